// cbm_stencil_tma.cuh — 3D medium stencils fed by the tensor memory
// accelerator.
//
// A block of kStX x kStY threads owns a kStX x kStTileY column of nodes over
// a run of z planes (the tiling of stencil_3d).  The planes of the column,
// each with a one-node y halo and a 16-byte x halo, stream from HBM into a
// ring of shared-memory stages by cp.async.bulk.tensor, one copy per plane
// issued by one thread and completed on the stage's mbarrier.  While plane z
// is computed from the stages of z - 1, z and z + 1, the next planes are in
// flight, so the loads never wait on registers and each block keeps several
// planes of bytes outstanding; in Float32 two planes are computed between
// barriers.  The x start of every copy is a
// multiple of 16 bytes (x0 - 16 / sizeof(T)); copies that reach beyond the
// field (the planes below 0 and above nz - 1, the halo of border tiles) read
// zeros, which only border nodes, whose values do not use them, would see.
//
// Same expressions as k_medium_grad / k_medium_de: lap = (l_x + l_y) + l_z,
// the DE reading medium_in() of every value, the divisions by dx^2 and 2 dx
// as over_dx2 / over_2dx.  Every wait on a stage is bounded; a wait that
// runs out sets kErrTimeout in the counters and the kernel goes on without
// blocking (its results are then void).
#pragma once
#include <cuda.h>  // CUtensorMap (the type only; the map is encoded on the host)

#include "cbm_kernels.cuh"

namespace cbm {

constexpr long long kTmaWaitCycles = 1ll << 31;  // about one second of SM clock

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(unsigned long long* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(unsigned long long* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(b)),
               "r"(bytes)
               : "memory");
}

// Wait for the completion of phase `parity` of barrier b, for at most
// kTmaWaitCycles; false when the bound ran out.
__device__ __forceinline__ bool mbar_wait(unsigned long long* b, unsigned parity) {
  const unsigned a = smem_addr(b);
  const long long t0 = clock64();
  while (true) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > kTmaWaitCycles) return false;
  }
}

// One tiled copy of the box at (x, y, z) of `map` into dst, completed on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// Geometry of the plane boxes: kStX + 2 * pad columns (pad = 16 bytes of
// elements), kStTileY + 2 rows, stages 128-byte aligned.
template <typename T>
struct TmaPlane {
  static constexpr int kPad = 16 / (int)sizeof(T);
  static constexpr int kBX = kStX + 2 * kPad;
  static constexpr int kBY = kStTileY + 2;
  static constexpr int kBytes = kBX * kBY * (int)sizeof(T);
  static constexpr int kStride = (kBytes + 127) / 128 * 128;
  static constexpr int kStages = sizeof(T) == 4 ? 6 : 4;
  static constexpr int kPlanes = sizeof(T) == 4 ? 2 : 1;  // planes computed between barriers
  static constexpr int kSmem = kStages * kStride + 128;  // + alignment slack
  // the planes read between two barriers (kPlanes + 2) and the next one in
  // flight fit the ring
  static_assert(kStages >= kPlanes + 3, "plane ring too short");
};

template <typename T, bool kDE, bool kScale>
__device__ __forceinline__ void stencil_3d_tma(const Params<T>& P, const CUtensorMap* map,
                                               int z_run) {
  using G = TmaPlane<T>;
  constexpr int S = G::kStages;
  extern __shared__ unsigned char tma_smem_raw[];
  __shared__ unsigned long long full[S];
  unsigned char* ring = tma_smem_raw + ((128 - (smem_addr(tma_smem_raw) & 127)) & 127);
  auto stage = [&](int i) -> const T* {
    return reinterpret_cast<const T*>(ring + (i % S) * G::kStride);
  };
  const int nx = P.n_medium[0], ny = P.n_medium[1], nz = P.n_medium[2];
  const int x0 = blockIdx.x * kStX, y0 = blockIdx.y * kStTileY;
  const int za = blockIdx.z * z_run;
  const int zb = za + z_run < nz ? za + z_run : nz;
  const int nplanes = zb - za + 2;  // planes za - 1 .. zb
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
  auto issue = [&](int i) {  // plane za - 1 + i into stage i % S
    unsigned long long* b = &full[i % S];
    mbar_expect_tx(b, (unsigned)G::kBytes);
    tma_load_3d(ring + (i % S) * G::kStride, map, x0 - G::kPad, y0 - 1, za - 1 + i, b);
  };
  if (lead) {
    for (int s = 0; s < S; ++s) mbar_init(&full[s], 1);
    mbar_fence_init();
  }
  __syncthreads();
  if (lead)
    for (int i = 0; i < S && i < nplanes; ++i) issue(i);
  bool ok = true;
  auto wait = [&](int i) {
    if (ok && !mbar_wait(&full[i % S], (unsigned)((i / S) & 1))) {
      ok = false;
      atomicOr(&P.ctr->err, kErrTimeout);
    }
  };
  auto in_val = [&](T v) { return kDE ? medium_in(P, v) : v; };
  const int x = x0 + threadIdx.x;
  // the column's nodes: in-plane offset, inside in x and y, present
  size_t nxy[kStRows];
  bool inxy[kStRows], here[kStRows];
#pragma unroll
  for (int r = 0; r < kStRows; ++r) {
    const int y = y0 + threadIdx.y + r * kStY;
    nxy[r] = (size_t)y * nx + x;
    here[r] = x < nx && y < ny;
    inxy[r] = x > 0 && x < nx - 1 && y > 0 && y < ny - 1;
  }
  const size_t plane = (size_t)nx * ny;
  // plane i of the run (z = za - 1 + i) from the stages of i - 1, i, i + 1
  auto compute = [&](int i) {
    const int z = za - 1 + i;
    const T* Sm = stage(i - 1);
    const T* Sc = stage(i);
    const T* Sp = stage(i + 1);
    const bool inz = z > 0 && z < nz - 1;
    const size_t zoff = (size_t)z * plane;
#pragma unroll
    for (int r = 0; r < kStRows; ++r) {
      if (here[r]) {
        const size_t n = zoff + nxy[r];
        const bool in = inxy[r] && inz;
        const int o = (threadIdx.y + r * kStY + 1) * G::kBX + threadIdx.x + G::kPad;
        if (kDE) {
          const T u = in_val(Sc[o]);
          if (!in) {
            P.c_nxt[n] = u;
          } else {
            const T l0 = over_dx2<kScale>(P, 0, (in_val(Sc[o + 1]) - (T)2 * u) + in_val(Sc[o - 1]));
            const T l1 =
                over_dx2<kScale>(P, 1, (in_val(Sc[o + G::kBX]) - (T)2 * u) + in_val(Sc[o - G::kBX]));
            const T l2 = over_dx2<kScale>(P, 2, (in_val(Sp[o]) - (T)2 * u) + in_val(Sm[o]));
            const T lap = (l0 + l1) + l2;
            const T k = P.diff_D * lap - P.decay * u;
            P.c_nxt[n] = u + P.dt * k;
          }
        } else {
          P.grad_nxt[0][n] = in ? over_2dx<kScale>(P, 0, Sc[o + 1] - Sc[o - 1]) : (T)0;
          P.grad_nxt[1][n] = in ? over_2dx<kScale>(P, 1, Sc[o + G::kBX] - Sc[o - G::kBX]) : (T)0;
          P.grad_nxt[2][n] = in ? over_2dx<kScale>(P, 2, Sp[o] - Sm[o]) : (T)0;
        }
      }
    }
  };
  wait(0);
  wait(1);
  // G::kPlanes planes a barrier: planes i .. i + kPlanes - 1 need the stages
  // of i - 1 .. i + kPlanes, which the ring holds
  for (int i = 1; i <= nplanes - 2; i += G::kPlanes) {
#pragma unroll
    for (int q = 0; q < G::kPlanes; ++q)
      if (i + q <= nplanes - 2) {
        wait(i + q + 1);
        compute(i + q);
      }
    __syncthreads();  // the stages of i - 1 .. i + kPlanes - 2 are read by no one any more
    if (lead)
#pragma unroll
      for (int q = 0; q < G::kPlanes; ++q)
        if (i - 1 + q + S < nplanes) issue(i - 1 + q + S);
  }
  // Every issued plane has been waited for on the normal path; after a wait
  // that ran out, the lead thread waits (bounded) for the copies still in
  // flight before the block's shared memory is released.
  if (lead && !ok) {
    const int last = nplanes < S ? nplanes : S;
    for (int i = nplanes - last; i < nplanes; ++i) mbar_wait(&full[i % S], (unsigned)((i / S) & 1));
  }
}

template <typename T>
__global__ void __launch_bounds__(kStX * kStY) k_medium_grad_3d_tma(Params<T> P,
                                                                   const __grid_constant__ CUtensorMap map,
                                                                   int z_run) {
  if (P.exact_scale) stencil_3d_tma<T, false, true>(P, &map, z_run);
  else stencil_3d_tma<T, false, false>(P, &map, z_run);
}

template <typename T>
__global__ void __launch_bounds__(kStX * kStY) k_medium_de_3d_tma(Params<T> P,
                                                                 const __grid_constant__ CUtensorMap map,
                                                                 int z_run) {
  pdl_wait();
  if (P.exact_scale) stencil_3d_tma<T, true, true>(P, &map, z_run);
  else stencil_3d_tma<T, true, false>(P, &map, z_run);
}

}  // namespace cbm
