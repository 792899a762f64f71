// cbm_common.cuh — constants, the device counter block and the small
// device helpers shared by every kernel of the library.
//
// Arithmetic follows the reference's expression order with no FMA
// contraction (the library is built with -fmad=false), so float and double
// results are bit-identical to a CPU evaluation of the same expressions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <utility>

#include "../../include/cbm_b200.h"
#include "../../include/cbm_rng.h"

namespace cbm {

constexpr int kTile = 256;          // threads per block of the per-agent kernels
constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanItems = 32;      // cells per thread in the cell scan (8192 per tile, so
                                    // the look-back spans few tiles)
constexpr int kScanTile = kTile * kScanItems;
constexpr long long kSpinLimit = 1ll << 20;  // bounded look-back wait

// Programmatic dependent launch.  A kernel launched with programmatic stream
// serialization is launched as the kernel before it on the stream completes,
// without the full gap between two launches; pdl_wait() returns once that
// kernel has completed and its writes are visible (at once for a plain
// launch), so a dependent kernel calls it before its first access to global
// memory.  No kernel here triggers its dependents early: blocks that wait
// resident for their predecessor would hold the SMs the concurrent branches
// of the step graph need.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Host side: launch kern on stream st, with programmatic stream
// serialization when `pdl` (then the operation before it on st must be a
// kernel launch, and kern calls pdl_wait() before its first global access).
// Errors are seen like those of <<<>>> launches, by cudaGetLastError.
template <typename... KP, typename... A>
inline void launch_serial(cudaStream_t st, bool pdl, void (*kern)(KP...), dim3 grid, dim3 block,
                          size_t smem, A&&... args) {
  cudaLaunchConfig_t lc = {};
  lc.gridDim = grid;
  lc.blockDim = block;
  lc.dynamicSmemBytes = smem;
  lc.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  lc.attrs = at;
  lc.numAttrs = pdl ? 1 : 0;
  cudaLaunchKernelEx(&lc, kern, std::forward<A>(args)...);
}

// device error bits (cbm_sync reports the first as a status code)
enum : int {
  kErrAgentOverflow = 1 << 0,
  kErrNeighborOverflow = 1 << 1,
  kErrTimeout = 1 << 2,
};

// Device counters.  Values that a step both reads and produces are indexed
// by step parity p: a step of parity p reads [p] and writes [p ^ 1].
struct Counters {
  long long N[2];
  long long step[2];
  double t[2];
  long long n_add;      // NAdd_ of the step in flight
  long long n_remove;   // NRemove_
  long long id_max;     // idMax_
  long long id_base;    // idMax_ before this step's births
  long long children;   // births requested (including dropped ones)
  long long slots;      // working slots of the step that ended (N + NAdd)
  int flag[2];          // flagRecomputeNeighbors_ of the step of that parity
  int err;              // kErr* bits
  unsigned scan_ticket; // tile tickets of the cell scan
  unsigned scan_epoch;  // generation of the cell-scan tile states
  int resort;           // the step that ended re-sorts its agents (grid rebuild)
  int events;           // births or deaths in the step in flight
  int list_valid;       // the Verlet list matches the current slots
  int list_written;     // this step wrote the Verlet list lazily
  unsigned fate_ticket; // tile tickets of the fused rule / births kernel
  unsigned fate_epoch;  // generation of its tile states
  unsigned de_ticket;   // tile tickets of the force kernel (reset by its last block)
  unsigned de_done;     // blocks of the force kernel that have finished
};

template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// Julia's float `÷` on a >= 0: round((a - rem(a, b)) / b), which is the exact
// floor of a / b (quotients below 4e6).  Fast path: when the correctly
// rounded quotient f has a fractional part farther than m from 0 and 1, the
// exact quotient lies within half an ulp of f (< m) and so in the same unit
// interval, and floor(f) is that floor; otherwise the remainder formula runs.
__device__ __forceinline__ int floordiv(double a, double b) {
  const double f = a / b;
  const double n = floor(f);
  const double fr = f - n;  // exact below 2^52
  const double m = f * 1e-12 + 1e-14;
  if (fr > m && fr < 1.0 - m) return (int)n;
  return (int)rint((a - fmod(a, b)) / b);
}
__device__ __forceinline__ int floordiv(float a, float b) {
  const float f = a / b;
  const float n = floorf(f);
  const float fr = f - n;  // exact below 2^23
  const float m = f * 1e-5f + 1e-6f;
  if (fr > m && fr < 1.0f - m) return (int)n;
  return (int)rintf((a - fmodf(a, b)) / b);
}

// cellPos, src/neighbors.jl:636-638, 0-based; a NaN coordinate goes to the
// first cell
template <typename T>
__device__ __forceinline__ int cell_pos1(T edge, T x, T lo, T hi, int n) {
  if (x > hi) return n - 1;
  if (!(x >= lo)) return 0;
  int p = floordiv(x - lo, edge) + 1;
  return p > n - 1 ? n - 1 : p;
}

// linear cell of a point, x fastest
template <typename T, int D>
__device__ __forceinline__ int cell_of(T edge, const T* lo, const T* hi, const int* nc,
                                       const T* x) {
  int lin = cell_pos1<T>(edge, x[0], lo[0], hi[0], nc[0]);
  if (D > 1) lin += nc[0] * cell_pos1<T>(edge, x[1], lo[1], hi[1], nc[1]);
  if (D > 2) lin += nc[0] * nc[1] * cell_pos1<T>(edge, x[2], lo[2], hi[2], nc[2]);
  return lin;
}

// cellInMesh, src/metrics.jl:18-20 (0-based, clamped at the top)
template <typename T>
__device__ __forceinline__ int cell_in_mesh(T dx, T x, T lo, T hi, int n) {
  if (x > hi) return n - 1;
  if (!(x >= lo)) return 0;
  int p = floordiv(x - lo, dx);
  return p > n - 1 ? n - 1 : p;
}

// cellPosNeigh, src/neighbors.jl:658-708: k-th of 3^D cells, x fastest,
// -1 outside the grid
template <int D>
__device__ __forceinline__ int cell_neigh(const int* nc, const int* q, int k) {
  int px = q[0] + (k % 3) - 1;
  if (px < 0 || px >= nc[0]) return -1;
  int lin = px;
  if (D > 1) {
    int py = q[1] + ((k / 3) % 3) - 1;
    if (py < 0 || py >= nc[1]) return -1;
    lin += nc[0] * py;
  }
  if (D > 2) {
    int pz = q[2] + (k / 9) - 1;
    if (pz < 0 || pz >= nc[2]) return -1;
    lin += nc[0] * nc[1] * pz;
  }
  return lin;
}

template <int D>
__device__ __forceinline__ void cell_coords(const int* nc, int pos, int* q) {
  q[0] = pos % nc[0];
  if (D > 1) q[1] = (pos / nc[0]) % nc[1];
  if (D > 2) q[2] = pos / (nc[0] * nc[1]);
}

// exclusive block scan of one int per thread (kTile threads)
__device__ __forceinline__ int block_exscan(int v, int* warp_sums, int* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    int s = lane < kTile / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kTile / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  int prefix = w > 0 ? warp_sums[w - 1] : 0;
  *total = warp_sums[kTile / 32 - 1];
  __syncthreads();
  return prefix + x - v;
}

// ---------------------------------------------------------------------------
// exclusive scan of per-cell counts (cumsum .- counts, src/neighbors.jl:934-937)
// in one pass with decoupled look-back.  Tiles take tickets in launch order so
// a tile only waits on tiles that are already running; the wait is bounded.
// Counts are zeroed for the next build.  The preceding histogram kernel resets
// the ticket counter and advances the tile-state epoch.
// ---------------------------------------------------------------------------
struct ScanArgs {
  int* count;                      // n counts, zeroed on exit
  int* start;                      // n + 1 exclusive offsets
  unsigned long long* state;       // n_tiles tile states: epoch | flag | value
  int n;
  int n_tiles;
  Counters* ctr;
  const int* due;                  // skip the scan when *due == 0 (nullptr: always)
};

// Shared-memory index of cell k of a tile: one padding word per 32 cells, so
// that a thread reading its 32 consecutive cells hits 32 different banks.
__device__ __forceinline__ int scan_pad(int k) { return k + (k >> 5); }

static __global__ void __launch_bounds__(kTile) k_scan_cells(ScanArgs A) {
  __shared__ int warp_sums[kTile / 32];
  __shared__ unsigned s_tile;
  __shared__ int s_prefix;
  __shared__ int s_cells[kScanTile + kScanTile / 32];
  pdl_wait();
  if (A.due && *A.due == 0) return;
  Counters* C = A.ctr;
  const unsigned epoch = C->scan_epoch;
  if (threadIdx.x == 0) s_tile = atomicAdd(&C->scan_ticket, 1u);
  __syncthreads();
  const int tile = (int)s_tile;
  if (tile >= A.n_tiles) {  // tickets were not reset: never index past the tile states
    if (threadIdx.x == 0) atomicOr(&C->err, kErrTimeout);
    return;
  }
  static_assert(kScanItems % 4 == 0 && kScanItems == 32, "int4 staging, 32 cells per thread");
  const int tile_base = tile * kScanTile;
  const bool full = tile_base + kScanTile <= A.n;
  // coalesced load of the tile's counts into shared memory
  if (full) {
#pragma unroll
    for (int v = 0; v < kScanItems / 4; ++v) {
      const int q = v * kTile + threadIdx.x;  // int4 index inside the tile
      const int4 a = reinterpret_cast<const int4*>(A.count + tile_base)[q];
      s_cells[scan_pad(4 * q)] = a.x;
      s_cells[scan_pad(4 * q + 1)] = a.y;
      s_cells[scan_pad(4 * q + 2)] = a.z;
      s_cells[scan_pad(4 * q + 3)] = a.w;
    }
  } else {
    for (int k = threadIdx.x; k < kScanTile; k += kTile)
      s_cells[scan_pad(k)] = tile_base + k < A.n ? A.count[tile_base + k] : 0;
  }
  __syncthreads();
  const int first = threadIdx.x * kScanItems;  // this thread's cells inside the tile
  int vals[kScanItems];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    vals[k] = s_cells[scan_pad(first + k)];
    sum += vals[k];
  }
  int total;
  int ex = block_exscan(sum, warp_sums, &total);
  const unsigned long long ep = (unsigned long long)epoch << 32;
  if (threadIdx.x < 32) {
    // warp look-back: lane l inspects tile (t - l); stop at the nearest tile
    // that has published its inclusive prefix, summing aggregates before it
    const int lane = threadIdx.x;
    if (tile == 0) {
      if (lane == 0) {
        s_prefix = 0;
        atomicExch(A.state, ep | (2ull << 30) | (unsigned)total);
      }
    } else {
      if (lane == 0) atomicExch(A.state + tile, ep | (1ull << 30) | (unsigned)total);
      int prefix = 0;
      int t = tile - 1;
      long long spins = 0;
      while (true) {
        const int idx = t - lane;
        unsigned flag = 2u, val = 0u;  // before tile 0: an inclusive prefix of 0
        if (idx >= 0) {
          unsigned long long s = atomicAdd(A.state + idx, 0ull);
          flag = ((s >> 32) == epoch) ? (unsigned)(s >> 30) & 3u : 0u;
          val = (unsigned)(s & 0x3fffffffu);
        }
        const unsigned incl = __ballot_sync(kFull, flag == 2u);
        const unsigned pend = __ballot_sync(kFull, flag == 0u);
        // lanes up to and including the first inclusive one must be ready
        const unsigned upto = incl ? ((incl & (0u - incl)) << 1) - 1u : kFull;
        if (pend & upto) {
          if (++spins > kSpinLimit) {
            if (lane == 0) atomicOr(&C->err, kErrTimeout);
            break;
          }
          continue;
        }
        unsigned mine = ((1u << lane) & upto) ? val : 0u;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(kFull, mine, o);
        prefix += (int)mine;
        if (incl) break;
        t -= 32;
      }
      if (lane == 0) {
        s_prefix = prefix;
        atomicExch(A.state + tile, ep | (2ull << 30) | (unsigned)(prefix + total));
      }
    }
  }
  __syncthreads();
  // exclusive offsets back into shared memory, then coalesced stores
  int run = s_prefix + ex;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    s_cells[scan_pad(first + k)] = run;
    run += vals[k];
  }
  // the thread holding the last cell writes the end sentinel
  if (A.n - 1 >= tile_base + first && A.n - 1 < tile_base + first + kScanItems) A.start[A.n] = run;
  __syncthreads();
  if (full) {
    // start is only 4-byte aligned for a shifted array, so it is written as
    // plain ints; counts are cleared as int4
#pragma unroll 8
    for (int k = threadIdx.x; k < kScanTile; k += kTile) A.start[tile_base + k] = s_cells[scan_pad(k)];
#pragma unroll
    for (int v = 0; v < kScanItems / 4; ++v)
      reinterpret_cast<int4*>(A.count + tile_base)[v * kTile + threadIdx.x] = make_int4(0, 0, 0, 0);
  } else {
    for (int k = threadIdx.x; k < kScanTile; k += kTile)
      if (tile_base + k < A.n) {
        A.start[tile_base + k] = s_cells[scan_pad(k)];
        A.count[tile_base + k] = 0;
      }
  }
}

}  // namespace cbm
