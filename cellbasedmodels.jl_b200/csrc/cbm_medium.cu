// cbm_medium.cu — the implicit medium integrator DGADI on the device.
//
// CBMIntegrators.DGADI (src/integrators.jl:817-937) advances the medium by
//   1. u .+= f(u)                        (the explicit part, no factor dt)
//   2. a Thomas solve along every line of x, then y, then z
//      (tridiagonal{1,2,3}D{x,y,z}{CPU,GPU}!, :141-428)
// with the border nodes fixed at their initial values (the reference never
// writes them into u_new, and copies u_new into u after each axis).
//
// Layout: field k, node (x, y, z) at k * nodes + x + n0 * (y + n1 * z).  Two
// copies of every field: a step reads one and writes the interior of the
// other, whose border nodes hold the uploaded values, so the copy back of the
// reference is a swap.
//
// The line recurrence (0-based, nodes 0 and n-1 are the Dirichlet ends):
//   c*_1 = sup / main                    d*_1 = (x_1 - sub x_0) / main
//   m_j  = 1.0 / (main - sub c*_{j-1})   (Float64: Julia promotes 1.0 / x)
//   c*_j = T(sup m_j)                    d*_j = T((x_j - sub d*_{j-1}) m_j)
//   d*_{n-2} = T(((x_{n-2} - sup x_{n-1}) - sub d*_{n-3}) m_{n-2})
//   x_{n-2} = d*_{n-2},  x_j = d*_j - c*_j x_{j+1}
// c*_j and m_j depend only on the diagonals, so every line of a field and
// axis shares one table of them (the same bits as recomputing them per line).
// One thread walks one line: lines along y and z are coalesced across
// threads; lines along x are served by L1 (each thread reads its own
// contiguous row).
#include <cuda_runtime.h>

#include <cmath>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/cbm_b200.h"

namespace {

constexpr int kSweepThreads = 128;

template <typename T>
struct FieldCoef {
  T sub[CBM_MEDIUM_MAX_FIELDS], main[CBM_MEDIUM_MAX_FIELDS], sup[CBM_MEDIUM_MAX_FIELDS];
  T decay[CBM_MEDIUM_MAX_FIELDS];
};

// Diagonals, c* and the pivots of every (field, axis): one thread each.
// r = dt / (dims dx^2) with dx of the last axis for every axis (the
// reference's column [l, dims]); the coefficients are formed in Float64 and
// rounded to the field precision.
template <typename T>
__global__ void k_dgadi_tables(cbm_medium_config k, int nmax, FieldCoef<T>* coef, T* cstar,
                               double* piv) {
  const int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= k.n_fields * 3) return;
  const int f = id / 3, a = id % 3;
  const int D = k.dims;
  const double dxl = (k.box_hi[D - 1] - k.box_lo[D - 1]) / (double)k.n[D - 1];
  const double r = k.dt / ((double)D * (dxl * dxl));
  const T sub = (T)(-k.diffusion[f] * r), sup = (T)(-k.diffusion[f] * r);
  const T main = (T)(1.0 + 2.0 * k.diffusion[f] * r);
  if (a == 0) {
    coef->sub[f] = sub;
    coef->main[f] = main;
    coef->sup[f] = sup;
    coef->decay[f] = (T)k.decay[f];
  }
  if (a >= D) return;
  const int n = k.n[a];
  T* cs = cstar + (size_t)id * nmax;
  double* pv = piv + (size_t)id * nmax;
  cs[1] = sup / main;
  for (int j = 2; j <= n - 2; ++j) {
    pv[j] = 1.0 / (double)(main - sub * cs[j - 1]);
    if (j <= n - 3) cs[j] = (T)((double)sup * pv[j]);
  }
}

// The explicit part u .+= f(u), f = s (c_max - u) - decay u, applies to the
// nodes that are interior in every axis: exactly the interior nodes of the
// lines along x through interior (y, z), whose solve reads nothing else.  So
// it is applied while those lines are loaded, inside the x solves.
template <typename T>
__device__ __forceinline__ T explicit_part(T u, T s, T cmax, T decay) {
  return u + (s * (cmax - u) - decay * u);
}

constexpr unsigned kFullMask = 0xffffffffu;

// Asynchronous copy of one element global -> shared (no register round trip,
// so a thread's copies are all in flight together); completed by
// cp_async_wait_all, made visible to the warp by __syncwarp.
template <typename T>
__device__ __forceinline__ void cp_async_elem(T* smem, const T* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (sizeof(T) == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(a), "l"(gmem) : "memory");
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;\n" ::: "memory");
}

// One line's solve in place: X(j) is node j of the line (ends 0 and n-1).
// The table entries and nodes of the next iteration are loaded one step
// ahead, so that only the arithmetic stays on the recurrence's chain.
template <typename T, typename F>
__device__ __forceinline__ void line_solve(F&& X, int n, T sub, T main, T sup, const T* cs,
                                           const double* pv) {
  T d = (X(1) - sub * X(0)) / main;
  X(1) = d;
  double pn = pv[2];
  T xn = X(2);
  for (int j = 2; j <= n - 3; ++j) {
    const double p = pn;
    const T xj = xn;
    pn = pv[j + 1];
    xn = X(j + 1);
    d = (T)((double)(xj - sub * d) * p);
    X(j) = d;
  }
  T x = (T)((double)((xn - sup * X(n - 1)) - sub * d) * pn);
  X(n - 2) = x;
  T cn = n - 3 >= 1 ? cs[n - 3] : (T)0;
  T dn = n - 3 >= 1 ? X(n - 3) : (T)0;
  for (int j = n - 3; j >= 1; --j) {
    const T c = cn, dj = dn;
    if (j > 1) {
      cn = cs[j - 1];
      dn = X(j - 1);
    }
    x = dj - c * x;
    X(j) = x;
  }
}

// The Thomas solves of axis A: one thread per (field, line through interior
// nodes of the other axes).  Reads xo, writes the line's interior of xn
// (d* first, then the solution in place).
template <typename T, int A, int D>
__global__ void __launch_bounds__(kSweepThreads)
    k_dgadi_sweep(const T* __restrict__ xo, T* __restrict__ xn, const FieldCoef<T>* __restrict__ coef,
                  const T* __restrict__ cstar, const double* __restrict__ piv, int nmax, int n0,
                  int n1, int n2, int nf, const T* __restrict__ src, T cmax) {
  const int len[3] = {n0, n1, n2};
  const long long stride[3] = {1, n0, (long long)n0 * n1};
  constexpr int B = A == 0 ? 1 : 0;  // the line's position: (b, c) interior
  constexpr int Cx = A == 2 ? 1 : 2;
  const int nb = B < D ? len[B] - 2 : 1, nc = Cx < D ? len[Cx] - 2 : 1;
  const long long lines = (long long)nb * nc;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= lines * nf) return;
  const int f = (int)(id / lines);
  const long long l = id - (long long)f * lines;
  const int ib = (int)(l % nb) + (B < D ? 1 : 0);
  const int ic = (int)(l / nb) + (Cx < D ? 1 : 0);
  const long long o =
      (long long)f * n0 * n1 * n2 + (long long)ib * stride[B] + (long long)ic * stride[Cx];
  const long long st = stride[A];
  const int n = len[A];
  const T sub = coef->sub[f], main = coef->main[f], sup = coef->sup[f];
  const T* cs = cstar + (size_t)(f * 3 + A) * nmax;
  const double* pv = piv + (size_t)(f * 3 + A) * nmax;
  const T* X = xo + o;
  T* Y = xn + o;
  // the interior to solve is copied to xn's line first, with the explicit
  // part along x (xn's ends are the uploaded border values, equal to xo's)
  if (A == 0) {
    const T* S = src + (o - (long long)f * n0 * n1 * n2);
    const T dec = coef->decay[f];
    for (int j = 1; j < n - 1; ++j) Y[j] = explicit_part(X[j], S[j], cmax, dec);
  } else {
    for (int j = 1; j < n - 1; ++j) Y[j * st] = X[j * st];
  }
  line_solve<T>([&](int j) -> T& { return Y[j * st]; }, n, sub, main, sup, cs, pv);
}

// The same solves with the lines of one warp staged in shared memory: 32
// lines per block, copied in and out with coalesced accesses (rows along x
// for axis 0; for axes 1 and 2, 32 consecutive lines at each position along
// them) and solved in place there.  Row r of the tile is line r of the block:
// at r * rowp + j for axis 0 (rowp odd, so the 32 rows fall in distinct
// banks), at j * 32 + r otherwise.
constexpr int kTileLines = 32;

template <typename T, int A, int D>
__global__ void __launch_bounds__(kTileLines)
    k_dgadi_sweep_tiled(const T* __restrict__ xo, T* __restrict__ xn,
                        const FieldCoef<T>* __restrict__ coef, const T* __restrict__ cstar,
                        const double* __restrict__ piv, int nmax, int n0, int n1, int n2, int nf,
                        int rowp, const T* __restrict__ src, T cmax) {
  extern __shared__ __align__(16) unsigned char med_smem[];
  T* tile = reinterpret_cast<T*>(med_smem);
  T* stile = tile + kTileLines * rowp;  // axis 0: the source rows
  const int len[3] = {n0, n1, n2};
  const long long stride[3] = {1, n0, (long long)n0 * n1};
  constexpr int B = A == 0 ? 1 : 0;
  constexpr int Cx = A == 2 ? 1 : 2;
  const int nb = B < D ? len[B] - 2 : 1, nc = Cx < D ? len[Cx] - 2 : 1;
  const long long lines = (long long)nb * nc;
  const int n = len[A];
  const long long st = stride[A];
  const int t = threadIdx.x;
  // global offset of the first node of line (block base + r), or -1 past the end
  auto line_base = [&](int r, int* field) -> long long {
    const long long id = (long long)blockIdx.x * kTileLines + r;
    if (id >= lines * nf) return -1;
    const int f = (int)(id / lines);
    const long long l = id - (long long)f * lines;
    const int ib = (int)(l % nb) + (B < D ? 1 : 0);
    const int ic = (int)(l / nb) + (Cx < D ? 1 : 0);
    *field = f;
    return (long long)f * n0 * n1 * n2 + (long long)ib * stride[B] + (long long)ic * stride[Cx];
  };
  int f = 0;
  const long long o = line_base(t, &f);
  auto at = [&](int r, int j) -> T& { return A == 0 ? tile[r * rowp + j] : tile[j * kTileLines + r]; };
  const long long fnodes = (long long)n0 * n1 * n2;
  if (A == 0) {
    for (int r = 0; r < kTileLines; ++r) {
      const long long orow = __shfl_sync(kFullMask, o, r);
      const int frow = __shfl_sync(kFullMask, f, r);
      if (orow < 0) break;
      const long long srow = orow - (long long)frow * fnodes;
      for (int j = t; j < n; j += kTileLines) {
        cp_async_elem(&at(r, j), xo + orow + j);
        cp_async_elem(&stile[r * rowp + j], src + srow + j);
      }
    }
  } else if (o >= 0) {
    for (int j = 0; j < n; ++j) cp_async_elem(&at(t, j), xo + o + j * st);
  }
  cp_async_wait_all();
  __syncwarp();
  if (o >= 0) {
    if (A == 0) {
      const T dec = coef->decay[f];
      for (int j = 1; j < n - 1; ++j) at(t, j) = explicit_part(at(t, j), stile[t * rowp + j], cmax, dec);
    }
    const T sub = coef->sub[f], main = coef->main[f], sup = coef->sup[f];
    const T* cs = cstar + (size_t)(f * 3 + A) * nmax;
    const double* pv = piv + (size_t)(f * 3 + A) * nmax;
    line_solve<T>([&](int j) -> T& { return at(t, j); }, n, sub, main, sup, cs, pv);
  }
  __syncwarp();
  if (A == 0) {
    for (int r = 0; r < kTileLines; ++r) {
      const long long orow = __shfl_sync(kFullMask, o, r);
      if (orow < 0) break;
      for (int j = 1 + t; j < n - 1; j += kTileLines) xn[orow + j] = at(r, j);
    }
  } else if (o >= 0) {
    for (int j = 1; j < n - 1; ++j) xn[o + j * st] = at(t, j);
  }
}

// A whole field in one block's shared memory: nsteps complete steps in one
// launch, one block per field (the fields do not interact).  Each step is the
// explicit part, then the lines of x, y, z, one thread per line and in place
// (the lines of one axis are disjoint and each writes only its interior),
// with a block barrier between phases.  Rows are stored with an odd pitch px
// so that the threads of the x phase fall in distinct banks; the source field
// follows the medium field.  The global copy is read once and written back
// once, in place.
constexpr int kFusedThreads = 256;

template <typename T, int D>
__global__ void __launch_bounds__(kFusedThreads)
    k_dgadi_fused(T* __restrict__ u, const T* __restrict__ src,
                  const FieldCoef<T>* __restrict__ coef, const T* __restrict__ cstar,
                  const double* __restrict__ piv, T cmax, int nmax, int n0, int n1, int n2,
                  int px, int nsteps) {
  extern __shared__ __align__(16) unsigned char med_smem[];
  T* sh = reinterpret_cast<T*>(med_smem);
  const int f = blockIdx.x;
  const int nodes = n0 * n1 * n2;
  const int snodes = px * n1 * n2;  // shared layout: x + px (y + n1 z)
  T* ss = sh + snodes;
  T* g = u + (size_t)f * nodes;
  for (int i = threadIdx.x; i < nodes; i += kFusedThreads) {
    const int x = i % n0, yz = i / n0;
    sh[x + px * yz] = g[i];
    ss[x + px * yz] = src[i];
  }
  __syncthreads();
  const T sub = coef->sub[f], main = coef->main[f], sup = coef->sup[f], dec = coef->decay[f];
  const int len[3] = {n0, n1, n2};
  const int sst[3] = {1, px, px * n1};
  for (int step = 0; step < nsteps; ++step) {
    for (int i = threadIdx.x; i < nodes; i += kFusedThreads) {
      const int x = i % n0;
      const int y = D > 1 ? (i / n0) % n1 : 0;
      const int z = D > 2 ? i / (n0 * n1) : 0;
      const bool in = x > 0 && x < n0 - 1 && (D < 2 || (y > 0 && y < n1 - 1)) &&
                      (D < 3 || (z > 0 && z < n2 - 1));
      if (!in) continue;
      const int k = x + px * (y + n1 * z);
      sh[k] = explicit_part(sh[k], ss[k], cmax, dec);
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
      const int nb = b < D ? len[b] - 2 : 1, nc = c < D ? len[c] - 2 : 1;
      const int n = len[a], st = sst[a];
      const T* cs = cstar + (size_t)(f * 3 + a) * nmax;
      const double* pv = piv + (size_t)(f * 3 + a) * nmax;
      for (int l = threadIdx.x; l < nb * nc; l += kFusedThreads) {
        const int ib = l % nb + (b < D ? 1 : 0), ic = l / nb + (c < D ? 1 : 0);
        T* X = sh + ib * sst[b] + ic * sst[c];
        line_solve<T>([&](int j) -> T& { return X[j * st]; }, n, sub, main, sup, cs, pv);
      }
      __syncthreads();
    }
  }
  for (int i = threadIdx.x; i < nodes; i += kFusedThreads) {
    const int x = i % n0, yz = i / n0;
    g[i] = sh[x + px * yz];
  }
}

// shared memory of the fused kernel (medium and source fields)
template <typename T>
size_t fused_bytes(const int* n, int dims) {
  size_t nodes = (size_t)(n[0] | 1);
  for (int d = 1; d < dims; ++d) nodes *= (size_t)n[d];
  return 2 * nodes * sizeof(T);
}
constexpr size_t kFusedMaxBytes = 200 * 1024;

// shared memory of one tiled sweep block along an axis of n nodes
template <typename T>
size_t tile_bytes(int axis, int n) {
  const int rowp = axis == 0 ? (n | 1) : n;
  return (axis == 0 ? 2 : 1) * (size_t)kTileLines * rowp * sizeof(T);
}
constexpr size_t kTileMaxBytes = 96 * 1024;

}  // namespace

struct cbm_medium {
  cbm_medium_config cfg{};
  int tsize = 4;
  int device = 0;
  cudaStream_t stream = nullptr;
  long long nodes = 0;
  int nmax = 0;
  void* u[2] = {nullptr, nullptr};
  void* src = nullptr;
  void* coef = nullptr;
  void* cstar = nullptr;
  double* piv = nullptr;
  int cur = 0;
  bool fused = false;  // the whole field fits one block's shared memory
  long long steps = 0;
  double t = 0;
  bool loaded = false;
  std::string err;
};

namespace {

std::string g_medium_create_error;

int mfail(cbm_medium* m, int code, const std::string& msg) {
  if (m) m->err = msg;
  else g_medium_create_error = msg;
  return code;
}

#define MED_TRY(m, call)                                                                    \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return mfail(m, CBM_ERR_CUDA, std::string(#call) + " failed: " + cudaGetErrorString(e_)); \
  } while (0)

void mfree(cbm_medium* m) {
  for (void* p : {m->u[0], m->u[1], m->src, m->coef, m->cstar, (void*)m->piv})
    if (p) cudaFree(p);
  m->u[0] = m->u[1] = m->src = m->coef = m->cstar = nullptr;
  m->piv = nullptr;
  if (m->stream) cudaStreamDestroy(m->stream);
  m->stream = nullptr;
}

template <typename T, int D>
int enqueue_step(cbm_medium* m) {
  const cbm_medium_config& k = m->cfg;
  const int n0 = k.n[0], n1 = D > 1 ? k.n[1] : 1, n2 = D > 2 ? k.n[2] : 1;
  const int nf = k.n_fields;
  T* u[2] = {(T*)m->u[0], (T*)m->u[1]};
  const auto* coef = (const FieldCoef<T>*)m->coef;
  const T* src = (const T*)m->src;
  const T cmax = (T)k.c_max;
  auto lines = [&](int a) {
    const int len[3] = {n0, n1, n2};
    long long l = 1;
    for (int d = 0; d < D; ++d)
      if (d != a) l *= len[d] - 2;
    return l * nf;
  };
  auto grid = [&](long long n) { return (unsigned)((n + kSweepThreads - 1) / kSweepThreads); };
  const T* cs = (const T*)m->cstar;
  const int len[3] = {n0, n1, n2};
  auto sweep = [&](auto axis) {
    constexpr int A = decltype(axis)::value;
    const size_t tb = tile_bytes<T>(A, len[A]);
    if (tb <= kTileMaxBytes) {
      const long long nl = lines(A);
      k_dgadi_sweep_tiled<T, A, D>
          <<<(unsigned)((nl + kTileLines - 1) / kTileLines), kTileLines, tb, m->stream>>>(
              u[m->cur], u[m->cur ^ 1], coef, cs, m->piv, m->nmax, n0, n1, n2, nf,
              A == 0 ? (len[A] | 1) : len[A], src, cmax);
    } else {
      k_dgadi_sweep<T, A, D><<<grid(lines(A)), kSweepThreads, 0, m->stream>>>(
          u[m->cur], u[m->cur ^ 1], coef, cs, m->piv, m->nmax, n0, n1, n2, nf, src, cmax);
    }
    m->cur ^= 1;
  };
  sweep(std::integral_constant<int, 0>());
  if constexpr (D > 1) sweep(std::integral_constant<int, 1>());
  if constexpr (D > 2) sweep(std::integral_constant<int, 2>());
  MED_TRY(m, cudaGetLastError());
  return CBM_OK;
}

template <typename T, int D>
int enqueue_fused(cbm_medium* m, int nsteps) {
  const cbm_medium_config& k = m->cfg;
  const int n0 = k.n[0], n1 = D > 1 ? k.n[1] : 1, n2 = D > 2 ? k.n[2] : 1;
  const size_t bytes = fused_bytes<T>(k.n, D);
  k_dgadi_fused<T, D><<<k.n_fields, kFusedThreads, bytes, m->stream>>>(
      (T*)m->u[m->cur], (const T*)m->src, (const FieldCoef<T>*)m->coef, (const T*)m->cstar,
      m->piv, (T)k.c_max, m->nmax, n0, n1, n2, n0 | 1, nsteps);
  MED_TRY(m, cudaGetLastError());
  return CBM_OK;
}
template <typename T>
int enqueue_fused_t(cbm_medium* m, int nsteps) {
  switch (m->cfg.dims) {
    case 1: return enqueue_fused<T, 1>(m, nsteps);
    case 2: return enqueue_fused<T, 2>(m, nsteps);
    default: return enqueue_fused<T, 3>(m, nsteps);
  }
}

template <typename T, int D>
bool set_tile_attrs_d(int bytes) {
  bool ok = cudaFuncSetAttribute(k_dgadi_sweep_tiled<T, 0, D>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
  if (D > 1)
    ok = ok && cudaFuncSetAttribute(k_dgadi_sweep_tiled<T, 1, D>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
  if (D > 2)
    ok = ok && cudaFuncSetAttribute(k_dgadi_sweep_tiled<T, 2, D>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess;
  ok = ok && cudaFuncSetAttribute(k_dgadi_fused<T, D>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)kFusedMaxBytes) == cudaSuccess;
  return ok;
}
template <typename T>
bool set_tile_attrs(int dims, int bytes) {
  switch (dims) {
    case 1: return set_tile_attrs_d<T, 1>(bytes);
    case 2: return set_tile_attrs_d<T, 2>(bytes);
    default: return set_tile_attrs_d<T, 3>(bytes);
  }
}

template <typename T>
int enqueue_step_t(cbm_medium* m) {
  switch (m->cfg.dims) {
    case 1: return enqueue_step<T, 1>(m);
    case 2: return enqueue_step<T, 2>(m);
    default: return enqueue_step<T, 3>(m);
  }
}

}  // namespace

extern "C" {

int cbm_medium_create(cbm_medium** out, const cbm_medium_config* cfg) {
  if (!out || !cfg) return mfail(nullptr, CBM_ERR_ARG, "null argument");
  *out = nullptr;
  const cbm_medium_config& k = *cfg;
  if (k.dims < 1 || k.dims > 3) return mfail(nullptr, CBM_ERR_ARG, "dims must be 1, 2 or 3");
  if (k.precision != CBM_F32 && k.precision != CBM_F64)
    return mfail(nullptr, CBM_ERR_ARG, "precision must be CBM_F32 or CBM_F64");
  if (k.n_fields < 1 || k.n_fields > CBM_MEDIUM_MAX_FIELDS)
    return mfail(nullptr, CBM_ERR_ARG, "n_fields must be 1 .. CBM_MEDIUM_MAX_FIELDS");
  long long nodes = 1;
  int nmax = 0;
  for (int d = 0; d < k.dims; ++d) {
    if (k.n[d] < 4)
      return mfail(nullptr, CBM_ERR_ARG, "every axis of a DGADI medium needs at least 4 nodes");
    nodes *= k.n[d];
    nmax = k.n[d] > nmax ? k.n[d] : nmax;
  }
  if (nodes * k.n_fields >= (1ll << 40)) return mfail(nullptr, CBM_ERR_ARG, "medium too large");
  if (!(k.dt > 0) || !(k.box_hi[k.dims - 1] > k.box_lo[k.dims - 1]))
    return mfail(nullptr, CBM_ERR_ARG, "dt and the last axis of the box must be positive");

  cbm_medium* m = new cbm_medium;
  m->cfg = k;
  for (int d = k.dims; d < 3; ++d) m->cfg.n[d] = 1;
  m->tsize = k.precision == CBM_F64 ? 8 : 4;
  m->nodes = nodes;
  m->nmax = nmax;
  cudaGetDevice(&m->device);
  const size_t fb = (size_t)nodes * k.n_fields * m->tsize;
  bool ok = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) == cudaSuccess;
  ok = ok && cudaMalloc(&m->u[0], fb) == cudaSuccess;
  ok = ok && cudaMalloc(&m->u[1], fb) == cudaSuccess;
  ok = ok && cudaMalloc(&m->src, (size_t)nodes * m->tsize) == cudaSuccess;
  ok = ok && cudaMalloc(&m->coef, sizeof(FieldCoef<double>)) == cudaSuccess;
  ok = ok && cudaMalloc(&m->cstar, (size_t)k.n_fields * 3 * nmax * m->tsize) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&m->piv, (size_t)k.n_fields * 3 * nmax * 8) == cudaSuccess;
  if (!ok) {
    mfree(m);
    delete m;
    return mfail(nullptr, CBM_ERR_NOMEM, "device allocation failed for the DGADI medium");
  }
  {
    // tiled sweeps may use up to kTileMaxBytes of dynamic shared memory
    const int big = (int)kTileMaxBytes;
    bool attr = true;
    if (m->tsize == 8) attr = set_tile_attrs<double>(k.dims, big);
    else attr = set_tile_attrs<float>(k.dims, big);
    if (!attr) {
      mfree(m);
      delete m;
      return mfail(nullptr, CBM_ERR_CUDA, "cudaFuncSetAttribute failed for the DGADI sweeps");
    }
  }
  const unsigned tb = (unsigned)((k.n_fields * 3 + 63) / 64);
  if (m->tsize == 8)
    k_dgadi_tables<double><<<tb, 64, 0, m->stream>>>(m->cfg, nmax, (FieldCoef<double>*)m->coef,
                                                     (double*)m->cstar, m->piv);
  else
    k_dgadi_tables<float><<<tb, 64, 0, m->stream>>>(m->cfg, nmax, (FieldCoef<float>*)m->coef,
                                                    (float*)m->cstar, m->piv);
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(m->stream) != cudaSuccess) {
    mfree(m);
    delete m;
    return mfail(nullptr, CBM_ERR_CUDA, "DGADI table set-up failed");
  }
  m->fused = (m->tsize == 8 ? fused_bytes<double>(m->cfg.n, k.dims)
                            : fused_bytes<float>(m->cfg.n, k.dims)) <= kFusedMaxBytes;
  *out = m;
  return CBM_OK;
}

void cbm_medium_destroy(cbm_medium* m) {
  if (!m) return;
  mfree(m);
  delete m;
}

const char* cbm_medium_last_error(const cbm_medium* m) {
  return m ? m->err.c_str() : g_medium_create_error.c_str();
}

int cbm_medium_upload(cbm_medium* m, const void* fields, const void* source) {
  if (!m || !fields) return mfail(m, CBM_ERR_ARG, "null argument");
  const size_t fb = (size_t)m->nodes * m->cfg.n_fields * m->tsize;
  MED_TRY(m, cudaMemcpyAsync(m->u[0], fields, fb, cudaMemcpyHostToDevice, m->stream));
  MED_TRY(m, cudaMemcpyAsync(m->u[1], m->u[0], fb, cudaMemcpyDeviceToDevice, m->stream));
  if (source)
    MED_TRY(m, cudaMemcpyAsync(m->src, source, (size_t)m->nodes * m->tsize,
                               cudaMemcpyHostToDevice, m->stream));
  else
    MED_TRY(m, cudaMemsetAsync(m->src, 0, (size_t)m->nodes * m->tsize, m->stream));
  MED_TRY(m, cudaStreamSynchronize(m->stream));
  m->cur = 0;
  m->steps = 0;
  m->t = 0;
  m->loaded = true;
  return CBM_OK;
}

int cbm_medium_step(cbm_medium* m, int32_t nsteps, int32_t flags) {
  if (!m) return mfail(m, CBM_ERR_ARG, "null medium");
  if (!m->loaded) return mfail(m, CBM_ERR_STATE, "cbm_medium_step before cbm_medium_upload");
  if (nsteps < 0) return mfail(m, CBM_ERR_ARG, "nsteps must be >= 0");
  if (m->fused && nsteps > 0) {
    const int rc = m->tsize == 8 ? enqueue_fused_t<double>(m, nsteps) : enqueue_fused_t<float>(m, nsteps);
    if (rc != CBM_OK) return rc;
    for (int s = 0; s < nsteps; ++s) {
      m->steps += 1;
      m->t += m->cfg.dt;  // obj.t += dt
    }
  } else {
    for (int s = 0; s < nsteps; ++s) {
      const int rc = m->tsize == 8 ? enqueue_step_t<double>(m) : enqueue_step_t<float>(m);
      if (rc != CBM_OK) return rc;
      m->steps += 1;
      m->t += m->cfg.dt;  // obj.t += dt
    }
  }
  if (flags & CBM_SYNC) MED_TRY(m, cudaStreamSynchronize(m->stream));
  return CBM_OK;
}

int cbm_medium_download(cbm_medium* m, void* fields, double* t) {
  if (!m || !fields) return mfail(m, CBM_ERR_ARG, "null argument");
  if (!m->loaded) return mfail(m, CBM_ERR_STATE, "cbm_medium_download before cbm_medium_upload");
  const size_t fb = (size_t)m->nodes * m->cfg.n_fields * m->tsize;
  MED_TRY(m, cudaMemcpyAsync(fields, m->u[m->cur], fb, cudaMemcpyDeviceToHost, m->stream));
  MED_TRY(m, cudaStreamSynchronize(m->stream));
  if (t) *t = m->t;
  return CBM_OK;
}

void* cbm_medium_stream(cbm_medium* m) { return m ? (void*)m->stream : nullptr; }

}  // extern "C"
