// cbm_adjoint.cu — exact gradients of a trajectory loss with respect to the
// interaction parameters and the initial positions, by a hand-written
// reverse (adjoint) sweep of the force + Euler step with checkpointing.
//
// Forward map (the 3D soft-sphere ODE of the reference's agentODE with
// Euler, src/integrators.jl:465-505): x_{n+1} = x_n + dt F(x_n; theta),
//   F_i = sum_j f(r_ij),  f(r) = (F(d)/d) r,  r = x_i - x_j, d = |r|,
//   F(d) = k (rho - d) for d < rho,  -a (d - rho) for rho <= d < r_att,
// with theta = (k, a, rho = 2r) and r_att = 3r.  Loss L = mean over agents and
// axes of (x_T - x*)^2.  Adjoint (lambda_n = dL/dx_n):
//   lambda_T = 2 (x_T - x*) / (3N)
//   lambda_n = lambda_{n+1} + dt J_n^T lambda_{n+1},
//   (J^T l)_i = sum_j [ s (l_i - l_j) + c r (r . (l_i - l_j)) ],
//     s = F/d,  c = (F'(d) d - F) / d^3   (the Hessian of the pair term is
//     s I + c r r^T, symmetric, and f_ji = -f_ij)
//   dL/dtheta += dt sum_i lambda_{n+1,i} . sum_j (dF/dtheta / d) r_ij.
// The cutoff r_att is held fixed in the derivative (a pair crossing it
// changes the force discontinuously; that measure-zero event has no
// derivative), which is also what forward-mode dual numbers of the same
// program compute.
//
// Memory: checkpoints every `checkpoint_every` steps; a segment is recomputed
// from its checkpoint, keeping its states and cell grids, and then swept
// backwards, so long trajectories need O(T/K + K) states instead of O(T).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cbm_b200.h"
#include "cbm_grid.cuh"

using namespace cbm;

namespace {

template <typename T>
struct AdjParams {
  const T* x[3];        // state x_n (index order)
  T* xn[3];             // x_{n+1} (forward) or unused
  const T* lam[3];      // lambda_{n+1}
  T* lam_out[3];        // lambda_n
  double* gpart;        // per block: running dL/dtheta partials (3 per block)
  const int* cell_start;
  const int* cell_agents;
  int n;
  int nc[3];
  T lo[3], hi[3];
  T edge;
  T dt, k, a, rho, ratt, cut2;
};

template <typename T>
__device__ __forceinline__ void neighbors3(const AdjParams<T>& A, int i, const T* xi, int* qc) {
  cell_coords<3>(A.nc, cell_of<T, 3>(A.edge, A.lo, A.hi, A.nc, xi), qc);
}

// forward Euler step: the reference's expression order, cells x fastest,
// ascending index inside a cell (same sums as the plain path's CellLinked)
template <typename T>
__global__ void __launch_bounds__(kTile) k_adj_forward(AdjParams<T> A) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= A.n) return;
  T xi[3] = {A.x[0][i], A.x[1][i], A.x[2][i]};
  int q[3];
  neighbors3(A, i, xi, q);
  T acc[3] = {(T)0, (T)0, (T)0};
  for (int kk = 0; kk < 27; ++kk) {
    const int pn = cell_neigh<3>(A.nc, q, kk);
    if (pn < 0) continue;
    for (int s = A.cell_start[pn]; s < A.cell_start[pn + 1]; ++s) {
      const int j = A.cell_agents[s];
      if (j == i) continue;
      T e[3];
      e[0] = xi[0] - A.x[0][j];
      T s2 = e[0] * e[0];
      e[1] = xi[1] - A.x[1][j];
      s2 = s2 + e[1] * e[1];
      e[2] = xi[2] - A.x[2][j];
      s2 = s2 + e[2] * e[2];
      if (s2 >= A.cut2) continue;
      const T dd = sqrt(s2);
      T F;
      if (dd < A.rho) F = A.k * (A.rho - dd);
      else if (dd < A.ratt) F = -(A.a * (dd - A.rho));
      else continue;
      const T sc = F / dd;
#pragma unroll
      for (int d = 0; d < 3; ++d) acc[d] = acc[d] + sc * e[d];
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) A.xn[d][i] = xi[d] + acc[d] * A.dt;
}

// one backward step: lambda_n from lambda_{n+1} at state x_n, and this
// step's dL/dtheta terms added to the block's running partial sums
template <typename T>
__global__ void __launch_bounds__(kTile) k_adj_backward(AdjParams<T> A) {
  __shared__ double red[3][kTile];
  const int i = blockIdx.x * kTile + threadIdx.x;
  double g[3] = {0.0, 0.0, 0.0};
  if (i < A.n) {
    const T xi[3] = {A.x[0][i], A.x[1][i], A.x[2][i]};
    const T li[3] = {A.lam[0][i], A.lam[1][i], A.lam[2][i]};
    int q[3];
    neighbors3(A, i, xi, q);
    T adj[3] = {(T)0, (T)0, (T)0};
    T gk = (T)0, ga = (T)0, gr = (T)0;
    for (int kk = 0; kk < 27; ++kk) {
      const int pn = cell_neigh<3>(A.nc, q, kk);
      if (pn < 0) continue;
      for (int s = A.cell_start[pn]; s < A.cell_start[pn + 1]; ++s) {
        const int j = A.cell_agents[s];
        if (j == i) continue;
        T r[3];
        r[0] = xi[0] - A.x[0][j];
        T s2 = r[0] * r[0];
        r[1] = xi[1] - A.x[1][j];
        s2 = s2 + r[1] * r[1];
        r[2] = xi[2] - A.x[2][j];
        s2 = s2 + r[2] * r[2];
        if (s2 >= A.cut2) continue;
        const T dd = sqrt(s2);
        T F, Fp, dk, da, drho;
        if (dd < A.rho) {
          F = A.k * (A.rho - dd);
          Fp = -A.k;
          dk = A.rho - dd;
          da = (T)0;
          drho = A.k;
        } else if (dd < A.ratt) {
          F = -(A.a * (dd - A.rho));
          Fp = -A.a;
          dk = (T)0;
          da = -(dd - A.rho);
          drho = A.a;
        } else {
          continue;
        }
        const T inv = (T)1 / dd;
        const T sc = F * inv;
        const T c = (Fp * dd - F) * inv * inv * inv;
        T dl[3];
        T rdl = (T)0, rli = (T)0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          dl[d] = li[d] - A.lam[d][j];
          rdl += r[d] * dl[d];
          rli += r[d] * li[d];
        }
#pragma unroll
        for (int d = 0; d < 3; ++d) adj[d] += sc * dl[d] + c * rdl * r[d];
        gk += dk * inv * rli;
        ga += da * inv * rli;
        gr += drho * inv * rli;
      }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) A.lam_out[d][i] = li[d] + A.dt * adj[d];
    g[0] = (double)(A.dt * gk);
    g[1] = (double)(A.dt * ga);
    g[2] = (double)(A.dt * gr);
  }
  // deterministic block sum (fixed tree), added to this block's running sum
#pragma unroll
  for (int m = 0; m < 3; ++m) red[m][threadIdx.x] = g[m];
  __syncthreads();
  for (int o = kTile / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int m = 0; m < 3; ++m) red[m][threadIdx.x] += red[m][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) A.gpart[blockIdx.x * 3 + threadIdx.x] += red[threadIdx.x][0];
}

// lambda_T = 2 (x_T - x*) / (3N) and per-block partial sums of the loss
template <typename T>
__global__ void __launch_bounds__(kTile) k_adj_loss(AdjParams<T> A, const T* tgt0, const T* tgt1,
                                                    const T* tgt2, double* lpart) {
  __shared__ double red[kTile];
  const int i = blockIdx.x * kTile + threadIdx.x;
  const T* tg[3] = {tgt0, tgt1, tgt2};
  double l = 0.0;
  if (i < A.n) {
    const T inv3n = (T)2 / (T)(3.0 * (double)A.n);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T e = A.x[d][i] - tg[d][i];
      A.lam_out[d][i] = inv3n * e;
      l += (double)e * (double)e;
    }
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int o = kTile / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) lpart[blockIdx.x] = red[0];
}

}  // namespace

struct cbm_adjoint {
  cbm_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<void*> allocs;
  size_t ts = 8;
  int n_max = 0;
  int nc[3] = {1, 1, 1};
  int n_cells = 1;
  int n_tiles = 1;
  int blocks = 1;
  // grid scratch
  int* cell_count = nullptr;
  unsigned long long* scan_state = nullptr;
  int* agent_cell = nullptr;
  int* agent_rank = nullptr;
  int* cell_tmp = nullptr;
  Counters* ctr = nullptr;
  double* gpart = nullptr;
  double* lpart = nullptr;
};

namespace {

std::string g_adj_error;

int afail(cbm_adjoint* a, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (a) a->err = buf;
  else g_adj_error = buf;
  return code;
}

#define ACUDA(a, call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return afail(a, CBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

// device buffers of one run, freed at the end of the run
struct RunBufs {
  std::vector<void*> v;
  bool ok = true;
  void* get(size_t bytes) {
    if (!ok) return nullptr;
    void* p = nullptr;
    if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    v.push_back(p);
    return p;
  }
  ~RunBufs() {
    for (void* p : v) cudaFree(p);
  }
};

template <typename T>
GridParams<T> grid_params(cbm_adjoint* a, const T* const* x, int n, int* cell_start,
                          int* cell_agents) {
  GridParams<T> G;
  memset(&G, 0, sizeof G);
  for (int d = 0; d < 3; ++d) {
    G.pos[d] = x[d];
    G.box_lo[d] = (T)a->cfg.box_lo[d];
    G.box_hi[d] = (T)a->cfg.box_hi[d];
    G.n_cells_d[d] = a->nc[d];
  }
  G.n = n;
  G.edge = (T)a->cfg.cell_edge;
  G.n_cells = a->n_cells;
  G.n_scan_tiles = a->n_tiles;
  G.ctr = a->ctr;
  G.cell_count = a->cell_count;
  G.cell_start = cell_start;
  G.scan_state = a->scan_state;
  G.agent_cell = a->agent_cell;
  G.agent_rank = a->agent_rank;
  G.cell_tmp = a->cell_tmp;
  G.cell_agents = cell_agents;
  return G;
}

template <typename T>
void build_grid(cbm_adjoint* a, const T* const* x, int n, int* cell_start, int* cell_agents) {
  GridParams<T> G = grid_params<T>(a, x, n, cell_start, cell_agents);
  const int nb = n > 0 ? (n + kTile - 1) / kTile : 1;
  k_grid_hist<T, 3><<<nb, kTile, 0, a->stream>>>(G);
  k_scan_cells<<<a->n_tiles, kTile, 0, a->stream>>>(grid_scan_args(G));
  k_grid_scatter<T><<<nb, kTile, 0, a->stream>>>(G);
  k_grid_stable<T><<<nb, kTile, 0, a->stream>>>(G);
}

template <typename T>
AdjParams<T> adj_params(cbm_adjoint* a, int n, const int* cell_start, const int* cell_agents) {
  AdjParams<T> A;
  memset(&A, 0, sizeof A);
  const cbm_config& k = a->cfg;
  A.cell_start = cell_start;
  A.cell_agents = cell_agents;
  A.n = n;
  for (int d = 0; d < 3; ++d) {
    A.nc[d] = a->nc[d];
    A.lo[d] = (T)k.box_lo[d];
    A.hi[d] = (T)k.box_hi[d];
  }
  A.edge = (T)k.cell_edge;
  A.dt = (T)k.dt;
  A.k = (T)k.k_rep;
  A.a = (T)k.k_att;
  A.rho = (T)k.r_rep;
  A.ratt = (T)k.r_att;
  double c = std::max(k.r_rep, k.r_att), v = c * c * (1.0 + 1e-5);
  T t = (T)v;
  A.cut2 = (double)t < v ? std::nextafter(t, (T)INFINITY) : t;
  A.gpart = a->gpart;
  return A;
}

template <typename T>
int run(cbm_adjoint* a, const void* const* x0h, int n, int nsteps, int K, const void* const* tgth,
        double* loss, double* dtheta, void* const* dx0h, void* const* xTh, bool backward) {
  const size_t S = sizeof(T), nb = (size_t)n * S;
  const int blocks = n > 0 ? (n + kTile - 1) / kTile : 1;
  const int nseg = (nsteps + K - 1) / K;
  RunBufs B;
  T* ckpt[3];
  T* seg[3];      // K + 1 states of a segment
  T* lamA[3];
  T* lamB[3];
  T* tgt[3];
  for (int d = 0; d < 3; ++d) {
    ckpt[d] = backward ? (T*)B.get(nb * (size_t)std::max(nseg, 1)) : nullptr;
    seg[d] = (T*)B.get(nb * (size_t)(backward ? K + 1 : 2));
    lamA[d] = (T*)B.get(nb);
    lamB[d] = (T*)B.get(nb);
    tgt[d] = (T*)B.get(nb);
  }
  int* starts = (int*)B.get((size_t)(a->n_cells + 1) * 4 * (size_t)K);
  int* agents = (int*)B.get((size_t)std::max(n, 1) * 4 * (size_t)K);
  double* gpart = (double*)B.get((size_t)blocks * 3 * 8);
  double* lpart = (double*)B.get((size_t)blocks * 8);
  if (!B.ok) return afail(a, CBM_ERR_NOMEM, "adjoint buffers do not fit");
  a->gpart = gpart;
  cudaStream_t st = a->stream;
  auto state = [&](T* const* base, int m, T** out) {
    for (int d = 0; d < 3; ++d) out[d] = base[d] + (size_t)m * n;
  };
  // forward sweep, keeping a checkpoint every K steps
  for (int d = 0; d < 3; ++d) {
    ACUDA(a, cudaMemcpyAsync(seg[d], x0h[d], nb, cudaMemcpyHostToDevice, st));
    if (tgth && tgth[d]) ACUDA(a, cudaMemcpyAsync(tgt[d], tgth[d], nb, cudaMemcpyHostToDevice, st));
  }
  for (int s = 0; s < nsteps; ++s) {
    T* cur[3];
    T* nxt[3];
    state(seg, s % 2, cur);
    state(seg, (s + 1) % 2, nxt);
    if (backward && s % K == 0)
      for (int d = 0; d < 3; ++d)
        ACUDA(a, cudaMemcpyAsync(ckpt[d] + (size_t)(s / K) * n, cur[d], nb, cudaMemcpyDeviceToDevice, st));
    build_grid<T>(a, (const T* const*)cur, n, starts, agents);
    AdjParams<T> A = adj_params<T>(a, n, starts, agents);
    for (int d = 0; d < 3; ++d) {
      A.x[d] = cur[d];
      A.xn[d] = nxt[d];
    }
    k_adj_forward<T><<<blocks, kTile, 0, st>>>(A);
  }
  T* xT[3];
  state(seg, nsteps % 2, xT);
  if (xTh)
    for (int d = 0; d < 3; ++d)
      if (xTh[d]) ACUDA(a, cudaMemcpyAsync(xTh[d], xT[d], nb, cudaMemcpyDeviceToHost, st));
  if (!backward) {
    ACUDA(a, cudaStreamSynchronize(st));
    return CBM_OK;
  }
  // loss and lambda_T
  {
    AdjParams<T> A = adj_params<T>(a, n, starts, agents);
    for (int d = 0; d < 3; ++d) {
      A.x[d] = xT[d];
      A.lam_out[d] = lamA[d];
    }
    k_adj_loss<T><<<blocks, kTile, 0, st>>>(A, tgt[0], tgt[1], tgt[2], lpart);
  }
  ACUDA(a, cudaMemsetAsync(gpart, 0, (size_t)blocks * 3 * 8, st));
  // backward sweep, segment by segment from the last
  T** lam_in = lamA;
  T** lam_out = lamB;
  for (int sg = nseg - 1; sg >= 0; --sg) {
    const int n0 = sg * K, n1 = std::min(n0 + K, nsteps), len = n1 - n0;
    T* base[3];
    for (int d = 0; d < 3; ++d) {
      base[d] = seg[d];
      ACUDA(a, cudaMemcpyAsync(seg[d], ckpt[d] + (size_t)sg * n, nb, cudaMemcpyDeviceToDevice, st));
    }
    // recompute the segment's states and keep each step's grid
    for (int m = 0; m < len; ++m) {
      T* cur[3];
      state(base, m, cur);
      int* gs = starts + (size_t)m * (a->n_cells + 1);
      int* ga = agents + (size_t)m * n;
      build_grid<T>(a, (const T* const*)cur, n, gs, ga);
      if (m + 1 < len) {
        T* nxt[3];
        state(base, m + 1, nxt);
        AdjParams<T> A = adj_params<T>(a, n, gs, ga);
        for (int d = 0; d < 3; ++d) {
          A.x[d] = cur[d];
          A.xn[d] = nxt[d];
        }
        k_adj_forward<T><<<blocks, kTile, 0, st>>>(A);
      }
    }
    for (int m = len - 1; m >= 0; --m) {
      T* cur[3];
      state(base, m, cur);
      AdjParams<T> A = adj_params<T>(a, n, starts + (size_t)m * (a->n_cells + 1), agents + (size_t)m * n);
      for (int d = 0; d < 3; ++d) {
        A.x[d] = cur[d];
        A.lam[d] = lam_in[d];
        A.lam_out[d] = lam_out[d];
      }
      k_adj_backward<T><<<blocks, kTile, 0, st>>>(A);
      std::swap(lam_in, lam_out);
    }
  }
  ACUDA(a, cudaGetLastError());
  std::vector<double> gp((size_t)blocks * 3), lp((size_t)blocks);
  ACUDA(a, cudaMemcpyAsync(gp.data(), gpart, gp.size() * 8, cudaMemcpyDeviceToHost, st));
  ACUDA(a, cudaMemcpyAsync(lp.data(), lpart, lp.size() * 8, cudaMemcpyDeviceToHost, st));
  if (dx0h)
    for (int d = 0; d < 3; ++d)
      if (dx0h[d]) ACUDA(a, cudaMemcpyAsync(dx0h[d], lam_in[d], nb, cudaMemcpyDeviceToHost, st));
  ACUDA(a, cudaStreamSynchronize(st));
  double l = 0.0, g[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < blocks; ++b) {  // fixed order: deterministic
    l += lp[(size_t)b];
    for (int m = 0; m < 3; ++m) g[m] += gp[(size_t)b * 3 + m];
  }
  if (loss) *loss = n > 0 ? l / (3.0 * (double)n) : 0.0;
  if (dtheta)
    for (int m = 0; m < 3; ++m) dtheta[m] = g[m];
  Counters hc;
  ACUDA(a, cudaMemcpy(&hc, a->ctr, sizeof hc, cudaMemcpyDeviceToHost));
  if (hc.err & kErrTimeout) return afail(a, CBM_ERR_TIMEOUT, "a bounded device-side wait gave up");
  return CBM_OK;
}

}  // namespace

extern "C" {

const char* cbm_adjoint_last_error(const cbm_adjoint* a) {
  return a ? a->err.c_str() : g_adj_error.c_str();
}

int cbm_adjoint_create(cbm_adjoint** out, const cbm_config* cfg) {
  if (!out || !cfg) return afail(nullptr, CBM_ERR_ARG, "null argument");
  *out = nullptr;
  const cbm_config& k = *cfg;
  if (k.dims != 3 || k.integrator != CBM_INT_EULER || k.force_mode != CBM_FORCE_DIRECT ||
      k.att_form != CBM_ATT_FROM_REP || k.neighbors != CBM_NEIGH_CELL_LINKED ||
      k.walls != CBM_WALLS_NONE || k.fate != CBM_FATE_NONE || k.medium || k.growth ||
      k.drift_linear != 0)
    return afail(nullptr, CBM_ERR_ARG,
                 "the adjoint covers the 3D soft-sphere Euler ODE with CellLinked neighbors "
                 "(no walls, fate, growth, medium or drift)");
  if (!(k.dt > 0) || !(k.cell_edge >= std::max(k.r_rep, k.r_att)) || !(k.r_att >= k.r_rep))
    return afail(nullptr, CBM_ERR_ARG, "need dt > 0, r_att >= r_rep and cell_edge >= r_att");
  if (k.n_max < 0 || k.n_max >= (1ll << 28)) return afail(nullptr, CBM_ERR_ARG, "n_max out of range");
  cbm_adjoint* a = new cbm_adjoint;
  a->cfg = k;
  a->ts = k.precision == CBM_F64 ? 8 : 4;
  a->n_max = (int)k.n_max;
  cudaGetDevice(&a->device);
  if (cudaStreamCreateWithFlags(&a->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete a;
    return afail(nullptr, CBM_ERR_CUDA, "cudaStreamCreate failed (is a CUDA device present?)");
  }
  long long nc = 1;
  for (int d = 0; d < 3; ++d) {
    a->nc[d] = (int)std::ceil((k.box_hi[d] - k.box_lo[d]) / k.cell_edge + 2.0);  // neighbors.jl:605
    nc *= a->nc[d];
  }
  if (nc >= (1ll << 28)) {
    cudaStreamDestroy(a->stream);
    delete a;
    return afail(nullptr, CBM_ERR_ARG, "cell grid too large");
  }
  a->n_cells = (int)nc;
  a->n_tiles = (a->n_cells + kScanTile - 1) / kScanTile;
  const size_t n = (size_t)std::max(a->n_max, 1);
  bool ok = true;
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (!ok || cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    a->allocs.push_back(p);
    return p;
  };
  a->cell_count = (int*)get((size_t)a->n_cells * 4);
  a->scan_state = (unsigned long long*)get((size_t)a->n_tiles * 8);
  a->agent_cell = (int*)get(n * 4);
  a->agent_rank = (int*)get(n * 4);
  a->cell_tmp = (int*)get(n * 4);
  a->ctr = (Counters*)get(sizeof(Counters));
  if (!ok) {
    for (void* p : a->allocs) cudaFree(p);
    cudaStreamDestroy(a->stream);
    delete a;
    return afail(nullptr, CBM_ERR_NOMEM, "device allocation failed");
  }
  cudaMemsetAsync(a->cell_count, 0, (size_t)a->n_cells * 4, a->stream);
  cudaMemsetAsync(a->scan_state, 0, (size_t)a->n_tiles * 8, a->stream);
  cudaMemsetAsync(a->ctr, 0, sizeof(Counters), a->stream);
  cudaStreamSynchronize(a->stream);
  *out = a;
  return CBM_OK;
}

void cbm_adjoint_destroy(cbm_adjoint* a) {
  if (!a) return;
  cudaSetDevice(a->device);
  cudaStreamSynchronize(a->stream);
  for (void* p : a->allocs) cudaFree(p);
  cudaStreamDestroy(a->stream);
  delete a;
}

int cbm_adjoint_run(cbm_adjoint* a, int64_t n, const void* const* x0, int32_t nsteps,
                    int32_t checkpoint_every, const void* const* target, double* loss,
                    double* dtheta, void* const* dx0, void* const* xT) {
  if (!a || !x0 || !target || nsteps < 0 || checkpoint_every < 1) return afail(a, CBM_ERR_ARG, "bad argument");
  if (n < 0 || n > a->n_max) return afail(a, CBM_ERR_ARG, "n exceeds n_max");
  cudaSetDevice(a->device);
  if (a->ts == 8)
    return run<double>(a, x0, (int)n, nsteps, checkpoint_every, target, loss, dtheta, dx0, xT, true);
  return run<float>(a, x0, (int)n, nsteps, checkpoint_every, target, loss, dtheta, dx0, xT, true);
}

int cbm_adjoint_forward(cbm_adjoint* a, int64_t n, const void* const* x0, int32_t nsteps,
                        void* const* xT) {
  if (!a || !x0 || nsteps < 0) return afail(a, CBM_ERR_ARG, "bad argument");
  if (n < 0 || n > a->n_max) return afail(a, CBM_ERR_ARG, "n exceeds n_max");
  cudaSetDevice(a->device);
  if (a->ts == 8)
    return run<double>(a, x0, (int)n, nsteps, 1, nullptr, nullptr, nullptr, nullptr, xT, false);
  return run<float>(a, x0, (int)n, nsteps, 1, nullptr, nullptr, nullptr, nullptr, xT, false);
}

void* cbm_adjoint_stream(cbm_adjoint* a) { return a ? (void*)a->stream : nullptr; }

}  // extern "C"
