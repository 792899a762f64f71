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
// from its checkpoint, keeping its states, cell grids and interacting pairs,
// and then swept backwards, so long trajectories need O(T/K + K) states
// instead of O(T).
//
// Layout and launches.  Each step's grid (counting sort by cell, ascending
// index inside a cell) is followed by a gather of the positions into slot
// order (double4/float4 with the agent index in w), so a thread walks its 27
// cells as 9 contiguous slot runs, in the reference's order.  The recompute
// pass records, per slot, the partner slots that carry a force term; the
// backward step visits only those pairs.  All buffers of a shape (n, steps,
// checkpoint interval) are kept, and the whole device part of a run is one
// CUDA graph replayed by later runs of the same shape; host copies of the
// inputs and results stay outside the graph.
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
struct AV4;
template <>
struct AV4<float> {
  using type = float4;
  __device__ static float enc(int i) { return __int_as_float(i); }
  __device__ static int dec(float w) { return __float_as_int(w); }
};
template <>
struct AV4<double> {
  using type = double4;
  __device__ static double enc(int i) { return __longlong_as_double((long long)i); }
  __device__ static int dec(double w) { return (int)__double_as_longlong(w); }
};

template <typename T>
struct AdjParams {
  using V4 = typename AV4<T>::type;
  T* xn[3];             // x_{n+1}, index order (forward)
  const V4* xs;         // x_n in slot order, w = agent index
  const V4* ls;         // lambda_{n+1} in slot order (backward)
  T* lam_out[3];        // lambda_n, index order (backward)
  const int* cell_start;
  int* pair_n;          // per slot: partners with a force term (recompute, backward)
  int* pair_list;       // entry k of slot s at k * n + s: the partner's slot
  int cap;
  double* gpart;        // per block: running dL/dtheta partials (3 per block)
  Counters* ctr;
  int n;
  int nc[3];
  T lo[3], hi[3];
  T edge;
  T dt, k, a, rho, ratt, cut2;
};

// x (index order) gathered into slot order, agent index in w
template <typename T>
__global__ void __launch_bounds__(kTile) k_adj_gather(const T* x0, const T* x1, const T* x2,
                                                      const int* agents, typename AV4<T>::type* out,
                                                      int n) {
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s >= n) return;
  const int j = agents[s];
  typename AV4<T>::type v;
  v.x = x0[j];
  v.y = x1[j];
  v.z = x2[j];
  v.w = AV4<T>::enc(j);
  out[s] = v;
}

// forward Euler step of the agent in slot s: the reference's expression
// order, cells x fastest, ascending index inside a cell (the plain path's
// CellLinked sums).  With LIST, the slots of the partners that carry a
// force term are recorded in order for the backward step.
template <typename T, bool LIST>
__global__ void __launch_bounds__(kTile) k_adj_forward(AdjParams<T> A) {
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s >= A.n) return;
  const typename AV4<T>::type me = A.xs[s];
  const int i = AV4<T>::dec(me.w);
  const T xi[3] = {me.x, me.y, me.z};
  int q[3];
  cell_coords<3>(A.nc, cell_of<T, 3>(A.edge, A.lo, A.hi, A.nc, xi), q);
  const int xa = max(q[0] - 1, 0), xb = min(q[0] + 1, A.nc[0] - 1);
  T acc[3] = {(T)0, (T)0, (T)0};
  int m = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = q[2] + dz;
    if (z < 0 || z >= A.nc[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = q[1] + dy;
      if (y < 0 || y >= A.nc[1]) continue;
      const int row = (z * A.nc[1] + y) * A.nc[0];
      const int t1 = A.cell_start[row + xb + 1];
      for (int t = A.cell_start[row + xa]; t < t1; ++t) {
        if (t == s) continue;
        const typename AV4<T>::type o = A.xs[t];
        T e[3];
        e[0] = xi[0] - o.x;
        T s2 = e[0] * e[0];
        e[1] = xi[1] - o.y;
        s2 = s2 + e[1] * e[1];
        e[2] = xi[2] - o.z;
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
        if (LIST) {
          if (m < A.cap) A.pair_list[(long long)m * A.n + s] = t;
          ++m;
        }
      }
    }
  }
  if (LIST) {
    A.pair_n[s] = m < A.cap ? m : A.cap;
    if (m > A.cap) atomicOr(&A.ctr->err, kErrNeighborOverflow);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) A.xn[d][i] = xi[d] + acc[d] * A.dt;
}

// one backward step at state x_n: lambda_n from lambda_{n+1} over the pairs
// recorded by the recompute pass, and this step's dL/dtheta terms added to
// the block's running partial sums
template <typename T>
__global__ void __launch_bounds__(kTile) k_adj_backward(AdjParams<T> A) {
  __shared__ double red[3][kTile];
  const int s = blockIdx.x * kTile + threadIdx.x;
  double g[3] = {0.0, 0.0, 0.0};
  if (s < A.n) {
    const typename AV4<T>::type me = A.xs[s];
    const typename AV4<T>::type lm = A.ls[s];
    const int i = AV4<T>::dec(me.w);
    const T xi[3] = {me.x, me.y, me.z};
    const T li[3] = {lm.x, lm.y, lm.z};
    T adj[3] = {(T)0, (T)0, (T)0};
    T gk = (T)0, ga = (T)0, gr = (T)0;
    const int m = A.pair_n[s];
    for (int kk = 0; kk < m; ++kk) {
      const int t = A.pair_list[(long long)kk * A.n + s];
      const typename AV4<T>::type o = A.xs[t];
      const typename AV4<T>::type lo = A.ls[t];
      T r[3];
      r[0] = xi[0] - o.x;
      T s2 = r[0] * r[0];
      r[1] = xi[1] - o.y;
      s2 = s2 + r[1] * r[1];
      r[2] = xi[2] - o.z;
      s2 = s2 + r[2] * r[2];
      const T dd = sqrt(s2);  // every recorded pair has dd < r_att
      T F, Fp, dk, da, drho;
      if (dd < A.rho) {
        F = A.k * (A.rho - dd);
        Fp = -A.k;
        dk = A.rho - dd;
        da = (T)0;
        drho = A.k;
      } else {
        F = -(A.a * (dd - A.rho));
        Fp = -A.a;
        dk = (T)0;
        da = -(dd - A.rho);
        drho = A.a;
      }
      const T inv = (T)1 / dd;
      const T sc = F * inv;
      const T c = (Fp * dd - F) * inv * inv * inv;
      const T dl[3] = {li[0] - lo.x, li[1] - lo.y, li[2] - lo.z};
      T rdl = (T)0, rli = (T)0;
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        rdl += r[d] * dl[d];
        rli += r[d] * li[d];
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) adj[d] += sc * dl[d] + c * rdl * r[d];
      gk += dk * inv * rli;
      ga += da * inv * rli;
      gr += drho * inv * rli;
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) A.lam_out[d][i] = li[d] + A.dt * adj[d];
    g[0] = (double)(A.dt * gk);
    g[1] = (double)(A.dt * ga);
    g[2] = (double)(A.dt * gr);
  }
  // deterministic block sum (fixed tree), added to this block's running sum
#pragma unroll
  for (int q = 0; q < 3; ++q) red[q][threadIdx.x] = g[q];
  __syncthreads();
  for (int o = kTile / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o)
#pragma unroll
      for (int q = 0; q < 3; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x < 3) A.gpart[blockIdx.x * 3 + threadIdx.x] += red[threadIdx.x][0];
}

// lambda_T = 2 (x_T - x*) / (3N) and per-block partial sums of the loss
template <typename T>
__global__ void __launch_bounds__(kTile) k_adj_loss(const T* x0, const T* x1, const T* x2,
                                                    const T* tgt0, const T* tgt1, const T* tgt2,
                                                    T* l0, T* l1, T* l2, int n, double* lpart) {
  __shared__ double red[kTile];
  const int i = blockIdx.x * kTile + threadIdx.x;
  const T* x[3] = {x0, x1, x2};
  const T* tg[3] = {tgt0, tgt1, tgt2};
  T* lo[3] = {l0, l1, l2};
  double l = 0.0;
  if (i < n) {
    const T inv3n = (T)2 / (T)(3.0 * (double)n);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const T e = x[d][i] - tg[d][i];
      lo[d][i] = inv3n * e;
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

// Device buffers and the captured graph of one run shape.
struct Plan {
  int n = -1, nsteps = -1, K = -1;
  bool backward = false;
  std::vector<void*> bufs;
  cudaGraphExec_t graph = nullptr;
  void* in_x[3] = {};    // x0 (index order)
  void* in_tgt[3] = {};  // target
  void* out_xT[3] = {};  // x_T (inside a state buffer)
  void* out_dx0[3] = {}; // lambda_0
  double* gpart = nullptr;
  double* lpart = nullptr;
  int blocks = 1;
  void release() {
    if (graph) cudaGraphExecDestroy(graph);
    graph = nullptr;
    for (void* p : bufs) cudaFree(p);
    bufs.clear();
    n = nsteps = K = -1;
  }
};

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
  int cap = 64;          // pair-row capacity of the recompute pass
  // grid scratch
  int* cell_count = nullptr;
  unsigned long long* scan_state = nullptr;
  int* agent_cell = nullptr;
  int* agent_rank = nullptr;
  int* cell_tmp = nullptr;
  Counters* ctr = nullptr;
  Plan plan[2];          // [0] forward only, [1] forward + backward
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

// grid of state x (index order) and its positions in slot order
template <typename T>
void build_grid(cbm_adjoint* a, T* const* x, int n, int* cell_start, int* cell_agents,
                typename AV4<T>::type* xs) {
  GridParams<T> G = grid_params<T>(a, (const T* const*)x, n, cell_start, cell_agents);
  const int nb = n > 0 ? (n + kTile - 1) / kTile : 1;
  k_grid_hist<T, 3><<<nb, kTile, 0, a->stream>>>(G);
  k_scan_cells<<<a->n_tiles, kTile, 0, a->stream>>>(grid_scan_args(G));
  k_grid_scatter<T><<<nb, kTile, 0, a->stream>>>(G);
  k_grid_stable<T><<<nb, kTile, 0, a->stream>>>(G);
  k_adj_gather<T><<<nb, kTile, 0, a->stream>>>(x[0], x[1], x[2], cell_agents, xs, n);
}

template <typename T>
AdjParams<T> adj_params(cbm_adjoint* a, int n) {
  AdjParams<T> A;
  memset(&A, 0, sizeof A);
  const cbm_config& k = a->cfg;
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
  A.cap = a->cap;
  A.ctr = a->ctr;
  return A;
}

// Buffers of a shape and the enqueue of its device work (captured once).
template <typename T>
int make_plan(cbm_adjoint* a, Plan& P, int n, int nsteps, int K, bool backward) {
  using V4 = typename AV4<T>::type;
  P.release();
  const size_t S = sizeof(T), nb = (size_t)std::max(n, 1) * S, n1 = (size_t)std::max(n, 1);
  const int blocks = n > 0 ? (n + kTile - 1) / kTile : 1;
  const int nseg = backward ? std::max((nsteps + K - 1) / K, 1) : 0;
  const int Kb = backward ? K : 1;
  bool ok = true;
  auto get = [&](size_t bytes) -> void* {
    void* p = nullptr;
    if (!ok || cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    P.bufs.push_back(p);
    return p;
  };
  T* fw[2][3];
  T* ckpt[3] = {};
  T* seg[3] = {};
  T* lam[2][3] = {};
  T* tgt[3] = {};
  for (int d = 0; d < 3; ++d) {
    P.in_x[d] = get(nb);
    fw[0][d] = (T*)get(nb);
    fw[1][d] = (T*)get(nb);
    if (backward) {
      tgt[d] = (T*)get(nb);
      P.in_tgt[d] = tgt[d];
      ckpt[d] = (T*)get(nb * (size_t)nseg);
      seg[d] = (T*)get(nb * (size_t)(K + 1));
      lam[0][d] = (T*)get(nb);
      lam[1][d] = (T*)get(nb);
    }
  }
  int* starts = (int*)get((size_t)(a->n_cells + 1) * 4 * (size_t)Kb);
  int* agents = (int*)get(n1 * 4 * (size_t)Kb);
  V4* xs = (V4*)get(n1 * sizeof(V4) * (size_t)Kb);
  V4* ls = backward ? (V4*)get(n1 * sizeof(V4)) : nullptr;
  int* pair_n = backward ? (int*)get(n1 * 4 * (size_t)K) : nullptr;
  int* pair_list = backward ? (int*)get(n1 * 4 * (size_t)a->cap * (size_t)K) : nullptr;
  P.gpart = (double*)get((size_t)blocks * 3 * 8);
  P.lpart = (double*)get((size_t)blocks * 8);
  if (!ok) {
    P.release();
    return afail(a, CBM_ERR_NOMEM, "adjoint buffers do not fit");
  }
  P.n = n;
  P.nsteps = nsteps;
  P.K = K;
  P.backward = backward;
  P.blocks = blocks;
  cudaStream_t st = a->stream;
  cudaGraph_t g = nullptr;
  ACUDA(a, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  // forward sweep, keeping a checkpoint every K steps
  for (int d = 0; d < 3; ++d)
    cudaMemcpyAsync(fw[0][d], P.in_x[d], nb, cudaMemcpyDeviceToDevice, st);
  for (int s = 0; s < nsteps; ++s) {
    T* const* cur = fw[s % 2];
    T* const* nxt = fw[(s + 1) % 2];
    if (backward && s % K == 0)
      for (int d = 0; d < 3; ++d)
        cudaMemcpyAsync(ckpt[d] + (size_t)(s / K) * n, cur[d], nb, cudaMemcpyDeviceToDevice, st);
    build_grid<T>(a, cur, n, starts, agents, xs);
    AdjParams<T> A = adj_params<T>(a, n);
    A.cell_start = starts;
    A.xs = xs;
    for (int d = 0; d < 3; ++d) A.xn[d] = nxt[d];
    k_adj_forward<T, false><<<blocks, kTile, 0, st>>>(A);
  }
  for (int d = 0; d < 3; ++d) P.out_xT[d] = fw[nsteps % 2][d];
  if (backward) {
    T* const* xT = fw[nsteps % 2];
    k_adj_loss<T><<<blocks, kTile, 0, st>>>(xT[0], xT[1], xT[2], tgt[0], tgt[1], tgt[2], lam[0][0],
                                            lam[0][1], lam[0][2], n, P.lpart);
    cudaMemsetAsync(P.gpart, 0, (size_t)blocks * 3 * 8, st);
    int li = 0;  // lam[li] holds lambda_{n+1}
    for (int sg = nseg - 1; sg >= 0; --sg) {
      const int n0 = sg * K, n1s = std::min(n0 + K, nsteps), len = n1s - n0;
      for (int d = 0; d < 3; ++d)
        cudaMemcpyAsync(seg[d], ckpt[d] + (size_t)sg * n, nb, cudaMemcpyDeviceToDevice, st);
      // recompute the segment, keeping each step's grid, slot positions and pairs
      for (int m = 0; m < len; ++m) {
        T* cur[3];
        T* nxt[3];
        for (int d = 0; d < 3; ++d) {
          cur[d] = seg[d] + (size_t)m * n;
          nxt[d] = seg[d] + (size_t)(m + 1) * n;
        }
        int* gs = starts + (size_t)m * (a->n_cells + 1);
        int* ga = agents + (size_t)m * n;
        V4* gx = xs + (size_t)m * n;
        build_grid<T>(a, cur, n, gs, ga, gx);
        AdjParams<T> A = adj_params<T>(a, n);
        A.cell_start = gs;
        A.xs = gx;
        A.pair_n = pair_n + (size_t)m * n;
        A.pair_list = pair_list + (size_t)m * n * a->cap;
        for (int d = 0; d < 3; ++d) A.xn[d] = nxt[d];
        k_adj_forward<T, true><<<blocks, kTile, 0, st>>>(A);
      }
      for (int m = len - 1; m >= 0; --m) {
        int* ga = agents + (size_t)m * n;
        const int nbk = n > 0 ? (n + kTile - 1) / kTile : 1;
        k_adj_gather<T><<<nbk, kTile, 0, st>>>(lam[li][0], lam[li][1], lam[li][2], ga, ls, n);
        AdjParams<T> A = adj_params<T>(a, n);
        A.xs = xs + (size_t)m * n;
        A.ls = ls;
        A.pair_n = pair_n + (size_t)m * n;
        A.pair_list = pair_list + (size_t)m * n * a->cap;
        A.gpart = P.gpart;
        for (int d = 0; d < 3; ++d) A.lam_out[d] = lam[li ^ 1][d];
        k_adj_backward<T><<<blocks, kTile, 0, st>>>(A);
        li ^= 1;
      }
    }
    for (int d = 0; d < 3; ++d) P.out_dx0[d] = lam[li][d];
  }
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (e != cudaSuccess) {
    P.release();
    return afail(a, CBM_ERR_CUDA, "adjoint graph capture failed: %s", cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&P.graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) {
    P.graph = nullptr;
    P.release();
    return afail(a, CBM_ERR_CUDA, "adjoint graph instantiate failed: %s", cudaGetErrorString(e));
  }
  return CBM_OK;
}

template <typename T>
int run(cbm_adjoint* a, const void* const* x0h, int n, int nsteps, int K, const void* const* tgth,
        double* loss, double* dtheta, void* const* dx0h, void* const* xTh, bool backward) {
  const size_t nb = (size_t)n * sizeof(T);
  if (backward && K > nsteps) K = std::max(nsteps, 1);  // one segment either way
  Plan& P = a->plan[backward ? 1 : 0];
  if (P.n != n || P.nsteps != nsteps || (backward && P.K != K) || !P.graph) {
    int rc = make_plan<T>(a, P, n, nsteps, backward ? K : 1, backward);
    if (rc) return rc;
  }
  cudaStream_t st = a->stream;
  for (int d = 0; d < 3; ++d) {
    if (nb) ACUDA(a, cudaMemcpyAsync(P.in_x[d], x0h[d], nb, cudaMemcpyHostToDevice, st));
    if (backward && nb) ACUDA(a, cudaMemcpyAsync(P.in_tgt[d], tgth[d], nb, cudaMemcpyHostToDevice, st));
  }
  ACUDA(a, cudaGraphLaunch(P.graph, st));
  if (xTh)
    for (int d = 0; d < 3; ++d)
      if (xTh[d] && nb) ACUDA(a, cudaMemcpyAsync(xTh[d], P.out_xT[d], nb, cudaMemcpyDeviceToHost, st));
  std::vector<double> gp, lp;
  if (backward) {
    gp.resize((size_t)P.blocks * 3);
    lp.resize((size_t)P.blocks);
    ACUDA(a, cudaMemcpyAsync(gp.data(), P.gpart, gp.size() * 8, cudaMemcpyDeviceToHost, st));
    ACUDA(a, cudaMemcpyAsync(lp.data(), P.lpart, lp.size() * 8, cudaMemcpyDeviceToHost, st));
    if (dx0h)
      for (int d = 0; d < 3; ++d)
        if (dx0h[d] && nb) ACUDA(a, cudaMemcpyAsync(dx0h[d], P.out_dx0[d], nb, cudaMemcpyDeviceToHost, st));
  }
  Counters hc;
  ACUDA(a, cudaMemcpyAsync(&hc, a->ctr, sizeof hc, cudaMemcpyDeviceToHost, st));
  ACUDA(a, cudaStreamSynchronize(st));
  if (hc.err) {
    int zero = 0;
    ACUDA(a, cudaMemcpy(&a->ctr->err, &zero, sizeof zero, cudaMemcpyHostToDevice));
    if (hc.err & kErrTimeout) return afail(a, CBM_ERR_TIMEOUT, "a bounded device-side wait gave up");
    if (hc.err & kErrNeighborOverflow)
      return afail(a, CBM_ERR_NEIGHBOR_OVERFLOW,
                   "an agent had more than %d interacting partners in one step", a->cap);
  }
  if (backward) {
    double l = 0.0, g[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < P.blocks; ++b) {  // fixed order: deterministic
      l += lp[(size_t)b];
      for (int m = 0; m < 3; ++m) g[m] += gp[(size_t)b * 3 + m];
    }
    if (loss) *loss = n > 0 ? l / (3.0 * (double)n) : 0.0;
    if (dtheta)
      for (int m = 0; m < 3; ++m) dtheta[m] = g[m];
  }
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
  a->cap = std::max(k.n_max_neighbors, 64);
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
  for (Plan& P : a->plan) P.release();
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
