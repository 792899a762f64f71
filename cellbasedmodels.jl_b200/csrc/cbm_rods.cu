// cbm_rods.cu — the rods2D model (src/models/rods.jl) on the device.
//
// One step, as step! runs rods2D with the Euler integrator:
//   1. agentStepDE!: every rod sums rodForces over its neighbors (the
//      CellLinked grid of the committed positions: 9 cells x fastest, rods
//      ascending inside a cell; or all rods) into the new copies fx__, fy__,
//      W__, pressure__, while u += du dt takes du from the committed (lagged)
//      fx, fy, W;
//   2. update!: the new copies are committed;
//   3. computeNeighbors!: the grid is rebuilt on the new positions.
// In rods2D the rods stay in index order.  rods2dGrowth (rods.jl:123-163)
// adds dt(l) = growth/(1 + alpha pressure) and, before step 1, the division
// rule, whose births and removals update! resolves by filling holes from the
// tail (rod_divide).  The force arithmetic is cbm_rods_math.h.
//
// The state is double-buffered: k_rod_step reads buffer a (committed) and
// writes buffer b, so 1 and 2 are one launch and the commit is a swap.  The
// same launch computes the cell of each new position and its atomic rank
// (assignCells); the scan, scatter and stable passes of cbm_grid.cuh finish
// the grid.  Four launches per step (seven with growth: the division flags,
// their scan and the holes come first), replayed from a CUDA graph of two
// steps.
//
// A rod's candidates are spread over a group of kRodLanes lanes: lane k takes
// candidates k, k + G, ...; after each chunk of G the group's terms are
// broadcast by shuffles and every lane adds them in candidate order, so the
// sums have the reference's order.  Only contacts add (a pair without contact
// contributes +0.0, which leaves a sum started at +0.0 unchanged).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/cbm_b200.h"
#include "../../include/cbm_rods_math.h"
#include "cbm_grid.cuh"

using namespace cbm;

namespace {

constexpr int kRodBlock = 128;
#ifndef CBM_ROD_LANES
#define CBM_ROD_LANES 8
#endif
constexpr int kRodLanes = CBM_ROD_LANES;  // lanes per rod
static_assert(kRodLanes == 4 || kRodLanes == 8 || kRodLanes == 16, "lanes per rod");

// the per-rod arrays that a step rewrites; d, l, m are constant in rods2D and
// single arrays, while rods2dGrowth rewrites (moves) every field, so there
// l, lTarget, d and m are double-buffered too
enum {
  kSX = 0, kSY, kSVX, kSVY, kSTH, kSOM, kSFX, kSFY, kSW, kSP, kSCOS, kSSIN,
  kSL, kSLT, kSD, kSM, kStateArrays
};
constexpr int kPlainArrays = kSL;  // arrays of the rods2D state

template <typename T>
struct RodStep {
  T* a[kStateArrays];  // committed
  T* b[kStateArrays];  // written
  const T* d;
  const T* l;
  const T* m;
  const int* cell_start;  // grid of a
  const int* cell_agents;
  int* cell_count;        // zero on entry (the scan clears it)
  int* agent_cell;        // cell and rank of b's positions
  int* agent_rank;
  Counters* ctr;
  int n;
  int full;               // all pairs instead of the grid
  T box_lo[2], box_hi[2], edge;
  int n_cells_d[3];
  T dt, beta, beta_w;
  CbmRodCoef<T> k;
  // rods2dGrowth
  const long long* cnt_a;  // {n, step} of a
  long long* cnt_b;        // {n, step} of b
  const int* div_rank;     // exclusive prefix of the division flags (n_max + 1)
  const int* holes;        // index of the k-th dividing rod
  int n_max;
  T growth, alpha, lt_lo, lt_hi;
  unsigned long long seed;
};

// cos and sin of the uploaded angles
template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_geom(T* const* a, int n) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= n) return;
  T c, s;
  cbm_rod_cossin<T>(a[kSTH][i], &c, &s);
  a[kSCOS][i] = c;
  a[kSSIN][i] = s;
}

template <typename T>
__device__ __forceinline__ T shfl_group(T v, int q) {
  return __shfl_sync(0xffffffffu, v, q, kRodLanes);
}

// assignCells for a row of b (neighbors.jl:763-821)
template <typename T>
__device__ __forceinline__ void rod_assign_cell(const RodStep<T>& R, int row, T x0, T y0) {
  const T x[2] = {x0, y0};
  const int c = cell_of<T, 2>(R.edge, R.box_lo, R.box_hi, R.n_cells_d, x);
  R.agent_cell[row] = c;
  R.agent_rank[row] = atomicAdd(R.cell_count + c, 1);
}

// The rows that @addAgent keeps: A = min(2D, n_max - n) (functionRule.jl:58-70
// drops a birth whose row would pass nMax_)
__device__ __forceinline__ int rod_births(int n, int D, int n_max) {
  return 2 * D < n_max - n ? 2 * D : n_max - n;
}

// rods2dGrowth's rule for a rod with l > lTarget (rods.jl:141-161), with the
// bookkeeping of @addAgent / @removeAgent and update! folded in.  The k-th
// dividing rod (index order) asks for rows n + 2k and n + 2k + 1, of which
// the first A exist, and leaves a hole at its own row.  update! then moves
// the highest surviving rows, newborns first and then old rows from the top,
// into the holes in ascending order while the hole lies below its source
// (kernelListSurvived / kernelFillHolesParameters, update.jl:15-84).  So
// newborn row s lands at holes[n + A - 1 - s] when that index is below D,
// and stays at s otherwise.  Fields not given to @addAgent are the parent's
// committed values.
template <typename T>
__device__ void rod_divide(const RodStep<T>& R, int i, int n) {
  const int D = R.div_rank[n], k = R.div_rank[i];
  const int A = rod_births(n, D, R.n_max);
  const long long step = R.cnt_a[1];
  const T x = R.a[kSX][i], y = R.a[kSY][i], c = R.a[kSCOS][i], s = R.a[kSSIN][i];
  const T l = R.a[kSL][i], d = R.a[kSD][i], om = R.a[kSOM][i];
  // CBMDistributions.uniform(a, b) = (b - a) rand() + a (src/random.jl:15)
  const T ww = ((T)0.1 - (T)-0.1) * cbm_uniform<T>(R.seed, step, (uint32_t)i, CBM_STREAM_ROD_TORQUE, 0u) +
               (T)-0.1;
  const T q = (l + d) / (T)4;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    if (2 * k + h >= A) continue;  // the birth found no row below n_max
    const int slot = n + 2 * k + h;
    const int m = n + A - 1 - slot;  // in [0, A)
    const int row = m < D ? R.holes[m] : slot;
    const T xs = h == 0 ? q * c + x : (-(l + d) / (T)4) * c + x;
    const T ys = h == 0 ? q * s + y : (-(l + d) / (T)4) * s + y;
    const T lt = (R.lt_hi - R.lt_lo) *
                     cbm_uniform<T>(R.seed, step, (uint32_t)i, CBM_STREAM_ROD_TARGET + (uint32_t)h, 0u) +
                 R.lt_lo;
    R.b[kSX][row] = xs;
    R.b[kSY][row] = ys;
    R.b[kSVX][row] = R.a[kSVX][i];
    R.b[kSVY][row] = R.a[kSVY][i];
    R.b[kSTH][row] = R.a[kSTH][i];
    R.b[kSOM][row] = h == 0 ? om + ww : om - ww;
    R.b[kSFX][row] = R.a[kSFX][i];
    R.b[kSFY][row] = R.a[kSFY][i];
    R.b[kSW][row] = R.a[kSW][i];
    R.b[kSP][row] = R.a[kSP][i];
    R.b[kSCOS][row] = c;
    R.b[kSSIN][row] = s;
    R.b[kSL][row] = (l - d) / (T)2;
    R.b[kSLT][row] = lt;
    R.b[kSD][row] = d;
    R.b[kSM][row] = R.a[kSM][i];
    if (!R.full) rod_assign_cell<T>(R, row, xs, ys);
  }
}

// Steps 1 and 2 of one step (rods.jl:86-118 with rodForces, :21-59), and the
// cell assignment of step 3 (assignCells, neighbors.jl:763-821)
template <typename T, bool GROW>
__global__ void __launch_bounds__(kRodBlock) k_rod_step(RodStep<T> R) {
  pdl_wait();
  const int t = blockIdx.x * kRodBlock + threadIdx.x;
  const int i = t / kRodLanes, lane = t % kRodLanes;
  const int n = GROW ? (int)R.cnt_a[0] : R.n;
  const bool live = i < n;
  if (t == 0 && !R.full) {
    R.ctr->scan_ticket = 0u;  // fresh tickets and tile-state generation for the scan
    R.ctr->scan_epoch = R.ctr->scan_epoch + 1u;
  }
  CbmRodGeom<T> g{(T)0, (T)0, (T)1, (T)0, (T)0};
  T d1 = (T)0, m1 = (T)1, vx1 = (T)0, vy1 = (T)0;
  if (live) {
    g = CbmRodGeom<T>{R.a[kSX][i], R.a[kSY][i], R.a[kSCOS][i], R.a[kSSIN][i], R.l[i]};
    d1 = R.d[i];
    m1 = R.m[i];
    vx1 = R.a[kSVX][i];
    vy1 = R.a[kSVY][i];
  }
  // candidate runs: all rods, or the three rows of x-neighbor cells
  int rs[3] = {0, 0, 0}, re[3] = {0, 0, 0};
  if (live) {
    if (R.full) {
      re[0] = n;
    } else {
      const T x[2] = {g.x, g.y};
      const int c = cell_of<T, 2>(R.edge, R.box_lo, R.box_hi, R.n_cells_d, x);
      const int nx = R.n_cells_d[0], ny = R.n_cells_d[1];
      const int qx = c % nx, qy = c / nx;
      const int x0 = qx > 0 ? qx - 1 : 0, x1 = qx < nx - 1 ? qx + 1 : nx - 1;
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        const int py = qy + r - 1;
        if (py < 0 || py >= ny) continue;
        rs[r] = R.cell_start[nx * py + x0];
        re[r] = R.cell_start[nx * py + x1 + 1];
      }
    }
  }
  const int group_shift = (threadIdx.x & 31) & ~(kRodLanes - 1);
  T fx = (T)0, fy = (T)0, w = (T)0, p = (T)0;
#pragma unroll 1
  for (int r = 0; r < 3; ++r) {
    const int chunks = __reduce_max_sync(0xffffffffu, (re[r] - rs[r] + kRodLanes - 1) / kRodLanes);
#pragma unroll 1
    for (int c = 0; c < chunks; ++c) {
      const int s = rs[r] + c * kRodLanes + lane;
      bool hit = false;
      T gx = (T)0, gy = (T)0, gw = (T)0, gp = (T)0;
      if (s < re[r]) {
        const int j = R.full ? s : R.cell_agents[s];
        if (j != i) {
          const CbmRodGeom<T> h{R.a[kSX][j], R.a[kSY][j], R.a[kSCOS][j], R.a[kSSIN][j], R.l[j]};
          hit = cbm_rod_forces<T>(g, d1, vx1, vy1, m1, h, R.d[j], R.a[kSVX][j], R.a[kSVY][j], R.k,
                                  &gx, &gy, &gw);
          if (hit) gp = sqrt(gx * gx + gy * gy);
        }
      }
      const unsigned hits = __ballot_sync(0xffffffffu, hit);
      if (hits == 0u) continue;
      const unsigned mine = (hits >> group_shift) & ((1u << kRodLanes) - 1u);
#pragma unroll
      for (int q = 0; q < kRodLanes; ++q) {
        const T ax = shfl_group(gx, q), ay = shfl_group(gy, q);
        const T aw = shfl_group(gw, q), ap = shfl_group(gp, q);
        if (mine & (1u << q)) {
          fx = fx + ax;
          fy = fy + ay;
          w = w + aw;
          p = p + ap;
        }
      }
    }
  }
  if (!live || lane != 0) return;
  int row = i;  // the final row of rod i
  if constexpr (GROW) {
    if (R.div_rank[i + 1] != R.div_rank[i]) {
      rod_divide<T>(R, i, n);
      return;
    }
    // with fewer births than parents, update! also moves old rows: rod i is
    // the (n - 1 - i - dividers above it)-th surviving old row from the top
    const int D = R.div_rank[n], A = rod_births(n, D, R.n_max);
    if (A < D) {
      const int q = A + (n - 1 - i) - (D - R.div_rank[i + 1]);
      if (q < D && R.holes[q] < i) row = R.holes[q];
    }
  }
  // Euler: u + du dt with the committed forces, then the commit of the sums
  const T dt = R.dt;
  const T vx = vx1, vy = vy1, om = R.a[kSOM][i], th = R.a[kSTH][i];
  const T d = d1, l = g.l, m = m1;
  const T dvx = -R.beta * vx + R.a[kSFX][i] / m;
  const T dvy = -R.beta * vy + R.a[kSFY][i] / m;
  const T den = (m * ((d + l) * (d + l))) / (T)12 + m * (d * d);
  const T dom = R.a[kSW][i] / den - R.beta_w * om;
  const T xn = g.x + vx * dt, yn = g.y + vy * dt, thn = th + om * dt;
  R.b[kSX][row] = xn;
  R.b[kSY][row] = yn;
  R.b[kSVX][row] = vx + dvx * dt;
  R.b[kSVY][row] = vy + dvy * dt;
  R.b[kSTH][row] = thn;
  R.b[kSOM][row] = om + dom * dt;
  R.b[kSFX][row] = fx;
  R.b[kSFY][row] = fy;
  R.b[kSW][row] = w;
  R.b[kSP][row] = p;
  T cn, sn;
  cbm_rod_cossin<T>(thn, &cn, &sn);
  R.b[kSCOS][row] = cn;
  R.b[kSSIN][row] = sn;
  if constexpr (GROW) {
    // dt(l) = growth/(1 + alpha pressure), the committed pressure (rods.jl:137-139)
    R.b[kSL][row] = l + (R.growth / ((T)1 + R.alpha * R.a[kSP][i])) * dt;
    R.b[kSLT][row] = R.a[kSLT][i];
    R.b[kSD][row] = d;
    R.b[kSM][row] = m;
  }
  if (!R.full) rod_assign_cell<T>(R, row, xn, yn);
}

// rods2dGrowth, before the step: the division flags l > lTarget of the
// committed rods (rods.jl:143), as counts for the scan that ranks them
template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_flags(RodStep<T> R, int* flags, Counters* dctr) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i == 0) {
    dctr->scan_ticket = 0u;  // fresh tickets and tile-state generation for the scan
    dctr->scan_epoch = dctr->scan_epoch + 1u;
  }
  if (i >= (int)R.cnt_a[0]) return;
  flags[i] = R.a[kSL][i] > R.a[kSLT][i] ? 1 : 0;
}

// holes[k] = index of the k-th dividing rod; the step's count and counter
template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_holes(RodStep<T> R, int* holes, Counters* ctr) {
  pdl_wait();
  const int i = blockIdx.x * kTile + threadIdx.x;
  const int n = (int)R.cnt_a[0];
  if (i == 0) {
    const int D = R.div_rank[n], A = rod_births(n, D, R.n_max);
    R.cnt_b[0] = n + A - D;  // N + NAdd - NRemove
    R.cnt_b[1] = R.cnt_a[1] + 1;
    if (A < 2 * D) atomicOr(&ctr->err, kErrAgentOverflow);  // births were dropped
  }
  if (i >= n) return;
  if (R.div_rank[i + 1] != R.div_rank[i]) holes[R.div_rank[i]] = i;
}

// k_grid_scatter / k_grid_stable of cbm_grid.cuh with the rod count on the device
template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_scatter(GridParams<T> G, const long long* cnt) {
  pdl_wait();
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= (int)cnt[0]) return;
  G.cell_tmp[G.cell_start[G.agent_cell[i]] + G.agent_rank[i]] = i;
}

template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_stable(GridParams<T> G, const long long* cnt) {
  pdl_wait();
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= (int)cnt[0]) return;
  const int c = G.agent_cell[i];
  const int s0 = G.cell_start[c], s1 = G.cell_start[c + 1];
  int r = 0;
  for (int s = s0; s < s1; ++s) r += ld(G.cell_tmp + s) < i;
  G.cell_agents[s0 + r] = i;
}

}  // namespace

struct cbm_rods {
  cbm_rods_config cfg{};
  int tsize = 4;
  cudaStream_t stream = nullptr;
  int n = 0;
  int cur = 0;                       // buffer holding the committed state
  void* st[2][kStateArrays] = {};    // double-buffered per-rod arrays
  void* dlm[3] = {};                 // d, l, m
  void** ptrs = nullptr;             // device copy of st (for k_rod_geom)
  // grid (CellLinked)
  int n_cells_d[3] = {1, 1, 1};
  int n_cells = 1;
  Counters* ctr = nullptr;
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  int* agent_cell = nullptr;
  int* agent_rank = nullptr;
  int* cell_tmp = nullptr;
  int* cell_agents = nullptr;
  unsigned long long* scan_state = nullptr;
  // rods2dGrowth: {n, step} per buffer on the device, the division ranks
  bool grow = false;
  long long* cnt = nullptr;          // cnt[2 * buf + 0] = n, cnt[2 * buf + 1] = step
  int* div_flags = nullptr;          // whole scan tiles, zero between steps
  int* div_rank = nullptr;           // n_max + 1
  int* holes = nullptr;              // n_max
  Counters* div_ctr = nullptr;
  unsigned long long* div_state = nullptr;
  int div_tiles = 0;
  long long cnt_host[4] = {0, 0, 0, 0};
  cudaGraphExec_t pair_graph[2] = {nullptr, nullptr};  // two steps starting at cur = 0 / 1
  bool loaded = false;
  std::string err;
};

namespace {

std::string g_rods_create_error;

int rfail(cbm_rods* r, int code, const std::string& msg) {
  if (r) r->err = msg;
  else g_rods_create_error = msg;
  return code;
}

#define ROD_TRY(r, call)                                                                    \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return rfail(r, CBM_ERR_CUDA, std::string(#call) + " failed: " + cudaGetErrorString(e_)); \
  } while (0)

void drop_graphs(cbm_rods* r) {
  for (cudaGraphExec_t& g : r->pair_graph)
    if (g) cudaGraphExecDestroy(g), g = nullptr;
}

void rfree(cbm_rods* r) {
  drop_graphs(r);
  for (auto& b : r->st)
    for (void*& p : b)
      if (p) cudaFree(p), p = nullptr;
  for (void*& p : r->dlm)
    if (p) cudaFree(p), p = nullptr;
  for (void* p : {(void*)r->ptrs, (void*)r->ctr, (void*)r->cell_count, (void*)r->cell_start,
                  (void*)r->agent_cell, (void*)r->agent_rank, (void*)r->cell_tmp,
                  (void*)r->cell_agents, (void*)r->scan_state, (void*)r->cnt,
                  (void*)r->div_flags, (void*)r->div_rank, (void*)r->holes, (void*)r->div_ctr,
                  (void*)r->div_state})
    if (p) cudaFree(p);
  r->ptrs = nullptr;
  r->ctr = nullptr;
  if (r->stream) cudaStreamDestroy(r->stream);
  r->stream = nullptr;
}

// field k of the C ABI (CBM_ROD_*) in buffer `buf`
void* field_ptr(cbm_rods* r, int buf, int k) {
  switch (k) {
    case CBM_ROD_X: return r->st[buf][kSX];
    case CBM_ROD_Y: return r->st[buf][kSY];
    case CBM_ROD_VX: return r->st[buf][kSVX];
    case CBM_ROD_VY: return r->st[buf][kSVY];
    case CBM_ROD_THETA: return r->st[buf][kSTH];
    case CBM_ROD_OMEGA: return r->st[buf][kSOM];
    case CBM_ROD_D: return r->grow ? r->st[buf][kSD] : r->dlm[0];
    case CBM_ROD_L: return r->grow ? r->st[buf][kSL] : r->dlm[1];
    case CBM_ROD_M: return r->grow ? r->st[buf][kSM] : r->dlm[2];
    case CBM_ROD_FX: return r->st[buf][kSFX];
    case CBM_ROD_FY: return r->st[buf][kSFY];
    case CBM_ROD_W: return r->st[buf][kSW];
    case CBM_ROD_L_TARGET: return r->grow ? r->st[buf][kSLT] : nullptr;
    default: return r->st[buf][kSP];
  }
}

template <typename T>
GridParams<T> grid_params(const cbm_rods* r) {
  GridParams<T> G;
  memset(&G, 0, sizeof G);
  G.pos[0] = (const T*)r->st[r->cur][kSX];
  G.pos[1] = (const T*)r->st[r->cur][kSY];
  for (int d = 0; d < 2; ++d) {
    G.box_lo[d] = (T)r->cfg.box_lo[d];
    G.box_hi[d] = (T)r->cfg.box_hi[d];
  }
  for (int d = 0; d < 3; ++d) G.n_cells_d[d] = r->n_cells_d[d];
  G.n = r->n;
  G.edge = (T)r->cfg.cell_edge;
  G.n_cells = r->n_cells;
  G.n_scan_tiles = (r->n_cells + kScanTile - 1) / kScanTile;
  G.ctr = r->ctr;
  G.cell_count = r->cell_count;
  G.cell_start = r->cell_start;
  G.scan_state = r->scan_state;
  G.agent_cell = r->agent_cell;
  G.agent_rank = r->agent_rank;
  G.cell_tmp = r->cell_tmp;
  G.cell_agents = r->cell_agents;
  return G;
}

// computeNeighbors! from scratch on the committed positions (after upload)
template <typename T>
void enqueue_full_grid(cbm_rods* r) {
  const GridParams<T> G = grid_params<T>(r);
  const unsigned nb = (unsigned)(r->n > 0 ? (r->n + kTile - 1) / kTile : 1);
  k_grid_hist<T, 2><<<nb, kTile, 0, r->stream>>>(G);
  k_scan_cells<<<G.n_scan_tiles, kTile, 0, r->stream>>>(grid_scan_args(G));
  k_grid_scatter<T><<<nb, kTile, 0, r->stream>>>(G);
  k_grid_stable<T><<<nb, kTile, 0, r->stream>>>(G);
}

template <typename T>
void enqueue_rod_step(cbm_rods* r) {
  RodStep<T> R;
  memset(&R, 0, sizeof R);
  const cbm_rods_config& k = r->cfg;
  for (int q = 0; q < kStateArrays; ++q) {
    R.a[q] = (T*)r->st[r->cur][q];
    R.b[q] = (T*)r->st[1 - r->cur][q];
  }
  R.d = (const T*)(r->grow ? r->st[r->cur][kSD] : r->dlm[0]);
  R.l = (const T*)(r->grow ? r->st[r->cur][kSL] : r->dlm[1]);
  R.m = (const T*)(r->grow ? r->st[r->cur][kSM] : r->dlm[2]);
  R.cell_start = r->cell_start;
  R.cell_agents = r->cell_agents;
  R.cell_count = r->cell_count;
  R.agent_cell = r->agent_cell;
  R.agent_rank = r->agent_rank;
  R.ctr = r->ctr;
  R.n = r->n;
  R.full = k.neighbors == CBM_NEIGH_FULL;
  for (int d = 0; d < 2; ++d) {
    R.box_lo[d] = (T)k.box_lo[d];
    R.box_hi[d] = (T)k.box_hi[d];
  }
  R.edge = (T)k.cell_edge;
  for (int d = 0; d < 3; ++d) R.n_cells_d[d] = r->n_cells_d[d];
  R.dt = (T)k.dt;
  R.beta = (T)k.beta;
  R.beta_w = (T)k.beta_w;
  R.k = CbmRodCoef<T>{(T)k.kn, (T)k.gamma_n, (T)k.gamma_t, (T)k.mu_cc};
  if (!r->grow) {
    const long long threads = (long long)(r->n > 0 ? r->n : 1) * kRodLanes;
    const unsigned nb = (unsigned)((threads + kRodBlock - 1) / kRodBlock);
    k_rod_step<T, false><<<nb, kRodBlock, 0, r->stream>>>(R);
    r->cur = 1 - r->cur;
    if (!R.full) {
      // the rest of computeNeighbors! on the new positions
      const GridParams<T> G = grid_params<T>(r);
      const unsigned ng = (unsigned)(r->n > 0 ? (r->n + kTile - 1) / kTile : 1);
      // each kernel follows a kernel on the stream: programmatic launches
      launch_serial(r->stream, true, k_scan_cells, dim3(G.n_scan_tiles), dim3(kTile), 0,
                    grid_scan_args(G));
      launch_serial(r->stream, true, k_grid_scatter<T>, dim3(ng), dim3(kTile), 0, G);
      launch_serial(r->stream, true, k_grid_stable<T>, dim3(ng), dim3(kTile), 0, G);
    }
    return;
  }
  // rods2dGrowth: the count lives on the device, launches cover n_max
  R.cnt_a = r->cnt + 2 * r->cur;
  R.cnt_b = r->cnt + 2 * (1 - r->cur);
  R.div_rank = r->div_rank;
  R.holes = r->holes;
  R.n_max = (int)k.n_max;
  R.growth = (T)k.growth;
  R.alpha = (T)k.alpha;
  R.lt_lo = (T)k.l_max - (T)k.sigma_l_target;
  R.lt_hi = (T)k.l_max + (T)k.sigma_l_target;
  R.seed = k.seed;
  const unsigned nt = (unsigned)((k.n_max + kTile - 1) / kTile);
  k_rod_flags<T><<<nt, kTile, 0, r->stream>>>(R, r->div_flags, r->div_ctr);
  ScanArgs A;
  A.count = r->div_flags;
  A.start = r->div_rank;
  A.state = r->div_state;
  A.n = (int)k.n_max;
  A.n_tiles = r->div_tiles;
  A.ctr = r->div_ctr;
  A.due = nullptr;
  // from here each kernel follows a kernel on the stream: programmatic launches
  launch_serial(r->stream, true, k_scan_cells, dim3(A.n_tiles), dim3(kTile), 0, A);
  launch_serial(r->stream, true, k_rod_holes<T>, dim3(nt), dim3(kTile), 0, R, r->holes, r->ctr);
  const long long threads = (long long)k.n_max * kRodLanes;
  const unsigned nb = (unsigned)((threads + kRodBlock - 1) / kRodBlock);
  launch_serial(r->stream, true, k_rod_step<T, true>, dim3(nb), dim3(kRodBlock), 0, R);
  r->cur = 1 - r->cur;
  if (!R.full) {
    const GridParams<T> G = grid_params<T>(r);
    const long long* cnt = r->cnt + 2 * r->cur;
    launch_serial(r->stream, true, k_scan_cells, dim3(G.n_scan_tiles), dim3(kTile), 0,
                  grid_scan_args(G));
    launch_serial(r->stream, true, k_rod_scatter<T>, dim3(nt), dim3(kTile), 0, G, cnt);
    launch_serial(r->stream, true, k_rod_stable<T>, dim3(nt), dim3(kTile), 0, G, cnt);
  }
}

void enqueue_one(cbm_rods* r) {
  if (r->tsize == 8) enqueue_rod_step<double>(r);
  else enqueue_rod_step<float>(r);
}

// a graph of two steps starting at the current buffer (which it leaves current)
int pair_graph(cbm_rods* r, cudaGraphExec_t* out) {
  cudaGraphExec_t& g = r->pair_graph[r->cur];
  if (!g) {
    cudaGraph_t graph = nullptr;
    ROD_TRY(r, cudaStreamBeginCapture(r->stream, cudaStreamCaptureModeThreadLocal));
    enqueue_one(r);
    enqueue_one(r);
    const cudaError_t e = cudaStreamEndCapture(r->stream, &graph);
    if (e != cudaSuccess)
      return rfail(r, CBM_ERR_CUDA, std::string("rods graph capture failed: ") + cudaGetErrorString(e));
    const cudaError_t ei = cudaGraphInstantiate(&g, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      g = nullptr;
      return rfail(r, CBM_ERR_CUDA,
                   std::string("rods graph instantiation failed: ") + cudaGetErrorString(ei));
    }
  }
  *out = g;
  return CBM_OK;
}

}  // namespace

extern "C" {

int cbm_rods_create(cbm_rods** out, const cbm_rods_config* cfg) {
  if (!out || !cfg) return rfail(nullptr, CBM_ERR_ARG, "null argument");
  *out = nullptr;
  const cbm_rods_config& k = *cfg;
  if (k.precision != CBM_F32 && k.precision != CBM_F64)
    return rfail(nullptr, CBM_ERR_ARG, "precision must be CBM_F32 or CBM_F64");
  if (k.neighbors != CBM_NEIGH_FULL && k.neighbors != CBM_NEIGH_CELL_LINKED)
    return rfail(nullptr, CBM_ERR_ARG, "rods need neighbors CBM_NEIGH_FULL or CBM_NEIGH_CELL_LINKED");
  if (k.n_max < 1 || k.n_max >= (1ll << 27))
    return rfail(nullptr, CBM_ERR_ARG, "n_max must be in [1, 2^27)");
  if (!(k.dt > 0)) return rfail(nullptr, CBM_ERR_ARG, "dt must be positive");
  for (int d = 0; d < 2; ++d)
    if (!(k.box_hi[d] > k.box_lo[d])) return rfail(nullptr, CBM_ERR_ARG, "empty simBox");
  if (k.growth_model != 0 && k.growth_model != 1)
    return rfail(nullptr, CBM_ERR_ARG, "growth_model must be 0 (rods2D) or 1 (rods2dGrowth)");
  if (k.growth_model && !(std::isfinite(k.growth) && std::isfinite(k.alpha) &&
                          std::isfinite(k.l_max) && std::isfinite(k.sigma_l_target)))
    return rfail(nullptr, CBM_ERR_ARG, "growth, alpha, l_max and sigma_l_target must be finite");
  cbm_rods* r = new cbm_rods;
  r->cfg = k;
  r->grow = k.growth_model != 0;
  r->tsize = k.precision == CBM_F64 ? 8 : 4;
  if (k.neighbors == CBM_NEIGH_CELL_LINKED) {
    if (!(k.cell_edge > 0)) {
      delete r;
      return rfail(nullptr, CBM_ERR_ARG, "cell_edge must be positive");
    }
    long long nc = 1;
    for (int d = 0; d < 2; ++d) {
      // nCells = ceil((hi - lo) / edge + 2), neighbors.jl:605
      const double v = std::ceil((k.box_hi[d] - k.box_lo[d]) / k.cell_edge + 2.0);
      if (!(v >= 1 && v < 1.0e8)) {
        delete r;
        return rfail(nullptr, CBM_ERR_ARG, "cell grid too large");
      }
      r->n_cells_d[d] = (int)v;
      nc *= (long long)v;
    }
    if (nc >= (1ll << 31) - 1) {
      delete r;
      return rfail(nullptr, CBM_ERR_ARG, "cell grid has too many cells");
    }
    r->n_cells = (int)nc;
  }
  const size_t n = (size_t)k.n_max, S = (size_t)r->tsize;
  bool ok = cudaStreamCreateWithFlags(&r->stream, cudaStreamNonBlocking) == cudaSuccess;
  const int arrays = r->grow ? kStateArrays : kPlainArrays;
  for (auto& b : r->st)
    for (int q = 0; q < arrays; ++q) ok = ok && cudaMalloc(&b[q], n * S) == cudaSuccess;
  if (!r->grow)
    for (void*& p : r->dlm) ok = ok && cudaMalloc(&p, n * S) == cudaSuccess;
  if (r->grow) {
    r->div_tiles = (int)((k.n_max + kScanTile - 1) / kScanTile);
    const size_t flag_ints = (size_t)r->div_tiles * kScanTile;
    ok = ok && cudaMalloc((void**)&r->cnt, 4 * sizeof(long long)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&r->div_flags, flag_ints * 4) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&r->div_rank, (n + 1) * 4) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&r->holes, n * 4) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&r->div_ctr, sizeof(Counters)) == cudaSuccess;
    ok = ok && cudaMalloc((void**)&r->div_state, (size_t)r->div_tiles * 8) == cudaSuccess;
    ok = ok && cudaMemsetAsync(r->cnt, 0, 4 * sizeof(long long), r->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(r->div_flags, 0, flag_ints * 4, r->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(r->div_ctr, 0, sizeof(Counters), r->stream) == cudaSuccess;
    ok = ok && cudaMemsetAsync(r->div_state, 0, (size_t)r->div_tiles * 8, r->stream) == cudaSuccess;
  }
  ok = ok && cudaMalloc((void**)&r->ptrs, 2 * kStateArrays * sizeof(void*)) == cudaSuccess;
  const int tiles = (r->n_cells + kScanTile - 1) / kScanTile;
  // whole scan tiles of counts: the scan loads and clears them as int4
  const size_t count_ints = (size_t)tiles * kScanTile;
  ok = ok && cudaMalloc((void**)&r->ctr, sizeof(Counters)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_count, count_ints * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_start, ((size_t)r->n_cells + 1) * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->agent_cell, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->agent_rank, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_tmp, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_agents, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->scan_state, (size_t)tiles * 8) == cudaSuccess;
  void* host_ptrs[2 * kStateArrays];
  for (int b = 0; b < 2; ++b)
    for (int q = 0; q < kStateArrays; ++q) host_ptrs[b * kStateArrays + q] = r->st[b][q];
  ok = ok && cudaMemcpyAsync(r->ptrs, host_ptrs, sizeof host_ptrs, cudaMemcpyHostToDevice,
                             r->stream) == cudaSuccess;
  ok = ok && cudaMemsetAsync(r->ctr, 0, sizeof(Counters), r->stream) == cudaSuccess;
  ok = ok && cudaMemsetAsync(r->cell_count, 0, count_ints * 4, r->stream) == cudaSuccess;
  ok = ok && cudaMemsetAsync(r->scan_state, 0, (size_t)tiles * 8, r->stream) == cudaSuccess;
  ok = ok && cudaStreamSynchronize(r->stream) == cudaSuccess;
  if (!ok) {
    rfree(r);
    delete r;
    return rfail(nullptr, CBM_ERR_NOMEM, "device allocation failed for the rods");
  }
  *out = r;
  return CBM_OK;
}

void cbm_rods_destroy(cbm_rods* r) {
  if (!r) return;
  rfree(r);
  delete r;
}

const char* cbm_rods_last_error(const cbm_rods* r) {
  return r ? r->err.c_str() : g_rods_create_error.c_str();
}

int cbm_rods_upload(cbm_rods* r, int64_t n, const void* const* fields) {
  if (!r || !fields) return rfail(r, CBM_ERR_ARG, "null argument");
  if (n < 0 || n > r->cfg.n_max) return rfail(r, CBM_ERR_ARG, "n must be in [0, n_max]");
  for (int q = 0; q < CBM_ROD_PRESSURE; ++q)
    if (!fields[q]) return rfail(r, CBM_ERR_ARG, "a rod field is missing");
  if (r->grow && !fields[CBM_ROD_L_TARGET])
    return rfail(r, CBM_ERR_ARG, "rods2dGrowth needs the lTarget field");
  ROD_TRY(r, cudaStreamSynchronize(r->stream));
  if ((int)n != r->n) drop_graphs(r);  // the graphs hold n in their launch shapes
  r->n = (int)n;
  r->cur = 0;
  const size_t b = (size_t)n * r->tsize;
  if (b) {
    for (int q = 0; q < CBM_ROD_PRESSURE; ++q)
      ROD_TRY(r, cudaMemcpyAsync(field_ptr(r, 0, q), fields[q], b, cudaMemcpyHostToDevice,
                                 r->stream));
    ROD_TRY(r, cudaMemsetAsync(field_ptr(r, 0, CBM_ROD_PRESSURE), 0, b, r->stream));
    if (r->grow)
      ROD_TRY(r, cudaMemcpyAsync(field_ptr(r, 0, CBM_ROD_L_TARGET), fields[CBM_ROD_L_TARGET], b,
                                 cudaMemcpyHostToDevice, r->stream));
  }
  ROD_TRY(r, cudaMemsetAsync(&r->ctr->err, 0, sizeof(int), r->stream));
  if (r->grow) {
    r->cnt_host[0] = n;
    r->cnt_host[1] = 0;
    r->cnt_host[2] = n;
    r->cnt_host[3] = 0;
    ROD_TRY(r, cudaMemcpyAsync(r->cnt, r->cnt_host, sizeof r->cnt_host, cudaMemcpyHostToDevice,
                               r->stream));
    ROD_TRY(r, cudaMemsetAsync(&r->div_ctr->err, 0, sizeof(int), r->stream));
  }
  const unsigned nb = (unsigned)(n > 0 ? (n + kTile - 1) / kTile : 1);
  if (r->tsize == 8) {
    k_rod_geom<double><<<nb, kTile, 0, r->stream>>>((double* const*)r->ptrs, (int)n);
    if (r->cfg.neighbors == CBM_NEIGH_CELL_LINKED) enqueue_full_grid<double>(r);
  } else {
    k_rod_geom<float><<<nb, kTile, 0, r->stream>>>((float* const*)r->ptrs, (int)n);
    if (r->cfg.neighbors == CBM_NEIGH_CELL_LINKED) enqueue_full_grid<float>(r);
  }
  ROD_TRY(r, cudaGetLastError());
  ROD_TRY(r, cudaStreamSynchronize(r->stream));
  r->loaded = true;
  return CBM_OK;
}

int cbm_rods_step(cbm_rods* r, int32_t nsteps, int32_t flags) {
  if (!r) return rfail(r, CBM_ERR_ARG, "null rods");
  if (!r->loaded) return rfail(r, CBM_ERR_STATE, "cbm_rods_step before cbm_rods_upload");
  if (nsteps < 0) return rfail(r, CBM_ERR_ARG, "nsteps must be >= 0");
  int s = 0;
  if (!(flags & CBM_NO_GRAPH)) {
    for (; s + 2 <= nsteps; s += 2) {
      cudaGraphExec_t g = nullptr;
      const int rc = pair_graph(r, &g);
      if (rc != CBM_OK) return rc;
      ROD_TRY(r, cudaGraphLaunch(g, r->stream));
    }
  }
  for (; s < nsteps; ++s) enqueue_one(r);
  ROD_TRY(r, cudaGetLastError());
  if (flags & CBM_SYNC) {
    int e[2] = {0, 0};
    ROD_TRY(r, cudaMemcpyAsync(&e[0], &r->ctr->err, sizeof(int), cudaMemcpyDeviceToHost, r->stream));
    if (r->grow)
      ROD_TRY(r, cudaMemcpyAsync(&e[1], &r->div_ctr->err, sizeof(int), cudaMemcpyDeviceToHost,
                                 r->stream));
    ROD_TRY(r, cudaStreamSynchronize(r->stream));
    const int bits = e[0] | e[1];
    if (bits & kErrAgentOverflow)
      return rfail(r, CBM_ERR_AGENT_OVERFLOW, "a division found no room below n_max");
    if (bits & kErrTimeout) return rfail(r, CBM_ERR_TIMEOUT, "a bounded wait of the cell scan gave up");
  }
  return CBM_OK;
}

int cbm_rods_download(cbm_rods* r, void* const* fields, int64_t* n_out) {
  if (!r || !fields) return rfail(r, CBM_ERR_ARG, "null argument");
  if (!r->loaded) return rfail(r, CBM_ERR_STATE, "cbm_rods_download before cbm_rods_upload");
  if (r->grow) {
    ROD_TRY(r, cudaMemcpyAsync(r->cnt_host, r->cnt, sizeof r->cnt_host, cudaMemcpyDeviceToHost,
                               r->stream));
    ROD_TRY(r, cudaStreamSynchronize(r->stream));
    r->n = (int)r->cnt_host[2 * r->cur];
  }
  const size_t b = (size_t)r->n * r->tsize;
  for (int q = 0; q < CBM_RODS_FIELDS; ++q) {
    void* src = field_ptr(r, r->cur, q);  // null: lTarget without rods2dGrowth
    if (fields[q] && src && b)
      ROD_TRY(r, cudaMemcpyAsync(fields[q], src, b, cudaMemcpyDeviceToHost, r->stream));
  }
  ROD_TRY(r, cudaStreamSynchronize(r->stream));
  if (n_out) *n_out = r->n;
  return CBM_OK;
}

void* cbm_rods_stream(cbm_rods* r) { return r ? (void*)r->stream : nullptr; }

}  // extern "C"
