// cbm_kernels.cuh — device kernels of the per-step path.
//
// Every kernel here reads the live agent count, step number and flags from
// the device counter block, so a whole step can be captured once in a CUDA
// graph and replayed without host round trips (the reference syncs the host
// after every stage and reads flagRecomputeNeighbors_ / NAdd_ on the host,
// src/neighbors.jl:548, src/CommunityStructure/update.jl:214).
//
// Arithmetic follows the reference's expression order with no FMA
// contraction (the library is built with -fmad=false), so float and double
// results are bit-identical to a CPU evaluation of the same expressions.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/cbm_b200.h"
#include "../../include/cbm_rng.h"

namespace cbm {

constexpr int kTile = 256;          // agents per block in every agent kernel
constexpr unsigned kFull = 0xffffffffu;
constexpr int kScanItems = 8;       // cells per thread in the cell scan
constexpr int kScanTile = kTile * kScanItems;
constexpr long long kSpinLimit = 1ll << 20;  // bounded look-back wait

// device error bits (reported through cbm_sync as the lowest set code)
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
  int flag[2];          // flagRecomputeNeighbors_ of the step of that parity
  int err;              // kErr* bits
  unsigned scan_ticket; // tile tickets of the cell scan
  unsigned scan_epoch;  // generation of the cell-scan tile states
  int pad;
};

template <typename T>
struct Params {
  // agent arrays: committed ("cur", parity p) and written ("nxt", p ^ 1)
  T* pos_cur[3];
  T* pos_nxt[3];
  T* pos_u[3];          // positions after the rule's wall reflection (u); = pos_cur without walls
  T* v_cur;
  T* v_nxt;
  T* f_cur[3];
  T* f_nxt[3];
  T* g;
  long long* id;
  long long* parent;
  unsigned char* fate;
  int* holes;
  int* blk_children;
  int* blk_deaths;
  int* blk_child_off;
  int* blk_death_off;
  // grid
  int* agent_cell;
  int* agent_rank;
  int* cell_count;
  int* cell_start;      // n_cells + 1
  int* cell_tmp;
  int* cell_agents;
  unsigned long long* scan_state;  // per scan tile: epoch | flag | value
  // Verlet
  int* nbr_n;
  int* nbr_list;        // column-major: slot k of agent i at k * n_max + i
  T* pos_old[3];
  // medium: committed / written
  T* c_cur;
  T* c_nxt;
  T* grad_cur[3];
  T* grad_nxt[3];
  Counters* ctr;
  // sizes
  int n_max;
  int n_blocks;         // agent tiles = ceil(n_max / kTile)
  int n_cells;
  int n_cells_d[3];
  int n_scan_tiles;
  int n_nodes;
  int n_medium[3];
  int max_nbrs;
  int parity;
  int births_only;      // k_agent_de: place the rule's births, integrate nothing
  // model
  int neighbors, integrator, force_mode, att_form, walls, fate_rule, growth, medium,
      medium_sampling;
  T box_lo[3], box_hi[3];
  T dt, sqrt_dt, sigma;
  T edge;               // grid cell edge
  T skin, rebuild_thr;
  T k_rep, r_rep, k_att, r_att;
  T wall_force, wall_range, drift_linear;
  T v_div, div_sep, p_death;
  T dx_m[3];
  T diff_D, decay, secretion_amt, chemotaxis;
  uint64_t seed;
  uint32_t community;
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// Julia's float `÷` on a >= 0: round((a - rem(a, b)) / b)
__device__ __forceinline__ int floordiv(double a, double b) {
  return (int)rint((a - fmod(a, b)) / b);
}
__device__ __forceinline__ int floordiv(float a, float b) {
  return (int)rintf((a - fmodf(a, b)) / b);
}

// cellPos, src/neighbors.jl:636-638, 0-based; NaN goes to the first cell
template <typename T>
__device__ __forceinline__ int cell_pos1(T edge, T x, T lo, T hi, int n) {
  if (x > hi) return n - 1;
  if (!(x >= lo)) return 0;
  int p = floordiv(x - lo, edge) + 1;
  return p > n - 1 ? n - 1 : p;
}

template <typename T, int D>
__device__ __forceinline__ int cell_of(const Params<T>& P, const T* x) {
  int lin = cell_pos1<T>(P.edge, x[0], P.box_lo[0], P.box_hi[0], P.n_cells_d[0]);
  if (D > 1) lin += P.n_cells_d[0] * cell_pos1<T>(P.edge, x[1], P.box_lo[1], P.box_hi[1], P.n_cells_d[1]);
  if (D > 2)
    lin += P.n_cells_d[0] * P.n_cells_d[1] *
           cell_pos1<T>(P.edge, x[2], P.box_lo[2], P.box_hi[2], P.n_cells_d[2]);
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

template <typename T, int D>
__device__ __forceinline__ int nearest_node(const Params<T>& P, const T* x) {
  int lin = cell_in_mesh<T>(P.dx_m[0], x[0], P.box_lo[0], P.box_hi[0], P.n_medium[0]);
  if (D > 1) lin += P.n_medium[0] * cell_in_mesh<T>(P.dx_m[1], x[1], P.box_lo[1], P.box_hi[1], P.n_medium[1]);
  if (D > 2)
    lin += P.n_medium[0] * P.n_medium[1] *
           cell_in_mesh<T>(P.dx_m[2], x[2], P.box_lo[2], P.box_hi[2], P.n_medium[2]);
  return lin;
}

// Nodes and weights of the multilinear stencil around x (nodes at the cell
// centres lo + (i + 1/2) dx, indices clamped to the grid).
template <typename T, int D>
__device__ __forceinline__ void bilinear(const Params<T>& P, const T* x, int* node, T* w) {
  int i0[3], i1[3];
  T tt[3];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    T s = (x[d] - P.box_lo[d]) / P.dx_m[d] - (T)0.5;
    T fl = floor(s);
    tt[d] = s - fl;
    int a = (int)fl, b = a + 1;
    int hi = P.n_medium[d] - 1;
    i0[d] = a < 0 ? 0 : (a > hi ? hi : a);
    i1[d] = b < 0 ? 0 : (b > hi ? hi : b);
  }
#pragma unroll
  for (int q = 0; q < (1 << D); ++q) {
    int lin = 0, mul = 1;
    T wq = (T)1;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      bool h = (q >> d) & 1;
      lin += (h ? i1[d] : i0[d]) * mul;
      mul *= P.n_medium[d];
      wq = wq * (h ? tt[d] : (T)1 - tt[d]);
    }
    node[q] = lin;
    w[q] = wq;
  }
}

// cellPosNeigh, src/neighbors.jl:658-708: k-th of 3^D cells, x fastest, -1 outside
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

template <typename T, int D>
__device__ __forceinline__ void load_pos(T* const* arr, int i, T* x) {
#pragma unroll
  for (int d = 0; d < D; ++d) x[d] = arr[d][i];
}

// Visit neighbor candidates of agent i in the reference's order.  `pos` are
// the positions used to locate i's own cell (u in the DE, x in a rule).
template <typename T, int D, typename F>
__device__ __forceinline__ void for_neighbors(const Params<T>& P, const T* xi, int i, int N,
                                              F&& body) {
  switch (P.neighbors) {
    case CBM_NEIGH_FULL:
      for (int j = 0; j < N; ++j)
        if (j != i) body(j);
      break;
    case CBM_NEIGH_CELL_LINKED: {
      int q[3];
      cell_coords<D>(P.n_cells_d, cell_of<T, D>(P, xi), q);
      constexpr int nk = D == 1 ? 3 : (D == 2 ? 9 : 27);
      for (int k = 0; k < nk; ++k) {
        int pn = cell_neigh<D>(P.n_cells_d, q, k);
        if (pn < 0) continue;
        int s0 = ld(P.cell_start + pn), s1 = ld(P.cell_start + pn + 1);
        for (int s = s0; s < s1; ++s) {
          int j = ld(P.cell_agents + s);
          if (j != i) body(j);
        }
      }
      break;
    }
    case CBM_NEIGH_VERLET_DISPLACEMENT:
    case CBM_NEIGH_CLVD: {
      int n = P.nbr_n[i];
      for (int k = 0; k < n; ++k) body(ld(P.nbr_list + (size_t)k * P.n_max + i));
      break;
    }
    default:
      break;
  }
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
// mediumStepRule!: gradient of the committed field (central differences
// inside, 0 on the border; the @∂ macro, src/AgentStructure/macros.jl:148-190)
// ---------------------------------------------------------------------------
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_medium_grad(Params<T> P) {
  int n = blockIdx.x * kTile + threadIdx.x;
  if (n >= P.n_nodes) return;
  int q[3] = {0, 0, 0};
  q[0] = n % P.n_medium[0];
  if (D > 1) q[1] = (n / P.n_medium[0]) % P.n_medium[1];
  if (D > 2) q[2] = n / (P.n_medium[0] * P.n_medium[1]);
  bool in = true;
#pragma unroll
  for (int d = 0; d < D; ++d) in = in && q[d] > 0 && q[d] < P.n_medium[d] - 1;
  int stride[3] = {1, P.n_medium[0], P.n_medium[0] * P.n_medium[1]};
#pragma unroll
  for (int d = 0; d < D; ++d)
    P.grad_nxt[d][n] = in ? (ld(P.c_cur + n + stride[d]) - ld(P.c_cur + n - stride[d])) /
                                ((T)2 * P.dx_m[d])
                          : (T)0;
}

// ---------------------------------------------------------------------------
// Bilinear secretion as a gather over medium nodes.  Atomic adds of unequal
// amounts would sum in an arbitrary order; here every node adds the
// contributions of the agents whose stencil covers it in ascending agent
// index, the order of the reference's serial agent loop.  The agents are
// found through the cell grid, which holds exactly the committed positions
// the rule reads when the grid is rebuilt every step (CellLinked).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool secretion_by_gather(const Params<T>& P) {
  return P.medium_sampling == CBM_MEDIUM_BILINEAR && P.neighbors == CBM_NEIGH_CELL_LINKED;
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_secrete_gather(Params<T> P) {
  constexpr int kMaxCells = D == 1 ? 4 : (D == 2 ? 16 : 64);
  const int n = blockIdx.x * kTile + threadIdx.x;
  if (n >= P.n_nodes) return;
  int q[3] = {0, 0, 0};
  q[0] = n % P.n_medium[0];
  if (D > 1) q[1] = (n / P.n_medium[0]) % P.n_medium[1];
  if (D > 2) q[2] = n / (P.n_medium[0] * P.n_medium[1]);
  // agents touching node q along an axis lie in x in [lo+(q-1/2)dx, lo+(q+3/2)dx)
  // (unbounded below for q = 0, above for the last node); widen by one cell
  int c0[3] = {0, 0, 0}, c1[3] = {0, 0, 0};
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int nc = P.n_cells_d[d];
    int a = q[d] == 0 ? 0
                      : cell_pos1<T>(P.edge, P.box_lo[d] + ((T)q[d] - (T)0.5) * P.dx_m[d],
                                     P.box_lo[d], P.box_hi[d], nc) - 1;
    int b = q[d] == P.n_medium[d] - 1
                ? nc - 1
                : cell_pos1<T>(P.edge, P.box_lo[d] + ((T)q[d] + (T)1.5) * P.dx_m[d],
                               P.box_lo[d], P.box_hi[d], nc) + 1;
    c0[d] = a < 0 ? 0 : a;
    c1[d] = b > nc - 1 ? nc - 1 : b;
  }
  int cur[kMaxCells], end[kMaxCells];
  int ncand = 0;
  bool all = true;
  for (int cz = c0[2]; cz <= c1[2]; ++cz)
    for (int cy = c0[1]; cy <= c1[1]; ++cy)
      for (int cx = c0[0]; cx <= c1[0]; ++cx) {
        if (ncand == kMaxCells) { all = false; continue; }
        int c = cx + P.n_cells_d[0] * (cy + P.n_cells_d[1] * cz);
        int s0 = P.cell_start[c], s1 = P.cell_start[c + 1];
        if (s0 < s1) { cur[ncand] = s0; end[ncand] = s1; ++ncand; }
      }
  const T amt = P.secretion_amt;
  T acc = P.c_cur[n];
  if (all) {
    while (true) {  // k-way merge: next smallest agent index among the cells
      int best = -1, bj = 0x7fffffff;
      for (int k = 0; k < ncand; ++k)
        if (cur[k] < end[k]) {
          int j = P.cell_agents[cur[k]];
          if (j < bj) { bj = j; best = k; }
        }
      if (best < 0) break;
      ++cur[best];
      T x[3];
      load_pos<T, D>(P.pos_cur, bj, x);
      int nodes[8];
      T w[8];
      bilinear<T, D>(P, x, nodes, w);
#pragma unroll
      for (int k = 0; k < (1 << D); ++k)
        if (nodes[k] == n) acc = acc + w[k] * amt;
    }
  } else {
    // the cell box is too large (cells much smaller than the medium spacing):
    // visit every agent in index order
    const int N = (int)P.ctr->N[P.parity];
    for (int j = 0; j < N; ++j) {
      T x[3];
      load_pos<T, D>(P.pos_cur, j, x);
      int nodes[8];
      T w[8];
      bilinear<T, D>(P, x, nodes, w);
#pragma unroll
      for (int k = 0; k < (1 << D); ++k)
        if (nodes[k] == n) acc = acc + w[k] * amt;
    }
  }
  P.c_cur[n] = acc;
}

// ---------------------------------------------------------------------------
// agentStepRule!: walls, secretion, fate decision + per-tile event counts
// (src/AgentStructure/functionRule.jl:9-111)
// ---------------------------------------------------------------------------
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_agent_rule(Params<T> P) {
  const int p = P.parity;
  const int N = (int)P.ctr->N[p];
  const int i = blockIdx.x * kTile + threadIdx.x;
  const bool live = i < N;
  int fate = 0;  // 0 none, 1 die, 2 divide (2 children + die), 3 one child
  if (live) {
    T x[3];
    load_pos<T, D>(P.pos_cur, i, x);
    if (P.walls == CBM_WALLS_REFLECT) {
#pragma unroll
      for (int d = 0; d < D; ++d) {
        T y = x[d];
        if (x[d] < P.box_lo[d]) y = (T)2 * P.box_lo[d] - x[d];
        else if (x[d] > P.box_hi[d]) y = (T)2 * P.box_hi[d] - x[d];
        P.pos_u[d][i] = y;
      }
    }
    if (P.medium && P.secretion_amt != (T)0 && !secretion_by_gather(P)) {
      if (P.medium_sampling == CBM_MEDIUM_NEAREST) {
        atomicAdd(P.c_cur + nearest_node<T, D>(P, x), P.secretion_amt);
      } else {
        int nodes[8];
        T w[8];
        bilinear<T, D>(P, x, nodes, w);
#pragma unroll
        for (int q = 0; q < (1 << D); ++q) atomicAdd(P.c_cur + nodes[q], w[q] * P.secretion_amt);
      }
    }
    if (P.fate_rule == CBM_FATE_VOLUME) {
      if (P.growth && P.v_cur[i] >= P.v_div) fate = 2;
      else if (P.p_death > (T)0 &&
               cbm_uniform<T>(P.seed, P.ctr->step[p], (uint32_t)i, CBM_STREAM_DEATH, P.community) <
                   P.p_death)
        fate = 1;
    } else if (P.fate_rule == CBM_FATE_ID_PARITY) {
      fate = (P.id[i] % 2 == 1) ? 1 : 3;
    }
  }
  if (i < P.n_max) P.fate[i] = (unsigned char)fate;
  int n_div = __syncthreads_count(fate == 2);
  int n_one = __syncthreads_count(fate == 3);
  int n_die = __syncthreads_count(fate == 1 || fate == 2);
  if (threadIdx.x == 0) {
    P.blk_children[blockIdx.x] = 2 * n_div + n_one;
    P.blk_deaths[blockIdx.x] = n_die;
  }
}

// Offsets of every tile's births and deaths; NAdd_ / NRemove_ / idMax_
// bookkeeping of @addAgent/@removeAgent (functionRule.jl:59-70,97-102).
// One block.
template <typename T>
__global__ void __launch_bounds__(1024) k_fate_scan(Params<T> P) {
  __shared__ long long s_c[1024], s_d[1024];
  const int p = P.parity;
  const int nb = P.n_blocks;
  const int per = (nb + 1023) / 1024;
  const int b0 = threadIdx.x * per;
  long long c = 0, d = 0;
  for (int b = b0; b < b0 + per && b < nb; ++b) {
    c += P.blk_children[b];
    d += P.blk_deaths[b];
  }
  s_c[threadIdx.x] = c;
  s_d[threadIdx.x] = d;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    long long yc = threadIdx.x >= o ? s_c[threadIdx.x - o] : 0;
    long long yd = threadIdx.x >= o ? s_d[threadIdx.x - o] : 0;
    __syncthreads();
    s_c[threadIdx.x] += yc;
    s_d[threadIdx.x] += yd;
    __syncthreads();
  }
  long long oc = s_c[threadIdx.x] - c, od = s_d[threadIdx.x] - d;
  for (int b = b0; b < b0 + per && b < nb; ++b) {
    P.blk_child_off[b] = (int)oc;
    P.blk_death_off[b] = (int)od;
    oc += P.blk_children[b];
    od += P.blk_deaths[b];
  }
  if (threadIdx.x == 1023) {
    Counters* C = P.ctr;
    long long N = C->N[p];
    long long tc = s_c[1023], td = s_d[1023];
    long long room = (long long)P.n_max - N;
    long long added = tc < room ? tc : room;
    if (added < tc) atomicOr(&C->err, kErrAgentOverflow);
    C->n_add = added;
    C->n_remove = td;
    C->children = tc;
    C->id_base = C->id_max;
    C->id_max += tc;  // ids are consumed even by dropped births
    if (tc > 0 || td > 0) C->flag[p] = 1;
  }
}

// ---------------------------------------------------------------------------
// agentStepDE!: fused neighbor force + Euler / EM update, births and holes
// (src/integrators.jl:465-505,683-734, functionDE.jl:13-117,
//  functionRule.jl:59-70,97-102)
// ---------------------------------------------------------------------------
template <typename T, int D>
__device__ __forceinline__ void place_births(const Params<T>& P, int i, int fate, int N) {
  __shared__ int warp_sums[kTile / 32];
  const int b = blockIdx.x;
  int has_events = P.blk_children[b] + P.blk_deaths[b];
  if (has_events == 0) return;  // uniform over the block
  const int nch = fate == 2 ? 2 : (fate == 3 ? 1 : 0);
  const int die = (fate == 1 || fate == 2) ? 1 : 0;
  int tot;
  int rc = block_exscan(nch, warp_sums, &tot) + P.blk_child_off[b];
  int rd = block_exscan(die, warp_sums, &tot) + P.blk_death_off[b];
  if (die) P.holes[rd] = i;
  if (nch == 0) return;
  T x[3];
  load_pos<T, D>(P.pos_cur, i, x);
  T a[3] = {0, 0, 0};
  if (fate == 2) {
    cbm_normals(P.seed, P.ctr->step[P.parity], (uint32_t)i, CBM_STREAM_DIVISION, P.community, D, a);
    T s = a[0] * a[0];
    if (D > 1) s = s + a[1] * a[1];
    if (D > 2) s = s + a[2] * a[2];
    T Ta = sqrt(s);
#pragma unroll
    for (int d = 0; d < D; ++d) a[d] = a[d] / Ta;
  }
  const long long idp = P.id[i];
  const T vv = P.v_cur[i];
  const T gg = P.g[i];
  for (int k = 0; k < nch; ++k) {
    long long slot = (long long)N + rc + k;
    if (slot >= P.n_max) break;  // dropped birth (counted in k_fate_scan)
    int s = (int)slot;
    if (fate == 2) {
#pragma unroll
      for (int d = 0; d < D; ++d)
        P.pos_nxt[d][s] = k == 0 ? x[d] + P.div_sep * a[d] : x[d] - P.div_sep * a[d];
      P.v_nxt[s] = vv / (T)2;
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) P.pos_nxt[d][s] = x[d];
      P.v_nxt[s] = vv;
    }
    if (P.force_mode == CBM_FORCE_LAGGED) {
#pragma unroll
      for (int d = 0; d < D; ++d) P.f_nxt[d][s] = P.f_cur[d][i];
    }
    P.g[s] = gg;
    P.id[s] = P.ctr->id_base + rc + k + 1;
    P.parent[s] = idp;
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_agent_de(Params<T> P) {
  const int p = P.parity;
  const int N = (int)P.ctr->N[p];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (P.fate_rule != CBM_FATE_NONE) {
    int fate = i < N ? P.fate[i] : 0;
    place_births<T, D>(P, i, fate, N);
  }
  if (i >= N || P.births_only) return;
  T* const* U = P.walls == CBM_WALLS_REFLECT ? P.pos_u : P.pos_cur;
  T xi[3];
  load_pos<T, D>(U, i, xi);
  T acc[3] = {(T)0, (T)0, (T)0};
  if (P.neighbors != CBM_NEIGH_NONE) {
    const T krep = P.k_rep, rrep = P.r_rep, katt = P.k_att, ratt = P.r_att;
    const bool from_rep = P.att_form == CBM_ATT_FROM_REP;
    for_neighbors<T, D>(P, xi, i, N, [&](int j) {
      T e[3];
      e[0] = xi[0] - ld(U[0] + j);
      T s2 = e[0] * e[0];
      if (D > 1) { e[1] = xi[1] - ld(U[1] + j); s2 = s2 + e[1] * e[1]; }
      if (D > 2) { e[2] = xi[2] - ld(U[2] + j); s2 = s2 + e[2] * e[2]; }
      T dist = sqrt(s2);
      T F;
      if (dist < rrep) F = krep * (rrep - dist);
      else if (dist < ratt) F = from_rep ? -(katt * (dist - rrep)) : -(katt * (ratt - dist));
      else return;
      T s = F / dist;
#pragma unroll
      for (int d = 0; d < D; ++d) acc[d] = acc[d] + s * e[d];
    });
  }
  if (P.walls == CBM_WALLS_PUSH) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (xi[d] < P.box_lo[d] + P.wall_range) acc[d] = acc[d] + P.wall_force;
      else if (xi[d] > P.box_hi[d] - P.wall_range) acc[d] = acc[d] - P.wall_force;
    }
  }
  T dv[3];
  if (P.force_mode == CBM_FORCE_LAGGED) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      P.f_nxt[d][i] = acc[d];
      dv[d] = P.f_cur[d][i];
    }
  } else {
#pragma unroll
    for (int d = 0; d < D; ++d) dv[d] = acc[d];
  }
  if (P.drift_linear != (T)0) {
#pragma unroll
    for (int d = 0; d < D; ++d) dv[d] = dv[d] + (-P.drift_linear) * xi[d];
  }
  if (P.medium && P.chemotaxis != (T)0) {
    T gv[3] = {(T)0, (T)0, (T)0};
    if (P.medium_sampling == CBM_MEDIUM_NEAREST) {
      int n = nearest_node<T, D>(P, xi);
#pragma unroll
      for (int d = 0; d < D; ++d) gv[d] = ld(P.grad_cur[d] + n);
    } else {
      int nodes[8];
      T w[8];
      bilinear<T, D>(P, xi, nodes, w);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        T s = (T)0;
#pragma unroll
        for (int q = 0; q < (1 << D); ++q) s = s + w[q] * ld(P.grad_cur[d] + nodes[q]);
        gv[d] = s;
      }
    }
    T s = gv[0] * gv[0];
    if (D > 1) s = s + gv[1] * gv[1];
    if (D > 2) s = s + gv[2] * gv[2];
    T den = (T)1 + sqrt(s);
#pragma unroll
    for (int d = 0; d < D; ++d) dv[d] = dv[d] + (P.chemotaxis * gv[d]) / den;
  }
  T xn[3];
  if (P.integrator == CBM_INT_EM) {
    T xi_n[3] = {(T)0, (T)0, (T)0};
    cbm_normals(P.seed, P.ctr->step[p], (uint32_t)i, CBM_STREAM_NOISE, P.community, D, xi_n);
#pragma unroll
    for (int d = 0; d < D; ++d) xn[d] = (xi[d] + dv[d] * P.dt) + (P.sigma * xi_n[d]) * P.sqrt_dt;
  } else {
#pragma unroll
    for (int d = 0; d < D; ++d) xn[d] = xi[d] + dv[d] * P.dt;
  }
#pragma unroll
  for (int d = 0; d < D; ++d) P.pos_nxt[d][i] = xn[d];
  if (P.growth) P.v_nxt[i] = P.v_cur[i] + P.g[i] * P.dt;
  else P.v_nxt[i] = P.v_cur[i];
  if (P.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT || P.neighbors == CBM_NEIGH_CLVD) {
    // verletDisplacement (neighbors.jl:367-391) on the new positions; when
    // agents are added or removed the flag is already set, so checking the
    // pre-compaction positions decides the same rebuild.
    T e = xn[0] - P.pos_old[0][i];
    T s = e * e;
    if (D > 1) { e = xn[1] - P.pos_old[1][i]; s = s + e * e; }
    if (D > 2) { e = xn[2] - P.pos_old[2][i]; s = s + e * e; }
    if (sqrt(s) >= P.rebuild_thr) P.ctr->flag[p] = 1;
  }
}

// ---------------------------------------------------------------------------
// mediumStepDE!: FTCS Euler step u <- u + dt (D lap(u) - lambda u) inside,
// du = 0 on the border (macros.jl:203-258)
// ---------------------------------------------------------------------------
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_medium_de(Params<T> P) {
  int n = blockIdx.x * kTile + threadIdx.x;
  if (n >= P.n_nodes) return;
  int q[3] = {0, 0, 0};
  q[0] = n % P.n_medium[0];
  if (D > 1) q[1] = (n / P.n_medium[0]) % P.n_medium[1];
  if (D > 2) q[2] = n / (P.n_medium[0] * P.n_medium[1]);
  bool in = true;
#pragma unroll
  for (int d = 0; d < D; ++d) in = in && q[d] > 0 && q[d] < P.n_medium[d] - 1;
  T u = P.c_cur[n];
  if (!in) {
    P.c_nxt[n] = u;
    return;
  }
  int stride[3] = {1, P.n_medium[0], P.n_medium[0] * P.n_medium[1]};
  T lap = (T)0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    T l = ((P.c_cur[n + stride[d]] - (T)2 * u) + P.c_cur[n - stride[d]]) / (P.dx_m[d] * P.dx_m[d]);
    lap = d == 0 ? l : lap + l;
  }
  T k = P.diff_D * lap - P.decay * u;
  P.c_nxt[n] = u + P.dt * k;
}

// ---------------------------------------------------------------------------
// update!: tail-fill compaction (kernelListSurvived + kernelFillHolesParameters,
// src/CommunityStructure/update.jl:15-119).  The k-th hole (ascending) takes
// the k-th survivor counted from the tail when the hole lies before it, which
// is the serial reference's permutation.
// ---------------------------------------------------------------------------
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_compact(Params<T> P) {
  const int p = P.parity;
  const Counters* C = P.ctr;
  const long long N = C->N[p];
  const long long R = C->n_remove;
  const long long total = N + C->n_add;
  const long long surv = total - R;
  const long long fills = R < surv ? R : surv;
  for (long long k = blockIdx.x * (long long)kTile + threadIdx.x; k < fills;
       k += (long long)gridDim.x * kTile) {
    // survivor with tail rank k: the largest q with #survivors in [q, total) >= k + 1,
    // #survivors in [q, total) = (total - q) - (R - #holes < q)
    long long lo = 0, hi = total - 1;
    while (lo < hi) {
      long long mid = (lo + hi + 1) >> 1;
      long long a = 0, b = R;  // lower_bound of mid in holes
      while (a < b) {
        long long m = (a + b) >> 1;
        if (P.holes[m] < mid) a = m + 1; else b = m;
      }
      long long s = (total - mid) - (R - a);
      if (s >= k + 1) lo = mid; else hi = mid - 1;
    }
    const int src = (int)lo, dst = P.holes[k];
    if (dst < src) {
#pragma unroll
      for (int d = 0; d < D; ++d) P.pos_nxt[d][dst] = P.pos_nxt[d][src];
      P.v_nxt[dst] = P.v_nxt[src];
      if (P.force_mode == CBM_FORCE_LAGGED) {
#pragma unroll
        for (int d = 0; d < D; ++d) P.f_nxt[d][dst] = P.f_nxt[d][src];
      }
      P.g[dst] = P.g[src];
      P.id[dst] = P.id[src];
      P.parent[dst] = P.parent[src];
    }
  }
}

// N <- N + NAdd - NRemove, t += dt, step += 1 (update.jl:201-298).  One thread.
template <typename T>
__global__ void k_commit(Params<T> P) {
  Counters* C = P.ctr;
  const int p = P.parity;
  C->N[p ^ 1] = C->N[p] + C->n_add - C->n_remove;
  C->n_add = 0;
  C->n_remove = 0;
  C->t[p ^ 1] = C->t[p] + (double)P.dt;
  C->step[p ^ 1] = C->step[p] + 1;
  C->flag[p ^ 1] = 0;
}

// ---------------------------------------------------------------------------
// computeNeighbors!: cell grid (counting sort, stable within a cell) and the
// Verlet list.  Kernels see the positions and N committed by update! (parity
// p ^ 1 of the step that ends) and do nothing unless a rebuild is due.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool rebuild_due(const Params<T>& P) {
  if (P.neighbors == CBM_NEIGH_CELL_LINKED) return true;
  return P.ctr->flag[P.parity] != 0;
}

// assignCells (neighbors.jl:763-821) + verletResetDisplacement (:438-487)
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_cells_hist(Params<T> P) {
  if (!rebuild_due(P)) return;
  const int N = (int)P.ctr->N[P.parity ^ 1];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i == 0) {
    // fresh tickets and tile-state generation for this build's k_cells_scan
    P.ctr->scan_ticket = 0u;
    P.ctr->scan_epoch = P.ctr->scan_epoch + 1u;
  }
  if (i >= N) return;
  T x[3];
  load_pos<T, D>(P.pos_nxt, i, x);
  int c = cell_of<T, D>(P, x);
  P.agent_cell[i] = c;
  P.agent_rank[i] = atomicAdd(P.cell_count + c, 1);
  if (P.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT || P.neighbors == CBM_NEIGH_CLVD) {
#pragma unroll
    for (int d = 0; d < D; ++d) P.pos_old[d][i] = x[d];
  }
}

// exclusive scan of the cell counts (cumsum .- counts, neighbors.jl:934-937)
// in one pass with decoupled look-back; counts are zeroed for the next build.
template <typename T>
__global__ void __launch_bounds__(kTile) k_cells_scan(Params<T> P) {
  __shared__ int warp_sums[kTile / 32];
  __shared__ unsigned s_tile;
  __shared__ int s_prefix;
  if (!rebuild_due(P)) return;
  Counters* C = P.ctr;
  const unsigned epoch = C->scan_epoch;
  if (threadIdx.x == 0) s_tile = atomicAdd(&C->scan_ticket, 1u);
  __syncthreads();
  const int tile = (int)s_tile;
  if (tile >= P.n_scan_tiles) {  // tickets were not reset: never index past the tile states
    if (threadIdx.x == 0) atomicOr(&C->err, kErrTimeout);
    return;
  }
  const int base = tile * kScanTile + threadIdx.x * kScanItems;
  int vals[kScanItems];
  int sum = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int c = base + k;
    vals[k] = c < P.n_cells ? P.cell_count[c] : 0;
    sum += vals[k];
  }
  int total;
  int ex = block_exscan(sum, warp_sums, &total);
  // publish aggregate, look back, publish inclusive prefix
  const unsigned long long ep = (unsigned long long)epoch << 32;
  if (threadIdx.x == 0) {
    if (tile == 0) {
      s_prefix = 0;
      atomicExch(P.scan_state + tile, ep | (2ull << 30) | (unsigned)total);
    } else {
      atomicExch(P.scan_state + tile, ep | (1ull << 30) | (unsigned)total);
      int prefix = 0;
      int t = tile - 1;
      long long spins = 0;
      while (t >= 0) {
        unsigned long long s = atomicAdd(P.scan_state + t, 0ull);
        unsigned flag = (unsigned)(s >> 30) & 3u;
        if ((s >> 32) != epoch || flag == 0) {
          if (++spins > kSpinLimit) {
            atomicOr(&C->err, kErrTimeout);
            break;
          }
          continue;
        }
        prefix += (int)(s & 0x3fffffffu);
        if (flag == 2) break;
        --t;
      }
      s_prefix = prefix;
      atomicExch(P.scan_state + tile, ep | (2ull << 30) | (unsigned)(prefix + total));
    }
  }
  __syncthreads();
  int run = s_prefix + ex;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    int c = base + k;
    if (c < P.n_cells) {
      P.cell_start[c] = run;
      P.cell_count[c] = 0;
    }
    run += vals[k];
  }
  // the thread holding the last cell writes the end sentinel
  if (base <= P.n_cells - 1 && P.n_cells - 1 < base + kScanItems) P.cell_start[P.n_cells] = run;
}

// sortAgentsInCells (neighbors.jl:837-899), first pass: scatter by the
// atomic rank taken in k_cells_hist
template <typename T>
__global__ void __launch_bounds__(kTile) k_cells_scatter(Params<T> P) {
  if (!rebuild_due(P)) return;
  const int N = (int)P.ctr->N[P.parity ^ 1];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  P.cell_tmp[P.cell_start[P.agent_cell[i]] + P.agent_rank[i]] = i;
}

// second pass: place every agent by its rank among the cell's agents with a
// smaller index, so agents are ascending within each cell as in the serial
// CPU reference (neighbors.jl:851-862)
template <typename T>
__global__ void __launch_bounds__(kTile) k_cells_stable(Params<T> P) {
  if (!rebuild_due(P)) return;
  const int N = (int)P.ctr->N[P.parity ^ 1];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  const int c = P.agent_cell[i];
  const int s0 = P.cell_start[c], s1 = P.cell_start[c + 1];
  int r = 0;
  for (int s = s0; s < s1; ++s) r += ld(P.cell_tmp + s) < i;
  P.cell_agents[s0 + r] = i;
}

// Verlet list over the cell grid: CLVD in cell order (verletNeighborsCLVD,
// neighbors.jl:1071-1131); VerletDisplacement sorted ascending
// (verletNeighbors, :92-133)
constexpr int kVdSortMax = 256;

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_verlet_list(Params<T> P) {
  if (!rebuild_due(P)) return;
  const int N = (int)P.ctr->N[P.parity ^ 1];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  T xi[3];
  load_pos<T, D>(P.pos_nxt, i, xi);
  const T skin = P.skin;
  const int M = P.max_nbrs;
  int n = 0;
  bool over = false;
  int q[3];
  cell_coords<D>(P.n_cells_d, cell_of<T, D>(P, xi), q);
  constexpr int nk = D == 1 ? 3 : (D == 2 ? 9 : 27);
  for (int k = 0; k < nk; ++k) {
    int pn = cell_neigh<D>(P.n_cells_d, q, k);
    if (pn < 0) continue;
    int s0 = ld(P.cell_start + pn), s1 = ld(P.cell_start + pn + 1);
    for (int s = s0; s < s1; ++s) {
      int j = ld(P.cell_agents + s);
      if (j == i) continue;
      T e = xi[0] - ld(P.pos_nxt[0] + j);
      T s2 = e * e;
      if (D > 1) { e = xi[1] - ld(P.pos_nxt[1] + j); s2 = s2 + e * e; }
      if (D > 2) { e = xi[2] - ld(P.pos_nxt[2] + j); s2 = s2 + e * e; }
      if (sqrt(s2) < skin) {
        if (n < M) P.nbr_list[(size_t)n * P.n_max + i] = j;
        else over = true;
        ++n;
      }
    }
  }
  if (over) atomicOr(&P.ctr->err, kErrNeighborOverflow);
  n = n < M ? n : M;
  if (P.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT && n > 1) {
    // insertion sort of the row (ascending j, the O(N^2) reference's order)
    for (int a = 1; a < n; ++a) {
      int key = P.nbr_list[(size_t)a * P.n_max + i];
      int b = a - 1;
      while (b >= 0 && P.nbr_list[(size_t)b * P.n_max + i] > key) {
        P.nbr_list[(size_t)(b + 1) * P.n_max + i] = P.nbr_list[(size_t)b * P.n_max + i];
        --b;
      }
      P.nbr_list[(size_t)(b + 1) * P.n_max + i] = key;
    }
  }
  P.nbr_n[i] = n;
}

// ---------------------------------------------------------------------------
// helpers for the host API
// ---------------------------------------------------------------------------
// the neighbor-counting rule of test/testCommunity.jl:359-415 on committed x
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_count_neighbors(Params<T> P, T radius, int* out) {
  const int N = (int)P.ctr->N[P.parity];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  T xi[3];
  load_pos<T, D>(P.pos_cur, i, xi);
  int n = 0;
  for_neighbors<T, D>(P, xi, i, N, [&](int j) {
    T e = xi[0] - P.pos_cur[0][j];
    T s2 = e * e;
    if (D > 1) { e = xi[1] - P.pos_cur[1][j]; s2 = s2 + e * e; }
    if (D > 2) { e = xi[2] - P.pos_cur[2][j]; s2 = s2 + e * e; }
    if (sqrt(s2) < radius) ++n;
  });
  out[i] = n;
}

// committed -> written copies for a stage that was skipped within a step
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_copy_agents(Params<T> P) {
  const int N = (int)P.ctr->N[P.parity];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  T* const* U = P.walls == CBM_WALLS_REFLECT ? P.pos_u : P.pos_cur;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    P.pos_nxt[d][i] = U[d][i];
    P.f_nxt[d][i] = P.f_cur[d][i];
  }
  P.v_nxt[i] = P.v_cur[i];
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_copy_medium(Params<T> P, int grad_only) {
  int n = blockIdx.x * kTile + threadIdx.x;
  if (n >= P.n_nodes) return;
  if (!grad_only) P.c_nxt[n] = P.c_cur[n];
#pragma unroll
  for (int d = 0; d < D; ++d) P.grad_nxt[d][n] = P.grad_cur[d][n];
}

template <typename T>
__global__ void __launch_bounds__(kTile) k_rng_fill(uint64_t seed, uint32_t community,
                                                    long long step, int kind, T a, T b,
                                                    long long n, T* out) {
  long long i = blockIdx.x * (long long)kTile + threadIdx.x;
  if (i >= n) return;
  T z;
  if (kind == 0) {
    cbm_normals(seed, step, (uint32_t)i, CBM_STREAM_USER, community, 1, &z);
    z = b * z + a;
  } else if (kind == 1) {
    z = (b - a) * cbm_uniform<T>(seed, step, (uint32_t)i, CBM_STREAM_USER, community) + a;
  } else {
    T u = cbm_uniform<T>(seed, step, (uint32_t)i, CBM_STREAM_USER, community);
    if (sizeof(T) == 8) z = -(T)cbm_log_f64((double)((T)1 - u)) * a;
    else z = -(T)cbm_log_f32((float)((T)1 - u)) * a;
  }
  out[i] = z;
}

}  // namespace cbm
