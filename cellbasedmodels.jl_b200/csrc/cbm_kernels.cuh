// cbm_kernels.cuh — the stepping engine's kernels.
//
// Layout.  The committed agent state (positions and the DE variables) is kept
// in "slots" sorted by grid cell and, inside a cell, by agent index: the order
// in which the reference visits neighbor candidates (src/neighbors.jl:715-747,
// cells x fastest, agents ascending inside a cell).  Positions are packed as
// float4 / double4, so a warp of consecutive slots reads its candidates'
// positions as a few contiguous runs instead of scattered loads.  Per-agent
// constants (growth rate, id, parent id) stay in agent-index order.  `IA`
// maps slot -> agent index and `inv` maps agent index -> slot.
//
// Every reference semantic that depends on the agent index is evaluated on
// the index: random keys, the ascending order inside a cell, birth slots
// (N + rank of the parent), and the tail-fill compaction (update.jl:15-119),
// which here relabels slots.  A step ends by re-sorting the working slots
// (survivors with their new indices plus newborns) by (cell, index): that one
// pass is the compaction gather and the grid rebuild of computeNeighbors!.
//
// Set A holds the committed state, set B the state being written by the
// current step (the reference's x__).  Every kernel reads N, the step and the
// flags from the device counter block, so a whole step is a static CUDA
// graph without host round trips (the reference reads flagRecomputeNeighbors_
// and NAdd_ on the host every step, src/neighbors.jl:548, update.jl:214).
#pragma once
#include <type_traits>

#include "cbm_common.cuh"

namespace cbm {

template <typename T>
struct V4T;
template <>
struct V4T<float> {
  using type = float4;
};
template <>
struct V4T<double> {
  using type = double4;
};

template <typename T>
struct Params {
  using V4 = typename V4T<T>::type;
  // slot-ordered state: committed (A) and written (B)
  V4* PA;
  V4* PB;
  T* VA;
  T* VB;
  V4* FA;               // lagged force
  V4* FB;
  int* IA;              // slot -> agent index
  int* IB;              // working labels (relabelled by the compaction, -1 = dead)
  V4* U;                // positions after the rule's wall reflection (walls only)
  // multi-stage integrators (Heun, RungeKutta4): stage positions, running sum
  // and derivative of every slot, and per launch of k_agent_de the stage
  // positions to read (XS) and where to store the derivative instead of
  // integrating (KOUT); no_prune turns the cell walk's face pruning off
  // (stage positions may lie outside the cells of the grid)
  V4* stage_h;
  V4* stage_s;
  V4* stage_k;
  const V4* XS;
  V4* KOUT;
  int no_prune;
  V4* POLD;             // positions at the last Verlet rebuild (slot order)
  int* inv;             // agent index -> slot of A
  int* cell_of_slot;    // cell of each A slot
  // agent-index-ordered constants
  T* G;
  long long* ID;
  long long* PAR;
  // index-ordered host exchange staging
  T* hx[3];
  T* hv;
  T* hf[3];
  // fate
  unsigned char* fate;
  int* holes;
  unsigned long long* fate_state;  // per tile: epoch | flag | children | deaths
  // re-sort
  int* s_cell;          // cell of each working slot (-1 dead)
  int* s_rank;          // atomic rank inside the cell
  int* s_key;           // agent index at each sorted position
  int* cell_count;
  int* cell_start;      // n_cells + 1
  const int* gather_box;  // per medium axis d, per node q: gather_cell_lo, then gather_cell_hi
  unsigned long long* scan_state;
  // Verlet list in slot space: entry k of the row of slot s at k * n_max + s
  int* nbr_n;
  int* nbr_list;
  // partner lists of the force walk: per block of k_agent_de, pair_cap4
  // blocks of four slots per thread (block j of thread t at j * kTile + t)
  int4* pair_list;
  int pair_cap4;
  // Float64 3D cell walks: the committed positions rounded to Float32, in
  // slot order, for the walk's filter (k_pos32); null otherwise
  float4* PA32;
  // Float32 3D cell walks: the committed positions as three rows x | y | z
  // of ps_stride floats (a multiple of four), for the walk's filter
  // (k_pos_rows); null otherwise
  float* PS;
  int ps_stride;
  // medium: committed / written
  T* c_cur;
  T* c_nxt;
  T* grad_cur[3];
  T* grad_nxt[3];
  Counters* ctr;
  const T* noise;       // EM increments given by the caller for this step (i * D + d), or null
  // sizes
  int n_max;
  int n_blocks;         // ceil(n_max / kTile)
  int n_cells;
  int n_cells_d[3];
  int n_scan_tiles;
  int n_nodes;
  int n_medium[3];
  int max_nbrs;
  int parity;
  // model
  int neighbors, integrator, force_mode, att_form, walls, fate_rule, growth, medium,
      medium_sampling;
  T box_lo[3], box_hi[3];
  T dt, sqrt_dt, sigma;
  double dt_time;           // the configured dt, by which the time t advances
  T edge;               // grid cell edge
  T skin, rebuild_thr;
  T k_rep, r_rep, k_att, r_att;
  // Squared-distance bounds above which sqrt(s2) is certain to fail the
  // reference's `d < cutoff` (resp. `d < skin`) test; pairs below them take
  // the exact test.  (cutoff^2 and skin^2 times 1 + 1e-5, rounded up.)
  T cut2, skin2;
  T skin2_lo;               // skin^2 times 1 - 1e-5, rounded down: below it d < skin for certain
  int force_in_list;        // (T)cutoff <= (T)skin: every pair with a force term is in the list
  T cut_reach, skin_reach;  // cutoff and skin times 1 + 1e-4: cell-pruning radii
  T wall_force, wall_range, drift_linear;
  T v_div, div_sep, p_death;
  T dx_m[3];
  T inv_dx[3], inv_dx2[3], inv_2dx[3];  // 1 / dx, 1 / dx^2, 1 / (2 dx) when powers of two, else 0
  int exact_scale;           // every axis of the medium has both reciprocals
  T diff_D, decay, secretion_amt, chemotaxis;
  T uptake_amt;             // uptake * dt (0: no uptake, and no clamp of the field)
  uint64_t seed;
  uint32_t community;
};

template <typename T>
__device__ __forceinline__ void to3(const typename V4T<T>::type& v, T* x) {
  x[0] = v.x;
  x[1] = v.y;
  x[2] = v.z;
}
template <typename T>
__device__ __forceinline__ typename V4T<T>::type from3(const T* x) {
  typename V4T<T>::type v;
  v.x = x[0];
  v.y = x[1];
  v.z = x[2];
  v.w = (T)0;
  return v;
}

template <typename T>
__device__ __forceinline__ bool is_verlet(const Params<T>& P) {
  return P.neighbors == CBM_NEIGH_CLVD || P.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT;
}

template <typename T, int D>
__device__ __forceinline__ int cell_of_pos(const Params<T>& P, const T* x) {
  return cell_of<T, D>(P.edge, P.box_lo, P.box_hi, P.n_cells_d, x);
}

template <typename T, int D>
__device__ __forceinline__ int nearest_node(const Params<T>& P, const T* x) {
  int lin = cell_in_mesh<T>(P.dx_m[0], x[0], P.box_lo[0], P.box_hi[0], P.n_medium[0]);
  if (D > 1)
    lin += P.n_medium[0] * cell_in_mesh<T>(P.dx_m[1], x[1], P.box_lo[1], P.box_hi[1], P.n_medium[1]);
  if (D > 2)
    lin += P.n_medium[0] * P.n_medium[1] *
           cell_in_mesh<T>(P.dx_m[2], x[2], P.box_lo[2], P.box_hi[2], P.n_medium[2]);
  return lin;
}

// v / dx on axis d: the product with the exact reciprocal when dx is a power
// of two (the same correctly rounded value), else the quotient.
template <typename T>
__device__ __forceinline__ T over_dx(const Params<T>& P, int d, T v) {
  return P.inv_dx[d] != (T)0 ? v * P.inv_dx[d] : v / P.dx_m[d];
}

// Clamped node indices i0 <= i1 of the multilinear stencil around x on each
// axis (nodes at the cell centres lo + (i + 1/2) dx) and the fractional
// offsets tt.
template <typename T, int D>
__device__ __forceinline__ void bilinear_axes(const Params<T>& P, const T* x, int* i0, int* i1,
                                              T* tt) {
#pragma unroll
  for (int d = 0; d < D; ++d) {
    T s = over_dx(P, d, x[d] - P.box_lo[d]) - (T)0.5;
    T fl = floor(s);
    tt[d] = s - fl;
    int a = (int)fl, b = a + 1;
    int hi = P.n_medium[d] - 1;
    i0[d] = a < 0 ? 0 : (a > hi ? hi : a);
    i1[d] = b < 0 ? 0 : (b > hi ? hi : b);
  }
}

// Weight of stencil node q (bit d of q: i1 rather than i0 on axis d).
template <typename T, int D>
__device__ __forceinline__ T bilinear_weight(const T* tt, int q) {
  T wq = (T)1;
#pragma unroll
  for (int d = 0; d < D; ++d) wq = wq * (((q >> d) & 1) ? tt[d] : (T)1 - tt[d]);
  return wq;
}

// Nodes and weights of the multilinear stencil around x (indices clamped to
// the grid).
template <typename T, int D>
__device__ __forceinline__ void bilinear(const Params<T>& P, const T* x, int* node, T* w) {
  int i0[3], i1[3];
  T tt[3];
  bilinear_axes<T, D>(P, x, i0, i1, tt);
#pragma unroll
  for (int q = 0; q < (1 << D); ++q) {
    int lin = 0, mul = 1;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      lin += (((q >> d) & 1) ? i1[d] : i0[d]) * mul;
      mul *= P.n_medium[d];
    }
    node[q] = lin;
    w[q] = bilinear_weight<T, D>(tt, q);
  }
}

// euclidean, src/metrics.jl:34-36: sqrt((a1-b1)^2 + (a2-b2)^2 + (a3-b3)^2)
template <typename T, int D>
__device__ __forceinline__ T dist(const T* a, const T* b) {
  T e = a[0] - b[0];
  T s = e * e;
  if (D > 1) { e = a[1] - b[1]; s = s + e * e; }
  if (D > 2) { e = a[2] - b[2]; s = s + e * e; }
  return sqrt(s);
}

// Visit the candidate slots of the 3^D cells around the cell holding x, in
// the reference's order (cells x fastest; a row of three x-neighbor cells is
// one contiguous run of slots).
template <typename T, int D, typename F>
__device__ __forceinline__ void for_cell_slots(const Params<T>& P, const T* x, F&& body) {
  int q[3] = {0, 0, 0};
  cell_coords<D>(P.n_cells_d, cell_of_pos<T, D>(P, x), q);
  const int nx = P.n_cells_d[0];
  const int x0 = q[0] > 0 ? q[0] - 1 : 0;
  const int x1 = q[0] < nx - 1 ? q[0] + 1 : nx - 1;
  constexpr int ny_rows = D > 1 ? 3 : 1;
  constexpr int nz_rows = D > 2 ? 3 : 1;
  for (int dz = 0; dz < nz_rows; ++dz) {
    int pz = D > 2 ? q[2] + dz - 1 : 0;
    if (D > 2 && (pz < 0 || pz >= P.n_cells_d[2])) continue;
    for (int dy = 0; dy < ny_rows; ++dy) {
      int py = D > 1 ? q[1] + dy - 1 : 0;
      if (D > 1 && (py < 0 || py >= P.n_cells_d[1])) continue;
      int row = nx * (py + P.n_cells_d[1] * pz);
      int s0 = ld(P.cell_start + row + x0), s1 = ld(P.cell_start + row + x1 + 1);
      for (int s = s0; s < s1; ++s) body(s);
    }
  }
}

// Per-thread force queue of k_agent_de, in shared memory (kQueue * 1 KB per
// block, 48 KB: the static limit).  48 entries hold every partner of nearly
// every agent of a colony at the packing density (about 17 on average), whose
// terms then follow the walk in one converged drain; in denser colonies a
// full queue moves to the thread's partner list in global memory.
#ifndef CBM_FORCE_QUEUE
#define CBM_FORCE_QUEUE 48
#endif
constexpr int kQueue = CBM_FORCE_QUEUE;

// Partner-list capacity of the force walk, in blocks of four slots per
// thread: 1024 slots (4 KB), more than the partners of an agent in a colony
// compressed to 4 agents per unit volume (about 600 at most).  A list that
// fills is evaluated where it stands, so the capacity bounds memory, not
// correctness.
constexpr int kPairCap4 = 256;
// Partner lists (and the persistent force grid that owns them) are used in
// 3D; in 1D and 2D an agent's 3 or 9 cells hold few partners, and the
// queue's drain serves them.
template <int D>
constexpr bool kPartnerLists = D == 3;
static_assert(kPairCap4 >= kQueue / 4, "a flush must fit an empty list");

// Asynchronous 16-byte copy global -> shared that bypasses L1 (each thread
// waits for its own copies; no block barrier is involved).
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
// list blocks fetched ahead of the one being evaluated, and the ring they
// land in (the force queue, empty by then: kQueue / 4 blocks per thread)
constexpr int kListAhead = 8;
constexpr int kListRing = kQueue / 4;
static_assert(kListRing > kListAhead, "the staging ring must exceed the prefetch depth");

template <typename T>
struct Eps;
template <>
struct Eps<float> {
  static constexpr float v = 1.1920929e-07f;
};
template <>
struct Eps<double> {
  static constexpr double v = 2.220446049250313e-16;
};

// Like for_cell_slots, but cells whose nearest face is farther than `reach`
// from x are skipped (their agents cannot pass a `d < reach` test), and the
// positions of a run are loaded four at a time.  body(slot, position).
// Skipping cells keeps the order of the visited candidates, so the sums that
// follow are unchanged.  The face gaps carry a margin for the rounding of the
// cell assignment; cells next to the ghost layer are never skipped.
template <typename T, int D, typename F>
__device__ __forceinline__ void walk_runs(const Params<T>& P, const T* x, T reach, F&& run,
                                          int cell = -1);

template <typename T, int D, typename F>
__device__ __forceinline__ void walk_cells(const Params<T>& P, const typename V4T<T>::type* X,
                                           const T* x, T reach, F&& body) {
  using V4 = typename V4T<T>::type;
  walk_runs<T, D>(P, x, reach, [&](int s0, int s1) {
    for (int s = s0; s < s1; ++s) body(s, X[s]);
  });
}

// The pruned cell walk as a sequence of contiguous slot runs run(s0, s1).
// `cell`, when given, is the linear cell of x (the grid's own assignment).
// The decisions of the 3^(D-1) rows are taken first and kept as a mask
// (three bits a row: visited, with the x-1 cell, with the x+1 cell), so the
// walk itself holds only the mask, x's cell column and its first row.
template <typename T, int D, typename F>
__device__ __forceinline__ void walk_runs(const Params<T>& P, const T* x, T reach, F&& run,
                                          int cell) {
  int q[3] = {0, 0, 0};
  if (cell >= 0) {
    q[0] = cell % P.n_cells_d[0];
    if (D > 1) q[1] = (cell / P.n_cells_d[0]) % P.n_cells_d[1];
    if (D > 2) q[2] = cell / (P.n_cells_d[0] * P.n_cells_d[1]);
  }
  T gm[3] = {(T)0, (T)0, (T)0}, gp[3] = {(T)0, (T)0, (T)0};
#pragma unroll
  for (int d = 0; d < D; ++d) {
    const int n = P.n_cells_d[d];
    const int c = cell >= 0 ? q[d] : cell_pos1<T>(P.edge, x[d], P.box_lo[d], P.box_hi[d], n);
    q[d] = c;
    if (c >= 2 && c <= n - 3 && !P.no_prune) {
      const T rel = x[d] - P.box_lo[d];
      const T k = (T)(c - 1);
      const T margin = (T)16 * Eps<T>::v * (fabs(rel) + (k + (T)1) * P.edge) + (T)1e-4 * reach;
      T a = rel - k * P.edge - margin;
      T b = (k + (T)1) * P.edge - rel - margin;
      gm[d] = a > (T)0 ? a : (T)0;
      gp[d] = b > (T)0 ? b : (T)0;
    }
  }
  const T r2 = reach * reach;
  const int nx = P.n_cells_d[0];
  constexpr int ny_rows = D > 1 ? 3 : 1;
  constexpr int nz_rows = D > 2 ? 3 : 1;
  unsigned mask = 0u;
#pragma unroll
  for (int dz = 0; dz < nz_rows; ++dz) {
#pragma unroll
    for (int dy = 0; dy < ny_rows; ++dy) {
      const int pz = D > 2 ? q[2] + dz - 1 : 0;
      const int py = D > 1 ? q[1] + dy - 1 : 0;
      if (D > 2 && (pz < 0 || pz >= P.n_cells_d[2])) continue;
      if (D > 1 && (py < 0 || py >= P.n_cells_d[1])) continue;
      const T gz = dz == 0 ? gm[2] : (dz == 2 ? gp[2] : (T)0);
      const T gy = dy == 0 ? gm[1] : (dy == 2 ? gp[1] : (T)0);
      const T gyz = (D > 1 ? gy * gy : (T)0) + (D > 2 ? gz * gz : (T)0);
      if (!(gyz < r2)) continue;
      const unsigned lo = (q[0] > 0 && gm[0] * gm[0] + gyz < r2) ? 2u : 0u;
      const unsigned hi = (q[0] < nx - 1 && gp[0] * gp[0] + gyz < r2) ? 4u : 0u;
      mask |= (1u | lo | hi) << (3 * (dz * ny_rows + dy));
    }
  }
  const int x0 = q[0];
  const int row0 = nx * ((D > 1 ? q[1] - 1 : 0) + P.n_cells_d[1] * (D > 2 ? q[2] - 1 : 0));
  for (int dz = 0; dz < nz_rows; ++dz)
    for (int dy = 0; dy < ny_rows; ++dy) {
      const unsigned m = mask >> (3 * (dz * ny_rows + dy));
      if (!(m & 1u)) continue;
      const int row = row0 + nx * (dy + P.n_cells_d[1] * dz);
      const int xa = x0 - (int)((m >> 1) & 1u), xb = x0 + (int)((m >> 2) & 1u);
      run(ld(P.cell_start + row + xa), ld(P.cell_start + row + xb + 1));
    }
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
// Bilinear secretion and uptake as a gather over medium nodes.  Atomic adds
// of unequal amounts would sum in an arbitrary order; here every node adds
// the contributions w (secretion dt - uptake dt c0) of the agents whose
// stencil covers it in ascending agent index, the order of the reference's
// serial agent loop (c0: the node's committed value).  The agents are
// found through the cell grid, which holds exactly the committed positions
// the rule reads when the grid is rebuilt every step (CellLinked).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ bool secretion_by_gather(const Params<T>& P) {
  return P.medium_sampling == CBM_MEDIUM_BILINEAR && P.neighbors == CBM_NEIGH_CELL_LINKED;
}

// Cell range on axis d of the agents whose stencil can cover node q: such
// agents lie in [lo + (q - 1/2) dx, lo + (q + 3/2) dx) (unbounded below for
// q = 0, above for the last node), widened by a rounding margin.  Both ends
// are non-decreasing in q.
template <typename T>
__device__ __forceinline__ T gather_margin(const Params<T>& P, int d) {
  return (T)1e-3 * P.dx_m[d] + (T)64 * Eps<T>::v * (fabs(P.box_lo[d]) + fabs(P.box_hi[d]));
}
template <typename T>
__device__ __forceinline__ int gather_cell_lo(const Params<T>& P, int d, int q) {
  return q == 0 ? 0
                : cell_pos1<T>(P.edge, P.box_lo[d] + ((T)q - (T)0.5) * P.dx_m[d] - gather_margin(P, d),
                               P.box_lo[d], P.box_hi[d], P.n_cells_d[d]);
}
template <typename T>
__device__ __forceinline__ int gather_cell_hi(const Params<T>& P, int d, int q) {
  return q == P.n_medium[d] - 1
             ? P.n_cells_d[d] - 1
             : cell_pos1<T>(P.edge, P.box_lo[d] + ((T)q + (T)1.5) * P.dx_m[d] + gather_margin(P, d),
                            P.box_lo[d], P.box_hi[d], P.n_cells_d[d]);
}

// The tables of gather_cell_lo / gather_cell_hi: for axis d (offset
// off[d] = 2 * (n_medium[0] + ... + n_medium[d-1])), entries q and
// n_medium[d] + q.  Filled once per context.
template <typename T>
__global__ void k_gather_box(Params<T> P, int* box, int dims) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  int off = 0;
  for (int d = 0; d < dims; ++d) {
    const int n = P.n_medium[d];
    if (q < n) {
      box[off + q] = gather_cell_lo(P, d, q);
      box[off + n + q] = gather_cell_hi(P, d, q);
    }
    off += 2 * n;
  }
}

// The gather of one node n by one thread: the agents of its cell box that
// touch it, sorted by index (or a k-way merge over the cells when more than
// kTouch touch it).  The path of crowded patches of k_secrete_rows.
template <typename T, int D>
__device__ __forceinline__ void secrete_node(const Params<T>& P, int n) {
  constexpr int kMaxCells = D == 1 ? 4 : (D == 2 ? 16 : 64);
  constexpr int kTouch = 32;  // agents collected per node before the merge fallback
  int q[3] = {0, 0, 0};
  q[0] = n % P.n_medium[0];
  if (D > 1) q[1] = (n / P.n_medium[0]) % P.n_medium[1];
  if (D > 2) q[2] = n / (P.n_medium[0] * P.n_medium[1]);
  const T amt = P.secretion_amt;
  const T c_com = P.c_cur[n];  // committed value: this thread is the node's only writer
  const bool upt = P.uptake_amt != (T)0;
  const T net = upt ? amt - P.uptake_amt * c_com : amt;  // secretion - first-order uptake
  T acc = c_com;
  auto add = [&](int slot) {
    T x[3];
    to3<T>(P.PA[slot], x);
    int nodes[8];
    T w[8];
    bilinear<T, D>(P, x, nodes, w);
#pragma unroll
    for (int k = 0; k < (1 << D); ++k)
      if (nodes[k] == n) acc = acc + w[k] * net;
  };
  // The stencil of bilinear() covers node q exactly when, on every axis, one
  // of its two clamped indices is q (the same expressions, without weights).
  auto touches = [&](int slot) {
    T x[3];
    to3<T>(P.PA[slot], x);
    bool t = true;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const T sd = over_dx(P, d, x[d] - P.box_lo[d]) - (T)0.5;
      const int a = (int)floor(sd), b = a + 1;
      const int hi = P.n_medium[d] - 1;
      const int i0 = a < 0 ? 0 : (a > hi ? hi : a);
      const int i1 = b < 0 ? 0 : (b > hi ? hi : b);
      t = t && (i0 == q[d] || i1 == q[d]);
    }
    return t;
  };
  int c0[3] = {0, 0, 0}, c1[3] = {0, 0, 0};
  int ncell = 1;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    c0[d] = gather_cell_lo(P, d, q[d]);
    c1[d] = gather_cell_hi(P, d, q[d]);
    ncell *= c1[d] - c0[d] + 1;
  }
  int tj[kTouch], ts[kTouch];
  int nt = 0;
  bool ok = ncell <= kMaxCells;
  for (int cz = c0[2]; ok && cz <= c1[2]; ++cz)
    for (int cy = c0[1]; ok && cy <= c1[1]; ++cy) {
      const int row = P.n_cells_d[0] * (cy + P.n_cells_d[1] * cz);
      const int s1 = P.cell_start[row + c1[0] + 1];
      for (int sl = P.cell_start[row + c0[0]]; sl < s1; ++sl) {
        if (!touches(sl)) continue;
        if (nt == kTouch) {
          ok = false;
          break;
        }
        const int j = P.IA[sl];
        int k = nt++;
        for (; k > 0 && tj[k - 1] > j; --k) {
          tj[k] = tj[k - 1];
          ts[k] = ts[k - 1];
        }
        tj[k] = j;
        ts[k] = sl;
      }
    }
  if (ok) {
    for (int k = 0; k < nt; ++k) add(ts[k]);
    P.c_cur[n] = acc;
    return;
  }
  // Fallback (a crowded node, or cells much smaller than the medium spacing):
  // k-way merge over the cells of the box widened by one cell, or every agent
  // in index order when even that box is too large.
#pragma unroll
  for (int d = 0; d < D; ++d) {
    c0[d] = c0[d] > 0 ? c0[d] - 1 : 0;
    c1[d] = c1[d] < P.n_cells_d[d] - 1 ? c1[d] + 1 : P.n_cells_d[d] - 1;
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
  if (all) {
    while (true) {  // k-way merge: next smallest agent index among the cells
      int best = -1, bj = 0x7fffffff;
      for (int k = 0; k < ncand; ++k)
        if (cur[k] < end[k]) {
          int j = P.IA[cur[k]];
          if (j < bj) { bj = j; best = k; }
        }
      if (best < 0) break;
      add(cur[best]++);
    }
  } else {
    const int N = (int)P.ctr->N[P.parity];
    for (int j = 0; j < N; ++j) add(P.inv[j]);
  }
  P.c_cur[n] = acc;
}

// The gather by patches: one warp takes the runs of 32 nodes along x of a
// patch of rows (4 x 4 (y, z) rows in 3D, 4 rows in 2D, 1 in 1D).  The
// patch's committed values and net rates are loaded into shared memory.  The
// union of the patch nodes' cell boxes is read at once: each lane takes one
// row of cells (one (y, z) pair of the box; its agents are contiguous slots),
// a warp scan numbers the candidates, and every lane takes one candidate of a
// chunk, computes its stencil (bilinear_axes, the expressions of bilinear())
// and the patch nodes it falls on.  The agents that touch the patch are
// appended to a warp list, and the list is ranked by agent index.  Groups of
// ranked entries add their terms with one lane per (entry, stencil node), in
// rounds that order the lanes sharing a node, so each node sums its terms in
// agent order and, within an agent, in stencil order: the sums of
// secrete_node.  A patch whose box has more than 32 rows, or that more than
// kCap agents touch, falls back to secrete_node for each of its nodes.  A
// node that no agent touches keeps its value and is not written.
template <int D>
struct GatherPatch {
  static constexpr int kY = D >= 2 ? 4 : 1, kZ = D > 2 ? 4 : 1;
  static constexpr int kRuns = kY * kZ;                // runs of 32 nodes a patch
  static constexpr int kCap = D == 3 ? 32 : 64;       // entries of the warp list
  static constexpr int kWarps = D == 3 ? 4 : (D == 2 ? 8 : 1);  // patches a block (along y)
};
constexpr unsigned short kNoNode = 0xffff;

template <typename T, int D>
__global__ void __launch_bounds__(GatherPatch<D>::kWarps * 32) k_secrete_rows(Params<T> P) {
  constexpr int K = 1 << D;
  constexpr int PY = GatherPatch<D>::kY, PZ = GatherPatch<D>::kZ, NP = GatherPatch<D>::kRuns;
  constexpr int CAP = GatherPatch<D>::kCap, W = GatherPatch<D>::kWarps;
  __shared__ int s_j[W][CAP];                   // agent index of entry e
  __shared__ unsigned short s_code[W][CAP][K];  // run * 32 + lane of stencil node k, or kNoNode
  __shared__ T s_w[W][CAP][K];
  __shared__ unsigned char s_perm[W][CAP];
  __shared__ T s_acc[W][NP * 32], s_net[W][NP * 32];
  __shared__ unsigned char s_tch[W][NP * 32];
  pdl_wait();
  const int lane = threadIdx.x & 31, wb = threadIdx.x >> 5;
  const int nx = P.n_medium[0];
  const int ny = D > 1 ? P.n_medium[1] : 1, nz = D > 2 ? P.n_medium[2] : 1;
  // grid: x runs, y patches (a block's warps), z patches
  const int x0 = blockIdx.x * 32;
  const int y0 = (blockIdx.y * W + wb) * PY, z0 = blockIdx.z * PZ;
  if (y0 >= ny) return;  // the whole warp
  const int xl = min(x0 + 31, nx - 1), yl = min(y0 + PY - 1, ny - 1), zl = min(z0 + PZ - 1, nz - 1);
  const int qx = x0 + lane;
  // the lane's nodes (run p: y0 + p % PY, z0 + p / PY): committed values
  // (this lane is their only writer) and net rates, secretion - uptake
  {
    const T amt = P.secretion_amt;
    const bool upt = P.uptake_amt != (T)0;
#pragma unroll
    for (int p = 0; p < NP; ++p) {
      const int y = y0 + p % PY, z = z0 + p / PY;
      const T v = (qx < nx && y < ny && z < nz) ? P.c_cur[qx + nx * (y + ny * z)] : (T)0;
      s_acc[wb][p * 32 + lane] = v;
      s_net[wb][p * 32 + lane] = upt ? amt - P.uptake_amt * v : amt;
      s_tch[wb][p * 32 + lane] = 0;
    }
  }
  const int* bx = P.gather_box;
  const int* by = bx + 2 * nx;
  const int* bz = by + 2 * ny;
  const int cx0 = ld(bx + x0), cx1 = ld(bx + nx + xl);
  const int cy0 = D > 1 ? ld(by + y0) : 0, cy1 = D > 1 ? ld(by + ny + yl) : 0;
  const int cz0 = D > 2 ? ld(bz + z0) : 0, cz1 = D > 2 ? ld(bz + nz + zl) : 0;
  const int nry = cy1 - cy0 + 1, nrows = nry * (cz1 - cz0 + 1);
  bool crowded = nrows > 32;
  int ne = 0;  // entries of the warp list
  if (!crowded) {
    int s0 = 0, cnt = 0;
    if (lane < nrows) {
      const int row = P.n_cells_d[0] * ((cy0 + lane % nry) + P.n_cells_d[1] * (cz0 + lane / nry));
      s0 = ld(P.cell_start + row + cx0);
      cnt = ld(P.cell_start + row + cx1 + 1) - s0;
    }
    int inc = cnt;  // inclusive scan of the rows' counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, inc, o);
      if (lane >= o) inc += y;
    }
    const int m_all = __shfl_sync(kFull, inc, 31);
    const unsigned below = (1u << lane) - 1u;
    for (int base = 0; base < m_all; base += 32) {
      const int m = base + lane;
      int r = 0;  // row of candidate m: the rows that end at or before it
      for (int k = 0; k < nrows; ++k) r += __shfl_sync(kFull, inc, k) <= m;
      const int rr = r < 31 ? r : 31;
      const int sl = __shfl_sync(kFull, s0, rr) + m - (__shfl_sync(kFull, inc, rr) -
                                                       __shfl_sync(kFull, cnt, rr));
      bool hit = false;
      unsigned short code[K];
      T w[K];
      int j = 0;
      if (m < m_all) {
        T x[3];
        to3<T>(P.PA[sl], x);
        j = P.IA[sl];
        int i0[3] = {0, 0, 0}, i1[3] = {0, 0, 0};
        T tt[3];
        bilinear_axes<T, D>(P, x, i0, i1, tt);
#pragma unroll
        for (int k = 0; k < K; ++k) {
          const int ix = (k & 1) ? i1[0] : i0[0];
          const int iy = ((k >> 1) & 1) ? i1[1] : i0[1];
          const int iz = ((k >> 2) & 1) ? i1[2] : i0[2];
          bool on = ix >= x0 && ix <= xl;
          if (D > 1) on = on && iy >= y0 && iy <= yl;
          if (D > 2) on = on && iz >= z0 && iz <= zl;
          const int run = (D > 2 ? (iz - z0) * PY : 0) + (D > 1 ? iy - y0 : 0);
          code[k] = on ? (unsigned short)(run * 32 + ix - x0) : kNoNode;
          w[k] = bilinear_weight<T, D>(tt, k);
          hit = hit || on;
        }
      }
      const unsigned hits = __ballot_sync(kFull, hit);
      if (ne + __popc(hits) > CAP) {
        crowded = true;
        break;
      }
      if (hit) {
        const int e = ne + __popc(hits & below);
        s_j[wb][e] = j;
#pragma unroll
        for (int k = 0; k < K; ++k) {
          s_code[wb][e][k] = code[k];
          s_w[wb][e][k] = w[k];
        }
      }
      ne += __popc(hits);
    }
  }
  if (crowded) {
#pragma unroll 1
    for (int p = 0; p < NP; ++p) {
      const int y = y0 + p % PY, z = z0 + p / PY;
      if (qx < nx && y < ny && z < nz) secrete_node<T, D>(P, qx + nx * (y + ny * z));
    }
    return;
  }
  if (ne == 0) return;
  __syncwarp();
  // rank by agent index (the indices are distinct): s_perm[rank] = entry
#pragma unroll
  for (int h = 0; h < CAP / 32; ++h) {
    const int e = h * 32 + lane;
    int r = -1;
    if (e < ne) {
      const int j = s_j[wb][e];
      r = 0;
      for (int f = 0; f < ne; ++f) r += s_j[wb][f] < j;
    }
    __syncwarp();
    if (r >= 0) s_perm[wb][r] = (unsigned char)e;
  }
  __syncwarp();
  // The ranked entries in groups of 32 / K, one lane per (entry, stencil
  // node), lanes in rank order and, within an entry, in stencil order.  Lanes
  // whose nodes coincide (a later entry on the same node, or a clamped
  // stencil that repeats a node) are ordered by lane: a lane's round is the
  // number of lower lanes with its node, and the rounds are applied in turn,
  // so every node takes its terms in rank and stencil order.
  constexpr int G = 32 / K;
  const int ge = lane / K, gk = lane % K;
  const unsigned lower = (1u << lane) - 1u;
  for (int base = 0; base < ne; base += G) {
    const int r = base + ge;
    int c = -1;
    T t = (T)0;
    if (r < ne) {
      const int e = s_perm[wb][r];
      const int code = s_code[wb][e][gk];
      if (code != kNoNode) {
        c = code;
        t = s_w[wb][e][gk];
      }
    }
    const unsigned same = __match_any_sync(kFull, c >= 0 ? c : 65536 + lane);
    const int round = c >= 0 ? __popc(same & lower) : 0;
    const int rounds = __reduce_max_sync(kFull, (unsigned)round) + 1;
    for (int q = 0; q < rounds; ++q) {
      if (c >= 0 && round == q) {
        s_acc[wb][c] = s_acc[wb][c] + t * s_net[wb][c];
        s_tch[wb][c] = 1;
      }
      __syncwarp();
    }
  }
#pragma unroll
  for (int p = 0; p < NP; ++p) {
    const int y = y0 + p % PY, z = z0 + p / PY;
    if (qx < nx && y < ny && z < nz && s_tch[wb][p * 32 + lane])
      P.c_cur[qx + nx * (y + ny * z)] = s_acc[wb][p * 32 + lane];
  }
}

// ---------------------------------------------------------------------------
// agentStepRule! of one agent index i < N: walls, secretion, and the fate
// decision (src/AgentStructure/functionRule.jl:9-111).  Returns 0 none,
// 1 die, 2 divide (two children, the parent is removed), 3 one child.
// ---------------------------------------------------------------------------
template <typename T, int D>
__device__ __forceinline__ int rule_agent(const Params<T>& P, int i, long long step) {
  const int s = P.inv[i];
  T x[3] = {(T)0, (T)0, (T)0};
  const bool exchange = P.medium && (P.secretion_amt != (T)0 || P.uptake_amt != (T)0);
  if (P.walls == CBM_WALLS_REFLECT || exchange) to3<T>(P.PA[s], x);
  if (P.walls == CBM_WALLS_REFLECT) {
    T y[3] = {x[0], x[1], x[2]};
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (x[d] < P.box_lo[d]) y[d] = (T)2 * P.box_lo[d] - x[d];
      else if (x[d] > P.box_hi[d]) y[d] = (T)2 * P.box_hi[d] - x[d];
    }
    P.U[s] = from3<T>(y);
  }
  if (exchange && !secretion_by_gather(P)) {
    // c__ += w (secretion dt - uptake dt c) with c the committed value, which
    // k_medium_snapshot copied to c_nxt before the rule (c_cur changes under
    // the atomics).  Nearest-node terms are equal for every agent of a node,
    // so their atomic sum does not depend on the order.
    const bool upt = P.uptake_amt != (T)0;
    if (P.medium_sampling == CBM_MEDIUM_NEAREST) {
      const int nn = nearest_node<T, D>(P, x);
      atomicAdd(P.c_cur + nn, upt ? P.secretion_amt - P.uptake_amt * P.c_nxt[nn] : P.secretion_amt);
    } else {
      int nodes[8];
      T w[8];
      bilinear<T, D>(P, x, nodes, w);
#pragma unroll
      for (int q = 0; q < (1 << D); ++q)
        atomicAdd(P.c_cur + nodes[q],
                  upt ? w[q] * (P.secretion_amt - P.uptake_amt * P.c_nxt[nodes[q]])
                      : w[q] * P.secretion_amt);
    }
  }
  int fate = 0;
  if (P.fate_rule == CBM_FATE_VOLUME) {
    if (P.growth && P.VA[s] >= P.v_div) fate = 2;
    else if (P.p_death > (T)0 &&
             cbm_uniform<T>(P.seed, step, (uint32_t)i, CBM_STREAM_DEATH, P.community) < P.p_death)
      fate = 1;
  } else if (P.fate_rule == CBM_FATE_ID_PARITY) {
    fate = (P.ID[i] % 2 == 1) ? 1 : 3;
  }
  return fate;
}

// agentStepRule! without births or deaths: one thread per agent index
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_agent_rule(Params<T> P) {
  const int p = P.parity;
  const int N = (int)P.ctr->N[p];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i < N) rule_agent<T, D>(P, i, P.ctr->step[p]);
}

// Tile state of the fate scan: epoch (4 bits) | flag (2) | children (29) |
// deaths (29).  Every launch rewrites every tile's state, so a state from the
// previous launch differs from the current one in the epoch.
__device__ __forceinline__ unsigned long long fate_word(unsigned epoch, unsigned flag,
                                                        unsigned long long children,
                                                        unsigned long long deaths) {
  return ((unsigned long long)(epoch & 15u) << 60) | ((unsigned long long)flag << 58) |
         (children << 29) | deaths;
}

// ---------------------------------------------------------------------------
// agentStepRule! with @addAgent / @removeAgent (functionRule.jl:9-111), one
// kernel: each tile of kFateTile agent indices (kFateItems consecutive ones
// per thread) decides the fates, ranks its births and deaths, takes their
// offsets from the preceding tiles with a decoupled look-back (tiles numbered
// in launch order, bounded wait), and then places its newborns and holes in
// agent-index order.  Newborn k of the step gets index and working slot
// N + k (dropped beyond n_max, but its id is still consumed,
// functionRule.jl:59-70); its DE variables go to set B, its constants to
// index N + k; parameters not given to @addAgent are copied from the parent's
// committed values.  The last tile writes NAdd_, NRemove_ and idMax_
// (functionRule.jl:59-70,97-102) and resets the tile tickets.
// ---------------------------------------------------------------------------
#ifndef CBM_FATE_ITEMS
#define CBM_FATE_ITEMS 8
#endif
constexpr int kFateItems = CBM_FATE_ITEMS;  // agents per thread of k_agent_fate
constexpr int kFateTile = kTile * kFateItems;
__host__ __device__ inline int fate_tiles(long long n_max) {
  return n_max > 0 ? (int)((n_max + kFateTile - 1) / kFateTile) : 1;
}

template <typename T, int D>
__device__ __forceinline__ void place_births(const Params<T>& P, int i, int fate, int N,
                                             long long step, long long first_child,
                                             long long id_base) {
  const int nch = fate == 2 ? 2 : (fate == 3 ? 1 : 0);
  const int s = P.inv[i];
  T x[3];
  to3<T>(P.PA[s], x);
  T a[3] = {(T)0, (T)0, (T)0};
  if (fate == 2) {
    cbm_normals(P.seed, step, (uint32_t)i, CBM_STREAM_DIVISION, P.community, D, a);
    T ss = a[0] * a[0];
    if (D > 1) ss = ss + a[1] * a[1];
    if (D > 2) ss = ss + a[2] * a[2];
    T Ta = sqrt(ss);
#pragma unroll
    for (int d = 0; d < D; ++d) a[d] = a[d] / Ta;
  }
  const long long idp = P.ID[i];
  const T vv = P.VA[s];
  const T gg = P.G[i];
  for (int k = 0; k < nch; ++k) {
    const long long slot = (long long)N + first_child + k;
    if (slot >= P.n_max) break;  // dropped birth (its id is still consumed)
    const int ns = (int)slot;
    T y[3] = {x[0], x[1], x[2]};
    if (fate == 2) {
#pragma unroll
      for (int d = 0; d < D; ++d) y[d] = k == 0 ? x[d] + P.div_sep * a[d] : x[d] - P.div_sep * a[d];
      P.VB[ns] = vv / (T)2;
    } else {
      P.VB[ns] = vv;
    }
    P.PB[ns] = from3<T>(y);
    if (P.force_mode == CBM_FORCE_LAGGED) P.FB[ns] = P.FA[s];
    P.IB[ns] = ns;
    P.G[ns] = gg;
    P.ID[ns] = id_base + first_child + k + 1;
    P.PAR[ns] = idp;
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_agent_fate(Params<T> P) {
  __shared__ int warp_sums[kTile / 32];
  __shared__ unsigned s_tile;
  __shared__ long long s_off[2];
  Counters* C = P.ctr;
  const int p = P.parity;
  const int n_tiles = fate_tiles(P.n_max);
  if (threadIdx.x == 0) s_tile = atomicAdd(&C->fate_ticket, 1u);
  __syncthreads();
  const int tile = (int)s_tile;
  if (tile >= n_tiles) {  // tickets were not reset: never index past the tile states
    if (threadIdx.x == 0) atomicOr(&C->err, kErrTimeout);
    return;
  }
  // read before this tile publishes anything: the last tile updates id_max
  // and the epoch only after every tile's publication
  const unsigned epoch = C->fate_epoch;
  const int N = (int)C->N[p];
  const long long step = C->step[p];
  const long long id_base = C->id_max;  // idMax_ before this step's births
  const int i0 = tile * kFateTile + threadIdx.x * kFateItems;
  unsigned char fates[kFateItems];
  int mc = 0, md = 0;  // this thread's children and deaths
#pragma unroll
  for (int k = 0; k < kFateItems; ++k) {
    const int i = i0 + k;
    const int f = i < N ? rule_agent<T, D>(P, i, step) : 0;
    fates[k] = (unsigned char)f;
    if (i < P.n_max) P.fate[i] = (unsigned char)f;
    mc += f == 2 ? 2 : (f == 3 ? 1 : 0);
    md += (f == 1 || f == 2) ? 1 : 0;
  }
  // children in the high half, deaths in the low half (at most 4096 / 2048 a tile)
  int tot;
  const int ex = block_exscan((mc << 16) | md, warp_sums, &tot);
  const int tc = tot >> 16, td = tot & 0xffff;
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (tile == 0) {
      if (lane == 0) {
        s_off[0] = 0;
        s_off[1] = 0;
        __threadfence();
        atomicExch(P.fate_state, fate_word(epoch, 2u, (unsigned)tc, (unsigned)td));
      }
    } else {
      if (lane == 0) {
        __threadfence();
        atomicExch(P.fate_state + tile, fate_word(epoch, 1u, (unsigned)tc, (unsigned)td));
      }
      long long pc = 0, pd = 0;
      int t = tile - 1;
      long long spins = 0;
      const unsigned long long mask29 = (1ull << 29) - 1ull;
      while (true) {
        const int idx = t - lane;
        unsigned flag = 2u;  // before tile 0: an inclusive prefix of 0
        unsigned long long vc = 0, vd = 0;
        if (idx >= 0) {
          const unsigned long long w = atomicAdd(P.fate_state + idx, 0ull);
          flag = ((unsigned)(w >> 60) == (epoch & 15u)) ? (unsigned)(w >> 58) & 3u : 0u;
          vc = (w >> 29) & mask29;
          vd = w & mask29;
        }
        const unsigned incl = __ballot_sync(kFull, flag == 2u);
        const unsigned pend = __ballot_sync(kFull, flag == 0u);
        const unsigned upto = incl ? ((incl & (0u - incl)) << 1) - 1u : kFull;
        if (pend & upto) {
          if (++spins > kSpinLimit) {
            if (lane == 0) atomicOr(&C->err, kErrTimeout);
            break;
          }
          continue;
        }
        unsigned long long sc = ((1u << lane) & upto) ? vc : 0ull;
        unsigned long long sd = ((1u << lane) & upto) ? vd : 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          sc += __shfl_xor_sync(kFull, sc, o);
          sd += __shfl_xor_sync(kFull, sd, o);
        }
        pc += (long long)sc;
        pd += (long long)sd;
        if (incl) break;
        t -= 32;
      }
      if (lane == 0) {
        s_off[0] = pc;
        s_off[1] = pd;
        __threadfence();
        atomicExch(P.fate_state + tile, fate_word(epoch, 2u, (unsigned long long)(pc + tc),
                                                  (unsigned long long)(pd + td)));
      }
    }
  }
  __syncthreads();
  long long rc = s_off[0] + (ex >> 16), rd = s_off[1] + (ex & 0xffff);
  if (mc + md > 0) {
#pragma unroll 1
    for (int k = 0; k < kFateItems; ++k) {
      const int f = fates[k];
      if (f == 0) continue;
      const int i = i0 + k;
      if (f == 1 || f == 2) {
        if (rd < P.n_max) P.holes[rd] = i;
        ++rd;
      }
      if (f == 2 || f == 3) {
        place_births<T, D>(P, i, f, N, step, rc, id_base);
        rc += f == 2 ? 2 : 1;
      }
    }
  }
  if (tile == n_tiles - 1 && threadIdx.x == 0) {
    const long long tcs = s_off[0] + tc, tds = s_off[1] + td;
    const long long room = (long long)P.n_max - N;
    const long long added = tcs < room ? tcs : room;
    if (added < tcs) atomicOr(&C->err, kErrAgentOverflow);
    C->n_add = added;
    C->n_remove = tds;
    C->children = tcs;
    C->id_base = id_base;
    C->id_max = id_base + tcs;  // ids are consumed even by dropped births
    C->events = (tcs > 0 || tds > 0) ? 1 : 0;
    if (tcs > 0 || tds > 0) C->flag[p] = 1;
    C->fate_ticket = 0u;
    C->fate_epoch = epoch + 1u;
  }
}

// ---------------------------------------------------------------------------
// agentStepDE!: fused neighbor force + Euler / EM update, one thread per slot
// (src/integrators.jl:465-505,683-734, functionDE.jl:13-117)
// ---------------------------------------------------------------------------
// Packed pairs of float operations (sm_100 f32x2): one instruction, and per
// element the same IEEE rounding as the scalar operation.
__device__ __forceinline__ float2 f2_sub(float2 a, float2 b) {
  unsigned long long r;
  asm("sub.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)),
        "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}
__device__ __forceinline__ float2 f2_mul(float2 a, float2 b) {
  unsigned long long r;
  asm("mul.rn.f32x2 %0, %1, %2;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)),
        "l"(*reinterpret_cast<unsigned long long*>(&b)));
  return *reinterpret_cast<float2*>(&r);
}

__device__ __forceinline__ float2 f2_fma(float2 a, float2 b, float2 c) {
  unsigned long long r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;"
      : "=l"(r)
      : "l"(*reinterpret_cast<unsigned long long*>(&a)),
        "l"(*reinterpret_cast<unsigned long long*>(&b)),
        "l"(*reinterpret_cast<unsigned long long*>(&c)));
  return *reinterpret_cast<float2*>(&r);
}

// e = xi - xj and its squared norm, in the reference's order
// ((e0 e0 + e1 e1) + e2 e2); in Float32 the x and y halves are packed pairs.
template <typename T, int D>
__device__ __forceinline__ T pair_diff(const T* xi, const T* xj, T* e) {
  if constexpr (std::is_same<T, float>::value && D > 1) {
    const float2 d = f2_sub(make_float2(xi[0], xi[1]), make_float2(xj[0], xj[1]));
    const float2 q = f2_mul(d, d);
    e[0] = d.x;
    e[1] = d.y;
    T s2 = q.x + q.y;
    if (D > 2) {
      e[2] = xi[2] - xj[2];
      s2 = s2 + e[2] * e[2];
    }
    return s2;
  }
  e[0] = xi[0] - xj[0];
  T s2 = e[0] * e[0];
  if (D > 1) {
    e[1] = xi[1] - xj[1];
    s2 = s2 + e[1] * e[1];
  }
  if (D > 2) {
    e[2] = xi[2] - xj[2];
    s2 = s2 + e[2] * e[2];
  }
  return s2;
}

// Coefficients of the soft-sphere pair term.
template <typename T>
struct PairCoef {
  T cut2, rrep, ratt, krep, katt;
  bool from_rep;
};
template <typename T>
__device__ __forceinline__ PairCoef<T> pair_coef(const Params<T>& P) {
  return PairCoef<T>{P.cut2, P.r_rep, P.r_att, P.k_rep, P.k_att, P.att_form == CBM_ATT_FROM_REP};
}

// Soft-sphere pair term (repulsion inside r_rep, attraction up to r_att) of
// the difference e with squared norm s2, added to acc.
template <typename T, int D>
__device__ __forceinline__ void pair_term(const PairCoef<T>& c, const T* e, T s2, T* acc) {
  if (s2 >= c.cut2) return;  // d >= cutoff for certain (NaN takes the exact test)
  const T dd = sqrt(s2);
  T F;
  if (dd < c.rrep) F = c.krep * (c.rrep - dd);
  else if (dd < c.ratt) F = c.from_rep ? -(c.katt * (dd - c.rrep)) : -(c.katt * (c.ratt - dd));
  else return;
  const T sc = F / dd;
#pragma unroll
  for (int d = 0; d < D; ++d) acc[d] = acc[d] + sc * e[d];
}

// Terms of the first nblk stored partner blocks of slot s, oldest first.
// Out of line: it runs only when a partner list fills in the middle of a
// walk, and keeping it out of the walk keeps the walk's code small.
template <typename T, int D>
__device__ __noinline__ void list_terms(const PairCoef<T> c, const typename V4T<T>::type* U,
                                        const int4* list, int nblk, int s, const T* xi, T* acc) {
  for (int j = 0; j < nblk; ++j) {
    const int4 b = __ldcg(list + (size_t)j * kTile);
    const int qq[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (qq[u] == s) continue;
      T xj[3], e[3];
      to3<T>(U[qq[u]], xj);
      const T s2 = pair_diff<T, D>(xi, xj, e);
      pair_term<T, D>(c, e, s2, acc);
    }
  }
}

// Squared distance for the candidate filter only: x and y packed, z fused.
template <typename T, int D>
__device__ __forceinline__ T filter_s2(const T* xi, const T* xj) {
  if constexpr (std::is_same<T, float>::value && D > 2) {
    const float2 d = f2_sub(make_float2(xi[0], xi[1]), make_float2(xj[0], xj[1]));
    const float2 q = f2_mul(d, d);
    const float dz = xi[2] - xj[2];
    return __fmaf_rn(dz, dz, q.x + q.y);
  } else {
    T e[3];
    return pair_diff<T, D>(xi, xj, e);
  }
}

// Float32 squared distance of the filter from a rounded Float64 position
// (the packed form of filter_s2<float, 3>).
__device__ __forceinline__ float filter_s2_f32(const float* xi, const float4 v) {
  const float2 d = f2_sub(make_float2(xi[0], xi[1]), make_float2(v.x, v.y));
  const float2 q = f2_mul(d, d);
  const float dz = xi[2] - v.z;
  return __fmaf_rn(dz, dz, q.x + q.y);
}

// Bound of the Float32 filter of a Float64 walk for an agent at xi: every
// pair whose Float64 squared distance passes the evaluation's test s2 < cut2
// has a Float32 one (positions rounded to nearest, filter_s2_f32) below it.
// With u = 2^-24, X = max_k |xi_k| and c = sqrt(cut2) (1 + 1e-15) the exact
// distance is below c, so |xj_k| <= X + c and each Float32 difference is
// within E = u (2X + 2c)(1 + u) of the exact one; three roundings of the
// squares and sums give s2_32 < (1 + u)^3 (c + sqrt(3) E)^2 (Minkowski).  The
// bound is formed in Float64 with a relative margin of 1e-12 for its own
// roundings and rounded up to Float32.
__device__ __forceinline__ float f32_filter_bound(const double* xi, double cut2) {
  const double u = 5.9604644775390625e-08;
  double X = 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d) X = fmax(X, fabs(xi[d]));
  const double c = sqrt(cut2) * (1.0 + 1e-15);
  const double E = u * (2.0 * X + 2.0 * c) * (1.0 + u);
  const double r = c + 1.7320508075688775 * E;
  return __double2float_ru(r * r * (1.0 + 4.0 * u) * (1.0 + 1e-12));
}

// PS = the committed Float32 positions as rows x | y | z (slots below N).
template <typename T>
__global__ void __launch_bounds__(kTile) k_pos_rows(Params<T> P) {
  const int N = (int)P.ctr->N[P.parity];
  const int st = P.ps_stride;
  for (int s = blockIdx.x * kTile + threadIdx.x; s < N; s += gridDim.x * kTile) {
    const typename V4T<T>::type v = P.PA[s];
    P.PS[s] = (float)v.x;
    P.PS[st + s] = (float)v.y;
    P.PS[2 * st + s] = (float)v.z;
  }
}

// PA32 = the committed positions rounded to Float32 (slots below N).
template <typename T>
__global__ void __launch_bounds__(kTile) k_pos32(Params<T> P) {
  const int N = (int)P.ctr->N[P.parity];
  for (int s = blockIdx.x * kTile + threadIdx.x; s < N; s += gridDim.x * kTile) {
    const typename V4T<T>::type v = P.PA[s];
    P.PA32[s] = make_float4((float)v.x, (float)v.y, (float)v.z, 0.f);
  }
}

// The end of agentStepDE! for slot s once its pair forces are summed in acc:
// pushing walls, the lagged force, linear drift and chemotaxis, then the
// integrator (Euler or Euler-Maruyama), the commit of the written slot and
// the displacement check of the Verlet algorithms.  xi: the positions the
// step reads (the stage's, the rule's reflected ones, or the committed ones).
template <typename T, int D>
__device__ __forceinline__ void finish_agent(const Params<T>& P, const int s, const T* xi, T* acc) {
  const int p = P.parity;
  if (P.walls == CBM_WALLS_PUSH) {
#pragma unroll
    for (int d = 0; d < D; ++d) {
      if (xi[d] < P.box_lo[d] + P.wall_range) acc[d] = acc[d] + P.wall_force;
      else if (xi[d] > P.box_hi[d] - P.wall_range) acc[d] = acc[d] - P.wall_force;
    }
  }
  T dv[3];
  if (P.force_mode == CBM_FORCE_LAGGED) {
    T fc[3];
    to3<T>(P.FA[s], fc);
    P.FB[s] = from3<T>(acc);
#pragma unroll
    for (int d = 0; d < D; ++d) dv[d] = fc[d];
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
      int nn = nearest_node<T, D>(P, xi);
#pragma unroll
      for (int d = 0; d < D; ++d) gv[d] = ld(P.grad_cur[d] + nn);
    } else {
      int nodes[8];
      T w[8];
      bilinear<T, D>(P, xi, nodes, w);
#pragma unroll
      for (int d = 0; d < D; ++d) {
        T sm = (T)0;
#pragma unroll
        for (int q = 0; q < (1 << D); ++q) sm = sm + w[q] * ld(P.grad_cur[d] + nodes[q]);
        gv[d] = sm;
      }
    }
    T g2 = gv[0] * gv[0];
    if (D > 1) g2 = g2 + gv[1] * gv[1];
    if (D > 2) g2 = g2 + gv[2] * gv[2];
    T den = (T)1 + sqrt(g2);
#pragma unroll
    for (int d = 0; d < D; ++d) dv[d] = dv[d] + (P.chemotaxis * gv[d]) / den;
  }
  if (P.KOUT) {  // a stage of a multi-stage integrator: f(u) only
    P.KOUT[s] = from3<T>(dv);
    return;
  }
  const int i = ld(P.IA + s);  // agent index of the slot
  T xn[3] = {(T)0, (T)0, (T)0};
  if (P.integrator == CBM_INT_EM) {
    T xi_n[3] = {(T)0, (T)0, (T)0};
    if (P.noise) {
#pragma unroll
      for (int d = 0; d < D; ++d) xi_n[d] = P.noise[(size_t)i * D + d];
    } else {
      cbm_normals(P.seed, P.ctr->step[p], (uint32_t)i, CBM_STREAM_NOISE, P.community, D, xi_n);
    }
#pragma unroll
    for (int d = 0; d < D; ++d) xn[d] = (xi[d] + dv[d] * P.dt) + (P.sigma * xi_n[d]) * P.sqrt_dt;
  } else {
#pragma unroll
    for (int d = 0; d < D; ++d) xn[d] = xi[d] + dv[d] * P.dt;
  }
  P.PB[s] = from3<T>(xn);
  P.VB[s] = P.growth ? P.VA[s] + ld(P.G + i) * P.dt : P.VA[s];
  P.IB[s] = i;
  if (is_verlet(P) && !P.ctr->events) {
    // verletDisplacement (neighbors.jl:367-391) on the new positions; when
    // agents are added or removed this step the flag is already set and the
    // check is skipped.
    T xo[3];
    to3<T>(P.POLD[s], xo);
    if (dist<T, D>(xn, xo) >= P.rebuild_thr) P.ctr->flag[p] = 1;
  }
}

// Slot s of N; `list` is this thread's partner list (null: none); `live`
// holds the lanes of this warp whose slot is below N.
template <typename T, int D>
__device__ __forceinline__ void agent_de(const Params<T>& P, const int N, const int s,
                                         int4* const list, const unsigned live) {
  using V4 = typename V4T<T>::type;
  const int p = P.parity;
  if (s >= N) return;
  const bool reflect = P.walls == CBM_WALLS_REFLECT;
  // positions read by this launch: a stage's, the rule's reflected ones, or
  // the committed ones
  const V4* U = P.XS ? P.XS : (reflect ? P.U : P.PA);
  T xi[3];
  to3<T>(U[s], xi);
  T acc[3] = {(T)0, (T)0, (T)0};
  const T krep = P.k_rep, rrep = P.r_rep, katt = P.k_att, ratt = P.r_att;
  const T cut2 = P.cut2;
  // the filter's fused squared distance is within a few ulps of the
  // evaluation's; 2^-20 above the bound keeps every pair the evaluation keeps
  const T cut2f = cut2 * ((T)1 + (T)9.5367431640625e-07);
  const bool from_rep = P.att_form == CBM_ATT_FROM_REP;
  // pair term with the difference e = xi - xj and its squared norm s2
  const PairCoef<T> coef = pair_coef<T>(P);
  auto pair_e = [&](const T* e, T s2) { pair_term<T, D>(coef, e, s2, acc); };
  auto diff = [&](const T* xj, T* e) { return pair_diff<T, D>(xi, xj, e); };
  auto pair = [&](const T* xj) {
    T e[3];
    T s2 = diff(xj, e);
    pair_e(e, s2);
  };
  const int alg = P.neighbors;
  if (alg == CBM_NEIGH_FULL) {
    for (int j = 0; j < N; ++j) {
      if (j == ld(P.IA + s)) continue;
      T xj[3];
      to3<T>(U[ld(P.inv + j)], xj);
      pair(xj);
    }
  } else if (alg == CBM_NEIGH_CELL_LINKED ||
             (alg == CBM_NEIGH_CLVD && !P.ctr->list_valid && !reflect)) {
    // Two phases.  The walk over the 3^D cells only filters: candidates that
    // may be within the cutoff are queued, in visiting order, in this
    // thread's column of a shared buffer.  The force terms are then
    // evaluated from the queue (and the partner list it spills to), where
    // nearly every lane has work, in visiting order.
    //
    // For CLVD the grid is current, so the list the last rebuild defines
    // (candidates within `skin` of the committed positions, in cell order)
    // is this walk; the list is also written out when no birth or death this
    // step forces another rebuild.
    __shared__ __align__(16) int queue[kQueue * kTile];
    int nq = 0;
    // Queued pairs four at a time: loads and differences of four entries are
    // independent, their terms are then added in queue order.  The agent
    // itself (queued by the force-only filter) is skipped here.
    auto drain = [&]() {
      int k = 0;
      for (; k + 4 <= nq; k += 4) {
        int qq[4];
        T xx[4][3], ee[4][3], ss[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) qq[u] = queue[(k + u) * kTile + threadIdx.x];
#pragma unroll
        for (int u = 0; u < 4; ++u) to3<T>(U[qq[u]], xx[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) ss[u] = diff(xx[u], ee[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (qq[u] != s) pair_e(ee[u], ss[u]);
      }
      for (; k < nq; ++k) {
        const int q = queue[k * kTile + threadIdx.x];
        if (q == s) continue;
        T xj[3];
        to3<T>(U[q], xj);
        pair(xj);
      }
      nq = 0;
    };
    auto enqueue = [&](int q) {
      queue[nq * kTile + threadIdx.x] = q;
      if (++nq == kQueue) drain();
    };
    const bool clvd = alg == CBM_NEIGH_CLVD;
    if (!(clvd && (P.ctr->events == 0 || !P.force_in_list))) {
      // force-only walk (CellLinked, or a CLVD step that will rebuild anyway
      // and whose cutoff lies inside the list radius): four independent
      // candidates per iteration, then an in-order enqueue.  Every active lane
      // empties its queue when one of them may run out of room.
      auto push = [&](int q) {
        queue[nq * kTile + threadIdx.x] = q;
        ++nq;
      };
      // With a partner list, a full queue is not evaluated but appended to the
      // list in blocks of four (a remainder of up to three stays queued); the
      // terms follow the walk, once every lane has all its partners.  Lanes
      // find their partners in bursts that differ from lane to lane (in the
      // rows near each agent), so evaluating whenever one lane's queue fills
      // keeps few lanes busy; at the end each lane's loop is as long as its
      // own partner count.
      int nl4 = 0;  // blocks of four entries in the list
      auto eval4 = [&](const int4 b) {
        const int qq[4] = {b.x, b.y, b.z, b.w};
        T xx[4][3], ee[4][3], ss[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) to3<T>(U[qq[u]], xx[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u) ss[u] = diff(xx[u], ee[u]);
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (qq[u] != s) pair_e(ee[u], ss[u]);
      };
      // the stored blocks in order, fetched kListAhead blocks ahead into the
      // queue, empty by then.  Ring position r of this lane is 16 bytes of the
      // warp's own queue columns (rows 4r..4r+3, eight lanes a row), so only
      // this warp touches it; the warp syncs before (here) and after (between
      // slots) its lanes reuse the queue.
      auto eval_list_staged = [&]() {
        const int lane = threadIdx.x & 31;
        int* const ring0 = queue + (lane >> 3) * kTile + (threadIdx.x & ~31) + (lane & 7) * 4;
        auto ring = [&](int r) { return reinterpret_cast<int4*>(ring0 + r * 4 * kTile); };
#pragma unroll
        for (int j = 0; j < kListAhead; ++j) {
          if (j < nl4) cp_async16(ring(j), list + (size_t)j * kTile);
          cp_async_commit();
        }
        int r = 0, w = kListAhead;  // ring positions of block j and of block j + kListAhead
        for (int j = 0; j < nl4; ++j) {
          cp_async_wait<kListAhead - 1>();
          const int4 b = *ring(r);
          if (j + kListAhead < nl4) cp_async16(ring(w), list + (size_t)(j + kListAhead) * kTile);
          cp_async_commit();
          r = r + 1 == kListRing ? 0 : r + 1;
          w = w + 1 == kListRing ? 0 : w + 1;
          eval4(b);
        }
        cp_async_wait<0>();
        nl4 = 0;
      };
      // whole blocks of the queue to the list; up to three entries stay queued,
      // or, with `all`, the last block is padded with the agent itself
      auto flush = [&](bool all) {
        const int nb = all ? (nq + 3) >> 2 : nq >> 2;
        if (nl4 + nb > P.pair_cap4) {  // list full: its terms now, in order
          list_terms<T, D>(coef, U, list, nl4, s, xi, acc);
          nl4 = 0;
        }
        for (int b = 0; b < nb; ++b) {
          int e[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int k = 4 * b + u;
            e[u] = k < nq ? queue[k * kTile + threadIdx.x] : s;
          }
          __stcg(list + (size_t)(nl4 + b) * kTile, make_int4(e[0], e[1], e[2], e[3]));
        }
        nl4 += nb;
        const int r = all ? 0 : nq & 3;
        for (int k = 0; k < r; ++k)
          queue[k * kTile + threadIdx.x] = queue[(4 * nb + k) * kTile + threadIdx.x];
        nq = r;
      };
      auto room = [&](int k) {
        if (__any_sync(__activemask(), nq > kQueue - k)) {
          if constexpr (kPartnerLists<D>) flush(false);
          else drain();
        }
      };
      // the slot's cell is the grid's assignment of the committed position,
      // which the walk starts from unless the rule reflected it off a wall
      const int own_cell = (reflect || P.XS) ? -1 : ld(P.cell_of_slot + s);
      // Float64 walks filter in Float32 on the rounded copy of the positions,
      // with the bound widened for the rounding; the evaluation's exact test
      // decides every queued pair
      const float4* U32 = nullptr;
      float xi32[3] = {0.f, 0.f, 0.f};
      float cut2f32 = 0.f;
      if constexpr (std::is_same<T, double>::value && D == 3) {
        if (P.PA32 && U == P.PA) {
          U32 = P.PA32;
#pragma unroll
          for (int d = 0; d < 3; ++d) xi32[d] = (float)xi[d];
          cut2f32 = f32_filter_bound(xi, (double)cut2);
        }
      }
      // Float32 walks over the position rows: four candidates a step from
      // three 16-byte loads, their squared distances as packed pairs
      // (fl(dx dx), then two fused terms: three roundings, as the scalar
      // filter's, inside the widened cutoff)
      const float* PS = nullptr;
      float2 xx = make_float2(0.f, 0.f), yy = xx, zz = xx;
      if constexpr (std::is_same<T, float>::value && D == 3) {
        if (P.PS && U == P.PA) {
          PS = P.PS;
          xx = make_float2(xi[0], xi[0]);
          yy = make_float2(xi[1], xi[1]);
          zz = make_float2(xi[2], xi[2]);
        }
      }
      walk_runs<T, D>(P, xi, P.cut_reach, [&](int s0, int s1) {
        int q = s0;
        if constexpr (std::is_same<T, float>::value && D == 3) {
          if (PS) {
            // one check for room a group of eight candidates (a warp vote),
            // and one for a run's unaligned head and tail of up to three
            if (q & 3) room(4);
            for (; q < s1 && (q & 3); ++q) {  // to a multiple of four
              T xj[3];
              to3<T>(U[q], xj);
              if (filter_s2<T, D>(xi, xj) < cut2f) push(q);
            }
            const int st = P.ps_stride;
            auto four = [&](int r) {
              const float4 a = ld(reinterpret_cast<const float4*>(PS + r));
              const float4 b = ld(reinterpret_cast<const float4*>(PS + st + r));
              const float4 c = ld(reinterpret_cast<const float4*>(PS + 2 * st + r));
              const float2 dx0 = f2_sub(xx, make_float2(a.x, a.y)), dx1 = f2_sub(xx, make_float2(a.z, a.w));
              const float2 dy0 = f2_sub(yy, make_float2(b.x, b.y)), dy1 = f2_sub(yy, make_float2(b.z, b.w));
              const float2 dz0 = f2_sub(zz, make_float2(c.x, c.y)), dz1 = f2_sub(zz, make_float2(c.z, c.w));
              const float2 q0 = f2_fma(dz0, dz0, f2_fma(dy0, dy0, f2_mul(dx0, dx0)));
              const float2 q1 = f2_fma(dz1, dz1, f2_fma(dy1, dy1, f2_mul(dx1, dx1)));
              const float s2v[4] = {q0.x, q0.y, q1.x, q1.y};
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                queue[nq * kTile + threadIdx.x] = r + u;
                nq += s2v[u] < cut2f ? 1 : 0;
              }
            };
            for (; q + 8 <= s1; q += 8) {
              room(8);
              four(q);
              four(q + 4);
            }
            if (q + 4 <= s1) {
              room(4);
              four(q);
              q += 4;
            }
            if (q < s1) room(4);
            for (; q < s1; ++q) {
              T xj[3];
              to3<T>(U[q], xj);
              if (filter_s2<T, D>(xi, xj) < cut2f) push(q);
            }
            return;
          }
        }
        if constexpr (std::is_same<T, double>::value && D == 3) {
          if (U32) {
            auto four = [&](int r) {
              float s2v[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) s2v[u] = filter_s2_f32(xi32, U32[r + u]);
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                queue[nq * kTile + threadIdx.x] = r + u;
                nq += s2v[u] < cut2f32 ? 1 : 0;
              }
            };
            for (; q + 8 <= s1; q += 8) {
              room(8);
              four(q);
              four(q + 4);
            }
            if (q + 4 <= s1) {
              room(4);
              four(q);
              q += 4;
            }
            if (q < s1) room(4);
            for (; q < s1; ++q)
              if (filter_s2_f32(xi32, U32[q]) < cut2f32) push(q);
            return;
          }
        }
        // every candidate is written at the queue's end and kept only when it
        // may be inside the cutoff (room() left space for the group); the
        // agent itself is skipped in the drain
        auto four = [&](int r) {
          T s2v[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            T xj[3];
            to3<T>(U[r + u], xj);
            s2v[u] = filter_s2<T, D>(xi, xj);
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            queue[nq * kTile + threadIdx.x] = r + u;
            nq += s2v[u] < cut2f ? 1 : 0;
          }
        };
        // candidates a check for room: eight in 1D and 2D; four in 3D, whose
        // main walks take the paths above and where a longer loop here would
        // cost the kernel registers
        constexpr int kGroup = D == 3 ? 4 : 8;
        for (; q + kGroup <= s1; q += kGroup) {
          room(kGroup);
#pragma unroll
          for (int g = 0; g < kGroup; g += 4) four(q + g);
        }
        if (kGroup == 8 && q + 4 <= s1) {
          room(4);
          four(q);
          q += 4;
        }
        if (q < s1) room(4);
        for (; q < s1; ++q) {
          T xj[3];
          to3<T>(U[q], xj);
          if (filter_s2<T, D>(xi, xj) < cut2f) push(q);
        }
      }, own_cell);
      // a warp with a stored list evaluates from the list, every entry of the
      // queue appended first; otherwise the queue is drained below
      if constexpr (kPartnerLists<D>) {
        __syncwarp(live);
        if (__any_sync(live, nl4 > 0)) {
          flush(true);
          __syncwarp(live);  // every lane's queue is read before the rings overwrite it
          eval_list_staged();
        }
      }
    } else {
      const bool write = !P.ctr->events;
      const T skin2 = P.skin2, skin2_lo = P.skin2_lo;
      int n = 0;
      bool over = false;
      walk_cells<T, D>(P, U, xi, write ? P.skin_reach : P.cut_reach, [&](int q, const V4& v) {
        if (q == s) return;
        T xj[3], e[3];
        to3<T>(v, xj);
        const T s2 = diff(xj, e);
        if (s2 >= skin2) return;                                   // d >= skin for certain
        if (!write && s2 >= cut2) return;                          // in the list, no force
        if (!(s2 < skin2_lo) && !(sqrt(s2) < P.skin)) return;      // exact test near skin
        if (write) {
          if (n < P.max_nbrs) P.nbr_list[(size_t)n * P.n_max + s] = q;
          else over = true;
          ++n;
        }
        if (s2 < cut2) enqueue(q);
      });
      if (write) {
        if (over) atomicOr(&P.ctr->err, kErrNeighborOverflow);
        P.nbr_n[s] = n < P.max_nbrs ? n : P.max_nbrs;
        if (s == 0) P.ctr->list_written = 1;
      }
    }
    drain();
  } else if (alg == CBM_NEIGH_CLVD && !P.ctr->list_valid) {
    // The grid is current, so the list the last rebuild defines (candidates
    // within `skin` of the committed positions, in cell order) is walked
    // directly.  It is also written out when no birth or death this step
    // forces another rebuild.
    const bool write = !P.ctr->events;
    T xa[3];
    to3<T>(P.PA[s], xa);
    int n = 0;
    bool over = false;
    const T skin2 = P.skin2;
    for_cell_slots<T, D>(P, xa, [&](int q) {
      if (q == s) return;
      T xj[3], e[3];
      to3<T>(U[q], xj);
      T s2 = diff(xj, e);
      if (reflect) {
        // list membership is decided on the committed positions
        T xb[3];
        to3<T>(P.PA[q], xb);
        if (!(dist<T, D>(xa, xb) < P.skin)) return;
      } else {
        if (s2 >= skin2) return;                       // d >= skin for certain
        if (!write && s2 >= cut2) return;              // in the list, no force
        if (!(sqrt(s2) < P.skin)) return;
      }
      if (write) {
        if (n < P.max_nbrs) P.nbr_list[(size_t)n * P.n_max + s] = q;
        else over = true;
      }
      ++n;
      pair_e(e, s2);
    });
    if (write) {
      if (over) atomicOr(&P.ctr->err, kErrNeighborOverflow);
      P.nbr_n[s] = n < P.max_nbrs ? n : P.max_nbrs;
      if (s == 0) P.ctr->list_written = 1;
    }
  } else if (is_verlet(P)) {
    const int n = P.nbr_n[s];
    for (int k = 0; k < n; ++k) {
      T xj[3];
      to3<T>(U[ld(P.nbr_list + (size_t)k * P.n_max + s)], xj);
      pair(xj);
    }
  }
  finish_agent<T, D>(P, s, xi, acc);
}

// One block per resident slot of the device, so each thread owns one region
// of the partner-list scratch.  Warp w first takes run w of 32 slots, then
// further runs from a ticket counter until the N slots are done (small
// colonies need no ticket).  The last block to finish resets the counter for
// the next launch.
template <typename T, int D>
__global__ void __launch_bounds__(kTile, sizeof(T) == 4 ? 4 : 3) k_agent_de(Params<T> P) {
  Counters* C = P.ctr;
  const int N = (int)C->N[P.parity];
  if constexpr (!kPartnerLists<D>) {  // one thread per slot, grid over n_max
    const int slot = (int)blockIdx.x * kTile + (int)threadIdx.x;
    agent_de<T, D>(P, N, slot, nullptr, __ballot_sync(kFull, slot < N));
    return;
  }
  const int n_runs = (N + 31) >> 5;
  const int lane = threadIdx.x & 31;
  const int n_warps = (int)gridDim.x * (kTile / 32);
  int4* const list =
      P.pair_list ? P.pair_list + (size_t)blockIdx.x * P.pair_cap4 * kTile + threadIdx.x : nullptr;
  int run = (int)blockIdx.x * (kTile / 32) + (int)(threadIdx.x >> 5);
  while (run < n_runs) {
    const int slot = (run << 5) + lane;
    agent_de<T, D>(P, N, slot, list, __ballot_sync(kFull, slot < N));
    __syncwarp();
    int t = 0;
    if (lane == 0) t = (int)atomicAdd(&C->de_ticket, 1u);
    run = n_warps + __shfl_sync(kFull, t, 0);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&C->de_done, 1u) == gridDim.x - 1) {
      C->de_ticket = 0u;
      C->de_done = 0u;
    }
  }
}

// ---------------------------------------------------------------------------
// Stage combinations of the multi-stage agent integrators over the slots of
// existing agents, with the reference's broadcast expressions element by
// element (src/integrators.jl: Heun :541-571, RungeKutta4 :606-666):
//   Heun  h1 = u + du dt;  u = (h1 + (u + du2 dt)) / 2
//   RK4   h1 = u + (k1 dt)/2, u + (k2 dt)/2, u + k3 dt;
//         u = u + ((((k1 + 2 k2) + 2 k3) + k4) dt) / 6
// The volume v is a DE variable with dv = g when growth is on; its stage
// values do not enter f, so only its final combination is formed.
// ---------------------------------------------------------------------------
//   EulerHeun (:775-810, the CPU branch):
//         h1 = (u + f1 dt) + (g xi1) sqrt(dt)
//         u = u + (((f1 + f2) dt) + ((g + g) xi2) sqrt(dt)) / 2
//         with g = sigma for positions, 0 for the volume, and xi2 a fresh draw
enum { kHeunStage = 0, kHeunFinal = 1, kRk1 = 2, kRk2 = 3, kRk3 = 4, kRkFinal = 5, kEhStage = 6,
       kEhFinal = 7 };

// verletDisplacement (neighbors.jl:367-391) on the new position xn of slot s,
// as k_agent_de does it for the single-stage integrators
template <typename T, int D>
__device__ __forceinline__ void stage_displacement(const Params<T>& P, int s, const T* xn) {
  if (is_verlet(P) && !P.ctr->events) {
    T xo[3];
    to3<T>(P.POLD[s], xo);
    if (dist<T, D>(xn, xo) >= P.rebuild_thr) P.ctr->flag[P.parity] = 1;
  }
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_stage_combine(Params<T> P, int op) {
  const int N = (int)P.ctr->N[P.parity];
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s >= N) return;
  const bool reflect = P.walls == CBM_WALLS_REFLECT;
  T u[3], k[3];
  to3<T>((reflect ? P.U : P.PA)[s], u);
  to3<T>(P.stage_k[s], k);
  const T dt = P.dt;
  T o[3] = {(T)0, (T)0, (T)0};
  if (op == kHeunStage || op == kRk3) {
#pragma unroll
    for (int d = 0; d < D; ++d) o[d] = u[d] + k[d] * dt;
  } else if (op == kRk1 || op == kRk2) {
#pragma unroll
    for (int d = 0; d < D; ++d) o[d] = u[d] + (k[d] * dt) / (T)2;
  }
  if (op == kEhStage || op == kEhFinal) {
    const int i = ld(P.IA + s);
    T xi[3] = {(T)0, (T)0, (T)0};
    cbm_normals(P.seed, P.ctr->step[P.parity], (uint32_t)i,
                op == kEhStage ? CBM_STREAM_NOISE : CBM_STREAM_NOISE_FINAL, P.community, D, xi);
    if (op == kEhStage) {
      P.stage_s[s] = P.stage_k[s];  // f1
#pragma unroll
      for (int d = 0; d < D; ++d) o[d] = (u[d] + k[d] * dt) + (P.sigma * xi[d]) * P.sqrt_dt;
      P.stage_h[s] = from3<T>(o);
      return;
    }
    T f1[3];
    to3<T>(P.stage_s[s], f1);
#pragma unroll
    for (int d = 0; d < D; ++d)
      o[d] = u[d] + (((f1[d] + k[d]) * dt) + ((P.sigma + P.sigma) * xi[d]) * P.sqrt_dt) / (T)2;
    const T v = P.VA[s];
    P.PB[s] = from3<T>(o);
    P.VB[s] = P.growth ? v + ((ld(P.G + i) + ld(P.G + i)) * dt) / (T)2 : v;
    P.IB[s] = i;
    stage_displacement<T, D>(P, s, o);
    return;
  }
  if (op == kRk1) {
    P.stage_s[s] = P.stage_k[s];
  } else if (op == kRk2 || op == kRk3 || op == kRkFinal) {
    T a[3];
    to3<T>(P.stage_s[s], a);
#pragma unroll
    for (int d = 0; d < D; ++d) a[d] = op == kRkFinal ? a[d] + k[d] : a[d] + (T)2 * k[d];
    P.stage_s[s] = from3<T>(a);
    if (op == kRkFinal) {
#pragma unroll
      for (int d = 0; d < D; ++d) o[d] = u[d] + (a[d] * dt) / (T)6;
    }
  }
  if (op != kHeunFinal && op != kRkFinal) {
    P.stage_h[s] = from3<T>(o);
    return;
  }
  const int i = ld(P.IA + s);
  const T v = P.VA[s];
  T vn = v;
  if (op == kHeunFinal) {
    T h[3];
    to3<T>(P.stage_h[s], h);
#pragma unroll
    for (int d = 0; d < D; ++d) o[d] = (h[d] + (u[d] + k[d] * dt)) / (T)2;
    if (P.growth) {
      const T g = ld(P.G + i);
      const T hv = v + g * dt;
      vn = (hv + (v + g * dt)) / (T)2;
    }
  } else if (P.growth) {
    const T g = ld(P.G + i);
    vn = v + ((((g + (T)2 * g) + (T)2 * g) + g) * dt) / (T)6;
  }
  P.PB[s] = from3<T>(o);
  P.VB[s] = vn;
  P.IB[s] = i;
  stage_displacement<T, D>(P, s, o);
}

// ---------------------------------------------------------------------------
// mediumStepDE!: FTCS Euler step u <- u + dt (D lap(u) - lambda u) inside,
// du = 0 on the border (macros.jl:203-258)
// ---------------------------------------------------------------------------
// The field as the DE step reads it: clamped at zero when uptake is on.
template <typename T>
__device__ __forceinline__ T medium_in(const Params<T>& P, T v) {
  return (P.uptake_amt != (T)0 && v < (T)0) ? (T)0 : v;
}

// v / (dx dx) and v / (2 dx) on axis d.  With kScale the divisor is a power
// of two, and the product with its exact reciprocal is the same correctly
// rounded value as the quotient (subnormal results, zeros and infinities
// included), without a division.
template <bool kScale, typename T>
__device__ __forceinline__ T over_dx2(const Params<T>& P, int d, T v) {
  return kScale ? v * P.inv_dx2[d] : v / (P.dx_m[d] * P.dx_m[d]);
}
template <bool kScale, typename T>
__device__ __forceinline__ T over_2dx(const Params<T>& P, int d, T v) {
  return kScale ? v * P.inv_2dx[d] : v / ((T)2 * P.dx_m[d]);
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_medium_de(Params<T> P) {
  pdl_wait();
  int n = blockIdx.x * kTile + threadIdx.x;
  if (n >= P.n_nodes) return;
  int q[3] = {0, 0, 0};
  q[0] = n % P.n_medium[0];
  if (D > 1) q[1] = (n / P.n_medium[0]) % P.n_medium[1];
  if (D > 2) q[2] = n / (P.n_medium[0] * P.n_medium[1]);
  bool in = true;
#pragma unroll
  for (int d = 0; d < D; ++d) in = in && q[d] > 0 && q[d] < P.n_medium[d] - 1;
  T u = medium_in(P, P.c_cur[n]);
  if (!in) {
    P.c_nxt[n] = u;
    return;
  }
  int stride[3] = {1, P.n_medium[0], P.n_medium[0] * P.n_medium[1]};
  T lap = (T)0;
#pragma unroll
  for (int d = 0; d < D; ++d) {
    T l = ((medium_in(P, P.c_cur[n + stride[d]]) - (T)2 * u) + medium_in(P, P.c_cur[n - stride[d]])) /
          (P.dx_m[d] * P.dx_m[d]);
    lap = d == 0 ? l : lap + l;
  }
  T k = P.diff_D * lap - P.decay * u;
  P.c_nxt[n] = u + P.dt * k;
}

// ---------------------------------------------------------------------------
// 2D medium stencils on shared-memory tiles: a block of kStX x kStY threads
// covers a kStX x (kStY * kStRows) tile of nodes and stages it with a
// one-node halo, so every node is read from HBM/L2 once per block.  Same
// expressions as k_medium_grad / k_medium_de.
// ---------------------------------------------------------------------------
constexpr int kStX = 32, kStY = 8, kStRows = 4;
constexpr int kStTileY = kStY * kStRows;

template <typename T>
__device__ __forceinline__ void stage_tile2(const Params<T>& P, T (*tile)[kStX + 2], int x0, int y0,
                                            bool clamp) {
  const int nx = P.n_medium[0], ny = P.n_medium[1];
  for (int k = threadIdx.y * kStX + threadIdx.x; k < (kStTileY + 2) * (kStX + 2); k += kStX * kStY) {
    const int ty = k / (kStX + 2), tx = k % (kStX + 2);
    const int gx = x0 + tx - 1, gy = y0 + ty - 1;
    const T v = (gx >= 0 && gx < nx && gy >= 0 && gy < ny) ? P.c_cur[(size_t)gy * nx + gx] : (T)0;
    tile[ty][tx] = clamp ? medium_in(P, v) : v;
  }
  __syncthreads();
}

template <typename T, bool kScale>
__device__ __forceinline__ void medium_grad_2d(const Params<T>& P) {
  __shared__ T tile[kStTileY + 2][kStX + 2];
  const int nx = P.n_medium[0], ny = P.n_medium[1];
  const int x0 = blockIdx.x * kStX, y0 = blockIdx.y * kStTileY;
  stage_tile2<T>(P, tile, x0, y0, false);
  const int x = x0 + threadIdx.x;
  if (x >= nx) return;
#pragma unroll
  for (int r = 0; r < kStRows; ++r) {
    const int ty = threadIdx.y + r * kStY, y = y0 + ty;
    if (y >= ny) break;
    const size_t n = (size_t)y * nx + x;
    const bool in = x > 0 && x < nx - 1 && y > 0 && y < ny - 1;
    const int tx = threadIdx.x + 1, tyy = ty + 1;
    P.grad_nxt[0][n] = in ? over_2dx<kScale>(P, 0, tile[tyy][tx + 1] - tile[tyy][tx - 1]) : (T)0;
    P.grad_nxt[1][n] = in ? over_2dx<kScale>(P, 1, tile[tyy + 1][tx] - tile[tyy - 1][tx]) : (T)0;
  }
}

template <typename T>
__global__ void __launch_bounds__(kStX * kStY) k_medium_grad_2d(Params<T> P) {
  if (P.exact_scale) medium_grad_2d<T, true>(P);
  else medium_grad_2d<T, false>(P);
}

template <typename T, bool kScale>
__device__ __forceinline__ void medium_de_2d(const Params<T>& P) {
  __shared__ T tile[kStTileY + 2][kStX + 2];
  const int nx = P.n_medium[0], ny = P.n_medium[1];
  const int x0 = blockIdx.x * kStX, y0 = blockIdx.y * kStTileY;
  stage_tile2<T>(P, tile, x0, y0, true);
  const int x = x0 + threadIdx.x;
  if (x >= nx) return;
#pragma unroll
  for (int r = 0; r < kStRows; ++r) {
    const int ty = threadIdx.y + r * kStY, y = y0 + ty;
    if (y >= ny) break;
    const size_t n = (size_t)y * nx + x;
    const int tx = threadIdx.x + 1, tyy = ty + 1;
    const T u = tile[tyy][tx];
    if (!(x > 0 && x < nx - 1 && y > 0 && y < ny - 1)) {
      P.c_nxt[n] = u;
      continue;
    }
    const T l0 = over_dx2<kScale>(P, 0, (tile[tyy][tx + 1] - (T)2 * u) + tile[tyy][tx - 1]);
    const T l1 = over_dx2<kScale>(P, 1, (tile[tyy + 1][tx] - (T)2 * u) + tile[tyy - 1][tx]);
    const T lap = l0 + l1;
    const T k = P.diff_D * lap - P.decay * u;
    P.c_nxt[n] = u + P.dt * k;
  }
}

template <typename T>
__global__ void __launch_bounds__(kStX * kStY) k_medium_de_2d(Params<T> P) {
  pdl_wait();
  if (P.exact_scale) medium_de_2d<T, true>(P);
  else medium_de_2d<T, false>(P);
}

// ---------------------------------------------------------------------------
// 3D medium stencils (7-point), marching along z: a block of kStX x kStY
// threads owns a kStX x kStTileY column of nodes over a run of z planes.  Each
// thread keeps its kStRows nodes of the planes z-1, z and z+1 in registers;
// plane z is staged in shared memory with a one-node x/y halo for the
// in-plane neighbours.  The march is pipelined: while plane z is computed,
// the values of plane z+2 and the halo of plane z+1 are already in flight,
// and the staged tiles alternate between two buffers, so a plane costs one
// block barrier and no exposed load latency.  Every node of the run is read
// from HBM once, plus the halo and the two planes that close the run.  Same
// expressions as k_medium_grad / k_medium_de: lap = (l_x + l_y) + l_z.
// ---------------------------------------------------------------------------
template <typename T, bool kDE>
__device__ __forceinline__ void stencil_3d(const Params<T>& P, int z_run) {
  __shared__ T tile[2][kStTileY + 2][kStX + 2];
  const int nx = P.n_medium[0], ny = P.n_medium[1], nz = P.n_medium[2];
  const int x0 = blockIdx.x * kStX, y0 = blockIdx.y * kStTileY;
  const int za = blockIdx.z * z_run;
  const int zb = za + z_run < nz ? za + z_run : nz;
  const size_t plane = (size_t)nx * (size_t)ny;
  auto read = [&](int gx, int gy, int gz) -> T {
    if (gx < 0 || gx >= nx || gy < 0 || gy >= ny || gz < 0 || gz >= nz) return (T)0;
    const T v = P.c_cur[(size_t)gz * plane + (size_t)gy * nx + gx];
    return kDE ? medium_in(P, v) : v;
  };
  const int x = x0 + threadIdx.x;
  const int t = threadIdx.y * kStX + threadIdx.x;
  // the halo node this thread stages: x-halo columns, then y-halo rows
  int hx = 0, hy = 0, hr = 0, hc = 0;
  const bool halo = t < 2 * kStTileY + 2 * kStX;
  if (t < kStTileY) {
    hx = x0 - 1, hy = y0 + t, hr = t + 1, hc = 0;
  } else if (t < 2 * kStTileY) {
    hx = x0 + kStX, hy = y0 + t - kStTileY, hr = t - kStTileY + 1, hc = kStX + 1;
  } else if (t < 2 * kStTileY + kStX) {
    hx = x0 + t - 2 * kStTileY, hy = y0 - 1, hr = 0, hc = t - 2 * kStTileY + 1;
  } else if (halo) {
    hx = x0 + t - 2 * kStTileY - kStX, hy = y0 + kStTileY, hr = kStTileY + 1,
    hc = t - 2 * kStTileY - kStX + 1;
  }
  T lo[kStRows], mid[kStRows], hi[kStRows], nxt[kStRows];
#pragma unroll
  for (int r = 0; r < kStRows; ++r) {
    const int y = y0 + threadIdx.y + r * kStY;
    lo[r] = read(x, y, za - 1);
    mid[r] = read(x, y, za);
    hi[r] = read(x, y, za + 1);
    tile[0][threadIdx.y + r * kStY + 1][threadIdx.x + 1] = mid[r];
  }
  if (halo) tile[0][hr][hc] = read(hx, hy, za);
  int buf = 0;
  for (int z = za; z < zb; ++z) {
    // in flight during this plane: plane z + 2 and the halo of plane z + 1
#pragma unroll
    for (int r = 0; r < kStRows; ++r) nxt[r] = read(x, y0 + threadIdx.y + r * kStY, z + 2);
    const T hnext = halo ? read(hx, hy, z + 1) : (T)0;
    __syncthreads();  // tile[buf] complete; tile[buf ^ 1] no longer read
#pragma unroll
    for (int r = 0; r < kStRows; ++r) {
      const int ty = threadIdx.y + r * kStY, y = y0 + ty;
      if (x < nx && y < ny) {
        const size_t n = (size_t)z * plane + (size_t)y * nx + x;
        const bool in = x > 0 && x < nx - 1 && y > 0 && y < ny - 1 && z > 0 && z < nz - 1;
        const int tx = threadIdx.x + 1, tyy = ty + 1;
        if (kDE) {
          const T u = mid[r];
          if (!in) {
            P.c_nxt[n] = u;
          } else {
            const T l0 = ((tile[buf][tyy][tx + 1] - (T)2 * u) + tile[buf][tyy][tx - 1]) /
                         (P.dx_m[0] * P.dx_m[0]);
            const T l1 = ((tile[buf][tyy + 1][tx] - (T)2 * u) + tile[buf][tyy - 1][tx]) /
                         (P.dx_m[1] * P.dx_m[1]);
            const T l2 = ((hi[r] - (T)2 * u) + lo[r]) / (P.dx_m[2] * P.dx_m[2]);
            const T lap = (l0 + l1) + l2;
            const T k = P.diff_D * lap - P.decay * u;
            P.c_nxt[n] = u + P.dt * k;
          }
        } else {
          P.grad_nxt[0][n] =
              in ? (tile[buf][tyy][tx + 1] - tile[buf][tyy][tx - 1]) / ((T)2 * P.dx_m[0]) : (T)0;
          P.grad_nxt[1][n] =
              in ? (tile[buf][tyy + 1][tx] - tile[buf][tyy - 1][tx]) / ((T)2 * P.dx_m[1]) : (T)0;
          P.grad_nxt[2][n] = in ? (hi[r] - lo[r]) / ((T)2 * P.dx_m[2]) : (T)0;
        }
      }
      // plane z + 1 into the other buffer, then shift the column
      tile[buf ^ 1][ty + 1][threadIdx.x + 1] = hi[r];
      lo[r] = mid[r];
      mid[r] = hi[r];
      hi[r] = nxt[r];
    }
    if (halo) tile[buf ^ 1][hr][hc] = hnext;
    buf ^= 1;
  }
}

template <typename T>
__global__ void __launch_bounds__(kStX * kStY) k_medium_grad_3d(Params<T> P, int z_run) {
  stencil_3d<T, false>(P, z_run);
}

template <typename T>
__global__ void __launch_bounds__(kStX * kStY) k_medium_de_3d(Params<T> P, int z_run) {
  pdl_wait();
  stencil_3d<T, true>(P, z_run);
}

// The committed field, copied before an agent rule that adds to it with
// atomics and takes up from it: the uptake reads the value before the rule.
template <typename T>
__global__ void __launch_bounds__(kTile) k_medium_snapshot(Params<T> P) {
  const int n = blockIdx.x * kTile + threadIdx.x;
  if (n < P.n_nodes) P.c_nxt[n] = P.c_cur[n];
}

// ---------------------------------------------------------------------------
// update!: tail-fill compaction (kernelListSurvived + kernelFillHolesParameters,
// src/CommunityStructure/update.jl:15-119).  The k-th hole (ascending) takes
// the k-th survivor counted from the tail when the hole lies before it, which
// is the serial reference's permutation.  Agent constants move in index
// order; slot-ordered variables keep their slot and get relabelled.
// ---------------------------------------------------------------------------
constexpr int kCompactThreads = 1024;

// Survivors that fill holes all lie in the tail [N_new, N + NAdd)
// and holes before N_new are exactly as many, so the tail is walked from its
// end in chunks, survivors are ranked by a block scan, and the k-th survivor
// from the tail moves into the k-th hole.
//
// When the step's births are at least its removals (a growing colony), the
// tail holds newborns only, which all survive: the k-th survivor from the
// tail is then slot total-1-k, and every block relabels its share directly.
template <typename T, int D>
__global__ void __launch_bounds__(kCompactThreads) k_compact(Params<T> P) {
  __shared__ int warp_sums[kCompactThreads / 32];
  __shared__ int s_total;
  const int p = P.parity;
  const Counters* C = P.ctr;
  const long long N = C->N[p];
  const long long R = C->n_remove;
  const long long total = N + C->n_add;
  const long long n_new = total - R;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (n_new >= N) {
    for (long long k = (long long)blockIdx.x * kCompactThreads + tid; k < R;
         k += (long long)gridDim.x * kCompactThreads) {
      const int dst = P.holes[k];
      const int src = (int)(total - 1 - k);  // a newborn: working slot == index
      P.IB[P.inv[dst]] = -1;                 // the dead agent's slot leaves the sort
      P.G[dst] = P.G[src];
      P.ID[dst] = P.ID[src];
      P.PAR[dst] = P.PAR[src];
      P.IB[src] = dst;
    }
    return;
  }
  if (blockIdx.x != 0) return;
  for (long long k = tid; k < R; k += kCompactThreads)
    P.IB[P.inv[P.holes[k]]] = -1;  // every dead agent's slot leaves the sort
  long long offset = 0;            // survivors already ranked
  for (long long base = 0; base < total - n_new; base += kCompactThreads) {
    const long long q = total - 1 - base - tid;
    bool live = false;
    if (q >= n_new) {
      live = true;
      if (q < N) {
        const int f = P.fate[q];
        live = !(f == 1 || f == 2);
      }
    }
    // exclusive block scan of `live`
    unsigned bal = __ballot_sync(kFull, live);
    int in_warp = __popc(bal & ((1u << lane) - 1u));
    if (lane == 0) warp_sums[w] = __popc(bal);
    __syncthreads();
    if (w == 0) {
      int v = warp_sums[lane];
      int x = v;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(kFull, x, o);
        if (lane >= o) x += y;
      }
      warp_sums[lane] = x - v;
      if (lane == 31) s_total = x;
    }
    __syncthreads();
    if (live) {
      const long long k = offset + warp_sums[w] + in_warp;  // tail rank of q
      if (k < R) {
        const int dst = P.holes[k];
        const int src = (int)q;
        if (dst < src) {
          P.G[dst] = P.G[src];
          P.ID[dst] = P.ID[src];
          P.PAR[dst] = P.PAR[src];
          // newborns sit in working slot == index; survivors in their A slot
          P.IB[src < N ? P.inv[src] : src] = dst;
        }
      }
    }
    offset += s_total;
    __syncthreads();
  }
}

// N <- N + NAdd - NRemove, t += dt, step += 1 (update.jl:201-298), and the
// re-sort decision of computeNeighbors!.  One thread.
template <typename T>
__global__ void k_commit(Params<T> P) {
  Counters* C = P.ctr;
  const int p = P.parity;
  C->slots = C->N[p] + C->n_add;
  C->N[p ^ 1] = C->N[p] + C->n_add - C->n_remove;
  C->n_add = 0;
  C->n_remove = 0;
  C->t[p ^ 1] = C->t[p] + P.dt_time;
  C->step[p ^ 1] = C->step[p] + 1;
  C->flag[p ^ 1] = 0;
  C->resort = (P.neighbors == CBM_NEIGH_CELL_LINKED || C->flag[p]) ? 1 : 0;
  C->events = 0;
  if (C->list_written) C->list_valid = 1;
  C->list_written = 0;
}

// ---------------------------------------------------------------------------
// End of step: B -> A.  Without a re-sort the working slots are copied; with
// one, live working slots are counting-sorted by (cell, agent index) into A
// (the grid rebuild of computeNeighbors!, neighbors.jl:918-979, and the
// compaction gather in one pass).
// ---------------------------------------------------------------------------
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_sort_hist(Params<T> P) {
  pdl_wait();
  const Counters* C = P.ctr;
  const int s = blockIdx.x * kTile + threadIdx.x;
  const long long slots = C->slots;
  if (!C->resort) {
    if (s < slots) {
      P.PA[s] = P.PB[s];
      P.VA[s] = P.VB[s];
      if (P.force_mode == CBM_FORCE_LAGGED) P.FA[s] = P.FB[s];
    }
    return;
  }
  if (s == 0) {
    P.ctr->scan_ticket = 0u;  // fresh tickets and tile-state generation for the scan
    P.ctr->scan_epoch = C->scan_epoch + 1u;
  }
  // The lanes of a warp hold consecutive slots, mostly of one cell in a
  // dense community: the lanes of each cell take their ranks with one atomic
  // add (any ranks 0 .. count-1 of a cell do, since the placement orders
  // the cell's agents by index).  Every lane of the warp gets here.
  int c = -1;
  if (s < slots && P.IB[s] >= 0) {
    T x[3];
    to3<T>(P.PB[s], x);
    c = cell_of_pos<T, D>(P, x);
  }
  if (s < slots) P.s_cell[s] = c;
  const unsigned peers = __match_any_sync(kFull, c);
  if (c >= 0) {
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(P.cell_count + c, __popc(peers));
    base = __shfl_sync(peers, base, leader);
    P.s_rank[s] = base + __popc(peers & ((1u << lane) - 1u));
  }
}

template <typename T>
__global__ void __launch_bounds__(kTile) k_sort_scatter(Params<T> P) {
  pdl_wait();
  const Counters* C = P.ctr;
  if (!C->resort) return;
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s >= C->slots) return;
  const int c = P.s_cell[s];
  if (c < 0) return;
  P.s_key[P.cell_start[c] + P.s_rank[s]] = P.IB[s];
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_sort_place(Params<T> P) {
  pdl_wait();
  const Counters* C = P.ctr;
  if (!C->resort) return;
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s == 0) P.ctr->list_valid = 0;
  if (s >= C->slots) return;
  const int c = P.s_cell[s];
  if (c < 0) return;
  const int key = P.IB[s];
  const int s0 = P.cell_start[c], s1 = P.cell_start[c + 1];
  // rank among the cell's keys (the cells of a dense colony hold a hundred
  // and more): four keys a load between the aligned ends
  int r = 0, q = s0;
  for (const int qa = min(s1, (s0 + 3) & ~3); q < qa; ++q) r += ld(P.s_key + q) < key;
  for (; q + 4 <= s1; q += 4) {
    const int4 k4 = ld(reinterpret_cast<const int4*>(P.s_key + q));
    r += (int)(k4.x < key) + (int)(k4.y < key) + (int)(k4.z < key) + (int)(k4.w < key);
  }
  for (; q < s1; ++q) r += ld(P.s_key + q) < key;
  const int ns = s0 + r;
  const typename V4T<T>::type x = P.PB[s];
  P.PA[ns] = x;
  P.VA[ns] = P.VB[s];
  if (P.force_mode == CBM_FORCE_LAGGED) P.FA[ns] = P.FB[s];
  P.IA[ns] = key;
  P.inv[key] = ns;
  P.cell_of_slot[ns] = c;
  if (is_verlet(P)) P.POLD[ns] = x;  // verletResetDisplacement (neighbors.jl:438-487)
}

// Verlet list of the committed slots over the grid: CLVD in cell order
// (verletNeighborsCLVD, neighbors.jl:1071-1131); VerletDisplacement ascending
// in agent index (verletNeighbors, :92-133).  Entries are slots.
constexpr int kVdSortMax = 256;

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_verlet_list(Params<T> P, int only_if_resorted) {
  if (only_if_resorted && !P.ctr->resort) return;
  const int N = (int)P.ctr->N[P.parity];
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s == 0) P.ctr->list_valid = 1;
  if (s >= N) return;
  T xi[3];
  to3<T>(P.PA[s], xi);
  const int M = P.max_nbrs;
  int n = 0;
  bool over = false;
  walk_cells<T, D>(P, P.PA, xi, P.skin_reach, [&](int q, const typename V4T<T>::type& v) {
    if (q == s) return;
    T xj[3];
    to3<T>(v, xj);
    if (dist<T, D>(xi, xj) < P.skin) {
      if (n < M) P.nbr_list[(size_t)n * P.n_max + s] = q;
      else over = true;
      ++n;
    }
  });
  if (over) atomicOr(&P.ctr->err, kErrNeighborOverflow);
  n = n < M ? n : M;
  if (P.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT && n > 1) {
    // insertion sort of the row by agent index (the O(N^2) reference's order)
    for (int a = 1; a < n; ++a) {
      int keyslot = P.nbr_list[(size_t)a * P.n_max + s];
      int key = P.IA[keyslot];
      int b = a - 1;
      while (b >= 0 && P.IA[P.nbr_list[(size_t)b * P.n_max + s]] > key) {
        P.nbr_list[(size_t)(b + 1) * P.n_max + s] = P.nbr_list[(size_t)b * P.n_max + s];
        --b;
      }
      P.nbr_list[(size_t)(b + 1) * P.n_max + s] = keyslot;
    }
  }
  P.nbr_n[s] = n;
}

// ---------------------------------------------------------------------------
// host exchange and inspection
// ---------------------------------------------------------------------------
// index-ordered staging -> working slots (identity), before the first sort
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_pack_upload(Params<T> P, int N) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  T x[3] = {(T)0, (T)0, (T)0}, f[3] = {(T)0, (T)0, (T)0};
#pragma unroll
  for (int d = 0; d < D; ++d) {
    x[d] = P.hx[d][i];
    f[d] = P.hf[d][i];
  }
  P.PB[i] = from3<T>(x);
  P.FB[i] = from3<T>(f);
  P.VB[i] = P.hv[i];
  P.IB[i] = i;
}

// slot-ordered set (which: 0 committed A, 1 written B, 2 reflected U) ->
// index-ordered staging
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_gather_download(Params<T> P, int N, int which) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  const int s = P.inv[i];
  T x[3], f[3];
  to3<T>(which == 0 ? P.PA[s] : (which == 1 ? P.PB[s] : P.U[s]), x);
  to3<T>(which == 1 ? P.FB[s] : P.FA[s], f);
#pragma unroll
  for (int d = 0; d < D; ++d) {
    P.hx[d][i] = x[d];
    P.hf[d][i] = f[d];
  }
  P.hv[i] = which == 1 ? P.VB[s] : P.VA[s];
}

// committed -> working slots, for an update! without a DE stage
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_copy_ab(Params<T> P, int use_u) {
  const int N = (int)P.ctr->N[P.parity];
  const int s = blockIdx.x * kTile + threadIdx.x;
  if (s >= N) return;
  P.PB[s] = use_u ? P.U[s] : P.PA[s];
  P.VB[s] = P.VA[s];
  P.FB[s] = P.FA[s];
  P.IB[s] = P.IA[s];
}

template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_copy_medium(Params<T> P, int grad_only) {
  int n = blockIdx.x * kTile + threadIdx.x;
  if (n >= P.n_nodes) return;
  if (!grad_only) P.c_nxt[n] = P.c_cur[n];
#pragma unroll
  for (int d = 0; d < D; ++d) P.grad_nxt[d][n] = P.grad_cur[d][n];
}

// the neighbor-counting rule of test/testCommunity.jl:359-415 on committed x
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_count_neighbors(Params<T> P, T radius, int* out) {
  const int N = (int)P.ctr->N[P.parity];
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= N) return;
  const int s = P.inv[i];
  T xi[3];
  to3<T>(P.PA[s], xi);
  int n = 0;
  auto visit = [&](int q) {
    T xj[3];
    to3<T>(P.PA[q], xj);
    if (dist<T, D>(xi, xj) < radius) ++n;
  };
  if (P.neighbors == CBM_NEIGH_FULL) {
    for (int j = 0; j < N; ++j)
      if (j != i) visit(P.inv[j]);
  } else if (P.neighbors == CBM_NEIGH_CELL_LINKED) {
    for_cell_slots<T, D>(P, xi, [&](int q) {
      if (q != s) visit(q);
    });
  } else if (is_verlet(P) && P.ctr->list_valid) {
    const int m = P.nbr_n[s];
    for (int k = 0; k < m; ++k) visit(P.nbr_list[(size_t)k * P.n_max + s]);
  } else if (P.neighbors == CBM_NEIGH_CLVD) {
    for_cell_slots<T, D>(P, xi, [&](int q) {
      if (q == s) return;
      T xj[3];
      to3<T>(P.PA[q], xj);
      if (dist<T, D>(xi, xj) < P.skin) visit(q);
    });
  }
  out[i] = n;
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
