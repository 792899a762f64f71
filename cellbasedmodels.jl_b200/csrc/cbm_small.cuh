// cbm_small.cuh — small CellLinked communities stepped by one launch.
//
// A community of a few thousand agents (the 2D aggregation of 4096 agents)
// costs far less than the launches of its step graph: the graph's seven
// kernels each wait for the previous one to drain.  Here one launch of a
// single thread-block cluster (up to 16 blocks of 1024 threads, scheduled
// together on one GPC) runs all the steps of a cbm_step call.  Its blocks
// meet at three hardware cluster barriers a step (barrier.cluster with
// release / acquire), between the phases:
//
//   DE     agentStepDE! of every slot over the grid of the committed
//          positions (the rule's wall reflection computed on the fly), four
//          lanes an agent, the same sums in the same order as k_agent_de,
//          into the working set B; then the histogram of the new cells
//   scan   update!'s counters (k_commit); every block scans the cell counts
//          into shared memory (the cell grid of these communities fits one
//          block), block 0 stores the offsets, and agent indices are
//          scattered by (cell, arrival)
//   place  the stable placement B -> A by (cell, agent index) of
//          k_sort_place, and the counts are cleared for the next step
//
// The state after the launch is the one the step graphs leave.  Every block
// takes every barrier (the loops are uniform), so no wait depends on a
// condition that could fail to arrive.
#pragma once
#include "cbm_kernels.cuh"

namespace cbm {

constexpr int kSmallThreads = 1024;
constexpr int kSmallMaxBlocks = 16;     // blocks of the cluster (16 needs the non-portable size)
constexpr int kSmallMaxAgents = 32768;  // communities stepped by one launch (fate-free CellLinked)
constexpr int kSmallMaxCells = 8192;    // cell grids a block scans in shared memory

// Barrier of the cluster's blocks: every thread arrives with release and
// waits with acquire, so the global writes before it are visible after it.
__device__ __forceinline__ void cluster_barrier() {
  asm volatile(
      "barrier.cluster.arrive.release;\n\t"
      "barrier.cluster.wait.acquire;" ::: "memory");
}

// Exclusive scan of counts[0, n) by one block into out[0, n]; out[n] = total.
__device__ __forceinline__ void block_scan_counts(const int* counts, int n, int* out,
                                                  int* warp_sums) {
  const int per = (n + kSmallThreads - 1) / kSmallThreads;
  const int c0 = min(n, (int)threadIdx.x * per), c1 = min(n, c0 + per);
  int local = 0;
  for (int c = c0; c < c1; ++c) {
    const int v = counts[c];
    out[c] = v;
    local += v;
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[w] = x;
  __syncthreads();
  if (w == 0) {
    int v = lane < kSmallThreads / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(kFull, v, o);
      if (lane >= o) v += y;
    }
    if (lane < kSmallThreads / 32) warp_sums[lane] = v;
  }
  __syncthreads();
  int run = (w > 0 ? warp_sums[w - 1] : 0) + x - local;
  for (int c = c0; c < c1; ++c) {
    const int v = out[c];
    out[c] = run;
    run += v;
  }
  if (threadIdx.x == kSmallThreads - 1) out[n] = warp_sums[kSmallThreads / 32 - 1];
  __syncthreads();
}

// agentStepDE! of slot s for CellLinked, by the kSmallLanes lanes of a group
// (lane gl of the group takes candidates gl, gl + kSmallLanes, ... of each
// run): the candidates of the 3^D cells in the reference's order, the pair
// terms of each chunk added in candidate order through the group's shuffles,
// so the sums are those of k_agent_de (skipping cells with no partner, as its
// pruning does, changes no sum).  With reflecting walls the rule's reflected
// positions are computed from the committed ones, here for xi and every
// candidate.  The group's first lane integrates.
constexpr int kSmallLanes = 4;

template <typename T, int D>
__device__ __forceinline__ void small_de(const Params<T>& P, int s) {
  constexpr int L = kSmallLanes;
  const int lane = threadIdx.x & 31, gl = lane & (L - 1);
  const unsigned gmask = ((1u << L) - 1u) << (lane & ~(L - 1));
  const bool reflect = P.walls == CBM_WALLS_REFLECT;
  auto pos = [&](int q, T* x) {
    to3<T>(P.PA[q], x);
    if (reflect) {
#pragma unroll
      for (int d = 0; d < D; ++d) {
        if (x[d] < P.box_lo[d]) x[d] = (T)2 * P.box_lo[d] - x[d];
        else if (x[d] > P.box_hi[d]) x[d] = (T)2 * P.box_hi[d] - x[d];
      }
    }
  };
  T xi[3] = {(T)0, (T)0, (T)0};
  pos(s, xi);
  T acc[3] = {(T)0, (T)0, (T)0};
  const PairCoef<T> coef = pair_coef<T>(P);
  int q3[3] = {0, 0, 0};
  cell_coords<D>(P.n_cells_d, cell_of_pos<T, D>(P, xi), q3);
  const int nx = P.n_cells_d[0];
  const int x0 = q3[0] > 0 ? q3[0] - 1 : 0, x1 = q3[0] < nx - 1 ? q3[0] + 1 : nx - 1;
  constexpr int ny_rows = D > 1 ? 3 : 1, nz_rows = D > 2 ? 3 : 1;
  for (int dz = 0; dz < nz_rows; ++dz) {
    const int pz = D > 2 ? q3[2] + dz - 1 : 0;
    if (D > 2 && (pz < 0 || pz >= P.n_cells_d[2])) continue;
    for (int dy = 0; dy < ny_rows; ++dy) {
      const int py = D > 1 ? q3[1] + dy - 1 : 0;
      if (D > 1 && (py < 0 || py >= P.n_cells_d[1])) continue;
      const int row = nx * (py + P.n_cells_d[1] * pz);
      const int s0 = ld(P.cell_start + row + x0), s1 = ld(P.cell_start + row + x1 + 1);
      for (int base = s0; base < s1; base += L) {
        const int q = base + gl;
        bool has = false;
        T t[3] = {(T)0, (T)0, (T)0};
        if (q < s1 && q != s) {
          T xj[3], e[3];
          pos(q, xj);
          const T s2 = pair_diff<T, D>(xi, xj, e);
          if (s2 < coef.cut2) {
            const T dd = sqrt(s2);
            T F = (T)0;
            if (dd < coef.rrep) {
              F = coef.krep * (coef.rrep - dd);
              has = true;
            } else if (dd < coef.ratt) {
              F = coef.from_rep ? -(coef.katt * (dd - coef.rrep)) : -(coef.katt * (coef.ratt - dd));
              has = true;
            }
            if (has) {
              const T sc = F / dd;
#pragma unroll
              for (int d = 0; d < D; ++d) t[d] = sc * e[d];
            }
          }
        }
        // the chunk's terms, added in candidate order by every lane of the group
#pragma unroll
        for (int u = 0; u < L; ++u) {
          const bool hu = __shfl_sync(gmask, has ? 1 : 0, u, L) != 0;
          T tu[3];
#pragma unroll
          for (int d = 0; d < D; ++d) tu[d] = __shfl_sync(gmask, t[d], u, L);
          if (hu) {
#pragma unroll
            for (int d = 0; d < D; ++d) acc[d] = acc[d] + tu[d];
          }
        }
      }
    }
  }
  if (gl == 0) finish_agent<T, D>(P, s, xi, acc);
}

// nsteps steps; P0 has the parity of the first step, P1 the other one.  The
// counts of the histogram are complete after the first barrier.  The
// counters' commit is made by the cluster's last thread in the placement
// phase (no thread reads those counters before the next step) so that it
// stays off the scan's path.
template <typename T, int D>
__global__ void __launch_bounds__(kSmallThreads) k_small_steps(Params<T> P0, Params<T> P1,
                                                               int nsteps, int n_cells) {
  extern __shared__ int s_start[];  // n_cells + 1 offsets of the grid being built
  __shared__ int warp_sums[kSmallThreads / 32];
  const int tid = (int)(blockIdx.x * kSmallThreads + threadIdx.x);
  const int nth = (int)(gridDim.x * kSmallThreads);
  for (int t = 0; t < nsteps; ++t) {
    const Params<T>& P = (t & 1) ? P1 : P0;
    Counters* C = P.ctr;
    const int p = P.parity;
    const int N = (int)C->N[p];
    // DE, kSmallLanes lanes an agent; the histogram of the new cells follows
    // in the same phase (the agent's own written position is all it reads).
    // Slots are dealt to the blocks in turn (slot s to block s mod blocks),
    // so every block holds agents from all over the community and the dense
    // clumps do not all fall to the same block.
    const int groups = kSmallThreads / kSmallLanes;
    for (int s = (int)(threadIdx.x / kSmallLanes) * (int)gridDim.x + (int)blockIdx.x; s < N;
         s += groups * (int)gridDim.x) {
      small_de<T, D>(P, s);
      if ((threadIdx.x & (kSmallLanes - 1)) == 0) {  // k_sort_hist
        T x[3];
        to3<T>(P.PB[s], x);
        const int c = cell_of_pos<T, D>(P, x);
        P.s_cell[s] = c;
        P.s_rank[s] = atomicAdd(P.cell_count + c, 1);
      }
    }
    cluster_barrier();
    block_scan_counts(P.cell_count, n_cells, s_start, warp_sums);
    if (blockIdx.x == 0)
      for (int c = threadIdx.x; c <= n_cells; c += kSmallThreads) P.cell_start[c] = s_start[c];
    for (int s = tid; s < N; s += nth) P.s_key[s_start[P.s_cell[s]] + P.s_rank[s]] = P.IB[s];
    cluster_barrier();
    for (int s = tid; s < N; s += nth) {  // stable placement by agent index (k_sort_place)
      const int c = P.s_cell[s];
      const int key = P.IB[s];
      const int s0 = s_start[c], s1 = s_start[c + 1];
      int r = 0;
      for (int q = s0; q < s1; ++q) r += P.s_key[q] < key;
      const int ns = s0 + r;
      P.PA[ns] = P.PB[s];
      P.VA[ns] = P.VB[s];
      P.IA[ns] = key;
      P.inv[key] = ns;
      P.cell_of_slot[ns] = c;
    }
    for (int c = tid; c < n_cells; c += nth) P.cell_count[c] = 0;
    if (tid == nth - 1) {  // update!'s counters, as k_commit (no births or deaths here)
      C->slots = C->N[p];
      C->N[p ^ 1] = C->N[p];
      C->n_add = 0;
      C->n_remove = 0;
      C->t[p ^ 1] = C->t[p] + P.dt_time;
      C->step[p ^ 1] = C->step[p] + 1;
      C->flag[p ^ 1] = 0;
      C->resort = 1;
      C->events = 0;
      C->list_written = 0;
      C->list_valid = 0;  // the grid was rebuilt (computeNeighbors!)
    }
    cluster_barrier();
  }
}

}  // namespace cbm
