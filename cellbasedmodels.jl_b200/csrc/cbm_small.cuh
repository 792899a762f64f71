// cbm_small.cuh — small CellLinked communities stepped by one launch.
//
// A community of a few thousand agents (the 2D aggregation of 4096 agents)
// costs far less than the launches of its step graph: the graph's seven
// kernels each wait for the previous one to drain.  Here one cooperative
// launch runs all the steps of a cbm_step call.  Its blocks meet at grid
// barriers between the phases of a step:
//
//   DE     agentStepDE! of every slot over the grid of the committed
//          positions (the rule's wall reflection computed on the fly), the
//          same sums in the same order as k_agent_de, into the working set B
//   commit update!'s counters (k_commit), the histogram of the new cells
//   scan   every block scans the cell counts into shared memory (the cell
//          grid of these communities fits one block); block 0 stores the
//          offsets; agent indices are scattered by (cell, arrival)
//   place  the stable placement B -> A by (cell, agent index) of k_sort_place,
//          and the counts are cleared for the next step
//
// so the state after the launch is the one the step graphs leave.  Each
// barrier's wait is bounded: a block that gives up sets the timeout bit and
// an abort flag, and every block leaves at its next barrier.
#pragma once
#include "cbm_kernels.cuh"

namespace cbm {

constexpr int kSmallThreads = 256;
constexpr int kSmallMaxAgents = 32768;  // communities stepped by one launch (fate-free CellLinked)
constexpr int kSmallMaxCells = 8192;    // cell grids a block scans in shared memory
constexpr unsigned kBarrierPolls = 1u << 23;  // polls (about 0.1 us each) before a wait gives up

struct SmallBarrier {
  unsigned* count;  // blocks arrived at the current barrier (0 at launch)
  unsigned* gen;    // barriers passed
  int* abort;       // a wait gave up (0 at launch)
};

// Grid barrier of the cooperative launch.  Returns false when a wait gave up
// (here or in another block); the caller then leaves.
__device__ __forceinline__ bool small_barrier(const SmallBarrier& B, Counters* C) {
  __shared__ int s_go;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned* gen = B.gen;
    volatile int* abort = B.abort;
    const unsigned g = *gen;
    __threadfence();
    if (atomicAdd(B.count, 1u) == gridDim.x - 1) {
      atomicExch(B.count, 0u);
      __threadfence();
      atomicAdd(B.gen, 1u);
    } else {
      unsigned polls = 0;
      while (*gen == g && *abort == 0) {
        if (++polls == kBarrierPolls) {
          atomicOr(&C->err, kErrTimeout);
          atomicExch(B.abort, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    s_go = *abort == 0;
  }
  __syncthreads();
  return s_go != 0;
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

// agentStepDE! of slot s for CellLinked without a queue: the candidates of
// the 3^D cells in the reference's order, each pair term added in that order
// (skipping cells with no partner, as k_agent_de's pruning does, changes no
// sum).  With reflecting walls the rule's reflected positions are computed
// from the committed ones, here for xi and every candidate.
template <typename T, int D>
__device__ __forceinline__ void small_de(const Params<T>& P, int s) {
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
  for_cell_slots<T, D>(P, xi, [&](int q) {
    if (q == s) return;
    T xj[3], e[3];
    pos(q, xj);
    const T s2 = pair_diff<T, D>(xi, xj, e);
    pair_term<T, D>(coef, e, s2, acc);
  });
  finish_agent<T, D>(P, s, xi, acc);
}

// nsteps steps; P0 has the parity of the first step, P1 the other one.
template <typename T, int D>
__global__ void __launch_bounds__(kSmallThreads) k_small_steps(Params<T> P0, Params<T> P1,
                                                               SmallBarrier bar, int nsteps,
                                                               int n_cells) {
  extern __shared__ int s_start[];  // n_cells + 1 offsets of the grid being built
  __shared__ int warp_sums[kSmallThreads / 32];
  const int tid = (int)(blockIdx.x * kSmallThreads + threadIdx.x);
  const int nth = (int)(gridDim.x * kSmallThreads);
  for (int t = 0; t < nsteps; ++t) {
    const Params<T>& P = (t & 1) ? P1 : P0;
    Counters* C = P.ctr;
    const int p = P.parity;
    const int N = (int)C->N[p];
    for (int s = tid; s < N; s += nth) small_de<T, D>(P, s);
    if (!small_barrier(bar, C)) return;
    if (tid == 0) {  // update!'s counters, as k_commit (no births or deaths here)
      C->slots = C->N[p];
      C->N[p ^ 1] = C->N[p];
      C->n_add = 0;
      C->n_remove = 0;
      C->t[p ^ 1] = C->t[p] + P.dt_time;
      C->step[p ^ 1] = C->step[p] + 1;
      C->flag[p ^ 1] = 0;
      C->resort = 1;
      C->events = 0;
      if (C->list_written) C->list_valid = 1;
      C->list_written = 0;
    }
    for (int s = tid; s < N; s += nth) {  // histogram of the new cells (k_sort_hist)
      T x[3];
      to3<T>(P.PB[s], x);
      const int c = cell_of_pos<T, D>(P, x);
      P.s_cell[s] = c;
      P.s_rank[s] = atomicAdd(P.cell_count + c, 1);
    }
    if (!small_barrier(bar, C)) return;
    block_scan_counts(P.cell_count, n_cells, s_start, warp_sums);
    if (blockIdx.x == 0)
      for (int c = threadIdx.x; c <= n_cells; c += kSmallThreads) P.cell_start[c] = s_start[c];
    for (int s = tid; s < N; s += nth) P.s_key[s_start[P.s_cell[s]] + P.s_rank[s]] = P.IB[s];
    if (!small_barrier(bar, C)) return;
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
    if (tid == 0) C->list_valid = 0;
    if (!small_barrier(bar, C)) return;
  }
}

}  // namespace cbm
