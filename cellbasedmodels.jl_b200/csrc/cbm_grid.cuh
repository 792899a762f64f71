// cbm_grid.cuh — the CellLinked grid over agents in index order (agent i at
// position i of the input arrays): counting sort by cell, stable inside a
// cell (src/neighbors.jl:763-979).  Used by the allocation-free entry point;
// the stepping engine sorts its own slot-ordered state (cbm_kernels.cuh).
#pragma once

#include "cbm_common.cuh"

namespace cbm {

template <typename T>
struct GridParams {
  const T* pos[3];       // positions, index order
  int n;                 // agents
  T box_lo[3], box_hi[3];
  T edge;
  int n_cells_d[3];
  int n_cells;
  int n_scan_tiles;
  Counters* ctr;
  int* cell_count;       // zero on entry, zero on exit
  int* cell_start;       // n_cells + 1
  unsigned long long* scan_state;
  int* agent_cell;       // n
  int* agent_rank;       // n (atomic rank inside the cell)
  int* cell_tmp;         // n
  int* cell_agents;      // n (cellAssignedToAgent_)
};

// assignCells (neighbors.jl:763-821)
template <typename T, int D>
__global__ void __launch_bounds__(kTile) k_grid_hist(GridParams<T> G) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i == 0) {
    G.ctr->scan_ticket = 0u;  // fresh tickets and tile-state generation for the scan
    G.ctr->scan_epoch = G.ctr->scan_epoch + 1u;
  }
  if (i >= G.n) return;
  T x[3];
#pragma unroll
  for (int d = 0; d < D; ++d) x[d] = G.pos[d][i];
  int c = cell_of<T, D>(G.edge, G.box_lo, G.box_hi, G.n_cells_d, x);
  G.agent_cell[i] = c;
  G.agent_rank[i] = atomicAdd(G.cell_count + c, 1);
}

// sortAgentsInCells (neighbors.jl:837-899), first pass: scatter by atomic rank
template <typename T>
__global__ void __launch_bounds__(kTile) k_grid_scatter(GridParams<T> G) {
  pdl_wait();
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= G.n) return;
  G.cell_tmp[G.cell_start[G.agent_cell[i]] + G.agent_rank[i]] = i;
}

// second pass: rank among the cell's agents with a smaller index, so agents
// are ascending inside each cell as in the serial CPU reference (:851-862)
template <typename T>
__global__ void __launch_bounds__(kTile) k_grid_stable(GridParams<T> G) {
  pdl_wait();
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= G.n) return;
  const int c = G.agent_cell[i];
  const int s0 = G.cell_start[c], s1 = G.cell_start[c + 1];
  int r = 0;
  for (int s = s0; s < s1; ++s) r += ld(G.cell_tmp + s) < i;
  G.cell_agents[s0 + r] = i;
}

template <typename T>
ScanArgs grid_scan_args(const GridParams<T>& G) {
  ScanArgs A;
  A.count = G.cell_count;
  A.start = G.cell_start;
  A.state = G.scan_state;
  A.n = G.n_cells;
  A.n_tiles = G.n_scan_tiles;
  A.ctr = G.ctr;
  A.due = nullptr;
  return A;
}

}  // namespace cbm
