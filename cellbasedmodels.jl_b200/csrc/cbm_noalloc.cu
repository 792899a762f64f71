// cbm_noalloc.cu — cbm_cell_grid_noalloc: the counting-sort cell grid built
// without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need a
// grid: code that runs while a framework is capturing the stream into a CUDA
// graph (cudaMalloc is refused in a thread whose stream is being captured in
// global or thread-local mode), hosts whose device memory is owned by a pool
// allocator that must see every byte (for instance a Julia process whose
// CUDA.jl pool holds the GPU), and real-time loops that cannot take the
// latency of cudaMalloc/cudaFree.  They pass device pointers for the
// positions and the three output arrays; the scratch memory lives in the
// file-scope array below.
#include <cuda_runtime.h>

#include <cstddef>
#include <mutex>
#include <string>

#include "../../include/cbm_b200.h"
#include "cbm_grid.cuh"

using namespace cbm;

namespace {

// Scratch layout inside g_noalloc_scratch (bytes):
//   Counters | cell_count[MAX_CELLS] | agent_rank[MAX_AGENTS] |
//   cell_tmp[MAX_AGENTS] | scan_state[MAX_SCAN_TILES]
constexpr size_t kCtrBytes = 256;
constexpr size_t kMaxScanTiles = (CBM_NOALLOC_MAX_CELLS + kScanTile - 1) / kScanTile;
constexpr size_t kCountOff = kCtrBytes;
constexpr size_t kRankOff = kCountOff + (size_t)CBM_NOALLOC_MAX_CELLS * 4;
constexpr size_t kTmpOff = kRankOff + (size_t)CBM_NOALLOC_MAX_AGENTS * 4;
constexpr size_t kScanOff = kTmpOff + (size_t)CBM_NOALLOC_MAX_AGENTS * 4;
constexpr size_t kScratchBytes = kScanOff + kMaxScanTiles * 8;
static_assert(sizeof(Counters) <= kCtrBytes, "counter block does not fit");

// Every GPU that loads the library holds this array until the process exits.
// All calls share it and it keeps the last call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_ptr[kMaxDevices] = {};
// The last argument error of this host thread: each thread reads the
// message of its own failed call, and no two threads share the string.
thread_local std::string g_noalloc_error;

int nfail(int code, const char* msg) {
  g_noalloc_error = msg;
  return code;
}

// One-thread set-up of the counter block for this call: agent count, fresh
// scan tickets; everything a call needs zeroed is cleared here or by memset.
__global__ void k_noalloc_setup(Counters* ctr, int n) {
  ctr->N[0] = n;
  ctr->N[1] = n;
  ctr->flag[0] = ctr->flag[1] = 1;
  ctr->err = 0;
  ctr->scan_ticket = 0u;
}

template <typename T, int D>
void launch(const void* const* pos, int n, const double* lo, const double* hi, double edge,
            const int* ncd, int n_cells, int32_t* agent_cell, int32_t* cell_start,
            int32_t* cell_agents, unsigned char* base, cudaStream_t st) {
  GridParams<T> G;
  memset(&G, 0, sizeof G);
  for (int d = 0; d < 3; ++d) {
    G.pos[d] = d < D ? (const T*)pos[d] : nullptr;
    G.box_lo[d] = (T)lo[d];
    G.box_hi[d] = (T)hi[d];
    G.n_cells_d[d] = ncd[d];
  }
  G.n = n;
  G.edge = (T)edge;
  G.n_cells = n_cells;
  G.n_scan_tiles = (n_cells + kScanTile - 1) / kScanTile;
  G.ctr = (Counters*)base;
  G.cell_count = (int*)(base + kCountOff);
  G.agent_rank = (int*)(base + kRankOff);
  G.cell_tmp = (int*)(base + kTmpOff);
  G.scan_state = (unsigned long long*)(base + kScanOff);
  G.agent_cell = agent_cell;
  G.cell_start = cell_start;
  G.cell_agents = cell_agents;
  const int nb = n > 0 ? (n + kTile - 1) / kTile : 1;
  k_noalloc_setup<<<1, 1, 0, st>>>(G.ctr, n);
  cudaMemsetAsync(G.cell_count, 0, (size_t)n_cells * 4, st);
  k_grid_hist<T, D><<<nb, kTile, 0, st>>>(G);
  k_scan_cells<<<G.n_scan_tiles, kTile, 0, st>>>(grid_scan_args(G));
  k_grid_scatter<T><<<nb, kTile, 0, st>>>(G);
  k_grid_stable<T><<<nb, kTile, 0, st>>>(G);
}

}  // namespace

extern "C" const char* cbm_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

extern "C" int cbm_noalloc_status(void* stream) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return nfail(CBM_ERR_CUDA, "no usable CUDA device");
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) return CBM_OK;  // no call has run on this device
  }
  // The error bits of the counter block in the static array, read after the
  // work queued on `stream` (the last call's launches included) has finished.
  int err = 0;
  cudaError_t e = cudaMemcpyFromSymbolAsync(&err, g_noalloc_scratch, sizeof err,
                                            offsetof(Counters, err), cudaMemcpyDeviceToHost,
                                            (cudaStream_t)stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize((cudaStream_t)stream);
  if (e != cudaSuccess) return nfail(CBM_ERR_CUDA, cudaGetErrorString(e));
  if (err & kErrTimeout)
    return nfail(CBM_ERR_TIMEOUT,
                 "the cell scan's bounded wait gave up: cell_start and cell_agents are incomplete");
  return CBM_OK;
}

extern "C" int cbm_cell_grid_noalloc(const void* x, const void* y, const void* z, int32_t n_agents,
                                     int32_t dims, int32_t precision, const double* box_lo,
                                     const double* box_hi, double cell_edge, int32_t* agent_cell,
                                     int32_t* cell_start, int32_t* cell_agents, void* stream) {
  if (dims < 1 || dims > 3) return nfail(CBM_ERR_ARG, "dims must be 1, 2 or 3");
  if (precision != CBM_F32 && precision != CBM_F64)
    return nfail(CBM_ERR_ARG, "precision must be CBM_F32 or CBM_F64");
  if (!box_lo || !box_hi || !(cell_edge > 0)) return nfail(CBM_ERR_ARG, "bad box or cell_edge");
  if (n_agents < 0 || n_agents > CBM_NOALLOC_MAX_AGENTS)
    return nfail(CBM_ERR_ARG,
                 "n_agents exceeds CBM_NOALLOC_MAX_AGENTS (524288) of the static scratch array");
  const void* pos[3] = {x, y, z};
  int ncd[3] = {1, 1, 1};
  long long nc = 1;
  for (int d = 0; d < dims; ++d) {
    if (!(box_hi[d] > box_lo[d])) return nfail(CBM_ERR_ARG, "empty box");
    double v = ceil((box_hi[d] - box_lo[d]) / cell_edge + 2.0);  // nCells_, neighbors.jl:605
    if (!(v >= 1 && v <= (double)CBM_NOALLOC_MAX_CELLS))
      return nfail(CBM_ERR_ARG, "cell grid exceeds CBM_NOALLOC_MAX_CELLS (1048576)");
    ncd[d] = (int)v;
    nc *= (long long)v;
  }
  if (nc > CBM_NOALLOC_MAX_CELLS)
    return nfail(CBM_ERR_ARG, "cell grid exceeds CBM_NOALLOC_MAX_CELLS (1048576)");
  for (int d = 0; d < dims; ++d)
    if (n_agents && !pos[d]) return nfail(CBM_ERR_ARG, "a position array is NULL");
  if (!cell_start || (n_agents && (!agent_cell || !cell_agents)))
    return nfail(CBM_ERR_ARG, "an output array is NULL");

  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices)
    return nfail(CBM_ERR_CUDA, "no usable CUDA device");
  void* base = nullptr;
  {
    // set-up, once per device, with that device current: the host-side name
    // of the array is not a device address, so fetch the real one
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_ptr[dev]) {
      cudaError_t e = cudaGetSymbolAddress(&g_scratch_ptr[dev], g_noalloc_scratch);
      if (e != cudaSuccess) {
        g_scratch_ptr[dev] = nullptr;
        return nfail(CBM_ERR_CUDA, cudaGetErrorString(e));
      }
    }
    base = g_scratch_ptr[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* b = (unsigned char*)base;
  if (precision == CBM_F64) {
    if (dims == 1) launch<double, 1>(pos, n_agents, box_lo, box_hi, cell_edge, ncd, (int)nc, agent_cell, cell_start, cell_agents, b, st);
    else if (dims == 2) launch<double, 2>(pos, n_agents, box_lo, box_hi, cell_edge, ncd, (int)nc, agent_cell, cell_start, cell_agents, b, st);
    else launch<double, 3>(pos, n_agents, box_lo, box_hi, cell_edge, ncd, (int)nc, agent_cell, cell_start, cell_agents, b, st);
  } else {
    if (dims == 1) launch<float, 1>(pos, n_agents, box_lo, box_hi, cell_edge, ncd, (int)nc, agent_cell, cell_start, cell_agents, b, st);
    else if (dims == 2) launch<float, 2>(pos, n_agents, box_lo, box_hi, cell_edge, ncd, (int)nc, agent_cell, cell_start, cell_agents, b, st);
    else launch<float, 3>(pos, n_agents, box_lo, box_hi, cell_edge, ncd, (int)nc, agent_cell, cell_start, cell_agents, b, st);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return nfail(CBM_ERR_CUDA, cudaGetErrorString(e));
  return CBM_OK;
}
