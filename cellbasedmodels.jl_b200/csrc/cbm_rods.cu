// cbm_rods.cu — the rods2D model (src/models/rods.jl) on the device.
//
// One step, as step! runs rods2D with the Euler integrator:
//   1. agentStepDE!: every rod sums rodForces over its neighbors (the
//      CellLinked grid of the committed positions, 9 cells x fastest, rods
//      ascending inside a cell; or all rods) into the new copies fx__, fy__,
//      W__, pressure__, then u += du dt with du from the committed (lagged)
//      fx, fy, W (k_rod_forces, then k_rod_update);
//   2. update!: the new copies are committed (k_rod_update);
//   3. computeNeighbors!: the grid is rebuilt on the new positions
//      (the stable counting sort of cbm_grid.cuh).
// Rods stay in index order (no division or death in rods2D).  The force
// arithmetic is cbm_rods_math.h.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>

#include "../../include/cbm_b200.h"
#include "../../include/cbm_rods_math.h"
#include "cbm_grid.cuh"

using namespace cbm;

namespace {

template <typename T>
struct RodParams {
  T* f[CBM_RODS_FIELDS];     // committed fields, index order
  T* fnew[4];                // fx__, fy__, W__, pressure__
  T* cs[2];                  // cos, sin of theta
  const int* cell_start;     // n_cells + 1
  const int* cell_agents;
  int n;
  int full;                  // all pairs instead of the grid
  T box_lo[2], box_hi[2], edge;
  int n_cells_d[3];
  T dt, beta, beta_w;
  CbmRodCoef<T> k;
};

template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_geom(RodParams<T> R) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= R.n) return;
  T c, s;
  cbm_rod_cossin<T>(R.f[CBM_ROD_THETA][i], &c, &s);
  R.cs[0][i] = c;
  R.cs[1][i] = s;
}

// the neighbor sum of rod i (@loopOverNeighbors with rodForces, rods.jl:94-111)
template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_forces(RodParams<T> R) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= R.n) return;
  const CbmRodGeom<T> a{R.f[CBM_ROD_X][i], R.f[CBM_ROD_Y][i], R.cs[0][i], R.cs[1][i],
                        R.f[CBM_ROD_L][i]};
  const T d1 = R.f[CBM_ROD_D][i], m1 = R.f[CBM_ROD_M][i];
  const T vx1 = R.f[CBM_ROD_VX][i], vy1 = R.f[CBM_ROD_VY][i];
  T fx = (T)0, fy = (T)0, w = (T)0, p = (T)0;
  auto pair = [&](int j) {
    if (j == i) return;
    const CbmRodGeom<T> b{R.f[CBM_ROD_X][j], R.f[CBM_ROD_Y][j], R.cs[0][j], R.cs[1][j],
                          R.f[CBM_ROD_L][j]};
    T gx, gy, gw;
    if (!cbm_rod_forces<T>(a, d1, vx1, vy1, m1, b, R.f[CBM_ROD_D][j], R.f[CBM_ROD_VX][j],
                           R.f[CBM_ROD_VY][j], R.k, &gx, &gy, &gw))
      return;
    fx = fx + gx;
    fy = fy + gy;
    w = w + gw;
    p = p + sqrt(gx * gx + gy * gy);
  };
  if (R.full) {
    for (int j = 0; j < R.n; ++j) pair(j);
  } else {
    const T x[2] = {a.x, a.y};
    const int c = cell_of<T, 2>(R.edge, R.box_lo, R.box_hi, R.n_cells_d, x);
    const int nx = R.n_cells_d[0], ny = R.n_cells_d[1];
    const int qx = c % nx, qy = c / nx;
    for (int dy = -1; dy <= 1; ++dy) {
      const int py = qy + dy;
      if (py < 0 || py >= ny) continue;
      for (int dx = -1; dx <= 1; ++dx) {
        const int px = qx + dx;
        if (px < 0 || px >= nx) continue;
        const int cell = px + nx * py;
        const int s1 = R.cell_start[cell + 1];
        for (int s = R.cell_start[cell]; s < s1; ++s) pair(R.cell_agents[s]);
      }
    }
  }
  R.fnew[0][i] = fx;
  R.fnew[1][i] = fy;
  R.fnew[2][i] = w;
  R.fnew[3][i] = p;
}

// Euler over the ODE of rods2D (rods.jl:113-118) with the committed forces,
// then update!: the new copies become the committed fx, fy, W, pressure
template <typename T>
__global__ void __launch_bounds__(kTile) k_rod_update(RodParams<T> R) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i >= R.n) return;
  const T dt = R.dt;
  const T x = R.f[CBM_ROD_X][i], y = R.f[CBM_ROD_Y][i];
  const T vx = R.f[CBM_ROD_VX][i], vy = R.f[CBM_ROD_VY][i];
  const T th = R.f[CBM_ROD_THETA][i], om = R.f[CBM_ROD_OMEGA][i];
  const T d = R.f[CBM_ROD_D][i], l = R.f[CBM_ROD_L][i], m = R.f[CBM_ROD_M][i];
  const T dvx = -R.beta * vx + R.f[CBM_ROD_FX][i] / m;
  const T dvy = -R.beta * vy + R.f[CBM_ROD_FY][i] / m;
  const T den = (m * ((d + l) * (d + l))) / (T)12 + m * (d * d);
  const T dom = R.f[CBM_ROD_W][i] / den - R.beta_w * om;
  R.f[CBM_ROD_X][i] = x + vx * dt;
  R.f[CBM_ROD_Y][i] = y + vy * dt;
  R.f[CBM_ROD_VX][i] = vx + dvx * dt;
  R.f[CBM_ROD_VY][i] = vy + dvy * dt;
  R.f[CBM_ROD_THETA][i] = th + om * dt;
  R.f[CBM_ROD_OMEGA][i] = om + dom * dt;
  R.f[CBM_ROD_FX][i] = R.fnew[0][i];
  R.f[CBM_ROD_FY][i] = R.fnew[1][i];
  R.f[CBM_ROD_W][i] = R.fnew[2][i];
  R.f[CBM_ROD_PRESSURE][i] = R.fnew[3][i];
}

}  // namespace

struct cbm_rods {
  cbm_rods_config cfg{};
  int tsize = 4;
  cudaStream_t stream = nullptr;
  int n = 0;
  void* f[CBM_RODS_FIELDS] = {};
  void* fnew[4] = {};
  void* cs[2] = {};
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

void rfree(cbm_rods* r) {
  for (void*& p : r->f)
    if (p) cudaFree(p), p = nullptr;
  for (void*& p : r->fnew)
    if (p) cudaFree(p), p = nullptr;
  for (void*& p : r->cs)
    if (p) cudaFree(p), p = nullptr;
  for (void* p : {(void*)r->ctr, (void*)r->cell_count, (void*)r->cell_start, (void*)r->agent_cell,
                  (void*)r->agent_rank, (void*)r->cell_tmp, (void*)r->cell_agents,
                  (void*)r->scan_state})
    if (p) cudaFree(p);
  r->ctr = nullptr;
  if (r->stream) cudaStreamDestroy(r->stream);
  r->stream = nullptr;
}

template <typename T>
RodParams<T> rod_params(const cbm_rods* r) {
  RodParams<T> R;
  memset(&R, 0, sizeof R);
  const cbm_rods_config& k = r->cfg;
  for (int q = 0; q < CBM_RODS_FIELDS; ++q) R.f[q] = (T*)r->f[q];
  for (int q = 0; q < 4; ++q) R.fnew[q] = (T*)r->fnew[q];
  R.cs[0] = (T*)r->cs[0];
  R.cs[1] = (T*)r->cs[1];
  R.cell_start = r->cell_start;
  R.cell_agents = r->cell_agents;
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
  return R;
}

// computeNeighbors!: the CellLinked grid of the committed positions
template <typename T>
void enqueue_grid(cbm_rods* r) {
  if (r->cfg.neighbors != CBM_NEIGH_CELL_LINKED) return;
  GridParams<T> G;
  memset(&G, 0, sizeof G);
  G.pos[0] = (const T*)r->f[CBM_ROD_X];
  G.pos[1] = (const T*)r->f[CBM_ROD_Y];
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
  const unsigned nb = (unsigned)(r->n > 0 ? (r->n + kTile - 1) / kTile : 1);
  cudaMemsetAsync(G.cell_count, 0, (size_t)r->n_cells * 4, r->stream);
  k_grid_hist<T, 2><<<nb, kTile, 0, r->stream>>>(G);
  k_scan_cells<<<G.n_scan_tiles, kTile, 0, r->stream>>>(grid_scan_args(G));
  k_grid_scatter<T><<<nb, kTile, 0, r->stream>>>(G);
  k_grid_stable<T><<<nb, kTile, 0, r->stream>>>(G);
}

template <typename T>
int enqueue_rod_step(cbm_rods* r) {
  const RodParams<T> R = rod_params<T>(r);
  const unsigned nb = (unsigned)(r->n > 0 ? (r->n + kTile - 1) / kTile : 1);
  k_rod_geom<T><<<nb, kTile, 0, r->stream>>>(R);
  k_rod_forces<T><<<nb, kTile, 0, r->stream>>>(R);
  k_rod_update<T><<<nb, kTile, 0, r->stream>>>(R);
  enqueue_grid<T>(r);
  ROD_TRY(r, cudaGetLastError());
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
  if (k.n_max < 1 || k.n_max >= (1ll << 30)) return rfail(nullptr, CBM_ERR_ARG, "n_max must be in [1, 2^30)");
  if (!(k.dt > 0)) return rfail(nullptr, CBM_ERR_ARG, "dt must be positive");
  for (int d = 0; d < 2; ++d)
    if (!(k.box_hi[d] > k.box_lo[d])) return rfail(nullptr, CBM_ERR_ARG, "empty simBox");
  cbm_rods* r = new cbm_rods;
  r->cfg = k;
  r->tsize = k.precision == CBM_F64 ? 8 : 4;
  if (k.neighbors == CBM_NEIGH_CELL_LINKED) {
    if (!(k.cell_edge > 0)) {
      delete r;
      return rfail(nullptr, CBM_ERR_ARG, "cell_edge must be positive");
    }
    long long nc = 1;
    for (int d = 0; d < 2; ++d) {
      // nCells_ = ceil((hi - lo) / edge + 2), neighbors.jl:605
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
  for (int q = 0; q < CBM_RODS_FIELDS; ++q) ok = ok && cudaMalloc(&r->f[q], n * S) == cudaSuccess;
  for (int q = 0; q < 4; ++q) ok = ok && cudaMalloc(&r->fnew[q], n * S) == cudaSuccess;
  for (int q = 0; q < 2; ++q) ok = ok && cudaMalloc(&r->cs[q], n * S) == cudaSuccess;
  const int tiles = (r->n_cells + kScanTile - 1) / kScanTile;
  ok = ok && cudaMalloc((void**)&r->ctr, sizeof(Counters)) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_count, (size_t)r->n_cells * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_start, ((size_t)r->n_cells + 1) * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->agent_cell, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->agent_rank, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_tmp, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->cell_agents, n * 4) == cudaSuccess;
  ok = ok && cudaMalloc((void**)&r->scan_state, (size_t)tiles * 8) == cudaSuccess;
  ok = ok && cudaMemsetAsync(r->ctr, 0, sizeof(Counters), r->stream) == cudaSuccess;
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
  r->n = (int)n;
  const size_t b = (size_t)n * r->tsize;
  for (int q = 0; q < CBM_ROD_PRESSURE; ++q)
    if (b) ROD_TRY(r, cudaMemcpyAsync(r->f[q], fields[q], b, cudaMemcpyHostToDevice, r->stream));
  if (b) ROD_TRY(r, cudaMemsetAsync(r->f[CBM_ROD_PRESSURE], 0, b, r->stream));
  if (r->tsize == 8) enqueue_grid<double>(r);
  else enqueue_grid<float>(r);
  ROD_TRY(r, cudaGetLastError());
  ROD_TRY(r, cudaStreamSynchronize(r->stream));
  r->loaded = true;
  return CBM_OK;
}

int cbm_rods_step(cbm_rods* r, int32_t nsteps, int32_t flags) {
  if (!r) return rfail(r, CBM_ERR_ARG, "null rods");
  if (!r->loaded) return rfail(r, CBM_ERR_STATE, "cbm_rods_step before cbm_rods_upload");
  if (nsteps < 0) return rfail(r, CBM_ERR_ARG, "nsteps must be >= 0");
  for (int s = 0; s < nsteps; ++s) {
    const int rc = r->tsize == 8 ? enqueue_rod_step<double>(r) : enqueue_rod_step<float>(r);
    if (rc != CBM_OK) return rc;
  }
  if (flags & CBM_SYNC) ROD_TRY(r, cudaStreamSynchronize(r->stream));
  return CBM_OK;
}

int cbm_rods_download(cbm_rods* r, void* const* fields, int64_t* n_out) {
  if (!r || !fields) return rfail(r, CBM_ERR_ARG, "null argument");
  if (!r->loaded) return rfail(r, CBM_ERR_STATE, "cbm_rods_download before cbm_rods_upload");
  const size_t b = (size_t)r->n * r->tsize;
  for (int q = 0; q < CBM_RODS_FIELDS; ++q)
    if (fields[q] && b)
      ROD_TRY(r, cudaMemcpyAsync(fields[q], r->f[q], b, cudaMemcpyDeviceToHost, r->stream));
  ROD_TRY(r, cudaStreamSynchronize(r->stream));
  if (n_out) *n_out = r->n;
  return CBM_OK;
}

void* cbm_rods_stream(cbm_rods* r) { return r ? (void*)r->stream : nullptr; }

}  // extern "C"
