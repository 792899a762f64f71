// cbm_batch.cu — many independent communities advanced by one persistent
// kernel (the parameter-sweep / model-fitting workload: the reference's
// fitting drivers run one whole simulation per parameter set,
// src/fitting/gridSearch.jl:19-65, and its README notes there is no
// batching, README.md:63).
//
// Each community is a 3D soft-sphere Community with Euler–Maruyama noise and
// CLVD neighbors (cell grid + Verlet list rebuilt when a displacement reaches
// the threshold, src/neighbors.jl:997-1275), Float32.  One CTA owns one
// community at a time and runs all requested steps of it with CTA barriers
// only; communities are taken from a work queue in descending size (longest
// processing time first), so the launch is persistent and load-balanced.
// A community's trajectory is bit-identical to the plain path (cbm_create
// with the same parameters and `community` index): same list order (cells x
// fastest, ascending index inside a cell), same expression order, same
// counter-based noise keyed by the community index.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/cbm_b200.h"
#include "cbm_common.cuh"

using namespace cbm;

namespace {

struct Comm {
  int n;                // agents
  int n_cells;
  int nc[3];
  float lo[3], hi[3];
  float k_rep, r_rep, k_att, r_att, sigma;
  float cut2;           // squared-cutoff bound (see bound2 in cbm_api.cu)
  long long off;        // agent offset
  long long cell_off;   // cell offset (n_cells + 1 entries per community)
  uint32_t community;   // index in the random stream
  int pad;
};

struct BatchParams {
  const Comm* comms;
  const int* order;     // communities by descending size
  int n_comm;
  int* head;            // work-queue head
  float4* P[2];         // positions, ping-pong by per-community parity
  float4* pold;
  int* parity;          // per community: which P holds the current positions
  int* rebuild;         // per community: the next step starts with a rebuild
  long long* step;      // per community step counter
  int* cell_count;
  int* cell_start;
  int* agent_cell;
  int* agent_rank;
  int* tmp;
  int* cell_agents;
  int* nbr_n;
  int* nbr_list;        // per community: entry k of agent i at off*M + k*n + i
  int max_nbrs;
  float dt, sqrt_dt;
  float edge, skin, skin2, skin2_lo, thr;
  uint64_t seed;
  int* err;
};

__device__ __forceinline__ void f4to3(const float4& v, float* x) {
  x[0] = v.x;
  x[1] = v.y;
  x[2] = v.z;
}

// CTA-wide exclusive scan of one int per thread
template <int NT>
__device__ __forceinline__ int cta_exscan(int v, int* warp_sums, int* total) {
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
    int s = lane < NT / 32 ? warp_sums[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(kFull, s, o);
      if (lane >= o) s += y;
    }
    if (lane < NT / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  int prefix = w > 0 ? warp_sums[w - 1] : 0;
  *total = warp_sums[NT / 32 - 1];
  __syncthreads();
  return prefix + x - v;
}

// Grid (counting sort, stable inside a cell) and CLVD list of one community
// from positions X (neighbors.jl:918-979,1071-1131).
template <int NT>
__device__ void cta_rebuild(const BatchParams& B, const Comm& C, const float4* X, int* warp_sums) {
  const int n = C.n, tid = threadIdx.x;
  int* count = B.cell_count + C.cell_off;
  int* start = B.cell_start + C.cell_off;
  int* acell = B.agent_cell + C.off;
  int* arank = B.agent_rank + C.off;
  int* tmp = B.tmp + C.off;
  int* cagents = B.cell_agents + C.off;
  for (int i = tid; i < n; i += NT) {
    float x[3];
    f4to3(X[i], x);
    int c = cell_of<float, 3>(B.edge, C.lo, C.hi, C.nc, x);
    acell[i] = c;
    arank[i] = atomicAdd(count + c, 1);
    B.pold[C.off + i] = X[i];  // verletResetDisplacement
  }
  __syncthreads();
  int carry = 0;
  for (int base = 0; base < C.n_cells; base += NT) {
    const int c = base + tid;
    const int v = c < C.n_cells ? count[c] : 0;
    int tot;
    const int ex = cta_exscan<NT>(v, warp_sums, &tot);
    if (c < C.n_cells) {
      start[c] = carry + ex;
      count[c] = 0;
    }
    carry += tot;
  }
  if (tid == 0) start[C.n_cells] = carry;
  __syncthreads();
  for (int i = tid; i < n; i += NT) tmp[start[acell[i]] + arank[i]] = i;
  __syncthreads();
  for (int i = tid; i < n; i += NT) {
    const int c = acell[i];
    const int s0 = start[c], s1 = start[c + 1];
    int r = 0;
    for (int s = s0; s < s1; ++s) r += tmp[s] < i;
    cagents[s0 + r] = i;
  }
  __syncthreads();
  const int M = B.max_nbrs;
  int* list = B.nbr_list + C.off * (long long)M;
  for (int i = tid; i < n; i += NT) {
    float xi[3];
    f4to3(X[i], xi);
    int q[3];
    cell_coords<3>(C.nc, cell_of<float, 3>(B.edge, C.lo, C.hi, C.nc, xi), q);
    int m = 0;
    bool over = false;
    for (int k = 0; k < 27; ++k) {
      const int pn = cell_neigh<3>(C.nc, q, k);
      if (pn < 0) continue;
      for (int s = start[pn]; s < start[pn + 1]; ++s) {
        const int j = cagents[s];
        if (j == i) continue;
        float xj[3];
        f4to3(X[j], xj);
        float e = xi[0] - xj[0];
        float s2 = e * e;
        e = xi[1] - xj[1];
        s2 = s2 + e * e;
        e = xi[2] - xj[2];
        s2 = s2 + e * e;
        if (s2 >= B.skin2) continue;
        if (!(s2 < B.skin2_lo) && !(sqrtf(s2) < B.skin)) continue;
        if (m < M) list[(long long)m * n + i] = j;
        else over = true;
        ++m;
      }
    }
    if (over) atomicOr(B.err, kErrNeighborOverflow);
    B.nbr_n[C.off + i] = m < M ? m : M;
  }
  __syncthreads();
}

template <int NT>
__global__ void __launch_bounds__(NT) k_batch(BatchParams B, int nsteps) {
  __shared__ int s_comm;
  __shared__ int s_flag;
  __shared__ int warp_sums[NT / 32];
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(B.head, 1);
      s_comm = q < B.n_comm ? B.order[q] : -1;
    }
    __syncthreads();
    const int ci = s_comm;
    if (ci < 0) return;
    const Comm C = B.comms[ci];
    int par = B.parity[ci];
    int rebuild = B.rebuild[ci];
    long long step = B.step[ci];
    const int M = B.max_nbrs;
    const int* list = B.nbr_list + C.off * (long long)M;
    for (int t = 0; t < nsteps; ++t) {
      const float4* Xc = B.P[par] + C.off;
      float4* Xn = B.P[par ^ 1] + C.off;
      if (rebuild) cta_rebuild<NT>(B, C, Xc, warp_sums);
      if (threadIdx.x == 0) s_flag = 0;
      __syncthreads();
      for (int i = threadIdx.x; i < C.n; i += NT) {
        float xi[3];
        f4to3(Xc[i], xi);
        float acc[3] = {0.f, 0.f, 0.f};
        const int m = B.nbr_n[C.off + i];
        for (int k = 0; k < m; ++k) {
          float xj[3];
          f4to3(Xc[list[(long long)k * C.n + i]], xj);
          float e[3];
          e[0] = xi[0] - xj[0];
          float s2 = e[0] * e[0];
          e[1] = xi[1] - xj[1];
          s2 = s2 + e[1] * e[1];
          e[2] = xi[2] - xj[2];
          s2 = s2 + e[2] * e[2];
          if (s2 >= C.cut2) continue;
          const float dd = sqrtf(s2);
          float F;
          if (dd < C.r_rep) F = C.k_rep * (C.r_rep - dd);
          else if (dd < C.r_att) F = -(C.k_att * (dd - C.r_rep));
          else continue;
          const float sc = F / dd;
#pragma unroll
          for (int d = 0; d < 3; ++d) acc[d] = acc[d] + sc * e[d];
        }
        float z[3];
        cbm_normals(B.seed, step, (uint32_t)i, CBM_STREAM_NOISE, C.community, 3, z);
        float xn[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) xn[d] = (xi[d] + acc[d] * B.dt) + (C.sigma * z[d]) * B.sqrt_dt;
        Xn[i] = make_float4(xn[0], xn[1], xn[2], 0.f);
        float xo[3];
        f4to3(B.pold[C.off + i], xo);
        float e = xn[0] - xo[0];
        float s2 = e * e;
        e = xn[1] - xo[1];
        s2 = s2 + e * e;
        e = xn[2] - xo[2];
        s2 = s2 + e * e;
        if (sqrtf(s2) >= B.thr) s_flag = 1;  // verletDisplacement (neighbors.jl:367-391)
      }
      __syncthreads();
      rebuild = s_flag;
      par ^= 1;
      ++step;
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      B.parity[ci] = par;
      B.rebuild[ci] = rebuild;
      B.step[ci] = step;
    }
    __syncthreads();
  }
}

template <typename T>
T bound2(double r, bool up) {
  if (!(r > 0)) return (T)0;
  double v = r * r * (up ? 1.0 + 1e-5 : 1.0 - 1e-5);
  T t = (T)v;
  if (up && (double)t < v) t = std::nextafter(t, (T)INFINITY);
  if (!up && (double)t > v) t = std::nextafter(t, (T)0);
  return t;
}

}  // namespace

struct cbm_batch {
  cbm_config base{};
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string err;
  std::vector<void*> allocs;       // agent-sized and per-community buffers
  std::vector<void*> cell_allocs;  // cell arrays (depend on the list radius)
  std::vector<Comm> comms;
  std::vector<int> order;
  long long total = 0, total_cells = 0;
  double cutoff = 0;               // largest interaction cutoff of the communities
  Comm* d_comms = nullptr;
  int* d_order = nullptr;
  int* d_head = nullptr;
  float4* P[2] = {};
  float4* pold = nullptr;
  int* parity = nullptr;
  int* rebuild = nullptr;
  long long* step = nullptr;
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  int* agent_cell = nullptr;
  int* agent_rank = nullptr;
  int* tmp = nullptr;
  int* cell_agents = nullptr;
  int* nbr_n = nullptr;
  int* nbr_list = nullptr;
  int* d_err = nullptr;
  cbm_batch_tuning tune{256, 2, 0.3, 0.0};
  std::map<int, cudaGraphExec_t> graphs;  // per nsteps
  int n_sm = 148;
};

namespace {

std::string g_batch_create_error;

int bfail(cbm_batch* b, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (b) b->err = buf;
  else g_batch_create_error = buf;
  return code;
}

#define BCUDA(b, call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return bfail(b, CBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

void* balloc(std::vector<void*>& list, size_t bytes, bool* ok) {
  if (!*ok) return nullptr;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes ? bytes : 16) != cudaSuccess) {
    *ok = false;
    return nullptr;
  }
  list.push_back(p);
  return p;
}

void drop_graphs(cbm_batch* b) {
  for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
  b->graphs.clear();
}

void free_batch(cbm_batch* b) {
  drop_graphs(b);
  for (void* p : b->allocs) cudaFree(p);
  for (void* p : b->cell_allocs) cudaFree(p);
  b->allocs.clear();
  b->cell_allocs.clear();
  if (b->stream) cudaStreamDestroy(b->stream);
  b->stream = nullptr;
}

double list_radius(const cbm_batch* b) { return b->cutoff + b->tune.skin; }

BatchParams batch_params(const cbm_batch* b) {
  BatchParams B;
  memset(&B, 0, sizeof B);
  B.comms = b->d_comms;
  B.order = b->d_order;
  B.n_comm = (int)b->comms.size();
  B.head = b->d_head;
  B.P[0] = b->P[0];
  B.P[1] = b->P[1];
  B.pold = b->pold;
  B.parity = b->parity;
  B.rebuild = b->rebuild;
  B.step = b->step;
  B.cell_count = b->cell_count;
  B.cell_start = b->cell_start;
  B.agent_cell = b->agent_cell;
  B.agent_rank = b->agent_rank;
  B.tmp = b->tmp;
  B.cell_agents = b->cell_agents;
  B.nbr_n = b->nbr_n;
  B.nbr_list = b->nbr_list;
  B.max_nbrs = b->base.n_max_neighbors;
  B.dt = (float)b->base.dt;
  B.sqrt_dt = std::sqrt((float)b->base.dt);
  const double R = list_radius(b);  // cell edge = list radius, as CLVD(skin=R, cellEdge=R)
  B.edge = (float)R;
  B.skin = (float)R;
  B.skin2 = bound2<float>(R, true);
  B.skin2_lo = bound2<float>(R, false);
  // rebuild when a displacement reaches half the skin
  B.thr = (float)(b->tune.rebuild_threshold > 0 ? b->tune.rebuild_threshold : b->tune.skin / 2.0);
  B.seed = b->base.seed;
  B.err = b->d_err;
  return B;
}

int enqueue_batch(cbm_batch* b, int nsteps) {
  BatchParams B = batch_params(b);
  cudaMemsetAsync(b->d_head, 0, sizeof(int), b->stream);
  const int grid = b->n_sm * std::max(1, b->tune.ctas_per_sm);
  switch (b->tune.threads) {
    case 128: k_batch<128><<<grid, 128, 0, b->stream>>>(B, nsteps); break;
    case 512: k_batch<512><<<grid, 512, 0, b->stream>>>(B, nsteps); break;
    case 1024: k_batch<1024><<<grid, 1024, 0, b->stream>>>(B, nsteps); break;
    default: k_batch<256><<<grid, 256, 0, b->stream>>>(B, nsteps); break;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bfail(b, CBM_ERR_CUDA, "batch launch failed: %s", cudaGetErrorString(e));
  return CBM_OK;
}

int batch_sync(cbm_batch* b) {
  BCUDA(b, cudaStreamSynchronize(b->stream));
  int err = 0;
  BCUDA(b, cudaMemcpy(&err, b->d_err, sizeof err, cudaMemcpyDeviceToHost));
  if (err) {
    int zero = 0;
    BCUDA(b, cudaMemcpy(b->d_err, &zero, sizeof zero, cudaMemcpyHostToDevice));
    if (err & kErrNeighborOverflow)
      return bfail(b, CBM_ERR_NEIGHBOR_OVERFLOW, "a Verlet row exceeded n_max_neighbors: list truncated");
  }
  return CBM_OK;
}

// cell arrays and descriptors for the current list radius; every community
// rebuilds its list at its next step
int apply_tuning(cbm_batch* b) {
  drop_graphs(b);
  for (void* p : b->cell_allocs) cudaFree(p);
  b->cell_allocs.clear();
  const double R = list_radius(b);
  b->total_cells = 0;
  for (Comm& C : b->comms) {
    long long nc = 1;
    for (int d = 0; d < 3; ++d) {
      // nCells_ = ceil((hi - lo) / edge + 2), neighbors.jl:605
      C.nc[d] = (int)std::ceil(((double)C.hi[d] - (double)C.lo[d]) / R + 2.0);
      nc *= C.nc[d];
    }
    if (nc >= (1ll << 30)) return bfail(b, CBM_ERR_ARG, "a community's cell grid is too large");
    C.n_cells = (int)nc;
    C.cell_off = b->total_cells;
    b->total_cells += nc + 1;
  }
  bool ok = true;
  b->cell_count = (int*)balloc(b->cell_allocs, (size_t)b->total_cells * 4, &ok);
  b->cell_start = (int*)balloc(b->cell_allocs, (size_t)b->total_cells * 4, &ok);
  if (!ok) return bfail(b, CBM_ERR_NOMEM, "cell arrays do not fit");
  BCUDA(b, cudaMemsetAsync(b->cell_count, 0, (size_t)b->total_cells * 4, b->stream));
  BCUDA(b, cudaMemcpyAsync(b->d_comms, b->comms.data(), b->comms.size() * sizeof(Comm),
                           cudaMemcpyHostToDevice, b->stream));
  std::vector<int> ones(b->comms.size(), 1);
  BCUDA(b, cudaMemcpyAsync(b->rebuild, ones.data(), ones.size() * 4, cudaMemcpyHostToDevice, b->stream));
  BCUDA(b, cudaStreamSynchronize(b->stream));
  return CBM_OK;
}

}  // namespace

extern "C" {

const char* cbm_batch_last_error(const cbm_batch* b) {
  return b ? b->err.c_str() : g_batch_create_error.c_str();
}

int cbm_batch_create(cbm_batch** out, const cbm_config* base, int32_t n_comm,
                     const cbm_community_desc* descs) {
  if (!out || !base || !descs || n_comm < 1)
    return bfail(nullptr, CBM_ERR_ARG, "null argument or no community");
  *out = nullptr;
  if (base->dims != 3 || base->precision != CBM_F32 || base->integrator != CBM_INT_EM ||
      base->neighbors != CBM_NEIGH_CLVD)
    return bfail(nullptr, CBM_ERR_ARG,
                 "the batched form runs 3D Float32 Euler-Maruyama communities with CLVD");
  if (!(base->dt > 0) || base->n_max_neighbors < 1)
    return bfail(nullptr, CBM_ERR_ARG, "dt and n_max_neighbors must be positive");
  cbm_batch* b = new cbm_batch;
  b->base = *base;
  cudaGetDevice(&b->device);
  cudaDeviceGetAttribute(&b->n_sm, cudaDevAttrMultiProcessorCount, b->device);
  if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete b;
    return bfail(nullptr, CBM_ERR_CUDA, "cudaStreamCreate failed (is a CUDA device present?)");
  }
  b->comms.resize((size_t)n_comm);
  for (int c = 0; c < n_comm; ++c) {
    const cbm_community_desc& d = descs[c];
    if (d.n < 0 || d.n >= (1 << 26)) {
      free_batch(b);
      delete b;
      return bfail(nullptr, CBM_ERR_ARG, "community %d size out of range", c);
    }
    Comm& C = b->comms[(size_t)c];
    memset(&C, 0, sizeof C);
    C.n = (int)d.n;
    for (int k = 0; k < 3; ++k) {
      C.lo[k] = (float)d.box_lo[k];
      C.hi[k] = (float)d.box_hi[k];
      if (!(d.box_hi[k] > d.box_lo[k])) {
        free_batch(b);
        delete b;
        return bfail(nullptr, CBM_ERR_ARG, "community %d has an empty box", c);
      }
    }
    C.k_rep = (float)d.k_rep;
    C.r_rep = (float)d.r_rep;
    C.k_att = (float)d.k_att;
    C.r_att = (float)d.r_att;
    C.sigma = (float)d.sigma;
    C.cut2 = bound2<float>(std::max(d.r_rep, d.r_att), true);
    C.community = d.community;
    C.off = b->total;
    b->total += C.n;
    b->cutoff = std::max(b->cutoff, std::max(d.r_rep, d.r_att));
  }
  if (b->total >= (1ll << 30) || b->total * (long long)base->n_max_neighbors >= (1ll << 40)) {
    free_batch(b);
    delete b;
    return bfail(nullptr, CBM_ERR_ARG, "too many agents in the batch");
  }
  b->order.resize((size_t)n_comm);
  for (int c = 0; c < n_comm; ++c) b->order[(size_t)c] = c;
  std::stable_sort(b->order.begin(), b->order.end(),
                   [&](int a, int c) { return b->comms[(size_t)a].n > b->comms[(size_t)c].n; });
  const size_t n = (size_t)std::max(b->total, 1ll), nc = (size_t)n_comm;
  bool ok = true;
  b->P[0] = (float4*)balloc(b->allocs, n * 16, &ok);
  b->P[1] = (float4*)balloc(b->allocs, n * 16, &ok);
  b->pold = (float4*)balloc(b->allocs, n * 16, &ok);
  b->agent_cell = (int*)balloc(b->allocs, n * 4, &ok);
  b->agent_rank = (int*)balloc(b->allocs, n * 4, &ok);
  b->tmp = (int*)balloc(b->allocs, n * 4, &ok);
  b->cell_agents = (int*)balloc(b->allocs, n * 4, &ok);
  b->nbr_n = (int*)balloc(b->allocs, n * 4, &ok);
  b->nbr_list = (int*)balloc(b->allocs, n * (size_t)base->n_max_neighbors * 4, &ok);
  b->parity = (int*)balloc(b->allocs, nc * 4, &ok);
  b->rebuild = (int*)balloc(b->allocs, nc * 4, &ok);
  b->step = (long long*)balloc(b->allocs, nc * 8, &ok);
  b->d_comms = (Comm*)balloc(b->allocs, nc * sizeof(Comm), &ok);
  b->d_order = (int*)balloc(b->allocs, nc * 4, &ok);
  b->d_head = (int*)balloc(b->allocs, 4, &ok);
  b->d_err = (int*)balloc(b->allocs, 4, &ok);
  if (!ok) {
    free_batch(b);
    delete b;
    return bfail(nullptr, CBM_ERR_NOMEM, "device allocation failed for %lld agents", (long long)n);
  }
  cudaMemsetAsync(b->P[0], 0, n * 16, b->stream);
  cudaMemsetAsync(b->parity, 0, nc * 4, b->stream);
  cudaMemsetAsync(b->step, 0, nc * 8, b->stream);
  cudaMemsetAsync(b->d_err, 0, 4, b->stream);
  cudaMemcpyAsync(b->d_order, b->order.data(), nc * 4, cudaMemcpyHostToDevice, b->stream);
  // defaults: skin from the base config (list radius - cutoff) when given
  if (base->skin > b->cutoff) b->tune.skin = base->skin - b->cutoff;
  b->tune.rebuild_threshold = base->rebuild_threshold;
  int rc = apply_tuning(b);
  if (rc) {
    g_batch_create_error = b->err;
    free_batch(b);
    delete b;
    return rc;
  }
  *out = b;
  return CBM_OK;
}

void cbm_batch_destroy(cbm_batch* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  cudaStreamSynchronize(b->stream);
  free_batch(b);
  delete b;
}

int cbm_batch_set_tuning(cbm_batch* b, const cbm_batch_tuning* t) {
  if (!b || !t) return CBM_ERR_ARG;
  if (t->threads != 128 && t->threads != 256 && t->threads != 512 && t->threads != 1024)
    return bfail(b, CBM_ERR_ARG, "threads must be 128, 256, 512 or 1024");
  if (t->ctas_per_sm < 1 || t->ctas_per_sm > 8 || !(t->skin > 0))
    return bfail(b, CBM_ERR_ARG, "ctas_per_sm must be in [1, 8] and skin positive");
  cudaSetDevice(b->device);
  BCUDA(b, cudaStreamSynchronize(b->stream));
  b->tune = *t;
  return apply_tuning(b);
}

int cbm_batch_get_tuning(cbm_batch* b, cbm_batch_tuning* t) {
  if (!b || !t) return CBM_ERR_ARG;
  *t = b->tune;
  return CBM_OK;
}

int cbm_batch_upload(cbm_batch* b, int32_t c, const cbm_state_view* h) {
  if (!b || !h || c < 0 || c >= (int)b->comms.size()) return bfail(b, CBM_ERR_ARG, "bad community");
  const Comm& C = b->comms[(size_t)c];
  if (h->N != C.n) return bfail(b, CBM_ERR_ARG, "community %d holds %d agents, got %lld", c, C.n, (long long)h->N);
  if (C.n && (!h->pos[0] || !h->pos[1] || !h->pos[2])) return bfail(b, CBM_ERR_ARG, "positions are NULL");
  cudaSetDevice(b->device);
  std::vector<float4> packed((size_t)C.n);
  const float* x = (const float*)h->pos[0];
  const float* y = (const float*)h->pos[1];
  const float* z = (const float*)h->pos[2];
  for (int i = 0; i < C.n; ++i) packed[(size_t)i] = make_float4(x[i], y[i], z[i], 0.f);
  BCUDA(b, cudaStreamSynchronize(b->stream));
  if (C.n) BCUDA(b, cudaMemcpy(b->P[0] + C.off, packed.data(), (size_t)C.n * 16, cudaMemcpyHostToDevice));
  int zero = 0, one = 1;
  long long st = h->step;
  BCUDA(b, cudaMemcpy(b->parity + c, &zero, 4, cudaMemcpyHostToDevice));
  BCUDA(b, cudaMemcpy(b->rebuild + c, &one, 4, cudaMemcpyHostToDevice));
  BCUDA(b, cudaMemcpy(b->step + c, &st, 8, cudaMemcpyHostToDevice));
  return CBM_OK;
}

int cbm_batch_download(cbm_batch* b, int32_t c, cbm_state_view* h) {
  if (!b || !h || c < 0 || c >= (int)b->comms.size()) return bfail(b, CBM_ERR_ARG, "bad community");
  const Comm& C = b->comms[(size_t)c];
  if (h->capacity < C.n) return bfail(b, CBM_ERR_ARG, "host capacity too small");
  cudaSetDevice(b->device);
  BCUDA(b, cudaStreamSynchronize(b->stream));
  int par = 0;
  long long st = 0;
  BCUDA(b, cudaMemcpy(&par, b->parity + c, 4, cudaMemcpyDeviceToHost));
  BCUDA(b, cudaMemcpy(&st, b->step + c, 8, cudaMemcpyDeviceToHost));
  std::vector<float4> packed((size_t)C.n);
  if (C.n) BCUDA(b, cudaMemcpy(packed.data(), b->P[par] + C.off, (size_t)C.n * 16, cudaMemcpyDeviceToHost));
  float* x = (float*)h->pos[0];
  float* y = (float*)h->pos[1];
  float* z = (float*)h->pos[2];
  for (int i = 0; i < C.n; ++i) {
    if (x) x[i] = packed[(size_t)i].x;
    if (y) y[i] = packed[(size_t)i].y;
    if (z) z[i] = packed[(size_t)i].z;
  }
  h->N = C.n;
  h->step = st;
  h->t = (double)st * b->base.dt;
  return CBM_OK;
}

int cbm_batch_step(cbm_batch* b, int32_t nsteps, int32_t flags) {
  if (!b || nsteps < 0) return CBM_ERR_ARG;
  cudaSetDevice(b->device);
  if (nsteps == 0) return flags & CBM_SYNC ? batch_sync(b) : CBM_OK;
  if (flags & CBM_NO_GRAPH) {
    int rc = enqueue_batch(b, nsteps);
    if (rc) return rc;
  } else {
    auto it = b->graphs.find(nsteps);
    if (it == b->graphs.end()) {
      cudaGraph_t g = nullptr;
      BCUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      int rc = enqueue_batch(b, nsteps);
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (rc) return rc;
      if (e != cudaSuccess) return bfail(b, CBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
      cudaGraphExec_t ge = nullptr;
      e = cudaGraphInstantiate(&ge, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return bfail(b, CBM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
      it = b->graphs.emplace(nsteps, ge).first;
    }
    BCUDA(b, cudaGraphLaunch(it->second, b->stream));
  }
  return flags & CBM_SYNC ? batch_sync(b) : CBM_OK;
}

void* cbm_batch_stream(cbm_batch* b) { return b ? (void*)b->stream : nullptr; }

int cbm_batch_autotune(cbm_batch* b, int32_t trial_steps, cbm_batch_tuning* best_out) {
  if (!b || trial_steps < 1) return CBM_ERR_ARG;
  cudaSetDevice(b->device);
  BCUDA(b, cudaStreamSynchronize(b->stream));
  const size_t n = (size_t)std::max(b->total, 1ll), nc = b->comms.size();
  // the trials run on a copy of the state, which is put back afterwards
  std::vector<float4> p0(n), p1(n);
  std::vector<int> par(nc), reb(nc);
  std::vector<long long> st(nc);
  BCUDA(b, cudaMemcpy(p0.data(), b->P[0], n * 16, cudaMemcpyDeviceToHost));
  BCUDA(b, cudaMemcpy(p1.data(), b->P[1], n * 16, cudaMemcpyDeviceToHost));
  BCUDA(b, cudaMemcpy(par.data(), b->parity, nc * 4, cudaMemcpyDeviceToHost));
  BCUDA(b, cudaMemcpy(st.data(), b->step, nc * 8, cudaMemcpyDeviceToHost));
  const cbm_batch_tuning start = b->tune;
  const int threads[] = {128, 256, 512, 1024};
  const int ctas[] = {1, 2, 4};
  const double skins[] = {0.15, 0.3, 0.6};
  cbm_batch_tuning best = start;
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  for (double sk : skins)
    for (int th : threads)
      for (int cp : ctas) {
        if (th * cp > 2048) continue;
        cbm_batch_tuning t{th, cp, sk, 0.0};
        if (cbm_batch_set_tuning(b, &t)) continue;
        BCUDA(b, cudaMemcpy(b->P[0], p0.data(), n * 16, cudaMemcpyHostToDevice));
        BCUDA(b, cudaMemcpy(b->P[1], p1.data(), n * 16, cudaMemcpyHostToDevice));
        BCUDA(b, cudaMemcpy(b->parity, par.data(), nc * 4, cudaMemcpyHostToDevice));
        BCUDA(b, cudaMemcpy(b->step, st.data(), nc * 8, cudaMemcpyHostToDevice));
        cudaEventRecord(e0, b->stream);
        int rc = enqueue_batch(b, trial_steps);
        cudaEventRecord(e1, b->stream);
        if (rc) continue;
        if (batch_sync(b)) continue;  // an overflowing list disqualifies the setting
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) {
          best_ms = ms;
          best = t;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  int rc = cbm_batch_set_tuning(b, &best);
  if (rc) return rc;
  BCUDA(b, cudaMemcpy(b->P[0], p0.data(), n * 16, cudaMemcpyHostToDevice));
  BCUDA(b, cudaMemcpy(b->P[1], p1.data(), n * 16, cudaMemcpyHostToDevice));
  BCUDA(b, cudaMemcpy(b->parity, par.data(), nc * 4, cudaMemcpyHostToDevice));
  BCUDA(b, cudaMemcpy(b->step, st.data(), nc * 8, cudaMemcpyHostToDevice));
  if (best_out) *best_out = best;
  return CBM_OK;
}

}  // extern "C"
