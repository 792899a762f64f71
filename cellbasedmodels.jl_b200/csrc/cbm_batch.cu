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
  float4* P[2];         // positions in slot order, ping-pong by per-community parity;
                        // w holds the agent index (int bits)
  float4* pold;         // slot order: positions at the last rebuild
  int* parity;          // per community: which P holds the current positions
  int* rebuild;         // per community: the next step starts with a rebuild
  long long* step;      // per community step counter
  int* cell_count;      // zero between rebuilds
  int* cell_start;      // n_cells + 1 per community
  int* key;             // rebuild scratch: cell of an old slot
  int* rank;            // rebuild scratch: arrival rank of an old slot in its cell
  int* sidx;            // rebuild scratch: agent index by (cell, arrival)
  int* nbr_n;
  int* nbr_list;        // per community: entry k of slot q at off*M + k*n + q
  int max_nbrs;
  int tile;             // communities of at most this many agents gather from shared memory
  float dt, sqrt_dt;
  float edge, skin, skin2, skin2_lo, thr;
  uint64_t seed;
  int* err;
};

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

__device__ __forceinline__ int agent_index(const float4& p) { return __float_as_int(p.w); }

// Grid rebuild of one community (neighbors.jl:918-979): counting sort of the
// agents by cell, ascending agent index inside a cell, from X (old slot
// order) into Xs, which becomes the new slot order.  The slot order is then
// the CLVD walk order: cells x fastest, ascending index inside a cell.
template <int NT>
__device__ void cta_sort(const BatchParams& B, const Comm& C, const float4* X, float4* Xs,
                         int* warp_sums) {
  const int n = C.n, tid = threadIdx.x;
  int* count = B.cell_count + C.cell_off;
  int* start = B.cell_start + C.cell_off;
  int* key = B.key + C.off;
  int* rank = B.rank + C.off;
  int* sidx = B.sidx + C.off;
  for (int s = tid; s < n; s += NT) {
    const float4 p = X[s];
    const float x[3] = {p.x, p.y, p.z};
    const int c = cell_of<float, 3>(B.edge, C.lo, C.hi, C.nc, x);
    key[s] = c;
    rank[s] = atomicAdd(count + c, 1);
  }
  __syncthreads();
  // exclusive scan of the counts: a run of cells per thread
  const int nc = C.n_cells;
  const int per = (nc + NT - 1) / NT;
  const int c0 = min(nc, tid * per), c1 = min(nc, c0 + per);
  int local = 0;
  for (int c = c0; c < c1; ++c) local += count[c];
  int total;
  int run = cta_exscan<NT>(local, warp_sums, &total);
  for (int c = c0; c < c1; ++c) {
    const int v = count[c];
    start[c] = run;
    run += v;
    count[c] = 0;
  }
  if (tid == 0) start[nc] = total;
  __syncthreads();
  for (int s = tid; s < n; s += NT) sidx[start[key[s]] + rank[s]] = agent_index(X[s]);
  __syncthreads();
  for (int s = tid; s < n; s += NT) {
    const float4 p = X[s];
    const int c = key[s], me = agent_index(p);
    const int s0 = start[c], s1 = start[c + 1];
    int r = 0;
    for (int u = s0; u < s1; ++u) r += sidx[u] < me;
    Xs[s0 + r] = p;
    B.pold[C.off + s0 + r] = p;  // verletResetDisplacement
  }
  __syncthreads();
}

// position of slot j: from the shared-memory tile or from global memory
template <bool SM>
__device__ __forceinline__ void pos_of(const float4* X, const float* sx, const float* sy,
                                       const float* sz, int j, float* xj) {
  if (SM) {
    xj[0] = sx[j];
    xj[1] = sy[j];
    xj[2] = sz[j];
  } else {
    const float4 p = X[j];
    xj[0] = p.x;
    xj[1] = p.y;
    xj[2] = p.z;
  }
}

// one pair of the soft-sphere force (the expression order of the plain path)
__device__ __forceinline__ void pair_force(const Comm& C, const float* xi, const float* xj,
                                           float* acc) {
  float e[3];
  e[0] = xi[0] - xj[0];
  float s2 = e[0] * e[0];
  e[1] = xi[1] - xj[1];
  s2 = s2 + e[1] * e[1];
  e[2] = xi[2] - xj[2];
  s2 = s2 + e[2] * e[2];
  if (s2 >= C.cut2) return;
  const float dd = sqrtf(s2);
  float F;
  if (dd < C.r_rep) F = C.k_rep * (C.r_rep - dd);
  else if (dd < C.r_att) F = -(C.k_att * (dd - C.r_rep));
  else return;
  const float sc = F / dd;
#pragma unroll
  for (int d = 0; d < 3; ++d) acc[d] = acc[d] + sc * e[d];
}

// The same pair term as pair_force, returned instead of added: t = (F/d) e.
__device__ __forceinline__ bool pair_term3(const Comm& C, const float* xi, const float* xj,
                                           float* t) {
  float e[3];
  e[0] = xi[0] - xj[0];
  float s2 = e[0] * e[0];
  e[1] = xi[1] - xj[1];
  s2 = s2 + e[1] * e[1];
  e[2] = xi[2] - xj[2];
  s2 = s2 + e[2] * e[2];
  if (s2 >= C.cut2) return false;
  const float dd = sqrtf(s2);
  float F;
  if (dd < C.r_rep) F = C.k_rep * (C.r_rep - dd);
  else if (dd < C.r_att) F = -(C.k_att * (dd - C.r_rep));
  else return false;
  const float sc = F / dd;
#pragma unroll
  for (int d = 0; d < 3; ++d) t[d] = sc * e[d];
  return true;
}

// L lanes of a warp that share one agent (lanes_per_agent): the lane's place
// in its group and the group's lanes.
template <int L>
struct Group {
  int gl;
  unsigned mask;
  __device__ Group() {
    const int lane = threadIdx.x & 31;
    gl = lane & (L - 1);
    mask = (L == 32 ? 0xffffffffu : ((1u << L) - 1u)) << (lane & ~(L - 1));
  }
};

// The terms of the group's lanes added to acc in lane order (the list order
// of the entries the lanes hold); every lane of the group keeps the same acc.
template <int L>
__device__ __forceinline__ void group_add(const Group<L>& g, bool has, const float* t, float* acc) {
#pragma unroll
  for (int u = 0; u < L; ++u) {
    const int hu = __shfl_sync(g.mask, has ? 1 : 0, u, L);
    const float t0 = __shfl_sync(g.mask, t[0], u, L);
    const float t1 = __shfl_sync(g.mask, t[1], u, L);
    const float t2 = __shfl_sync(g.mask, t[2], u, L);
    if (hu) {
      acc[0] = acc[0] + t0;
      acc[1] = acc[1] + t1;
      acc[2] = acc[2] + t2;
    }
  }
}

// Rebuild step of slot q with L lanes: lane u of the group takes candidates
// u, u + L, ... of each run; the list row is written at the places the
// group's ballot gives (candidate order), and the terms are added in
// candidate order by group_add.
template <bool SM, int L>
__device__ __forceinline__ void build_row_group(const BatchParams& B, const Comm& C,
                                                const float4* X, const float* sx, const float* sy,
                                                const float* sz, int q, const float* xi, int* list,
                                                int* nbr_n, float* acc) {
  const Group<L> g;
  const int n = C.n, M = B.max_nbrs;
  const int* start = B.cell_start + C.cell_off;
  int q3[3];
  cell_coords<3>(C.nc, cell_of<float, 3>(B.edge, C.lo, C.hi, C.nc, xi), q3);
  const int xa = max(q3[0] - 1, 0), xb = min(q3[0] + 1, C.nc[0] - 1);
  const int shift = (threadIdx.x & 31) & ~(L - 1);
  int m = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = q3[2] + dz;
    if (z < 0 || z >= C.nc[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = q3[1] + dy;
      if (y < 0 || y >= C.nc[1]) continue;
      const int row = (z * C.nc[1] + y) * C.nc[0];
      const int s1 = start[row + xb + 1];
      for (int base = start[row + xa]; base < s1; base += L) {
        const int s = base + g.gl;
        bool in = false, has = false;
        float t[3] = {0.f, 0.f, 0.f};
        if (s < s1 && s != q) {
          float xj[3];
          pos_of<SM>(X, sx, sy, sz, s, xj);
          float e = xi[0] - xj[0];
          float s2 = e * e;
          e = xi[1] - xj[1];
          s2 = s2 + e * e;
          e = xi[2] - xj[2];
          s2 = s2 + e * e;
          in = s2 < B.skin2 && (s2 < B.skin2_lo || sqrtf(s2) < B.skin);
          if (in) has = pair_term3(C, xi, xj, t);
        }
        const unsigned gb = (__ballot_sync(g.mask, in) >> shift) & ((1u << L) - 1u);
        if (in) {
          const int pos = m + __popc(gb & ((1u << g.gl) - 1u));
          if (pos < M) list[(long long)pos * n + q] = s;
        }
        m += __popc(gb);
        group_add<L>(g, has, t, acc);
      }
    }
  }
  if (g.gl == 0) {
    if (m > M) atomicOr(B.err, kErrNeighborOverflow);
    nbr_n[q] = m < M ? m : M;
  }
}

// Non-rebuild step of slot q with L lanes: lane u takes list entries u,
// u + L, ...; the terms are added in list order.
template <bool SM, int L>
__device__ __forceinline__ void list_row_group(const BatchParams& B, const Comm& C,
                                               const float4* X, const float* sx, const float* sy,
                                               const float* sz, int q, const float* xi,
                                               const int* list, const int* nbr_n, float* acc) {
  const Group<L> g;
  const int n = C.n;
  const int m = nbr_n[q];
  const int* row = list + q;
  for (int k0 = 0; k0 < m; k0 += L) {
    const int k = k0 + g.gl;
    bool has = false;
    float t[3] = {0.f, 0.f, 0.f};
    if (k < m) {
      float xj[3];
      pos_of<SM>(X, sx, sy, sz, row[(long long)k * n], xj);
      has = pair_term3(C, xi, xj, t);
    }
    group_add<L>(g, has, t, acc);
  }
}

// Rebuild step of slot q: the CLVD list row (verletNeighborsCLVD,
// neighbors.jl:1071-1131 as intended: the 27 cells x fastest, d < list
// radius) and, in the same pass and the same order, the force.  For fixed
// (dz, dy) the cells x-1..x+1 are one contiguous run of slots.
template <bool SM>
__device__ __forceinline__ void build_row(const BatchParams& B, const Comm& C, const float4* X,
                                          const float* sx, const float* sy, const float* sz,
                                          int q, const float* xi, int* list, int* nbr_n,
                                          float* acc) {
  const int n = C.n, M = B.max_nbrs;
  const int* start = B.cell_start + C.cell_off;
  int q3[3];
  cell_coords<3>(C.nc, cell_of<float, 3>(B.edge, C.lo, C.hi, C.nc, xi), q3);
  const int xa = max(q3[0] - 1, 0), xb = min(q3[0] + 1, C.nc[0] - 1);
  int m = 0;
  for (int dz = -1; dz <= 1; ++dz) {
    const int z = q3[2] + dz;
    if (z < 0 || z >= C.nc[2]) continue;
    for (int dy = -1; dy <= 1; ++dy) {
      const int y = q3[1] + dy;
      if (y < 0 || y >= C.nc[1]) continue;
      const int row = (z * C.nc[1] + y) * C.nc[0];
      const int s1 = start[row + xb + 1];
      for (int s = start[row + xa]; s < s1; ++s) {
        if (s == q) continue;
        float xj[3];
        pos_of<SM>(X, sx, sy, sz, s, xj);
        float e = xi[0] - xj[0];
        float s2 = e * e;
        e = xi[1] - xj[1];
        s2 = s2 + e * e;
        e = xi[2] - xj[2];
        s2 = s2 + e * e;
        if (s2 >= B.skin2) continue;
        if (!(s2 < B.skin2_lo) && !(sqrtf(s2) < B.skin)) continue;
        if (m < M) list[(long long)m * n + q] = s;
        ++m;
        pair_force(C, xi, xj, acc);
      }
    }
  }
  if (m > M) atomicOr(B.err, kErrNeighborOverflow);
  nbr_n[q] = m < M ? m : M;
}

// Non-rebuild step of slot q: the force over the list row, four entries in
// flight, summed in list order.
template <bool SM>
__device__ __forceinline__ void list_row(const BatchParams& B, const Comm& C, const float4* X,
                                         const float* sx, const float* sy, const float* sz,
                                         int q, const float* xi, const int* list,
                                         const int* nbr_n, float* acc) {
  const int n = C.n;
  const int m = nbr_n[q];
  const int* row = list + q;
  int k = 0;
  for (; k + 4 <= m; k += 4) {
    int j[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) j[u] = row[(long long)(k + u) * n];
    float xj[4][3];
#pragma unroll
    for (int u = 0; u < 4; ++u) pos_of<SM>(X, sx, sy, sz, j[u], xj[u]);
#pragma unroll
    for (int u = 0; u < 4; ++u) pair_force(C, xi, xj[u], acc);
  }
  for (; k < m; ++k) {
    float xj[3];
    pos_of<SM>(X, sx, sy, sz, row[(long long)k * n], xj);
    pair_force(C, xi, xj, acc);
  }
}

// all requested steps of one community
template <int NT, bool SM, int L>
__device__ void run_comm(const BatchParams& B, const Comm& C, int ci, int nsteps, float* sx,
                         float* sy, float* sz, int* warp_sums, int* s_flag) {
  int par = B.parity[ci];
  int rebuild = B.rebuild[ci];
  long long step = B.step[ci];
  const int n = C.n;
  int* list = B.nbr_list + C.off * (long long)B.max_nbrs;
  int* nbr_n = B.nbr_n + C.off;
  const float4* pold = B.pold + C.off;
  if (threadIdx.x == 0) s_flag[0] = s_flag[1] = 0;
  for (int t = 0; t < nsteps; ++t) {
    if (rebuild) {
      cta_sort<NT>(B, C, B.P[par] + C.off, B.P[par ^ 1] + C.off, warp_sums);
      par ^= 1;
    }
    const float4* Xc = B.P[par] + C.off;
    float4* Xn = B.P[par ^ 1] + C.off;
    if (SM) {
      for (int s = threadIdx.x; s < n; s += NT) {
        const float4 p = Xc[s];
        sx[s] = p.x;
        sy[s] = p.y;
        sz[s] = p.z;
      }
    }
    __syncthreads();
    // the flag of the next step: every thread has read it last step
    if (threadIdx.x == 0) s_flag[(t + 1) & 1] = 0;
    // L lanes per agent: the group of lanes (threadIdx.x / L) shares slot q
    for (int q = (int)threadIdx.x / L; q < n; q += NT / L) {
      const float4 me = Xc[q];
      const float xi[3] = {me.x, me.y, me.z};
      float acc[3] = {0.f, 0.f, 0.f};
      if constexpr (L == 1) {
        if (rebuild) build_row<SM>(B, C, Xc, sx, sy, sz, q, xi, list, nbr_n, acc);
        else list_row<SM>(B, C, Xc, sx, sy, sz, q, xi, list, nbr_n, acc);
      } else {
        if (rebuild) build_row_group<SM, L>(B, C, Xc, sx, sy, sz, q, xi, list, nbr_n, acc);
        else list_row_group<SM, L>(B, C, Xc, sx, sy, sz, q, xi, list, nbr_n, acc);
        if ((threadIdx.x & (L - 1)) != 0) continue;  // the group's first lane integrates
      }
      float z[3];
      cbm_normals(B.seed, step, (uint32_t)agent_index(me), CBM_STREAM_NOISE, C.community, 3, z);
      float xn[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) xn[d] = (xi[d] + acc[d] * B.dt) + (C.sigma * z[d]) * B.sqrt_dt;
      Xn[q] = make_float4(xn[0], xn[1], xn[2], me.w);
      const float4 po = pold[q];
      float e = xn[0] - po.x;
      float s2 = e * e;
      e = xn[1] - po.y;
      s2 = s2 + e * e;
      e = xn[2] - po.z;
      s2 = s2 + e * e;
      if (sqrtf(s2) >= B.thr) s_flag[t & 1] = 1;  // verletDisplacement (neighbors.jl:367-391)
    }
    __syncthreads();
    rebuild = s_flag[t & 1];
    par ^= 1;
    ++step;
  }
  if (threadIdx.x == 0) {
    B.parity[ci] = par;
    B.rebuild[ci] = rebuild;
    B.step[ci] = step;
  }
}

// MINB: resident CTAs per SM the register allocation must allow (the
// tuning's ctas_per_sm when it is 1 or 2)
template <int NT, int MINB, int L>
__global__ void __launch_bounds__(NT, MINB) k_batch(BatchParams B, int nsteps) {
  extern __shared__ float s_tile[];
  __shared__ int s_comm;
  __shared__ int s_flag[2];
  __shared__ int warp_sums[NT / 32];
  float* sx = s_tile;
  float* sy = s_tile + B.tile;
  float* sz = s_tile + 2 * B.tile;
  for (;;) {
    if (threadIdx.x == 0) {
      const int q = atomicAdd(B.head, 1);
      s_comm = q < B.n_comm ? B.order[q] : -1;
    }
    __syncthreads();
    const int ci = s_comm;
    if (ci < 0) return;
    const Comm C = B.comms[ci];
    if (C.n <= B.tile) run_comm<NT, true, L>(B, C, ci, nsteps, sx, sy, sz, warp_sums, s_flag);
    else run_comm<NT, false, L>(B, C, ci, nsteps, sx, sy, sz, warp_sums, s_flag);
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
  int* key = nullptr;
  int* rank = nullptr;
  int* sidx = nullptr;
  int* nbr_n = nullptr;
  int* nbr_list = nullptr;
  int* d_err = nullptr;
  cbm_batch_tuning tune{256, 2, 0.3, 0.0, 0, 1};
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

using BatchKernel = void (*)(BatchParams, int);

// registers limited for two resident CTAs when the tuning asks for two or more
template <int NT, int L>
void launch_batch_l(cbm_batch* b, const BatchParams& B, int nsteps, int grid, size_t smem) {
  if (b->tune.ctas_per_sm >= 2) k_batch<NT, 2, L><<<grid, NT, smem, b->stream>>>(B, nsteps);
  else k_batch<NT, 1, L><<<grid, NT, smem, b->stream>>>(B, nsteps);
}
template <int NT>
void launch_batch(cbm_batch* b, const BatchParams& B, int nsteps, int grid, size_t smem) {
  switch (b->tune.lanes_per_agent) {
    case 2: launch_batch_l<NT, 2>(b, B, nsteps, grid, smem); break;
    case 4: launch_batch_l<NT, 4>(b, B, nsteps, grid, smem); break;
    default: launch_batch_l<NT, 1>(b, B, nsteps, grid, smem); break;
  }
}

// dynamic shared memory of a position tile (x, y, z arrays)
constexpr int kMaxTileBytes = 220 * 1024;
size_t tile_bytes(int tile_agents) { return (size_t)std::max(tile_agents, 0) * 3 * sizeof(float); }

int set_smem_limit(cbm_batch* b) {
  const int bytes = (int)tile_bytes(b->tune.tile_agents);
  for (const BatchKernel k :
       {k_batch<128, 1, 1>, k_batch<128, 2, 1>, k_batch<256, 1, 1>, k_batch<256, 2, 1>,
        k_batch<512, 1, 1>, k_batch<512, 2, 1>, k_batch<1024, 1, 1>, k_batch<1024, 2, 1>,
        k_batch<128, 1, 2>, k_batch<128, 2, 2>, k_batch<256, 1, 2>, k_batch<256, 2, 2>,
        k_batch<512, 1, 2>, k_batch<512, 2, 2>, k_batch<1024, 1, 2>, k_batch<1024, 2, 2>,
        k_batch<128, 1, 4>, k_batch<128, 2, 4>, k_batch<256, 1, 4>, k_batch<256, 2, 4>,
        k_batch<512, 1, 4>, k_batch<512, 2, 4>, k_batch<1024, 1, 4>, k_batch<1024, 2, 4>})
    BCUDA(b, cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return CBM_OK;
}

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
  B.key = b->key;
  B.rank = b->rank;
  B.sidx = b->sidx;
  B.tile = b->tune.tile_agents;
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
  const size_t smem = tile_bytes(b->tune.tile_agents);
  switch (b->tune.threads) {
    case 128: launch_batch<128>(b, B, nsteps, grid, smem); break;
    case 512: launch_batch<512>(b, B, nsteps, grid, smem); break;
    case 1024: launch_batch<1024>(b, B, nsteps, grid, smem); break;
    default: launch_batch<256>(b, B, nsteps, grid, smem); break;
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
  if (int rc = set_smem_limit(b)) return rc;
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
  b->key = (int*)balloc(b->allocs, n * 4, &ok);
  b->rank = (int*)balloc(b->allocs, n * 4, &ok);
  b->sidx = (int*)balloc(b->allocs, n * 4, &ok);
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
  if (t->tile_agents < 0 || tile_bytes(t->tile_agents) > (size_t)kMaxTileBytes)
    return bfail(b, CBM_ERR_ARG, "tile_agents must be in [0, %d]", kMaxTileBytes / 12);
  if (t->lanes_per_agent != 0 && t->lanes_per_agent != 1 && t->lanes_per_agent != 2 &&
      t->lanes_per_agent != 4)
    return bfail(b, CBM_ERR_ARG, "lanes_per_agent must be 1, 2 or 4");
  cudaSetDevice(b->device);
  BCUDA(b, cudaStreamSynchronize(b->stream));
  b->tune = *t;
  if (b->tune.lanes_per_agent == 0) b->tune.lanes_per_agent = 1;
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
  for (int i = 0; i < C.n; ++i) {
    float w;
    memcpy(&w, &i, sizeof w);  // the agent index rides in w
    packed[(size_t)i] = make_float4(x[i], y[i], z[i], w);
  }
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
  // slot order -> index order
  for (int s = 0; s < C.n; ++s) {
    const float4& p = packed[(size_t)s];
    int i;
    memcpy(&i, &p.w, sizeof i);
    if (i < 0 || i >= C.n) return bfail(b, CBM_ERR_CUDA, "community %d: corrupt agent index", c);
    if (x) x[i] = p.x;
    if (y) y[i] = p.y;
    if (z) z[i] = p.z;
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
  const int threads[] = {256, 512, 1024};
  const int ctas[] = {1, 2};
  const double skins[] = {0.3, 0.6, 1.0, 1.5};
  int largest = 0;
  for (const Comm& C : b->comms) largest = std::max(largest, C.n);
  cbm_batch_tuning best = start;
  float best_ms = 1e30f;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  // times trial_steps of tuning t on the saved state; the fastest is kept
  auto try_tuning = [&](const cbm_batch_tuning& t) {
    if (cbm_batch_set_tuning(b, &t)) return;
    if (cudaMemcpy(b->P[0], p0.data(), n * 16, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->P[1], p1.data(), n * 16, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->parity, par.data(), nc * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(b->step, st.data(), nc * 8, cudaMemcpyHostToDevice) != cudaSuccess)
      return;
    cudaEventRecord(e0, b->stream);
    int rc = enqueue_batch(b, trial_steps);
    cudaEventRecord(e1, b->stream);
    if (rc) return;
    if (batch_sync(b)) return;  // an overflowing list disqualifies the setting
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best_ms) {
      best_ms = ms;
      best = t;
    }
  };
  for (double sk : skins)
    for (int th : threads)
      for (int cp : ctas)
        for (int staged = 0; staged < 2; ++staged) {
        if (th * cp > 2048) continue;
        // tile: the shared memory a CTA can hold when cp CTAs share an SM
        const int fit = (int)std::min<long long>(kMaxTileBytes, 227 * 1024 / cp - 1024) / 12;
        const int tile = staged ? std::min(fit, largest) : 0;
        if (staged && tile < 1) continue;
        cbm_batch_tuning t{th, cp, sk, 0.0, tile, 1};
        try_tuning(t);
      }
  // agents per warp: the best setting with 2 and 4 lanes per agent
  const cbm_batch_tuning one_lane = best;
  for (int lanes : {2, 4}) {
    cbm_batch_tuning t = one_lane;
    t.lanes_per_agent = lanes;
    try_tuning(t);
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
