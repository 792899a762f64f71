// cbm_api.cu — host side of the C ABI declared in include/cbm_b200.h.
//
// A context owns every device buffer of one Community (capacity n_max) and
// one CUDA stream.  Its committed agent state lives in cell-sorted slots (set
// A) and each step writes set B (see cbm_kernels.cuh); a full step of each
// counter parity is captured once as a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <cmath>
#include <cstddef>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cbm_b200.h"
#include "cbm_kernels.cuh"
#include "cbm_small.cuh"
#include "cbm_stencil_tma.cuh"
#include <utility>

using namespace cbm;

// Steps of one chained step graph, replayed by cbm_step calls of at least
// this many steps when the medium has a gradient: inside the chain each
// step's update runs beside the next step's gradient.  Even, so that a chain
// leaves the parity as it found it.
constexpr int kChainSteps = 8;
static_assert(kChainSteps % 2 == 0, "a chain must keep the parity");
// Media of at most this many nodes are chained.  Their gradient is short
// next to the update it overlaps (1024^2 nodes: about 12 us against about
// 35); the gradient of a 256^3 field is an HBM-bound kernel of about 50 us,
// and chaining it measured slower.
constexpr long long kChainMaxNodes = 1ll << 22;

struct cbm_ctx {
  cbm_config cfg{};
  int device = 0;
  cudaStream_t stream = nullptr;
  // with a medium: the force kernel's branch of a step, forked from and
  // joined to `stream` by events (the kernel shares no buffer with the
  // medium kernels it overlaps); with a gradient as well, the branch of the
  // next step's gradient inside a chained step graph
  cudaStream_t side = nullptr, side2 = nullptr;
  cudaEvent_t fork_ev = nullptr, join_ev = nullptr, grad_fork_ev = nullptr, grad_ev = nullptr;
  size_t tsize = 4;
  std::string err;
  std::vector<void*> allocs;

  // slot-ordered state
  void* PA = nullptr;
  void* PB = nullptr;
  void* VA = nullptr;
  void* VB = nullptr;
  void* FA = nullptr;
  void* FB = nullptr;
  int* IA = nullptr;
  int* IB = nullptr;
  void* U = nullptr;
  void* POLD = nullptr;
  int* inv = nullptr;
  int* cell_of_slot = nullptr;
  // index-ordered constants and staging
  void* G = nullptr;
  long long* ID = nullptr;
  long long* PAR = nullptr;
  void* hx[3] = {};
  void* hv = nullptr;
  void* hf[3] = {};
  // fate
  unsigned char* fate = nullptr;
  int* holes = nullptr;
  unsigned long long* fate_state = nullptr;  // per tile of the fused rule / births kernel
  // sort and grid
  int* s_cell = nullptr;
  int* s_rank = nullptr;
  int* s_key = nullptr;
  int* cell_count = nullptr;
  int* cell_start = nullptr;
  unsigned long long* scan_state = nullptr;
  // Verlet
  int* nbr_n = nullptr;
  int* nbr_list = nullptr;
  // medium
  void* c[2] = {};
  void* grad[2][3] = {};
  int* gather_box = nullptr;  // cell-box tables of the secretion gather (k_gather_box)
  // 3D medium: tensor maps of c[0] and c[1] for the TMA-fed stencils
  CUtensorMap tmap_c[2];
  bool tma_medium = false;
  Counters* ctr = nullptr;
  Counters* h_ctr = nullptr;   // pinned staging of the counters an upload writes
  int* scratch_int = nullptr;  // n_max ints for inspection calls
  void* ext_noise = nullptr;   // EM increments of cbm_step_noise (n_max * dims reals, lazy)
  bool ext_noise_on = false;   // the step being enqueued reads ext_noise

  int n_blocks = 0;
  int n_sm = 148;             // multiprocessors of the device (grid of the compaction)
  int de_blocks = 1;          // persistent grid of the force kernel
  void* pair_list = nullptr;  // its partner lists (cell walks only)
  void* pos32 = nullptr;      // Float64 3D cell walks: positions rounded to Float32
  void* pos_rows = nullptr;   // Float32 3D cell walks: positions as rows x | y | z
  int rows_stride = 0;
  void* stage[3] = {nullptr, nullptr, nullptr};  // Heun / RK4: h, running sum, derivative
  int n_cells = 1;
  int n_cells_d[3] = {1, 1, 1};
  int n_scan_tiles = 1;
  int n_nodes = 0;
  bool grid_exposed = false;  // CellLinked / CLVD: the reference has a cell grid
  bool has_list = false;      // CLVD / VerletDisplacement

  // host-side bookkeeping
  bool loaded = false;
  int parity = 0;
  bool rule_done = false, de_done = false, mrule_done = false, mde_done = false;
  cudaGraphExec_t graph[2] = {nullptr, nullptr};   // step graphs of each parity
  cudaGraphExec_t tgraph[2] = {nullptr, nullptr};  // the same with kernel timing events
  cudaGraphExec_t chain[2] = {nullptr, nullptr};   // kChainSteps steps from each parity
  // small fate-free communities: all steps of a call in one cluster launch
  long long n_loaded = 0;         // N of the last upload (fixed without births and deaths)

  // per-kernel event timing: of eager steps (cbm_profile_step, `marks`) and,
  // when graph timing is on, inside the step graph of each parity
  // (`gmarks[p]`, re-recorded by every replay)
  bool prof = false;
  struct Mark {
    const char* name;
    cudaEvent_t ev[2];
  };
  std::vector<Mark> marks;
  size_t mark_used = 0;
  bool graph_timing = false;
  std::vector<Mark> gmarks[2];
  size_t gmark_used[2] = {0, 0};
  std::vector<Mark>* prof_set = nullptr;  // the set being recorded
  size_t* prof_used = nullptr;
};

extern "C" int cbm_sync(cbm_ctx* c);

namespace {

std::string g_create_error;

int fail(cbm_ctx* ctx, int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (ctx) ctx->err = buf;
  else g_create_error = buf;
  return code;
}

#define CUDA_TRY(ctx, call)                                                                \
  do {                                                                                     \
    cudaError_t e_ = (call);                                                               \
    if (e_ != cudaSuccess)                                                                 \
      return fail(ctx, CBM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(e_));      \
  } while (0)

int grid_blocks(long long n) { return n > 0 ? (int)((n + kTile - 1) / kTile) : 1; }

// device address of the counter block's re-sort flag
const int* resort_flag(const cbm_ctx* c) {
  return (const int*)((const char*)c->ctr + offsetof(Counters, resort));
}

// Brackets one kernel launch with events when profiling an eager step.
struct Prof {
  cbm_ctx* c;
  cbm_ctx::Mark* m = nullptr;
  Prof(cbm_ctx* ctx, const char* name) : c(ctx) {
    if (!c->prof) return;
    std::vector<cbm_ctx::Mark>& set = c->prof_set ? *c->prof_set : c->marks;
    size_t& used = c->prof_used ? *c->prof_used : c->mark_used;
    if (used == set.size()) {
      cbm_ctx::Mark mk{name, {nullptr, nullptr}};
      cudaEventCreate(&mk.ev[0]);
      cudaEventCreate(&mk.ev[1]);
      set.push_back(mk);
    }
    m = &set[used++];
    m->name = name;
    record(m->ev[0]);
  }
  ~Prof() {
    if (m) record(m->ev[1]);
  }
  // inside a stream capture an event record becomes a graph node only with
  // the external flag (a plain record there just orders the capture)
  void record(cudaEvent_t e) {
    if (c->prof_set) cudaEventRecordWithFlags(e, c->stream, cudaEventRecordExternal);
    else cudaEventRecord(e, c->stream);
  }
};
#define PROF(name) Prof prof_scope_(c, name)

// Launch on the context's stream with programmatic stream serialization,
// where the kernel before it on the stream is a kernel (no event between):
// the launch follows that kernel's completion without the full gap between
// launches, and the kernel's pdl_wait() orders its memory accesses after
// it.  A plain launch while kernels are timed (the event records sit
// between).
template <typename... KP, typename... A>
void launch_pdl(cbm_ctx* c, bool pdl, void (*kern)(KP...), dim3 grid, dim3 block, size_t smem,
                A&&... args) {
  launch_serial(c->stream, pdl && !c->prof, kern, grid, block, smem, std::forward<A>(args)...);
}

// r^2 (1 + 1e-5) rounded up to T: a squared distance at or above it has a
// correctly rounded sqrt >= (T)r, so the exact `d < r` test can be skipped
template <typename T>
T bound2(double r) {
  if (!(r > 0)) return (T)0;
  double v = r * r * (1.0 + 1e-5);
  T t = (T)v;
  return (double)t < v ? std::nextafter(t, (T)INFINITY) : t;
}

// r^2 (1 - 1e-5) rounded down to T: a squared distance below it has a
// correctly rounded sqrt < (T)r
template <typename T>
T bound2_lo(double r) {
  if (!(r > 0)) return (T)0;
  double v = r * r * (1.0 - 1e-5);
  T t = (T)v;
  return (double)t > v ? std::nextafter(t, (T)0) : t;
}

// 1 / v when v > 0 is a power of two whose reciprocal is representable
// (exactly), else 0.
template <typename T>
T exact_reciprocal(T v) {
  if (!(v > (T)0) || !std::isfinite(v)) return (T)0;
  int e = 0;
  if (std::frexp(v, &e) != (T)0.5) return (T)0;
  const T r = std::ldexp((T)1, 1 - e);
  return (r > (T)0 && std::isfinite(r) && r * v == (T)1) ? r : (T)0;
}

template <typename T>
Params<T> params(const cbm_ctx* c, int parity) {
  using V4 = typename V4T<T>::type;
  Params<T> P;
  memset(&P, 0, sizeof P);
  const cbm_config& k = c->cfg;
  const int p = parity, q = parity ^ 1;
  P.PA = (V4*)c->PA;
  P.PB = (V4*)c->PB;
  P.VA = (T*)c->VA;
  P.VB = (T*)c->VB;
  P.FA = (V4*)c->FA;
  P.FB = (V4*)c->FB;
  P.IA = c->IA;
  P.IB = c->IB;
  P.U = (V4*)c->U;
  P.stage_h = (V4*)c->stage[0];
  P.stage_s = (V4*)c->stage[1];
  P.stage_k = (V4*)c->stage[2];
  P.POLD = (V4*)c->POLD;
  P.inv = c->inv;
  P.cell_of_slot = c->cell_of_slot;
  P.G = (T*)c->G;
  P.ID = c->ID;
  P.PAR = c->PAR;
  for (int d = 0; d < 3; ++d) {
    P.hx[d] = (T*)c->hx[d];
    P.hf[d] = (T*)c->hf[d];
    P.grad_cur[d] = (T*)c->grad[p][d];
    P.grad_nxt[d] = (T*)c->grad[q][d];
  }
  P.hv = (T*)c->hv;
  P.fate = c->fate;
  P.holes = c->holes;
  P.fate_state = c->fate_state;
  P.noise = c->ext_noise_on ? (const T*)c->ext_noise : nullptr;
  P.s_cell = c->s_cell;
  P.s_rank = c->s_rank;
  P.s_key = c->s_key;
  P.cell_count = c->cell_count;
  P.cell_start = c->cell_start;
  P.gather_box = c->gather_box;
  P.scan_state = c->scan_state;
  P.nbr_n = c->nbr_n;
  P.nbr_list = c->nbr_list;
  P.pair_list = (int4*)c->pair_list;
  P.pair_cap4 = kPairCap4;
  P.PA32 = (float4*)c->pos32;
  P.PS = (float*)c->pos_rows;
  P.ps_stride = c->rows_stride;
  P.c_cur = (T*)c->c[p];
  P.c_nxt = (T*)c->c[q];
  P.ctr = c->ctr;
  P.n_max = (int)k.n_max;
  P.n_blocks = c->n_blocks;
  P.n_cells = c->n_cells;
  for (int d = 0; d < 3; ++d) {
    P.n_cells_d[d] = c->n_cells_d[d];
    P.n_medium[d] = d < k.dims && k.medium ? k.n_medium[d] : 1;
    P.box_lo[d] = (T)k.box_lo[d];
    P.box_hi[d] = (T)k.box_hi[d];
    // dx = (hi - lo) / NMedium in Float64 (communityStructure.jl:274)
    P.dx_m[d] = d < k.dims && k.medium ? (T)((k.box_hi[d] - k.box_lo[d]) / (double)k.n_medium[d])
                                       : (T)1;
  }
  P.exact_scale = k.medium ? 1 : 0;
  for (int d = 0; d < 3; ++d) {
    P.inv_dx[d] = P.inv_dx2[d] = P.inv_2dx[d] = (T)0;
    if (d < k.dims && k.medium) {
      P.inv_dx[d] = exact_reciprocal<T>(P.dx_m[d]);
      P.inv_dx2[d] = exact_reciprocal<T>(P.dx_m[d] * P.dx_m[d]);
      P.inv_2dx[d] = exact_reciprocal<T>((T)2 * P.dx_m[d]);
      if (P.inv_dx2[d] == (T)0 || P.inv_2dx[d] == (T)0) P.exact_scale = 0;
    }
  }
  P.n_scan_tiles = c->n_scan_tiles;
  P.n_nodes = c->n_nodes;
  P.max_nbrs = k.n_max_neighbors;
  P.parity = parity;
  P.neighbors = k.neighbors;
  P.integrator = k.integrator;
  P.force_mode = k.force_mode;
  P.att_form = k.att_form;
  P.walls = k.walls;
  P.fate_rule = k.fate;
  P.growth = k.growth;
  P.medium = k.medium;
  P.medium_sampling = k.medium_sampling;
  P.dt = (T)k.dt;
  P.dt_time = k.dt;
  P.sqrt_dt = std::sqrt((T)k.dt);
  P.sigma = (T)k.sigma;
  P.edge = (T)(k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT ? k.skin : k.cell_edge);
  P.skin = (T)k.skin;
  P.rebuild_thr = k.rebuild_threshold > 0 ? (T)k.rebuild_threshold : (T)k.skin / (T)2;
  P.k_rep = (T)k.k_rep;
  P.r_rep = (T)k.r_rep;
  P.k_att = (T)k.k_att;
  P.r_att = (T)k.r_att;
  P.cut2 = bound2<T>(k.r_rep > k.r_att ? k.r_rep : k.r_att);
  P.skin2 = bound2<T>(k.skin);
  P.skin2_lo = bound2_lo<T>(k.skin);
  P.force_in_list = (T)(k.r_rep > k.r_att ? k.r_rep : k.r_att) <= (T)k.skin ? 1 : 0;
  P.cut_reach = (T)((k.r_rep > k.r_att ? k.r_rep : k.r_att) * (1.0 + 1e-4));
  P.skin_reach = (T)(k.skin * (1.0 + 1e-4));
  P.wall_force = (T)k.wall_force;
  P.wall_range = (T)k.wall_range;
  P.drift_linear = (T)k.drift_linear;
  P.v_div = (T)k.v_div;
  P.div_sep = (T)k.div_sep;
  P.p_death = (T)k.p_death;
  P.diff_D = (T)k.diff_D;
  P.decay = (T)k.decay;
  P.secretion_amt = (T)k.secretion * (T)k.dt;
  P.uptake_amt = (T)k.uptake * (T)k.dt;
  P.chemotaxis = (T)k.chemotaxis;
  P.seed = k.seed;
  P.community = k.community;
  return P;
}

// agents add to the medium (secretion) or take from it (uptake)
bool exchanges(const cbm_config& k) { return k.medium && (k.secretion != 0 || k.uptake != 0); }
bool uses_gather(const cbm_config& k) {
  return exchanges(k) && k.medium_sampling == CBM_MEDIUM_BILINEAR &&
         k.neighbors == CBM_NEIGH_CELL_LINKED;
}
bool rule_needed(const cbm_config& k) {
  return k.walls == CBM_WALLS_REFLECT || (exchanges(k) && !uses_gather(k)) ||
         k.fate != CBM_FATE_NONE;
}
// the atomic rule path reads the committed field from a snapshot
bool needs_snapshot(const cbm_config& k) { return k.uptake != 0 && exchanges(k) && !uses_gather(k); }

// blocks of the 2D shared-memory stencils (one tile per block)
dim3 stencil_grid(const cbm_ctx* c) {
  const int nx = c->cfg.n_medium[0] > 0 ? c->cfg.n_medium[0] : 1;
  const int ny = c->cfg.n_medium[1] > 0 ? c->cfg.n_medium[1] : 1;
  return dim3((unsigned)((nx + kStX - 1) / kStX), (unsigned)((ny + kStTileY - 1) / kStTileY));
}

// z planes per block of the 3D stencils: about twelve blocks for every SM
// (two to three waves of the TMA-fed blocks, five or six of which are
// resident; each block works through its planes one after another, so more
// and shorter runs keep more planes in flight: measured 0.061 ms at four,
// 0.051 ms at twelve for the 256^3 FTCS step), and runs of at least 8
// planes (each run also reads the two planes that close it)
int stencil_z_run(const cbm_ctx* c) {
  const dim3 g = stencil_grid(c);
  const long long xy = (long long)g.x * g.y;
  const int nz = c->cfg.n_medium[2] > 0 ? c->cfg.n_medium[2] : 1;
  const long long want = 12LL * (c->n_sm > 0 ? c->n_sm : 148);
  long long runs = (want + xy - 1) / xy;
  if (runs < 1) runs = 1;
  long long z_run = (nz + runs - 1) / runs;
  if (z_run < 8) z_run = 8;
  return (int)z_run;
}
dim3 stencil_grid_3d(const cbm_ctx* c) {
  dim3 g = stencil_grid(c);
  const int nz = c->cfg.n_medium[2] > 0 ? c->cfg.n_medium[2] : 1;
  const int zr = stencil_z_run(c);
  g.z = (unsigned)((nz + zr - 1) / zr);
  return g;
}

// Tensor maps of the two medium buffers for the TMA-fed 3D stencils: the
// field as an (nx, ny, nz) array of reals, boxes of one plane of a column
// tile (TmaPlane), zeros outside.  Needs rows of a multiple of 16 bytes (the
// strides of a tensor map); other shapes keep the register-pipelined
// stencils.  cuTensorMapEncodeTiled is reached through the runtime's driver
// entry point, so the library does not link the driver library itself.
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                   const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                   const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                   CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled_fn() {
  static EncodeTiledFn fn = []() -> EncodeTiledFn {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      return nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

template <typename T>
bool encode_medium_maps(cbm_ctx* c) {
  using G = TmaPlane<T>;
  const cbm_config& k = c->cfg;
  if (!k.medium || k.dims != 3) return false;
  const unsigned long long nx = k.n_medium[0], ny = k.n_medium[1], nz = k.n_medium[2];
  if ((nx * sizeof(T)) % 16 != 0) return false;
  EncodeTiledFn enc = encode_tiled_fn();
  if (!enc) return false;
  const cuuint64_t dim[3] = {nx, ny, nz};
  const cuuint64_t stride[2] = {nx * sizeof(T), nx * ny * sizeof(T)};
  const cuuint32_t box[3] = {(cuuint32_t)G::kBX, (cuuint32_t)G::kBY, 1};
  const cuuint32_t estride[3] = {1, 1, 1};
  for (int q = 0; q < 2; ++q)
    if (enc(&c->tmap_c[q],
            sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
            c->c[q], dim, stride, box, estride, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
      return false;
  return true;
}

// ---- stage launches (enqueue only) -----------------------------------------
template <typename T, int D>
void enqueue_medium_rule(cbm_ctx* c, const Params<T>& P) {
  if (c->cfg.medium && c->cfg.chemotaxis != 0) {
    PROF("k_medium_grad");
    if (D == 2)
      k_medium_grad_2d<T><<<stencil_grid(c), dim3(kStX, kStY), 0, c->stream>>>(P);
    else if (D == 3)
      if (c->tma_medium)
        k_medium_grad_3d_tma<T><<<stencil_grid_3d(c), dim3(kStX, kStY), TmaPlane<T>::kSmem,
                                  c->stream>>>(P, c->tmap_c[P.parity], stencil_z_run(c));
      else
        k_medium_grad_3d<T><<<stencil_grid_3d(c), dim3(kStX, kStY), 0, c->stream>>>(P, stencil_z_run(c));
    else
      k_medium_grad<T, D><<<grid_blocks(c->n_nodes), kTile, 0, c->stream>>>(P);
  }
}

template <typename T, int D>
void enqueue_agent_rule(cbm_ctx* c, const Params<T>& P, bool pdl_gather = false) {
  const cbm_config& k = c->cfg;
  if (needs_snapshot(k)) {
    PROF("k_medium_snapshot");
    k_medium_snapshot<T><<<grid_blocks(c->n_nodes), kTile, 0, c->stream>>>(P);
  }
  if (uses_gather(k)) {
    PROF("k_secrete_rows");
    const int nm[3] = {c->cfg.n_medium[0], D > 1 ? c->cfg.n_medium[1] : 1,
                       D > 2 ? c->cfg.n_medium[2] : 1};
    const int py = (nm[1] + GatherPatch<D>::kY - 1) / GatherPatch<D>::kY;
    constexpr int W = GatherPatch<D>::kWarps;
    const dim3 grid((unsigned)((nm[0] + 31) / 32), (unsigned)((py + W - 1) / W),
                    (unsigned)((nm[2] + GatherPatch<D>::kZ - 1) / GatherPatch<D>::kZ));
    launch_pdl(c, pdl_gather, k_secrete_rows<T, D>, grid, dim3(W * 32), 0, P);
  }
  if (!rule_needed(k)) return;
  if (k.fate != CBM_FATE_NONE) {
    PROF("k_agent_fate");
    k_agent_fate<T, D><<<fate_tiles(c->cfg.n_max), kTile, 0, c->stream>>>(P);
  } else {
    PROF("k_agent_rule");
    k_agent_rule<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(P);
  }
}

template <typename T, int D>
void enqueue_agent_de(cbm_ctx* c, const Params<T>& P) {
  const unsigned grid = kPartnerLists<D> ? c->de_blocks : c->n_blocks;
  const int integ = c->cfg.integrator;
  if (c->pos32) {
    PROF("k_pos32");
    k_pos32<T><<<c->n_blocks, kTile, 0, c->stream>>>(P);
  }
  if (c->pos_rows) {
    PROF("k_pos_rows");
    k_pos_rows<T><<<c->n_blocks, kTile, 0, c->stream>>>(P);
  }
  if (integ != CBM_INT_HEUN && integ != CBM_INT_RK4 && integ != CBM_INT_EULER_HEUN) {
    PROF("k_agent_de");
    k_agent_de<T, D><<<grid, kTile, 0, c->stream>>>(P);
    return;
  }
  // multi-stage: f at u, then at each stage's positions (own cell from the
  // position, no face pruning), each followed by its combination
  auto stage = [&](bool at_h, int op) {
    Params<T> Q = P;
    Q.KOUT = Q.stage_k;
    if (at_h) {
      Q.XS = Q.stage_h;
      Q.no_prune = 1;
    }
    {
      PROF("k_agent_de");
      k_agent_de<T, D><<<grid, kTile, 0, c->stream>>>(Q);
    }
    PROF("k_stage_combine");
    k_stage_combine<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(P, op);
  };
  if (integ == CBM_INT_HEUN) {
    stage(false, kHeunStage);
    stage(true, kHeunFinal);
  } else if (integ == CBM_INT_EULER_HEUN) {
    stage(false, kEhStage);
    stage(true, kEhFinal);
  } else {
    stage(false, kRk1);
    stage(true, kRk2);
    stage(true, kRk3);
    stage(true, kRkFinal);
  }
}

template <typename T, int D>
void enqueue_medium_de(cbm_ctx* c, const Params<T>& P, bool pdl = false) {
  if (c->cfg.medium) {
    PROF("k_medium_de");
    if (D == 2)
      launch_pdl(c, pdl, k_medium_de_2d<T>, stencil_grid(c), dim3(kStX, kStY), 0, P);
    else if (D == 3)
      if (c->tma_medium)
        launch_pdl(c, pdl, k_medium_de_3d_tma<T>, stencil_grid_3d(c), dim3(kStX, kStY),
                   (size_t)TmaPlane<T>::kSmem, P, c->tmap_c[P.parity], stencil_z_run(c));
      else
        launch_pdl(c, pdl, k_medium_de_3d<T>, stencil_grid_3d(c), dim3(kStX, kStY), 0, P,
                   stencil_z_run(c));
    else
      launch_pdl(c, pdl, k_medium_de<T, D>, dim3(grid_blocks(c->n_nodes)), dim3(kTile), 0, P);
  }
}

// update!: compaction, commit, then B -> A (copy, or re-sort = grid rebuild)
template <typename T, int D>
void enqueue_update(cbm_ctx* c, const Params<T>& P) {
  if (c->cfg.fate != CBM_FATE_NONE) {
    PROF("k_compact");
    k_compact<T, D><<<c->n_sm, kCompactThreads, 0, c->stream>>>(P);
  }
  {
    PROF("k_commit");
    k_commit<T><<<1, 1, 0, c->stream>>>(P);
  }
  // the four sort kernels follow one another on the stream
  {
    PROF("k_sort_hist");
    launch_pdl(c, true, k_sort_hist<T, D>, dim3(c->n_blocks), dim3(kTile), 0, P);
  }
  {
    PROF("k_scan_cells");
    ScanArgs A{c->cell_count, c->cell_start, c->scan_state, c->n_cells, c->n_scan_tiles, c->ctr,
               resort_flag(c)};
    launch_pdl(c, true, k_scan_cells, dim3(c->n_scan_tiles), dim3(kTile), 0, A);
  }
  {
    PROF("k_sort_scatter");
    launch_pdl(c, true, k_sort_scatter<T>, dim3(c->n_blocks), dim3(kTile), 0, P);
  }
  PROF("k_sort_place");
  launch_pdl(c, true, k_sort_place<T, D>, dim3(c->n_blocks), dim3(kTile), 0, P);
}

// computeNeighbors! after update!: the grid was rebuilt by the re-sort; a
// VerletDisplacement list is rebuilt eagerly (ascending agent order), a CLVD
// list is walked from the grid by the next DE stage.  Q has the parity of the
// step that starts.
template <typename T, int D>
void enqueue_neighbors(cbm_ctx* c, const Params<T>& Q) {
  if (c->cfg.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT) {
    PROF("k_verlet_list");
    k_verlet_list<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(Q, 1);
  }
}

int kernels_per_step(const cbm_ctx* c) {
  const cbm_config& k = c->cfg;
  int n = 0;
  if (k.medium && k.chemotaxis != 0) n += 1;
  if (needs_snapshot(k)) n += 1;
  if (uses_gather(k)) n += 1;
  if (rule_needed(k)) n += 1;           // rule (with births and deaths when fate is on)
  if (k.fate != CBM_FATE_NONE) n += 1;  // compaction
  n += 1;                               // agent DE
  if (c->pos32) n += 1;                 // its Float32 positions (Float64 3D walks)
  if (c->pos_rows) n += 1;              // its position rows (Float32 3D walks)
  if (k.medium) n += 1;
  n += 5;                               // commit, sort hist, scan, scatter, place
  if (k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT) n += 1;
  return n;
}

template <typename T, int D>
void enqueue_full_step(cbm_ctx* c, int parity, bool grad_ahead = false, bool next_grad = false) {
  Params<T> P = params<T>(c, parity);
  // The force kernel reads the committed positions and gradient and writes
  // the next state; the medium kernels read and write only the field and
  // its gradient.  With a medium the two run as parallel branches: the
  // force kernel on `side`, forked after the last kernel it depends on (the
  // agents' rule when there is one, else at the start of the step) and
  // joined before the update.  Per-kernel timing keeps them in series.  A
  // failed event call is seen like a failed launch (by the capture, or by
  // cudaGetLastError after an eager step).
  const bool fork = c->side && !c->prof;
  const bool early = fork && !rule_needed(c->cfg);
  auto agent_de = [&] {
    cudaEventRecord(c->fork_ev, c->stream);
    cudaStreamWaitEvent(c->side, c->fork_ev, 0);
    cudaStream_t main = c->stream;
    c->stream = c->side;
    enqueue_agent_de<T, D>(c, P);
    c->stream = main;
    cudaEventRecord(c->join_ev, c->side);
  };
  if (early) agent_de();
  // the gradient reads only the committed c: it may precede the secretion,
  // and in a chained graph the previous step enqueued it beside its update
  if (grad_ahead) cudaStreamWaitEvent(c->stream, c->grad_ev, 0);
  else enqueue_medium_rule<T, D>(c, P);
  // programmatic launches where the kernel before is one on this stream:
  // the secretion after the gradient, the FTCS after the secretion
  const bool grad_before = !grad_ahead && c->cfg.medium && c->cfg.chemotaxis != 0;
  enqueue_agent_rule<T, D>(c, P, grad_before && !needs_snapshot(c->cfg));
  if (!fork) enqueue_agent_de<T, D>(c, P);
  else if (!early) agent_de();
  enqueue_medium_de<T, D>(c, P, early && uses_gather(c->cfg) && !rule_needed(c->cfg));
  if (fork) cudaStreamWaitEvent(c->stream, c->join_ev, 0);
  if (next_grad) {
    // The next step's gradient reads the field just written and writes the
    // gradient buffer this step's force kernel has read (joined above); the
    // update touches neither, so the two run side by side.
    cudaEventRecord(c->grad_fork_ev, c->stream);
    cudaStreamWaitEvent(c->side2, c->grad_fork_ev, 0);
    cudaStream_t main = c->stream;
    c->stream = c->side2;
    enqueue_medium_rule<T, D>(c, params<T>(c, parity ^ 1));
    c->stream = main;
    cudaEventRecord(c->grad_ev, c->side2);
  }
  enqueue_update<T, D>(c, P);
  enqueue_neighbors<T, D>(c, params<T>(c, parity ^ 1));
}

// dispatch on (precision, dims)
template <template <typename, int> class Fn, typename... A>
void dispatch(cbm_ctx* c, A... a) {
  if (c->cfg.precision == CBM_F64) {
    switch (c->cfg.dims) {
      case 1: Fn<double, 1>::run(c, a...); break;
      case 2: Fn<double, 2>::run(c, a...); break;
      default: Fn<double, 3>::run(c, a...); break;
    }
  } else {
    switch (c->cfg.dims) {
      case 1: Fn<float, 1>::run(c, a...); break;
      case 2: Fn<float, 2>::run(c, a...); break;
      default: Fn<float, 3>::run(c, a...); break;
    }
  }
}

// resident blocks of the force kernel per multiprocessor
template <typename T, int D>
struct DEOccupancy {
  static void run(cbm_ctx*, int* bps) {
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(bps, k_agent_de<T, D>, kTile, 0) !=
            cudaSuccess ||
        *bps < 1)
      *bps = 1;
  }
};

template <typename T, int D>
struct FullStep {
  static void run(cbm_ctx* c, int parity) { enqueue_full_step<T, D>(c, parity); }
};
// kChainSteps steps from parity p; each step after the first takes the
// gradient its predecessor enqueued beside its update
template <typename T, int D>
struct ChainSteps {
  static void run(cbm_ctx* c, int parity) {
    for (int i = 0; i < kChainSteps; ++i)
      enqueue_full_step<T, D>(c, parity ^ (i & 1), i > 0, i + 1 < kChainSteps);
  }
};
template <typename T, int D>
struct StageRule {
  static void run(cbm_ctx* c) {
    Params<T> P = params<T>(c, c->parity);
    if (!c->mrule_done) enqueue_medium_rule<T, D>(c, P);
    enqueue_agent_rule<T, D>(c, P);
  }
};
template <typename T, int D>
struct StageDE {
  static void run(cbm_ctx* c) { enqueue_agent_de<T, D>(c, params<T>(c, c->parity)); }
};
template <typename T, int D>
struct StageMediumRule {
  static void run(cbm_ctx* c) { enqueue_medium_rule<T, D>(c, params<T>(c, c->parity)); }
};
template <typename T, int D>
struct StageMediumDE {
  static void run(cbm_ctx* c) { enqueue_medium_de<T, D>(c, params<T>(c, c->parity)); }
};
template <typename T, int D>
struct StageUpdate {
  static void run(cbm_ctx* c, int copy_agents, int use_u, int copy_c, int copy_grad) {
    Params<T> P = params<T>(c, c->parity);
    if (copy_agents) k_copy_ab<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(P, use_u);
    if (c->cfg.medium && (copy_c || copy_grad))
      k_copy_medium<T, D><<<grid_blocks(c->n_nodes), kTile, 0, c->stream>>>(P, copy_c ? 0 : 1);
    enqueue_update<T, D>(c, P);
  }
};
template <typename T, int D>
struct StageNeighbors {
  static void run(cbm_ctx* c) { enqueue_neighbors<T, D>(c, params<T>(c, c->parity)); }
};
template <typename T, int D>
struct BuildList {  // the list of the current slots, on request
  static void run(cbm_ctx* c) {
    k_verlet_list<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(params<T>(c, c->parity), 0);
  }
};
template <typename T, int D>
struct CountNeighbors {
  static void run(cbm_ctx* c, double radius, int* out) {
    k_count_neighbors<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(params<T>(c, c->parity),
                                                                  (T)radius, out);
  }
};
template <typename T, int D>
struct Pack {
  static void run(cbm_ctx* c, int N) {
    k_pack_upload<T, D><<<grid_blocks(N), kTile, 0, c->stream>>>(params<T>(c, c->parity), N);
  }
};
template <typename T, int D>
struct Gather {
  static void run(cbm_ctx* c, int N, int which) {
    k_gather_download<T, D><<<grid_blocks(N), kTile, 0, c->stream>>>(params<T>(c, c->parity), N,
                                                                      which);
  }
};
template <typename T, int D>
struct FirstSort {  // the re-sort half of update!, for loadToPlatform!
  static void run(cbm_ctx* c) {
    Params<T> P = params<T>(c, c->parity);
    k_sort_hist<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(P);
    ScanArgs A{c->cell_count, c->cell_start, c->scan_state, c->n_cells, c->n_scan_tiles, c->ctr,
               resort_flag(c)};
    k_scan_cells<<<c->n_scan_tiles, kTile, 0, c->stream>>>(A);
    k_sort_scatter<T><<<c->n_blocks, kTile, 0, c->stream>>>(P);
    k_sort_place<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(P);
    if (c->cfg.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT)
      k_verlet_list<T, D><<<c->n_blocks, kTile, 0, c->stream>>>(P, 0);
  }
};

int check_launch(cbm_ctx* c) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(c, CBM_ERR_CUDA, "kernel launch failed: %s", cudaGetErrorString(e));
  return CBM_OK;
}

void* dalloc(cbm_ctx* c, size_t bytes, bool* ok) {
  if (!*ok) return nullptr;
  if (bytes == 0) bytes = 16;
  void* p = nullptr;
  if (cudaMalloc(&p, bytes) != cudaSuccess) {
    *ok = false;
    return nullptr;
  }
  c->allocs.push_back(p);
  return p;
}

void free_all(cbm_ctx* c) {
  for (auto& m : c->marks) {
    cudaEventDestroy(m.ev[0]);
    cudaEventDestroy(m.ev[1]);
  }
  c->marks.clear();
  for (int q = 0; q < 2; ++q) {
    if (c->graph[q]) cudaGraphExecDestroy(c->graph[q]);
    if (c->tgraph[q]) cudaGraphExecDestroy(c->tgraph[q]);
    if (c->chain[q]) cudaGraphExecDestroy(c->chain[q]);
  }
  for (int q = 0; q < 2; ++q) {
    for (auto& m : c->gmarks[q]) {
      cudaEventDestroy(m.ev[0]);
      cudaEventDestroy(m.ev[1]);
    }
    c->gmarks[q].clear();
  }
  for (void* p : c->allocs) cudaFree(p);
  if (c->h_ctr) cudaFreeHost(c->h_ctr);
  c->h_ctr = nullptr;
  c->allocs.clear();
  if (c->side) cudaStreamDestroy(c->side);
  if (c->side2) cudaStreamDestroy(c->side2);
  for (cudaEvent_t e : {c->fork_ev, c->join_ev, c->grad_fork_ev, c->grad_ev})
    if (e) cudaEventDestroy(e);
  c->side = c->side2 = nullptr;
  c->fork_ev = c->join_ev = c->grad_fork_ev = c->grad_ev = nullptr;
  if (c->stream) cudaStreamDestroy(c->stream);
  c->stream = nullptr;
}

int flags_to_status(int err) {
  if (err & kErrAgentOverflow) return CBM_ERR_AGENT_OVERFLOW;
  if (err & kErrNeighborOverflow) return CBM_ERR_NEIGHBOR_OVERFLOW;
  if (err & kErrTimeout) return CBM_ERR_TIMEOUT;
  return CBM_OK;
}

int read_counters(cbm_ctx* c, Counters* h) {
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  CUDA_TRY(c, cudaMemcpy(h, c->ctr, sizeof(Counters), cudaMemcpyDeviceToHost));
  return CBM_OK;
}

void reset_stage_flags(cbm_ctx* c) {
  c->rule_done = c->de_done = c->mrule_done = c->mde_done = false;
}

// CLVD builds its list lazily; inspection calls build it when missing
int ensure_list(cbm_ctx* c) {
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  if (!hc.list_valid) {
    dispatch<BuildList>(c);
    rc = check_launch(c);
    if (rc) return rc;
    return cbm_sync(c);  // reports a row that exceeded n_max_neighbors
  }
  return CBM_OK;
}

}  // namespace

// ============================================================================
// C ABI
// ============================================================================
extern "C" {

const char* cbm_version(void) { return "cbm_b200 0.2.0 (sm_100a)"; }

const char* cbm_last_error(const cbm_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int cbm_create(cbm_ctx** out, const cbm_config* cfg) {
  if (!out || !cfg) return fail(nullptr, CBM_ERR_ARG, "null argument");
  *out = nullptr;
  const cbm_config& k = *cfg;
  if (k.dims < 1 || k.dims > 3) return fail(nullptr, CBM_ERR_ARG, "dims must be 1, 2 or 3");
  if (k.precision != CBM_F32 && k.precision != CBM_F64)
    return fail(nullptr, CBM_ERR_ARG, "precision must be CBM_F32 or CBM_F64");
  if (k.n_max < 0 || k.n_max >= (1ll << 30))
    return fail(nullptr, CBM_ERR_ARG, "n_max must be in [0, 2^30)");
  // the births/deaths scan packs two prefix counts of up to 2 n_max into 29 bits each
  if (k.fate != CBM_FATE_NONE && k.n_max >= (1ll << 28))
    return fail(nullptr, CBM_ERR_ARG, "with births and deaths n_max must be below 2^28");
  if (!(k.dt > 0)) return fail(nullptr, CBM_ERR_ARG, "dt must be positive");
  if (k.neighbors < CBM_NEIGH_NONE || k.neighbors > CBM_NEIGH_CLVD)
    return fail(nullptr, CBM_ERR_ARG, "unknown neighbor algorithm %d", k.neighbors);
  if (k.integrator < CBM_INT_EULER || k.integrator > CBM_INT_EULER_HEUN)
    return fail(nullptr, CBM_ERR_ARG, "unknown integrator %d", k.integrator);
  const bool multistage = k.integrator == CBM_INT_HEUN || k.integrator == CBM_INT_RK4 ||
                          k.integrator == CBM_INT_EULER_HEUN;
  if (multistage) {
    if (k.integrator != CBM_INT_EULER_HEUN && k.sigma != 0)
      return fail(nullptr, CBM_ERR_ARG, "Heun and RungeKutta4 integrate ODEs: sigma must be 0");
    if (k.force_mode == CBM_FORCE_LAGGED)
      return fail(nullptr, CBM_ERR_ARG, "multi-stage integrators need force_mode = CBM_FORCE_DIRECT");
    if (k.neighbors == CBM_NEIGH_CLVD)
      return fail(nullptr, CBM_ERR_ARG,
                  "multi-stage integrators need neighbors NONE, FULL, CELL_LINKED or "
                  "VERLET_DISPLACEMENT");
  }
  for (int d = 0; d < k.dims; ++d)
    if (!(k.box_hi[d] > k.box_lo[d])) return fail(nullptr, CBM_ERR_ARG, "empty simBox on axis %d", d);
  const bool cells = k.neighbors == CBM_NEIGH_CELL_LINKED || k.neighbors == CBM_NEIGH_CLVD;
  const bool list = k.neighbors == CBM_NEIGH_CLVD || k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT;
  if (cells && !(k.cell_edge > 0)) return fail(nullptr, CBM_ERR_ARG, "cell_edge must be positive");
  if (list && !(k.skin > 0)) return fail(nullptr, CBM_ERR_ARG, "skin must be positive");
  if (k.neighbors == CBM_NEIGH_CLVD && k.cell_edge < k.skin)
    return fail(nullptr, CBM_ERR_ARG, "CLVD needs cell_edge >= skin");
  if (list && (k.n_max_neighbors < 1 ||
               (k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT && k.n_max_neighbors > kVdSortMax)))
    return fail(nullptr, CBM_ERR_ARG, "n_max_neighbors must be in [1, %d]",
                k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT ? kVdSortMax : (1 << 20));
  if (k.medium) {
    for (int d = 0; d < k.dims; ++d)
      if (k.n_medium[d] < 1) return fail(nullptr, CBM_ERR_ARG, "n_medium[%d] must be >= 1", d);
  }
  if (!(k.uptake >= 0) || k.uptake > 1e300)
    return fail(nullptr, CBM_ERR_ARG, "uptake must be finite and >= 0");
  if (k.uptake != 0 && !k.medium) return fail(nullptr, CBM_ERR_ARG, "uptake needs a medium");

  cbm_ctx* c = new cbm_ctx;
  c->cfg = k;
  c->tsize = k.precision == CBM_F64 ? 8 : 4;
  cudaGetDevice(&c->device);
  cudaDeviceGetAttribute(&c->n_sm, cudaDevAttrMultiProcessorCount, c->device);
  // Chained step graphs (a medium with a gradient, of at most
  // kChainMaxNodes nodes): the library's stream takes the greatest priority
  // and the branches keep the least, so that the update and the medium
  // chain go first and the force kernel and the next gradient fill the SMs
  // they leave (with equal priorities the chained 1024^2 chemotaxis step
  // measured 9-13 % slower).
  long long med_nodes = 1;
  for (int d = 0; d < k.dims && k.medium && med_nodes <= kChainMaxNodes; ++d)
    med_nodes *= k.n_medium[d] > 0 ? k.n_medium[d] : 1;  // stops past the bound: no overflow
  const bool chained = k.medium && k.chemotaxis != 0 && med_nodes <= kChainMaxNodes;
  int prio_least = 0, prio_greatest = 0;
  cudaError_t se = cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
  if (se == cudaSuccess)
    se = chained ? cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, prio_greatest)
                 : cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if (se != cudaSuccess) {
    int rc = fail(nullptr, CBM_ERR_CUDA, "cudaStreamCreate failed (is a CUDA device present?)");
    delete c;
    return rc;
  }
  if ((k.medium && (cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
                    cudaEventCreateWithFlags(&c->fork_ev, cudaEventDisableTiming) != cudaSuccess ||
                    cudaEventCreateWithFlags(&c->join_ev, cudaEventDisableTiming) != cudaSuccess)) ||
      (chained && (cudaStreamCreateWithFlags(&c->side2, cudaStreamNonBlocking) != cudaSuccess ||
                   cudaEventCreateWithFlags(&c->grad_fork_ev, cudaEventDisableTiming) != cudaSuccess ||
                   cudaEventCreateWithFlags(&c->grad_ev, cudaEventDisableTiming) != cudaSuccess))) {
    int rc = fail(nullptr, CBM_ERR_CUDA, "creating the branch streams of the step graph failed");
    free_all(c);
    delete c;
    return rc;
  }
  const size_t n = (size_t)(k.n_max > 0 ? k.n_max : 1);
  const size_t S = c->tsize, S4 = 4 * c->tsize;
  c->n_blocks = grid_blocks((long long)n);
  c->grid_exposed = cells;
  c->has_list = list;
  // slots are sorted by cell for every algorithm; without a grid there is one cell
  if (cells || k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT) {
    double e = k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT ? k.skin : k.cell_edge;
    long long nc = 1;
    for (int d = 0; d < k.dims; ++d) {
      // nCells_ = ceil((hi - lo) / edge + 2), neighbors.jl:605 (Float64 on the host)
      double v = std::ceil((k.box_hi[d] - k.box_lo[d]) / e + 2.0);
      if (!(v >= 1 && v < 2.0e9)) {
        int rc = fail(nullptr, CBM_ERR_ARG, "cell grid too large on axis %d", d);
        free_all(c);
        delete c;
        return rc;
      }
      c->n_cells_d[d] = (int)v;
      nc *= (long long)v;
    }
    if (nc >= (1ll << 31) - 1) {
      int rc = fail(nullptr, CBM_ERR_ARG, "cell grid has too many cells (%lld)", nc);
      free_all(c);
      delete c;
      return rc;
    }
    c->n_cells = (int)nc;
  }
  c->n_scan_tiles = (c->n_cells + kScanTile - 1) / kScanTile;
  if (k.medium) {
    long long nn = 1;
    for (int d = 0; d < k.dims; ++d) nn *= k.n_medium[d];
    if (nn >= (1ll << 31)) {
      int rc = fail(nullptr, CBM_ERR_ARG, "medium grid too large");
      free_all(c);
      delete c;
      return rc;
    }
    c->n_nodes = (int)nn;
  }

  bool ok = true;
  c->PA = dalloc(c, n * S4, &ok);
  c->PB = dalloc(c, n * S4, &ok);
  c->VA = dalloc(c, n * S, &ok);
  c->VB = dalloc(c, n * S, &ok);
  c->FA = dalloc(c, n * S4, &ok);
  c->FB = dalloc(c, n * S4, &ok);
  c->IA = (int*)dalloc(c, n * 4, &ok);
  c->IB = (int*)dalloc(c, n * 4, &ok);
  if (k.walls == CBM_WALLS_REFLECT) c->U = dalloc(c, n * S4, &ok);
  if (k.integrator == CBM_INT_HEUN || k.integrator == CBM_INT_RK4 ||
      k.integrator == CBM_INT_EULER_HEUN)
    for (int q = 0; q < 3; ++q) c->stage[q] = dalloc(c, n * S4, &ok);
  if (list) c->POLD = dalloc(c, n * S4, &ok);
  c->inv = (int*)dalloc(c, n * 4, &ok);
  c->cell_of_slot = (int*)dalloc(c, n * 4, &ok);
  c->G = dalloc(c, n * S, &ok);
  c->ID = (long long*)dalloc(c, n * 8, &ok);
  c->PAR = (long long*)dalloc(c, n * 8, &ok);
  for (int d = 0; d < 3; ++d) {
    c->hx[d] = dalloc(c, n * S, &ok);
    c->hf[d] = dalloc(c, n * S, &ok);
  }
  c->hv = dalloc(c, n * S, &ok);
  c->fate = (unsigned char*)dalloc(c, n, &ok);
  c->holes = (int*)dalloc(c, n * 4, &ok);
  c->fate_state = (unsigned long long*)dalloc(c, (size_t)c->n_blocks * 8, &ok);
  c->s_cell = (int*)dalloc(c, n * 4, &ok);
  c->s_rank = (int*)dalloc(c, n * 4, &ok);
  c->s_key = (int*)dalloc(c, n * 4, &ok);
  c->cell_count = (int*)dalloc(c, (size_t)c->n_cells * 4, &ok);
  c->cell_start = (int*)dalloc(c, ((size_t)c->n_cells + 1) * 4, &ok);
  c->scan_state = (unsigned long long*)dalloc(c, (size_t)c->n_scan_tiles * 8, &ok);
  c->scratch_int = (int*)dalloc(c, n * 4, &ok);
  {
    // one partner-list region per resident block of the force kernel
    int bps = 1;
    dispatch<DEOccupancy>(c, &bps);
    const long long resident = (long long)c->n_sm * bps;
    c->de_blocks = (int)(resident < c->n_blocks ? resident : c->n_blocks);
    if (cells && k.dims == 3)
      c->pair_list = dalloc(c, (size_t)c->de_blocks * kTile * kPairCap4 * sizeof(int4), &ok);
    if (cells && k.dims == 3 && c->tsize == 8) c->pos32 = dalloc(c, n * sizeof(float4), &ok);
    if (cells && k.dims == 3 && c->tsize == 4) {
      c->rows_stride = (int)((n + 3) & ~(size_t)3);  // rows start on 16 bytes
      c->pos_rows = dalloc(c, 3 * (size_t)c->rows_stride * sizeof(float), &ok);
    }
  }
  if (list) {
    c->nbr_n = (int*)dalloc(c, n * 4, &ok);
    c->nbr_list = (int*)dalloc(c, n * (size_t)k.n_max_neighbors * 4, &ok);
  }
  if (k.medium) {
    for (int q = 0; q < 2; ++q) {
      c->c[q] = dalloc(c, (size_t)c->n_nodes * S, &ok);
      for (int d = 0; d < 3; ++d) c->grad[q][d] = dalloc(c, (size_t)c->n_nodes * S, &ok);
    }
    size_t nb = 0;
    for (int d = 0; d < k.dims; ++d) nb += 2 * (size_t)k.n_medium[d];
    c->gather_box = (int*)dalloc(c, nb * 4, &ok);
  }
  c->ctr = (Counters*)dalloc(c, sizeof(Counters), &ok);
  if (ok && cudaMallocHost((void**)&c->h_ctr, sizeof(Counters)) != cudaSuccess) {
    c->h_ctr = nullptr;
    ok = false;
  }
  if (!ok) {
    int rc = fail(nullptr, CBM_ERR_NOMEM, "device allocation failed for n_max=%lld", (long long)k.n_max);
    free_all(c);
    delete c;
    return rc;
  }
  c->tma_medium = c->tsize == 8 ? encode_medium_maps<double>(c) : encode_medium_maps<float>(c);
  if (k.medium) {
    int nmax = 1;
    for (int d = 0; d < k.dims; ++d) nmax = k.n_medium[d] > nmax ? (int)k.n_medium[d] : nmax;
    const unsigned blocks = (unsigned)((nmax + 255) / 256);
    if (c->tsize == 8)
      k_gather_box<double><<<blocks, 256, 0, c->stream>>>(params<double>(c, 0), c->gather_box, k.dims);
    else
      k_gather_box<float><<<blocks, 256, 0, c->stream>>>(params<float>(c, 0), c->gather_box, k.dims);
  }
  cudaMemsetAsync(c->cell_count, 0, (size_t)c->n_cells * 4, c->stream);
  cudaMemsetAsync(c->scan_state, 0, (size_t)c->n_scan_tiles * 8, c->stream);
  cudaMemsetAsync(c->fate_state, 0, (size_t)c->n_blocks * 8, c->stream);
  cudaMemsetAsync(c->ctr, 0, sizeof(Counters), c->stream);
  if (cudaStreamSynchronize(c->stream) != cudaSuccess) {
    int rc = fail(nullptr, CBM_ERR_CUDA, "device initialisation failed");
    free_all(c);
    delete c;
    return rc;
  }
  *out = c;
  return CBM_OK;
}

void cbm_destroy(cbm_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  free_all(ctx);
  delete ctx;
}

// ids 1..N for an upload that gives none (Community numbers its agents from 1)
static __global__ void k_default_ids(long long* id, int n) {
  const int i = blockIdx.x * kTile + threadIdx.x;
  if (i < n) id[i] = (long long)i + 1;
}

int cbm_upload(cbm_ctx* c, const cbm_state_view* h) {
  if (!c || !h) return fail(c, CBM_ERR_ARG, "null argument");
  cudaSetDevice(c->device);
  const cbm_config& k = c->cfg;
  if (h->N < 0 || h->N > k.n_max)
    return fail(c, CBM_ERR_ARG, "N=%lld exceeds n_max=%lld", (long long)h->N, (long long)k.n_max);
  const size_t N = (size_t)h->N, S = c->tsize, nm = (size_t)k.n_max;
  for (int d = 0; d < k.dims; ++d)
    if (N && !h->pos[d]) return fail(c, CBM_ERR_ARG, "pos[%d] is NULL", d);
  if (k.growth && N && (!h->v || !h->g)) return fail(c, CBM_ERR_ARG, "growth needs v and g");
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  cudaStream_t st = c->stream;
  // the epochs of the counters being replaced, read before anything is
  // enqueued, so that the copies, the counters and the first sort follow one
  // another with one synchronisation at the end
  Counters old;
  CUDA_TRY(c, cudaMemcpy(&old, c->ctr, sizeof old, cudaMemcpyDeviceToHost));
  // staging: index order; absent fields are zeros (loadToPlatform! pads with
  // zeros), and so is every field beyond N.  A field given by the caller is
  // copied into [0, N) and cleared beyond it only.
  auto stage = [&](void* dst, const void* src, size_t elem) -> cudaError_t {
    const size_t from = (src && N) ? N : 0;
    cudaError_t e = cudaSuccess;
    if (from) e = cudaMemcpyAsync(dst, src, N * elem, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && nm > from)
      e = cudaMemsetAsync((char*)dst + from * elem, 0, (nm - from) * elem, st);
    return e;
  };
  for (int d = 0; d < 3; ++d) {
    CUDA_TRY(c, stage(c->hx[d], d < k.dims ? h->pos[d] : nullptr, S));
    CUDA_TRY(c, stage(c->hf[d], d < k.dims ? h->f[d] : nullptr, S));
  }
  CUDA_TRY(c, stage(c->hv, h->v, S));
  CUDA_TRY(c, stage(c->G, h->g, S));
  CUDA_TRY(c, stage(c->PAR, h->parent, 8));
  // ids: the caller's (copied straight from its array), else 1..N; zero beyond N
  CUDA_TRY(c, stage(c->ID, h->id, 8));
  if (N && !h->id) k_default_ids<<<grid_blocks((long long)N), kTile, 0, st>>>(c->ID, (int)N);
  if (k.medium) {
    const size_t nb = (size_t)c->n_nodes * S;
    for (int q = 0; q < 2; ++q) {
      if (h->medium_c) CUDA_TRY(c, cudaMemcpyAsync(c->c[q], h->medium_c, nb, cudaMemcpyHostToDevice, st));
      else CUDA_TRY(c, cudaMemsetAsync(c->c[q], 0, nb, st));
      for (int d = 0; d < 3; ++d) {
        if (d < k.dims && h->medium_grad[d])
          CUDA_TRY(c, cudaMemcpyAsync(c->grad[q][d], h->medium_grad[d], nb, cudaMemcpyHostToDevice, st));
        else CUDA_TRY(c, cudaMemsetAsync(c->grad[q][d], 0, nb, st));
      }
    }
  }
  CUDA_TRY(c, cudaMemsetAsync(c->cell_count, 0, (size_t)c->n_cells * 4, st));
  Counters hc;
  memset(&hc, 0, sizeof hc);
  hc.N[0] = hc.N[1] = h->N;
  hc.step[0] = hc.step[1] = h->step;
  hc.t[0] = hc.t[1] = h->t;
  hc.id_max = h->id_max > 0 ? h->id_max : h->N;
  hc.slots = h->N;
  hc.resort = 1;  // flagRecomputeNeighbors_ = [1] and computeNeighbors! at load (communityStructure.jl:480,648)
  hc.scan_epoch = old.scan_epoch + 1;  // keep the epoch monotonic so stale tile states never match
  hc.fate_epoch = old.fate_epoch + 1;
  *c->h_ctr = hc;  // pinned: the copy is ordered on the stream, without a wait
  CUDA_TRY(c, cudaMemcpyAsync(c->ctr, c->h_ctr, sizeof hc, cudaMemcpyHostToDevice, st));
  c->parity = 0;
  reset_stage_flags(c);
  c->loaded = true;
  c->n_loaded = h->N;
  dispatch<Pack>(c, (int)N);
  dispatch<FirstSort>(c);
  int rc = check_launch(c);
  if (rc) return rc;
  return cbm_sync(c);
}

int cbm_download(cbm_ctx* c, cbm_state_view* h, int32_t which) {
  if (!c || !h) return fail(c, CBM_ERR_ARG, "null argument");
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  const cbm_config& k = c->cfg;
  const int p = c->parity;
  const long long N = hc.N[p];
  if (h->capacity < N)
    return fail(c, CBM_ERR_ARG, "host capacity %lld < N=%lld", (long long)h->capacity, N);
  h->N = N;
  h->t = hc.t[p];
  h->step = hc.step[p];
  h->id_max = hc.id_max;
  const size_t S = c->tsize, nb = (size_t)N * S;
  const bool nw = which == CBM_VIEW_NEW;
  const int src = nw && c->de_done ? 1 : (nw && c->rule_done && c->U ? 2 : 0);
  if (N) {
    dispatch<Gather>(c, (int)N, src);
    rc = check_launch(c);
    if (rc) return rc;
  }
  // the copies follow the gather on the context's stream, one
  // synchronisation for all of them
  cudaStream_t st = c->stream;
  for (int d = 0; d < k.dims; ++d) {
    if (h->pos[d] && N) CUDA_TRY(c, cudaMemcpyAsync(h->pos[d], c->hx[d], nb, cudaMemcpyDeviceToHost, st));
    if (h->f[d] && N) CUDA_TRY(c, cudaMemcpyAsync(h->f[d], c->hf[d], nb, cudaMemcpyDeviceToHost, st));
  }
  if (h->v && N) CUDA_TRY(c, cudaMemcpyAsync(h->v, c->hv, nb, cudaMemcpyDeviceToHost, st));
  if (h->g && N) CUDA_TRY(c, cudaMemcpyAsync(h->g, c->G, nb, cudaMemcpyDeviceToHost, st));
  if (h->id && N) CUDA_TRY(c, cudaMemcpyAsync(h->id, c->ID, (size_t)N * 8, cudaMemcpyDeviceToHost, st));
  if (h->parent && N)
    CUDA_TRY(c, cudaMemcpyAsync(h->parent, c->PAR, (size_t)N * 8, cudaMemcpyDeviceToHost, st));
  if (k.medium) {
    const size_t mb = (size_t)c->n_nodes * S;
    const int qc = nw && c->mde_done ? p ^ 1 : p;
    const int qg = nw && c->mrule_done ? p ^ 1 : p;
    if (h->medium_c) CUDA_TRY(c, cudaMemcpyAsync(h->medium_c, c->c[qc], mb, cudaMemcpyDeviceToHost, st));
    for (int d = 0; d < k.dims; ++d)
      if (h->medium_grad[d])
        CUDA_TRY(c, cudaMemcpyAsync(h->medium_grad[d], c->grad[qg][d], mb, cudaMemcpyDeviceToHost, st));
  }
  CUDA_TRY(c, cudaStreamSynchronize(st));
  return CBM_OK;
}

int cbm_agent_step_rule(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  dispatch<StageRule>(c);
  if (c->cfg.medium && c->cfg.chemotaxis != 0) c->mrule_done = true;
  c->rule_done = true;
  return check_launch(c);
}

int cbm_agent_step_de(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  const cbm_config& k = c->cfg;
  if (!c->rule_done && k.walls == CBM_WALLS_REFLECT)
    CUDA_TRY(c, cudaMemcpyAsync(c->U, c->PA, (size_t)k.n_max * 4 * c->tsize,
                                cudaMemcpyDeviceToDevice, c->stream));
  dispatch<StageDE>(c);
  c->de_done = true;
  return check_launch(c);
}

int cbm_medium_step_rule(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  if (!c->mrule_done) dispatch<StageMediumRule>(c);
  if (c->cfg.medium && c->cfg.chemotaxis != 0) c->mrule_done = true;
  return check_launch(c);
}

int cbm_medium_step_de(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  dispatch<StageMediumDE>(c);
  if (c->cfg.medium) c->mde_done = true;
  return check_launch(c);
}

int cbm_update(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  const cbm_config& k = c->cfg;
  int copy_agents = c->de_done ? 0 : 1;
  int use_u = (c->rule_done && k.walls == CBM_WALLS_REFLECT) ? 1 : 0;
  int copy_c = (k.medium && !c->mde_done) ? 1 : 0;
  int copy_grad = (k.medium && !c->mrule_done) ? 1 : 0;
  dispatch<StageUpdate>(c, copy_agents, use_u, copy_c, copy_grad);
  c->parity ^= 1;
  reset_stage_flags(c);
  return check_launch(c);
}

int cbm_compute_neighbors(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  dispatch<StageNeighbors>(c);
  return check_launch(c);
}

int cbm_sync(cbm_ctx* c) {
  if (!c) return CBM_ERR_ARG;
  cudaSetDevice(c->device);
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  if (hc.err) {
    int code = flags_to_status(hc.err);
    int zero = 0;
    CUDA_TRY(c, cudaMemcpy(&c->ctr->err, &zero, sizeof zero, cudaMemcpyHostToDevice));
    const char* what = code == CBM_ERR_AGENT_OVERFLOW
                           ? "agent capacity n_max reached: births were dropped"
                           : code == CBM_ERR_NEIGHBOR_OVERFLOW
                                 ? "a Verlet row exceeded n_max_neighbors: list truncated"
                                 : "a bounded device-side wait gave up";
    return fail(c, code, "%s (device flags 0x%x)", what, hc.err);
  }
  return CBM_OK;
}

}  // extern "C"

// A fate-free CellLinked community small enough for one cluster launch of all
// its steps (cbm_small.cuh)
bool small_eligible(const cbm_ctx* c) {
  const cbm_config& k = c->cfg;
  return k.neighbors == CBM_NEIGH_CELL_LINKED && k.fate == CBM_FATE_NONE && !k.growth &&
         !k.medium && k.force_mode == CBM_FORCE_DIRECT &&
         (k.integrator == CBM_INT_EULER || k.integrator == CBM_INT_EM) &&
         c->n_cells <= kSmallMaxCells && c->n_loaded > 0 && c->n_loaded <= kSmallMaxAgents;
}

template <typename T, int D>
struct SmallSteps {
  static void run(cbm_ctx* c, int nsteps, cudaError_t* err) {
    Params<T> P0 = params<T>(c, c->parity), P1 = params<T>(c, c->parity ^ 1);
    int n_cells = c->n_cells;
    const size_t smem = (size_t)(n_cells + 1) * sizeof(int);
    auto kern = k_small_steps<T, D>;
    // one cluster: as many blocks as four lanes an agent need, up to 16
    long long want = (c->n_loaded * kSmallLanes + kSmallThreads - 1) / kSmallThreads;
    int blocks = (int)std::max<long long>(1, std::min<long long>(want, kSmallMaxBlocks));
    *err = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (*err != cudaSuccess) return;
    cudaLaunchConfig_t lc = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    lc.blockDim = dim3(kSmallThreads);
    lc.dynamicSmemBytes = smem;
    lc.stream = c->stream;
    lc.attrs = attr;
    lc.numAttrs = 1;
    for (;; blocks /= 2) {  // the largest cluster the device can schedule
      attr[0].val.clusterDim.x = (unsigned)blocks;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      lc.gridDim = dim3((unsigned)blocks);
      int clusters = 0;
      if ((cudaOccupancyMaxActiveClusters(&clusters, kern, &lc) == cudaSuccess && clusters > 0) ||
          blocks == 1)
        break;
    }
    *err = cudaLaunchKernelEx(&lc, kern, P0, P1, nsteps, n_cells);
  }
};

extern "C" {

int cbm_step(cbm_ctx* c, int32_t nsteps, int32_t flags) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  if (nsteps < 0) return fail(c, CBM_ERR_ARG, "nsteps must be >= 0");
  cudaSetDevice(c->device);
  if (c->rule_done || c->de_done || c->mrule_done || c->mde_done)
    return fail(c, CBM_ERR_STATE, "a step is half done through the stage calls; call cbm_update first");
  const bool use_graph = !(flags & CBM_NO_GRAPH);
  if (use_graph && nsteps > 0 && !c->graph_timing && small_eligible(c)) {
    cudaError_t e = cudaSuccess;
    dispatch<SmallSteps>(c, (int)nsteps, &e);
    if (e != cudaSuccess) return fail(c, CBM_ERR_CUDA, "small-community launch failed: %s", cudaGetErrorString(e));
    if (nsteps & 1) c->parity ^= 1;
    if (flags & CBM_SYNC) return cbm_sync(c);
    return CBM_OK;
  }
  for (int s = 0; s < nsteps; ++s) {
    const int p = c->parity;
    if (use_graph && !c->graph_timing && c->side2 && nsteps - s >= kChainSteps) {
      if (!c->chain[p]) {
        cudaGraph_t g = nullptr;
        CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        dispatch<ChainSteps>(c, p);
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (e != cudaSuccess) return fail(c, CBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        // the nodes keep the priorities of the streams they were captured on
        e = cudaGraphInstantiate(&c->chain[p], g, cudaGraphInstantiateFlagUseNodePriority);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(c, CBM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
      }
      CUDA_TRY(c, cudaGraphLaunch(c->chain[p], c->stream));
      s += kChainSteps - 1;  // an even count: the parity is unchanged
      continue;
    }
    if (use_graph) {
      cudaGraphExec_t* graphs = c->graph_timing ? c->tgraph : c->graph;
      if (!graphs[p]) {
        cudaGraph_t g = nullptr;
        CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
        if (c->graph_timing) {  // event records around each kernel become graph nodes
          c->prof = true;
          c->prof_set = &c->gmarks[p];
          c->prof_used = &c->gmark_used[p];
          c->gmark_used[p] = 0;
        }
        dispatch<FullStep>(c, p);
        c->prof = false;
        c->prof_set = nullptr;
        c->prof_used = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g);
        if (e != cudaSuccess) return fail(c, CBM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(e));
        e = cudaGraphInstantiate(&graphs[p], g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return fail(c, CBM_ERR_CUDA, "graph instantiate failed: %s", cudaGetErrorString(e));
      }
      CUDA_TRY(c, cudaGraphLaunch(graphs[p], c->stream));
    } else {
      dispatch<FullStep>(c, p);
      int rc = check_launch(c);
      if (rc) return rc;
    }
    c->parity ^= 1;
  }
  if (flags & CBM_SYNC) return cbm_sync(c);
  return CBM_OK;
}

int cbm_step_noise(cbm_ctx* c, const void* noise, int32_t flags) {
  if (!c) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  if (c->cfg.integrator != CBM_INT_EM)
    return fail(c, CBM_ERR_ARG, "external noise needs the Euler-Maruyama integrator");
  if (c->rule_done || c->de_done || c->mrule_done || c->mde_done)
    return fail(c, CBM_ERR_STATE, "a step is half done through the stage calls; call cbm_update first");
  cudaSetDevice(c->device);
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  const long long N = hc.N[c->parity];
  const size_t bytes = (size_t)N * (size_t)c->cfg.dims * c->tsize;
  if (N > 0 && !noise) return fail(c, CBM_ERR_ARG, "noise is NULL");
  if (!c->ext_noise) {
    CUDA_TRY(c, cudaMalloc(&c->ext_noise,
                           (size_t)(c->cfg.n_max > 0 ? c->cfg.n_max : 1) * c->cfg.dims * c->tsize));
    c->allocs.push_back(c->ext_noise);
  }
  if (bytes) CUDA_TRY(c, cudaMemcpyAsync(c->ext_noise, noise, bytes, cudaMemcpyHostToDevice, c->stream));
  c->ext_noise_on = true;  // read by params() for this step only; the step graphs keep the stream
  dispatch<FullStep>(c, c->parity);
  c->ext_noise_on = false;
  rc = check_launch(c);
  if (rc) return rc;
  c->parity ^= 1;
  // the host buffer is borrowed for the call only
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (flags & CBM_SYNC) return cbm_sync(c);
  return CBM_OK;
}

int cbm_get_counters(cbm_ctx* c, int64_t* N, int64_t* n_add, int64_t* n_remove, int64_t* id_max,
                     int32_t* flag_recompute, int64_t* stepc) {
  if (!c) return CBM_ERR_ARG;
  cudaSetDevice(c->device);
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  const int p = c->parity;
  if (N) *N = hc.N[p];
  if (n_add) *n_add = hc.n_add;
  if (n_remove) *n_remove = hc.n_remove;
  if (id_max) *id_max = hc.id_max;
  // flag of the step in flight, or of the step that just ended
  if (flag_recompute) *flag_recompute = (c->rule_done || c->de_done) ? hc.flag[p] : hc.flag[p ^ 1];
  if (stepc) *stepc = hc.step[p];
  return CBM_OK;
}

int cbm_grid_shape(cbm_ctx* c, int32_t* n3) {
  if (!c || !n3) return CBM_ERR_ARG;
  for (int d = 0; d < 3; ++d) n3[d] = c->grid_exposed ? c->n_cells_d[d] : 1;
  return CBM_OK;
}

int cbm_get_grid(cbm_ctx* c, int32_t* agent_cell, int32_t* cell_start, int32_t* cell_count,
                 int32_t* cell_agents) {
  if (!c) return CBM_ERR_ARG;
  if (!c->grid_exposed) return fail(c, CBM_ERR_STATE, "this neighbor algorithm has no cell grid");
  cudaSetDevice(c->device);
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  const long long N = hc.N[c->parity];
  std::vector<int> start((size_t)c->n_cells + 1), ia((size_t)N), inv((size_t)N), cos((size_t)N);
  CUDA_TRY(c, cudaMemcpy(start.data(), c->cell_start, start.size() * 4, cudaMemcpyDeviceToHost));
  if (N) {
    CUDA_TRY(c, cudaMemcpy(ia.data(), c->IA, (size_t)N * 4, cudaMemcpyDeviceToHost));
    CUDA_TRY(c, cudaMemcpy(inv.data(), c->inv, (size_t)N * 4, cudaMemcpyDeviceToHost));
    CUDA_TRY(c, cudaMemcpy(cos.data(), c->cell_of_slot, (size_t)N * 4, cudaMemcpyDeviceToHost));
  }
  for (int q = 0; q < c->n_cells; ++q) {
    if (cell_start) cell_start[q] = start[q];
    if (cell_count) cell_count[q] = start[q + 1] - start[q];
  }
  for (long long i = 0; i < N; ++i) {
    if (cell_agents) cell_agents[i] = ia[(size_t)i];  // slots are in cell order
    if (agent_cell) agent_cell[i] = cos[(size_t)inv[(size_t)i]];
  }
  return CBM_OK;
}

int cbm_get_neighbors(cbm_ctx* c, int32_t* counts, int32_t* list, int64_t cap) {
  if (!c) return CBM_ERR_ARG;
  if (!c->has_list) return fail(c, CBM_ERR_STATE, "this neighbor algorithm has no Verlet list");
  cudaSetDevice(c->device);
  int rc = ensure_list(c);
  if (rc) return rc;
  Counters hc;
  rc = read_counters(c, &hc);
  if (rc) return rc;
  const long long N = hc.N[c->parity];
  const long long M = c->cfg.n_max_neighbors, nmax = c->cfg.n_max;
  if (list && cap < N * M) return fail(c, CBM_ERR_ARG, "list capacity %lld < N*n_max_neighbors", (long long)cap);
  std::vector<int> n((size_t)N), ia((size_t)N), inv((size_t)N), col;
  if (N) {
    CUDA_TRY(c, cudaMemcpy(n.data(), c->nbr_n, (size_t)N * 4, cudaMemcpyDeviceToHost));
    CUDA_TRY(c, cudaMemcpy(ia.data(), c->IA, (size_t)N * 4, cudaMemcpyDeviceToHost));
    CUDA_TRY(c, cudaMemcpy(inv.data(), c->inv, (size_t)N * 4, cudaMemcpyDeviceToHost));
  }
  if (list && N) {
    col.resize((size_t)(nmax * M));
    CUDA_TRY(c, cudaMemcpy(col.data(), c->nbr_list, col.size() * 4, cudaMemcpyDeviceToHost));
  }
  for (long long i = 0; i < N; ++i) {
    const long long s = inv[(size_t)i];
    if (counts) counts[i] = n[(size_t)s];
    if (list)
      for (long long q = 0; q < M; ++q)
        list[i * M + q] = q < n[(size_t)s] ? ia[(size_t)col[(size_t)(q * nmax + s)]] : -1;
  }
  return CBM_OK;
}

int cbm_count_neighbors(cbm_ctx* c, double radius, int32_t* out) {
  if (!c || !out) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  cudaSetDevice(c->device);
  Counters hc;
  int rc = read_counters(c, &hc);
  if (rc) return rc;
  const long long N = hc.N[c->parity];
  dispatch<CountNeighbors>(c, radius, c->scratch_int);
  rc = check_launch(c);
  if (rc) return rc;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  if (N) CUDA_TRY(c, cudaMemcpy(out, c->scratch_int, (size_t)N * 4, cudaMemcpyDeviceToHost));
  return CBM_OK;
}

int cbm_rng_fill(cbm_ctx* c, int32_t kind, double a, double b, int64_t n, int64_t stepc, void* out) {
  if (!c || !out || n < 0) return CBM_ERR_ARG;
  if (kind < 0 || kind > 2) return fail(c, CBM_ERR_ARG, "kind must be 0, 1 or 2");
  cudaSetDevice(c->device);
  void* buf = nullptr;
  const size_t bytes = (size_t)(n > 0 ? n : 1) * c->tsize;
  CUDA_TRY(c, cudaMallocAsync(&buf, bytes, c->stream));
  const int blocks = grid_blocks(n);
  if (n > 0) {
    if (c->cfg.precision == CBM_F64)
      k_rng_fill<double><<<blocks, kTile, 0, c->stream>>>(c->cfg.seed, c->cfg.community, stepc, kind, a,
                                                         b, n, (double*)buf);
    else
      k_rng_fill<float><<<blocks, kTile, 0, c->stream>>>(c->cfg.seed, c->cfg.community, stepc, kind,
                                                        (float)a, (float)b, n, (float*)buf);
  }
  int rc = check_launch(c);
  if (!rc && n > 0) {
    cudaError_t e = cudaMemcpyAsync(out, buf, (size_t)n * c->tsize, cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) rc = fail(c, CBM_ERR_CUDA, "copy failed: %s", cudaGetErrorString(e));
  }
  cudaFreeAsync(buf, c->stream);
  cudaError_t e = cudaStreamSynchronize(c->stream);
  if (!rc && e != cudaSuccess) rc = fail(c, CBM_ERR_CUDA, "rng fill failed: %s", cudaGetErrorString(e));
  return rc;
}

void* cbm_stream(cbm_ctx* c) { return c ? (void*)c->stream : nullptr; }

int cbm_profile_step(cbm_ctx* c, int32_t max_kernels, float* ms, const char** names,
                     int32_t* n_kernels) {
  if (!c || !n_kernels) return CBM_ERR_ARG;
  if (!c->loaded) return fail(c, CBM_ERR_STATE, "community not uploaded");
  if (c->rule_done || c->de_done || c->mrule_done || c->mde_done)
    return fail(c, CBM_ERR_STATE, "a step is half done through the stage calls; call cbm_update first");
  cudaSetDevice(c->device);
  c->prof = true;
  c->mark_used = 0;
  dispatch<FullStep>(c, c->parity);
  c->prof = false;
  int rc = check_launch(c);
  if (rc) return rc;
  c->parity ^= 1;
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *n_kernels = (int32_t)c->mark_used;
  for (size_t q = 0; q < c->mark_used && (int)q < max_kernels; ++q) {
    float t = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&t, c->marks[q].ev[0], c->marks[q].ev[1]));
    if (ms) ms[q] = t;
    if (names) names[q] = c->marks[q].name;
  }
  return cbm_sync(c);
}

int cbm_kernels_per_step(cbm_ctx* c) { return c ? kernels_per_step(c) : 0; }

int cbm_set_kernel_timing(cbm_ctx* c, int32_t on) {
  if (!c) return CBM_ERR_ARG;
  cudaSetDevice(c->device);
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  c->graph_timing = on != 0;  // the two sets of step graphs are kept apart
  return CBM_OK;
}

int cbm_kernel_times(cbm_ctx* c, int32_t max_kernels, float* ms, const char** names,
                     int32_t* n_kernels) {
  if (!c || !n_kernels) return CBM_ERR_ARG;
  if (!c->graph_timing) return fail(c, CBM_ERR_STATE, "kernel timing is off (cbm_set_kernel_timing)");
  cudaSetDevice(c->device);
  const int p = c->parity ^ 1;  // the parity of the step replayed last
  if (!c->tgraph[p]) return fail(c, CBM_ERR_STATE, "no step graph has been replayed yet");
  CUDA_TRY(c, cudaStreamSynchronize(c->stream));
  *n_kernels = (int32_t)c->gmark_used[p];
  for (size_t q = 0; q < c->gmark_used[p] && (int)q < max_kernels; ++q) {
    float t = 0.f;
    CUDA_TRY(c, cudaEventElapsedTime(&t, c->gmarks[p][q].ev[0], c->gmarks[p][q].ev[1]));
    if (ms) ms[q] = t;
    if (names) names[q] = c->gmarks[p][q].name;
  }
  return CBM_OK;
}

}  // extern "C"
