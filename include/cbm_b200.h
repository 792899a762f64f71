/*
 * cbm_b200.h — C ABI of the B200 per-step path of CellBasedModels.jl.
 *
 * The reference runs one simulation step as (src/CommunityStructure/step.jl:96-107)
 *     agentStepRule! -> agentStepDE! -> mediumStepRule! -> mediumStepDE!
 *     -> modelStepRule! -> modelStepDE! -> update! -> computeNeighbors!
 * over a Community whose state lives on a Platform (src/platforms.jl:1-121).
 * This library is that Platform for one fixed model family (soft spheres with
 * repulsion/adhesion, Euler or Euler–Maruyama, volume growth with division and
 * death, an FTCS-diffused medium with secretion and chemotaxis), evaluated by
 * hand-written sm_100a kernels.  A Julia `B200 <: Platform` binds these entry
 * points with `ccall`; every entry point names the reference function it
 * replaces.
 *
 * Conventions
 *  - All functions return CBM_OK (0) or a CBM_ERR_* code; cbm_last_error()
 *    gives the message.  The device never traps: device-side faults of the
 *    model (capacity or neighbor-list overflow) are recorded in a flag word and
 *    reported at the next synchronising call.
 *  - Indices are 0-based inside the library; agent ids are kept as given.
 *  - Host pointers are borrowed for the duration of the call only.
 *  - One context = one CUDA stream; a context is not re-entrant.  Different
 *    contexts may be driven from different host threads.
 *  - Arrays of reals are `float` when cfg.precision == CBM_F32 and `double`
 *    when CBM_F64 (void* in the signatures).
 */
#ifndef CBM_B200_H
#define CBM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
#define CBM_OK 0
#define CBM_ERR_ARG 1              /* invalid argument or configuration */
#define CBM_ERR_CUDA 2             /* a CUDA runtime call failed */
#define CBM_ERR_AGENT_OVERFLOW 3   /* births dropped: N would exceed n_max */
#define CBM_ERR_NEIGHBOR_OVERFLOW 4 /* a Verlet row needed more than n_max_neighbors */
#define CBM_ERR_TIMEOUT 5          /* a bounded device-side wait gave up */
#define CBM_ERR_STATE 6            /* call out of order (e.g. step before upload) */
#define CBM_ERR_NOMEM 7            /* device allocation failed */

/* ---- enumerations ------------------------------------------------------- */
enum { CBM_F32 = 0, CBM_F64 = 1 };

/* src/neighbors.jl: Full :26, VerletDisplacement :310, CellLinked :587, CLVD :997 */
enum {
  CBM_NEIGH_NONE = 0,       /* no pair interactions */
  CBM_NEIGH_FULL = 1,       /* all pairs, ascending j            (neighbors.jl:36-38) */
  CBM_NEIGH_CELL_LINKED = 2, /* cell grid rebuilt every step     (neighbors.jl:587-979) */
  CBM_NEIGH_VERLET_DISPLACEMENT = 3, /* list, ascending j, rebuilt on displacement (:310-570) */
  CBM_NEIGH_CLVD = 4        /* list built over the cell grid, cell order (:997-1275) */
};

/* src/integrators.jl: Euler :465-505, EM :683-734, Heun :516-573,
 * RungeKutta4 :583-668, EulerHeun :744-814.  Heun and RungeKutta4 integrate
 * ODEs (sigma = 0); EulerHeun integrates the SDE as the reference's CPU path
 * does (the final update draws fresh noise).  The multi-stage integrators
 * evaluate f at every stage over the neighbor structure of the last rebuild;
 * they need neighbors NONE, FULL, CELL_LINKED or VERLET_DISPLACEMENT and
 * force_mode = CBM_FORCE_DIRECT. */
enum { CBM_INT_EULER = 0, CBM_INT_EM = 1, CBM_INT_HEUN = 2, CBM_INT_RK4 = 3, CBM_INT_EULER_HEUN = 4 };

/* How the pair force enters dt(x).
 *  DIRECT: dt(x) += F(d)/d * (x - x[j]) inside @loopOverNeighbors.
 *  LAGGED: fx__ accumulates the pair force; dt(x) = fx reads the value committed
 *          at the previous update! (docs/src/Aggregation.md:81-114). */
enum { CBM_FORCE_DIRECT = 0, CBM_FORCE_LAGGED = 1 };

/* Adhesion branch for r_rep <= d < r_att:
 *  FROM_REP: F = -k_att (d - r_rep)   (linear growth past contact)
 *  TO_ATT:   F = -k_att (r_att - d)   (docs/src/Aggregation.md:96-99) */
enum { CBM_ATT_FROM_REP = 0, CBM_ATT_TO_ATT = 1 };

/* Walls.  REFLECT: agentRule sets x = 2 lo - x / 2 hi - x.  PUSH: the ODE adds
 * +wall_force within wall_range of lo and -wall_force within wall_range of hi
 * (docs/src/Aggregation.md:101-111). */
enum { CBM_WALLS_NONE = 0, CBM_WALLS_REFLECT = 1, CBM_WALLS_PUSH = 2 };

/* Agent fate rule evaluated in agentStepRule!.
 *  VOLUME: if v >= v_div divide into two daughters at +-div_sep along a random
 *          unit vector with v/2 each (@addAgent x2 + @removeAgent, docs/src/
 *          Development.md:153-190), elseif uniform(0,1) < p_death die.
 *  ID_PARITY: odd ids die, even ids add one child that copies the parent
 *          (test/testCommunity.jl:239-316). */
enum { CBM_FATE_NONE = 0, CBM_FATE_VOLUME = 1, CBM_FATE_ID_PARITY = 2 };

/* Where agents read and write the medium.  NEAREST is the reference's
 * cellInMesh (src/metrics.jl:18-20); BILINEAR spreads over the two (four,
 * eight) surrounding medium nodes with multilinear weights w_q.
 *
 * Secretion and uptake happen in the agent rule, in agent order, as the
 * reference's `c__[node] += ...` statements would (auxiliar.jl:353-365): agent
 * i adds to each node q of its stencil
 *     w_q * (secretion * dt - (uptake * dt) * c_q)
 * where c_q is the committed value of node q (the field before this step's
 * rule), so the uptake is first order in the local concentration.  With
 * uptake = 0 the term is w_q * secretion * dt.  With uptake > 0 the medium's DE
 * step reads the field clamped at zero, max(c, 0), on every node: an uptake
 * larger than the node holds leaves it empty, never negative. */
enum { CBM_MEDIUM_NEAREST = 0, CBM_MEDIUM_BILINEAR = 1 };

/* cbm_step flags */
#define CBM_SYNC 1          /* synchronise and report device flags before returning */
#define CBM_NO_GRAPH 2      /* launch kernels one by one instead of replaying a graph */

/* cbm_download / cbm_upload `which` */
#define CBM_VIEW_COMMITTED 0 /* x  : values committed by the last update! */
#define CBM_VIEW_NEW 1       /* x__: values written by this step's rule / DE */

/* ---- configuration (ABM(...) + Community(...) keyword arguments) --------- */
typedef struct cbm_config {
  int32_t dims;          /* 1, 2 or 3 (ABM(dims, ...)) */
  int32_t precision;     /* CBM_F32 | CBM_F64 (src/constants.jl:1-4) */
  int64_t n_max;         /* agent capacity = N + preallocateAgents (nMax_) */
  double box_lo[3];      /* simBox[:,1] */
  double box_hi[3];      /* simBox[:,2] */
  double dt;
  uint64_t seed;         /* key of the counter-based stream (cbm_rng.h) */
  uint32_t community;    /* community index inside the random stream */
  int32_t neighbors;     /* CBM_NEIGH_* */
  int32_t n_max_neighbors; /* Verlet row capacity (nMaxNeighbors) */
  int32_t integrator;    /* CBM_INT_* */
  double cell_edge;      /* CellLinked / CLVD cellEdge */
  double skin;           /* Verlet list radius (the reference's `skin`) */
  double rebuild_threshold; /* rebuild when a displacement >= this; <= 0 means skin/2 */
  double sigma;          /* EM noise amplitude: dt(x) = sigma in agentSDE */
  int32_t force_mode;    /* CBM_FORCE_* */
  int32_t att_form;      /* CBM_ATT_* */
  double k_rep;          /* repulsion stiffness (k) */
  double r_rep;          /* repulsion range (2r) */
  double k_att;          /* adhesion stiffness (a) */
  double r_att;          /* interaction cutoff (3r); no pair term for d >= r_att */
  int32_t walls;         /* CBM_WALLS_* */
  int32_t fate;          /* CBM_FATE_* */
  double wall_force;
  double wall_range;
  double drift_linear;   /* dt(x) += -drift_linear * x  (test/testCommunity.jl:418-464) */
  int32_t growth;        /* 1: volume v is a DE variable with dt(v) = g */
  int32_t medium;        /* 1: coupled medium field c on an n_medium grid */
  double v_div;          /* division volume */
  double div_sep;        /* daughters at +-div_sep along the division axis */
  double p_death;        /* per-step death probability */
  int32_t n_medium[3];   /* NMedium; node spacing dx = (hi - lo) / n_medium */
  int32_t medium_sampling; /* CBM_MEDIUM_* */
  double diff_D;         /* medium diffusion coefficient */
  double decay;          /* medium decay rate lambda */
  double secretion;      /* amount per unit time each agent adds to c */
  double chemotaxis;     /* dt(x) += chemotaxis * dc/dx / (1 + |grad c|) */
  double uptake;         /* first-order uptake rate per agent (CBM_MEDIUM_* above) */
} cbm_config;

/* ---- state exchanged with the host (Community fields) ------------------- */
typedef struct cbm_state_view {
  int64_t N;             /* number of agents */
  int64_t capacity;      /* length of the host agent arrays (download) */
  double t;              /* time */
  int64_t step;          /* step counter: the random stream's step key */
  int64_t id_max;        /* idMax_ */
  void* pos[3];          /* x, y, z */
  void* v;               /* volume (growth) or NULL */
  void* g;               /* growth rate (growth) or NULL */
  void* f[3];            /* lagged force fx, fy, fz (CBM_FORCE_LAGGED) or NULL */
  int64_t* id;           /* ids or NULL (upload: NULL means 1..N) */
  int64_t* parent;       /* id of the parent at birth (0 = initial agent) or NULL */
  void* medium_c;        /* medium field, x fastest, prod(n_medium) nodes, or NULL */
  void* medium_grad[3];  /* committed gradient fields (chemotaxis) or NULL */
} cbm_state_view;

typedef struct cbm_ctx cbm_ctx;

/* ---- library ------------------------------------------------------------- */
const char* cbm_version(void);
/* Message of the last failed call on ctx (or of the last failed cbm_create
 * when ctx is NULL). */
const char* cbm_last_error(const cbm_ctx* ctx);

/* ---- lifetime ------------------------------------------------------------ */
/* Replaces ABM(...) + Community(...) + CBMNeighbors.initialize!
 * (src/AgentStructure/agentStructure.jl:131-304, src/CommunityStructure/
 * communityStructure.jl:108-186, src/neighbors.jl:601-619,1021-1047):
 * validates cfg and allocates every device buffer for n_max agents. */
int cbm_create(cbm_ctx** out, const cbm_config* cfg);
/* Frees the device buffers and the stream. */
void cbm_destroy(cbm_ctx* ctx);

/* loadToPlatform! (src/CommunityStructure/communityStructure.jl:606-654):
 * copies N agents (and the medium) to the device, zero-pads to n_max, resets
 * NAdd_/NRemove_/flagSurvive_, computes neighbors.  Synchronous. */
int cbm_upload(cbm_ctx* ctx, const cbm_state_view* host);
/* bringFromPlatform! (communityStructure.jl:663-712): copies the first N
 * agents back (which = CBM_VIEW_COMMITTED or CBM_VIEW_NEW).  Synchronous;
 * fails with CBM_ERR_ARG if host->capacity < N. */
int cbm_download(cbm_ctx* ctx, cbm_state_view* host, int32_t which);

/* ---- stepping (src/CommunityStructure/step.jl) ---------------------------- */
/* step! x nsteps (step.jl:96-107).  Enqueues the steps (as CUDA graph replays
 * unless CBM_NO_GRAPH) and returns; CBM_SYNC waits and reports device flags.
 * With a medium, the force kernel of a step runs beside the medium kernels,
 * and with a medium gradient on at most 2^22 nodes a call of 8 steps or more
 * replays graphs of 8 chained steps, in which each step's update runs beside
 * the next step's gradient; the results are those of the steps made one by
 * one. */
int cbm_step(cbm_ctx* ctx, int32_t nsteps, int32_t flags);
/* One step! whose Euler–Maruyama increments are given instead of drawn:
 * noise[i * dims + d] ~ N(0,1) for the N agents in index order, in the
 * context's precision (the agentSDE draws of integrators.jl:718-724, fed to
 * both this library and a CPU run).  Divisions and deaths keep their
 * counter-based draws.  Runs without the step graph; noise is borrowed for
 * the call only.  Needs integrator == CBM_INT_EM. */
int cbm_step_noise(cbm_ctx* ctx, const void* noise, int32_t flags);
/* The stages of step!, for custom loops (docs/src/Usage_Community.md:236-345) */
int cbm_agent_step_rule(cbm_ctx* ctx);   /* agentStepRule!  step.jl:6-14 */
int cbm_agent_step_de(cbm_ctx* ctx);     /* agentStepDE!    step.jl:51-59 */
int cbm_medium_step_rule(cbm_ctx* ctx);  /* mediumStepRule! step.jl:28-36 */
int cbm_medium_step_de(cbm_ctx* ctx);    /* mediumStepDE!   step.jl:81-89 */
int cbm_update(cbm_ctx* ctx);            /* update!         update.jl:310-320 */
int cbm_compute_neighbors(cbm_ctx* ctx); /* computeNeighbors! neighbors.jl:18 */
/* Waits for the stream and returns the first device flag as a status. */
int cbm_sync(cbm_ctx* ctx);

/* ---- inspection ----------------------------------------------------------- */
/* N, NAdd_, NRemove_, idMax_, flagRecomputeNeighbors_ and the step counter.
 * Synchronous. */
int cbm_get_counters(cbm_ctx* ctx, int64_t* N, int64_t* n_add, int64_t* n_remove,
                     int64_t* id_max, int32_t* flag_recompute, int64_t* step);
/* Number of cells per axis of the cell grid (nCells_, neighbors.jl:605). */
int cbm_grid_shape(cbm_ctx* ctx, int32_t* n_cells3);
/* CellLinked arrays (neighbors.jl:601-619), 0-based: cell of each agent
 * (N), first slot of each cell (prod(nCells)), agents per cell
 * (prod(nCells)), agent indices in cell order (N) (cellAssignedToAgent_). */
int cbm_get_grid(cbm_ctx* ctx, int32_t* agent_cell, int32_t* cell_start,
                 int32_t* cell_count, int32_t* cell_agents);
/* Verlet arrays (neighbors.jl:314-331): counts (N) and the row-major list
 * list[i * n_max_neighbors + k] (N x n_max_neighbors); cap = list length. */
int cbm_get_neighbors(cbm_ctx* ctx, int32_t* counts, int32_t* list, int64_t cap);
/* The reference's neighbor-counting rule (test/testCommunity.jl:359-415):
 * out[i] = number of neighbors j of i (per the configured algorithm) with
 * euclidean distance < radius. */
int cbm_count_neighbors(cbm_ctx* ctx, double radius, int32_t* out);

/* Fills out[n] with draws of the shared stream (cbm_rng.h) on the device:
 * kind 0 normal(mu=a, sigma=b), 1 uniform(a, b), 2 exponential(theta=a)
 * (src/random.jl:8-22).  out is a host array of the context's precision. */
int cbm_rng_fill(cbm_ctx* ctx, int32_t kind, double a, double b, int64_t n, int64_t step,
                 void* out);

/* The context's CUDA stream (cudaStream_t), for event timing by the caller. */
void* cbm_stream(cbm_ctx* ctx);
/* Number of kernels one step launches with this configuration. */
int cbm_kernels_per_step(cbm_ctx* ctx);
/* Runs one step! with kernels launched one by one, each bracketed by CUDA
 * events on the context's stream (the reference has no stage timers; its
 * evolve! only offers a progressMessage callback, step.jl:129,146).  Writes
 * up to max_kernels durations (ms) and static kernel names; *n_kernels gets
 * the number of kernels the step launched.  Synchronous. */
int cbm_profile_step(cbm_ctx* ctx, int32_t max_kernels, float* ms, const char** names,
                     int32_t* n_kernels);
/* Kernel timing inside the step graphs (no reference counterpart; the
 * reference has no stage timers).  With on != 0, cbm_step replays a second
 * set of step graphs (captured at first use) with a CUDA event recorded
 * before and after every kernel, which every replay records again; on = 0
 * goes back to the plain graphs, which stay as they were.  The small
 * communities' single launch is not used while timing is on.  Synchronises
 * the stream. */
int cbm_set_kernel_timing(cbm_ctx* ctx, int32_t on);
/* After a graph-replayed cbm_step with kernel timing on: the durations (ms)
 * and static names of the kernels of the last step replayed, up to
 * max_kernels; *n_kernels gets their number.  Synchronises the stream. */
int cbm_kernel_times(cbm_ctx* ctx, int32_t max_kernels, float* ms, const char** names,
                     int32_t* n_kernels);

/* ---- batched communities ----------------------------------------------------
 * Many independent communities (parameter sweeps, model fitting: the
 * reference's fitting drivers run one whole simulation per parameter set,
 * src/fitting/gridSearch.jl:19-65) advanced by one persistent kernel, each
 * step count captured as one CUDA graph.  Every community is a 3D Float32
 * soft-sphere community with Euler-Maruyama noise and CLVD neighbors whose
 * trajectory is bit-identical to the plain path (cbm_create) with
 * neighbors = CLVD, skin = cell_edge = cutoff + tuning.skin,
 * rebuild_threshold = tuning.skin / 2 (unless set) and the same `community`.
 * The base configuration gives dims = 3, precision = CBM_F32,
 * integrator = CBM_INT_EM, neighbors = CBM_NEIGH_CLVD, dt, seed,
 * n_max_neighbors, and an initial skin (list radius) and rebuild threshold. */
typedef struct cbm_community_desc {
  int64_t n;             /* agents (fixed: no division or death) */
  double box_lo[3];
  double box_hi[3];
  double k_rep, r_rep, k_att, r_att; /* force parameters, as in cbm_config */
  double sigma;          /* EM noise amplitude */
  uint32_t community;    /* index in the random stream */
  int32_t pad;
} cbm_community_desc;

typedef struct cbm_batch_tuning {
  int32_t threads;       /* threads per CTA (one CTA runs one community): 128..1024 */
  int32_t ctas_per_sm;   /* resident CTAs per SM of the persistent grid */
  double skin;           /* Verlet skin: list radius = cutoff + skin */
  double rebuild_threshold; /* displacement that triggers a rebuild; <= 0: skin / 2 */
  int32_t tile_agents;   /* communities of at most this many agents gather neighbor
                            positions from a shared-memory tile (12 B per agent,
                            at most 220 KiB); 0: every gather goes through L1/L2 */
  int32_t lanes_per_agent; /* lanes that share one agent's list and pair terms: 1, 2 or 4
                            (32, 16 or 8 agents a warp; 0 means 1); the terms are added
                            in list order whatever the lanes */
} cbm_batch_tuning;

typedef struct cbm_batch cbm_batch;

int cbm_batch_create(cbm_batch** out, const cbm_config* base, int32_t n_communities,
                     const cbm_community_desc* communities);
void cbm_batch_destroy(cbm_batch* b);
const char* cbm_batch_last_error(const cbm_batch* b);
/* loadToPlatform! / bringFromPlatform! of community c (positions only) */
int cbm_batch_upload(cbm_batch* b, int32_t c, const cbm_state_view* host);
int cbm_batch_download(cbm_batch* b, int32_t c, cbm_state_view* host);
/* nsteps steps of every community in one persistent launch (graph replay
 * unless CBM_NO_GRAPH); CBM_SYNC waits and reports device flags */
int cbm_batch_step(cbm_batch* b, int32_t nsteps, int32_t flags);
int cbm_batch_set_tuning(cbm_batch* b, const cbm_batch_tuning* tuning);
int cbm_batch_get_tuning(cbm_batch* b, cbm_batch_tuning* tuning);
/* Times trial_steps on a copy of the current state for every candidate
 * (threads x CTAs per SM x shared-memory tile x skin), keeps the fastest and
 * restores the state.  A candidate whose lists overflow is skipped. */
int cbm_batch_autotune(cbm_batch* b, int32_t trial_steps, cbm_batch_tuning* best);
void* cbm_batch_stream(cbm_batch* b);

/* ---- adjoint (differentiable trajectories) ---------------------------------
 * Exact gradients of L = mean((x_T - target)^2) over a trajectory of the 3D
 * soft-sphere Euler ODE (agentODE + CBMIntegrators.Euler,
 * src/integrators.jl:465-505) with respect to theta = (k_rep, k_att, r_rep)
 * — (k, a, equilibrium distance 2r) — and to the initial positions, by a
 * hand-written reverse sweep with step checkpointing: states are kept every
 * checkpoint_every steps and each segment is recomputed before it is swept
 * backwards.  The configuration must be dims = 3, Euler, CBM_FORCE_DIRECT,
 * CBM_ATT_FROM_REP, CBM_NEIGH_CELL_LINKED, without walls, fate, growth,
 * medium or drift; the cutoff r_att is held fixed in the derivative.  The
 * forward map is the plain path's, bit for bit.  Arrays are host arrays of
 * the configured precision (x, y, z each). */
typedef struct cbm_adjoint cbm_adjoint;
int cbm_adjoint_create(cbm_adjoint** out, const cbm_config* cfg);
void cbm_adjoint_destroy(cbm_adjoint* a);
const char* cbm_adjoint_last_error(const cbm_adjoint* a);
/* loss, dtheta[3] = dL/d(k_rep, k_att, r_rep); dx0 (may be NULL) = dL/dx0;
 * xT (may be NULL) = final positions */
int cbm_adjoint_run(cbm_adjoint* a, int64_t n, const void* const* x0, int32_t nsteps,
                    int32_t checkpoint_every, const void* const* target, double* loss,
                    double* dtheta, void* const* dx0, void* const* xT);
/* the same forward trajectory without the backward sweep (for timing) */
int cbm_adjoint_forward(cbm_adjoint* a, int64_t n, const void* const* x0, int32_t nsteps,
                        void* const* xT);
void* cbm_adjoint_stream(cbm_adjoint* a);

/* ---- implicit medium: Douglas–Gunn ADI ------------------------------------
 * CBMIntegrators.DGADI (src/integrators.jl:817-937) on a medium of n_fields
 * fields over n[0] x n[1] x n[2] nodes (x fastest; unused axes have 1 node).
 * One step, as DifferentialEquations.step!(::DGADI) (:875-933):
 *   1. the explicit part is added to every field, u .+= f(u) (no factor dt,
 *      as in the reference), with the medium model
 *        f_k = s (c_max - u_k) - decay_k u_k   at interior nodes, 0 on the border
 *      (s a static source field; the mediumODE of examples/Implementation.ipynb
 *      is decay = 0);
 *   2. one Thomas solve per axis, x then y then z, along the lines through
 *      interior nodes (tridiagonal{1,2,3}D{x,y,z}, :141-428), with
 *        sub = super = -D_k r,  main = 1 + 2 D_k r,
 *        r = dt / (dims * dx^2), dx = (box_hi - box_lo) / n of the LAST axis
 *      for every axis (the reference reads column [l, dims] of its table),
 *      and the two border nodes of each line as Dirichlet values.  In Float32
 *      the pivots 1.0 / (...) are Float64, as Julia promotes them.
 * Border nodes keep their uploaded values (the reference never writes them).
 * Every axis needs at least 4 nodes.  A medium whose field fits one SM's
 * shared memory runs all steps of a call in one launch; a larger one enqueues
 * one launch per axis and step. */
#define CBM_MEDIUM_MAX_FIELDS 8
typedef struct cbm_medium_config {
  int32_t dims;                           /* 1, 2 or 3 */
  int32_t precision;                      /* CBM_F32 or CBM_F64 */
  int32_t n[3];                           /* nodes per axis (NMedium) */
  int32_t n_fields;                       /* 1 .. CBM_MEDIUM_MAX_FIELDS */
  double box_lo[3], box_hi[3];            /* simBox */
  double dt;
  double diffusion[CBM_MEDIUM_MAX_FIELDS]; /* D_k (difussionCoefs) */
  double decay[CBM_MEDIUM_MAX_FIELDS];     /* decay_k */
  double c_max;                           /* target of the source term */
} cbm_medium_config;

typedef struct cbm_medium cbm_medium;
int cbm_medium_create(cbm_medium** out, const cbm_medium_config* cfg);
void cbm_medium_destroy(cbm_medium* m);
const char* cbm_medium_last_error(const cbm_medium* m);
/* fields: n_fields blocks of prod(n) reals (field k, then x fastest); source:
 * prod(n) reals, or NULL for s = 0.  Host arrays of the configured precision.
 * Sets t = 0. */
int cbm_medium_upload(cbm_medium* m, const void* fields, const void* source);
/* nsteps DGADI steps; flags & CBM_SYNC waits for them. */
int cbm_medium_step(cbm_medium* m, int32_t nsteps, int32_t flags);
/* fields as in upload; *t (if not NULL) = steps taken x dt since the upload. */
int cbm_medium_download(cbm_medium* m, void* fields, double* t);
void* cbm_medium_stream(cbm_medium* m);

/* ---- rods: the rods2D model (src/models/rods.jl) ---------------------------
 * 2D rods of diameter d, length l and mass m, after Volfson et al.  The ODE
 * of rods2D (rods.jl:86-118), integrated by Euler:
 *   dt(x) = vx, dt(y) = vy, dt(vx) = -beta vx + fx/m, dt(vy) = -beta vy + fy/m,
 *   dt(theta) = omega, dt(omega) = W/(m (d+l)^2/12 + m d^2) - beta_w omega,
 * where fx, fy, W (and pressure) are summed over the neighbors with
 * rodForces (:21-59) and CBMMetrics.rodIntersection (src/metrics.jl:128-246).
 * Assigned inside the ODE, they are written to the new copy and read lagged:
 * dt(vx) uses the fx committed by the previous step, as the reference's code
 * generator has it.  Neighbors: the CellLinked grid over the committed
 * positions (cell_edge), in the reference's order, or all pairs (FULL).
 * cos and sin are the library's own series (the same bits on host and
 * device); delta^1.5 = delta sqrt(delta), delta^0.5 = sqrt(delta). */
typedef struct cbm_rods_config {
  int32_t precision;        /* CBM_F32 or CBM_F64 */
  int32_t neighbors;        /* CBM_NEIGH_FULL or CBM_NEIGH_CELL_LINKED */
  int64_t n_max;            /* rod capacity */
  double box_lo[2], box_hi[2];
  double cell_edge;
  double dt;
  double kn, gamma_n, gamma_t, mu_cc, mu_cw, beta, beta_w;
  /* rods2dGrowth (rods.jl:123-163) when growth_model != 0:
   *   dt(l) = growth/(1 + alpha pressure), pressure lagged like fx;
   *   the rule, before the ODE: a rod with l > lTarget divides into two rods
   *   at x +- (l+d)/4 (cos, sin)(theta), l = (l-d)/2, omega +- ww,
   *   ww = uniform(-.1, .1), lTarget = uniform(l_max - sigma_l_target,
   *   l_max + sigma_l_target) each (the other fields are the parent's), and
   *   is removed; update! fills the holes from the tail as the reference.
   * uniform(a, b) = (b - a) u + a with u the shared stream of cbm_rng.h
   * (seed, step, parent index, CBM_STREAM_ROD_*). */
  int32_t growth_model;
  int32_t pad0;
  double growth, alpha, sigma_l_target, l_max;
  uint64_t seed;
} cbm_rods_config;

typedef struct cbm_rods cbm_rods;
int cbm_rods_create(cbm_rods** out, const cbm_rods_config* cfg);
void cbm_rods_destroy(cbm_rods* r);
const char* cbm_rods_last_error(const cbm_rods* r);
/* The per-rod fields, each an array of n reals of the configured precision,
 * in this order (CBM_RODS_FIELDS of them; pressure is read by download only;
 * lTarget is used by rods2dGrowth only). */
#define CBM_RODS_FIELDS 14
enum {
  CBM_ROD_X = 0, CBM_ROD_Y, CBM_ROD_VX, CBM_ROD_VY, CBM_ROD_THETA, CBM_ROD_OMEGA, CBM_ROD_D,
  CBM_ROD_L, CBM_ROD_M, CBM_ROD_FX, CBM_ROD_FY, CBM_ROD_W, CBM_ROD_PRESSURE, CBM_ROD_L_TARGET
};
/* fields[k] for k < CBM_ROD_PRESSURE are read (host arrays), and
 * fields[CBM_ROD_L_TARGET] with growth_model; sets the step to 0 */
int cbm_rods_upload(cbm_rods* r, int64_t n, const void* const* fields);
/* With growth_model, flags & CBM_SYNC also reports CBM_ERR_AGENT_OVERFLOW when
 * births were dropped for want of rows below n_max; as in the reference, the
 * step drops them in order and still removes every parent. */
int cbm_rods_step(cbm_rods* r, int32_t nsteps, int32_t flags);
/* fields[k] (host arrays of at least n reals, or NULL) receive the fields;
 * *n_out = n (with growth_model the current count, read back from the device) */
int cbm_rods_download(cbm_rods* r, void* const* fields, int64_t* n_out);
void* cbm_rods_stream(cbm_rods* r);

/* ---- allocation-free cell grid -------------------------------------------
 * This entry point has no counterpart in the reference.  It is for callers
 * that cannot allocate device memory when they need a grid: code running
 * while a framework captures the stream into a CUDA graph (cudaMalloc is
 * refused in a capturing thread), hosts whose device memory belongs to a pool
 * allocator that must account for every byte (such as a Julia process whose
 * CUDA.jl pool owns the GPU), and real-time loops that cannot wait for
 * cudaMalloc/cudaFree.
 *
 * It builds the same CellLinked grid as cbm_upload/cbm_compute_neighbors
 * (cellPos + counting sort, ascending agent index within a cell,
 * src/neighbors.jl:636-638,918-979) for n_agents positions x, y, z (device
 * arrays of the given precision; y/z may be NULL below 2/3 dims) and writes,
 * 0-based, agent_cell[n_agents], cell_start[prod(nCells) + 1] (the last entry
 * is n_agents) and cell_agents[n_agents], all caller-allocated device arrays.
 * Work is enqueued on `stream` (a cudaStream_t, NULL for the legacy default
 * stream); the call returns before it finishes.
 *
 * Scratch memory is a static device array inside the library (about 8.4 MB,
 * held by every GPU that loads the library until the process exits), so
 * n_agents <= CBM_NOALLOC_MAX_AGENTS and prod(nCells) <= CBM_NOALLOC_MAX_CELLS;
 * larger requests return CBM_ERR_ARG.  All calls share that array and it keeps
 * the last call's contents: calls that overlap on the GPU (on different
 * streams, or from different host threads without ordering) race and corrupt
 * each other's results.  The first call on a device looks up the array's
 * device address (once per device, with that device current); make that first
 * call before any stream capture begins.  Errors are described by
 * cbm_noalloc_last_error(). */
#define CBM_NOALLOC_MAX_AGENTS 524288
#define CBM_NOALLOC_MAX_CELLS 1048576
int cbm_cell_grid_noalloc(const void* x, const void* y, const void* z, int32_t n_agents,
                          int32_t dims, int32_t precision, const double* box_lo,
                          const double* box_hi, double cell_edge, int32_t* agent_cell,
                          int32_t* cell_start, int32_t* cell_agents, void* stream);
const char* cbm_noalloc_last_error(void);
/* Status of the last cbm_cell_grid_noalloc call on the current device: waits
 * for `stream` (the stream that call was given), then reads the error bits
 * that its kernels left in the static scratch array.  CBM_ERR_TIMEOUT means
 * the cell scan's bounded wait gave up and the grid it wrote is incomplete.
 * It synchronises the stream, so call it outside any stream capture.  It
 * allocates nothing.  The message of a failed call (of either function) is
 * kept per host thread and read with cbm_noalloc_last_error(). */
int cbm_noalloc_status(void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CBM_B200_H */
