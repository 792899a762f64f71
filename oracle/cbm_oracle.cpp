/*
 * cbm_oracle.cpp — TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference's per-step path (CellBasedModels.jl
 * v0.1.1, CPU platform), used by the tests and by bench.py's CPU baseline as
 * the checker.  Nothing in the product links, loads or calls this file.
 *
 * It follows the reference's data layout and loop order, 0-based:
 *   - committed agent arrays (x, v, fx ...) and their "__" copies, the
 *     DE state u, exactly as loadToPlatform!/linkVariables set them up
 *     (src/CommunityStructure/communityStructure.jl:606-654,724-743);
 *   - agentStepRule! as a serial loop over agents with @addAgent/@removeAgent
 *     (src/AgentStructure/functionRule.jl:9-111);
 *   - agentStepDE!: cleanArray, the generated f(du,u,p,t) with
 *     @loopOverNeighbors, then the Euler / EM update
 *     (src/integrators.jl:442-505,683-734, src/AgentStructure/functionDE.jl:13-117);
 *   - mediumStepRule!/mediumStepDE!: central difference and @∂2 FTCS with an
 *     Euler step u <- u + dt f(u) (src/AgentStructure/macros.jl:148-311);
 *   - update!: kernelListSurvived, kernelFillHolesParameters, commit
 *     (src/CommunityStructure/update.jl:15-298);
 *   - computeNeighbors!: CellLinked serial assign / cumsum / sort, Verlet
 *     displacement check + rebuild, CLVD list over the cell grid
 *     (src/neighbors.jl:92-133,367-570,636-979,1071-1131).
 *   - the implicit medium integrator DGADI: explicit part, then one Thomas
 *     solve per axis with u_new/c_star/d_star as the reference keeps them
 *     (src/integrators.jl:141-428,817-937).
 * Random draws come from the shared counter-based stream (include/cbm_rng.h)
 * so that the device path and this checker see the same numbers.
 *
 * Build: oracle/build.sh (g++ -O2 -ffp-contract=off -fopenmp).  Single-thread
 * and OpenMP runs give identical bits: every parallel loop writes per-agent
 * results whose summation order is fixed.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/cbm_b200.h"
#include "../include/cbm_rng.h"

namespace {

int g_threads = 1;

template <typename T>
struct Com {
  cbm_config cfg;
  int dims = 3;
  int64_t N = 0, nMax = 0, NAdd = 0, NRemove = 0, idMax = 0, step = 0;
  double t = 0;
  bool loaded = false;
  int err = 0;  // first model fault seen (CBM_ERR_*), sticky until read

  // agent arrays: committed and "__" (u rows for DE variables)
  std::vector<T> x[3], x_[3];
  std::vector<T> v, v_;
  std::vector<T> g;
  std::vector<T> f[3], f_[3];
  std::vector<int64_t> id, parent;
  std::vector<int64_t> flagSurvive, holeFromRemoveAt, repositionAgentInPos;
  int flagRecompute = 1;

  // neighbors
  int64_t nCells[3] = {1, 1, 1};
  T edge = 0;
  std::vector<int64_t> cellAssignedToAgent, cellNumAgents, cellCumSum;
  std::vector<int64_t> neighborN;
  std::vector<int32_t> neighborList;  // column-major (nMax x nMaxNeighbors); indices < 2^31
  std::vector<T> posOld[3], accumulatedDistance;
  const T* ext_noise = nullptr;  // EM increments given by the caller for one step (i * D + d)

  // medium: committed c, u (c__), gradient committed / new
  int64_t nm[3] = {1, 1, 1};
  int64_t nNodes = 0;
  T dxm[3] = {1, 1, 1};
  std::vector<T> c, c_, gr[3], gr_[3];

  std::vector<T> du[4];  // scratch of the integrator
};

template <typename T>
inline T rint_t(T a) { return std::rint(a); }
template <typename T>
inline T fmod_t(T a, T b) { return std::fmod(a, b); }

/* Julia's float `÷` (round((a - rem(a,b))/b)), a >= 0 here. */
template <typename T>
inline int64_t floordiv(T a, T b) {
  return (int64_t)rint_t((a - fmod_t(a, b)) / b);
}

/* cellPos, src/neighbors.jl:636-638 (0-based).  A NaN coordinate falls in
 * the first cell. */
template <typename T>
inline int64_t cellPos1(T edge, T x, T lo, T hi, int64_t n) {
  if (x > hi) return n - 1;
  if (!(x >= lo)) return 0;
  int64_t p = floordiv<T>(x - lo, edge) + 1;
  return p > n - 1 ? n - 1 : p;
}

/* cellInMesh, src/metrics.jl:18-20 (0-based, clamped at the top). */
template <typename T>
inline int64_t cellInMesh(T dx, T x, T lo, T hi, int64_t n) {
  if (x > hi) return n - 1;
  if (!(x >= lo)) return 0;
  int64_t p = floordiv<T>(x - lo, dx);
  return p > n - 1 ? n - 1 : p;
}

template <typename T>
inline T euclid(const Com<T>& C, const std::vector<T>* a, int64_t i, const std::vector<T>* b,
                int64_t j) {
  T s = 0;
  for (int d = 0; d < C.dims; ++d) {
    T e = a[d][i] - b[d][j];
    s = (d == 0) ? e * e : s + e * e;
  }
  return std::sqrt(s);
}

template <typename T>
int64_t cellOf(const Com<T>& C, const std::vector<T>* P, int64_t i) {
  int64_t lin = 0, mul = 1;
  for (int d = 0; d < C.dims; ++d) {
    int64_t p = cellPos1<T>(C.edge, P[d][i], (T)C.cfg.box_lo[d], (T)C.cfg.box_hi[d], C.nCells[d]);
    lin += p * mul;
    mul *= C.nCells[d];
  }
  return lin;
}

/* cellPosNeigh, src/neighbors.jl:658-708: k-th of 3^d neighbor cells, x
 * fastest, -1 outside the grid.  (2D uses nX for the row stride.) */
template <typename T>
int64_t cellNeigh(const Com<T>& C, int64_t pos, int k) {
  int64_t q[3] = {0, 0, 0};
  int64_t r = pos;
  for (int d = 0; d < C.dims; ++d) { q[d] = r % C.nCells[d]; r /= C.nCells[d]; }
  int off[3] = {k % 3 - 1, (k / 3) % 3 - 1, k / 9 - 1};
  int64_t lin = 0, mul = 1;
  for (int d = 0; d < C.dims; ++d) {
    int64_t p = q[d] + off[d];
    if (p < 0 || p >= C.nCells[d]) return -1;
    lin += p * mul;
    mul *= C.nCells[d];
  }
  return lin;
}

/* Walk the neighbors of agent i as @loopOverNeighbors does, with positions P
 * (u inside the DE, committed x inside a rule). */
template <typename T, typename F>
void forNeighbors(const Com<T>& C, const std::vector<T>* P, int64_t i, int64_t N, F&& body) {
  switch (C.cfg.neighbors) {
    case CBM_NEIGH_FULL:
      for (int64_t j = 0; j < N; ++j)
        if (j != i) body(j);
      break;
    case CBM_NEIGH_CELL_LINKED: {
      int64_t pos = cellOf(C, P, i);
      int nk = C.dims == 1 ? 3 : (C.dims == 2 ? 9 : 27);
      for (int k = 0; k < nk; ++k) {
        int64_t pn = cellNeigh(C, pos, k);
        if (pn < 0) continue;
        for (int64_t s = C.cellCumSum[pn] - C.cellNumAgents[pn]; s < C.cellCumSum[pn]; ++s) {
          int64_t j = C.cellAssignedToAgent[s];
          if (j != i) body(j);
        }
      }
      break;
    }
    case CBM_NEIGH_VERLET_DISPLACEMENT:
    case CBM_NEIGH_CLVD:
      for (int64_t k = 0; k < C.neighborN[i]; ++k) body(C.neighborList[i + k * C.nMax]);
      break;
    default:
      break;
  }
}

template <typename T>
void alloc(Com<T>& C) {
  const cbm_config& k = C.cfg;
  C.dims = k.dims;
  C.nMax = k.n_max;
  size_t n = (size_t)C.nMax;
  for (int d = 0; d < 3; ++d) {
    C.x[d].assign(n, 0); C.x_[d].assign(n, 0);
    C.f[d].assign(n, 0); C.f_[d].assign(n, 0);
    C.posOld[d].assign(n, 0);
  }
  C.v.assign(n, 0); C.v_.assign(n, 0); C.g.assign(n, 0);
  C.id.assign(n, 0); C.parent.assign(n, 0);
  C.flagSurvive.assign(n, 1); C.holeFromRemoveAt.assign(n, 0); C.repositionAgentInPos.assign(n, 0);
  for (int d = 0; d < 4; ++d) C.du[d].assign(n, 0);
  C.accumulatedDistance.assign(n, 0);
  C.edge = (T)(k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT ? k.skin : k.cell_edge);
  int64_t nc = 1;
  for (int d = 0; d < C.dims; ++d) {
    if (k.neighbors == CBM_NEIGH_CELL_LINKED || k.neighbors == CBM_NEIGH_CLVD) {
      // nCells_ = ceil((hi - lo)/edge + 2), src/neighbors.jl:605
      // evaluated in Float64 on the host in both reference platforms
      double e = k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT ? k.skin : k.cell_edge;
      C.nCells[d] = (int64_t)std::ceil((k.box_hi[d] - k.box_lo[d]) / e + 2.0);
    } else {
      C.nCells[d] = 1;
    }
    nc *= C.nCells[d];
  }
  C.cellAssignedToAgent.assign(n, 0);
  C.cellNumAgents.assign((size_t)nc, 0);
  C.cellCumSum.assign((size_t)nc, 0);
  C.neighborN.assign(n, 0);
  if (k.neighbors == CBM_NEIGH_VERLET_DISPLACEMENT || k.neighbors == CBM_NEIGH_CLVD)
    C.neighborList.assign(n * (size_t)k.n_max_neighbors, 0);
  C.nNodes = 0;
  if (k.medium) {
    C.nNodes = 1;
    for (int d = 0; d < C.dims; ++d) {
      C.nm[d] = k.n_medium[d];
      C.dxm[d] = (T)((k.box_hi[d] - k.box_lo[d]) / (double)k.n_medium[d]);  // communityStructure.jl:274
      C.nNodes *= C.nm[d];
    }
    C.c.assign((size_t)C.nNodes, 0); C.c_.assign((size_t)C.nNodes, 0);
    for (int d = 0; d < 3; ++d) { C.gr[d].assign((size_t)C.nNodes, 0); C.gr_[d].assign((size_t)C.nNodes, 0); }
  }
}

/* ---------------------------------------------------------------------------
 * computeNeighbors!
 * ------------------------------------------------------------------------- */
template <typename T>
void buildCells(Com<T>& C) {
  // neighborsCellLinked{d}CPU!, src/neighbors.jl:918-979
  std::fill(C.cellNumAgents.begin(), C.cellNumAgents.end(), 0);
  for (int64_t i = 0; i < C.N; ++i) C.cellNumAgents[cellOf(C, C.x, i)] += 1;  // assignCells :776-786
  int64_t acc = 0;
  for (size_t c = 0; c < C.cellNumAgents.size(); ++c) {  // cumsum! .- counts :934-937
    C.cellCumSum[c] = acc;
    acc += C.cellNumAgents[c];
  }
  for (int64_t i = 0; i < C.N; ++i) {  // sortAgentsInCells :851-862
    int64_t p = cellOf(C, C.x, i);
    C.cellCumSum[p] += 1;
    C.cellAssignedToAgent[C.cellCumSum[p] - 1] = i;
  }
}

template <typename T>
void verletDisplacement(Com<T>& C) {
  // verletDisplacementCPU!, src/neighbors.jl:367-391
  T thr = C.cfg.rebuild_threshold > 0 ? (T)C.cfg.rebuild_threshold : (T)C.cfg.skin / (T)2;
  for (int64_t i = 0; i < C.N; ++i) {
    C.accumulatedDistance[i] = euclid(C, C.x, i, C.posOld, i);
    if (C.accumulatedDistance[i] >= thr) C.flagRecompute = 1;
  }
}

template <typename T>
void appendNeighbor(Com<T>& C, int64_t i, int64_t j) {
  int64_t k = C.neighborN[i];
  if (k >= C.cfg.n_max_neighbors) {
#pragma omp atomic write
    C.err = CBM_ERR_NEIGHBOR_OVERFLOW;
    return;
  }
  C.neighborList[i + k * C.nMax] = (int32_t)j;
  C.neighborN[i] = k + 1;
}

template <typename T>
void computeNeighbors(Com<T>& C) {
  const int alg = C.cfg.neighbors;
  if (alg == CBM_NEIGH_CELL_LINKED) {
    buildCells(C);
    return;
  }
  if (alg != CBM_NEIGH_VERLET_DISPLACEMENT && alg != CBM_NEIGH_CLVD) return;
  verletDisplacement(C);
  if (C.flagRecompute != 1) return;
  const T skin = (T)C.cfg.skin;
  if (alg == CBM_NEIGH_CLVD) buildCells(C);  // neighborsCLVD, :1206-1228
  std::fill(C.neighborN.begin(), C.neighborN.end(), 0);
  std::fill(C.accumulatedDistance.begin(), C.accumulatedDistance.end(), 0);
  C.flagRecompute = 0;
  for (int64_t i = 0; i < C.N; ++i)  // verletResetDisplacement :438-487
    for (int d = 0; d < C.dims; ++d) C.posOld[d][i] = C.x[d][i];
  if (alg == CBM_NEIGH_VERLET_DISPLACEMENT) {
    // verletNeighborsCPU!, :92-133: ascending j
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int64_t i = 0; i < C.N; ++i)
      for (int64_t j = 0; j < C.N; ++j)
        if (i != j && euclid(C, C.x, i, C.x, j) < skin) appendNeighbor(C, i, j);
  } else {
    // verletNeighborsCLVD{d}CPU!, :1071-1131: cell order, ascending within a cell
    const int nk = C.dims == 1 ? 3 : (C.dims == 2 ? 9 : 27);
#pragma omp parallel for schedule(static) num_threads(g_threads)
    for (int64_t i = 0; i < C.N; ++i) {
      int64_t pos = cellOf(C, C.x, i);
      for (int k = 0; k < nk; ++k) {
        int64_t pn = cellNeigh(C, pos, k);
        if (pn < 0) continue;
        for (int64_t s = C.cellCumSum[pn] - C.cellNumAgents[pn]; s < C.cellCumSum[pn]; ++s) {
          int64_t j = C.cellAssignedToAgent[s];
          if (j != i && euclid(C, C.x, i, C.x, j) < skin) appendNeighbor(C, i, j);
        }
      }
    }
  }
}

/* ---------------------------------------------------------------------------
 * agentStepRule!
 * ------------------------------------------------------------------------- */
template <typename T>
void bilinear(const Com<T>& C, const T* p, int64_t* node, T* w) {
  // corners of the medium cell whose nodes (cell centres lo + (i+1/2) dx)
  // surround p; node indices clamped to the grid.
  int64_t i0[3], i1[3];
  T tt[3];
  for (int d = 0; d < C.dims; ++d) {
    T s = (p[d] - (T)C.cfg.box_lo[d]) / C.dxm[d] - (T)0.5;
    T fl = std::floor(s);
    tt[d] = s - fl;
    int64_t a = (int64_t)fl;
    int64_t b = a + 1;
    a = a < 0 ? 0 : (a > C.nm[d] - 1 ? C.nm[d] - 1 : a);
    b = b < 0 ? 0 : (b > C.nm[d] - 1 ? C.nm[d] - 1 : b);
    i0[d] = a; i1[d] = b;
  }
  int nc = 1 << C.dims;
  for (int q = 0; q < nc; ++q) {
    int64_t lin = 0, mul = 1;
    T wq = 1;
    for (int d = 0; d < C.dims; ++d) {
      bool hi = (q >> d) & 1;
      lin += (hi ? i1[d] : i0[d]) * mul;
      mul *= C.nm[d];
      wq = wq * (hi ? tt[d] : (T)1 - tt[d]);
    }
    node[q] = lin;
    w[q] = wq;
  }
}

template <typename T>
int64_t nearestNode(const Com<T>& C, const T* p) {
  int64_t lin = 0, mul = 1;
  for (int d = 0; d < C.dims; ++d) {
    lin += cellInMesh<T>(C.dxm[d], p[d], (T)C.cfg.box_lo[d], (T)C.cfg.box_hi[d], C.nm[d]) * mul;
    mul *= C.nm[d];
  }
  return lin;
}

/* @addAgent, src/AgentStructure/functionRule.jl:9-79.  Returns the new slot
 * or -1 when nMax is reached (the birth is dropped; the id is consumed). */
template <typename T>
int64_t addAgent(Com<T>& C, int64_t i) {
  int64_t slot = C.N + C.NAdd;
  C.NAdd += 1;
  int64_t idNew = ++C.idMax;
  if (slot < C.nMax) {
    C.id[slot] = idNew;
    C.flagRecompute = 1;
    C.flagSurvive[slot] = 1;
    // parameters not given to @addAgent are copied from the parent
    for (int d = 0; d < C.dims; ++d) {
      C.x_[d][slot] = C.x[d][i];
      C.f_[d][slot] = C.f[d][i];
    }
    C.v_[slot] = C.v[i];
    C.g[slot] = C.g[i];
    C.parent[slot] = C.id[i];
    return slot;
  }
  C.NAdd -= 1;
  if (!C.err) C.err = CBM_ERR_AGENT_OVERFLOW;
  return -1;
}

/* @removeAgent, functionRule.jl:89-111 */
template <typename T>
void removeAgent(Com<T>& C, int64_t i) {
  C.holeFromRemoveAt[C.NRemove] = i;
  C.NRemove += 1;
  C.flagSurvive[i] = 0;
  C.flagRecompute = 1;
}

template <typename T>
void agentStepRule(Com<T>& C) {
  const cbm_config& k = C.cfg;
  const int D = C.dims;
  const T amt = (T)k.secretion * (T)k.dt;
  const T upt = (T)k.uptake * (T)k.dt;
  for (int64_t i = 0; i < C.N; ++i) {
    T p[3];
    for (int d = 0; d < D; ++d) p[d] = C.x[d][i];
    if (k.walls == CBM_WALLS_REFLECT) {
      for (int d = 0; d < D; ++d) {
        T lo = (T)k.box_lo[d], hi = (T)k.box_hi[d];
        if (p[d] < lo) C.x_[d][i] = (T)2 * lo - p[d];
        else if (p[d] > hi) C.x_[d][i] = (T)2 * hi - p[d];
      }
    }
    if (k.medium && (k.secretion != 0 || k.uptake != 0)) {
      // c__[node] += w (secretion dt - uptake dt c[node]) at the agent, c the
      // committed field (auxiliar.jl:353-365 writes c__ inside the rule); the
      // uptake term is this library's first-order sink, absent when uptake = 0
      if (k.medium_sampling == CBM_MEDIUM_NEAREST) {
        int64_t n = nearestNode(C, p);
        C.c_[n] = C.c_[n] + (k.uptake != 0 ? amt - upt * C.c[n] : amt);
      } else {
        int64_t nodes[8];
        T w[8];
        bilinear(C, p, nodes, w);
        for (int q = 0; q < (1 << D); ++q)
          C.c_[nodes[q]] =
              C.c_[nodes[q]] + (k.uptake != 0 ? w[q] * (amt - upt * C.c[nodes[q]]) : w[q] * amt);
      }
    }
    if (k.fate == CBM_FATE_VOLUME) {
      if (k.growth && C.v[i] >= (T)k.v_div) {
        T a[3] = {0, 0, 0};
        cbm_normals(k.seed, C.step, (uint32_t)i, CBM_STREAM_DIVISION, k.community, D, a);
        T s = 0;
        for (int d = 0; d < D; ++d) s = (d == 0) ? a[d] * a[d] : s + a[d] * a[d];
        T Ta = std::sqrt(s);
        for (int d = 0; d < D; ++d) a[d] = a[d] / Ta;
        T rsep = (T)k.div_sep;
        T vh = C.v[i] / (T)2;
        int64_t s1 = addAgent(C, i);
        if (s1 >= 0) {
          for (int d = 0; d < D; ++d) C.x_[d][s1] = p[d] + rsep * a[d];
          C.v_[s1] = vh;
        }
        int64_t s2 = addAgent(C, i);
        if (s2 >= 0) {
          for (int d = 0; d < D; ++d) C.x_[d][s2] = p[d] - rsep * a[d];
          C.v_[s2] = vh;
        }
        removeAgent(C, i);
      } else if (k.p_death > 0 &&
                 cbm_uniform<T>(k.seed, C.step, (uint32_t)i, CBM_STREAM_DEATH, k.community) <
                     (T)k.p_death) {
        removeAgent(C, i);
      }
    } else if (k.fate == CBM_FATE_ID_PARITY) {
      if (C.id[i] % 2 == 1) removeAgent(C, i);
      else addAgent(C, i);
    }
  }
}

/* ---------------------------------------------------------------------------
 * agentStepDE!
 * ------------------------------------------------------------------------- */
template <typename T>
void sampleGrad(const Com<T>& C, const T* p, T* gv) {
  const int D = C.dims;
  if (C.cfg.medium_sampling == CBM_MEDIUM_NEAREST) {
    int64_t n = nearestNode(C, p);
    for (int d = 0; d < D; ++d) gv[d] = C.gr[d][n];
  } else {
    int64_t nodes[8];
    T w[8];
    bilinear(C, p, nodes, w);
    for (int d = 0; d < D; ++d) {
      T s = 0;
      for (int q = 0; q < (1 << D); ++q) s = s + w[q] * C.gr[d][nodes[q]];
      gv[d] = s;
    }
  }
}

// f(du, u, p, t) of agentStepDE! for agents 0..N-1, with the positions of u
// in X (the DE state, or a stage of a multi-stage integrator): the neighbor
// loop's own cell is computed from X, its occupants are the last rebuild's.
template <typename T>
void evalF(Com<T>& C, const std::vector<T>* X, std::vector<T>* out) {
  const cbm_config& k = C.cfg;
  const int D = C.dims;
  const int64_t N = C.N;
  const T krep = (T)k.k_rep, rrep = (T)k.r_rep, katt = (T)k.k_att, ratt = (T)k.r_att;
  const bool lagged = k.force_mode == CBM_FORCE_LAGGED;
#pragma omp parallel for schedule(static) num_threads(g_threads)
  for (int64_t i = 0; i < N; ++i) {
    T acc[3] = {0, 0, 0};  // cleanArray: du = 0 (integrators.jl:442-450)
    T pi[3];
    for (int d = 0; d < D; ++d) pi[d] = X[d][i];
    if (k.neighbors != CBM_NEIGH_NONE) {
      forNeighbors(C, X, i, N, [&](int64_t j) {
        T e[3];
        T s2 = 0;
        for (int d = 0; d < D; ++d) {
          e[d] = pi[d] - X[d][j];
          s2 = (d == 0) ? e[d] * e[d] : s2 + e[d] * e[d];
        }
        T dist = std::sqrt(s2);
        T F;
        if (dist < rrep) F = krep * (rrep - dist);
        else if (dist < ratt) F = k.att_form == CBM_ATT_FROM_REP ? -(katt * (dist - rrep))
                                                                : -(katt * (ratt - dist));
        else return;
        T s = F / dist;
        for (int d = 0; d < D; ++d) acc[d] = acc[d] + s * e[d];
      });
    }
    if (k.walls == CBM_WALLS_PUSH) {
      for (int d = 0; d < D; ++d) {
        if (pi[d] < (T)k.box_lo[d] + (T)k.wall_range) acc[d] = acc[d] + (T)k.wall_force;
        else if (pi[d] > (T)k.box_hi[d] - (T)k.wall_range) acc[d] = acc[d] - (T)k.wall_force;
      }
    }
    T dv[3];
    if (lagged) {
      for (int d = 0; d < D; ++d) { C.f_[d][i] = acc[d]; dv[d] = C.f[d][i]; }
    } else {
      for (int d = 0; d < D; ++d) dv[d] = acc[d];
    }
    if (k.drift_linear != 0)
      for (int d = 0; d < D; ++d) dv[d] = dv[d] + (-(T)k.drift_linear) * pi[d];
    if (k.medium && k.chemotaxis != 0) {
      T gv[3] = {0, 0, 0};
      sampleGrad(C, pi, gv);
      T s = 0;
      for (int d = 0; d < D; ++d) s = (d == 0) ? gv[d] * gv[d] : s + gv[d] * gv[d];
      T den = (T)1 + std::sqrt(s);
      for (int d = 0; d < D; ++d) dv[d] = dv[d] + ((T)k.chemotaxis * gv[d]) / den;
    }
    for (int d = 0; d < D; ++d) out[d][i] = dv[d];
  }
}

// Heun (src/integrators.jl:541-571) and RungeKutta4 (:606-666) over 1:N,
// each broadcast element by element.  The volume is a DE variable with
// dt(v) = g when growth is on; f does not read it.
template <typename T>
void multiStage(Com<T>& C) {
  const cbm_config& k = C.cfg;
  const int D = C.dims;
  const int64_t N = C.N;
  const T dt = (T)k.dt;
  std::vector<T> h[3], kk[3], acc[3];
  for (int d = 0; d < 3; ++d) {
    h[d].assign(C.x_[d].size(), 0);
    kk[d].assign(C.x_[d].size(), 0);
    acc[d].assign(C.x_[d].size(), 0);
  }
  if (k.integrator == CBM_INT_EULER_HEUN) {
    // EulerHeun (:775-810), the CPU branch; g = sigma for positions, 0 for v
    const T sq = std::sqrt(dt), sig = (T)k.sigma;
    evalF(C, C.x_, acc);  // f1
    for (int64_t i = 0; i < N; ++i) {
      T xi[3] = {0, 0, 0};
      cbm_normals(k.seed, C.step, (uint32_t)i, CBM_STREAM_NOISE, k.community, D, xi);
      for (int d = 0; d < D; ++d) h[d][i] = (C.x_[d][i] + acc[d][i] * dt) + (sig * xi[d]) * sq;
    }
    evalF(C, h, kk);  // f2
    for (int64_t i = 0; i < N; ++i) {
      T xi[3] = {0, 0, 0};
      cbm_normals(k.seed, C.step, (uint32_t)i, CBM_STREAM_NOISE_FINAL, k.community, D, xi);
      for (int d = 0; d < D; ++d)
        C.x_[d][i] = C.x_[d][i] + (((acc[d][i] + kk[d][i]) * dt) + ((sig + sig) * xi[d]) * sq) / (T)2;
      if (k.growth) C.v_[i] = C.v_[i] + ((C.g[i] + C.g[i]) * dt) / (T)2;
    }
    return;
  }
  if (k.integrator == CBM_INT_HEUN) {
    evalF(C, C.x_, kk);
    for (int64_t i = 0; i < N; ++i)
      for (int d = 0; d < D; ++d) h[d][i] = C.x_[d][i] + kk[d][i] * dt;
    evalF(C, h, kk);
    for (int64_t i = 0; i < N; ++i) {
      for (int d = 0; d < D; ++d) C.x_[d][i] = (h[d][i] + (C.x_[d][i] + kk[d][i] * dt)) / (T)2;
      if (k.growth) {
        const T v = C.v_[i], g = C.g[i];
        const T hv = v + g * dt;
        C.v_[i] = (hv + (v + g * dt)) / (T)2;
      }
    }
    return;
  }
  // k1: h = u + (k1 dt)/2; k2: h = u + (k2 dt)/2; k3: h = u + k3 dt; k4
  evalF(C, C.x_, kk);
  for (int64_t i = 0; i < N; ++i)
    for (int d = 0; d < D; ++d) {
      acc[d][i] = kk[d][i];
      h[d][i] = C.x_[d][i] + (kk[d][i] * dt) / (T)2;
    }
  for (int st = 2; st <= 4; ++st) {
    evalF(C, h, kk);
    for (int64_t i = 0; i < N; ++i)
      for (int d = 0; d < D; ++d) {
        acc[d][i] = st == 4 ? acc[d][i] + kk[d][i] : acc[d][i] + (T)2 * kk[d][i];
        if (st == 2) h[d][i] = C.x_[d][i] + (kk[d][i] * dt) / (T)2;
        if (st == 3) h[d][i] = C.x_[d][i] + kk[d][i] * dt;
      }
  }
  for (int64_t i = 0; i < N; ++i) {
    for (int d = 0; d < D; ++d) C.x_[d][i] = C.x_[d][i] + (acc[d][i] * dt) / (T)6;
    if (k.growth) {
      const T v = C.v_[i], g = C.g[i];
      C.v_[i] = v + ((((g + (T)2 * g) + (T)2 * g) + g) * dt) / (T)6;
    }
  }
}

template <typename T>
void agentStepDE(Com<T>& C) {
  const cbm_config& k = C.cfg;
  const int D = C.dims;
  const int64_t N = C.N;
  const T dt = (T)k.dt;
  if (k.integrator == CBM_INT_HEUN || k.integrator == CBM_INT_RK4 ||
      k.integrator == CBM_INT_EULER_HEUN) {
    multiStage(C);
    return;
  }
  evalF(C, C.x_, C.du);
  // integrator update over 1:N (integrators.jl:495-496 / :720-721)
  const T sq = std::sqrt(dt);
  const T sig = (T)k.sigma;
  for (int64_t i = 0; i < N; ++i) {
    if (k.integrator == CBM_INT_EM) {
      T xi[3] = {0, 0, 0};
      if (C.ext_noise) {
        for (int d = 0; d < D; ++d) xi[d] = C.ext_noise[i * D + d];
      } else {
        cbm_normals(k.seed, C.step, (uint32_t)i, CBM_STREAM_NOISE, k.community, D, xi);
      }
      for (int d = 0; d < D; ++d) C.x_[d][i] = (C.x_[d][i] + C.du[d][i] * dt) + (sig * xi[d]) * sq;
    } else {
      for (int d = 0; d < D; ++d) C.x_[d][i] = C.x_[d][i] + C.du[d][i] * dt;
    }
    if (k.growth) C.v_[i] = C.v_[i] + C.g[i] * dt;
  }
}

/* ---------------------------------------------------------------------------
 * mediumStepRule! / mediumStepDE!
 * ------------------------------------------------------------------------- */
template <typename T>
bool interiorNode(const Com<T>& C, int64_t n, int64_t* q) {
  int64_t r = n;
  bool in = true;
  for (int d = 0; d < C.dims; ++d) {
    q[d] = r % C.nm[d];
    r /= C.nm[d];
    if (q[d] == 0 || q[d] == C.nm[d] - 1) in = false;  // @mediumInside, macros.jl:240-255
  }
  return in;
}

template <typename T>
void mediumStepRule(Com<T>& C) {
  if (!C.cfg.medium || C.cfg.chemotaxis == 0) return;
  // gx = @∂(1,c) inside, 0 on the border (macros.jl:148-190)
  int64_t stride[3] = {1, C.nm[0], C.nm[0] * C.nm[1]};
  for (int64_t n = 0; n < C.nNodes; ++n) {
    int64_t q[3];
    bool in = interiorNode(C, n, q);
    for (int d = 0; d < C.dims; ++d)
      C.gr_[d][n] = in ? (C.c[n + stride[d]] - C.c[n - stride[d]]) / ((T)2 * C.dxm[d]) : (T)0;
  }
}

template <typename T>
void mediumStepDE(Com<T>& C) {
  if (!C.cfg.medium) return;
  const T D = (T)C.cfg.diff_D, lam = (T)C.cfg.decay, dt = (T)C.cfg.dt;
  int64_t stride[3] = {1, C.nm[0], C.nm[0] * C.nm[1]};
  if (C.cfg.uptake != 0)  // with uptake the step reads the field clamped at zero
    for (int64_t n = 0; n < C.nNodes; ++n)
      if (C.c_[n] < (T)0) C.c_[n] = (T)0;
  std::vector<T> k(C.nNodes, (T)0);
  for (int64_t n = 0; n < C.nNodes; ++n) {
    int64_t q[3];
    if (!interiorNode(C, n, q)) continue;  // du stays 0 on the border
    T u = C.c_[n];
    T lap = 0;
    for (int d = 0; d < C.dims; ++d) {
      // @∂2: (m[i+1] - 2 m[i] + m[i-1]) / dx^2, macros.jl:203-258
      T l = ((C.c_[n + stride[d]] - (T)2 * u) + C.c_[n - stride[d]]) / (C.dxm[d] * C.dxm[d]);
      lap = (d == 0) ? l : lap + l;
    }
    k[n] = D * lap - lam * u;
  }
  for (int64_t n = 0; n < C.nNodes; ++n) C.c_[n] = C.c_[n] + dt * k[n];  // u = uprev + dt*k
}

/* ---------------------------------------------------------------------------
 * update!
 * ------------------------------------------------------------------------- */
template <typename T, typename V>
void fillHoles(Com<T>& C, std::vector<V>& par, int64_t count) {
  // kernelFillHolesParametersCPU!, update.jl:67-84
  for (int64_t k = 0; k < count; ++k) {
    int64_t posNew = C.holeFromRemoveAt[k], posOld = C.repositionAgentInPos[k];
    if (posNew < posOld) par[posNew] = par[posOld];
  }
}

template <typename T>
void update(Com<T>& C) {
  const int D = C.dims;
  if (C.cfg.fate != CBM_FATE_NONE) {
    // kernelListSurvived, update.jl:15-33
    int64_t count = 0;
    int64_t lastPos = C.N + C.NAdd - 1;
    while (C.NRemove > count && lastPos >= 0) {
      if (C.flagSurvive[lastPos] == 1) C.repositionAgentInPos[count++] = lastPos;
      lastPos -= 1;
    }
    // entries beyond `count` would only touch rows >= the new N
    fillHoles(C, C.id, count);
    fillHoles(C, C.parent, count);
    for (int d = 0; d < D; ++d) { fillHoles(C, C.x_[d], count); fillHoles(C, C.f_[d], count); }
    fillHoles(C, C.v_, count);
    fillHoles(C, C.g, count);
  }
  C.N = C.N + C.NAdd - C.NRemove;
  C.NAdd = 0;
  C.NRemove = 0;
  for (int64_t i = 0; i < C.N; ++i) C.flagSurvive[i] = 1;
  // commit par <- par__ (kernelUpdateParameters, update.jl:126-158)
  for (int64_t i = 0; i < C.N; ++i) {
    for (int d = 0; d < D; ++d) { C.x[d][i] = C.x_[d][i]; C.f[d][i] = C.f_[d][i]; }
    C.v[i] = C.v_[i];
  }
  if (C.cfg.medium) {
    C.c = C.c_;
    for (int d = 0; d < D; ++d) C.gr[d] = C.gr_[d];
  }
  C.t = C.t + C.cfg.dt;
  C.step += 1;
}

template <typename T>
void step(Com<T>& C) {
  // step!, step.jl:96-107 (model stages are empty in this family)
  agentStepRule(C);
  agentStepDE(C);
  mediumStepRule(C);
  mediumStepDE(C);
  update(C);
  computeNeighbors(C);
}

/* ---------------------------------------------------------------------------
 * host exchange
 * ------------------------------------------------------------------------- */
template <typename T>
int upload(Com<T>& C, const cbm_state_view* h) {
  const int D = C.dims;
  if (h->N < 0 || h->N > C.nMax) return CBM_ERR_ARG;
  alloc(C);
  C.N = h->N;
  C.t = h->t;
  C.step = h->step;
  C.idMax = h->id_max > 0 ? h->id_max : h->N;
  C.NAdd = C.NRemove = 0;
  C.err = 0;
  for (int64_t i = 0; i < C.N; ++i) {
    for (int d = 0; d < D; ++d) {
      C.x[d][i] = ((const T*)h->pos[d])[i];
      C.f[d][i] = h->f[d] ? ((const T*)h->f[d])[i] : (T)0;
    }
    C.v[i] = h->v ? ((const T*)h->v)[i] : (T)0;
    C.g[i] = h->g ? ((const T*)h->g)[i] : (T)0;
    C.id[i] = h->id ? h->id[i] : i + 1;
    C.parent[i] = h->parent ? h->parent[i] : 0;
  }
  for (int d = 0; d < 3; ++d) { C.x_[d] = C.x[d]; C.f_[d] = C.f[d]; }
  C.v_ = C.v;
  if (C.cfg.medium) {
    for (int64_t n = 0; n < C.nNodes; ++n) {
      C.c[n] = h->medium_c ? ((const T*)h->medium_c)[n] : (T)0;
      for (int d = 0; d < D; ++d)
        C.gr[d][n] = h->medium_grad[d] ? ((const T*)h->medium_grad[d])[n] : (T)0;
    }
    C.c_ = C.c;
    for (int d = 0; d < 3; ++d) C.gr_[d] = C.gr[d];
  }
  C.flagRecompute = 1;  // loadBaseParameters!, communityStructure.jl:480
  C.loaded = true;
  computeNeighbors(C);  // communityStructure.jl:648
  return CBM_OK;
}

template <typename T>
int download(Com<T>& C, cbm_state_view* h, int which) {
  const int D = C.dims;
  if (h->capacity < C.N) return CBM_ERR_ARG;
  h->N = C.N;
  h->t = C.t;
  h->step = C.step;
  h->id_max = C.idMax;
  const bool nw = which == CBM_VIEW_NEW;
  for (int64_t i = 0; i < C.N; ++i) {
    for (int d = 0; d < D; ++d) {
      if (h->pos[d]) ((T*)h->pos[d])[i] = nw ? C.x_[d][i] : C.x[d][i];
      if (h->f[d]) ((T*)h->f[d])[i] = nw ? C.f_[d][i] : C.f[d][i];
    }
    if (h->v) ((T*)h->v)[i] = nw ? C.v_[i] : C.v[i];
    if (h->g) ((T*)h->g)[i] = C.g[i];
    if (h->id) h->id[i] = C.id[i];
    if (h->parent) h->parent[i] = C.parent[i];
  }
  if (C.cfg.medium) {
    for (int64_t n = 0; n < C.nNodes; ++n) {
      if (h->medium_c) ((T*)h->medium_c)[n] = nw ? C.c_[n] : C.c[n];
      for (int d = 0; d < D; ++d)
        if (h->medium_grad[d]) ((T*)h->medium_grad[d])[n] = nw ? C.gr_[d][n] : C.gr[d][n];
    }
  }
  return CBM_OK;
}

struct Handle {
  int prec;
  void* p;
};

template <typename T>
Com<T>* as(Handle* h) { return (Com<T>*)h->p; }

// ---- implicit medium: DGADI (src/integrators.jl:141-428, 817-937) ---------
// The reference's arrays: u (the medium ODE state), u_new, c_star, d_star,
// all copies of u0 (DGADI(problem, ...) :844-856), shape (field, x, y, z)
// with x fastest inside a field here.
template <typename T>
struct Med {
  cbm_medium_config cfg;
  int64_t nodes = 0;
  std::vector<T> u, u_new, c_star, d_star, src;
  double t = 0;
};

// One line of tridiagonal{1,2,3}D{x,y,z}CPU! (:141-269), 0-based: nodes 0 and
// n-1 are the Dirichlet ends.  1.0 / (...) is Float64 (Julia promotes the
// Float32 denominator), so the pivots and the products with them are formed
// in Float64 and rounded to T when stored.
template <typename T>
void thomasLine(const T* xo, T* xn, T* cs, T* ds, int64_t st, int n, T sub, T main, T sup) {
  auto X = [&](int j) { return xo[(int64_t)j * st]; };
  auto C = [&](int j) -> T& { return cs[(int64_t)j * st]; };
  auto Dd = [&](int j) -> T& { return ds[(int64_t)j * st]; };
  C(1) = sup / main;
  Dd(1) = (X(1) - sub * X(0)) / main;
  for (int j = 2; j <= n - 3; ++j) {
    const double m = 1.0 / (double)(main - sub * C(j - 1));
    C(j) = (T)((double)sup * m);
    Dd(j) = (T)((double)(X(j) - sub * Dd(j - 1)) * m);
  }
  const double m = 1.0 / (double)(main - sub * C(n - 3));
  Dd(n - 2) = (T)((double)((X(n - 2) - sup * X(n - 1)) - sub * Dd(n - 3)) * m);
  xn[(int64_t)(n - 2) * st] = Dd(n - 2);
  for (int j = n - 3; j >= 1; --j)
    xn[(int64_t)j * st] = Dd(j) - C(j) * xn[(int64_t)(j + 1) * st];
}

// DifferentialEquations.step!(::DGADI) (:875-933)
template <typename T>
void medStep(Med<T>& M) {
  const cbm_medium_config& k = M.cfg;
  const int D = k.dims;
  const int n0 = k.n[0], n1 = D > 1 ? k.n[1] : 1, n2 = D > 2 ? k.n[2] : 1;
  const int64_t N = M.nodes;
  // du = f(u) inside (@mediumInside), then u .+= du
  for (int f = 0; f < k.n_fields; ++f) {
    const T cmax = (T)k.c_max, dec = (T)k.decay[f];
    T* u = M.u.data() + f * N;
    for (int z = 0; z < n2; ++z)
      for (int y = 0; y < n1; ++y)
        for (int x = 0; x < n0; ++x) {
          const bool in = x > 0 && x < n0 - 1 && (D < 2 || (y > 0 && y < n1 - 1)) &&
                          (D < 3 || (z > 0 && z < n2 - 1));
          if (!in) continue;
          const int64_t i = x + (int64_t)n0 * (y + (int64_t)n1 * z);
          const T du = M.src[i] * (cmax - u[i]) - dec * u[i];
          u[i] = u[i] + du;
        }
  }
  // r = dt / (dims dx^2) per axis; every axis reads the last one's
  const double dxl = (k.box_hi[D - 1] - k.box_lo[D - 1]) / (double)k.n[D - 1];
  const double r = k.dt / ((double)D * (dxl * dxl));
  const int64_t stride[3] = {1, n0, (int64_t)n0 * n1};
  const int len[3] = {n0, n1, n2};
  for (int a = 0; a < D; ++a) {
    // lines along axis a through interior nodes of the other axes
    const int b = a == 0 ? 1 : 0, c = a == 2 ? 1 : 2;
    const int lb = b < D ? len[b] : 1, lc = c < D ? len[c] : 1;
    for (int f = 0; f < k.n_fields; ++f) {
      const T sub = (T)(-k.diffusion[f] * r), sup = (T)(-k.diffusion[f] * r);
      const T main = (T)(1.0 + 2.0 * k.diffusion[f] * r);
      for (int ic = (c < D ? 1 : 0); ic < (c < D ? lc - 1 : 1); ++ic)
        for (int ib = (b < D ? 1 : 0); ib < (b < D ? lb - 1 : 1); ++ib) {
          const int64_t o = f * N + (int64_t)ib * stride[b] + (int64_t)ic * stride[c];
          thomasLine<T>(M.u.data() + o, M.u_new.data() + o, M.c_star.data() + o,
                        M.d_star.data() + o, stride[a], len[a], sub, main, sup);
        }
    }
    M.u = M.u_new;  // obj.u .= obj.u_new
  }
  M.t += k.dt;
}

}  // namespace

#define DISPATCH(h, expr)                          \
  do {                                             \
    if ((h)->prec == CBM_F64) { auto* C = as<double>(h); expr; } \
    else { auto* C = as<float>(h); expr; }         \
  } while (0)

extern "C" {

void oracle_set_threads(int n) { g_threads = n > 0 ? n : 1; }

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void* oracle_create(const cbm_config* cfg) {
  if (!cfg || cfg->dims < 1 || cfg->dims > 3 || cfg->n_max < 0) return nullptr;
  Handle* h = new Handle;
  h->prec = cfg->precision;
  if (h->prec == CBM_F64) {
    auto* C = new Com<double>;
    C->cfg = *cfg;
    alloc(*C);
    h->p = C;
  } else {
    auto* C = new Com<float>;
    C->cfg = *cfg;
    alloc(*C);
    h->p = C;
  }
  return h;
}

void oracle_destroy(void* vh) {
  Handle* h = (Handle*)vh;
  if (!h) return;
  if (h->prec == CBM_F64) delete as<double>(h);
  else delete as<float>(h);
  delete h;
}

int oracle_upload(void* vh, const cbm_state_view* s) {
  int rc = 0;
  DISPATCH((Handle*)vh, rc = upload(*C, s));
  return rc;
}

int oracle_download(void* vh, cbm_state_view* s, int which) {
  int rc = 0;
  DISPATCH((Handle*)vh, rc = download(*C, s, which));
  return rc;
}

/* stage: 0 agentRule, 1 agentDE, 2 mediumRule, 3 mediumDE, 4 update, 5 neighbors */
int oracle_stage(void* vh, int stage) {
  DISPATCH((Handle*)vh, {
    switch (stage) {
      case 0: agentStepRule(*C); break;
      case 1: agentStepDE(*C); break;
      case 2: mediumStepRule(*C); break;
      case 3: mediumStepDE(*C); break;
      case 4: update(*C); break;
      case 5: computeNeighbors(*C); break;
      default: return CBM_ERR_ARG;
    }
  });
  return CBM_OK;
}

int oracle_step(void* vh, int nsteps) {
  DISPATCH((Handle*)vh, for (int s = 0; s < nsteps; ++s) step(*C));
  return CBM_OK;
}

/* one step whose EM increments are given: noise[i * dims + d] for the N
 * agents in index order, in the context's precision */
int oracle_step_noise(void* vh, const void* noise) {
  DISPATCH((Handle*)vh, {
    using TT = typename std::remove_reference<decltype(C->g)>::type::value_type;
    C->ext_noise = (const TT*)noise;
    step(*C);
    C->ext_noise = nullptr;
  });
  return CBM_OK;
}

/* returns and clears the first model fault */
int oracle_take_error(void* vh) {
  int e = 0;
  DISPATCH((Handle*)vh, { e = C->err; C->err = 0; });
  return e;
}

int oracle_get_counters(void* vh, int64_t* N, int64_t* nadd, int64_t* nrem, int64_t* idmax,
                        int32_t* flag, int64_t* stepc) {
  DISPATCH((Handle*)vh, {
    *N = C->N; *nadd = C->NAdd; *nrem = C->NRemove; *idmax = C->idMax;
    *flag = C->flagRecompute; *stepc = C->step;
  });
  return CBM_OK;
}

int oracle_grid_shape(void* vh, int32_t* n3) {
  DISPATCH((Handle*)vh, for (int d = 0; d < 3; ++d) n3[d] = (int32_t)C->nCells[d]);
  return CBM_OK;
}

int oracle_get_grid(void* vh, int32_t* agent_cell, int32_t* cell_start, int32_t* cell_count,
                    int32_t* cell_agents) {
  DISPATCH((Handle*)vh, {
    for (int64_t i = 0; i < C->N; ++i) {
      agent_cell[i] = (int32_t)cellOf(*C, C->x, i);
      cell_agents[i] = (int32_t)C->cellAssignedToAgent[i];
    }
    for (size_t c = 0; c < C->cellNumAgents.size(); ++c) {
      cell_count[c] = (int32_t)C->cellNumAgents[c];
      cell_start[c] = (int32_t)(C->cellCumSum[c] - C->cellNumAgents[c]);
    }
  });
  return CBM_OK;
}

int oracle_get_neighbors(void* vh, int32_t* counts, int32_t* list, int64_t cap) {
  DISPATCH((Handle*)vh, {
    int64_t m = C->cfg.n_max_neighbors;
    if (cap < C->N * m) return CBM_ERR_ARG;
    for (int64_t i = 0; i < C->N; ++i) {
      counts[i] = (int32_t)C->neighborN[i];
      for (int64_t k = 0; k < m; ++k)
        list[i * m + k] = k < C->neighborN[i] ? (int32_t)C->neighborList[i + k * C->nMax] : -1;
    }
  });
  return CBM_OK;
}

int oracle_count_neighbors(void* vh, double radius, int32_t* out) {
  DISPATCH((Handle*)vh, {
    auto r = (decltype(C->edge))radius;
    for (int64_t i = 0; i < C->N; ++i) {
      int32_t n = 0;
      forNeighbors(*C, C->x, i, C->N, [&](int64_t j) {
        if (euclid(*C, C->x, i, C->x, j) < r) n += 1;
      });
      out[i] = n;
    }
  });
  return CBM_OK;
}

/* kind 0 normal(a,b), 1 uniform(a,b), 2 exponential(a): src/random.jl:8-22 */
int oracle_rng_fill(int precision, uint64_t seed, uint32_t community, int kind, double a,
                    double b, int64_t n, int64_t stepc, void* out) {
  for (int64_t i = 0; i < n; ++i) {
    if (precision == CBM_F64) {
      double z;
      if (kind == 0) { cbm_normals(seed, stepc, (uint32_t)i, CBM_STREAM_USER, community, 1, &z); z = b * z + a; }
      else if (kind == 1) z = (b - a) * cbm_uniform_f64(seed, stepc, (uint32_t)i, CBM_STREAM_USER, community) + a;
      else z = -cbm_log_f64(1.0 - cbm_uniform_f64(seed, stepc, (uint32_t)i, CBM_STREAM_USER, community)) * a;
      ((double*)out)[i] = z;
    } else {
      float z;
      if (kind == 0) { cbm_normals(seed, stepc, (uint32_t)i, CBM_STREAM_USER, community, 1, &z); z = (float)b * z + (float)a; }
      else if (kind == 1) z = ((float)b - (float)a) * cbm_uniform_f32(seed, stepc, (uint32_t)i, CBM_STREAM_USER, community) + (float)a;
      else z = -cbm_log_f32(1.0f - cbm_uniform_f32(seed, stepc, (uint32_t)i, CBM_STREAM_USER, community)) * (float)a;
      ((float*)out)[i] = z;
    }
  }
  return CBM_OK;
}

/* the `dims` normals of one (step, agent, stream) of the shared stream */
void oracle_normals(int precision, uint64_t seed, int64_t stepc, uint32_t agent, uint32_t stream,
                    uint32_t community, int dims, void* out) {
  if (precision == CBM_F64) cbm_normals(seed, stepc, agent, stream, community, dims, (double*)out);
  else cbm_normals(seed, stepc, agent, stream, community, dims, (float*)out);
}

/* own log / cos-sin, exposed for accuracy tests */
struct MedHandle {
  int prec;
  void* p;
};

void* oracle_medium_create(const cbm_medium_config* cfg) {
  if (!cfg || cfg->dims < 1 || cfg->dims > 3 || cfg->n_fields < 1 ||
      cfg->n_fields > CBM_MEDIUM_MAX_FIELDS)
    return nullptr;
  int64_t nodes = 1;
  for (int d = 0; d < cfg->dims; ++d) {
    if (cfg->n[d] < 4) return nullptr;
    nodes *= cfg->n[d];
  }
  MedHandle* h = new MedHandle;
  h->prec = cfg->precision;
  auto init = [&](auto* M) {
    M->cfg = *cfg;
    for (int d = cfg->dims; d < 3; ++d) M->cfg.n[d] = 1;
    M->nodes = nodes;
    const size_t tot = (size_t)nodes * cfg->n_fields;
    M->u.assign(tot, 0);
    M->u_new.assign(tot, 0);
    M->c_star.assign(tot, 0);
    M->d_star.assign(tot, 0);
    M->src.assign((size_t)nodes, 0);
  };
  if (h->prec == CBM_F64) {
    auto* M = new Med<double>;
    init(M);
    h->p = M;
  } else {
    auto* M = new Med<float>;
    init(M);
    h->p = M;
  }
  return h;
}

void oracle_medium_destroy(void* vh) {
  MedHandle* h = (MedHandle*)vh;
  if (!h) return;
  if (h->prec == CBM_F64) delete (Med<double>*)h->p;
  else delete (Med<float>*)h->p;
  delete h;
}

int oracle_medium_upload(void* vh, const void* fields, const void* source) {
  MedHandle* h = (MedHandle*)vh;
  auto up = [&](auto* M) {
    using T = typename std::remove_reference<decltype(M->u[0])>::type;
    const T* f = (const T*)fields;
    std::copy(f, f + M->u.size(), M->u.begin());
    M->u_new = M->u;
    M->c_star = M->u;
    M->d_star = M->u;
    if (source) std::copy((const T*)source, (const T*)source + M->nodes, M->src.begin());
    else std::fill(M->src.begin(), M->src.end(), (T)0);
    M->t = 0;
  };
  if (h->prec == CBM_F64) up((Med<double>*)h->p);
  else up((Med<float>*)h->p);
  return CBM_OK;
}

int oracle_medium_step(void* vh, int nsteps) {
  MedHandle* h = (MedHandle*)vh;
  for (int s = 0; s < nsteps; ++s) {
    if (h->prec == CBM_F64) medStep(*(Med<double>*)h->p);
    else medStep(*(Med<float>*)h->p);
  }
  return CBM_OK;
}

int oracle_medium_download(void* vh, void* fields, double* t) {
  MedHandle* h = (MedHandle*)vh;
  auto down = [&](auto* M) {
    using T = typename std::remove_reference<decltype(M->u[0])>::type;
    std::copy(M->u.begin(), M->u.end(), (T*)fields);
    if (t) *t = M->t;
  };
  if (h->prec == CBM_F64) down((Med<double>*)h->p);
  else down((Med<float>*)h->p);
  return CBM_OK;
}

double oracle_log_f64(double x) { return cbm_log_f64(x); }
float oracle_log_f32(float x) { return cbm_log_f32(x); }
void oracle_cossin_f64(double w, double* c, double* s) { cbm_cossin_turns_f64(w, c, s); }
void oracle_cossin_f32(float w, float* c, float* s) { cbm_cossin_turns_f32(w, c, s); }
void oracle_philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1,
                   uint32_t* out) {
  cbm_u32x4 r = cbm_philox4x32_10(c0, c1, c2, c3, k0, k1);
  for (int i = 0; i < 4; ++i) out[i] = r.v[i];
}

}  // extern "C"

/* ---------------------------------------------------------------------------
 * Forward-mode dual numbers of the soft-sphere Euler trajectory: the
 * gradient check for the adjoint.  It stands in for a ForwardDiff gradient of
 * the reference's CPU path (ForwardDiff 0.10.36 is in the reference's
 * Manifest.toml but Julia cannot run here).  Directions 0..2 carry
 * d/d(k_rep, k_att, r_rep); further directions carry d/d of chosen initial
 * coordinates.  The cutoff r_att is a plain number (held fixed), as in the
 * adjoint.  Pairs come from a cell grid rebuilt every step, in the
 * reference's CellLinked order; agents are evaluated in parallel (each
 * agent's sum is sequential, so the result does not depend on the threads).
 * ------------------------------------------------------------------------- */
namespace {

constexpr int kDualMax = 12;

struct Dual {
  double v;
  double d[kDualMax];
};

int g_dual_k = 3;

inline Dual dconst(double v) {
  Dual r;
  r.v = v;
  for (int q = 0; q < kDualMax; ++q) r.d[q] = 0.0;
  return r;
}
inline Dual operator+(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v + b.v;
  for (int q = 0; q < g_dual_k; ++q) r.d[q] = a.d[q] + b.d[q];
  return r;
}
inline Dual operator-(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v - b.v;
  for (int q = 0; q < g_dual_k; ++q) r.d[q] = a.d[q] - b.d[q];
  return r;
}
inline Dual operator*(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v * b.v;
  for (int q = 0; q < g_dual_k; ++q) r.d[q] = a.d[q] * b.v + a.v * b.d[q];
  return r;
}
inline Dual operator/(const Dual& a, const Dual& b) {
  Dual r;
  r.v = a.v / b.v;
  for (int q = 0; q < g_dual_k; ++q) r.d[q] = (a.d[q] * b.v - a.v * b.d[q]) / (b.v * b.v);
  return r;
}
inline Dual dsqrt(const Dual& a) {
  Dual r;
  r.v = std::sqrt(a.v);
  for (int q = 0; q < g_dual_k; ++q) r.d[q] = a.d[q] / (2.0 * r.v);
  return r;
}

}  // namespace

extern "C" int oracle_adjoint_dual(const cbm_config* cfg, int64_t n, const double* const* x0,
                                   int nsteps, const double* const* target, int n_seed,
                                   const int64_t* seed_agent, const int32_t* seed_axis,
                                   double* loss, double* dtheta, double* dx0_seeded) {
  if (n_seed < 0 || 3 + n_seed > kDualMax) return CBM_ERR_ARG;
  g_dual_k = 3 + n_seed;
  std::vector<Dual> x[3], xn[3];
  for (int d = 0; d < 3; ++d) {
    x[d].resize((size_t)n);
    xn[d].resize((size_t)n);
    for (int64_t i = 0; i < n; ++i) x[d][(size_t)i] = dconst(x0[d][i]);
  }
  for (int s = 0; s < n_seed; ++s) x[seed_axis[s]][(size_t)seed_agent[s]].d[3 + s] = 1.0;
  Dual k = dconst(cfg->k_rep), a = dconst(cfg->k_att), rho = dconst(cfg->r_rep);
  k.d[0] = 1.0;
  a.d[1] = 1.0;
  rho.d[2] = 1.0;
  const double ratt = cfg->r_att;
  const Dual dt = dconst(cfg->dt);
  // The pair set and the order of the sums are the reference's CellLinked
  // ones, with the grid rebuilt from the committed positions every step:
  // agent i visits the 3^3 cells around its own (cellPosNeigh order, x
  // fastest, neighbors.jl:658-708) and, inside a cell, the agents in
  // ascending index (neighbors.jl:715-747).  Agents beyond simBox fall in the
  // ghost layer (cellPos, neighbors.jl:636-638), so the set is not every pair
  // within the cutoff.
  int64_t ncell[3];
  for (int d = 0; d < 3; ++d)
    ncell[d] = (int64_t)std::ceil((cfg->box_hi[d] - cfg->box_lo[d]) / cfg->cell_edge + 2.0);
  const int64_t n_cells = ncell[0] * ncell[1] * ncell[2];
  std::vector<int64_t> cell((size_t)n), start((size_t)n_cells + 1), order((size_t)n);
  for (int st = 0; st < nsteps; ++st) {
    std::fill(start.begin(), start.end(), 0);
    for (int64_t i = 0; i < n; ++i) {
      int64_t lin = 0, mul = 1;
      for (int d = 0; d < 3; ++d) {
        lin += cellPos1<double>(cfg->cell_edge, x[d][(size_t)i].v, cfg->box_lo[d], cfg->box_hi[d],
                                ncell[d]) * mul;
        mul *= ncell[d];
      }
      cell[(size_t)i] = lin;
      ++start[(size_t)lin + 1];
    }
    for (int64_t c = 0; c < n_cells; ++c) start[(size_t)c + 1] += start[(size_t)c];
    {
      std::vector<int64_t> fill(start.begin(), start.end() - 1);
      for (int64_t i = 0; i < n; ++i) order[(size_t)fill[(size_t)cell[(size_t)i]]++] = i;
    }
#pragma omp parallel for schedule(dynamic, 64) num_threads(g_threads)
    for (int64_t i = 0; i < n; ++i) {
      Dual acc[3] = {dconst(0), dconst(0), dconst(0)};
      const int64_t c = cell[(size_t)i];
      const int64_t q[3] = {c % ncell[0], (c / ncell[0]) % ncell[1], c / (ncell[0] * ncell[1])};
      for (int nb = 0; nb < 27; ++nb) {
        const int64_t p[3] = {q[0] + nb % 3 - 1, q[1] + (nb / 3) % 3 - 1, q[2] + nb / 9 - 1};
        if (p[0] < 0 || p[1] < 0 || p[2] < 0 || p[0] >= ncell[0] || p[1] >= ncell[1] ||
            p[2] >= ncell[2])
          continue;
        const int64_t cn = p[0] + ncell[0] * (p[1] + ncell[1] * p[2]);
        for (int64_t s = start[(size_t)cn]; s < start[(size_t)cn + 1]; ++s) {
          const int64_t j = order[(size_t)s];
          if (j == i) continue;
          double ev[3];
          for (int d = 0; d < 3; ++d) ev[d] = x[d][(size_t)i].v - x[d][(size_t)j].v;
          if (!(ev[0] * ev[0] + ev[1] * ev[1] + ev[2] * ev[2] < ratt * ratt * (1.0 + 1e-9)))
            continue;  // beyond the cutoff for certain
          Dual e[3];
          for (int d = 0; d < 3; ++d) e[d] = x[d][(size_t)i] - x[d][(size_t)j];
          Dual s2 = e[0] * e[0] + e[1] * e[1] + e[2] * e[2];
          Dual dd = dsqrt(s2);
          Dual F;
          if (dd.v < rho.v) F = k * (rho - dd);
          else if (dd.v < ratt) F = dconst(0) - a * (dd - rho);
          else continue;
          Dual sc = F / dd;
          for (int d = 0; d < 3; ++d) acc[d] = acc[d] + sc * e[d];
        }
      }
      for (int d = 0; d < 3; ++d) xn[d][(size_t)i] = x[d][(size_t)i] + acc[d] * dt;
    }
    for (int d = 0; d < 3; ++d) x[d].swap(xn[d]);
  }
  Dual L = dconst(0);
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) {
      Dual e = x[d][(size_t)i] - dconst(target[d][i]);
      L = L + e * e;
    }
  L = L / dconst(3.0 * (double)n);
  *loss = L.v;
  for (int q = 0; q < 3; ++q) dtheta[q] = L.d[q];
  for (int s = 0; s < n_seed; ++s) dx0_seeded[s] = L.d[3 + s];
  return CBM_OK;
}

/* ---------------------------------------------------------------------------
 * rods2D (src/models/rods.jl:61-121) with the Euler integrator: rodForces
 * (rods.jl:21-59) over @loopOverNeighbors, fx/fy/W/pressure written to their
 * "__" copies while du reads the committed (lagged) fx, fy, W, then update!
 * and computeNeighbors! (CellLinked, or all pairs).  The geometry follows
 * CBMMetrics (src/metrics.jl:137-246) statement by statement.  cos/sin of
 * theta are the shared series of include/cbm_rng.h on theta/(2 pi) reduced to
 * [0, 1); x^1.5 is x*sqrt(x) and x^.5 is sqrt(x); in Float32 every constant
 * is Float32.
 * ------------------------------------------------------------------------- */
namespace {

template <typename T>
T jlMin(T a, T b) {
  if (std::isnan(a) || std::isnan(b)) return a + b;
  if (a == b) return std::signbit(b) ? b : a;
  return b < a ? b : a;
}
template <typename T>
T jlMax(T a, T b) {
  if (std::isnan(a) || std::isnan(b)) return a + b;
  if (a == b) return std::signbit(a) ? b : a;
  return b > a ? b : a;
}

template <typename T>
void rodCosSin(T theta, T& c, T& s) {
  T w = theta * (T)0.15915494309189535;
  w = w - std::floor(w);
  if (w >= (T)1) w = w - (T)1;
  if constexpr (std::is_same<T, double>::value) cbm_cossin_turns_f64(w, &c, &s);
  else cbm_cossin_turns_f32(w, &c, &s);
}

/* point2line: projection of (x1, y1) on the line through (x2, y2) at theta2 */
template <typename T>
void point2line(T x1, T y1, T x2, T y2, T c2, T s2, T& px, T& py) {
  T cx = x2 - x1;
  T cy = y2 - y1;
  T t = s2 * cx - c2 * cy;
  px = t * s2 + x1;
  py = -t * c2 + y1;
}

/* pointInsideRod: the point clamped to the rod's segment, scaled by sep */
template <typename T>
void pointInsideRod(T x1, T y1, T l1, T px, T py, T sep, T& ox, T& oy) {
  T ex = x1 - px, ey = y1 - py;
  T d = jlMax(std::sqrt(ex * ex + ey * ey), (T)0.00000001);
  T ux = (px - x1) / d;
  T uy = (py - y1) / d;
  T a = sep * jlMin(d, l1 / (T)2);
  ox = a * ux + x1;
  oy = a * uy + y1;
}

template <typename T>
void intersection2lines(T x1, T y1, T c1, T s1, T x2, T y2, T c2, T s2, T& px, T& py) {
  T cx = x1 - x2, cy = y1 - y2;
  T nrm = c1 * s2 - s1 * c2;
  if (std::fabs(nrm) > (T)0.0000001) {
    T sc = (-s2 * cx + c2 * cy) / nrm;
    px = sc * c1 + x1;
    py = sc * s1 + y1;
  } else {
    px = (x1 + x2) / (T)2;
    py = (y1 + y2) / (T)2;
  }
}

template <typename T>
void rodIntersection(T x1, T y1, T l1, T c1, T s1, T x2, T y2, T l2, T c2, T s2, T& xa, T& ya,
                     T& xb, T& yb) {
  const T sep = (T)0.99;
  xa = x1; ya = y1; xb = x2; yb = y2;
  T px, py;
  intersection2lines(x1, y1, c1, s1, x2, y2, c2, s2, px, py);
  T e0 = x1 - px, e1 = y1 - py;
  T d1 = std::sqrt(e0 * e0 + e1 * e1);
  e0 = x2 - px; e1 = y2 - py;
  T d2 = std::sqrt(e0 * e0 + e1 * e1);
  T nrm = c1 * s2 - s1 * c2;
  if (std::fabs(nrm) < (T)0.000001) {
    T qx, qy;
    point2line(px, py, x1, y1, c1, s1, qx, qy);
    pointInsideRod(x1, y1, l1, qx, qy, sep, xa, ya);
    point2line(px, py, x2, y2, c2, s2, qx, qy);
    pointInsideRod(x2, y2, l2, qx, qy, sep, xb, yb);
  } else if (d1 <= l1 / (T)2 && d2 <= l2 / (T)2) {
    pointInsideRod(x1, y1, l1, px, py, sep, xa, ya);
    pointInsideRod(x2, y2, l2, px, py, sep, xb, yb);
  } else if (d1 <= l1 / (T)2 && d2 > l2 / (T)2) {
    pointInsideRod(x2, y2, l2, px, py, sep, xb, yb);
    point2line(xb, yb, x1, y1, c1, s1, xa, ya);
  } else if (d1 > l1 / (T)2 && d2 <= l2 / (T)2) {
    pointInsideRod(x1, y1, l1, px, py, sep, xa, ya);
    point2line(xa, ya, x2, y2, c2, s2, xb, yb);
  } else {
    pointInsideRod(x2, y2, l2, px, py, sep, xb, yb);
    point2line(xb, yb, x1, y1, c1, s1, xa, ya);
    e0 = x1 - xa; e1 = y1 - ya;
    d2 = std::sqrt(e0 * e0 + e1 * e1);
    if (d2 > l1 / (T)2) {
      pointInsideRod(x1, y1, l1, px, py, sep, xa, ya);
      T qx, qy;
      point2line(xa, ya, x2, y2, c2, s2, qx, qy);
      e0 = x2 - qx; e1 = y2 - qy;
      d2 = std::sqrt(e0 * e0 + e1 * e1);
      if (d2 < l2 / (T)2) { xb = qx; yb = qy; }
    }
  }
}

template <typename T>
struct Rods {
  cbm_rods_config cfg;
  int64_t n = 0;
  int64_t step = 0;
  int err = 0;
  std::vector<T> f[CBM_RODS_FIELDS];
  std::vector<T> cosT, sinT, fx_, fy_, w_, p_;
  int64_t nc[2] = {1, 1};
  std::vector<int64_t> cellCount, cellStart, cellAgents;
};

template <typename T>
int64_t rodCell(const Rods<T>& R, int64_t i) {
  const T edge = (T)R.cfg.cell_edge;
  int64_t px = cellPos1<T>(edge, R.f[CBM_ROD_X][i], (T)R.cfg.box_lo[0], (T)R.cfg.box_hi[0], R.nc[0]);
  int64_t py = cellPos1<T>(edge, R.f[CBM_ROD_Y][i], (T)R.cfg.box_lo[1], (T)R.cfg.box_hi[1], R.nc[1]);
  return px + R.nc[0] * py;
}

/* computeNeighbors! (CellLinked): counts, cumulative sum, rods in index order
 * inside each cell */
template <typename T>
void rodGrid(Rods<T>& R) {
  if (R.cfg.neighbors != CBM_NEIGH_CELL_LINKED) return;
  const int64_t ncell = R.nc[0] * R.nc[1];
  R.cellCount.assign((size_t)ncell, 0);
  R.cellStart.assign((size_t)ncell + 1, 0);
  R.cellAgents.assign((size_t)R.n, 0);
  std::vector<int64_t> cell((size_t)R.n);
  for (int64_t i = 0; i < R.n; ++i) R.cellCount[cell[i] = rodCell(R, i)]++;
  for (int64_t c = 0; c < ncell; ++c) R.cellStart[c + 1] = R.cellStart[c] + R.cellCount[c];
  std::vector<int64_t> fill(R.cellStart.begin(), R.cellStart.end() - 1);
  for (int64_t i = 0; i < R.n; ++i) R.cellAgents[fill[cell[i]]++] = i;
}

template <typename T>
void rodStep(Rods<T>& R) {
  const int64_t N = R.n;
  const T kn = (T)R.cfg.kn, gn = (T)R.cfg.gamma_n, gt = (T)R.cfg.gamma_t, mucc = (T)R.cfg.mu_cc;
  std::vector<T>* F = R.f;
  for (int64_t i = 0; i < N; ++i) rodCosSin(F[CBM_ROD_THETA][i], R.cosT[i], R.sinT[i]);
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < N; ++i) {
    T sfx = 0, sfy = 0, sw = 0, sp = 0;
    const T x = F[CBM_ROD_X][i], y = F[CBM_ROD_Y][i], d = F[CBM_ROD_D][i], l = F[CBM_ROD_L][i];
    const T vx = F[CBM_ROD_VX][i], vy = F[CBM_ROD_VY][i], m = F[CBM_ROD_M][i];
    auto pair = [&](int64_t j) {
      if (j == i) return;
      T xa, ya, xb, yb;
      rodIntersection(x, y, l, R.cosT[i], R.sinT[i], F[CBM_ROD_X][j], F[CBM_ROD_Y][j],
                      F[CBM_ROD_L][j], R.cosT[j], R.sinT[j], xa, ya, xb, yb);
      T rij = std::sqrt((xa - xb) * (xa - xb) + (ya - yb) * (ya - yb));
      if (!(rij > (T)0 && rij < (d + F[CBM_ROD_D][j]) / (T)2)) return;  // Fij = 0: adds +0
      T dl = d - rij;
      T me = m / (T)2;
      T nx = (xa - xb) / rij;
      T ny = (ya - yb) / rij;
      T wx = vx - F[CBM_ROD_VX][j];
      T wy = vy - F[CBM_ROD_VY][j];
      T vn = nx * wx + ny * wy;
      T fn = kn * (dl * std::sqrt(dl)) - gn * me * dl * vn;
      T ft = -jlMin(gt * me * std::sqrt(dl), mucc * fn);
      T fx = fn * nx + ft * (wx - vn * nx);
      T fy = fn * ny + ft * (wy - vn * ny);
      T w = (xa - x) * fy - (ya - y) * fx;
      sfx += fx;
      sfy += fy;
      sw += w;
      sp += std::sqrt(fx * fx + fy * fy);
    };
    if (R.cfg.neighbors == CBM_NEIGH_FULL) {
      for (int64_t j = 0; j < N; ++j) pair(j);
    } else {
      const int64_t c = rodCell(R, i);
      const int64_t cx = c % R.nc[0], cy = c / R.nc[0];
      for (int k = 0; k < 9; ++k) {
        const int64_t qx = cx + k % 3 - 1, qy = cy + k / 3 - 1;
        if (qx < 0 || qx >= R.nc[0] || qy < 0 || qy >= R.nc[1]) continue;
        const int64_t cc = qx + R.nc[0] * qy;
        for (int64_t s = R.cellStart[cc]; s < R.cellStart[cc + 1]; ++s) pair(R.cellAgents[s]);
      }
    }
    R.fx_[i] = sfx;
    R.fy_[i] = sfy;
    R.w_[i] = sw;
    R.p_[i] = sp;
  }
  const T dt = (T)R.cfg.dt, beta = (T)R.cfg.beta, bw = (T)R.cfg.beta_w;
  for (int64_t i = 0; i < N; ++i) {
    const T vx = F[CBM_ROD_VX][i], vy = F[CBM_ROD_VY][i], om = F[CBM_ROD_OMEGA][i];
    const T d = F[CBM_ROD_D][i], l = F[CBM_ROD_L][i], m = F[CBM_ROD_M][i];
    // du of rods.jl:111-116, then Euler u + dt du (integrators.jl Euler)
    T ax = -beta * vx + F[CBM_ROD_FX][i] / m;
    T ay = -beta * vy + F[CBM_ROD_FY][i] / m;
    T aw = F[CBM_ROD_W][i] / (m * ((d + l) * (d + l)) / (T)12 + m * (d * d)) - bw * om;
    F[CBM_ROD_X][i] += vx * dt;
    F[CBM_ROD_Y][i] += vy * dt;
    F[CBM_ROD_VX][i] = vx + ax * dt;
    F[CBM_ROD_VY][i] = vy + ay * dt;
    F[CBM_ROD_THETA][i] += om * dt;
    F[CBM_ROD_OMEGA][i] = om + aw * dt;
  }
  // update!: commit the "__" copies
  F[CBM_ROD_FX] = R.fx_;
  F[CBM_ROD_FY] = R.fy_;
  F[CBM_ROD_W] = R.w_;
  F[CBM_ROD_PRESSURE] = R.p_;
  rodGrid(R);
}

/* rods2dGrowth (rods.jl:123-163): step! with the reference's bookkeeping.
 * agentStepRule! writes the daughters into the "__" copies at rows N + NAdd
 * (@addAgent: the fields not given are the parent's committed values) and
 * records the parent in holeFromRemoveAt (@removeAgent,
 * functionRule.jl:9-111); agentStepDE! integrates rows < N from the committed
 * state; update! fills the holes from the surviving tail
 * (kernelListSurvived / kernelFillHolesParameters, update.jl:15-84) and
 * commits.  Births beyond n_max are dropped in order and every parent is
 * still removed (functionRule.jl:58-70); the overflow is also reported. */
template <typename T>
void rodStepGrowth(Rods<T>& R) {
  const int64_t N = R.n, nMax = R.cfg.n_max;
  std::vector<T>* F = R.f;
  const T kn = (T)R.cfg.kn, gn = (T)R.cfg.gamma_n, gt = (T)R.cfg.gamma_t, mucc = (T)R.cfg.mu_cc;
  for (int64_t i = 0; i < N; ++i) rodCosSin(F[CBM_ROD_THETA][i], R.cosT[i], R.sinT[i]);
  std::vector<T> G[CBM_RODS_FIELDS];
  for (int q = 0; q < CBM_RODS_FIELDS; ++q) G[q] = F[q];
  // agentStepRule!
  std::vector<int64_t> holes;
  std::vector<char> survive((size_t)nMax, 1);
  int64_t nAdd = 0;
  {
    const T lo = (T)R.cfg.l_max - (T)R.cfg.sigma_l_target;
    const T hi = (T)R.cfg.l_max + (T)R.cfg.sigma_l_target;
    for (int64_t i = 0; i < N; ++i) {
      const T l = F[CBM_ROD_L][i];
      if (!(l > F[CBM_ROD_L_TARGET][i])) continue;
      const T d = F[CBM_ROD_D][i], x = F[CBM_ROD_X][i], y = F[CBM_ROD_Y][i];
      const T om = F[CBM_ROD_OMEGA][i];
      // ww = CBMDistributions.uniform(-.1,.1) = (l1 - l0) rand() + l0 (random.jl:15)
      const T ww = ((T)0.1 - (T)-0.1) *
                       cbm_uniform<T>(R.cfg.seed, R.step, (uint32_t)i, CBM_STREAM_ROD_TORQUE, 0u) +
                   (T)-0.1;
      for (int h = 0; h < 2; ++h) {
        // @addAgent: i1New_ = N + NAdd_ + 1 is kept only if nMax_ >= i1New_
        const int64_t slot = N + nAdd;
        if (slot >= nMax) {
          R.err = CBM_ERR_AGENT_OVERFLOW;
          continue;
        }
        nAdd += 1;
        for (int q = 0; q < CBM_RODS_FIELDS; ++q) G[q][slot] = F[q][i];
        const T sg = h == 0 ? (l + d) / (T)4 : -(l + d) / (T)4;
        G[CBM_ROD_X][slot] = sg * R.cosT[i] + x;
        G[CBM_ROD_Y][slot] = sg * R.sinT[i] + y;
        G[CBM_ROD_L][slot] = (l - d) / (T)2;
        G[CBM_ROD_OMEGA][slot] = h == 0 ? om + ww : om - ww;
        G[CBM_ROD_L_TARGET][slot] =
            (hi - lo) * cbm_uniform<T>(R.cfg.seed, R.step, (uint32_t)i,
                                       CBM_STREAM_ROD_TARGET + (uint32_t)h, 0u) + lo;
      }
      holes.push_back(i);  // @removeAgent
      survive[(size_t)i] = 0;
    }
  }
  // agentStepDE!: the neighbor sums and Euler from the committed state
  const T dt = (T)R.cfg.dt, beta = (T)R.cfg.beta, bw = (T)R.cfg.beta_w;
  const T growth = (T)R.cfg.growth, alpha = (T)R.cfg.alpha;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t i = 0; i < N; ++i) {
    T sfx = 0, sfy = 0, sw = 0, sp = 0;
    const T x = F[CBM_ROD_X][i], y = F[CBM_ROD_Y][i], d = F[CBM_ROD_D][i], l = F[CBM_ROD_L][i];
    const T vx = F[CBM_ROD_VX][i], vy = F[CBM_ROD_VY][i], m = F[CBM_ROD_M][i];
    auto pair = [&](int64_t j) {
      if (j == i) return;
      T xa, ya, xb, yb;
      rodIntersection(x, y, l, R.cosT[i], R.sinT[i], F[CBM_ROD_X][j], F[CBM_ROD_Y][j],
                      F[CBM_ROD_L][j], R.cosT[j], R.sinT[j], xa, ya, xb, yb);
      T rij = std::sqrt((xa - xb) * (xa - xb) + (ya - yb) * (ya - yb));
      if (!(rij > (T)0 && rij < (d + F[CBM_ROD_D][j]) / (T)2)) return;
      T dl = d - rij;
      T me = m / (T)2;
      T nx = (xa - xb) / rij;
      T ny = (ya - yb) / rij;
      T wx = vx - F[CBM_ROD_VX][j];
      T wy = vy - F[CBM_ROD_VY][j];
      T vn = nx * wx + ny * wy;
      T fn = kn * (dl * std::sqrt(dl)) - gn * me * dl * vn;
      T ft = -jlMin(gt * me * std::sqrt(dl), mucc * fn);
      T fx = fn * nx + ft * (wx - vn * nx);
      T fy = fn * ny + ft * (wy - vn * ny);
      sfx += fx;
      sfy += fy;
      sw += (xa - x) * fy - (ya - y) * fx;
      sp += std::sqrt(fx * fx + fy * fy);
    };
    if (R.cfg.neighbors == CBM_NEIGH_FULL) {
      for (int64_t j = 0; j < N; ++j) pair(j);
    } else {
      const int64_t c = rodCell(R, i);
      const int64_t cx = c % R.nc[0], cy = c / R.nc[0];
      for (int k = 0; k < 9; ++k) {
        const int64_t qx = cx + k % 3 - 1, qy = cy + k / 3 - 1;
        if (qx < 0 || qx >= R.nc[0] || qy < 0 || qy >= R.nc[1]) continue;
        const int64_t cc = qx + R.nc[0] * qy;
        for (int64_t s = R.cellStart[cc]; s < R.cellStart[cc + 1]; ++s) pair(R.cellAgents[s]);
      }
    }
    const T om = F[CBM_ROD_OMEGA][i];
    T ax = -beta * vx + F[CBM_ROD_FX][i] / m;
    T ay = -beta * vy + F[CBM_ROD_FY][i] / m;
    T aw = F[CBM_ROD_W][i] / (m * ((d + l) * (d + l)) / (T)12 + m * (d * d)) - bw * om;
    T al = growth / ((T)1 + alpha * F[CBM_ROD_PRESSURE][i]);  // rods.jl:138
    G[CBM_ROD_X][i] = x + vx * dt;
    G[CBM_ROD_Y][i] = y + vy * dt;
    G[CBM_ROD_VX][i] = vx + ax * dt;
    G[CBM_ROD_VY][i] = vy + ay * dt;
    G[CBM_ROD_THETA][i] = F[CBM_ROD_THETA][i] + om * dt;
    G[CBM_ROD_OMEGA][i] = om + aw * dt;
    G[CBM_ROD_L][i] = l + al * dt;
    G[CBM_ROD_FX][i] = sfx;
    G[CBM_ROD_FY][i] = sfy;
    G[CBM_ROD_W][i] = sw;
    G[CBM_ROD_PRESSURE][i] = sp;
  }
  // update!
  std::vector<int64_t> repo;
  int64_t lastPos = N + nAdd - 1;
  while ((int64_t)holes.size() > (int64_t)repo.size() && lastPos >= 0) {
    if (survive[(size_t)lastPos]) repo.push_back(lastPos);
    lastPos -= 1;
  }
  for (int q = 0; q < CBM_RODS_FIELDS; ++q)
    for (size_t k = 0; k < repo.size(); ++k)
      if (holes[k] < repo[k]) G[q][(size_t)holes[k]] = G[q][(size_t)repo[k]];
  R.n = N + nAdd - (int64_t)holes.size();
  for (int q = 0; q < CBM_RODS_FIELDS; ++q) F[q] = G[q];
  R.step += 1;
  rodGrid(R);
}

struct RodHandle {
  int prec;
  void* p;
};

}  // namespace

extern "C" {

void* oracle_rods_create(const cbm_rods_config* cfg) {
  if (!cfg) return nullptr;
  RodHandle* h = new RodHandle;
  h->prec = cfg->precision;
  auto init = [&](auto* R) {
    R->cfg = *cfg;
    if (cfg->neighbors == CBM_NEIGH_CELL_LINKED)
      for (int d = 0; d < 2; ++d)
        R->nc[d] = (int64_t)std::ceil((cfg->box_hi[d] - cfg->box_lo[d]) / cfg->cell_edge + 2.0);
  };
  if (h->prec == CBM_F64) {
    auto* R = new Rods<double>;
    init(R);
    h->p = R;
  } else {
    auto* R = new Rods<float>;
    init(R);
    h->p = R;
  }
  return h;
}

void oracle_rods_destroy(void* vh) {
  RodHandle* h = (RodHandle*)vh;
  if (!h) return;
  if (h->prec == CBM_F64) delete (Rods<double>*)h->p;
  else delete (Rods<float>*)h->p;
  delete h;
}

/* fields: CBM_ROD_PRESSURE arrays of n (pressure starts at zero) */
int oracle_rods_upload(void* vh, int64_t n, const void* const* fields) {
  RodHandle* h = (RodHandle*)vh;
  auto up = [&](auto* R) {
    using T = typename std::remove_reference<decltype(R->cosT[0])>::type;
    R->n = n;
    R->step = 0;
    R->err = 0;
    const bool grow = R->cfg.growth_model != 0;
    const size_t rows = grow ? (size_t)std::max<int64_t>(n, R->cfg.n_max) : (size_t)n;
    for (int q = 0; q < CBM_RODS_FIELDS; ++q) {
      R->f[q].assign(rows, (T)0);
      if (q < CBM_ROD_PRESSURE || (grow && q == CBM_ROD_L_TARGET))
        std::copy((const T*)fields[q], (const T*)fields[q] + n, R->f[q].begin());
    }
    for (auto* v : {&R->cosT, &R->sinT, &R->fx_, &R->fy_, &R->w_, &R->p_}) v->assign(rows, (T)0);
    rodGrid(*R);
  };
  if (h->prec == CBM_F64) up((Rods<double>*)h->p);
  else up((Rods<float>*)h->p);
  return CBM_OK;
}

int oracle_rods_step(void* vh, int nsteps) {
  RodHandle* h = (RodHandle*)vh;
  for (int s = 0; s < nsteps; ++s) {
    if (h->prec == CBM_F64) {
      auto& R = *(Rods<double>*)h->p;
      if (R.cfg.growth_model) rodStepGrowth(R);
      else rodStep(R);
    } else {
      auto& R = *(Rods<float>*)h->p;
      if (R.cfg.growth_model) rodStepGrowth(R);
      else rodStep(R);
    }
  }
  return CBM_OK;
}

int oracle_rods_download(void* vh, void* const* fields) {
  RodHandle* h = (RodHandle*)vh;
  auto down = [&](auto* R) {
    using T = typename std::remove_reference<decltype(R->cosT[0])>::type;
    for (int q = 0; q < CBM_RODS_FIELDS; ++q)
      if (fields[q]) std::copy(R->f[q].begin(), R->f[q].begin() + R->n, (T*)fields[q]);
  };
  if (h->prec == CBM_F64) down((Rods<double>*)h->p);
  else down((Rods<float>*)h->p);
  return CBM_OK;
}

/* one uniform u in [0, 1) of the shared stream, for transcriptions in tests */
double oracle_uniform_f64(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                          uint32_t community) {
  return cbm_uniform_f64(seed, step, agent, stream, community);
}

float oracle_uniform_f32(uint64_t seed, int64_t step, uint32_t agent, uint32_t stream,
                         uint32_t community) {
  return cbm_uniform_f32(seed, step, agent, stream, community);
}

/* the rod count and the error code (CBM_ERR_AGENT_OVERFLOW) of the last steps */
int64_t oracle_rods_count(void* vh, int* err) {
  RodHandle* h = (RodHandle*)vh;
  if (h->prec == CBM_F64) {
    auto& R = *(Rods<double>*)h->p;
    if (err) *err = R.err;
    return R.n;
  }
  auto& R = *(Rods<float>*)h->p;
  if (err) *err = R.err;
  return R.n;
}

/* rodForces of one pair, for the pin against a transcription of rods.jl */
int oracle_rod_pair_f64(const double* a, const double* b, const double* k, double* out) {
  double c1, s1, c2, s2;
  rodCosSin(a[4], c1, s1);
  rodCosSin(b[4], c2, s2);
  double xa, ya, xb, yb;
  rodIntersection(a[0], a[1], a[3], c1, s1, b[0], b[1], b[3], c2, s2, xa, ya, xb, yb);
  out[3] = xa; out[4] = ya; out[5] = xb; out[6] = yb;
  out[0] = out[1] = out[2] = 0.0;
  double rij = std::sqrt((xa - xb) * (xa - xb) + (ya - yb) * (ya - yb));
  if (!(rij > 0.0 && rij < (a[2] + b[2]) / 2.0)) return 0;
  double dl = a[2] - rij, me = a[7] / 2.0;
  double nx = (xa - xb) / rij, ny = (ya - yb) / rij;
  double wx = a[5] - b[5], wy = a[6] - b[6];
  double vn = nx * wx + ny * wy;
  double fn = k[0] * (dl * std::sqrt(dl)) - k[1] * me * dl * vn;
  double ft = -jlMin(k[2] * me * std::sqrt(dl), k[3] * fn);
  out[0] = fn * nx + ft * (wx - vn * nx);
  out[1] = fn * ny + ft * (wy - vn * ny);
  out[2] = (xa - a[0]) * out[1] - (ya - a[1]) * out[0];
  return 1;
}

}  // extern "C"
