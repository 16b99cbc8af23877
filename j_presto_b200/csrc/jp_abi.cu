// jp_abi.cu -- host side of the engine: the C ABI of include/jpgpu.h.
//
// jp_create derives, in C++ on the host, what md_run's set-up derives in Fortran:
//   * chgmod = q*sqrt(332.06378/eps)                      inpcls.f90:215-227
//   * SHAKE groups ordered 2/3/4 atoms, squared lengths     setshk.f90 redshk/modshk
//   * bonds/angles whose pair is a SHAKE constraint dropped setshk.f90 reabnd/reaang
//   * 1-4 pairs of torsions with nbf=1, scales min(s_i,s_j) incel.f90:972-987,
//                                                           inptpl.f90:453-462, incel.f90:1084
//   * ZD constants, dself, excess list                       incel.f90:29-39, :627-689
//   * degrees of freedom (whole / per sub-system)            md.f90:116-183
// and lays out device memory (see jp_common.cuh).  jp_step replays one CUDA graph per
// MD step (forces + integration) and one per list rebuild.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <new>
#include <set>
#include <string>
#include <vector>

#include "jp_kernels.h"

using namespace jp;

namespace {

struct Timing {
  bool enabled = false;
  double total_ms = 0.0;
  double phase_ms[4] = {0, 0, 0, 0};
  int launches[4] = {0, 0, 0, 0};
};

// The dynamic state an MD step changes, copied aside on the device so that a step whose
// SHAKE failed can be undone (verlethe.f90:552-574 restores cord, vel and lambda and redoes
// the step with half the time step): coordinates, velocities, lambda and its velocity, the
// CMM far-field cache, the energy histograms, the step counters, and the per-step energy
// and temperature record of the history row being written.
struct Snap {
  double *x = nullptr, *v = nullptr, *lam = nullptr, *gwk = nullptr;
  long long *cmm_e = nullptr;
  unsigned long long *hist = nullptr;
  int *ctr = nullptr;
  double *ene_row = nullptr, *temp_row = nullptr;
  unsigned long long *acnt = nullptr, *acnt2 = nullptr;   // ALSD lambda histograms
  double *af = nullptr, *af2 = nullptr;
  int row = 0;   // history row the record copies belong to
};

}  // namespace

struct jp_ctx {
  int nrep = 0;
  jp_params prm{};
  int device = 0;
  int natom = 0, nblk = 0, nslot = 0, nunit = 0, nterm = 0, nsub = 0, nkeys = 0, nkin = 8;
  int ncol = 0;
  int tile_cap_total = 0, nchunk = 0;
  std::vector<Rep> reps;
  std::vector<int> rep_natom;
  DevPtrs P{};
  ZdConst zc{};
  IntConst ic{};
  double qscale = 1.0;
  bool fp64 = false;
  bool minimg = true;
  int pair_warps = 0;
  int nsm = 148;                    // the device's SM count
  bool alsd = false;                // some replica has ALSD classes (lambda)
  bool split = false;               // some replica keeps partial-McMD class-1 forces apart
  bool classes = false;             // alsd or split: class energies are kept
  bool cmm = false;                 // CAL15M= CMM
  bool hbond = false;               // some type pair has the 10-12 H-bond term
  int hb_cap = 0;                   // capacity of the H-bond pair list
  int nres = 0;                     // restraint and CAP terms
  int ngroups = 0;                  // SHAKE groups (units of 2-4 atoms)
  int cmm_ncell[6] = {0, 0, 0, 0, 0, 0};   // cells per level over all replicas
  int cmm_nlev = 0;                 // most levels of any replica
  int cano_grid = 1;
  int hist_cap = 1024;
  long long idloop = 0;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;       // the bonded kernel's branch of the step graph
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaGraphExec_t g_step = nullptr, g_rebuild = nullptr;
  int *scan_scratch = nullptr;
  std::vector<void *> allocs;
  cudaEvent_t ev_a = nullptr, ev_b = nullptr;
  std::vector<cudaEvent_t> tev;
  Timing tm;
  int launches_step = 0, launches_rebuild = 0;
  bool rebuild_pending = false;     // the list rebuild due after the last step taken
  // block-shape tuning: per replica and candidate the xy column grid, the compact tiles
  // the list needed with it, and the candidate kept
  std::vector<int> tune_grid;       // [nrep][JP_TUNE_CANDIDATES][2]
  std::vector<long long> tune_tiles;  // [nrep][JP_TUNE_CANDIDATES]
  std::vector<int> tune_pick;       // [nrep]
  Snap snap[3];                     // segment start, step start, a sub-step's accepted state
  bool snap_ready = false;
  int nstep_retry = 0;              // steps redone with a halved time step (all calls)
};

namespace {

const char *g_last_err = "";

#define CK(call)                                                      \
  do {                                                                \
    cudaError_t e_ = (call);                                          \
    if (e_ != cudaSuccess) {                                          \
      g_last_err = cudaGetErrorString(e_);                            \
      std::fprintf(stderr, "jpgpu: %s at %s:%d\n", g_last_err, __FILE__, __LINE__); \
      return JP_E_CUDA;                                               \
    }                                                                 \
  } while (0)

template <class T>
int dalloc(jp_ctx *c, T **p, size_t n) {
  if (n == 0) n = 1;
  void *q = nullptr;
  cudaError_t e = cudaMalloc(&q, n * sizeof(T));
  if (e != cudaSuccess) {
    g_last_err = cudaGetErrorString(e);
    return JP_E_CUDA;
  }
  cudaMemset(q, 0, n * sizeof(T));
  c->allocs.push_back(q);
  *p = static_cast<T *>(q);
  return 0;
}

template <class T>
int dput(jp_ctx *c, T **p, const std::vector<T> &h) {
  int r = dalloc(c, p, h.size());
  if (r) return r;
  if (!h.empty()) {
    cudaError_t e = cudaMemcpy(*p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { g_last_err = cudaGetErrorString(e); return JP_E_CUDA; }
  }
  return 0;
}

constexpr double kEekcal = 332.06378;
// column-edge factors the block-shape tuner tries (1 = columns of edge (32/density)^(1/3),
// near-cubic 32-atom blocks); kTuneDefault is the unit factor
constexpr double kTuneScale[JP_TUNE_CANDIDATES] = {0.84, 0.92, 1.0, 1.09, 1.19};
constexpr int kTuneDefault = 2;

void set_grid(Rep &R, const int *g) {
  for (int k = 0; k < 2; ++k) {
    R.grid[k] = g[k];
    R.cell[k] = R.box[k] / g[k];
  }
}
// bound of a grid-barrier wait in the integration (SM cycles: about one second)
constexpr long long kDefaultWaitCycles = 2000000000LL;
constexpr int kGeCap = JP_GE_MAX_WINDOWS * (JP_GE_MAX_DEG + 3);   // doubles per replica

// a .nf weight in the device layout: per window [low, high, c0..cndeg]
void pack_ge(const jp_ge &g, double *dst) {
  int o = 0;
  for (int w = 0; w < g.nwindow; ++w) {
    dst[o++] = g.low[w];
    dst[o++] = g.high[w];
    for (int k = 0; k <= g.ndeg; ++k) dst[o++] = g.coef[w * (g.ndeg + 1) + k];
  }
}

// ---- rebuild: cells + tiles -------------------------------------------------------------
void enqueue_rebuild(jp_ctx *c) {
  DevPtrs &P = c->P;
  cudaStream_t st = c->st;
  const int nt = 256;
  cudaMemsetAsync(P.hist, 0, sizeof(int) * (c->nkeys + 1), st);
  cudaMemsetAsync(P.cursor, 0, sizeof(int) * (c->nkeys + 1), st);
  cudaMemsetAsync(P.rep_hmax, 0, sizeof(float) * 3 * c->nrep, st);
  int ncmm = 0;
  if (c->cmm) {   // celpar_CB + celoth + celpol: cells and multipoles at this rebuild
    int ntot = 0;
    for (int l = 1; l <= c->cmm_nlev; ++l) ntot += c->cmm_ncell[l];
    cudaMemsetAsync(P.cmm_c0, 0, sizeof(double) * 3 * c->nrep, st);
    cudaMemsetAsync(P.cmm_pop, 0, sizeof(int) * ntot, st);
    cudaMemsetAsync(P.cmm_raw, 0, sizeof(double) * 10 * c->cmm_ncell[1], st);
    launch_cmm_rebuild(P, c->natom, c->nrep, c->cmm_ncell[1], c->cmm_ncell, c->cmm_nlev, st);
    ncmm = 3 + std::max(0, c->cmm_nlev - 1);
  }
  k_cell_key<<<(c->natom + nt - 1) / nt, nt, 0, st>>>(P, c->natom);
  int nl = 10;   // the single kernels below
  nl += scan_exclusive(P.hist, P.hist_scan, c->nkeys + 1, c->scan_scratch, nullptr, st);
  k_scatter<<<(c->natom + nt - 1) / nt, nt, 0, st>>>(P, c->natom);
  k_sort_bins<<<(c->nkeys + nt - 1) / nt, nt, 0, st>>>(P, c->nkeys);
  k_col_count<<<(c->ncol + nt - 1) / nt, nt, 0, st>>>(P, c->ncol);
  nl += scan_exclusive(P.col_nb, P.col_blk, c->ncol + 1, c->scan_scratch, nullptr, st);
  k_clear_slots<<<(c->nslot + nt - 1) / nt, nt, 0, st>>>(P, c->nslot, c->zc.nt1 - 1);
  k_fill_slots<<<(c->natom + nt - 1) / nt, nt, 0, st>>>(P, c->natom);
  k_excl_slots<<<(c->natom + nt - 1) / nt, nt, 0, st>>>(P, c->natom);
  k_block_setup<<<(c->nblk * 32 + nt - 1) / nt, nt, 0, st>>>(P, c->nblk, c->qscale);
  if (c->fp64) k_fill_pos_d<<<(c->nslot + nt - 1) / nt, nt, 0, st>>>(P, c->nslot, c->qscale);
  const double rlim = c->zc.rlim;   // rc + 1.5; CMM: the farthest near-field pair
  const double rc = c->prm.cutoff;
  const int nwb = (c->nchunk * 32 + 127) / 128;
  launch_tile_scan(P, c->nchunk, rlim * rlim, (float)rlim, rc * rc, c->cmm, st);
  nl += scan_exclusive(P.chunk_cnt, P.chunk_off, c->nchunk + 1, c->scan_scratch, P.ntiles, st);
  for (int h = 0; h < 2; ++h)   // the entries of each half block
    nl += scan_exclusive(P.chunk_ent + h * (c->nchunk + 1), P.chunk_eoff + h * (c->nchunk + 1), c->nchunk + 1,
                         c->scan_scratch, nullptr, st);
  k_tile_emit<<<nwb, 128, 0, st>>>(P, c->nchunk, c->cmm ? 1 : 0);
  nl += launch_compact_tiles(P, c->nblk, c->nchunk, c->nsm, c->cmm, c->scan_scratch, st);
  if (c->hbond) launch_hb_list(P, c->hb_cap, c->zc.nt1, c->nblk, st);
  c->launches_rebuild = nl + (c->fp64 ? 1 : 0) + ncmm + (c->hbond ? 1 : 0);
}

// ---- one MD step ------------------------------------------------------------------------
void enqueue_zero(jp_ctx *c, bool count) {
  DevPtrs &P = c->P;
  cudaStream_t st = c->st;
  if (c->fp64) cudaMemsetAsync(P.grd, 0, sizeof(double) * 3 * c->natom, st);
  else cudaMemsetAsync(P.frc, 0, sizeof(long long) * 3 * c->natom, st);
  if (c->split && c->fp64) cudaMemsetAsync(P.grd1, 0, sizeof(double) * 3 * c->natom, st);
  if (c->split && !c->fp64) cudaMemsetAsync(P.frc1, 0, sizeof(long long) * 3 * c->natom, st);
  cudaMemsetAsync(P.ene_fix, 0, sizeof(long long) * (16 * c->nrep + 1), st);   // + tile counter
  if (c->classes) cudaMemsetAsync(P.ene_cls, 0, sizeof(long long) * 4 * c->nrep, st);
  if (count) cudaMemsetAsync(P.pair_cnt, 0, sizeof(long long) * c->nrep, st);
}

// the non-bonded forces: pair tiles, and with CMM the far field (recomputed every CMMUPD
// steps by the step counter, or always with force_far: a single-point evaluation)
void enqueue_pair(jp_ctx *c, bool count, bool force_far = false) {
  if (c->fp64) launch_pair_fp64(c->P, c->zc, c->pair_warps, count, c->alsd, c->split, c->st);
  else launch_pair_mixed(c->P, c->zc, c->pair_warps, count, c->alsd, c->split, c->st);
  if (c->hbond) launch_hbond(c->P, c->hb_cap, c->zc.rc2, c->zc.nt1, c->fp64, c->classes, c->st);
  if (c->cmm) launch_cmm_far(c->P, c->natom, c->nrep, c->fp64, force_far, c->qscale * c->qscale, c->st);
}

void enqueue_forces(jp_ctx *c, bool count, bool force_far = false) {
  enqueue_zero(c, count);
  enqueue_pair(c, count, force_far);
}

void enqueue_bonded(jp_ctx *c) {
  launch_bonded(c->P, c->nterm, c->fp64, c->zc.bcoeff, c->zc.fcoeff, c->classes, c->st);
  launch_restraints(c->P, c->nres, c->fp64, c->classes, c->st);
}

void enqueue_integrate(jp_ctx *c) {
  DevPtrs &P = c->P;
  if (c->ic.ge_prescaled) launch_ge_scale(P, c->ic, c->st);
  launch_integrate(P, c->ic, c->nunit, c->fp64, c->cano_grid, c->st);
}

void drop_graphs(jp_ctx *c) {
  if (c->g_step) cudaGraphExecDestroy(c->g_step);
  if (c->g_rebuild) cudaGraphExecDestroy(c->g_rebuild);
  c->g_step = c->g_rebuild = nullptr;
}

int launches_per_step(const jp_ctx *c) {
  int n = 1;                       // pair
  n += c->nterm > 0 ? 1 : 0;      // bonded
  n += integrate_launches(c->ic, c->cano_grid);   // the integration (one or per-phase kernels)
  n += c->ic.ge_prescaled ? 1 : 0; // k_ge_scale
  n += c->cmm ? 2 : 0;             // k_cmm_far, k_cmm_energy
  n += c->hbond ? 1 : 0;           // k_hbond
  n += c->nres > 0 ? 1 : 0;        // k_restraints
  return n;
}

int capture(jp_ctx *c, cudaGraphExec_t *out, bool rebuild) {
  cudaGraph_t g;
  CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
  if (rebuild) {
    enqueue_rebuild(c);
  } else {
    // forces and energy slots start at zero (the integration of the previous step, or the
    // call that last used them, left them so); the bonded terms run beside the pair tiles
    // (both only add into the accumulators, as order-independent integer sums on the mixed
    // path), joined before the integration
    if (c->classes) cudaMemsetAsync(c->P.ene_cls, 0, sizeof(long long) * 4 * c->nrep, c->st);
    CK(cudaEventRecord(c->ev_fork, c->st));
    CK(cudaStreamWaitEvent(c->st2, c->ev_fork, 0));
    launch_bonded(c->P, c->nterm, c->fp64, c->zc.bcoeff, c->zc.fcoeff, c->classes, c->st2);
    launch_restraints(c->P, c->nres, c->fp64, c->classes, c->st2);
    CK(cudaEventRecord(c->ev_join, c->st2));
    enqueue_pair(c, false);
    CK(cudaStreamWaitEvent(c->st, c->ev_join, 0));
    enqueue_integrate(c);
  }
  CK(cudaStreamEndCapture(c->st, &g));
  CK(cudaGraphInstantiate(out, g, 0));
  CK(cudaGraphDestroy(g));
  return 0;
}

int check_status(jp_ctx *c) {
  unsigned s = 0;
  CK(cudaMemcpy(&s, c->P.status, sizeof(unsigned), cudaMemcpyDeviceToHost));
  if (s == 0) return JP_OK;
  CK(cudaMemset(c->P.status, 0, sizeof(unsigned)));
  // an integration that stopped early left its barrier, sums and accumulators: clear them
  CK(cudaMemset(c->P.bar, 0, sizeof(unsigned) * 4));
  if (c->fp64) CK(cudaMemset(c->P.grd, 0, sizeof(double) * 3 * c->natom));
  else CK(cudaMemset(c->P.frc, 0, sizeof(long long) * 3 * c->natom));
  if (c->split && c->fp64) CK(cudaMemset(c->P.grd1, 0, sizeof(double) * 3 * c->natom));
  if (c->split && !c->fp64) CK(cudaMemset(c->P.frc1, 0, sizeof(long long) * 3 * c->natom));
  CK(cudaMemset(c->P.ene_fix, 0, sizeof(long long) * (16 * c->nrep + 1)));
  CK(cudaMemset(c->P.kin_fix, 0, sizeof(long long) * c->nkin * c->nsub));
  if (c->ic.stop) CK(cudaMemset(c->P.com, 0, sizeof(double) * c->ic.ncom * c->ic.nrep * 16));
  if (s & ERR_TIMEOUT) return JP_E_TIMEOUT;
  if (s & ERR_LIST_OVERFLOW) return JP_E_LIST_OVERFLOW;
  if (s & ERR_NONFINITE) return JP_E_NONFINITE;
  if (s & ERR_FIX_OVERFLOW) return JP_E_FIXED_OVERFLOW;
  if (s & ERR_FREE_WINDOW) return JP_E_FREE_WINDOW;
  if (s & ERR_CMM_GRID) return JP_E_CELL_OVERFLOW;
  if (s & ERR_STOP_MASS) return JP_E_STOP_MASS;
  if (s & ERR_STOP_SINGULAR) return JP_E_STOP_SINGULAR;
  if (s & ERR_SHAKE_SINGULAR) return JP_E_SHAKE_SINGULAR;
  if (s & ERR_SHAKE_NOCONV) return JP_W_SHAKE_NOT_CONVERGED;
  return JP_E_INVALID;
}

// ---- undoing a step: SHAKE failure retry (verlethe.f90:552-574, :745-752) ------------------
__global__ void k_check_finite(const double *a, long long n, unsigned *status) {
  bool bad = false;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    bad |= !isfinite(a[i]);
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(status, ERR_NONFINITE);
}

int snap_alloc(jp_ctx *c) {
  if (c->snap_ready) return 0;
  int e = 0;
  for (Snap &S : c->snap) {
    e |= dalloc(c, &S.x, 3 * (size_t)c->natom);
    e |= dalloc(c, &S.v, 3 * (size_t)c->natom);
    e |= dalloc(c, &S.lam, 2 * (size_t)c->nrep);
    if (c->cmm) {
      e |= dalloc(c, &S.gwk, 3 * (size_t)c->natom);
      e |= dalloc(c, &S.cmm_e, (size_t)c->nrep);
    }
    e |= dalloc(c, &S.hist, (size_t)c->nrep * JP_GE_MAX_BINS);
    e |= dalloc(c, &S.ctr, 2);
    e |= dalloc(c, &S.ene_row, (size_t)c->nrep * JP_MAXENE);
    e |= dalloc(c, &S.temp_row, (size_t)c->nrep);
    if (c->P.alsd_cnt) {
      e |= dalloc(c, &S.acnt, (size_t)c->nrep * JP_ALSD_MAX_LBINS);
      e |= dalloc(c, &S.af, (size_t)c->nrep * JP_ALSD_MAX_LBINS);
      e |= dalloc(c, &S.acnt2, (size_t)c->nrep * JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS);
      e |= dalloc(c, &S.af2, (size_t)c->nrep * JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS);
    }
  }
  if (e) return JP_E_CUDA;
  c->snap_ready = true;
  return 0;
}

// copy the whole state (to = true: into S; false: back from S), history row `row`
int snap_copy(jp_ctx *c, Snap &S, bool to, int row) {
  DevPtrs &P = c->P;
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  auto cp = [&](void *snap, void *live, size_t bytes) {
    return to ? cudaMemcpyAsync(snap, live, bytes, k, c->st) : cudaMemcpyAsync(live, snap, bytes, k, c->st);
  };
  if (to) S.row = row;
  const size_t n3 = 3 * (size_t)c->natom * sizeof(double);
  CK(cp(S.x, P.x, n3));
  CK(cp(S.v, P.v, n3));
  CK(cp(S.lam, P.lam, 2 * (size_t)c->nrep * sizeof(double)));
  if (c->cmm) {
    CK(cp(S.gwk, P.gwk, n3));
    CK(cp(S.cmm_e, P.cmm_e, (size_t)c->nrep * sizeof(long long)));
  }
  CK(cp(S.hist, P.ge_hist, (size_t)c->nrep * JP_GE_MAX_BINS * sizeof(unsigned long long)));
  CK(cp(S.ctr, P.step_ctr, 2 * sizeof(int)));
  CK(cp(S.ene_row, P.ene_hist + (size_t)S.row * c->nrep * JP_MAXENE, (size_t)c->nrep * JP_MAXENE * sizeof(double)));
  CK(cp(S.temp_row, P.temp_hist + (size_t)S.row * c->nrep, (size_t)c->nrep * sizeof(double)));
  if (S.acnt) {
    const size_t n1 = (size_t)c->nrep * JP_ALSD_MAX_LBINS, n2 = n1 * JP_ALSD_MAX_EBINS;
    CK(cp(S.acnt, P.alsd_cnt, n1 * sizeof(unsigned long long)));
    CK(cp(S.af, P.alsd_f, n1 * sizeof(double)));
    CK(cp(S.acnt2, P.alsd_cnt2, n2 * sizeof(unsigned long long)));
    CK(cp(S.af2, P.alsd_f2, n2 * sizeof(double)));
  }
  if (!to) launch_update_pos(P, c->nslot, c->fp64, c->qscale, c->st);
  return 0;
}

// the part of the state that belongs to replica r (S's history row)
int snap_copy_rep(jp_ctx *c, Snap &S, bool to, int r) {
  DevPtrs &P = c->P;
  const Rep &R = c->reps[r];
  const cudaMemcpyKind k = cudaMemcpyDeviceToDevice;
  auto cp = [&](void *snap, void *live, size_t bytes) {
    return to ? cudaMemcpyAsync(snap, live, bytes, k, c->st) : cudaMemcpyAsync(live, snap, bytes, k, c->st);
  };
  const size_t a3 = 3 * (size_t)R.atom0, n3 = 3 * (size_t)R.natom * sizeof(double);
  CK(cp(S.x + a3, P.x + a3, n3));
  CK(cp(S.v + a3, P.v + a3, n3));
  CK(cp(S.lam + 2 * r, P.lam + 2 * r, 2 * sizeof(double)));
  if (c->cmm) {
    CK(cp(S.gwk + a3, P.gwk + a3, n3));
    CK(cp(S.cmm_e + r, P.cmm_e + r, sizeof(long long)));
  }
  const size_t h = (size_t)r * JP_GE_MAX_BINS;
  CK(cp(S.hist + h, P.ge_hist + h, JP_GE_MAX_BINS * sizeof(unsigned long long)));
  const size_t e = ((size_t)S.row * c->nrep + r) * JP_MAXENE;
  CK(cp(S.ene_row + (size_t)r * JP_MAXENE, P.ene_hist + e, JP_MAXENE * sizeof(double)));
  CK(cp(S.temp_row + r, P.temp_hist + (size_t)S.row * c->nrep + r, sizeof(double)));
  if (S.acnt) {
    const size_t o1 = (size_t)r * JP_ALSD_MAX_LBINS, n2 = (size_t)JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS;
    CK(cp(S.acnt + o1, P.alsd_cnt + o1, JP_ALSD_MAX_LBINS * sizeof(unsigned long long)));
    CK(cp(S.af + o1, P.alsd_f + o1, JP_ALSD_MAX_LBINS * sizeof(double)));
    CK(cp(S.acnt2 + r * n2, P.alsd_cnt2 + r * n2, n2 * sizeof(unsigned long long)));
    CK(cp(S.af2 + r * n2, P.alsd_f2 + r * n2, n2 * sizeof(double)));
  }
  if (!to) launch_update_pos(P, c->nslot, c->fp64, c->qscale, c->st);
  return 0;
}

// after an integration that failed: the status word, barrier, sums and accumulators back to
// their between-steps state (what check_status clears), without mapping the status
int clear_after_failure(jp_ctx *c) {
  DevPtrs &P = c->P;
  CK(cudaMemsetAsync(P.status, 0, sizeof(unsigned), c->st));
  CK(cudaMemsetAsync(P.bar, 0, sizeof(unsigned) * 4, c->st));
  if (c->fp64) CK(cudaMemsetAsync(P.grd, 0, sizeof(double) * 3 * c->natom, c->st));
  else CK(cudaMemsetAsync(P.frc, 0, sizeof(long long) * 3 * c->natom, c->st));
  if (c->split && c->fp64) CK(cudaMemsetAsync(P.grd1, 0, sizeof(double) * 3 * c->natom, c->st));
  if (c->split && !c->fp64) CK(cudaMemsetAsync(P.frc1, 0, sizeof(long long) * 3 * c->natom, c->st));
  CK(cudaMemsetAsync(P.ene_fix, 0, sizeof(long long) * (16 * c->nrep + 1), c->st));
  CK(cudaMemsetAsync(P.kin_fix, 0, sizeof(long long) * c->nkin * c->nsub, c->st));
  if (c->ic.stop) CK(cudaMemsetAsync(P.com, 0, sizeof(double) * c->ic.ncom * c->ic.nrep * 16, c->st));
  if (c->classes) CK(cudaMemsetAsync(P.ene_cls, 0, sizeof(long long) * 4 * c->nrep, c->st));
  CK(cudaMemsetAsync(P.rep_fail, 0, sizeof(int) * c->nrep, c->st));
  return 0;
}

int read_status(jp_ctx *c, unsigned *s) {
  CK(cudaMemcpyAsync(s, c->P.status, sizeof(unsigned), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return 0;
}

constexpr unsigned kShakeBits = ERR_SHAKE_NOCONV | ERR_SHAKE_SINGULAR;

// A step whose SHAKE failed in some replicas (the device state is the failed step's result,
// `pre` holds the state before it, history row `row`).  As verlethe.f90:552-574 does for its
// one system, each failing replica goes back to its state before the step and redoes it in
// sub-steps: on a failure the sub-step is undone and the time step halved (jshk, ishk
// doubled), after each successful sub-step ishk advances and two completed halves merge
// back (:745-752), until ishk = jshk; below 1 % of dt the step is abandoned (-9999).
// Replicas are independent, so the others keep the step they completed.  Each sub-step
// runs the whole force and integration sequence on every replica with the reduced time
// step and keeps only the redone replica's result.
int retry_step(jp_ctx *c, Snap &pre, int row) {
  std::vector<int> fail(c->nrep, 0);
  CK(cudaMemcpyAsync(fail.data(), c->P.rep_fail, sizeof(int) * c->nrep, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  if (int e = clear_after_failure(c)) return e;
  // a step that started from non-finite coordinates or velocities is not a SHAKE failure
  for (const double *a : {pre.x, pre.v})
    k_check_finite<<<64, 256, 0, c->st>>>(a, 3LL * c->natom, c->P.status);
  unsigned st0 = 0;
  if (int e = read_status(c, &st0)) return e;
  if (st0) return check_status(c);
  Snap &post = c->snap[2];
  for (int r = 0; r < c->nrep; ++r)
    if (fail[r])
      if (int e = snap_copy_rep(c, pre, false, r)) return e;
  if (int e = snap_copy(c, post, true, row)) return e;
  int ctr_pre[2];
  CK(cudaMemcpyAsync(ctr_pre, pre.ctr, sizeof(ctr_pre), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  const double dt = c->prm.dt;
  IntConst ic = c->ic;
  for (int r = 0; r < c->nrep; ++r) {
    if (!fail[r]) continue;
    double T = 0.5 * dt;
    int ishk = 0, jshk = 2;
    ++c->nstep_retry;
    for (;;) {
      // one sub-step of every replica from the saved state; replica r's result is kept
      CK(cudaMemcpyAsync(c->P.step_ctr, ctr_pre, sizeof(ctr_pre), cudaMemcpyHostToDevice, c->st));
      ic.dt = T;
      // the step's histogram visit is the one of its last sub-step (the .ene record GEprep
      // reads holds the energy of that sub-step): only a sub-step that would complete the
      // step records; if it fails its record is undone with the rest of its state
      ic.no_hist = ishk + 1 != jshk;
      enqueue_forces(c, false);
      enqueue_bonded(c);
      if (ic.ge_prescaled) launch_ge_scale(c->P, ic, c->st);
      launch_integrate(c->P, ic, c->nunit, c->fp64, c->cano_grid, c->st);
      unsigned st = 0;
      if (int e = read_status(c, &st)) return e;
      if (st & ERR_TIMEOUT) return check_status(c);
      int fr = 0;
      CK(cudaMemcpyAsync(&fr, c->P.rep_fail + r, sizeof(int), cudaMemcpyDeviceToHost, c->st));
      CK(cudaStreamSynchronize(c->st));
      if (int e = clear_after_failure(c)) return e;
      if (!fr)
        if (int e = snap_copy_rep(c, post, true, r)) return e;
      if (int e = snap_copy(c, post, false, row)) return e;
      if (fr) {
        if (T < 0.01 * dt) {
          CK(cudaMemcpyAsync(c->P.step_ctr, ctr_pre, sizeof(ctr_pre), cudaMemcpyHostToDevice, c->st));
          CK(cudaStreamSynchronize(c->st));
          return JP_E_SHAKE_ABORT;
        }
        jshk *= 2;
        ishk *= 2;
        T *= 0.5;
        continue;
      }
      ++ishk;
      if (ishk == jshk) break;
      if (ishk % 2 == 0) { jshk /= 2; ishk /= 2; T *= 2.0; }
    }
  }
  // the step is done: counters one step on
  const int ctr_post[2] = {ctr_pre[0] + 1, ctr_pre[1] + 1};
  CK(cudaMemcpyAsync(c->P.step_ctr, ctr_post, sizeof(ctr_post), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return JP_OK;
}

int validate(const jp_system *sys, int nrep, const jp_params *prm) {
  if (!sys || nrep <= 0 || !prm) return JP_E_INVALID;
  if (prm->cutoff <= 0.0 || prm->dt <= 0.0 || prm->dielectric <= 0.0) return JP_E_INVALID;
  if (prm->method < JP_METHOD_CONS || prm->method > JP_METHOD_GE) return JP_E_INVALID;
  if (prm->method == JP_METHOD_CONS && !(prm->taut > 0.0)) return JP_E_INVALID;
  if (prm->stop_center < 0 || prm->stop_center > JP_STOP_NONE || prm->stop_natom < 0) return JP_E_INVALID;
  if (prm->cal15m != JP_CAL15M_ZD && prm->cal15m != JP_CAL15M_ATOM && prm->cal15m != JP_CAL15M_CMM)
    return JP_E_INVALID;
  if (prm->cal15m == JP_CAL15M_CMM) {   // inpmd.f90:283-288, :525-528; CMM without clusters
    if (prm->bounda != JP_BOUND_NONE || prm->alsd != JP_ALSD_NONE) return JP_E_INVALID;
    if (!(prm->cmm_cell > 0.0) || prm->cmm_levels < 1 || prm->cmm_levels > 5 || prm->cmm_update < 1)
      return JP_E_INVALID;
    if (prm->update > 0 && prm->update % prm->cmm_update != 0) return JP_E_INVALID;
  }
  if (prm->bounda != JP_BOUND_PBC && prm->bounda != JP_BOUND_NONE) return JP_E_INVALID;
  if (prm->precision != JP_PREC_FP64 && prm->precision != JP_PREC_MIXED) return JP_E_INVALID;
  if (prm->alsd < JP_ALSD_NONE || prm->alsd > JP_GEPS_XOR) return JP_E_INVALID;
  const bool lmd = prm->alsd == JP_ALSD_LMD || prm->alsd == JP_ALSD_LMD2;
  const bool geps = prm->alsd >= JP_GEPS_AND;
  if (lmd) {   // verlethe only; lambda^(1/2) needs lambda > 0
    if (prm->method <= JP_METHOD_MICR || !std::isfinite(prm->lambda0)) return JP_E_INVALID;
    if (prm->alsd == JP_ALSD_LMD2 && !(prm->lambda0 > 0.0)) return JP_E_INVALID;
  }
  for (int r = 0; r < nrep && prm->alsd != JP_ALSD_NONE; ++r) {
    if (!sys[r].cluster) continue;
    bool any = false;
    for (int i = 0; i < sys[r].natom; ++i) {   // region codes: A 1, B 2 (partial McMD only)
      const int v = sys[r].cluster[i];
      if (v < 0 || v > (geps ? 2 : 1)) return JP_E_INVALID;
      any |= v != 0;
    }
    // partial McMD combines the classes only under the McMD weight or a pseudo temperature
    // (verlet.f90:118-142, verlethe.f90:170-238); md_run would integrate class 2 alone
    if (geps && any && prm->method != JP_METHOD_GE && !(prm->psetmp > 1.0e-10)) return JP_E_INVALID;
  }
  const double rlim = prm->cutoff + 1.5;
  for (int r = 0; r < nrep; ++r) {
    const jp_system &s = sys[r];
    if (s.natom <= 0 || !s.cord || !s.mass || !s.charge || !s.atype || !s.c6 || !s.c12 || !s.excl_ptr)
      return JP_E_INVALID;
    if (prm->bounda == JP_BOUND_PBC)
      for (int k = 0; k < 3; ++k)
        if (!(s.box[k] > 2.0 * rlim)) return JP_E_INVALID;   // unique minimum image
    if (s.ntype != sys[0].ntype) return JP_E_INVALID;
    if (prm->stop_natom > s.natom) return JP_E_INVALID;
    const size_t nt2 = (size_t)s.ntype * s.ntype;
    for (size_t q = 0; q < nt2; ++q)
      if (s.c6[q] != sys[0].c6[q] || s.c12[q] != sys[0].c12[q]) return JP_E_INVALID;
    // H-bond tables: 0/1 flags, symmetric, finite parameters, the same in every replica;
    // the 10-12 pairs belong to the cut-off variants (enear_ZD_*, enear_ACT_*) only
    if ((s.hbond == nullptr) != (sys[0].hbond == nullptr)) return JP_E_INVALID;
    if (s.hbond) {
      if (!s.c10 || !s.c12h) return JP_E_INVALID;
      const int nt = s.ntype;
      bool any = false;
      for (int i = 0; i < nt; ++i)
        for (int j = 0; j < nt; ++j) {
          const size_t q = (size_t)i * nt + j, qt = (size_t)j * nt + i;
          const int f = s.hbond[q];
          if ((f != 0 && f != 1) || f != s.hbond[qt] || f != sys[0].hbond[q]) return JP_E_INVALID;
          if (!f) continue;
          any = true;
          if (!std::isfinite(s.c10[q]) || !std::isfinite(s.c12h[q]) || s.c10[q] != s.c10[qt] ||
              s.c12h[q] != s.c12h[qt] || s.c10[q] != sys[0].c10[q] || s.c12h[q] != sys[0].c12h[q])
            return JP_E_INVALID;
        }
      if (any && prm->cal15m == JP_CAL15M_CMM) return JP_E_INVALID;
    }
    // CELRES residues: CMM only, atom ranges inside the system, no atom in two of them
    if (s.ncelres < 0 || (s.ncelres > 0 && (!s.celres || prm->cal15m != JP_CAL15M_CMM)))
      return JP_E_INVALID;
    if (s.ncelres > 0) {
      std::vector<char> seen(s.natom, 0);
      for (int i = 0; i < s.ncelres; ++i) {
        const int f = s.celres[2 * i] - s.index_base, l = s.celres[2 * i + 1] - s.index_base;
        if (f < 0 || l >= s.natom || f > l) return JP_E_INVALID;
        for (int a = f; a <= l; ++a) {
          if (seen[a]) return JP_E_INVALID;
          seen[a] = 1;
        }
      }
    }
    for (int i = 0; i < s.ntors; ++i) {
      int n = (int)std::lround(s.tors_nrot[i]);
      if (n < 1 || n > 6 || s.tors_div[i] == 0) return JP_E_INVALID;
    }
    for (int i = 0; i < s.nimpr; ++i) {
      int n = (int)std::lround(s.impr_nrot[i]);
      if (n < 1 || n > 6 || s.impr_div[i] == 0) return JP_E_INVALID;
    }
    for (int g = 0; g < s.nshake; ++g)
      if (s.shake_n[g] < 2 || s.shake_n[g] > 4) return JP_E_INVALID;
    if (prm->method == JP_METHOD_GE && !s.ge) return JP_E_INVALID;
    // every index that reaches a kernel must be in range
    const int b = s.index_base, n = s.natom;
    auto okatom = [&](int a) { return a - b >= 0 && a - b < n; };
    for (int i = 0; i < n; ++i) {
      if (s.atype[i] - b < 0 || s.atype[i] - b >= s.ntype) return JP_E_INVALID;
      if (s.molecule && s.molecule[i] - b < 0) return JP_E_INVALID;
      if (!(s.mass[i] > 0.0)) return JP_E_INVALID;
      if (s.excl_ptr[i + 1] < s.excl_ptr[i]) return JP_E_INVALID;
    }
    if (s.excl_ptr[0] != 0) return JP_E_INVALID;
    for (int p = 0; p < s.excl_ptr[n]; ++p)
      if (!okatom(s.excl_idx[p])) return JP_E_INVALID;
    for (int i = 0; i < 2 * s.nbond; ++i) if (!okatom(s.bond[i])) return JP_E_INVALID;
    for (int i = 0; i < 3 * s.nangle; ++i) if (!okatom(s.angle[i])) return JP_E_INVALID;
    for (int i = 0; i < 4 * s.ntors; ++i) if (!okatom(s.tors[i])) return JP_E_INVALID;
    for (int i = 0; i < 4 * s.nimpr; ++i) if (!okatom(s.impr[i])) return JP_E_INVALID;
    for (int g = 0; g < s.nshake; ++g)
      for (int k = 0; k < s.shake_n[g]; ++k)
        if (!okatom(s.shake_atoms[4 * g + k])) return JP_E_INVALID;
    if (s.restraints) {   // every array present for its count, indices in range, finite values
      const jp_restraints &q = *s.restraints;
      auto fin = [](double v) { return std::isfinite(v); };
      if (q.npos < 0 || q.ndist < 0 || q.ndihe < 0 || q.ncap_group < 0 || q.ncap_atom < 0)
        return JP_E_INVALID;
      if (q.npos && (!q.pos_atom || !q.pos_k || !q.pos_ref)) return JP_E_INVALID;
      for (int i = 0; i < q.npos; ++i)
        if (!okatom(q.pos_atom[i]) || !fin(q.pos_k[i]) || !fin(q.pos_ref[3 * i]) ||
            !fin(q.pos_ref[3 * i + 1]) || !fin(q.pos_ref[3 * i + 2]))
          return JP_E_INVALID;
      if (q.ndist && (!q.dist_iptr || !q.dist_iatom || !q.dist_jptr || !q.dist_jatom || !q.dist_lo ||
                      !q.dist_up || !q.dist_klo || !q.dist_kup || q.dist_iptr[0] != 0 || q.dist_jptr[0] != 0))
        return JP_E_INVALID;
      for (int i = 0; i < q.ndist; ++i) {
        // non-empty groups without a common atom (r = 0 would make <r^-6> infinite)
        if (q.dist_iptr[i + 1] <= q.dist_iptr[i] || q.dist_jptr[i + 1] <= q.dist_jptr[i]) return JP_E_INVALID;
        if (!fin(q.dist_lo[i]) || !fin(q.dist_up[i]) || !(q.dist_lo[i] <= q.dist_up[i]) ||
            !fin(q.dist_klo[i]) || !fin(q.dist_kup[i]))
          return JP_E_INVALID;
        for (int p = q.dist_iptr[i]; p < q.dist_iptr[i + 1]; ++p) {
          if (!okatom(q.dist_iatom[p])) return JP_E_INVALID;
          for (int u = q.dist_jptr[i]; u < q.dist_jptr[i + 1]; ++u)
            if (!okatom(q.dist_jatom[u]) || q.dist_jatom[u] == q.dist_iatom[p]) return JP_E_INVALID;
        }
      }
      if (q.ndihe && (!q.dihe_atom || !q.dihe_lo || !q.dihe_up || !q.dihe_klo || !q.dihe_kup))
        return JP_E_INVALID;
      for (int i = 0; i < q.ndihe; ++i) {
        for (int k = 0; k < 4; ++k) if (!okatom(q.dihe_atom[4 * i + k])) return JP_E_INVALID;
        if (!fin(q.dihe_lo[i]) || !fin(q.dihe_up[i]) || !(q.dihe_lo[i] <= q.dihe_up[i]) ||
            !fin(q.dihe_klo[i]) || !fin(q.dihe_kup[i]))
          return JP_E_INVALID;
      }
      if (q.ncap_group || q.ncap_atom) {   // dnecap is called from dneres_CB only
        if (prm->bounda != JP_BOUND_NONE) return JP_E_INVALID;
        if (!fin(q.cap_center[0]) || !fin(q.cap_center[1]) || !fin(q.cap_center[2]) ||
            !(q.cap_radius >= 0.0) || !(q.cap_atom_radius >= 0.0) || !fin(q.cap_radius) ||
            !fin(q.cap_atom_radius) || !fin(q.cap_k) || !fin(q.cap_atom_k))
          return JP_E_INVALID;
        if ((q.ncap_group && !q.cap_group) || (q.ncap_atom && !q.cap_atom)) return JP_E_INVALID;
        if (q.cap_shape < 0 || q.cap_shape > JP_CAP_ELLIPSOID) return JP_E_INVALID;
        if (q.cap_function < 0 || q.cap_function > JP_CAP_BIQUADRATIC) return JP_E_INVALID;
        if (q.cap_function == JP_CAP_BIQUADRATIC && q.cap_shape > JP_CAP_SPHERE) return JP_E_INVALID;
        if (q.cap_function == JP_CAP_BIQUADRATIC && (!(q.cap_radius > 0.0) || !(q.cap_atom_radius > 0.0)))
          return JP_E_INVALID;
        for (int k = 0; k < 6 && q.cap_shape == JP_CAP_BOX; k += 2)
          if (!fin(q.cap_wall[k]) || !fin(q.cap_wall[k + 1]) || !(q.cap_wall[k] <= q.cap_wall[k + 1]) ||
              !fin(q.cap_atom_wall[k]) || !fin(q.cap_atom_wall[k + 1]) ||
              !(q.cap_atom_wall[k] <= q.cap_atom_wall[k + 1]))
            return JP_E_INVALID;
        for (int k = 0; k < 3 && q.cap_shape == JP_CAP_ELLIPSOID; ++k)
          if (!(q.cap_ellipse[k] > 0.0) || !(q.cap_atom_ellipse[k] > 0.0) || !fin(q.cap_ellipse[k]) ||
              !fin(q.cap_atom_ellipse[k]))
            return JP_E_INVALID;
        for (int i = 0; i < q.ncap_group; ++i)
          if (!okatom(q.cap_group[2 * i]) || !okatom(q.cap_group[2 * i + 1]) ||
              q.cap_group[2 * i] > q.cap_group[2 * i + 1])
            return JP_E_INVALID;
        for (int i = 0; i < q.ncap_atom; ++i) if (!okatom(q.cap_atom[i])) return JP_E_INVALID;
      }
    }
    if (s.ge && (s.ge->nwindow < 1 || s.ge->ndeg < 0 || s.ge->nwindow > JP_GE_MAX_WINDOWS ||
                 s.ge->ndeg > JP_GE_MAX_DEG || !s.ge->coef || !s.ge->low || !s.ge->high))
      return JP_E_INVALID;
  }
  return 0;
}

}  // namespace

// =======================================================================================
namespace {

// conj (conj.f90) for one replica on the host over device force evaluations: the search
// direction (mksrdc with mksdc1 / mksdc2 / mksrdg, chksrd) and the line search (linsrc).
// Returns a JP code; fills iters / eneval / rmsf / state like the steepest-descent path.
int minimize_conj(jp_ctx *c, int r, const jp_min_params *mp, int32_t *iters, double *eneval,
                  double *rmsf_out, int32_t *state) {
  const Rep &R = c->reps[r];
  const int n = R.natom, m = 3 * n;
  std::vector<double> x(m), g(m), grado(m, 0.0), difgrd(m, 0.0), d(m, 0.0), dold(m, 0.0),
      drst(m, 0.0), trycor(m);
  double e[JP_MAXENE];
  int rc = jp_get_state(c, r, x.data(), nullptr);
  if (rc != JP_OK) return rc;
  auto dot = [m](const std::vector<double> &a, const std::vector<double> &b) {
    double t = 0.0;
    for (int k = 0; k < m; ++k) t += a[k] * b[k];
    return t;
  };
  auto unit = [&](std::vector<double> &v) {
    const double f = 1.0 / std::sqrt(dot(v, v));
    for (double &w : v) w *= f;
  };
  rc = jp_energy_grad(c, r, x.data(), e, g.data());
  if (rc != JP_OK) return rc;
  double stp = mp->step0 * std::sqrt((double)n), dtdifg = 0.0;
  double rms = std::sqrt(dot(g, g) / n);
  int mode = 1, nsrch = 0, nrst = 0, it = 0, st = 0;
  bool done = false;
  while (!done) {
    // search direction: 1 steepest descent, 3 start a restart cycle, 2 continue it
    double gd;
    for (;;) {
      if (mode == 2 && std::fabs(dot(grado, g)) / dot(g, g) >= 0.2) mode = 3;
      if (mode == 1) {
        const double f = -1.0 / std::sqrt(dot(g, g));
        for (int k = 0; k < m; ++k) d[k] = f * g[k];
        dold = d;
      } else if (mode == 2) {
        dold = d;
        double beta = 0.0, den = 0.0, gam = 0.0;
        for (int k = 0; k < m; ++k) {
          const double dg = g[k] - grado[k];
          beta += g[k] * dg;
          den += dold[k] * dg;
          gam += g[k] * difgrd[k];
        }
        if (den != 0.0) {
          beta /= den;
          gam /= dtdifg;
          for (int k = 0; k < m; ++k) d[k] = beta * dold[k] + gam * drst[k] - g[k];
          unit(d);
        }
      } else {
        dold = d;
        drst = d;
        double beta = 0.0, den = 0.0;
        for (int k = 0; k < m; ++k) {
          difgrd[k] = g[k] - grado[k];
          beta += g[k] * difgrd[k];
          den += dold[k] * difgrd[k];
        }
        dtdifg = den;
        if (den != 0.0) {
          beta /= den;
          for (int k = 0; k < m; ++k) d[k] = beta * dold[k] - g[k];
          unit(d);
        }
        nrst = nsrch;
      }
      gd = dot(g, d);
      if (gd < 0.0) break;   // downhill: keep it
      mode = 1;
    }
    ++nsrch;
    if (mode == 1) mode = 3;
    else if (mode == 3) mode = 2;
    if (nsrch - nrst == 3 * n) mode = 3;
    grado = g;
    // line search along d from trycor
    const double gd0 = gd;
    bool bracket = false;
    int j = 0;
    double s_lo = 0.0, s_hi = 0.0, gd_lo = gd0, gd_hi = 0.0;
    trycor = x;
    for (;;) {
      if (it != 0 && mp->update > 0 && it % mp->update == 0) {
        rc = jp_rebuild_cells(c, r);
        if (rc != JP_OK) return rc;
      }
      for (int k = 0; k < m; ++k) x[k] = trycor[k] + stp * d[k];
      ++it;
      ++j;
      rc = jp_energy_grad(c, r, x.data(), e, g.data());
      if (rc != JP_OK) return rc;
      const double gdn = dot(g, d);
      rms = std::sqrt(dot(g, g) / n);
      if (rms <= mp->convgr) { st = 1; done = true; break; }
      if (it >= mp->max_loop) { done = true; break; }
      if (j == mp->line_max) break;
      if (std::fabs(gdn / gd0) <= mp->line_conv) break;
      if (!bracket && gdn < 0.0) {   // still downhill: double the step
        s_lo = stp;
        gd_lo = gdn;
        stp = 2.0 * s_lo;
        continue;
      }
      if (gdn < 0.0) { s_lo = stp; gd_lo = gdn; }
      else { s_hi = stp; gd_hi = gdn; }
      bracket = true;
      stp = s_lo - (s_hi - s_lo) / (gd_hi - gd_lo) * gd_lo;   // secant on g.d
    }
  }
  if (iters) iters[r] = it;
  if (rmsf_out) rmsf_out[r] = rms;
  if (state) state[r] = st;
  if (eneval) std::memcpy(eneval + (size_t)r * JP_MAXENE, e, sizeof(e));
  return JP_OK;
}

int flush_rebuild(jp_ctx *c);   // below, beside the step loop

// Block-shape tuning (the role of md_run's SIMD_check.f90:1-42 for its vector length): the
// pair kernels' work is proportional to the compact tiles of the list, so each replica's
// list is built with every candidate column grid and the grid needing the fewest compact
// tiles is kept (ties to the unit factor, then to the smaller factor).  The count is exact
// and deterministic, so the choice does not depend on timing noise, and a replica's choice
// depends on its own atoms only (batched with others it chooses as it would alone).
// Without tuning every replica keeps the unit factor.  Ends with the list built for the
// chosen shapes.
int tune_blocks(jp_ctx *c, bool tune) {
  const int nq = JP_TUNE_CANDIDATES;
  c->tune_tiles.assign((size_t)c->nrep * nq, -1);
  c->tune_pick.assign(c->nrep, kTuneDefault);
  std::vector<int> cnt(2 * (size_t)c->nblk);   // pair records per unit (two per block)
  for (int q = 0; q < (tune ? nq : 0); ++q) {
    for (int r = 0; r < c->nrep; ++r) set_grid(c->reps[r], c->tune_grid.data() + ((size_t)r * nq + q) * 2);
    CK(cudaMemcpy(c->P.reps, c->reps.data(), sizeof(Rep) * c->nrep, cudaMemcpyHostToDevice));
    enqueue_rebuild(c);
    CK(cudaMemcpyAsync(cnt.data(), c->P.ct_cnt, sizeof(int) * 2 * c->nblk, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    int rs = check_status(c);
    if (rs < 0) return rs;
    for (int r = 0; r < c->nrep; ++r) {
      long long t = 0;
      for (int b = c->reps[r].blk0; b < c->reps[r].blk0 + c->reps[r].nblk; ++b) t += cnt[2 * b] + cnt[2 * b + 1];
      c->tune_tiles[(size_t)r * nq + q] = t;
    }
  }
  for (int r = 0; r < c->nrep && tune; ++r) {
    const long long *t = &c->tune_tiles[(size_t)r * nq];
    int best = kTuneDefault;
    for (int q = 0; q < nq; ++q)
      if (t[q] < t[best]) best = q;
    c->tune_pick[r] = best;
  }
  for (int r = 0; r < c->nrep; ++r)
    set_grid(c->reps[r], c->tune_grid.data() + ((size_t)r * nq + c->tune_pick[r]) * 2);
  CK(cudaMemcpy(c->P.reps, c->reps.data(), sizeof(Rep) * c->nrep, cudaMemcpyHostToDevice));
  enqueue_rebuild(c);
  CK(cudaStreamSynchronize(c->st));
  return check_status(c);
}

}  // namespace

extern "C" {

void jp_default_params(jp_params *p) {
  std::memset(p, 0, sizeof(*p));
  p->precision = JP_PREC_MIXED;
  p->method = JP_METHOD_CANO;      // inpmd.f90:126 intele(9)=3
  p->dt = 2.0;                     // inpmd.f90:127
  p->cutoff = 12.0;                // main.f90:155 fycutl
  p->dielectric = 1.0;             // main.f90:155 fydiel
  p->update = 10;                  // inpmd.f90:126 intele(4)
  p->temp = 300.0;
  p->temp_start = 300.0;
  p->heat_loop = 0;
  p->tempco = 2;                   // inpmd.f90:148 intele(63)=2
  p->shake_method = JP_SHAKE_HBON;
  p->shake_tol = 1.0e-6;           // main.f90:167 fustol
  p->shake_maxit = 1000;           // main.f90:166 iuslop
  p->icslop = 3;                   // main.f90:166
  p->fcstol = 1.0e-3;              // main.f90:167
  p->psetmp = 0.0;
  p->device = 0;
  p->alsd = JP_ALSD_NONE;
  p->lambda0 = 1.0;
  p->lambda_mass = 0.0;
  p->lambda_temp_control = 0;
  p->scale_terms = 0;
  p->taut = 40.0;                  // inpmd.f90:125 reaele(11)
  p->stop_center = JP_STOP_NONE;   // inpmd.f90:124 intele(8)=4
  p->stop_natom = 0;
  p->cal15m = JP_CAL15M_ZD;
  p->bounda = JP_BOUND_PBC;
  p->cmm_levels = 3;               // inpinp.f90:86 intele(16)
  p->cmm_cell = 6.0;               // inpinp.f90:86 reaele(17)
  p->cmm_update = 5;
  p->tune_blocks = 1;               // inpmd.f90:151 intele(66)
}

const char *jp_strerror(int code) {
  switch (code) {
    case JP_OK: return "ok";
    case JP_W_SHAKE_NOT_CONVERGED: return "SHAKE not converged (warning)";
    case JP_E_SHAKE_SINGULAR: return "SHAKE gradient matrix singular";
    case JP_E_SHAKE_ABORT: return "SHAKE failed after time-step halving";
    case JP_E_INVALID: return "invalid argument or topology";
    case JP_E_CELL_OVERFLOW: return "cell table overflow";
    case JP_E_LIST_OVERFLOW: return "pair-tile list overflow";
    case JP_E_NONFINITE: return "non-finite coordinate or force";
    case JP_E_FIXED_OVERFLOW: return "fixed-point force overflow";
    case JP_E_CUDA: return g_last_err;
    case JP_E_NO_DEVICE: return "no CUDA device";
    case JP_E_TIMEOUT: return "device wait timed out";
    case JP_E_NOALLOC_LIMIT: return "natom above JP_NOALLOC_MAX_ATOMS, the static scratch size";
    case JP_E_FREE_WINDOW: return "BOUNDA= NO: an atom left the window of the context (re-create it)";
    case JP_E_STOP_MASS: return "centre-of-mass stop: the stopped atoms have no mass";
    case JP_E_STOP_SINGULAR: return "centre-of-mass stop: inertia tensor of the stopped atoms is singular";
    case JP_E_MIN_STEP: return "minimisation: the step length fell below 1e-10 A per degree of freedom";
    default: return "unknown error";
  }
}

int jp_create(const jp_system *sys, int32_t nrep, const jp_params *prm, jp_ctx **out) {
  if (!out) return JP_E_INVALID;
  *out = nullptr;
  int v = validate(sys, nrep, prm);
  if (v) return v;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return JP_E_NO_DEVICE;
  if (prm->device < 0 || prm->device >= ndev) return JP_E_INVALID;
  CK(cudaSetDevice(prm->device));

  jp_ctx *c = new (std::nothrow) jp_ctx();
  if (!c) return JP_E_INVALID;
  c->nrep = nrep;
  c->prm = *prm;
  c->device = prm->device;
  c->fp64 = prm->precision == JP_PREC_FP64;
  const double ccoef = kEekcal / prm->dielectric;
  c->qscale = std::sqrt(ccoef);
  const double rc = prm->cutoff;
  const double rlim = rc + 1.5;

  // ---- host-side topology derivation -----------------------------------------------
  std::vector<double> hx, hv, hmass, himass, hchg;
  std::vector<int> htyp, hrep, hexp{0}, hexi;
  std::vector<Unit> units;
  std::vector<Term> terms_by_kind[6];
  std::vector<double> hnfr, hge, hlam;
  std::vector<Rep> reps(nrep);
  const int ntype = sys[0].ntype;
  const int nt1 = ntype + 1;
  std::vector<float2> ljf(nt1 * nt1, make_float2(0.f, 0.f));
  std::vector<double2> ljd(nt1 * nt1, make_double2(0.0, 0.0));
  // H-bond type pairs: (C10, C12h) and their flags; the pair kernels' 12-6 table is zero
  // there (those pairs keep only their Coulomb term in the tiles), the 1-4 table is not
  std::vector<double2> hbt(nt1 * nt1, make_double2(0.0, 0.0));
  std::vector<int> hbp(nt1 * nt1, 0), hbty(nt1, 0);
  for (int i = 0; i < ntype; ++i)
    for (int j = 0; j < ntype; ++j) {
      const int q = i * ntype + j;
      ljd[i * nt1 + j] = make_double2(sys[0].c6[q], sys[0].c12[q]);
      ljf[i * nt1 + j] = make_float2((float)sys[0].c6[q], (float)sys[0].c12[q]);
      if (sys[0].hbond && sys[0].hbond[q]) {
        hbt[i * nt1 + j] = make_double2(sys[0].c10[q], sys[0].c12h[q]);
        hbp[i * nt1 + j] = 1;
        hbty[i] = 1;
      }
    }
  const std::vector<double2> lj14 = ljd;
  for (int q = 0; q < nt1 * nt1; ++q)
    if (hbp[q]) {
      ljd[q] = make_double2(0.0, 0.0);
      ljf[q] = make_float2(0.f, 0.f);
    }
  c->hbond = std::find(hbp.begin(), hbp.end(), 1) != hbp.end();
  int atom0 = 0, blk0 = 0, key0 = 0, sub0 = 0, col0 = 0;
  std::vector<Restr> hres;          // restraints and CAP terms of all replicas
  std::vector<int2> hres_cmm;       // CELRES: each atom's residue range (empty: no CELRES)
  double celres_rmax = 0.0;         // largest distance of a CELRES atom from its residue centre
  int N_all = 0;
  for (int r = 0; r < nrep; ++r) N_all += sys[r].natom;
  std::vector<int> hres_idx;        // atoms of the distance-restraint groups
  std::vector<int> hcol_rep;
  for (int r = 0; r < nrep; ++r) {
    const jp_system &s = sys[r];
    const int b = s.index_base;
    const int n = s.natom;
    Rep &R = reps[r];
    std::memset(&R, 0, sizeof(Rep));
    R.atom0 = atom0;
    R.natom = n;
    R.blk0 = blk0;
    // BOUNDA= NO: a periodic box in which no two atoms of the replica can be half a box
    // apart, so that minimum image is the identity and the periodic cell list, tiles and
    // kernels give exactly the free-boundary pair set (the *_CB variants).  The atoms must
    // stay in a window around their initial bounding box (checked at each list rebuild).
    double box[3], vol = 1.0;
    R.free_bnd = prm->bounda == JP_BOUND_NONE ? 1 : 0;
    for (int k = 0; k < 3; ++k) {
      box[k] = s.box[k];
      if (R.free_bnd) {
        double lo = s.cord[k], hi = s.cord[k];
        for (int i = 1; i < n; ++i) {
          lo = std::min(lo, s.cord[3 * i + k]);
          hi = std::max(hi, s.cord[3 * i + k]);
        }
        const double half = 0.5 * (hi - lo) + 10.0 + 0.1 * (hi - lo);
        R.win_lo[k] = 0.5 * (lo + hi) - half;
        R.win_hi[k] = 0.5 * (lo + hi) + half;
        box[k] = std::max(4.0 * half + 2.0, 2.0 * rlim + 2.0);   // separations < 2 half < box / 2
        vol *= std::max(hi - lo, 10.0);
      } else {
        vol *= box[k];
      }
    }
    // CMM cell levels (incel.f90:29-57): nlev raised until 2^(nlev+1) CELSIZ covers the
    // largest extent; nv = 4 * 2^(nlev-l) cells of edge CELSIZ * 2^(l-1) per level
    R.cmm = prm->cal15m == JP_CAL15M_CMM ? 1 : 0;
    if (R.cmm) {
      double ext = 0.0;
      for (int k = 0; k < 3; ++k) {
        double lo = s.cord[k], hi = s.cord[k];
        for (int i = 1; i < n; ++i) {
          lo = std::min(lo, s.cord[3 * i + k]);
          hi = std::max(hi, s.cord[3 * i + k]);
        }
        ext = std::max(ext, hi - lo);
      }
      int nlev = prm->cmm_levels;
      if (std::ldexp(1.0, nlev + 1) * prm->cmm_cell < ext)
        nlev = (int)std::ceil(std::log(ext / prm->cmm_cell) / std::log(2.0) - 1.0);
      if (nlev > 5) { delete c; return JP_E_INVALID; }
      R.nlev = nlev;
      for (int l = 1; l <= nlev; ++l) {
        R.nv[l] = 4 << (nlev - l);
        R.siz[l] = prm->cmm_cell * (double)(1 << (l - 1));
      }
      R.idelay = (int)std::ceil(rc / R.siz[1]);
      R.cmm_upd = prm->cmm_update;
      if (s.ext_cmm) {   // setextCMM.f90:17-33: 4 levels, the same grid as the file's
        const jp_ext_cmm &x = *s.ext_cmm;
        if (x.nlev != 4 || nlev != 4 || !x.flag || !x.pot ||
            !(std::fabs(x.cell - prm->cmm_cell) <= 1e-9 * prm->cmm_cell)) { delete c; return JP_E_INVALID; }
        R.ext = 1;
        for (int k = 0; k < 3; ++k) R.ext_c0[k] = x.center[k];
      }
    } else if (s.ext_cmm) {
      delete c;
      return JP_E_INVALID;   // an external environment belongs to a CMM run
    }
    // xy columns of edge ~(32/density)^(1/3) so that 32 z-sorted atoms fill a near-cubic
    // block; 0.25 A z bins inside a column
    const double dens = n / vol;
    const double edge = std::cbrt((double)kTile / dens);
    for (int k = 0; k < 3; ++k) {
      R.box[k] = box[k];
      R.invbox[k] = 1.0 / box[k];
    }
    // the block-shape candidates: column edges scaled by kTuneScale; the columns, sort keys
    // and blocks are laid out for the candidate with the most columns, so any of them can
    // be taken later without reallocating
    int ncol_cap = 0;
    for (int q = 0; q < JP_TUNE_CANDIDATES; ++q) {
      int g[2];
      for (int k = 0; k < 2; ++k)
        g[k] = std::max(1, std::min(512, (int)std::lround(box[k] / (edge * kTuneScale[q]))));
      c->tune_grid.push_back(g[0]);
      c->tune_grid.push_back(g[1]);
      ncol_cap = std::max(ncol_cap, g[0] * g[1]);
    }
    set_grid(R, c->tune_grid.data() + ((size_t)r * JP_TUNE_CANDIDATES + kTuneDefault) * 2);
    R.grid[2] = std::max(1, (int)std::ceil(box[2] / 0.25));
    R.cell[2] = box[2] / R.grid[2];
    R.col0 = col0;
    R.ncol = ncol_cap;
    col0 += R.ncol;
    for (int q = 0; q < R.ncol; ++q) hcol_rep.push_back(r);
    R.key0 = key0;
    key0 += R.ncol * R.grid[2];
    // block capacity: every column wastes less than one block
    R.nblk = (n + kTile - 1) / kTile + R.ncol;
    // ALSD cluster (inpcls.f90 icls): the atom's class bit rides in bit 30 of its LJ type
    const bool ralsd = (prm->alsd == JP_ALSD_LMD || prm->alsd == JP_ALSD_LMD2) && s.cluster;
    std::vector<int> inA(n, 0);
    if (ralsd)
      for (int i = 0; i < n; ++i) inA[i] = s.cluster[i] ? 1 : 0;
    // partial McMD (GEPSME= AND / OR / XOR): region codes A 0, B 1, neither 2 in bits 28-29
    // of the LJ type, and the replica's class-1 table (n_matrix = 1, inpcls.f90:298-325); a
    // replica without cluster atoms (nfrag = 1) keeps one class and plain McMD
    std::vector<int> icl(n, 2);
    bool rsplit = false;
    unsigned tab1 = 0;
    if (prm->alsd >= JP_GEPS_AND && s.cluster) {
      bool hasA = false, hasB = false;
      for (int i = 0; i < n; ++i) {
        if (s.cluster[i] == 1) { icl[i] = 0; hasA = true; }
        else if (s.cluster[i] == 2) { icl[i] = 1; hasB = true; }
      }
      rsplit = hasA || hasB;
      auto bit = [](int a, int c2) { return (1u << (3 * a + c2)) | (1u << (3 * c2 + a)); };
      if (!hasB) {   // nfrag = 2: region A and the rest
        tab1 = prm->alsd == JP_GEPS_AND ? bit(0, 0) : prm->alsd == JP_GEPS_OR ? bit(0, 0) | bit(0, 2) : bit(0, 2);
      } else {       // nfrag = 3: A, B and the rest
        tab1 = prm->alsd == JP_GEPS_AND ? bit(0, 0) | bit(1, 1) : prm->alsd == JP_GEPS_OR ? bit(0, 0) | bit(0, 1)
                                                                                     : bit(0, 1);
      }
    }
    R.split = rsplit ? 1 : 0;
    R.cls_tab = tab1;
    R.cls_over = 0;
    auto pcls = [&](int a1, int a2) {
      if (rsplit) return ((tab1 >> (3 * icl[a1] + icl[a2])) & 1u) ? 0 : 2;
      return ralsd ? 2 - inA[a1] - inA[a2] : 2;
    };
    for (int i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) {
        hx.push_back(s.cord[3 * i + k]);
        hv.push_back(s.vel ? s.vel[3 * i + k] : 0.0);
      }
      hmass.push_back(s.mass[i]);
      himass.push_back(1.0 / s.mass[i]);
      hchg.push_back(s.charge[i]);
      htyp.push_back((s.atype[i] - b) | (inA[i] << 30) | (rsplit ? icl[i] << kRegionShift : 0));
      hrep.push_back(r);
    }
    // exclusions
    for (int i = 0; i < n; ++i) {
      std::vector<int> L;
      for (int p = s.excl_ptr[i]; p < s.excl_ptr[i + 1]; ++p) L.push_back(atom0 + s.excl_idx[p] - b);
      std::sort(L.begin(), L.end());
      for (int q : L) hexi.push_back(q);
      hexp.push_back((int)hexi.size());
    }
    // sub-systems
    // sub-systems: molecule-entry ids renumbered densely, empty ids removed (md.f90:133-151)
    std::vector<int> mol(n, 0);
    int nmol = 1;
    if (s.molecule && prm->tempco == 2) {
      // with clusters each molecule splits into its cluster and non-cluster part (md.f90
      // ixamol2 = (ixamol - 1) * nfrag + icls, renumbered densely)
      auto key = [&](int i) {
        return ralsd ? 2 * (s.molecule[i] - b) + (inA[i] ? 0 : 1) : rsplit ? 3 * (s.molecule[i] - b) + icl[i]
                                                                          : s.molecule[i] - b;
      };
      std::vector<int> u;
      for (int i = 0; i < n; ++i) u.push_back(key(i));
      std::sort(u.begin(), u.end());
      u.erase(std::unique(u.begin(), u.end()), u.end());
      for (int i = 0; i < n; ++i) mol[i] = (int)(std::lower_bound(u.begin(), u.end(), key(i)) - u.begin());
      nmol = (int)u.size();
    }
    R.sub0 = sub0;
    R.nsub = nmol;
    std::vector<double> nfr(nmol, 0.0);
    for (int i = 0; i < n; ++i) nfr[mol[i]] += 3.0;
    // SHAKE groups -> units
    const bool shk = prm->shake_method != JP_SHAKE_NONE && s.nshake > 0;
    std::set<std::pair<int, int>> cpairs;
    std::vector<char> in_group(n, 0);
    std::vector<Unit> ru;
    static const int pl[6][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 0}, {2, 3}, {1, 3}};
    if (shk) {
      for (int ng = 2; ng <= 4; ++ng)   // md_run order: 2-, 3-, then 4-atom groups
        for (int g = 0; g < s.nshake; ++g) {
          if (s.shake_n[g] != ng) continue;
          Unit u;
          std::memset(&u, 0, sizeof(u));
          u.n = ng;
          u.rep = r;
          for (int k = 0; k < 4; ++k) u.a[k] = k < ng ? atom0 + s.shake_atoms[4 * g + k] - b : -1;
          const int nc = ng * (ng - 1) / 2;
          for (int q = 0; q < 6; ++q) {
            const double d = q < nc ? s.shake_dist[6 * g + q] : 0.0;
            u.d2[q] = d * d;
          }
          for (int q = 0; q < nc; ++q) {
            int a1 = u.a[pl[q][0]] - atom0, a2 = u.a[pl[q][1]] - atom0;
            cpairs.insert({std::min(a1, a2), std::max(a1, a2)});
          }
          for (int k = 0; k < ng; ++k) {
            if (in_group[u.a[k] - atom0]) { delete c; return JP_E_INVALID; }
            in_group[u.a[k] - atom0] = 1;
          }
          u.sub = sub0 + mol[u.a[0] - atom0];
          // a group's atoms share one temperature (they do when sub-systems follow
          // molecules and residues); a group split across sub-systems is rejected
          for (int k = 1; k < ng; ++k)
            if (mol[u.a[k] - atom0] != mol[u.a[0] - atom0]) { delete c; return JP_E_INVALID; }
          nfr[mol[u.a[0] - atom0]] -= (double)nc;
          ru.push_back(u);
        }
    }
    for (int i = 0; i < n; ++i)
      if (!in_group[i]) {
        Unit u;
        std::memset(&u, 0, sizeof(u));
        u.n = 1;
        u.rep = r;
        u.a[0] = atom0 + i;
        u.a[1] = u.a[2] = u.a[3] = -1;
        u.sub = sub0 + mol[i];
        ru.push_back(u);
      }
    // centre-of-mass stop (md.f90:116-121, :186-216): 3 (translation or rotation) or 6 fewer
    // degrees of freedom, taken from the sub-systems of the first molecule in proportion to
    // their DOF; the stopped atoms are the first stop_natom (ixcend(nstpcn))
    R.stop_n = 0;
    if (prm->stop_center >= JP_STOP_TRANS && prm->stop_center <= JP_STOP_BOTH) {
      int lead = n;   // leading atoms with atom 1's molecule id
      if (s.molecule) {
        lead = 1;
        while (lead < n && s.molecule[lead] == s.molecule[0]) ++lead;
      }
      R.stop_n = prm->stop_natom > 0 ? prm->stop_natom : lead;
      const double drop = prm->stop_center == JP_STOP_BOTH ? 6.0 : 3.0;
      int ifrg = 0;
      for (int i = 0; i < lead; ++i) ifrg = std::max(ifrg, mol[i] + 1);
      if (ifrg >= 2) {
        double sum = 0.0;
        for (int q = 0; q < ifrg; ++q) sum += nfr[q];
        std::vector<double> ratio(ifrg);
        for (int q = 0; q < ifrg; ++q) ratio[q] = nfr[q] / sum;
        for (int q = 0; q < ifrg; ++q) nfr[q] -= drop * ratio[q];
      } else {
        nfr[0] -= drop;
      }
    }
    std::stable_sort(ru.begin(), ru.end(), [](const Unit &x, const Unit &y) {
      return x.sub != y.sub ? x.sub < y.sub : x.n < y.n;   // warps uniform in sub-system and group size
    });
    R.unit0 = (int)units.size();
    R.nunit = (int)ru.size();
    units.insert(units.end(), ru.begin(), ru.end());
    // ALSD lambda: mass (inpcls.f90:350-360), its degree of freedom (md.f90:122-123,
    // :220-228) and the sub-system whose temperature holds its kinetic term (caltmp/caltmp2)
    R.lam_mode = ralsd ? prm->alsd : JP_ALSD_NONE;
    R.lam_ke_sub = -1;
    if (ralsd) {
      R.lam_m = prm->lambda_mass;
      if (!(R.lam_m > 0.0)) {
        R.lam_m = 0.0;
        for (int i = 0; i < n; ++i) if (inA[i]) R.lam_m += s.mass[i];
      }
      R.lam_im = R.lam_m > 0.0 ? 1.0 / R.lam_m : 0.0;
      R.lam_tc = prm->lambda_temp_control ? 1 : 0;
      const bool dof = R.lam_tc && prm->method == JP_METHOD_GE;
      if (prm->tempco == 1) {
        R.lam_ke_sub = R.sub0;
        if (dof) nfr[0] += 1.0;
      } else if (dof) {
        int best = 0;
        for (int q = 1; q < nmol; ++q) if (nfr[q] > nfr[best]) best = q;
        nfr[best] += 1.0;
        R.lam_ke_sub = R.sub0 + best;
      }
    }
    hlam.push_back(prm->lambda0);
    hlam.push_back(0.0);
    for (double f : nfr) hnfr.push_back(f);
    sub0 += nmol;
    auto constrained = [&](int a1, int a2) {
      return shk && cpairs.count({std::min(a1, a2), std::max(a1, a2)}) > 0;
    };
    // bonded terms
    std::vector<double> dwork(s.charge, s.charge + n);
    std::vector<double> dwk((size_t)3 * n, 0.0);   // the same by class (incel.f90:629-654)
    for (int i = 0; i < n; ++i) dwk[(size_t)pcls(i, i) * n + i] += s.charge[i];
    const int sct = prm->scale_terms;
    auto mkterm = [&](int kind) {
      Term t;
      std::memset(&t, 0, sizeof(t));
      t.kind = kind;
      t.rep = r;
      t.idiv = 1;
      t.cls = 2;
      return t;
    };
    const bool zd = prm->cal15m == JP_CAL15M_ZD;   // ATOM: no self or excess term
    auto excess = [&](int a1, int a2) {   // incel.f90:635-654, :665-688
      if (!zd) return;
      dwork[a1] += s.charge[a2];
      dwork[a2] += s.charge[a1];
      const int cl = pcls(a1, a2);
      dwk[(size_t)cl * n + a1] += s.charge[a2];
      dwk[(size_t)cl * n + a2] += s.charge[a1];
      Term t = mkterm(T_EXCESS);
      t.a[0] = atom0 + a1;
      t.a[1] = atom0 + a2;
      t.p0 = ccoef * s.charge[a1] * s.charge[a2];
      t.cls = cl;
      terms_by_kind[T_EXCESS].push_back(t);
    };
    for (int i = 0; i < s.nbond; ++i) {
      int a1 = s.bond[2 * i] - b, a2 = s.bond[2 * i + 1] - b;
      excess(a1, a2);
      if (constrained(a1, a2)) continue;
      Term t = mkterm(T_BOND);
      t.a[0] = atom0 + a1;
      t.a[1] = atom0 + a2;
      t.p0 = s.bond_k[i];
      t.p1 = s.bond_r0[i];
      if (sct & JP_SCALE_BOND) t.cls = pcls(a1, a2);   // incel.f90:705-712
      terms_by_kind[T_BOND].push_back(t);
    }
    for (int i = 0; i < s.nangle; ++i) {
      int a1 = s.angle[3 * i] - b, a2 = s.angle[3 * i + 1] - b, a3 = s.angle[3 * i + 2] - b;
      excess(a1, a3);
      if (constrained(a1, a3)) continue;
      Term t = mkterm(T_ANGLE);
      t.a[0] = atom0 + a1;
      t.a[1] = atom0 + a2;
      t.a[2] = atom0 + a3;
      t.p0 = s.angle_k[i];
      t.p1 = s.angle_theta0[i];
      if (sct & JP_SCALE_ANGLE) t.cls = pcls(a1, a3);  // :735-742
      terms_by_kind[T_ANGLE].push_back(t);
    }
    for (int i = 0; i < s.ntors; ++i) {
      Term t = mkterm(T_TORS);
      for (int k = 0; k < 4; ++k) t.a[k] = atom0 + s.tors[4 * i + k] - b;
      t.p0 = s.tors_k[i];
      t.p1 = s.tors_nrot[i];
      t.p2 = s.tors_phase[i];
      t.idiv = s.tors_div[i];
      if ((sct & JP_SCALE_TORS) && !(s.tors_unscaled && s.tors_unscaled[i]))   // :838-866
        t.cls = pcls(s.tors[4 * i + 1] - b, s.tors[4 * i + 2] - b);
      terms_by_kind[T_TORS].push_back(t);
      if (s.tors_nbf && s.tors_nbf[i] == 1) {
        const int a1 = s.tors[4 * i] - b, a4 = s.tors[4 * i + 3] - b;
        excess(a1, a4);
        const int t1 = s.atype[a1] - b, t4 = s.atype[a4] - b;
        Term p = mkterm(T_P14);
        p.a[0] = atom0 + a1;
        p.a[1] = atom0 + a4;
        p.a[2] = t1 * nt1 + t4;   // LJ table index
        p.p0 = std::min(s.s14_vdw[t1], s.s14_vdw[t4]);
        p.p1 = std::min(s.s14_ele[t1], s.s14_ele[t4]) * ccoef * s.charge[a1] * s.charge[a4];
        p.cls = pcls(a1, a4);   // :758-787
        terms_by_kind[T_P14].push_back(p);
      }
    }
    for (int i = 0; i < s.nimpr; ++i) {
      Term t = mkterm(T_IMPR);
      for (int k = 0; k < 4; ++k) t.a[k] = atom0 + s.impr[4 * i + k] - b;
      t.p0 = s.impr_k[i];
      t.p1 = s.impr_nrot[i];
      t.p2 = s.impr_phase[i];
      t.idiv = s.impr_div[i];
      if ((sct & JP_SCALE_IMPR) && ralsd) {   // n_matrix(min icls, max icls), :911-917
        int na = 0;
        for (int k = 0; k < 4; ++k) na += inA[s.impr[4 * i + k] - b];
        t.cls = na == 4 ? 0 : (na > 0 ? 1 : 2);
      } else if ((sct & JP_SCALE_IMPR) && rsplit) {
        int lo = 2, hi = 0;
        for (int k = 0; k < 4; ++k) {
          lo = std::min(lo, icl[s.impr[4 * i + k] - b]);
          hi = std::max(hi, icl[s.impr[4 * i + k] - b]);
        }
        t.cls = ((tab1 >> (3 * lo + hi)) & 1u) ? 0 : 2;
      }
      terms_by_kind[T_IMPR].push_back(t);
    }
    double ds = 0.0;
    for (int i = 0; i < n; ++i) ds += s.charge[i] * dwork[i];
    R.dself = zd ? -(1.5 / rc) * ds * 0.5 * ccoef : 0.0;
    for (int k = 0; k < 3; ++k) {
      double d = 0.0;
      for (int i = 0; i < n; ++i) d += s.charge[i] * dwk[(size_t)k * n + i];
      R.dself_cls[k] = zd ? -(1.5 / rc) * d * 0.5 * ccoef : 0.0;
    }
    // GE weight: a fixed slot per replica, per window [low, high, c0..cndeg]
    R.ge_off = r * kGeCap;
    R.hist_off = r * JP_GE_MAX_BINS;
    hge.resize((size_t)(r + 1) * kGeCap, 0.0);
    if (s.ge) {
      R.ge_nwin = s.ge->nwindow;
      R.ge_ndeg = s.ge->ndeg;
      R.ge_alphalw = s.ge->alphalw;
      R.ge_alphaup = s.ge->alphaup;
      R.ge_celw = s.ge->celw;
      R.ge_ceup = s.ge->ceup;
      R.ge_tempce = s.ge->tempce;
      R.ge_lower = s.ge->lower;
      R.ge_upper = s.ge->upper;
      pack_ge(*s.ge, hge.data() + R.ge_off);
    }
    if (s.ncelres > 0) {   // CELRES residues (global atom ids); their largest radius
      if (hres_cmm.empty()) hres_cmm.assign(N_all, make_int2(-1, -1));
      for (int i = 0; i < s.ncelres; ++i) {
        const int f = s.celres[2 * i] - b, l = s.celres[2 * i + 1] - b;
        double cen[3] = {0.0, 0.0, 0.0};
        for (int a = f; a <= l; ++a)
          for (int k = 0; k < 3; ++k) cen[k] += s.cord[3 * a + k];
        for (int k = 0; k < 3; ++k) cen[k] /= (double)(l - f + 1);
        for (int a = f; a <= l; ++a) {
          hres_cmm[atom0 + a] = make_int2(atom0 + f, atom0 + l);
          double d2 = 0.0;
          for (int k = 0; k < 3; ++k) d2 += (s.cord[3 * a + k] - cen[k]) * (s.cord[3 * a + k] - cen[k]);
          celres_rmax = std::max(celres_rmax, std::sqrt(d2));
        }
      }
    }
    if (s.restraints) {   // dneres: POSITI, DISTAN, DIHEDR, SETBOU sphere CAP
      const jp_restraints &q = *s.restraints;
      auto item = [&](int kind) {
        Restr t;
        std::memset(&t, 0, sizeof(t));
        t.kind = kind;
        t.rep = r;
        return t;
      };
      for (int i = 0; i < q.npos; ++i) {
        Restr t = item(R_POS);
        t.a[0] = atom0 + q.pos_atom[i] - b;
        for (int k = 0; k < 3; ++k) t.p[k] = q.pos_ref[3 * i + k];
        t.p[3] = q.pos_k[i];
        hres.push_back(t);
      }
      for (int i = 0; i < q.ndist; ++i) {
        Restr t = item(R_DIST);
        t.a[0] = (int)hres_idx.size();
        for (int p = q.dist_iptr[i]; p < q.dist_iptr[i + 1]; ++p) hres_idx.push_back(atom0 + q.dist_iatom[p] - b);
        t.a[1] = t.a[2] = (int)hres_idx.size();
        for (int p = q.dist_jptr[i]; p < q.dist_jptr[i + 1]; ++p) hres_idx.push_back(atom0 + q.dist_jatom[p] - b);
        t.a[3] = (int)hres_idx.size();
        t.p[0] = q.dist_lo[i];
        t.p[1] = q.dist_up[i];
        t.p[2] = q.dist_klo[i];
        t.p[3] = q.dist_kup[i];
        hres.push_back(t);
      }
      for (int i = 0; i < q.ndihe; ++i) {
        Restr t = item(R_DIHE);
        for (int k = 0; k < 4; ++k) t.a[k] = atom0 + q.dihe_atom[4 * i + k] - b;
        t.p[0] = q.dihe_lo[i];
        t.p[1] = q.dihe_up[i];
        t.p[2] = q.dihe_klo[i];
        t.p[3] = q.dihe_kup[i];
        hres.push_back(t);
      }
      const int quartic = q.cap_function == JP_CAP_BIQUADRATIC;   // sphere only (validated)
      const int shape = quartic ? kCapSphereQuartic : q.cap_shape == 0 ? JP_CAP_SPHERE : q.cap_shape;
      auto shape_params = [&](Restr &t, const double *wall, const double *ell) {
        if (shape == JP_CAP_BOX) for (int k = 0; k < 6; ++k) t.p[6 + k] = wall[k];
        if (shape == JP_CAP_ELLIPSOID) for (int k = 0; k < 3; ++k) t.p[6 + k] = ell[k];
      };
      for (int i = 0; i < q.ncap_group; ++i) {
        Restr t = item(R_CAPG);
        t.a[0] = atom0 + q.cap_group[2 * i] - b;
        t.a[1] = atom0 + q.cap_group[2 * i + 1] - b;
        t.a[2] = shape;
        double m = 0.0;
        for (int a = q.cap_group[2 * i] - b; a <= q.cap_group[2 * i + 1] - b; ++a) m += s.mass[a];
        for (int k = 0; k < 3; ++k) t.p[k] = q.cap_center[k];
        t.p[3] = q.cap_radius;
        t.p[4] = q.cap_k;
        t.p[5] = 1.0 / m;
        shape_params(t, q.cap_wall, q.cap_ellipse);
        hres.push_back(t);
      }
      for (int i = 0; i < q.ncap_atom; ++i) {
        Restr t = item(R_CAPA);
        t.a[0] = atom0 + q.cap_atom[i] - b;
        t.a[1] = shape;
        for (int k = 0; k < 3; ++k) t.p[k] = q.cap_center[k];
        t.p[3] = q.cap_atom_radius;
        t.p[4] = q.cap_atom_k;
        shape_params(t, q.cap_atom_wall, q.cap_atom_ellipse);
        hres.push_back(t);
      }
    }
    atom0 += n;
    blk0 += R.nblk;
  }
  // CMM cells of all replicas, level-major: level 1 of every replica, then level 2, ...
  c->cmm = prm->cal15m == JP_CAL15M_CMM;
  if (c->cmm) {
    int off = 0;
    for (int l = 1; l <= 5; ++l) {
      const int base = off;
      for (int r = 0; r < nrep; ++r) {
        Rep &R = reps[r];
        if (!R.cmm || l > R.nlev) continue;
        R.cell_off[l] = off;
        off += R.nv[l] * R.nv[l] * R.nv[l];
        c->cmm_nlev = std::max(c->cmm_nlev, R.nlev);
      }
      c->cmm_ncell[l] = off - base;
    }
  }
  c->reps = reps;
  c->natom = atom0;
  c->nblk = blk0;
  c->nslot = blk0 * kTile;
  c->nunit = (int)units.size();
  for (const Unit &u : units) c->ngroups += u.n >= 2 ? 1 : 0;
  c->nsub = sub0;
  c->nkeys = key0;
  c->ncol = col0;
  c->nkin = std::max(8, 2 * prm->icslop + 2);
  std::vector<Term> terms;
  for (auto &v2 : terms_by_kind) terms.insert(terms.end(), v2.begin(), v2.end());
  c->nterm = (int)terms.size();
  std::vector<int> hblk_rep(c->nblk);
  for (int r = 0; r < nrep; ++r)
    for (int bb = 0; bb < reps[r].nblk; ++bb) hblk_rep[reps[r].blk0 + bb] = r;
  // tile-list chunks: (i-block, j0) for j0 = i, i+32, ... inside the replica
  std::vector<int> chunk_i, chunk_j0, blk_chunk0(c->nblk + 1, 0);
  for (int bb = 0; bb < c->nblk; ++bb) {
    const Rep &R = reps[hblk_rep[bb]];
    blk_chunk0[bb] = (int)chunk_i.size();
    for (int j0 = bb; j0 < R.blk0 + R.nblk; j0 += 32) {
      chunk_i.push_back(bb);
      chunk_j0.push_back(j0);
    }
  }
  blk_chunk0[c->nblk] = (int)chunk_i.size();
  c->nchunk = (int)chunk_i.size();
  c->tile_cap_total = c->nchunk * 32;   // every candidate could be a tile: no overflow

  // ---- device allocation ---------------------------------------------------------------
  DevPtrs &P = c->P;
  int e = 0;
  const int N = c->natom;
  e |= dput(c, &P.x, hx);
  e |= dput(c, &P.v, hv);
  e |= dalloc(c, &P.x0, 3 * (size_t)N);
  e |= dalloc(c, &P.vback, 3 * (size_t)N);
  e |= dalloc(c, &P.xback, 3 * (size_t)N);
  e |= dalloc(c, &P.forcec, 3 * (size_t)N);
  e |= dput(c, &P.mass, hmass);
  e |= dput(c, &P.imass, himass);
  e |= dput(c, &P.chg, hchg);
  e |= dput(c, &P.typ, htyp);
  e |= dput(c, &P.rep_of, hrep);
  e |= dalloc(c, &P.slot_of, (size_t)N);
  e |= dalloc(c, &P.frc, 3 * (size_t)N);
  e |= dalloc(c, &P.grd, 3 * (size_t)N);
  bool anysplit = false;   // partial McMD: the class-1 gradient set
  for (int r = 0; r < nrep; ++r) anysplit |= reps[r].split != 0;
  if (anysplit && c->fp64) e |= dalloc(c, &P.grd1, 3 * (size_t)N);
  if (anysplit && !c->fp64) e |= dalloc(c, &P.frc1, 3 * (size_t)N);
  e |= dput(c, &P.excl_ptr, hexp);
  e |= dput(c, &P.excl_idx, hexi);
  e |= dalloc(c, &P.excl_slot, hexi.size());
  e |= dalloc(c, &P.pos_f, (size_t)c->nslot);
  e |= dalloc(c, &P.pos_d, (size_t)c->nslot);
  e |= dalloc(c, &P.off, 3 * (size_t)c->nslot);
  e |= dalloc(c, &P.styp, (size_t)c->nslot);
  e |= dalloc(c, &P.satom, (size_t)c->nslot);
  e |= dput(c, &P.blk_rep, hblk_rep);
  e |= dalloc(c, &P.blk_ctr, (size_t)c->nblk);
  e |= dalloc(c, &P.blk_half, (size_t)c->nblk);
  e |= dalloc(c, &P.blk_ref, 3 * (size_t)c->nblk);
  e |= dput(c, &P.chunk_i, chunk_i);
  e |= dput(c, &P.chunk_j0, chunk_j0);
  e |= dalloc(c, &P.chunk_nz, (size_t)c->nchunk);
  e |= dalloc(c, &P.chunk_cnt, (size_t)c->nchunk + 1);
  e |= dalloc(c, &P.chunk_off, (size_t)c->nchunk + 1);
  e |= dalloc(c, &P.tmp_masks, (size_t)c->tile_cap_total * 32);
  e |= dalloc(c, &P.tiles, (size_t)c->tile_cap_total);
  e |= dalloc(c, &P.tile_shift, (size_t)c->tile_cap_total);
  e |= dalloc(c, &P.tile_src, (size_t)c->tile_cap_total);
  // compact tiles: at most one per tile (an i-block's j entries never outnumber 32 per tile)
  e |= dput(c, &P.blk_chunk0, blk_chunk0);
  // pair records: at most one per tile and half (a unit's records never outnumber the tiles
  // of its block), plus one so that the kernels' record pairs stay inside the arrays
  const size_t rec_cap = 2 * (size_t)c->tile_cap_total + 2;
  e |= dalloc(c, &P.ct_cnt, 2 * (size_t)c->nblk + 1);
  e |= dalloc(c, &P.ct_off, 2 * (size_t)c->nblk + 1);
  e |= dalloc(c, &P.ct_blk, rec_cap);
  e |= dalloc(c, &P.ct_info, rec_cap);
  e |= dalloc(c, &P.tmp_occ, (size_t)c->nchunk * 32 * 2);
  e |= dalloc(c, &P.chunk_ent, 2 * ((size_t)c->nchunk + 1));
  e |= dalloc(c, &P.chunk_eoff, 2 * ((size_t)c->nchunk + 1));
  e |= dalloc(c, &P.tile_occ, 2 * (size_t)c->tile_cap_total);
  e |= dalloc(c, &P.tile_eoff, 2 * (size_t)c->tile_cap_total);
  e |= dalloc(c, &P.ct_j, rec_cap * 32);
  e |= dalloc(c, &P.ct_mask, rec_cap * kHalf);
  e |= dalloc(c, &P.nctiles, 1);
  if (c->cmm) e |= dalloc(c, &P.ct_mask_el, rec_cap * kHalf);
  if (c->cmm) {
    int ntot = 0;
    for (int l = 1; l <= 5; ++l) ntot += c->cmm_ncell[l];
    e |= dalloc(c, &P.tmp_masks_el, (size_t)c->tile_cap_total * 32);
    e |= dalloc(c, &P.cmm_cell, (size_t)N);
    if (!hres_cmm.empty()) e |= dput(c, &P.cmm_res, hres_cmm);
    e |= dalloc(c, &P.gwk, 3 * (size_t)N);
    e |= dalloc(c, &P.cmm_pop, (size_t)ntot);
    e |= dalloc(c, &P.cmm_pot, 13 * (size_t)ntot);
    e |= dalloc(c, &P.cmm_raw, 10 * (size_t)c->cmm_ncell[1]);
    e |= dalloc(c, &P.cmm_c0, 3 * (size_t)nrep);
    e |= dalloc(c, &P.cmm_e, (size_t)nrep);
    e |= dalloc(c, &P.cmm_enew, (size_t)nrep);
    e |= dalloc(c, &P.ene_ext, (size_t)nrep);
    // external environments on the level-1 cells (zeros for replicas without one)
    std::vector<unsigned char> hflag((size_t)c->cmm_ncell[1], 0);
    std::vector<double> hpot((size_t)13 * c->cmm_ncell[1], 0.0);
    for (int r = 0; r < nrep; ++r) {
      const Rep &R = c->reps[r];
      if (!R.ext) continue;
      const size_t nc = (size_t)R.nv[1] * R.nv[1] * R.nv[1];
      for (size_t q = 0; q < nc; ++q) {
        hflag[R.cell_off[1] + q] = sys[r].ext_cmm->flag[q] ? 1 : 0;
        for (int k = 0; k < 13; ++k) hpot[(R.cell_off[1] + q) * 13 + k] = sys[r].ext_cmm->pot[q * 13 + k];
      }
    }
    e |= dput(c, &P.ext_flag, hflag);
    e |= dput(c, &P.ext_pot, hpot);
  }
  e |= dalloc(c, &P.ntiles, 1);
  e |= dalloc(c, &P.key, (size_t)N);
  e |= dalloc(c, &P.hist, (size_t)c->nkeys + 1);        // +1: sentinel for the scan
  e |= dalloc(c, &P.hist_scan, (size_t)c->nkeys + 1);
  e |= dalloc(c, &P.cursor, (size_t)c->nkeys + 1);
  e |= dput(c, &P.col_rep, hcol_rep);
  e |= dalloc(c, &P.col_nb, (size_t)c->ncol + 1);
  e |= dalloc(c, &P.col_blk, (size_t)c->ncol + 1);
  e |= dalloc(c, &P.rep_hmax, 3 * (size_t)nrep);
  e |= dalloc(c, &P.sorted, (size_t)N);
  e |= dput(c, &P.units, units);
  std::vector<int> small_idx, quad_idx;
  for (int i = 0; i < (int)units.size(); ++i) (units[i].n == 4 ? quad_idx : small_idx).push_back(i);
  e |= dput(c, &P.small_idx, small_idx);
  e |= dput(c, &P.quad_idx, quad_idx);
  e |= dput(c, &P.terms, terms);
  e |= dput(c, &P.reps, reps);
  e |= dput(c, &P.ge_coef, hge);
  e |= dalloc(c, &P.ge_hist, (size_t)nrep * JP_GE_MAX_BINS);
  e |= dalloc(c, &P.mlp, (size_t)nrep * kMlpSlot);
  e |= dput(c, &P.lam, hlam);
  e |= dalloc(c, &P.ene_cls, (size_t)nrep * 4);
  e |= dalloc(c, &P.com, (size_t)std::max(1, prm->icslop) * nrep * 16);
  e |= dalloc(c, &P.ene_fix, 16 * (size_t)nrep + 1);
  if (!e) P.tile_ctr = reinterpret_cast<int *>(P.ene_fix + 16 * (size_t)nrep);
  e |= dalloc(c, &P.kin_fix, (size_t)c->nkin * c->nsub);
  e |= dput(c, &P.nfr, hnfr);
  e |= dalloc(c, &P.scale, (size_t)nrep);
  e |= dalloc(c, &P.done, (size_t)nrep);
  e |= dalloc(c, &P.rep_fail, (size_t)nrep);
  e |= dalloc(c, &P.lam_dew, (size_t)nrep);
  e |= dalloc(c, &P.lam_step, (size_t)5 * nrep);
  if (prm->alsd != JP_ALSD_NONE) {
    e |= dalloc(c, &P.alsd_cnt, (size_t)nrep * JP_ALSD_MAX_LBINS);
    e |= dalloc(c, &P.alsd_f, (size_t)nrep * JP_ALSD_MAX_LBINS);
    e |= dalloc(c, &P.alsd_cnt2, (size_t)nrep * JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS);
    e |= dalloc(c, &P.alsd_f2, (size_t)nrep * JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS);
  }
  e |= dalloc(c, &P.status, 1);
  e |= dalloc(c, &P.bar, 4);
  P.wait_cycles = kDefaultWaitCycles;
  e |= dalloc(c, &P.pair_cnt, (size_t)nrep);
  e |= dalloc(c, &P.ene_hist, (size_t)c->hist_cap * nrep * JP_MAXENE);
  e |= dalloc(c, &P.temp_hist, (size_t)c->hist_cap * nrep);
  e |= dalloc(c, &P.step_ctr, 2);
  e |= dput(c, &P.lj_f, ljf);
  e |= dput(c, &P.lj_d, ljd);
  e |= dput(c, &P.lj14, lj14);
  c->nres = (int)hres.size();
  if (c->nres) {
    e |= dput(c, &P.restr, hres);
    if (!hres_idx.empty()) e |= dput(c, &P.res_idx, hres_idx);
  }
  if (c->hbond) {
    // listed pairs of an atom are bounded by the atoms within the list radius at a density
    // of 0.2 per A^3 (liquid water holds 0.1); each marked pair is counted at both atoms
    long long nhb = 0;
    for (int a = 0; a < N; ++a) nhb += hbty[htyp[a] & kTypeMask];
    const double rl = rc + 1.5;
    const long long per = (long long)std::ceil(0.2 * 4.0 / 3.0 * std::acos(-1.0) * rl * rl * rl);
    c->hb_cap = (int)std::min<long long>(std::max<long long>(nhb * per, 1024), 1LL << 30);
    e |= dput(c, &P.hb_tab, hbt);
    e |= dput(c, &P.hb_pair, hbp);
    e |= dput(c, &P.hb_type, hbty);
    e |= dalloc(c, &P.hb_list, (size_t)c->hb_cap);
    e |= dalloc(c, &P.hb_n, 1);
  }
  e |= dalloc(c, &c->scan_scratch,
              (size_t)std::max(std::max(c->nkeys, c->ncol), c->nchunk) / 1024 + 4);
  if (e) { jp_destroy(c); return JP_E_CUDA; }
  // the tile-row prefix must cover the sentinel entry; row_cnt[nblk] stays 0
  // ---- constants ---------------------------------------------------------------------------
  // ZD constants (incel.f90:655-658); the atom cut-off is the same pair formula with all
  // three zero: E = qi qj / r, F = qi qj / r^3 d (enear.f90 #ACT lines)
  const bool zd = prm->cal15m == JP_CAL15M_ZD;
  c->zc.rc2 = rc * rc;
  c->zc.zcore = zd ? 1.5 / rc : 0.0;
  c->zc.fcoeff = zd ? 1.0 / (rc * rc * rc) : 0.0;
  c->zc.bcoeff = 0.5 * c->zc.fcoeff;
  c->zc.rlim = rc + 1.5;
  c->zc.cmm = c->cmm ? 1 : 0;
  if (c->cmm) {   // near field without cut-off, out to two level-1 cells along a diagonal
    double s1 = 0.0;
    for (int r = 0; r < nrep; ++r) s1 = std::max(s1, c->reps[r].siz[1]);
    c->zc.rc2 = 1.0e30;
    // CELRES: atoms sit up to a residue radius away from the centre that picks their cell
    // (1 A more for the deformation of a residue between rebuilds)
    const double rres = hres_cmm.empty() ? 0.0 : 2.0 * (celres_rmax + 1.0);
    c->zc.rlim = std::max(2.0 * std::sqrt(3.0) * s1 + rres, rc) * 1.0001 + 0.01;
  }
  c->zc.nt1 = nt1;
  IntConst &ic = c->ic;
  ic.dt = prm->dt;
  ic.temp = prm->temp;
  ic.temp_start = prm->temp_start;
  ic.heat_loop = prm->heat_loop;
  ic.tempco = prm->tempco;
  ic.shake_method = prm->shake_method;
  ic.shake_tol = prm->shake_tol;
  ic.shake_maxit = prm->shake_maxit;
  ic.icslop = prm->icslop;
  ic.fcstol = prm->fcstol;
  ic.psetmp = prm->psetmp;
  ic.method = prm->method;
  ic.nrep = nrep;
  ic.nsub_total = c->nsub;
  ic.natom = N;
  ic.nkin = c->nkin;
  ic.nsmall = (int)small_idx.size();
  ic.nquad = (int)quad_idx.size();
  ic.qbase = (ic.nsmall + 31) / 32 * 32;
  ic.nvirt = ic.qbase + (8 * ic.nquad + 31) / 32 * 32;
  ic.ge_prescaled = 0;
  ic.stop = (prm->stop_center >= JP_STOP_TRANS && prm->stop_center <= JP_STOP_BOTH) ? prm->stop_center : 0;
  ic.ncom = std::max(1, prm->icslop);
  ic.taut = prm->taut;
  ic.alsd = 0;
  for (int r = 0; r < nrep; ++r) ic.alsd |= reps[r].lam_mode != 0;
  c->alsd = ic.alsd != 0;
  ic.split = anysplit ? 1 : 0;
  c->split = anysplit;
  c->classes = c->alsd || c->split;
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
  c->nsm = std::max(1, nsm);
  // one wave: every warp resident at once, each with an equal share of the tiles
  c->pair_warps = std::max(1, nsm) * (256 / 32) * pair_blocks_per_sm(c->fp64, c->zc.nt1);
  c->cano_grid = cano_grid(c->fp64, c->device);
  CK(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  CK(cudaStreamCreateWithFlags(&c->st2, cudaStreamNonBlocking));
  CK(cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming));
  CK(cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming));
  CK(cudaEventCreate(&c->ev_a));
  CK(cudaEventCreate(&c->ev_b));
  int rs = tune_blocks(c, prm->tune_blocks != 0);
  if (rs < 0) { jp_destroy(c); return rs; }
  *out = c;
  return JP_OK;
}

void jp_destroy(jp_ctx *c) {
  if (!c) return;
  cudaSetDevice(c->device);
  if (c->st) cudaStreamSynchronize(c->st);
  if (c->g_step) cudaGraphExecDestroy(c->g_step);
  if (c->g_rebuild) cudaGraphExecDestroy(c->g_rebuild);
  for (void *p : c->allocs) cudaFree(p);
  for (auto ev : c->tev) cudaEventDestroy(ev);
  if (c->ev_a) cudaEventDestroy(c->ev_a);
  if (c->ev_b) cudaEventDestroy(c->ev_b);
  if (c->st) cudaStreamDestroy(c->st);
  if (c->st2) cudaStreamDestroy(c->st2);
  if (c->ev_fork) cudaEventDestroy(c->ev_fork);
  if (c->ev_join) cudaEventDestroy(c->ev_join);
  delete c;
}

int jp_rebuild_cells(jp_ctx *c, int32_t replica) {
  if (!c || replica < -1 || replica >= c->nrep) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  c->rebuild_pending = false;
  enqueue_rebuild(c);   // all replicas share one pass
  CK(cudaStreamSynchronize(c->st));
  return check_status(c);
}

int jp_set_state(jp_ctx *c, int32_t r, const double *cord, const double *vel) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  if (int e = flush_rebuild(c)) return e;
  const Rep &R = c->reps[r];
  if (cord) CK(cudaMemcpyAsync(c->P.x + 3 * (size_t)R.atom0, cord, sizeof(double) * 3 * R.natom,
                               cudaMemcpyHostToDevice, c->st));
  if (vel) CK(cudaMemcpyAsync(c->P.v + 3 * (size_t)R.atom0, vel, sizeof(double) * 3 * R.natom,
                              cudaMemcpyHostToDevice, c->st));
  if (cord) launch_update_pos(c->P, c->nslot, c->fp64, c->qscale, c->st);
  CK(cudaStreamSynchronize(c->st));
  return JP_OK;
}

int jp_get_state(jp_ctx *c, int32_t r, double *cord, double *vel) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  const Rep &R = c->reps[r];
  if (cord) CK(cudaMemcpyAsync(cord, c->P.x + 3 * (size_t)R.atom0, sizeof(double) * 3 * R.natom,
                               cudaMemcpyDeviceToHost, c->st));
  if (vel) CK(cudaMemcpyAsync(vel, c->P.v + 3 * (size_t)R.atom0, sizeof(double) * 3 * R.natom,
                              cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return JP_OK;
}

// One dnergy of every replica, synchronised: the accumulators then hold its gradients and
// energies (cord: the replica's new coordinates first, nullable)
int eval_forces(jp_ctx *c, int32_t r, const double *cord) {
  if (int e = flush_rebuild(c)) return e;
  const Rep &R = c->reps[r];
  if (cord) {
    CK(cudaMemcpyAsync(c->P.x + 3 * (size_t)R.atom0, cord, sizeof(double) * 3 * R.natom,
                       cudaMemcpyHostToDevice, c->st));
    launch_update_pos(c->P, c->nslot, c->fp64, c->qscale, c->st);
  }
  enqueue_forces(c, true, true);
  enqueue_bonded(c);
  CK(cudaStreamSynchronize(c->st));
  CK(cudaGetLastError());
  return JP_OK;
}

// the replica's eneval from the energy slots (the ZD self term into ELE15)
int read_eneval(jp_ctx *c, int32_t r, double *eneval) {
  long long ef[16];
  CK(cudaMemcpy(ef, c->P.ene_fix + 16 * (size_t)r, sizeof(ef), cudaMemcpyDeviceToHost));
  double tot = 0.0;
  for (int k = 1; k < JP_MAXENE; ++k) {
    eneval[k] = (double)ef[k] * kEneInv;
    if (k == JP_E_ELE15) eneval[k] += c->reps[r].dself;
    tot += eneval[k];
  }
  eneval[0] = tot;
  return JP_OK;
}

// the replica's gradient in accumulator set `set` (0: frc / grd, 1: the class-1 set frc1 /
// grd1), written to out or, with add, added to it
int read_grad(jp_ctx *c, int32_t r, int set, double *out, bool add) {
  const Rep &R = c->reps[r];
  const size_t n3 = 3 * (size_t)R.natom;
  std::vector<double> g(n3);
  if (c->fp64) {
    CK(cudaMemcpy(g.data(), (set ? c->P.grd1 : c->P.grd) + 3 * (size_t)R.atom0, sizeof(double) * n3,
                  cudaMemcpyDeviceToHost));
  } else {
    std::vector<long long> f(n3);
    CK(cudaMemcpy(f.data(), (set ? c->P.frc1 : c->P.frc) + 3 * (size_t)R.atom0, sizeof(long long) * n3,
                  cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n3; ++i) g[i] = (double)f[i] * kFrcInv;
  }
  for (size_t i = 0; i < n3; ++i) out[i] = add ? out[i] + g[i] : g[i];
  return JP_OK;
}

// steps start from zero force and energy accumulators; the class energies stay readable
// (jp_get_lambda) until the next step clears them
int clear_eval(jp_ctx *c) {
  if (c->fp64) CK(cudaMemsetAsync(c->P.grd, 0, sizeof(double) * 3 * c->natom, c->st));
  else CK(cudaMemsetAsync(c->P.frc, 0, sizeof(long long) * 3 * c->natom, c->st));
  if (c->split && c->fp64) CK(cudaMemsetAsync(c->P.grd1, 0, sizeof(double) * 3 * c->natom, c->st));
  if (c->split && !c->fp64) CK(cudaMemsetAsync(c->P.frc1, 0, sizeof(long long) * 3 * c->natom, c->st));
  CK(cudaMemsetAsync(c->P.ene_fix, 0, sizeof(long long) * (16 * c->nrep + 1), c->st));
  CK(cudaStreamSynchronize(c->st));
  return JP_OK;
}

int jp_energy_grad(jp_ctx *c, int32_t r, const double *cord, double *eneval, double *grad) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  if (int e = eval_forces(c, r, cord)) return e;
  if (eneval)
    if (int e = read_eneval(c, r, eneval)) return e;
  if (grad) {   // classes 1 and 2 together for a partial-McMD replica
    if (int e = read_grad(c, r, 0, grad, false)) return e;
    if (c->reps[r].split)
      if (int e = read_grad(c, r, 1, grad, true)) return e;
  }
  if (int e = clear_eval(c)) return e;
  return check_status(c);
}

// the class-weight override of replica r (jp_energy_grad_cls on an ALSD replica): weights of
// one class (cls 0..2) or back to lambda's (cls < 0)
int set_cls_override(jp_ctx *c, int32_t r, int cls) {
  Rep &R = c->reps[r];
  R.cls_over = cls >= 0 ? 1 : 0;
  for (int k = 0; k < 3; ++k) R.cls_w[k] = k == cls ? 1.0 : 0.0;
  CK(cudaMemcpyAsync(c->P.reps + r, &R, sizeof(Rep), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  return JP_OK;
}

int jp_energy_grad_cls(jp_ctx *c, int32_t r, const double *cord, double *eneval, double *ecls, double *grad,
                       int32_t *nfrg_out) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  const Rep &R = c->reps[r];
  const int nfrg = R.lam_mode ? 3 : R.split ? 2 : 1;
  if (nfrg_out) *nfrg_out = nfrg;
  const size_t n3 = 3 * (size_t)R.natom;
  if (nfrg == 3) {   // one evaluation per class, the weights set to that class alone
    for (int q = 0; q < 3; ++q) {
      if (int e = set_cls_override(c, r, q)) return e;
      int e = eval_forces(c, r, q == 0 ? cord : nullptr);
      if (!e && eneval && q == 0) e = read_eneval(c, r, eneval);
      if (!e && grad) e = read_grad(c, r, 0, grad + q * n3, false);
      if (!e && ecls) {
        long long ef[4];
        CK(cudaMemcpy(ef, c->P.ene_cls + 4 * (size_t)r, sizeof(ef), cudaMemcpyDeviceToHost));
        ecls[q] = (double)ef[q] * kEneInv + R.dself_cls[q];
      }
      if (!e) e = clear_eval(c);
      if (!e) e = check_status(c);
      if (e) {
        set_cls_override(c, r, -1);
        return e;
      }
    }
    return set_cls_override(c, r, -1);
  }
  if (int e = eval_forces(c, r, cord)) return e;
  if (eneval)
    if (int e = read_eneval(c, r, eneval)) return e;
  if (nfrg == 2) {   // partial McMD: class 1 in the frc1 / grd1 set, class 2 in frc / grd
    if (grad) {
      if (int e = read_grad(c, r, 1, grad, false)) return e;
      if (int e = read_grad(c, r, 0, grad + n3, false)) return e;
    }
    if (ecls) {
      long long ef[4];
      CK(cudaMemcpy(ef, c->P.ene_cls + 4 * (size_t)r, sizeof(ef), cudaMemcpyDeviceToHost));
      ecls[0] = (double)ef[0] * kEneInv + R.dself_cls[0];
      ecls[1] = (double)ef[2] * kEneInv + R.dself_cls[2];
    }
  } else {
    if (grad)
      if (int e = read_grad(c, r, 0, grad, false)) return e;
    if (ecls) {
      double ev[JP_MAXENE];
      if (int e = read_eneval(c, r, ev)) return e;
      ecls[0] = ev[0];
    }
  }
  if (int e = clear_eval(c)) return e;
  return check_status(c);
}

int jp_ge_hist_setup(jp_ctx *c, int32_t r, double emin, double emax, int32_t nbin, int32_t nbor) {
  if (!c || r < -1 || r >= c->nrep || nbin < 0 || nbor < 0) return JP_E_INVALID;
  if (nbin > 0 && (!(emax > emin) || nbin + 2 * nbor > JP_GE_MAX_BINS)) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  for (int q = (r < 0 ? 0 : r); q < (r < 0 ? c->nrep : r + 1); ++q) {
    Rep &R = c->reps[q];
    const double de = nbin > 0 ? (emax - emin) / nbin : 1.0;
    R.hist_n = nbin > 0 ? nbin + 2 * nbor : 0;
    R.hist_min = emin - de * nbor;
    R.hist_inv = 1.0 / de;
    CK(cudaMemset(c->P.ge_hist + R.hist_off, 0, sizeof(unsigned long long) * JP_GE_MAX_BINS));
    CK(cudaMemcpy(c->P.reps + q, &R, sizeof(Rep), cudaMemcpyHostToDevice));
  }
  return JP_OK;
}

int jp_ge_hist_get(jp_ctx *c, int32_t r, double *counts, int32_t clear) {
  if (!c || r < 0 || r >= c->nrep || !counts) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  const Rep &R = c->reps[r];
  std::vector<unsigned long long> h(R.hist_n);
  if (R.hist_n > 0)
    CK(cudaMemcpy(h.data(), c->P.ge_hist + R.hist_off, sizeof(unsigned long long) * R.hist_n,
                  cudaMemcpyDeviceToHost));
  for (int i = 0; i < R.hist_n; ++i) counts[i] = (double)h[i];
  if (clear) CK(cudaMemset(c->P.ge_hist + R.hist_off, 0, sizeof(unsigned long long) * JP_GE_MAX_BINS));
  return JP_OK;
}

int jp_ge_set(jp_ctx *c, int32_t r, const jp_ge *g) {
  if (!c || r < 0 || r >= c->nrep || !g) return JP_E_INVALID;
  if (c->prm.method != JP_METHOD_GE) return JP_E_INVALID;
  if (g->nwindow < 1 || g->nwindow > JP_GE_MAX_WINDOWS || g->ndeg < 0 || g->ndeg > JP_GE_MAX_DEG ||
      !g->coef || !g->low || !g->high || !(g->ceup > g->celw))
    return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  Rep &R = c->reps[r];
  std::vector<double> slot(kGeCap, 0.0);
  pack_ge(*g, slot.data());
  R.ge_nwin = g->nwindow;
  R.ge_ndeg = g->ndeg;
  R.ge_alphalw = g->alphalw;
  R.ge_alphaup = g->alphaup;
  R.ge_celw = g->celw;
  R.ge_ceup = g->ceup;
  R.ge_tempce = g->tempce;
  R.ge_lower = g->lower;
  R.ge_upper = g->upper;
  CK(cudaMemcpy(c->P.ge_coef + R.ge_off, slot.data(), sizeof(double) * kGeCap, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->P.reps + r, &R, sizeof(Rep), cudaMemcpyHostToDevice));
  return JP_OK;
}

int jp_alsd_hist_setup(jp_ctx *c, int32_t r, double lmin, double lmax, int32_t nbin, int32_t nbor,
                       double emin, double emax, int32_t ne) {
  if (!c || r < 0 || r >= c->nrep || nbin < 0 || nbor < 0 || ne < 0) return JP_E_INVALID;
  if (!c->P.alsd_cnt || c->reps[r].lam_mode == JP_ALSD_NONE) return JP_E_INVALID;
  if (nbin > 0 && (!(lmax > lmin) || nbin + 2 * nbor > JP_ALSD_MAX_LBINS)) return JP_E_INVALID;
  if (ne > 0 && (!(emax > emin) || ne > JP_ALSD_MAX_EBINS)) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  if (int e = flush_rebuild(c)) return e;
  CK(cudaStreamSynchronize(c->st));
  Rep &R = c->reps[r];
  const double dl = nbin > 0 ? (lmax - lmin) / nbin : 1.0;
  R.alsd_nl = nbin > 0 ? nbin + 2 * nbor : 0;
  R.alsd_lmin = lmin - dl * nbor;
  R.alsd_linv = 1.0 / dl;
  R.alsd_ne = nbin > 0 ? ne : 0;
  R.alsd_emin = emin;
  R.alsd_einv = ne > 0 ? ne / (emax - emin) : 0.0;
  const size_t n1 = JP_ALSD_MAX_LBINS, n2 = (size_t)JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS;
  CK(cudaMemset(c->P.alsd_cnt + r * n1, 0, sizeof(unsigned long long) * n1));
  CK(cudaMemset(c->P.alsd_f + r * n1, 0, sizeof(double) * n1));
  CK(cudaMemset(c->P.alsd_cnt2 + r * n2, 0, sizeof(unsigned long long) * n2));
  CK(cudaMemset(c->P.alsd_f2 + r * n2, 0, sizeof(double) * n2));
  CK(cudaMemcpy(c->P.reps + r, &R, sizeof(Rep), cudaMemcpyHostToDevice));
  return JP_OK;
}

int jp_alsd_hist_get(jp_ctx *c, int32_t r, double *counts, double *dedl, double *counts2, double *dedl2,
                     int32_t clear) {
  if (!c || r < 0 || r >= c->nrep || !c->P.alsd_cnt) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  const Rep &R = c->reps[r];
  const int nl = R.alsd_nl, ne = R.alsd_ne;
  const size_t n1 = JP_ALSD_MAX_LBINS, n2 = (size_t)JP_ALSD_MAX_EBINS * JP_ALSD_MAX_LBINS;
  std::vector<unsigned long long> h(n2);
  std::vector<double> f(n2);
  if (nl > 0) {
    CK(cudaMemcpy(h.data(), c->P.alsd_cnt + r * n1, sizeof(unsigned long long) * nl, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(f.data(), c->P.alsd_f + r * n1, sizeof(double) * nl, cudaMemcpyDeviceToHost));
    for (int i = 0; i < nl; ++i) {
      if (counts) counts[i] = (double)h[i];
      if (dedl) dedl[i] = f[i];
    }
  }
  if (ne > 0 && (counts2 || dedl2)) {
    CK(cudaMemcpy(h.data(), c->P.alsd_cnt2 + r * n2, sizeof(unsigned long long) * n2, cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(f.data(), c->P.alsd_f2 + r * n2, sizeof(double) * n2, cudaMemcpyDeviceToHost));
    for (int a = 0; a < ne; ++a)
      for (int i = 0; i < nl; ++i) {
        if (counts2) counts2[(size_t)a * nl + i] = (double)h[(size_t)a * JP_ALSD_MAX_LBINS + i];
        if (dedl2) dedl2[(size_t)a * nl + i] = f[(size_t)a * JP_ALSD_MAX_LBINS + i];
      }
  }
  if (clear) {
    CK(cudaMemset(c->P.alsd_cnt + r * n1, 0, sizeof(unsigned long long) * n1));
    CK(cudaMemset(c->P.alsd_f + r * n1, 0, sizeof(double) * n1));
    CK(cudaMemset(c->P.alsd_cnt2 + r * n2, 0, sizeof(unsigned long long) * n2));
    CK(cudaMemset(c->P.alsd_f2 + r * n2, 0, sizeof(double) * n2));
  }
  return JP_OK;
}

// whether any replica's force-scaling step needs k_ge_scale (a network weight)
void update_prescale(jp_ctx *c) {
  int any = 0;
  for (int q = 0; q < c->nrep; ++q) any |= c->reps[q].mlp_on != 0;
  if (any != c->ic.ge_prescaled) {   // the step graph changes: capture it again
    c->ic.ge_prescaled = any;
    drop_graphs(c);
  }
}

int jp_alsd_set_mlp(jp_ctx *c, int32_t r, const float *params, double emin, double emax) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  if (c->prm.method != JP_METHOD_GE || c->reps[r].lam_mode == JP_ALSD_NONE) return JP_E_INVALID;
  if (params && !(emax > emin)) return JP_E_INVALID;
  const int np = jp_mlp_nparam(2, 2);
  if (np < 0 || np > kMlpSlot) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  Rep &R = c->reps[r];
  R.mlp_on = params ? 2 : 0;
  R.mlp_e0 = emin;
  R.mlp_e1 = emax;
  if (params)
    CK(cudaMemcpy(c->P.mlp + (size_t)r * kMlpSlot, params, sizeof(float) * np, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->P.reps + r, &R, sizeof(Rep), cudaMemcpyHostToDevice));
  update_prescale(c);
  return JP_OK;
}

int jp_ge_set_mlp(jp_ctx *c, int32_t r, const float *params) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  if (c->prm.method != JP_METHOD_GE || c->reps[r].lam_mode != JP_ALSD_NONE) return JP_E_INVALID;
  const int np = jp_mlp_nparam(1, 1);
  if (np < 0 || np > kMlpSlot) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  Rep &R = c->reps[r];
  R.mlp_on = params ? 1 : 0;
  if (params) CK(cudaMemcpy(c->P.mlp + (size_t)r * kMlpSlot, params, sizeof(float) * np,
                            cudaMemcpyHostToDevice));
  CK(cudaMemcpy(c->P.reps + r, &R, sizeof(Rep), cudaMemcpyHostToDevice));
  update_prescale(c);
  return JP_OK;
}

int jp_get_lambda(jp_ctx *c, int32_t r, double *lam2, double *ecls) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  if (lam2) CK(cudaMemcpy(lam2, c->P.lam + 2 * r, sizeof(double) * 2, cudaMemcpyDeviceToHost));
  if (ecls) {
    long long ef[4] = {0, 0, 0, 0};
    if (c->classes) CK(cudaMemcpy(ef, c->P.ene_cls + 4 * (size_t)r, sizeof(ef), cudaMemcpyDeviceToHost));
    for (int k = 0; k < 3; ++k) ecls[k] = (double)ef[k] * kEneInv + c->reps[r].dself_cls[k];
  }
  return JP_OK;
}

int jp_set_lambda(jp_ctx *c, int32_t r, double lambda, double lambda_v) {
  if (!c || r < 0 || r >= c->nrep || !std::isfinite(lambda) || !std::isfinite(lambda_v))
    return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  CK(cudaStreamSynchronize(c->st));
  const double v[2] = {lambda, lambda_v};
  CK(cudaMemcpy(c->P.lam + 2 * r, v, sizeof(v), cudaMemcpyHostToDevice));
  return JP_OK;
}

int jp_pair_count(jp_ctx *c, int32_t r, int64_t *count) {
  if (!c || r < 0 || r >= c->nrep || !count) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  long long v = 0;
  CK(cudaMemcpy(&v, c->P.pair_cnt + r, sizeof(long long), cudaMemcpyDeviceToHost));
  *count = v;
  return JP_OK;
}

int jp_set_timing(jp_ctx *c, int enable) {
  if (!c) return JP_E_INVALID;
  c->tm.enabled = enable != 0;
  return JP_OK;
}

void jp_default_min_params(jp_min_params *p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->method = JP_MIN_STEEP;   // inpmin.f90 defaults: METHOD= STEE, UPDATE 10, CONVGR 0.1,
  p->max_loop = 1000;         // ISTEPL 0.01, step-length factors 1.2 / 0.6
  p->update = 10;
  p->convgr = 0.1;
  p->step0 = 0.01;
  p->up = 1.2;
  p->down = 0.6;
  p->line_conv = 0.1;         // line-search convergence rate and limit (inpmin.f90 :90-92)
  p->line_max = 10;
}


int jp_minimize(jp_ctx *c, const jp_min_params *mp, int32_t *iters, double *eneval, double *rmsf,
                int32_t *state) {
  if (!c || !mp) return JP_E_INVALID;
  if ((mp->method != JP_MIN_STEEP && mp->method != JP_MIN_CONJ) || mp->max_loop < 1 || mp->update < 0 ||
      !(mp->convgr >= 0.0) || !(mp->step0 > 0.0) || !std::isfinite(mp->convgr) || !std::isfinite(mp->step0))
    return JP_E_INVALID;
  if (mp->method == JP_MIN_STEEP &&
      (!(mp->up > 0.0) || !(mp->down > 0.0) || !std::isfinite(mp->up) || !std::isfinite(mp->down)))
    return JP_E_INVALID;
  if (c->split) return JP_E_INVALID;   // the class-1 gradient set has no role in the minimiser
  CK(cudaSetDevice(c->device));
  if (int e = flush_rebuild(c)) return e;
  if (mp->method == JP_MIN_CONJ) {   // conj.f90:48-53: no SHAKE with conjugate gradients
    if (mp->line_max < 1 || !(mp->line_conv >= 0.0) || !std::isfinite(mp->line_conv)) return JP_E_INVALID;
    if (c->prm.shake_method != JP_SHAKE_NONE && c->ngroups > 0) return JP_E_INVALID;
    for (int r = 0; r < c->nrep; ++r) {
      const int rc = minimize_conj(c, r, mp, iters, eneval, rmsf, state);
      if (rc != JP_OK) return rc;
    }
    enqueue_rebuild(c);
    CK(cudaStreamSynchronize(c->st));
    return check_status(c);
  }
  if (!c->P.mins && dalloc(c, &c->P.mins, (size_t)c->nrep)) return JP_E_CUDA;
  DevPtrs &P = c->P;
  cudaStream_t st = c->st;
  const bool shake = c->prm.shake_method != JP_SHAKE_NONE && c->nunit > 0;
  const int nmax = mp->max_loop;
  CK(cudaMemsetAsync(P.mins, 0, sizeof(MinState) * c->nrep, st));
  // the first evaluation (mini.f90 inimin) at the current positions
  enqueue_zero(c, false);
  enqueue_pair(c, false, true);
  enqueue_bonded(c);
  launch_min_init(P, c->natom, c->nrep, c->fp64, mp->step0, mp->convgr, st);
  // one linsrd iteration of every replica, replayed as a graph
  cudaGraph_t g;
  cudaGraphExec_t gx = nullptr;
  CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  launch_min_move(P, c->natom, c->fp64, nmax, shake, st);
  if (shake) {
    launch_shake_only(P, c->ic, 0, c->nunit, st);
    launch_min_commit(P, c->natom, nmax, st);
  }
  launch_update_pos(P, c->nslot, c->fp64, c->qscale, st);
  enqueue_zero(c, false);
  enqueue_pair(c, false, true);   // CMM: the far field at every evaluation
  enqueue_bonded(c);
  launch_min_decide(P, c->natom, c->nrep, c->fp64, nmax, mp->up, mp->down, mp->convgr, st);
  CK(cudaStreamEndCapture(st, &g));
  const cudaError_t ie = cudaGraphInstantiate(&gx, g, 0);
  cudaGraphDestroy(g);
  CK(ie);
  std::vector<MinState> hs(c->nrep);
  int it = 0;
  cudaError_t err = cudaSuccess;
  while (it < nmax && err == cudaSuccess) {
    const int chunk = std::min(nmax - it, 64);
    for (int k = 0; k < chunk && err == cudaSuccess; ++k) {
      err = cudaGraphLaunch(gx, st);
      ++it;
      if (mp->update > 0 && it % mp->update == 0) enqueue_rebuild(c);   // steep.f90:51-54
    }
    if (err != cudaSuccess) break;
    unsigned stat = 0;
    err = cudaMemcpyAsync(&stat, P.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaMemcpyAsync(hs.data(), P.mins, sizeof(MinState) * c->nrep,
                                                  cudaMemcpyDeviceToHost, st);
    if (err == cudaSuccess) err = cudaStreamSynchronize(st);
    if (err != cudaSuccess || stat != 0) break;
    bool running = false;
    for (const MinState &m : hs) running |= m.state == 0 && m.iters < nmax;
    if (!running) break;
  }
  cudaGraphExecDestroy(gx);
  CK(err);
  // leave what the MD step expects: zero accumulators and a list built at these positions
  if (c->fp64) CK(cudaMemsetAsync(P.grd, 0, sizeof(double) * 3 * c->natom, st));
  else CK(cudaMemsetAsync(P.frc, 0, sizeof(long long) * 3 * c->natom, st));
  CK(cudaMemsetAsync(P.ene_fix, 0, sizeof(long long) * (16 * c->nrep + 1), st));
  enqueue_rebuild(c);
  CK(cudaMemcpyAsync(hs.data(), P.mins, sizeof(MinState) * c->nrep, cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  CK(cudaGetLastError());
  bool step_err = false;
  for (int r = 0; r < c->nrep; ++r) {
    const MinState &m = hs[r];
    if (iters) iters[r] = m.iters;
    if (rmsf) rmsf[r] = m.rmsf;
    if (state) state[r] = m.state;
    if (eneval) std::memcpy(eneval + (size_t)r * JP_MAXENE, m.ene, sizeof(m.ene));
    step_err |= m.state == 2;
  }
  const int rs = check_status(c);
  if (rs != JP_OK) return rs;
  return step_err ? JP_E_MIN_STEP : JP_OK;
}

int jp_tile_shape(jp_ctx *c, int32_t r, double *column_scale, int64_t *tiles) {
  if (!c || r < 0 || r >= c->nrep) return JP_E_INVALID;
  if (column_scale) *column_scale = kTuneScale[c->tune_pick[r]];
  if (tiles)
    for (int q = 0; q < JP_TUNE_CANDIDATES; ++q) tiles[q] = c->tune_tiles[(size_t)r * JP_TUNE_CANDIDATES + q];
  return JP_OK;
}

int jp_set_wait_limit(jp_ctx *c, int64_t cycles) {
  if (!c || cycles < 0) return JP_E_INVALID;
  c->P.wait_cycles = cycles > 0 ? (long long)cycles : kDefaultWaitCycles;
  drop_graphs(c);   // the step graph holds the limit it was captured with
  return JP_OK;
}

int jp_set_grid_limit(jp_ctx *c, int32_t blocks) {
  if (!c || blocks < 0) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  const int full = cano_grid(c->fp64, c->device);
  c->cano_grid = blocks > 0 ? std::min((int)blocks, full) : full;
  drop_graphs(c);
  return JP_OK;
}

int jp_last_timing(jp_ctx *c, double *total_ms, double *phase_ms4, int32_t *launches4) {
  if (!c) return JP_E_INVALID;
  if (total_ms) *total_ms = c->tm.total_ms;
  for (int k = 0; k < 4; ++k) {
    if (phase_ms4) phase_ms4[k] = c->tm.phase_ms[k];
    if (launches4) launches4[k] = c->tm.launches[k];
  }
  return JP_OK;
}

int jp_list_stats(jp_ctx *c, int64_t *ntiles, int64_t *npairs_listed, int64_t *nslots) {
  if (!c) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  if (int e = flush_rebuild(c)) return e;
  CK(cudaStreamSynchronize(c->st));
  int nt = 0;
  CK(cudaMemcpy(&nt, c->P.nctiles, sizeof(int), cudaMemcpyDeviceToHost));
  if (ntiles) *ntiles = nt;
  if (nslots) *nslots = c->nslot;
  if (npairs_listed) {
    std::vector<unsigned> m((size_t)nt * kHalf);
    if (nt) CK(cudaMemcpy(m.data(), c->P.ct_mask, sizeof(unsigned) * m.size(), cudaMemcpyDeviceToHost));
    int64_t s = 0;
    for (unsigned v : m) s += __builtin_popcount(v);
    *npairs_listed = s;
  }
  return JP_OK;
}

int jp_launch_counts(jp_ctx *c, int32_t *per_step, int32_t *per_rebuild) {
  if (!c) return JP_E_INVALID;
  if (per_step) *per_step = launches_per_step(c);
  if (per_rebuild) *per_rebuild = c->launches_rebuild;
  return JP_OK;
}

}  // extern "C"

namespace {

// the list rebuild due after the last step of a jp_step call, run before anything that uses
// the list (the next step, a force evaluation, a state change)
int flush_rebuild(jp_ctx *c) {
  if (!c->rebuild_pending) return 0;
  c->rebuild_pending = false;
  if (c->g_rebuild) CK(cudaGraphLaunch(c->g_rebuild, c->st));
  else enqueue_rebuild(c);
  return 0;
}

// what a call returns for steps [done, done + chunk): the energy and temperature records
// and, after its last step, the state of every replica; then the status word.  Copies on
// the context's stream, ahead of the one synchronisation that ends the chunk.
int enqueue_tail(jp_ctx *c, int done, int chunk, double *ene_out, double *temp_out, double *xout,
                 double *vout, bool last) {
  DevPtrs &P = c->P;
  CK(cudaEventRecord(c->ev_b, c->st));
  if (ene_out)
    CK(cudaMemcpyAsync(ene_out + (size_t)done * c->nrep * JP_MAXENE, P.ene_hist,
                       sizeof(double) * (size_t)chunk * c->nrep * JP_MAXENE, cudaMemcpyDeviceToHost, c->st));
  if (temp_out)
    CK(cudaMemcpyAsync(temp_out + (size_t)done * c->nrep, P.temp_hist, sizeof(double) * (size_t)chunk * c->nrep,
                       cudaMemcpyDeviceToHost, c->st));
  if (last && xout)
    CK(cudaMemcpyAsync(xout, P.x, sizeof(double) * 3 * (size_t)c->natom, cudaMemcpyDeviceToHost, c->st));
  if (last && vout)
    CK(cudaMemcpyAsync(vout, P.v, sizeof(double) * 3 * (size_t)c->natom, cudaMemcpyDeviceToHost, c->st));
  return 0;
}

// nsteps iterations of runmd's loop body; xout/vout (nullable, all replicas) receive the
// state after the last step
int step_impl(jp_ctx *c, int nsteps, double *ene_out, double *temp_out, double *xout, double *vout) {
  if (!c->tm.enabled && !c->g_step) {
    if (capture(c, &c->g_step, false)) return JP_E_CUDA;
    if (capture(c, &c->g_rebuild, true)) return JP_E_CUDA;
  }
  for (int k = 0; k < 4; ++k) { c->tm.phase_ms[k] = 0.0; c->tm.launches[k] = 0; }
  c->tm.total_ms = 0.0;
  // SHAKE failures of verlethe are redone with a halved time step; verlet (MICR, CONS)
  // returns the failure, as md_run stops there (verlet.f90:203, md.f90:557)
  const bool retry = c->prm.method >= JP_METHOD_CANO && c->prm.shake_method != JP_SHAKE_NONE;
  if (retry && !c->tm.enabled)
    if (int e = snap_alloc(c)) return e;
  auto due = [&]() { return c->prm.update > 0 && c->idloop % c->prm.update == 0; };
  int done = 0;
  while (done < nsteps) {
    const int chunk = std::min(nsteps - done, c->hist_cap);
    const bool last = done + chunk == nsteps;
    CK(cudaMemsetAsync(c->P.step_ctr + 1, 0, sizeof(int), c->st));
    CK(cudaEventRecord(c->ev_a, c->st));
    unsigned st = 0;
    if (c->tm.enabled) {
      if (int e = flush_rebuild(c)) return e;
      const size_t need = (size_t)chunk * 8;
      while (c->tev.size() < need) {
        cudaEvent_t ev;
        CK(cudaEventCreate(&ev));
        c->tev.push_back(ev);
      }
      std::vector<int> rebuilt(chunk, 0);
      for (int s = 0; s < chunk; ++s) {
        cudaEvent_t *E = &c->tev[(size_t)s * 8];
        enqueue_zero(c, false);
        CK(cudaEventRecord(E[0], c->st));
        enqueue_pair(c, false);
        CK(cudaEventRecord(E[1], c->st));
        enqueue_bonded(c);
        CK(cudaEventRecord(E[2], c->st));
        enqueue_integrate(c);
        CK(cudaEventRecord(E[3], c->st));
        c->idloop += 1;
        if (due()) {
          enqueue_rebuild(c);
          rebuilt[s] = 1;
        }
        CK(cudaEventRecord(E[4], c->st));
      }
      if (int e = enqueue_tail(c, done, chunk, ene_out, temp_out, xout, vout, last)) return e;
      if (int e = read_status(c, &st)) return e;
      for (int s = 0; s < chunk; ++s) {
        cudaEvent_t *E = &c->tev[(size_t)s * 8];
        float ms;
        for (int k = 0; k < 3; ++k) {
          CK(cudaEventElapsedTime(&ms, E[k], E[k + 1]));
          c->tm.phase_ms[k] += ms;
          c->tm.launches[k] += 1;
        }
        if (rebuilt[s]) {
          CK(cudaEventElapsedTime(&ms, E[3], E[4]));
          c->tm.phase_ms[3] += ms;
          c->tm.launches[3] += 1;
        }
      }
    } else if (!retry) {
      for (int s = 0; s < chunk; ++s) {
        if (int e = flush_rebuild(c)) return e;
        CK(cudaGraphLaunch(c->g_step, c->st));
        c->idloop += 1;
        c->rebuild_pending = due();
      }
      if (int e = enqueue_tail(c, done, chunk, ene_out, temp_out, xout, vout, last)) return e;
      if (int e = read_status(c, &st)) return e;
    } else {
      // verlethe with SHAKE: segments that end at a list rebuild, each started from a copy of
      // the state.  A segment in which SHAKE failed is redone from that copy one step at a
      // time, and the failing step goes through retry_step.  A segment holds no rebuild, so
      // the copy and the pair list stay consistent.
      for (int s = 0; s < chunk;) {
        if (int e = flush_rebuild(c)) return e;
        int seg = chunk - s;
        if (c->prm.update > 0) seg = std::min<long long>(seg, c->prm.update - c->idloop % c->prm.update);
        const bool tail = s + seg == chunk;
        if (int e = snap_copy(c, c->snap[0], true, s)) return e;
        for (int k = 0; k < seg; ++k) CK(cudaGraphLaunch(c->g_step, c->st));
        if (tail)
          if (int e = enqueue_tail(c, done, chunk, ene_out, temp_out, xout, vout, last)) return e;
        if (int e = read_status(c, &st)) return e;
        if (st & ERR_TIMEOUT) return check_status(c);
        if (st & kShakeBits) {
          if (int e = clear_after_failure(c)) return e;
          if (int e = snap_copy(c, c->snap[0], false, s)) return e;
          for (int k = 0; k < seg; ++k) {
            if (int e = snap_copy(c, c->snap[1], true, s + k)) return e;
            CK(cudaGraphLaunch(c->g_step, c->st));
            if (int e = read_status(c, &st)) return e;
            if ((st & kShakeBits) && !(st & ERR_TIMEOUT)) {
              const int rc = retry_step(c, c->snap[1], s + k);
              if (rc != JP_OK) return rc;
            } else if (st) {
              return check_status(c);
            }
          }
          if (tail) {
            if (int e = enqueue_tail(c, done, chunk, ene_out, temp_out, xout, vout, last)) return e;
            if (int e = read_status(c, &st)) return e;
          }
        }
        if (st) return check_status(c);
        c->idloop += seg;
        s += seg;
        c->rebuild_pending = due();
      }
    }
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev_a, c->ev_b));
    c->tm.total_ms += ms;
    if (st) return check_status(c);
    done += chunk;
  }
  return JP_OK;
}

}  // namespace

extern "C" {

int jp_step(jp_ctx *c, int32_t nsteps, double *ene_out, double *temp_out) {
  if (!c || nsteps < 0) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  if (nsteps == 0) return JP_OK;
  return step_impl(c, nsteps, ene_out, temp_out, nullptr, nullptr);
}

int jp_step_io(jp_ctx *c, int32_t nsteps, const double *cord_in, const double *vel_in, double *cord_out,
               double *vel_out, double *ene_out, double *temp_out) {
  if (!c || nsteps < 0) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  if (int e = flush_rebuild(c)) return e;
  const size_t n3 = sizeof(double) * 3 * (size_t)c->natom;
  if (cord_in) CK(cudaMemcpyAsync(c->P.x, cord_in, n3, cudaMemcpyHostToDevice, c->st));
  if (vel_in) CK(cudaMemcpyAsync(c->P.v, vel_in, n3, cudaMemcpyHostToDevice, c->st));
  if (cord_in) launch_update_pos(c->P, c->nslot, c->fp64, c->qscale, c->st);
  if (nsteps == 0) {
    if (cord_out) CK(cudaMemcpyAsync(cord_out, c->P.x, n3, cudaMemcpyDeviceToHost, c->st));
    if (vel_out) CK(cudaMemcpyAsync(vel_out, c->P.v, n3, cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    return JP_OK;
  }
  return step_impl(c, nsteps, ene_out, temp_out, cord_out, vel_out);
}

int jp_shake(jp_ctx *c, int32_t r, double *r1, const double *r2) {
  if (!c || r < 0 || r >= c->nrep || !r1 || !r2) return JP_E_INVALID;
  CK(cudaSetDevice(c->device));
  const Rep &R = c->reps[r];
  const size_t n3 = 3 * (size_t)R.natom;
  CK(cudaMemcpyAsync(c->P.xback + 3 * (size_t)R.atom0, r1, sizeof(double) * n3, cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->P.x0 + 3 * (size_t)R.atom0, r2, sizeof(double) * n3, cudaMemcpyHostToDevice, c->st));
  launch_shake_only(c->P, c->ic, R.unit0, R.nunit, c->st);
  CK(cudaMemcpyAsync(r1, c->P.xback + 3 * (size_t)R.atom0, sizeof(double) * n3, cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return check_status(c);
}

}  // extern "C"
