// jp_common.cuh -- device-side data layout shared by the engine's kernels.
//
// Layout in HBM (all replicas concatenated; "atom" = original md_run order, "slot" =
// cell-sorted order padded to 32-atom blocks):
//   atoms : x, v      double[N][3]   master FP64 state (cord, vel of md_run)
//           frc       long long[N][3] 64-bit fixed-point gradient (mixed path)
//           grd       double[N][3]   FP64 gradient (FP64 path)
//   slots : pos_f     float4[S]      (x-off, y-off, z-off, q*sqrt(332/eps)) block-local
//           pos_d     double4[S]     (x, y, z, q*sqrt(332/eps)) absolute (FP64 path)
//           off       double[S][3]   block frame origin of the slot (ref + L*image)
//           styp      int[S]         LJ type (padding -> dummy zero type)
//           satom     int[S]         atom of the slot, -1 for padding
//   blocks: 32 slots each; tiles = (i-block, j-block) pairs with a 32x32 interaction mask.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "jpgpu.h"

namespace jp {

constexpr int kTile = 32;
constexpr int kHalf = 16;   // i atoms of a pair record: half a block
// fixed-point scales: forces 2^32 per kcal/mol/A, energies 2^32 per kcal/mol,
// kinetic sums (m v^2, amu A^2/fs^2) 2^40.
constexpr double kFrcScale = 4294967296.0;
constexpr double kFrcInv = 1.0 / 4294967296.0;
constexpr double kEneScale = 4294967296.0;
constexpr double kEneInv = 1.0 / 4294967296.0;
constexpr double kKinScale = 1099511627776.0;
constexpr double kKinInv = 1.0 / 1099511627776.0;
// Largest magnitude of one fixed-point contribution (2^56 in scaled units: a force term of
// 1.7e7 kcal/mol/A, an energy term of 1.7e7 kcal/mol).  Each accumulator receives at most a
// few hundred contributions per step, so sums of terms below this bound stay inside the
// 64-bit range; a term beyond it is reported instead of wrapping the sum.
constexpr double kFixLim = 72057594037927936.0;

constexpr double kConvcv = 4.184e-4;       // md.f90:56
constexpr double kGas = 8.31451;           // PHYCNS gascst
constexpr double kJouCal = 4.184;

// error bits of the device status word
enum : unsigned {
  ERR_SHAKE_NOCONV = 1u, ERR_SHAKE_SINGULAR = 2u, ERR_NONFINITE = 4u,
  ERR_FIX_OVERFLOW = 8u, ERR_LIST_OVERFLOW = 16u, ERR_SORT = 32u, ERR_TIMEOUT = 64u,
  ERR_STOP_MASS = 128u, ERR_STOP_SINGULAR = 256u, ERR_FREE_WINDOW = 512u, ERR_CMM_GRID = 1024u
};

// per-replica constants
struct Rep {
  int atom0, natom;        // atom range
  int blk0, nblk;          // block range (slots [32*blk0, 32*(blk0+nblk)))
  int unit0, nunit;        // integration units
  int sub0, nsub;          // temperature sub-systems (global ids)
  int key0;                // first sort key of the replica
  int col0, ncol;          // first global xy column, number of columns
  int grid[3];             // columns in x, in y; z bins per column
  double box[3], invbox[3];
  double cell[3];          // column edge in x, in y; z-bin height
  double dself;
  int ge_off, ge_nwin, ge_ndeg;   // offset into the GE coefficient array
  double ge_alphalw, ge_alphaup, ge_celw, ge_ceup, ge_tempce;
  double ge_lower, ge_upper;      // ALSD linear walls below celw / above ceup
  int hist_off, hist_n;           // energy histogram slot and bin count (0 = off)
  double hist_min, hist_inv;      // lower edge of bin 0 and 1 / bin width
  int mlp_on;                     // 1: McMD weight from the surrogate network instead of the
                                  // polynomial; 2: ALSD weight in lambda from the (E, lambda) network
  double mlp_e0, mlp_e1;          // energy range the (E, lambda) network's first input spans
  // ALSD weight iteration: lambda bins (0 = off) and (E, lambda) energy bins of the replica's
  // histograms, lower edges and inverse widths
  int alsd_nl, alsd_ne;
  double alsd_lmin, alsd_linv, alsd_emin, alsd_einv;
  // ALSD (cluster classes AA / AB / BB scaled by powers of lambda)
  int lam_mode;                   // JP_ALSD_*; 0 = off
  int lam_ke_sub;                 // sub-system whose temperature holds lambda's kinetic term, -1 none
  int lam_tc;                     // lambda velocity coupled to the thermostat
  int stop_n;                     // centre-of-mass stop: atoms [atom0, atom0 + stop_n); 0 = off
  double lam_m, lam_im;           // lambda mass and its inverse
  double dself_cls[3];            // ZD self term by class
  // GEPSME= AND / OR / XOR with cluster atoms (partial McMD, nfrg = 2): class-1 terms
  // (bit 3 ca + cb of cls_tab set for atom regions ca, cb: 0 A, 1 B, 2 neither) accumulate
  // into frc1 / grd1, class-2 terms into frc / grd; class energies in slots 0 and 2
  int split;
  unsigned cls_tab;
  // class weights set to one class at a time (cls_over = 1) while dnergy's per-class
  // outputs of an ALSD replica are evaluated; cls_w[AA, AB, BB]
  int cls_over;
  double cls_w[3];
  // BOUNDA= NO: the periodic box is a container large enough that minimum image is the
  // identity while every atom stays in [win_lo, win_hi]
  int free_bnd;
  double win_lo[3], win_hi[3];
  // CMM (CAL15M= CMM): levels 1..nlev (index 0 unused), nv cells per axis, edge siz;
  // cell_off = first global cell of the level in the CMM cell arrays (x fastest)
  int cmm, nlev, idelay, cmm_upd;
  int nv[6], cell_off[6];
  double siz[6];
  int ext;                        // EXTCMM= environment on the level-1 cells (ext_flag, ext_pot)
  double ext_c0[3];               // its grid centre, used instead of the atoms' centroid
};

// class weight of a term (verlethe.f90:116-163): class 0 = AA, 1 = AB, 2 = BB
__host__ __device__ __forceinline__ double lam_factor(int mode, double lam, int cls) {
  if (mode == JP_ALSD_NONE || cls == 2) return 1.0;
  if (cls == 0) return mode == JP_ALSD_LMD ? lam * lam : lam;
  return mode == JP_ALSD_LMD ? lam : sqrt(lam);
}
// the same, or the replica's one-class weights while its per-class outputs are evaluated
__host__ __device__ __forceinline__ double cls_weight(const Rep& R, double lam, int cls) {
  return R.cls_over ? R.cls_w[cls] : lam_factor(R.lam_mode, lam, cls);
}
// LJ type in the low bits of typ/styp; bit 30 = ALSD cluster atom; bits 28-29 = the atom's
// region code (0 A, 1 B, 2 neither) in a partial-McMD replica
constexpr int kTypeMask = 0xffff;
constexpr int kRegionShift = 28;

// integration unit: a SHAKE group (2-4 atoms) or a lone atom (n = 1)
struct Unit {
  int n;
  int a[4];
  int sub;                 // sub-system of its atoms
  int rep;
  double d2[6];            // squared constraint lengths, md_run pair order
};

// bonded term of any kind, flattened
enum : int { T_BOND = 0, T_ANGLE = 1, T_TORS = 2, T_IMPR = 3, T_P14 = 4, T_EXCESS = 5 };
struct Term {
  int kind;
  int rep;
  int a[4];
  double p0, p1, p2;       // bond: k, r0 | angle: k, t0 | tors: k, nrot, phase | 14: svdw, sele
  int idiv;
  int cls;                 // ALSD class 0 = AA, 1 = AB, 2 = BB
};

// restraint or CAP term of one replica (jp_restraint.cu); atoms are global ids
enum : int { R_POS = 0, R_DIST = 1, R_DIHE = 2, R_CAPG = 3, R_CAPA = 4 };
constexpr int kCapSphereQuartic = 4;   // CAP shape code: sphere with the half-biquadratic function
struct Restr {
  int kind;
  int rep;
  int a[4];        // POS, CAPA: atom | DIST: group i = res_idx[a0, a1), group j = res_idx[a2, a3)
                   // | DIHE: the four atoms | CAPG: first and last atom of the group
                   // | CAPG: a[2], CAPA: a[1] = shape (JP_CAP_*)
  double p[12];    // POS: ref xyz, k | DIST, DIHE: lo, up, k_lo, k_up
                   // | CAPG, CAPA: centre xyz, radius, k, 1 / group mass (CAPG), then
                   //   walls lo/hi x, y, z (box) or 1 / semi-axis^2 x, y, z (ellipsoid)
};

// steepest-descent minimisation state of one replica (jp_minimize.cu)
struct MinState {
  double stp;               // step length (A, whole replica)
  double e_old;             // total energy of the last evaluation
  double gsum, gsum_new;    // sum |g|^2 of the last evaluation / being summed
  double rmsf;              // sqrt(gsum / natom)
  int state;                // 0 running, 1 converged, 2 step length too small
  int iters;                // iterations done
  double ene[JP_MAXENE];    // energies of the last evaluation
};

struct DevPtrs {
  // bound of every grid-barrier wait of the cooperative integration, in SM clock cycles
  long long wait_cycles;
  // atoms
  double *x, *v, *x0, *vback, *xback, *forcec;
  double *mass, *imass, *chg;
  int *typ, *rep_of, *slot_of;
  long long *frc;
  double *grd;
  long long *frc1;                // partial McMD: class-1 gradient (fixed point / FP64 path)
  double *grd1;
  // exclusions (global atom ids)
  int *excl_ptr, *excl_idx;
  int *excl_slot;                 // slot of each partner after the last sort
  // slots / blocks
  float4 *pos_f;
  double4 *pos_d;
  double *off;
  int *styp, *satom;
  int *blk_rep;
  float4 *blk_ctr, *blk_half;     // bbox (wrapped frame) centre / half extent
  double *blk_ref;                // [B][3]
  // tile-list build: chunk = (i-block, 32 candidate j-blocks from j0)
  int *chunk_i, *chunk_j0;        // static per context
  unsigned *chunk_nz;             // non-empty candidates of the chunk (bit b = j0+b)
  int *chunk_cnt, *chunk_off;     // their count and its exclusive scan [nchunk+1]
  unsigned *tmp_masks;            // [nchunk*32][32] masks of the chunk candidates
  // tiles
  int2 *tiles;                    // dense (i-block, j-block)
  float4 *tile_shift;             // dense min-image shift of block refs (mixed path)
  int *tile_src;                  // [T] where each tile's mask rows are in tmp_masks: chunk * 32 + candidate
  int *ntiles;                    // device scalar
  // compact tiles (what the pair kernels run on): an i-block and 32 j entries
  int *blk_chunk0;                // [nblk+1] first chunk of each i-block (static)
  int *ct_cnt, *ct_off;           // pair records per unit (2 i-block + half) and their scan [2 nblk+1]
  int *ct_blk;                    // [CT] unit of each pair record
  int4 *ct_info;                  // [CT] what the emit needs of each record: its first source tile,
                                  // the global entry of its slot 0, the end of its unit's entries,
                                  // and (end of its block's tiles) << 1 | half
  unsigned *tmp_occ;              // [nchunk*32][2] occupied j lanes of each chunk candidate, per half
  int *chunk_ent, *chunk_eoff;    // per half [2][nchunk+1]: entries per chunk, their exclusive scan
  unsigned *tile_occ;             // [T][2] occupied j lanes of each tile, per half
  int *tile_eoff;                 // [T][2] first entry of each tile in its half's order (global)
  float4 *ct_j;                   // [CT][32] (image shift into the i frame, slot bits; -1 = empty)
  unsigned *ct_mask, *ct_mask_el; // [CT][32] rotated masks (listed pairs; CMM Coulomb pairs)
  int *nctiles;                   // device scalar
  // cell sort
  unsigned *key;                  // per atom
  int *hist, *hist_scan, *cursor; // per key
  int *sorted;                    // compact order -> atom
  int *col_rep;                   // replica of each xy column (static)
  int *col_nb, *col_blk;          // blocks per column and their exclusive scan [ncol+1]
  float *rep_hmax;                // largest block half-extent per replica [nrep][3]
  // units / terms
  Unit *units;
  int *small_idx, *quad_idx;      // units of 1-3 atoms / of 4 atoms, in unit order
  Term *terms;
  // replicas
  Rep *reps;
  double *ge_coef;                // JP_GE_MAX_WINDOWS * (JP_GE_MAX_DEG + 3) per replica
  unsigned long long *ge_hist;    // JP_GE_MAX_BINS per replica
  float *mlp;                     // surrogate network parameters, kMlpSlot per replica
  double *lam;                    // ALSD lambda and its velocity [nrep][2]
  long long *ene_cls;             // class energies AA, AB, BB (fixed point) [nrep][4]
  double *com;                    // centre-of-mass stop sums [ncom][nrep][16]
  // CMM: per atom its level-1 cell (0-based ix | iy << 8 | iz << 16) and far-field gradient;
  // per cell (all levels, all replicas) population and 13 multipole coefficients; level-1
  // raw sums; per replica the centroid sums and the far-field energy (last and being built)
  int *cmm_cell;
  int2 *cmm_res;                  // CELRES: first / last atom of the atom's residue, (-1, -1) none
  double *gwk;
  int *cmm_pop;
  double *cmm_pot, *cmm_raw, *cmm_c0;
  long long *cmm_e, *cmm_enew;
  long long *ene_ext;             // EXTCMM energy of the step, per replica (fixed point)
  unsigned *tmp_masks_el;         // CMM tiles: pairs with the Coulomb term (as tmp_masks)
  unsigned char *ext_flag;        // EXTCMM: occupied external level-1 cells (CMM cell index)
  double *ext_pot;                // their 13 coefficients
  // accumulators
  long long *ene_fix;             // [nrep][16], then the pair kernels' tile counter
  int *tile_ctr;                  // next unclaimed tile (zeroed with ene_fix every step)
  long long *kin_fix;             // [nslots_kin][nsub_total]
  double *nfr;                    // DOF per sub-system
  double *scale;                  // per replica force scale (GE / pseudo-T)
  int *done;                      // per replica SHAKE-thermostat loop finished
  int *rep_fail;                  // per replica: a SHAKE group failed this step (1)
  // ALSD weight iteration, per replica: counts and sums of dE/dlambda of the cluster energy
  // per lambda bin [nrep][JP_ALSD_MAX_LBINS], and per (E, lambda) bin
  // [nrep][JP_ALSD_MAX_EBINS][JP_ALSD_MAX_LBINS]; allocated only with ALSD replicas
  unsigned long long *alsd_cnt, *alsd_cnt2;
  double *alsd_f, *alsd_f2;
  double *lam_dew;                // [nrep] the lambda weight term of the step from the network
  double *lam_step;               // [5 nrep] lambda's state through a step of per-phase launches
  unsigned *status;               // error bits
  unsigned *bar;                  // grid barrier of the cooperative integrator [4]
  long long *pair_cnt;            // [nrep]
  double *ene_hist;               // [max_steps][nrep][15]
  double *temp_hist;              // [max_steps][nrep]
  int *step_ctr;                  // device step counter (idloop)
  // LJ tables [(nt+1)^2]: the pair kernels' (C6, C12), zero for H-bond type pairs; the
  // 1-4 terms' (C6, C12) of every type pair
  float2 *lj_f;
  double2 *lj_d;
  double2 *lj14;
  // H-bond 10-12 term: (C10, C12h) and flag per type pair, flag per type; the listed
  // H-bond pairs (atom ids) of the last rebuild and their count
  double2 *hb_tab;
  int *hb_pair, *hb_type;
  int2 *hb_list;
  int *hb_n;
  // restraints and CAP terms, and the atoms of the distance-restraint groups
  Restr *restr;
  int *res_idx;
  MinState *mins;                 // [nrep], allocated by the first jp_minimize
};

// v * scale rounded to a 64-bit integer.  A product beyond +-kFixLim sets ERR_FIX_OVERFLOW
// in *status (ERR_NONFINITE for a NaN or an infinity) and the contribution is dropped, so
// the call that made it returns an error instead of a silently wrapped sum.
__device__ __forceinline__ long long to_fix(double v, double scale, unsigned *status) {
  const double s = v * scale;
  if (!(fabs(s) < kFixLim)) {
    atomicOr(status, isfinite(s) ? ERR_FIX_OVERFLOW : ERR_NONFINITE);
    return 0;
  }
  return __double2ll_rn(s);
}

// The same for an FP32 force at the force scale 2^32: v * 2^32 is exact in FP32, and its
// conversion rounds as the FP64 one does (a float above 2^24 is already an integer), so the
// result equals to_fix((double)v, kFrcScale, status) without the FP64 arithmetic.
__device__ __forceinline__ long long to_fix_f(float v, unsigned *status) {
  const float s = v * 4294967296.0f;
  if (!(fabsf(s) < 72057594037927936.0f)) {
    atomicOr(status, isfinite(v) ? ERR_FIX_OVERFLOW : ERR_NONFINITE);
    return 0;
  }
  return __float2ll_rn(s);
}

__device__ __forceinline__ void atomic_add_ll(long long *p, long long v) {
  atomicAdd(reinterpret_cast<unsigned long long *>(p), static_cast<unsigned long long>(v));
}

__host__ __device__ __forceinline__ double anint(double x) { return round(x); }

// gradient of one atom from a term evaluated in FP64, times its ALSD class weight fs:
// FP64 atomics on the FP64 path, 64-bit fixed point on the mixed path; c1: a class-1 term of
// a partial-McMD replica (into frc1 / grd1)
template <bool FP64>
__device__ __forceinline__ void add_grad(const DevPtrs& P, double fs, int a, double gx, double gy,
                                         double gz, bool c1 = false) {
  gx *= fs; gy *= fs; gz *= fs;   // ALSD class weight (1 otherwise)
  if (FP64) {
    double* g = c1 ? P.grd1 : P.grd;
    atomicAdd(&g[3 * a + 0], gx);
    atomicAdd(&g[3 * a + 1], gy);
    atomicAdd(&g[3 * a + 2], gz);
  } else {
    long long* f = c1 ? P.frc1 : P.frc;
    atomic_add_ll(&f[3 * a + 0], to_fix(gx, kFrcScale, P.status));
    atomic_add_ll(&f[3 * a + 1], to_fix(gy, kFrcScale, P.status));
    atomic_add_ll(&f[3 * a + 2], to_fix(gz, kFrcScale, P.status));
  }
}

// warp-aggregated energy add keyed by (replica, slot)
__device__ __forceinline__ void add_energy(const DevPtrs& P, int rep, int slot, double e) {
  const int key = rep * 16 + slot;
  const unsigned full = 0xffffffffu;
  const int k0 = __shfl_sync(full, key, 0);
  const bool uni = __all_sync(full, key == k0);
  if (uni) {
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(full, e, o);
    if ((threadIdx.x & 31) == 0) atomic_add_ll(&P.ene_fix[key], to_fix(e, kEneScale, P.status));
  } else if (e != 0.0) {
    atomic_add_ll(&P.ene_fix[key], to_fix(e, kEneScale, P.status));
  }
}

// warp-aggregated add of a term's energy to its replica's ALSD class total
__device__ __forceinline__ void add_cls_energy(const DevPtrs& P, int rep, int cls, double e) {
  const int key = rep * 4 + cls;
  const unsigned full = 0xffffffffu;
  const int k0 = __shfl_sync(full, key, 0);
  if (__all_sync(full, key == k0)) {
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(full, e, o);
    if ((threadIdx.x & 31) == 0 && e != 0.0) atomic_add_ll(&P.ene_cls[key], to_fix(e, kEneScale, P.status));
  } else if (e != 0.0) {
    atomic_add_ll(&P.ene_cls[key], to_fix(e, kEneScale, P.status));
  }
}

}  // namespace jp
