// jp_kernels.h -- kernel entry points shared between the engine's translation units.
#pragma once
#include "jp_common.cuh"

namespace jp {

// cells / tiles (jp_cells.cu)
__global__ void k_cell_key(DevPtrs P, int natom);
__global__ void k_scatter(DevPtrs P, int natom);
__global__ void k_sort_bins(DevPtrs P, int nkeys);
__global__ void k_col_count(DevPtrs P, int ncol);
__global__ void k_clear_slots(DevPtrs P, int nslot, int dummy_type);
__global__ void k_fill_slots(DevPtrs P, int natom);
__global__ void k_excl_slots(DevPtrs P, int natom);
__global__ void k_block_setup(DevPtrs P, int nblk, double qscale);
__global__ void k_fill_pos_d(DevPtrs P, int nslot, double qscale);
// CMM: masks from the level-1 cells (neighbours: Coulomb + LJ into masks and masks_el;
// cells up to idelay apart and r^2 < rc2: LJ only) instead of the list radius
void launch_tile_scan(const DevPtrs& P, int nchunk, double rlim2, float rlimf, double rc2, bool cmm,
                      cudaStream_t st);
__global__ void k_tile_emit(DevPtrs P, int nchunk, int cmm);
// compact tiles of every i-block from the tile list (count, scan, emit); returns the launches
int launch_compact_tiles(const DevPtrs& P, int nblk, int nchunk, int nsm, bool cmm, int* scan_scratch,
                         cudaStream_t st);
// deterministic exclusive scan of n ints (total: the sum, or null); returns the launches
int scan_exclusive(const int* in, int* out, int n, int* scratch, int* total, cudaStream_t st);

// ZD pair constants
struct ZdConst {
  double rc2, zcore, bcoeff, fcoeff;
  double rlim;             // list radius rc + 1.5 (CMM: the farthest listed pair)
  int nt1;                 // LJ table stride (ntype + 1 incl. the dummy type)
  int cmm;                 // CMM near field: no cut-off, Coulomb only where masks_el says
};

// cell multipole method (jp_cmm.cu): cells and multipoles at a list rebuild (before the tile
// scan), and the far field of a step (every cmm_upd steps, or always with force)
void launch_cmm_rebuild(const DevPtrs& P, int natom, int nrep, int ncell1, const int* ncell_lvl,
                        int nlev_max, cudaStream_t st);
void launch_cmm_far(const DevPtrs& P, int natom, int nrep, bool fp64, bool force, double ccoef,
                    cudaStream_t st);

// pair kernels (jp_pair.cu)
// alsd: some replica has ALSD classes; split: some replica keeps partial-McMD class-1 forces
// apart (frc1 / grd1)
void launch_pair_mixed(const DevPtrs& P, const ZdConst& z, int nwarps, bool count, bool alsd, bool split,
                       cudaStream_t st);
void launch_pair_fp64(const DevPtrs& P, const ZdConst& z, int nwarps, bool count, bool alsd, bool split,
                      cudaStream_t st);
// co-resident blocks per SM of the (non-counting) pair kernel: the grid is one full wave
int pair_blocks_per_sm(bool fp64, int nt1);
void launch_update_pos(const DevPtrs& P, int nslot, bool fp64, double qscale, cudaStream_t st);

// H-bond 10-12 pairs (jp_hbond.cu): their list at a rebuild (after the tile list), their
// term at every force evaluation
void launch_hb_list(const DevPtrs& P, int cap, int nt1, int nblk, cudaStream_t st);
void launch_hbond(const DevPtrs& P, int cap, double rc2, int nt1, bool fp64, bool alsd, cudaStream_t st);

// restraints and CAP boundary (jp_restraint.cu)
void launch_restraints(const DevPtrs& P, int n, bool fp64, bool alsd, cudaStream_t st);

// steepest-descent minimisation (jp_minimize.cu)
void launch_min_init(const DevPtrs& P, int natom, int nrep, bool fp64, double step0, double convgr,
                     cudaStream_t st);
void launch_min_move(const DevPtrs& P, int natom, bool fp64, int max_loop, bool shake, cudaStream_t st);
void launch_min_commit(const DevPtrs& P, int natom, int max_loop, cudaStream_t st);
void launch_min_decide(const DevPtrs& P, int natom, int nrep, bool fp64, int max_loop, double up,
                       double down, double convgr, cudaStream_t st);

// bonded (jp_bonded.cu)
void launch_bonded(const DevPtrs& P, int nterm, bool fp64, double zb, double zf, bool alsd,
                   cudaStream_t st);

// integration (jp_integrate.cu)
struct IntConst {
  double dt;
  double temp, temp_start;
  int heat_loop;
  int tempco;              // 1 whole-system, 2 per sub-system
  int shake_method;        // 0 none, 1 exact 2-atom, 2 iterative 2-atom
  double shake_tol;
  int shake_maxit;
  int icslop;
  double fcstol;
  double psetmp;
  int method;
  int nrep;
  int nsub_total;
  int natom;
  int nkin;                // kinetic-sum slots; the last one is MICR's
  // virtual lanes of the CANO/GE kernel: [0, nsmall) one 1-3 atom unit each (small_idx),
  // [qbase, nvirt) eight lanes per 4-atom group (quad_idx); qbase and nvirt are multiples of 32
  int nsmall, nquad, qbase, nvirt;
  int ge_prescaled;        // force scales computed by k_ge_scale before the integration kernel
  int alsd;                // some replica runs ALSD (lambda carried by the integration kernel)
  int split;               // some replica keeps partial-McMD class-1 forces apart (frc1 / grd1)
  int stop;                // STOPCE 1 translation, 2 rotation, 3 both; 0 = off
  int ncom;                // centre-of-mass sum slots (one per velocity update of a step)
  double taut;             // METHOD= CONS relaxation time (fs)
  int no_hist;             // record no histogram visit (a sub-step of a redone step that is
                           // not its last)
};
int cano_grid(bool fp64, int device);   // co-resident blocks of the integration kernels
// energies of the step, force scale, verlet (MICR) or verlethe (CANO/GE) with SHAKE,
// temperatures and step counters: one cooperative launch, or for a CANO/GE system with more
// virtual lanes than the cooperative grid (grid_max blocks) holds, one launch per phase
void launch_integrate(const DevPtrs& P, const IntConst& c, int nunit, bool fp64, int grid_max,
                      cudaStream_t st);
int integrate_launches(const IntConst& c, int grid_max);   // kernels launch_integrate launches
void launch_shake_only(const DevPtrs& P, const IntConst& c, int unit0, int nunit, cudaStream_t st);
// per-replica force scale of this step (McMD polynomial or surrogate network) into P.scale
void launch_ge_scale(const DevPtrs& P, const IntConst& c, cudaStream_t st);
constexpr int kMlpSlot = 4608;   // floats per replica >= jp_mlp_nparam(2, 2)

}  // namespace jp
