/*
 * jpgpu.h -- C ABI of the B200 engine for md_run's per-step force/integrate path.
 *
 * The reference (j_presto md_run, Fortran 90 + OpenMP) has no plugin or FFI layer: its
 * routines share state through modules.  Each entry point below replaces one reference call
 * site, named in its comment as file:line inside src_md_run/.  A Fortran driver binds these
 * through iso_c_binding (a bind(C) interface per entry point); the bundled Python/ctypes
 * host does the same.
 *
 * Conventions
 *   - Units follow md_run: Angstrom, fs, amu, kcal/mol, e.  Velocities in Angstrom/fs.
 *   - real(8) cord(3,N) column-major == C double[N][3]; grad likewise (dE/dx, i.e. -force).
 *   - Atom indices in jp_system are 0-based unless jp_system.index_base == 1 (Fortran arrays
 *     can then be passed unchanged).
 *   - The caller owns every host array; the library copies in and out and keeps no host
 *     pointer after a call returns.  The library owns all device memory inside jp_ctx.
 *   - Return codes mirror md_run's `ier`: 0 ok, >0 warning, <0 fatal (JP_E_* below).
 *   - One host thread per jp_ctx; calls on one context are not re-entrant.
 */
#ifndef JPGPU_H
#define JPGPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JP_MAXENE 15      /* energy slots, md_run COMPAR.f90:37 maxene */
#define JP_MAXNFRG 3      /* cluster-pair classes (ALSD), md_run inpcls.f90 n_matrix */

/* energy slot indices (0-based) of eneval/enevcc, md_run dnergy.f90:17-35 */
enum {
  JP_E_TOTAL = 0, JP_E_BOND = 1, JP_E_ANGLE = 2, JP_E_TORS = 3, JP_E_IMPR = 4,
  JP_E_VDW14 = 5, JP_E_ELE14 = 6, JP_E_VDW15 = 7, JP_E_ELE15 = 8, JP_E_HBOND = 9,
  JP_E_POSRES = 10, JP_E_DISTRES = 11, JP_E_DIHERES = 12, JP_E_CAP = 13
};

/* precision of the force path */
enum { JP_PREC_FP64 = 0, JP_PREC_MIXED = 1 };

/* METHOD= keyword (md_run inpmd.f90:65, stored as idfvsl) */
enum { JP_METHOD_CONS = 1, JP_METHOD_MICR = 2, JP_METHOD_CANO = 3, JP_METHOD_GE = 4 };

/* SHAKEM= keyword (inpmd.f90:71, iyfshk): 0 = no SHAKE */
enum { JP_SHAKE_NONE = 0, JP_SHAKE_HBON = 1, JP_SHAKE_ALLB = 2 };

/* return codes.  Positive values are warnings (md_run ier > 0). */
enum {
  JP_OK = 0,
  JP_W_SHAKE_NOT_CONVERGED = 1,   /* shake.f90:304 ier=1 */
  JP_E_SHAKE_SINGULAR = -2,       /* shake.f90:288 ier=-2 */
  JP_E_SHAKE_ABORT = -9999,       /* verlethe.f90:567 dt halving exhausted */
  JP_E_INVALID = -100,            /* bad argument / inconsistent topology */
  JP_E_CELL_OVERFLOW = -128,      /* celpar.f90 ier=28 analogue: too many tiles */
  JP_E_LIST_OVERFLOW = -151,      /* cutoff.f90 ier=51 analogue */
  JP_E_NONFINITE = -200,          /* non-finite force or coordinate */
  JP_E_FIXED_OVERFLOW = -201,     /* a force contribution left the 64-bit fixed-point range */
  JP_E_CUDA = -300,               /* CUDA runtime error */
  JP_E_NO_DEVICE = -301,
  JP_E_TIMEOUT = -302,            /* a bounded device wait ran out */
  JP_E_NOALLOC_LIMIT = -110,      /* natom above JP_NOALLOC_MAX_ATOMS (jp_nonbond_noalloc) */
  JP_E_STOP_MASS = -121,          /* remotv ier=-1: the stopped atoms have no mass */
  JP_E_STOP_SINGULAR = -122,      /* remotv ier=-2: their inertia tensor is singular */
  JP_E_FREE_WINDOW = -130,        /* BOUNDA= NO: an atom left the window the context was
                                     built for (re-create it from the current state) */
  JP_E_MIN_STEP = -140            /* steep.f90:235-243 ier=-2: the step length fell below
                                     1e-10 A per degree of freedom */
};

/* Generalized-ensemble weight (.nf file, md_run inmcmd.f90:22-40; verlethe.f90:196-321). */
typedef struct jp_ge {
  int32_t nwindow, ndeg;
  const double *coef;        /* [nwindow][ndeg+1]  c(0:ndeg, iwin) */
  const double *low, *high;  /* [nwindow] window bounds in reduced coordinate */
  double alphalw, alphaup;   /* d lnP/dE outside [celw, ceup] */
  double celw, ceup;         /* energy (or lambda) range */
  double tempce;             /* temperature T0 of the weight */
  double lower, upper;       /* ALSD linear wall slopes (LMD only) */
} jp_ge;

/* Frozen external environment of a CMM run (EXTCMM=, setextCMM.f90 / enear_extCMM.f90): the
 * level-1 multipoles of the cells of a surrounding system, on the same cell grid as the
 * simulated one, which is then centred on `center` instead of the atoms' centroid (celpar.f90
 * :54-70).  Each atom interacts with the occupied external cells among its own level-1 cell
 * and its 26 neighbours: the multipole expansion, softened inside 1.5 CELSIZ of the cell
 * centre (enear_extCMM.f90:58-164).  Only 4 cell levels are supported (setextCMM.f90:20). */
typedef struct jp_ext_cmm {
  int32_t nlev;              /* cell levels of the file: must equal the run's (4) */
  double cell;               /* its level-1 cell size: must equal CELSIZ */
  double center[3];          /* grid centre (celx, cely, celz) */
  const uint8_t *flag;       /* [nv1^3] 1 = external cell occupied (exflag1), x fastest */
  const double *pot;         /* [nv1^3][13] its multipoles in the engine's layout: q, p_x..z,
                                Q_xx/2, Q_yy/2, Q_zz/2, Q_xx, Q_yy, Q_zz, Q_xy, Q_yz, Q_zx
                                (setextCMM.f90:44-68 forms this from the file's 10 arrays) */
} jp_ext_cmm;

/* Capacity of a replica's weight and of its energy histogram (fixed when the context is
 * created, so the weight can be replaced between runs without re-capturing anything). */
#define JP_GE_MAX_WINDOWS 16
#define JP_GE_MAX_DEG 15
#define JP_GE_MAX_BINS 4096

/* One McMD weight iteration (GEprep distrib_MULT + lstsquare_final), see jp_ge_fit. */
typedef struct jp_ge_fit_params {
  double emin, emax;         /* minE, maxE of the histogram (distrib_MULT) */
  int32_t nbin, nbor;        /* nBIN bins in [emin, emax] plus nBOR border bins each side */
  double next_emin, next_emax; /* nxminE, nxmaxE: energy range of the new weight */
  double next_temp;          /* nxT: its temperature T0 */
  int32_t nwindow, ndeg;     /* Nwindow, NfitDIM of the new polynomial */
  int32_t ignore_empty;      /* igndat: drop bins with no estimate (weights sqrt(count)) */
  int32_t neglect_low, neglect_high;  /* FneglectL/H: leave the border bins out of the fit */
} jp_ge_fit_params;

/* Restraints and the spherical CAP boundary of one replica (dneres.f90 dneres_PB/_CB,
 * called from dnergy.f90:70-74).  The caller reads psr/dsr/dhr/CAPbound files as md_run
 * does and passes the finished force constants.  Atom indices use jp_system.index_base.
 * Energies go to the slots md_run uses (enevcc(11..14)): JP_E_POSRES .. JP_E_CAP; with
 * ALSD they belong to class BB and are not scaled (grad(:,:,nfrg)). */
typedef struct jp_restraints {
  /* POSITI (dposc, dneres.f90:48-101): E = 1/2 sum k |x - ref|^2, minimum image under
   * BOUNDA= PBC; k = fugcns = (mass *) delta * boltzk * T * w (psr.f90:214-216, inpmd.f90:547) */
  int32_t npos;
  const int32_t *pos_atom;     /* [npos] iugpnt */
  const double *pos_k;         /* [npos] fugcns (kcal/mol/A^2) */
  const double *pos_ref;       /* [npos][3] fucord of those atoms */
  /* DISTAN (ddistc, dneres.f90:107-221): R = <r^-6>^(-1/6) over all pairs of group i x
   * group j (minimum image); E = k_up (R^2 - up^2)^2 if R > up, k_lo (R^2 - lo^2)^2 if
   * R < lo, else 0; k = boltzk * T * w / 2 * fudupr / fudlow */
  int32_t ndist;
  const int32_t *dist_iptr;    /* [ndist+1] CSR of group i's atoms (iuipnt) */
  const int32_t *dist_iatom;
  const int32_t *dist_jptr;    /* [ndist+1] CSR of group j's atoms (iujpnt) */
  const int32_t *dist_jatom;
  const double *dist_lo, *dist_up;     /* furlow, furupr (A) */
  const double *dist_klo, *dist_kup;
  /* DIHEDR (dcdihe, dneres.f90:227-378): phi in [0, 2 pi) as the torsion term defines it;
   * outside [lo, up] E = k (phi - wall)^2 from the nearer wall, across 2 pi;
   * k_up = boltzk T w / (2 fudelu^2), k_lo = boltzk T w / (2 fudell^2) */
  int32_t ndihe;
  const int32_t *dihe_atom;    /* [ndihe][4] iudhcp */
  const double *dihe_lo, *dihe_up;     /* fucdlw, fucdup (radian, 0 <= lo <= up < 2 pi) */
  const double *dihe_klo, *dihe_kup;
  /* SETBOU sphere CAP (dnecap iufcap = 1, capshp = 1, dnecap.f90:80-122, :428-437), no
   * minimum image: the centre of mass C of each group (a range of atoms, chains of the
   * INCLUDE list) has E = 1/2 k (|C - centre| - radius)^2 outside the sphere, its gradient
   * shared by the atoms in proportion to their mass; each listed solute atom has
   * E = 1/2 k_atom (|x - centre| - radius_atom)^2 outside radius_atom = radius - BUFFER */
  int32_t ncap_group;
  const int32_t *cap_group;    /* [ncap_group][2] first and last atom (fechn) */
  int32_t ncap_atom;
  const int32_t *cap_atom;     /* [ncap_atom] iamcap */
  double cap_center[3];        /* fxcbou */
  double cap_radius, cap_k;            /* furcap, fukcap */
  double cap_atom_radius, cap_atom_k;  /* furcap_pro, fukcap_pro */
  /* SETBOU shape (capshp, dnecap.f90:82-250, half-harmonic function): JP_CAP_SPHERE (or 0)
   * as above; JP_CAP_BOX: each coordinate of a group's centre of mass minus cap_center
   * outside [cap_wall[2k], cap_wall[2k+1]] adds 1/2 k (distance to the wall)^2, each
   * coordinate of a listed atom (absolute) likewise with cap_atom_wall (celwal, celwal_pro,
   * compared as dnecap.f90:126-193 compares them); JP_CAP_ELLIPSOID: with
   * s = sum_k c_k^2 e_k > 1 (e = 1 / semi-axis^2, c = position - cap_center) the term is
   * 1/2 k (|c| (1 - s^-1/2))^2 and its gradient k (1 - s^-1/2) c, as dnecap.f90:206-246
   * writes it */
  int32_t cap_shape;
  double cap_wall[6], cap_atom_wall[6];          /* x lo, x hi, y lo, y hi, z lo, z hi */
  double cap_ellipse[3], cap_atom_ellipse[3];    /* fxellp, fxellp_pro */
  /* CAP function (iufcap): 1 (or 0) half-harmonic as above; 2 half-biquadratic, sphere
   * only (dnecap.f90:253-281): with s = (d^2 - R^2) / R^2 > 0 the term is 1/4 k R^2 s^2
   * and its gradient k s c.  The plane-and-cylinder functions 3 and 4 are not built. */
  int32_t cap_function;
} jp_restraints;

enum { JP_CAP_SPHERE = 1, JP_CAP_BOX = 2, JP_CAP_ELLIPSOID = 3 };
enum { JP_CAP_HARMONIC = 1, JP_CAP_BIQUADRATIC = 2 };

/* One replica's system: topology, parameters and coordinates.
 * Mirrors md_run's COMBAS/COMERG/COMMIS module arrays. */
typedef struct jp_system {
  int32_t natom;
  int32_t index_base;          /* 0 (C) or 1 (Fortran) for every atom index below */
  double box[3];               /* PBC cell lengths fxcell(1:3) (BOUNDA= PBC) */
  const double *cord;          /* [natom][3] initial coordinates */
  const double *vel;           /* [natom][3] initial velocities, v(t-dt/2); NULL = zero */
  const double *mass;          /* [natom] fxmass */
  const double *charge;        /* [natom] fxchrg (e) */
  const int32_t *atype;        /* [natom] LJ type ixatyp */
  const int32_t *molecule;     /* [natom] molecule-entry id ixamol (sub-system for TEMPCO);
                                  NULL = one sub-system */
  int32_t ntype;
  const double *c6;            /* [ntype][ntype] fynbpp(1,:,:)  E = C12/r^12 - C6/r^6 */
  const double *c12;           /* [ntype][ntype] fynbpp(2,:,:) */
  const double *s14_vdw;       /* [ntype] fy14sv, 1-4 vdW scale */
  const double *s14_ele;       /* [ntype] fy14se, 1-4 electrostatic scale */
  const int32_t *excl_ptr;     /* [natom+1] CSR of 1-2/1-3/1-4 partners (ix14lt, symmetric) */
  const int32_t *excl_idx;
  int32_t nbond;
  const int32_t *bond;         /* [nbond][2] iypbnd */
  const double *bond_k, *bond_r0;          /* fyfbnd, fyqbnd */
  int32_t nangle;
  const int32_t *angle;        /* [nangle][3] iypang */
  const double *angle_k, *angle_theta0;    /* fyfang, fyqang (radian) */
  int32_t ntors;
  const int32_t *tors;         /* [ntors][4] iyptor */
  const double *tors_k, *tors_nrot, *tors_phase;   /* fyftor, fytrot, fytphs (radian) */
  const int32_t *tors_div, *tors_nbf;              /* iytdiv, iytnbf (1 = 1-4 pair counted) */
  int32_t nimpr;
  const int32_t *impr;         /* [nimpr][4] iypimp */
  const double *impr_k, *impr_nrot, *impr_phase;
  const int32_t *impr_div;
  int32_t nshake;
  const int32_t *shake_n;      /* [nshake] atoms in group (2..4) = iuhshk+1 */
  const int32_t *shake_atoms;  /* [nshake][4] iuashk */
  const double *shake_dist;    /* [nshake][6] target distances d0 in md_run pair order
                                  (1,2),(2,3),(3,1),(4,1),(3,4),(2,4) -- setshk.f90 redshk */
  const jp_ge *ge;             /* McMD weight for METHOD= GE; NULL otherwise */
  const int32_t *cluster;      /* [natom] 1 = atom of region A (CLUSTA, inpcls.f90 icls = 1:
                                  the lambda-scaled cluster of ALSD), 2 = atom of region B
                                  (CLUSTB; GEPSME= AND / OR / XOR only), else 0; NULL = none */
  const jp_ext_cmm *ext_cmm;   /* EXTCMM= environment (CAL15M= CMM only); NULL = none */
  /* Hydrogen-bond 10-12 term (md_run iyeflg(10), on when a type pair has iyppid = 2,
   * incel.f90:170-171; CAL15M= ZD and ATOM): a listed 1-5 pair whose types are marked
   * in hbond keeps its Coulomb term but has E = C12h/r^12 - C10/r^10 instead of the 12-6
   * term, with the same cut-off, summed into JP_E_HBOND (cutoff.f90:98-154 splits the
   * pairs off, enear.f90:330-516 evaluates them).  1-4 pairs keep c6/c12 (dnergv.f90:490).
   * The three tables are shared by all replicas, like c6/c12.  NULL hbond = no such pair. */
  const int32_t *hbond;        /* [ntype][ntype] 1 = iyppid 2, else 0; symmetric */
  const double *c10;           /* [ntype][ntype] fynbpp(3,:,:) of the marked pairs */
  const double *c12h;          /* [ntype][ntype] fynbpp(4,:,:) of the marked pairs */
  const jp_restraints *restraints;   /* POSITI / DISTAN / DIHEDR / SETBOU; NULL = none */
  const int32_t *tors_unscaled;  /* [ntors] 1 = the torsion stays in class BB (unscaled) even
                                    with JP_SCALE_TORS: SCALET's peptide-bond exemption
                                    (scale_tor 2/3, incel.f90:846-866), which the caller
                                    decides from atom and residue names; NULL = none */
  /* CELRES (CAL15M= CMM only, celpar.f90:131-153): every atom of these residues goes to the
   * level-1 cell of the residue's geometric centre instead of its own */
  int32_t ncelres;
  const int32_t *celres;       /* [ncelres][2] first and last atom of each residue */
} jp_system;

/* Run parameters shared by all replicas of a context (md.inp EXE> MD keywords). */
typedef struct jp_params {
  int32_t precision;     /* JP_PREC_FP64 or JP_PREC_MIXED */
  int32_t method;        /* METHOD= (JP_METHOD_CONS / MICR / CANO / GE) */
  double dt;             /* TIMEST (fs) */
  double cutoff;         /* CUTLEN (Angstrom), ZD cut-off */
  double dielectric;     /* DIEVAL */
  int32_t update;        /* UPDATE: pair-list rebuild interval (steps) */
  double temp;           /* SETTEM (K) */
  double temp_start;     /* STARTT (K) */
  int32_t heat_loop;     /* HEATLO (steps); 0 = no heating ramp */
  int32_t tempco;        /* TEMPCO: 1 = one temperature, 2 = per sub-system (itmeth) */
  int32_t shake_method;  /* SHAKEM (JP_SHAKE_*) */
  double shake_tol;      /* COVSHK */
  int32_t shake_maxit;   /* LIMSHK */
  int32_t icslop;        /* SHAKE <-> thermostat iterations (md_run default 3) */
  double fcstol;         /* their tolerance (md_run default 1e-3) */
  double psetmp;         /* PSETMP pseudo temperature; 0 = off */
  int32_t device;        /* CUDA device ordinal */
  /* Adaptive lambda square dynamics (ALSD, CLSTMETHOD= LMD / LMD2, inpcls.f90, verlethe.f90
   * :110-165, :240-321): with jp_system.cluster set, every term of class AA / AB / BB
   * (both / one / no atom in the cluster) enters the forces times lambda^2 / lambda / 1
   * (LMD) or lambda / sqrt(lambda) / 1 (LMD2); lambda moves under
   * f = -2 E_AA lambda - E_AB - dew (LMD), dew the McMD weight in lambda (METHOD= GE). */
  int32_t alsd;          /* GEPSME= (cluster_method): JP_ALSD_* or JP_GEPS_* */
  double lambda0;        /* initial lambda (LAMBDA) */
  double lambda_mass;    /* its mass; 0 = total mass of the cluster (inpcls.f90:350-360) */
  int32_t lambda_temp_control;  /* lambda velocity coupled to the thermostat (l_temp_control) */
  int32_t scale_terms;   /* SCALET: JP_SCALE_* bits; non-bonded terms are always scaled */
  /* METHOD= CONS (verlet.f90:31-34, :172-176, scalet.f90): before each position update the
   * velocities are scaled by sqrt(1 + dt/taut (T0/T - 1)), at most 2, T the temperature
   * of v(t-dt/2) over all degrees of freedom. */
  double taut;           /* TAUTEM relaxation time (fs), > 0 for METHOD= CONS */
  /* STOPCE (remotv.f90, called by verlet.f90:157-158 and verlethe.f90:490-492, :706-709):
   * after each velocity update the centre-of-mass translation and/or rotation of the first
   * stop_natom atoms is removed, positions at time t giving the centre and the inertia
   * tensor; the degrees of freedom drop by 3 / 6 (md.f90:116-121, :186-216). */
  int32_t stop_center;   /* JP_STOP_TRANS / ROT / BOTH; JP_STOP_NONE (or 0) = off */
  int32_t stop_natom;    /* ixcend(nstpcn): atoms 1..stop_natom; 0 = the leading atoms that
                            share atom 1's molecule id (all atoms without molecule ids) */
  /* CAL15M (cmmdo.f90:27-74): JP_CAL15M_ZD (zero-dipole, the default), JP_CAL15M_ATOM
   * (atom cut-off, enear_ACT_*: E = qi qj / r and the LJ term for r <= CUTLEN, no self or
   * excess term) or JP_CAL15M_CMM (cell multipole method, BOUNDA= NO only: exact Coulomb
   * and LJ between atoms of neighbouring level-1 cells, LJ out to CUTLEN from the cells
   * within CUTLEN, and the far field of up to 5 cell levels by multipoles). */
  int32_t cal15m;
  /* BOUNDA (inpmd.f90:72): JP_BOUND_PBC (the box of jp_system) or JP_BOUND_NONE (no
   * boundary, the *_CB variants: no minimum image; the box of jp_system is ignored). */
  int32_t bounda;
  int32_t cmm_levels;    /* CELLVL: cell levels of the CMM (raised to fit the system, <= 5) */
  double cmm_cell;       /* CELSIZ: edge of a level-1 CMM cell (Angstrom) */
  int32_t cmm_update;    /* CMMUPD: far-field interval (steps); UPDATE must be a multiple */
  /* Block-shape tuning at jp_create (no md.inp keyword; the counterpart of md_run's
   * SIMD_check autotuning of its vector length): 1 (default) = build each replica's list
   * with JP_TUNE_CANDIDATES column grids and keep the one whose list has the fewest
   * pair records (see jp_tile_shape); 0 = near-cubic 32-atom blocks for every replica. */
  int32_t tune_blocks;
} jp_params;

#define JP_TUNE_CANDIDATES 5   /* column-edge factors 0.84, 0.92, 1, 1.09, 1.19 */

enum { JP_ALSD_NONE = 0, JP_ALSD_LMD = 1, JP_ALSD_LMD2 = 2 };
/* GEPSME= AND / OR / XOR (inpinp.f90:44-54, n_matrix inpcls.f90:298-325): partial McMD.
 * With jp_system.cluster set, every term belongs to class 1 or 2 by the regions of its atoms
 * (n_matrix of the region pair: AND -- both atoms in A, or both in B; OR -- both in A, or one
 * in A and one in B, or (without B) at least one in A; XOR -- one in A and one in B, or
 * (without B) exactly one in A); bonded terms that SCALET leaves unscaled are class 2.  The
 * class-1 forces are scaled and the class-2 forces are not (verlet.f90:118-142,
 * verlethe.f90:170-238 with nfrg = 2): by the McMD weight of the class-1 potential energy
 * (METHOD= GE) or by SETTEM/PSETMP (PSETMP > 0, any other METHOD).  Without GE or PSETMP
 * md_run integrates the class-2 forces alone, so that combination is refused.  Replicas
 * without cluster atoms run plain McMD / pseudo temperature on their whole energy.  Not with
 * CAL15M= CMM or jp_minimize. */
enum { JP_GEPS_AND = 3, JP_GEPS_OR = 4, JP_GEPS_XOR = 5 };
enum { JP_SCALE_BOND = 1, JP_SCALE_ANGLE = 2, JP_SCALE_TORS = 4, JP_SCALE_IMPR = 8 };
enum { JP_STOP_TRANS = 1, JP_STOP_ROT = 2, JP_STOP_BOTH = 3, JP_STOP_NONE = 4 };   /* STOPCE */
enum { JP_CAL15M_CMM = 1, JP_CAL15M_ATOM = 2, JP_CAL15M_ZD = 4 };                  /* CAL15M */
enum { JP_BOUND_NONE = 0, JP_BOUND_PBC = 1 };                                       /* BOUNDA */

typedef struct jp_ctx jp_ctx;

/* Fill *prm with md_run's defaults (inpmd.f90:120-160, main.f90:134-174). */
void jp_default_params(jp_params *prm);

/* Set-up after incel (md.f90:82): copies topology, derives the ZD excess list, dself and
 * 1-4 pairs (incel.f90:627-689, :755-787, :1084-1087), drops SHAKE-constrained bonds and
 * angles (setshk.f90 reabnd/reaang), builds the first pair list (celprp).
 * `sys` points at nrep replica systems; all replicas share `prm`. */
int jp_create(const jp_system *sys, int32_t nrep, const jp_params *prm, jp_ctx **out);

/* celprp(iprint,ilflag,ier) (md.f90:657, :888, :1059, :1138): rebuild cells and the pair
 * list from the current device coordinates.  replica = -1 rebuilds all. */
int jp_rebuild_cells(jp_ctx *ctx, int32_t replica);

/* dnergy(eneval, enevcc) (verlet.f90:63, verlethe.f90:103, staver.f90:41).
 * If cord != NULL it replaces the replica's coordinates first (the pair list is NOT
 * rebuilt; call jp_rebuild_cells for a list at these coordinates).  Outputs are nullable:
 * eneval[JP_MAXENE], grad[natom][3] (dE/dx, kcal/mol/Angstrom). */
int jp_energy_grad(jp_ctx *ctx, int32_t replica, const double *cord, double *eneval,
                   double *grad);

/* dnergy's outputs by class (dnergy.f90:2-84: the class totals enevcc(1, 1:nfrg) and the
 * gradient grad(3, N, 1:nfrg) before verlethe combines the classes).  nfrg = 1 for a replica
 * without cluster atoms, 3 for ALSD (classes AA, AB, BB), 2 for GEPSME= AND / OR / XOR
 * (classes 1, 2); *nfrg_out receives it.  ecls[nfrg] (nullable) the class totals, the ZD self
 * term included; grad[nfrg][natom][3] (nullable) each class's unscaled gradient (dE/dx);
 * eneval[JP_MAXENE] (nullable) as jp_energy_grad.  cord as jp_energy_grad.  An ALSD replica
 * is evaluated once per class (the class weights set to one class at a time). */
int jp_energy_grad_cls(jp_ctx *ctx, int32_t replica, const double *cord, double *eneval,
                       double *ecls, double *grad, int32_t *nfrg_out);

/* nsteps iterations of runmd's loop body (md.f90:519-694): one verlet (MICR) or verlethe
 * (CANO/GE) step including SHAKE, then the pair-list rebuild every UPDATE steps.
 * ene_out (nullable) receives [nsteps][nrep][JP_MAXENE] potential energies at time t of
 * each step (the NAMETO .ene values, md.f90:578-601); temp_out (nullable) [nsteps][nrep]
 * the instantaneous temperature of v(t+dt/2). */
int jp_step(jp_ctx *ctx, int32_t nsteps, double *ene_out, double *temp_out);

/* jp_step with the state in host memory, for a driver that keeps cord/vel itself: the
 * coordinates and velocities of all replicas (concatenated in replica order, [natom_total][3];
 * NULL = keep the device's) are copied in, nsteps steps run, and the state after the last
 * step (NULL = not wanted), the energies and the temperatures are copied out, all queued on
 * the context's stream ahead of one synchronisation (a second one only when a SHAKE failure
 * has to be redone).  Equivalent to jp_set_state + jp_step + jp_get_state for every replica
 * (md.f90:544-553 with the state exchange of outrst.f90:56-61).  Pinned host buffers make
 * the copies asynchronous. */
int jp_step_io(jp_ctx *ctx, int32_t nsteps, const double *cord_in, const double *vel_in,
               double *cord_out, double *vel_out, double *ene_out, double *temp_out);

/* shake_PB(r1, r2, iprint, ier) (verlet.f90:196): constrain r1 against reference r2,
 * both [natom][3] host arrays of one replica.  Test hook. */
int jp_shake(jp_ctx *ctx, int32_t replica, double *r1, const double *r2);

/* Coordinates/velocities of one replica for restart and monitor output
 * (outrst.f90:56-61, monmd.f90).  Any pointer may be NULL. */
int jp_get_state(jp_ctx *ctx, int32_t replica, double *cord, double *vel);
int jp_set_state(jp_ctx *ctx, int32_t replica, const double *cord, const double *vel);

/* ALSD state of one replica: lam2 = {lambda, lambda velocity}; ecls (nullable) = the
 * energies of classes AA, AB, BB (unscaled) at the last force evaluation. */
int jp_get_lambda(jp_ctx *ctx, int32_t replica, double *lam2, double *ecls);
int jp_set_lambda(jp_ctx *ctx, int32_t replica, double lambda, double lambda_v);

/* Number of pair interactions within the cut-off evaluated at the last force call
 * (counts r <= rc among listed pairs, one per unordered pair), per replica. */
int jp_pair_count(jp_ctx *ctx, int32_t replica, int64_t *count);

/* Timing.  jp_set_timing(ctx, 1) makes jp_step launch its kernels directly (no CUDA graph)
 * with CUDA events around each phase; 0 (default) replays one captured graph per step.
 * jp_last_timing returns the device time of the last jp_step call (events on the
 * context's stream around all of its kernels) and, in timing mode, the summed time of each
 * phase: [0] pair kernel, [1] bonded, [2] integrate+SHAKE, [3] list rebuild, plus
 * launches[0..3] = number of launches timed per phase (nullable arrays). */
int jp_set_timing(jp_ctx *ctx, int enable);

/* Caps the integration kernel's grid at `blocks` (0 = the co-resident maximum, the default).
 * A step whose integration lanes exceed the grid runs the grid-stride form, with the unit
 * state in the atom arrays between phases, as large systems do.  Test and tuning hook. */
int jp_set_grid_limit(jp_ctx *ctx, int32_t blocks);

/* Bound of every grid-barrier wait inside the cooperative integration kernel, in SM clock
 * cycles (0 = the default, 2e9: about one second).  A wait that runs out makes the kernel
 * record the timeout and every block return at its next barrier; the step then returns
 * JP_E_TIMEOUT with the barrier, sums and accumulators cleared, so the context stays usable
 * after jp_set_state.  No counterpart in the reference (md_run has no device waits). */
int jp_set_wait_limit(jp_ctx *ctx, int64_t cycles);

/* The block shape jp_create chose for `replica`: the column-edge factor kept (1 = columns of
 * edge (32/density)^(1/3)) and, per candidate, the pair records its list needed
 * (tiles[JP_TUNE_CANDIDATES], -1 when tuning was off).  md_run's counterpart is the
 * vector length SIMD_check.f90 picks and prints. */
int jp_tile_shape(jp_ctx *ctx, int32_t replica, double *column_scale, int64_t *tiles);
int jp_last_timing(jp_ctx *ctx, double *total_ms, double *phase_ms4, int32_t *launches4);

/* Kernel launches per jp_step step (excluding list rebuilds) and per list rebuild. */
int jp_launch_counts(jp_ctx *ctx, int32_t *per_step, int32_t *per_rebuild);

/* Pair-list statistics of the current list, all replicas: pair records (the pair kernels'
 * work units: half a block, 16 i atoms, with 32 j entries: 512 pair slots), pair slots set
 * in their masks (pairs
 * within rc+1.5 at the last rebuild, exclusions removed), and the number of atoms padded
 * into blocks. */
int jp_list_stats(jp_ctx *ctx, int64_t *ntiles, int64_t *npairs_listed, int64_t *nslots);

/* FP32 FMA throughput of `device` in TFLOP/s (best of 5 timed FMA-chain launches): the
 * peak the pair kernel's FP32 arithmetic is measured against. */
int jp_calibrate_fp32(int32_t device, double *tflops);

/* McMD iteration support (GEprep, src_GEprep/distrib_MULT.f90:60-445).
 * jp_ge_hist_setup: from now on every MD step adds the potential energy E(t) of `replica`
 * (-1 = all) to an energy histogram of nbin + 2 nbor bins of width (emax-emin)/nbin starting
 * nbor bins below emin (distrib_MULT's binning, including its bin-index truncation);
 * nbin + 2 nbor <= JP_GE_MAX_BINS; nbin = 0 switches it off.  Counts start at zero.
 * jp_ge_hist_get: the counts [nbin + 2 nbor] as doubles; clear != 0 zeroes them. */
int jp_ge_hist_setup(jp_ctx *ctx, int32_t replica, double emin, double emax, int32_t nbin,
                     int32_t nbor);
int jp_ge_hist_get(jp_ctx *ctx, int32_t replica, double *counts, int32_t clear);

/* ALSD weight iteration (GEprep distrib_ALSD.f90:40-120, input_lambda_data :613-669).
 * jp_alsd_hist_setup: from now on every MD step of `replica` (an ALSD replica) adds, at the
 * bin of its lambda (nbin bins of (lmax - lmin) / nbin from lmin, plus nbor border bins each
 * side; a lambda below the first bin's edge is not counted, as int(u + 1) >= 1 decides in
 * the reference), one count and the lambda derivative of its cluster energy, 2 lambda E_AA +
 * E_AB (LMD) or E_AA + E_AB / (2 sqrt(lambda)) (LMD2), E_AA and E_AB the class energies of
 * the step; with ne > 0 also one count and that derivative at the (E, lambda) bin, E the
 * total potential energy on ne bins of [emin, emax] (outside: not counted).  nbin + 2 nbor
 * <= JP_ALSD_MAX_LBINS, ne <= JP_ALSD_MAX_EBINS; nbin = 0 switches it off.  A step redone
 * after a SHAKE failure counts each of its accepted sub-steps.
 * jp_alsd_hist_get: counts and derivative sums [nbin + 2 nbor], and (nullable) the (E, lambda)
 * counts and sums [ne][nbin + 2 nbor]; clear != 0 zeroes them. */
#define JP_ALSD_MAX_LBINS 64
#define JP_ALSD_MAX_EBINS 256
int jp_alsd_hist_setup(jp_ctx *ctx, int32_t replica, double lmin, double lmax, int32_t nbin,
                       int32_t nbor, double emin, double emax, int32_t ne);
int jp_alsd_hist_get(jp_ctx *ctx, int32_t replica, double *counts, double *dedl, double *counts2,
                     double *dedl2, int32_t clear);

/* The ALSD weight of `replica` from a network instead of its polynomial in lambda: the
 * lambda force's weight term R T0 P(lambda) (verlethe.f90:289-320) takes P = net(x)[0] with
 * x = ((E - emin) / (emax - emin), lambda), E the step's total potential energy, params
 * jp_mlp_nparam(2, 2) floats (output 1, the network's d lnP/dE, is not applied: the
 * reference's ALSD has no weight in E); outside [celw, ceup] in lambda the linear walls are
 * added as before.  params NULL goes back to the polynomial.  METHOD= GE ALSD replicas only;
 * the next jp_step re-captures its step graph.  No counterpart in the reference. */
int jp_alsd_set_mlp(jp_ctx *ctx, int32_t replica, const float *params, double emin, double emax);

/* Replace the McMD weight of `replica` (the .nf read by inmcmd.f90) for the following steps;
 * nwindow <= JP_GE_MAX_WINDOWS, ndeg <= JP_GE_MAX_DEG.  METHOD= GE contexts only. */
int jp_ge_set(jp_ctx *ctx, int32_t replica, const jp_ge *ge);

/* Host only.  lstsquare_final.f90: weighted least-squares fit of Y(X) by `nwindow`
 * polynomials of degree `ndim` on equal windows of [minv, maxv] (X ascending), continuous in
 * value and slope; coe[nwindow][ndim+1], low/high[nwindow] out; resid[2] (nullable) the
 * weighted residual error and its spread (Resierr, Resierr2). */
int jp_lstsq_windows(int32_t nwindow, int32_t ndat, int32_t ndim, double minv, double maxv,
                     const double *X, const double *Y, const double *wei, double *coe,
                     double *low, double *high, double *resid);

/* Host only.  distrib_MULT.f90:286-445: from a histogram hist[nbin + 2 nbor] sampled with the
 * weight `old`, the differential density of states d lnN/dE = d lnP/dE + (d lnN/dE of old),
 * fitted on [next_emin, next_emax]; the new weight goes to `out`, whose coefficient arrays
 * are the caller's coef[nwindow][ndeg+1], low/high[nwindow]; resid[2] nullable.  Run
 * weights (fw) and flatness acceleration of GEprep are not supported (all weights 1). */
int jp_ge_fit(const double *hist, const jp_ge_fit_params *fp, const jp_ge *old, double *coef,
              double *low, double *high, jp_ge *out, double *resid);

/* Host only.  The fit data of jp_ge_fit (distrib_MULT.f90:322-420): points x (reduced energy
 * of the next range), y = d lnN/dE and weights w, each of capacity nbin + 2 nbor; *ndat out. */
int jp_ge_dlnn(const double *hist, const jp_ge_fit_params *fp, const jp_ge *old, double *x,
               double *y, double *w, int32_t *ndat);

/* Weight surrogate network: nin -> 64 -> 64 -> nout (tanh), FP32, nin, nout <= 2.  It stands
 * in for the polynomial of jp_ge_fit (nin = nout = 1: reduced energy -> d lnN/dE; ALSD:
 * (E, lambda) -> its two derivatives).  Parameters are one flat float vector of
 * jp_mlp_nparam(nin, nout) entries (layout in csrc/jp_mlp.cuh).
 * jp_mlp_init: Glorot-uniform weights from `seed`, input/target normalisation from the data
 *   of each of nnet networks (samples off[k]..off[k+1]-1 of x[][nin], y[][nout]).
 * jp_mlp_train: `epochs` full-batch Adam steps (learning rate lr) of all nnet networks at once
 *   on `device`, one CUDA block per network, minimising sum w (net - y)^2 / sum w in
 *   normalised units; params in/out [nnet][np]; loss[nnet] at the final parameters;
 *   grad[nnet][np] (nullable) the gradient there (epochs = 0: at the given parameters).
 * jp_mlp_forward: y[n][nout] of one network at x[n][nin] on `device`. */
#define JP_MLP_HIDDEN 64
#define JP_MLP_MAXIO 2
int32_t jp_mlp_nparam(int32_t nin, int32_t nout);
int jp_mlp_init(int32_t nin, int32_t nout, int32_t nnet, const float *x, const float *y,
                const int32_t *off, uint64_t seed, float *params);
int jp_mlp_train(int32_t nin, int32_t nout, int32_t nnet, const float *x, const float *y,
                 const float *w, const int32_t *off, int32_t epochs, float lr, int32_t device,
                 float *params, float *loss, float *grad);
int jp_mlp_forward(int32_t nin, int32_t nout, const float *params, const float *x, int32_t n,
                   int32_t device, float *y);

/* McMD force scaling by the network instead of the polynomial for `replica` (METHOD= GE):
 * inside [celw, ceup] of its current weight d lnN/dE = net(x), x the reduced energy;
 * outside, alphalw / alphaup as before.  params: jp_mlp_nparam(1, 1) floats, or NULL to go
 * back to the polynomial.  The next jp_step re-captures its step graph. */
int jp_ge_set_mlp(jp_ctx *ctx, int32_t replica, const float *params);

const char *jp_strerror(int code);
void jp_destroy(jp_ctx *ctx);

/* Energy minimisation (EXE> MIN, mini.f90 runmin -> steep.f90 steep/linsrd): steepest
 * descent with an adaptive step length.  Each iteration moves every atom along
 * -grad/|grad| (the whole replica's gradient normalised) by the step length, applies SHAKE
 * to the moved positions when the context has SHAKE groups, evaluates dnergy, and
 * multiplies the step length by `up` when the energy fell, else by `down`; the move is kept
 * either way.  It stops when the RMS gradient sqrt(sum |g|^2 / natom) <= convgr (checked
 * before each move), after max_loop iterations, when the step length falls below 1e-10 A
 * per degree of freedom (JP_E_MIN_STEP) or when SHAKE fails.  The pair list is rebuilt
 * every `update` iterations and once at the end.  METHOD= CONJ is not built. */
enum { JP_MIN_STEEP = 1, JP_MIN_CONJ = 2 };
typedef struct jp_min_params {
  int32_t method;        /* JP_MIN_STEEP (METHOD= STEE) or JP_MIN_CONJ (METHOD= CONJ) */
  int32_t max_loop;      /* LOOPLI: iterations (force evaluations after the first), >= 1 */
  int32_t update;        /* UPDATE: list rebuild interval in iterations (default 10) */
  double convgr;         /* CONVGR: RMS gradient threshold, kcal/mol/A (default 0.1) */
  double step0;          /* ISTEPL: initial step length per atom, A (default 0.01); the
                            step length starts at step0 * sqrt(natom) */
  double up, down;       /* STEE step-length factors (md_run defaults 1.2 and 0.6) */
  double line_conv;      /* CONJ: a line search ends at |g.d| <= line_conv |g.d|_start (0.1) */
  int32_t line_max;      /* CONJ: at most line_max evaluations per line search (10) */
} jp_min_params;

void jp_default_min_params(jp_min_params *p);

/* METHOD= CONJ (conj.f90): conjugate gradients with Powell's restarts (mksrdc, a steepest-
 * descent direction whenever a direction is not downhill) and a line search that doubles
 * the step until the directional derivative changes sign, then takes secant steps (linsrc);
 * the search ends on line_conv or line_max, the minimisation on convgr or max_loop.  The
 * reference refuses SHAKE here, and so does this call (JP_E_INVALID).  The iteration runs
 * on the host over device force evaluations, one replica after the other.
 *
 * STEE minimises every replica of the context at once, each with its own step length and
 * stop condition (md_run minimises one system; replicas here are independent).  Per replica
 * (arrays of nrep, each may be NULL): iters = iterations done, eneval[JP_MAXENE] = the
 * energies of the last evaluation, rmsf = its RMS gradient, state = 0 still running at
 * max_loop, 1 converged, 2 step length too small.  Returns JP_OK, JP_E_MIN_STEP if any
 * replica ended with state 2, or the SHAKE codes (a SHAKE failure stops every replica).
 * Velocities are left as they were. */
int jp_minimize(jp_ctx *ctx, const jp_min_params *mp, int32_t *iters, double *eneval,
                double *rmsf, int32_t *state);

/* Largest system jp_nonbond_noalloc accepts: its static scratch array holds
 * 32 + 3 * JP_NOALLOC_MAX_ATOMS doubles (384.25 KiB) on each device. */
#define JP_NOALLOC_MAX_ATOMS 16384

/* No counterpart in the reference: an entry point that allocates no device memory, for
 * callers that cannot allocate.  The ZD + LJ non-bonded part of dnergy -- the pair terms
 * within `cutoff` under the minimum image, the ZD excess of every excluded pair and the ZD
 * self term -- of ONE system given entirely in caller-owned DEVICE buffers, by an
 * O(N^2) all-pairs variant of the FP64 tile kernel (no pair list).
 *   cord[natom][3], charge[natom] (e), atype[natom], c6/c12[ntype][ntype] as in jp_system,
 *   excl_ptr[natom+1] / excl_idx: symmetric exclusion CSR as in jp_system (the ZD excess
 *   is applied to each excluded pair once), index_base 0 or 1 for atype and excl_idx;
 *   box[3] is a HOST array, each edge > 2 * cutoff.
 *   Outputs (device): grad[natom][3] = dE/dx; ene[0] = ZD Coulomb (jp_energy_grad's
 *   JP_E_ELE15 slot, self term included), ene[1] = LJ (JP_E_VDW15).
 *   stream: a cudaStream_t of the current device (NULL = legacy default stream).
 * Work runs on `stream` in the current device's context; the call returns after it has
 * finished.  natom > JP_NOALLOC_MAX_ATOMS returns JP_E_NOALLOC_LIMIT before any device
 * work; an atom or type index out of range returns JP_E_INVALID, a non-finite result
 * JP_E_NONFINITE.
 * Scratch: one static device array shared by every call on a device; each call clears it
 * on `stream` first.  Calls whose device work overlaps (different streams or host threads
 * on one device) race on it and corrupt each other's results: serialise them.  The first
 * call on each device looks up that device's copy of the array (cudaGetSymbolAddress,
 * which may load the library's module); make that first call before any stream capture.
 * Calls no cudaMalloc, cudaFree or other allocating routine. */
int jp_nonbond_noalloc(int32_t natom, const double *cord, const double *charge,
                       const int32_t *atype, int32_t ntype, const double *c6, const double *c12,
                       const int32_t *excl_ptr, const int32_t *excl_idx, int32_t index_base,
                       const double box[3], double cutoff, double dielectric, double *grad,
                       double *ene, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* JPGPU_H */
