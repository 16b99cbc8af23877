// oracle.cpp -- TEST INFRASTRUCTURE ONLY.
//
// CPU/OpenMP FP64 restatement of j_presto md_run's per-step force/integrate path, used as
// the correctness oracle for the CUDA engine (tests, smoke check, bench CPU baseline).
// It is never linked into or called by the product library.
//
// Every routine cites the md_run source (src_md_run/<file>:<line>) it follows.  The
// reference itself cannot be compiled in this environment (no Fortran compiler), and the
// reference ships no tests or golden vectors, so parity against the reference is
// unpinned: the oracle is checked against known-answer vectors derived independently from
// the closed-form formulas (tests/golden/) and against analytic identities
// (finite-difference gradients, energy conservation, constraint satisfaction).
//
// Build: oracle/Makefile -> oracle/liboracle.so (C ABI, see or_* below).

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>
#include <array>
#include <algorithm>
#include <omp.h>

#include "../include/jpgpu.h"

namespace {

// PHYCNS.f90 constants
constexpr double kPi = 3.141592653589793;
constexpr double kGas = 8.31451;         // gascst J/mol/K
constexpr double kJouCal = 4.184;        // joucal
constexpr double kEekcal = 332.06378;    // eekcal
constexpr double kEps = 1.0e-10;         // eps
constexpr double kConvcv = 4.184e-4;     // md.f90:56 fdcvcv

inline double anint(double x) { return std::round(x); }  // Fortran anint: half away from 0

struct Shake {
  int n;            // atoms 2..4
  int a[4];
  double d2[6];     // squared target distances, pair order (1,2),(2,3),(3,1),(4,1),(3,4),(2,4)
};

struct Ctx {
  // ---- topology (0-based) ----
  int n = 0;
  double box[3], invbox[3];
  std::vector<double> mass, imass, chg, chgmod;
  std::vector<int> typ, mol;
  int ntype = 0;
  std::vector<double> c6, c12;
  // restraints (dneres.f90) and the sphere CAP (dnecap.f90); atom indices 0-based
  struct PosRes { int a; double k, ref[3]; };
  struct DistRes { std::vector<int> gi, gj; double lo, up, klo, kup; };
  struct DiheRes { int a[4]; double lo, up, klo, kup; };
  std::vector<PosRes> posres;
  std::vector<DistRes> distres;
  std::vector<DiheRes> diheres;
  std::vector<std::pair<int, int>> cap_groups;   // first, last atom (fechn)
  std::vector<int> cap_atoms;                    // iamcap
  double cap_c[3] = {0, 0, 0}, cap_r = 0, cap_k = 0, cap_ra = 0, cap_ka = 0;
  int cap_shape = 1;                             // capshp: 1 sphere, 2 box, 3 ellipsoid
  int cap_func = 1;                              // iufcap: 1 half-harmonic, 2 half-biquadratic
  double cap_wall[6] = {0}, cap_awall[6] = {0}, cap_ell[3] = {0}, cap_aell[3] = {0};
  // CELRES: each atom's residue (first, last atom), -1 = the atom's own position picks its
  // cell; empty = none
  std::vector<int> res_first, res_last;
  // H-bond type pairs (iyppid = 2) and their 10-12 parameters fynbpp(3:4,:,:); empty = none
  std::vector<int> hbp;
  std::vector<double> c10, c12h;
  std::vector<std::vector<int>> excl;  // sorted partner list per atom
  // cls: ALSD class of the term, 0 = AA, 1 = AB, 2 = BB (n_matrix, inpcls.f90:297-325);
  // 2 for every term without clusters
  struct Bond { int i, j; double k, r0; int cls; };
  struct Angle { int i, j, k; double kf, t0; int cls; };
  struct Tors { int a[4]; double k, nrot, phase; int div; int cls; };
  struct P14 { int i, j; double svdw, sele; int cls; };
  std::vector<Bond> bonds;       // active bonds (SHAKE-constrained removed)
  std::vector<Angle> angles;     // active angles
  std::vector<Tors> tors, imprs;
  std::vector<P14> p14;
  std::vector<std::array<int, 3>> excess;   // (i, j, cls)
  std::vector<Shake> sk2, sk3, sk4;
  int nconstr = 0;
  // ---- ZD constants (incel.f90:29-39, :655-662) ----
  double rc, rlim, rlim2, irlim2, zcore, fcoeff, bcoeff, ccoef, dself;
  // ---- ALSD (inpcls.f90, verlethe.f90:110-165, :240-321, :400-450) ----
  int alsd = 0;
  std::vector<int> inA;               // 1 = atom of the lambda-scaled cluster
  double lam = 1.0, lam_v = 0.0, lam_m = 0.0, lam_im = 0.0;
  bool lam_tc = false, lam_dof = false;
  int ifg_lambda = -1;                // sub-system carrying lambda's degree of freedom
  double ecls[3] = {0.0, 0.0, 0.0};   // class energies (unscaled) of the last force call
  double dself_cls[3] = {0.0, 0.0, 0.0};
  // ---- partial McMD (GEPSME= AND / OR / XOR, nfrg = 2: inpcls.f90:160-183, :298-325;
  // verlet.f90:118-142, verlethe.f90:170-238) ----
  int geps = 0;                       // JP_GEPS_*; 0 = none
  bool split = false;                 // geps with cluster atoms: classes 1 and 2 kept apart
  std::vector<int> icl;               // region code: 0 = A (CLUSTA), 1 = B (CLUSTB), 2 = neither
  unsigned tab1 = 0;                  // bit 3 ca + cb set: n_matrix of the regions = 1
  int pcls(int a, int b) const {      // slot of a term's class: 0 AA / class 1, 1 AB, 2 BB / class 2
    if (split) return ((tab1 >> (3 * icl[a] + icl[b])) & 1u) ? 0 : 2;
    return alsd ? 2 - inA[a] - inA[b] : 2;
  }
  // the class weights can be set to one class at a time (per-class gradients)
  bool fover = false;
  double fo[3] = {1.0, 1.0, 1.0};
  void factors(double* f) const {     // class weights of the gradient
    if (fover) { f[0] = fo[0]; f[1] = fo[1]; f[2] = fo[2]; return; }
    if (alsd == JP_ALSD_LMD) { f[0] = lam * lam; f[1] = lam; f[2] = 1.0; }
    else if (alsd == JP_ALSD_LMD2) { f[0] = lam; f[1] = std::sqrt(lam); f[2] = 1.0; }
    else { f[0] = f[1] = f[2] = 1.0; }
  }
  // ---- run parameters ----
  jp_params prm;
  jp_ge ge{};
  std::vector<double> ge_coef, ge_low, ge_high;
  bool has_ge = false;
  // ---- DOF (md.f90:116-228) ----
  int idnfre = 0;
  int stop_n = 0;               // centre-of-mass stop: atoms 0..stop_n-1 (ixcend(nstpcn))
  bool pbc = true;              // BOUNDA= PBC; false: no boundary (*_CB variants)
  int nsub = 1;
  std::vector<double> nfrmol;   // per sub-system DOF
  // ---- pair list: half list (j listed under i) of pairs within rlim at build ----
  std::vector<std::vector<int>> nb;
  // ---- CMM (CAL15M= CMM): levels 1..nlev (index 0 unused) ----
  bool cmm = false;
  int nlev = 0, idelay = 0, nv[6] = {0, 0, 0, 0, 0, 0};
  double siz[6] = {0, 0, 0, 0, 0, 0};
  std::vector<double> cen[6];            // [3][nv] cell centres per level (celpar_CB)
  std::vector<int> pop[6];               // atoms per cell [nv^3], x fastest
  std::vector<double> pot[6];            // 13 coefficients per cell (celpol)
  std::vector<int> cell1;                // level-1 cell (1-based ix, iy, iz) of each atom
  std::vector<std::vector<char>> nbt;    // per listed pair: 1 = Coulomb + LJ, 0 = LJ only
  std::vector<double> gwk;               // far-field gradient of the last update
  double ecmm = 0.0;                     // its energy (sum over levels)
  bool itwin = true;                     // recompute the far field at the next force call
  bool ext = false;                      // EXTCMM= environment on the level-1 grid
  double ext_c0[3] = {0, 0, 0};          // its grid centre
  std::vector<unsigned char> ext_flag;   // [nv1^3] occupied external cells
  std::vector<double> ext_pot;           // [nv1^3][13]
  double eext = 0.0;                     // its energy at the last force call
  int cmm_err = 0;                       // error of the last rebuild (an atom off the grid)
  // ---- state ----
  std::vector<double> cord, vel, grad;
  long long idloop = 0;
  long long npair_last = 0;
  int nthreads = 1;
};

// minimum image (the *_PB variants); the identity with BOUNDA= NO (*_CB)
inline void minimg(const Ctx& c, double* d) {
  if (!c.pbc) return;
  for (int k = 0; k < 3; ++k) d[k] -= c.box[k] * anint(d[k] * c.invbox[k]);
}

// ---------------------------------------------------------------------------------------
// Pair list: every pair with r^2 <= rlim^2 (minimum image) that is not a 1-2/1-3/1-4
// partner.  Semantics of cutatm_PB (cutoff.f90:166-505: `dd .le. rlim2`) followed by
// the itab14 removal (cutoff.f90:50-96).  A plain cell grid replaces the reference's
// cell hierarchy; the resulting pair SET is the same.
// ---------------------------------------------------------------------------------------
int cmm_rebuild(Ctx& c);

void build_list(Ctx& c) {
  if (c.cmm) {
    c.cmm_err = cmm_rebuild(c);
    return;
  }
  const int n = c.n;
  c.nb.assign(n, {});
  const double* x = c.cord.data();
  int g[3] = {1, 1, 1};
  if (c.pbc)
    for (int k = 0; k < 3; ++k) g[k] = std::max(1, (int)std::floor(c.box[k] / c.rlim));
  const bool brute = !c.pbc || (g[0] < 3 || g[1] < 3 || g[2] < 3);   // all pairs without a box
  std::vector<int> cellof(n), head, next(n, -1);
  if (!brute) {
    head.assign(g[0] * g[1] * g[2], -1);
    for (int i = n - 1; i >= 0; --i) {
      int ci[3];
      for (int k = 0; k < 3; ++k) {
        double w = x[3 * i + k] - c.box[k] * std::floor(x[3 * i + k] * c.invbox[k]);
        int q = (int)(w / c.box[k] * g[k]);
        if (q >= g[k]) q = g[k] - 1;
        if (q < 0) q = 0;
        ci[k] = q;
      }
      int id = (ci[2] * g[1] + ci[1]) * g[0] + ci[0];
      cellof[i] = id;
      next[i] = head[id];
      head[id] = i;
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; ++i) {
    std::vector<int>& L = c.nb[i];
    auto consider = [&](int j) {
      if (j <= i) return;
      double d[3] = {x[3 * i] - x[3 * j], x[3 * i + 1] - x[3 * j + 1], x[3 * i + 2] - x[3 * j + 2]};
      minimg(c, d);
      double dd = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (dd <= c.rlim2) {
        if (std::binary_search(c.excl[i].begin(), c.excl[i].end(), j)) return;
        L.push_back(j);
      }
    };
    if (brute) {
      for (int j = i + 1; j < n; ++j) consider(j);
    } else {
      int id = cellof[i];
      int cx = id % g[0], cy = (id / g[0]) % g[1], cz = id / (g[0] * g[1]);
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int jx = (cx + dx + g[0]) % g[0], jy = (cy + dy + g[1]) % g[1], jz = (cz + dz + g[2]) % g[2];
            for (int j = head[(jz * g[1] + jy) * g[0] + jx]; j >= 0; j = next[j]) consider(j);
          }
      std::sort(L.begin(), L.end());
    }
  }
}

// ---------------------------------------------------------------------------------------
// CMM (CAL15M= CMM, BOUNDA= NO).  Cell geometry of incel.f90:41-57 / mk_c (:1245-1276),
// re-centred on the atoms' centroid at each rebuild (celpar.f90 celpar_CB :36-53); atom
// cells as celpar.f90:90-116; level populations celoth.f90; multipoles celpol.f90 (level 1
// from the atoms, then level to level); near tables neartb.f90 (Coulomb + LJ between atoms
// of neighbouring level-1 cells; LJ only for cells up to idelay apart and dd < rc^2 at the
// rebuild; 1-2/1-3/1-4 partners removed); far field cmmdo.f90:80-170, :181-290 over the
// cell lists of mk_cm (incel.f90:1098-1240).
// ---------------------------------------------------------------------------------------
inline int cidx(const Ctx& c, int l, int ix, int iy, int iz) {   // 1-based indices
  return ((iz - 1) * c.nv[l] + (iy - 1)) * c.nv[l] + (ix - 1);
}

inline int lvup(int i) { return (i + 1) / 2; }

// returns 0 or JP_E_CELL_OVERFLOW (an atom outside the level-1 grid, celpar ier=28)
int cmm_rebuild(Ctx& c) {
  const int n = c.n;
  const double* x = c.cord.data();
  double cord0[3];
  const double rtmp = 1.0 / (double)n;
  for (int k = 0; k < 3; ++k) {
    double sum = 0.0;
    for (int i = 0; i < n; ++i) sum += x[3 * i + k];
    cord0[k] = c.ext ? c.ext_c0[k] : sum * rtmp;   // EXTCMM: the file's centre (celpar.f90:54-70)
  }
  for (int l = 1; l <= c.nlev; ++l) {
    const int m = c.nv[l];
    c.cen[l].assign(3 * m, 0.0);
    const double r = -0.5 * (m + 1);
    for (int i = 1; i <= m; ++i)
      for (int k = 0; k < 3; ++k) c.cen[l][3 * (i - 1) + k] = c.siz[l] * ((double)i + r) + cord0[k];
    c.pop[l].assign((size_t)m * m * m, 0);
    c.pot[l].assign((size_t)13 * m * m * m, 0.0);
  }
  // level-1 cells of the atoms
  const double half = c.siz[1] * 0.5, rr = 1.0 / c.siz[1];
  const double org[3] = {c.cen[1][0] - half, c.cen[1][1] - half, c.cen[1][2] - half};
  const int nv1 = c.nv[1];
  c.cell1.assign(3 * n, 0);
  std::vector<std::vector<int>> members((size_t)nv1 * nv1 * nv1);
  for (int i = 0; i < n; ++i) {
    int m[3];
    double p[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    if (!c.res_first.empty() && c.res_first[i] >= 0) {   // CELRES (celpar.f90:131-153)
      const int k1 = c.res_first[i], k2 = c.res_last[i];
      const double rt = 1.0 / (double)(k2 - k1 + 1);
      for (int k = 0; k < 3; ++k) {
        double sum = 0.0;
        for (int a = k1; a <= k2; ++a) sum += x[3 * a + k];
        p[k] = sum * rt;
      }
    }
    for (int k = 0; k < 3; ++k) {
      m[k] = (int)((p[k] - org[k]) * rr) + 1;   // Fortran int(): toward zero
      if (m[k] < 1 || m[k] > nv1) return JP_E_CELL_OVERFLOW;
      c.cell1[3 * i + k] = m[k];
    }
    const int id = cidx(c, 1, m[0], m[1], m[2]);
    c.pop[1][id] += 1;
    members[id].push_back(i);
  }
  // populations of the upper levels (celoth)
  for (int l = 2; l <= c.nlev; ++l)
    for (int iz = 1; iz <= c.nv[l - 1]; ++iz)
      for (int iy = 1; iy <= c.nv[l - 1]; ++iy)
        for (int ix = 1; ix <= c.nv[l - 1]; ++ix)
          c.pop[l][cidx(c, l, lvup(ix), lvup(iy), lvup(iz))] += c.pop[l - 1][cidx(c, l - 1, ix, iy, iz)];
  // level-1 multipoles about the cell centres, raw charges (celpol.f90:27-80)
  for (int iz = 1; iz <= nv1; ++iz)
    for (int iy = 1; iy <= nv1; ++iy)
      for (int ix = 1; ix <= nv1; ++ix) {
        const int id = cidx(c, 1, ix, iy, iz);
        if (members[id].empty()) continue;
        const double g[3] = {c.cen[1][3 * (ix - 1)], c.cen[1][3 * (iy - 1) + 1], c.cen[1][3 * (iz - 1) + 2]};
        double qz = 0, rx = 0, ry = 0, rz = 0, rxx = 0, ryy = 0, rzz = 0, rxy = 0, ryz = 0, rzx = 0;
        for (int a : members[id]) {
          const double cc = c.chg[a];
          const double dx = x[3 * a] - g[0], dy = x[3 * a + 1] - g[1], dz = x[3 * a + 2] - g[2];
          qz += cc;
          rx += cc * dx; ry += cc * dy; rz += cc * dz;
          const double dxx = dx * dx, dyy = dy * dy, dzz = dz * dz;
          rxx += cc * (2 * dxx - dyy - dzz);
          ryy += cc * (2 * dyy - dzz - dxx);
          rzz += cc * (2 * dzz - dxx - dyy);
          rxy += cc * dx * dy; ryz += cc * dy * dz; rzx += cc * dz * dx;
        }
        double* q = &c.pot[1][(size_t)13 * id];
        const double v[13] = {qz, rx, ry, rz, rxx * 0.5, ryy * 0.5, rzz * 0.5, rxx, ryy, rzz,
                              rxy * 3.0, ryz * 3.0, rzx * 3.0};
        for (int k = 0; k < 13; ++k) q[k] = v[k];
      }
  // level l-1 -> l, children in celpol's order (x fastest), shifted to the parent centre
  for (int l = 2; l <= c.nlev; ++l)
    for (int iz = 1; iz <= c.nv[l]; ++iz)
      for (int iy = 1; iy <= c.nv[l]; ++iy)
        for (int ix = 1; ix <= c.nv[l]; ++ix) {
          const int id = cidx(c, l, ix, iy, iz);
          if (c.pop[l][id] == 0) continue;
          double qz = 0, rx = 0, ry = 0, rz = 0, rxx = 0, ryy = 0, rzz = 0, rxy = 0, ryz = 0, rzx = 0;
          for (int jj = 0; jj < 8; ++jj) {
            const int mx = 2 * ix - 1 + (jj & 1), my = 2 * iy - 1 + ((jj >> 1) & 1), mz = 2 * iz - 1 + ((jj >> 2) & 1);
            const int cid = cidx(c, l - 1, mx, my, mz);
            if (c.pop[l - 1][cid] == 0) continue;
            const double* p = &c.pot[l - 1][(size_t)13 * cid];
            const double qq = p[0];
            qz += qq;
            const double xx = c.cen[l - 1][3 * (mx - 1)] - c.cen[l][3 * (ix - 1)];
            const double yy = c.cen[l - 1][3 * (my - 1) + 1] - c.cen[l][3 * (iy - 1) + 1];
            const double zz = c.cen[l - 1][3 * (mz - 1) + 2] - c.cen[l][3 * (iz - 1) + 2];
            const double ax = p[1], ay = p[2], az = p[3];
            rx += ax + qq * xx; ry += ay + qq * yy; rz += az + qq * zz;
            const double dxx = xx * xx, dyy = yy * yy, dzz = zz * zz;
            const double xax = xx * ax, yay = yy * ay, zaz = zz * az;
            rxx += p[4] + 2 * xax - yay - zaz + qq * (dxx - 0.5 * (dyy + dzz));
            ryy += p[5] + 2 * yay - zaz - xax + qq * (dyy - 0.5 * (dzz + dxx));
            rzz += p[6] + 2 * zaz - xax - yay + qq * (dzz - 0.5 * (dxx + dyy));
            rxy += p[10] * 0.5 + (yy * ax + xx * ay + xx * yy * qq) * 1.5;
            ryz += p[11] * 0.5 + (zz * ay + yy * az + yy * zz * qq) * 1.5;
            rzx += p[12] * 0.5 + (xx * az + zz * ax + zz * xx * qq) * 1.5;
          }
          double* q = &c.pot[l][(size_t)13 * id];
          const double v[13] = {qz, rx, ry, rz, rxx, ryy, rzz, rxx * 2.0, ryy * 2.0, rzz * 2.0,
                                rxy * 2.0, ryz * 2.0, rzx * 2.0};
          for (int k = 0; k < 13; ++k) q[k] = v[k];
        }
  // near tables (neartb): all pairs of neighbouring cells, LJ-only pairs out to idelay cells
  c.nb.assign(n, {});
  c.nbt.assign(n, {});
  const double rc2 = c.rc * c.rc;
#pragma omp parallel for schedule(dynamic, 32)
  for (int i = 0; i < n; ++i) {
    for (int j = i + 1; j < n; ++j) {
      int cheb = 0;
      for (int k = 0; k < 3; ++k) cheb = std::max(cheb, std::abs(c.cell1[3 * i + k] - c.cell1[3 * j + k]));
      char kind;
      if (cheb <= 1) {
        kind = 1;
      } else if (c.idelay > 1 && cheb <= c.idelay) {
        const double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
        if (!(dx * dx + dy * dy + dz * dz < rc2)) continue;
        kind = 0;
      } else {
        continue;
      }
      if (std::binary_search(c.excl[i].begin(), c.excl[i].end(), j)) continue;
      c.nb[i].push_back(j);
      c.nbt[i].push_back(kind);
    }
  }
  return 0;
}

// external environment (enear_extCMM.f90:2-174): each atom against the occupied external
// cells among its level-1 cell and the 26 around it (clipped to the grid); within 1.5 cell
// sizes of a cell centre the expansion is taken on that sphere and blended inward
// (:58-125), beyond it the plain expansion (:126-160).  Returns the energy (times 0.5, as
// md_run adds it), gradient added to grad.
double cmm_ext(Ctx& c, const double* x, double* grad) {
  const int nv1 = c.nv[1];
  const double RR = 1.5 * c.siz[1], RR2 = RR * RR, RR_2 = 3.0 * c.siz[1];
  const double iRR = 1.0 / RR, iRR3 = iRR * iRR * iRR, iRR5 = iRR3 * iRR * iRR;
  const double i3RR5 = 3.0 * iRR5, i5RR7 = 5.0 * iRR5 * iRR * iRR;
  double etot = 0.0;
  for (int i = 0; i < c.n; ++i) {
    const int mx = c.cell1[3 * i], my = c.cell1[3 * i + 1], mz = c.cell1[3 * i + 2];
    const double q2 = c.ccoef * c.chg[i];
    for (int jz = std::max(1, mz - 1); jz <= std::min(nv1, mz + 1); ++jz)
      for (int jy = std::max(1, my - 1); jy <= std::min(nv1, my + 1); ++jy)
        for (int jx = std::max(1, mx - 1); jx <= std::min(nv1, mx + 1); ++jx) {
          const int id = cidx(c, 1, jx, jy, jz);
          if (!c.ext_flag[id]) continue;
          const double* q = &c.ext_pot[(size_t)13 * id];
          double dx = x[3 * i] - c.cen[1][3 * (jx - 1)];
          double dy = x[3 * i + 1] - c.cen[1][3 * (jy - 1) + 1];
          double dz = x[3 * i + 2] - c.cen[1][3 * (jz - 1) + 2];
          const double dd2 = dx * dx + dy * dy + dz * dz;
          double e, f[3];
          if (dd2 < RR2) {
            const double scal = std::sqrt(RR2 / dd2);
            dx *= scal; dy *= scal; dz *= scal;
            const double aa1 = q[1] * dx + q[2] * dy + q[3] * dz;
            const double aa2 = q[4] * dx * dx + q[5] * dy * dy + q[6] * dz * dz + q[10] * dx * dy +
                               q[11] * dy * dz + q[12] * dz * dx;
            const double e0 = q[0] * iRR + aa1 * iRR3 + aa2 * iRR5;
            const double c4 = aa1 * i3RR5 + aa2 * i5RR7;
            f[0] = -(q[0] * dx - q[1]) * iRR3 + (q[7] * dx + q[10] * dy + q[12] * dz) * iRR5 - c4 * dx;
            f[1] = -(q[0] * dy - q[2]) * iRR3 + (q[10] * dx + q[8] * dy + q[11] * dz) * iRR5 - c4 * dy;
            f[2] = -(q[0] * dz - q[3]) * iRR3 + (q[12] * dx + q[11] * dy + q[9] * dz) * iRR5 - c4 * dz;
            const double fn = std::sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
            const double r = std::sqrt(dd2), b = fn * r;
            const double sf = r * iRR3 * (6.0 * e0 * (r - RR) + b * (3.0 * r - RR_2)) / fn;
            for (int k = 0; k < 3; ++k) f[k] *= sf;
            const double t = r * iRR;
            e = (2.0 * e0 + b) * t * t * t - (3.0 * e0 + b) * t * t + 2.0 * e0;
          } else {
            const double d2i = 1.0 / dd2, di = std::sqrt(d2i), d3i = di * d2i, d5i = d3i * d2i;
            const double d7i = d5i * d2i;
            const double aa1 = q[1] * dx + q[2] * dy + q[3] * dz;
            const double aa2 = q[4] * dx * dx + q[5] * dy * dy + q[6] * dz * dz + q[10] * dx * dy +
                               q[11] * dy * dz + q[12] * dz * dx;
            e = q[0] * di + aa1 * d3i + aa2 * d5i;
            const double c4 = aa1 * 3.0 * d5i + aa2 * 5.0 * d7i;
            f[0] = -(q[0] * dx - q[1]) * d3i + (q[7] * dx + q[10] * dy + q[12] * dz) * d5i - c4 * dx;
            f[1] = -(q[0] * dy - q[2]) * d3i + (q[10] * dx + q[8] * dy + q[11] * dz) * d5i - c4 * dy;
            f[2] = -(q[0] * dz - q[3]) * d3i + (q[12] * dx + q[11] * dy + q[9] * dz) * d5i - c4 * dz;
          }
          etot += e * q2;
          for (int k = 0; k < 3; ++k) grad[3 * i + k] += f[k] * q2;
        }
  }
  return 0.5 * etot;
}

// far field of every atom (cmmdo.f90:85-160, compute_particle_multipole :181-290) into
// c.gwk (gradient) and c.ecmm (energy), from the multipoles of the last rebuild
void cmm_far(Ctx& c, const double* x) {
  const int n = c.n;
  c.gwk.assign(3 * (size_t)n, 0.0);
  double ecmm[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < n; ++i) {
    int a[3] = {c.cell1[3 * i], c.cell1[3 * i + 1], c.cell1[3 * i + 2]};
    double gx = 0, gy = 0, gz = 0;
    for (int l = 1; l <= c.nlev; ++l) {
      if (l > 1)
        for (int k = 0; k < 3; ++k) a[k] = lvup(a[k]);
      const int m = c.nv[l];
      int lo[3], hi[3], nlo[3], nhi[3];
      for (int k = 0; k < 3; ++k) {
        nlo[k] = std::max(1, a[k] - 1);
        nhi[k] = std::min(m, a[k] + 1);
        if (l < c.nlev) {   // children of the parent's neighbours (mk_cm)
          const int p = lvup(a[k]), m1 = c.nv[l + 1];
          lo[k] = std::max(1, p - 1) * 2 - 1;
          hi[k] = std::min(m1, p + 1) * 2;
        } else {            // the top level: every cell
          lo[k] = 1;
          hi[k] = m;
        }
      }
      double e = 0.0;
      for (int kz = lo[2]; kz <= hi[2]; ++kz)
        for (int ky = lo[1]; ky <= hi[1]; ++ky)
          for (int kx = lo[0]; kx <= hi[0]; ++kx) {
            if (kx >= nlo[0] && kx <= nhi[0] && ky >= nlo[1] && ky <= nhi[1] && kz >= nlo[2] && kz <= nhi[2])
              continue;
            const int id = cidx(c, l, kx, ky, kz);
            if (c.pop[l][id] == 0) continue;
            const double* q = &c.pot[l][(size_t)13 * id];
            const double dx = x[3 * i] - c.cen[l][3 * (kx - 1)];
            const double dy = x[3 * i + 1] - c.cen[l][3 * (ky - 1) + 1];
            const double dz = x[3 * i + 2] - c.cen[l][3 * (kz - 1) + 2];
            const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
            const double dd2i = 1.0 / (dx2 + dy2 + dz2);
            const double ddi = std::sqrt(dd2i);
            const double dd3i = ddi * dd2i, dd5i = dd3i * dd2i;
            const double dxy = dx * dy, dyz = dy * dz, dzx = dz * dx;
            const double aa1 = q[1] * dx + q[2] * dy + q[3] * dz;
            const double aa2 = q[4] * dx2 + q[5] * dy2 + q[6] * dz2 + q[10] * dxy + q[11] * dyz + q[12] * dzx;
            e += q[0] * ddi + aa1 * dd3i + aa2 * dd5i;
            const double bbx = (q[0] * dx - q[1]) * dd3i, bby = (q[0] * dy - q[2]) * dd3i,
                         bbz = (q[0] * dz - q[3]) * dd3i;
            const double c2x = q[7] * dx + q[10] * dy + q[12] * dz;
            const double c2y = q[10] * dx + q[8] * dy + q[11] * dz;
            const double c2z = q[12] * dx + q[11] * dy + q[9] * dz;
            const double cc4 = aa1 * 3.0 + aa2 * dd2i * 5.0;
            gx += -bbx + (c2x - cc4 * dx) * dd5i;
            gy += -bby + (c2y - cc4 * dy) * dd5i;
            gz += -bbz + (c2z - cc4 * dz) * dd5i;
          }
      ecmm[l] += c.ccoef * c.chg[i] * e;   // chgmod2 = ccoef * charge (inpcls.f90:223)
    }
    const double q2 = c.ccoef * c.chg[i];
    c.gwk[3 * i] = gx * q2;
    c.gwk[3 * i + 1] = gy * q2;
    c.gwk[3 * i + 2] = gz * q2;
  }
  double tot = 0.0;
  for (int l = 1; l <= c.nlev; ++l) tot += ecmm[l] * 0.5;
  c.ecmm = tot;
  c.itwin = false;
}

// ---------------------------------------------------------------------------------------
// dneres_PB / dneres_CB (dneres.f90:2-43): position (dposc :48-101), distance (ddistc
// :107-221) and dihedral (dcdihe :227-378) restraints, then the sphere CAP (dnecap.f90
// :80-122, :428-437; called from dneres_CB only).  Gradients unscaled (grad(:,:,nfrg)),
// energies into enevcc(11..14) and the BB class.
// ---------------------------------------------------------------------------------------
void restraints(Ctx& c, const double* x, double* ene, double* grad) {
  double epos = 0.0;
  for (const auto& r : c.posres) {
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = x[3 * r.a + k] - r.ref[k];
    minimg(c, d);
    epos += r.k * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int k = 0; k < 3; ++k) grad[3 * r.a + k] += r.k * d[k];
  }
  epos *= 0.5;
  double enoe = 0.0;
  for (const auto& r : c.distres) {
    auto sep = [&](int p, int q, double* d) {
      for (int k = 0; k < 3; ++k) d[k] = x[3 * p + k] - x[3 * q + k];
      minimg(c, d);
      return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    };
    const double npair = (double)(r.gi.size() * r.gj.size());
    double tot = 0.0, d[3];
    for (int p : r.gi)
      for (int q : r.gj) {
        const double r2 = sep(p, q, d);
        tot += 1.0 / (r2 * r2 * r2);
      }
    const double rave = std::pow(tot / npair, -1.0 / 6.0);
    double r0 = 1.0, cst = 0.0;
    if (rave > r.up) { r0 = r.up; cst = r.kup; }
    else if (rave < r.lo) { r0 = r.lo; cst = r.klo; }
    const double dr2 = rave * rave - r0 * r0;
    enoe += cst * dr2 * dr2;
    if (rave >= r.lo && rave <= r.up) continue;
    const double coef = 4.0 * cst * dr2 * std::pow(rave, 8) / npair;
    for (int side = 0; side < 2; ++side) {
      const auto& A = side ? r.gj : r.gi;
      const auto& B = side ? r.gi : r.gj;
      for (int p : A) {
        double td[3] = {0, 0, 0};
        for (int q : B) {
          const double r2 = sep(p, q, d);
          const double r8i = 1.0 / (r2 * r2 * r2 * r2);
          for (int k = 0; k < 3; ++k) td[k] += d[k] * r8i;
        }
        for (int k = 0; k < 3; ++k) grad[3 * p + k] += coef * td[k];
      }
    }
  }
  double edhc = 0.0;
  for (const auto& r : c.diheres) {
    const int* ia = r.a;
    double d21[3], d32[3], d43[3];
    for (int k = 0; k < 3; ++k) {
      d21[k] = x[3 * ia[1] + k] - x[3 * ia[0] + k];
      d32[k] = x[3 * ia[2] + k] - x[3 * ia[1] + k];
      d43[k] = x[3 * ia[3] + k] - x[3 * ia[2] + k];
    }
    minimg(c, d21);
    minimg(c, d32);
    minimg(c, d43);
    double p12[3] = {d21[1] * d32[2] - d32[1] * d21[2], d21[2] * d32[0] - d32[2] * d21[0],
                     d21[0] * d32[1] - d32[0] * d21[1]};
    double p23[3] = {d32[1] * d43[2] - d43[1] * d32[2], d32[2] * d43[0] - d43[2] * d32[0],
                     d32[0] * d43[1] - d43[0] * d32[1]};
    double r12 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
    double r23 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
    double r12r23 = std::sqrt(r12 * r23);
    if (r12r23 <= 0.0) continue;
    r12r23 = 1.0 / r12r23;
    const double s1223 = p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2];
    const double cosp = std::max(std::min(s1223 * r12r23, 1.0), -1.0);
    const double p123[3] = {p12[1] * p23[2] - p23[1] * p12[2], p12[2] * p23[0] - p23[2] * p12[0],
                            p12[0] * p23[1] - p23[0] * p12[1]};
    const double s32123 = d32[0] * p123[0] + d32[1] * p123[1] + d32[2] * p123[2];
    double phi = std::acos(cosp);
    if (s32123 < 0.0) phi = 2.0 * kPi - phi;
    double phi0 = 0.0, phi1 = 0.0, cons0 = 0.0, cons1 = 0.0;
    if (phi > r.up) { phi0 = r.up; phi1 = r.lo + 2.0 * kPi; cons0 = r.kup; cons1 = r.klo; }
    else if (phi < r.lo) { phi0 = r.up - 2.0 * kPi; phi1 = r.lo; cons0 = r.kup; cons1 = r.klo; }
    const double dl0 = phi - phi0, dl1 = phi1 - phi;
    double dphi, cst;
    if (dl0 < dl1) { dphi = dl0; cst = cons0; }
    else { dphi = -dl1; cst = cons1; }
    edhc += cst * dphi * dphi;
    if (std::fabs(phi) < kEps || std::fabs(phi - kPi) < kEps) continue;
    const double q12 = s1223 / r12, q23 = s1223 / r23;
    const double wr = -2.0 * cst * dphi / std::sin(phi) * r12r23;
    const double w1 = d21[0] + d32[0], w2 = d21[1] + d32[1], w3 = d21[2] + d32[2];
    double w[9];
    w[0] = d32[2] * p23[1] - d32[1] * p23[2] - q12 * (d32[2] * p12[1] - d32[1] * p12[2]);
    w[1] = d32[0] * p23[2] - d32[2] * p23[0] - q12 * (d32[0] * p12[2] - d32[2] * p12[0]);
    w[2] = d32[1] * p23[0] - d32[0] * p23[1] - q12 * (d32[1] * p12[0] - d32[0] * p12[1]);
    w[3] = -w3 * p23[1] + d43[2] * p12[1] + w2 * p23[2] - d43[1] * p12[2] -
           q12 * (-w3 * p12[1] + w2 * p12[2]) - q23 * (d43[2] * p23[1] - d43[1] * p23[2]);
    w[4] = w3 * p23[0] - d43[2] * p12[0] - w1 * p23[2] + d43[0] * p12[2] -
           q12 * (w3 * p12[0] - w1 * p12[2]) - q23 * (d43[0] * p23[2] - d43[2] * p23[0]);
    w[5] = -w2 * p23[0] + d43[1] * p12[0] + w1 * p23[1] - d43[0] * p12[1] -
           q12 * (-w2 * p12[0] + w1 * p12[1]) - q23 * (d43[1] * p23[0] - d43[0] * p23[1]);
    w[6] = d32[2] * p12[1] - d32[1] * p12[2] - q23 * (d32[2] * p23[1] - d32[1] * p23[2]);
    w[7] = d32[0] * p12[2] - d32[2] * p12[0] - q23 * (d32[0] * p23[2] - d32[2] * p23[0]);
    w[8] = d32[1] * p12[0] - d32[0] * p12[1] - q23 * (d32[1] * p23[0] - d32[0] * p23[1]);
    for (int k = 0; k < 3; ++k) {
      grad[3 * ia[0] + k] += wr * w[k];
      grad[3 * ia[1] + k] += wr * w[3 + k];
      grad[3 * ia[2] + k] -= wr * (w[k] + w[3 + k] + w[6 + k]);
      grad[3 * ia[3] + k] += wr * w[6 + k];
    }
  }
  // CAP (dnecap.f90 iufcap 1): sum of squared overshoots times k, halved at the end
  // (:121, :202, :249); Tcord = centre of mass - fxcbou for groups, Tcod per atom
  double ecap = 0.0;
  auto cap = [&](const double* T, const double* Tbox, double k, double r, const double* wall,
                 const double* ell, double* tg) {
    tg[0] = tg[1] = tg[2] = 0.0;
    if (c.cap_shape == JP_CAP_BOX) {   // capshp 2 (:123-202): walls per coordinate
      for (int d = 0; d < 3; ++d) {
        double dist = 0.0;
        if (Tbox[d] < wall[2 * d]) dist = Tbox[d] - wall[2 * d];
        else if (Tbox[d] > wall[2 * d + 1]) dist = Tbox[d] - wall[2 * d + 1];
        else continue;
        ecap += k * dist * dist;
        tg[d] = dist * k;
      }
      return;
    }
    const double d2 = T[0] * T[0] + T[1] * T[1] + T[2] * T[2];
    if (c.cap_shape == JP_CAP_ELLIPSOID) {   // capshp 3 (:205-246)
      const double s2 = T[0] * T[0] * ell[0] + T[1] * T[1] * ell[1] + T[2] * T[2] * ell[2];
      if (s2 <= 1.0) return;
      const double rt = 1.0 - std::sqrt(1.0 / s2);
      const double dist = std::sqrt(d2) * rt;
      ecap += k * dist * dist;
      for (int d = 0; d < 3; ++d) tg[d] = T[d] * rt * k;
      return;
    }
    if (d2 <= r * r) return;   // capshp 1 (:83-122)
    const double d = std::sqrt(d2), over = d - r;
    ecap += k * over * over;
    for (int m = 0; m < 3; ++m) tg[m] = T[m] * (k * over / d);
  };
  if (c.cap_func == JP_CAP_BIQUADRATIC) {   // iufcap 2 (dnecap.f90:253-281), sphere
    double eg = 0.0, ea = 0.0;
    const double r2 = c.cap_r * c.cap_r, r2a = c.cap_ra * c.cap_ra;
    for (const auto& g : c.cap_groups) {
      double m = 0.0, C[3] = {0, 0, 0};
      for (int a = g.first; a <= g.second; ++a) {
        m += c.mass[a];
        for (int k = 0; k < 3; ++k) C[k] += c.mass[a] * x[3 * a + k];
      }
      for (int k = 0; k < 3; ++k) C[k] = C[k] / m - c.cap_c[k];
      const double dist = C[0] * C[0] + C[1] * C[1] + C[2] * C[2];
      const double d3 = std::max((dist - r2) / r2, 0.0);
      eg += d3 * d3 * r2;
      for (int a = g.first; a <= g.second; ++a)
        for (int k = 0; k < 3; ++k) grad[3 * a + k] += C[k] * c.cap_k * d3 * (c.mass[a] / m);
    }
    for (int a : c.cap_atoms) {
      double T[3];
      for (int k = 0; k < 3; ++k) T[k] = x[3 * a + k] - c.cap_c[k];
      const double dist = T[0] * T[0] + T[1] * T[1] + T[2] * T[2];
      if (dist <= r2a) continue;
      const double d3 = (dist - r2a) / r2a;
      ea += d3 * d3 * r2a;
      for (int k = 0; k < 3; ++k) grad[3 * a + k] += c.cap_ka * d3 * T[k];
    }
    ecap = (eg * c.cap_k + ea * c.cap_ka) * 0.25;
  }
  for (const auto& g : c.cap_groups) {   // centre of mass of each included chain
    if (c.cap_func == JP_CAP_BIQUADRATIC) break;
    double m = 0.0, C[3] = {0, 0, 0}, tg[3];
    for (int a = g.first; a <= g.second; ++a) {
      m += c.mass[a];
      for (int k = 0; k < 3; ++k) C[k] += c.mass[a] * x[3 * a + k];
    }
    for (int k = 0; k < 3; ++k) C[k] = C[k] / m - c.cap_c[k];
    cap(C, C, c.cap_k, c.cap_r, c.cap_wall, c.cap_ell, tg);
    for (int a = g.first; a <= g.second; ++a)   // :428-437, shared by mass
      for (int k = 0; k < 3; ++k) grad[3 * a + k] += tg[k] * (c.mass[a] / m);
  }
  for (int a : c.cap_atoms) {
    if (c.cap_func == JP_CAP_BIQUADRATIC) break;
    double T[3], tg[3];
    for (int k = 0; k < 3; ++k) T[k] = x[3 * a + k] - c.cap_c[k];
    cap(T, x + 3 * a, c.cap_ka, c.cap_ra, c.cap_awall, c.cap_aell, tg);   // box: absolute coordinates
    for (int k = 0; k < 3; ++k) grad[3 * a + k] += tg[k];
  }
  if (c.cap_func != JP_CAP_BIQUADRATIC) ecap *= 0.5;
  ene[JP_E_POSRES] += epos;
  ene[JP_E_DISTRES] += enoe;
  ene[JP_E_DIHERES] += edhc;
  ene[JP_E_CAP] += ecap;
  c.ecls[2] += epos + enoe + edhc + ecap;
}

// ---------------------------------------------------------------------------------------
// dnergy (dnergy.f90:2-84) -> dnergv_PB (dnergv.f90:2-59): bonds, angles, torsions,
// impropers, 1-4, then cmmdo -> enear_ZD_redu_PB (enear.f90, #ZD #REDU #PB lines).
// ene[15] gets enevcc(:,1); grad = dE/dx.
// ---------------------------------------------------------------------------------------
void energy_grad(Ctx& c, const double* x, double* ene, double* grad) {
  const int n = c.n;
  for (int k = 0; k < JP_MAXENE; ++k) ene[k] = 0.0;
  std::fill(grad, grad + 3 * n, 0.0);
  // ALSD: term gradients enter times f[class] (verlethe.f90:116-163: grad(:,:,3) =
  // lambda^2 grad(:,:,1) + lambda grad(:,:,2) + grad(:,:,3)); class energies unscaled
  double f[3];
  c.factors(f);
  double* ec = c.ecls;
  for (int k = 0; k < 3; ++k) ec[k] = c.dself_cls[k];

  // bonds: dnebnd_PB (dnergv.f90:65-122)
  for (const auto& b : c.bonds) {
    double d[3] = {x[3 * b.i] - x[3 * b.j], x[3 * b.i + 1] - x[3 * b.j + 1], x[3 * b.i + 2] - x[3 * b.j + 2]};
    minimg(c, d);
    double r12 = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double dif = r12 - b.r0;
    double coef = b.k * dif;
    ene[JP_E_BOND] += coef * dif;
    ec[b.cls] += coef * dif;
    coef = f[b.cls] * 2.0 * coef / r12;
    for (int k = 0; k < 3; ++k) {
      grad[3 * b.i + k] += coef * d[k];
      grad[3 * b.j + k] -= coef * d[k];
    }
  }
  // angles: dneang_PB (dnergv.f90:128-207)
  for (const auto& a : c.angles) {
    double d12[3], d32[3];
    for (int k = 0; k < 3; ++k) {
      d12[k] = x[3 * a.i + k] - x[3 * a.j + k];
      d32[k] = x[3 * a.k + k] - x[3 * a.j + k];
    }
    minimg(c, d12);
    minimg(c, d32);
    double r12 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
    double r32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
    double r12r32 = std::sqrt(1.0 / (r12 * r32));
    double cost = d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2];
    r12 = 1.0 / r12;
    r32 = 1.0 / r32;
    cost = std::min(cost * r12r32, 1.0);
    cost = std::max(cost, -1.0);
    double theta = std::acos(cost);
    double dif = theta - a.t0;
    double coef = a.kf * dif;
    ene[JP_E_ANGLE] += coef * dif;
    ec[a.cls] += coef * dif;
    double sint = std::max(std::sin(theta), kEps);
    coef = -f[a.cls] * 2.0 * coef / sint;
    double w[6];
    double rt = cost * r12;
    for (int k = 0; k < 3; ++k) w[k] = coef * (d32[k] * r12r32 - d12[k] * rt);
    rt = cost * r32;
    for (int k = 0; k < 3; ++k) w[3 + k] = coef * (d12[k] * r12r32 - d32[k] * rt);
    for (int k = 0; k < 3; ++k) {
      grad[3 * a.i + k] += w[k];
      grad[3 * a.j + k] -= (w[k] + w[3 + k]);
      grad[3 * a.k + k] += w[3 + k];
    }
  }
  // torsions / impropers: dnetor_PB (dnergv.f90:223-434)
  auto tors = [&](const std::vector<Ctx::Tors>& T, int slot) {
    for (const auto& t : T) {
      const int* ia = t.a;
      double d21[3], d32[3], d43[3];
      for (int k = 0; k < 3; ++k) {
        d21[k] = x[3 * ia[1] + k] - x[3 * ia[0] + k];
        d32[k] = x[3 * ia[2] + k] - x[3 * ia[1] + k];
        d43[k] = x[3 * ia[3] + k] - x[3 * ia[2] + k];
      }
      minimg(c, d21);
      minimg(c, d32);
      minimg(c, d43);
      double p12[3] = {d21[1] * d32[2] - d32[1] * d21[2], d21[2] * d32[0] - d32[2] * d21[0],
                       d21[0] * d32[1] - d32[0] * d21[1]};
      double p23[3] = {d32[1] * d43[2] - d43[1] * d32[2], d32[2] * d43[0] - d43[2] * d32[0],
                       d32[0] * d43[1] - d43[0] * d32[1]};
      double r12 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
      double r23 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
      double r12r23 = std::sqrt(r12 * r23);
      if (!(r12r23 > 0.0)) continue;
      r12r23 = 1.0 / r12r23;
      double s1223 = p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2];
      double cosp = s1223 * r12r23;
      if (cosp > 1.0) cosp = 1.0;
      else if (cosp < -1.0) cosp = -1.0;
      double p123[3] = {p12[1] * p23[2] - p23[1] * p12[2], p12[2] * p23[0] - p23[2] * p12[0],
                        p12[0] * p23[1] - p23[0] * p12[1]};
      double s32123 = d32[0] * p123[0] + d32[1] * p123[1] + d32[2] * p123[2];
      double phi = std::acos(cosp);
      if (s32123 < 0.0) phi = 2.0 * kPi - phi;
      double phimod = t.nrot * phi + t.phase;
      double div = 1.0 / (double)t.div;
      ene[slot] += t.k * (1.0 + std::cos(phimod)) * div;
      ec[t.cls] += t.k * (1.0 + std::cos(phimod)) * div;
      double sinp = std::sin(phi);
      int nrot = (int)anint(t.nrot);
      double w0 = 0.0;
      switch (nrot) {
        case 1: w0 = 1.0; break;
        case 2: w0 = 2.0 * cosp; break;
        case 3: w0 = -4.0 * sinp * sinp + 3.0; break;
        case 4: w0 = (-8.0 * sinp * sinp + 4.0) * cosp; break;
        case 5: w0 = (16.0 * sinp * sinp - 20.0) * sinp * sinp + 5.0; break;
        case 6: w0 = cosp * (6.0 + 32.0 * cosp * cosp * (cosp * cosp - 1.0)); break;
        default: w0 = 0.0;
      }
      w0 = f[t.cls] * std::cos(t.phase) * t.nrot * t.k * div * w0 * r12r23;
      double w1 = d21[0] + d32[0], w2 = d21[1] + d32[1], w3 = d21[2] + d32[2];
      double q12 = s1223 / r12, q23 = s1223 / r23;
      double w[9];
      w[0] = d32[2] * p23[1] - d32[1] * p23[2] - q12 * (d32[2] * p12[1] - d32[1] * p12[2]);
      w[1] = d32[0] * p23[2] - d32[2] * p23[0] - q12 * (d32[0] * p12[2] - d32[2] * p12[0]);
      w[2] = d32[1] * p23[0] - d32[0] * p23[1] - q12 * (d32[1] * p12[0] - d32[0] * p12[1]);
      w[3] = -w3 * p23[1] + d43[2] * p12[1] + w2 * p23[2] - d43[1] * p12[2] -
             q12 * (-w3 * p12[1] + w2 * p12[2]) - q23 * (d43[2] * p23[1] - d43[1] * p23[2]);
      w[4] = w3 * p23[0] - d43[2] * p12[0] - w1 * p23[2] + d43[0] * p12[2] -
             q12 * (w3 * p12[0] - w1 * p12[2]) - q23 * (d43[0] * p23[2] - d43[2] * p23[0]);
      w[5] = -w2 * p23[0] + d43[1] * p12[0] + w1 * p23[1] - d43[0] * p12[1] -
             q12 * (-w2 * p12[0] + w1 * p12[1]) - q23 * (d43[1] * p23[0] - d43[0] * p23[1]);
      w[6] = d32[2] * p12[1] - d32[1] * p12[2] - q23 * (d32[2] * p23[1] - d32[1] * p23[2]);
      w[7] = d32[0] * p12[2] - d32[2] * p12[0] - q23 * (d32[0] * p23[2] - d32[2] * p23[0]);
      w[8] = d32[1] * p12[0] - d32[0] * p12[1] - q23 * (d32[1] * p23[0] - d32[0] * p23[1]);
      for (int k = 0; k < 9; ++k) w[k] *= w0;
      for (int k = 0; k < 3; ++k) {
        grad[3 * ia[0] + k] += w[k];
        grad[3 * ia[1] + k] += w[3 + k];
        grad[3 * ia[2] + k] -= (w[k] + w[3 + k] + w[6 + k]);
        grad[3 * ia[3] + k] += w[6 + k];
      }
    }
  };
  tors(c.tors, JP_E_TORS);
  tors(c.imprs, JP_E_IMPR);
  // 1-4 vdW + electrostatics: dne14_PB (dnergv.f90:440-516)
  for (const auto& p : c.p14) {
    double d[3] = {x[3 * p.i] - x[3 * p.j], x[3 * p.i + 1] - x[3 * p.j + 1], x[3 * p.i + 2] - x[3 * p.j + 2]};
    minimg(c, d);
    double r14 = 1.0 / (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double r141 = std::sqrt(r14);
    double r146 = r14 * r14 * r14;
    double r1412 = r146 * r146;
    int ti = c.typ[p.i], tj = c.typ[p.j];
    double co6 = c.c6[ti * c.ntype + tj] * r146;
    double co12 = c.c12[ti * c.ntype + tj] * r1412;
    ene[JP_E_VDW14] += p.svdw * (-co6 + co12);
    ec[p.cls] += p.svdw * (-co6 + co12);
    double coef = r14 * p.svdw * (-2.0 * co12 + co6) * 6.0;
    double w[3] = {coef * d[0], coef * d[1], coef * d[2]};
    coef = p.sele * r141;
    ene[JP_E_ELE14] += coef;
    ec[p.cls] += coef;
    coef = coef * (-r14);
    for (int k = 0; k < 3; ++k) {
      w[k] += coef * d[k];
      grad[3 * p.i + k] += f[p.cls] * w[k];
      grad[3 * p.j + k] -= f[p.cls] * w[k];
    }
  }

  if (f[2] == 1.0) {
    restraints(c, x, ene, grad);
  } else {   // restraint gradients belong to the last class (grad(:,:,nfrg))
    std::vector<double> rg((size_t)3 * n, 0.0);
    restraints(c, x, ene, rg.data());
    for (int k = 0; k < 3 * n; ++k) grad[k] += f[2] * rg[k];
  }

  // ZD + LJ pair loop: enear_ZD_redu_PB (enear.f90:107-257, #ZD #REDU #PB lines),
  // per-thread gradient copies stand in for the OpenMP reduction(+:Tgrad).
  const int nt = c.nthreads;
  std::vector<double> tg((size_t)nt * 3 * n, 0.0);
  double eel = 0.0, evdw = 0.0, ehb = 0.0;
  double ec0 = 0.0, ec1 = 0.0, ec2 = 0.0;
  long long npair = 0;
#pragma omp parallel num_threads(nt) reduction(+ : eel, evdw, ehb, npair, ec0, ec1, ec2)
  {
    double* G = tg.data() + (size_t)omp_get_thread_num() * 3 * n;
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
      const double xi = x[3 * i], yi = x[3 * i + 1], zi = x[3 * i + 2];
      const double chgi = c.chgmod[i];
      const int it1 = c.typ[i];
      double gwx = 0, gwy = 0, gwz = 0;
      for (size_t q = 0; q < c.nb[i].size(); ++q) {
        const int j = c.nb[i][q];
        double d[3] = {xi - x[3 * j], yi - x[3 * j + 1], zi - x[3 * j + 2]};
        minimg(c, d);
        double dd2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        double dd2i = 1.0 / dd2;
        double co = (dd2i - c.irlim2 >= 0.0) ? 1.0 : 0.0;   // sign(0.5,dd2i-irlim2)+0.5
        double coel = co;
        if (c.cmm) {   // enear_CMM: no cut-off; the LJ-only table has no Coulomb term
          co = 1.0;
          coel = c.nbt[i][q] ? 1.0 : 0.0;
        }
        double ddi = std::sqrt(dd2i);
        double dd6i = dd2i * dd2i * dd2i * co;
        double ee = chgi * c.chgmod[j] * coel;
        const double epair = ee * (ddi + c.bcoeff * dd2 - c.zcore);
        eel += epair;
        int it2 = c.typ[j];
        const int tp = it2 * c.ntype + it1;
        double v1, v2, p1;
        if (!c.hbp.empty() && c.hbp[tp]) {
          // the itbhyd pairs (cutoff.f90:98-154): 10-12 instead of 12-6, into ehydcn
          // (enear.f90:415-440, #ZD / #ACT lines)
          const double dd10i = dd2i * dd2i * dd2i * dd2i * dd2i * co;
          v1 = c.c10[tp] * dd10i;
          v2 = c.c12h[tp] * dd10i * dd2i;
          p1 = 10.0;
          ehb += -v1 + v2;
        } else {
          v1 = c.c6[tp] * dd6i;
          v2 = c.c12[tp] * dd6i * dd6i;
          p1 = 6.0;
          evdw += -v1 + v2;
        }
        const int pc = c.pcls(i, j);
        (pc == 0 ? ec0 : pc == 1 ? ec1 : ec2) += epair + (-v1 + v2);
        double cc = f[pc] * (ee * (dd2i * ddi - c.fcoeff) + (-p1 * v1 + 12.0 * v2) * dd2i);
        double fx = d[0] * cc, fy = d[1] * cc, fz = d[2] * cc;
        gwx += fx; gwy += fy; gwz += fz;
        G[3 * j] += fx; G[3 * j + 1] += fy; G[3 * j + 2] += fz;
        npair += (coel > 0.0) ? 1 : 0;
      }
      G[3 * i] -= gwx; G[3 * i + 1] -= gwy; G[3 * i + 2] -= gwz;
    }
  }
  for (int t = 0; t < nt; ++t) {
    const double* G = tg.data() + (size_t)t * 3 * n;
    for (int k = 0; k < 3 * n; ++k) grad[k] += G[k];
  }
  c.npair_last = npair;
  ec[0] += ec0; ec[1] += ec1; ec[2] += ec2;
  // ZD excess of excluded pairs (enear.f90:518-555) and self term (enear.f90:571)
  double eexc = 0.0;
  for (const auto& e : c.excess) {
    int a = e[0], b = e[1];
    double d[3] = {x[3 * a] - x[3 * b], x[3 * a + 1] - x[3 * b + 1], x[3 * a + 2] - x[3 * b + 2]};
    minimg(c, d);
    double dd2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    double cc = c.chgmod[a] * c.chgmod[b];
    eexc += cc * c.bcoeff * dd2;
    ec[e[2]] += cc * c.bcoeff * dd2;
    cc *= f[e[2]] * c.fcoeff;
    for (int k = 0; k < 3; ++k) {
      grad[3 * a + k] += d[k] * cc;
      grad[3 * b + k] -= d[k] * cc;
    }
  }
  if (c.cmm) {   // far field: recomputed when itwin is set, else the last one again
    if (c.itwin) cmm_far(c, x);
    for (int k = 0; k < 3 * n; ++k) grad[k] += c.gwk[k];
    eel += c.ecmm;
    if (c.ext) {   // the external environment, every force call (cmmdo.f90:82)
      c.eext = cmm_ext(c, x, grad);
      eel += c.eext;
    }
  }
  ene[JP_E_VDW15] += evdw;
  ene[JP_E_HBOND] += ehb;
  ene[JP_E_ELE15] += eel + c.dself + eexc;
  double tot = 0.0;
  for (int k = 1; k < JP_MAXENE; ++k) tot += ene[k];
  ene[JP_E_TOTAL] = tot;
}

// ---------------------------------------------------------------------------------------
// SHAKE (shake.f90): shak2e (687-755), shak2i (568-681), shake3 (113-327), shake4 (333-562)
// Returns 0, 1 (not converged) or -2 (singular).
// ---------------------------------------------------------------------------------------
const int kParlis[6][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 0}, {2, 3}, {1, 3}};

int ludeco(double A[6][6], int n, double epsl, int* ip) {  // simulu.f90 ludeco
  for (int k = 0; k < n; ++k) ip[k] = k;
  for (int k = 0; k < n; ++k) {
    int l = k;
    double al = std::fabs(A[ip[l]][k]);
    for (int i = k + 1; i < n; ++i)
      if (std::fabs(A[ip[i]][k]) > al) { l = i; al = std::fabs(A[ip[l]][k]); }
    if (l != k) std::swap(ip[k], ip[l]);
    if (std::fabs(A[ip[k]][k]) < epsl) return -1;
    A[ip[k]][k] = 1.0 / A[ip[k]][k];
    for (int i = k + 1; i < n; ++i) {
      A[ip[i]][k] *= A[ip[k]][k];
      for (int j = k + 1; j < n; ++j) A[ip[i]][j] -= A[ip[i]][k] * A[ip[k]][j];
    }
  }
  return 0;
}

int simulu(double A[6][6], int n, const double* B, double* X) {  // simulu.f90 simulu
  int ip[6];
  if (ludeco(A, n, kEps * kEps * kEps, ip) != 0) return -1;
  for (int i = 0; i < n; ++i) {
    double t = B[ip[i]];
    for (int j = 0; j < i; ++j) t -= A[ip[i]][j] * X[j];
    X[i] = t;
  }
  for (int i = n - 1; i >= 0; --i) {
    double t = X[i];
    for (int j = i + 1; j < n; ++j) t -= A[ip[i]][j] * X[j];
    X[i] = t * A[ip[i]][i];
  }
  return 0;
}

int shake_all(Ctx& c, double* r1, const double* r2) {
  const double tol = c.prm.shake_tol;
  const int maxit = c.prm.shake_maxit;
  int ier = 0;
  auto vec = [&](const double* r, int a, int b, double* d) {
    for (int k = 0; k < 3; ++k) d[k] = r[3 * a + k] - r[3 * b + k];
    minimg(c, d);
  };
  // two-atom groups
  if (!c.sk2.empty()) {
    if (c.prm.shake_method == JP_SHAKE_HBON) {   // shak2e: exact quadratic
      for (const auto& g : c.sk2) {
        int ia = g.a[0], ja = g.a[1];
        double im1 = c.imass[ia], im2 = c.imass[ja];
        double i3 = im1 + im2, i4 = i3 * i3;
        double d1[3], d2[3];
        vec(r1, ja, ia, d1);
        vec(r2, ja, ia, d2);
        double d1d1 = d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2];
        double d1d2 = d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2];
        double d2d2 = d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2];
        double A = i4 * d2d2, B = i3 * d1d2, C = d1d1 - g.d2[0];
        double G = (B - std::sqrt(B * B - C * A)) / A;
        for (int k = 0; k < 3; ++k) {
          r1[3 * ia + k] += im1 * G * d2[k];
          r1[3 * ja + k] -= im2 * G * d2[k];
        }
      }
    } else {                                     // shak2i: iterative
      const int ng = (int)c.sk2.size();
      std::vector<char> ok(ng, 0);
      std::vector<double> d2s(3 * ng);
      for (int q = 0; q < ng; ++q) vec(r2, c.sk2[q].a[0], c.sk2[q].a[1], &d2s[3 * q]);
      bool conv = false;
      for (int it = 0; it < maxit && !conv; ++it) {
        for (int q = 0; q < ng; ++q) {
          const auto& g = c.sk2[q];
          double im1 = c.imass[g.a[0]], im2 = c.imass[g.a[1]];
          double i3 = 0.5 / (im1 + im2);
          double d1[3];
          vec(r1, g.a[0], g.a[1], d1);
          double dif = g.d2[0] - (d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
          double inpro = d1[0] * d2s[3 * q] + d1[1] * d2s[3 * q + 1] + d1[2] * d2s[3 * q + 2];
          double G = (dif * i3) / inpro;
          for (int k = 0; k < 3; ++k) {
            r1[3 * g.a[0] + k] += im1 * G * d2s[3 * q + k];
            r1[3 * g.a[1] + k] -= im2 * G * d2s[3 * q + k];
          }
        }
        int nok = 0;
        for (int q = 0; q < ng; ++q) {
          if (ok[q]) { ++nok; continue; }
          const auto& g = c.sk2[q];
          double d1[3];
          vec(r1, g.a[0], g.a[1], d1);
          double dif = g.d2[0] - (d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
          ok[q] = std::fabs(dif / g.d2[0]) < tol;
          nok += ok[q];
        }
        conv = (nok == ng);
      }
      if (!conv) return 1;
    }
  }
  // three-atom (triangle) groups: shake3 Newton with closed-form 3x3 inverse
  int numerr = 0, notconv = 0;
  for (const auto& g : c.sk3) {
    const int* a = g.a;
    double im[3] = {c.imass[a[0]], c.imass[a[1]], c.imass[a[2]]};
    double cg[3][3] = {{im[0] + im[1], -im[1], -im[0]},
                       {-im[1], im[1] + im[2], -im[2]},
                       {-im[0], -im[2], im[2] + im[0]}};
    double d1[3][3], d2[3][3];
    vec(r1, a[0], a[1], d1[0]); vec(r1, a[1], a[2], d1[1]); vec(r1, a[2], a[0], d1[2]);
    vec(r2, a[0], a[1], d2[0]); vec(r2, a[1], a[2], d2[1]); vec(r2, a[2], a[0], d2[2]);
    double G[6] = {0, 0, 0, 0, 0, 0};
    bool ok = false;
    for (int it = 0; it < maxit; ++it) {
      double B[3];
      for (int q = 0; q < 3; ++q) B[q] = g.d2[q] - (d1[q][0] * d1[q][0] + d1[q][1] * d1[q][1] + d1[q][2] * d1[q][2]);
      if (std::fabs(B[0]) < tol * g.d2[0] && std::fabs(B[1]) < tol * g.d2[1] && std::fabs(B[2]) < tol * g.d2[2]) {
        ok = true;
        for (int k = 0; k < 3; ++k) {
          r1[3 * a[0] + k] += im[0] * (G[3] * d2[0][k] - G[5] * d2[2][k]);
          r1[3 * a[1] + k] += im[1] * (-G[3] * d2[0][k] + G[4] * d2[1][k]);
          r1[3 * a[2] + k] += im[2] * (-G[4] * d2[1][k] + G[5] * d2[2][k]);
        }
        break;
      }
      double gf[3][3];
      for (int ig = 0; ig < 3; ++ig)
        for (int q = 0; q < 3; ++q)
          gf[q][ig] = 2.0 * cg[q][ig] * (d1[q][0] * d2[ig][0] + d1[q][1] * d2[ig][1] + d1[q][2] * d2[ig][2]);
      double deta = gf[0][0] * gf[1][1] * gf[2][2] + gf[0][1] * gf[1][2] * gf[2][0] + gf[0][2] * gf[1][0] * gf[2][1] -
                    gf[0][0] * gf[1][2] * gf[2][1] - gf[0][1] * gf[1][0] * gf[2][2] - gf[0][2] * gf[1][1] * gf[2][0];
      if (deta == 0.0) ++numerr;
      else deta = 1.0 / deta;
      double db[3][3];
      db[0][0] = gf[1][1] * gf[2][2] - gf[1][2] * gf[2][1];
      db[0][1] = gf[2][1] * gf[0][2] - gf[2][2] * gf[0][1];
      db[0][2] = gf[0][1] * gf[1][2] - gf[0][2] * gf[1][1];
      db[1][0] = gf[1][2] * gf[2][0] - gf[1][0] * gf[2][2];
      db[1][1] = gf[2][2] * gf[0][0] - gf[2][0] * gf[0][2];
      db[1][2] = gf[0][2] * gf[1][0] - gf[0][0] * gf[1][2];
      db[2][0] = gf[1][0] * gf[2][1] - gf[1][1] * gf[2][0];
      db[2][1] = gf[2][0] * gf[0][1] - gf[2][1] * gf[0][0];
      db[2][2] = gf[0][0] * gf[1][1] - gf[0][1] * gf[1][0];
      for (int q = 0; q < 3; ++q) G[q] = deta * (db[q][0] * B[0] + db[q][1] * B[1] + db[q][2] * B[2]);
      for (int q = 0; q < 3; ++q) G[3 + q] += G[q];
      for (int q = 0; q < 3; ++q)
        for (int k = 0; k < 3; ++k)
          d1[q][k] += cg[q][0] * d2[0][k] * G[0] + cg[q][1] * d2[1][k] * G[1] + cg[q][2] * d2[2][k] * G[2];
    }
    if (!ok) ++notconv;
  }
  if (numerr) return -2;
  if (notconv) return 1;
  // four-atom groups: shake4 Newton + LU (simulu)
  for (const auto& g : c.sk4) {
    const int* a = g.a;
    double im[4] = {c.imass[a[0]], c.imass[a[1]], c.imass[a[2]], c.imass[a[3]]};
    const double cg[6][6] = {
        {im[0] + im[1], -im[1], -im[0], -im[0], 0.0, -im[1]},
        {-im[1], im[1] + im[2], -im[2], 0.0, -im[2], im[1]},
        {-im[0], -im[2], im[2] + im[0], im[0], im[2], 0.0},
        {-im[0], 0.0, im[0], im[3] + im[0], -im[3], -im[3]},
        {0.0, -im[2], im[2], -im[3], im[2] + im[3], im[3]},
        {-im[1], im[1], 0.0, -im[3], im[3], im[1] + im[3]}};
    const int nc = 6;
    double d1[6][3], d2[6][3], wk[6][3], G[6] = {0, 0, 0, 0, 0, 0};
    for (int q = 0; q < nc; ++q) {
      vec(r1, a[kParlis[q][0]], a[kParlis[q][1]], d1[q]);
      vec(r2, a[kParlis[q][0]], a[kParlis[q][1]], d2[q]);
      for (int k = 0; k < 3; ++k) wk[q][k] = d1[q][k];
    }
    bool ok = false;
    for (int it = 0; it < maxit; ++it) {
      double B[6];
      bool flg = true;
      for (int q = 0; q < nc; ++q) {
        B[q] = g.d2[q] - (wk[q][0] * wk[q][0] + wk[q][1] * wk[q][1] + wk[q][2] * wk[q][2]);
        if (std::fabs(B[q]) >= tol * g.d2[q]) flg = false;
      }
      if (flg) {
        ok = true;
        for (int k = 0; k < 3; ++k) {
          r1[3 * a[0] + k] += im[0] * (G[0] * d2[0][k] - G[2] * d2[2][k] - G[3] * d2[3][k]);
          r1[3 * a[1] + k] += im[1] * (-G[0] * d2[0][k] + G[1] * d2[1][k] + G[5] * d2[5][k]);
          r1[3 * a[2] + k] += im[2] * (-G[1] * d2[1][k] + G[2] * d2[2][k] + G[4] * d2[4][k]);
          r1[3 * a[3] + k] += im[3] * (G[3] * d2[3][k] - G[4] * d2[4][k] - G[5] * d2[5][k]);
        }
        break;
      }
      double gf[6][6];
      for (int ig = 0; ig < nc; ++ig)
        for (int q = 0; q < nc; ++q)
          gf[q][ig] = 2.0 * cg[q][ig] * (wk[q][0] * d2[ig][0] + wk[q][1] * d2[ig][1] + wk[q][2] * d2[ig][2]);
      for (int ig = 0; ig < nc; ++ig)
        for (int q = 0; q < nc; ++q) B[q] += gf[q][ig] * G[ig];
      if (simulu(gf, nc, B, G) != 0) ++numerr;
      for (int q = 0; q < nc; ++q)
        for (int k = 0; k < 3; ++k) wk[q][k] = d1[q][k];
      for (int ig = 0; ig < nc; ++ig)
        for (int q = 0; q < nc; ++q)
          for (int k = 0; k < 3; ++k) wk[q][k] += cg[q][ig] * d2[ig][k] * G[ig];
    }
    if (!ok) ++notconv;
  }
  if (numerr) return -2;
  if (notconv) return 1;
  return ier;
}

// caltmp (caltmp.f90:2-48): T of the whole system from v
// caltmp (caltmp.f90:1-48): ek starts with lambda's kinetic term l_mas*l_vel^2 (zero
// without ALSD)
double caltmp(const Ctx& c, const double* v, double lvt = 0.0) {
  double ek = c.lam_m * lvt * lvt;
  for (int i = 0; i < c.n; ++i)
    ek += c.mass[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
  ek *= 1.0e7;
  return ek / (kGas * (double)c.idnfre);
}

// caltmp2 (caltmp.f90:54-110): per sub-system temperatures
void caltmp2(const Ctx& c, const double* v, double* tf, double lvt = 0.0) {
  for (int s = 0; s < c.nsub; ++s) tf[s] = 0.0;
  for (int i = 0; i < c.n; ++i)
    tf[c.mol[i]] += c.mass[i] * (v[3 * i] * v[3 * i] + v[3 * i + 1] * v[3 * i + 1] + v[3 * i + 2] * v[3 * i + 2]);
  if (c.lam_tc && c.ifg_lambda >= 0) tf[c.ifg_lambda] += c.lam_m * lvt * lvt;   // caltmp.f90:98-99
  for (int s = 0; s < c.nsub; ++s) tf[s] = tf[s] * 1.0e7 / (c.nfrmol[s] * kGas);
}

// McMD weight d lnP/dE at energy e (verlethe.f90:196-230), returns dew (force scale)
double mcmd_scale(const Ctx& c, double e) {
  const jp_ge& g = c.ge;
  double dprobl;
  if (e <= g.celw) dprobl = g.alphalw;
  else if (e >= g.ceup) dprobl = g.alphaup;
  else {
    double rt = (e - g.celw) / (g.ceup - g.celw);
    int i = 0;
    for (i = 0; i < g.nwindow; ++i)
      if (rt < c.ge_high[i]) break;
    if (i >= g.nwindow) i = g.nwindow - 1;
    rt -= c.ge_low[i];
    const double* cf = &c.ge_coef[(size_t)i * (g.ndeg + 1)];
    dprobl = cf[0];
    for (int j = 1; j <= g.ndeg; ++j) dprobl += cf[j] * std::pow(rt, j);
  }
  return (kGas / kJouCal) * 1.0e-3 * g.tempce * dprobl;
}

// ALSD weight d lnP/dlambda (verlethe.f90:240-262): polynomial in lambda itself (window
// search on lambda, no reduction) plus the linear walls below celw / above ceup; dew
double alsd_dew(const Ctx& c) {
  const jp_ge& g = c.ge;
  const double lam = c.lam;
  int i = g.nwindow - 1;
  for (int j = 0; j < g.nwindow; ++j)
    if (lam < c.ge_high[j]) { i = j; break; }
  const double rt = lam - c.ge_low[i];
  const double* cf = &c.ge_coef[(size_t)i * (g.ndeg + 1)];
  double dprobl = cf[0];
  for (int j = 1; j <= g.ndeg; ++j) dprobl += cf[j] * std::pow(rt, j);
  if (lam < g.celw) dprobl += g.lower * (g.celw - lam);
  else if (lam > g.ceup) dprobl += g.upper * (lam - g.ceup);
  return (kGas / kJouCal) * 1.0e-3 * g.tempce * dprobl;
}

// remotv (remotv.f90:2-131): remove the centre-of-mass translation (STOPCE 1, 3) and/or
// rotation (2, 3) of atoms 0..stop_n-1 from c.vel, centre and inertia from positions xp.
// Direct sums over the atoms, as the reference forms them.  Returns 0, -1 (no mass) or -2
// (singular inertia tensor).
int remotv(Ctx& c, const double* xp) {
  const int na = c.stop_n, idf = c.prm.stop_center;
  double tot = 0.0;
  for (int i = 0; i < na; ++i) tot += c.mass[i];
  if (tot <= 0.0) return -1;
  tot = 1.0 / tot;
  double cen[3] = {0, 0, 0}, tv[3] = {0, 0, 0}, av[3] = {0, 0, 0};
  for (int i = 0; i < na; ++i)
    for (int k = 0; k < 3; ++k) {
      cen[k] += c.mass[i] * xp[3 * i + k];
      if (idf == JP_STOP_TRANS || idf == JP_STOP_BOTH) tv[k] += c.mass[i] * c.vel[3 * i + k];
    }
  for (int k = 0; k < 3; ++k) { cen[k] *= tot; tv[k] *= tot; }
  std::vector<double> d((size_t)3 * na);
  for (int i = 0; i < na; ++i)
    for (int k = 0; k < 3; ++k) d[3 * i + k] = xp[3 * i + k] - cen[k];
  if (idf == JP_STOP_ROT || idf == JP_STOP_BOTH) {
    double ixx = 0, iyy = 0, izz = 0, ixy = 0, iyz = 0, izx = 0;
    for (int i = 0; i < na; ++i) {
      const double m = c.mass[i], dx = d[3 * i], dy = d[3 * i + 1], dz = d[3 * i + 2];
      ixx += m * (dy * dy + dz * dz);
      iyy += m * (dz * dz + dx * dx);
      izz += m * (dx * dx + dy * dy);
      ixy -= m * dx * dy;
      iyz -= m * dy * dz;
      izx -= m * dz * dx;
    }
    double det = ixx * iyy * izz + 2.0 * ixy * iyz * izx - iyz * iyz * ixx - izx * izx * iyy - ixy * ixy * izz;
    if (det == 0.0) return -2;
    det = 1.0 / det;
    double inv[3][3];
    inv[0][0] = (iyy * izz - iyz * iyz) * det;
    inv[0][1] = inv[1][0] = (iyz * izx - izz * ixy) * det;
    inv[0][2] = inv[2][0] = (ixy * iyz - izx * iyy) * det;
    inv[1][1] = (izz * ixx - izx * izx) * det;
    inv[1][2] = inv[2][1] = (izx * ixy - ixx * iyz) * det;
    inv[2][2] = (ixx * iyy - ixy * ixy) * det;
    for (int i = 0; i < na; ++i) {   // angular velocity: inverse tensor times angular momentum
      const double* v = &c.vel[3 * i];
      const double dx = d[3 * i], dy = d[3 * i + 1], dz = d[3 * i + 2];
      const double l[3] = {dy * v[2] - dz * v[1], dz * v[0] - dx * v[2], dx * v[1] - dy * v[0]};
      for (int k = 0; k < 3; ++k)
        av[k] += c.mass[i] * (inv[k][0] * l[0] + inv[k][1] * l[1] + inv[k][2] * l[2]);
    }
  }
  for (int i = 0; i < na; ++i) {
    double* v = &c.vel[3 * i];
    const double dx = d[3 * i], dy = d[3 * i + 1], dz = d[3 * i + 2];
    v[0] = v[0] - av[1] * dz + av[2] * dy - tv[0];
    v[1] = v[1] - av[2] * dx + av[0] * dz - tv[1];
    v[2] = v[2] - av[0] * dy + av[1] * dx - tv[2];
  }
  return 0;
}

inline bool stop_on(const Ctx& c) {
  return c.prm.stop_center >= JP_STOP_TRANS && c.prm.stop_center <= JP_STOP_BOTH && c.stop_n > 0;
}

// error code of the engine for remotv's ier
inline int remotv_code(int ier) { return ier == -1 ? JP_E_STOP_MASS : JP_E_STOP_SINGULAR; }

// One verlet step (verlet.f90:2-226), METHOD= MICR or CONS: pseudo-temperature force scale,
// velocity update, centre-of-mass stop, Berendsen scaling (scalet.f90), positions, SHAKE.
void split_force(Ctx& c, double* ene);

int step_verlet(Ctx& c, double* ene) {
  const int n = c.n;
  std::vector<double> x0(c.cord);
  const bool cons = c.prm.method == JP_METHOD_CONS;
  const double tempc = cons ? caltmp(c, c.vel.data()) : 0.0;   // T of v(t-dt/2), verlet.f90:31-34
  if (c.split) {
    split_force(c, ene);
  } else {
    energy_grad(c, c.cord.data(), ene, c.grad.data());
    if (c.prm.psetmp > kEps)   // verlet.f90:118-142
      for (auto& g : c.grad) g *= c.prm.temp / c.prm.psetmp;
  }
  const double dt = c.prm.dt;
  double rt = -dt * kConvcv;
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) c.vel[3 * i + k] += rt * c.grad[3 * i + k] / c.mass[i];
  if (stop_on(c)) {
    const int ier = remotv(c, x0.data());
    if (ier) return remotv_code(ier);
  }
  if (cons && tempc > 0.0) {   // scalet.f90:30-45
    double lam = std::sqrt(1.0 + (dt / c.prm.taut) * (c.prm.temp / tempc - 1.0));
    if (lam >= 2.0) lam = 2.0;
    for (auto& v : c.vel) v *= lam;
  }
  for (int i = 0; i < 3 * n; ++i) c.cord[i] += dt * c.vel[i];
  if (c.prm.shake_method != JP_SHAKE_NONE) {
    int ier = shake_all(c, c.cord.data(), x0.data());
    if (ier != 0) return ier;
    rt = 1.0 / dt;
    for (int i = 0; i < 3 * n; ++i) c.vel[i] = (c.cord[i] - x0[i]) * rt;
  }
  return 0;
}

// One verlethe step (verlethe.f90:2-758), METHOD= CANO or GE (McMD), itmeth 1 or 2,
// with the SHAKE <-> thermostat loop (icslop) and SHAKE-failure dt halving.
// dnergy and verlethe's scaling of the gradient (verlethe.f90:103-321): the pseudo
// temperature (CANO), the McMD weight (GE) or the ALSD class combination (done inside
// energy_grad) with the lambda force; c.grad gets the gradient the integration uses, the
// return value is lambda_f.  This is the state that FDEBUG dumps (verlethe.f90:325-387).
// partial McMD: the class-1 gradient into g1 and the class-2 gradient into g2, from two
// evaluations with the class weights set to one class each (the energies do not depend on
// them; c.ecls holds the class totals afterwards)
void split_eval(Ctx& c, double* ene, double* g1, double* g2) {
  c.fover = true;
  c.fo[0] = 1.0; c.fo[1] = 0.0; c.fo[2] = 0.0;
  energy_grad(c, c.cord.data(), ene, g1);
  c.fo[0] = 0.0; c.fo[2] = 1.0;
  energy_grad(c, c.cord.data(), ene, g2);
  c.fover = false;
}

// grad(:,:,2) = grad(:,:,1) * dew + grad(:,:,2) (verlet.f90:130-141, verlethe.f90:176-187,
// :223-234): dew the McMD weight of the class-1 energy epotcc(1,1) (METHOD= GE) or
// SETTEM / PSETMP
void split_force(Ctx& c, double* ene) {
  std::vector<double> g2(c.grad.size());
  split_eval(c, ene, c.grad.data(), g2.data());
  const double dew = c.prm.method == JP_METHOD_GE ? mcmd_scale(c, c.ecls[0]) : c.prm.temp / c.prm.psetmp;
  for (size_t k = 0; k < g2.size(); ++k) c.grad[k] = c.grad[k] * dew + g2[k];
}

double verlethe_force(Ctx& c, double* ene) {
  double lambda_f = 0.0;
  if (c.split) {
    split_force(c, ene);
    return lambda_f;
  }
  energy_grad(c, c.cord.data(), ene, c.grad.data());
  if (c.alsd) {
    // forces already combined by class (energy_grad); lambda force (verlethe.f90:289-320)
    if (c.prm.method == JP_METHOD_GE) {
      const double dew = alsd_dew(c);
      if (c.alsd == JP_ALSD_LMD) lambda_f = -2.0 * c.ecls[0] * c.lam - c.ecls[1] - dew;
      else lambda_f = -c.ecls[0] - 0.5 * c.ecls[1] / std::sqrt(c.lam) - dew;
    }
  } else if (c.prm.method == JP_METHOD_CANO) {
    if (c.prm.psetmp > kEps) {
      double dew = c.prm.temp / c.prm.psetmp;
      for (auto& g : c.grad) g *= dew;
    }
  } else if (c.prm.method == JP_METHOD_GE) {
    double dew = mcmd_scale(c, ene[JP_E_TOTAL]);
    for (auto& g : c.grad) g *= dew;
  }
  return lambda_f;
}

int step_verlethe(Ctx& c, double* ene) {
  const int n = c.n;
  const double deltt = c.prm.dt;
  const double temps = c.prm.temp, tmpsta = c.prm.temp_start;
  const int idhtlp = c.prm.heat_loop;
  const double i_idhtlp = idhtlp > 0 ? 1.0 / (double)idhtlp : 0.0;
  const long long idloop = c.idloop;
  const bool whole = (c.prm.tempco == 1);
  const bool shk = (c.prm.shake_method != JP_SHAKE_NONE);
  double Tdeltt = deltt;
  int ishk = 0, jshk = 1;
  std::vector<double> cordm1(3 * n), velback(3 * n), velt(3 * n), cordback(3 * n), forcec(3 * n);
  std::vector<double> tf(c.nsub), chif(c.nsub);
  auto target_t = [&]() {
    if (idhtlp <= 0 || idloop > idhtlp) return temps;
    return tmpsta + ((temps - tmpsta) * i_idhtlp) * (double)idloop;
  };
  double lmd_back = c.lam, lmd_vback = c.lam_v, lambda_f = 0.0;
  for (;;) {
    cordm1 = c.cord;
    velback = c.vel;
    lmd_back = c.lam;
    lmd_vback = c.lam_v;
  redo:
    lambda_f = verlethe_force(c, ene);
    double* g = c.grad.data();
    // velocity at 1/2 dt without SHAKE force (verlethe.f90:390-398)
    double rt = 0.5 * Tdeltt * kConvcv;
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < 3; ++k) velt[3 * i + k] = c.vel[3 * i + k] - rt * g[3 * i + k] * c.imass[i];
    double lambda_vt = c.lam_v;
    if (c.lam_im != 0.0) lambda_vt = c.lam_v + rt * lambda_f * c.lam_im;   // :403-404
    // temperature control (verlethe.f90:400-470)
    const double tt = target_t();
    const double lstep = Tdeltt * kConvcv * lambda_f * c.lam_im;
    if (whole) {
      double tempc = shk ? caltmp(c, velt.data(), lambda_vt) : temps;
      double chi = std::sqrt(tt / tempc);
      double a = chi * Tdeltt * kConvcv, b = 2.0 * chi - 1.0;
      for (int i = 0; i < n; ++i)
        for (int k = 0; k < 3; ++k) c.vel[3 * i + k] = b * c.vel[3 * i + k] - a * g[3 * i + k] * c.imass[i];
      if (c.lam_im != 0.0) {   // :439-445
        if (c.lam_tc) c.lam_v = b * c.lam_v + a * lambda_f * c.lam_im;
        else c.lam_v = c.lam_v + lstep;
      }
    } else {
      if (shk) caltmp2(c, velt.data(), tf.data(), lambda_vt);
      else std::fill(tf.begin(), tf.end(), temps);
      for (int s = 0; s < c.nsub; ++s) chif[s] = std::sqrt(tt / tf[s]);
      for (int i = 0; i < n; ++i) {
        double chi = chif[c.mol[i]];
        double a = chi * Tdeltt * kConvcv, b = 2.0 * chi - 1.0;
        for (int k = 0; k < 3; ++k) c.vel[3 * i + k] = b * c.vel[3 * i + k] - a * g[3 * i + k] * c.imass[i];
      }
      // :475-481; without a lambda sub-system (CANO) the uncoupled update is taken
      if (c.lam_tc && c.ifg_lambda >= 0) {
        const double chi = chif[c.ifg_lambda];
        c.lam_v = (2.0 * chi - 1.0) * c.lam_v + chi * Tdeltt * kConvcv * lambda_f * c.lam_im;
      } else {
        c.lam_v = c.lam_v + lstep;
      }
    }
    if (stop_on(c)) {   // verlethe.f90:490-492, positions at time t
      const int ier = remotv(c, c.cord.data());
      if (ier) return remotv_code(ier);
    }
    for (int i = 0; i < 3 * n; ++i) c.cord[i] += Tdeltt * c.vel[i];
    c.lam = c.lam + Tdeltt * c.lam_v;                                        // :516
    lambda_vt = (lmd_vback + c.lam_v) * 0.5;                                 // :529
    if (shk) {
      std::fill(forcec.begin(), forcec.end(), 0.0);
      bool retry = false;
      for (int numite = 1; numite <= c.prm.icslop; ++numite) {
        cordback = c.cord;
        int ier = shake_all(c, c.cord.data(), cordm1.data());
        if (ier != 0) {
          c.cord = cordm1;
          c.vel = velback;
          c.lam = lmd_back;
          c.lam_v = lmd_vback;
          if (Tdeltt < 0.01 * deltt) return JP_E_SHAKE_ABORT;
          jshk *= 2; ishk *= 2;
          Tdeltt *= 0.5;
          retry = true;
          break;
        }
        double ri = 1.0 / Tdeltt;
        for (int i = 0; i < 3 * n; ++i) {
          c.vel[i] = (c.cord[i] - cordm1[i]) * ri;
          velt[i] = (velback[i] + c.vel[i]) * 0.5;
        }
        const double tshu = target_t();
        if (whole) {
          double tempc = caltmp(c, velt.data(), lambda_vt);
          if (std::fabs(tempc - tshu) < c.prm.fcstol * tshu) break;
        } else {
          caltmp2(c, velt.data(), tf.data(), lambda_vt);
          double mn = *std::min_element(tf.begin(), tf.end()), mx = *std::max_element(tf.begin(), tf.end());
          if (std::max(std::fabs(mn - tshu), std::fabs(mx - tshu)) < c.prm.fcstol * tshu) break;
        }
        if (numite == c.prm.icslop) break;
        double r2 = 1.0 / (Tdeltt * Tdeltt), h = 0.5 * Tdeltt;
        for (int i = 0; i < n; ++i)
          for (int k = 0; k < 3; ++k) {
            int q = 3 * i + k;
            forcec[q] += r2 * (c.cord[q] - cordback[q]);
            velt[q] = h * (-kConvcv * g[q] * c.imass[i] + forcec[q]) + velback[q];
          }
        if (whole) {
          double tempc = caltmp(c, velt.data(), lambda_vt);
          double chi = std::sqrt(tt / tempc);
          double a = chi * Tdeltt, b = 2.0 * chi - 1.0;
          for (int i = 0; i < n; ++i)
            for (int k = 0; k < 3; ++k) {
              int q = 3 * i + k;
              c.vel[q] = (-kConvcv * g[q] * c.imass[i] + forcec[q]) * a + velback[q] * b;
            }
        } else {
          caltmp2(c, velt.data(), tf.data(), lambda_vt);
          for (int s = 0; s < c.nsub; ++s) chif[s] = std::sqrt(tt / tf[s]);
          for (int i = 0; i < n; ++i) {
            double chi = chif[c.mol[i]];
            double a = chi * Tdeltt, b = 2.0 * chi - 1.0;
            for (int k = 0; k < 3; ++k) {
              int q = 3 * i + k;
              c.vel[q] = b * velback[q] + a * (-kConvcv * g[q] * c.imass[i] + forcec[q]);
            }
          }
        }
        if (stop_on(c)) {   // verlethe.f90:706-709
          const int ier = remotv(c, cordm1.data());
          if (ier) return remotv_code(ier);
        }
        for (int i = 0; i < 3 * n; ++i) c.cord[i] = cordm1[i] + Tdeltt * c.vel[i];
      }
      if (retry) goto redo;
    }
    ++ishk;
    if (ishk == jshk) break;
    if (ishk % 2 == 0) { jshk /= 2; ishk /= 2; Tdeltt *= 2.0; }
  }
  return 0;
}

template <class T>
T* arr(const T* p, size_t n, std::vector<T>& store) {
  store.assign(p, p + n);
  return store.data();
}

}  // namespace

// =======================================================================================
// C ABI for the Python test harness
// =======================================================================================
extern "C" {

void* or_create(const jp_system* s, const jp_params* prm, int nthreads) {
  Ctx* c = new Ctx();
  const int b = s->index_base;
  const int n = s->natom;
  c->n = n;
  c->prm = *prm;
  c->nthreads = nthreads > 0 ? nthreads : omp_get_max_threads();
  c->pbc = prm->bounda == JP_BOUND_PBC;
  for (int k = 0; k < 3; ++k) { c->box[k] = s->box[k]; c->invbox[k] = 1.0 / s->box[k]; }
  c->mass.assign(s->mass, s->mass + n);
  c->imass.resize(n);
  for (int i = 0; i < n; ++i) c->imass[i] = 1.0 / c->mass[i];   // md.f90:62-71 ifxmass
  c->chg.assign(s->charge, s->charge + n);
  c->typ.resize(n);
  for (int i = 0; i < n; ++i) c->typ[i] = s->atype[i] - b;
  c->mol.assign(n, 0);
  c->alsd = ((prm->alsd == JP_ALSD_LMD || prm->alsd == JP_ALSD_LMD2) && s->cluster) ? prm->alsd : 0;
  c->inA.assign(n, 0);
  if (c->alsd)
    for (int i = 0; i < n; ++i) c->inA[i] = s->cluster[i] ? 1 : 0;
  c->geps = (prm->alsd >= JP_GEPS_AND && prm->alsd <= JP_GEPS_XOR) ? prm->alsd : 0;
  c->icl.assign(n, 2);
  if (c->geps && s->cluster) {
    bool hasA = false, hasB = false;
    for (int i = 0; i < n; ++i) {
      if (s->cluster[i] == 1) { c->icl[i] = 0; hasA = true; }
      else if (s->cluster[i] == 2) { c->icl[i] = 1; hasB = true; }
    }
    c->split = hasA || hasB;   // nfrag > 1, nfrg = 2
    // n_matrix(icls_a, icls_b) = 1 (inpcls.f90:298-325) on the region codes A 0, B 1,
    // neither 2; without region B the nfrag = 2 matrix (A, the rest)
    auto bit = [](int a, int b) { return (1u << (3 * a + b)) | (1u << (3 * b + a)); };
    unsigned t = 0;
    if (!hasB) {
      if (c->geps == JP_GEPS_AND) t = bit(0, 0);
      else if (c->geps == JP_GEPS_OR) t = bit(0, 0) | bit(0, 2);
      else t = bit(0, 2);
    } else {
      if (c->geps == JP_GEPS_AND) t = bit(0, 0) | bit(1, 1);
      else if (c->geps == JP_GEPS_OR) t = bit(0, 0) | bit(0, 1);
      else t = bit(0, 1);
    }
    c->tab1 = t;
  }
  if (s->molecule && prm->tempco == 2) {
    // sub-system ids renumbered densely in order, empty ids removed (md.f90:133-151);
    // with clusters each molecule splits into its cluster and non-cluster part (ixamol2)
    std::vector<int> ids;
    for (int i = 0; i < n; ++i)
      ids.push_back(c->alsd    ? 2 * (s->molecule[i] - b) + (c->inA[i] ? 0 : 1)
                    : c->split ? 3 * (s->molecule[i] - b) + c->icl[i]
                               : s->molecule[i] - b);
    std::vector<int> u(ids);
    std::sort(u.begin(), u.end());
    u.erase(std::unique(u.begin(), u.end()), u.end());
    for (int i = 0; i < n; ++i) c->mol[i] = (int)(std::lower_bound(u.begin(), u.end(), ids[i]) - u.begin());
  }
  c->ntype = s->ntype;
  c->c6.assign(s->c6, s->c6 + (size_t)s->ntype * s->ntype);
  c->c12.assign(s->c12, s->c12 + (size_t)s->ntype * s->ntype);
  if (s->hbond) {
    const size_t nt2 = (size_t)s->ntype * s->ntype;
    c->hbp.assign(s->hbond, s->hbond + nt2);
    c->c10.assign(s->c10, s->c10 + nt2);
    c->c12h.assign(s->c12h, s->c12h + nt2);
  }
  if (s->ncelres > 0 && s->celres) {
    c->res_first.assign(n, -1);
    c->res_last.assign(n, -1);
    for (int i = 0; i < s->ncelres; ++i)
      for (int a = s->celres[2 * i] - b; a <= s->celres[2 * i + 1] - b; ++a) {
        c->res_first[a] = s->celres[2 * i] - b;
        c->res_last[a] = s->celres[2 * i + 1] - b;
      }
  }
  if (s->restraints) {
    const jp_restraints& q = *s->restraints;
    for (int i = 0; i < q.npos; ++i)
      c->posres.push_back({q.pos_atom[i] - b, q.pos_k[i],
                           {q.pos_ref[3 * i], q.pos_ref[3 * i + 1], q.pos_ref[3 * i + 2]}});
    for (int i = 0; i < q.ndist; ++i) {
      Ctx::DistRes d;
      for (int p = q.dist_iptr[i]; p < q.dist_iptr[i + 1]; ++p) d.gi.push_back(q.dist_iatom[p] - b);
      for (int p = q.dist_jptr[i]; p < q.dist_jptr[i + 1]; ++p) d.gj.push_back(q.dist_jatom[p] - b);
      d.lo = q.dist_lo[i]; d.up = q.dist_up[i]; d.klo = q.dist_klo[i]; d.kup = q.dist_kup[i];
      c->distres.push_back(d);
    }
    for (int i = 0; i < q.ndihe; ++i) {
      Ctx::DiheRes d;
      for (int k = 0; k < 4; ++k) d.a[k] = q.dihe_atom[4 * i + k] - b;
      d.lo = q.dihe_lo[i]; d.up = q.dihe_up[i]; d.klo = q.dihe_klo[i]; d.kup = q.dihe_kup[i];
      c->diheres.push_back(d);
    }
    for (int i = 0; i < q.ncap_group; ++i)
      c->cap_groups.push_back({q.cap_group[2 * i] - b, q.cap_group[2 * i + 1] - b});
    for (int i = 0; i < q.ncap_atom; ++i) c->cap_atoms.push_back(q.cap_atom[i] - b);
    for (int k = 0; k < 3; ++k) c->cap_c[k] = q.cap_center[k];
    c->cap_r = q.cap_radius; c->cap_k = q.cap_k;
    c->cap_ra = q.cap_atom_radius; c->cap_ka = q.cap_atom_k;
    c->cap_shape = q.cap_shape == 0 ? JP_CAP_SPHERE : q.cap_shape;
    c->cap_func = q.cap_function == 0 ? JP_CAP_HARMONIC : q.cap_function;
    for (int k = 0; k < 6; ++k) { c->cap_wall[k] = q.cap_wall[k]; c->cap_awall[k] = q.cap_atom_wall[k]; }
    for (int k = 0; k < 3; ++k) { c->cap_ell[k] = q.cap_ellipse[k]; c->cap_aell[k] = q.cap_atom_ellipse[k]; }
  }
  // exclusions (inpcls.f90:229-290 itab14)
  c->excl.assign(n, {});
  for (int i = 0; i < n; ++i) {
    for (int p = s->excl_ptr[i]; p < s->excl_ptr[i + 1]; ++p) c->excl[i].push_back(s->excl_idx[p] - b);
    std::sort(c->excl[i].begin(), c->excl[i].end());
  }
  // chgmod (inpcls.f90:215-227)
  c->ccoef = kEekcal / prm->dielectric;
  const double fac = std::sqrt(c->ccoef);
  c->chgmod.resize(n);
  for (int i = 0; i < n; ++i) c->chgmod[i] = fac * c->chg[i];
  // SHAKE groups (setshk.f90 redshk: fudshk = d^2; modshk orders 2,3,4-atom groups)
  auto pairkey = [](int a, int bb) { return a < bb ? ((long long)a << 32) | bb : ((long long)bb << 32) | a; };
  std::vector<long long> cpairs;
  for (int gi = 0; gi < s->nshake; ++gi) {
    Shake g;
    g.n = s->shake_n[gi];
    for (int k = 0; k < 4; ++k) g.a[k] = k < g.n ? s->shake_atoms[4 * gi + k] - b : -1;
    int nc = g.n * (g.n - 1) / 2;
    for (int q = 0; q < 6; ++q) g.d2[q] = q < nc ? s->shake_dist[6 * gi + q] * s->shake_dist[6 * gi + q] : 0.0;
    for (int q = 0; q < nc; ++q) cpairs.push_back(pairkey(g.a[kParlis[q][0]], g.a[kParlis[q][1]]));
    c->nconstr += nc;
    if (g.n == 2) c->sk2.push_back(g);
    else if (g.n == 3) c->sk3.push_back(g);
    else c->sk4.push_back(g);
  }
  std::sort(cpairs.begin(), cpairs.end());
  const bool shk = prm->shake_method != JP_SHAKE_NONE && s->nshake > 0;
  if (!shk) { c->sk2.clear(); c->sk3.clear(); c->sk4.clear(); c->nconstr = 0; c->prm.shake_method = JP_SHAKE_NONE; }
  auto constrained = [&](int a, int bb) { return shk && std::binary_search(cpairs.begin(), cpairs.end(), pairkey(a, bb)); };
  // bonds / angles, dropping SHAKE-constrained ones (setshk.f90 reabnd/reaang)
  for (int i = 0; i < s->nbond; ++i) {
    int a = s->bond[2 * i] - b, bb = s->bond[2 * i + 1] - b;
    if (constrained(a, bb)) continue;
    const int cl = (prm->scale_terms & JP_SCALE_BOND) ? c->pcls(a, bb) : 2;   // incel.f90:705-712
    c->bonds.push_back({a, bb, s->bond_k[i], s->bond_r0[i], cl});
  }
  for (int i = 0; i < s->nangle; ++i) {
    int a = s->angle[3 * i] - b, m = s->angle[3 * i + 1] - b, z = s->angle[3 * i + 2] - b;
    if (constrained(a, z)) continue;
    const int cl = (prm->scale_terms & JP_SCALE_ANGLE) ? c->pcls(a, z) : 2;   // :735-742
    c->angles.push_back({a, m, z, s->angle_k[i], s->angle_theta0[i], cl});
  }
  for (int i = 0; i < s->ntors; ++i) {
    Ctx::Tors t;
    for (int k = 0; k < 4; ++k) t.a[k] = s->tors[4 * i + k] - b;
    t.k = s->tors_k[i]; t.nrot = s->tors_nrot[i]; t.phase = s->tors_phase[i]; t.div = s->tors_div[i];
    // class of the central pair (incel.f90:838-845); SCALET's peptide-bond exemption
    // (scale_tor 2/3, :846-866) keeps the marked torsions unscaled
    const bool fixed = s->tors_unscaled && s->tors_unscaled[i];
    t.cls = ((prm->scale_terms & JP_SCALE_TORS) && !fixed) ? c->pcls(t.a[1], t.a[2]) : 2;
    c->tors.push_back(t);
    // 1-4 pairs (incel.f90:972-987, mknopm inptpl.f90:453-462, incel.f90:1084-1087)
    if (s->tors_nbf[i] == 1) {
      int a1 = t.a[0], a4 = t.a[3];
      int t1 = c->typ[a1], t4 = c->typ[a4];
      double sv = std::min(s->s14_vdw[t1], s->s14_vdw[t4]);
      double se = std::min(s->s14_ele[t1], s->s14_ele[t4]);
      c->p14.push_back({a1, a4, sv, se * c->ccoef * c->chg[a1] * c->chg[a4], c->pcls(a1, a4)});
    }
  }
  for (int i = 0; i < s->nimpr; ++i) {
    Ctx::Tors t;
    for (int k = 0; k < 4; ++k) t.a[k] = s->impr[4 * i + k] - b;
    t.k = s->impr_k[i]; t.nrot = s->impr_nrot[i]; t.phase = s->impr_phase[i]; t.div = s->impr_div[i];
    t.cls = 2;
    if ((prm->scale_terms & JP_SCALE_IMPR) && c->alsd) {   // n_matrix(min icls, max icls) :911-917
      int na = 0;
      for (int k = 0; k < 4; ++k) na += c->inA[t.a[k]];
      t.cls = na == 4 ? 0 : (na > 0 ? 1 : 2);
    } else if ((prm->scale_terms & JP_SCALE_IMPR) && c->split) {
      int lo = 2, hi = 0;
      for (int k = 0; k < 4; ++k) { lo = std::min(lo, c->icl[t.a[k]]); hi = std::max(hi, c->icl[t.a[k]]); }
      t.cls = ((c->tab1 >> (3 * lo + hi)) & 1u) ? 0 : 2;
    }
    c->imprs.push_back(t);
  }
  // ZD constants, dself and excess list (incel.f90:29-39, :627-689)
  c->rc = prm->cutoff;
  c->rlim = c->rc + 1.5;
  c->rlim2 = c->rlim * c->rlim;
  c->irlim2 = 1.0 / (c->rc * c->rc);
  {
    double rtmp = 1.0 / c->rc;
    c->zcore = 1.5 * rtmp;
    c->fcoeff = rtmp * rtmp * rtmp;
    c->bcoeff = 0.5 * c->fcoeff;
  }
  // CAL15M= ATOM (enear.f90 #ACT lines): E = qi qj co / r, F = qi qj co / r^3 d, which is
  // the ZD formula with zcore = bcoeff = fcoeff = 0; no self or excess term (#ZD only)
  const bool zd = prm->cal15m == JP_CAL15M_ZD;
  if (!zd) c->zcore = c->fcoeff = c->bcoeff = 0.0;
  std::vector<double> dwork(c->chg);   // self term
  std::vector<double> dwk((size_t)3 * n, 0.0);   // per class (incel.f90:629-654)
  for (int i = 0; i < n; ++i) dwk[(size_t)c->pcls(i, i) * n + i] += c->chg[i];
  auto addx = [&](int a, int bb) {
    if (!zd) return;
    dwork[a] += c->chg[bb];
    dwork[bb] += c->chg[a];
    const int cl = c->pcls(a, bb);
    dwk[(size_t)cl * n + a] += c->chg[bb];
    dwk[(size_t)cl * n + bb] += c->chg[a];
    c->excess.push_back({a, bb, cl});
  };
  for (int i = 0; i < s->nbond; ++i) addx(s->bond[2 * i] - b, s->bond[2 * i + 1] - b);
  for (int i = 0; i < s->nangle; ++i) addx(s->angle[3 * i] - b, s->angle[3 * i + 2] - b);
  for (int i = 0; i < s->ntors; ++i)
    if (s->tors_nbf[i] == 1) addx(s->tors[4 * i] - b, s->tors[4 * i + 3] - b);
  double ds = 0.0;
  for (int i = 0; i < n; ++i) ds += c->chg[i] * dwork[i];
  c->dself = -c->zcore * ds * 0.5 * c->ccoef;
  for (int k = 0; k < 3; ++k) {
    double d = 0.0;
    for (int i = 0; i < n; ++i) d += c->chg[i] * dwk[(size_t)k * n + i];
    c->dself_cls[k] = -c->zcore * d * 0.5 * c->ccoef;
  }
  // GE weight
  if (s->ge) {
    c->has_ge = true;
    c->ge = *s->ge;
    size_t nc = (size_t)s->ge->nwindow * (s->ge->ndeg + 1);
    c->ge_coef.assign(s->ge->coef, s->ge->coef + nc);
    c->ge_low.assign(s->ge->low, s->ge->low + s->ge->nwindow);
    c->ge_high.assign(s->ge->high, s->ge->high + s->ge->nwindow);
  }
  // DOF (md.f90:116-131, :133-183)
  c->idnfre = 3 * n - c->nconstr;
  c->nsub = 1;
  for (int i = 0; i < n; ++i) c->nsub = std::max(c->nsub, c->mol[i] + 1);
  c->nfrmol.assign(c->nsub, 0.0);
  for (int i = 0; i < n; ++i) c->nfrmol[c->mol[i]] += 3.0;
  for (const auto* v : {&c->sk2, &c->sk3, &c->sk4})
    for (const auto& g : *v) c->nfrmol[c->mol[g.a[0]]] -= (double)(g.n * (g.n - 1) / 2);
  // centre-of-mass stop (md.f90:116-121, :186-216): 3 or 6 fewer, taken from the
  // sub-systems of the first molecule in proportion to their DOF
  if (prm->stop_center >= JP_STOP_TRANS && prm->stop_center <= JP_STOP_BOTH) {
    int iatm = n;   // leading atoms with atom 1's molecule id
    if (s->molecule) {
      iatm = 1;
      while (iatm < n && s->molecule[iatm] == s->molecule[0]) ++iatm;
    }
    c->stop_n = prm->stop_natom > 0 ? prm->stop_natom : iatm;
    const int drop = prm->stop_center == JP_STOP_BOTH ? 6 : 3;
    c->idnfre -= drop;
    int ifrg = 0;
    for (int i = 0; i < iatm; ++i) ifrg = std::max(ifrg, c->mol[i] + 1);
    if (ifrg >= 2) {
      double sum = 0.0;
      for (int q = 0; q < ifrg; ++q) sum += c->nfrmol[q];
      std::vector<double> ratio(ifrg);
      for (int q = 0; q < ifrg; ++q) ratio[q] = c->nfrmol[q] / sum;
      for (int q = 0; q < ifrg; ++q) c->nfrmol[q] -= drop * ratio[q];
    } else {
      c->nfrmol[0] -= drop;
    }
  }
  // lambda: mass (inpcls.f90:350-360) and its degree of freedom (md.f90:122-123, :220-228)
  if (c->alsd) {
    c->lam = prm->lambda0;
    c->lam_v = 0.0;
    c->lam_m = prm->lambda_mass;
    if (!(c->lam_m > 0.0)) {
      c->lam_m = 0.0;
      for (int i = 0; i < n; ++i) if (c->inA[i]) c->lam_m += c->mass[i];
    }
    c->lam_im = c->lam_m > 0.0 ? 1.0 / c->lam_m : 0.0;
    c->lam_tc = prm->lambda_temp_control != 0;
    c->lam_dof = c->lam_tc && prm->method == JP_METHOD_GE;
    if (c->lam_dof) {
      c->idnfre += 1;
      int best = 0;
      for (int s2 = 1; s2 < c->nsub; ++s2) if (c->nfrmol[s2] > c->nfrmol[best]) best = s2;
      c->ifg_lambda = best;
      c->nfrmol[best] += 1.0;
    }
  }
  // CMM geometry (incel.f90:29-57): rlim = CUTLEN, level sizes, nlev raised to the extent
  c->cmm = prm->cal15m == JP_CAL15M_CMM;
  if (c->cmm) {
    double ext = 0.0;
    for (int k = 0; k < 3; ++k) {
      double lo = s->cord[k], hi = s->cord[k];
      for (int i = 1; i < n; ++i) {
        lo = std::min(lo, s->cord[3 * i + k]);
        hi = std::max(hi, s->cord[3 * i + k]);
      }
      ext = std::max(ext, hi - lo);
    }
    int nlev = prm->cmm_levels;
    const double cminsiz = prm->cmm_cell;
    if (std::ldexp(1.0, nlev + 1) * cminsiz < ext)
      nlev = (int)std::ceil(std::log(ext / cminsiz) / std::log(2.0) - 1.0);
    c->nlev = nlev;
    for (int l = 1; l <= nlev; ++l) {
      c->nv[l] = 4 << (nlev - l);
      c->siz[l] = cminsiz * (double)(1 << (l - 1));
    }
    c->idelay = (int)std::ceil(c->rc / c->siz[1]);
    c->itwin = true;
    if (s->ext_cmm) {   // setextCMM.f90: the file's level-1 cells on this grid
      const int nc = c->nv[1] * c->nv[1] * c->nv[1];
      c->ext = true;
      for (int k = 0; k < 3; ++k) c->ext_c0[k] = s->ext_cmm->center[k];
      c->ext_flag.assign(s->ext_cmm->flag, s->ext_cmm->flag + nc);
      c->ext_pot.assign(s->ext_cmm->pot, s->ext_cmm->pot + (size_t)13 * nc);
    }
  }
  // state
  c->cord.assign(s->cord, s->cord + 3 * n);
  c->vel.assign(3 * n, 0.0);
  if (s->vel) c->vel.assign(s->vel, s->vel + 3 * n);
  c->grad.assign(3 * n, 0.0);
  build_list(*c);
  return c;
}

void or_destroy(void* h) { delete (Ctx*)h; }

void or_set_state(void* h, const double* cord, const double* vel) {
  Ctx* c = (Ctx*)h;
  if (cord) std::memcpy(c->cord.data(), cord, sizeof(double) * 3 * c->n);
  if (vel) std::memcpy(c->vel.data(), vel, sizeof(double) * 3 * c->n);
}

void or_get_state(void* h, double* cord, double* vel) {
  Ctx* c = (Ctx*)h;
  if (cord) std::memcpy(cord, c->cord.data(), sizeof(double) * 3 * c->n);
  if (vel) std::memcpy(vel, c->vel.data(), sizeof(double) * 3 * c->n);
}

void or_rebuild(void* h) { build_list(*(Ctx*)h); }

long long or_npairs_listed(void* h) {
  Ctx* c = (Ctx*)h;
  long long s = 0;
  for (auto& L : c->nb) s += (long long)L.size();
  return s;
}

long long or_npairs_cut(void* h) { return ((Ctx*)h)->npair_last; }

double or_dself(void* h) { return ((Ctx*)h)->dself; }
int or_dof(void* h) { return ((Ctx*)h)->idnfre; }

int or_energy_grad(void* h, const double* cord, double* ene, double* grad) {
  Ctx* c = (Ctx*)h;
  if (cord) std::memcpy(c->cord.data(), cord, sizeof(double) * 3 * c->n);
  const bool keep = c->itwin;
  c->itwin = true;   // a single-point evaluation takes the far field at these coordinates
  energy_grad(*c, c->cord.data(), ene, grad);
  c->itwin = keep;   // and leaves the step loop's far-field cadence as it was
  return 0;
}

// CMM state of level l (1-based): returns nv (0 without CMM); pot [nv^3][13], pop [nv^3],
// cen [nv][3] (each nullable).  Test hook.
// dnergy's per-class outputs: enevcc(1, 1:nfrg) and grad(3, N, 1:nfrg) (unscaled), one
// evaluation per class with the class weights set to that class; returns nfrg
int or_energy_grad_cls(void* h, const double* cord, double* ene, double* ecls, double* grad) {
  Ctx& c = *(Ctx*)h;
  if (cord) std::copy(cord, cord + 3 * c.n, c.cord.begin());
  const int nfrg = c.alsd ? 3 : c.split ? 2 : 1;
  const int slot[3][3] = {{2, 2, 2}, {0, 2, 2}, {0, 1, 2}};
  std::vector<double> g((size_t)3 * c.n);
  for (int q = 0; q < nfrg; ++q) {
    const int k = slot[nfrg - 1][q];
    c.fover = true;
    for (int z = 0; z < 3; ++z) c.fo[z] = z == k ? 1.0 : 0.0;
    if (nfrg == 1) c.fo[0] = c.fo[1] = c.fo[2] = 1.0;
    energy_grad(c, c.cord.data(), ene, g.data());
    c.fover = false;
    if (ecls) ecls[q] = nfrg == 1 ? ene[JP_E_TOTAL] : c.ecls[k];
    if (grad) std::copy(g.begin(), g.end(), grad + (size_t)q * 3 * c.n);
  }
  return nfrg;
}

int or_cmm_level(void* h, int l, double* pot, int* pop, double* cen) {
  Ctx* c = (Ctx*)h;
  if (!c->cmm || l < 1 || l > c->nlev) return 0;
  const size_t nc = (size_t)c->nv[l] * c->nv[l] * c->nv[l];
  if (pot) std::memcpy(pot, c->pot[l].data(), sizeof(double) * 13 * nc);
  if (pop) std::memcpy(pop, c->pop[l].data(), sizeof(int) * nc);
  if (cen) std::memcpy(cen, c->cen[l].data(), sizeof(double) * 3 * c->nv[l]);
  return c->nv[l];
}

int or_cmm_nlev(void* h) { return ((Ctx*)h)->cmm ? ((Ctx*)h)->nlev : 0; }

// far-field energy of the last force call; gwk (nullable) [natom][3] its gradient.
// Test hook.
double or_cmm_far(void* h, double* gwk) {
  Ctx* c = (Ctx*)h;
  if (!c->cmm) return 0.0;
  if (gwk) std::memcpy(gwk, c->gwk.data(), sizeof(double) * 3 * c->n);
  return c->ecmm;
}

int or_shake(void* h, double* r1, const double* r2) { return shake_all(*(Ctx*)h, r1, r2); }

// what md_run's FDEBUG dumps to 1stp_force.bin at the first step (verlethe.f90:382-387):
// eneval, lambda_f and the gradient after verlethe's scaling, at the current coordinates
// (METHOD= CANO / GE; MICR and CONS have no dump: the plain gradient and lambda_f = 0)
void or_first_force(void* h, double* ene, double* lambda_f, double* grad) {
  Ctx* c = (Ctx*)h;
  const bool keep = c->itwin;
  c->itwin = true;
  double lf = 0.0;
  if (c->prm.method >= JP_METHOD_CANO) lf = verlethe_force(*c, ene);
  else energy_grad(*c, c->cord.data(), ene, c->grad.data());
  c->itwin = keep;
  if (lambda_f) *lambda_f = lf;
  if (grad) std::memcpy(grad, c->grad.data(), sizeof(double) * 3 * c->n);
}

double or_temperature(void* h, const double* v) {
  Ctx* c = (Ctx*)h;
  return caltmp(*c, v ? v : c->vel.data());
}

// steepest-descent minimisation: steep (steep.f90:2-92) with linsrd (:98-246), RMS gradient
// by calrsf (calrsf.f90), search direction by mksrdg (-grad / |grad|).  All atoms variable;
// returns ier (0, steep's -2 for a vanishing step, SHAKE's code); iters, ene, rmsf, state
// (0 loop limit, 1 converged, 2 step too small) describe the end.
int or_minimize(void* h, int max_loop, int update, double convgr, double step0, double up, double down,
                int* iters, double* ene_out, double* rmsf_out, int* state) {
  Ctx* c = (Ctx*)h;
  const int n = c->n;
  double* x = c->cord.data();
  std::vector<double> g(3 * (size_t)n), xref;
  double ene[JP_MAXENE];
  auto evaluate = [&]() {
    c->itwin = true;
    energy_grad(*c, x, ene, g.data());
  };
  auto gsum = [&]() {
    double s2 = 0.0;
    for (double v : g) s2 += v * v;
    return s2;
  };
  evaluate();
  double stp = step0 * std::sqrt((double)n);
  int iloop = 0, ier = 0, st = 0;
  double rmsf = std::sqrt(gsum() / n);
  const bool shake = c->prm.shake_method != JP_SHAKE_NONE && !(c->sk2.empty() && c->sk3.empty() && c->sk4.empty());
  for (;;) {
    if (rmsf <= convgr) { st = 1; break; }
    const double conv = -1.0 / std::sqrt(gsum());
    const double epold = ene[JP_E_TOTAL];
    if (shake) xref.assign(x, x + 3 * (size_t)n);
    for (int k = 0; k < 3 * n; ++k) x[k] += stp * conv * g[k];
    if (shake) {
      ier = shake_all(*c, x, xref.data());
      if (ier != 0) break;
    }
    ++iloop;
    evaluate();
    rmsf = std::sqrt(gsum() / n);
    if (ene[JP_E_TOTAL] < epold) {
      stp *= up;
    } else {
      stp *= down;
      if (stp / std::sqrt(3.0 * n) < kEps) { st = 2; ier = -2; break; }
    }
    if (update > 0 && iloop % update == 0) build_list(*c);
    if (iloop == max_loop) break;
  }
  if (iters) *iters = iloop;
  if (ene_out) std::memcpy(ene_out, ene, sizeof(ene));
  if (rmsf_out) *rmsf_out = rmsf;
  if (state) *state = st;
  build_list(*c);
  return ier;
}

// conjugate-gradient minimisation: conj (conj.f90:2-116) -- search directions by mksrdc
// (:122-216: steepest descent, then Powell's restart scheme, mksdc2 starting a restart
// cycle and mksdc1 continuing it, back to steepest descent whenever a direction is not
// downhill) and the line search linsrc (:465-658: doubling until the directional
// derivative changes sign, then secant steps; stop at |g.d| <= fncovl |g.d at the start|
// or after inllpl evaluations).  SHAKE is refused (conj.f90:48-53).  Returns ier (0, or
// -1 with SHAKE groups); iters, ene, rmsf, state (0 loop limit, 1 converged).
int or_minimize_conj(void* h, int max_loop, int update, double convgr, double step0, double line_conv,
                     int line_max, int* iters, double* ene_out, double* rmsf_out, int* state) {
  Ctx* c = (Ctx*)h;
  if (c->prm.shake_method != JP_SHAKE_NONE && !(c->sk2.empty() && c->sk3.empty() && c->sk4.empty()))
    return -1;
  const int n = c->n, m = 3 * n;
  double* x = c->cord.data();
  std::vector<double> g(m), grado(m, 0.0), difgrd(m, 0.0), d(m, 0.0), dold(m, 0.0), drst(m, 0.0),
      trycor(m);
  double ene[JP_MAXENE];
  auto evaluate = [&]() {
    c->itwin = true;
    energy_grad(*c, x, ene, g.data());
  };
  auto dot = [&](const std::vector<double>& a, const std::vector<double>& b) {
    double s2 = 0.0;
    for (int k = 0; k < m; ++k) s2 += a[k] * b[k];
    return s2;
  };
  auto normalise = [&](std::vector<double>& v) {
    const double r = 1.0 / std::sqrt(dot(v, v));
    for (double& w : v) w *= r;
  };
  evaluate();
  double stplen = step0 * std::sqrt((double)n), dtdifg = 0.0;
  int ifsrdr = 1, insrdr = 0, inrsdr = 0, iloop = 0, inloop = 0, st = 0;
  double rmsf = std::sqrt(dot(g, g) / n);
  for (;;) {
    // mksrdc
    double dirgrd;
    for (;;) {
      if (ifsrdr == 2 && std::fabs(dot(grado, g)) / dot(g, g) >= 0.2) ifsrdr = 3;
      if (ifsrdr == 1) {   // mksrdg
        const double conv = -1.0 / std::sqrt(dot(g, g));
        for (int k = 0; k < m; ++k) d[k] = conv * g[k];
        dold = d;
      } else if (ifsrdr == 2) {   // mksdc1
        dold = d;
        double beta = 0.0, rss = 0.0, ganma = 0.0;
        for (int k = 0; k < m; ++k) {
          const double dif = g[k] - grado[k];
          beta += g[k] * dif;
          rss += dold[k] * dif;
          ganma += g[k] * difgrd[k];
        }
        if (rss != 0.0) {
          beta /= rss;
          ganma /= dtdifg;
          for (int k = 0; k < m; ++k) d[k] = beta * dold[k] + ganma * drst[k] - g[k];
          normalise(d);
        }
      } else {   // mksdc2
        dold = d;
        drst = d;
        double beta = 0.0, rss = 0.0;
        for (int k = 0; k < m; ++k) {
          difgrd[k] = g[k] - grado[k];
          beta += g[k] * difgrd[k];
          rss += dold[k] * difgrd[k];
        }
        dtdifg = rss;
        if (rss != 0.0) {
          beta /= rss;
          for (int k = 0; k < m; ++k) d[k] = beta * dold[k] - g[k];
          normalise(d);
        }
        inrsdr = insrdr;
      }
      dirgrd = dot(g, d);   // chksrd
      if (dirgrd < 0.0) break;
      ifsrdr = 1;
    }
    insrdr += 1;
    if (ifsrdr == 1) ifsrdr = 3;
    else if (ifsrdr == 3) ifsrdr = 2;
    if (insrdr - inrsdr == 3 * n) ifsrdr = 3;
    grado = g;
    // linsrc
    const double dirgrs = dirgrd;
    bool onfind = false, stop = false;
    int jloop = 0;
    double dirgrn = dirgrs, stplnn = 0.0, stplnp = 0.0, dirgrp = 0.0;
    trycor.assign(x, x + m);
    for (;;) {
      if (iloop != 0 && update > 0 && inloop % update == 0) build_list(*c);
      for (int k = 0; k < m; ++k) x[k] = trycor[k] + stplen * d[k];
      ++inloop; ++iloop; ++jloop;
      evaluate();
      const double dg = dot(g, d);
      rmsf = std::sqrt(dot(g, g) / n);
      if (rmsf <= convgr) { st = 1; stop = true; break; }
      if (iloop >= max_loop) { stop = true; break; }
      if (jloop == line_max) break;
      if (std::fabs(dg / dirgrs) <= line_conv) break;
      if (!onfind) {
        if (dg < 0.0) {
          stplnn = stplen; dirgrn = dg;
          stplen = stplnn * 2.0;
        } else {
          onfind = true;
          stplnp = stplen; dirgrp = dg;
          stplen = stplnn - (stplnp - stplnn) / (dirgrp - dirgrn) * dirgrn;
        }
      } else {
        if (dg < 0.0) { stplnn = stplen; dirgrn = dg; }
        else { stplnp = stplen; dirgrp = dg; }
        stplen = stplnn - (stplnp - stplnn) / (dirgrp - dirgrn) * dirgrn;
      }
    }
    if (stop) break;
  }
  if (iters) *iters = iloop;
  if (ene_out) std::memcpy(ene_out, ene, sizeof(ene));
  if (rmsf_out) *rmsf_out = rmsf;
  if (state) *state = st;
  build_list(*c);
  return 0;
}

// nsteps of runmd (md.f90:519-694): verlet or verlethe, then celprp every UPDATE steps.
int or_run(void* h, int nsteps, double* ene_out, double* temp_out) {
  Ctx* c = (Ctx*)h;
  double ene[JP_MAXENE];
  for (int s = 0; s < nsteps; ++s) {
    c->idloop += 1;
    int ier;
    if (c->prm.method <= JP_METHOD_MICR) ier = step_verlet(*c, ene);
    else ier = step_verlethe(*c, ene);
    if (ier != 0) return ier;
    if (ene_out) std::memcpy(ene_out + (size_t)s * JP_MAXENE, ene, sizeof(ene));
    if (temp_out) temp_out[s] = caltmp(*c, c->vel.data());
    if (c->prm.update > 0 && c->idloop % c->prm.update == 0) {
      build_list(*c);
      if (c->cmm_err) return c->cmm_err;
    }
    // CMM far-field marker for the next step (md.f90:680-684)
    if (c->cmm) c->itwin = c->idloop % c->prm.cmm_update == 0;
  }
  return 0;
}

double or_mcmd_scale(void* h, double e) { return mcmd_scale(*(Ctx*)h, e); }

// remotv on a given velocity set (in/out) with positions xp; returns ier (0, -1, -2).
// Test hook.
int or_remotv(void* h, const double* xp, double* vel) {
  Ctx* c = (Ctx*)h;
  std::vector<double> keep(c->vel);
  std::memcpy(c->vel.data(), vel, sizeof(double) * 3 * c->n);
  const int ier = remotv(*c, xp);
  std::memcpy(vel, c->vel.data(), sizeof(double) * 3 * c->n);
  c->vel.swap(keep);
  return ier;
}

// DOF of each sub-system (nfrmol); returns their number
int or_nfrmol(void* h, double* out) {
  Ctx* c = (Ctx*)h;
  if (out) std::memcpy(out, c->nfrmol.data(), sizeof(double) * c->nsub);
  return c->nsub;
}

void or_get_lambda(void* h, double* lam2, double* ecls) {
  Ctx* c = (Ctx*)h;
  if (lam2) { lam2[0] = c->lam; lam2[1] = c->lam_v; }
  if (ecls) for (int k = 0; k < 3; ++k) ecls[k] = c->ecls[k];
}

void or_set_lambda(void* h, double lam, double lam_v) {
  Ctx* c = (Ctx*)h;
  c->lam = lam;
  c->lam_v = lam_v;
}

}  // extern "C"
