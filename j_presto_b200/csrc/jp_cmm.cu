// jp_cmm.cu -- cell multipole method (CAL15M= CMM, BOUNDA= NO): cells and multipoles at a
// list rebuild, far field of a step.
//
// Replaces celpar_CB (src_md_run/celpar.f90:36-116: cells re-centred on the atoms'
// centroid), celoth (celoth.f90: level populations), celpol (celpol.f90: level-1 moments
// about the cell centres from the raw charges, then level-to-level translation) and the
// far-field part of cmmdo (cmmdo.f90:80-170, compute_particle_multipole :181-290) over the
// interaction lists of mk_cm (incel.f90:1098-1240).  The near field (neighbouring level-1
// cells, plus LJ out to CUTLEN) is the tile pair kernel with CMM masks (jp_cells.cu,
// jp_pair.cu).
//
// Geometry: level l has nv[l] = 4 * 2^(nlev-l) cells of edge siz[l] = CELSIZ * 2^(l-1) per
// axis, centres siz[l] * (i - (nv[l]+1)/2) + centroid (i = 1..nv[l]); an atom's level-1
// index is int((x - (centre_1 - siz[1]/2)) / siz[1]) + 1.  Multipole layout per cell (13):
// [q, p_x, p_y, p_z, Q_xx/2, Q_yy/2, Q_zz/2, Q_xx, Q_yy, Q_zz, Q_xy, Q_yz, Q_zx] with the
// traceless Q_ab = sum q (3 d_a d_b - d^2 delta_ab).
//
// One thread per atom (assignment, far field) or per cell (moments, translation).  Sums into
// a cell are FP64 atomics (their order varies in the last bits); the far-field energy is
// reduced per warp and added in 64-bit fixed point.
#include "jp_kernels.h"

namespace jp {

constexpr int kCmmRaw = 10;   // level-1 raw sums per cell

__device__ __forceinline__ double cmm_cen(const Rep& R, const double* c0, int l, int i, int k) {
  const double r = -0.5 * (R.nv[l] + 1);
  return R.siz[l] * ((double)i + r) + c0[k];
}

// the grid centre: the atoms' centroid at the last rebuild, or the external environment's
__device__ __forceinline__ void cmm_centroid(const DevPtrs& P, const Rep& R, int rep, double* c0) {
  const double rtmp = 1.0 / (double)R.natom;
  for (int k = 0; k < 3; ++k) c0[k] = R.ext ? R.ext_c0[k] : __ldcg(&P.cmm_c0[3 * rep + k]) * rtmp;
}

// replica and local index of global cell g of level l (-1: no CMM replica holds it)
__device__ int cmm_cell_rep(const DevPtrs& P, int nrep, int l, int g, int& local) {
  for (int r = 0; r < nrep; ++r) {
    const Rep& R = P.reps[r];
    if (!R.cmm || l > R.nlev) continue;
    const int n = R.nv[l] * R.nv[l] * R.nv[l];
    if (g >= R.cell_off[l] && g < R.cell_off[l] + n) {
      local = g - R.cell_off[l];
      return r;
    }
  }
  return -1;
}

__global__ void k_cmm_centroid(DevPtrs P, int natom) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const int rep = P.rep_of[a];
  if (!P.reps[rep].cmm || P.reps[rep].ext) return;
  for (int k = 0; k < 3; ++k) atomicAdd(&P.cmm_c0[3 * rep + k], P.x[3 * a + k]);
}

// level-1 cell of each atom (celpar.f90:90-116), its population and raw moments
__global__ void k_cmm_assign(DevPtrs P, int natom) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const int rep = P.rep_of[a];
  const Rep& R = P.reps[rep];
  if (!R.cmm) return;
  double c0[3];
  cmm_centroid(P, R, rep, c0);
  const int nv1 = R.nv[1];
  const double half = R.siz[1] * 0.5, rr = 1.0 / R.siz[1];
  int m[3];
  double x[3];
  bool bad = false;
  // CELRES: the cell of the residue's geometric centre (celpar.f90:131-153)
  const int2 res = P.cmm_res ? P.cmm_res[a] : make_int2(-1, -1);
  double p[3];
  for (int k = 0; k < 3; ++k) {
    x[k] = P.x[3 * a + k];
    p[k] = x[k];
  }
  if (res.x >= 0) {
    for (int k = 0; k < 3; ++k) p[k] = 0.0;
    for (int b = res.x; b <= res.y; ++b)
      for (int k = 0; k < 3; ++k) p[k] += P.x[3 * b + k];
    const double inv = 1.0 / (double)(res.y - res.x + 1);
    for (int k = 0; k < 3; ++k) p[k] *= inv;
  }
  for (int k = 0; k < 3; ++k) {
    const double org = cmm_cen(R, c0, 1, 1, k) - half;
    const double u = (p[k] - org) * rr;
    m[k] = (u > -1.0 && u < (double)nv1) ? (int)u + 1 : 0;   // int(): toward zero
    bad |= m[k] < 1 || m[k] > nv1;
  }
  if (bad) {
    atomicOr(P.status, ERR_CMM_GRID);
    P.cmm_cell[a] = -1;
    return;
  }
  P.cmm_cell[a] = (m[0] - 1) | ((m[1] - 1) << 8) | ((m[2] - 1) << 16);
  const int cell = R.cell_off[1] + ((m[2] - 1) * nv1 + (m[1] - 1)) * nv1 + (m[0] - 1);
  atomicAdd(&P.cmm_pop[cell], 1);
  const double q = P.chg[a];
  double d[3];
  for (int k = 0; k < 3; ++k) d[k] = x[k] - cmm_cen(R, c0, 1, m[k], k);
  const double dxx = d[0] * d[0], dyy = d[1] * d[1], dzz = d[2] * d[2];
  const double v[kCmmRaw] = {q, q * d[0], q * d[1], q * d[2],
                             q * (2 * dxx - dyy - dzz), q * (2 * dyy - dzz - dxx),
                             q * (2 * dzz - dxx - dyy), q * d[0] * d[1], q * d[1] * d[2],
                             q * d[2] * d[0]};
  double* raw = P.cmm_raw + (size_t)cell * kCmmRaw;
  for (int k = 0; k < kCmmRaw; ++k) atomicAdd(&raw[k], v[k]);
}

// level-1 coefficients from the raw sums (celpol.f90:27-80)
__global__ void k_cmm_level1(DevPtrs P, int ncell1) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= ncell1) return;
  const double* r = P.cmm_raw + (size_t)g * kCmmRaw;
  double* q = P.cmm_pot + (size_t)g * 13;
  if (P.cmm_pop[g] == 0) {
    for (int k = 0; k < 13; ++k) q[k] = 0.0;
    return;
  }
  const double v[13] = {r[0], r[1], r[2], r[3], r[4] * 0.5, r[5] * 0.5, r[6] * 0.5,
                        r[4], r[5], r[6], r[7] * 3.0, r[8] * 3.0, r[9] * 3.0};
  for (int k = 0; k < 13; ++k) q[k] = v[k];
}

// level l-1 -> l (celoth.f90 populations, celpol.f90:84-460 translation): the 8 children in
// celpol's order (x fastest), each shifted from its centre to the parent's
__global__ void k_cmm_m2m(DevPtrs P, int nrep, int l, int ncell_l, int cell_base) {
  const int g = cell_base + blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= cell_base + ncell_l) return;
  int local = 0;
  const int rep = cmm_cell_rep(P, nrep, l, g, local);
  if (rep < 0) return;
  const Rep& R = P.reps[rep];
  const int nv = R.nv[l], nc = R.nv[l - 1];
  const int ix = local % nv + 1, iy = (local / nv) % nv + 1, iz = local / (nv * nv) + 1;
  double c0[3];
  cmm_centroid(P, R, rep, c0);
  const double px = cmm_cen(R, c0, l, ix, 0), py = cmm_cen(R, c0, l, iy, 1), pz = cmm_cen(R, c0, l, iz, 2);
  int pop = 0;
  double qz = 0, rx = 0, ry = 0, rz = 0, rxx = 0, ryy = 0, rzz = 0, rxy = 0, ryz = 0, rzx = 0;
  for (int jj = 0; jj < 8; ++jj) {
    const int mx = 2 * ix - 1 + (jj & 1), my = 2 * iy - 1 + ((jj >> 1) & 1), mz = 2 * iz - 1 + ((jj >> 2) & 1);
    const int cid = R.cell_off[l - 1] + ((mz - 1) * nc + (my - 1)) * nc + (mx - 1);
    const int np = P.cmm_pop[cid];
    if (np == 0) continue;
    pop += np;
    const double* p = P.cmm_pot + (size_t)cid * 13;
    const double qq = p[0];
    qz += qq;
    const double xx = cmm_cen(R, c0, l - 1, mx, 0) - px;
    const double yy = cmm_cen(R, c0, l - 1, my, 1) - py;
    const double zz = cmm_cen(R, c0, l - 1, mz, 2) - pz;
    const double ax = p[1], ay = p[2], az = p[3];
    rx += ax + qq * xx;
    ry += ay + qq * yy;
    rz += az + qq * zz;
    const double dxx = xx * xx, dyy = yy * yy, dzz = zz * zz;
    const double xax = xx * ax, yay = yy * ay, zaz = zz * az;
    rxx += p[4] + 2 * xax - yay - zaz + qq * (dxx - 0.5 * (dyy + dzz));
    ryy += p[5] + 2 * yay - zaz - xax + qq * (dyy - 0.5 * (dzz + dxx));
    rzz += p[6] + 2 * zaz - xax - yay + qq * (dzz - 0.5 * (dxx + dyy));
    rxy += p[10] * 0.5 + (yy * ax + xx * ay + xx * yy * qq) * 1.5;
    ryz += p[11] * 0.5 + (zz * ay + yy * az + yy * zz * qq) * 1.5;
    rzx += p[12] * 0.5 + (xx * az + zz * ax + zz * xx * qq) * 1.5;
  }
  P.cmm_pop[g] = pop;
  double* q = P.cmm_pot + (size_t)g * 13;
  if (pop == 0) {
    for (int k = 0; k < 13; ++k) q[k] = 0.0;
    return;
  }
  const double v[13] = {qz, rx, ry, rz, rxx, ryy, rzz, rxx * 2.0, ryy * 2.0, rzz * 2.0,
                        rxy * 2.0, ryz * 2.0, rzx * 2.0};
  for (int k = 0; k < 13; ++k) q[k] = v[k];
}

void launch_cmm_rebuild(const DevPtrs& P, int natom, int nrep, int ncell1, const int* ncell_lvl,
                        int nlev_max, cudaStream_t st) {
  const int nt = 256;
  k_cmm_centroid<<<(natom + nt - 1) / nt, nt, 0, st>>>(P, natom);
  k_cmm_assign<<<(natom + nt - 1) / nt, nt, 0, st>>>(P, natom);
  k_cmm_level1<<<(ncell1 + nt - 1) / nt, nt, 0, st>>>(P, ncell1);
  int base = ncell1;
  for (int l = 2; l <= nlev_max; ++l) {
    const int n = ncell_lvl[l];
    if (n > 0) k_cmm_m2m<<<(n + nt - 1) / nt, nt, 0, st>>>(P, nrep, l, n, base);
    base += n;
  }
}

// far field of one atom (cmmdo.f90:181-290): the multipole expansion of every non-empty far
// cell at every level; returns sum over levels of the potential, gradient in g (per unit
// charge of the atom)
__device__ double cmm_far_atom(const DevPtrs& P, const Rep& R, const double* c0, int cell,
                               const double* x, double* g) {
  int a[3] = {(cell & 255) + 1, ((cell >> 8) & 255) + 1, ((cell >> 16) & 255) + 1};
  double e = 0.0;
  g[0] = g[1] = g[2] = 0.0;
  for (int l = 1; l <= R.nlev; ++l) {
    if (l > 1)
      for (int k = 0; k < 3; ++k) a[k] = (a[k] + 1) / 2;
    const int m = R.nv[l];
    int lo[3], hi[3], nlo[3], nhi[3];
    for (int k = 0; k < 3; ++k) {
      nlo[k] = max(1, a[k] - 1);
      nhi[k] = min(m, a[k] + 1);
      if (l < R.nlev) {   // children of the parent's neighbours (mk_cm)
        const int p = (a[k] + 1) / 2, m1 = R.nv[l + 1];
        lo[k] = max(1, p - 1) * 2 - 1;
        hi[k] = min(m1, p + 1) * 2;
      } else {            // top level: every cell
        lo[k] = 1;
        hi[k] = m;
      }
    }
    for (int kz = lo[2]; kz <= hi[2]; ++kz) {
      const double dz = x[2] - cmm_cen(R, c0, l, kz, 2);
      const bool nz = kz >= nlo[2] && kz <= nhi[2];
      for (int ky = lo[1]; ky <= hi[1]; ++ky) {
        const double dy = x[1] - cmm_cen(R, c0, l, ky, 1);
        const bool nyz = nz && ky >= nlo[1] && ky <= nhi[1];
        for (int kx = lo[0]; kx <= hi[0]; ++kx) {
          if (nyz && kx >= nlo[0] && kx <= nhi[0]) continue;
          const int id = R.cell_off[l] + ((kz - 1) * m + (ky - 1)) * m + (kx - 1);
          if (__ldg(&P.cmm_pop[id]) == 0) continue;
          const double* q = P.cmm_pot + (size_t)id * 13;
          const double dx = x[0] - cmm_cen(R, c0, l, kx, 0);
          const double dx2 = dx * dx, dy2 = dy * dy, dz2 = dz * dz;
          const double dd2i = 1.0 / (dx2 + dy2 + dz2);
          const double ddi = sqrt(dd2i);
          const double dd3i = ddi * dd2i, dd5i = dd3i * dd2i;
          const double aa1 = q[1] * dx + q[2] * dy + q[3] * dz;
          const double aa2 = q[4] * dx2 + q[5] * dy2 + q[6] * dz2 + q[10] * dx * dy + q[11] * dy * dz +
                             q[12] * dz * dx;
          e += q[0] * ddi + aa1 * dd3i + aa2 * dd5i;
          const double c4 = aa1 * 3.0 + aa2 * dd2i * 5.0;
          g[0] += -(q[0] * dx - q[1]) * dd3i + (q[7] * dx + q[10] * dy + q[12] * dz - c4 * dx) * dd5i;
          g[1] += -(q[0] * dy - q[2]) * dd3i + (q[10] * dx + q[8] * dy + q[11] * dz - c4 * dy) * dd5i;
          g[2] += -(q[0] * dz - q[3]) * dd3i + (q[12] * dx + q[11] * dy + q[9] * dz - c4 * dz) * dd5i;
        }
      }
    }
  }
  return e;
}

// external environment of one atom (enear_extCMM.f90:58-164): the occupied external cells
// among its level-1 cell and the 26 around it; within R = 1.5 cell sizes of a cell centre the
// expansion on that sphere, blended inward by a cubic in r.  Returns the energy per unit
// charge (before md_run's factor 0.5), gradient per unit charge in g.
__device__ double cmm_ext_atom(const DevPtrs& P, const Rep& R, const double* c0, int cell,
                               const double* x, double* g) {
  const int nv1 = R.nv[1];
  const int mx = (cell & 255) + 1, my = ((cell >> 8) & 255) + 1, mz = ((cell >> 16) & 255) + 1;
  const double RR = 1.5 * R.siz[1], RR2 = RR * RR, RR_2 = 3.0 * R.siz[1];
  const double iRR = 1.0 / RR, iRR3 = iRR * iRR * iRR, iRR5 = iRR3 * iRR * iRR;
  const double i3RR5 = 3.0 * iRR5, i5RR7 = 5.0 * iRR5 * iRR * iRR;
  double e = 0.0;
  g[0] = g[1] = g[2] = 0.0;
  for (int jz = max(1, mz - 1); jz <= min(nv1, mz + 1); ++jz)
    for (int jy = max(1, my - 1); jy <= min(nv1, my + 1); ++jy)
      for (int jx = max(1, mx - 1); jx <= min(nv1, mx + 1); ++jx) {
        const int id = R.cell_off[1] + ((jz - 1) * nv1 + (jy - 1)) * nv1 + (jx - 1);
        if (!P.ext_flag[id]) continue;
        const double* q = P.ext_pot + (size_t)id * 13;
        double dx = x[0] - cmm_cen(R, c0, 1, jx, 0);
        double dy = x[1] - cmm_cen(R, c0, 1, jy, 1);
        double dz = x[2] - cmm_cen(R, c0, 1, jz, 2);
        const double dd2 = dx * dx + dy * dy + dz * dz;
        double ec, f[3];
        if (dd2 < RR2) {
          const double scal = sqrt(RR2 / dd2);
          dx *= scal; dy *= scal; dz *= scal;
          const double aa1 = q[1] * dx + q[2] * dy + q[3] * dz;
          const double aa2 = q[4] * dx * dx + q[5] * dy * dy + q[6] * dz * dz + q[10] * dx * dy +
                             q[11] * dy * dz + q[12] * dz * dx;
          const double e0 = q[0] * iRR + aa1 * iRR3 + aa2 * iRR5;
          const double c4 = aa1 * i3RR5 + aa2 * i5RR7;
          f[0] = -(q[0] * dx - q[1]) * iRR3 + (q[7] * dx + q[10] * dy + q[12] * dz) * iRR5 - c4 * dx;
          f[1] = -(q[0] * dy - q[2]) * iRR3 + (q[10] * dx + q[8] * dy + q[11] * dz) * iRR5 - c4 * dy;
          f[2] = -(q[0] * dz - q[3]) * iRR3 + (q[12] * dx + q[11] * dy + q[9] * dz) * iRR5 - c4 * dz;
          const double fn = sqrt(f[0] * f[0] + f[1] * f[1] + f[2] * f[2]);
          const double r = sqrt(dd2), b = fn * r;
          const double sf = r * iRR3 * (6.0 * e0 * (r - RR) + b * (3.0 * r - RR_2)) / fn;
          for (int k = 0; k < 3; ++k) f[k] *= sf;
          const double t = r * iRR;
          ec = (2.0 * e0 + b) * t * t * t - (3.0 * e0 + b) * t * t + 2.0 * e0;
        } else {
          const double d2i = 1.0 / dd2, di = sqrt(d2i), d3i = di * d2i, d5i = d3i * d2i;
          const double d7i = d5i * d2i;
          const double aa1 = q[1] * dx + q[2] * dy + q[3] * dz;
          const double aa2 = q[4] * dx * dx + q[5] * dy * dy + q[6] * dz * dz + q[10] * dx * dy +
                             q[11] * dy * dz + q[12] * dz * dx;
          ec = q[0] * di + aa1 * d3i + aa2 * d5i;
          const double c4 = aa1 * 3.0 * d5i + aa2 * 5.0 * d7i;
          f[0] = -(q[0] * dx - q[1]) * d3i + (q[7] * dx + q[10] * dy + q[12] * dz) * d5i - c4 * dx;
          f[1] = -(q[0] * dy - q[2]) * d3i + (q[10] * dx + q[8] * dy + q[11] * dz) * d5i - c4 * dy;
          f[2] = -(q[0] * dz - q[3]) * d3i + (q[12] * dx + q[11] * dy + q[9] * dz) * d5i - c4 * dz;
        }
        e += ec;
        for (int k = 0; k < 3; ++k) g[k] += f[k];
      }
  return e;
}

// warp sum of each lane's energy into a replica's fixed-point slot (rep -1: nothing)
__device__ __forceinline__ void warp_energy(const DevPtrs& P, long long* dst, int rep, double e) {
  const unsigned full = 0xffffffffu;
  const unsigned has = __ballot_sync(full, rep >= 0);
  if (has == 0u) return;
  const int r0 = __shfl_sync(full, rep, __ffs(has) - 1);
  if (__all_sync(full, rep < 0 || rep == r0)) {
    double v = rep >= 0 ? e : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(full, v, o);
    if ((threadIdx.x & 31) == 0) atomic_add_ll(&dst[r0], to_fix(v, kEneScale, P.status));
  } else if (rep >= 0) {
    atomic_add_ll(&dst[rep], to_fix(e, kEneScale, P.status));
  }
}

__device__ __forceinline__ bool cmm_due(const DevPtrs& P, const Rep& R, bool force) {
  return force || (P.step_ctr[0] % R.cmm_upd) == 0;
}

// far field of each atom when due (into gwk, energy into cmm_enew), then gwk into the forces
__global__ void k_cmm_far(DevPtrs P, int natom, int fp64, int force, double ccoef) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  int rep = -1, rep_x = -1;
  double e = 0.0, ex = 0.0;
  if (a < natom) {
    const int r = P.rep_of[a];
    const Rep& R = P.reps[r];
    if (R.cmm) {
      const int cell = P.cmm_cell[a];
      const double q2 = ccoef * P.chg[a];   // chgmod2 (inpcls.f90:223)
      double c0[3], x[3], g[3];
      cmm_centroid(P, R, r, c0);
      for (int k = 0; k < 3; ++k) x[k] = P.x[3 * a + k];
      if (cmm_due(P, R, force != 0) && cell >= 0) {
        e = 0.5 * q2 * cmm_far_atom(P, R, c0, cell, x, g);
        for (int k = 0; k < 3; ++k) P.gwk[3 * a + k] = g[k] * q2;
        rep = r;
      }
      if (cell >= 0) {
        double gx[3] = {0.0, 0.0, 0.0};
        if (R.ext) {   // the external environment, every step (cmmdo.f90:82)
          ex = 0.5 * q2 * cmm_ext_atom(P, R, c0, cell, x, gx);
          rep_x = r;
        }
        for (int k = 0; k < 3; ++k) {
          const double gk = P.gwk[3 * a + k] + gx[k] * q2;
          if (fp64) atomicAdd(&P.grd[3 * a + k], gk);
          else atomic_add_ll(&P.frc[3 * a + k], to_fix(gk, kFrcScale, P.status));
        }
      }
    }
  }
  // warp-level energy sums (one replica per warp as a rule; mixed warps add per lane)
  warp_energy(P, P.cmm_enew, rep, e);
  warp_energy(P, P.ene_ext, rep_x, ex);
}

// the far-field energy of the step into ELE15: the new sum when due, else the last one
__global__ void k_cmm_energy(DevPtrs P, int nrep, int force) {
  for (int r = threadIdx.x; r < nrep; r += blockDim.x) {
    const Rep& R = P.reps[r];
    if (!R.cmm) continue;
    if (cmm_due(P, R, force != 0)) {
      P.cmm_e[r] = P.cmm_enew[r];
      P.cmm_enew[r] = 0;
    }
    atomic_add_ll(&P.ene_fix[r * 16 + JP_E_ELE15], P.cmm_e[r] + P.ene_ext[r]);
    P.ene_ext[r] = 0;
  }
}

void launch_cmm_far(const DevPtrs& P, int natom, int nrep, bool fp64, bool force, double ccoef,
                    cudaStream_t st) {
  const int nt = 128;
  k_cmm_far<<<(natom + nt - 1) / nt, nt, 0, st>>>(P, natom, fp64 ? 1 : 0, force ? 1 : 0, ccoef);
  k_cmm_energy<<<1, 128, 0, st>>>(P, nrep, force ? 1 : 0);
}

}  // namespace jp
