// jp_restraint.cu -- restraints and the CAP boundary (dneres.f90, dnecap.f90).
//
//   position  (dposc,  dneres.f90:48-101):  E = 1/2 k |x - ref|^2,       dE/dx = k (x - ref)
//   distance  (ddistc, dneres.f90:107-221): R = <r^-6>^(-1/6) over the pairs of two atom
//             groups; outside [lo, up] E = k (R^2 - r0^2)^2, r0 the crossed bound, and
//             dE/dx_i = 4 k (R^2 - r0^2) R^8 / n  sum_j r_ij^-8 (x_i - x_j)
//   dihedral  (dcdihe, dneres.f90:227-378): phi in [0, 2 pi); outside [lo, up] E =
//             k (phi - wall)^2 measured from the nearer wall (the far one across 2 pi)
//   CAP       (dnecap.f90:80-281 and :428-437): terms on a group's centre of mass (gradient
//             shared by mass) or a listed atom: half-harmonic outside a sphere, outside box
//             walls per coordinate or outside an ellipsoid (iufcap 1), half-biquadratic
//             outside a sphere (iufcap 2)
// Minimum image as in the _PB variants under BOUNDA= PBC; none under BOUNDA= NO (_CB).
// One restraint per thread, FP64 arithmetic on both paths (they are few); forces go to the
// class-BB accumulators with weight 1 (grad(:,:,nfrg)), energies to enevcc(11..14).
#include "jp_kernels.h"

namespace jp {

constexpr int kResThreads = 128;

__device__ __forceinline__ void res_image(const Rep& R, double* d) {
  if (R.free_bnd) return;
  for (int k = 0; k < 3; ++k) d[k] -= R.box[k] * anint(d[k] * R.invbox[k]);
}

template <bool FP64>
__device__ __forceinline__ void res_dist(const DevPtrs& P, const Rep& R, const Restr& Q, double& e,
                                         double wg) {
  const double* x = P.x;
  const int* idx = P.res_idx;
  const int n = (Q.a[1] - Q.a[0]) * (Q.a[3] - Q.a[2]);
  double s6 = 0.0;
  for (int p = Q.a[0]; p < Q.a[1]; ++p)
    for (int q = Q.a[2]; q < Q.a[3]; ++q) {
      double d[3];
      for (int k = 0; k < 3; ++k) d[k] = x[3 * idx[p] + k] - x[3 * idx[q] + k];
      res_image(R, d);
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      s6 += 1.0 / (r2 * r2 * r2);
    }
  const double rave = pow(s6 / (double)n, -1.0 / 6.0);
  const double lo = Q.p[0], up = Q.p[1];
  double r0 = 1.0, k = 0.0;
  if (rave > up) { r0 = up; k = Q.p[3]; }
  else if (rave < lo) { r0 = lo; k = Q.p[2]; }
  const double dr2 = rave * rave - r0 * r0;
  e = k * dr2 * dr2;
  if (rave >= lo && rave <= up) return;
  double r8 = rave * rave;
  r8 *= r8;
  r8 *= r8;
  const double coef = 4.0 * k * dr2 * r8 / (double)n;
  // each atom of either group: coef * sum over the other group of r^-8 (x_self - x_other)
  for (int side = 0; side < 2; ++side) {
    const int a0 = side ? Q.a[2] : Q.a[0], a1 = side ? Q.a[3] : Q.a[1];
    const int b0 = side ? Q.a[0] : Q.a[2], b1 = side ? Q.a[1] : Q.a[3];
    for (int p = a0; p < a1; ++p) {
      double td[3] = {0.0, 0.0, 0.0};
      for (int q = b0; q < b1; ++q) {
        double d[3];
        for (int kk = 0; kk < 3; ++kk) d[kk] = x[3 * idx[p] + kk] - x[3 * idx[q] + kk];
        res_image(R, d);
        double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        r2 *= r2;
        const double r8i = 1.0 / (r2 * r2);
        for (int kk = 0; kk < 3; ++kk) td[kk] += d[kk] * r8i;
      }
      add_grad<FP64>(P, coef * wg, idx[p], td[0], td[1], td[2]);
    }
  }
}

template <bool FP64>
__device__ __forceinline__ void res_dihe(const DevPtrs& P, const Rep& R, const Restr& Q, double& e,
                                         double wg) {
  constexpr double kTwoPi = 2.0 * 3.141592653589793;
  const double* x = P.x;
  double d21[3], d32[3], d43[3];
  for (int k = 0; k < 3; ++k) {
    d21[k] = x[3 * Q.a[1] + k] - x[3 * Q.a[0] + k];
    d32[k] = x[3 * Q.a[2] + k] - x[3 * Q.a[1] + k];
    d43[k] = x[3 * Q.a[3] + k] - x[3 * Q.a[2] + k];
  }
  res_image(R, d21);
  res_image(R, d32);
  res_image(R, d43);
  const double p12[3] = {d21[1] * d32[2] - d32[1] * d21[2], d21[2] * d32[0] - d32[2] * d21[0],
                         d21[0] * d32[1] - d32[0] * d21[1]};
  const double p23[3] = {d32[1] * d43[2] - d43[1] * d32[2], d32[2] * d43[0] - d43[2] * d32[0],
                         d32[0] * d43[1] - d43[0] * d32[1]};
  const double r12 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
  const double r23 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
  double r12r23 = sqrt(r12 * r23);
  if (!(r12r23 > 0.0)) return;   // collinear bonds: no angle, no term
  r12r23 = 1.0 / r12r23;
  const double s1223 = p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2];
  const double cosp = fmin(fmax(s1223 * r12r23, -1.0), 1.0);
  const double p123[3] = {p12[1] * p23[2] - p23[1] * p12[2], p12[2] * p23[0] - p23[2] * p12[0],
                          p12[0] * p23[1] - p23[0] * p12[1]};
  const double s32123 = d32[0] * p123[0] + d32[1] * p123[1] + d32[2] * p123[2];
  double phi = acos(cosp);
  if (s32123 < 0.0) phi = kTwoPi - phi;
  // walls: above up the upper wall and the lower one shifted by 2 pi, below lo the lower
  // wall and the upper one shifted by -2 pi; the nearer of the two counts
  const double lo = Q.p[0], up = Q.p[1];
  double w0 = 0.0, w1 = 0.0, k0 = 0.0, k1 = 0.0;
  if (phi > up) { w0 = up; w1 = lo + kTwoPi; k0 = Q.p[3]; k1 = Q.p[2]; }
  else if (phi < lo) { w0 = up - kTwoPi; w1 = lo; k0 = Q.p[3]; k1 = Q.p[2]; }
  const double dp0 = phi - w0, dp1 = w1 - phi;
  double dphi, kk;
  if (dp0 < dp1) { dphi = dp0; kk = k0; }
  else { dphi = -dp1; kk = k1; }
  e = kk * dphi * dphi;
  if (fabs(phi) < 1.0e-10 || fabs(phi - 0.5 * kTwoPi) < 1.0e-10) return;
  const double wr = -2.0 * kk * dphi / sin(phi) * r12r23;
  const double v1 = d21[0] + d32[0], v2 = d21[1] + d32[1], v3 = d21[2] + d32[2];
  const double q12 = s1223 / r12, q23 = s1223 / r23;
  double w[9];
  w[0] = d32[2] * p23[1] - d32[1] * p23[2] - q12 * (d32[2] * p12[1] - d32[1] * p12[2]);
  w[1] = d32[0] * p23[2] - d32[2] * p23[0] - q12 * (d32[0] * p12[2] - d32[2] * p12[0]);
  w[2] = d32[1] * p23[0] - d32[0] * p23[1] - q12 * (d32[1] * p12[0] - d32[0] * p12[1]);
  w[3] = -v3 * p23[1] + d43[2] * p12[1] + v2 * p23[2] - d43[1] * p12[2] -
         q12 * (-v3 * p12[1] + v2 * p12[2]) - q23 * (d43[2] * p23[1] - d43[1] * p23[2]);
  w[4] = v3 * p23[0] - d43[2] * p12[0] - v1 * p23[2] + d43[0] * p12[2] -
         q12 * (v3 * p12[0] - v1 * p12[2]) - q23 * (d43[0] * p23[2] - d43[2] * p23[0]);
  w[5] = -v2 * p23[0] + d43[1] * p12[0] + v1 * p23[1] - d43[0] * p12[1] -
         q12 * (-v2 * p12[0] + v1 * p12[1]) - q23 * (d43[1] * p23[0] - d43[0] * p23[1]);
  w[6] = d32[2] * p12[1] - d32[1] * p12[2] - q23 * (d32[2] * p23[1] - d32[1] * p23[2]);
  w[7] = d32[0] * p12[2] - d32[2] * p12[0] - q23 * (d32[0] * p23[2] - d32[2] * p23[0]);
  w[8] = d32[1] * p12[0] - d32[0] * p12[1] - q23 * (d32[1] * p23[0] - d32[0] * p23[1]);
  add_grad<FP64>(P, wr * wg, Q.a[0], w[0], w[1], w[2]);
  add_grad<FP64>(P, wr * wg, Q.a[1], w[3], w[4], w[5]);
  add_grad<FP64>(P, wr * wg, Q.a[2], -(w[0] + w[3] + w[6]), -(w[1] + w[4] + w[7]), -(w[2] + w[5] + w[8]));
  add_grad<FP64>(P, wr * wg, Q.a[3], w[6], w[7], w[8]);
}

// one CAP term of a group centre or an atom: c = position - centre, xa = what the box walls
// are compared with (c for groups, the absolute position for atoms, dnecap.f90:126-193);
// energy e and gradient g (before the mass share of a group); false when nothing acts
__device__ __forceinline__ bool cap_term(const Restr& Q, int shape, const double* c, const double* xa,
                                         double& e, double* g) {
  const double k = Q.p[4];
  if (shape == JP_CAP_BOX) {
    bool any = false;
    double s2 = 0.0;
    for (int d = 0; d < 3; ++d) {
      g[d] = 0.0;
      const double lo = Q.p[6 + 2 * d], hi = Q.p[7 + 2 * d];
      double dd = 0.0;
      if (xa[d] < lo) dd = xa[d] - lo;
      else if (xa[d] > hi) dd = xa[d] - hi;
      else continue;
      any = true;
      s2 += dd * dd;
      g[d] = k * dd;
    }
    e = 0.5 * k * s2;
    return any;
  }
  if (shape == JP_CAP_ELLIPSOID) {
    const double s = c[0] * c[0] * Q.p[6] + c[1] * c[1] * Q.p[7] + c[2] * c[2] * Q.p[8];
    if (!(s > 1.0)) return false;
    const double rt = 1.0 - sqrt(1.0 / s);
    const double dist = sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) * rt;
    e = 0.5 * k * dist * dist;
    for (int d = 0; d < 3; ++d) g[d] = c[d] * rt * k;
    return true;
  }
  const double d2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];   // sphere
  if (shape == kCapSphereQuartic) {   // half-biquadratic (dnecap.f90:253-281)
    const double r2 = Q.p[3] * Q.p[3];
    if (!(d2 > r2)) return false;
    const double sq = (d2 - r2) / r2;
    e = 0.25 * k * sq * sq * r2;
    for (int m = 0; m < 3; ++m) g[m] = k * sq * c[m];
    return true;
  }
  if (!(d2 > Q.p[3] * Q.p[3])) return false;
  const double d = sqrt(d2), dd = d - Q.p[3];
  e = 0.5 * k * dd * dd;
  for (int m = 0; m < 3; ++m) g[m] = k * dd / d * c[m];
  return true;
}

template <bool FP64>
__global__ void __launch_bounds__(kResThreads) k_restraints(DevPtrs P, int n, int alsd) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  int slot = JP_E_POSRES, rep = 0;
  if (t < n) {
    const Restr Q = P.restr[t];
    rep = Q.rep;
    const Rep& R = P.reps[rep];
    const double* x = P.x;
    // restraint gradients are class BB / class 2 (grad(:,:,nfrg)): weight 1, or the BB weight
    // while an ALSD replica's per-class outputs are evaluated
    const double wg = R.cls_over ? R.cls_w[2] : 1.0;
    switch (Q.kind) {
      case R_POS: {
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = x[3 * Q.a[0] + k] - Q.p[k];
        res_image(R, d);
        e = 0.5 * Q.p[3] * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        add_grad<FP64>(P, Q.p[3] * wg, Q.a[0], d[0], d[1], d[2]);
        break;
      }
      case R_DIST:
        slot = JP_E_DISTRES;
        res_dist<FP64>(P, R, Q, e, wg);
        break;
      case R_DIHE:
        slot = JP_E_DIHERES;
        res_dihe<FP64>(P, R, Q, e, wg);
        break;
      case R_CAPG: {   // centre of mass of atoms a[0] .. a[1]; p[5] = 1 / their mass
        slot = JP_E_CAP;
        double c[3] = {0.0, 0.0, 0.0}, g[3];
        for (int a = Q.a[0]; a <= Q.a[1]; ++a)
          for (int k = 0; k < 3; ++k) c[k] += P.mass[a] * x[3 * a + k];
        for (int k = 0; k < 3; ++k) c[k] = c[k] * Q.p[5] - Q.p[k];
        if (cap_term(Q, Q.a[2], c, c, e, g))
          for (int a = Q.a[0]; a <= Q.a[1]; ++a)
            add_grad<FP64>(P, Q.p[5] * P.mass[a] * wg, a, g[0], g[1], g[2]);
        break;
      }
      case R_CAPA: {
        slot = JP_E_CAP;
        double c[3], xa[3], g[3];
        for (int k = 0; k < 3; ++k) {
          xa[k] = x[3 * Q.a[0] + k];
          c[k] = xa[k] - Q.p[k];
        }
        if (cap_term(Q, Q.a[1], c, xa, e, g)) add_grad<FP64>(P, wg, Q.a[0], g[0], g[1], g[2]);
        break;
      }
    }
  }
  if (__any_sync(0xffffffffu, t < n)) {
    add_energy(P, rep, slot, e);
    if (alsd) add_cls_energy(P, rep, 2, e);
  }
}

void launch_restraints(const DevPtrs& P, int n, bool fp64, bool alsd, cudaStream_t st) {
  if (n <= 0) return;
  const int nb = (n + kResThreads - 1) / kResThreads;
  if (fp64) k_restraints<true><<<nb, kResThreads, 0, st>>>(P, n, alsd ? 1 : 0);
  else k_restraints<false><<<nb, kResThreads, 0, st>>>(P, n, alsd ? 1 : 0);
}

}  // namespace jp
