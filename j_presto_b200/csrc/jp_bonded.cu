// jp_bonded.cu -- bonded terms, 1-4 pairs and the zero-dipole excess of excluded pairs.
//
// Replaces dnergv_PB's bonded part (src_md_run/dnergv.f90): dnebnd (65-122), dneang
// (128-207), dnetor for torsions and impropers (223-434, closed-form derivative for
// n <= 6), dne14 (440-516), and the ZD excess loop of enear (enear.f90:518-555).
// md_run parallelises these over write-conflict-free colour groups (incel.f90:693-946);
// here every term is one thread and gradients are added atomically (64-bit fixed point
// on the mixed path, FP64 on the FP64 path).  Arithmetic is FP64 on both paths: these
// terms are few and latency-bound.
#include "jp_kernels.h"

namespace jp {

struct Img {
  double b[3], ib[3];
  __device__ void apply(double* d) const {
    for (int k = 0; k < 3; ++k) d[k] -= b[k] * anint(d[k] * ib[k]);
  }
};

template <bool FP64>
__global__ void __launch_bounds__(256) k_bonded(DevPtrs P, int nterm, double zb, double zf,
                                                int alsd) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  double e1 = 0.0, e2 = 0.0;
  int slot1 = JP_E_BOND, slot2 = -1, rep = 0, cls = 2;
  if (t < nterm) {
    const Term T = P.terms[t];
    rep = T.rep;
    const Rep& R = P.reps[rep];
    double fs = 1.0;
    bool c1 = false;   // a class-1 term of a partial-McMD replica
    if (alsd && R.lam_mode) {
      cls = T.cls;
      fs = cls_weight(R, P.lam[2 * rep], cls);
    } else if (alsd && R.split) {
      cls = T.cls;
      c1 = cls == 0;
    }
    Img im;
    for (int k = 0; k < 3; ++k) { im.b[k] = R.box[k]; im.ib[k] = R.invbox[k]; }
    const double* x = P.x;
    switch (T.kind) {
      case T_BOND: {
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = x[3 * T.a[0] + k] - x[3 * T.a[1] + k];
        im.apply(d);
        const double r12 = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double dif = r12 - T.p1;
        double coef = T.p0 * dif;
        e1 = coef * dif;
        coef = 2.0 * coef / r12;
        add_grad<FP64>(P, fs, T.a[0], coef * d[0], coef * d[1], coef * d[2], c1);
        add_grad<FP64>(P, fs, T.a[1], -coef * d[0], -coef * d[1], -coef * d[2], c1);
        slot1 = JP_E_BOND;
        break;
      }
      case T_ANGLE: {
        double d12[3], d32[3];
        for (int k = 0; k < 3; ++k) {
          d12[k] = x[3 * T.a[0] + k] - x[3 * T.a[1] + k];
          d32[k] = x[3 * T.a[2] + k] - x[3 * T.a[1] + k];
        }
        im.apply(d12);
        im.apply(d32);
        double r12 = d12[0] * d12[0] + d12[1] * d12[1] + d12[2] * d12[2];
        double r32 = d32[0] * d32[0] + d32[1] * d32[1] + d32[2] * d32[2];
        const double r12r32 = sqrt(1.0 / (r12 * r32));
        double cost = d12[0] * d32[0] + d12[1] * d32[1] + d12[2] * d32[2];
        r12 = 1.0 / r12;
        r32 = 1.0 / r32;
        cost = fmin(cost * r12r32, 1.0);
        cost = fmax(cost, -1.0);
        const double theta = acos(cost);
        const double dif = theta - T.p1;
        double coef = T.p0 * dif;
        e1 = coef * dif;
        const double sint = fmax(sin(theta), 1.0e-10);
        coef = -2.0 * coef / sint;
        double w[6];
        double rt = cost * r12;
        for (int k = 0; k < 3; ++k) w[k] = coef * (d32[k] * r12r32 - d12[k] * rt);
        rt = cost * r32;
        for (int k = 0; k < 3; ++k) w[3 + k] = coef * (d12[k] * r12r32 - d32[k] * rt);
        add_grad<FP64>(P, fs, T.a[0], w[0], w[1], w[2], c1);
        add_grad<FP64>(P, fs, T.a[1], -(w[0] + w[3]), -(w[1] + w[4]), -(w[2] + w[5]), c1);
        add_grad<FP64>(P, fs, T.a[2], w[3], w[4], w[5], c1);
        slot1 = JP_E_ANGLE;
        break;
      }
      case T_TORS:
      case T_IMPR: {
        slot1 = T.kind == T_TORS ? JP_E_TORS : JP_E_IMPR;
        double d21[3], d32[3], d43[3];
        for (int k = 0; k < 3; ++k) {
          d21[k] = x[3 * T.a[1] + k] - x[3 * T.a[0] + k];
          d32[k] = x[3 * T.a[2] + k] - x[3 * T.a[1] + k];
          d43[k] = x[3 * T.a[3] + k] - x[3 * T.a[2] + k];
        }
        im.apply(d21);
        im.apply(d32);
        im.apply(d43);
        const double p12[3] = {d21[1] * d32[2] - d32[1] * d21[2], d21[2] * d32[0] - d32[2] * d21[0],
                               d21[0] * d32[1] - d32[0] * d21[1]};
        const double p23[3] = {d32[1] * d43[2] - d43[1] * d32[2], d32[2] * d43[0] - d43[2] * d32[0],
                               d32[0] * d43[1] - d43[0] * d32[1]};
        const double r12 = p12[0] * p12[0] + p12[1] * p12[1] + p12[2] * p12[2];
        const double r23 = p23[0] * p23[0] + p23[1] * p23[1] + p23[2] * p23[2];
        double r12r23 = sqrt(r12 * r23);
        if (!(r12r23 > 0.0)) break;
        r12r23 = 1.0 / r12r23;
        const double s1223 = p12[0] * p23[0] + p12[1] * p23[1] + p12[2] * p23[2];
        double cosp = s1223 * r12r23;
        cosp = fmin(fmax(cosp, -1.0), 1.0);
        const double p123[3] = {p12[1] * p23[2] - p23[1] * p12[2], p12[2] * p23[0] - p23[2] * p12[0],
                                p12[0] * p23[1] - p23[0] * p12[1]};
        const double s32123 = d32[0] * p123[0] + d32[1] * p123[1] + d32[2] * p123[2];
        double phi = acos(cosp);
        if (s32123 < 0.0) phi = 2.0 * 3.141592653589793 - phi;
        const double div = 1.0 / (double)T.idiv;
        e1 = T.p0 * (1.0 + cos(T.p1 * phi + T.p2)) * div;
        const double sinp = sin(phi);
        double w0;
        switch ((int)anint(T.p1)) {
          case 1: w0 = 1.0; break;
          case 2: w0 = 2.0 * cosp; break;
          case 3: w0 = -4.0 * sinp * sinp + 3.0; break;
          case 4: w0 = (-8.0 * sinp * sinp + 4.0) * cosp; break;
          case 5: w0 = (16.0 * sinp * sinp - 20.0) * sinp * sinp + 5.0; break;
          case 6: w0 = cosp * (6.0 + 32.0 * cosp * cosp * (cosp * cosp - 1.0)); break;
          default: w0 = 0.0;
        }
        w0 = cos(T.p2) * T.p1 * T.p0 * div * w0 * r12r23;
        const double w1 = d21[0] + d32[0], w2 = d21[1] + d32[1], w3 = d21[2] + d32[2];
        const double q12 = s1223 / r12, q23 = s1223 / r23;
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
        add_grad<FP64>(P, fs, T.a[0], w[0], w[1], w[2], c1);
        add_grad<FP64>(P, fs, T.a[1], w[3], w[4], w[5], c1);
        add_grad<FP64>(P, fs, T.a[2], -(w[0] + w[3] + w[6]), -(w[1] + w[4] + w[7]), -(w[2] + w[5] + w[8]), c1);
        add_grad<FP64>(P, fs, T.a[3], w[6], w[7], w[8], c1);
        break;
      }
      case T_P14: {
        slot1 = JP_E_VDW14;
        slot2 = JP_E_ELE14;
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = x[3 * T.a[0] + k] - x[3 * T.a[1] + k];
        im.apply(d);
        const double r14 = 1.0 / (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        const double r141 = sqrt(r14);
        const double r146 = r14 * r14 * r14;
        const double r1412 = r146 * r146;
        // p0 = svdw, p1 = sele*ccoef*q1*q4, a[2] = LJ table index
        const double2 lj = P.lj14[T.a[2]];
        const double co6 = lj.x * r146, co12 = lj.y * r1412;
        e1 = T.p0 * (-co6 + co12);
        double coef = r14 * T.p0 * (-2.0 * co12 + co6) * 6.0;
        double w[3] = {coef * d[0], coef * d[1], coef * d[2]};
        coef = T.p1 * r141;
        e2 = coef;
        coef *= -r14;
        for (int k = 0; k < 3; ++k) w[k] += coef * d[k];
        add_grad<FP64>(P, fs, T.a[0], w[0], w[1], w[2], c1);
        add_grad<FP64>(P, fs, T.a[1], -w[0], -w[1], -w[2], c1);
        break;
      }
      case T_EXCESS: {
        slot1 = JP_E_ELE15;
        double d[3];
        for (int k = 0; k < 3; ++k) d[k] = x[3 * T.a[0] + k] - x[3 * T.a[1] + k];
        im.apply(d);
        const double dd2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        double cc = T.p0;   // chgmod(a)*chgmod(b)
        e1 = cc * zb * dd2;
        cc *= zf;
        add_grad<FP64>(P, fs, T.a[0], d[0] * cc, d[1] * cc, d[2] * cc, c1);
        add_grad<FP64>(P, fs, T.a[1], -d[0] * cc, -d[1] * cc, -d[2] * cc, c1);
        break;
      }
    }
  }
  // the term list is sorted by kind then replica, so most warps are uniform
  if (__any_sync(0xffffffffu, t < nterm)) {
    add_energy(P, rep, slot1, e1);
    const bool has2 = __any_sync(0xffffffffu, slot2 >= 0);
    if (has2) add_energy(P, rep, slot2 >= 0 ? slot2 : JP_E_ELE14, e2);
    if (alsd) add_cls_energy(P, rep, cls, e1 + e2);
  }
}

void launch_bonded(const DevPtrs& P, int nterm, bool fp64, double zb, double zf, bool alsd,
                   cudaStream_t st) {
  if (nterm <= 0) return;
  const int nb = (nterm + 255) / 256;
  if (fp64) k_bonded<true><<<nb, 256, 0, st>>>(P, nterm, zb, zf, alsd ? 1 : 0);
  else k_bonded<false><<<nb, 256, 0, st>>>(P, nterm, zb, zf, alsd ? 1 : 0);
}

}  // namespace jp
