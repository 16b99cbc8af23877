// jp_integrate.cu -- leap-frog integration fused with SHAKE, temperature control and the
// generalized-ensemble force scaling.
//
// Replaces verlet (src_md_run/verlet.f90:2-226, METHOD= MICR), verlethe (verlethe.f90:2-758,
// METHOD= CANO and GE/McMD), shake_PB (shake.f90:2-755) and caltmp/caltmp2 (caltmp.f90).
// One thread owns one integration unit: a SHAKE group (2-4 atoms, all pair distances
// constrained) or a lone atom, so SHAKE needs no inter-thread communication.  Everything
// is FP64.  Kinetic-energy sums for the thermostat are 64-bit fixed point (order
// independent); all replicas are processed by the same launches and each replica keeps
// its own temperatures, SHAKE<->thermostat iteration count and force scale.
#include <algorithm>

#include "jp_kernels.h"
#include "jp_mlp.cuh"

namespace jp {

constexpr int kCom = 16;   // centre-of-mass stop sums per replica and slot

// Loop over the 1-4 atoms of an integration unit.  The trip count is fixed at 4 and fully
// unrolled with a guard: the per-unit arrays then live in registers.  (A runtime trip count
// over these small local arrays produced wrong values on sm_100a with nvcc 12.9.)
#define JP_UNIT_LOOP(q) _Pragma("unroll") for (int q = 0; q < 4; ++q) if (q < u.n)
// the same over a 1-3 atom unit (the units of the small lanes: 4-atom groups take eight lanes)
#define JP_SMALL_LOOP(q) _Pragma("unroll") for (int q = 0; q < 3; ++q) if (q < u.n)

__host__ __device__ __forceinline__ void mimg(const Rep& R, double* d) {
  for (int k = 0; k < 3; ++k) d[k] -= R.box[k] * anint(d[k] * R.invbox[k]);
}

// A partial-McMD replica scales its class-1 gradient alone (verlet.f90:130-141,
// verlethe.f90:176-187, :223-234: grad(:,:,2) = grad(:,:,1) dew + grad(:,:,2)); the class-1
// set exists only in contexts with such replicas (a uniform test of a kernel parameter)
template <bool FP64>
__device__ __forceinline__ void split_grad(const DevPtrs& P, int a, double s, double* g) {
  if (FP64 ? P.grd1 == nullptr : P.frc1 == nullptr) return;
  if (!P.reps[P.rep_of[a]].split) return;
  for (int k = 0; k < 3; ++k) {
    const double g1 = FP64 ? P.grd1[3 * a + k] : (double)P.frc1[3 * a + k] * kFrcInv;
    const double g2 = FP64 ? P.grd[3 * a + k] : (double)P.frc[3 * a + k] * kFrcInv;
    g[k] = g1 * s + g2;
  }
}

template <bool FP64>
__device__ __forceinline__ void load_grad(const DevPtrs& P, int a, double s, double* g) {
  if (FP64) {
    for (int k = 0; k < 3; ++k) g[k] = P.grd[3 * a + k] * s;
  } else {
    for (int k = 0; k < 3; ++k) g[k] = (double)P.frc[3 * a + k] * kFrcInv * s;
  }
  split_grad<FP64>(P, a, s, g);
}

__host__ __device__ __noinline__ int shake_group4(const Rep& R, const Unit& u, const double* im,
                                                 double r1[4][3], const double r2[4][3],
                                                 double tol, int maxit);

// ---- SHAKE on one group (r1 constrained against reference r2) --------------------------
// returns 0 converged, 1 not converged, -2 singular.  2- and 3-atom groups: inlined, works on
// register arrays; 4-atom groups: shake_group4, out of line.
__host__ __device__ __forceinline__ int shake_small(const Rep& R, int n, const double* len2,
                                                    const double* im, double (*r1)[3],
                                                    const double (*r2)[3], int method, double tol,
                                                    int maxit) {
  if (n == 2) {
    double d1[3], d2[3];
    if (method == JP_SHAKE_HBON) {   // shak2e (shake.f90:687-755): exact quadratic
      for (int k = 0; k < 3; ++k) { d1[k] = r1[1][k] - r1[0][k]; d2[k] = r2[1][k] - r2[0][k]; }
      mimg(R, d1);
      mimg(R, d2);
      const double i3 = im[0] + im[1], i4 = i3 * i3;
      const double d1d1 = d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2];
      const double d1d2 = d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2];
      const double d2d2 = d2[0] * d2[0] + d2[1] * d2[1] + d2[2] * d2[2];
      const double A = i4 * d2d2, B = i3 * d1d2, C = d1d1 - len2[0];
      const double G = (B - sqrt(B * B - C * A)) / A;
      for (int k = 0; k < 3; ++k) {
        r1[0][k] += im[0] * G * d2[k];
        r1[1][k] -= im[1] * G * d2[k];
      }
      return 0;
    }
    // shak2i (shake.f90:568-681): iterate this constraint to its own tolerance
    for (int k = 0; k < 3; ++k) d2[k] = r2[0][k] - r2[1][k];
    mimg(R, d2);
    const double i3 = 0.5 / (im[0] + im[1]);
    for (int it = 0; it < maxit; ++it) {
      for (int k = 0; k < 3; ++k) d1[k] = r1[0][k] - r1[1][k];
      mimg(R, d1);
      double dif = len2[0] - (d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
      const double inpro = d1[0] * d2[0] + d1[1] * d2[1] + d1[2] * d2[2];
      const double G = dif * i3 / inpro;
      for (int k = 0; k < 3; ++k) {
        r1[0][k] += im[0] * G * d2[k];
        r1[1][k] -= im[1] * G * d2[k];
      }
      for (int k = 0; k < 3; ++k) d1[k] = r1[0][k] - r1[1][k];
      mimg(R, d1);
      dif = len2[0] - (d1[0] * d1[0] + d1[1] * d1[1] + d1[2] * d1[2]);
      if (fabs(dif / len2[0]) < tol) return 0;
    }
    return 1;
  }
  if (n == 3) {   // shake3 (shake.f90:113-327): Newton, closed-form 3x3 inverse
    const double cg[3][3] = {{im[0] + im[1], -im[1], -im[0]},
                             {-im[1], im[1] + im[2], -im[2]},
                             {-im[0], -im[2], im[2] + im[0]}};
    const int pa[3][2] = {{0, 1}, {1, 2}, {2, 0}};
    double d1[3][3], d2[3][3];
    for (int q = 0; q < 3; ++q) {
      for (int k = 0; k < 3; ++k) {
        d1[q][k] = r1[pa[q][0]][k] - r1[pa[q][1]][k];
        d2[q][k] = r2[pa[q][0]][k] - r2[pa[q][1]][k];
      }
      mimg(R, d1[q]);
      mimg(R, d2[q]);
    }
    double G[6] = {0, 0, 0, 0, 0, 0};
    bool singular = false;
    for (int it = 0; it < maxit; ++it) {
      double B[3];
      for (int q = 0; q < 3; ++q) B[q] = len2[q] - (d1[q][0] * d1[q][0] + d1[q][1] * d1[q][1] + d1[q][2] * d1[q][2]);
      if (fabs(B[0]) < tol * len2[0] && fabs(B[1]) < tol * len2[1] && fabs(B[2]) < tol * len2[2]) {
        for (int k = 0; k < 3; ++k) {
          r1[0][k] += im[0] * (G[3] * d2[0][k] - G[5] * d2[2][k]);
          r1[1][k] += im[1] * (-G[3] * d2[0][k] + G[4] * d2[1][k]);
          r1[2][k] += im[2] * (-G[4] * d2[1][k] + G[5] * d2[2][k]);
        }
        return singular ? -2 : 0;
      }
      double gf[3][3];
      for (int ig = 0; ig < 3; ++ig)
        for (int q = 0; q < 3; ++q)
          gf[q][ig] = 2.0 * cg[q][ig] * (d1[q][0] * d2[ig][0] + d1[q][1] * d2[ig][1] + d1[q][2] * d2[ig][2]);
      double deta = gf[0][0] * gf[1][1] * gf[2][2] + gf[0][1] * gf[1][2] * gf[2][0] +
                    gf[0][2] * gf[1][0] * gf[2][1] - gf[0][0] * gf[1][2] * gf[2][1] -
                    gf[0][1] * gf[1][0] * gf[2][2] - gf[0][2] * gf[1][1] * gf[2][0];
      if (deta == 0.0) singular = true;
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
    return singular ? -2 : 1;
  }
  return 1;
}

__host__ __device__ int shake_group(const Rep& R, const Unit& u, const double* im, double r1[4][3],
                                    const double r2[4][3], int method, double tol, int maxit) {
  if (u.n <= 3) return shake_small(R, u.n, u.d2, im, r1, r2, method, tol, maxit);
  return shake_group4(R, u, im, r1, r2, tol, maxit);
}

// coefficient matrix coeg of shake4 (shake.f90:363-398): entry (q, ig) from the inverse
// masses; evaluated at each use (static q, ig fold to one add or a sign) instead of being
// held as a 6x6 array
__host__ __device__ __forceinline__ double cg4(int q, int ig, const double* im) {
  switch (q * 6 + ig) {
    case 0: return im[0] + im[1];  case 1: return -im[1];  case 2: return -im[0];
    case 3: return -im[0];         case 4: return 0.0;     case 5: return -im[1];
    case 6: return -im[1];         case 7: return im[1] + im[2];  case 8: return -im[2];
    case 9: return 0.0;            case 10: return -im[2]; case 11: return im[1];
    case 12: return -im[0];        case 13: return -im[2]; case 14: return im[2] + im[0];
    case 15: return im[0];         case 16: return im[2];  case 17: return 0.0;
    case 18: return -im[0];        case 19: return 0.0;    case 20: return im[0];
    case 21: return im[3] + im[0]; case 22: return -im[3]; case 23: return -im[3];
    case 24: return 0.0;           case 25: return -im[2]; case 26: return im[2];
    case 27: return -im[3];        case 28: return im[2] + im[3]; case 29: return im[3];
    case 30: return -im[1];        case 31: return im[1];  case 32: return 0.0;
    case 33: return -im[3];        case 34: return im[3];  default: return im[1] + im[3];
  }
}

// n == 4: shake4 (shake.f90:333-562): Newton with LU (simulu.f90).  Kept out of line: only
// X-H3 groups take it, and inlining its 6x6 system would raise the register demand of every
// integration kernel.
__host__ __device__ __noinline__ int shake_group4(const Rep& R, const Unit& u, const double* im,
                                                 double r1[4][3], const double r2[4][3],
                                                 double tol, int maxit) {
  const int pa[6][2] = {{0, 1}, {1, 2}, {2, 0}, {3, 0}, {2, 3}, {1, 3}};
  double d1[6][3], d2[6][3], wk[6][3], G[6] = {0, 0, 0, 0, 0, 0};
  for (int q = 0; q < 6; ++q) {
    for (int k = 0; k < 3; ++k) {
      d1[q][k] = r1[pa[q][0]][k] - r1[pa[q][1]][k];
      d2[q][k] = r2[pa[q][0]][k] - r2[pa[q][1]][k];
    }
    mimg(R, d1[q]);
    mimg(R, d2[q]);
    for (int k = 0; k < 3; ++k) wk[q][k] = d1[q][k];
  }
  bool singular = false;
  for (int it = 0; it < maxit; ++it) {
    double B[6];
    bool ok = true;
    for (int q = 0; q < 6; ++q) {
      B[q] = u.d2[q] - (wk[q][0] * wk[q][0] + wk[q][1] * wk[q][1] + wk[q][2] * wk[q][2]);
      if (fabs(B[q]) >= tol * u.d2[q]) ok = false;
    }
    if (ok) {
      for (int k = 0; k < 3; ++k) {
        r1[0][k] += im[0] * (G[0] * d2[0][k] - G[2] * d2[2][k] - G[3] * d2[3][k]);
        r1[1][k] += im[1] * (-G[0] * d2[0][k] + G[1] * d2[1][k] + G[5] * d2[5][k]);
        r1[2][k] += im[2] * (-G[1] * d2[1][k] + G[2] * d2[2][k] + G[4] * d2[4][k]);
        r1[3][k] += im[3] * (G[3] * d2[3][k] - G[4] * d2[4][k] - G[5] * d2[5][k]);
      }
      return singular ? -2 : 0;
    }
    double A[6][6];
#pragma unroll
    for (int ig = 0; ig < 6; ++ig)
#pragma unroll
      for (int q = 0; q < 6; ++q)
        A[q][ig] = 2.0 * cg4(q, ig, im) * (wk[q][0] * d2[ig][0] + wk[q][1] * d2[ig][1] + wk[q][2] * d2[ig][2]);
    for (int ig = 0; ig < 6; ++ig)
      for (int q = 0; q < 6; ++q) B[q] += A[q][ig] * G[ig];
    // LU with partial pivoting (simulu.f90 ludeco + solve): the same pivot choice and
    // elimination order as md_run's row-permutation form, with the pivot row swapped in
    // registers (static indices only, so nothing goes to local memory)
    bool lu_ok = true;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      int pr = k;
      double al = fabs(A[k][k]);
#pragma unroll
      for (int i = k + 1; i < 6; ++i)
        if (fabs(A[i][k]) > al) { pr = i; al = fabs(A[i][k]); }
#pragma unroll
      for (int i = k + 1; i < 6; ++i) {
        const bool sw = (pr == i);
#pragma unroll
        for (int j = 0; j < 6; ++j) {
          const double t = A[k][j];
          A[k][j] = sw ? A[i][j] : t;
          A[i][j] = sw ? t : A[i][j];
        }
        const double tb = B[k];
        B[k] = sw ? B[i] : tb;
        B[i] = sw ? tb : B[i];
      }
      if (fabs(A[k][k]) < 1.0e-30) lu_ok = false;
      const double piv = 1.0 / A[k][k];
#pragma unroll
      for (int i = k + 1; i < 6; ++i) {
        const double f = A[i][k] * piv;
#pragma unroll
        for (int j = k + 1; j < 6; ++j) A[i][j] -= f * A[k][j];
        B[i] -= f * B[k];
      }
      A[k][k] = piv;
    }
    if (!lu_ok) {
      singular = true;
    } else {
#pragma unroll
      for (int i = 5; i >= 0; --i) {
        double t = B[i];
#pragma unroll
        for (int j = i + 1; j < 6; ++j) t -= A[i][j] * G[j];
        G[i] = t * A[i][i];
      }
    }
    for (int q = 0; q < 6; ++q)
      for (int k = 0; k < 3; ++k) wk[q][k] = d1[q][k];
#pragma unroll
    for (int ig = 0; ig < 6; ++ig)
#pragma unroll
      for (int q = 0; q < 6; ++q)
        for (int k = 0; k < 3; ++k) wk[q][k] += cg4(q, ig, im) * d2[ig][k] * G[ig];
  }
  return singular ? -2 : 1;
}

// An atom's force accumulator back to zero once its owner has read it for the last time in
// the step: the next step's pair, bonded and far-field kernels add into zeros (no memset).
template <bool FP64>
__device__ __forceinline__ void zero_force(const DevPtrs& P, int a) {
  if (FP64) {
    P.grd[3 * a] = 0.0; P.grd[3 * a + 1] = 0.0; P.grd[3 * a + 2] = 0.0;
    if (P.grd1) { P.grd1[3 * a] = 0.0; P.grd1[3 * a + 1] = 0.0; P.grd1[3 * a + 2] = 0.0; }
  } else {
    P.frc[3 * a] = 0; P.frc[3 * a + 1] = 0; P.frc[3 * a + 2] = 0;
    if (P.frc1) { P.frc1[3 * a] = 0; P.frc1[3 * a + 1] = 0; P.frc1[3 * a + 2] = 0; }
  }
}

// a SHAKE failure (shake.f90 ier 1 or -2) of a group of replica `rep`: the status bit, and
// the replica's flag that the host reads to redo its step with a halved time step
__device__ __forceinline__ void shake_status(const DevPtrs& P, int ier, int rep) {
  if (ier == 1) atomicOr(P.status, ERR_SHAKE_NOCONV);
  else if (ier == -2) atomicOr(P.status, ERR_SHAKE_SINGULAR);
  P.rep_fail[rep] = 1;
}

// warp-aggregated fixed-point add of m v^2 into kin_fix[slot][sub]
__device__ __forceinline__ void add_kin(const DevPtrs& P, int nsub_total, int kslot, int sub, double e) {
  const unsigned full = 0xffffffffu;
  const int s0 = __shfl_sync(full, sub, 0);
  long long* dst = P.kin_fix + (size_t)kslot * nsub_total;
  if (__all_sync(full, sub == s0)) {
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(full, e, o);
    if ((threadIdx.x & 31) == 0 && s0 >= 0) atomic_add_ll(&dst[s0], to_fix(e, kKinScale, P.status));
  } else if (sub >= 0 && e != 0.0) {
    atomic_add_ll(&dst[sub], to_fix(e, kKinScale, P.status));
  }
}

__device__ __forceinline__ void write_slot(const DevPtrs& P, int a, const double* x, bool fp64) {
  const int s = P.slot_of[a];
  if (fp64) {
    double4 p = P.pos_d[s];
    p.x = x[0]; p.y = x[1]; p.z = x[2];
    P.pos_d[s] = p;
  } else {
    float4 p = P.pos_f[s];
    p.x = (float)(x[0] - P.off[3 * s]);
    p.y = (float)(x[1] - P.off[3 * s + 1]);
    p.z = (float)(x[2] - P.off[3 * s + 2]);
    P.pos_f[s] = p;
  }
}

// target temperature with the heating ramp (verlethe.f90:412-416)
__device__ __forceinline__ double target_temp(const IntConst& c, long long idloop) {
  if (c.heat_loop <= 0 || idloop > c.heat_loop) return c.temp;
  return c.temp_start + ((c.temp - c.temp_start) / (double)c.heat_loop) * (double)idloop;
}

__device__ __forceinline__ double sub_temp(const DevPtrs& P, const IntConst& c, int kslot, int sub) {
  // L2-coherent load: inside the cooperative kernel other blocks wrote this sum before the
  // last grid barrier, and L1 may still hold the line from an earlier phase
  const double ek = (double)__ldcg(&P.kin_fix[(size_t)kslot * c.nsub_total + sub]) * kKinInv;
  return ek * 1.0e7 / (kGas * P.nfr[sub]);
}

// converged after iteration `it` (kinetic slot 2*it-1)?  verlethe.f90:614-623
__device__ bool cano_conv(const DevPtrs& P, const IntConst& c, const Rep& R, int it, double tt) {
  const int ks = 2 * it - 1;
  double mn = 1e300, mx = -1e300;
  for (int s = R.sub0; s < R.sub0 + R.nsub; ++s) {
    if (P.nfr[s] <= 0.0) continue;
    const double t = sub_temp(P, c, ks, s);
    mn = fmin(mn, t);
    mx = fmax(mx, t);
  }
  return fmax(fabs(mn - tt), fabs(mx - tt)) < c.fcstol * tt;
}

// iteration `it` of the SHAKE <-> thermostat loop still running for this replica?
__device__ bool cano_active(const DevPtrs& P, const IntConst& c, const Rep& R, int it, bool after_check,
                            double tt) {
  const int last = after_check ? it : it - 1;
  for (int q = 1; q <= last; ++q) {
    if (q == c.icslop) return false;
    if (cano_conv(P, c, R, q, tt)) return false;
  }
  return true;
}

// ---- per-replica preparation --------------------------------------------------------
// force scale of replica r for this step: McMD weight (verlethe.f90:196-238) from the total
// potential energy, or the pseudo-temperature factor (verlet.f90:118-142)
__device__ double rep_scale_poly(const DevPtrs& P, const IntConst& c, int r);

__device__ __forceinline__ double rep_scale(const DevPtrs& P, const IntConst& c, int r) {
  if (c.ge_prescaled) return __ldcg(&P.scale[r]);
  return rep_scale_poly(P, c, r);
}

// the energy of the McMD weight: the potential energy, or a partial-McMD replica's class-1
// energy epotcc(1,1) (verlethe.f90:199-210)
__device__ __forceinline__ double mcmd_energy(const DevPtrs& P, const Rep& R, int r) {
  if (R.split) return (double)__ldcg(&P.ene_cls[4 * r]) * kEneInv + R.dself_cls[0];
  double tot = R.dself;
  for (int k = 1; k < JP_MAXENE; ++k) tot += (double)__ldcg(&P.ene_fix[r * 16 + k]) * kEneInv;
  return tot;
}

__device__ double rep_scale_poly(const DevPtrs& P, const IntConst& c, int r) {
  const Rep& R = P.reps[r];
  if (R.lam_mode) return 1.0;   // ALSD: the weight acts on lambda, forces go by class
  if (c.method == JP_METHOD_GE && R.ge_nwin > 0) {
    const double tot = mcmd_energy(P, R, r);
    double dprobl;
    if (tot <= R.ge_celw) dprobl = R.ge_alphalw;
    else if (tot >= R.ge_ceup) dprobl = R.ge_alphaup;
    else {
      double rt = (tot - R.ge_celw) / (R.ge_ceup - R.ge_celw);
      const double* cf = P.ge_coef + R.ge_off;   // per window: low, high, c0..cndeg
      const int stride = R.ge_ndeg + 3;
      int i = 0;
      for (i = 0; i < R.ge_nwin; ++i)
        if (rt < cf[i * stride + 1]) break;
      if (i >= R.ge_nwin) i = R.ge_nwin - 1;
      rt -= cf[i * stride + 0];
      const double* cc = cf + i * stride + 2;
      dprobl = cc[0];
      for (int j = 1; j <= R.ge_ndeg; ++j) dprobl += cc[j] * pow(rt, (double)j);
    }
    return (kGas / kJouCal) * 1.0e-3 * R.ge_tempce * dprobl;
  }
  if (c.psetmp > 1.0e-10) return c.temp / c.psetmp;
  return 1.0;
}

// ---- ALSD lambda (verlethe.f90:240-321, :400-450, :516-530) -----------------------------
// McMD weight in lambda: the polynomial in lambda itself (window search on lambda, no
// reduction) plus the linear walls; returns dew
__device__ double alsd_dew(const DevPtrs& P, const Rep& R, double lam) {
  const double* cf = P.ge_coef + R.ge_off;   // per window: low, high, c0..cndeg
  const int stride = R.ge_ndeg + 3;
  int i = R.ge_nwin - 1;
  for (int j = 0; j < R.ge_nwin; ++j)
    if (lam < cf[j * stride + 1]) { i = j; break; }
  const double rt = lam - cf[i * stride];
  const double* cc = cf + i * stride + 2;
  double dprobl = cc[0];
  for (int j = 1; j <= R.ge_ndeg; ++j) dprobl += cc[j] * pow(rt, (double)j);
  if (lam < R.ge_celw) dprobl += R.ge_lower * (R.ge_celw - lam);
  else if (lam > R.ge_ceup) dprobl += R.ge_upper * (lam - R.ge_ceup);
  return (kGas / kJouCal) * 1.0e-3 * R.ge_tempce * dprobl;
}

// the lambda weight term from the network's d lnP/dlambda (k_ge_scale), walls added
__device__ __forceinline__ double alsd_walls(const Rep& R, double lam, double dprobl) {
  if (lam < R.ge_celw) dprobl += R.ge_lower * (R.ge_celw - lam);
  else if (lam > R.ge_ceup) dprobl += R.ge_upper * (lam - R.ge_ceup);
  return (kGas / kJouCal) * 1.0e-3 * R.ge_tempce * dprobl;
}

// lambda of one replica through one step, carried by one thread
struct LamStep {
  double lam, lv, lvback, lf, lvt;
};

__device__ __forceinline__ void lam_add_ke(const DevPtrs& P, const IntConst& c, const Rep& R, int kslot,
                                           double lvt) {
  if (R.lam_ke_sub >= 0)
    atomic_add_ll(&P.kin_fix[(size_t)kslot * c.nsub_total + R.lam_ke_sub],
                  to_fix(R.lam_m * lvt * lvt, kKinScale, P.status));
}

// phase 1: the lambda force from the class energies and lambda's half-step velocity
__device__ void lam_begin(const DevPtrs& P, const IntConst& c, int r, LamStep& L, bool shk) {
  const Rep& R = P.reps[r];
  L.lam = P.lam[2 * r];
  L.lv = P.lam[2 * r + 1];
  L.lvback = L.lv;
  L.lf = 0.0;
  if (c.method == JP_METHOD_GE) {
    const double eaa = (double)__ldcg(&P.ene_cls[4 * r]) * kEneInv + R.dself_cls[0];
    const double eab = (double)__ldcg(&P.ene_cls[4 * r + 1]) * kEneInv + R.dself_cls[1];
    const double dew = R.mlp_on == 2 ? alsd_walls(R, L.lam, __ldcg(&P.lam_dew[r])) : alsd_dew(P, R, L.lam);
    L.lf = R.lam_mode == JP_ALSD_LMD ? -2.0 * eaa * L.lam - eab - dew
                                     : -eaa - 0.5 * eab / sqrt(L.lam) - dew;
  }
  L.lvt = L.lv;
  if (R.lam_im != 0.0) L.lvt = L.lv + 0.5 * c.dt * kConvcv * L.lf * R.lam_im;
  if (shk) lam_add_ke(P, c, R, 0, L.lvt);
}

// phase 2: thermostat-coupled (or free) velocity update, position, the loop's velocity
__device__ void lam_advance(const DevPtrs& P, const IntConst& c, int r, LamStep& L, double tt,
                            bool shk) {
  const Rep& R = P.reps[r];
  const double step = c.dt * kConvcv * L.lf * R.lam_im;
  bool coupled = R.lam_tc && R.lam_im != 0.0;
  int sub = R.lam_ke_sub;
  if (c.tempco == 1) sub = R.sub0;
  else coupled = coupled && sub >= 0;
  if (coupled) {
    const double chi = sqrt(tt / (shk ? sub_temp(P, c, 0, sub) : c.temp));
    L.lv = (2.0 * chi - 1.0) * L.lv + chi * step;
  } else {
    L.lv += step;
  }
  L.lam += c.dt * L.lv;
  L.lvt = (L.lvback + L.lv) * 0.5;
  if (shk) lam_add_ke(P, c, R, 1, L.lvt);
}

// k_ge_scale: one warp per replica.  McMD replicas with the surrogate network evaluate
// d lnN/dE = net(x) at the reduced energy x inside [celw, ceup] (alphalw / alphaup outside,
// as verlethe.f90:196-238 does for the polynomial); all others as rep_scale_poly.
__global__ void __launch_bounds__(32) k_ge_scale(DevPtrs P, IntConst c) {
  const int r = blockIdx.x;
  const Rep& R = P.reps[r];
  double s;
  if (c.method == JP_METHOD_GE && R.mlp_on == 2) {
    // ALSD: d lnP/dlambda of the (E, lambda) network for the lambda force; atoms unscaled
    double tot = R.dself;
    for (int k = 1; k < JP_MAXENE; ++k) tot += (double)__ldcg(&P.ene_fix[r * 16 + k]) * kEneInv;
    const float x[2] = {(float)((tot - R.mlp_e0) / (R.mlp_e1 - R.mlp_e0)), (float)P.lam[2 * r]};
    float y[2];
    mlp_forward_warp(P.mlp + (size_t)r * kMlpSlot, 2, 2, x, y);
    if (threadIdx.x == 0) {
      P.lam_dew[r] = (double)y[0];
      P.scale[r] = 1.0;
    }
    return;
  }
  if (c.method == JP_METHOD_GE && R.ge_nwin > 0 && R.mlp_on) {
    const double tot = mcmd_energy(P, R, r);
    double dprobl;
    if (tot <= R.ge_celw) {
      dprobl = R.ge_alphalw;
    } else if (tot >= R.ge_ceup) {
      dprobl = R.ge_alphaup;
    } else {
      const float x = (float)((tot - R.ge_celw) / (R.ge_ceup - R.ge_celw));
      float y;
      mlp_forward_warp(P.mlp + (size_t)r * kMlpSlot, 1, 1, &x, &y);
      dprobl = (double)y;
    }
    s = (kGas / kJouCal) * 1.0e-3 * R.ge_tempce * dprobl;
  } else {
    s = rep_scale_poly(P, c, r);
  }
  if (threadIdx.x == 0) P.scale[r] = s;
}

void launch_ge_scale(const DevPtrs& P, const IntConst& c, cudaStream_t st) {
  k_ge_scale<<<c.nrep, 32, 0, st>>>(P, c);
}

// energies of this step (time t) into the per-step history: eneval(15) of dnergy
__device__ void write_ene_hist(const DevPtrs& P, const IntConst& c, int r) {
  const Rep& R = P.reps[r];
  double e[JP_MAXENE];
  double tot = 0.0;
  for (int k = 1; k < JP_MAXENE; ++k) {
    e[k] = (double)__ldcg(&P.ene_fix[r * 16 + k]) * kEneInv;
    if (k == JP_E_ELE15) e[k] += R.dself;
    tot += e[k];
  }
  e[0] = tot;
  if (R.hist_n > 0 && !c.no_hist) {   // distrib_MULT.f90:95: k = int((E - minEc)/EbinSZ) + 1
    const double u = ((R.split ? mcmd_energy(P, R, r) : tot) - R.hist_min) * R.hist_inv;
    if (u > -1.0 && u < (double)R.hist_n) atomicAdd(&P.ge_hist[R.hist_off + (int)u], 1ull);
  }
  double* out = P.ene_hist + ((size_t)P.step_ctr[1] * c.nrep + r) * JP_MAXENE;
  for (int k = 0; k < JP_MAXENE; ++k) out[k] = e[k];
  if (R.alsd_nl > 0 && !c.no_hist) {   // distrib_ALSD input_lambda_data: int((lambda - minEc)/bin + 1)
    const double lam = P.lam[2 * r];
    const double u = (lam - R.alsd_lmin) * R.alsd_linv;
    if (u >= 0.0 && u < (double)R.alsd_nl) {
      const double eaa = (double)__ldcg(&P.ene_cls[4 * r]) * kEneInv + R.dself_cls[0];
      const double eab = (double)__ldcg(&P.ene_cls[4 * r + 1]) * kEneInv + R.dself_cls[1];
      const double dedl = R.lam_mode == JP_ALSD_LMD ? 2.0 * eaa * lam + eab : eaa + 0.5 * eab / sqrt(lam);
      const int k = (int)u;
      const size_t o = (size_t)r * JP_ALSD_MAX_LBINS + k;
      P.alsd_cnt[o] += 1ull;   // one thread per replica: a plain sum is deterministic
      P.alsd_f[o] += dedl;
      if (R.alsd_ne > 0) {
        const double v = (tot - R.alsd_emin) * R.alsd_einv;
        if (v >= 0.0 && v < (double)R.alsd_ne) {
          const size_t o2 = ((size_t)r * JP_ALSD_MAX_EBINS + (int)v) * JP_ALSD_MAX_LBINS + k;
          P.alsd_cnt2[o2] += 1ull;
          P.alsd_f2[o2] += dedl;
        }
      }
    }
  }
}

// Grid barrier for a cooperative launch (all blocks co-resident).  bar[0] counts arrivals
// over the whole launch (never reset inside it): barrier number e is passed once it reaches
// e * gridDim.x.  bar[2] is the abort flag.  The wait is bounded by P.wait_cycles of SM
// clock (about 1 s by default): on timeout the kernel records ERR_TIMEOUT, raises abort and
// every block returns at its next barrier.  `epoch` is the block's arrival target, advanced
// by each call.

__device__ __forceinline__ bool grid_barrier(const DevPtrs& P, unsigned& epoch) {
  __shared__ int s_ok;
  __syncthreads();
  epoch += gridDim.x;
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned* vb = P.bar;
    __threadfence();
    atomicAdd(&P.bar[0], 1u);
    const long long t0 = clock64();
    while (vb[0] < epoch) {
      if (vb[2] != 0u) { ok = 0; break; }
      if (clock64() - t0 > P.wait_cycles) {
        atomicOr(P.status, ERR_TIMEOUT);
        atomicExch(&P.bar[2], 1u);
        ok = 0;
        break;
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// end of step, one block after all others have finished: temperature of each replica (the kinetic
// slot of the last SHAKE pass, i.e. of (v(t-dt/2)+v(t+dt/2))/2) and the step counters
__device__ void finish_block(const DevPtrs& P, const IntConst& c, double tt) {
  const int h = P.step_ctr[1];
  for (int r = threadIdx.x; r < c.nrep; r += blockDim.x) {
    const Rep& R = P.reps[r];
    int ks = c.nkin - 1;   // MICR
    if (c.method > JP_METHOD_MICR && c.shake_method != JP_SHAKE_NONE) {   // verlethe
      int q = 1;
      for (; q < c.icslop; ++q)
        if (cano_conv(P, c, R, q, tt)) break;
      ks = 2 * q - 1;
    }
    double ek = 0.0, nf = 0.0;
    for (int s = R.sub0; s < R.sub0 + R.nsub; ++s) {
      ek += (double)__ldcg(&P.kin_fix[(size_t)ks * c.nsub_total + s]) * kKinInv;
      nf += P.nfr[s];
    }
    P.temp_hist[(size_t)h * c.nrep + r] =
        (c.method <= JP_METHOD_MICR || c.shake_method != JP_SHAKE_NONE) ? ek * 1.0e7 / (kGas * nf) : -1.0;
  }
  __syncthreads();
  // the next step starts from zero kinetic (and centre-of-mass) sums and a fresh barrier:
  // every other block has left its last barrier and read its last sum
  const int nk = c.nkin * c.nsub_total;
  for (int i = threadIdx.x; i < nk; i += blockDim.x) P.kin_fix[i] = 0;
  // the step's energies have been read (write_ene_hist, the force scale); the pair kernels'
  // tile counter follows them
  for (int i = threadIdx.x; i < 16 * c.nrep + 1; i += blockDim.x) P.ene_fix[i] = 0;
  if (c.stop)
    for (int i = threadIdx.x; i < c.ncom * c.nrep * kCom; i += blockDim.x) P.com[i] = 0.0;
  if (threadIdx.x == 0) {
    P.step_ctr[0] += 1;
    P.step_ctr[1] += 1;
    P.bar[0] = 0u;
    P.bar[1] = 0u;
    P.bar[2] = 0u;
    P.bar[3] = 0u;
  }
}

// is any replica still iterating the SHAKE <-> thermostat loop at pass `it`?  The same answer
// in every block: all read the kinetic sums completed before the last grid barrier.
// The block also keeps each replica's answer in s_act (replicas below kActCache), so the
// lanes of the pass read a shared flag instead of re-reading the kinetic sums.
constexpr int kActCache = 1024;

__device__ bool any_active(const DevPtrs& P, const IntConst& c, int it, double tt,
                           unsigned char* s_act) {
  int act = 0;
  for (int r = threadIdx.x; r < c.nrep; r += blockDim.x) {
    const bool a = cano_active(P, c, P.reps[r], it, true, tt);
    if (r < kActCache) s_act[r] = a ? 1 : 0;
    act |= a ? 1 : 0;
  }
  return __syncthreads_or(act) != 0;   // also publishes s_act to the block
}

// is replica r still iterating at pass `it` (after any_active filled s_act)?
__device__ __forceinline__ bool rep_active(const DevPtrs& P, const IntConst& c, const unsigned char* s_act,
                                           int r, int it, double tt) {
  return r < kActCache ? s_act[r] != 0 : cano_active(P, c, P.reps[r], it, true, tt);
}

// the last block to finish the step computes the temperatures and advances the step counters
__device__ void finish_last(const DevPtrs& P, const IntConst& c, double tt) {
  __shared__ int s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    s_last = atomicAdd(&P.bar[3], 1u) == gridDim.x - 1;
    __threadfence();
  }
  __syncthreads();
  if (s_last) finish_block(P, c, tt);
}

// ---- centre-of-mass stop (remotv.f90:2-131) ----------------------------------------------
// One reduction per velocity update: over the stopped atoms of a replica, with positions at
// time t (x0) and the velocity just updated (v), the sums
//   [0] m, [1-3] m x0, [4-6] m v, [7-9] m x0_k^2, [10] m x0 y0, [11] m y0 z0, [12] m z0 x0,
//   [13-15] m (x0 cross v).
// Centre, inertia tensor about the centre (parallel-axis shift) and angular momentum about
// the centre follow from them, so the correction v -= tv + w x (x0 - centre) needs one grid
// barrier.  The sums are FP64 atomics (their order, hence the last bits, varies run to run).
__device__ __forceinline__ bool stopped(const Rep& R, int a) { return a - R.atom0 < R.stop_n; }

__device__ __forceinline__ void com_terms(double m, const double* x0, const double* v, double* w) {
  w[0] += m;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    w[1 + k] += m * x0[k];
    w[4 + k] += m * v[k];
    w[7 + k] += m * x0[k] * x0[k];
  }
  w[10] += m * x0[0] * x0[1];
  w[11] += m * x0[1] * x0[2];
  w[12] += m * x0[2] * x0[0];
  w[13] += m * (x0[1] * v[2] - x0[2] * v[1]);
  w[14] += m * (x0[2] * v[0] - x0[0] * v[2]);
  w[15] += m * (x0[0] * v[1] - x0[1] * v[0]);
}

// adds each lane's sums to slot `slot` of replica `rep` (-1: the lane has none).  Called by
// all 32 lanes of a warp at one site.
__device__ void com_add(const DevPtrs& P, const IntConst& c, int slot, int rep, const double* w) {
  const unsigned full = 0xffffffffu;
  const unsigned has = __ballot_sync(full, rep >= 0);
  if (has == 0u) return;
  const int r0 = __shfl_sync(full, rep, __ffs(has) - 1);
  double* dst = P.com + (size_t)slot * c.nrep * kCom;
  if (__all_sync(full, rep < 0 || rep == r0)) {
#pragma unroll
    for (int k = 0; k < kCom; ++k) {
      double v = rep >= 0 ? w[k] : 0.0;
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(full, v, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(&dst[(size_t)r0 * kCom + k], v);
    }
  } else if (rep >= 0) {
    for (int k = 0; k < kCom; ++k) atomicAdd(&dst[(size_t)rep * kCom + k], w[k]);
  }
}

struct ComFix {
  double cen[3], tv[3], w[3];   // centre, translation and angular velocity to remove
};

// remotv's translational velocity (STOPCE 1, 3) and angular velocity (2, 3) of replica `rep`
// from the completed sums of slot `slot`.  False (error recorded) without mass or with a
// singular inertia tensor; the determinant test is relative to the tensor's scale, as the
// sums are shifted by the parallel-axis theorem.
__device__ bool com_fix(const DevPtrs& P, const IntConst& c, int slot, int rep, ComFix& F) {
  const double* s = P.com + ((size_t)slot * c.nrep + rep) * kCom;
  double q[kCom];
#pragma unroll
  for (int k = 0; k < kCom; ++k) q[k] = __ldcg(&s[k]);
  if (!(q[0] > 0.0)) {
    atomicOr(P.status, ERR_STOP_MASS);
    return false;
  }
  const double M = q[0], im = 1.0 / M;
  const bool tr = c.stop == JP_STOP_TRANS || c.stop == JP_STOP_BOTH;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    F.cen[k] = q[1 + k] * im;
    F.tv[k] = tr ? q[4 + k] * im : 0.0;
    F.w[k] = 0.0;
  }
  if (c.stop == JP_STOP_ROT || c.stop == JP_STOP_BOTH) {
    const double* r = F.cen;
    const double cxx = q[7] - M * r[0] * r[0], cyy = q[8] - M * r[1] * r[1], czz = q[9] - M * r[2] * r[2];
    const double cxy = q[10] - M * r[0] * r[1], cyz = q[11] - M * r[1] * r[2], czx = q[12] - M * r[2] * r[0];
    const double ixx = cyy + czz, iyy = czz + cxx, izz = cxx + cyy;
    const double ixy = -cxy, iyz = -cyz, izx = -czx;
    const double det = ixx * iyy * izz + 2.0 * ixy * iyz * izx - iyz * iyz * ixx - izx * izx * iyy -
                       ixy * ixy * izz;
    const double tr3 = (ixx + iyy + izz) * (1.0 / 3.0);
    if (!(fabs(det) > 1.0e-12 * tr3 * tr3 * tr3)) {
      atomicOr(P.status, ERR_STOP_SINGULAR);
      return false;
    }
    const double id = 1.0 / det;
    const double i11 = (iyy * izz - iyz * iyz) * id, i12 = (iyz * izx - izz * ixy) * id;
    const double i13 = (ixy * iyz - izx * iyy) * id, i22 = (izz * ixx - izx * izx) * id;
    const double i23 = (izx * ixy - ixx * iyz) * id, i33 = (ixx * iyy - ixy * ixy) * id;
    // angular momentum about the centre: sum m x0 x v - centre x sum m v
    const double l0 = q[13] - (r[1] * q[6] - r[2] * q[5]);
    const double l1 = q[14] - (r[2] * q[4] - r[0] * q[6]);
    const double l2 = q[15] - (r[0] * q[5] - r[1] * q[4]);
    F.w[0] = i11 * l0 + i12 * l1 + i13 * l2;
    F.w[1] = i12 * l0 + i22 * l1 + i23 * l2;
    F.w[2] = i13 * l0 + i23 * l1 + i33 * l2;
  }
  return true;
}

// velocity to remove from an atom at x0: tv + w x (x0 - centre)
__device__ __forceinline__ void com_delta(const ComFix& F, const double* x0, double* d) {
  const double r0 = x0[0] - F.cen[0], r1 = x0[1] - F.cen[1], r2 = x0[2] - F.cen[2];
  d[0] = F.tv[0] + F.w[1] * r2 - F.w[2] * r1;
  d[1] = F.tv[1] + F.w[2] * r0 - F.w[0] * r2;
  d[2] = F.tv[2] + F.w[0] * r1 - F.w[1] * r0;
}

// does a unit of n atoms a[0..n) (n <= NA) hold a stopped atom?
template <int NA>
__device__ __forceinline__ bool unit_stopped(const Rep& R, int n, const int* a) {
  bool any = false;
#pragma unroll
  for (int q = 0; q < NA; ++q) any |= q < n && stopped(R, a[q]);
  return any;
}

// ---- METHOD= MICR: verlet.f90 fused with SHAKE, one cooperative launch ------------------
template <bool FP64>
__device__ __forceinline__ double micr_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s) {
  const Rep& R = P.reps[u.rep];
  const double rt = -c.dt * kConvcv;
  double x0[4][3], x1[4][3], vb[4][3], im[4];
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double g[3];
    load_grad<FP64>(P, a, s, g);
    im[q] = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      x0[q][k] = P.x[3 * a + k];
      vb[q][k] = P.v[3 * a + k];
      const double v = vb[q][k] + rt * g[k] * im[q];
      x1[q][k] = x0[q][k] + c.dt * v;
      P.v[3 * a + k] = v;
    }
  }
  if (u.n >= 2 && c.shake_method != JP_SHAKE_NONE) {
    const int ier = shake_group(R, u, im, x1, x0, c.shake_method, c.shake_tol, c.shake_maxit);
    if (ier) shake_status(P, ier, u.rep);
    const double ri = 1.0 / c.dt;
    JP_UNIT_LOOP(q)
      for (int k = 0; k < 3; ++k) P.v[3 * u.a[q] + k] = (x1[q][k] - x0[q][k]) * ri;
  }
  bool bad = false;
  double ke = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      P.x[3 * a + k] = x1[q][k];
      const double vm = 0.5 * (vb[q][k] + P.v[3 * a + k]);
      vv += vm * vm;
      bad |= !isfinite(x1[q][k]);
    }
    ke += P.mass[a] * vv;
    write_slot(P, a, x1[q], FP64);
  }
  if (bad) atomicOr(P.status, ERR_NONFINITE);
  return ke;
}

// METHOD= CONS and the centre-of-mass stop split the step at grid barriers:
// (CONS) temperature of v(t-dt/2) | velocity update, its centre-of-mass sums | the
// correction, Berendsen factor, positions, SHAKE.  v(t-dt/2) waits in vback.
template <bool FP64>
__device__ __forceinline__ int micr_vel(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                        double* w) {
  const Rep& R = P.reps[u.rep];
  const double rt = -c.dt * kConvcv;
  bool any = false;
#pragma unroll
  for (int k = 0; k < kCom; ++k) w[k] = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double g[3], x0[3], v[3];
    load_grad<FP64>(P, a, s, g);
    const double im = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      const double vb = P.v[3 * a + k];
      P.vback[3 * a + k] = vb;
      v[k] = vb + rt * g[k] * im;
      P.v[3 * a + k] = v[k];
      x0[k] = P.x[3 * a + k];
    }
    if (c.stop && stopped(R, a)) {
      com_terms(P.mass[a], x0, v, w);
      any = true;
    }
  }
  return any ? u.rep : -1;
}

// Berendsen factor of scalet.f90:30-45 from the temperature of v(t-dt/2) (kinetic slot 0,
// all degrees of freedom of the replica); 1 when that temperature is not positive
__device__ double berendsen(const DevPtrs& P, const IntConst& c, const Rep& R) {
  double ek = 0.0, nf = 0.0;
  for (int s = R.sub0; s < R.sub0 + R.nsub; ++s) {
    ek += (double)__ldcg(&P.kin_fix[s]) * kKinInv;
    nf += P.nfr[s];
  }
  const double tempc = ek * 1.0e7 / (kGas * nf);
  if (!(tempc > 0.0)) return 1.0;
  const double lam = sqrt(1.0 + (c.dt / c.taut) * (c.temp / tempc - 1.0));
  return lam >= 2.0 ? 2.0 : lam;
}

template <bool FP64>
__device__ __forceinline__ double micr_pos(const DevPtrs& P, const IntConst& c, const Unit& u) {
  const Rep& R = P.reps[u.rep];
  ComFix F;
  const bool fix = c.stop && unit_stopped<4>(R, u.n, u.a) && com_fix(P, c, 0, u.rep, F);
  const double lam = c.method == JP_METHOD_CONS ? berendsen(P, c, R) : 1.0;
  double x0[4][3], x1[4][3], vb[4][3], im[4];
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    im[q] = P.imass[a];
    double d[3] = {0.0, 0.0, 0.0};
    for (int k = 0; k < 3; ++k) x0[q][k] = P.x[3 * a + k];
    if (fix && stopped(R, a)) com_delta(F, x0[q], d);
    for (int k = 0; k < 3; ++k) {
      vb[q][k] = P.vback[3 * a + k];
      const double v = (P.v[3 * a + k] - d[k]) * lam;
      x1[q][k] = x0[q][k] + c.dt * v;
      P.v[3 * a + k] = v;
    }
  }
  if (u.n >= 2 && c.shake_method != JP_SHAKE_NONE) {
    const int ier = shake_group(R, u, im, x1, x0, c.shake_method, c.shake_tol, c.shake_maxit);
    if (ier) shake_status(P, ier, u.rep);
    const double ri = 1.0 / c.dt;
    JP_UNIT_LOOP(q)
      for (int k = 0; k < 3; ++k) P.v[3 * u.a[q] + k] = (x1[q][k] - x0[q][k]) * ri;
  }
  bool bad = false;
  double ke = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      P.x[3 * a + k] = x1[q][k];
      const double vm = 0.5 * (vb[q][k] + P.v[3 * a + k]);
      vv += vm * vm;
      bad |= !isfinite(x1[q][k]);
    }
    ke += P.mass[a] * vv;
    write_slot(P, a, x1[q], FP64);
  }
  if (bad) atomicOr(P.status, ERR_NONFINITE);
  return ke;
}

// SPLIT: METHOD= CONS or the centre-of-mass stop (a separate instantiation, so that the
// plain MICR kernel keeps its register allocation)
template <bool FP64, bool SPLIT>
__global__ void __launch_bounds__(64) k_micr_fused(DevPtrs P, IntConst c, int nunit) {
  const int nthr = gridDim.x * blockDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt < c.nrep) write_ene_hist(P, c, gt);
  if (SPLIT) {
    unsigned epoch = 0;
    if (c.method == JP_METHOD_CONS) {   // verlet.f90:31-34
      for (int base = 0; base < nunit; base += nthr) {
        const int t = base + gt;
        double ke = 0.0;
        int sub = -1;
        if (t < nunit) {
          const Unit u = P.units[t];
          sub = u.sub;
          JP_UNIT_LOOP(q) {
            const int a = u.a[q];
            const double* v = P.v + 3 * a;
            ke += P.mass[a] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
          }
        }
        add_kin(P, c.nsub_total, 0, sub, ke);
      }
      if (!grid_barrier(P, epoch)) return;
    }
    for (int base = 0; base < nunit; base += nthr) {   // verlet.f90:144-154
      const int t = base + gt;
      double w[kCom];
      int rep = -1;
      if (t < nunit) {
        const Unit u = P.units[t];
        rep = micr_vel<FP64>(P, c, u, rep_scale(P, c, u.rep), w);
        JP_UNIT_LOOP(q) zero_force<FP64>(P, u.a[q]);
      }
      if (c.stop) com_add(P, c, 0, rep, w);
    }
    if (c.stop && !grid_barrier(P, epoch)) return;
    for (int base = 0; base < nunit; base += nthr) {   // verlet.f90:157-215
      const int t = base + gt;
      double ke = 0.0;
      int sub = -1;
      if (t < nunit) {
        const Unit u = P.units[t];
        sub = u.sub;
        ke = micr_pos<FP64>(P, c, u);
      }
      add_kin(P, c.nsub_total, c.nkin - 1, sub, ke);
    }
  } else {
    for (int base = 0; base < nunit; base += nthr) {
      const int t = base + gt;
      double ke = 0.0;
      int sub = -1;
      if (t < nunit) {
        const Unit u = P.units[t];
        sub = u.sub;
        ke = micr_unit<FP64>(P, c, u, rep_scale(P, c, u.rep));
        JP_UNIT_LOOP(q) zero_force<FP64>(P, u.a[q]);
      }
      add_kin(P, c.nsub_total, c.nkin - 1, sub, ke);
    }
  }
  finish_last(P, c, c.temp);
}

// ---- METHOD= CANO / GE: verlethe.f90 ----------------------------------------------------
// Streaming form of a 1-3 atom unit: its state lives in the atom arrays between phases (the
// per-phase launches below; 4-atom groups take the eight-lane form further down).  Each
// function reads everything it needs of the unit's atoms before it writes anything: the atom
// arrays are separate pointers that the compiler must assume may overlap, so a store placed
// between two loads holds the later load back until the store's own inputs have arrived, and
// a unit would wait for memory once per atom component instead of once.

// an atom's slot record, read ahead of the position update that rewrites it (write_slot)
struct SlotRef {
  int s;
  float w;          // the mixed path's scaled charge (pos_f.w)
  double o[3];      // the mixed path's block frame origin of the slot
  double w64;       // the FP64 path's scaled charge (pos_d.w)
};

template <bool FP64>
__device__ __forceinline__ void slot_load(const DevPtrs& P, int a, SlotRef& r) {
  r.s = P.slot_of[a];
  if (FP64) {
    r.w64 = P.pos_d[r.s].w;
  } else {
    r.w = P.pos_f[r.s].w;
    for (int k = 0; k < 3; ++k) r.o[k] = P.off[3 * r.s + k];
  }
}

template <bool FP64>
__device__ __forceinline__ void slot_store(const DevPtrs& P, const SlotRef& r, const double* x) {
  if (FP64) P.pos_d[r.s] = make_double4(x[0], x[1], x[2], r.w64);
  else P.pos_f[r.s] = make_float4((float)(x[0] - r.o[0]), (float)(x[1] - r.o[1]), (float)(x[2] - r.o[2]), r.w);
}

// phase 1 (verlethe.f90:380-398): back up x, v; velt = v - dt/2 c g/m; KE(velt) -> slot 0
template <bool FP64>
__device__ __forceinline__ double cano1_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s) {
  const double rt = 0.5 * c.dt * kConvcv;
  double g[3][3], v[3][3], x[3][3], im[3], m[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    load_grad<FP64>(P, a, s, g[q]);
    im[q] = P.imass[a];
    m[q] = P.mass[a];
    for (int k = 0; k < 3; ++k) {
      v[q][k] = P.v[3 * a + k];
      x[q][k] = P.x[3 * a + k];
    }
  }
  double ke = 0.0;
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      P.x0[3 * a + k] = x[q][k];
      P.vback[3 * a + k] = v[q][k];
      const double vt = v[q][k] - rt * g[q][k] * im[q];
      vv += vt * vt;
    }
    ke += m[q] * vv;
  }
  return ke;
}

// phase 2 (verlethe.f90:400-516): chi from slot 0; v = (2chi-1)v - chi dt c g/m; x += dt v
template <bool FP64>
__device__ __forceinline__ void cano2_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                           double tt) {
  const bool shk = c.shake_method != JP_SHAKE_NONE;
  const double tempc = shk ? sub_temp(P, c, 0, u.sub) : c.temp;
  const double chi = sqrt(tt / tempc);
  const double a1 = chi * c.dt * kConvcv, b1 = 2.0 * chi - 1.0;
  double g[3][3], v[3][3], x[3][3], im[3];
  SlotRef sl[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    load_grad<FP64>(P, a, s, g[q]);
    im[q] = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      v[q][k] = P.v[3 * a + k];
      x[q][k] = P.x[3 * a + k];
    }
    if (!shk) slot_load<FP64>(P, a, sl[q]);
  }
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    for (int k = 0; k < 3; ++k) {
      const double vn = b1 * v[q][k] - a1 * g[q][k] * im[q];
      x[q][k] += c.dt * vn;
      P.v[3 * a + k] = vn;
      P.x[3 * a + k] = x[q][k];
      P.forcec[3 * a + k] = 0.0;
    }
    if (!shk) slot_store<FP64>(P, sl[q], x[q]);
  }
}

// The SHAKE pass after a velocity update of a 1-3 atom unit, on positions in registers: x1
// (the updated positions) is written to xback, constrained against x0, and becomes x with
// v = (x1 - x0)/dt; returns the kinetic term of (vb + v)/2, vb = v(t - dt/2).
template <bool FP64>
__device__ __forceinline__ double shake_finish_unit(const DevPtrs& P, const IntConst& c, const Unit& u,
                                                    const double* im, const double* m, const SlotRef* sl,
                                                    double (*x1)[3], const double (*x0)[3],
                                                    const double (*vb)[3]) {
  JP_SMALL_LOOP(q)
    for (int k = 0; k < 3; ++k) P.xback[3 * u.a[q] + k] = x1[q][k];
  if (u.n >= 2) {
    const int ier = shake_small(P.reps[u.rep], u.n, u.d2, im, x1, x0, c.shake_method, c.shake_tol,
                                c.shake_maxit);
    if (ier) shake_status(P, ier, u.rep);
  }
  const double ri = 1.0 / c.dt;
  bool bad = false;
  double ke = 0.0;
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double v = (x1[q][k] - x0[q][k]) * ri;
      P.v[3 * a + k] = v;
      P.x[3 * a + k] = x1[q][k];
      const double vt = 0.5 * (vb[q][k] + v);
      vv += vt * vt;
      bad |= !isfinite(x1[q][k]);
    }
    ke += m[q] * vv;
    slot_store<FP64>(P, sl[q], x1[q]);
  }
  if (bad) atomicOr(P.status, ERR_NONFINITE);
  return ke;
}

// phase 3 of an iteration (verlethe.f90:524-612): SHAKE, v = (x-x0)/dt,
// velt = (vback+v)/2, KE(velt)
template <bool FP64>
__device__ __forceinline__ double cano3_unit(const DevPtrs& P, const IntConst& c, const Unit& u) {
  double x1[3][3], x0[3][3], vb[3][3], im[3], m[3];
  SlotRef sl[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    im[q] = P.imass[a];
    m[q] = P.mass[a];
    for (int k = 0; k < 3; ++k) {
      x1[q][k] = P.x[3 * a + k];
      x0[q][k] = P.x0[3 * a + k];
      vb[q][k] = P.vback[3 * a + k];
    }
    slot_load<FP64>(P, a, sl[q]);
  }
  return shake_finish_unit<FP64>(P, c, u, im, m, sl, x1, x0, vb);
}

// phase 4 (verlethe.f90:625-640): forcec += (x - xback)/dt^2; velt; KE
template <bool FP64>
__device__ __forceinline__ double cano4_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s) {
  const double r2 = 1.0 / (c.dt * c.dt), h = 0.5 * c.dt;
  double g[3][3], fc[3][3], x[3][3], xb[3][3], vb[3][3], im[3], m[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    load_grad<FP64>(P, a, s, g[q]);
    im[q] = P.imass[a];
    m[q] = P.mass[a];
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * a + k;
      fc[q][k] = P.forcec[i];
      x[q][k] = P.x[i];
      xb[q][k] = P.xback[i];
      vb[q][k] = P.vback[i];
    }
  }
  double ke = 0.0;
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double f = fc[q][k] + r2 * (x[q][k] - xb[q][k]);
      P.forcec[3 * a + k] = f;
      const double vt = h * (-kConvcv * g[q][k] * im[q] + f) + vb[q][k];
      vv += vt * vt;
    }
    ke += m[q] * vv;
  }
  return ke;
}

// phase 5 (verlethe.f90:641-718): chi from slot 2*it; v = chi dt (-c g/m + forcec) +
// (2chi-1) vback; x = x0 + dt v
template <bool FP64>
__device__ __forceinline__ void cano5_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                           int it, double tt) {
  const double chi = sqrt(tt / sub_temp(P, c, 2 * it, u.sub));
  const double a1 = chi * c.dt, b1 = 2.0 * chi - 1.0;
  double g[3][3], fc[3][3], vb[3][3], x0[3][3], im[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    load_grad<FP64>(P, a, s, g[q]);
    im[q] = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * a + k;
      fc[q][k] = P.forcec[i];
      vb[q][k] = P.vback[i];
      x0[q][k] = P.x0[i];
    }
  }
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    for (int k = 0; k < 3; ++k) {
      const double v = (-kConvcv * g[q][k] * im[q] + fc[q][k]) * a1 + vb[q][k] * b1;
      P.v[3 * a + k] = v;
      P.x[3 * a + k] = x0[q][k] + c.dt * v;
    }
  }
}

// phase 2 then phase 3 with SHAKE and no centre-of-mass stop (the form of cano2_unit followed
// by cano3_unit): phase 1 left x0 = x and vback = v, so both come from one read of x and v
template <bool FP64>
__device__ __forceinline__ double cano23_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                              double tt) {
  const double chi = sqrt(tt / sub_temp(P, c, 0, u.sub));
  const double a1 = chi * c.dt * kConvcv, b1 = 2.0 * chi - 1.0;
  double x1[3][3], x0[3][3], vb[3][3], g[3][3], im[3], m[3];
  SlotRef sl[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    load_grad<FP64>(P, a, s, g[q]);
    im[q] = P.imass[a];
    m[q] = P.mass[a];
    for (int k = 0; k < 3; ++k) {
      vb[q][k] = P.v[3 * a + k];
      x0[q][k] = P.x[3 * a + k];
    }
    slot_load<FP64>(P, a, sl[q]);
  }
  JP_SMALL_LOOP(q)
    for (int k = 0; k < 3; ++k) {
      const double v = b1 * vb[q][k] - a1 * g[q][k] * im[q];
      x1[q][k] = x0[q][k] + c.dt * v;
      P.forcec[3 * u.a[q] + k] = 0.0;
    }
  return shake_finish_unit<FP64>(P, c, u, im, m, sl, x1, x0, vb);
}

// phase 5 then phase 3 (cano5_unit followed by cano3_unit), no centre-of-mass stop
template <bool FP64>
__device__ __forceinline__ double cano53_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                              int it, double tt) {
  const double chi = sqrt(tt / sub_temp(P, c, 2 * it, u.sub));
  const double a1 = chi * c.dt, b1 = 2.0 * chi - 1.0;
  double x1[3][3], x0[3][3], vb[3][3], g[3][3], fc[3][3], im[3], m[3];
  SlotRef sl[3];
  JP_SMALL_LOOP(q) {
    const int a = u.a[q];
    load_grad<FP64>(P, a, s, g[q]);
    im[q] = P.imass[a];
    m[q] = P.mass[a];
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * a + k;
      vb[q][k] = P.vback[i];
      x0[q][k] = P.x0[i];
      fc[q][k] = P.forcec[i];
    }
    slot_load<FP64>(P, a, sl[q]);
  }
  JP_SMALL_LOOP(q)
    for (int k = 0; k < 3; ++k) {
      const double v = (-kConvcv * g[q][k] * im[q] + fc[q][k]) * a1 + vb[q][k] * b1;
      x1[q][k] = x0[q][k] + c.dt * v;
    }
  return shake_finish_unit<FP64>(P, c, u, im, m, sl, x1, x0, vb);
}

// Resident form: a 1-3 atom unit keeps its state through every phase of the step on chip:
// positions x, x0, v(t-dt/2), forcec and the shift of the last SHAKE pass in shared memory
// (component-major, 9 values per state per thread), scalars in registers.  v(t+dt/2) is
// recomputed from x and x0 after each SHAKE pass; the scaled gradient is re-read (it is not
// written during the step).
constexpr int kIntThreads = 64;

struct UnitScal {
  int n, sub, rep;
  int a[3];
  double d2[3], im[3], m[3];
};

struct UnitSmem {
  double x[9][kIntThreads], x0[9][kIntThreads], vb[9][kIntThreads];
  double dxs[9][kIntThreads], fc[9][kIntThreads];
};

template <bool FP64>
__device__ __forceinline__ void ru_grad(const DevPtrs& P, int a, double s, double* g) {
  if (FP64) {
    for (int k = 0; k < 3; ++k) g[k] = __ldg(&P.grd[3 * a + k]) * s;
  } else {
    for (int k = 0; k < 3; ++k) g[k] = (double)__ldg(&P.frc[3 * a + k]) * kFrcInv * s;
  }
  split_grad<FP64>(P, a, s, g);
}

__device__ __forceinline__ void ru_load(const DevPtrs& P, const Unit& u, UnitScal& U, UnitSmem& S,
                                        int tid) {
  U.n = u.n; U.sub = u.sub; U.rep = u.rep;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    U.d2[q] = u.d2[q];
    const bool on = q < u.n;
    const int a = on ? u.a[q] : u.a[0];
    U.a[q] = a;
    U.im[q] = on ? P.imass[a] : 0.0;
    U.m[q] = on ? P.mass[a] : 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      S.x[3 * q + k][tid] = P.x[3 * a + k];
      S.vb[3 * q + k][tid] = P.v[3 * a + k];
    }
  }
}

// phase 1: x0 = x, KE of v(t-dt/2) - dt/2 c g/m
template <bool FP64>
__device__ __forceinline__ double ru_cano1(const DevPtrs& P, const IntConst& c, const UnitScal& U,
                                           UnitSmem& S, int tid, double s) {
  const double rt = 0.5 * c.dt * kConvcv;
  double ke = 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double g[3];
    ru_grad<FP64>(P, U.a[q], s, g);
    double vv = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      S.x0[3 * q + k][tid] = S.x[3 * q + k][tid];
      const double vt = S.vb[3 * q + k][tid] - rt * g[k] * U.im[q];
      vv += vt * vt;
    }
    ke += U.m[q] * vv;
  }
  return ke;
}

// phase 2: v = (2chi-1) v - chi dt c g/m; x += dt v; forcec = 0
template <bool FP64>
__device__ __forceinline__ void ru_cano2(const DevPtrs& P, const IntConst& c, const UnitScal& U,
                                         UnitSmem& S, int tid, double s, double chi, bool shk) {
  const double a1 = chi * c.dt * kConvcv, b1 = 2.0 * chi - 1.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double g[3];
    ru_grad<FP64>(P, U.a[q], s, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * q + k;
      const double v = b1 * S.vb[i][tid] - a1 * g[k] * U.im[q];
      S.x[i][tid] += c.dt * v;
      S.fc[i][tid] = 0.0;
      if (!shk) S.dxs[i][tid] = v;   // no SHAKE: the new velocity, stored at the end
    }
  }
}

// phase 3: SHAKE + KE of (v(t-dt/2) + v(t+dt/2))/2
__device__ __forceinline__ double ru_cano3(const DevPtrs& P, const IntConst& c, const UnitScal& U,
                                           UnitSmem& S, int tid) {
  double x[3][3], x0[3][3];
#pragma unroll
  for (int q = 0; q < 3; ++q)
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      x[q][k] = S.x[3 * q + k][tid];
      x0[q][k] = S.x0[3 * q + k][tid];
    }
  if (U.n >= 2) {
    const int ier = shake_small(P.reps[U.rep], U.n, U.d2, U.im, x, x0, c.shake_method,
                                c.shake_tol, c.shake_maxit);
    if (ier) shake_status(P, ier, U.rep);
  }
  const double ri = 1.0 / c.dt;
  double ke = 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double vv = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * q + k;
      S.dxs[i][tid] = x[q][k] - S.x[i][tid];
      S.x[i][tid] = x[q][k];
      const double vt = 0.5 * (S.vb[i][tid] + (x[q][k] - x0[q][k]) * ri);
      vv += vt * vt;
    }
    ke += U.m[q] * vv;
  }
  return ke;
}

// phase 4: forcec += (x - xback)/dt^2; KE of dt/2 (-c g/m + forcec) + v(t-dt/2)
template <bool FP64>
__device__ __forceinline__ double ru_cano4(const DevPtrs& P, const IntConst& c, const UnitScal& U,
                                           UnitSmem& S, int tid, double s) {
  const double r2 = 1.0 / (c.dt * c.dt), h = 0.5 * c.dt;
  double ke = 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double g[3];
    ru_grad<FP64>(P, U.a[q], s, g);
    double vv = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * q + k;
      const double fc = S.fc[i][tid] + r2 * S.dxs[i][tid];
      S.fc[i][tid] = fc;
      const double vt = h * (-kConvcv * g[k] * U.im[q] + fc) + S.vb[i][tid];
      vv += vt * vt;
    }
    ke += U.m[q] * vv;
  }
  return ke;
}

// phase 5: v = chi dt (-c g/m + forcec) + (2chi-1) v(t-dt/2); x = x0 + dt v
template <bool FP64>
__device__ __forceinline__ void ru_cano5(const DevPtrs& P, const IntConst& c, const UnitScal& U,
                                         UnitSmem& S, int tid, double s, double chi) {
  const double a1 = chi * c.dt, b1 = 2.0 * chi - 1.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    double g[3];
    ru_grad<FP64>(P, U.a[q], s, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * q + k;
      const double v = (-kConvcv * g[k] * U.im[q] + S.fc[i][tid]) * a1 + S.vb[i][tid] * b1;
      S.x[i][tid] = S.x0[i][tid] + c.dt * v;
    }
  }
}

// ---- 4-atom SHAKE groups: eight lanes per group ------------------------------------------
// Lanes 0-3 of an aligned group of 8 hold the group's atoms (state in the shared-memory slot
// of the lane, component 0-2); lanes 0-5 hold its constraints in md_run's pair order
// (shake.f90 parlis: 1-2, 2-3, 3-1, 4-1, 3-4, 2-4).  Warps that carry 4-atom groups carry
// nothing else, so every lane of such a warp runs the same code and the width-8 shuffles
// below are always warp-convergent.
struct QLane {
  int sl;            // lane in the group (0-7)
  int a;             // atom of this lane (sl < 4), else -1
  int sub, rep;      // -1 / 0 for lanes of an empty group
  bool grp;          // the group exists
  double im, m;      // inverse mass, mass of the atom (0 without one)
  double len2;       // squared length of constraint sl (sl < 6)
};

__device__ __forceinline__ QLane ql_make(const DevPtrs& P, const IntConst& c, int v) {
  QLane q;
  const int g = (v - c.qbase) >> 3;
  q.sl = v & 7;
  q.grp = g < c.nquad;
  q.a = -1; q.sub = -1; q.rep = 0; q.im = 0.0; q.m = 0.0; q.len2 = 1.0;
  if (q.grp) {
    const Unit& u = P.units[P.quad_idx[g]];
    q.sub = u.sub;
    q.rep = u.rep;
    if (q.sl < 4) {
      q.a = u.a[q.sl];
      q.im = P.imass[q.a];
      q.m = P.mass[q.a];
    }
    if (q.sl < 6) q.len2 = u.d2[q.sl];
  }
  return q;
}

// 1/a by Newton's iteration for the reciprocal, y <- y + y (1 - a y), from the hardware's
// approximate reciprocal: each step squares the relative error, two give full double
// precision (within an ulp of the rounded quotient) for the normal, well-scaled pivots of
// the 4-atom SHAKE solve, at a fraction of an IEEE division's latency
__device__ __forceinline__ double recip_nr(double a) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  y = fma(y, fma(-a, y, 1.0), y);
  y = fma(y, fma(-a, y, 1.0), y);
  return y;
}

__device__ __forceinline__ double sum8(double v) {
  v += __shfl_xor_sync(0xffffffffu, v, 4, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 2, 8);
  v += __shfl_xor_sync(0xffffffffu, v, 1, 8);
  return v;
}

// kinetic sum of a quad warp: one value per group (replicated in its 8 lanes)
__device__ __forceinline__ void add_kin_quad(const DevPtrs& P, int nsub_total, int kslot, int sub,
                                             double ke_grp) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  long long* dst = P.kin_fix + (size_t)kslot * nsub_total;
  const int s0 = __shfl_sync(full, sub, 0);
  double e = (lane & 7) == 0 ? ke_grp : 0.0;
  if (__all_sync(full, sub == s0)) {
    e += __shfl_xor_sync(full, e, 8);
    e += __shfl_xor_sync(full, e, 16);
    if (lane == 0 && s0 >= 0) atomic_add_ll(&dst[s0], to_fix(e, kKinScale, P.status));
  } else if ((lane & 7) == 0 && sub >= 0 && ke_grp != 0.0) {
    atomic_add_ll(&dst[sub], to_fix(ke_grp, kKinScale, P.status));
  }
}

// shake4 (shake.f90:333-562) for one group spread over its 8 lanes: each constraint lane
// builds its row of the Newton matrix, the LU with partial pivoting (simulu) eliminates the
// rows held by the lanes that are not yet pivots, and back substitution broadcasts G one
// entry at a time.  Same iteration, pivot rule, elimination arithmetic and convergence test
// as the serial form.  x (in/out) and x0 are this lane's atom (lanes 0-3).  Returns 0, 1 (not
// converged) or -2 (singular), the same value in all lanes of the group.
__device__ int quad_shake(const Rep& R, const QLane& q, double x[3], const double x0[3], double tol,
                          int maxit) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int sl = q.sl;
  const int pi_ = sl == 0 ? 0 : sl == 1 ? 1 : sl == 2 ? 2 : sl == 3 ? 3 : sl == 4 ? 2 : 1;
  const int pj_ = sl == 0 ? 1 : sl == 1 ? 2 : sl == 2 ? 0 : sl == 3 ? 0 : 3;
  const bool con = q.grp && sl < 6;
  double d1[3], d2[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double xi = __shfl_sync(full, x[k], pi_, 8), xj = __shfl_sync(full, x[k], pj_, 8);
    const double yi = __shfl_sync(full, x0[k], pi_, 8), yj = __shfl_sync(full, x0[k], pj_, 8);
    d1[k] = xi - xj;
    d2[k] = yi - yj;
  }
  mimg(R, d1);
  mimg(R, d2);
  double D2[6][3], im4[4], cr[6];
#pragma unroll
  for (int ig = 0; ig < 6; ++ig)
#pragma unroll
    for (int k = 0; k < 3; ++k) D2[ig][k] = __shfl_sync(full, d2[k], ig, 8);
#pragma unroll
  for (int a = 0; a < 4; ++a) im4[a] = __shfl_sync(full, q.im, a, 8);
#pragma unroll
  for (int ig = 0; ig < 6; ++ig) cr[ig] = sl < 6 ? cg4(sl, ig, im4) : 0.0;
  double wk[3] = {d1[0], d1[1], d1[2]};
  double G[6] = {0, 0, 0, 0, 0, 0};
  bool done = !q.grp;
  bool singular = false;
  int ret = 0;
  for (int it = 0; it < maxit; ++it) {
    const double B0 = q.len2 - (wk[0] * wk[0] + wk[1] * wk[1] + wk[2] * wk[2]);
    const bool bad = con && fabs(B0) >= tol * q.len2;
    const unsigned gbits = (__ballot_sync(full, bad) >> (lane & 24)) & 0xffu;
    if (!done && gbits == 0u) {   // converged: 3) modify r1 (shake.f90:478-489)
      done = true;
      ret = singular ? -2 : 0;
      if (sl < 4) {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          double w;
          if (sl == 0) w = G[0] * D2[0][k] - G[2] * D2[2][k] - G[3] * D2[3][k];
          else if (sl == 1) w = -G[0] * D2[0][k] + G[1] * D2[1][k] + G[5] * D2[5][k];
          else if (sl == 2) w = -G[1] * D2[1][k] + G[2] * D2[2][k] + G[4] * D2[4][k];
          else w = G[3] * D2[3][k] - G[4] * D2[4][k] - G[5] * D2[5][k];
          x[k] += q.im * w;
        }
      }
    }
    if (__all_sync(full, done)) return q.grp ? ret : 0;
    // gradient matrix row of this constraint and the right-hand side
    double A[6];
#pragma unroll
    for (int ig = 0; ig < 6; ++ig)
      A[ig] = 2.0 * cr[ig] * (wk[0] * D2[ig][0] + wk[1] * D2[ig][1] + wk[2] * D2[ig][2]);
    double B = B0;
#pragma unroll
    for (int ig = 0; ig < 6; ++ig) B += A[ig] * G[ig];
    // LU with partial pivoting over the constraint lanes
    bool used = !con;
    bool lu_ok = true;
    int perm[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
      double bv = used ? -1.0 : fabs(A[k]);
      int bl = sl;
#pragma unroll
      for (int off = 4; off > 0; off >>= 1) {
        const double ov = __shfl_xor_sync(full, bv, off, 8);
        const int ol = __shfl_xor_sync(full, bl, off, 8);
        if (ov > bv || (ov == bv && ol < bl)) { bv = ov; bl = ol; }
      }
      perm[k] = bl;
      double pk[6];
#pragma unroll
      for (int j = k; j < 6; ++j) pk[j] = __shfl_sync(full, A[j], bl, 8);
      const double pb = __shfl_sync(full, B, bl, 8);
      if (fabs(pk[k]) < 1.0e-30) lu_ok = false;
      const double piv = recip_nr(pk[k]);
      if (sl == bl) {
        used = true;
        A[k] = piv;
      } else if (!used) {
        const double f = A[k] * piv;
#pragma unroll
        for (int j = k + 1; j < 6; ++j) A[j] -= f * pk[j];
        B -= f * pb;
      }
    }
    // back substitution: every lane of the warp runs the shuffles (lu_ok and done differ
    // between the groups of a warp); only a live group with a regular matrix takes the result
    const bool take = lu_ok && !done;
    if (!lu_ok && !done) singular = true;
#pragma unroll
    for (int i = 5; i >= 0; --i) {
      double t = B;
#pragma unroll
      for (int j = i + 1; j < 6; ++j) t -= A[j] * G[j];
      const double gi = __shfl_sync(full, t * A[i], perm[i], 8);
      if (take) G[i] = gi;
    }
    if (!done) {
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        double w = d1[k];
#pragma unroll
        for (int ig = 0; ig < 6; ++ig) w += cr[ig] * D2[ig][k] * G[ig];
        wk[k] = w;
      }
    }
  }
  if (!done) ret = singular ? -2 : 1;
  return q.grp ? ret : 0;
}

// the per-atom phases of a quad lane, on its shared-memory slot (component 0-2)
template <bool FP64, class SM>
__device__ __forceinline__ double q_cano1(const DevPtrs& P, const IntConst& c, const QLane& q,
                                          SM& S, int tid, double s) {
  double ke = 0.0;
  if (q.a >= 0) {
    const double rt = 0.5 * c.dt * kConvcv;
    double g[3];
    ru_grad<FP64>(P, q.a, s, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      S.x0[k][tid] = S.x[k][tid];
      const double vt = S.vb[k][tid] - rt * g[k] * q.im;
      ke += vt * vt;
    }
    ke *= q.m;
  }
  return sum8(ke);
}

template <bool FP64, class SM>
__device__ __forceinline__ void q_cano2(const DevPtrs& P, const IntConst& c, const QLane& q,
                                        SM& S, int tid, double s, double chi) {
  if (q.a < 0) return;
  const double a1 = chi * c.dt * kConvcv, b1 = 2.0 * chi - 1.0;
  double g[3];
  ru_grad<FP64>(P, q.a, s, g);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = b1 * S.vb[k][tid] - a1 * g[k] * q.im;
    S.x[k][tid] += c.dt * v;
    S.fc[k][tid] = 0.0;
  }
}

template <class SM>
__device__ __forceinline__ double q_cano3(const DevPtrs& P, const IntConst& c, const QLane& q,
                                          SM& S, int tid) {
  double x[3], x0[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    x[k] = S.x[k][tid];
    x0[k] = S.x0[k][tid];
  }
  const int ier = quad_shake(P.reps[q.rep], q, x, x0, c.shake_tol, c.shake_maxit);
  if (ier && q.sl == 0) shake_status(P, ier, q.rep);
  double ke = 0.0;
  if (q.a >= 0) {
    const double ri = 1.0 / c.dt;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      S.dxs[k][tid] = x[k] - S.x[k][tid];
      S.x[k][tid] = x[k];
      const double vt = 0.5 * (S.vb[k][tid] + (x[k] - x0[k]) * ri);
      ke += vt * vt;
    }
    ke *= q.m;
  }
  return sum8(ke);
}

template <bool FP64, class SM>
__device__ __forceinline__ double q_cano4(const DevPtrs& P, const IntConst& c, const QLane& q,
                                          SM& S, int tid, double s) {
  double ke = 0.0;
  if (q.a >= 0) {
    const double r2 = 1.0 / (c.dt * c.dt), h = 0.5 * c.dt;
    double g[3];
    ru_grad<FP64>(P, q.a, s, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      const double fc = S.fc[k][tid] + r2 * S.dxs[k][tid];
      S.fc[k][tid] = fc;
      const double vt = h * (-kConvcv * g[k] * q.im + fc) + S.vb[k][tid];
      ke += vt * vt;
    }
    ke *= q.m;
  }
  return sum8(ke);
}

template <bool FP64, class SM>
__device__ __forceinline__ void q_cano5(const DevPtrs& P, const IntConst& c, const QLane& q,
                                        SM& S, int tid, double s, double chi) {
  if (q.a < 0) return;
  const double a1 = chi * c.dt, b1 = 2.0 * chi - 1.0;
  double g[3];
  ru_grad<FP64>(P, q.a, s, g);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double v = (-kConvcv * g[k] * q.im + S.fc[k][tid]) * a1 + S.vb[k][tid] * b1;
    S.x[k][tid] = S.x0[k][tid] + c.dt * v;
  }
}

// streaming form of a quad lane: its slot is filled from and returned to the atom arrays
// around each phase (x, x0, v(t-dt/2) = vback, forcec, and x - xback for the SHAKE shift)
template <class SM>
__device__ __forceinline__ void q_fetch(const DevPtrs& P, const QLane& q, SM& S, int tid, bool first) {
  if (q.a < 0) return;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int i = 3 * q.a + k;
    S.x[k][tid] = P.x[i];
    if (first) {
      S.vb[k][tid] = P.v[i];
      S.fc[k][tid] = 0.0;
      S.dxs[k][tid] = 0.0;
    } else {
      S.x0[k][tid] = P.x0[i];
      S.vb[k][tid] = P.vback[i];
      S.fc[k][tid] = P.forcec[i];
      S.dxs[k][tid] = P.x[i] - P.xback[i];
    }
  }
}

template <class SM>
__device__ __forceinline__ void q_spill(const DevPtrs& P, const IntConst& c, const QLane& q, SM& S,
                                        int tid, bool fp64) {
  if (q.a < 0) return;
  const double ri = 1.0 / c.dt;
  double xq[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const int i = 3 * q.a + k;
    xq[k] = S.x[k][tid];
    P.x[i] = xq[k];
    P.x0[i] = S.x0[k][tid];
    P.vback[i] = S.vb[k][tid];
    P.forcec[i] = S.fc[k][tid];
    P.xback[i] = xq[k] - S.dxs[k][tid];
    P.v[i] = (xq[k] - S.x0[k][tid]) * ri;
  }
  if (!isfinite(xq[0]) || !isfinite(xq[1]) || !isfinite(xq[2])) atomicOr(P.status, ERR_NONFINITE);
  write_slot(P, q.a, xq, fp64);
}

// Centre-of-mass stop in the CANO/GE kernel (verlethe.f90:490-492, :706-709).  After a
// velocity update a lane holds x0 (time t) and x = x0 + dt v; its stopped atoms add their sums
// (v recovered as (x - x0)/dt), and after the grid barrier the correction moves x by
// -dt (tv + w x (x0 - centre)) (and v without SHAKE), which is the remotv-corrected velocity
// carried into the position update.
__device__ __forceinline__ int com_small(const DevPtrs& P, const IntConst& c, const UnitScal& U,
                                         const UnitSmem& S, int tid, double* w) {
  const Rep& R = P.reps[U.rep];
  const double ri = 1.0 / c.dt;
  bool any = false;
#pragma unroll
  for (int k = 0; k < kCom; ++k) w[k] = 0.0;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q < U.n && stopped(R, U.a[q])) {
      double x0[3], v[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        x0[k] = S.x0[3 * q + k][tid];
        v[k] = (S.x[3 * q + k][tid] - x0[k]) * ri;
      }
      com_terms(U.m[q], x0, v, w);
      any = true;
    }
  }
  return any ? U.rep : -1;
}

__device__ __forceinline__ void fix_small(const DevPtrs& P, const IntConst& c, int slot, const UnitScal& U,
                                          UnitSmem& S, int tid, bool shk) {
  const Rep& R = P.reps[U.rep];
  ComFix F;
  if (!unit_stopped<3>(R, U.n, U.a) || !com_fix(P, c, slot, U.rep, F)) return;
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q < U.n && stopped(R, U.a[q])) {
      double x0[3], d[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) x0[k] = S.x0[3 * q + k][tid];
      com_delta(F, x0, d);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        S.x[3 * q + k][tid] -= c.dt * d[k];
        if (!shk) S.dxs[3 * q + k][tid] -= d[k];
      }
    }
  }
}

template <class SM>
__device__ __forceinline__ int com_quad(const DevPtrs& P, const IntConst& c, const QLane& q, const SM& S,
                                        int tid, double* w) {
#pragma unroll
  for (int k = 0; k < kCom; ++k) w[k] = 0.0;
  if (q.a < 0 || !stopped(P.reps[q.rep], q.a)) return -1;
  const double ri = 1.0 / c.dt;
  double x0[3], v[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    x0[k] = S.x0[k][tid];
    v[k] = (S.x[k][tid] - x0[k]) * ri;
  }
  com_terms(q.m, x0, v, w);
  return q.rep;
}

template <class SM>
__device__ __forceinline__ void fix_quad(const DevPtrs& P, const IntConst& c, int slot, const QLane& q,
                                         SM& S, int tid) {
  ComFix F;
  if (q.a < 0 || !stopped(P.reps[q.rep], q.a) || !com_fix(P, c, slot, q.rep, F)) return;
  double x0[3], d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) x0[k] = S.x0[k][tid];
  com_delta(F, x0, d);
#pragma unroll
  for (int k = 0; k < 3; ++k) S.x[k][tid] -= c.dt * d[k];
}

// streaming form: the unit's x0 and x in the atom arrays
__device__ __forceinline__ int com_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double* w) {
  const Rep& R = P.reps[u.rep];
  const double ri = 1.0 / c.dt;
  bool any = false;
#pragma unroll
  for (int k = 0; k < kCom; ++k) w[k] = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    if (stopped(R, a)) {
      double x0[3], v[3];
      for (int k = 0; k < 3; ++k) {
        x0[k] = P.x0[3 * a + k];
        v[k] = (P.x[3 * a + k] - x0[k]) * ri;
      }
      com_terms(P.mass[a], x0, v, w);
      any = true;
    }
  }
  return any ? u.rep : -1;
}

__device__ __forceinline__ void fix_unit(const DevPtrs& P, const IntConst& c, int slot, const Unit& u,
                                         bool shk, bool fp64) {
  const Rep& R = P.reps[u.rep];
  ComFix F;
  if (!unit_stopped<4>(R, u.n, u.a) || !com_fix(P, c, slot, u.rep, F)) return;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    if (stopped(R, a)) {
      double x0[3], d[3];
      for (int k = 0; k < 3; ++k) x0[k] = P.x0[3 * a + k];
      com_delta(F, x0, d);
      for (int k = 0; k < 3; ++k) {
        P.x[3 * a + k] -= c.dt * d[k];
        if (!shk) P.v[3 * a + k] -= d[k];
      }
      if (!shk) write_slot(P, a, P.x + 3 * a, fp64);
    }
  }
}

// Whole step for all replicas, one cooperative launch, when every virtual lane has a thread of
// its own: [0, nsmall) one 1-3 atom unit each, [qbase, nvirt) eight lanes per 4-atom group, all
// unit state on chip for the whole step, a grid barrier between phases.
template <bool FP64, bool STOP>
__global__ void __launch_bounds__(kIntThreads) k_cano_fused(DevPtrs P, IntConst c) {
  __shared__ UnitSmem S;
  __shared__ unsigned char s_act[kActCache];   // replicas still in the SHAKE<->thermostat loop
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const int tid = threadIdx.x;
  const double tt = target_temp(c, (long long)P.step_ctr[0] + 1);
  const bool shk = c.shake_method != JP_SHAKE_NONE;
  unsigned epoch = 0;
  if (gt < c.nrep) write_ene_hist(P, c, gt);
  // ALSD: thread r carries lambda of replica r (c.alsd: some replica has clusters)
  LamStep L{};
  const bool lam_thread = c.alsd && gt < c.nrep && P.reps[gt].lam_mode != 0;
  if (lam_thread) lam_begin(P, c, gt, L, shk);
  // the lane's state (warp-uniform kinds: qbase and nvirt are multiples of 32)
  UnitScal U;
  QLane Q;
  const bool small = gt < c.nsmall;
  const bool quad = gt >= c.qbase && gt < c.nvirt;
  double s = 1.0;
  if (small) {
    const Unit u = P.units[P.small_idx[gt]];
    ru_load(P, u, U, S, tid);
    s = rep_scale(P, c, u.rep);
  } else if (quad) {
    Q = ql_make(P, c, gt);
    q_fetch(P, Q, S, tid, true);
    s = rep_scale(P, c, Q.rep);
  }
  // phase 1 (verlethe.f90:380-398); with the centre-of-mass stop also without SHAKE (x0)
  if (shk || STOP) {
    if (quad) {   // warp-uniform: one kinetic-sum call site per warp kind
      add_kin_quad(P, c.nsub_total, 0, Q.sub, q_cano1<FP64>(P, c, Q, S, tid, s));
    } else {
      const double ke = small ? ru_cano1<FP64>(P, c, U, S, tid, s) : 0.0;
      add_kin(P, c.nsub_total, 0, small ? U.sub : -1, ke);
    }
    if (!grid_barrier(P, epoch)) return;
  }
  if (lam_thread) lam_advance(P, c, gt, L, tt, shk);
  // phase 2 (verlethe.f90:400-516) + phase 3 of the first SHAKE pass; the centre-of-mass
  // stop puts its sums and a grid barrier between the two (com slot 0)
  constexpr bool split = STOP;   // c.stop != 0
  {
    double w[kCom];
    if (quad) {
      const double chi = Q.grp ? sqrt(tt / sub_temp(P, c, 0, Q.sub)) : 1.0;
      q_cano2<FP64>(P, c, Q, S, tid, s, chi);
      if (split) com_add(P, c, 0, com_quad(P, c, Q, S, tid, w), w);
      else add_kin_quad(P, c.nsub_total, 1, Q.sub, q_cano3(P, c, Q, S, tid));
    } else {
      double ke = 0.0;
      if (small) {
        const double chi = sqrt(tt / (shk ? sub_temp(P, c, 0, U.sub) : c.temp));
        ru_cano2<FP64>(P, c, U, S, tid, s, chi, shk);
        if (shk && !split) ke = ru_cano3(P, c, U, S, tid);
      }
      if (split) com_add(P, c, 0, small ? com_small(P, c, U, S, tid, w) : -1, w);
      else if (shk) add_kin(P, c.nsub_total, 1, small ? U.sub : -1, ke);
    }
  }
  if (split) {
    if (!grid_barrier(P, epoch)) return;
    // the correction, then phase 3
    if (quad) {
      fix_quad(P, c, 0, Q, S, tid);
      add_kin_quad(P, c.nsub_total, 1, Q.sub, q_cano3(P, c, Q, S, tid));
    } else {
      double ke = 0.0;
      if (small) {
        fix_small(P, c, 0, U, S, tid, shk);
        if (shk) ke = ru_cano3(P, c, U, S, tid);
      }
      if (shk) add_kin(P, c.nsub_total, 1, small ? U.sub : -1, ke);
    }
  }
  if (shk) {
    for (int it = 1; it < c.icslop; ++it) {
      if (!grid_barrier(P, epoch)) return;
      if (!any_active(P, c, it, tt, s_act)) break;
      // lambda's velocity stays (v_back + v)/2 through the loop (verlethe.f90:529)
      const bool lam_act = lam_thread && rep_active(P, c, s_act, gt, it, tt);
      if (lam_act) {
        lam_add_ke(P, c, P.reps[gt], 2 * it, L.lvt);
        lam_add_ke(P, c, P.reps[gt], 2 * it + 1, L.lvt);
      }
      // phase 4 (verlethe.f90:625-640)
      if (quad) {
        const bool act = Q.grp && rep_active(P, c, s_act, Q.rep, it, tt);
        const double ke = q_cano4<FP64>(P, c, Q, S, tid, s);
        add_kin_quad(P, c.nsub_total, 2 * it, act ? Q.sub : -1, act ? ke : 0.0);
      } else {
        const bool act = small && rep_active(P, c, s_act, U.rep, it, tt);
        const double ke = act ? ru_cano4<FP64>(P, c, U, S, tid, s) : 0.0;
        add_kin(P, c.nsub_total, 2 * it, act ? U.sub : -1, ke);
      }
      if (!grid_barrier(P, epoch)) return;
      // phase 5 (verlethe.f90:641-718) + phase 3 of the next SHAKE pass; with the
      // centre-of-mass stop: phase 5 and the sums (com slot it), barrier, correction + phase 3
      if (split) {
        double w[kCom];
        int rep = -1;
        if (!quad) {
          if (small && rep_active(P, c, s_act, U.rep, it, tt)) {
            ru_cano5<FP64>(P, c, U, S, tid, s, sqrt(tt / sub_temp(P, c, 2 * it, U.sub)));
            rep = com_small(P, c, U, S, tid, w);
          }
        } else if (Q.grp && rep_active(P, c, s_act, Q.rep, it, tt)) {
          q_cano5<FP64>(P, c, Q, S, tid, s, sqrt(tt / sub_temp(P, c, 2 * it, Q.sub)));
          rep = com_quad(P, c, Q, S, tid, w);
        }
        com_add(P, c, it, rep, w);
        if (!grid_barrier(P, epoch)) return;
        // the correction, then phase 3
        if (!quad) {
          const bool act = small && rep_active(P, c, s_act, U.rep, it, tt);
          double ke = 0.0;
          if (act) {
            fix_small(P, c, it, U, S, tid, shk);
            ke = ru_cano3(P, c, U, S, tid);
          }
          add_kin(P, c.nsub_total, 2 * it + 1, act ? U.sub : -1, ke);
        } else {
          const bool act = Q.grp && rep_active(P, c, s_act, Q.rep, it, tt);
          double sx[3], sdx[3];
#pragma unroll
          for (int k = 0; k < 3; ++k) { sx[k] = S.x[k][tid]; sdx[k] = S.dxs[k][tid]; }
          if (act) fix_quad(P, c, it, Q, S, tid);
          const double ke = q_cano3(P, c, Q, S, tid);
          if (!act && Q.a >= 0) {
#pragma unroll
            for (int k = 0; k < 3; ++k) { S.x[k][tid] = sx[k]; S.dxs[k][tid] = sdx[k]; }
          }
          add_kin_quad(P, c.nsub_total, 2 * it + 1, act ? Q.sub : -1, act ? ke : 0.0);
        }
        continue;
      }
      if (!quad) {
        const bool act = small && rep_active(P, c, s_act, U.rep, it, tt);
        double ke = 0.0;
        if (act) {
          ru_cano5<FP64>(P, c, U, S, tid, s, sqrt(tt / sub_temp(P, c, 2 * it, U.sub)));
          ke = ru_cano3(P, c, U, S, tid);
        }
        add_kin(P, c.nsub_total, 2 * it + 1, act ? U.sub : -1, ke);
      } else {
        // the whole warp runs the SHAKE (its shuffles); inactive groups keep their state
        const bool act = Q.grp && rep_active(P, c, s_act, Q.rep, it, tt);
        double sx[3], sdx[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) { sx[k] = S.x[k][tid]; sdx[k] = S.dxs[k][tid]; }
        if (act) q_cano5<FP64>(P, c, Q, S, tid, s, sqrt(tt / sub_temp(P, c, 2 * it, Q.sub)));
        const double ke = q_cano3(P, c, Q, S, tid);
        if (!act && Q.a >= 0) {
#pragma unroll
          for (int k = 0; k < 3; ++k) { S.x[k][tid] = sx[k]; S.dxs[k][tid] = sdx[k]; }
        }
        add_kin_quad(P, c.nsub_total, 2 * it + 1, act ? Q.sub : -1, act ? ke : 0.0);
      }
    }
  }
  // the lane's new state back to memory
  if (small) {
    bool bad = false;
    const double ri = 1.0 / c.dt;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      if (q < U.n) {
        const int a = U.a[q];
        double xq[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
          const int i = 3 * q + k;
          xq[k] = S.x[i][tid];
          P.x[3 * a + k] = xq[k];
          P.v[3 * a + k] = shk ? (xq[k] - S.x0[i][tid]) * ri : S.dxs[i][tid];
          bad |= !isfinite(xq[k]);
        }
        write_slot(P, a, xq, FP64);
      }
    }
    if (bad) atomicOr(P.status, ERR_NONFINITE);
#pragma unroll
    for (int q = 0; q < 3; ++q)
      if (q < U.n) zero_force<FP64>(P, U.a[q]);
  } else if (quad) {
    q_spill(P, c, Q, S, tid, FP64);
    if (Q.a >= 0) zero_force<FP64>(P, Q.a);
  }
  if (lam_thread) {
    P.lam[2 * gt] = L.lam;
    P.lam[2 * gt + 1] = L.lv;
  }
  finish_last(P, c, tt);
}

// ---- METHOD= CANO / GE, streaming form: one launch per phase -------------------------------
// A system with more virtual lanes than the cooperative launch holds at once runs its step as
// a chain of ordinary launches with one virtual lane per thread, so that every lane's loads
// are in flight together: each launch is one phase of the form above, the launch boundary
// stands where that form has a grid barrier, and a lane's state is in the atom arrays between
// launches (x, x0, v, vback, xback, forcec).  A launch for a SHAKE <-> thermostat pass that no
// replica still runs returns at once.  Lambda's state through the step is kept in lam_step.
enum : int {
  PH_BEGIN = 0,     // energy record, lambda force; phase 1
  PH_UPDATE = 1,    // lambda advance; phase 2, then phase 3 (with the stop: its sums, slot 0)
  PH_FIX = 2,       // with the stop: correction by the sums of slot `it`, then phase 3
  PH_CORR = 3,      // pass `it`: phase 4
  PH_RESCALE = 4,   // pass `it`: phase 5, then phase 3 (with the stop: its sums, slot it)
  PH_END = 5        // forces cleared, lambda stored, temperatures and step counters
};

// blocks per SM the unit-lane launches are compiled for (their registers: 65,536 / (64 x this));
// on C4 a bound of 8 (128 registers, with spills) measured 3 % slower than 4 (no spills)
constexpr int kPhaseBlocks = 4;

// shared-memory state of the 4-atom group lanes of a launch (component 0-2)
struct QuadSmem {
  double x[3][kIntThreads], x0[3][kIntThreads], vb[3][kIntThreads];
  double dxs[3][kIntThreads], fc[3][kIntThreads];
};

__device__ __forceinline__ void lam_save(const DevPtrs& P, int r, const LamStep& L) {
  double* d = P.lam_step + 5 * r;
  d[0] = L.lam; d[1] = L.lv; d[2] = L.lvback; d[3] = L.lf; d[4] = L.lvt;
}

__device__ __forceinline__ void lam_load(const DevPtrs& P, int r, LamStep& L) {
  const double* d = P.lam_step + 5 * r;
  L.lam = d[0]; L.lv = d[1]; L.lvback = d[2]; L.lf = d[3]; L.lvt = d[4];
}

// KIND 0: the 1-3 atom units [0, nsmall) and the per-replica threads (energy record,
// lambda); KIND 1: the 4-atom group lanes [qbase, nvirt) (a launch of its own, as their
// SHAKE needs several times the registers); KIND 2 (PH_END only): every lane.
template <bool FP64, bool STOP, int PH, int KIND>
__global__ void __launch_bounds__(kIntThreads, KIND == 1 ? 4 : kPhaseBlocks) k_cano_phase(DevPtrs P, IntConst c, int it) {
  __shared__ QuadSmem S;
  __shared__ unsigned char s_act[kActCache];
  const int v = (KIND == 1 ? c.qbase : 0) + blockIdx.x * blockDim.x + threadIdx.x;
  const int tid = threadIdx.x;
  const double tt = target_temp(c, (long long)P.step_ctr[0] + 1);
  const bool shk = c.shake_method != JP_SHAKE_NONE;
  const bool lam_thread = KIND != 1 && c.alsd && v < c.nrep && P.reps[v].lam_mode != 0;
  const bool small = KIND != 1 && v < c.nsmall;
  const bool quad = KIND != 0 && v >= c.qbase && v < c.nvirt;   // warp-uniform (multiples of 32)
  constexpr bool split = STOP;
  if (PH == PH_BEGIN) {
    if (KIND == 0 && v < c.nrep) write_ene_hist(P, c, v);
    if (lam_thread) {
      LamStep L{};
      lam_begin(P, c, v, L, shk);
      lam_save(P, v, L);
    }
    if (!(shk || STOP)) return;
    if (quad) {
      const QLane q = ql_make(P, c, v);
      q_fetch(P, q, S, tid, true);
      const double ke = q_cano1<FP64>(P, c, q, S, tid, rep_scale(P, c, q.rep));
      q_spill(P, c, q, S, tid, FP64);
      add_kin_quad(P, c.nsub_total, 0, q.sub, ke);
    } else {
      double ke = 0.0;
      int sub = -1;
      if (small) {
        const Unit u = P.units[P.small_idx[v]];
        sub = u.sub;
        ke = cano1_unit<FP64>(P, c, u, rep_scale(P, c, u.rep));
      }
      add_kin(P, c.nsub_total, 0, sub, ke);
    }
  } else if (PH == PH_UPDATE) {
    if (lam_thread) {
      LamStep L;
      lam_load(P, v, L);
      lam_advance(P, c, v, L, tt, shk);
      lam_save(P, v, L);
    }
    double w[kCom];
    if (quad) {
      const QLane q = ql_make(P, c, v);
      q_fetch(P, q, S, tid, false);
      const double chi = q.grp ? sqrt(tt / sub_temp(P, c, 0, q.sub)) : 1.0;
      q_cano2<FP64>(P, c, q, S, tid, rep_scale(P, c, q.rep), chi);
      if (split) {
        const int rep = com_quad(P, c, q, S, tid, w);
        q_spill(P, c, q, S, tid, FP64);
        com_add(P, c, 0, rep, w);
      } else {
        const double ke = q_cano3(P, c, q, S, tid);
        q_spill(P, c, q, S, tid, FP64);
        add_kin_quad(P, c.nsub_total, 1, q.sub, ke);
      }
    } else {
      double ke = 0.0;
      int sub = -1, rep = -1;
      if (small) {
        const Unit u = P.units[P.small_idx[v]];
        if (split || !shk) {
          cano2_unit<FP64>(P, c, u, rep_scale(P, c, u.rep), tt);
          if (split) rep = com_unit(P, c, u, w);
        } else {
          sub = u.sub;
          ke = cano23_unit<FP64>(P, c, u, rep_scale(P, c, u.rep), tt);
        }
      }
      if (split) com_add(P, c, 0, rep, w);
      else if (shk) add_kin(P, c.nsub_total, 1, sub, ke);
    }
  } else if (PH == PH_FIX) {
    // after phase 2 (it = 0, every replica) or after phase 5 of pass it
    if (it > 0 && !any_active(P, c, it, tt, s_act)) return;
    const int ks = it == 0 ? 1 : 2 * it + 1;
    if (quad) {
      const QLane q = ql_make(P, c, v);
      const bool act = it == 0 || (q.grp && rep_active(P, c, s_act, q.rep, it, tt));
      q_fetch(P, q, S, tid, false);
      if (act) fix_quad(P, c, it, q, S, tid);
      const double ke = q_cano3(P, c, q, S, tid);
      if (act) q_spill(P, c, q, S, tid, FP64);
      add_kin_quad(P, c.nsub_total, ks, act ? q.sub : -1, act ? ke : 0.0);
    } else {
      double ke = 0.0;
      int sub = -1;
      if (small) {
        const Unit u = P.units[P.small_idx[v]];
        if (it == 0 || rep_active(P, c, s_act, u.rep, it, tt)) {
          fix_unit(P, c, it, u, shk, FP64);
          if (shk) {
            sub = u.sub;
            ke = cano3_unit<FP64>(P, c, u);
          }
        }
      }
      if (shk) add_kin(P, c.nsub_total, ks, sub, ke);
    }
  } else if (PH == PH_CORR) {
    if (!any_active(P, c, it, tt, s_act)) return;
    // lambda's velocity stays (v_back + v)/2 through the loop (verlethe.f90:529)
    if (lam_thread && rep_active(P, c, s_act, v, it, tt)) {
      LamStep L;
      lam_load(P, v, L);
      lam_add_ke(P, c, P.reps[v], 2 * it, L.lvt);
      lam_add_ke(P, c, P.reps[v], 2 * it + 1, L.lvt);
    }
    if (quad) {
      const QLane q = ql_make(P, c, v);
      const bool act = q.grp && rep_active(P, c, s_act, q.rep, it, tt);
      q_fetch(P, q, S, tid, false);
      const double ke = q_cano4<FP64>(P, c, q, S, tid, rep_scale(P, c, q.rep));
      if (act) q_spill(P, c, q, S, tid, FP64);
      add_kin_quad(P, c.nsub_total, 2 * it, act ? q.sub : -1, act ? ke : 0.0);
    } else {
      double ke = 0.0;
      int sub = -1;
      if (small) {
        const Unit u = P.units[P.small_idx[v]];
        if (rep_active(P, c, s_act, u.rep, it, tt)) {
          sub = u.sub;
          ke = cano4_unit<FP64>(P, c, u, rep_scale(P, c, u.rep));
        }
      }
      add_kin(P, c.nsub_total, 2 * it, sub, ke);
    }
  } else if (PH == PH_RESCALE) {
    if (!any_active(P, c, it, tt, s_act)) return;
    if (split) {
      double w[kCom];
      int rep = -1;
      if (quad) {
        const QLane q = ql_make(P, c, v);
        if (q.grp && rep_active(P, c, s_act, q.rep, it, tt)) {
          q_fetch(P, q, S, tid, false);
          q_cano5<FP64>(P, c, q, S, tid, rep_scale(P, c, q.rep), sqrt(tt / sub_temp(P, c, 2 * it, q.sub)));
          rep = com_quad(P, c, q, S, tid, w);
          q_spill(P, c, q, S, tid, FP64);
        }
      } else if (small) {
        const Unit u = P.units[P.small_idx[v]];
        if (rep_active(P, c, s_act, u.rep, it, tt)) {
          cano5_unit<FP64>(P, c, u, rep_scale(P, c, u.rep), it, tt);
          rep = com_unit(P, c, u, w);
        }
      }
      com_add(P, c, it, rep, w);
    } else if (quad) {
      const QLane q = ql_make(P, c, v);
      const bool act = q.grp && rep_active(P, c, s_act, q.rep, it, tt);
      q_fetch(P, q, S, tid, false);
      if (act)
        q_cano5<FP64>(P, c, q, S, tid, rep_scale(P, c, q.rep), sqrt(tt / sub_temp(P, c, 2 * it, q.sub)));
      const double ke = q_cano3(P, c, q, S, tid);   // the whole warp runs the SHAKE shuffles
      if (act) q_spill(P, c, q, S, tid, FP64);
      add_kin_quad(P, c.nsub_total, 2 * it + 1, act ? q.sub : -1, act ? ke : 0.0);
    } else {
      double ke = 0.0;
      int sub = -1;
      if (small) {
        const Unit u = P.units[P.small_idx[v]];
        if (rep_active(P, c, s_act, u.rep, it, tt)) {
          sub = u.sub;
          ke = cano53_unit<FP64>(P, c, u, rep_scale(P, c, u.rep), it, tt);
        }
      }
      add_kin(P, c.nsub_total, 2 * it + 1, sub, ke);
    }
  } else {   // PH_END
    if (quad) {
      const QLane q = ql_make(P, c, v);
      if (q.a >= 0) zero_force<FP64>(P, q.a);
    } else if (small) {
      const Unit u = P.units[P.small_idx[v]];
      JP_UNIT_LOOP(q) zero_force<FP64>(P, u.a[q]);
    }
    if (lam_thread) {
      LamStep L;
      lam_load(P, v, L);
      P.lam[2 * v] = L.lam;
      P.lam[2 * v + 1] = L.lv;
    }
    finish_last(P, c, tt);
  }
}

// ---- standalone SHAKE (test hook): r1 constrained against r2, positions in xback / x0 -----
__global__ void k_shake_only(DevPtrs P, IntConst c, int unit0, int nunit) {
  const int tt = blockIdx.x * blockDim.x + threadIdx.x;
  if (tt >= nunit) return;
  const int t = unit0 + tt;
  const Unit u = P.units[t];
  if (u.n < 2) return;
  const Rep& R = P.reps[u.rep];
  double x1[4][3], x0[4][3], im[4];
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    im[q] = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      x1[q][k] = P.xback[3 * a + k];
      x0[q][k] = P.x0[3 * a + k];
    }
  }
  const int ier = shake_group(R, u, im, x1, x0, c.shake_method, c.shake_tol, c.shake_maxit);
  if (ier) shake_status(P, ier, u.rep);
  JP_UNIT_LOOP(q)
    for (int k = 0; k < 3; ++k) P.xback[3 * u.a[q] + k] = x1[q][k];
}

// ---- launches -----------------------------------------------------------------------------
template <class K>
static int coop_grid(K kernel, int device) {
  int nsm = 0, per = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 64, 0);
  return nsm * (per > 0 ? per : 1);
}

int cano_grid(bool fp64, int device) {
  // the smallest co-resident grid among the cooperative integration kernels of this precision
  int g;
  if (fp64) {
    g = coop_grid(k_cano_fused<true, false>, device);
    g = std::min(g, coop_grid(k_cano_fused<true, true>, device));
    g = std::min(g, coop_grid(k_micr_fused<true, false>, device));
    g = std::min(g, coop_grid(k_micr_fused<true, true>, device));
  } else {
    g = coop_grid(k_cano_fused<false, false>, device);
    g = std::min(g, coop_grid(k_cano_fused<false, true>, device));
    g = std::min(g, coop_grid(k_micr_fused<false, false>, device));
    g = std::min(g, coop_grid(k_micr_fused<false, true>, device));
  }
  return g;
}

template <class... Args>
static void coop_launch(void (*kernel)(Args...), int grid, cudaStream_t st, Args... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(64);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cudaLaunchKernelEx(&cfg, kernel, args...);
}

// does a CANO/GE step of this system take the per-phase launches (more virtual lanes than
// the cooperative grid holds)?
static bool cano_streaming(const IntConst& c, int grid_max) {
  if (c.method <= JP_METHOD_MICR) return false;
  const int want = std::max(1, (c.nvirt + kIntThreads - 1) / kIntThreads);
  return want > grid_max;
}

// one phase: the unit lanes (and per-replica threads), then the 4-atom group lanes
template <bool FP64, bool STOP, int PH>
static void launch_phase(const DevPtrs& P, const IntConst& c, int it, cudaStream_t st) {
  const int g0 = (std::max(c.nsmall, c.nrep) + kIntThreads - 1) / kIntThreads;
  const int g1 = (c.nvirt - c.qbase + kIntThreads - 1) / kIntThreads;
  k_cano_phase<FP64, STOP, PH, 0><<<g0, kIntThreads, 0, st>>>(P, c, it);
  if (g1 > 0) k_cano_phase<FP64, STOP, PH, 1><<<g1, kIntThreads, 0, st>>>(P, c, it);
}

template <bool FP64, bool STOP>
static void launch_cano_phases(const DevPtrs& P, const IntConst& c, cudaStream_t st) {
  const bool shk = c.shake_method != JP_SHAKE_NONE;
  launch_phase<FP64, STOP, PH_BEGIN>(P, c, 0, st);
  launch_phase<FP64, STOP, PH_UPDATE>(P, c, 0, st);
  if (STOP) launch_phase<FP64, STOP, PH_FIX>(P, c, 0, st);
  if (shk) {
    for (int it = 1; it < c.icslop; ++it) {
      launch_phase<FP64, STOP, PH_CORR>(P, c, it, st);
      launch_phase<FP64, STOP, PH_RESCALE>(P, c, it, st);
      if (STOP) launch_phase<FP64, STOP, PH_FIX>(P, c, it, st);
    }
  }
  const int grid = (std::max(c.nvirt, c.nrep) + kIntThreads - 1) / kIntThreads;
  k_cano_phase<FP64, STOP, PH_END, 2><<<grid, kIntThreads, 0, st>>>(P, c, 0);
}

int integrate_launches(const IntConst& c, int grid_max) {
  if (!cano_streaming(c, grid_max)) return 1;
  const bool stop = c.stop != 0, shk = c.shake_method != JP_SHAKE_NONE;
  int phases = 2 + (stop ? 1 : 0);
  if (shk) phases += std::max(0, c.icslop - 1) * (stop ? 3 : 2);
  int n = phases * (c.nvirt > c.qbase ? 2 : 1) + 1;            // + PH_END
  if (c.method == JP_METHOD_GE && !c.ge_prescaled) n += 1;   // k_ge_scale
  return n;
}

void launch_integrate(const DevPtrs& P, const IntConst& c, int nunit, bool fp64, int grid_max,
                      cudaStream_t st) {
  // bar, the kinetic sums and the centre-of-mass sums are zero here: created so, and reset
  // by the last block of the previous integration (or by the host after an error)
  const bool verlet = c.method <= JP_METHOD_MICR;   // MICR or CONS
  const bool stop = c.stop != 0;
  if (verlet) {
    const int want = std::max(1, (nunit + kIntThreads - 1) / kIntThreads);
    const int grid = std::min(want, grid_max);
    const bool split = stop || c.method == JP_METHOD_CONS;
    if (fp64) coop_launch(split ? k_micr_fused<true, true> : k_micr_fused<true, false>, grid, st, P, c, nunit);
    else coop_launch(split ? k_micr_fused<false, true> : k_micr_fused<false, false>, grid, st, P, c, nunit);
  } else if (!cano_streaming(c, grid_max)) {
    const int grid = std::max(1, (c.nvirt + kIntThreads - 1) / kIntThreads);
    if (fp64) coop_launch(stop ? k_cano_fused<true, true> : k_cano_fused<true, false>, grid, st, P, c);
    else coop_launch(stop ? k_cano_fused<false, true> : k_cano_fused<false, false>, grid, st, P, c);
  } else {
    // every lane of every phase reads the replica's force scale: McMD polynomials are
    // evaluated once per replica beforehand
    IntConst cs = c;
    if (c.method == JP_METHOD_GE && !c.ge_prescaled) {
      launch_ge_scale(P, c, st);
      cs.ge_prescaled = 1;
    }
    if (fp64) {
      if (stop) launch_cano_phases<true, true>(P, cs, st);
      else launch_cano_phases<true, false>(P, cs, st);
    } else {
      if (stop) launch_cano_phases<false, true>(P, cs, st);
      else launch_cano_phases<false, false>(P, cs, st);
    }
  }
}

void launch_shake_only(const DevPtrs& P, const IntConst& c, int unit0, int nunit, cudaStream_t st) {
  if (nunit <= 0) return;
  k_shake_only<<<(nunit + 127) / 128, 128, 0, st>>>(P, c, unit0, nunit);
}

}  // namespace jp
