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

namespace jp {

// Loop over the 1-4 atoms of an integration unit.  The trip count is fixed at 4 and fully
// unrolled with a guard: the per-unit arrays then live in registers.  (A runtime trip count
// over these small local arrays produced wrong values on sm_100a with nvcc 12.9.)
#define JP_UNIT_LOOP(q) _Pragma("unroll") for (int q = 0; q < 4; ++q) if (q < u.n)

__host__ __device__ __forceinline__ void mimg(const Rep& R, double* d) {
  for (int k = 0; k < 3; ++k) d[k] -= R.box[k] * anint(d[k] * R.invbox[k]);
}

template <bool FP64>
__device__ __forceinline__ void load_grad(const DevPtrs& P, int a, double s, double* g) {
  if (FP64) {
    for (int k = 0; k < 3; ++k) g[k] = P.grd[3 * a + k] * s;
  } else {
    for (int k = 0; k < 3; ++k) g[k] = (double)P.frc[3 * a + k] * kFrcInv * s;
  }
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

__device__ __forceinline__ void shake_status(const DevPtrs& P, int ier) {
  if (ier == 1) atomicOr(P.status, ERR_SHAKE_NOCONV);
  else if (ier == -2) atomicOr(P.status, ERR_SHAKE_SINGULAR);
}

// warp-aggregated fixed-point add of m v^2 into kin_fix[slot][sub]
__device__ __forceinline__ void add_kin(const DevPtrs& P, int nsub_total, int kslot, int sub, double e) {
  const unsigned full = 0xffffffffu;
  const int s0 = __shfl_sync(full, sub, 0);
  long long* dst = P.kin_fix + (size_t)kslot * nsub_total;
  if (__all_sync(full, sub == s0)) {
    for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(full, e, o);
    if ((threadIdx.x & 31) == 0 && s0 >= 0) atomic_add_ll(&dst[s0], to_fix(e, kKinScale));
  } else if (sub >= 0 && e != 0.0) {
    atomic_add_ll(&dst[sub], to_fix(e, kKinScale));
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
__device__ double rep_scale(const DevPtrs& P, const IntConst& c, int r) {
  const Rep& R = P.reps[r];
  if (c.method == JP_METHOD_GE && R.ge_nwin > 0) {
    double tot = R.dself;
    for (int k = 1; k < JP_MAXENE; ++k) tot += (double)__ldcg(&P.ene_fix[r * 16 + k]) * kEneInv;
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
  double* out = P.ene_hist + ((size_t)P.step_ctr[1] * c.nrep + r) * JP_MAXENE;
  for (int k = 0; k < JP_MAXENE; ++k) out[k] = e[k];
}

// Grid barrier for a cooperative launch (all blocks co-resident).  bar[0] arrivals,
// bar[1] generation, bar[2] abort.  The wait is bounded (~1 s of SM clock): on timeout the
// kernel records ERR_TIMEOUT, raises abort and every block returns at its next barrier.
constexpr long long kBarrierCycles = 2000000000LL;

__device__ __forceinline__ bool grid_barrier(const DevPtrs& P) {
  __shared__ int s_ok;
  unsigned* bar = P.bar;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    volatile unsigned* vb = bar;
    const unsigned gen = vb[1];
    __threadfence();
    if (atomicAdd(&bar[0], 1u) == gridDim.x - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicAdd(&bar[1], 1u);
    } else {
      const long long t0 = clock64();
      while (vb[1] == gen) {
        if (vb[2] != 0u) { ok = 0; break; }
        if (clock64() - t0 > kBarrierCycles) {
          atomicOr(P.status, ERR_TIMEOUT);
          atomicExch(&bar[2], 1u);
          ok = 0;
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// end of step, block 0 after the final barrier: temperature of each replica (the kinetic
// slot of the last SHAKE pass, i.e. of (v(t-dt/2)+v(t+dt/2))/2) and the step counters
__device__ void finish_block(const DevPtrs& P, const IntConst& c, double tt) {
  const int h = P.step_ctr[1];
  for (int r = threadIdx.x; r < c.nrep; r += blockDim.x) {
    const Rep& R = P.reps[r];
    int ks = c.nkin - 1;   // MICR
    if (c.method != JP_METHOD_MICR && c.shake_method != JP_SHAKE_NONE) {
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
        (c.method == JP_METHOD_MICR || c.shake_method != JP_SHAKE_NONE) ? ek * 1.0e7 / (kGas * nf) : -1.0;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    P.step_ctr[0] += 1;
    P.step_ctr[1] += 1;
  }
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
    if (ier) shake_status(P, ier);
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

template <bool FP64>
__global__ void __launch_bounds__(64) k_micr_fused(DevPtrs P, IntConst c, int nunit) {
  const int nthr = gridDim.x * blockDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt < c.nrep) write_ene_hist(P, c, gt);
  for (int base = 0; base < nunit; base += nthr) {
    const int t = base + gt;
    double ke = 0.0;
    int sub = -1;
    if (t < nunit) {
      const Unit u = P.units[t];
      sub = u.sub;
      ke = micr_unit<FP64>(P, c, u, rep_scale(P, c, u.rep));
    }
    add_kin(P, c.nsub_total, c.nkin - 1, sub, ke);
  }
  if (!grid_barrier(P)) return;
  if (blockIdx.x == 0) finish_block(P, c, c.temp);
}

// ---- METHOD= CANO / GE: verlethe.f90 ----------------------------------------------------
// Streaming form: one unit's state lives in global memory between phases (any number of
// units per thread; also used for 4-atom groups by the register-resident form).

// phase 1 (verlethe.f90:380-398): back up x, v; velt = v - dt/2 c g/m; KE(velt) -> slot 0
template <bool FP64>
__device__ __noinline__ double cano1_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s) {
  const double rt = 0.5 * c.dt * kConvcv;
  double ke = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double g[3];
    load_grad<FP64>(P, a, s, g);
    const double im = P.imass[a];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double v = P.v[3 * a + k];
      P.x0[3 * a + k] = P.x[3 * a + k];
      P.vback[3 * a + k] = v;
      const double vt = v - rt * g[k] * im;
      vv += vt * vt;
    }
    ke += P.mass[a] * vv;
  }
  return ke;
}

// phase 2 (verlethe.f90:400-516): chi from slot 0; v = (2chi-1)v - chi dt c g/m; x += dt v
template <bool FP64>
__device__ __noinline__ void cano2_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                        double tt) {
  double tempc = c.temp;
  if (c.shake_method != JP_SHAKE_NONE) tempc = sub_temp(P, c, 0, u.sub);
  const double chi = sqrt(tt / tempc);
  const double a1 = chi * c.dt * kConvcv, b1 = 2.0 * chi - 1.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double g[3];
    load_grad<FP64>(P, a, s, g);
    const double im = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      const double v = b1 * P.v[3 * a + k] - a1 * g[k] * im;
      P.v[3 * a + k] = v;
      P.x[3 * a + k] += c.dt * v;
      P.forcec[3 * a + k] = 0.0;
    }
    if (c.shake_method == JP_SHAKE_NONE) write_slot(P, a, P.x + 3 * a, FP64);
  }
}

// phase 3 of an iteration (verlethe.f90:524-612): SHAKE, v = (x-x0)/dt,
// velt = (vback+v)/2, KE(velt)
template <bool FP64>
__device__ __noinline__ double cano3_unit(const DevPtrs& P, const IntConst& c, const Unit& u) {
  const Rep& R = P.reps[u.rep];
  double x1[4][3], x0[4][3], im[4];
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    im[q] = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      x1[q][k] = P.x[3 * a + k];
      x0[q][k] = P.x0[3 * a + k];
      P.xback[3 * a + k] = x1[q][k];
    }
  }
  if (u.n >= 2) {
    const int ier = shake_group(R, u, im, x1, x0, c.shake_method, c.shake_tol, c.shake_maxit);
    if (ier) shake_status(P, ier);
  }
  const double ri = 1.0 / c.dt;
  bool bad = false;
  double ke = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      const double v = (x1[q][k] - x0[q][k]) * ri;
      P.v[3 * a + k] = v;
      P.x[3 * a + k] = x1[q][k];
      const double vt = 0.5 * (P.vback[3 * a + k] + v);
      vv += vt * vt;
      bad |= !isfinite(x1[q][k]);
    }
    ke += P.mass[a] * vv;
    write_slot(P, a, x1[q], FP64);
  }
  if (bad) atomicOr(P.status, ERR_NONFINITE);
  return ke;
}

// phase 4 (verlethe.f90:625-640): forcec += (x - xback)/dt^2; velt; KE
template <bool FP64>
__device__ __noinline__ double cano4_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s) {
  const double r2 = 1.0 / (c.dt * c.dt), h = 0.5 * c.dt;
  double ke = 0.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double g[3];
    load_grad<FP64>(P, a, s, g);
    const double im = P.imass[a];
    double vv = 0.0;
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * a + k;
      const double fc = P.forcec[i] + r2 * (P.x[i] - P.xback[i]);
      P.forcec[i] = fc;
      const double vt = h * (-kConvcv * g[k] * im + fc) + P.vback[i];
      vv += vt * vt;
    }
    ke += P.mass[a] * vv;
  }
  return ke;
}

// phase 5 (verlethe.f90:641-718): chi from slot 2*it; v = chi dt (-c g/m + forcec) +
// (2chi-1) vback; x = x0 + dt v
template <bool FP64>
__device__ __noinline__ void cano5_unit(const DevPtrs& P, const IntConst& c, const Unit& u, double s,
                                        int it, double tt) {
  const double chi = sqrt(tt / sub_temp(P, c, 2 * it, u.sub));
  const double a1 = chi * c.dt, b1 = 2.0 * chi - 1.0;
  JP_UNIT_LOOP(q) {
    const int a = u.a[q];
    double g[3];
    load_grad<FP64>(P, a, s, g);
    const double im = P.imass[a];
    for (int k = 0; k < 3; ++k) {
      const int i = 3 * a + k;
      const double v = (-kConvcv * g[k] * im + P.forcec[i]) * a1 + P.vback[i] * b1;
      P.v[i] = v;
      P.x[i] = P.x0[i] + c.dt * v;
    }
  }
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
__device__ __forceinline__ void ru_grad(const DevPtrs& P, const UnitScal& U, int q, double s, double* g) {
  if (FP64) {
    for (int k = 0; k < 3; ++k) g[k] = __ldg(&P.grd[3 * U.a[q] + k]) * s;
  } else {
    for (int k = 0; k < 3; ++k) g[k] = (double)__ldg(&P.frc[3 * U.a[q] + k]) * kFrcInv * s;
  }
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
    ru_grad<FP64>(P, U, q, s, g);
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
    if (ier) shake_status(P, ier);
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

// whole step for all replicas, one launch; units of 1-3 atoms held in registers when every
// unit has its own thread (RESIDENT), else streamed through global memory
template <bool FP64, bool RESIDENT>
__global__ void __launch_bounds__(kIntThreads) k_cano_fused(DevPtrs P, IntConst c, int nunit) {
  const int nthr = gridDim.x * blockDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  const double tt = target_temp(c, (long long)P.step_ctr[0] + 1);
  const bool shk = c.shake_method != JP_SHAKE_NONE;
  if (gt < c.nrep) write_ene_hist(P, c, gt);
  if (RESIDENT) {
    // ---------------- one unit per thread --------------------------------------------
    __shared__ UnitSmem S;
    const int tid = threadIdx.x;
    const bool have = gt < nunit;
    Unit u;
    u.n = 0; u.sub = -1; u.rep = 0;
    if (have) u = P.units[gt];
    const bool reg = have && u.n <= 3;
    const double s = have ? rep_scale(P, c, u.rep) : 1.0;
    UnitScal U;
    if (reg) ru_load(P, u, U, S, tid);
    const int sub = have ? u.sub : -1;
    if (shk) {
      double ke = 0.0;
      if (reg) ke = ru_cano1<FP64>(P, c, U, S, tid, s);
      else if (have) ke = cano1_unit<FP64>(P, c, u, s);
      add_kin(P, c.nsub_total, 0, sub, ke);
      if (!grid_barrier(P)) return;
    }
    // phase 2 (+ phase 3 of the first SHAKE pass)
    {
      double ke = 0.0;
      if (reg) {
        const double tempc = shk ? sub_temp(P, c, 0, U.sub) : c.temp;
        const double chi = sqrt(tt / tempc);
        const double a1 = chi * c.dt * kConvcv, b1 = 2.0 * chi - 1.0;
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          double g[3];
          ru_grad<FP64>(P, U, q, s, g);
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            const int i = 3 * q + k;
            const double v = b1 * S.vb[i][tid] - a1 * g[k] * U.im[q];
            S.x[i][tid] += c.dt * v;
            S.fc[i][tid] = 0.0;
            if (!shk) S.dxs[i][tid] = v;   // no SHAKE: the new velocity, stored below
          }
        }
        if (shk) ke = ru_cano3(P, c, U, S, tid);
      } else if (have) {
        cano2_unit<FP64>(P, c, u, s, tt);
        if (shk) ke = cano3_unit<FP64>(P, c, u);
      }
      if (shk) add_kin(P, c.nsub_total, 1, sub, ke);
    }
    if (shk) {
      for (int it = 1; it < c.icslop; ++it) {
        if (!grid_barrier(P)) return;
        const bool act = have && cano_active(P, c, P.reps[u.rep], it, true, tt);
        double ke = 0.0;
        if (act) {   // phase 4
          if (reg) {
            const double r2 = 1.0 / (c.dt * c.dt), h = 0.5 * c.dt;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              double g[3];
              ru_grad<FP64>(P, U, q, s, g);
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
          } else {
            ke = cano4_unit<FP64>(P, c, u, s);
          }
        }
        add_kin(P, c.nsub_total, 2 * it, act ? sub : -1, ke);
        if (!grid_barrier(P)) return;
        ke = 0.0;
        if (act) {   // phase 5 + phase 3 of the next pass
          if (reg) {
            const double chi = sqrt(tt / sub_temp(P, c, 2 * it, U.sub));
            const double a1 = chi * c.dt, b1 = 2.0 * chi - 1.0;
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              double g[3];
              ru_grad<FP64>(P, U, q, s, g);
#pragma unroll
              for (int k = 0; k < 3; ++k) {
                const int i = 3 * q + k;
                const double v = (-kConvcv * g[k] * U.im[q] + S.fc[i][tid]) * a1 + S.vb[i][tid] * b1;
                S.x[i][tid] = S.x0[i][tid] + c.dt * v;
              }
            }
            ke = ru_cano3(P, c, U, S, tid);
          } else {
            cano5_unit<FP64>(P, c, u, s, it, tt);
            ke = cano3_unit<FP64>(P, c, u);
          }
        }
        add_kin(P, c.nsub_total, 2 * it + 1, act ? sub : -1, ke);
      }
    }
    if (reg) {   // the unit's new state back to memory
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
    }
  } else {
    // ---------------- streaming: grid-stride over units ------------------------------
    if (shk) {
      for (int base = 0; base < nunit; base += nthr) {
        const int t = base + gt;
        double ke = 0.0;
        int sub = -1;
        if (t < nunit) {
          const Unit u = P.units[t];
          sub = u.sub;
          ke = cano1_unit<FP64>(P, c, u, rep_scale(P, c, u.rep));
        }
        add_kin(P, c.nsub_total, 0, sub, ke);
      }
      if (!grid_barrier(P)) return;
    }
    for (int base = 0; base < nunit; base += nthr) {
      const int t = base + gt;
      double ke = 0.0;
      int sub = -1;
      if (t < nunit) {
        const Unit u = P.units[t];
        cano2_unit<FP64>(P, c, u, rep_scale(P, c, u.rep), tt);
        if (shk) {
          sub = u.sub;
          ke = cano3_unit<FP64>(P, c, u);
        }
      }
      if (shk) add_kin(P, c.nsub_total, 1, sub, ke);
    }
    if (shk) {
      for (int it = 1; it < c.icslop; ++it) {
        if (!grid_barrier(P)) return;
        for (int base = 0; base < nunit; base += nthr) {
          const int t = base + gt;
          double ke = 0.0;
          int sub = -1;
          if (t < nunit) {
            const Unit u = P.units[t];
            if (cano_active(P, c, P.reps[u.rep], it, true, tt)) {
              sub = u.sub;
              ke = cano4_unit<FP64>(P, c, u, rep_scale(P, c, u.rep));
            }
          }
          add_kin(P, c.nsub_total, 2 * it, sub, ke);
        }
        if (!grid_barrier(P)) return;
        for (int base = 0; base < nunit; base += nthr) {
          const int t = base + gt;
          double ke = 0.0;
          int sub = -1;
          if (t < nunit) {
            const Unit u = P.units[t];
            if (cano_active(P, c, P.reps[u.rep], it, true, tt)) {
              cano5_unit<FP64>(P, c, u, rep_scale(P, c, u.rep), it, tt);
              sub = u.sub;
              ke = cano3_unit<FP64>(P, c, u);
            }
          }
          add_kin(P, c.nsub_total, 2 * it + 1, sub, ke);
        }
      }
    }
  }
  if (!grid_barrier(P)) return;
  if (blockIdx.x == 0) finish_block(P, c, tt);
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
  if (ier) shake_status(P, ier);
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
  // the smallest co-resident grid among the integration kernels of this precision
  int g;
  if (fp64) {
    g = coop_grid(k_cano_fused<true, true>, device);
    g = std::min(g, coop_grid(k_cano_fused<true, false>, device));
    g = std::min(g, coop_grid(k_micr_fused<true>, device));
  } else {
    g = coop_grid(k_cano_fused<false, true>, device);
    g = std::min(g, coop_grid(k_cano_fused<false, false>, device));
    g = std::min(g, coop_grid(k_micr_fused<false>, device));
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

void launch_integrate(const DevPtrs& P, const IntConst& c, int nunit, bool fp64, int grid_max,
                      cudaStream_t st) {
  cudaMemsetAsync(P.bar, 0, sizeof(unsigned) * 4, st);
  const int want = std::max(1, (nunit + 63) / 64);
  const int grid = std::min(want, grid_max);
  const bool resident = want <= grid_max;
  if (c.method == JP_METHOD_MICR) {
    if (fp64) coop_launch(k_micr_fused<true>, grid, st, P, c, nunit);
    else coop_launch(k_micr_fused<false>, grid, st, P, c, nunit);
  } else if (resident) {
    if (fp64) coop_launch(k_cano_fused<true, true>, grid, st, P, c, nunit);
    else coop_launch(k_cano_fused<false, true>, grid, st, P, c, nunit);
  } else {
    if (fp64) coop_launch(k_cano_fused<true, false>, grid, st, P, c, nunit);
    else coop_launch(k_cano_fused<false, false>, grid, st, P, c, nunit);
  }
}

void launch_shake_only(const DevPtrs& P, const IntConst& c, int unit0, int nunit, cudaStream_t st) {
  if (nunit <= 0) return;
  k_shake_only<<<(nunit + 127) / 128, 128, 0, st>>>(P, c, unit0, nunit);
}

}  // namespace jp
