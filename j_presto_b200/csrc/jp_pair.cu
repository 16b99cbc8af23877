// jp_pair.cu -- zero-dipole (ZD) cut-off Coulomb + Lennard-Jones pair kernels.
//
// Replaces enear_ZD_{redu,high,doub}_PB (src_md_run/enear.f90:2-593, lines tagged #ZD #PB):
//   co   = [r <= rc]                                  (enear.f90:134, sign(0.5,dd2i-irlim2)+.5)
//   E_el += qi qj co (1/r + b r^2 - z)                 (enear.f90:138-141)
//   E_lj += co (C12/r^12 - C6/r^6)                      (enear.f90:199-210)
//   dE/dxi = -d [qi qj co (1/r^3 - f) + co (12 C12/r^12 - 6 C6/r^6)/r^2],  d = xi - xj
// with q = charge * sqrt(332.06378/eps) (chgmod, inpcls.f90:215-227), b = 1/(2 rc^3),
// f = 1/rc^3, z = 1.5/rc (incel.f90:655-658).
//
// Work unit: a tile = (i-block, j-block) of 32 x 32 cell-sorted atoms with an interaction
// mask fixed at list-build time.  One warp per tile: lane l holds i-atom l; the j-atoms and
// their force accumulators rotate one lane per step through warp shuffles, so after 32
// steps every lane has seen every j and each j-force is back in the lane that loaded it.
// Newton's third law: each unordered pair is evaluated once.
//
// Warps take tiles one at a time from a global counter, so all finish together whatever
// their tiles hold (tile work varies with the mask).
// Mixed path: FP32 pair arithmetic on block-local coordinates (|x| < ~10 A), forces and
// energies summed per tile in FP32 then added as 64-bit fixed point (2^-32 kcal/mol/A) with
// integer atomics -- order independent, so results are bit-identical run to run.
// FP64 path: the same tiles in FP64 with absolute coordinates and FP64 force atomics.
#include "jp_kernels.h"

namespace jp {

constexpr int kPairThreads = 256;
constexpr int kPairClaim = 1;   // tiles a warp claims at a time

// a warp's energies (ELE15, VDW15; ALSD class AA / AB, BB the rest) and pair count into the
// replica's slots: 64-bit fixed point, summed per tile, so the totals do not depend on which
// warp took which tile (the kernels claim their tiles dynamically)
__device__ __forceinline__ void flush_fix(const DevPtrs& P, int rep, long long eel, long long elj,
                                          long long eaa, long long eab, long long npair, bool count,
                                          bool alsd) {
  for (int o = 16; o > 0; o >>= 1) {
    eel += __shfl_xor_sync(0xffffffffu, eel, o);
    elj += __shfl_xor_sync(0xffffffffu, elj, o);
    if (alsd) {
      eaa += __shfl_xor_sync(0xffffffffu, eaa, o);
      eab += __shfl_xor_sync(0xffffffffu, eab, o);
    }
    if (count) npair += __shfl_xor_sync(0xffffffffu, npair, o);
  }
  if ((threadIdx.x & 31) == 0 && rep >= 0) {
    atomic_add_ll(&P.ene_fix[rep * 16 + JP_E_ELE15], eel);
    atomic_add_ll(&P.ene_fix[rep * 16 + JP_E_VDW15], elj);
    if (alsd) {
      atomic_add_ll(&P.ene_cls[rep * 4 + 0], eaa);
      atomic_add_ll(&P.ene_cls[rep * 4 + 1], eab);
      atomic_add_ll(&P.ene_cls[rep * 4 + 2], eel + elj - eaa - eab);
    }
    if (count) atomicAdd(reinterpret_cast<unsigned long long*>(&P.pair_cnt[rep]),
                         static_cast<unsigned long long>(npair));
  }
}

// One 32x32 tile: lane = i atom; the j atoms are staged in the warp's shared-memory slice
// and read at (lane + k) & 31 in step k; the j-force accumulators rotate one lane per step
// (3 shuffles) so that after 32 steps each is back in the lane of its atom.
// ALSD: ci = cluster bit of the i atom; a pair with nA cluster atoms has its force times
// f2 (nA = 2, class AA), f1 (AB) or 1 (BB), and its energy also goes to ea (AA) / eb (AB).
// CMM: no cut-off (rc2 is huge) and the Coulomb term only for the pairs of `me` (the
// neighbouring-cell pairs; the rest of the tile's pairs are LJ only)
template <bool MINIMG, bool COUNT, bool ALSD, bool CMM>
__device__ __forceinline__ void tile_mixed(const float4* __restrict__ sj_pos, const int* __restrict__ sj_typ,
                                           const float2* __restrict__ s_lj, int nt1, float4 pi, int ti,
                                           float4 sh, unsigned m, unsigned me, int lane, float bx, float by, float bz,
                                           float ibx, float iby, float ibz, float rc2, float zb, float zf,
                                           float zc, float& fix, float& fiy, float& fiz, float& gjx,
                                           float& gjy, float& gjz, float& te, float& tl, int& tn,
                                           int ci, float f1, float f2, float& ea, float& eb) {
  const float xi = pi.x + sh.x, yi = pi.y + sh.y, zi = pi.z + sh.z;
  const int row = (ALSD ? (ti & kTypeMask) : ti) * nt1;
#pragma unroll 4
  for (int k = 0; k < 32; ++k) {
    const int jl = (lane + k) & 31;
    if (m & 1u) {
      const float4 pj = sj_pos[jl];
      float dx = xi - pj.x, dy = yi - pj.y, dz = zi - pj.z;
      if (MINIMG) {
        dx -= bx * rintf(dx * ibx);
        dy -= by * rintf(dy * iby);
        dz -= bz * rintf(dz * ibz);
      }
      const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (r2 <= rc2) {
        const float rinv = rsqrtf(r2);
        const float r2inv = rinv * rinv;
        const float r6inv = r2inv * r2inv * r2inv;
        const int tjr = sj_typ[jl];
        const float2 lj = s_lj[row + (ALSD ? (tjr & kTypeMask) : tjr)];
        const float qq = CMM ? ((me & 1u) ? pi.w * pj.w : 0.f) : pi.w * pj.w;
        const float v1 = lj.x * r6inv;
        const float v2 = lj.y * r6inv * r6inv;
        float fs;
        if (ALSD) {
          const float e = qq * (rinv + fmaf(zb, r2, -zc)) + (v2 - v1);
          te = fmaf(qq, rinv + fmaf(zb, r2, -zc), te);
          tl += v2 - v1;
          const int na = ci + (tjr >> 30);
          if (na == 2) ea += e;
          else if (na == 1) eb += e;
          fs = (na == 2 ? f2 : na == 1 ? f1 : 1.f) *
               fmaf(qq, fmaf(rinv, r2inv, -zf), (12.f * v2 - 6.f * v1) * r2inv);
        } else {
          te = fmaf(qq, rinv + fmaf(zb, r2, -zc), te);
          tl += v2 - v1;
          fs = fmaf(qq, fmaf(rinv, r2inv, -zf), (12.f * v2 - 6.f * v1) * r2inv);
        }
        const float fx = dx * fs, fy = dy * fs, fz = dz * fs;
        fix -= fx; fiy -= fy; fiz -= fz;
        gjx += fx; gjy += fy; gjz += fz;
        if (COUNT && (!CMM || (me & 1u))) ++tn;
      }
    }
    m >>= 1;
    if (CMM) me >>= 1;
    const int src = (lane + 1) & 31;
    gjx = __shfl_sync(0xffffffffu, gjx, src);
    gjy = __shfl_sync(0xffffffffu, gjy, src);
    gjz = __shfl_sync(0xffffffffu, gjz, src);
  }
}

template <bool COUNT, bool ALSD, bool CMM>
__global__ void __launch_bounds__(kPairThreads)
k_pair_mixed(DevPtrs P, ZdConst z) {
  extern __shared__ float2 s_lj[];
  __shared__ float4 s_jpos[kPairThreads];
  __shared__ int s_jtyp[kPairThreads];
  const int nlj = z.nt1 * z.nt1;
  for (int i = threadIdx.x; i < nlj; i += blockDim.x) s_lj[i] = P.lj_f[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  float4* sj_pos = s_jpos + (threadIdx.x & ~31);
  int* sj_typ = s_jtyp + (threadIdx.x & ~31);
  const int T = *P.ntiles;
  const float rc2 = (float)z.rc2, zb = (float)z.bcoeff, zf = (float)z.fcoeff, zc = (float)z.zcore;
  int cur_bi = -1, cur_rep = -1, ai = -1, ti = 0;
  float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
  long long gix = 0, giy = 0, giz = 0;
  long long eel = 0, elj = 0, eaa = 0, eab = 0;   // fixed point, per tile
  long long npair = 0;
  bool mi = true;
  float bx = 0.f, by = 0.f, bz = 0.f, ibx = 0.f, iby = 0.f, ibz = 0.f;
  float f1 = 1.f, f2 = 1.f;
  // tiles are claimed kPairClaim at a time from a global counter (row order: consecutive
  // tiles mostly share their i block), so warps finish together whatever their tiles hold
  for (;;) {
  int t0 = 0;
  if (lane == 0) t0 = atomicAdd(P.tile_ctr, kPairClaim);
  t0 = __shfl_sync(0xffffffffu, t0, 0);
  if (t0 >= T) break;
  const int t1 = min(T, t0 + kPairClaim);
  for (int t = t0; t < t1; ++t) {
    const int2 ij = P.tiles[t];
    if (ij.x != cur_bi) {
      if (ai >= 0 && (gix | giy | giz)) {
        atomic_add_ll(&P.frc[3 * ai + 0], gix);
        atomic_add_ll(&P.frc[3 * ai + 1], giy);
        atomic_add_ll(&P.frc[3 * ai + 2], giz);
      }
      gix = giy = giz = 0;
      cur_bi = ij.x;
      const int s = cur_bi * kTile + lane;
      pi = P.pos_f[s];
      ti = P.styp[s];
      ai = P.satom[s];
      const int rep = P.blk_rep[cur_bi];
      if (rep != cur_rep) {
        if (cur_rep >= 0) {
          flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD);
        }
        eel = elj = eaa = eab = 0;
        npair = 0;
        cur_rep = rep;
        const Rep& R = P.reps[rep];
        bx = (float)R.box[0]; by = (float)R.box[1]; bz = (float)R.box[2];
        ibx = (float)R.invbox[0]; iby = (float)R.invbox[1]; ibz = (float)R.invbox[2];
        if (ALSD) {
          const double lam = P.lam[2 * rep];
          f1 = (float)lam_factor(R.lam_mode, lam, 1);
          f2 = (float)lam_factor(R.lam_mode, lam, 0);
        }
        // Per-pair minimum image is needed only if a listed pair could reach half a box
        // length: |d| <= rlim + 2*(h_i + h_j) + motion since the build (2 A margin).
        mi = false;
        for (int k = 0; k < 3; ++k)
          if (0.5 * R.box[k] < z.rlim + 4.0 * (double)P.rep_hmax[3 * rep + k] + 2.0) mi = true;
      }
    }
    const float4 sh = P.tile_shift[t];
    const unsigned m = P.masks[(size_t)t * 32 + lane];
    const unsigned me = CMM ? P.masks_el[(size_t)t * 32 + lane] : 0u;
    const int sj = ij.y * kTile + lane;
    __syncwarp();
    sj_pos[lane] = P.pos_f[sj];
    sj_typ[lane] = P.styp[sj];
    __syncwarp();
    float gjx = 0.f, gjy = 0.f, gjz = 0.f;
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float te = 0.f, tl = 0.f, ea = 0.f, eb = 0.f;
    int tn = 0;
    const int ci = ALSD ? (ti >> 30) : 0;
    if (mi)
      tile_mixed<true, COUNT, ALSD, CMM>(sj_pos, sj_typ, s_lj, z.nt1, pi, ti, sh, m, me, lane, bx, by, bz, ibx,
                                    iby, ibz, rc2, zb, zf, zc, fix, fiy, fiz, gjx, gjy, gjz, te, tl, tn,
                                    ci, f1, f2, ea, eb);
    else
      tile_mixed<false, COUNT, ALSD, CMM>(sj_pos, sj_typ, s_lj, z.nt1, pi, ti, sh, m, me, lane, bx, by, bz, ibx,
                                     iby, ibz, rc2, zb, zf, zc, fix, fiy, fiz, gjx, gjy, gjz, te, tl,
                                     tn, ci, f1, f2, ea, eb);
    const int aj = P.satom[sj];
    if (aj >= 0 && (gjx != 0.f || gjy != 0.f || gjz != 0.f)) {
      atomic_add_ll(&P.frc[3 * aj + 0], to_fix((double)gjx, kFrcScale));
      atomic_add_ll(&P.frc[3 * aj + 1], to_fix((double)gjy, kFrcScale));
      atomic_add_ll(&P.frc[3 * aj + 2], to_fix((double)gjz, kFrcScale));
    }
    gix += to_fix((double)fix, kFrcScale);
    giy += to_fix((double)fiy, kFrcScale);
    giz += to_fix((double)fiz, kFrcScale);
    eel += to_fix((double)te, kEneScale);
    elj += to_fix((double)tl, kEneScale);
    if (ALSD) { eaa += to_fix((double)ea, kEneScale); eab += to_fix((double)eb, kEneScale); }
    if (COUNT) npair += tn;
  }
  }
  if (ai >= 0 && (gix | giy | giz)) {
    atomic_add_ll(&P.frc[3 * ai + 0], gix);
    atomic_add_ll(&P.frc[3 * ai + 1], giy);
    atomic_add_ll(&P.frc[3 * ai + 2], giz);
  }
  flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD);
}

template <bool COUNT, bool ALSD, bool CMM>
__global__ void __launch_bounds__(kPairThreads)
k_pair_fp64(DevPtrs P, ZdConst z) {
  extern __shared__ double2 s_ljd[];
  const int nlj = z.nt1 * z.nt1;
  for (int i = threadIdx.x; i < nlj; i += blockDim.x) s_ljd[i] = P.lj_d[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int T = *P.ntiles;
  const double irlim2 = 1.0 / z.rc2;
  int cur_bi = -1, cur_rep = -1, ai = -1, ti = 0;
  double4 pi = make_double4(0, 0, 0, 0);
  double gix = 0, giy = 0, giz = 0;
  long long eel = 0, elj = 0, eaa = 0, eab = 0;   // fixed point, per tile
  long long npair = 0;
  double bx = 0, by = 0, bz = 0, ibx = 0, iby = 0, ibz = 0;
  double f1 = 1.0, f2 = 1.0;
  // tiles claimed one at a time, as in the mixed kernel
  for (;;) {
  int t = 0;
  if (lane == 0) t = atomicAdd(P.tile_ctr, 1);
  t = __shfl_sync(0xffffffffu, t, 0);
  if (t >= T) break;
  {
    const int2 ij = P.tiles[t];
    if (ij.x != cur_bi) {
      if (ai >= 0) {
        atomicAdd(&P.grd[3 * ai + 0], gix);
        atomicAdd(&P.grd[3 * ai + 1], giy);
        atomicAdd(&P.grd[3 * ai + 2], giz);
      }
      gix = giy = giz = 0;
      cur_bi = ij.x;
      const int s = cur_bi * kTile + lane;
      pi = P.pos_d[s];
      ti = P.styp[s];
      ai = P.satom[s];
      const int rep = P.blk_rep[cur_bi];
      if (rep != cur_rep) {
        if (cur_rep >= 0) {
          flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD);
        }
        eel = elj = eaa = eab = 0;
        npair = 0;
        cur_rep = rep;
        const Rep& R = P.reps[rep];
        bx = R.box[0]; by = R.box[1]; bz = R.box[2];
        ibx = R.invbox[0]; iby = R.invbox[1]; ibz = R.invbox[2];
        if (ALSD) {
          f1 = lam_factor(R.lam_mode, P.lam[2 * rep], 1);
          f2 = lam_factor(R.lam_mode, P.lam[2 * rep], 0);
        }
      }
    }
    unsigned m = P.masks[(size_t)t * 32 + lane];
    unsigned me = CMM ? P.masks_el[(size_t)t * 32 + lane] : 0u;
    const int sj = ij.y * kTile + lane;
    double4 pj = P.pos_d[sj];
    int tj = P.styp[sj];
    const int row = (ALSD ? (ti & kTypeMask) : ti) * z.nt1;
    const int ci = ALSD ? (ti >> 30) : 0;
    double gjx = 0, gjy = 0, gjz = 0;
    int tn = 0;
    double te = 0.0, tl = 0.0, ta = 0.0, tb = 0.0;   // this tile's energies
#pragma unroll 2
    for (int k = 0; k < 32; ++k) {
      if (m & 1u) {
        double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
        dx -= bx * anint(dx * ibx);
        dy -= by * anint(dy * iby);
        dz -= bz * anint(dz * ibz);
        const double dd2 = dx * dx + dy * dy + dz * dz;
        const double dd2i = 1.0 / dd2;
        if (dd2i - irlim2 >= 0.0) {
          const double ddi = sqrt(dd2i);
          const double dd6i = dd2i * dd2i * dd2i;
          const double ee = CMM ? ((me & 1u) ? pi.w * pj.w : 0.0) : pi.w * pj.w;
          const double epair = ee * (ddi + z.bcoeff * dd2 - z.zcore);
          te += epair;
          const double2 lj = s_ljd[row + (ALSD ? (tj & kTypeMask) : tj)];
          const double v1 = lj.x * dd6i;
          const double v2 = lj.y * dd6i * dd6i;
          tl += -v1 + v2;
          double cc = ee * (dd2i * ddi - z.fcoeff) + (-6.0 * v1 + 12.0 * v2) * dd2i;
          if (ALSD) {
            const int na = ci + (tj >> 30);
            if (na == 2) { ta += epair + (-v1 + v2); cc *= f2; }
            else if (na == 1) { tb += epair + (-v1 + v2); cc *= f1; }
          }
          const double fx = dx * cc, fy = dy * cc, fz = dz * cc;
          gix -= fx; giy -= fy; giz -= fz;
          gjx += fx; gjy += fy; gjz += fz;
          if (COUNT && (!CMM || (me & 1u))) ++tn;
        }
      }
      m >>= 1;
      if (CMM) me >>= 1;
      const int src = (lane + 1) & 31;
      pj.x = __shfl_sync(0xffffffffu, pj.x, src);
      pj.y = __shfl_sync(0xffffffffu, pj.y, src);
      pj.z = __shfl_sync(0xffffffffu, pj.z, src);
      pj.w = __shfl_sync(0xffffffffu, pj.w, src);
      tj = __shfl_sync(0xffffffffu, tj, src);
      gjx = __shfl_sync(0xffffffffu, gjx, src);
      gjy = __shfl_sync(0xffffffffu, gjy, src);
      gjz = __shfl_sync(0xffffffffu, gjz, src);
    }
    const int aj = P.satom[sj];
    if (aj >= 0 && (gjx != 0.0 || gjy != 0.0 || gjz != 0.0)) {
      atomicAdd(&P.grd[3 * aj + 0], gjx);
      atomicAdd(&P.grd[3 * aj + 1], gjy);
      atomicAdd(&P.grd[3 * aj + 2], gjz);
    }
    if (COUNT) npair += tn;
    eel += to_fix(te, kEneScale);
    elj += to_fix(tl, kEneScale);
    if (ALSD) { eaa += to_fix(ta, kEneScale); eab += to_fix(tb, kEneScale); }
  }
  }
  if (ai >= 0) {
    atomicAdd(&P.grd[3 * ai + 0], gix);
    atomicAdd(&P.grd[3 * ai + 1], giy);
    atomicAdd(&P.grd[3 * ai + 2], giz);
  }
  flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD);
}

int pair_blocks_per_sm(bool fp64, int nt1) {
  int per = 0;
  if (fp64)
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair_fp64<false, false, false>, kPairThreads,
                                                  sizeof(double2) * nt1 * nt1);
  else
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair_mixed<false, false, false>, kPairThreads,
                                                  sizeof(float2) * nt1 * nt1);
  return per > 0 ? per : 1;
}

void launch_pair_mixed(const DevPtrs& P, const ZdConst& z, int nwarps, bool, bool count, bool alsd,
                       cudaStream_t st) {
  const int wpb = kPairThreads / 32;
  const int nb = (nwarps + wpb - 1) / wpb;
  const size_t sh = sizeof(float2) * z.nt1 * z.nt1;
  if (z.cmm) {
    if (count) k_pair_mixed<true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
  } else if (alsd) {
    if (count) k_pair_mixed<true, true, false><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, true, false><<<nb, kPairThreads, sh, st>>>(P, z);
  } else {
    if (count) k_pair_mixed<true, false, false><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, false, false><<<nb, kPairThreads, sh, st>>>(P, z);
  }
}

void launch_pair_fp64(const DevPtrs& P, const ZdConst& z, int nwarps, bool count, bool alsd,
                      cudaStream_t st) {
  const int wpb = kPairThreads / 32;
  const int nb = (nwarps + wpb - 1) / wpb;
  const size_t sh = sizeof(double2) * z.nt1 * z.nt1;
  if (z.cmm) {
    if (count) k_pair_fp64<true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_fp64<false, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
  } else if (alsd) {
    if (count) k_pair_fp64<true, true, false><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_fp64<false, true, false><<<nb, kPairThreads, sh, st>>>(P, z);
  } else {
    if (count) k_pair_fp64<true, false, false><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_fp64<false, false, false><<<nb, kPairThreads, sh, st>>>(P, z);
  }
}

// slot positions from the master coordinates (after an external coordinate change)
__global__ void k_update_pos(DevPtrs P, int nslot, int fp64, double qscale) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslot) return;
  int a = P.satom[s];
  if (a < 0) return;
  const double x = P.x[3 * a], y = P.x[3 * a + 1], zz = P.x[3 * a + 2];
  if (fp64) {
    P.pos_d[s] = make_double4(x, y, zz, qscale * P.chg[a]);
  } else {
    P.pos_f[s] = make_float4((float)(x - P.off[3 * s]), (float)(y - P.off[3 * s + 1]),
                             (float)(zz - P.off[3 * s + 2]), (float)(qscale * P.chg[a]));
  }
}

void launch_update_pos(const DevPtrs& P, int nslot, bool fp64, double qscale, cudaStream_t st) {
  k_update_pos<<<(nslot + 255) / 256, 256, 0, st>>>(P, nslot, fp64 ? 1 : 0, qscale);
}

}  // namespace jp
