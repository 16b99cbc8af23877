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
// Work unit: a pair record (jp_cells.cu) = half an i-block (16 cell-sorted atoms) and 32 j
// entries (j atoms with at least one listed pair in the half block, each with the image
// shift of its block) with an interaction mask fixed at list-build time.  One warp takes two
// consecutive records, a half-warp each: lane l (l < 16 of its half) holds i atom l and at
// step k (k < 16) meets entries a = (l + k) & 15 and b = 16 + a; the j-force accumulators of
// a and b rotate one lane per step inside the half-warp (warp shuffles), so after 16 steps
// lane l holds those of entries l and 16 + l, the ones it gathered.  Newton's third law:
// each unordered pair is evaluated once.
//
// Warps take short runs of consecutive record pairs from a global counter, so all finish
// together whatever their records hold.
// Mixed path: FP32 pair arithmetic on block-local coordinates (|x| < ~30 A), every step of a
// record branch-free (a pair outside the mask or the cut-off contributes an exact zero);
// forces summed per record in FP32, energies in FP32 over 4 steps then in FP64, both added
// as 64-bit fixed point (2^-32 kcal/mol/A) with integer atomics -- order independent, so
// results are bit-identical run to run.  A warp keeps two record pairs in flight ahead of
// the one it computes: the bulk-copy engine (cp.async.bulk, completion on an mbarrier)
// brings the entries and masks of the pair after next into shared memory, and the gathers
// of the next pair's j atoms are issued before the current pair's arithmetic.
// FP64 path: the same records in FP64 with absolute coordinates, per-pair minimum image and
// FP64 force atomics.
#include "jp_kernels.h"

namespace jp {

constexpr int kPairThreads = 256;
constexpr long long kCopyWaitCycles = 2000000000LL;
constexpr int kPairWarps = kPairThreads / 32;

// ---- bulk copies into shared memory (TMA engine, no tensor map) -------------------------
__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long* bar) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(bar)) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// arm the barrier for `bytes` of incoming copies and start one copy of `bytes` (a multiple
// of 16, both addresses 16-byte aligned) from global to shared memory
__device__ __forceinline__ void mbar_expect(unsigned long long* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void bulk_load(void* dst, const void* src, unsigned bytes, unsigned long long* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// the shared-memory buffer is about to be overwritten by the async proxy after generic reads
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// wait for phase `parity` of the barrier, at most `limit` SM cycles; false on timeout
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, long long limit) {
  const long long t0 = clock64();
  for (;;) {
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

// each half-warp's energies (ELE15, VDW15; ALSD class AA / AB, BB the rest) and pair count
// into the slots of its replica: 64-bit fixed point, summed per record, so the totals do not
// depend on which warp took which record (the kernels claim their records dynamically).  The
// two halves of a warp may work for different replicas: the sums stay inside each half.
__device__ __forceinline__ void flush_fix(const DevPtrs& P, int rep, long long eel, long long elj,
                                          long long eaa, long long eab, long long npair, bool count,
                                          bool alsd) {
  for (int o = 8; o > 0; o >>= 1) {
    eel += __shfl_xor_sync(0xffffffffu, eel, o);
    elj += __shfl_xor_sync(0xffffffffu, elj, o);
    if (alsd) {
      eaa += __shfl_xor_sync(0xffffffffu, eaa, o);
      eab += __shfl_xor_sync(0xffffffffu, eab, o);
    }
    if (count) npair += __shfl_xor_sync(0xffffffffu, npair, o);
  }
  if ((threadIdx.x & 15) == 0 && rep >= 0) {
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

// Per-warp shared memory of the mixed kernel: two bulk-copy buffers (entries and masks of a
// record pair: record 0 in entries 0-31 and masks 0-15, record 1 in 32-63 and 16-31) and the
// staged j atoms of the pair being computed.  Half-warp h stages its record at [32 h, 32 h +
// 32): lane l's entries a = l and b = 16 + l side by side, stored twice (at 32 h + l and
// 32 h + l + 16) so that step k reads slot 32 h + l + k at a constant offset.
struct __align__(16) MixStage {
  float4 ent[2][64];
  unsigned msk[2][32];
  unsigned msk_el[2][32];
  float4 p2[64];      // x_a, x_b, y_a, y_b
  float4 q2[64];      // z_a, z_b, q_a, q_b
  int2 t2[64];        // their LJ type words (with TRI: x = the type-triple index a * nt1 + b)
  unsigned long long bar[2];
};

// rsqrt.approx without the IEEE-mode denormal fix-up: its argument is a squared distance of
// a listed pair (far above the FP32 denormal range) or a masked slot's 1 or 1e30
__device__ __forceinline__ float rsqrt_ftz(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// Nearest integer of v (ties to even, as rintf) for |v| < 2^22, on the FMA pipe: adding and
// subtracting 1.5 * 2^23 rounds v at the unit place in round-to-nearest-even (the explicit
// _rn adds are never contracted or reassociated).  The minimum-image multiples are a few
// units at most.
__device__ __forceinline__ float2 rint2(float2 v) {
  const float2 m = make_float2(12582912.f, 12582912.f), nm = make_float2(-12582912.f, -12582912.f);
  return __fadd2_rn(__fadd2_rn(v, m), nm);
}

__device__ __forceinline__ float rint1(float v) {
  return __fadd_rn(__fadd_rn(v, 12582912.f), -12582912.f);
}

// One record, two pairs per step in packed FP32x2 arithmetic (Blackwell's FFMA2 / FADD2 /
// FMUL2): at step k (k < 16) lane l of the half-warp meets entries a = (l + k) & 15 and
// b = 16 + a, staged at sidx + k (sidx = 32 h + l).  A slot outside the mask or the cut-off
// takes r^2 = 1e30 (its r^-6 = 1e-90 is zero in FP32) and a zero charge product, so it
// contributes an exact zero without a branch.  The j-force accumulators of a and b move one
// lane per step (from lane src = l + 1 of the same half); after 16 steps lane l holds those
// of entries l and 16 + l, returned in (gja, gjb).  Energies in FP32 over 4 steps, then FP64.
// TRI: the LJ parameters of both pairs come from one 16-byte record of the type-triple
// table (i type, a type, b type) -> (C6_a, C6_b, C12_a, C12_b), indexed by row3 (the i type)
// plus the staged a * nt1 + b; else from two type-pair records.
template <bool MINIMG, bool COUNT, bool TRI>
__device__ __forceinline__ void tile_mixed2(const MixStage& S, const float2* __restrict__ s_lj,
                                            const float4* __restrict__ s_lj3, int row,
                                            float4 pi, unsigned m, int sidx, int src, float bx, float by,
                                            float bz, float ibx, float iby, float ibz, float rc2, float zb,
                                            float zf, float zc, float& fix, float& fiy, float& fiz,
                                            float3& gja, float3& gjb, double& te, double& tl, int& tn) {
  const unsigned full = 0xffffffffu;
  const float2 m1 = make_float2(-1.f, -1.f);
  const float2 px = make_float2(pi.x, pi.x), py = make_float2(pi.y, pi.y), pz = make_float2(pi.z, pi.z);
  const float2 pw = make_float2(pi.w, pi.w);
  const float2 zb2 = make_float2(zb, zb), mzc = make_float2(-zc, -zc), mzf = make_float2(-zf, -zf);
  const float2 c12 = make_float2(12.f, 12.f), cm6 = make_float2(-6.f, -6.f);
  float2 fx = make_float2(0.f, 0.f), fy = fx, fz = fx;   // i force, a and b halves (sign: -sum)
  float2 gx = fx, gy = fx, gz = fx;                      // j forces of the a and b entries
#pragma unroll 1
  for (int k0 = 0; k0 < 16; k0 += 4) {
    const float4* __restrict__ sp = S.p2 + sidx + k0;
    const float4* __restrict__ sq = S.q2 + sidx + k0;
    const int2* __restrict__ st = S.t2 + sidx + k0;
    const unsigned ma = m >> k0, mb = m >> (k0 + 16);
    float2 te4 = make_float2(0.f, 0.f), tl4 = te4;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 a = sp[k];
      const float4 b = sq[k];
      float2 dx = __ffma2_rn(make_float2(a.x, a.y), m1, px);
      float2 dy = __ffma2_rn(make_float2(a.z, a.w), m1, py);
      float2 dz = __ffma2_rn(make_float2(b.x, b.y), m1, pz);
      if (MINIMG) {
        dx = __ffma2_rn(make_float2(-bx, -bx), rint2(__fmul2_rn(dx, make_float2(ibx, ibx))), dx);
        dy = __ffma2_rn(make_float2(-by, -by), rint2(__fmul2_rn(dy, make_float2(iby, iby))), dy);
        dz = __ffma2_rn(make_float2(-bz, -bz), rint2(__fmul2_rn(dz, make_float2(ibz, ibz))), dz);
      }
      const float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
      const bool ia = ((ma >> k) & 1u) && r2.x <= rc2;
      const bool ib = ((mb >> k) & 1u) && r2.y <= rc2;
      const float2 rinv = make_float2(rsqrt_ftz(ia ? r2.x : 1e30f), rsqrt_ftz(ib ? r2.y : 1e30f));
      const float2 r2i = __fmul2_rn(rinv, rinv);
      const float2 r6 = __fmul2_rn(__fmul2_rn(r2i, r2i), r2i);
      float2 c6, c12v;
      if (TRI) {
        const float4 lj = s_lj3[row + st[k].x];
        c6 = make_float2(lj.x, lj.y);
        c12v = make_float2(lj.z, lj.w);
      } else {
        const int2 t = st[k];
        const float2 lja = s_lj[row + t.x], ljb = s_lj[row + t.y];
        c6 = make_float2(lja.x, ljb.x);
        c12v = make_float2(lja.y, ljb.y);
      }
      const float2 qf = __fmul2_rn(pw, make_float2(b.z, b.w));
      const float2 qq = make_float2(ia ? qf.x : 0.f, ib ? qf.y : 0.f);
      const float2 v1 = __fmul2_rn(c6, r6);
      const float2 v2 = __fmul2_rn(__fmul2_rn(c12v, r6), r6);
      const float2 eel = __fmul2_rn(qq, __fadd2_rn(rinv, __ffma2_rn(zb2, r2, mzc)));
      const float2 elj = __ffma2_rn(v1, m1, v2);
      const float2 fs = __ffma2_rn(qq, __ffma2_rn(rinv, r2i, mzf),
                                   __fmul2_rn(__ffma2_rn(c12, v2, __fmul2_rn(cm6, v1)), r2i));
      te4 = __fadd2_rn(te4, eel);
      tl4 = __fadd2_rn(tl4, elj);
      const float2 ffx = __fmul2_rn(dx, fs), ffy = __fmul2_rn(dy, fs), ffz = __fmul2_rn(dz, fs);
      fx = __ffma2_rn(ffx, m1, fx);
      fy = __ffma2_rn(ffy, m1, fy);
      fz = __ffma2_rn(ffz, m1, fz);
      gx = __fadd2_rn(gx, ffx);
      gy = __fadd2_rn(gy, ffy);
      gz = __fadd2_rn(gz, ffz);
      if (COUNT) tn += (ia ? 1 : 0) + (ib ? 1 : 0);
      gx.x = __shfl_sync(full, gx.x, src); gx.y = __shfl_sync(full, gx.y, src);
      gy.x = __shfl_sync(full, gy.x, src); gy.y = __shfl_sync(full, gy.y, src);
      gz.x = __shfl_sync(full, gz.x, src); gz.y = __shfl_sync(full, gz.y, src);
    }
    te += (double)te4.x + (double)te4.y;
    tl += (double)tl4.x + (double)tl4.y;
  }
  fix += fx.x + fx.y;
  fiy += fy.x + fy.y;
  fiz += fz.x + fz.y;
  gja = make_float3(gx.x, gy.x, gz.x);
  gjb = make_float3(gx.y, gy.y, gz.y);
}

// what a lane gathers for a record pair before computing it: its two j entries a = l and
// b = 16 + l of its record (position in the i block's frame with the charge, type word,
// atom), its mask rows and its record's unit (-1: no record)
struct Gather {
  float4 pa, pb;
  int ta, tb, aa, ab;
  unsigned m, me;
  int unit;
};

// One pair in the scalar form, branch-free like the packed step: d = x_i - x_j, and the
// force scalar fs (F = -fs d on the i atom) and energies, all zero outside the mask (`bit`)
// or the cut-off.  CMM: the Coulomb term only where `elbit` is set.
template <bool MINIMG, bool CMM>
__device__ __forceinline__ void pair_scalar(float4 pi, float xj, float yj, float zj, float qj, float2 lj,
                                            bool bit, bool elbit, float bx, float by, float bz, float ibx,
                                            float iby, float ibz, float rc2, float zb, float zf, float zc,
                                            float& dx, float& dy, float& dz, float& fs, float& eel,
                                            float& elj, bool& in) {
  dx = pi.x - xj;
  dy = pi.y - yj;
  dz = pi.z - zj;
  if (MINIMG) {
    dx = fmaf(-bx, rint1(dx * ibx), dx);
    dy = fmaf(-by, rint1(dy * iby), dy);
    dz = fmaf(-bz, rint1(dz * ibz), dz);
  }
  const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  in = bit && r2 <= rc2;
  const float rinv = rsqrt_ftz(in ? r2 : 1.f);
  const float r2inv = rinv * rinv;
  const float r6inv = r2inv * r2inv * r2inv;
  const float qq = (CMM ? elbit : true) ? pi.w * qj : 0.f;
  const float v1 = lj.x * r6inv;
  const float v2 = lj.y * r6inv * r6inv;
  const float e1 = qq * (rinv + fmaf(zb, r2, -zc));
  const float e2 = v2 - v1;
  const float f = fmaf(qq, fmaf(rinv, r2inv, -zf), fmaf(12.f, v2, -6.f * v1) * r2inv);
  fs = in ? f : 0.f;
  eel = in ? e1 : 0.f;
  elj = in ? e2 : 0.f;
}

// One record in the scalar form (ALSD, CMM and partial-McMD variants), the two entries of a
// step one after the other, same staging and rotation as tile_mixed2.  ALSD: ci = cluster bit
// of the i atom; a pair with nA cluster atoms has its force times f2 (nA = 2, class AA), f1
// (AB) or f0 (BB: 1 but while per-class outputs are evaluated), and its energy also goes to
// ea (AA) / eb (AB).  SPLIT (partial McMD): the pair's class from the regions of its atoms
// (bit cj of trow: class 1), the class-1 forces in accumulators of their own (fi[3..5],
// gj[6..11], rotated like the others) and the class-1 energy in ea.  CMM: no cut-off (rc2 is
// huge) and the Coulomb term only for the pairs of `me`.  gj[0..5]: entries a and b.
template <bool MINIMG, bool COUNT, bool ALSD, bool CMM, bool SPLIT>
__device__ __forceinline__ void tile_scalar(const MixStage& S, const float2* __restrict__ s_lj, int row,
                                            float4 pi, unsigned m, unsigned me, int sidx, int src, float bx,
                                            float by, float bz, float ibx, float iby, float ibz, float rc2,
                                            float zb, float zf, float zc, float (&fi)[6], float (&gj)[12],
                                            double& te, double& tl, int& tn, int ci, float f0, float f1,
                                            float f2, unsigned trow, double& ea, double& eb) {
  const unsigned full = 0xffffffffu;
  constexpr int NG = SPLIT ? 12 : 6;
#pragma unroll 1
  for (int k0 = 0; k0 < 16; k0 += 4) {
    float te4 = 0.f, tl4 = 0.f, ea4 = 0.f, eb4 = 0.f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float4 a = S.p2[sidx + k0 + k];
      const float4 b = S.q2[sidx + k0 + k];
      const int2 t = S.t2[sidx + k0 + k];
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int tj = e ? t.y : t.x;
        const int sh = k0 + k + 16 * e;
        const float2 lj = s_lj[row + ((ALSD || SPLIT) ? (tj & kTypeMask) : tj)];
        float dx, dy, dz, fs, eel, elj;
        bool in;
        pair_scalar<MINIMG, CMM>(pi, e ? a.y : a.x, e ? a.w : a.z, e ? b.y : b.x, e ? b.w : b.z, lj,
                                 ((m >> sh) & 1u) != 0u, ((me >> sh) & 1u) != 0u, bx, by, bz, ibx, iby, ibz,
                                 rc2, zb, zf, zc, dx, dy, dz, fs, eel, elj, in);
        te4 += eel;
        tl4 += elj;
        float fs1 = 0.f;
        if (SPLIT) {
          const bool c1 = ((trow >> ((tj >> kRegionShift) & 3)) & 1u) != 0u;
          ea4 += c1 ? eel + elj : 0.f;
          fs1 = c1 ? fs : 0.f;
          fs -= fs1;
        } else if (ALSD) {
          const int na = ci + ((tj >> 30) & 1);
          ea4 += na == 2 ? eel + elj : 0.f;
          eb4 += na == 1 ? eel + elj : 0.f;
          fs *= na == 2 ? f2 : (na == 1 ? f1 : f0);
        }
        const float fx = dx * fs, fy = dy * fs, fz = dz * fs;
        fi[0] -= fx; fi[1] -= fy; fi[2] -= fz;
        gj[3 * e + 0] += fx; gj[3 * e + 1] += fy; gj[3 * e + 2] += fz;
        if (SPLIT) {
          const float hx = dx * fs1, hy = dy * fs1, hz = dz * fs1;
          fi[3] -= hx; fi[4] -= hy; fi[5] -= hz;
          gj[6 + 3 * e + 0] += hx; gj[6 + 3 * e + 1] += hy; gj[6 + 3 * e + 2] += hz;
        }
        if (COUNT) tn += (in && (CMM ? ((me >> sh) & 1u) != 0u : true)) ? 1 : 0;
      }
#pragma unroll
      for (int q = 0; q < NG; ++q) gj[q] = __shfl_sync(full, gj[q], src);
    }
    te += (double)te4;
    tl += (double)tl4;
    if (ALSD || SPLIT) {
      ea += (double)ea4;
      eb += (double)eb4;
    }
  }
}

// dynamic shared memory of the mixed kernel: the type-pair (C6, C12) table, and with TRI the
// type-triple table after it (16-byte aligned)
__host__ __device__ constexpr size_t lj_pair_bytes(int nt1) { return ((size_t)nt1 * nt1 * 8 + 15) / 16 * 16; }
__host__ __device__ constexpr size_t lj_tri_bytes(int nt1) { return (size_t)nt1 * nt1 * nt1 * 16; }
constexpr int kTriMaxTypes = 16;   // the triple table up to 16 types (64 KiB)

template <bool COUNT, bool ALSD, bool CMM, bool SPLIT = false, bool TRI = false>
__global__ void __launch_bounds__(kPairThreads, 2)
k_pair_mixed(DevPtrs P, ZdConst z) {
  extern __shared__ float2 s_lj[];
  __shared__ MixStage s_stage[kPairWarps];
  const unsigned full = 0xffffffffu;
  const int nlj = z.nt1 * z.nt1;
  float4* s_lj3 = reinterpret_cast<float4*>(reinterpret_cast<char*>(s_lj) + lj_pair_bytes(z.nt1));
  for (int i = threadIdx.x; i < nlj; i += blockDim.x) s_lj[i] = P.lj_f[i];
  if (TRI)
    for (int i = threadIdx.x; i < nlj * z.nt1; i += blockDim.x) {
      const int ti = i / nlj, ta = (i / z.nt1) % z.nt1, tb = i % z.nt1;
      const float2 a = P.lj_f[ti * z.nt1 + ta], b = P.lj_f[ti * z.nt1 + tb];
      s_lj3[i] = make_float4(a.x, b.x, a.y, b.y);
    }
  const int lane = threadIdx.x & 31;
  const int hw = lane >> 4, lp = lane & (kHalf - 1);   // half-warp, lane inside it
  const int sidx = 32 * hw + lp;                        // this lane's staging slot
  const int src = ((lp + 1) & (kHalf - 1)) | (hw << 4); // rotation: from the next lane of the half
  MixStage& S = s_stage[threadIdx.x >> 5];
  if (lane == 0) {
    mbar_init(&S.bar[0]);
    mbar_init(&S.bar[1]);
  }
  __syncthreads();
  const int T = *P.nctiles;         // records
  const int TU = (T + 1) >> 1;      // record pairs: a warp's work units
  // a 1.2-KiB copy lands in microseconds; the bound (about a second of SM clock) only ends
  // the wait on a broken device, and it is not the integrator's adjustable barrier bound:
  // a block must never leave with one of its copies still in flight
  const long long wlim = kCopyWaitCycles;
  const float rc2 = (float)z.rc2, zb = (float)z.bcoeff, zf = (float)z.fcoeff, zc = (float)z.zcore;
  const unsigned txb = CMM ? 1280u : 1152u;
  unsigned phase = 0u, pend = 0u;   // per buffer: barrier parity to wait for; copy in flight
  bool ok = true;

  // record pairs are claimed in runs of `run` consecutive ones: the records of a unit are
  // consecutive, so a run mostly keeps its i atoms (no reload, no i-force flush between
  // records); the run is short enough that every warp still gets several (8 per warp at most
  // of the total, 1 to 16 pairs)
  const int run = max(1, min(16, TU / (int)(gridDim.x * kPairWarps * 8)));
  int run_next = 0, run_end = 0;
  auto claim = [&]() {
    if (run_next >= run_end) {
      int t = 0;
      if (lane == 0) t = atomicAdd(P.tile_ctr, run);
      t = __shfl_sync(full, t, 0);
      run_next = t;
      run_end = min(t + run, TU);
    }
    return run_next < run_end ? run_next++ : TU;
  };
  // the entries and masks of records 2t and 2t + 1 into buffer b (one past the last record
  // is padding inside the arrays: read, never used)
  auto issue = [&](int t, int b) {
    if (lane == 0) {
      fence_proxy_async();
      mbar_expect(&S.bar[b], txb);
      bulk_load(S.ent[b], P.ct_j + (size_t)t * 64, 1024u, &S.bar[b]);
      bulk_load(S.msk[b], P.ct_mask + (size_t)t * 32, 128u, &S.bar[b]);
      if (CMM) bulk_load(S.msk_el[b], P.ct_mask_el + (size_t)t * 32, 128u, &S.bar[b]);
    }
    pend |= 1u << b;
  };
  auto gather1 = [&](float4 e, bool valid, float4& p, int& ty, int& at) {
    const int sj = valid ? __float_as_int(e.w) : -1;
    if (sj >= 0) {
      const float4 q = P.pos_f[sj];
      p = make_float4(q.x - e.x, q.y - e.y, q.z - e.z, q.w);   // into the i block's frame
      ty = P.styp[sj];
      at = P.satom[sj];
    } else {
      p = make_float4(0.f, 0.f, 0.f, 0.f);
      ty = z.nt1 - 1;   // the zero dummy type
      at = -1;
    }
  };
  // pair t's copy has landed in buffer b: start the gathers of this lane's two entries
  auto fetch = [&](int t, int b, Gather& G) {
    if (!mbar_wait(&S.bar[b], (phase >> b) & 1u, wlim)) {
      ok = false;
      atomicOr(P.status, ERR_TIMEOUT);
      return;
    }
    phase ^= 1u << b;
    pend &= ~(1u << b);
    const int rec = 2 * t + hw;
    const bool valid = rec < T;
    G.m = valid ? S.msk[b][lane] : 0u;
    G.me = CMM && valid ? S.msk_el[b][lane] : 0u;
    G.unit = valid ? P.ct_blk[rec] : -1;
    gather1(S.ent[b][32 * hw + lp], valid, G.pa, G.ta, G.aa);
    gather1(S.ent[b][32 * hw + kHalf + lp], valid, G.pb, G.tb, G.ab);
  };

  int cur_unit = -2, cur_rep = -1, rep = -1, ai = -1, ti = 0;
  float4 pi = make_float4(0.f, 0.f, 0.f, 0.f);
  long long gix = 0, giy = 0, giz = 0;
  long long gix1 = 0, giy1 = 0, giz1 = 0;   // partial McMD: class-1 i forces
  long long eel = 0, elj = 0, eaa = 0, eab = 0;
  long long npair = 0;
  bool mi = false;
  float bx = 0.f, by = 0.f, bz = 0.f, ibx = 0.f, iby = 0.f, ibz = 0.f;
  float f0 = 1.f, f1 = 1.f, f2 = 1.f;
  unsigned tab = 0u;

  int t = claim(), tn = TU;
  Gather G;
  if (t < TU) {
    issue(t, 0);
    tn = claim();
    if (tn < TU) issue(tn, 1);
    fetch(t, 0, G);
  }
  int b = 0;
  while (t < TU && ok) {
    // this lane's two entries into the stage, twice
    __syncwarp();
    {
      const float4 p2 = make_float4(G.pa.x, G.pb.x, G.pa.y, G.pb.y);
      const float4 q2 = make_float4(G.pa.z, G.pb.z, G.pa.w, G.pb.w);
      const int2 t2 = TRI ? make_int2(G.ta * z.nt1 + G.tb, 0) : make_int2(G.ta, G.tb);
      S.p2[sidx] = p2;
      S.p2[sidx + kHalf] = p2;
      S.q2[sidx] = q2;
      S.q2[sidx + kHalf] = q2;
      S.t2[sidx] = t2;
      S.t2[sidx + kHalf] = t2;
    }
    const unsigned m = G.m, me = G.me;
    const int aa = G.aa, ab = G.ab, unit = G.unit;
    // the lane's i atom: a new unit flushes the last one's force and loads the new atom
    if (unit != cur_unit) {
      if (ai >= 0 && (gix | giy | giz)) {
        atomic_add_ll(&P.frc[3 * ai + 0], gix);
        atomic_add_ll(&P.frc[3 * ai + 1], giy);
        atomic_add_ll(&P.frc[3 * ai + 2], giz);
      }
      if (SPLIT && ai >= 0 && (gix1 | giy1 | giz1)) {
        atomic_add_ll(&P.frc1[3 * ai + 0], gix1);
        atomic_add_ll(&P.frc1[3 * ai + 1], giy1);
        atomic_add_ll(&P.frc1[3 * ai + 2], giz1);
      }
      gix = giy = giz = 0;
      gix1 = giy1 = giz1 = 0;
      cur_unit = unit;
      if (unit >= 0) {
        const int si = (unit >> 1) * kTile + (unit & 1) * kHalf + lp;
        pi = P.pos_f[si];
        ti = P.styp[si];
        ai = P.satom[si];
        rep = P.blk_rep[unit >> 1];
      } else {
        pi = make_float4(0.f, 0.f, 0.f, 0.f);
        ti = z.nt1 - 1;
        ai = -1;
      }
    }
    // a new replica in either half: both halves' energies go to their replicas so far
    if (__any_sync(full, rep != cur_rep)) {
      flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD || SPLIT);
      eel = elj = eaa = eab = 0;
      npair = 0;
      if (rep != cur_rep) {
        cur_rep = rep;
        const Rep& R = P.reps[rep];
        bx = (float)R.box[0]; by = (float)R.box[1]; bz = (float)R.box[2];
        ibx = (float)R.invbox[0]; iby = (float)R.invbox[1]; ibz = (float)R.invbox[2];
        if (ALSD) {
          const double lam = P.lam[2 * rep];
          f0 = (float)cls_weight(R, lam, 2);
          f1 = (float)cls_weight(R, lam, 1);
          f2 = (float)cls_weight(R, lam, 0);
        }
        if (SPLIT) tab = R.split ? R.cls_tab : 0u;
        // Per-pair minimum image is needed only where a pair within the cut-off can have
        // another image than its tile's.  Per axis the tile's image puts the two block
        // references at most box/2 apart, and a pair's separation differs from theirs by at
        // most h_i + h_j <= 2 h_max plus the atoms' motion since the build (2 A margin), so
        // in the tile's image |d| <= box/2 + 2 h_max + 2; in any other image |d| >= box - rc.
        // Both hold at once only if box/2 <= rc + 2 h_max + 2.  CMM (no cut-off): the
        // farthest near-field pair rlim in place of rc, with twice the block margin.
        mi = false;
        for (int k = 0; k < 3; ++k) {
          const double h = (double)P.rep_hmax[3 * rep + k];
          const double reach = CMM ? z.rlim + 4.0 * h : sqrt(z.rc2) + 2.0 * h;
          if (0.5 * R.box[k] < reach + 2.0) mi = true;
        }
      }
    }
    const bool wmi = __any_sync(full, mi);   // one image form for the whole warp
    __syncwarp();
    // buffer b is free again: the pair after next goes into it; the next pair's gathers
    // are issued before this pair's arithmetic
    int t2 = TU;
    if (tn < TU) {
      t2 = claim();
      if (t2 < TU) issue(t2, b);
    }
    Gather Gn;
    if (tn < TU) fetch(tn, b ^ 1, Gn);
    float fix = 0.f, fiy = 0.f, fiz = 0.f;
    float3 gja = make_float3(0.f, 0.f, 0.f), gjb = gja, gja1 = gja, gjb1 = gja;
    double te = 0.0, tl = 0.0, ea = 0.0, eb = 0.0;
    int tn_pairs = 0;
    const int ci = ALSD ? ((ti >> 30) & 1) : 0;
    const int row = ((ALSD || SPLIT) ? (ti & kTypeMask) : ti) * z.nt1;
    if (ALSD || CMM || SPLIT) {
      float fi6[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      float gj[12] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
      const unsigned trow = SPLIT ? tab >> (3 * ((ti >> kRegionShift) & 3)) : 0u;
      if (wmi)
        tile_scalar<true, COUNT, ALSD, CMM, SPLIT>(S, s_lj, row, pi, m, me, sidx, src, bx, by, bz, ibx, iby,
                                                   ibz, rc2, zb, zf, zc, fi6, gj, te, tl, tn_pairs, ci, f0,
                                                   f1, f2, trow, ea, eb);
      else
        tile_scalar<false, COUNT, ALSD, CMM, SPLIT>(S, s_lj, row, pi, m, me, sidx, src, bx, by, bz, ibx, iby,
                                                    ibz, rc2, zb, zf, zc, fi6, gj, te, tl, tn_pairs, ci, f0,
                                                    f1, f2, trow, ea, eb);
      fix = fi6[0]; fiy = fi6[1]; fiz = fi6[2];
      gja = make_float3(gj[0], gj[1], gj[2]);
      gjb = make_float3(gj[3], gj[4], gj[5]);
      if (SPLIT) {
        gja1 = make_float3(gj[6], gj[7], gj[8]);
        gjb1 = make_float3(gj[9], gj[10], gj[11]);
        gix1 += to_fix_f(fi6[3], P.status);
        giy1 += to_fix_f(fi6[4], P.status);
        giz1 += to_fix_f(fi6[5], P.status);
      }
    } else if (wmi) {
      tile_mixed2<true, COUNT, TRI>(S, s_lj, s_lj3, TRI ? ti * nlj : row, pi, m, sidx, src, bx, by, bz, ibx,
                                    iby, ibz, rc2, zb, zf, zc, fix, fiy, fiz, gja, gjb, te, tl, tn_pairs);
    } else {
      tile_mixed2<false, COUNT, TRI>(S, s_lj, s_lj3, TRI ? ti * nlj : row, pi, m, sidx, src, bx, by, bz,
                                     ibx, iby, ibz, rc2, zb, zf, zc, fix, fiy, fiz, gja, gjb, te, tl,
                                     tn_pairs);
    }
    auto add_j = [&](long long* f, int aj, float3 g) {
      if (aj >= 0 && (g.x != 0.f || g.y != 0.f || g.z != 0.f)) {
        atomic_add_ll(&f[3 * aj + 0], to_fix_f(g.x, P.status));
        atomic_add_ll(&f[3 * aj + 1], to_fix_f(g.y, P.status));
        atomic_add_ll(&f[3 * aj + 2], to_fix_f(g.z, P.status));
      }
    };
    add_j(P.frc, aa, gja);
    add_j(P.frc, ab, gjb);
    if (SPLIT) {
      add_j(P.frc1, aa, gja1);
      add_j(P.frc1, ab, gjb1);
    }
    gix += to_fix_f(fix, P.status);
    giy += to_fix_f(fiy, P.status);
    giz += to_fix_f(fiz, P.status);
    eel += to_fix(te, kEneScale, P.status);
    elj += to_fix(tl, kEneScale, P.status);
    if (ALSD || SPLIT) {
      eaa += to_fix(ea, kEneScale, P.status);
      eab += to_fix(eb, kEneScale, P.status);
    }
    if (COUNT) npair += tn_pairs;
    t = tn;
    tn = t2;
    G = Gn;
    b ^= 1;
  }
  if (ai >= 0 && (gix | giy | giz)) {
    atomic_add_ll(&P.frc[3 * ai + 0], gix);
    atomic_add_ll(&P.frc[3 * ai + 1], giy);
    atomic_add_ll(&P.frc[3 * ai + 2], giz);
  }
  if (SPLIT && ai >= 0 && (gix1 | giy1 | giz1)) {
    atomic_add_ll(&P.frc1[3 * ai + 0], gix1);
    atomic_add_ll(&P.frc1[3 * ai + 1], giy1);
    atomic_add_ll(&P.frc1[3 * ai + 2], giz1);
  }
  flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD || SPLIT);
  // a copy still in flight (only after a timed-out wait) must land before the block exits
  for (int k = 0; k < 2; ++k)
    if ((pend >> k) & 1u) mbar_wait(&S.bar[k], (phase >> k) & 1u, wlim);
}

// Per-warp shared memory of the FP64 kernel: each half-warp's record, entries a and b of
// every lane, twice (see MixStage).
struct __align__(16) F64Stage {
  double4 pa[64], pb[64];
  int2 t[64];
};

template <bool COUNT, bool ALSD, bool CMM, bool SPLIT = false>
__global__ void __launch_bounds__(kPairThreads)
k_pair_fp64(DevPtrs P, ZdConst z) {
  extern __shared__ double2 s_ljd[];
  __shared__ F64Stage s_stage[kPairWarps];
  const unsigned full = 0xffffffffu;
  const int nlj = z.nt1 * z.nt1;
  for (int i = threadIdx.x; i < nlj; i += blockDim.x) s_ljd[i] = P.lj_d[i];
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int hw = lane >> 4, lp = lane & (kHalf - 1);
  const int sidx = 32 * hw + lp;
  const int src = ((lp + 1) & (kHalf - 1)) | (hw << 4);
  F64Stage& S = s_stage[threadIdx.x >> 5];
  const int T = *P.nctiles;
  const int TU = (T + 1) >> 1;
  const double irlim2 = 1.0 / z.rc2;
  int cur_unit = -2, cur_rep = -1, rep = -1, ai = -1, ti = 0;
  double4 pi = make_double4(0, 0, 0, 0);
  double gix = 0, giy = 0, giz = 0;
  double gix1 = 0, giy1 = 0, giz1 = 0;            // partial McMD: class-1 i forces
  long long eel = 0, elj = 0, eaa = 0, eab = 0;   // fixed point, per record
  long long npair = 0;
  double bx = 0, by = 0, bz = 0, ibx = 0, iby = 0, ibz = 0;
  double f0 = 1.0, f1 = 1.0, f2 = 1.0;
  unsigned tab = 0u;
  auto flush_i = [&]() {
    if (ai >= 0) {
      atomicAdd(&P.grd[3 * ai + 0], gix);
      atomicAdd(&P.grd[3 * ai + 1], giy);
      atomicAdd(&P.grd[3 * ai + 2], giz);
      if (SPLIT) {
        atomicAdd(&P.grd1[3 * ai + 0], gix1);
        atomicAdd(&P.grd1[3 * ai + 1], giy1);
        atomicAdd(&P.grd1[3 * ai + 2], giz1);
      }
    }
    gix = giy = giz = 0;
    gix1 = giy1 = giz1 = 0;
  };
  for (;;) {
    int t = 0;
    if (lane == 0) t = atomicAdd(P.tile_ctr, 1);
    t = __shfl_sync(full, t, 0);
    if (t >= TU) break;
    const int rec = 2 * t + hw;
    const bool valid = rec < T;
    const int unit = valid ? P.ct_blk[rec] : -1;
    if (unit != cur_unit) {
      flush_i();
      cur_unit = unit;
      if (unit >= 0) {
        const int si = (unit >> 1) * kTile + (unit & 1) * kHalf + lp;
        pi = P.pos_d[si];
        ti = P.styp[si];
        ai = P.satom[si];
        rep = P.blk_rep[unit >> 1];
      } else {
        pi = make_double4(0, 0, 0, 0);
        ti = z.nt1 - 1;
        ai = -1;
      }
    }
    if (__any_sync(full, rep != cur_rep)) {
      flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD || SPLIT);
      eel = elj = eaa = eab = 0;
      npair = 0;
      if (rep != cur_rep) {
        cur_rep = rep;
        const Rep& R = P.reps[rep];
        bx = R.box[0]; by = R.box[1]; bz = R.box[2];
        ibx = R.invbox[0]; iby = R.invbox[1]; ibz = R.invbox[2];
        if (ALSD) {
          f0 = cls_weight(R, P.lam[2 * rep], 2);
          f1 = cls_weight(R, P.lam[2 * rep], 1);
          f2 = cls_weight(R, P.lam[2 * rep], 0);
        }
        if (SPLIT) tab = R.split ? R.cls_tab : 0u;
      }
    }
    const unsigned m = valid ? P.ct_mask[(size_t)rec * kHalf + lp] : 0u;
    const unsigned me = CMM && valid ? P.ct_mask_el[(size_t)rec * kHalf + lp] : 0u;
    int aj[2], tjv[2];
    double4 pj[2];
    for (int e = 0; e < 2; ++e) {
      const int sj = valid ? __float_as_int(P.ct_j[(size_t)rec * 32 + kHalf * e + lp].w) : -1;
      pj[e] = sj >= 0 ? P.pos_d[sj] : make_double4(0.0, 0.0, 0.0, 0.0);
      tjv[e] = sj >= 0 ? P.styp[sj] : z.nt1 - 1;
      aj[e] = sj >= 0 ? P.satom[sj] : -1;
    }
    __syncwarp();
    S.pa[sidx] = pj[0];
    S.pa[sidx + kHalf] = pj[0];
    S.pb[sidx] = pj[1];
    S.pb[sidx + kHalf] = pj[1];
    S.t[sidx] = make_int2(tjv[0], tjv[1]);
    S.t[sidx + kHalf] = make_int2(tjv[0], tjv[1]);
    __syncwarp();
    const int row = ((ALSD || SPLIT) ? (ti & kTypeMask) : ti) * z.nt1;
    const int ci = ALSD ? ((ti >> 30) & 1) : 0;
    const unsigned trow = SPLIT ? tab >> (3 * ((ti >> kRegionShift) & 3)) : 0u;
    constexpr int NG = SPLIT ? 12 : 6;
    double gj[12] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};   // entries a, b; class 1 a, b
    int tn = 0;
    double te = 0.0, tl = 0.0, ta = 0.0, tb = 0.0;   // this record's energies
#pragma unroll 2
    for (int k = 0; k < kHalf; ++k) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int sh = k + kHalf * e;
        if ((m >> sh) & 1u) {
          const double4 q = e ? S.pb[sidx + k] : S.pa[sidx + k];
          const int tj = e ? S.t[sidx + k].y : S.t[sidx + k].x;
          double dx = pi.x - q.x, dy = pi.y - q.y, dz = pi.z - q.z;
          dx -= bx * anint(dx * ibx);
          dy -= by * anint(dy * iby);
          dz -= bz * anint(dz * ibz);
          const double dd2 = dx * dx + dy * dy + dz * dz;
          const double dd2i = 1.0 / dd2;
          if (dd2i - irlim2 >= 0.0) {
            const double ddi = sqrt(dd2i);
            const double dd6i = dd2i * dd2i * dd2i;
            const bool elp = CMM ? ((me >> sh) & 1u) != 0u : true;
            const double ee = elp ? pi.w * q.w : 0.0;
            const double epair = ee * (ddi + z.bcoeff * dd2 - z.zcore);
            te += epair;
            const double2 lj = s_ljd[row + ((ALSD || SPLIT) ? (tj & kTypeMask) : tj)];
            const double v1 = lj.x * dd6i;
            const double v2 = lj.y * dd6i * dd6i;
            tl += -v1 + v2;
            double cc = ee * (dd2i * ddi - z.fcoeff) + (-6.0 * v1 + 12.0 * v2) * dd2i;
            bool c1 = false;
            if (SPLIT) {   // partial McMD: class 1 by the regions of the two atoms
              c1 = ((trow >> ((tj >> kRegionShift) & 3)) & 1u) != 0u;
              if (c1) ta += epair + (-v1 + v2);
            } else if (ALSD) {
              const int na = ci + ((tj >> 30) & 1);
              if (na == 2) { ta += epair + (-v1 + v2); cc *= f2; }
              else if (na == 1) { tb += epair + (-v1 + v2); cc *= f1; }
              else cc *= f0;
            }
            const double fx = dx * cc, fy = dy * cc, fz = dz * cc;
            if (SPLIT && c1) {
              gix1 -= fx; giy1 -= fy; giz1 -= fz;
              gj[6 + 3 * e] += fx; gj[7 + 3 * e] += fy; gj[8 + 3 * e] += fz;
            } else {
              gix -= fx; giy -= fy; giz -= fz;
              gj[3 * e] += fx; gj[1 + 3 * e] += fy; gj[2 + 3 * e] += fz;
            }
            if (COUNT && elp) ++tn;
          }
        }
      }
#pragma unroll
      for (int q = 0; q < NG; ++q) gj[q] = __shfl_sync(full, gj[q], src);
    }
    for (int e = 0; e < 2; ++e) {
      if (aj[e] >= 0 && (gj[3 * e] != 0.0 || gj[1 + 3 * e] != 0.0 || gj[2 + 3 * e] != 0.0)) {
        atomicAdd(&P.grd[3 * aj[e] + 0], gj[3 * e]);
        atomicAdd(&P.grd[3 * aj[e] + 1], gj[1 + 3 * e]);
        atomicAdd(&P.grd[3 * aj[e] + 2], gj[2 + 3 * e]);
      }
      if (SPLIT && aj[e] >= 0 && (gj[6 + 3 * e] != 0.0 || gj[7 + 3 * e] != 0.0 || gj[8 + 3 * e] != 0.0)) {
        atomicAdd(&P.grd1[3 * aj[e] + 0], gj[6 + 3 * e]);
        atomicAdd(&P.grd1[3 * aj[e] + 1], gj[7 + 3 * e]);
        atomicAdd(&P.grd1[3 * aj[e] + 2], gj[8 + 3 * e]);
      }
    }
    if (COUNT) npair += tn;
    eel += to_fix(te, kEneScale, P.status);
    elj += to_fix(tl, kEneScale, P.status);
    if (ALSD || SPLIT) { eaa += to_fix(ta, kEneScale, P.status); eab += to_fix(tb, kEneScale, P.status); }
  }
  flush_i();
  flush_fix(P, cur_rep, eel, elj, eaa, eab, npair, COUNT, ALSD || SPLIT);
}

// the mixed kernels that read the type-triple table need more than the default 48 KiB of
// dynamic shared memory above 12 types: raised once, when a context is created
static void allow_tri_smem(int nt1) {
  const int b = (int)(lj_pair_bytes(nt1) + lj_tri_bytes(nt1));
  cudaFuncSetAttribute(k_pair_mixed<false, false, false, false, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, b);
  cudaFuncSetAttribute(k_pair_mixed<true, false, false, false, true>,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, b);
}

int pair_blocks_per_sm(bool fp64, int nt1) {
  int per = 0;
  if (fp64) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair_fp64<false, false, false>, kPairThreads,
                                                  sizeof(double2) * nt1 * nt1);
  } else if (nt1 <= kTriMaxTypes) {
    allow_tri_smem(nt1);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair_mixed<false, false, false, false, true>,
                                                  kPairThreads, lj_pair_bytes(nt1) + lj_tri_bytes(nt1));
  } else {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_pair_mixed<false, false, false>, kPairThreads,
                                                  lj_pair_bytes(nt1));
  }
  return per > 0 ? per : 1;
}

void launch_pair_mixed(const DevPtrs& P, const ZdConst& z, int nwarps, bool count, bool alsd, bool split,
                       cudaStream_t st) {
  const int nb = (nwarps + kPairWarps - 1) / kPairWarps;
  const size_t sh = lj_pair_bytes(z.nt1);
  if (split) {
    if (count) k_pair_mixed<true, true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
  } else if (z.cmm) {
    if (count) k_pair_mixed<true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
  } else if (alsd) {
    if (count) k_pair_mixed<true, true, false><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, true, false><<<nb, kPairThreads, sh, st>>>(P, z);
  } else if (z.nt1 <= kTriMaxTypes) {   // LJ pairs from the type-triple table
    const size_t sh3 = lj_pair_bytes(z.nt1) + lj_tri_bytes(z.nt1);
    if (count) k_pair_mixed<true, false, false, false, true><<<nb, kPairThreads, sh3, st>>>(P, z);
    else k_pair_mixed<false, false, false, false, true><<<nb, kPairThreads, sh3, st>>>(P, z);
  } else {
    if (count) k_pair_mixed<true, false, false><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_mixed<false, false, false><<<nb, kPairThreads, sh, st>>>(P, z);
  }
}

void launch_pair_fp64(const DevPtrs& P, const ZdConst& z, int nwarps, bool count, bool alsd, bool split,
                      cudaStream_t st) {
  const int nb = (nwarps + kPairWarps - 1) / kPairWarps;
  const size_t sh = sizeof(double2) * z.nt1 * z.nt1;
  if (split) {
    if (count) k_pair_fp64<true, true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
    else k_pair_fp64<false, true, false, true><<<nb, kPairThreads, sh, st>>>(P, z);
  } else if (z.cmm) {
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
