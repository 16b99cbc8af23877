// jp_hbond.cu -- the hydrogen-bond 10-12 term of the listed 1-5 pairs.
//
// md_run switches it on when a type pair has iyppid = 2 (incel.f90:170-171, iyeflg(10)).
// cutoff_PB then moves every listed pair of such types out of the 12-6 tables into
// itbhyd (cutoff.f90:98-154), and enear evaluates those pairs with their usual Coulomb
// term plus, instead of the 12-6 term (enear.f90:330-516, #ZD / #ACT lines),
//   E_hb += co (C12h/r^12 - C10/r^10),   dE/dxi = -co (12 C12h/r^12 - 10 C10/r^10)/r^2 d,
// d = xi - xj, co = [r <= rc], C10 = fynbpp(3,.,.), C12h = fynbpp(4,.,.).
//
// Here the pairs stay in the tiles, where the pair kernels' 12-6 table is zero for these
// type pairs, so the tiles give their Coulomb term; at each list rebuild k_hb_list copies
// the marked pairs of the tile masks into a compact list of atom pairs, and every force
// evaluation k_hbond adds their 10-12 term from the FP64 master coordinates (FP64
// arithmetic on both paths: the pairs are few).  ALSD: class weight of the pair as in the
// tiles, energy also into the class totals.
#include "jp_kernels.h"

namespace jp {

constexpr int kHbThreads = 256;

// one warp per tile: lane l holds i slot l of the tile and its mask (bit k = j slot
// (l + k) & 31); the marked pairs go to hb_list through one atomic per warp
__global__ void __launch_bounds__(kHbThreads) k_hb_list(DevPtrs P, int cap, int nt1) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (kHbThreads / 32);
  const int T = *P.ntiles;
  for (int t = (blockIdx.x * kHbThreads + threadIdx.x) >> 5; t < T; t += nw) {
    const int2 ij = P.tiles[t];
    const int si = ij.x * kTile + lane, sj = ij.y * kTile + lane;
    const int ti = P.styp[si] & kTypeMask, tj = P.styp[sj] & kTypeMask;
    const bool hi = P.hb_type[ti] != 0;
    if (!__any_sync(full, hi) || !__any_sync(full, P.hb_type[tj] != 0)) continue;
    const unsigned m = P.tmp_masks[(size_t)P.tile_src[t] * 32 + lane];
    unsigned hm = 0;
    for (int k = 0; k < 32; ++k) {
      const int tk = __shfl_sync(full, tj, (lane + k) & 31);
      if (hi && ((m >> k) & 1u) && P.hb_pair[ti * nt1 + tk]) hm |= 1u << k;
    }
    const int cnt = __popc(hm);
    int incl = cnt;
    for (int o = 1; o < 32; o <<= 1) {
      const int v = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += v;
    }
    const int total = __shfl_sync(full, incl, 31);
    if (total == 0) continue;
    int base = 0;
    if (lane == 31) base = atomicAdd(P.hb_n, total);
    base = __shfl_sync(full, base, 31);
    if (lane == 31 && base + total > cap) atomicOr(P.status, ERR_LIST_OVERFLOW);
    int pos = base + incl - cnt;
    const int ai = P.satom[si];
    while (hm) {
      const int k = __ffs(hm) - 1;
      hm &= hm - 1;
      if (pos < cap) P.hb_list[pos] = make_int2(ai, P.satom[ij.y * kTile + ((lane + k) & 31)]);
      ++pos;
    }
  }
}

// every listed H-bond pair once; the loop bound is block-uniform, so whole warps reach the
// warp-aggregated energy adds
template <bool FP64, bool ALSD>
__global__ void __launch_bounds__(kHbThreads) k_hbond(DevPtrs P, int cap, double rc2, int nt1) {
  const int n = min(*P.hb_n, cap);
  const int stride = gridDim.x * kHbThreads;
  for (int b0 = blockIdx.x * kHbThreads; b0 < n; b0 += stride) {
    const int q = b0 + threadIdx.x;
    double e = 0.0;
    int rep = 0, cls = 2;
    if (q < n) {
      const int2 pr = P.hb_list[q];
      rep = P.rep_of[pr.x];
      const Rep& R = P.reps[rep];
      double d[3];
      for (int k = 0; k < 3; ++k) {
        d[k] = P.x[3 * pr.x + k] - P.x[3 * pr.y + k];
        d[k] -= R.box[k] * anint(d[k] * R.invbox[k]);
      }
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 <= rc2) {
        const int ti = P.typ[pr.x], tj = P.typ[pr.y];
        const double2 h = P.hb_tab[(ti & kTypeMask) * nt1 + (tj & kTypeMask)];
        const double dd2i = 1.0 / r2;
        const double dd4i = dd2i * dd2i;
        const double v1 = h.x * (dd4i * dd4i * dd2i);   // C10 / r^10
        const double v2 = h.y * (dd4i * dd4i * dd4i);   // C12h / r^12
        e = v2 - v1;
        double fs = 1.0;
        bool c1 = false;   // class 1 of a partial-McMD replica
        if (ALSD && R.split) {
          const int ci = (ti >> kRegionShift) & 3, cj = (tj >> kRegionShift) & 3;
          cls = ((R.cls_tab >> (3 * ci + cj)) & 1u) ? 0 : 2;
          c1 = cls == 0;
        } else if (ALSD) {
          cls = 2 - (((ti >> 30) & 1) + ((tj >> 30) & 1));
          fs = cls_weight(R, P.lam[2 * rep], cls);
        }
        const double cc = (12.0 * v2 - 10.0 * v1) * dd2i;
        add_grad<FP64>(P, fs, pr.x, -d[0] * cc, -d[1] * cc, -d[2] * cc, c1);
        add_grad<FP64>(P, fs, pr.y, d[0] * cc, d[1] * cc, d[2] * cc, c1);
      }
    }
    add_energy(P, rep, JP_E_HBOND, e);
    if (ALSD) add_cls_energy(P, rep, cls, e);
  }
}

static int hb_blocks(int cap) {
  return std::max(1, std::min((cap + kHbThreads - 1) / kHbThreads, 148 * 8));
}

void launch_hb_list(const DevPtrs& P, int cap, int nt1, int nblk, cudaStream_t st) {
  cudaMemsetAsync(P.hb_n, 0, sizeof(int), st);
  // eight warps a block, four blocks per block of atoms: about one warp per tile
  const int nb = std::max(1, std::min(nblk * 4, 148 * 8));
  k_hb_list<<<nb, kHbThreads, 0, st>>>(P, cap, nt1);
}

void launch_hbond(const DevPtrs& P, int cap, double rc2, int nt1, bool fp64, bool alsd, cudaStream_t st) {
  const int nb = hb_blocks(cap);
  if (fp64) {
    if (alsd) k_hbond<true, true><<<nb, kHbThreads, 0, st>>>(P, cap, rc2, nt1);
    else k_hbond<true, false><<<nb, kHbThreads, 0, st>>>(P, cap, rc2, nt1);
  } else {
    if (alsd) k_hbond<false, true><<<nb, kHbThreads, 0, st>>>(P, cap, rc2, nt1);
    else k_hbond<false, false><<<nb, kHbThreads, 0, st>>>(P, cap, rc2, nt1);
  }
}

}  // namespace jp
