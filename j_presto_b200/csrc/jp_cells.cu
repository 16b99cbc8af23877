// jp_cells.cu -- device cell-list build and pair-tile list (replaces md_run celprp/celpar/
// cutoff: src_md_run/celprp.f90:2-175, celpar.f90:2-244, cutoff.f90:2-505).
//
// Pipeline (every UPDATE steps, all replicas in one pass):
//   1. k_cell_key      radix binning: wrapped position -> fine cell -> Morton key per replica
//   2. scan            counting-sort offsets (deterministic exclusive scan)
//   3. k_scatter       bin atoms; k_sort_bins makes the order within a bin deterministic
//   4. k_fill_slots    compact order -> 32-atom blocks padded per replica
//   5. k_block_setup   per-block bounding box, frame origin, block-local coordinates
//   6. k_tile_scan_chunks  one warp per (i-block, 32 candidate j-blocks): bounding-box test
//                      of the 32 candidates at once, warp-ballot compaction of the
//                      survivors, then the exact 32x32 interaction mask in FP64:
//                      r^2 <= (rc+1.5)^2 at build time (cutatm `dd .le. rlim2`), minus
//                      1-2/1-3/1-4 partners (cutoff.f90:50-96).
//   7. scan of the per-chunk tile counts, k_tile_emit writes one dense list in row-major,
//      ascending-j order (deterministic).
#include "jp_common.cuh"
#include "jp_kernels.h"

namespace jp {

// Binning: atoms go to xy columns of edge ~(32/density)^(1/3) (~6.8 A for water) and,
// inside a column, to 0.25 A z bins.  The key orders atoms by (replica, column, z), so each
// column's atoms are z-sorted and a column cut into runs of 32 gives near-cubic blocks.
__global__ void k_cell_key(DevPtrs P, int natom) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const Rep& R = P.reps[P.rep_of[a]];
  int c[3];
  bool out = false;
  for (int k = 0; k < 3; ++k) {
    const double x = P.x[3 * a + k];
    out |= R.free_bnd && !(x >= R.win_lo[k] && x <= R.win_hi[k]);
    const double w = x - R.box[k] * floor(x * R.invbox[k]);
    int q = (int)(w / R.cell[k]);
    c[k] = q < 0 ? 0 : (q >= R.grid[k] ? R.grid[k] - 1 : q);
  }
  if (out) atomicOr(P.status, ERR_FREE_WINDOW);
  const unsigned key = (unsigned)(R.key0 + (c[1] * R.grid[0] + c[0]) * R.grid[2] + c[2]);
  P.key[a] = key;
  atomicAdd(&P.hist[key], 1);
}

__global__ void k_scatter(DevPtrs P, int natom) {
  int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  unsigned key = P.key[a];
  int pos = P.hist_scan[key] + atomicAdd(&P.cursor[key], 1);
  P.sorted[pos] = a;
}

// deterministic order inside each bin: ascending atom index (bins hold a few atoms)
__global__ void k_sort_bins(DevPtrs P, int nkeys) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nkeys) return;
  int n = P.hist[k];
  if (n < 2) return;
  int* s = P.sorted + P.hist_scan[k];
  for (int i = 1; i < n; ++i) {
    int v = s[i];
    int j = i - 1;
    while (j >= 0 && s[j] > v) { s[j + 1] = s[j]; --j; }
    s[j + 1] = v;
  }
}

// blocks each column needs: ceil(atoms in column / 32)
__global__ void k_col_count(DevPtrs P, int ncol) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncol) return;
  const int r = P.col_rep[c];
  const Rep& R = P.reps[r];
  const int k0 = R.key0 + (c - R.col0) * R.grid[2];
  const int n = P.hist_scan[k0 + R.grid[2]] - P.hist_scan[k0];
  P.col_nb[c] = (n + kTile - 1) / kTile;
}

__global__ void k_clear_slots(DevPtrs P, int nslot, int dummy_type) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslot) return;
  P.satom[s] = -1;
  P.styp[s] = dummy_type;
}

// sorted position -> slot: block = replica's first block + blocks of the columns before this
// one (a column never shares a block with another), lane = rank inside the column
__global__ void k_fill_slots(DevPtrs P, int natom) {
  const int pos = blockIdx.x * blockDim.x + threadIdx.x;
  if (pos >= natom) return;
  const int a = P.sorted[pos];
  const Rep& R = P.reps[P.rep_of[a]];
  const int col = R.col0 + ((int)P.key[a] - R.key0) / R.grid[2];
  const int kcol = R.key0 + (col - R.col0) * R.grid[2];
  const int rank = pos - P.hist_scan[kcol];
  const int blk = R.blk0 + (P.col_blk[col] - P.col_blk[R.col0]) + rank / kTile;
  const int slot = blk * kTile + (rank % kTile);
  P.slot_of[a] = slot;
  P.satom[slot] = a;
  P.styp[slot] = P.typ[a];
}

// one warp per block
__global__ void k_block_setup(DevPtrs P, int nblk, double qscale) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= nblk) return;
  const int slot = warp * kTile + lane;
  const int a = P.satom[slot];
  const Rep& R = P.reps[P.blk_rep[warp]];
  double w[3] = {0, 0, 0}, img[3] = {0, 0, 0};
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    if (a >= 0) {
      double x = P.x[3 * a + k];
      img[k] = floor(x * R.invbox[k]);
      w[k] = x - R.box[k] * img[k];
      lo[k] = w[k];
      hi[k] = w[k];
    } else {
      lo[k] = 1e300;
      hi[k] = -1e300;
    }
    for (int o = 16; o > 0; o >>= 1) {
      lo[k] = fmin(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], o));
      hi[k] = fmax(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], o));
    }
  }
  double ref[3];
  for (int k = 0; k < 3; ++k) ref[k] = 0.5 * (lo[k] + hi[k]);
  if (lane == 0) {
    P.blk_ref[3 * warp + 0] = ref[0];
    P.blk_ref[3 * warp + 1] = ref[1];
    P.blk_ref[3 * warp + 2] = ref[2];
    P.blk_ctr[warp] = make_float4((float)ref[0], (float)ref[1], (float)ref[2], 0.f);
    // an empty block (capacity not used this rebuild) gets a -inf extent: it never passes
    // the bounding-box test
    P.blk_half[warp] = make_float4((float)(0.5 * (hi[0] - lo[0])) + 1e-4f,
                                   (float)(0.5 * (hi[1] - lo[1])) + 1e-4f,
                                   (float)(0.5 * (hi[2] - lo[2])) + 1e-4f, 0.f);
    if (lo[0] <= hi[0]) {   // largest block half-extent per replica (non-negative floats
                            // order like their bit patterns)
      const int r = P.blk_rep[warp];
      for (int k = 0; k < 3; ++k)
        atomicMax(reinterpret_cast<int*>(&P.rep_hmax[3 * r + k]),
                  __float_as_int((float)(0.5 * (hi[k] - lo[k]))));
    }
  }
  double o[3];
  for (int k = 0; k < 3; ++k) o[k] = ref[k] + R.box[k] * img[k];
  P.off[3 * slot + 0] = o[0];
  P.off[3 * slot + 1] = o[1];
  P.off[3 * slot + 2] = o[2];
  if (a >= 0) {
    float q = (float)((double)qscale * P.chg[a]);
    P.pos_f[slot] = make_float4((float)(P.x[3 * a] - o[0]), (float)(P.x[3 * a + 1] - o[1]),
                                (float)(P.x[3 * a + 2] - o[2]), q);
  } else {
    P.pos_f[slot] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// FP64 slot positions (absolute master coordinates) + charges; used every step by the FP64
// path and after a rebuild by both paths.
__global__ void k_fill_pos_d(DevPtrs P, int nslot, double qscale) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nslot) return;
  int a = P.satom[s];
  if (a >= 0) P.pos_d[s] = make_double4(P.x[3 * a], P.x[3 * a + 1], P.x[3 * a + 2], qscale * P.chg[a]);
  else P.pos_d[s] = make_double4(0.0, 0.0, 0.0, 0.0);
}

// slot of every exclusion partner, refreshed after each sort: lets the tile build clear
// excluded pairs per partner instead of searching the partner list per pair
__global__ void k_excl_slots(DevPtrs P, int natom) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  for (int p = P.excl_ptr[a]; p < P.excl_ptr[a + 1]; ++p) P.excl_slot[p] = P.slot_of[P.excl_idx[p]];
}

constexpr int kExclReg = 8;   // exclusion partners held in registers per i-atom

// Tile list, pass A: one warp per chunk = (i-block, 32 consecutive candidate j-blocks
// starting at j0 >= i, same replica).  Bounding-box test of the 32 candidates at once, then
// for each survivor the exact mask; non-empty masks go to the chunk's scratch slots.
// CMM: level-1 cells ci / cj (packed 0-based x | y << 8 | z << 16, -1 = off the grid);
// neighbours (neartb.f90 first table) set mask and mel, cells up to idelay apart with
// r^2 < rc2 at the rebuild (neartb.f90:330-370, the LJ-only table) set mask only
template <bool CMM>
__device__ __forceinline__ unsigned tile_mask(const DevPtrs& P, const Rep& R, int bi, int bj, int lane,
                                              int ai, double xi, double yi, double zi,
                                              const int (&ps)[kExclReg], int pb, int pe,
                                              double rlim2, int ci, double rc2, unsigned& mel) {
  const int aj = P.satom[bj * kTile + lane];
  double xj = 0, yj = 0, zj = 0;
  int cj = -1;
  if (aj >= 0) {
    xj = P.x[3 * aj]; yj = P.x[3 * aj + 1]; zj = P.x[3 * aj + 2];
    if (CMM) cj = P.cmm_cell[aj];
  }
  unsigned mask = 0;
  mel = 0;
  const double bx = R.box[0], by = R.box[1], bz = R.box[2];
  const double ibx = R.invbox[0], iby = R.invbox[1], ibz = R.invbox[2];
  const int idelay = R.idelay;
  for (int k = 0; k < 32; ++k) {
    const int src = (lane + k) & 31;
    const double xk = __shfl_sync(0xffffffffu, xj, src);
    const double yk = __shfl_sync(0xffffffffu, yj, src);
    const double zk = __shfl_sync(0xffffffffu, zj, src);
    const int ak = __shfl_sync(0xffffffffu, aj, src);
    const int ck = CMM ? __shfl_sync(0xffffffffu, cj, src) : 0;
    if (ai < 0 || ak < 0) continue;
    if (bj == bi && (k == 0 || k > 16 || (k == 16 && lane >= 16))) continue;
    double dx = xi - xk, dy = yi - yk, dz = zi - zk;
    dx -= bx * anint(dx * ibx);
    dy -= by * anint(dy * iby);
    dz -= bz * anint(dz * ibz);
    const double d2 = dx * dx + dy * dy + dz * dz;
    if (CMM) {
      if (ci < 0 || ck < 0) continue;
      const int cheb = max(abs((ci & 255) - (ck & 255)),
                           max(abs(((ci >> 8) & 255) - ((ck >> 8) & 255)), abs((ci >> 16) - (ck >> 16))));
      if (cheb <= 1) {
        mask |= 1u << k;
        mel |= 1u << k;
      } else if (idelay > 1 && cheb <= idelay && d2 < rc2) {
        mask |= 1u << k;
      }
    } else if (d2 <= rlim2) {
      mask |= 1u << k;
    }
  }
  // 1-2/1-3/1-4 partners of the i-atom that sit in block bj: lane l sees slot
  // bj*32 + ((l+k)&31) at bit k
  if (mask) {
#pragma unroll
    for (int q = 0; q < kExclReg; ++q)
      if ((ps[q] >> 5) == bj) mask &= ~(1u << (((ps[q] & 31) - lane) & 31));
    for (int p = pb + kExclReg; p < pe; ++p) {
      const int sp = P.excl_slot[p];
      if ((sp >> 5) == bj) mask &= ~(1u << (((sp & 31) - lane) & 31));
    }
  }
  mel &= mask;
  return mask;
}

// Fast form of the mask (no CMM, large box): lane = j atom; the i block is read from shared
// memory one atom per step (a broadcast) and a ballot gives that i atom's row of the tile at
// once; lane i keeps row i and rotates it into the kernels' layout (bit k = j (i + k) & 31).
// Coordinates are wrapped (x - box floor(x / box)) and the tile's image is the block
// references' minimum image n, exact for every pair the list can hold when box/2 > list
// radius + block extents (the condition of the pair kernels' per-tile shift).
struct IStage {
  double x[kTile], y[kTile], z[kTile];
  float xf[kTile], yf[kTile], zf[kTile];   // the same relative to the i block's reference
  float4 live[kTile];                      // a candidate's live i atoms, compacted (x, y, z, lane)
};

// The exact list radius decides in FP64, but almost every pair is far from it: the mask is
// first built in FP32 on coordinates relative to the i block's reference (|x| <~ 25 A, so
// d^2 is good to ~3e-4 A^2), and a tile with any pair within `band` of rlim^2 is redone by
// tile_mask_fast in FP64; the FP32 mask is returned only where every decision is certain,
// so the list is the FP64 list.  `unsure` is warp-uniform.
// A j atom in the i frame is its block-local position (pos_f, relative to its block's
// reference in the wrapped frame) plus block bj's reference shifted by the tiles' image into
// the i block's frame.  Only the i atoms within the list radius of block bj's bounding box
// (with a margin of 1e-4 rlim^2 + 1e-3 A^2, far wider than `band` and the FP32 rounding) can
// list a pair; the rows of the others are certainly empty, and the loop skips them.
// PIMG (a box at most twice the list radius plus two block extents): the tiles' image is not
// every pair's, so each pair takes its own minimum image in FP32 and no i atom is culled.
template <bool PIMG>
__device__ __forceinline__ unsigned tile_row_f32(const DevPtrs& P, const Rep& R, int bi, int bj, int lane,
                                                 IStage& S, float rlim2f, float band, bool& unsure) {
  const int aj = P.satom[bj * kTile + lane];
  float cj[3];   // block bj's reference (its bounding-box centre) in the i block's frame
  for (int k = 0; k < 3; ++k) {
    const double d = P.blk_ref[3 * bi + k] - P.blk_ref[3 * bj + k];
    cj[k] = (float)(R.box[k] * anint(d * R.invbox[k]) - d);
  }
  const float4 pj = P.pos_f[bj * kTile + lane];
  const float r[3] = {pj.x + cj[0], pj.y + cj[1], pj.z + cj[2]};
  unsigned live;
  if (PIMG) {   // every real i atom (padding slots sit at 1e18)
    live = __ballot_sync(0xffffffffu, S.xf[lane] < 1.0e17f);
  } else {
    const float4 hj = P.blk_half[bj];
    const float gx = fmaxf(fabsf(S.xf[lane] - cj[0]) - hj.x, 0.f);
    const float gy = fmaxf(fabsf(S.yf[lane] - cj[1]) - hj.y, 0.f);
    const float gz = fmaxf(fabsf(S.zf[lane] - cj[2]) - hj.z, 0.f);
    live = __ballot_sync(0xffffffffu, fmaf(gx, gx, fmaf(gy, gy, gz * gz)) <= rlim2f * 1.0001f + 1e-3f);
  }
  const float bx = (float)R.box[0], by = (float)R.box[1], bz = (float)R.box[2];
  const float ibx = (float)R.invbox[0], iby = (float)R.invbox[1], ibz = (float)R.invbox[2];
  unsigned row = 0;
  bool u = false;
  // the live i atoms compacted in shared memory, so each pass reads two of them by
  // position instead of scanning the bit mask (bit scans run on the XU pipe); two i atoms
  // per pass: two independent distance chains and ballots
  const int nlive = __popc(live);
  __syncwarp();   // the previous candidate's passes are done with S.live
  if ((live >> lane) & 1u)
    S.live[__popc(live & ((1u << lane) - 1u))] = make_float4(S.xf[lane], S.yf[lane], S.zf[lane], __int_as_float(lane));
  __syncwarp();
  auto d2of = [&](float4 a) {
    float dx = a.x - r[0], dy = a.y - r[1], dz = a.z - r[2];
    if (PIMG) {
      dx = fmaf(-bx, rintf(dx * ibx), dx);
      dy = fmaf(-by, rintf(dy * iby), dy);
      dz = fmaf(-bz, rintf(dz * ibz), dz);
    }
    return fmaf(dx, dx, fmaf(dy, dy, dz * dz));
  };
  for (int q = 0; q < nlive; q += 2) {   // warp-uniform
    const bool has2 = q + 1 < nlive;
    const float4 a = S.live[q];
    const float4 c = S.live[has2 ? q + 1 : q];
    const float d2 = d2of(a), e2 = d2of(c);
    const bool in = aj >= 0 && d2 <= rlim2f;
    const bool in2 = aj >= 0 && has2 && e2 <= rlim2f;
    u |= aj >= 0 && fabsf(d2 - rlim2f) < band;
    u |= aj >= 0 && has2 && fabsf(e2 - rlim2f) < band;
    const unsigned b = __ballot_sync(0xffffffffu, in);
    const unsigned b2 = __ballot_sync(0xffffffffu, in2);
    if (lane == __float_as_int(a.w)) row = b;
    if (has2 && lane == __float_as_int(c.w)) row = b2;
  }
  unsure = __any_sync(0xffffffffu, u);
  return row;
}

// row i of a tile (bit j: pair (i, j) within the list radius) into the kernels' rotated
// layout, each unordered pair once, exclusions removed
__device__ __forceinline__ unsigned finish_mask(const DevPtrs& P, int bi, int bj, int lane, unsigned row,
                                                const int (&ps)[kExclReg], int pb, int pe) {
  unsigned mask = __funnelshift_r(row, row, lane);
  if (bj == bi) mask &= lane < 16 ? 0x1fffeu : 0xfffeu;   // each unordered pair once, no self pair
  if (mask) {
#pragma unroll
    for (int q = 0; q < kExclReg; ++q)
      if ((ps[q] >> 5) == bj) mask &= ~(1u << (((ps[q] & 31) - lane) & 31));
    for (int p = pb + kExclReg; p < pe; ++p) {
      const int sp = P.excl_slot[p];
      if ((sp >> 5) == bj) mask &= ~(1u << (((sp & 31) - lane) & 31));
    }
  }
  return mask;
}

__device__ __forceinline__ unsigned tile_mask_fast(const DevPtrs& P, const Rep& R, int bi, int bj, int lane,
                                                   int ai, const IStage& S, const int (&ps)[kExclReg],
                                                   int pb, int pe, double rlim2) {
  const int aj = P.satom[bj * kTile + lane];
  double xj = 0.0, yj = 0.0, zj = 0.0;
  if (aj >= 0) {
    double w[3];
    for (int k = 0; k < 3; ++k) {
      const double x = P.x[3 * aj + k];
      const double n = anint((P.blk_ref[3 * bi + k] - P.blk_ref[3 * bj + k]) * R.invbox[k]);
      w[k] = (x - R.box[k] * floor(x * R.invbox[k])) + R.box[k] * n;
    }
    xj = w[0]; yj = w[1]; zj = w[2];
  }
  unsigned row = 0;
#pragma unroll 8
  for (int i = 0; i < kTile; ++i) {
    const double dx = S.x[i] - xj, dy = S.y[i] - yj, dz = S.z[i] - zj;
    const bool in = aj >= 0 && dx * dx + dy * dy + dz * dz <= rlim2;
    const unsigned b = __ballot_sync(0xffffffffu, in);
    if (lane == i) row = b;
  }
  if (ai < 0) row = 0;
  return finish_mask(P, bi, bj, lane, row, ps, pb, pe);
}

template <bool CMM>
__global__ void __launch_bounds__(128, 6) k_tile_scan_chunks(DevPtrs P, int nchunk, double rlim2, float rlimf,
                                                          double rc2) {
  const float rlim2f = (float)rlim2;
  __shared__ IStage s_i[4];
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nchunk) return;
  const int bi = P.chunk_i[w], j0 = P.chunk_j0[w];
  const int rep = P.blk_rep[bi];
  const Rep& R = P.reps[rep];
  // exact when a pair within the list radius cannot be another image than the blocks':
  // box/2 > list radius + the two blocks' half extents (largest of the replica)
  bool fast = !CMM;
  for (int k = 0; k < 3; ++k)
    if (!(0.5 * R.box[k] > sqrt(rlim2) + 2.0 * (double)P.rep_hmax[3 * rep + k] + 0.01)) fast = false;
  const int bend = R.blk0 + R.nblk;
  const float4 ci = P.blk_ctr[bi], hi = P.blk_half[bi];
  const int bj = j0 + lane;
  bool cand = false;
  if (bj < bend) {
    const float4 cj = P.blk_ctr[bj], hj = P.blk_half[bj];
    float dx = ci.x - cj.x, dy = ci.y - cj.y, dz = ci.z - cj.z;
    dx -= (float)R.box[0] * rintf(dx * (float)R.invbox[0]);
    dy -= (float)R.box[1] * rintf(dy * (float)R.invbox[1]);
    dz -= (float)R.box[2] * rintf(dz * (float)R.invbox[2]);
    const float gx = fmaxf(fabsf(dx) - hi.x - hj.x, 0.f);
    const float gy = fmaxf(fabsf(dy) - hi.y - hj.y, 0.f);
    const float gz = fmaxf(fabsf(dz) - hi.z - hj.z, 0.f);
    cand = gx * gx + gy * gy + gz * gz <= rlimf * rlimf * 1.0001f + 1e-3f;
  }
  unsigned ball = __ballot_sync(0xffffffffu, cand);
  unsigned nz = 0;
  int nent0 = 0, nent1 = 0;   // entries of the two half blocks (rows 0-15, 16-31)
  if (ball) {
    const int ai = P.satom[bi * kTile + lane];
    double xi = 0, yi = 0, zi = 0;
    int pb = 0, pe = 0, ci = -1;
    int ps[kExclReg];
    if (ai >= 0) {
      xi = P.x[3 * ai]; yi = P.x[3 * ai + 1]; zi = P.x[3 * ai + 2];
      pb = P.excl_ptr[ai];
      pe = P.excl_ptr[ai + 1];
      if (CMM) ci = P.cmm_cell[ai];
    }
#pragma unroll
    for (int q = 0; q < kExclReg; ++q) ps[q] = pb + q < pe ? P.excl_slot[pb + q] : -64;
    IStage& S = s_i[threadIdx.x >> 5];
    if (!CMM) {   // the i block, wrapped, for the broadcast reads
      S.x[lane] = xi - R.box[0] * floor(xi * R.invbox[0]);
      S.y[lane] = yi - R.box[1] * floor(yi * R.invbox[1]);
      S.z[lane] = zi - R.box[2] * floor(zi * R.invbox[2]);
      // padding slots far away: they never list a pair nor make a tile uncertain
      S.xf[lane] = ai >= 0 ? (float)(S.x[lane] - P.blk_ref[3 * bi + 0]) : 1.0e18f;
      S.yf[lane] = ai >= 0 ? (float)(S.y[lane] - P.blk_ref[3 * bi + 1]) : 1.0e18f;
      S.zf[lane] = ai >= 0 ? (float)(S.z[lane] - P.blk_ref[3 * bi + 2]) : 1.0e18f;
      __syncwarp();
    }
    // the FP32 mask's uncertainty band: every coordinate tile_row_f32 works with is below
    // M = rlim + 3 h_max in magnitude (h_max: the replica's largest block half extent) and
    // carries at most 2.5 roundings of 2^-24 M, a difference one more, so |error of d^2| <=
    // 2 sqrt(3) rlim 5 2^-24 M + 3 2^-24 rlim^2; pairs within 4 times that of rlim^2 are
    // decided in FP64 (about 1.5e-3 A^2 for water blocks at rc = 12 A)
    const float hm = fmaxf(P.rep_hmax[3 * rep], fmaxf(P.rep_hmax[3 * rep + 1], P.rep_hmax[3 * rep + 2]));
    // with per-pair images (a small box) the coordinates before imaging reach the box edge
    const float mb = fast ? rlimf + 3.f * hm
                          : fmaxf(rlimf + 3.f * hm, (float)fmax(R.box[0], fmax(R.box[1], R.box[2])) + 3.f * hm);
    const float band = 4.f * 5.9604645e-8f * (17.33f * rlimf * mb + 3.f * rlimf * rlimf);
    while (ball) {
      const int b = __ffs(ball) - 1;
      ball &= ball - 1;
      unsigned mel = 0;
      unsigned m;
      bool unsure = true;
      if (!CMM) {
        unsigned row = fast ? tile_row_f32<false>(P, R, bi, j0 + b, lane, S, rlim2f, band, unsure)
                            : tile_row_f32<true>(P, R, bi, j0 + b, lane, S, rlim2f, band, unsure);
        if (!unsure) {
          if (ai < 0) row = 0;
          m = finish_mask(P, bi, j0 + b, lane, row, ps, pb, pe);
        }
      }
      if (unsure)
        m = fast ? tile_mask_fast(P, R, bi, j0 + b, lane, ai, S, ps, pb, pe, rlim2)
                 : tile_mask<CMM>(P, R, bi, j0 + b, lane, ai, xi, yi, zi, ps, pb, pe, rlim2, ci, rc2, mel);
      if (__any_sync(0xffffffffu, m != 0)) {
        P.tmp_masks[((size_t)w * 32 + b) * 32 + lane] = m;
        if (CMM) P.tmp_masks_el[((size_t)w * 32 + b) * 32 + lane] = mel;
        // the j lanes some i atom of each half block lists: the entries this tile
        // contributes to the two halves' pair records
        const unsigned rowj = __funnelshift_l(m, m, lane);
        const unsigned occ0 = __reduce_or_sync(0xffffffffu, lane < kHalf ? rowj : 0u);
        const unsigned occ1 = __reduce_or_sync(0xffffffffu, lane < kHalf ? 0u : rowj);
        if (lane == 0) {
          P.tmp_occ[((size_t)w * 32 + b) * 2 + 0] = occ0;
          P.tmp_occ[((size_t)w * 32 + b) * 2 + 1] = occ1;
        }
        nent0 += __popc(occ0);
        nent1 += __popc(occ1);
        nz |= 1u << b;
      }
    }
  }
  if (lane == 0) {
    P.chunk_nz[w] = nz;
    P.chunk_cnt[w] = __popc(nz);
    P.chunk_ent[w] = nent0;
    P.chunk_ent[nchunk + 1 + w] = nent1;
  }
}

// pass C: copy non-empty tiles to the dense list at the scanned offsets (row-major, j order)
void launch_tile_scan(const DevPtrs& P, int nchunk, double rlim2, float rlimf, double rc2, bool cmm,
                      cudaStream_t st) {
  const int nwb = (nchunk * 32 + 127) / 128;
  if (cmm) k_tile_scan_chunks<true><<<nwb, 128, 0, st>>>(P, nchunk, rlim2, rlimf, rc2);
  else k_tile_scan_chunks<false><<<nwb, 128, 0, st>>>(P, nchunk, rlim2, rlimf, rc2);
}

__global__ void k_tile_emit(DevPtrs P, int nchunk, int cmm) {
  const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (w >= nchunk) return;
  const unsigned nz = P.chunk_nz[w];
  if (!nz) return;
  const int bi = P.chunk_i[w], j0 = P.chunk_j0[w];
  const int t0 = P.chunk_off[w];
  const int cnt = __popc(nz);
  // lane q: the chunk's q-th tile's occupied j lanes of each half block and its first entry
  // in that half's entry order (global)
  for (int h = 0; h < 2; ++h) {
    const int b = lane < cnt ? (int)__fns(nz, 0, lane + 1) : 0;
    const unsigned occ = lane < cnt ? P.tmp_occ[((size_t)w * 32 + b) * 2 + h] : 0u;
    int e = __popc(occ);
    for (int o = 1; o < 32; o <<= 1) {   // inclusive scan over the lanes
      const int y = __shfl_up_sync(0xffffffffu, e, o);
      if (lane >= o) e += y;
    }
    if (lane < cnt) {
      P.tile_occ[2 * (size_t)(t0 + lane) + h] = occ;
      P.tile_eoff[2 * (size_t)(t0 + lane) + h] = P.chunk_eoff[h * (nchunk + 1) + w] + e - __popc(occ);
    }
  }
  if (lane < cnt) {   // lane q: the chunk's q-th tile, its block pair and image shift
    const Rep& R = P.reps[P.blk_rep[bi]];
    const int bj = j0 + (int)__fns(nz, 0, lane + 1);
    P.tiles[t0 + lane] = make_int2(bi, bj);
    P.tile_src[t0 + lane] = w * 32 + (bj - j0);   // its mask rows stay where the scan wrote them
    float sh[3];
    for (int k = 0; k < 3; ++k) {
      const double d = P.blk_ref[3 * bi + k] - P.blk_ref[3 * bj + k];
      sh[k] = (float)(d - R.box[k] * anint(d * R.invbox[k]));
    }
    P.tile_shift[t0 + lane] = make_float4(sh[0], sh[1], sh[2], 0.f);
  }
}

// ---- pair records ------------------------------------------------------------------------
// The pair kernels run on pair records: a half block (16 i atoms: rows 0-15 or 16-31 of an
// i-block, unit u = 2 i-block + half) with 32 j entries, the j atoms of that block's tiles
// that at least one of the 16 i atoms lists, taken in tile order (ascending j block,
// ascending slot).  A 32 x 32 tile of two blocks holds ~26 % listed pairs at the md_run list
// radius; keeping only the j atoms a half block lists raises that to ~55 %, because 16 atoms
// span a smaller volume than 32 (within the cut-off: 32 % of the slots with whole blocks,
// 39 % with half blocks), and the pair kernels' work per pair falls in proportion.  The
// listed pair set is unchanged.  Each entry carries its tile's image shift (into the i
// block's frame) and its slot; the mask of i atom l (0..15) has bit k = entry (l + k) & 15
// and bit 16 + k = entry 16 + ((l + k) & 15), the order in which the kernels meet them.

// tiles of i-block bi: [chunk_off[blk_chunk0[bi]], chunk_off[blk_chunk0[bi + 1]]); the
// entries of its half h: [eoff_h[blk_chunk0[bi]], eoff_h[blk_chunk0[bi + 1]]) in global
// order, eoff_h = chunk_eoff + h (nchunk + 1) (the tile scan counts each tile's occupied j
// lanes per half, the tile emit places each tile's entries)

// per unit (one thread each): the pair records it needs
__global__ void k_ct_count(DevPtrs P, int nblk, int nchunk) {
  const int u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= 2 * nblk) return;
  const int b = u >> 1, h = u & 1;
  const int* eoff = P.chunk_eoff + h * (nchunk + 1);
  const int ne = eoff[P.blk_chunk0[b + 1]] - eoff[P.blk_chunk0[b]];
  P.ct_cnt[u] = (ne + 31) >> 5;
}

// per tile (one thread each, after the scan of ct_cnt) and half: the records of the unit
// whose first slot falls among the tile's entries of that half get their unit and, for the
// emit, the tile as their first source tile, their first slot's global entry, the end of the
// unit's entries and of the block's tiles (a tile holds at most 32 entries, so at most two
// records start in it)
__global__ void k_ct_index(DevPtrs P, int nchunk) {
  const int T = *P.ntiles;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
    const int b = P.tiles[t].x;
    const int c0 = P.blk_chunk0[b], c1 = P.blk_chunk0[b + 1];
    const int tl = P.chunk_off[c1] - 1;   // the block's last tile
    for (int h = 0; h < 2; ++h) {
      const int* eoff = P.chunk_eoff + h * (nchunk + 1);
      const int e0 = eoff[c0];
      const int lo = P.tile_eoff[2 * (size_t)t + h] - e0;
      const int hi = t < tl ? P.tile_eoff[2 * (size_t)(t + 1) + h] - e0 : eoff[c1] - e0;
      const int u = 2 * b + h;
      for (int k = (lo + 31) >> 5; 32 * k < hi; ++k) {
        P.ct_blk[P.ct_off[u] + k] = u;
        P.ct_info[P.ct_off[u] + k] = make_int4(t, e0 + 32 * k, eoff[c1], ((tl + 1) << 1) | h);
      }
    }
  }
}

// a record row (bit e: entry e) into the kernels' order for i atom l: each 16-bit half
// rotated right by l
__device__ __forceinline__ unsigned record_row(unsigned row, int l) {
  const unsigned lo = row & 0xffffu, hi = row >> 16;
  const unsigned rl = ((lo >> l) | (lo << (16 - l))) & 0xffffu;
  const unsigned rh = ((hi >> l) | (hi << (16 - l))) & 0xffffu;
  return rl | (rh << 16);
}

// One warp per record, lane p for slot p.  The record's source tiles are consecutive from
// ct_info's first tile and at most 32 (each holds at least one entry and the first covers
// slot 0), so lane q reads source tile q's entry offset, occupancy, j block, image shift and
// mask rows' place in one coalesced pass; each slot finds its tile and its rank among the
// tile's entries by shuffles, and writes its entry.  Record row r (i atom 16 h + r) is then
// one ballot: every slot contributes the bit of its j lane in row 16 h + r of its tile, so no
// lane packs bits and lane r keeps row r.
__global__ void k_ct_emit(DevPtrs P, int nchunk, int cmm) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int nw = (gridDim.x * blockDim.x) >> 5;
  const int T = *P.nctiles;
  for (int ct = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ct < T; ct += nw) {
    const int4 info = P.ct_info[ct];
    const int ts = info.x, s0 = info.y, e1 = info.z, t1 = info.w >> 1, h = info.w & 1;
    const int tq = ts + lane;   // lane q: source tile q
    int qb = 32, qy = 0, qs = 0;
    unsigned qocc = 0u;
    float4 qsh = make_float4(0.f, 0.f, 0.f, 0.f);
    if (tq < t1) {
      qb = P.tile_eoff[2 * (size_t)tq + h] - s0;   // slot of the tile's first entry (may be < 0)
      if (qb < 32) {
        qocc = P.tile_occ[2 * (size_t)tq + h];
        qy = P.tiles[tq].y;
        qsh = P.tile_shift[tq];
        qs = P.tile_src[tq];
      }
    }
    const int nt = __popc(__ballot_sync(full, tq < t1 && qb < 32));   // lanes 0 .. nt-1
    unsigned cur = 0u, cur_el = 0u;
    int src = -1, kk = 0;   // this slot's source tile and its rank among the tile's entries
    for (int j = 0; j < nt; ++j) {   // warp-uniform: every lane looks for its slot
      const int base = __shfl_sync(full, qb, j);
      const int n = __popc(__shfl_sync(full, qocc, j));   // both shuffles by every lane
      const int k = lane - base;
      if (k >= 0 && k < n) {
        src = j;
        kk = k;
      }
    }
    const int sy = __shfl_sync(full, qy, src & 31);
    const unsigned socc = __shfl_sync(full, qocc, src & 31);
    const int sm = __shfl_sync(full, qs, src & 31);   // the source tile's rows in tmp_masks
    const float shx = __shfl_sync(full, qsh.x, src & 31);
    const float shy = __shfl_sync(full, qsh.y, src & 31);
    const float shz = __shfl_sync(full, qsh.z, src & 31);
    const bool live = src >= 0 && s0 + lane < e1;
    const int jl = live ? (int)__fns(socc, 0, kk + 1) : 0;   // the slot's j lane in its tile
    float4 ent = make_float4(0.f, 0.f, 0.f, __int_as_float(-1));
    if (live) ent = make_float4(shx, shy, shz, __int_as_float(sy * kTile + jl));
    P.ct_j[(size_t)ct * 32 + lane] = ent;
    // record row r (bit p: slot p) is one ballot: slot p's bit is bit jl of row 16 h + r of its
    // source tile (stored rotated: bit k is j lane (row + k) & 31); lane r keeps row r
    {
      const unsigned* rows = P.tmp_masks + (size_t)(live ? sm : 0) * 32 + kHalf * h;
      unsigned m[kHalf];
#pragma unroll
      for (int r = 0; r < kHalf; ++r) m[r] = live ? rows[r] : 0u;
#pragma unroll
      for (int r = 0; r < kHalf; ++r) {
        const unsigned row = __ballot_sync(full, (m[r] >> ((jl - kHalf * h - r) & 31)) & 1u);
        if (lane == r) cur = row;
      }
      if (cmm) {
        const unsigned* rows_el = P.tmp_masks_el + (size_t)(live ? sm : 0) * 32 + kHalf * h;
#pragma unroll
        for (int r = 0; r < kHalf; ++r) m[r] = live ? rows_el[r] : 0u;
#pragma unroll
        for (int r = 0; r < kHalf; ++r) {
          const unsigned row = __ballot_sync(full, (m[r] >> ((jl - kHalf * h - r) & 31)) & 1u);
          if (lane == r) cur_el = row;
        }
      }
    }
    if (lane < kHalf) {
      P.ct_mask[(size_t)ct * kHalf + lane] = record_row(cur, lane);
      if (cmm) P.ct_mask_el[(size_t)ct * kHalf + lane] = record_row(cur_el, lane);
    }
  }
}

int launch_compact_tiles(const DevPtrs& P, int nblk, int nchunk, int nsm, bool cmm, int* scan_scratch,
                         cudaStream_t st) {
  const int nb = (2 * nblk + 127) / 128;
  k_ct_count<<<nb, 128, 0, st>>>(P, nblk, nchunk);
  const int ns = scan_exclusive(P.ct_cnt, P.ct_off, 2 * nblk + 1, scan_scratch, P.nctiles, st);
  k_ct_index<<<nsm * 4, 256, 0, st>>>(P, nchunk);
  k_ct_emit<<<nsm * 8, 256, 0, st>>>(P, nchunk, cmm ? 1 : 0);
  return 3 + ns;
}

// ---- deterministic exclusive scan (3 passes) --------------------------------------------
__global__ void k_scan_block_sums(const int* in, int n, int* bsum) {
  __shared__ int sh[1024];
  int i = blockIdx.x * 1024 + threadIdx.x;
  int v = i < n ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 512; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] += sh[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) bsum[blockIdx.x] = sh[0];
}

// single block: exclusive scan of nb block sums (any nb)
__global__ void k_scan_small(int* bsum, int nb) {
  __shared__ int sh[1024];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int b0 = 0; b0 < nb; b0 += 1024) {
    int i = b0 + threadIdx.x;
    int v = i < nb ? bsum[i] : 0;
    sh[threadIdx.x] = v;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
      int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
      __syncthreads();
      sh[threadIdx.x] += t;
      __syncthreads();
    }
    if (i < nb) bsum[i] = carry + sh[threadIdx.x] - v;
    __syncthreads();
    if (threadIdx.x == 1023) carry += sh[1023];
    __syncthreads();
  }
}

__global__ void k_scan_final(const int* in, int n, const int* bsum, int* out, int* total) {
  __shared__ int sh[1024];
  int i = blockIdx.x * 1024 + threadIdx.x;
  int v = i < n ? in[i] : 0;
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int t = threadIdx.x >= o ? sh[threadIdx.x - o] : 0;
    __syncthreads();
    sh[threadIdx.x] += t;
    __syncthreads();
  }
  if (i < n) out[i] = bsum[blockIdx.x] + sh[threadIdx.x] - v;
  if (i == n - 1 && total) *total = bsum[blockIdx.x] + sh[threadIdx.x];
}

// one block for up to kScanOneMax values: thread t sums its run of consecutive values, the
// 1024 run sums are scanned with warp shuffles, and each thread writes its run's prefixes
constexpr int kScanOneMax = 1 << 13;   // above it the three-pass scan is faster

__global__ void __launch_bounds__(1024) k_scan_one(const int* in, int n, int* out, int* total) {
  __shared__ int wsum[32];
  const unsigned full = 0xffffffffu;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int per = (n + 1023) / 1024;
  const int b = min(t * per, n), e = min(b + per, n);
  int s = 0;
  for (int i = b; i < e; ++i) s += in[i];
  int x = s;   // inclusive scan of the run sums: within the warp, then over the warps
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(full, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int w = wsum[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(full, w, o);
      if (lane >= o) w += y;
    }
    wsum[lane] = w;
  }
  __syncthreads();
  int run = x - s + (wid > 0 ? wsum[wid - 1] : 0);
  for (int i = b; i < e; ++i) {
    const int v = in[i];
    out[i] = run;
    run += v;
  }
  if (t == 0 && total) *total = wsum[31];
}

int scan_exclusive(const int* in, int* out, int n, int* scratch, int* total, cudaStream_t st) {
  if (n <= kScanOneMax) {
    k_scan_one<<<1, 1024, 0, st>>>(in, n, out, total);
    return 1;
  }
  int nb = (n + 1023) / 1024;
  k_scan_block_sums<<<nb, 1024, 0, st>>>(in, n, scratch);
  k_scan_small<<<1, 1024, 0, st>>>(scratch, nb);
  k_scan_final<<<nb, 1024, 0, st>>>(in, n, scratch, out, total);
  return 3;
}

}  // namespace jp
