// jp_noalloc.cu -- jp_nonbond_noalloc: the ZD + LJ non-bonded energy and gradient of one
// system from caller-owned device buffers, with every intermediate in one static device
// array, so that a call allocates no device memory.
//
// It is a variant of the FP64 tile kernel in jp_pair.cu (same pair formula, same 32 x 32
// warp tile with the j atoms rotating through shuffles) that needs no pair list: the tiles
// are all (i-block, j-block) pairs of 32 atoms in input order with j-block >= i-block, and
// the exclusion mask of a tile is built on the fly from the exclusion CSR.  Pairs are
// summed within the cut-off under the minimum image, so the result equals what the
// list-based path gives right after a list rebuild.  Work is O(N^2): meant for systems up
// to JP_NOALLOC_MAX_ATOMS atoms.
//
// Scratch: g_nb_scratch, a file-scope __device__ array (one instance per device):
//   [0]            ZD pair energy           (FP64 atomics)
//   [1]            LJ energy
//   [2]            ZD excess + self energy
//   [3]            status bits (unsigned, low 4 bytes)
//   [4 .. 32)      unused (keeps the force block 256-byte aligned)
//   [32 .. 32+3N)  gradient accumulators dE/dx [N][3]
// The first 32 + 3N words must start at zero; every call clears them with
// cudaMemsetAsync on its stream before the first kernel.  All calls on a device share the
// array: calls whose work overlaps on the GPU (two streams, two host threads) race and
// corrupt each other's results.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>

#include "jp_common.cuh"

namespace jp {
namespace {

constexpr int kHdr = 32;                       // header words before the gradient block
constexpr int kNbThreads = 256;
constexpr int kMaxDevices = 64;
enum : unsigned { NB_BAD_INDEX = 1u, NB_NONFINITE = 2u };

static __device__ __align__(256) double g_nb_scratch[kHdr + 3 * JP_NOALLOC_MAX_ATOMS];

std::mutex g_mu;
std::atomic<double*> g_ptr[kMaxDevices];
int g_nsm[kMaxDevices];   // SM count of each device, written before its g_ptr is published

struct NbArgs {
  int natom, ntype, base;
  const double *x, *q;
  const int *typ;
  const double *c6, *c12;
  const int *eptr, *eidx;
  double box[3], ibox[3];
  double ccoef, irc2, zb, zf, zc, dself_coef;
};

__device__ __forceinline__ void set_status(double* scr, unsigned bits) {
  atomicOr(reinterpret_cast<unsigned*>(scr + 3), bits);
}

// exclusion range [p0, p1) of atom i; false (and NB_BAD_INDEX) unless the CSR row is sane:
// excl_ptr starts at 0, never decreases and no atom has more partners than there are atoms
__device__ __forceinline__ bool excl_range(double* scr, const NbArgs& a, int i, int& p0, int& p1) {
  p0 = a.eptr[i];
  p1 = a.eptr[i + 1];
  if (p0 < 0 || p1 < p0 || p1 - p0 > a.natom || (i == 0 && p0 != 0)) {
    set_status(scr, NB_BAD_INDEX);
    p0 = p1 = 0;
    return false;
  }
  return true;
}

__device__ __forceinline__ void warp_add(double* dst, double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(dst, v);
}

// One warp per (i-block, j-block) tile, j-block >= i-block, grid-stride over nb x nb.
__global__ void __launch_bounds__(kNbThreads) k_nb_tiles(double* scr, NbArgs a) {
  const int lane = threadIdx.x & 31;
  const int nb = (a.natom + 31) >> 5;
  const long long ntile = (long long)nb * nb;
  const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  double* grad = scr + kHdr;
  double eel = 0.0, elj = 0.0;
  for (long long t = gw; t < ntile; t += nw) {
    const int bi = (int)(t / nb), bj = (int)(t % nb);
    if (bj < bi) continue;                    // warp-uniform
    const int i = bi * 32 + lane, j = bj * 32 + lane;
    const bool iv = i < a.natom, jv = j < a.natom;
    double xi = 0, yi = 0, zi = 0, qi = 0;
    int ti = 0;
    unsigned m = 0u;
    if (iv) {
      xi = a.x[3 * i]; yi = a.x[3 * i + 1]; zi = a.x[3 * i + 2];
      qi = a.q[i];
      ti = a.typ[i] - a.base;
      if (ti < 0 || ti >= a.ntype) { set_status(scr, NB_BAD_INDEX); ti = 0; }
      // candidate j lanes: existing atoms, upper triangle on the diagonal tile
      const int nj = min(32, a.natom - bj * 32);
      m = nj >= 32 ? 0xffffffffu : ((1u << nj) - 1u);
      if (bj == bi) m &= lane == 31 ? 0u : (0xffffffffu << (lane + 1));
      int p0, p1;
      excl_range(scr, a, i, p0, p1);
      for (int p = p0; p < p1; ++p) {
        const int e = a.eidx[p] - a.base;
        if (e < 0 || e >= a.natom) { set_status(scr, NB_BAD_INDEX); continue; }
        if ((e >> 5) == bj) m &= ~(1u << (e & 31));
      }
      // bit k <-> j lane (lane + k) & 31, the order the rotation below visits them in
      m = (m >> lane) | (m << ((32 - lane) & 31));
    }
    double xj = 0, yj = 0, zj = 0, qj = 0;
    int tj = 0;
    if (jv) {
      xj = a.x[3 * j]; yj = a.x[3 * j + 1]; zj = a.x[3 * j + 2];
      qj = a.q[j];
      tj = a.typ[j] - a.base;
      if (tj < 0 || tj >= a.ntype) { set_status(scr, NB_BAD_INDEX); tj = 0; }
    }
    // start the rotation at j lane = own lane (k = 0)
    double gix = 0, giy = 0, giz = 0, gjx = 0, gjy = 0, gjz = 0;
    for (int k = 0; k < 32; ++k) {
      if (m & 1u) {
        double dx = xi - xj, dy = yi - yj, dz = zi - zj;
        dx -= a.box[0] * anint(dx * a.ibox[0]);
        dy -= a.box[1] * anint(dy * a.ibox[1]);
        dz -= a.box[2] * anint(dz * a.ibox[2]);
        const double dd2 = dx * dx + dy * dy + dz * dz;
        const double dd2i = 1.0 / dd2;
        if (dd2i - a.irc2 >= 0.0) {
          const double ddi = sqrt(dd2i);
          const double dd6i = dd2i * dd2i * dd2i;
          const double ee = a.ccoef * qi * qj;
          eel += ee * (ddi + a.zb * dd2 - a.zc);
          const int l = ti * a.ntype + tj;
          const double v1 = __ldg(a.c6 + l) * dd6i;
          const double v2 = __ldg(a.c12 + l) * dd6i * dd6i;
          elj += -v1 + v2;
          const double cc = ee * (dd2i * ddi - a.zf) + (-6.0 * v1 + 12.0 * v2) * dd2i;
          const double fx = dx * cc, fy = dy * cc, fz = dz * cc;
          gix -= fx; giy -= fy; giz -= fz;
          gjx += fx; gjy += fy; gjz += fz;
        }
      }
      m >>= 1;
      const int src = (lane + 1) & 31;
      xj = __shfl_sync(0xffffffffu, xj, src);
      yj = __shfl_sync(0xffffffffu, yj, src);
      zj = __shfl_sync(0xffffffffu, zj, src);
      qj = __shfl_sync(0xffffffffu, qj, src);
      tj = __shfl_sync(0xffffffffu, tj, src);
      gjx = __shfl_sync(0xffffffffu, gjx, src);
      gjy = __shfl_sync(0xffffffffu, gjy, src);
      gjz = __shfl_sync(0xffffffffu, gjz, src);
    }
    // after 32 steps each lane holds the j-force of its own j atom again
    if (iv && (gix != 0.0 || giy != 0.0 || giz != 0.0)) {
      atomicAdd(grad + 3 * i + 0, gix);
      atomicAdd(grad + 3 * i + 1, giy);
      atomicAdd(grad + 3 * i + 2, giz);
    }
    if (jv && (gjx != 0.0 || gjy != 0.0 || gjz != 0.0)) {
      atomicAdd(grad + 3 * j + 0, gjx);
      atomicAdd(grad + 3 * j + 1, gjy);
      atomicAdd(grad + 3 * j + 2, gjz);
    }
  }
  warp_add(scr + 0, eel);
  warp_add(scr + 1, elj);
}

// ZD excess of the excluded pairs (each once, j > i) and the ZD self term
// dself = -(z/2) ccoef sum_i q_i (q_i + sum_{j excl i} q_j)   (incel.f90:627-689).
__global__ void __launch_bounds__(kNbThreads) k_nb_excl(double* scr, NbArgs a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double* grad = scr + kHdr;
  double e = 0.0;
  if (i < a.natom) {
    const double qi = a.q[i];
    double qs = qi;
    const double xi = a.x[3 * i], yi = a.x[3 * i + 1], zi = a.x[3 * i + 2];
    double gx = 0, gy = 0, gz = 0;
    int p0, p1;
    excl_range(scr, a, i, p0, p1);
    for (int p = p0; p < p1; ++p) {
      const int j = a.eidx[p] - a.base;
      if (j < 0 || j >= a.natom) continue;     // flagged by k_nb_tiles
      const double qj = a.q[j];
      qs += qj;
      if (j <= i) continue;
      double dx = xi - a.x[3 * j], dy = yi - a.x[3 * j + 1], dz = zi - a.x[3 * j + 2];
      dx -= a.box[0] * anint(dx * a.ibox[0]);
      dy -= a.box[1] * anint(dy * a.ibox[1]);
      dz -= a.box[2] * anint(dz * a.ibox[2]);
      const double dd2 = dx * dx + dy * dy + dz * dz;
      double cc = a.ccoef * qi * qj;
      e += cc * a.zb * dd2;
      cc *= a.zf;
      gx += dx * cc; gy += dy * cc; gz += dz * cc;
      atomicAdd(grad + 3 * j + 0, -dx * cc);
      atomicAdd(grad + 3 * j + 1, -dy * cc);
      atomicAdd(grad + 3 * j + 2, -dz * cc);
    }
    if (gx != 0.0 || gy != 0.0 || gz != 0.0) {
      atomicAdd(grad + 3 * i + 0, gx);
      atomicAdd(grad + 3 * i + 1, gy);
      atomicAdd(grad + 3 * i + 2, gz);
    }
    e += a.dself_coef * qi * qs;
  }
  warp_add(scr + 2, e);
}

// gradient and the two energies out of the scratch array
__global__ void __launch_bounds__(kNbThreads) k_nb_out(double* scr, int natom, double* grad,
                                                       double* ene) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  if (k < 3 * natom) {
    const double g = scr[kHdr + k];
    bad = !isfinite(g);
    grad[k] = g;
  }
  if (k == 0) {
    ene[0] = scr[0] + scr[2];
    ene[1] = scr[1];
    bad |= !isfinite(ene[0]) || !isfinite(ene[1]);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) set_status(scr, NB_NONFINITE);
}

// Set-up, once per device, with that device current: the address of this device's
// instance of g_nb_scratch and the device's SM count (the tile kernel's grid cap).
int scratch_of_current_device(double** out, int* nsm) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return JP_E_NO_DEVICE;
  if (dev < 0 || dev >= kMaxDevices) return JP_E_NO_DEVICE;
  double* p = g_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lk(g_mu);
    p = g_ptr[dev].load(std::memory_order_relaxed);
    if (!p) {
      void* sym = nullptr;
      if (cudaGetSymbolAddress(&sym, g_nb_scratch) != cudaSuccess || !sym) return JP_E_CUDA;
      if (reinterpret_cast<uintptr_t>(sym) % 256 != 0) return JP_E_CUDA;
      int sms = 0;
      if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return JP_E_CUDA;
      g_nsm[dev] = sms;
      p = static_cast<double*>(sym);
      g_ptr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  *nsm = g_nsm[dev];
  return JP_OK;
}

}  // namespace
}  // namespace jp

using namespace jp;

extern "C" int jp_nonbond_noalloc(int32_t natom, const double *cord, const double *charge,
                                  const int32_t *atype, int32_t ntype, const double *c6,
                                  const double *c12, const int32_t *excl_ptr,
                                  const int32_t *excl_idx, int32_t index_base,
                                  const double box[3], double cutoff, double dielectric,
                                  double *grad, double *ene, void *stream) {
  if (natom > JP_NOALLOC_MAX_ATOMS) return JP_E_NOALLOC_LIMIT;
  if (natom < 1 || ntype < 1 || (index_base != 0 && index_base != 1)) return JP_E_INVALID;
  if (!cord || !charge || !atype || !c6 || !c12 || !excl_ptr || !excl_idx || !box || !grad ||
      !ene)
    return JP_E_INVALID;
  if (!(cutoff > 0.0) || !(dielectric > 0.0)) return JP_E_INVALID;
  for (int k = 0; k < 3; ++k)   // one image within the cut-off
    if (!(box[k] > 2.0 * cutoff) || !std::isfinite(box[k])) return JP_E_INVALID;
  double* scr = nullptr;
  int nsm = 0;
  int rc = scratch_of_current_device(&scr, &nsm);
  if (rc != JP_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  NbArgs a;
  a.natom = natom; a.ntype = ntype; a.base = index_base;
  a.x = cord; a.q = charge; a.typ = atype; a.c6 = c6; a.c12 = c12;
  a.eptr = excl_ptr; a.eidx = excl_idx;
  for (int k = 0; k < 3; ++k) { a.box[k] = box[k]; a.ibox[k] = 1.0 / box[k]; }
  const double rc3 = cutoff * cutoff * cutoff;
  a.ccoef = 332.06378 / dielectric;             // inpcls.f90:215-227
  a.irc2 = 1.0 / (cutoff * cutoff);
  a.zb = 0.5 / rc3; a.zf = 1.0 / rc3; a.zc = 1.5 / cutoff;   // incel.f90:655-658
  a.dself_coef = -0.5 * a.zc * a.ccoef;

  if (cudaMemsetAsync(scr, 0, sizeof(double) * (kHdr + 3 * (size_t)natom), st) != cudaSuccess)
    return JP_E_CUDA;
  const int nb = (natom + 31) / 32;
  const long long warps = (long long)nb * nb;
  const int wpb = kNbThreads / 32;
  const int grid = (int)std::min<long long>((warps + wpb - 1) / wpb, (long long)nsm * 16);
  k_nb_tiles<<<grid, kNbThreads, 0, st>>>(scr, a);
  k_nb_excl<<<(natom + kNbThreads - 1) / kNbThreads, kNbThreads, 0, st>>>(scr, a);
  k_nb_out<<<(3 * natom + kNbThreads - 1) / kNbThreads, kNbThreads, 0, st>>>(scr, natom, grad, ene);
  if (cudaGetLastError() != cudaSuccess) return JP_E_CUDA;
  unsigned status = 0;
  if (cudaMemcpyAsync(&status, scr + 3, sizeof(unsigned), cudaMemcpyDeviceToHost, st) !=
          cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return JP_E_CUDA;
  if (status & NB_BAD_INDEX) return JP_E_INVALID;
  if (status & NB_NONFINITE) return JP_E_NONFINITE;
  return JP_OK;
}
