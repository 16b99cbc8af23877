// jp_minimize.cu -- steepest-descent minimisation (steep.f90 steep / linsrd) of all replicas.
//
// One iteration of linsrd per replica, every decision on the device so that iterations
// replay as a CUDA graph without a host round trip:
//   move    x <- x - stp g / |g|       (steep.f90:31 mksrdg, :128-131)   unless stopped
//   SHAKE   against the positions before the move (:118-150), then commit
//   dnergy  the usual force kernels
//   decide  E < E_old ? stp *= up : stp *= down, stop below 1e-10 A per degree of freedom
//           (:228-243); RMS gradient, stop at convgr (:28-35, calrsf.f90)
// State per replica in MinState; a replica that stopped keeps its positions.
#include "jp_kernels.h"

namespace jp {

constexpr int kMinThreads = 256;

__device__ __forceinline__ bool min_running(const MinState& M, int max_loop) {
  return M.state == 0 && M.iters < max_loop;
}

template <bool FP64>
__device__ __forceinline__ double grad_of(const DevPtrs& P, int i) {
  if (FP64) return P.grd[i];
  return (double)P.frc[i] * kFrcInv;
}

// sum |g|^2 per replica into gsum_new (warp-aggregated when a warp holds one replica)
template <bool FP64>
__global__ void __launch_bounds__(kMinThreads) k_min_gsum(DevPtrs P, int natom) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0;
  int r = 0;
  if (a < natom) {
    r = P.rep_of[a];
    for (int k = 0; k < 3; ++k) {
      const double g = grad_of<FP64>(P, 3 * a + k);
      s += g * g;
    }
  }
  const unsigned full = 0xffffffffu;
  const int r0 = __shfl_sync(full, r, 0);
  if (__all_sync(full, r == r0)) {
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(full, s, o);
    if ((threadIdx.x & 31) == 0 && s != 0.0) atomicAdd(&P.mins[r0].gsum_new, s);
  } else if (s != 0.0) {
    atomicAdd(&P.mins[r].gsum_new, s);
  }
}

// energies of the evaluation just done (eneval convention: dself in ELE15, total in 0)
__device__ __forceinline__ void min_energies(const DevPtrs& P, int r, double* e) {
  double tot = 0.0;
  for (int k = 1; k < JP_MAXENE; ++k) {
    e[k] = (double)P.ene_fix[r * 16 + k] * kEneInv;
    if (k == JP_E_ELE15) e[k] += P.reps[r].dself;
    tot += e[k];
  }
  e[0] = tot;
}

// the first evaluation (mini.f90 inimin): start values and the convergence check
__global__ void k_min_init(DevPtrs P, int nrep, double step0, double convgr) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrep) return;
  MinState& M = P.mins[r];
  const double n = (double)P.reps[r].natom;
  min_energies(P, r, M.ene);
  M.stp = step0 * sqrt(n);
  M.e_old = M.ene[0];
  M.gsum = M.gsum_new;
  M.gsum_new = 0.0;
  M.rmsf = sqrt(M.gsum / n);
  M.iters = 0;
  M.state = M.rmsf <= convgr ? 1 : 0;
}

// move along -g/|g|; with SHAKE the moved positions go to xback, the old ones to x0
template <bool FP64>
__global__ void __launch_bounds__(kMinThreads) k_min_move(DevPtrs P, int natom, int max_loop, int shake) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const MinState& M = P.mins[P.rep_of[a]];
  const bool go = *P.status == 0 && min_running(M, max_loop);
  const double f = go ? -M.stp / sqrt(M.gsum) : 0.0;
  for (int k = 0; k < 3; ++k) {
    const double x = P.x[3 * a + k];
    const double xn = x + f * grad_of<FP64>(P, 3 * a + k);
    if (shake) {
      P.x0[3 * a + k] = x;
      P.xback[3 * a + k] = xn;
    } else {
      P.x[3 * a + k] = xn;
    }
  }
}

// SHAKE's result becomes the positions of the replicas that moved
__global__ void __launch_bounds__(kMinThreads) k_min_commit(DevPtrs P, int natom, int max_loop) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  if (!min_running(P.mins[P.rep_of[a]], max_loop)) return;
  for (int k = 0; k < 3; ++k) P.x[3 * a + k] = P.xback[3 * a + k];
}

__global__ void k_min_decide(DevPtrs P, int nrep, int max_loop, double up, double down, double convgr) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= nrep) return;
  MinState& M = P.mins[r];
  const double gnew = M.gsum_new;
  M.gsum_new = 0.0;
  if (*P.status != 0 || !min_running(M, max_loop)) return;
  const double n = (double)P.reps[r].natom;
  M.iters += 1;
  min_energies(P, r, M.ene);
  if (M.ene[0] < M.e_old) {
    M.stp *= up;
  } else {
    M.stp *= down;
    if (M.stp / sqrt(3.0 * n) < 1.0e-10) M.state = 2;
  }
  M.e_old = M.ene[0];
  M.gsum = gnew;
  M.rmsf = sqrt(gnew / n);
  if (M.state == 0 && M.rmsf <= convgr) M.state = 1;
}

void launch_min_init(const DevPtrs& P, int natom, int nrep, bool fp64, double step0, double convgr,
                     cudaStream_t st) {
  const int nb = (natom + kMinThreads - 1) / kMinThreads;
  if (fp64) k_min_gsum<true><<<nb, kMinThreads, 0, st>>>(P, natom);
  else k_min_gsum<false><<<nb, kMinThreads, 0, st>>>(P, natom);
  k_min_init<<<(nrep + 63) / 64, 64, 0, st>>>(P, nrep, step0, convgr);
}

void launch_min_move(const DevPtrs& P, int natom, bool fp64, int max_loop, bool shake, cudaStream_t st) {
  const int nb = (natom + kMinThreads - 1) / kMinThreads;
  if (fp64) k_min_move<true><<<nb, kMinThreads, 0, st>>>(P, natom, max_loop, shake ? 1 : 0);
  else k_min_move<false><<<nb, kMinThreads, 0, st>>>(P, natom, max_loop, shake ? 1 : 0);
}

void launch_min_commit(const DevPtrs& P, int natom, int max_loop, cudaStream_t st) {
  k_min_commit<<<(natom + kMinThreads - 1) / kMinThreads, kMinThreads, 0, st>>>(P, natom, max_loop);
}

void launch_min_decide(const DevPtrs& P, int natom, int nrep, bool fp64, int max_loop, double up,
                       double down, double convgr, cudaStream_t st) {
  const int nb = (natom + kMinThreads - 1) / kMinThreads;
  if (fp64) k_min_gsum<true><<<nb, kMinThreads, 0, st>>>(P, natom);
  else k_min_gsum<false><<<nb, kMinThreads, 0, st>>>(P, natom);
  k_min_decide<<<(nrep + 63) / 64, 64, 0, st>>>(P, nrep, max_loop, up, down, convgr);
}

}  // namespace jp
