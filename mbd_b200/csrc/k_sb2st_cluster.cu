// Band -> tridiagonal bulge chasing with the band held in the distributed
// shared memory of one thread-block cluster per matrix (the second stage of
// the two-stage reduction behind PDSYEV('N','L'), UTILS.f90:835), FP64.
//
// The sweeps and tasks are those of k_sb2st.cu: sweep i annihilates column i
// below the subdiagonal; its task k works on rows r = i + 1 + 32 k: the
// diagonal block D = A[r, r + 32)^2 (two-sided with the task's reflector H)
// and the block below it O = A[r + 32, r + 64) x [r, r + 32) (O <- O H, the
// next reflector H' from O's first column, O <- H' O).  Task (i, k) must
// follow tasks (i, k - 1) and (i - 1, k + 1).  Here every task runs at step
// t = 2 i + k: both predecessors run at step t - 1, and the tasks of one step
// touch disjoint entries (consecutive ones are 63 rows apart), so a cluster
// barrier between steps is the only synchronisation -- no flags, no polling,
// and no block ever leaves shared memory.  Per entry the operations and
// their order are those of the flag-synchronised kernel, so the two give the
// same band bit for bit.
//
// Layout: CTA c of a cluster of C holds band rows [c R, (c + 1) R), R =
// ceil(n / C), row q at band[(q - c R) * SLD + d] = A(q, q - d), d = 0 .. 64.
// A block that straddles two CTAs is read and written through the cluster
// window (map_shared_rank).  SLD = 66 makes the per-lane row walks (stride
// SLD + 1 = 67 doubles) and column walks (stride 1) free of bank conflicts.
// A task runs on a warp pair of the CTA holding its row r (owner computes):
// the D-warp updates D, the O-warp O; the O-warp hands H' to the CTA holding
// row r + 32 (the next task's owner) through a ring of reflector slots
// indexed by (step parity, sweep mod 16).  R <= 6 * 63 keeps the tasks of a
// CTA in one step within its 6 warp pairs.
//
// Clusters are persistent over the batch's matrices (largest first); the
// band never returns to global memory, only d and e do.  Matrices larger
// than C_max * R_max rows take the flag-synchronised kernel (k_sb2st.cu).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace mbd {
namespace {

constexpr int B = kBand;                      // 32
constexpr int SLD = 66;                       // shared band row stride (doubles)
constexpr int PAIRS = 6;
constexpr int THREADS = PAIRS * 64;
constexpr int kMaxRows = PAIRS * (2 * B - 1);   // 378: at most PAIRS tasks per CTA and step
constexpr int kMaxCluster = 16;
constexpr int RSLOT = B + 8;                  // v[32], tau, padding
constexpr int kRing = 16;                     // reflector slots, by sweep mod 16

size_t smem_bytes(int R) {
  return sizeof(double) * ((size_t)R * SLD + 2 * kRing * RSLOT + (size_t)PAIRS * (RSLOT + 2 * B));
}

__device__ __forceinline__ void pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(pair + 1) : "memory");
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// Householder reflector of x (lane l holds x[l], length len): H x = beta e_1
// (the same arithmetic as k_sb2st.cu).  Returns tau; v (lane l) with v[0] = 1.
__device__ __forceinline__ double make_reflector(double x, int len, double* v, double* beta) {
  const int l = threadIdx.x & 31;
  const double xn2 = warp_sum((l >= 1 && l < len) ? x * x : 0.0);
  const double alpha = __shfl_sync(0xffffffffu, x, 0);
  double tau = 0.0, b = alpha, scale = 0.0;
  if (len >= 2 && xn2 > 0.0) {
    b = -copysign(sqrt(alpha * alpha + xn2), alpha);
    tau = (b - alpha) / b;
    scale = 1.0 / (alpha - b);
  }
  *v = (l == 0) ? 1.0 : ((l < len && tau != 0.0) ? x * scale : 0.0);
  *beta = b;
  return tau;
}

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// Rows [r, r + 64) of a task, r in this CTA: row r + q is at base0 + q SLD
// (this CTA's shared memory) while q < lim, in the next CTA at
// base1 + (q - lim) SLD after.  LOCAL: every row the task touches is here, so
// all accesses are plain shared-memory ones (the cluster window is only taken
// by the few tasks that straddle two CTAs).
template <bool LOCAL>
struct Rows {
  double* base0;
  double* base1;
  int lim;
  __device__ __forceinline__ double* row(int q) const {
    if (LOCAL) return base0 + q * SLD;
    return (q < lim) ? base0 + q * SLD : base1 + (q - lim) * SLD;
  }
};

// One task (i, k) at step t on warp pair `pair`: the O-warp builds the
// reflector (k = 0), updates O and hands H' on; the D-warp updates D.
template <bool LOCAL>
__device__ __forceinline__ void chase_task(const Rows<LOCAL>& rm, int n, int r, int i, int k, int t, int R,
                                           double* refl, double* const* peer_refl, double* pv, double* pw,
                                           double* ps, int pair, bool owarp, int rank) {
  const int l = threadIdx.x & 31;
  const int L = min(B, n - r);
  const int rn = r + B;
  const int Ln = max(0, min(B, n - rn));
  // the task's reflector H (v, tau)
  const double* vsrc;
  if (k == 0) {
    if (owarp) {
      // from column i: x[l] = A(r + l, i), band row r + l at d = l + 1
      double* xp = rm.row(l) + 1 + l;
      const double x = (l < L) ? *xp : 0.0;
      double vl, beta;
      const double tau0 = make_reflector(x, L, &vl, &beta);
      if (l < L) *xp = (l == 0) ? beta : (tau0 != 0.0 ? 0.0 : x);
      pv[l] = vl;
      if (l == 0) pv[B] = tau0;
    }
    pair_sync(pair);
    vsrc = pv;
  } else {
    vsrc = refl + ((t & 1) * kRing + (i % kRing)) * RSLOT;
  }
  const double tau = vsrc[B];
  if (!owarp) {
    // ---- D <- H D H:  w = tau D v - (tau^2 / 2)(v^T D v) v;  D -= v w^T + w v^T
    double dr[B];   // dr[j] = D(l, j)
#pragma unroll
    for (int j = 0; j < B; ++j) {
      const int q = (j <= l) ? l : j;
      dr[j] = (q < L) ? rm.row(q)[(j <= l) ? l - j : j - l] : 0.0;
    }
    if (tau != 0.0) {
      const double vlD = vsrc[l];
      double dv = 0.0;
#pragma unroll
      for (int j = 0; j < B; ++j) dv += dr[j] * vsrc[j];
      const double vdv = warp_sum(vlD * dv);
      const double wl = tau * dv - 0.5 * tau * tau * vdv * vlD;
      pw[l] = wl;
      __syncwarp();
#pragma unroll
      for (int j = 0; j < B; ++j) dr[j] -= vlD * pw[j] + wl * vsrc[j];
      if (l < L) {
        double* own = rm.row(l);
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (j <= l) own[l - j] = dr[j];
      }
    }
  } else {
    // ---- O <- O H;  H' from O[:, 0];  O <- H' O
    // orow[j] = O(l, j) = A(rn + l, r + j): band row rn + l at d = B + l - j
    double* orowp = rm.row(B + l) + B + l;
    double orow[B];
#pragma unroll
    for (int j = 0; j < B; ++j) orow[j] = (l < Ln && j < L) ? orowp[-j] : 0.0;
    if (tau != 0.0) {
      double ov = 0.0;
#pragma unroll
      for (int j = 0; j < B; ++j) ov += orow[j] * vsrc[j];
#pragma unroll
      for (int j = 0; j < B; ++j) orow[j] -= tau * ov * vsrc[j];
    }
    double v2 = 0.0, tau2 = 0.0, beta2 = 0.0;
    if (Ln > 0) {
      tau2 = make_reflector(orow[0], Ln, &v2, &beta2);
      if (tau2 != 0.0) {
        // column sums s_l = sum_q v2[q] O(q, l): the rows go to the band
        // first, then lane l walks column l
        if (l < Ln) {
#pragma unroll
          for (int j = 0; j < B; ++j)
            if (j < L) orowp[-j] = orow[j];
        }
        ps[l] = v2;
        __syncwarp();
        double sj = 0.0;
#pragma unroll
        for (int q = 0; q < B; ++q) {
          const double oql = (q < Ln && l < L) ? rm.row(B + q)[B + q - l] : 0.0;
          sj += ps[q] * oql;
        }
        __syncwarp();
        ps[l] = sj;
        __syncwarp();
#pragma unroll
        for (int j = 0; j < B; ++j) orow[j] -= tau2 * v2 * ps[j];
        orow[0] = (l == 0) ? beta2 : 0.0;
      }
      if (l < Ln) {
#pragma unroll
        for (int j = 0; j < B; ++j)
          if (j < L) orowp[-j] = orow[j];
      }
      // H' to the owner of row rn, for task (i, k + 1) at step t + 1 (through
      // the cluster window only when that is another CTA)
      const int owner = rn / R;
      double* slot = (owner == rank ? refl : peer_refl[owner]) + ((((t + 1) & 1) * kRing) + (i % kRing)) * RSLOT;
      slot[l] = v2;
      if (l == 0) slot[B] = tau2;
    }
  }
}

__global__ void __launch_bounds__(THREADS, 1) sb2st_cluster_kernel(const BandJob* jobs, int n_jobs, int rmax) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double* peer_band[kMaxCluster];
  __shared__ double* peer_refl[kMaxCluster];
  cg::cluster_group cl = cg::this_cluster();
  const int C = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int tid = threadIdx.x, warp = tid >> 5;
  const int pair = warp >> 1;
  const bool owarp = (warp & 1) != 0;
  double* band = sm;
  double* refl = sm + (size_t)rmax * SLD;          // [2][kRing][RSLOT]
  double* pv = refl + 2 * kRing * RSLOT + pair * (RSLOT + 2 * B);   // this pair: k = 0 reflector
  double* pw = pv + RSLOT;                         // D-warp: w
  double* ps = pw + B;                             // O-warp: column sums / v2
  if (tid < C) {
    peer_band[tid] = cl.map_shared_rank(band, tid);
    peer_refl[tid] = cl.map_shared_rank(refl, tid);
  }
  __syncthreads();
  const int cid = blockIdx.x / C, ncl = gridDim.x / C;
  for (int job = cid; job < n_jobs; job += ncl) {
    const BandJob jb = jobs[job];
    const int n = jb.n;
    // CTAs used for this matrix: at least 64 rows each, so that the rows
    // [r, r + 64) of a task lie in at most two CTAs
    const int Cj = min(C, max(1, n / (2 * B)));
    const int R = (n + Cj - 1) / Cj;
    const int lo = min(n, rank * R), hi = min(n, lo + R);
    {
      const int cnt = (hi - lo) * kBandLd;
      const double* src = jb.Br + (size_t)lo * kBandLd;
      for (int e = tid; e < cnt; e += THREADS) {
        const int q = e / kBandLd;
        band[q * SLD + (e - q * kBandLd)] = __ldcg(src + e);
      }
    }
    cl.sync();
    double* next_band = peer_band[min(rank + 1, C - 1)];
    const int tmax = 2 * (n - 3);
    for (int t = 0; t <= tmax; ++t) {
      // this CTA's tasks at step t: r = 32 t + 1 - 63 i in [lo, hi); pair p
      // takes the p-th largest sweep index
      const int i = floor_div(32 * t + 1 - lo, 2 * B - 1) - pair;
      const int r = 32 * t + 1 - (2 * B - 1) * i;
      const int k = t - 2 * i;
      if (i >= 0 && k >= 0 && r < hi && r < n) {
        if (min(n, r + 2 * B) <= hi) {
          const Rows<true> rm{band + (r - lo) * SLD, nullptr, 0};
          chase_task(rm, n, r, i, k, t, R, refl, peer_refl, pv, pw, ps, pair, owarp, rank);
        } else {
          const Rows<false> rm{band + (r - lo) * SLD, next_band, hi - r};
          chase_task(rm, n, r, i, k, t, R, refl, peer_refl, pv, pw, ps, pair, owarp, rank);
        }
      }
      cl.sync();
    }
    // d[q] = A(q, q), e[q - 1] = A(q, q - 1) of this CTA's rows
    for (int q = lo + tid; q < hi; q += THREADS) {
      jb.d[q] = band[(q - lo) * SLD];
      if (q >= 1) jb.e[q - 1] = band[(q - lo) * SLD + 1];
    }
    cl.sync();
  }
}

// Largest cluster this device can run the kernel with (0: none), probed once.
int g_cmax = -1;

int probe_cmax() {
  if (g_cmax >= 0) return g_cmax;
  g_cmax = 0;
  if (cudaFuncSetAttribute(sb2st_cluster_kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess ||
      cudaFuncSetAttribute(sb2st_cluster_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem_bytes(kMaxRows)) != cudaSuccess) {
    cudaGetLastError();
    return g_cmax;
  }
  for (int C = kMaxCluster; C >= 1; --C) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(THREADS);
    cfg.dynamicSmemBytes = smem_bytes(kMaxRows);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, sb2st_cluster_kernel, &cfg) == cudaSuccess && clusters >= 1) {
      g_cmax = C;
      break;
    }
    cudaGetLastError();
  }
  return g_cmax;
}

}  // namespace

int sb2st_cluster_max_n() { return probe_cmax() * kMaxRows; }

int sb2st_cluster_cmax() { return probe_cmax(); }

int sb2st_cluster_min(int n) { return std::max(1, (n + kMaxRows - 1) / kMaxRows); }

int sb2st_cluster_size(int max_n, int n_jobs, int num_sms, int want_c) {
  const int cmax = probe_cmax();
  if (cmax < 1 || max_n > cmax * kMaxRows) return 0;
  const int cmin = sb2st_cluster_min(max_n);
  // at most 64 rows per CTA of the largest matrix and no more clusters' worth
  // of CTAs than the SMs can hold for the batch
  const int chi = std::max(cmin, std::min({cmax, std::max(1, num_sms / std::max(1, n_jobs)),
                                            std::max(1, max_n / (2 * B))}));
  if (want_c > 0) return std::max(cmin, std::min(want_c, chi));
  // default: spare SMs go to wider clusters (fewer tasks per CTA and step)
  return chi;
}

cudaError_t launch_sb2st_cluster(const BandJob* jobs, int n_jobs, int max_n, int C, cudaStream_t s) {
  if (n_jobs < 1) return cudaSuccess;
  if (C < 1 || max_n > C * kMaxRows) return cudaErrorInvalidValue;
  // rows per CTA: ceil(n / C) for the matrices that use the whole cluster,
  // below 128 for those that use fewer CTAs (n / 64 of them)
  const int rmax = std::min(kMaxRows, std::max((max_n + C - 1) / C, 2 * 2 * B));
  cudaLaunchConfig_t cfg{};
  cfg.blockDim = dim3(THREADS);
  cfg.dynamicSmemBytes = smem_bytes(rmax);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  cfg.gridDim = dim3(C);
  int clusters = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&clusters, sb2st_cluster_kernel, &cfg);
  if (e != cudaSuccess) return e;
  const int Q = std::max(1, std::min(n_jobs, clusters));
  cfg.gridDim = dim3(Q * C);
  return cudaLaunchKernelEx(&cfg, sb2st_cluster_kernel, jobs, n_jobs, rmax);
}

}  // namespace mbd
