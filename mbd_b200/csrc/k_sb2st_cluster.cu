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
// and no block ever leaves shared memory.  The operations per entry are those
// of the flag-synchronised kernel, with sums taken in another order (below),
// so the two agree to rounding.
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

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// ---- arithmetic of one task ------------------------------------------------
// A task works with one warp per block, lane l holding row l of the block in
// registers (for the symmetric diagonal block only its lower triangle, which
// is band row l of the block).  Sums of 32 terms run as four interleaved
// partial sums (terms m mod 4 in partial m, combined as (s0 + s1) + (s2 + s3)):
// an FP64 FMA has a latency of about 13-23 cycles on B200, so a single
// 32-term chain would cost 400-700 cycles.  Sums across the lanes (a block's
// columns) go through shuffles, not through shared memory: reading a column
// of the band with one lane per row was measured several times slower than
// the arithmetic of the whole task.
namespace chase {

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

// sum_{j < 32} a(j) b(j) in four interleaved partial sums
template <class FA, class FB>
__device__ __forceinline__ double dot32(FA a, FB b) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
  for (int j = 0; j < B; j += 4) {
    s0 = fma(a(j), b(j), s0);
    s1 = fma(a(j + 1), b(j + 1), s1);
    s2 = fma(a(j + 2), b(j + 2), s2);
    s3 = fma(a(j + 3), b(j + 3), s3);
  }
  return (s0 + s1) + (s2 + s3);
}

// Householder reflector of x (lane l holds x[l], length len): H x = beta e_1,
// H = I - tau v v^T.  Returns tau; *v (lane l) with v[0] = 1; beta through
// *beta.  tau = 0 (H = I) when len < 2 or x[1 ..] = 0.
__device__ __forceinline__ double make_reflector(double x, int len, double* v, double* beta) {
  const int l = threadIdx.x & 31;
  const double xn2 = warp_sum((l >= 1 && l < len) ? x * x : 0.0);
  const double alpha = __shfl_sync(0xffffffffu, x, 0);
  double tau = 0.0, b = alpha, scale = 0.0;
  if (len >= 2 && xn2 > 0.0) {
    b = -copysign(sqrt(fma(alpha, alpha, xn2)), alpha);
    tau = (b - alpha) / b;
    scale = 1.0 / (alpha - b);
  }
  *v = (l == 0) ? 1.0 : ((l < len && tau != 0.0) ? x * scale : 0.0);
  *beta = b;
  return tau;
}

// D <- H D H on the lower triangle of D, held by diagonal offset: lane l has
// lo[m] = D(l, l - m) (0 for m > l), which is band row l of the block.  The
// upper half of (D v)_l, sum_{m >= 1} D(l + m, l) v(l + m), comes from the
// lanes below by shuffles (lane q sends D(q, q - m) v(q) to lane q - m), so
// no lane reads another lane's row: a walk down a column across the lanes
// made the shared-memory loads of a full row per lane several times slower
// than the whole update.  v(j) reads the reflector (any j in [0, 32)), vl =
// v(l); wsm: 32 doubles of this warp's shared memory.
template <class FV>
__device__ __forceinline__ void d_update_lower(double (&lo)[B], FV v, double vl, double tau, double* wsm) {
  const int l = threadIdx.x & 31;
  double s[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
  for (int m = 0; m < B; ++m) s[m & 3] = fma(lo[m], (m <= l) ? v(l - m) : 0.0, s[m & 3]);
#pragma unroll
  for (int m = 1; m < B; ++m) {
    const double u = __shfl_down_sync(0xffffffffu, lo[m] * vl, m);
    s[m & 3] += (l + m < B) ? u : 0.0;
  }
  const double dv = (s[0] + s[1]) + (s[2] + s[3]);
  const double vdv = warp_sum(vl * dv);
  const double wl = fma(tau, dv, -(0.5 * tau * tau * vdv * vl));
  wsm[l] = wl;
  __syncwarp();
#pragma unroll
  for (int m = 0; m < B; ++m)
    if (m <= l) lo[m] -= fma(vl, wsm[l - m], wl * v(l - m));
  __syncwarp();
}

// s_l = sum over the lanes q of c_q(l), where lane q supplies c(j) for every
// j (a butterfly reduce-scatter: five rounds of 16, 8, 4, 2, 1 shuffles, in
// each a lane keeps the half of its values whose index bit matches its own
// lane bit and adds the partner's copy of it).
template <class FC>
__device__ __forceinline__ double reduce_scatter32(FC c) {
  const int l = threadIdx.x & 31;
  double a16[16], a8[8], a4[4], a2[2];
  bool b = (l & 16) != 0;
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const double lo_ = c(p), hi_ = c(p + 16);
    a16[p] = (b ? hi_ : lo_) + __shfl_xor_sync(0xffffffffu, b ? lo_ : hi_, 16);
  }
  b = (l & 8) != 0;
#pragma unroll
  for (int p = 0; p < 8; ++p)
    a8[p] = (b ? a16[p + 8] : a16[p]) + __shfl_xor_sync(0xffffffffu, b ? a16[p] : a16[p + 8], 8);
  b = (l & 4) != 0;
#pragma unroll
  for (int p = 0; p < 4; ++p)
    a4[p] = (b ? a8[p + 4] : a8[p]) + __shfl_xor_sync(0xffffffffu, b ? a8[p] : a8[p + 4], 4);
  b = (l & 2) != 0;
#pragma unroll
  for (int p = 0; p < 2; ++p)
    a2[p] = (b ? a4[p + 2] : a4[p]) + __shfl_xor_sync(0xffffffffu, b ? a4[p] : a4[p + 2], 2);
  b = (l & 1) != 0;
  return (b ? a2[1] : a2[0]) + __shfl_xor_sync(0xffffffffu, b ? a2[0] : a2[1], 1);
}

// O <- H' O with H' = I - tau2 v2 v2^T for the block O held a row per lane
// (lane l: orow[j] = O(l, j), v2 = v2[l]): s = O^T v2 by a reduce-scatter
// across the lanes, then O -= (tau2 v2) s^T; O(., 0) becomes beta2 e_1.
// ssm: 32 doubles of this warp's shared memory.
__device__ __forceinline__ void o_left_rs(double (&orow)[B], double v2, double tau2, double beta2, double* ssm) {
  const int l = threadIdx.x & 31;
  const double sl = reduce_scatter32([&](int j) { return v2 * orow[j]; });
  ssm[l] = sl;
  __syncwarp();
  const double t = tau2 * v2;
#pragma unroll
  for (int j = 0; j < B; ++j) orow[j] = fma(-t, ssm[j], orow[j]);
  orow[0] = (l == 0) ? beta2 : 0.0;
  __syncwarp();
}

// O <- O H for the block O below D (lane l: orow[j] = O(l, j)).
template <class FV>
__device__ __forceinline__ void o_right(double (&orow)[B], FV v, double tau) {
  const double t = tau * dot32([&](int j) { return orow[j]; }, v);
#pragma unroll
  for (int j = 0; j < B; ++j) orow[j] = fma(-t, v(j), orow[j]);
}

}  // namespace chase

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

// One task (i, k) at step t on warp pair `pair`: the O-warp updates O and
// hands H' on, the D-warp updates D (and for k = 0 builds the next sweep's
// first reflector).
template <bool LOCAL>
__device__ __forceinline__ void chase_task(const Rows<LOCAL>& rm, int n, int r, int i, int k, int t, int R,
                                           double* refl, double* const* peer_refl, double* pv, double* pw,
                                           double* ps, int pair, bool owarp, int rank) {
  const int l = threadIdx.x & 31;
  const int L = min(B, n - r);
  const int rn = r + B;
  const int Ln = max(0, min(B, n - rn));
  // the task's reflector H (v, tau): from the slot of (step parity, sweep),
  // where the previous task of the sweep left it -- for k = 0 the D-warp of
  // task (i - 1, 0) two steps earlier, which also left beta (the reflector
  // of column i is known as soon as that task has updated the column)
  const double* vsrc = refl + ((t & 1) * kRing + (i % kRing)) * RSLOT;
  if (k == 0) {
    if (i == 0) {
      if (owarp) {
        // the first sweep's reflector from column 0: x[l] = A(r + l, 0), band
        // row r + l at d = l + 1
        double* xp = rm.row(l) + 1 + l;
        const double x = (l < L) ? *xp : 0.0;
        double vl, beta;
        const double tau0 = chase::make_reflector(x, L, &vl, &beta);
        if (l < L) *xp = (l == 0) ? beta : (tau0 != 0.0 ? 0.0 : x);
        pv[l] = vl;
        if (l == 0) pv[B] = tau0;
      }
      pair_sync(pair);
      vsrc = pv;
    } else if (owarp && vsrc[B] != 0.0 && l < L) {
      // column i <- beta e_1 (H x = beta e_1; with tau = 0 it stays as it is)
      rm.row(l)[1 + l] = (l == 0) ? vsrc[B + 1] : 0.0;
    }
  }
  // task (i, 0) builds the reflector of sweep i + 1 from column i + 1, which
  // it finishes: rows r + 1 .. r + 31 of it are column 0 of D (the D-warp's
  // registers after its update), row r + 32 is O(0, 0) = beta' of the O-warp
  const bool pre = (k == 0) && (i + 4 <= n);
  const int bar_beta = 7 + pair;   // named barrier of the O-warp -> D-warp hand-off of beta'
  const double tau = vsrc[B];
  if (!owarp) {
    // ---- D <- H D H:  w = tau D v - (tau^2 / 2)(v^T D v) v;  D -= v w^T + w v^T
    // on the lower triangle, lane l holding band row r + l: lo[m] = D(l, l - m)
    double lo[B];
    double* rowp = rm.row(l);
#pragma unroll
    for (int m = 0; m < B; ++m) lo[m] = (m <= l && l < L) ? rowp[m] : 0.0;
    if (tau != 0.0) {
      chase::d_update_lower(lo, [&](int j) { return vsrc[j]; }, vsrc[l], tau, pw);
      if (l < L) {
#pragma unroll
        for (int m = 0; m < B; ++m)
          if (m <= l) rowp[m] = lo[m];
      }
    }
    if (pre) {
      // x[l] = A(r + 1 + l, r) = D(l + 1, 0): band row r + 1 + l at d = l + 1
      // (as this warp just stored it), and for l = 31 O(0, 0) once the O-warp
      // has made its reflector
      __syncwarp();
      double x = (l + 1 < L) ? rm.row(l + 1)[l + 1] : 0.0;
      if (Ln > 0) {
        asm volatile("bar.sync %0, 64;" ::"r"(bar_beta) : "memory");
        if (l == B - 1) x = pv[B + 2];
      }
      const int Lx = min(B, n - r - 1);
      double vx, betax;
      const double taux = chase::make_reflector(x, Lx, &vx, &betax);
      // for task (i + 1, 0) at step t + 2 (same parity), in the CTA of row r + 1
      const int owner = (r + 1) / R;
      double* slot = (owner == rank ? refl : peer_refl[owner]) + ((t & 1) * kRing + ((i + 1) % kRing)) * RSLOT;
      slot[l] = vx;
      if (l == 0) {
        slot[B] = taux;
        slot[B + 1] = betax;
      }
    }
  } else {
    // ---- O <- O H;  H' from O[:, 0];  O <- H' O
    // orow[j] = O(l, j) = A(rn + l, r + j): band row rn + l at d = B + l - j
    double* orowp = rm.row(B + l) + B + l;
    double orow[B];
#pragma unroll
    for (int j = 0; j < B; ++j) orow[j] = (l < Ln && j < L) ? orowp[-j] : 0.0;
    if (tau != 0.0) chase::o_right(orow, [&](int j) { return vsrc[j]; }, tau);
    double v2 = 0.0, tau2 = 0.0, beta2 = 0.0;
    if (Ln > 0) {
      tau2 = chase::make_reflector(orow[0], Ln, &v2, &beta2);
      if (pre) {
        if (l == 0) pv[B + 2] = beta2;   // O(0, 0) after this task: beta2 (or alpha when tau2 = 0)
        asm volatile("bar.arrive %0, 64;" ::"r"(bar_beta) : "memory");
      }
      if (tau2 != 0.0) chase::o_left_rs(orow, v2, tau2, beta2, ps);
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
