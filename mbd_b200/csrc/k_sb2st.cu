// Stage 2 of the two-stage tridiagonalisation: symmetric band (half-bandwidth
// kBand) -> tridiagonal by bulge chasing with Householder reflectors of
// length kBand, FP64, for every band of a batch in ONE persistent
// cooperative launch.
//
// Band storage per matrix: Br[r][d] = A(r, r - d), d = 0 .. 2 kBand; the
// diagonals beyond kBand hold the bulges between sweeps.  Sweep i annihilates
// column i below the subdiagonal; its task k (rows r_k = i + 1 + k kBand):
//   k = 0: reflector H from column i (A(r_0 .. r_0 + kBand, i)).
//   D_k <- H D_k H            (diagonal block, rows/cols [r_k, r_k + kBand))
//   O   <- O H                (O = A[r_k + kBand .. + kBand, r_k .. + kBand))
//   H'  from O[:, 0];  O <- H' O;  carry H' to task k + 1.
// Task (i, k) touches columns [r_k, r_k + kBand) and must follow task
// (i-1, k+1), the last task of the previous sweep that touches one of them.
// Of that task it needs only the diagonal block (its D(0,0) is the last
// diagonal entry of (i, k)'s D block, its column 0 the last column of
// (i, k)'s O block) and the corner O(0,0) of its O block (the last entry of
// (i, k)'s O block): every other entry the two tasks touch is disjoint.  So
// each sweep publishes two counts: one when its D-warp has stored a task's D
// block, one as soon as its O-warp has the next reflector's beta and has
// stored it as O(0,0) (the rest of the O block, which (i, k) does not touch,
// is stored later).  The two counts share one 64-bit word per sweep item
// (D-warp count in the low half, O-warp count in the high half, each
// advanced by a release add), so the next sweep's O-warp polls a single word
// (bounded) until both halves reach k + 2; its D-warp follows through the
// pair barrier.  Earlier tasks of sweep i-1 are complete by then: task k + 1
// started after the pair barrier that closed task k.
//
// Work items are (matrix, sweep) pairs ordered by sweep, then matrix; warp w
// takes items w, w + W, ...  Every wait points to an item of lower index, so
// the lowest unfinished item always progresses (all CTAs are co-resident).
// Lane l of a warp holds row l of D (D-warp) or of O (O-warp) in registers;
// the blocks move between the band and shared memory a band row per load or
// store instruction (coalesced), and between shared memory and registers a
// matrix row per lane.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "wait_limit.cuh"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int B = kBand;
constexpr int LD = kBandLd;
constexpr int WARPS = 4;

// Shared memory of one warp pair (one sweep item): the reflector of the
// current and of the next task (double-buffered by task parity), D-warp and
// O-warp scratch.
struct PairSmem {
  double v[2][B];
  double w[B];
  double s[B];
  double Ot[B][B + 1];   // O-warp: the O block, row-major (row l at Ot[l])
  double Ds[B][B];       // D-warp: band rows of D, Ds[i][d] = A(r + i, r + i - d)
  int go;             // the O-warp's decision after its wait, read by both warps
};

__device__ __forceinline__ void pair_sync(int pair) {
  asm volatile("bar.sync %0, 64;" ::"r"(pair + 1) : "memory");
}

__device__ __forceinline__ double warp_sum(double x) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
  return x;
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// one published count (low half: D-warp, high half: O-warp)
__device__ __forceinline__ void add_release(unsigned long long* p, unsigned long long v) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
constexpr unsigned long long kCountD = 1ull, kCountO = 1ull << 32;

__device__ __forceinline__ int both_counts(unsigned long long v) {
  return min((int)(unsigned)(v & 0xffffffffull), (int)(unsigned)(v >> 32));
}

// Lane 0 spins (bounded) with acquire loads until both counts of *p reach
// target; the warp barrier after it orders every lane's later reads behind
// that acquire (a second acquire load by every lane would add an L2 round
// trip to each link of the sweep-to-sweep chain).
__device__ bool wait_progress(const unsigned long long* p, int target, int* err) {
  int ok = 1;
  if ((threadIdx.x & 31) == 0) {
    // tight polling first (the predecessor is usually one task away), then
    // exponential back-off so that far-behind warps do not load the L2; the
    // error flag and the clock are read every 64 polls (an extra load per poll
    // would sit behind the acquire and double the detection latency)
    const long long lim = wait_limit_cycles();
    const long long t0 = clock64();
    unsigned ns = 0, polls = 0;
    while (both_counts(ld_acquire(p)) < target) {
      if ((++polls & 63u) == 0) {
        if (*(volatile int*)err != 0 || clock64() - t0 > lim) {
          atomicCAS(err, 0, MBD_ERR_TIMEOUT);
          ok = 0;
          break;
        }
      }
      if (polls > 256) {
        __nanosleep(ns);
        ns = min(2 * ns + 16, 256u);
      }
    }
  }
  ok = __shfl_sync(0xffffffffu, ok, 0);
  __syncwarp();
  return ok != 0;
}

// Householder reflector of x (lane l holds x[l], length len): H x = beta e_1.
// Returns tau; v[l] (lane l) with v[0] = 1; beta through *beta.
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

// Warp pair p of a CTA owns one sweep item at a time: warp 2p updates the
// diagonal block D two-sided, warp 2p + 1 the block O below it (right apply,
// next reflector, left apply); they meet at a named barrier once per task.
constexpr int PAIRS = WARPS / 2;
__global__ void __launch_bounds__(WARPS * 32) sb2st_kernel(const BandJob* jobs, const SweepItem* items,
                                                           int n_items, unsigned long long* progress, int* err,
                                                           int stall_item) {
  __shared__ PairSmem psm[PAIRS];
  const int warp = threadIdx.x / 32, l = threadIdx.x & 31;
  const int pair = warp / 2;
  const bool owarp = (warp & 1) != 0;
  PairSmem& S = psm[pair];
  const int W = gridDim.x * PAIRS;
  for (int t = blockIdx.x * PAIRS + pair; t < n_items; t += W) {
    const SweepItem it = items[t];
    const BandJob jb = jobs[it.job];
    const int n = jb.n, i = it.sweep;
    double* Br = jb.Br;
    const int K = (n - i - 1 + B - 1) / B;           // tasks of sweep i
    const int Kp = (n - i + B - 1) / B;              // tasks of sweep i - 1
    double tau = 0.0, vl = 0.0;                      // current reflector (O-warp registers)
    // D-warp: rows 0 .. B-2 of the next task's D block go into S.Ds during
    // this task, once the D-warp has stored and published (the D-warp waits
    // for the O-warp at the end of a task anyway); the next task then loads
    // only its last row after its wait
    bool have_pf = false;
    for (int k = 0; k < K; ++k) {
      // the O-warp waits for the previous sweep and decides for the pair; the
      // D-warp follows it through the barrier (one decision, both warps leave
      // together)
      if (owarp) {
        bool ok;
        if (t == stall_item && k == 0)   // a count nothing reaches: the wait runs out
          ok = wait_progress(progress + t, 1 << 30, err);
        else
          ok = it.pred < 0 || wait_progress(progress + it.pred, min(k + 2, Kp), err);
        if (l == 0) S.go = ok;
      }
      pair_sync(pair);
      if (!S.go) return;
      const int r = i + 1 + k * B;
      const int L = min(B, n - r);
      const int rn = r + B;
      const int Ln = max(0, min(B, n - rn));
      double* vcur = S.v[k & 1];
      if (k == 0) {
        if (owarp) {
          // reflector from column i: x[l] = A(i + 1 + l, i) = Br[i + 1 + l][1 + l]
          const double x = (l < L) ? __ldcg(Br + (size_t)(r + l) * LD + 1 + l) : 0.0;
          double beta;
          tau = make_reflector(x, L, &vl, &beta);
          if (l < L) Br[(size_t)(r + l) * LD + 1 + l] = (l == 0) ? beta : (tau != 0.0 ? 0.0 : x);
          vcur[l] = vl;
          S.w[0] = tau;   // tau for the D-warp (S.w is free before its first use)
        }
        pair_sync(pair);
      }
      if (!owarp) {
        // ---- D <- H D H:  w = tau D v - (tau^2 / 2)(v^T D v) v;  D -= v w^T + w v^T
        const double tauD = (k == 0) ? S.w[0] : S.w[1];
        __syncwarp();
        // band rows r .. r + L - 1, diagonals d <= row (the lower triangle of D)
        const double* rowsD = Br + (size_t)r * LD + l;
        if (have_pf) {
          S.Ds[B - 1][l] = (B - 1 < L) ? __ldcg(rowsD + (size_t)(B - 1) * LD) : 0.0;
        } else {
#pragma unroll
          for (int i = 0; i < B; ++i) S.Ds[i][l] = (i < L && l <= i) ? __ldcg(rowsD + (size_t)i * LD) : 0.0;
        }
        __syncwarp();
        double dr[B];   // dr[j] = D(l, j): Ds[l][l - j] below the diagonal, Ds[j][j - l] above
        const double* ds = &S.Ds[0][0];
#pragma unroll
        for (int j = 0; j < B; ++j) dr[j] = ds[(j <= l) ? (B + 1) * l - j : (B + 1) * j - l];
        if (tauD != 0.0) {
          const double vlD = vcur[l];
          double dv = 0.0;
#pragma unroll
          for (int j = 0; j < B; ++j) dv += dr[j] * vcur[j];
          const double vdv = warp_sum(vlD * dv);
          const double wl = tauD * dv - 0.5 * tauD * tauD * vdv * vlD;
          __syncwarp();
          S.w[l] = wl;
          __syncwarp();
#pragma unroll
          for (int j = 0; j < B; ++j) dr[j] -= vlD * S.w[j] + wl * vcur[j];
#pragma unroll
          for (int j = 0; j < B; ++j)
            if (j <= l) S.Ds[l][l - j] = dr[j];
          __syncwarp();
          double* rowsW = Br + (size_t)r * LD + l;
#pragma unroll
          for (int i = 0; i < B; ++i)
            if (i < L && l <= i) rowsW[(size_t)i * LD] = S.Ds[i][l];
        }
        // the warp barrier orders every lane's stores before lane 0's release
        __syncwarp();
        if (l == 0) add_release(progress + t, kCountD);
        // rows 0 .. B-2 of the next task's D block: global rows [r + B,
        // r + 2B - 1), all inside the D block of the previous sweep's task
        // k + 1 (published: this task waited for its D count), touched by no
        // task that runs before the next one
        // (lane l reads and writes only column l of S.Ds here, after its last
        // read of this task's block)
        have_pf = k + 1 < K;
        if (have_pf) {
          const int L1 = min(B, n - rn);
          const double* rows1 = Br + (size_t)rn * LD + l;
#pragma unroll
          for (int i = 0; i < B - 1; ++i) S.Ds[i][l] = (i < L1 && l <= i) ? __ldcg(rows1 + (size_t)i * LD) : 0.0;
        }
      } else {
        // ---- O <- O H;  next reflector from O[:, 0];  O <- H' O
        // band row rn + q holds O(q, j) at diagonal B + q - j: lane l reads j = B - 1 - l
        const double* rowsO = Br + (size_t)rn * LD + 1 + l;
        const bool jin = (B - 1 - l) < L;
#pragma unroll
        for (int q = 0; q < B; ++q)
          S.Ot[q][B - 1 - l] = (q < Ln && jin) ? __ldcg(rowsO + (size_t)q * (LD + 1)) : 0.0;
        __syncwarp();
        double orow[B];
#pragma unroll
        for (int j = 0; j < B; ++j) orow[j] = S.Ot[l][j];
        __syncwarp();
        if (tau != 0.0) {
          double ov = 0.0;
#pragma unroll
          for (int j = 0; j < B; ++j) ov += orow[j] * vcur[j];
#pragma unroll
          for (int j = 0; j < B; ++j) orow[j] -= tau * ov * vcur[j];
        }
        double v2 = 0.0, tau2 = 0.0, beta2 = 0.0;
        if (Ln > 0) {
          tau2 = make_reflector(orow[0], Ln, &v2, &beta2);
          // O(0,0) is final now (beta2; the entry itself when there is no
          // reflection): store it and publish it for the next sweep
          if (l == 0) {
            Br[(size_t)rn * LD + B] = beta2;
            add_release(progress + t, kCountO);
          }
          if (tau2 != 0.0) {
#pragma unroll
            for (int j = 0; j < B; ++j) S.Ot[l][j] = orow[j];
            S.v[(k + 1) & 1][l] = v2;
            __syncwarp();
            double sj = 0.0;
#pragma unroll
            for (int q = 0; q < B; ++q) sj += S.v[(k + 1) & 1][q] * S.Ot[q][l];   // column l of v2^T O
            __syncwarp();
            S.s[l] = sj;
            __syncwarp();
#pragma unroll
            for (int j = 0; j < B; ++j) orow[j] -= tau2 * v2 * S.s[j];
            orow[0] = (l == 0) ? beta2 : 0.0;
          }
          // the rows of O back to the band
#pragma unroll
          for (int j = 0; j < B; ++j) S.Ot[l][j] = orow[j];
          __syncwarp();
          double* rowsOW = Br + (size_t)rn * LD + 1 + l;
#pragma unroll
          for (int q = 0; q < B; ++q)   // O(0,0) (q = 0, lane B - 1) is stored already
            if (q < Ln && jin && (q > 0 || l != B - 1)) rowsOW[(size_t)q * (LD + 1)] = S.Ot[q][B - 1 - l];
        } else if (l == 0) {
          add_release(progress + t, kCountO);   // no O block
        }
        S.v[(k + 1) & 1][l] = v2;
        tau = tau2;
        vl = v2;
      }
      // Publication is a release store at GPU scope by one lane, cumulative
      // over the writes a barrier ordered before it (no separate fence: a
      // __threadfence() cost ~7 % of the launch).  The barrier below closes
      // the task for the pair (the next task's first barrier orders S.w[1]
      // before the D-warp reads it).
      pair_sync(pair);
      if (owarp && l == 0) S.w[1] = tau;   // the next task's tau for the D-warp
    }
  }
}

// d[r] = A(r, r), e[r] = A(r + 1, r) after the last sweep
__global__ void extract_kernel(const BandJob* jobs) {
  const BandJob jb = jobs[blockIdx.y];
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= jb.n) return;
  jb.d[r] = jb.Br[(size_t)r * LD];
  if (r + 1 < jb.n) jb.e[r] = jb.Br[(size_t)(r + 1) * LD + 1];
}

}  // namespace

cudaError_t init_sb2st_attributes() { return cudaSuccess; }

int sb2st_max_ctas(int num_sms) {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, sb2st_kernel, WARPS * 32, 0) != cudaSuccess || nb < 1)
    nb = 1;
  return nb * num_sms;
}

cudaError_t launch_sb2st(const BandJob* jobs, int n_jobs, const SweepItem* items, int n_items, int* progress,
                         int* err, int num_sms, int max_n, long long sweeps_in_flight, int stall_item,
                         cudaStream_t s) {
  if (n_jobs < 1) return cudaSuccess;
  if (n_items > 0) {
    cudaError_t e = cudaMemsetAsync(progress, 0, 2 * sizeof(int) * (size_t)n_items, s);
    if (e != cudaSuccess) return e;
    // workers: about three times the sweeps that can be in flight at once (a
    // matrix keeps about n / (2 kBand) sweeps busy), within co-residency
    int grid = sb2st_max_ctas(num_sms);
    const long long want_pairs = 3LL * sweeps_in_flight + 4 * PAIRS;
    const int need = (int)((std::min<long long>(want_pairs, n_items) + PAIRS - 1) / PAIRS);
    if (grid > need) grid = need;
    unsigned long long* prog64 = reinterpret_cast<unsigned long long*>(progress);
    void* args[] = {(void*)&jobs, (void*)&items, (void*)&n_items, (void*)&prog64, (void*)&err, (void*)&stall_item};
    e = cudaLaunchCooperativeKernel((const void*)sb2st_kernel, dim3(grid), dim3(WARPS * 32), args, 0, s);
    if (e != cudaSuccess) return e;
  }
  extract_kernel<<<dim3((max_n + 255) / 256, n_jobs), 256, 0, s>>>(jobs);
  return cudaGetLastError();
}

MBD_WAIT_LIMIT_SETTER(set_wait_limit_sb2st)

}  // namespace mbd
