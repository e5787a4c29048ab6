// Eigenvalues of the symmetric tridiagonal matrix and the MBD energy
// (the eigenvalue half of PDSYEV('N','L') at UTILS.f90:835, energy at
// UTILS.f90:839-867).
//
// bisect_kernel: each eigenvalue by 9-way multisection (8 lanes evaluate 8
// shifts per step) on a division-free Sturm count -- the three-term
// determinant recurrence p_i = (d_i - x) p_{i-1} - e_{i-1}^2 p_{i-2} with
// power-of-two rescaling; the number of sign changes of p_0..p_n is the number
// of eigenvalues below x.  d and e^2 are staged in shared memory.
// energy_kernel: E = 0.5 sum_{lambda>=0} sqrt(lambda)/n_SL - 0.5 sum 3 omega
// with compensated (TwoSum) summation; NIMAG = #lambda<0.
#include <cuda_runtime.h>

#include "kernels.h"

namespace mbd {
namespace {

// Number of eigenvalues of the symmetric tridiagonal (d, e) below x; e2 = e^2.
// The three-term recurrence is homogeneous in (p, p_prev), so rescaling both
// by a power of two changes no sign and no count.  CHECK steps run between
// two magnitude checks; with CHECK = 4 a step's FMA is the only link of the
// dependency chain (the check and its branch sit on it once per 4 steps).
// One step grows max(|p|, |p_prev|) by at most G = |d_i - x| + e_{i-1}^2
// <= 2 tn + tn^2 (tn bounds |d|, |e| and the shifts); the caller takes
// CHECK = 4 only for tn < 2^32, where G^4 < 2^260: after a check the pair
// stays below 2^500 (or 2^523 scaled down to 2^23) and 4 steps keep it
// below 2^783.  Cancellation can shrink p by much more per step, but a tiny
// p only matters through its sign, which an FMA rounds correctly even below
// the normal range.
template <int CHECK>
__device__ __forceinline__ void sturm_rescale(double& p, double& pm) {
  const double big = 0x1p500, small = 0x1p-500;
  const double m = fmax(fabs(p), fabs(pm));
  if (m > big) {
    p *= small;
    pm *= small;
  } else if (m < small && m != 0.0) {
    p *= big;
    pm *= big;
  }
}

__device__ __forceinline__ void sturm_step(double di, double e2i, double x, double& p, double& pm, bool& neg,
                                           int& cnt) {
  const double pn = fma(di - x, p, -e2i * pm);
  const bool nn = (pn == 0.0) ? !neg : (pn < 0.0);
  cnt += (nn != neg);
  neg = nn;
  pm = p;
  p = pn;
}

template <int CHECK>
__device__ int sturm_count(const double* d, const double* e2, int n, double x) {
  double pm = 1.0;
  double p = d[0] - x;
  bool neg = (p <= 0.0);               // a zero takes the sign opposite to its predecessor (+1)
  int cnt = neg ? 1 : 0;
  int i = 1;
  for (; i + CHECK <= n; i += CHECK) {
#pragma unroll
    for (int u = 0; u < CHECK; ++u) sturm_step(d[i + u], e2[i + u - 1], x, p, pm, neg, cnt);
    sturm_rescale<CHECK>(p, pm);
  }
  for (; i < n; ++i) {
    sturm_step(d[i], e2[i - 1], x, p, pm, neg, cnt);
    sturm_rescale<1>(p, pm);
  }
  return cnt;
}

constexpr int kLanesPerEig = 8;

// blockDim 256: 32 eigenvalues per CTA, 8 lanes each.  sh = [d | e^2] when
// staged (n small enough for shared memory), else global memory is read.
__device__ __forceinline__ void bisect_block(const double* d, const double* e, const double* e2g, int n, int staged,
                                             double* ev, int block, double* sh) {
  const double* dd = d;
  const double* ee = e2g;
  if (staged) {
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      sh[i] = d[i];
      if (i < n - 1) sh[n + i] = e[i] * e[i];
    }
    dd = sh;
    ee = sh + n;
  }
  __syncthreads();
  // Gershgorin interval (every CTA computes it)
  __shared__ double s_lo[256], s_hi[256];
  double lo = 1e308, hi = -1e308;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double rad = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - rad);
    hi = fmax(hi, d[i] + rad);
  }
  s_lo[threadIdx.x] = lo;
  s_hi[threadIdx.x] = hi;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      s_lo[threadIdx.x] = fmin(s_lo[threadIdx.x], s_lo[threadIdx.x + h]);
      s_hi[threadIdx.x] = fmax(s_hi[threadIdx.x], s_hi[threadIdx.x + h]);
    }
    __syncthreads();
  }
  lo = s_lo[0];
  hi = s_hi[0];
  const double tn = fmax(fabs(lo), fabs(hi));
  lo -= 4.0 * 2.2e-16 * tn + 1e-300;
  hi += 4.0 * 2.2e-16 * tn + 1e-300;
  // |d_i - x| + e_{i-1}^2 <= 2 tn + tn^2 for every shift x in [lo, hi]
  const bool few_checks = tn < 0x1p32;
  const int gid = block * blockDim.x + threadIdx.x;
  const int k = gid / kLanesPerEig;
  const int q = gid % kLanesPerEig;
  const int lane = threadIdx.x % 32;
  const int base = lane & ~(kLanesPerEig - 1);
  const unsigned gmask = ((1u << kLanesPerEig) - 1u) << base;
  if (k >= n) return;   // whole lane groups leave together
  // invariant: count(lo) <= k < count(hi)
  for (int it = 0; it < 64; ++it) {
    const double wdt = hi - lo;
    if (wdt <= 2.0 * 1.1102230246251565e-16 * fmax(fabs(lo), fabs(hi))) break;
    const double x = lo + wdt * (double)(q + 1) / (double)(kLanesPerEig + 1);
    const bool above = (x > lo && x < hi) ? ((few_checks ? sturm_count<4>(dd, ee, n, x)
                                                         : sturm_count<1>(dd, ee, n, x)) > k)
                                          : (x >= hi);
    const unsigned bits = (__ballot_sync(gmask, above) & gmask) >> base;
    const double xprev = __shfl_up_sync(gmask, x, 1, kLanesPerEig);
    const int first = bits ? (__ffs(bits) - 1) : kLanesPerEig;
    // new interval (all 8 lanes compute the same)
    const double xs = __shfl_sync(gmask, x, base + min(first, kLanesPerEig - 1));
    const double xp = __shfl_sync(gmask, xprev, base + min(first, kLanesPerEig - 1));
    double nlo, nhi;
    if (first == kLanesPerEig) {
      nlo = xs;                    // x of lane 7
      nhi = hi;
    } else {
      nhi = xs;
      nlo = (first == 0) ? lo : xp;
    }
    if (!(nlo >= lo && nhi <= hi && nlo < nhi)) break;   // no progress possible
    lo = nlo;
    hi = nhi;
  }
  if (q == 0) ev[k] = 0.5 * (lo + hi);
}

__global__ void __launch_bounds__(256) bisect_kernel(const double* d, const double* e, const double* e2g, int n,
                                                     int staged, double* ev) {
  extern __shared__ double sh[];
  bisect_block(d, e, e2g, n, staged, ev, blockIdx.x, sh);
}

// blockIdx.y = job; blocks past a job's eigenvalues leave before any barrier.
__global__ void __launch_bounds__(256) bisect_batch_kernel(const EigJob* jobs) {
  extern __shared__ double sh[];
  const EigJob jb = jobs[blockIdx.y];
  if ((long long)blockIdx.x * blockDim.x >= (long long)jb.n * kLanesPerEig) return;
  bisect_block(jb.d, jb.e, nullptr, jb.n, 1, jb.ev, blockIdx.x, sh);
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& err) {
  s = a + b;
  const double bb = s - a;
  err = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ void energy_block(const double* ev, int n, int nsl, const double* scalars, double* out) {
  __shared__ double ss[1024], sc[1024];
  __shared__ int sn[1024];
  double s = 0.0, comp = 0.0;
  int neg = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double l = ev[k];
    if (l >= 0.0) {
      double t, e2;
      two_sum(s, sqrt(l), t, e2);
      s = t;
      comp += e2;
    } else {
      ++neg;
    }
  }
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = comp;
  sn[threadIdx.x] = neg;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) {
      double t, e2;
      two_sum(ss[threadIdx.x], ss[threadIdx.x + h], t, e2);
      ss[threadIdx.x] = t;
      sc[threadIdx.x] += sc[threadIdx.x + h] + e2;
      sn[threadIdx.x] += sn[threadIdx.x + h];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double e_int = ss[0] + sc[0];
    const double e_nonint = scalars[1];
    out[0] = (0.5 * e_int) / nsl - (0.5 * e_nonint);     // UTILS.f90:858
    out[1] = e_int;
    out[2] = (double)sn[0];
  }
}

__global__ void __launch_bounds__(1024) energy_kernel(const double* ev, int n, int nsl, const double* scalars,
                                                      double* out) {
  energy_block(ev, n, nsl, scalars, out);
}

__global__ void __launch_bounds__(1024) energy_batch_kernel(const EigJob* jobs) {
  const EigJob jb = jobs[blockIdx.x];
  energy_block(jb.ev, jb.n, jb.nsl, jb.scalars, jb.out);
}

__global__ void square_kernel(const double* e, double* e2, int m) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) e2[i] = e[i] * e[i];
}

}  // namespace

constexpr size_t kBisectMaxSmem = 200 * 1024;

static_assert(2 * sizeof(double) * kEigBatchMaxN <= kBisectMaxSmem, "batched bisection stages d and e^2");

cudaError_t init_eigval_attributes() {
  cudaError_t e = cudaFuncSetAttribute(bisect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBisectMaxSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(bisect_batch_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBisectMaxSmem);
}

// ev must hold 2n doubles: [0, n) eigenvalues, [n, 2n) scratch for e^2.
void launch_tridiag_eigenvalues(const double* d, const double* e, int n, double* ev, cudaStream_t s) {
  const size_t need = sizeof(double) * 2 * (size_t)n;
  const int staged = need <= kBisectMaxSmem;
  double* e2 = ev + n;
  if (!staged && n > 1) square_kernel<<<(n + 255) / 256, 256, 0, s>>>(e, e2, n - 1);
  const long long threads = (long long)n * kLanesPerEig;
  const int blocks = (int)((threads + 255) / 256);
  bisect_kernel<<<blocks, 256, staged ? need : 0, s>>>(d, e, e2, n, staged, ev);
}

// Same as launch_tridiag_eigenvalues with the e^2 scratch given separately
// (n doubles), so ev needs only n doubles.
void launch_tridiag_eigenvalues_scratch(const double* d, const double* e, int n, double* ev, double* e2,
                                        cudaStream_t s) {
  const size_t need = sizeof(double) * 2 * (size_t)n;
  const int staged = need <= kBisectMaxSmem;
  if (!staged && n > 1) square_kernel<<<(n + 255) / 256, 256, 0, s>>>(e, e2, n - 1);
  const long long threads = (long long)n * kLanesPerEig;
  const int blocks = (int)((threads + 255) / 256);
  bisect_kernel<<<blocks, 256, staged ? need : 0, s>>>(d, e, e2, n, staged, ev);
}

void launch_energy(const double* ev, int n, int nsl, const double* scalars, double* out, cudaStream_t s) {
  energy_kernel<<<1, 1024, 0, s>>>(ev, n, nsl, scalars, out);
}

void launch_eigen_batch(const EigJob* jobs_dev, int n_jobs, int max_n, cudaStream_t s) {
  if (n_jobs < 1 || max_n < 1) return;
  const long long threads = (long long)max_n * kLanesPerEig;
  const dim3 grid((unsigned)((threads + 255) / 256), (unsigned)n_jobs);
  bisect_batch_kernel<<<grid, 256, sizeof(double) * 2 * (size_t)max_n, s>>>(jobs_dev);
}

void launch_energy_batch(const EigJob* jobs_dev, int n_jobs, cudaStream_t s) {
  if (n_jobs < 1) return;
  energy_batch_kernel<<<n_jobs, 1024, 0, s>>>(jobs_dev);
}

}  // namespace mbd
