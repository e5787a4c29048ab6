// Eigenvectors of a real symmetric matrix (JOBZ = 'V' of the PDSYEV call at
// UTILS.f90:835, which the reference makes with JOBZ = 'N' and so never
// forms them):
//   1. A = Q T Q^T by the one-stage Householder reduction (k_tridiag.cu) with
//      its reflectors saved, Q = H_0 H_1 ... H_{n-2};
//   2. T's eigenvalues by bisection (k_eigval.cu);
//   3. T's eigenvectors, one thread per eigenvalue: a twisted factorisation
//      N_r D_r N_r^T of T - lambda I with the twist r at the smallest |gamma_r|
//      gives the vector in O(n) (Fernando; Parlett and Dhillon); eigenvalues
//      closer than a cluster tolerance are solved together by one thread,
//      inverse iteration from fixed pseudo-random starts with modified
//      Gram-Schmidt inside the cluster (the scheme of LAPACK's DSTEIN);
//   4. Newton-Schulz steps Z <- Z (3 I - Z^T Z) / 2 until Z^T Z = I to
//      ~1e-15 (vectors of eigenvalues a small gap apart carry errors of
//      eps ||T|| / gap; the step removes them to second order);
//   5. X = Q Z by compact-WY blocks of 128 reflectors, applied last block
//      first: X <- X - V (T_b (V^T X)).
// The dense products run on FP64 tensor-core MMA (mma.sync m8n8k4) in one
// row-major GEMM kernel.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#include "kernels.h"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

// ---- row-major DGEMM on FP64 MMA ------------------------------------------
// C (M x N, row-major, ldc) = alpha op(A) op(B) + beta C with
//   op(A)(i, k) = TA ? A[k * lda + i] : A[i * lda + k]
//   op(B)(k, j) = TB ? B[j * ldb + k] : B[k * ldb + j]
// 64 x 64 tiles of C per CTA, 4 warps of 32 x 32 (4 x 4 MMA tiles), K in
// chunks of 32 staged through shared memory, the next chunk's loads in
// registers while the current one is multiplied.
constexpr int GT = 64;         // C tile
constexpr int GK = 32;         // K chunk
constexpr int GS = GK + 4;     // shared row stride (doubles), 4 (mod 16): conflict-free fragments
constexpr int GTHREADS = 128;
constexpr int GLOADS = GT * GK / GTHREADS;   // 16 values of each operand per thread and chunk

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// element e (0 .. GT*GK) of a chunk: (row of the tile, k) with the index that
// is contiguous in global memory running fastest
template <bool KFAST>
__device__ __forceinline__ void chunk_pos(int e, int* r, int* k) {
  if (KFAST) {
    *r = e / GK;
    *k = e % GK;
  } else {
    *r = e % GT;
    *k = e / GT;
  }
}

template <bool TA, bool TB>
__global__ void __launch_bounds__(GTHREADS) dgemm_rm_kernel(int M, int N, int K, double alpha, const double* __restrict__ A,
                                                            size_t lda, const double* __restrict__ B, size_t ldb,
                                                            double beta, double* __restrict__ C, size_t ldc) {
  __shared__ __align__(16) double As[GT * GS];   // As[i][k] = op(A)(i0 + i, k0 + k)
  __shared__ __align__(16) double Bs[GT * GS];   // Bs[j][k] = op(B)(k0 + k, j0 + j)
  const int i0 = blockIdx.y * GT, j0 = blockIdx.x * GT;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, q4 = lane & 3;
  const int r0 = (warp / 2) * 32, c0 = (warp % 2) * 32;
  double ra[GLOADS], rb[GLOADS];
  auto load = [&](int k0) {
#pragma unroll
    for (int u = 0; u < GLOADS; ++u) {
      const int e = tid + GTHREADS * u;
      int r, k;
      chunk_pos<!TA>(e, &r, &k);
      const int gi = i0 + r, gk = k0 + k;
      ra[u] = (gi < M && gk < K) ? (TA ? A[(size_t)gk * lda + gi] : A[(size_t)gi * lda + gk]) : 0.0;
      chunk_pos<TB>(e, &r, &k);
      const int gj = j0 + r, gk2 = k0 + k;
      rb[u] = (gj < N && gk2 < K) ? (TB ? B[(size_t)gj * ldb + gk2] : B[(size_t)gk2 * ldb + gj]) : 0.0;
    }
  };
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[i][q][0] = acc[i][q][1] = 0.0;
  load(0);
  for (int k0 = 0; k0 < K; k0 += GK) {
#pragma unroll
    for (int u = 0; u < GLOADS; ++u) {
      const int e = tid + GTHREADS * u;
      int r, k;
      chunk_pos<!TA>(e, &r, &k);
      As[r * GS + k] = ra[u];
      chunk_pos<TB>(e, &r, &k);
      Bs[r * GS + k] = rb[u];
    }
    __syncthreads();
    if (k0 + GK < K) load(k0 + GK);
#pragma unroll
    for (int kk = 0; kk < GK; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = As[(r0 + i * 8 + g) * GS + kk + q4];
#pragma unroll
      for (int q = 0; q < 4; ++q) bf[q] = Bs[(c0 + q * 8 + g) * GS + kk + q4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) dmma(acc[i][q][0], acc[i][q][1], af[i], bf[q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int gi = i0 + r0 + i * 8 + g, gj = j0 + c0 + q * 8 + 2 * q4 + h;
        if (gi < M && gj < N) {
          double* c = C + (size_t)gi * ldc + gj;
          *c = beta == 0.0 ? alpha * acc[i][q][h] : alpha * acc[i][q][h] + beta * *c;
        }
      }
}

// ---- eigenvectors of the tridiagonal ---------------------------------------
// Fixed pseudo-random start in [-1, 1) for component i of vector k.
__device__ __forceinline__ double start_value(int i, int k) {
  unsigned long long x = ((unsigned long long)(unsigned)k << 32) ^ (unsigned long long)(unsigned)i;
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  x ^= x >> 31;
  return (double)(x >> 11) * 0x1.0p-52 - 1.0;
}

__device__ __forceinline__ double guard(double p, double pivmin) { return fabs(p) < pivmin ? -pivmin : p; }

// Vector of the isolated eigenvalue lam into column k of Z (row-major,
// Z[i * ldz + k]); s1(i) is this thread's scratch.
template <class S1>
__device__ void twisted_vector(const double* __restrict__ d, const double* __restrict__ e, int n, double lam,
                               double pivmin, double* Z, size_t ldz, int k, S1 s1) {
  // D-: T - lam I = U- D- U-^T from the bottom
  double dm = guard(d[n - 1] - lam, pivmin);
  s1(n - 1) = dm;
  for (int i = n - 2; i >= 0; --i) {
    dm = guard((d[i] - lam) - e[i] * (e[i] / dm), pivmin);
    s1(i) = dm;
  }
  // D+ from the top, L+ into the column; gamma_i = D+_i + D-_i - (d_i - lam)
  double dp = guard(d[0] - lam, pivmin);
  double best = fabs(s1(0));
  int r = 0;
  for (int i = 1; i < n; ++i) {
    const double lp = e[i - 1] / dp;
    Z[(size_t)(i - 1) * ldz + k] = lp;
    const double a = d[i] - lam;
    dp = guard(a - lp * e[i - 1], pivmin);
    const double gm = fabs(dp + s1(i) - a);
    if (gm < best) {
      best = gm;
      r = i;
    }
  }
  // N_r^T z = e_r: z_r = 1, outwards from r (through a zero component by the
  // row of T - lam I that links the two neighbours)
  double nrm2 = 1.0;
  Z[(size_t)r * ldz + k] = 1.0;
  double z1 = 1.0, z2 = 0.0;   // z_{i+1}, z_{i+2}
  for (int i = r - 1; i >= 0; --i) {
    double z = -Z[(size_t)i * ldz + k] * z1;
    if (z1 == 0.0 && i + 2 < n && e[i] != 0.0) z = -(e[i + 1] * z2) / e[i];
    Z[(size_t)i * ldz + k] = z;
    nrm2 += z * z;
    z2 = z1;
    z1 = z;
  }
  z1 = 1.0;   // z_i
  z2 = 0.0;   // z_{i-1}
  for (int i = r; i < n - 1; ++i) {
    double z = -(e[i] / s1(i + 1)) * z1;
    if (z1 == 0.0 && i >= 1 && e[i] != 0.0) z = -(e[i - 1] * z2) / e[i];
    Z[(size_t)(i + 1) * ldz + k] = z;
    nrm2 += z * z;
    z2 = z1;
    z1 = z;
  }
  const double sc = 1.0 / sqrt(nrm2);
  for (int i = 0; i < n; ++i) Z[(size_t)i * ldz + k] *= sc;
}

// Vectors of the cluster lo..hi into columns lo..hi: three steps of inverse
// iteration each, shifts at least `pert` apart, Gram-Schmidt (twice) against
// the cluster's earlier vectors after every step.
template <class S1, class S2>
__device__ void cluster_vectors(const double* __restrict__ d, const double* __restrict__ e, const double* __restrict__ ev,
                                int n, int lo, int hi, double pivmin, double pert, double* Z, size_t ldz, S1 s1,
                                S2 s2) {
  double prev = 0.0;
  for (int k = lo; k <= hi; ++k) {
    double sigma = ev[k];
    if (k > lo && sigma < prev + pert) sigma = prev + pert;
    prev = sigma;
    // T - sigma I = L D L^T
    double dd = guard(d[0] - sigma, pivmin);
    s1(0) = dd;
    for (int i = 1; i < n; ++i) {
      const double l = e[i - 1] / dd;
      s2(i - 1) = l;
      dd = guard((d[i] - sigma) - l * e[i - 1], pivmin);
      s1(i) = dd;
    }
    for (int i = 0; i < n; ++i) Z[(size_t)i * ldz + k] = start_value(i, k);
    for (int it = 0; it < 3; ++it) {
      double u = Z[k];
      for (int i = 1; i < n; ++i) {
        u = Z[(size_t)i * ldz + k] - s2(i - 1) * u;
        Z[(size_t)i * ldz + k] = u;
      }
      double y = Z[(size_t)(n - 1) * ldz + k] / s1(n - 1), ymax = fabs(y);
      Z[(size_t)(n - 1) * ldz + k] = y;
      for (int i = n - 2; i >= 0; --i) {
        y = Z[(size_t)i * ldz + k] / s1(i) - s2(i) * y;
        Z[(size_t)i * ldz + k] = y;
        ymax = fmax(ymax, fabs(y));
      }
      const double inv = ymax > 0.0 ? 1.0 / ymax : 1.0;
      for (int i = 0; i < n; ++i) Z[(size_t)i * ldz + k] *= inv;
      for (int pass = 0; pass < 2; ++pass)
        for (int j = lo; j < k; ++j) {
          double dot = 0.0;
          for (int i = 0; i < n; ++i) dot += Z[(size_t)i * ldz + j] * Z[(size_t)i * ldz + k];
          for (int i = 0; i < n; ++i) Z[(size_t)i * ldz + k] -= dot * Z[(size_t)i * ldz + j];
        }
      double nrm2 = 0.0;
      for (int i = 0; i < n; ++i) nrm2 += Z[(size_t)i * ldz + k] * Z[(size_t)i * ldz + k];
      const double sc = nrm2 > 0.0 ? 1.0 / sqrt(nrm2) : 0.0;
      for (int i = 0; i < n; ++i) Z[(size_t)i * ldz + k] *= sc;
    }
  }
}

// Thread t takes eigenvalues t, t + nthr, ...; its scratch is interleaved
// with the other threads' (element i at S[i * nthr + t]) so a warp's
// accesses coalesce, and so do its writes of Z's row-major columns.
__global__ void __launch_bounds__(128) tri_vectors_kernel(const double* __restrict__ d, const double* __restrict__ e,
                                                          const double* __restrict__ ev, int n, double ctol,
                                                          double pivmin, double pert, double* Z, size_t ldz,
                                                          double* S, int nthr) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nthr) return;
  double* S1 = S;
  double* S2 = S + (size_t)n * nthr;
  auto s1 = [=](int i) -> double& { return S1[(size_t)i * nthr + t]; };
  auto s2 = [=](int i) -> double& { return S2[(size_t)i * nthr + t]; };
  for (int k = t; k < n; k += nthr) {
    if (n == 1) {
      Z[0] = 1.0;
      continue;
    }
    int lo = k, hi = k;
    while (lo > 0 && ev[lo] - ev[lo - 1] <= ctol) --lo;
    while (hi < n - 1 && ev[hi + 1] - ev[hi] <= ctol) ++hi;
    if (lo == hi) twisted_vector(d, e, n, ev[k], pivmin, Z, ldz, k, s1);
    else if (k == lo) cluster_vectors(d, e, ev, n, lo, hi, pivmin, pert, Z, ldz, s1, s2);
  }
}

// ---- Newton-Schulz and compact WY -----------------------------------------
// G <- 3/2 I - G/2 in place; *dev = max |G - I| (non-negative doubles order
// as their bit patterns).
__global__ void ns_prepare_kernel(double* G, int n, unsigned long long* dev) {
  const size_t total = (size_t)n * n;
  double m = 0.0;
  for (size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    const double gv = G[idx];
    const double dv = i == j ? gv - 1.0 : gv;
    m = fmax(m, fabs(dv));
    G[idx] = (i == j ? 1.5 : 0.0) - 0.5 * gv;
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dev, (unsigned long long)__double_as_longlong(m));
}

// T (nb x nb, row-major, upper) of the forward compact-WY form
// H_0 ... H_{kb-1} = I - V T V^T from the Gram matrix S = V^T V (row-major,
// ld nb) and the taus: T(j,j) = tau_j, T(0:j, j) = -tau_j T(0:j, 0:j) S(0:j, j).
__global__ void wy_t_kernel(const double* __restrict__ S, const double* __restrict__ tau, int kb, int nb, double* T) {
  const int i = threadIdx.x;   // blockDim.x == nb
  for (int c = 0; c < nb; ++c) T[i * nb + c] = 0.0;
  __syncthreads();
  for (int j = 0; j < kb; ++j) {
    double v = 0.0;
    if (i < j) {
      for (int l = i; l < j; ++l) v += T[i * nb + l] * S[l * nb + j];
      v *= -tau[j];
    } else if (i == j) {
      v = tau[j];
    }
    __syncthreads();
    if (i <= j) T[i * nb + j] = v;
    __syncthreads();
  }
}

}  // namespace

void dgemm_rm(bool ta, bool tb, int M, int N, int K, double alpha, const double* A, size_t lda, const double* B,
              size_t ldb, double beta, double* C, size_t ldc, cudaStream_t s) {
  if (M <= 0 || N <= 0) return;
  dim3 grid((N + GT - 1) / GT, (M + GT - 1) / GT);
  if (!ta && !tb) dgemm_rm_kernel<false, false><<<grid, GTHREADS, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  else if (ta && !tb) dgemm_rm_kernel<true, false><<<grid, GTHREADS, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  else if (!ta && tb) dgemm_rm_kernel<false, true><<<grid, GTHREADS, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
  else dgemm_rm_kernel<true, true><<<grid, GTHREADS, 0, s>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc);
}

int tri_vectors_threads(int n) { return std::max(1, std::min(n, 8192)); }

size_t eigh_scratch_doubles(int n) { return 2 * (size_t)n * tri_vectors_threads(n); }

void launch_tri_vectors(const double* d, const double* e, const double* ev, int n, double tnorm, double* Z, size_t ldz,
                        double* S, cudaStream_t s) {
  const int nthr = tri_vectors_threads(n);
  const double eps = 0x1.0p-52;
  const double scale = std::max(tnorm, 1e-250);   // a zero matrix: one cluster, normal pivot floor
  const double ctol = 1e-10 * scale;               // eigenvalues this close are solved as one cluster
  const double pivmin = scale * 0x1.0p-80;
  const double pert = 4.0 * eps * scale;           // minimum shift separation inside a cluster
  tri_vectors_kernel<<<(nthr + 127) / 128, 128, 0, s>>>(d, e, ev, n, ctol, pivmin, pert, Z, ldz, S, nthr);
}

void launch_ns_prepare(double* G, int n, unsigned long long* dev, cudaStream_t s) {
  const size_t total = (size_t)n * n;
  const unsigned blocks = (unsigned)std::min<size_t>(4096, (total + 255) / 256);
  ns_prepare_kernel<<<std::max(1u, blocks), 256, 0, s>>>(G, n, dev);
}

void launch_wy_t(const double* S, const double* tau, int kb, int nb, double* T, cudaStream_t s) {
  wy_t_kernel<<<1, nb, 0, s>>>(S, tau, kb, nb, T);
}

}  // namespace mbd
