// FP64 relay factorisation and solve (the plain path): blocked right-looking
// Cholesky A = L L^T on row-major lower matrices, batched over the 21
// frequency matrices (PDPOTRF('L') at UTILS.f90:469), the 3-RHS solve
// X = A^-1 [I;I;..;I] (PDPOTRS at UTILS.f90:473) and the reductions of
// get_screened_alpha / MBD_at_rsSCS (UTILS.f90:479-495, 272-315, 731-741).
//
// Per 64-column step k0:
//   potrf_diag   factor the 64x64 diagonal block in shared memory and store
//                its inverse Linv (used by the panel and by the solves);
//   trsm_panel   L[r, k0:k0+64] = A[r, k0:k0+64] Linv^T for rows below;
//   syrk_mma     A[trail] -= P P^T on the lower 64x64 tiles (FP64 tensor-core MMA).
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"

namespace mbd {
namespace {

constexpr int NB = kCholNB;  // 64

__device__ __forceinline__ double* mat_ptr(const BatchMat& m, int b) { return m.A + (size_t)b * m.stride; }

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) potrf_diag_kernel(BatchMat m, int k0, double* Linv,
                                                        size_t linv_stride, int* info) {
  extern __shared__ double dyn_smem[];
  double (*S)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(dyn_smem);
  double (*X)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(dyn_smem + NB * (NB + 1));
  __shared__ int s_bad;
  const int b = blockIdx.x;
  double* A = mat_ptr(m, b);
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    int r = idx / NB, c = idx % NB;
    double v = 0.0;
    if (r < nbk && c < nbk && c <= r) v = A[(size_t)(k0 + r) * m.ld + k0 + c];
    if (r == c && r >= nbk) v = 1.0;      // identity padding keeps the block SPD
    S[r][c] = v;
    X[r][c] = 0.0;
  }
  __syncthreads();
  for (int c = 0; c < NB; ++c) {
    if (tid == 0) {
      double piv = S[c][c];
      if (!(piv > 0.0)) {                 // not SPD (or NaN): record the first failing column
        if (!s_bad && c < nbk) {
          s_bad = 1;
          atomicCAS(&info[b], 0, k0 + c + 1);
        }
        piv = 1.0;
      }
      S[c][c] = sqrt(piv);
    }
    __syncthreads();
    const double inv = 1.0 / S[c][c];
    for (int r = c + 1 + tid; r < NB; r += blockDim.x) S[r][c] *= inv;
    __syncthreads();
    const int rem = NB - c - 1;
    for (int idx = tid; idx < rem * rem; idx += blockDim.x) {
      int r = c + 1 + idx / rem, q = c + 1 + idx % rem;
      if (q <= r) S[r][q] -= S[r][c] * S[q][c];
    }
    __syncthreads();
  }
  // Inverse of the lower-triangular factor, row by row:
  // X[i][j] = -(sum_{k=j}^{i-1} S[i][k] X[k][j]) / S[i][i]; X[i][i] = 1/S[i][i].
  for (int i = 0; i < NB; ++i) {
    const double dinv = 1.0 / S[i][i];
    for (int j = tid; j <= i; j += blockDim.x) {
      if (j == i) {
        X[i][i] = dinv;
      } else {
        double acc = 0.0;
        for (int k = j; k < i; ++k) acc += S[i][k] * X[k][j];
        X[i][j] = -acc * dinv;
      }
    }
    __syncthreads();
  }
  double* Li = Linv + (size_t)b * linv_stride + (size_t)(k0 / NB) * NB * NB;
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    int r = idx / NB, c = idx % NB;
    Li[idx] = X[r][c];
    if (r < nbk && c < nbk && c <= r) A[(size_t)(k0 + r) * m.ld + k0 + c] = S[r][c];
  }
}

// ---------------------------------------------------------------------------
// Rows [k0+64 + 64*blockIdx.x, +64): P = A_panel Linv^T, in place.
__global__ void __launch_bounds__(256) trsm_panel_kernel(BatchMat m, int k0, const double* Linv,
                                                        size_t linv_stride) {
  extern __shared__ double dyn_smem[];
  double (*Ls)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(dyn_smem);
  double (*As)[NB + 1] = reinterpret_cast<double (*)[NB + 1]>(dyn_smem + NB * (NB + 1));
  const int b = blockIdx.y;
  double* A = mat_ptr(m, b);
  const int r0 = k0 + NB + blockIdx.x * NB;
  const int tid = threadIdx.x;
  const double* Li = Linv + (size_t)b * linv_stride + (size_t)(k0 / NB) * NB * NB;
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    int r = idx / NB, c = idx % NB;
    Ls[r][c] = Li[idx];
    As[r][c] = (r0 + r < m.n && k0 + c < m.n) ? A[(size_t)(r0 + r) * m.ld + k0 + c] : 0.0;
  }
  __syncthreads();
  // thread -> rows (tid/16)*4..+3, cols (tid%16) + 16*q
  const int tr = (tid / 16) * 4, tc = tid % 16;
  double acc[4][4] = {};
  for (int l = 0; l < NB; ++l) {
    double a[4], w[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) a[u] = As[tr + u][l];
#pragma unroll
    for (int q = 0; q < 4; ++q) w[q] = Ls[tc + 16 * q][l];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[u][q] += a[u] * w[q];
  }
  const int nbk = min(NB, m.n - k0);
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int r = r0 + tr + u, c = tc + 16 * q;
      if (r < m.n && c < nbk) A[(size_t)r * m.ld + k0 + c] = acc[u][q];
    }
}

// ---------------------------------------------------------------------------
// SYRK on the trailing lower triangle: C[t0.., t0..] -= P P^T, P = A[t0.., k0:k0+64],
// on FP64 tensor-core MMAs (mma.sync m8n8k4, FP64 in and out).

__device__ __forceinline__ void tri_index(int t, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

// D = A B + D with A 8x4 (row), B 4x8 (col), D 8x8 in FP64:
// a = A[lane/4][lane%4], b = B[lane%4][lane/4], d = D[lane/4][2*(lane%4) + {0,1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// 16-byte asynchronous copy global -> shared; src_bytes < 16 zero-fills the rest.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}

constexpr int MT = 64;            // tile edge
constexpr int MFS = MT + 4;       // shared row stride: the 8 x 4 fragment loads of a half-warp hit 16 bank pairs
constexpr size_t kSyrkSmem = sizeof(double) * 3 * MT * MFS;

// One lower 64 x 64 tile (I, J) of the trailing matrix per CTA, 4 warps each
// a 32 x 32 quarter (4 x 4 MMA tiles).  The panel rows of block I and J and
// the tile itself go to shared memory together (cp.async, zero-filled past
// the matrix), the product is subtracted there and the tile goes back a row
// per warp instruction.
__global__ void __launch_bounds__(128) syrk_mma_kernel(BatchMat m, int k0) {
  extern __shared__ __align__(16) double dsm[];
  double* Pi = dsm;                // [64][MFS]: P rows of block I
  double* Pj = dsm + MT * MFS;     // [64][MFS]: P rows of block J
  double* Cs = dsm + 2 * MT * MFS; // [64][MFS]: the tile (I, J)
  const int b = blockIdx.y;
  double* A = mat_ptr(m, b);
  const int t0 = k0 + NB;
  const int msz = m.n - t0;
  int ti, tj;
  tri_index(blockIdx.x, &ti, &tj);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, q4 = lane & 3;
  double* T = A + (size_t)t0 * m.ld;   // row t0 of the matrix
  for (int e = tid; e < MT * (NB / 2); e += 128) {
    const int r = e / (NB / 2), c = 2 * (e % (NB / 2));
    const int gi = ti * MT + r, gj = tj * MT + r;
    cp_async16(Pi + r * MFS + c, T + (size_t)(gi < msz ? gi : 0) * m.ld + k0 + c, gi < msz ? 16 : 0);
    cp_async16(Pj + r * MFS + c, T + (size_t)(gj < msz ? gj : 0) * m.ld + k0 + c, gj < msz ? 16 : 0);
  }
  for (int e = tid; e < MT * (MT / 2); e += 128) {
    const int r = e / (MT / 2), c = 2 * (e % (MT / 2));
    const int gr = ti * MT + r, gc = tj * MT + c;
    const bool rok = gr < msz;
    const int bytes = rok ? (gc + 1 < msz ? 16 : (gc < msz ? 8 : 0)) : 0;
    cp_async16(Cs + r * MFS + c, T + (size_t)(rok ? gr : 0) * m.ld + t0 + (bytes ? gc : 0), bytes);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  const int r0 = (warp / 2) * 32, c0 = (warp % 2) * 32;
  if (!(ti == tj && c0 > r0)) {   // the strictly upper quarter of a diagonal tile is not stored
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][q][0] = acc[i][q][1] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < NB; kk += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = Pi[(r0 + i * 8 + g) * MFS + kk + q4];
#pragma unroll
      for (int q = 0; q < 4; ++q) bf[q] = Pj[(c0 + q * 8 + g) * MFS + kk + q4];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int q = 0; q < 4; ++q) dmma(acc[i][q][0], acc[i][q][1], af[i], bf[q]);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int h = 0; h < 2; ++h) Cs[(r0 + i * 8 + g) * MFS + c0 + q * 8 + 2 * q4 + h] -= acc[i][q][h];
  }
  __syncthreads();
  for (int e = tid; e < MT * MT; e += 128) {
    const int r = e / MT, c = e % MT;
    const int gr = ti * MT + r, gc = tj * MT + c;
    if (gr < msz && gc < msz && (ti != tj || c <= r)) T[(size_t)gr * m.ld + t0 + gc] = Cs[r * MFS + c];
  }
}

// ---------------------------------------------------------------------------
__global__ void init_rhs_kernel(double* Y, size_t ystride, int n, int batch) {
  size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  size_t total = (size_t)n * 3 * batch;
  if (idx >= total) return;
  int b = (int)(idx / ((size_t)n * 3));
  int rem = (int)(idx % ((size_t)n * 3));
  int r = rem / 3, c = rem % 3;
  Y[(size_t)b * ystride + (size_t)r * 3 + c] = (r % 3 == c) ? 1.0 : 0.0;
}

// Forward step for block k0: z_k = Linv_k w_k; w[rows below] -= L[rows, k] z_k.
// Every CTA recomputes z_k in shared memory; CTA 0 stores it into Z.  The
// working right-hand side W is only read at block k and only written below
// it, so no CTA reads a value another CTA of the same launch writes.
__global__ void __launch_bounds__(256) trsv_fwd_kernel(BatchMat m, int k0, const double* Linv,
                                                      size_t linv_stride, double* W, double* Z,
                                                      size_t ystride) {
  __shared__ double yk[NB][3];
  __shared__ double bk[NB][3];
  const int b = blockIdx.y;
  const double* A = m.A + (size_t)b * m.stride;
  double* y = W + (size_t)b * ystride;
  double* z = Z + (size_t)b * ystride;
  const double* Li = Linv + (size_t)b * linv_stride + (size_t)(k0 / NB) * NB * NB;
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) {
    int r = idx / 3, c = idx % 3;
    bk[r][c] = (r < nbk) ? y[(size_t)(k0 + r) * 3 + c] : 0.0;
  }
  __syncthreads();
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) {
    int r = idx / 3, c = idx % 3;
    double acc = 0.0;
    for (int l = 0; l <= r; ++l) acc += Li[r * NB + l] * bk[l][c];
    yk[r][c] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int idx = tid; idx < nbk * 3; idx += blockDim.x) z[(size_t)(k0 + idx / 3) * 3 + idx % 3] = yk[idx / 3][idx % 3];
  // warp per row
  const int warp = tid / 32, lane = tid % 32;
  const int rows_per_cta = 64;
  const int rbase = k0 + nbk + blockIdx.x * rows_per_cta;
  for (int rr = warp; rr < rows_per_cta; rr += blockDim.x / 32) {
    const int r = rbase + rr;
    if (r >= m.n) break;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int l = lane; l < nbk; l += 32) {
      double a = A[(size_t)r * m.ld + k0 + l];
      s0 += a * yk[l][0];
      s1 += a * yk[l][1];
      s2 += a * yk[l][2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
      y[(size_t)r * 3 + 0] -= s0;
      y[(size_t)r * 3 + 1] -= s1;
      y[(size_t)r * 3 + 2] -= s2;
    }
  }
}

// Backward step for block k0: x_k = Linv_k^T z_k; z[rows above] -= L[k, rows]^T x_k.
__global__ void __launch_bounds__(256) trsv_bwd_kernel(BatchMat m, int k0, const double* Linv,
                                                      size_t linv_stride, double* Zw, double* X,
                                                      size_t ystride) {
  __shared__ double xk[NB][3];
  __shared__ double bk[NB][3];
  const int b = blockIdx.y;
  const double* A = m.A + (size_t)b * m.stride;
  double* y = Zw + (size_t)b * ystride;
  double* xo = X + (size_t)b * ystride;
  const double* Li = Linv + (size_t)b * linv_stride + (size_t)(k0 / NB) * NB * NB;
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) {
    int r = idx / 3, c = idx % 3;
    bk[r][c] = (r < nbk) ? y[(size_t)(k0 + r) * 3 + c] : 0.0;
  }
  __syncthreads();
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) {
    int r = idx / 3, c = idx % 3;
    double acc = 0.0;
    for (int l = r; l < NB; ++l) acc += Li[l * NB + r] * bk[l][c];   // (Linv^T)[r][l] = Linv[l][r]
    xk[r][c] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int idx = tid; idx < nbk * 3; idx += blockDim.x) xo[(size_t)(k0 + idx / 3) * 3 + idx % 3] = xk[idx / 3][idx % 3];
  // columns j < k0, one thread per j (coalesced along the rows of block k)
  const int j = blockIdx.x * blockDim.x + tid;
  if (j >= k0) return;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = 0; i < nbk; ++i) {
    double a = A[(size_t)(k0 + i) * m.ld + j];
    s0 += a * xk[i][0];
    s1 += a * xk[i][1];
    s2 += a * xk[i][2];
  }
  y[(size_t)j * 3 + 0] -= s0;
  y[(size_t)j * 3 + 1] -= s1;
  y[(size_t)j * 3 + 2] -= s2;
}

// ---------------------------------------------------------------------------
// alpha_i = tr X_i / 3 and M = sum_i X_i per frequency (UTILS.f90:487-491).
__global__ void __launch_bounds__(256) relay_reduce_kernel(EpilogueArgs a) {
  const int f = blockIdx.x;
  const double* X = a.X + (size_t)f * a.xstride;
  double m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int i = threadIdx.x; i < a.N; i += blockDim.x) {
    const double* x = X + (size_t)(3 * i) * 3;
    a.alpha_iw[(size_t)f * a.N + i] = (x[0] / 3.0 + x[4] / 3.0) + x[8] / 3.0;
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] += x[k];
  }
  __shared__ double red[9][256];
#pragma unroll
  for (int k = 0; k < 9; ++k) red[k][threadIdx.x] = m[k];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int k = 0; k < 9; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < 9) a.molpol[f * 9 + threadIdx.x] = red[threadIdx.x][0];
}

// C6_i, alpha_eff, R_vdW_eff, omega (UTILS.f90:302-315, 731-741); block 0
// also forms the system C6 (UTILS.f90:272-288) and sum 3 omega (UTILS.f90:846-848).

__global__ void __launch_bounds__(256) relay_post_kernel(EpilogueArgs a, const double* w) {
  __shared__ double red[256];
  __shared__ int bad[256];
  double s3w = 0.0;
  int nbad = 0;
  for (int i = threadIdx.x; i < a.N; i += blockDim.x) {
    double c6 = 0.0;
    for (int f = 1; f < 21; ++f) {
      double al = a.alpha_iw[(size_t)f * a.N + i];
      c6 = c6 + (w[f] * al * al);
    }
    c6 = c6 * 0.954929658551372;
    const double ae = a.alpha_iw[i];
    a.c6_eff[i] = c6;
    a.alpha_eff[i] = ae;
    a.rvdw_eff[i] = a.r0[i] * pow(ae / a.alpha0[i], 0.33333333333333333333);
    const double om = (4.0 / 3.0) * c6 / (ae * ae);
    a.omega[i] = om;
    s3w += 3.0 * om;
    if (!(ae > 0.0)) ++nbad;
  }
  red[threadIdx.x] = s3w;
  bad[threadIdx.x] = nbad;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) {
      red[threadIdx.x] += red[threadIdx.x + s];
      bad[threadIdx.x] += bad[threadIdx.x + s];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    double c6m = 0.0;
    for (int f = 1; f < 21; ++f) {
      const double* M = a.molpol + f * 9;
      double iso = (M[0] + M[4] + M[8]) / 3.0;
      c6m = c6m + (w[f] * iso * iso);
    }
    a.scalars[0] = 0.954929658551372 * c6m;
    a.scalars[1] = red[0];
    a.scalars[2] = (double)bad[0];
  }
}

}  // namespace

constexpr size_t kPairSmem = 2 * NB * (NB + 1) * sizeof(double);

cudaError_t init_chol_attributes() {
  cudaError_t e = cudaFuncSetAttribute(syrk_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kSyrkSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(potrf_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmem);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(trsm_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPairSmem);
  return e;
}

void launch_potrf_diag_f64(const BatchMat& m, int k0, double* Linv, size_t linv_stride, int* info,
                           cudaStream_t s) {
  potrf_diag_kernel<<<m.batch, 256, kPairSmem, s>>>(m, k0, Linv, linv_stride, info);
}

void launch_trsm_panel_f64(const BatchMat& m, int k0, const double* Linv, size_t linv_stride,
                           cudaStream_t s) {
  int rows = m.n - k0 - NB;
  if (rows <= 0) return;
  dim3 grid((rows + NB - 1) / NB, m.batch);
  trsm_panel_kernel<<<grid, 256, kPairSmem, s>>>(m, k0, Linv, linv_stride);
}

void launch_syrk_lower_f64(const BatchMat& m, int k0, cudaStream_t s) {
  int msz = m.n - k0 - NB;
  if (msz <= 0) return;
  int nt = (msz + MT - 1) / MT;
  dim3 grid(nt * (nt + 1) / 2, m.batch);
  syrk_mma_kernel<<<grid, 128, kSyrkSmem, s>>>(m, k0);
}

void launch_init_rhs(double* Y, size_t ystride, int n, int batch, cudaStream_t s) {
  size_t total = (size_t)n * 3 * batch;
  init_rhs_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(Y, ystride, n, batch);
}

void launch_trsv_fwd_step(const BatchMat& m, int k0, const double* Linv, size_t linv_stride, double* W,
                          double* Z, size_t ystride, cudaStream_t s) {
  int nbk = std::min(NB, m.n - k0);
  int rows = m.n - k0 - nbk;
  int ctas = std::max(1, (rows + 63) / 64);
  dim3 grid(ctas, m.batch);
  trsv_fwd_kernel<<<grid, 256, 0, s>>>(m, k0, Linv, linv_stride, W, Z, ystride);
}

void launch_trsv_bwd_step(const BatchMat& m, int k0, const double* Linv, size_t linv_stride, double* Zw,
                          double* X, size_t ystride, cudaStream_t s) {
  int ctas = std::max(1, (k0 + 255) / 256);
  dim3 grid(ctas, m.batch);
  trsv_bwd_kernel<<<grid, 256, 0, s>>>(m, k0, Linv, linv_stride, Zw, X, ystride);
}

void launch_relay_epilogue(const EpilogueArgs& a, cudaStream_t s) {
  relay_reduce_kernel<<<21, 256, 0, s>>>(a);
}

void launch_relay_post(const EpilogueArgs& a, const double* weights_dev, cudaStream_t s) {
  relay_post_kernel<<<1, 256, 0, s>>>(a, weights_dev);
}

}  // namespace mbd
