// Mixed-precision relay solve pieces: the FP32 128x128 diagonal-block
// factorisation, triangular solves with the FP32 factor (FP64 right-hand
// sides and accumulation), and the FP64 residual R = B - A X of the lower-
// stored FP64 relay matrices used by the iterative refinement
// (PDPOTRF/PDPOTRS of UTILS.f90:469-473, refined to FP64 accuracy).
#include <cuda_runtime.h>

#include <algorithm>

#include "tc3.h"

namespace mbd {
namespace {

constexpr int NB = kMixNB;   // 128
constexpr int LDS = NB + 1;

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(512) potrf_diag_f32_kernel(BatchMat32 m, int k0, float* linv_hi, float* linv_lo,
                                                            size_t l_bstride, int* info) {
  extern __shared__ float fsm[];
  float (*S)[LDS] = reinterpret_cast<float (*)[LDS]>(fsm);
  float (*X)[LDS] = reinterpret_cast<float (*)[LDS]>(fsm + NB * LDS);
  __shared__ int s_bad;
  const int b = blockIdx.x;
  float* A = m.A + (size_t)b * m.stride;
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  if (tid == 0) s_bad = 0;
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    const int r = idx / NB, c = idx % NB;
    float v = 0.f;
    if (r < nbk && c < nbk && c <= r) v = A[(size_t)(k0 + r) * m.ld + k0 + c];
    if (r == c && r >= nbk) v = 1.f;
    S[r][c] = v;
    X[r][c] = 0.f;
  }
  __syncthreads();
  for (int c = 0; c < NB; ++c) {
    if (tid == 0) {
      float piv = S[c][c];
      if (!(piv > 0.f)) {
        if (!s_bad && c < nbk) {
          s_bad = 1;
          atomicCAS(&info[b], 0, k0 + c + 1);
        }
        piv = 1.f;
      }
      S[c][c] = sqrtf(piv);
    }
    __syncthreads();
    const float inv = 1.f / S[c][c];
    for (int r = c + 1 + tid; r < NB; r += blockDim.x) S[r][c] *= inv;
    __syncthreads();
    const int rem = NB - c - 1;
    for (int idx = tid; idx < rem * rem; idx += blockDim.x) {
      const int r = c + 1 + idx / rem, q = c + 1 + idx % rem;
      if (q <= r) S[r][q] = fmaf(-S[r][c], S[q][c], S[r][q]);
    }
    __syncthreads();
  }
  // X = S^-1 row by row; 4 threads per column j split the dot product.
  const int j = tid / 4, part = tid % 4;
  for (int i = 0; i < NB; ++i) {
    const float dinv = 1.f / S[i][i];
    float acc = 0.f;
    if (j < i)
      for (int k = j + part; k < i; k += 4) acc = fmaf(S[i][k], X[k][j], acc);
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (part == 0) {
      if (j < i) X[i][j] = -acc * dinv;
      else if (j == i) X[i][i] = dinv;
    }
    __syncthreads();
  }
  float* lh = linv_hi + (size_t)b * l_bstride + (size_t)k0 * NB;
  float* ll = linv_lo + (size_t)b * l_bstride + (size_t)k0 * NB;
  for (int idx = tid; idx < NB * NB; idx += blockDim.x) {
    const int r = idx / NB, c = idx % NB;
    const float x = X[r][c];
    const float h = tf32_hi(x);
    lh[idx] = h;
    ll[idx] = x - h;
    if (r < nbk && c < nbk && c <= r) A[(size_t)(k0 + r) * m.ld + k0 + c] = S[r][c];
  }
}

// ---------------------------------------------------------------------------
// Forward step at block k0: z_k = Linv_k w_k (into Z); w[rows below] -= L[rows, k] z_k.
__global__ void __launch_bounds__(256) fwd_f32_kernel(BatchMat32 m, int k0, const float* lh, const float* ll,
                                                     size_t l_bstride, double* W, double* Z, size_t ystride) {
  __shared__ double zk[NB][3];
  __shared__ double wk[NB][3];
  const int b = blockIdx.y;
  const float* A = m.A + (size_t)b * m.stride;
  double* w = W + (size_t)b * ystride;
  const float* Lh = lh + (size_t)b * l_bstride + (size_t)k0 * NB;
  const float* Ll = ll + (size_t)b * l_bstride + (size_t)k0 * NB;
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) wk[idx / 3][idx % 3] = (idx / 3 < nbk) ? w[(size_t)k0 * 3 + idx] : 0.0;
  __syncthreads();
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) {
    const int r = idx / 3, c = idx % 3;
    double acc = 0.0;
    for (int l = 0; l <= r; ++l) acc += ((double)Lh[r * NB + l] + (double)Ll[r * NB + l]) * wk[l][c];
    zk[r][c] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int idx = tid; idx < nbk * 3; idx += blockDim.x) Z[(size_t)b * ystride + (size_t)k0 * 3 + idx] = zk[idx / 3][idx % 3];
  const int warp = tid / 32, lane = tid % 32;
  const int rbase = k0 + nbk + blockIdx.x * 64;
  for (int rr = warp; rr < 64; rr += 8) {
    const int r = rbase + rr;
    if (r >= m.n) break;
    double s0 = 0, s1 = 0, s2 = 0;
    for (int l = lane; l < nbk; l += 32) {
      const double a = A[(size_t)r * m.ld + k0 + l];
      s0 += a * zk[l][0];
      s1 += a * zk[l][1];
      s2 += a * zk[l][2];
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      s0 += __shfl_xor_sync(0xffffffffu, s0, o);
      s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    }
    if (lane == 0) {
      w[(size_t)r * 3 + 0] -= s0;
      w[(size_t)r * 3 + 1] -= s1;
      w[(size_t)r * 3 + 2] -= s2;
    }
  }
}

// Backward step at block k0: x_k = Linv_k^T z_k (into D); z[rows above] -= L[k, rows]^T x_k.
__global__ void __launch_bounds__(256) bwd_f32_kernel(BatchMat32 m, int k0, const float* lh, const float* ll,
                                                     size_t l_bstride, double* Zw, double* D, size_t ystride) {
  __shared__ double xk[NB][3];
  __shared__ double zk[NB][3];
  const int b = blockIdx.y;
  const float* A = m.A + (size_t)b * m.stride;
  double* z = Zw + (size_t)b * ystride;
  const float* Lh = lh + (size_t)b * l_bstride + (size_t)k0 * NB;
  const float* Ll = ll + (size_t)b * l_bstride + (size_t)k0 * NB;
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) zk[idx / 3][idx % 3] = (idx / 3 < nbk) ? z[(size_t)k0 * 3 + idx] : 0.0;
  __syncthreads();
  for (int idx = tid; idx < NB * 3; idx += blockDim.x) {
    const int r = idx / 3, c = idx % 3;
    double acc = 0.0;
    for (int l = r; l < NB; ++l) acc += ((double)Lh[l * NB + r] + (double)Ll[l * NB + r]) * zk[l][c];
    xk[r][c] = acc;
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int idx = tid; idx < nbk * 3; idx += blockDim.x) D[(size_t)b * ystride + (size_t)k0 * 3 + idx] = xk[idx / 3][idx % 3];
  const int jc = blockIdx.x * blockDim.x + tid;
  if (jc >= k0) return;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int i = 0; i < nbk; ++i) {
    const double a = A[(size_t)(k0 + i) * m.ld + jc];
    s0 += a * xk[i][0];
    s1 += a * xk[i][1];
    s2 += a * xk[i][2];
  }
  z[(size_t)jc * 3 + 0] -= s0;
  z[(size_t)jc * 3 + 1] -= s1;
  z[(size_t)jc * 3 + 2] -= s2;
}

// ---------------------------------------------------------------------------
// Residual R = B - A X, A lower-stored FP64: tile partials, then row sums.
constexpr int RT = 64;

__device__ __forceinline__ void rt_index(int t, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

__global__ void axpy_kernel(double* X, const double* D, size_t total) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < total) X[i] += D[i];
}

// One CTA (192 threads) per lower tile (I, J): row partial (rows of I) and
// column partial (rows of J), each 64 x 3, into partial[b][I][J] / [b][J][I].
__global__ void __launch_bounds__(192) res_tile_kernel(const double* A64, size_t a_stride, int ld, int n,
                                                      const double* X, size_t ystride, double* partial, int nt) {
  __shared__ double Ts[RT][RT + 1];
  __shared__ double xI[RT][3], xJ[RT][3];
  int ti, tj;
  rt_index(blockIdx.x, &ti, &tj);
  const int b = blockIdx.y;
  const double* A = A64 + (size_t)b * a_stride;
  const double* x = X + (size_t)b * ystride;
  const int tid = threadIdx.x;
  const bool diag = ti == tj;
  for (int idx = tid; idx < RT * RT; idx += blockDim.x) {
    const int r = idx / RT, c = idx % RT;
    const int gr = ti * RT + r, gc = tj * RT + c;
    double v = 0.0;
    if (gr < n && gc < n && (!diag || c <= r)) v = A[(size_t)gr * ld + gc];
    Ts[r][c] = v;
  }
  for (int idx = tid; idx < RT * 3; idx += blockDim.x) {
    const int r = idx / 3, q = idx % 3;
    const int gi = ti * RT + r, gj = tj * RT + r;
    xI[r][q] = gi < n ? x[(size_t)gi * 3 + q] : 0.0;
    xJ[r][q] = gj < n ? x[(size_t)gj * 3 + q] : 0.0;
  }
  __syncthreads();
  const int r = tid / 3, q = tid % 3;   // 64 x 3
  double rs = 0.0, cs = 0.0;
  for (int c = 0; c < RT; ++c) rs += Ts[r][c] * xJ[c][q];                 // row part
  for (int c = 0; c < RT; ++c)                                             // column part (strict lower on diag)
    if (!diag || c > r) cs += Ts[c][r] * xI[c][q];
  double* pr = partial + (size_t)b * nt * nt * RT * 3;
  if (!diag) {
    pr[((size_t)ti * nt + tj) * RT * 3 + tid] = rs;
    pr[((size_t)tj * nt + ti) * RT * 3 + tid] = cs;
  } else {
    pr[((size_t)ti * nt + ti) * RT * 3 + tid] = rs + cs;
  }
}

// R[row] = B[row] - sum_J partial[b][I][J][row]; per-block squared norms.
__global__ void __launch_bounds__(192) res_reduce_kernel(const double* partial, int nt, int n, double* R,
                                                        size_t ystride, double* normpart) {
  const int I = blockIdx.x, b = blockIdx.y;
  const int tid = threadIdx.x;
  const int r = tid / 3, q = tid % 3;
  const int gr = I * RT + r;
  const double* pr = partial + (size_t)b * nt * nt * RT * 3 + (size_t)I * nt * RT * 3 + tid;
  double y = 0.0;
  for (int J = 0; J < nt; ++J) y += pr[(size_t)J * RT * 3];
  double res = 0.0;
  if (gr < n) {
    res = ((gr % 3) == q ? 1.0 : 0.0) - y;
    R[(size_t)b * ystride + (size_t)gr * 3 + q] = res;
  }
  __shared__ double red[192];
  red[tid] = res * res;
  __syncthreads();
  if (tid == 0) {
    double s = 0.0;
    for (int k = 0; k < 192; ++k) s += red[k];
    normpart[(size_t)b * nt + I] = s;
  }
}

__global__ void norm_final_kernel(const double* normpart, int nt, double* rnorm2) {
  const int b = blockIdx.x;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int I = 0; I < nt; ++I) s += normpart[(size_t)b * nt + I];
    rnorm2[b] = s;
  }
}

}  // namespace

constexpr size_t kPotrf32Smem = 2 * NB * LDS * sizeof(float);

cudaError_t init_mixed_attributes() {
  return cudaFuncSetAttribute(potrf_diag_f32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPotrf32Smem);
}

void launch_potrf_diag_f32(const BatchMat32& m, int k0, float* linv_hi, float* linv_lo, size_t l_bstride, int* info,
                           cudaStream_t s) {
  potrf_diag_f32_kernel<<<m.batch, 512, kPotrf32Smem, s>>>(m, k0, linv_hi, linv_lo, l_bstride, info);
}

void launch_solve_f32(const BatchMat32& m, const float* linv_hi, const float* linv_lo, size_t l_bstride, double* R,
                      double* Z, double* D, size_t ystride, cudaStream_t s) {
  const int nblk = (m.n + NB - 1) / NB;
  for (int k0 = 0; k0 < m.n; k0 += NB) {
    const int nbk = std::min(NB, m.n - k0);
    const int rows = m.n - k0 - nbk;
    const int ctas = std::max(1, (rows + 63) / 64);
    fwd_f32_kernel<<<dim3(ctas, m.batch), 256, 0, s>>>(m, k0, linv_hi, linv_lo, l_bstride, R, Z, ystride);
  }
  for (int k0 = (nblk - 1) * NB; k0 >= 0; k0 -= NB) {
    const int ctas = std::max(1, (k0 + 255) / 256);
    bwd_f32_kernel<<<dim3(ctas, m.batch), 256, 0, s>>>(m, k0, linv_hi, linv_lo, l_bstride, Z, D, ystride);
  }
}

size_t relay_residual_ws_doubles(int n, int batch) {
  const int nt = (n + RT - 1) / RT;
  return (size_t)batch * nt * nt * RT * 3 + (size_t)batch * nt;
}

void launch_relay_residual(const double* A64, size_t a_stride, int ld, int n, int batch, double* X, const double* D,
                           double* R, size_t ystride, double* partial, double* rnorm2, cudaStream_t s) {
  const int nt = (n + RT - 1) / RT;
  if (D) {
    const size_t total = (size_t)batch * ystride;
    axpy_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(X, D, total);
  }
  res_tile_kernel<<<dim3(nt * (nt + 1) / 2, batch), 192, 0, s>>>(A64, a_stride, ld, n, X, ystride, partial, nt);
  double* normpart = partial + (size_t)batch * nt * nt * RT * 3;
  res_reduce_kernel<<<dim3(nt, batch), 192, 0, s>>>(partial, nt, n, R, ystride, normpart);
  norm_final_kernel<<<batch, 32, 0, s>>>(normpart, nt, rnorm2);
}

}  // namespace mbd
