// Mixed-precision relay solve pieces: the FP32 128x128 diagonal-block
// factorisation, triangular solves with the FP32 factor (FP64 right-hand
// sides and accumulation), and the FP64 residual R = B - A X of the lower-
// stored FP64 relay matrices used by the iterative refinement
// (PDPOTRF/PDPOTRS of UTILS.f90:469-473, refined to FP64 accuracy).
//
// The triangular solves are sync-free single launches: each CTA takes a
// ticket (atomicAdd) that fixes its 128-row block in dependency order, then
// waits on per-block ready flags of the blocks it needs (bounded spins), so
// a CTA only ever waits for CTAs that already started.
#include <cuda_runtime.h>

#include <algorithm>

#include "tc3.h"
#include "wait_limit.cuh"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int NB = kMixNB;   // 128
constexpr int LDS = NB + 1;

__device__ __forceinline__ float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

// ---------------------------------------------------------------------------
// 512 threads: thread t works on row t/4 with column phase t%4.
__global__ void __launch_bounds__(512) potrf_diag_f32_kernel(BatchMat32 m, int k0, float* linv_hi, float* linv_lo,
                                                            size_t l_bstride, int* info) {
  extern __shared__ float fsm[];
  float (*S)[LDS] = reinterpret_cast<float (*)[LDS]>(fsm);
  float (*X)[LDS] = reinterpret_cast<float (*)[LDS]>(fsm + NB * LDS);
  const int b = blockIdx.x;
  float* A = m.A + (size_t)b * m.stride;
  const int nbk = min(NB, m.n - k0);
  const int tid = threadIdx.x;
  const int r = tid / 4, part = tid % 4;
  for (int c = part; c < NB; c += 4) {
    float v = 0.f;
    if (r < nbk && c < nbk && c <= r) v = A[(size_t)(k0 + r) * m.ld + k0 + c];
    if (r == c && r >= nbk) v = 1.f;                 // identity padding keeps the block SPD
    S[r][c] = v;
    X[r][c] = 0.f;
  }
  __syncthreads();
  bool bad = false;
  for (int c = 0; c < NB; ++c) {
    float piv = S[c][c];
    if (!(piv > 0.f)) {
      if (c < nbk) bad = true;
      piv = 1.f;
    }
    const float d = sqrtf(piv);
    const float inv = 1.f / d;
    if (r > c && part == 0) S[r][c] *= inv;
    __syncthreads();
    if (r > c) {
      const float lrc = S[r][c];
      for (int q = c + 1 + part; q <= r; q += 4) S[r][q] = fmaf(-lrc, S[q][c], S[r][q]);
    } else if (r == c && part == 0) {
      S[c][c] = d;
    }
    __syncthreads();
  }
  if (bad && tid == 0) atomicCAS(&info[b], 0, k0 + 1);
  // X = S^-1 row by row; 4 threads per column j split the dot product.
  const int j = tid / 4;
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
  for (int c = part; c < NB; c += 4) {
    const float x = X[r][c];
    const float h = tf32_hi(x);
    lh[r * NB + c] = h;
    ll[r * NB + c] = x - h;
    if (r < nbk && c < nbk && c <= r) A[(size_t)(k0 + r) * m.ld + k0 + c] = S[r][c];
  }
}

// ---------------------------------------------------------------------------
// Sync-free triangular solves, one CTA (256 threads) per (matrix, 128-row block).
struct SolveArgs {
  BatchMat32 m;
  const float* lh;
  const float* ll;
  size_t l_bstride;
  const double* in;      // right-hand side (forward) / forward result (backward)
  double* out;           // result
  size_t ystride;
  int* flags;            // [batch][nblk] epoch of the last block completion
  int* ticket;
  int epoch;
  int nblk;
  int* err;
};

__device__ __forceinline__ int ld_acquire_flag(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Thread 0 of the waiting CTA polls with acquire loads; the CTA barrier after
// it orders the other threads' reads of the block behind the acquire.
__device__ bool wait_flag(const int* f, int epoch, int* err) {
  const long long lim = wait_limit_cycles();
  const long long t0 = clock64();
  while (ld_acquire_flag(f) != epoch) {
    if (*(volatile int*)err != 0 || clock64() - t0 > lim) {
      atomicCAS(err, 0, MBD_ERR_TIMEOUT);
      return false;
    }
    __nanosleep(64);
  }
  return true;
}

// The block's results are written by every thread before the CTA barrier;
// thread 0 then publishes them with a release store at GPU scope (cumulative
// over the writes the barrier ordered before it; no separate fence).
__device__ __forceinline__ void publish_flag(int* f, int epoch) {
  __syncthreads();
  if (threadIdx.x == 0) asm volatile("st.release.gpu.b32 [%0], %1;" ::"l"(f), "r"(epoch) : "memory");
}

// Forward: z_blk = Linv_blk (w_blk - sum_{k<blk} L_{blk,k} z_k).
// Warp w owns rows 16w..16w+15 of the block; lane l owns columns 4l..4l+3 of
// each 128-wide tile and keeps per-row partial sums until the end.
__global__ void __launch_bounds__(256) fwd_syncfree_kernel(SolveArgs a) {
  __shared__ int s_t;
  __shared__ double zk[NB][3];
  __shared__ double acc_s[NB][3];
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_t = atomicAdd(a.ticket, 1);
  __syncthreads();
  const int batch = a.m.batch;
  const int t = s_t;
  const int blk = t / batch, b = t % batch;
  const int n = a.m.n;
  const int r0 = blk * NB;
  const int nbk = min(NB, n - r0);
  const float* A = a.m.A + (size_t)b * a.m.stride;
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  double part[16][3];
#pragma unroll
  for (int u = 0; u < 16; ++u) part[u][0] = part[u][1] = part[u][2] = 0.0;
  for (int k = 0; k < blk; ++k) {
    if (threadIdx.x == 0) s_ok = wait_flag(a.flags + b * a.nblk + k, a.epoch, a.err);
    __syncthreads();
    if (!s_ok) return;
    for (int idx = threadIdx.x; idx < NB * 3; idx += blockDim.x)
      zk[idx / 3][idx % 3] = __ldcg(a.out + (size_t)b * a.ystride + (size_t)k * NB * 3 + idx);
    __syncthreads();
    const int c0 = k * NB + 4 * lane;
    const double z00 = zk[4 * lane][0], z01 = zk[4 * lane][1], z02 = zk[4 * lane][2];
    const double z10 = zk[4 * lane + 1][0], z11 = zk[4 * lane + 1][1], z12 = zk[4 * lane + 1][2];
    const double z20 = zk[4 * lane + 2][0], z21 = zk[4 * lane + 2][1], z22 = zk[4 * lane + 2][2];
    const double z30 = zk[4 * lane + 3][0], z31 = zk[4 * lane + 3][1], z32 = zk[4 * lane + 3][2];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const int row = r0 + warp * 16 + u;
      if (row < n) {
        const float4 l4 = *reinterpret_cast<const float4*>(A + (size_t)row * a.m.ld + c0);
        part[u][0] += l4.x * z00 + l4.y * z10 + l4.z * z20 + l4.w * z30;
        part[u][1] += l4.x * z01 + l4.y * z11 + l4.z * z21 + l4.w * z31;
        part[u][2] += l4.x * z02 + l4.y * z12 + l4.z * z22 + l4.w * z32;
      }
    }
  }
  // rhs - sum, gathered per row
#pragma unroll
  for (int u = 0; u < 16; ++u) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      double v = part[u][q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      part[u][q] = v;
    }
    const int rr = warp * 16 + u;
    if (lane < 3) {
      const double rhs = (rr < nbk) ? a.in[(size_t)b * a.ystride + (size_t)(r0 + rr) * 3 + lane] : 0.0;
      acc_s[rr][lane] = rhs - (lane == 0 ? part[u][0] : lane == 1 ? part[u][1] : part[u][2]);
    }
  }
  __syncthreads();
  // z_blk = Linv_blk acc (lower triangular)
  const float* Lh = a.lh + (size_t)b * a.l_bstride + (size_t)r0 * NB;
  const float* Ll = a.ll + (size_t)b * a.l_bstride + (size_t)r0 * NB;
  for (int idx = threadIdx.x; idx < NB * 3; idx += blockDim.x) {
    const int rr = idx / 3, q = idx % 3;
    double s = 0.0;
    for (int l = 0; l <= rr; ++l) s += ((double)Lh[rr * NB + l] + (double)Ll[rr * NB + l]) * acc_s[l][q];
    if (rr < nbk) a.out[(size_t)b * a.ystride + (size_t)(r0 + rr) * 3 + q] = s;
  }
  publish_flag(a.flags + b * a.nblk + blk, a.epoch);
}

// Backward: x_blk = Linv_blk^T (z_blk - sum_{k>blk} L_{k,blk}^T x_k).
// Thread t owns column c = t/2 of the block (half-row split by t%2).
__global__ void __launch_bounds__(256) bwd_syncfree_kernel(SolveArgs a) {
  __shared__ int s_t;
  __shared__ double xk[NB][3];
  __shared__ double acc_s[NB][3];
  __shared__ int s_ok;
  if (threadIdx.x == 0) s_t = atomicAdd(a.ticket, 1);
  __syncthreads();
  const int batch = a.m.batch;
  const int t = s_t;
  const int blk = a.nblk - 1 - t / batch, b = t % batch;
  const int n = a.m.n;
  const int c0 = blk * NB;
  const int nbk = min(NB, n - c0);
  const float* A = a.m.A + (size_t)b * a.m.stride;
  const int c = threadIdx.x % NB, half = threadIdx.x / NB;
  double p0 = 0.0, p1 = 0.0, p2 = 0.0;
  for (int k = a.nblk - 1; k > blk; --k) {
    if (threadIdx.x == 0) s_ok = wait_flag(a.flags + b * a.nblk + k, a.epoch, a.err);
    __syncthreads();
    if (!s_ok) return;
    for (int idx = threadIdx.x; idx < NB * 3; idx += blockDim.x)
      xk[idx / 3][idx % 3] = __ldcg(a.out + (size_t)b * a.ystride + (size_t)k * NB * 3 + idx);
    __syncthreads();
    const int kr = min(NB, n - k * NB);
    for (int rr = half; rr < kr; rr += 2) {
      const double l = A[(size_t)(k * NB + rr) * a.m.ld + c0 + c];
      p0 += l * xk[rr][0];
      p1 += l * xk[rr][1];
      p2 += l * xk[rr][2];
    }
    __syncthreads();
  }
  // combine the two row halves through shared memory
  __shared__ double hsum[2][NB][3];
  hsum[half][c][0] = p0;
  hsum[half][c][1] = p1;
  hsum[half][c][2] = p2;
  __syncthreads();
  for (int idx = threadIdx.x; idx < NB * 3; idx += blockDim.x) {
    const int cc = idx / 3, q = idx % 3;
    const double zin = (cc < nbk) ? a.in[(size_t)b * a.ystride + (size_t)(c0 + cc) * 3 + q] : 0.0;
    acc_s[cc][q] = zin - hsum[0][cc][q] - hsum[1][cc][q];
  }
  __syncthreads();
  const float* Lh = a.lh + (size_t)b * a.l_bstride + (size_t)c0 * NB;
  const float* Ll = a.ll + (size_t)b * a.l_bstride + (size_t)c0 * NB;
  for (int idx = threadIdx.x; idx < NB * 3; idx += blockDim.x) {
    const int rr = idx / 3, q = idx % 3;
    double s = 0.0;
    for (int l = rr; l < NB; ++l) s += ((double)Lh[l * NB + rr] + (double)Ll[l * NB + rr]) * acc_s[l][q];
    if (rr < nbk) a.out[(size_t)b * a.ystride + (size_t)(c0 + rr) * 3 + q] = s;
  }
  publish_flag(a.flags + b * a.nblk + blk, a.epoch);
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

size_t solve_sync_ints(int n, int batch) { return (size_t)batch * ((n + NB - 1) / NB) + 8; }

void launch_solve_f32(const BatchMat32& m, const float* linv_hi, const float* linv_lo, size_t l_bstride, double* R,
                      double* Z, double* D, size_t ystride, int* sync, int epoch, int* err, cudaStream_t s) {
  const int nblk = (m.n + NB - 1) / NB;
  int* ticket = sync;                 // [0] forward ticket, [1] backward ticket
  int* flags = sync + 8;              // [batch][nblk]
  cudaMemsetAsync(ticket, 0, 2 * sizeof(int), s);
  SolveArgs fa{m, linv_hi, linv_lo, l_bstride, R, Z, ystride, flags, ticket, 2 * epoch + 1, nblk, err};
  fwd_syncfree_kernel<<<nblk * m.batch, 256, 0, s>>>(fa);
  SolveArgs ba{m, linv_hi, linv_lo, l_bstride, Z, D, ystride, flags, ticket + 1, 2 * epoch + 2, nblk, err};
  bwd_syncfree_kernel<<<nblk * m.batch, 256, 0, s>>>(ba);
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

MBD_WAIT_LIMIT_SETTER(set_wait_limit_mixed)

}  // namespace mbd
