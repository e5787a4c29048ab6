// Message-passing network of the learned relay warm start: forward pass,
// loss, backward pass and Adam, FP32, one graph per geometry with the 21
// imaginary frequencies as 21 copies of the atom graph (node = f * N + i).
//
//   x      = [onehot(H, C, N, O, other), h_i, log alpha_i(iw_f), log(1 + w_f)]
//   h0     = silu(W0 x + b0)
//   layer l = 0..2:  m_i = sum_j (Wf_l e_ij) * h_j;  h_i += silu(Wu_l m_i + bu_l)
//   s_i = ws.h_i + bs,  a_i = wa.h_i + ca,  g_ij = wg.e_ij
//   S_i = (1 + s_i) I + sum_j a_j g_ij (u_ij u_ij^T - I/3),   X_i = alpha_i S_i
// e_ij: 16 Gaussian radial functions of |r_ij| times a cosine cut-off at 5 A;
// u_ij the unit vector from i to j.  Neighbour lists are symmetric (j in
// nbr(i) <=> i in nbr(j) with the same distance), so every backward scatter
// is written as a gather over the receiving node's own list.
#include <cuda_runtime.h>

#include "gnn.h"

namespace mbd {
namespace {

constexpr int H = kGnnHidden;
constexpr int NR = kGnnRbf;
constexpr int NI = kGnnIn;

__device__ __forceinline__ float sigm(float z) { return 1.0f / (1.0f + __expf(-z)); }
__device__ __forceinline__ float silu(float z) { return z * sigm(z); }
__device__ __forceinline__ float dsilu(float z) {
  const float s = sigm(z);
  return s * (1.0f + z * (1.0f - s));
}

__global__ void edge_kernel(const float* dvec, int E, float* efeat, float* eproj) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= E) return;
  const float dx = dvec[3 * e], dy = dvec[3 * e + 1], dz = dvec[3 * e + 2];
  const float r = sqrtf(dx * dx + dy * dy + dz * dz);
  const float ir = 1.0f / r;
  const float ux = dx * ir, uy = dy * ir, uz = dz * ir;
  const float rc = kGnnCutoffBohr;
  const float w = rc / (NR - 1);
  const float fc = 0.5f * (cosf(3.14159265358979f * r / rc) + 1.0f);
#pragma unroll
  for (int k = 0; k < NR; ++k) {
    const float t = (r - w * k) / w;
    efeat[(size_t)e * NR + k] = __expf(-0.5f * t * t) * fc;
  }
  float* p = eproj + (size_t)e * 6;
  p[0] = ux * ux - 1.0f / 3.0f;
  p[1] = uy * uy - 1.0f / 3.0f;
  p[2] = uz * uz - 1.0f / 3.0f;
  p[3] = ux * uy;
  p[4] = ux * uz;
  p[5] = uy * uz;
}

__global__ void features_kernel(const int* species, const double* hirsh, const double* alpha_w, const double* omega,
                                int N, int F, float* x) {
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N * F) return;
  const int f = node / N, i = node % N;
  float* xo = x + (size_t)node * NI;
  const int sp = species[i];
#pragma unroll
  for (int k = 0; k < 5; ++k) xo[k] = (k == sp) ? 1.0f : 0.0f;
  xo[5] = (float)hirsh[i];
  xo[6] = (float)log(alpha_w[(size_t)f * N + i]);
  xo[7] = (float)log1p(omega[f]);
}

// filt[l][e][k] = Wf_l[k] . e_e (l = 0..2), g[e] = wg . e_e
__global__ void filter_kernel(const float* P, const float* efeat, int E, float* filt, float* g) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long total = (long long)E * (kGnnLayers * H + 1);
  if (idx >= total) return;
  const int e = (int)(idx / (kGnnLayers * H + 1));
  const int c = (int)(idx % (kGnnLayers * H + 1));
  const float* ee = efeat + (size_t)e * NR;
  if (c == kGnnLayers * H) {
    const float* wg = P + kGnnOffWg;
    float s = 0.f;
#pragma unroll
    for (int q = 0; q < NR; ++q) s += wg[q] * ee[q];
    g[e] = s;
    return;
  }
  const int l = c / H, k = c % H;
  const float* W = P + kGnnOffWf(l) + k * NR;
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < NR; ++q) s += W[q] * ee[q];
  filt[((size_t)l * E + e) * H + k] = s;
}

__global__ void embed_kernel(const float* P, const float* x, int M, float* pre0, float* h0) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)M * H) return;
  const int node = (int)(idx / H), k = (int)(idx % H);
  const float* W = P + kGnnOffW0 + k * NI;
  const float* xi = x + (size_t)node * NI;
  float s = P[kGnnOffB0 + k];
#pragma unroll
  for (int q = 0; q < NI; ++q) s += W[q] * xi[q];
  pre0[idx] = s;
  h0[idx] = silu(s);
}

// m[f*N+i][k] = sum_{e in nbr(i)} filt[e][k] h[f*N+nbr[e]][k]
__global__ void conv_kernel(const float* h, const float* filt, const int* off, const int* nbr, int N, int F,
                            float* m) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)N * F * H) return;
  const int node = (int)(idx / H), k = (int)(idx % H);
  const int f = node / N, i = node % N;
  const float* hf = h + (size_t)f * N * H;
  float s = 0.f;
  for (int e = off[i]; e < off[i + 1]; ++e) s += filt[(size_t)e * H + k] * hf[(size_t)nbr[e] * H + k];
  m[idx] = s;
}

// u = Wu m + bu; h_out = h_in + silu(u).  256 threads = 4 nodes x 64 outputs.
__global__ void __launch_bounds__(256) dense_kernel(const float* P, int l, const float* m, const float* h_in,
                                                    float* u, float* h_out, int M) {
  __shared__ float Wt[H][H + 1];   // Wt[q][k] = Wu[k][q]
  __shared__ float ms[4][H];
  const float* W = P + kGnnOffWu(l);
  for (int t = threadIdx.x; t < H * H; t += blockDim.x) Wt[t % H][t / H] = W[t];
  const float bk = P[kGnnOffBu(l) + threadIdx.x % H];
  const int k = threadIdx.x % H, sub = threadIdx.x / H;
  for (int n0 = blockIdx.x * 4; n0 < M; n0 += gridDim.x * 4) {
    __syncthreads();
    const int node = n0 + sub;
    ms[sub][k] = node < M ? m[(size_t)node * H + k] : 0.f;
    __syncthreads();
    if (node < M) {
      float s = bk;
#pragma unroll 16
      for (int q = 0; q < H; ++q) s += Wt[q][k] * ms[sub][q];
      u[(size_t)node * H + k] = s;
      h_out[(size_t)node * H + k] = h_in[(size_t)node * H + k] + silu(s);
    }
  }
}

// s = ws.h + bs, a = wa.h + ca (one warp per node)
__global__ void sa_kernel(const float* P, const float* h, int M, float* s, float* a) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) / 32, lane = threadIdx.x % 32;
  if (warp >= M) return;
  const float* hn = h + (size_t)warp * H;
  float vs = P[kGnnOffWs + lane] * hn[lane] + P[kGnnOffWs + lane + 32] * hn[lane + 32];
  float va = P[kGnnOffWa + lane] * hn[lane] + P[kGnnOffWa + lane + 32] * hn[lane + 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vs += __shfl_xor_sync(0xffffffffu, vs, o);
    va += __shfl_xor_sync(0xffffffffu, va, o);
  }
  if (lane == 0) {
    s[warp] = vs + P[kGnnOffBs];
    a[warp] = va + P[kGnnOffCa];
  }
}

// S (row-major 3x3) per node
__global__ void tensor_kernel(const float* s, const float* a, const float* g, const float* eproj, const int* off,
                              const int* nbr, int N, int F, float* S) {
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N * F) return;
  const int f = node / N, i = node % N;
  float p[6] = {0, 0, 0, 0, 0, 0};
  for (int e = off[i]; e < off[i + 1]; ++e) {
    const float w = a[(size_t)f * N + nbr[e]] * g[e];
#pragma unroll
    for (int c = 0; c < 6; ++c) p[c] += w * eproj[(size_t)e * 6 + c];
  }
  const float d = 1.0f + s[node];
  float* o = S + (size_t)node * 9;
  o[0] = d + p[0];
  o[4] = d + p[1];
  o[8] = d + p[2];
  o[1] = o[3] = p[3];
  o[2] = o[6] = p[4];
  o[5] = o[7] = p[5];
}

// dS = 2 (S - S_true) / M; loss += ||S - S_true||^2 / M
__global__ void loss_kernel(const float* S, const float* St, int M, float* dS, double* loss) {
  __shared__ double red[256];
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  double l = 0.0;
  if (node < M) {
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const float d = S[(size_t)node * 9 + c] - St[(size_t)node * 9 + c];
      dS[(size_t)node * 9 + c] = 2.0f * d / (float)M;
      l += (double)d * d;
    }
  }
  red[threadIdx.x] = l;
  __syncthreads();
  for (int h = blockDim.x / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) red[threadIdx.x] += red[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicAdd(loss, red[0] / M);
}

__device__ __forceinline__ float dot_proj(const float* dS, const float* p) {
  return dS[0] * p[0] + dS[4] * p[1] + dS[8] * p[2] + (dS[1] + dS[3]) * p[3] + (dS[2] + dS[6]) * p[4] +
         (dS[5] + dS[7]) * p[5];
}

// ds = tr dS; da_j = sum_{e in nbr(j)} g_e <dS_nbr, P_e>; cw[f][e] = <dS_i, P_e> a_nbr
__global__ void readout_bwd_kernel(const float* dS, const float* a, const float* g, const float* eproj,
                                   const int* off, const int* nbr, int N, int F, int E, float* ds, float* da,
                                   float* cw) {
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= N * F) return;
  const int f = node / N, i = node % N;
  const float* dSi = dS + (size_t)node * 9;
  ds[node] = dSi[0] + dSi[4] + dSi[8];
  float acc = 0.f;
  for (int e = off[i]; e < off[i + 1]; ++e) {
    const int j = f * N + nbr[e];
    const float* pe = eproj + (size_t)e * 6;
    acc += g[e] * dot_proj(dS + (size_t)j * 9, pe);
    cw[(size_t)f * E + e] = dot_proj(dSi, pe) * a[j];
  }
  da[node] = acc;
}

// dh = ds ws + da wa
__global__ void readout_dh_kernel(const float* P, const float* ds, const float* da, int M, float* dh) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)M * H) return;
  const int node = (int)(idx / H), k = (int)(idx % H);
  dh[idx] = ds[node] * P[kGnnOffWs + k] + da[node] * P[kGnnOffWa + k];
}

// du = dh * silu'(u); dm = Wu^T du.  256 threads = 4 nodes x 64.
__global__ void __launch_bounds__(256) dense_bwd_kernel(const float* P, int l, const float* dh, const float* u,
                                                        float* du, float* dm, int M) {
  __shared__ float W[H][H + 1];   // W[k][q]
  __shared__ float ds_[4][H];
  const float* Wg = P + kGnnOffWu(l);
  for (int t = threadIdx.x; t < H * H; t += blockDim.x) W[t / H][t % H] = Wg[t];
  const int q = threadIdx.x % H, sub = threadIdx.x / H;
  for (int n0 = blockIdx.x * 4; n0 < M; n0 += gridDim.x * 4) {
    __syncthreads();
    const int node = n0 + sub;
    float d = 0.f;
    if (node < M) {
      d = dh[(size_t)node * H + q] * dsilu(u[(size_t)node * H + q]);
      du[(size_t)node * H + q] = d;
    }
    ds_[sub][q] = d;
    __syncthreads();
    if (node < M) {
      float s = 0.f;
#pragma unroll 16
      for (int k = 0; k < H; ++k) s += W[k][q] * ds_[sub][k];
      dm[(size_t)node * H + q] = s;
    }
  }
}

// dh_out[j] = dh_next[j] + sum_{e in nbr(j)} filt[e] * dm[nbr_e]
__global__ void conv_bwd_kernel(const float* dh_next, const float* dm, const float* filt, const int* off,
                                const int* nbr, int N, int F, float* dh_out) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)N * F * H) return;
  const int node = (int)(idx / H), k = (int)(idx % H);
  const int f = node / N, i = node % N;
  const float* dmf = dm + (size_t)f * N * H;
  float s = dh_next[idx];
  for (int e = off[i]; e < off[i + 1]; ++e) s += filt[(size_t)e * H + k] * dmf[(size_t)nbr[e] * H + k];
  dh_out[idx] = s;
}

// dfilt[e][k] = sum_f dm[f, src_e][k] h[f, nbr_e][k]
__global__ void dfilt_kernel(const float* dm, const float* h, const int* src, const int* nbr, int N, int F, int E,
                             float* dfilt) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)E * H) return;
  const int e = (int)(idx / H), k = (int)(idx % H);
  const int i = src[e], j = nbr[e];
  float s = 0.f;
  for (int f = 0; f < F; ++f) s += dm[((size_t)f * N + i) * H + k] * h[((size_t)f * N + j) * H + k];
  dfilt[idx] = s;
}

// dpre = dh * silu'(pre0) (in place into dh)
__global__ void embed_bwd_kernel(float* dh, const float* pre0, int M) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)M * H) return;
  dh[idx] *= dsilu(pre0[idx]);
}

// out[k1][k2] += sum_r A[r][k1] B[r % bmod][k2]  (B == nullptr: B = 1, K2 = 1).
// Each CTA sums a chunk of 64 rows in registers, then adds atomically.
constexpr int kOuterRows = 64;
__global__ void __launch_bounds__(256) outer_kernel(const float* A, int K1, const float* B, int K2, long long rows,
                                                    long long bmod, float* out) {
  __shared__ float As[kOuterRows][H + 1];
  __shared__ float Bs[kOuterRows][H + 1];
  const int nout = K1 * K2;
  float acc[16];
#pragma unroll
  for (int t = 0; t < 16; ++t) acc[t] = 0.f;
  for (long long r0 = (long long)blockIdx.x * kOuterRows; r0 < rows; r0 += (long long)gridDim.x * kOuterRows) {
    __syncthreads();
    for (int t = threadIdx.x; t < kOuterRows * K1; t += blockDim.x) {
      const int rr = t / K1, c = t % K1;
      const long long r = r0 + rr;
      As[rr][c] = r < rows ? A[r * K1 + c] : 0.f;
    }
    for (int t = threadIdx.x; t < kOuterRows * K2; t += blockDim.x) {
      const int rr = t / K2, c = t % K2;
      const long long r = r0 + rr;
      Bs[rr][c] = (r < rows) ? (B ? B[(r % bmod) * K2 + c] : 1.0f) : 0.f;
    }
    __syncthreads();
#pragma unroll
    for (int t = 0; t < 16; ++t) {
      const int o = threadIdx.x + 256 * t;
      if (o < nout) {
        const int k1 = o / K2, k2 = o % K2;
        float s = 0.f;
        for (int rr = 0; rr < kOuterRows; ++rr) s += As[rr][k1] * Bs[rr][k2];
        acc[t] += s;
      }
    }
  }
#pragma unroll
  for (int t = 0; t < 16; ++t) {
    const int o = threadIdx.x + 256 * t;
    if (o < nout) atomicAdd(out + o, acc[t]);
  }
}

__global__ void adam_kernel(float* P, float* G, float* m1, float* m2, int n, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float g = G[i];
  const float a = b1 * m1[i] + (1.f - b1) * g;
  const float b = b2 * m2[i] + (1.f - b2) * g * g;
  m1[i] = a;
  m2[i] = b;
  P[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  G[i] = 0.f;
}

// X0[f][3i+r][c] = alpha_w[f][i] S[f*N+i][r][c]
__global__ void warmstart_kernel(const float* S, const double* alpha_w, int N, int F, double* X, size_t ystride) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)N * F * 9) return;
  const int node = (int)(idx / 9), c = (int)(idx % 9);
  const int f = node / N, i = node % N;
  X[(size_t)f * ystride + (size_t)9 * i + c] = alpha_w[(size_t)f * N + i] * (double)S[idx];
}

// S_true[f*N+i][r][c] = X[f][3i+r][c] / alpha_w[f][i]
__global__ void targets_kernel(const double* X, size_t ystride, const double* alpha_w, int N, int F, float* St) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)N * F * 9) return;
  const int node = (int)(idx / 9), c = (int)(idx % 9);
  const int f = node / N, i = node % N;
  St[idx] = (float)(X[(size_t)f * ystride + (size_t)9 * i + c] / alpha_w[(size_t)f * N + i]);
}

// ---- the network's neighbour lists (radius graph), built on the device ----
// Every (atom i, image t, atom j) is tested with one warp per atom i, lanes
// over j; a ballot orders each warp's edges by (image, j), so the lists come
// out deterministic.  Coordinates are in bohr; the translations and distances
// use explicitly rounded FP64 operations (no contraction), so the count pass
// and the fill pass take the same decisions.

__device__ __forceinline__ void image_shift(const GraphBox& b, int n0, int n1, int n2, double* t) {
#pragma unroll
  for (int c = 0; c < 3; ++c)
    t[c] = __dadd_rn(__dadd_rn(__dmul_rn((double)n0, b.lat[c]), __dmul_rn((double)n1, b.lat[3 + c])),
                     __dmul_rn((double)n2, b.lat[6 + c]));
}

// false when no atom of image t can lie within the cut-off of xi (xi outside
// the image's bounding box widened by the cut-off and a rounding margin)
__device__ __forceinline__ bool image_near(const GraphBox& b, const double* xi, const double* t) {
  bool near = true;
#pragma unroll
  for (int c = 0; c < 3; ++c) near = near && xi[c] >= b.lo[c] + t[c] - b.pad && xi[c] <= b.hi[c] + t[c] + b.pad;
  return near;
}

template <bool FILL>
__global__ void __launch_bounds__(256) graph_kernel(const double* __restrict__ x, int N, GraphBox b,
                                                    const int* __restrict__ off_in, int* cnt_or_off,
                                                    int* __restrict__ nbr, int* __restrict__ src,
                                                    float* __restrict__ dvec) {
  const int lane = threadIdx.x & 31;
  const int i = (int)((blockIdx.x * (unsigned)blockDim.x + threadIdx.x) >> 5);
  if (i >= N) return;   // whole warps
  const double xi[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
  int pos = FILL ? off_in[i] : 0;
  if (FILL && lane == 0) {
    cnt_or_off[i] = pos;
    if (i == N - 1) cnt_or_off[N] = off_in[N];
  }
  for (int n0 = -b.rng[0]; n0 <= b.rng[0]; ++n0)
    for (int n1 = -b.rng[1]; n1 <= b.rng[1]; ++n1)
      for (int n2 = -b.rng[2]; n2 <= b.rng[2]; ++n2) {
        double t[3];
        image_shift(b, n0, n1, n2, t);
        if (!image_near(b, xi, t)) continue;   // uniform over the warp
        for (int j0 = 0; j0 < N; j0 += 32) {
          const int j = j0 + lane;
          bool ok = false;
          double d[3] = {0.0, 0.0, 0.0};
          if (j < N) {
#pragma unroll
            for (int c = 0; c < 3; ++c) d[c] = __dsub_rn(__dadd_rn(x[3 * j + c], t[c]), xi[c]);
            const double r2 = __dadd_rn(__dadd_rn(__dmul_rn(d[0], d[0]), __dmul_rn(d[1], d[1])), __dmul_rn(d[2], d[2]));
            ok = r2 < b.rc2 && r2 >= 1e-12;   // the atom itself (zero shift) has r = 0
          }
          const unsigned m = __ballot_sync(0xffffffffu, ok);
          if (FILL && ok) {
            const int e = pos + __popc(m & ((1u << lane) - 1u));
            nbr[e] = j;
            src[e] = i;
            dvec[3 * (size_t)e] = (float)d[0];
            dvec[3 * (size_t)e + 1] = (float)d[1];
            dvec[3 * (size_t)e + 2] = (float)d[2];
          }
          pos += __popc(m);
        }
      }
  if (!FILL && lane == 0) cnt_or_off[i] = pos;
}

// In-place exclusive scan of a[0..N) by one CTA; a[N] = *E = the total.
__global__ void __launch_bounds__(1024) graph_scan_kernel(int* a, int N, int* E) {
  __shared__ int wsum[32];
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  const int chunk = (N + 1023) / 1024;
  const int b0 = min(N, t * chunk), b1 = min(N, b0 + chunk);
  int mine = 0;
  for (int k = b0; k < b1; ++k) mine += a[k];
  int v = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) wsum[w] = v;
  __syncthreads();
  if (w == 0) {
    int q = wsum[lane];
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, q, o);
      if (lane >= o) q += u;
    }
    wsum[lane] = q;
  }
  __syncthreads();
  int run = v - mine + (w > 0 ? wsum[w - 1] : 0);
  for (int k = b0; k < b1; ++k) {
    const int c = a[k];
    a[k] = run;
    run += c;
  }
  if (t == 0) {
    a[N] = wsum[31];
    *E = wsum[31];
  }
}

inline unsigned blocks(long long n, int t) { return (unsigned)((n + t - 1) / t); }

void outer(const float* A, int K1, const float* B, int K2, long long rows, long long bmod, float* out,
           cudaStream_t s) {
  if (rows <= 0) return;
  const long long chunks = (rows + kOuterRows - 1) / kOuterRows;
  const unsigned g = (unsigned)(chunks < 592 ? chunks : 592);
  outer_kernel<<<g, 256, 0, s>>>(A, K1, B, K2, rows, bmod, out);
}

}  // namespace

size_t gnn_work_floats(int N, int F, int E, bool train) {
  const size_t M = (size_t)N * F;
  size_t f = M * H * (1 + 4 + 3 + 3)          // pre0, h0..h3, m0..m2, u0..u2
             + (size_t)kGnnLayers * E * H + E // filt, g
             + 2 * M + 9 * M;                 // s, a, S
  if (train) f += 9 * M + 4 * M * H + 2 * M + (size_t)E * H + (size_t)F * E + 9 * M;   // dS, dh*, ds/da, dfilt, cw, S_true
  return f + 512;   // 8-float alignment of every array of the layout
}

GnnWork gnn_work_layout(float* base, int N, int F, int E, bool train) {
  const size_t M = (size_t)N * F;
  GnnWork w{};
  float* p = base;
  auto take = [&](size_t n) {
    float* q = p;
    p += (n + 7) & ~size_t(7);
    return q;
  };
  w.pre0 = take(M * H);
  for (int l = 0; l <= kGnnLayers; ++l) w.h[l] = take(M * H);
  for (int l = 0; l < kGnnLayers; ++l) w.m[l] = take(M * H);
  for (int l = 0; l < kGnnLayers; ++l) w.u[l] = take(M * H);
  w.filt = take((size_t)kGnnLayers * E * H);
  w.g = take(E);
  w.s = take(M);
  w.a = take(M);
  w.S = take(9 * M);
  if (train) {
    w.dS = take(9 * M);
    w.dh = take(M * H);
    w.dh2 = take(M * H);
    w.du = take(M * H);
    w.dm = take(M * H);
    w.ds = take(M);
    w.da = take(M);
    w.dfilt = take((size_t)E * H);
    w.cw = take((size_t)F * E);
    w.S_true = take(9 * M);
  }
  return w;
}

void gnn_graph_count(const double* x, int N, const GraphBox& b, int* cnt, cudaStream_t s) {
  graph_kernel<false><<<blocks(32LL * N, 256), 256, 0, s>>>(x, N, b, nullptr, cnt, nullptr, nullptr, nullptr);
}

void gnn_graph_scan(int* cnt_off, int N, int* E, cudaStream_t s) {
  graph_scan_kernel<<<1, 1024, 0, s>>>(cnt_off, N, E);
}

void gnn_graph_fill(const double* x, int N, const GraphBox& b, const int* off_in, int* off, int* nbr, int* src,
                    float* dvec, cudaStream_t s) {
  graph_kernel<true><<<blocks(32LL * N, 256), 256, 0, s>>>(x, N, b, off_in, off, nbr, src, dvec);
}

void gnn_edges(const float* dvec, int E, float* efeat, float* eproj, cudaStream_t s) {
  if (E > 0) edge_kernel<<<blocks(E, 256), 256, 0, s>>>(dvec, E, efeat, eproj);
}

void gnn_features(const int* species, const double* hirsh, const double* alpha_w, const double* omega, int N, int F,
                  float* x, cudaStream_t s) {
  features_kernel<<<blocks((long long)N * F, 256), 256, 0, s>>>(species, hirsh, alpha_w, omega, N, F, x);
}

int gnn_forward(const float* P, const GnnGraph& g, const GnnWork& w, cudaStream_t s) {
  const int M = g.N * g.F;
  if (g.E > 0)
    filter_kernel<<<blocks((long long)g.E * (kGnnLayers * H + 1), 256), 256, 0, s>>>(P, g.efeat, g.E, w.filt, w.g);
  embed_kernel<<<blocks((long long)M * H, 256), 256, 0, s>>>(P, g.x, M, w.pre0, w.h[0]);
  const unsigned dg = blocks(M, 4) < 1184 ? blocks(M, 4) : 1184;
  for (int l = 0; l < kGnnLayers; ++l) {
    conv_kernel<<<blocks((long long)M * H, 256), 256, 0, s>>>(w.h[l], w.filt + (size_t)l * g.E * H, g.off, g.nbr,
                                                              g.N, g.F, w.m[l]);
    dense_kernel<<<dg, 256, 0, s>>>(P, l, w.m[l], w.h[l], w.u[l], w.h[l + 1], M);
  }
  sa_kernel<<<blocks((long long)M * 32, 256), 256, 0, s>>>(P, w.h[kGnnLayers], M, w.s, w.a);
  tensor_kernel<<<blocks(M, 128), 128, 0, s>>>(w.s, w.a, w.g, g.eproj, g.off, g.nbr, g.N, g.F, w.S);
  return 3 + 2 * kGnnLayers + (g.E > 0 ? 1 : 0);
}

int gnn_loss_backward(const float* P, const GnnGraph& g, const GnnWork& w, float* G, double* loss, cudaStream_t s) {
  const int M = g.N * g.F;
  int launches = 0;
  loss_kernel<<<blocks(M, 256), 256, 0, s>>>(w.S, w.S_true, M, w.dS, loss);
  readout_bwd_kernel<<<blocks(M, 128), 128, 0, s>>>(w.dS, w.a, w.g, g.eproj, g.off, g.nbr, g.N, g.F, g.E, w.ds, w.da,
                                                     w.cw);
  readout_dh_kernel<<<blocks((long long)M * H, 256), 256, 0, s>>>(P, w.ds, w.da, M, w.dh);
  launches += 3;
  const float* h3 = w.h[kGnnLayers];
  outer(w.ds, 1, h3, H, M, M, G + kGnnOffWs, s);
  outer(w.ds, 1, nullptr, 1, M, 1, G + kGnnOffBs, s);
  outer(w.da, 1, h3, H, M, M, G + kGnnOffWa, s);
  outer(w.da, 1, nullptr, 1, M, 1, G + kGnnOffCa, s);
  if (g.E > 0) outer(w.cw, 1, g.efeat, kGnnRbf, (long long)g.F * g.E, g.E, G + kGnnOffWg, s);
  launches += 5;
  const unsigned dg = blocks(M, 4) < 1184 ? blocks(M, 4) : 1184;
  float* dh = w.dh;
  float* dh_alt = w.dh2;
  for (int l = kGnnLayers - 1; l >= 0; --l) {
    dense_bwd_kernel<<<dg, 256, 0, s>>>(P, l, dh, w.u[l], w.du, w.dm, M);
    outer(w.du, H, w.m[l], H, M, M, G + kGnnOffWu(l), s);
    outer(w.du, H, nullptr, 1, M, 1, G + kGnnOffBu(l), s);
    conv_bwd_kernel<<<blocks((long long)M * H, 256), 256, 0, s>>>(dh, w.dm, w.filt + (size_t)l * g.E * H, g.off,
                                                                  g.nbr, g.N, g.F, dh_alt);
    launches += 4;
    if (g.E > 0) {
      dfilt_kernel<<<blocks((long long)g.E * H, 256), 256, 0, s>>>(w.dm, w.h[l], g.src, g.nbr, g.N, g.F, g.E,
                                                                   w.dfilt);
      outer(w.dfilt, H, g.efeat, kGnnRbf, g.E, g.E, G + kGnnOffWf(l), s);
      launches += 2;
    }
    float* t = dh;
    dh = dh_alt;
    dh_alt = t;
  }
  embed_bwd_kernel<<<blocks((long long)M * H, 256), 256, 0, s>>>(dh, w.pre0, M);
  outer(dh, H, g.x, kGnnIn, M, M, G + kGnnOffW0, s);
  outer(dh, H, nullptr, 1, M, 1, G + kGnnOffB0, s);
  return launches + 3;
}

void gnn_adam(float* P, float* G, float* m1, float* m2, int step, float lr, cudaStream_t s) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
  adam_kernel<<<blocks(kGnnParams, 256), 256, 0, s>>>(P, G, m1, m2, kGnnParams, lr, b1, b2, 1e-8f, c1, c2);
}

void gnn_warmstart(const float* S, const double* alpha_w, int N, int F, double* X, size_t ystride, cudaStream_t s) {
  warmstart_kernel<<<blocks((long long)N * F * 9, 256), 256, 0, s>>>(S, alpha_w, N, F, X, ystride);
}

void gnn_targets(const double* X, size_t ystride, const double* alpha_w, int N, int F, float* St, cudaStream_t s) {
  targets_kernel<<<blocks((long long)N * F * 9, 256), 256, 0, s>>>(X, ystride, alpha_w, N, F, St);
}

}  // namespace mbd
