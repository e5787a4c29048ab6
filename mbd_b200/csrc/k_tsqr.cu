// Panel QR of the dense -> band reduction (stage 1 of the two-stage
// reduction behind PDSYEV('N','L'), UTILS.f90:835) by TSQR with Householder
// reconstruction, FP64, in one thread-block cluster.
//
// The panel P = A[row0 .. row0 + m)[col0 .. col0 + 32) is split over the C
// CTAs of the cluster (R rows each).  Instead of one cluster-wide exchange
// per column (the Householder QR of k_sy2sb.cu), the cluster meets three
// times per panel:
//   1. every CTA: Householder QR of its own rows (CTA barriers only), local
//      compact-WY factor T_c and R_c; R_c goes to rank 0;            barrier 1
//   2. rank 0: Householder QR of the stacked R_c (32 C x 32; each block is
//      upper triangular, so only its fill is touched), explicit Q of that
//      tree, block c of it to CTA c;                                 barrier 2
//   3. every CTA: its rows of the panel's explicit Q,
//        Q_c = (I - V_c T_c V_c^T) [Q_tree,c; 0];
//      rank 0 reconstructs Householder vectors from the top 32 rows Q_1
//      (Ballard, Demmel, Grigori, Jacquelin, Nguyen, Solomonik, "Reconstructing
//      Householder vectors from tall-skinny QR", IPDPS 2014):
//        S = -sign(diag Q_1),  Q_1 - S = L_1 U (LU without pivoting),
//        V = [L_1; Q_2 U^-1],  T = -U S L_1^-T,  R_band = S R_tree,
//      so that P = (I - V T V^T) [R_band; 0]; U and S go to every CTA;  barrier 3
//   4. every CTA: V = Q U^-1 for its rows below the top 32.
// V (unit lower trapezoidal), T (upper triangular) and the band rows are the
// outputs of the per-column kernel, with the same meaning, so the trailing
// update is unchanged.  Pivots of Q_1 - S are at least 1 in magnitude by the
// choice of S, so the LU needs no pivoting.  A rank-deficient or zero panel
// is fine: its TSQR is still orthogonal (zero columns give tau = 0).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace mbd {
namespace {

constexpr int B = kBand;     // 32
constexpr int NW = 8;
constexpr int NT = NW * 32;
constexpr int LDT = B + 1;
constexpr unsigned FULL = 0xffffffffu;
constexpr int kTsqrMaxCluster = 16;

// One Householder step on column j of a block whose rows this thread block
// holds in registers (lane = column, warp w holds rows w + NW t), given the
// block's row count nr.  Returns tau; leaves v in x[.] of lane j below row j,
// beta at row j, and updates the columns right of j.  Column j of the
// compact-WY factor T (dlarft, forward) is formed by warp 0 from the same
// dots.  Two CTA barriers.
template <int RPW>
__device__ __forceinline__ void house_step(double (&x)[RPW], int j, int nr, double* nw, double* s_alpha,
                                           double (*dw)[B], double* gs, double (*Tm)[LDT]) {
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    if (r > j && r < nr) s += x[t] * x[t];
  }
  s = __shfl_sync(FULL, s, j);
  if (lane == 0) nw[warp] = s;
  if (j % NW == warp && lane == j) *s_alpha = (j < nr) ? x[j / NW] : 0.0;
  __syncthreads();
  double xn2 = 0.0;
#pragma unroll
  for (int w = 0; w < NW; ++w) xn2 += nw[w];
  const double alpha = *s_alpha;
  double tau = 0.0, scale = 0.0, beta = alpha;
  if (j < nr && xn2 > 0.0) {
    beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
    tau = (beta - alpha) / beta;
    scale = 1.0 / (alpha - beta);
  }
  // v on this warp's rows (from lane j's column), recomputed where it is
  // needed instead of held: RPW registers fewer
  auto vrow = [&](int t, double xj) {
    const int r = warp + NW * t;
    return (r < nr) ? (r > j ? xj * scale : (r == j ? 1.0 : 0.0)) : 0.0;
  };
  double d0 = 0.0, d1 = 0.0;
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const double vt = vrow(t, __shfl_sync(FULL, x[t], j));
    if (t & 1) d1 += vt * x[t];
    else d0 += vt * x[t];
  }
  dw[warp][lane] = d0 + d1;
  __syncthreads();
  double dc = 0.0;
#pragma unroll
  for (int w = 0; w < NW; ++w) dc += dw[w][lane];
  const double td = tau * dc;
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    const double vt = vrow(t, __shfl_sync(FULL, x[t], j));
    if (lane > j) x[t] -= vt * td;
    else if (lane == j && r >= j) x[t] = (r > j) ? vt : beta;
  }
  if (warp == 0) {
    // dots of columns c < j hold (V^T V)[c][j]
    gs[lane] = dc;
    __syncwarp();
    if (lane < j) {
      double acc = 0.0;
      for (int l = lane; l < j; ++l) acc += Tm[lane][l] * gs[l];
      Tm[lane][j] = -tau * acc;
    }
    if (lane == j) Tm[j][j] = tau;
    __syncwarp();
  }
}

template <int RPW>
__global__ void __launch_bounds__(NT) tsqr_panel_kernel(PanelArgs a) {
  // dynamic shared memory: six 32 x 33 blocks, then (rank 0) the stacked R_c
  extern __shared__ __align__(16) double dsm[];
  double (*Tl)[LDT] = reinterpret_cast<double (*)[LDT]>(dsm);               // local compact-WY factor
  double (*Vt)[LDT] = reinterpret_cast<double (*)[LDT]>(dsm + 1 * B * LDT); // local V, rows 0..31
  double (*Qt)[LDT] = reinterpret_cast<double (*)[LDT]>(dsm + 2 * B * LDT); // this CTA's block of the tree's Q
  double (*Wb)[LDT] = reinterpret_cast<double (*)[LDT]>(dsm + 3 * B * LDT); // scratch: T_c V_c,top^T Q_tree,c; rank 0: T_tree V_top^T, Q_1 - S
  double (*Uu)[LDT] = reinterpret_cast<double (*)[LDT]>(dsm + 4 * B * LDT); // U of the reconstruction
  double (*Tt)[LDT] = reinterpret_cast<double (*)[LDT]>(dsm + 5 * B * LDT); // rank 0: T of the tree, then the final T
  double* Rs = dsm + 6 * B * LDT;                                           // rank 0: the stacked R_c, [C * B][LDT]
  __shared__ double Ss[B];        // S of the reconstruction
  __shared__ double iu[B];        // 1 / U[k][k]
  __shared__ double dw[NW][B];
  __shared__ double nw[NW];
  __shared__ double gs[B];
  __shared__ double s_alpha;
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int C = (int)cl.num_blocks();
  const int m = a.m;
  const int R = a.rows_per_cta;
  const int lo = min(m, rank * R), hi = min(m, lo + R);
  const int nr = hi - lo;
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  double x[RPW];
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    x[t] = (r < nr) ? a.A[(size_t)(a.row0 + lo + r) * a.ld + a.col0 + lane] : 0.0;
  }
  for (int e = tid; e < B * LDT; e += NT) (&Tl[0][0])[e] = 0.0;
  __syncthreads();
  // ---- 1. local Householder QR
  for (int j = 0; j < B; ++j) house_step<RPW>(x, j, nr, nw, &s_alpha, dw, gs, Tl);
  __syncthreads();
  // local R (rows 0..31) to rank 0; local V rows 0..31 kept for step 3
  double* Rdst = cl.map_shared_rank(Rs, 0) + (size_t)rank * B * LDT;
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    if (r < B) {
      const bool in = r < nr;
      Rdst[r * LDT + lane] = (in && lane >= r) ? x[t] : 0.0;
      Vt[r][lane] = in ? (r > lane ? x[t] : (r == lane ? 1.0 : 0.0)) : 0.0;
    }
  }
  cl.sync();   // 1
  // ---- 2. rank 0: QR of the stacked R_c, explicit Q of the tree
  if (rank == 0) {
    const int M = C * B;
    for (int e = tid; e < B * LDT; e += NT) (&Tt[0][0])[e] = 0.0;
    __syncthreads();
    for (int j = 0; j < B; ++j) {
      // rows of column j's reflector: block 0 rows >= j, block c > 0 rows <= j
      double s = 0.0;
      for (int q = warp; q < M; q += NW) {
        const int c = q / B, r = q % B;
        if ((c == 0 && r > j) || (c > 0 && r <= j)) {
          const double y = Rs[q * LDT + j];
          s += y * y;
        }
      }
      s = __shfl_sync(FULL, s, 0);   // every lane summed the same column
      if (lane == 0) nw[warp] = s;
      __syncthreads();
      double xn2 = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) xn2 += nw[w];
      const double alpha = Rs[j * LDT + j];
      double tau = 0.0, scale = 0.0, beta = alpha;
      if (xn2 > 0.0) {
        beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        tau = (beta - alpha) / beta;
        scale = 1.0 / (alpha - beta);
      }
      // dots d_c = v^T (column c), over the reflector's rows
      double d = 0.0;
      for (int q = warp; q < M; q += NW) {
        const int c = q / B, r = q % B;
        double vq;
        if (c == 0) vq = (r > j) ? Rs[q * LDT + j] * scale : (r == j ? 1.0 : 0.0);
        else vq = (r <= j) ? Rs[q * LDT + j] * scale : 0.0;
        d += vq * Rs[q * LDT + lane];
      }
      dw[warp][lane] = d;
      __syncthreads();
      double dc = 0.0;
#pragma unroll
      for (int w = 0; w < NW; ++w) dc += dw[w][lane];
      // update columns right of j, store v in column j, beta on the diagonal
      for (int q = warp; q < M; q += NW) {
        const int c = q / B, r = q % B;
        const bool act = (c == 0) ? (r >= j) : (r <= j);
        if (!act) continue;
        const double yj = Rs[q * LDT + j];
        const double vq = (c == 0 && r == j) ? 1.0 : yj * scale;
        if (lane > j) Rs[q * LDT + lane] -= tau * dc * vq;
        __syncwarp();
        if (lane == j) Rs[q * LDT + j] = (c == 0 && r == j) ? beta : vq;
        __syncwarp();
      }
      if (warp == 0) {
        gs[lane] = dc;
        __syncwarp();
        if (lane < j) {
          double acc = 0.0;
          for (int l = lane; l < j; ++l) acc += Tt[lane][l] * gs[l];
          Tt[lane][j] = -tau * acc;
        }
        if (lane == j) Tt[j][j] = tau;
        __syncwarp();
      }
      __syncthreads();
    }
    // Q_tree = [I; 0] - V_tree (T_tree V_top^T);  Wb = T_tree V_top^T
    for (int e = tid; e < B * B; e += NT) {
      const int k = e / B, c = e % B;
      double acc = 0.0;
      for (int l = k; l <= c; ++l) acc += Tt[k][l] * (l == c ? 1.0 : Rs[c * LDT + l]);   // V_top[c][l], l <= c
      Wb[k][c] = acc;
    }
    __syncthreads();
    for (int q = warp; q < M; q += NW) {
      const int c = q / B, r = q % B;
      double acc = 0.0;
#pragma unroll 8
      for (int k = 0; k < B; ++k) {
        double vk;   // V_tree[q][k]
        if (c == 0) vk = (r > k) ? Rs[q * LDT + k] : (r == k ? 1.0 : 0.0);
        else vk = (k >= r) ? Rs[q * LDT + k] : 0.0;   // block c > 0: fill only at rows r <= k
        acc += vk * Wb[k][lane];
      }
      const double e0 = (q == lane) ? 1.0 : 0.0;
      cl.map_shared_rank(&Qt[0][0], c)[r * LDT + lane] = e0 - acc;
    }
  }
  cl.sync();   // 2
  // ---- 3. this CTA's rows of Q: Q_c = (I - V_c T_c V_c^T) [Qt; 0]
  // Wb = T_c (V_c,top^T Qt) (rank 0 is done with its Wb)
  {
    double w1[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + NT * u, k = e / B, c = e % B;
      double acc = 0.0;
      for (int r = k; r < B; ++r) acc += Vt[r][k] * Qt[r][c];
      w1[u] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + NT * u;
      Wb[e / B][e % B] = w1[u];   // W1
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + NT * u, k = e / B, c = e % B;
      double acc = 0.0;
      for (int l = k; l < B; ++l) acc += Tl[k][l] * Wb[l][c];
      w1[u] = acc;
    }
    __syncthreads();
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int e = tid + NT * u;
      Wb[e / B][e % B] = w1[u];   // W2 = T_c W1
    }
    __syncthreads();
  }
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    // V_c row r: column k from lane k (v below row k), 1 at r == k
    double acc = 0.0;
#pragma unroll
    for (int k = 0; k < B; ++k) {
      const double xk = __shfl_sync(FULL, x[t], k);
      const double vk = (r > k) ? xk : (r == k ? 1.0 : 0.0);
      acc += vk * Wb[k][lane];
    }
    const double y = (r < B) ? Qt[r][lane] : 0.0;
    x[t] = (r < nr) ? y - acc : 0.0;
  }
  // ---- rank 0: reconstruction from the top 32 rows
  if (rank == 0) {
    __syncthreads();
#pragma unroll
    for (int t = 0; t < RPW; ++t) {
      const int r = warp + NW * t;
      if (r < B) Wb[r][lane] = x[t];   // Q_1
    }
    __syncthreads();
    if (warp == 0) {
      // S and the LU of Q_1 - S (row per lane, no pivoting)
      const double q11 = Wb[lane][lane];
      const double sj = (q11 >= 0.0) ? -1.0 : 1.0;
      Ss[lane] = sj;
      Wb[lane][lane] = q11 - sj;
      __syncwarp();
      for (int k = 0; k < B; ++k) {
        if (lane > k) {
          const double l = Wb[lane][k] / Wb[k][k];
          Wb[lane][k] = l;
          for (int c = k + 1; c < B; ++c) Wb[lane][c] -= l * Wb[k][c];
        }
        __syncwarp();
      }
      // U (upper incl. diagonal) out of the LU, 1 / U[k][k]
      for (int c = 0; c < B; ++c) Uu[lane][c] = (c >= lane) ? Wb[lane][c] : 0.0;
      iu[lane] = 1.0 / Wb[lane][lane];
      __syncwarp();
      // T = -U S L_1^-T, row `lane` of T: solve L_1 y = -(U S)[lane][:]^T
      double y[B];
#pragma unroll
      for (int c = 0; c < B; ++c) {
        double acc = -Uu[lane][c] * Ss[c];
#pragma unroll
        for (int l = 0; l < c; ++l) acc -= Wb[c][l] * y[l];   // L_1[c][l], l < c
        y[c] = acc;
      }
#pragma unroll
      for (int c = 0; c < B; ++c) Tt[lane][c] = (c >= lane) ? y[c] : 0.0;
      __syncwarp();
    }
    __syncthreads();
    // U, S to every CTA
    for (int e = tid; e < C * B * LDT; e += NT) {
      const int c = e / (B * LDT), o = e % (B * LDT);
      if (c > 0) cl.map_shared_rank(&Uu[0][0], c)[o] = (&Uu[0][0])[o];
    }
    for (int e = tid; e < C * B; e += NT) {
      const int c = e / B, o = e % B;
      if (c > 0) {
        cl.map_shared_rank(Ss, c)[o] = Ss[o];
        cl.map_shared_rank(iu, c)[o] = iu[o];
      }
    }
    // outputs of rank 0: T, the band rows R_band = S R_tree, V rows 0..31 = L_1
    for (int e = tid; e < B * B; e += NT) {
      const int r = e / B, c = e % B;
      a.T[e] = Tt[r][c];
      if (c >= r) a.A[(size_t)(a.row0 + r) * a.ld + a.col0 + c] = Ss[r] * Rs[r * LDT + c];
      if (r < nr) a.V[(size_t)r * B + c] = (r > c) ? Wb[r][c] : (r == c ? 1.0 : 0.0);
    }
  }
  cl.sync();   // 3
  // ---- 4. V = Q U^-1 below the top 32 rows (forward substitution across
  // lanes, in place: lane k's value is final once step k is reached)
  for (int k = 0; k < B; ++k) {
    const double ukc = Uu[k][lane], ik = iu[k];
#pragma unroll
    for (int t = 0; t < RPW; ++t) {
      const double vk = __shfl_sync(FULL, x[t], k) * ik;
      if (lane == k) x[t] = vk;
      else if (lane > k) x[t] -= vk * ukc;
    }
  }
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    const int g = lo + r;
    if (r < nr && g >= B) a.V[(size_t)g * B + lane] = x[t];
  }
}

}  // namespace

size_t tsqr_smem_bytes(int C) { return sizeof(double) * (size_t)(6 + C) * B * LDT; }

int tsqr_max_rows_per_cta() { return NW * 48; }

cudaError_t init_tsqr_attributes() {
  cudaError_t e = cudaSuccess;
  for (auto k : {tsqr_panel_kernel<12>, tsqr_panel_kernel<24>, tsqr_panel_kernel<48>}) {
    e = cudaFuncSetAttribute(k, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)tsqr_smem_bytes(kTsqrMaxCluster));
    if (e != cudaSuccess) return e;
  }
  return e;
}

// rows_per_cta <= 384 and >= 32 (rank 0 holds the top 32 rows), C <= 16.
cudaError_t launch_tsqr_panel(const PanelArgs& pa, int C, cudaStream_t s) {
  if (C < 1 || C > kTsqrMaxCluster || pa.rows_per_cta < B || pa.rows_per_cta > NW * 48)
    return cudaErrorInvalidValue;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = tsqr_smem_bytes(C);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  const int rpw = (pa.rows_per_cta + NW - 1) / NW;
  if (rpw <= 12) return cudaLaunchKernelEx(&cfg, tsqr_panel_kernel<12>, pa);
  if (rpw <= 24) return cudaLaunchKernelEx(&cfg, tsqr_panel_kernel<24>, pa);
  return cudaLaunchKernelEx(&cfg, tsqr_panel_kernel<48>, pa);
}

}  // namespace mbd
