// Stage 1 of the two-stage tridiagonalisation of the CFDM Hamiltonian (the
// reduction half of PDSYEV('N','L') at UTILS.f90:835): symmetric dense ->
// band of half-bandwidth kBand, FP64, lower triangle, row-major.
//
// For each panel of kBand columns c0 = k*kBand (rows below the band r >= c0 +
// kBand, m of them):
//   qr_panel   Householder QR of the m x kBand panel in ONE thread-block
//              cluster: the panel's rows are spread over the CTAs' registers
//              (a lane per column; past 384 rows per CTA also shared
//              memory), cross-CTA sums are pushed into every CTA's shared
//              memory ahead of one or two hardware cluster barriers per
//              column.  Writes R in place (the band), V explicitly (unit
//              lower trapezoidal) and the compact-WY factor T (Q = I - V T
//              V^T, dlarft forward), whose Gram entries come from the same
//              dots.
//   symm       Y = A22 V (A22 the trailing m x m lower-stored block), row
//              blocks of 64 split over S column chunks (fixed-order partials)
//   yred       Y <- sum of the partials; Y <- Y T; block partials of V^T Y
//   mform      M = T^T (V^T Y)
//   zform      Z = Y - 1/2 V M
//   syr2k      A22 -= V Z^T + Z V^T (lower 64 x 64 tiles)
// so that A22 <- Q^T A22 Q.  Every reduction is summed in a fixed order: the
// result does not depend on scheduling.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>

#include "kernels.h"

namespace cg = cooperative_groups;

namespace mbd {
namespace {

constexpr int B = kBand;            // 32
constexpr int TL = 64;              // tile edge of symm / syr2k

// The cluster barrier in its two halves: work a CTA does between its arrive
// and its wait overlaps the other CTAs' arrival instead of delaying them.
__device__ __forceinline__ void cluster_arrive() { asm volatile("barrier.cluster.arrive.release.aligned;" ::: "memory"); }
__device__ __forceinline__ void cluster_wait() { asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory"); }

// Panel QR with the panel in registers: warp w of a CTA owns the local rows
// r = w + NW t (t < RPW), lane c holds column c of them in x[t].  One cluster
// barrier per column j (given ||x_j below row j||^2 and alpha = A(j, j)):
//   1. every CTA computes the same beta, tau from the same cluster sums.
//   2. lane j writes v (0 above row j, 1 at row j, x * scale below) to shared
//      memory for its warp; every lane c forms d_c = v^T x_c over its rows:
//      for c > j the update's coefficient, for c < j (column c already holds
//      v_c) the entry (V^T V)[c][j] of the compact-WY Gram matrix.  In the
//      same pass lane j + 1 sums, over its rows below row j + 1, x^2, v x and
//      v^2, and the owner of row j + 1 keeps x_{j+1}(j + 1) and v(j + 1).
//   3. CTA sums, ONE cluster barrier, cluster sums (fixed order everywhere).
//   4. x_c -= tau v d_c for c > j; lane j keeps v, row j gets beta.
//   5. the next column's norm below row j + 1 without another exchange:
//      ||x - tau d v||^2 = S_xx - 2 tau d S_vx + tau^2 d^2 S_vv, and
//      alpha' = x(j + 1) - tau d v(j + 1).  When the downdate cancels more than
//      90 % of S_xx the norm is summed again from the updated column (a
//      second barrier; every CTA takes the same branch).  On the matrices
//      studied (random symmetric, CFDM Hamiltonians) the ratio never fell
//      below 0.19 and the downdate matched the exact sum to 1.1e-15.
//   6. rank 0, warp 0: T[0:j, j] = -tau_j T[0:j, 0:j] (V^T V)[0:j, j],
//      T[j][j] = tau_j (dlarft, forward, columnwise) from the same dots.
// recv* are written by the other CTAs of the cluster (remote stores before
// the barrier) and read locally after it; double-buffered by column parity,
// a buffer is rewritten two columns later, after every CTA has passed the
// barrier of the column in between, so after its reads.
template <int NW, int RPW>
__global__ void __launch_bounds__(NW * 32) qr_panel_kernel(PanelArgs a) {
  constexpr int NT = NW * 32;
  constexpr unsigned FULL = 0xffffffffu;
  // receive buffers (double-buffered by column parity): every CTA pushes its
  // partial sums into every CTA's buffers with remote stores before the
  // cluster barrier and reads its own buffers after it
  __shared__ double recvN[2][kPanelMaxCluster];      // exact norm partials (first column, recomputes)
  __shared__ double recvA0;                          // alpha of the first column
  __shared__ double recvD[2][kPanelMaxCluster][B];   // dot sums, by rank
  __shared__ double recvS[2][kPanelMaxCluster][4];   // S_xx, S_vx, S_vv for the next column, by rank
  __shared__ double recvR[2][2];                     // from the owner of row j + 1: x_{j+1}(j + 1), v(j + 1)
  __shared__ double wn[NW];
  __shared__ double dw[NW][B];
  __shared__ double ds[NW][3];
  __shared__ double vs[NW][RPW];
  __shared__ double gs[B];
  __shared__ double Tm[B][B + 1];
  cg::cluster_group cl = cg::this_cluster();
  // T[0:jc, jc] = -tau_jc T[0:jc, 0:jc] (V^T V)[0:jc, jc], T[jc][jc] = tau_jc
  // (dlarft, forward, columnwise) from column jc's dots dcj (rank 0, warp 0)
  int jprev = -1;
  double dcprev = 0.0, tauprev = 0.0;
  auto t_column = [&](int jc, double dcj, double tauj) {
    const int ln = threadIdx.x % 32;
    gs[ln] = dcj;
    __syncwarp();
    if (ln < jc) {
      double t = 0.0;
      for (int l = ln; l < jc; ++l) t += Tm[ln][l] * gs[l];
      Tm[ln][jc] = -tauj * t;
    }
    if (ln == jc) Tm[jc][jc] = tauj;
    __syncwarp();
  };
  const int rank = (int)cl.block_rank();
  const int C = (int)cl.num_blocks();
  const int m = a.m;
  const int R = a.rows_per_cta;
  const int lo = rank * R, hi = min(m, lo + R);
  const int nr = max(0, hi - lo);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g0 = lo + warp;   // panel row of x[0]; x[t] holds row g0 + NW t
  double x[RPW];
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    x[t] = (r < nr) ? a.A[(size_t)(a.row0 + lo + r) * a.ld + a.col0 + lane] : 0.0;
  }
  if (rank == 0)
    for (int e = tid; e < B * (B + 1); e += NT) (&Tm[0][0])[e] = 0.0;
  const int nref = min(B, m);
  // exact ||x_c below row jr||^2 of column c = jr (lane jr's value), summed
  // over the cluster through recvN[par] (one barrier)
  auto exact_norm = [&](int jr, int par) -> double {
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int t = 0; t < RPW; ++t) {
      const double v = (g0 + NW * t > jr) ? x[t] : 0.0;
      if (t & 1) s1 += v * v;
      else s0 += v * v;
    }
    const double sj = __shfl_sync(FULL, s0 + s1, jr);
    if (lane == 0) wn[warp] = sj;
    __syncthreads();
    if (warp == 0) {
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < NW; ++q) t += wn[q];
      if (lane < C) cl.map_shared_rank(&recvN[0][0], lane)[par * kPanelMaxCluster + rank] = t;
    }
    cl.sync();
    double xn = 0.0;
    for (int q = 0; q < C; ++q) xn += recvN[par][q];
    return xn;
  };
  // row jr's entry of this lane's column (valid in the owner warp; jr - lo < 32)
  auto own_entry = [&](int jr) -> double {
    const int tj = (jr - lo) / NW;
    double v = 0.0;
#pragma unroll
    for (int t = 0; t < (RPW < 4 ? RPW : 4); ++t)
      if (t == tj) v = x[t];
    return v;
  };
  // column 0: exact norm and alpha (rank 0, warp 0 owns row 0)
  if (rank == 0 && warp == 0) {
    const double a0 = __shfl_sync(FULL, own_entry(0), 0);
    if (lane < C) *cl.map_shared_rank(&recvA0, lane) = a0;
  }
  double xn2 = exact_norm(0, 0);   // its barrier also delivers alpha
  double alpha = recvA0;
  for (int j = 0; j < nref; ++j) {
    const int par = j & 1;
    double tau = 0.0, scale = 0.0, beta = alpha;
    if (xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      tau = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    if (rank == 0 && tid == 0) a.tau[j] = tau;
    // v on this warp's rows
    if (lane == j) {
      if (g0 > j) {
#pragma unroll
        for (int t = 0; t < RPW; ++t) vs[warp][t] = x[t] * scale;
      } else {
#pragma unroll
        for (int t = 0; t < RPW; ++t) {
          const int g = g0 + NW * t;
          vs[warp][t] = g < j ? 0.0 : (g == j ? 1.0 : x[t] * scale);
        }
      }
    }
    __syncwarp();
    // dots (all lanes) and the next column's sums below row j + 1 (lane j + 1's)
    double d0 = 0.0, d1 = 0.0, sxx = 0.0, svx = 0.0, svv = 0.0;
    if (g0 > j + 1) {
#pragma unroll
      for (int t = 0; t < RPW; ++t) {
        const double v = vs[warp][t];
        if (t & 1) d1 += v * x[t];
        else d0 += v * x[t];
        sxx += x[t] * x[t];
        svv += v * v;
      }
      svx = d0 + d1;
    } else {
#pragma unroll
      for (int t = 0; t < RPW; ++t) {
        const double v = vs[warp][t];
        if (t & 1) d1 += v * x[t];
        else d0 += v * x[t];
        if (g0 + NW * t > j + 1) {
          sxx += x[t] * x[t];
          svx += v * x[t];
          svv += v * v;
        }
      }
    }
    dw[warp][lane] = d0 + d1;
    const int jn = j + 1 < B ? j + 1 : B - 1;
    {
      const double a0 = __shfl_sync(FULL, sxx, jn), a1 = __shfl_sync(FULL, svx, jn), a2 = __shfl_sync(FULL, svv, jn);
      if (lane == 0) {
        ds[warp][0] = a0;
        ds[warp][1] = a1;
        ds[warp][2] = a2;
      }
    }
    if (j + 1 < nref && j + 1 >= lo && j + 1 < hi && (j + 1 - lo) % NW == warp) {
      // the owner warp of row j + 1 pushes x_{j+1}(j + 1) and v(j + 1) to every CTA
      const double ex = __shfl_sync(FULL, own_entry(j + 1), j + 1);
      const double ev = vs[warp][(j + 1 - lo) / NW];
      if (lane < C) {
        double* pr = cl.map_shared_rank(&recvR[0][0], lane) + par * 2;
        pr[0] = ex;
        pr[1] = ev;
      }
    }
    __syncthreads();
    {
      // every warp forms the CTA's sums and pushes them to C / NW ranks
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < NW; ++q) t += dw[q][lane];
      double u = 0.0;
      if (lane < 3)
#pragma unroll
        for (int q = 0; q < NW; ++q) u += ds[q][lane];
      for (int q = warp; q < C; q += NW) {
        cl.map_shared_rank(&recvD[0][0][0], q)[(par * kPanelMaxCluster + rank) * B + lane] = t;
        if (lane < 3) cl.map_shared_rank(&recvS[0][0][0], q)[(par * kPanelMaxCluster + rank) * 4 + lane] = u;
      }
    }
    cluster_arrive();
    if (rank == 0 && warp == 0 && jprev >= 0) t_column(jprev, dcprev, tauprev);
    cluster_wait();
    // cluster sums in rank order
    double dc = 0.0, Sxx = 0.0, Svx = 0.0, Svv = 0.0;
    for (int q = 0; q < C; ++q) {
      dc += recvD[par][q][lane];
      Sxx += recvS[par][q][0];
      Svx += recvS[par][q][1];
      Svv += recvS[par][q][2];
    }
    const double rx = recvR[par][0], rv = recvR[par][1];
    // update the columns right of j
    const double tdc = (lane > j) ? tau * dc : 0.0;
#pragma unroll
    for (int t = 0; t < RPW; ++t) x[t] -= vs[warp][t] * tdc;
    if (lane == j) {
#pragma unroll
      for (int t = 0; t < RPW; ++t) {
        const int g = g0 + NW * t;
        if (g > j) x[t] = vs[warp][t];
        else if (g == j) x[t] = beta;
      }
    }
    // compact-WY factor, column j: built by rank 0's warp 0 inside the next
    // column's barrier (it needs only this column's dots and the earlier
    // columns of T), so that no CTA waits for it
    jprev = j;
    dcprev = dc;
    tauprev = tau;
    // the next column's norm and alpha
    if (j + 1 < nref) {
      const double dn = __shfl_sync(FULL, dc, j + 1);
      const double td = tau * dn;
      const double down = Sxx - 2.0 * td * Svx + td * td * Svv;
      alpha = rx - rv * td;
      xn2 = (down >= 0.1 * Sxx) ? down : exact_norm(j + 1, par);
    }
  }
  // write R (rows g <= c: the band) and V (explicit, unit lower trapezoidal)
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    if (r < nr) {
      const int g = lo + r;
      if (g <= lane) a.A[(size_t)(a.row0 + g) * a.ld + a.col0 + lane] = x[t];
      a.V[(size_t)g * B + lane] = g > lane ? x[t] : (g == lane ? 1.0 : 0.0);
    }
  }
  if (rank == 0 && warp == 0 && jprev >= 0) t_column(jprev, dcprev, tauprev);   // the last column of T
  if (rank == 0) {
    __syncthreads();
    for (int e = tid; e < B * B; e += NT) a.T[e] = Tm[e / B][e % B];
  }
  cl.sync();   // no CTA leaves while another may still read its shared memory
}

// The same factorisation with two cluster barriers per column: the norm of
// column j + 1 is summed from the updated column after a second exchange
// (no downdate).  For 48 rows per warp it measured faster than the one-barrier
// form (196 against 220 us for an m = 5296 panel): the extra sums of the
// downdate cost more than the barrier they save once the rows per warp grow.
// HYB: local rows beyond NW x RPW (up to kPanelMaxRowsPerCta) live in dynamic
// shared memory, Ps[i][c] for local row NW * RPW + i (row i belongs to warp
// i % NW as in the registers); they lie below row 383 of the panel, so they
// never meet the diagonal rows j, j + 1 < 32 and need no masks.
template <int NW, int RPW, bool HYB>
__global__ void __launch_bounds__(NW * 32) qr_panel2_kernel(PanelArgs a) {
  extern __shared__ __align__(16) double Ps[];   // HYB: [R - NW * RPW][QR_LD2]
  constexpr int QR_LD2 = B + 1;
  constexpr int RREG = NW * RPW;
  constexpr int NT = NW * 32;
  constexpr unsigned FULL = 0xffffffffu;
  // receive buffers (double-buffered by column parity): every CTA pushes its
  // partial sums into every CTA's buffers with remote stores before the
  // cluster barrier and reads its own buffers after it
  __shared__ double recvN[2][kPanelMaxCluster];      // CTA norm partials, by rank
  __shared__ double recvA[2];                        // alpha from the owner of row j
  __shared__ double recvD[2][kPanelMaxCluster][B];   // CTA dot sums, by rank
  __shared__ double wn[NW];
  __shared__ double dw[NW][B];
  __shared__ double vs[NW][RPW];
  __shared__ double gs[B];
  __shared__ double Tm[B][B + 1];
  cg::cluster_group cl = cg::this_cluster();
  // T[0:jc, jc] = -tau_jc T[0:jc, 0:jc] (V^T V)[0:jc, jc], T[jc][jc] = tau_jc
  // (dlarft, forward, columnwise) from column jc's dots dcj (rank 0, warp 0)
  int jprev = -1;
  double dcprev = 0.0, tauprev = 0.0;
  auto t_column = [&](int jc, double dcj, double tauj) {
    const int ln = threadIdx.x % 32;
    gs[ln] = dcj;
    __syncwarp();
    if (ln < jc) {
      double t = 0.0;
      for (int l = ln; l < jc; ++l) t += Tm[ln][l] * gs[l];
      Tm[ln][jc] = -tauj * t;
    }
    if (ln == jc) Tm[jc][jc] = tauj;
    __syncwarp();
  };
  const int rank = (int)cl.block_rank();
  const int C = (int)cl.num_blocks();
  const int m = a.m;
  const int R = a.rows_per_cta;
  const int lo = rank * R, hi = min(m, lo + R);
  const int nr = max(0, hi - lo);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g0 = lo + warp;   // panel row of x[0]; x[t] holds row g0 + NW t
  double x[RPW];
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    x[t] = (r < nr) ? a.A[(size_t)(a.row0 + lo + r) * a.ld + a.col0 + lane] : 0.0;
  }
  if (HYB)
    for (int i = warp; RREG + i < nr; i += NW)
      Ps[i * QR_LD2 + lane] = a.A[(size_t)(a.row0 + lo + RREG + i) * a.ld + a.col0 + lane];
  if (rank == 0)
    for (int e = tid; e < B * (B + 1); e += NT) (&Tm[0][0])[e] = 0.0;
  const int nref = min(B, m);
  // squared norm of this lane's column over the rows below row j
  double s_own;
  {
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int t = 0; t < RPW; ++t) {
      const double v = (g0 + NW * t > 0) ? x[t] : 0.0;
      if (t & 1) s1 += v * v;
      else s0 += v * v;
    }
    if (HYB)
      for (int i = warp; RREG + i < nr; i += NW) {
        const double v = Ps[i * QR_LD2 + lane];
        s0 += v * v;
      }
    s_own = s0 + s1;
  }
  for (int j = 0; j < nref; ++j) {
    const int par = j & 1;
    const double sj = __shfl_sync(FULL, s_own, j);
    if (lane == 0) wn[warp] = sj;
    // row j is local row j - lo < 32: warp (j - lo) % NW, slot t = (j - lo) / NW < 4;
    // the owner warp pushes alpha = A(j, j) to every CTA
    if (j >= lo && j < hi && (j - lo) % NW == warp) {
      const int tj = (j - lo) / NW;
      double aj = 0.0;
#pragma unroll
      for (int t = 0; t < (RPW < 4 ? RPW : 4); ++t)
        if (t == tj) aj = x[t];
      aj = __shfl_sync(FULL, aj, j);
      if (lane < C) cl.map_shared_rank(&recvA[0], lane)[par] = aj;
    }
    __syncthreads();
    if (warp == 0) {
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < NW; ++q) t += wn[q];
      if (lane < C) cl.map_shared_rank(&recvN[0][0], lane)[par * kPanelMaxCluster + rank] = t;
    }
    cluster_arrive();
    if (rank == 0 && warp == 0 && jprev >= 0) t_column(jprev, dcprev, tauprev);
    cluster_wait();
    double xn2 = 0.0;
    for (int q = 0; q < C; ++q) xn2 += recvN[par][q];
    const double alpha = recvA[par];
    double tau = 0.0, scale = 0.0, beta = alpha;
    if (xn2 > 0.0) {
      beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
      tau = (beta - alpha) / beta;
      scale = 1.0 / (alpha - beta);
    }
    if (rank == 0 && tid == 0) a.tau[j] = tau;
    // v on this warp's rows
    if (lane == j) {
      if (g0 > j) {
#pragma unroll
        for (int t = 0; t < RPW; ++t) vs[warp][t] = x[t] * scale;
      } else {
#pragma unroll
        for (int t = 0; t < RPW; ++t) {
          const int g = g0 + NW * t;
          vs[warp][t] = g < j ? 0.0 : (g == j ? 1.0 : x[t] * scale);
        }
      }
    }
    __syncwarp();
    double d0 = 0.0, d1 = 0.0;   // two accumulation chains
#pragma unroll
    for (int t = 0; t < RPW; ++t) {
      if (t & 1) d1 += vs[warp][t] * x[t];
      else d0 += vs[warp][t] * x[t];
    }
    if (HYB)
      for (int i = warp; RREG + i < nr; i += NW) d0 += (Ps[i * QR_LD2 + j] * scale) * Ps[i * QR_LD2 + lane];
    dw[warp][lane] = d0 + d1;
    __syncthreads();
    {
      // every warp forms the CTA's dot vector and pushes it to C / NW ranks
      double t = 0.0;
#pragma unroll
      for (int q = 0; q < NW; ++q) t += dw[q][lane];
      for (int q = warp; q < C; q += NW)
        cl.map_shared_rank(&recvD[0][0][0], q)[(par * kPanelMaxCluster + rank) * B + lane] = t;
    }
    cl.sync();
    double dc = 0.0;
    for (int q = 0; q < C; ++q) dc += recvD[par][q][lane];
    // update the columns right of j and the norms below row j + 1
    const double tdc = (lane > j) ? tau * dc : 0.0;
    double s0 = 0.0, s1 = 0.0;
    if (g0 > j + 1) {
#pragma unroll
      for (int t = 0; t < RPW; ++t) {
        x[t] -= vs[warp][t] * tdc;
        if (t & 1) s1 += x[t] * x[t];
        else s0 += x[t] * x[t];
      }
    } else {
#pragma unroll
      for (int t = 0; t < RPW; ++t) {
        x[t] -= vs[warp][t] * tdc;
        const double v = (g0 + NW * t > j + 1) ? x[t] : 0.0;
        if (t & 1) s1 += v * v;
        else s0 += v * v;
      }
    }
    if (HYB) {
      // lane j's column is read by every lane here and scaled to v after
      for (int i = warp; RREG + i < nr; i += NW) {
        double* pr = Ps + i * QR_LD2;
        const double y = pr[lane] - (pr[j] * scale) * tdc;
        if (lane > j) pr[lane] = y;
        s0 += y * y;
      }
      __syncwarp();
      if (lane == j)
        for (int i = warp; RREG + i < nr; i += NW) Ps[i * QR_LD2 + j] *= scale;
    }
    s_own = s0 + s1;
    if (lane == j) {
#pragma unroll
      for (int t = 0; t < RPW; ++t) {
        const int g = g0 + NW * t;
        if (g > j) x[t] = vs[warp][t];
        else if (g == j) x[t] = beta;
      }
    }
    // compact-WY factor, column j: built by rank 0's warp 0 inside the next
    // column's barrier (it needs only this column's dots and the earlier
    // columns of T), so that no CTA waits for it
    jprev = j;
    dcprev = dc;
    tauprev = tau;
  }
  // write R (rows g <= c: the band) and V (explicit, unit lower trapezoidal)
#pragma unroll
  for (int t = 0; t < RPW; ++t) {
    const int r = warp + NW * t;
    if (r < nr) {
      const int g = lo + r;
      if (g <= lane) a.A[(size_t)(a.row0 + g) * a.ld + a.col0 + lane] = x[t];
      a.V[(size_t)g * B + lane] = g > lane ? x[t] : (g == lane ? 1.0 : 0.0);
    }
  }
  if (HYB)   // rows below 383: V only
    for (int i = warp; RREG + i < nr; i += NW) a.V[(size_t)(lo + RREG + i) * B + lane] = Ps[i * QR_LD2 + lane];
  if (rank == 0 && warp == 0 && jprev >= 0) t_column(jprev, dcprev, tauprev);   // the last column of T
  if (rank == 0) {
    __syncthreads();
    for (int e = tid; e < B * B; e += NT) a.T[e] = Tm[e / B][e % B];
  }
  cl.sync();   // no CTA leaves while another may still read its shared memory
}

// Variants by rows per CTA: (warps, rows per warp); the last one keeps 384
// rows in registers and the rest in shared memory.
constexpr int kQrVariants = 4;
constexpr int kQrWarps[kQrVariants] = {8, 8, 8, 8};
constexpr int kQrRows[kQrVariants] = {12, 24, 48, kPanelMaxRowsPerCta / 8};
constexpr int kQrRegRows = 8 * 48;
int qr_variant(int R) {
  for (int v = 0; v < kQrVariants; ++v)
    if (R <= kQrWarps[v] * kQrRows[v]) return v;
  return -1;
}
using QrKernel = void (*)(PanelArgs);
QrKernel qr_kernel(int v) {
  switch (v) {
    case 0: return qr_panel_kernel<8, 12>;
    case 1: return qr_panel_kernel<8, 24>;
    case 2: return qr_panel2_kernel<8, 48, false>;
    default: return qr_panel2_kernel<8, 48, true>;
  }
}
// dynamic shared memory of variant v for R rows per CTA
size_t qr_smem_bytes(int v, int R) {
  return v == kQrVariants - 1 ? sizeof(double) * (B + 1) * (size_t)std::max(0, R - kQrRegRows) : 0;
}

// FP64 tensor-core MMA, D = A B + D with A 8x4 (row), B 4x8 (col), D 8x8:
// a = A[lane/4][lane%4], b = B[lane%4][lane/4], d = D[lane/4][2*(lane%4) + {0,1}].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Shared-memory row stride (doubles) making the 8 x 4 fragment loads of a
// half-warp hit 16 distinct bank pairs: stride = 4 (mod 16).
constexpr int FS = TL + 4;   // 68

// 16-byte asynchronous copy global -> shared; src_bytes < 16 zero-fills the rest.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(NPEND) : "memory");
}

// Y partials: Yp[s][r][c] = sum over column tiles J of chunk s of (A22 V)[r][c],
// row block I = blockIdx.x (64 rows), chunk s = blockIdx.y.  4 warps, each 16
// rows x 32 columns of the block (2 x 4 MMA tiles).  The stored lower tile
// that holds A22's block (I, J) -- (I, J) itself for J < I, (J, I) for J > I,
// the diagonal tile for J = I -- and the 64 rows of V of block J are copied to
// shared memory as they are stored (cp.async, two stages: the next J's copy
// runs under this J's MMAs); the MMA reads the tile in its orientation.
constexpr int FV = B + 4;                        // 36: V rows in shared memory (4 mod 16)
constexpr int kSymmStage = TL * FS + TL * FV;    // doubles per stage
constexpr size_t kSymmSmem = sizeof(double) * 2 * kSymmStage;

__device__ __forceinline__ void symm_stage(const double* A22, int ld, int m, const double* V, int I, int J,
                                           double* As, double* Vs) {
  const int tid = threadIdx.x;
  const int R0 = (J <= I ? I : J) * TL, C0 = (J <= I ? J : I) * TL;
  for (int idx = tid; idx < TL * (TL / 2); idx += blockDim.x) {
    const int u = idx / (TL / 2), w = 2 * (idx % (TL / 2));
    const int gr = R0 + u, gc = C0 + w;
    const bool rok = gr < m;
    const int bytes = rok ? (gc + 1 < m ? 16 : (gc < m ? 8 : 0)) : 0;
    cp_async16(As + u * FS + w, A22 + (size_t)(rok ? gr : 0) * ld + (bytes ? gc : 0), bytes);
  }
  for (int idx = tid; idx < TL * (B / 2); idx += blockDim.x) {
    const int k = idx / (B / 2), c = 2 * (idx % (B / 2));
    const int gk = J * TL + k;
    cp_async16(Vs + k * FV + c, V + (size_t)(gk < m ? gk : 0) * B + c, gk < m ? 16 : 0);
  }
}

// MODE 0: block (I, J) stored as is; 1: stored transposed; 2: diagonal tile (lower).
template <int MODE>
__device__ __forceinline__ void symm_mma(const double* As, const double* Vs, int warp, int g, int q4,
                                         double (&acc)[2][4][2]) {
#pragma unroll 4
  for (int k0 = 0; k0 < TL; k0 += 4) {
    double af[2], bf[4];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const int r = warp * 16 + i * 8 + g, k = k0 + q4;
      if (MODE == 0) af[i] = As[r * FS + k];
      else if (MODE == 1) af[i] = As[k * FS + r];
      else af[i] = As[(r > k ? r : k) * FS + (r > k ? k : r)];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) bf[q] = Vs[(k0 + q4) * FV + q * 8 + g];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q) dmma(acc[i][q][0], acc[i][q][1], af[i], bf[q]);
  }
}

__global__ void __launch_bounds__(128) symm_kernel(const double* A, int ld, int row0, int m, const double* V,
                                                   double* Yp, int chunk) {
  extern __shared__ __align__(16) double dsm[];
  const int I = blockIdx.x, s = blockIdx.y;
  const int nt = (m + TL - 1) / TL;
  const int J0 = s * chunk, J1 = min(nt, J0 + chunk);
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, q4 = lane & 3;
  double acc[2][4][2];
#pragma unroll
  for (int i = 0; i < 2; ++i)
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[i][q][0] = acc[i][q][1] = 0.0;
  const double* A22 = A + (size_t)row0 * ld + row0;
  if (J0 < J1) symm_stage(A22, ld, m, V, I, J0, dsm, dsm + TL * FS);
  cp_async_commit();
  for (int J = J0; J < J1; ++J) {
    const double* As = dsm + ((J - J0) & 1) * kSymmStage;
    const double* Vs = As + TL * FS;
    if (J + 1 < J1) {
      double* An = dsm + ((J + 1 - J0) & 1) * kSymmStage;
      symm_stage(A22, ld, m, V, I, J + 1, An, An + TL * FS);
    }
    cp_async_commit();
    cp_async_wait<1>();   // this J's stage has landed (the next may be in flight)
    __syncthreads();
    if (J < I) symm_mma<0>(As, Vs, warp, g, q4, acc);
    else if (J > I) symm_mma<1>(As, Vs, warp, g, q4, acc);
    else symm_mma<2>(As, Vs, warp, g, q4, acc);
    __syncthreads();      // the stage is read before the copy two steps on reuses it
  }
  double* out = Yp + (size_t)s * m * B;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const int gr = I * TL + warp * 16 + i * 8 + g;
    if (gr < m)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        out[(size_t)gr * B + q * 8 + 2 * q4] = acc[i][q][0];
        out[(size_t)gr * B + q * 8 + 2 * q4 + 1] = acc[i][q][1];
      }
  }
}

// Y = sum_s Yp[s]; Y <- Y T; Up[I] = V_I^T Y_I (64-row blocks, 256 threads).
__global__ void __launch_bounds__(256) yred_kernel(const double* Yp, int S, int m, const double* T, const double* V,
                                                   double* Y, double* Up) {
  __shared__ double Ts[B][B + 1];
  __shared__ double Ys[TL][B + 1];
  __shared__ double Vs[TL][B + 1];
  const int I = blockIdx.x, tid = threadIdx.x;
  for (int e = tid; e < B * B; e += 256) Ts[e / B][e % B] = T[e];
  for (int e = tid; e < TL * B; e += 256) {
    const int r = e / B, c = e % B, gr = I * TL + r;
    double y = 0.0, v = 0.0;
    if (gr < m) {
      for (int s = 0; s < S; ++s) y += Yp[((size_t)s * m + gr) * B + c];
      v = V[(size_t)gr * B + c];
    }
    Ys[r][c] = y;
    Vs[r][c] = v;
  }
  __syncthreads();
  double yt[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int e = tid + 256 * t, r = e / B, c = e % B;
    double x = 0.0;
    for (int l = 0; l <= c; ++l) x += Ys[r][l] * Ts[l][c];
    yt[t] = x;
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    const int e = tid + 256 * t, r = e / B, c = e % B, gr = I * TL + r;
    Ys[r][c] = yt[t];
    if (gr < m) Y[(size_t)gr * B + c] = yt[t];
  }
  __syncthreads();
#pragma unroll
  for (int t = 0; t < 4; ++t) {
    const int e = tid + 256 * t, p = e / B, c = e % B;
    double u = 0.0;
    for (int r = 0; r < TL; ++r) u += Vs[r][p] * Ys[r][c];
    Up[(size_t)I * B * B + e] = u;
  }
}

// M = T^T U, U = sum_I Up[I] (one CTA of B*B threads).
__global__ void __launch_bounds__(B* B) mform_kernel(const double* Up, int nt, const double* T, double* M) {
  __shared__ double Us[B][B + 1];
  __shared__ double Ts[B][B + 1];
  const int e = threadIdx.x, p = e / B, c = e % B;
  double u = 0.0;
  for (int I = 0; I < nt; ++I) u += Up[(size_t)I * B * B + e];
  Us[p][c] = u;
  Ts[p][c] = T[e];
  __syncthreads();
  double x = 0.0;
  for (int l = 0; l <= p; ++l) x += Ts[l][p] * Us[l][c];   // (T^T)[p][l] = T[l][p], l <= p
  M[e] = x;
}

// Z = Y - 1/2 V M (rows in blocks of 64, 256 threads)
__global__ void __launch_bounds__(256) zform_kernel(const double* Y, const double* V, const double* M, int m,
                                                    double* Z) {
  __shared__ double Ms[B][B + 1];
  __shared__ double Vs[TL][B + 1];
  const int I = blockIdx.x, tid = threadIdx.x;
  for (int e = tid; e < B * B; e += 256) Ms[e / B][e % B] = M[e];
  for (int e = tid; e < TL * B; e += 256) {
    const int r = e / B, c = e % B, gr = I * TL + r;
    Vs[r][c] = gr < m ? V[(size_t)gr * B + c] : 0.0;
  }
  __syncthreads();
  for (int e = tid; e < TL * B; e += 256) {
    const int r = e / B, c = e % B, gr = I * TL + r;
    if (gr >= m) continue;
    double x = 0.0;
#pragma unroll 8
    for (int l = 0; l < B; ++l) x += Vs[r][l] * Ms[l][c];
    Z[(size_t)gr * B + c] = Y[(size_t)gr * B + c] - 0.5 * x;
  }
}

// A22 -= V Z^T + Z V^T on lower 64 x 64 tiles: [V_I | Z_I] [Z_J | V_J]^T
// (K = 64) on FP64 MMAs; 4 warps, each a 32 x 32 quarter (4 x 4 MMA tiles).
// The two operand blocks and the A22 tile itself are copied to shared memory
// together (cp.async), the products are subtracted there and the tile goes
// back a row per warp instruction (coalesced).
constexpr size_t kSyr2kSmem = sizeof(double) * 3 * TL * FS;
// part: 0 every lower tile (one CTA each, triangular order), 1 the tiles of
// tile column 0 (the next panel's columns), 2 the lower tiles right of it.
__global__ void __launch_bounds__(128) syr2k_kernel(double* A, int ld, int row0, int m, const double* V,
                                                    const double* Z, int part) {
  extern __shared__ __align__(16) double dsm[];
  double* Li = dsm;                // [64][FS]: [V_I | Z_I]
  double* Lj = dsm + TL * FS;      // [64][FS]: [Z_J | V_J]
  double* Cs = dsm + 2 * TL * FS;  // [64][FS]: the A22 tile (I, J)
  int ti, tj;
  if (part == 1) {
    ti = (int)blockIdx.x;
    tj = 0;
  } else {
    ti = (int)((sqrt(8.0 * blockIdx.x + 1.0) - 1.0) * 0.5);
    while ((ti + 1) * (ti + 2) / 2 <= (int)blockIdx.x) ++ti;
    while (ti * (ti + 1) / 2 > (int)blockIdx.x) --ti;
    tj = (int)blockIdx.x - ti * (ti + 1) / 2;
    if (part == 2) {
      ++ti;
      ++tj;
    }
  }
  const int tid = threadIdx.x, warp = tid / 32, lane = tid % 32;
  const int g = lane >> 2, q4 = lane & 3;
  double* A22 = A + (size_t)row0 * ld + row0;
  for (int e = tid; e < TL * (B / 2); e += 128) {
    const int r = e / (B / 2), c = 2 * (e % (B / 2));
    const int gi = ti * TL + r, gj = tj * TL + r;
    const int bi = gi < m ? 16 : 0, bj = gj < m ? 16 : 0;
    const size_t oi = (size_t)(gi < m ? gi : 0) * B + c, oj = (size_t)(gj < m ? gj : 0) * B + c;
    cp_async16(Li + r * FS + c, V + oi, bi);
    cp_async16(Li + r * FS + B + c, Z + oi, bi);
    cp_async16(Lj + r * FS + c, Z + oj, bj);
    cp_async16(Lj + r * FS + B + c, V + oj, bj);
  }
  for (int e = tid; e < TL * (TL / 2); e += 128) {
    const int r = e / (TL / 2), c = 2 * (e % (TL / 2));
    const int gr = ti * TL + r, gc = tj * TL + c;
    const bool rok = gr < m;
    const int bytes = rok ? (gc + 1 < m ? 16 : (gc < m ? 8 : 0)) : 0;
    cp_async16(Cs + r * FS + c, A22 + (size_t)(rok ? gr : 0) * ld + (bytes ? gc : 0), bytes);
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  const int r0 = (warp / 2) * 32, c0 = (warp % 2) * 32;
  if (!(ti == tj && c0 > r0)) {   // the strictly upper quarter of a diagonal tile is not stored
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[i][q][0] = acc[i][q][1] = 0.0;
#pragma unroll 2
    for (int k0 = 0; k0 < 2 * B; k0 += 4) {
      double af[4], bf[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) af[i] = Li[(r0 + i * 8 + g) * FS + k0 + q4];
#pragma unroll
      for (int q = 0; q < 4; ++q) bf[q] = Lj[(c0 + q * 8 + g) * FS + k0 + q4];
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
        for (int h = 0; h < 2; ++h) Cs[(r0 + i * 8 + g) * FS + c0 + q * 8 + 2 * q4 + h] -= acc[i][q][h];
  }
  __syncthreads();
  for (int e = tid; e < TL * TL; e += 128) {
    const int r = e / TL, c = e % TL;
    const int gr = ti * TL + r, gc = tj * TL + c;
    if (gr < m && gc < m && (ti != tj || c <= r)) A22[(size_t)gr * ld + gc] = Cs[r * FS + c];
  }
}

// Br[r][d] = A(r, r - d) for d <= kBand, 0 for kBand < d <= 2 kBand.
__global__ void band_copy_kernel(const double* A, int ld, int n, double* Br) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * kBandLd) return;
  const int r = (int)(idx / kBandLd), d = (int)(idx % kBandLd);
  double x = 0.0;
  if (d <= B && r - d >= 0) x = A[(size_t)r * ld + (r - d)];
  Br[idx] = x;
}

}  // namespace

cudaError_t init_sy2sb_attributes() {
  {
    cudaError_t e = init_tsqr_attributes();
    if (e != cudaSuccess) return e;
  }
  for (int v = 0; v < kQrVariants; ++v) {
    cudaError_t e = cudaFuncSetAttribute(qr_kernel(v), cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return e;
    if (qr_smem_bytes(v, kPanelMaxRowsPerCta) > 0) {
      e = cudaFuncSetAttribute(qr_kernel(v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)qr_smem_bytes(v, kPanelMaxRowsPerCta));
      if (e != cudaSuccess) return e;
    }
  }
  cudaError_t e = cudaFuncSetAttribute(symm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSymmSmem);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(syr2k_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSyr2kSmem);
}

// Largest panel-QR cluster this device can run with every variant (0: none),
// probed once.
int probe_max_cluster() {
  for (int C = kPanelMaxCluster; C >= 1; C /= 2) {
    bool ok = true;
    for (int v = 0; v < kQrVariants && ok; ++v) {
      cudaLaunchConfig_t cfg{};
      cfg.gridDim = dim3(C);
      cfg.blockDim = dim3(kQrWarps[v] * 32);
      cfg.dynamicSmemBytes = qr_smem_bytes(v, kPanelMaxRowsPerCta);
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeClusterDimension;
      attr[0].val.clusterDim.x = C;
      attr[0].val.clusterDim.y = 1;
      attr[0].val.clusterDim.z = 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      int clusters = 0;
      if (cudaOccupancyMaxActiveClusters(&clusters, qr_kernel(v), &cfg) != cudaSuccess || clusters < 1) {
        cudaGetLastError();
        ok = false;
      }
    }
    if (ok) return C;
  }
  return 0;
}

int g_max_cluster = -1;

int sy2sb_max_cluster() {
  if (g_max_cluster < 0) g_max_cluster = probe_max_cluster();
  return g_max_cluster;
}

// Largest n whose panels fit the biggest cluster this device can run.
int sy2sb_max_n() {
  const int C = sy2sb_max_cluster();
  return C > 0 ? C * kPanelMaxRowsPerCta + kBand : 0;
}

size_t sy2sb_workspace_doubles(int n) {
  const int m = n;
  const int nt = (m + TL - 1) / TL;
  return (size_t)m * B * (4 + kSymmMaxSplit) + (size_t)nt * B * B + 3 * B * B + B + 256;
}

cudaError_t launch_sy2sb(double* A, int ld, int n, double* ws, double* Br, int num_sms, cudaStream_t s,
                         int rows_per_cta, int panel_qr, const Sy2sbLookAhead* la) {
  const int max_cluster = sy2sb_max_cluster();
  // panel rows per CTA the cluster size aims at: the caller's (autotuned)
  // choice, else MBD_B200_PANEL_ROWS, else the default
  static const int rows_env = [] {
    const char* e = std::getenv("MBD_B200_PANEL_ROWS");
    const int v = e ? std::atoi(e) : 0;
    return (v >= 32 && v <= kPanelMaxRowsPerCta) ? v : kPanelRowsTarget;
  }();
  const int rows_target = (rows_per_cta >= 32 && rows_per_cta <= kPanelMaxRowsPerCta) ? rows_per_cta : rows_env;
  const int nt_full = (n + TL - 1) / TL;
  double* Vb[2];
  Vb[0] = ws;
  double* Y = Vb[0] + (size_t)n * B;
  double* Z = Y + (size_t)n * B;
  double* Yp = Z + (size_t)n * B;
  double* Up = Yp + (size_t)n * B * kSymmMaxSplit;
  double* T = Up + (size_t)nt_full * B * B;
  double* M = T + B * B;
  double* tau = M + B * B;
  Vb[1] = tau + B + 64;   // the next panel's reflectors while this panel's are in use
  // panel QR of the columns c0 .. c0 + B - 1 in one cluster (a power of two of CTAs)
  auto panel_qr_launch = [&](int c0, double* V, cudaStream_t st, bool urgent) -> cudaError_t {
    const int row0 = c0 + B, m = n - row0;
    int C = 1;
    while (C * rows_target < m && C < max_cluster) C *= 2;
    while (C * kPanelMaxRowsPerCta < m) C *= 2;
    if (C > kPanelMaxCluster) return cudaErrorInvalidValue;   // the caller keeps n <= sy2sb_max_n()
    const int R = (m + C - 1) / C;
    PanelArgs pa{A, ld, row0, c0, m, R, V, T, tau};
    if (panel_qr == 1 && C >= 2 && R >= B && R <= tsqr_max_rows_per_cta()) {
      // TSQR with Householder reconstruction: three cluster exchanges per panel
      return launch_tsqr_panel(pa, C, st);
    }
    const int qv = qr_variant(R);
    if (qv < 0) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(C);
    cfg.blockDim = dim3(kQrWarps[qv] * 32);
    cfg.dynamicSmemBytes = qr_smem_bytes(qv, R);
    cfg.stream = st;
    cudaLaunchAttribute attr[2];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = C;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributePriority;
    attr[1].val.priority = urgent && la ? la->priority : 0;
    cfg.attrs = attr;
    cfg.numAttrs = urgent && la ? 2 : 1;
    return cudaLaunchKernelEx(&cfg, qr_kernel(qv), pa);
  };
  bool qr_done = false;   // this panel's QR was launched by the previous panel (look-ahead)
  int p = 0;
  for (int c0 = 0; c0 + B + 1 < n; c0 += B, ++p) {
    const int row0 = c0 + B, m = n - row0;
    double* V = Vb[p & 1];
    if (!qr_done) {
      cudaError_t e = panel_qr_launch(c0, V, s, false);
      if (e != cudaSuccess) return e;
    }
    qr_done = false;
    // two-sided update of the trailing block
    const int nt = (m + TL - 1) / TL;
    int S = (2 * num_sms + nt - 1) / nt;   // one wave at two CTAs per SM
    S = S < 1 ? 1 : (S > kSymmMaxSplit ? kSymmMaxSplit : S);
    if (S > nt) S = nt;
    const int chunk = (nt + S - 1) / S;
    S = (nt + chunk - 1) / chunk;
    symm_kernel<<<dim3(nt, S), 128, kSymmSmem, s>>>(A, ld, row0, m, V, Yp, chunk);
    yred_kernel<<<nt, 256, 0, s>>>(Yp, S, m, T, V, Y, Up);
    mform_kernel<<<1, B * B, 0, s>>>(Up, nt, T, M);
    zform_kernel<<<nt, 256, 0, s>>>(Y, V, M, m, Z);
    const int c1 = c0 + B;
    if (la && c1 + B + 1 < n) {
      // look-ahead: the next panel's columns (tile column 0) first, then its
      // QR on the auxiliary stream beside the rest of the update
      syr2k_kernel<<<nt, 128, kSyr2kSmem, s>>>(A, ld, row0, m, V, Z, 1);
      cudaError_t e = cudaEventRecord(la->ready, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(la->aux, la->ready, 0);
      if (e == cudaSuccess) e = panel_qr_launch(c1, Vb[(p + 1) & 1], la->aux, true);
      if (e == cudaSuccess) e = cudaEventRecord(la->done, la->aux);
      if (e != cudaSuccess) return e;
      if (nt > 1) syr2k_kernel<<<nt * (nt - 1) / 2, 128, kSyr2kSmem, s>>>(A, ld, row0, m, V, Z, 2);
      e = cudaStreamWaitEvent(s, la->done, 0);
      if (e != cudaSuccess) return e;
      qr_done = true;
    } else {
      syr2k_kernel<<<nt * (nt + 1) / 2, 128, kSyr2kSmem, s>>>(A, ld, row0, m, V, Z, 0);
    }
  }
  band_copy_kernel<<<(unsigned)(((long long)n * kBandLd + 255) / 256), 256, 0, s>>>(A, ld, n, Br);
  return cudaGetLastError();
}

int sy2sb_launches(int n) {
  int k = 0;
  for (int c0 = 0; c0 + B + 1 < n; c0 += B) k += 6;
  return k + 1;
}

}  // namespace mbd
