// Block conjugate gradients for the relay system of every frequency at once:
// A(iw_f) X_f = B with B = [I3; ...; I3] (3N x 3), A lower-stored FP64 --
// the solve of get_screened_alpha (UTILS.f90:469-473) by iteration instead of
// PDPOTRF/PDPOTRS, for the MIXED_LEARNED mode.
//
// Preconditioner M^-1: the exact inverses of the 64 x 64 diagonal tiles of A
// (block Jacobi over tiles; the atoms are in spatial order, so a tile holds
// about 21 neighbouring atoms and their strongest couplings).  Iteration (O'Leary's block CG, 3 right-hand sides, one
// recurrence per frequency):
//   Q = A P;  alpha = (P^T Q)^-1 (Z^T R);  X += P alpha;  R -= Q alpha
//   Z = M^-1 R;  beta = (Z_old^T R_old)^-1 (Z^T R);  P = Z + P beta
// Four launches per iteration, all frequencies at once (grid.y = f):
//   cg_tile    tile partials of A P (64 x 64 lower tiles serve both triangles)
//   cg_rows    Q = sum of the partials of each 64-row block; partials of P^T Q
//   cg_update  alpha; X, R, Z = M^-1 R of one 64-row tile per CTA; partials
//              of Z^T R, R^T R
//   cg_dir     beta; P; convergence test ||R||_F^2 <= tol2, after which every
//              later launch returns at once for that frequency
// The 3x3 sums are added in one fixed order by every CTA, so all CTAs of a
// launch take the same decisions.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"

namespace mbd {
namespace {

constexpr int CT = 64;       // tile edge (rows)
constexpr int AT = 64;       // atoms per CTA in the per-atom kernels
constexpr int kRed = 10;     // per-CTA partial sums: a 3x3 matrix and one scalar
// state[f][kCgState]: [0] stop (0 run, 1 converged, 2 breakdown, 3 negative
// curvature), [1] iterations, [2..10] Z^T R (even iterations), [11..19] Z^T R
// (odd), [20] R^T R, [kCgIndefinite] 1 when the relay matrix is shown not to
// be positive definite
constexpr int kZR0 = 2, kRR = 20;

__device__ __forceinline__ void cg_tri(int t, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

// out = m^-1 (3x3, row-major) by cofactors; false when singular or not finite.
__device__ __forceinline__ bool inv3(const double* m, double* out) {
  const double c00 = m[4] * m[8] - m[5] * m[7];
  const double c01 = m[5] * m[6] - m[3] * m[8];
  const double c02 = m[3] * m[7] - m[4] * m[6];
  const double det = m[0] * c00 + m[1] * c01 + m[2] * c02;
  if (!(fabs(det) > 0.0) || !isfinite(det)) return false;
  const double id = 1.0 / det;
  out[0] = c00 * id;
  out[1] = (m[2] * m[7] - m[1] * m[8]) * id;
  out[2] = (m[1] * m[5] - m[2] * m[4]) * id;
  out[3] = c01 * id;
  out[4] = (m[0] * m[8] - m[2] * m[6]) * id;
  out[5] = (m[2] * m[3] - m[0] * m[5]) * id;
  out[6] = c02 * id;
  out[7] = (m[1] * m[6] - m[0] * m[7]) * id;
  out[8] = (m[0] * m[4] - m[1] * m[3]) * id;
  return true;
}

// True when the symmetric part of m (3x3, row-major) has a clearly negative
// pivot in its LDL^T factorisation: some combination p of the search
// directions has p^T A p < 0, which no positive definite A allows.  Pivots
// within 1e-10 of the trace count as a (rank) breakdown, not as a proof.
__device__ __forceinline__ bool negative_curvature(const double* m) {
  const double a = m[0], b = 0.5 * (m[1] + m[3]), c = 0.5 * (m[2] + m[6]);
  const double d = m[4], e = 0.5 * (m[5] + m[7]), f = m[8];
  const double tol = 1e-10 * (fabs(a) + fabs(d) + fabs(f));
  if (a < -tol) return true;
  if (!(a > tol)) return false;
  const double d2 = d - b * b / a;
  if (d2 < -tol) return true;
  if (!(d2 > tol)) return false;
  const double e2 = e - b * c / a;
  const double d3 = f - c * c / a - e2 * e2 / d2;
  return d3 < -tol;
}

__device__ __forceinline__ void mul3(const double* a, const double* b, double* c) {
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) c[3 * i + j] = a[3 * i] * b[j] + a[3 * i + 1] * b[3 + j] + a[3 * i + 2] * b[6 + j];
}

// Sum of `cnt` partial records (kRed doubles each) in a fixed order by warp 0;
// the totals land in out[0..kRed) (shared memory) for the whole CTA.
__device__ void sum_records(const double* rec, int cnt, double* out) {
  if (threadIdx.x < 32) {
    double acc[kRed];
#pragma unroll
    for (int q = 0; q < kRed; ++q) acc[q] = 0.0;
    for (int k = threadIdx.x; k < cnt; k += 32)
#pragma unroll
      for (int q = 0; q < kRed; ++q) acc[q] += rec[(size_t)k * kRed + q];
#pragma unroll
    for (int q = 0; q < kRed; ++q) {
      double v = acc[q];
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
      if (threadIdx.x == 0) out[q] = v;
    }
  }
  __syncthreads();
}

// CTA-wide sums of vals[0..kRed) into dst (global), fixed order.
__device__ void cta_record(const double* vals, double* sm /* [kRed][32] */, double* dst) {
  const int lane = threadIdx.x % 32, warp = threadIdx.x / 32;
  const int nw = (blockDim.x + 31) / 32;
#pragma unroll
  for (int q = 0; q < kRed; ++q) {
    double v = vals[q];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) sm[q * 32 + warp] = v;
  }
  __syncthreads();
  if (threadIdx.x < kRed) {
    double s = 0.0;
    for (int w = 0; w < nw; ++w) s += sm[threadIdx.x * 32 + w];
    dst[threadIdx.x] = s;
  }
}

__device__ __forceinline__ bool stopped(const CgArgs& a, int f) { return a.state[f * kCgState] != 0.0; }

// Minv[f][I] = inverse of the diagonal tile A_II (rows beyond n: the
// identity): Cholesky L L^T = A_II in place, W = L^-1 column by column (W's
// column c kept as row c of the upper triangle, its diagonal in wd), then
// Minv = W^T W.  A tile that is not positive definite gets the identity (the
// iteration then cannot converge and the residual gate sends the geometry to
// the direct solve).
__global__ void __launch_bounds__(256) cg_tile_inv_kernel(CgArgs a) {
  __shared__ double T[CT][CT + 1];
  __shared__ double wd[CT];
  __shared__ int s_bad;
  const int I = blockIdx.x, f = blockIdx.y, tid = threadIdx.x;
  const double* A = a.A + (size_t)f * a.a_stride;
  for (int e = tid; e < CT * CT; e += blockDim.x) {
    const int r = e / CT, c = e % CT;
    const int gr = I * CT + r, gc = I * CT + c;
    double v = (r == c) ? 1.0 : 0.0;
    if (gr < a.n && gc < a.n) v = (c <= r) ? A[(size_t)gr * a.ld + gc] : A[(size_t)gc * a.ld + gr];
    T[r][c] = v;
  }
  if (tid == 0) s_bad = 0;
  __syncthreads();
  for (int k = 0; k < CT; ++k) {
    if (tid == 0) {
      const double d = T[k][k];
      if (!(d > 0.0) || !isfinite(d)) s_bad = 1;
      T[k][k] = sqrt(fmax(d, 1e-300));
    }
    __syncthreads();
    const double lkk = T[k][k];
    for (int i = k + 1 + tid; i < CT; i += blockDim.x) T[i][k] /= lkk;
    __syncthreads();
    const int w = CT - k - 1;
    for (int e = tid; e < w * w; e += blockDim.x) {
      const int i = k + 1 + e / w, j = k + 1 + e % w;
      if (j <= i) T[i][j] -= T[i][k] * T[j][k];
    }
    __syncthreads();
  }
  if (tid < CT) {
    // W(i, c) = (delta_ic - sum_{c <= k < i} L(i, k) W(k, c)) / L(i, i); W(k, c) at T[c][k] (k > c)
    const int c = tid;
    const double wcc = 1.0 / T[c][c];
    wd[c] = wcc;
    for (int i = c + 1; i < CT; ++i) {
      double sum = T[i][c] * wcc;
      for (int k = c + 1; k < i; ++k) sum += T[i][k] * T[c][k];
      T[c][i] = -sum / T[i][i];
    }
  }
  __syncthreads();
  double* M = a.Minv + ((size_t)f * a.nt + I) * CT * CT;
  for (int e = tid; e < CT * CT; e += blockDim.x) {
    const int i = e / CT, j = e % CT;
    double sum = 0.0;
    if (s_bad) {
      sum = (i == j) ? 1.0 : 0.0;
    } else {
      // (W^T W)(i, j) = sum_{k >= max(i, j)} W(k, i) W(k, j)
      const int k0 = i > j ? i : j;
      for (int k = k0; k < CT; ++k) sum += (k == i ? wd[i] : T[i][k]) * (k == j ? wd[j] : T[j][k]);
    }
    M[e] = sum;
  }
}

// partial[f][I][J][64 x 3] = A_IJ v_J, and A_IJ^T v_I into [J][I] (I > J).
// Grid-stride over (tile, frequency) items, so that the launches after every
// frequency has converged cost a few microseconds.  Thread (ty, tx) of 16 x 16
// holds the 16 tile entries of rows ty + 16 i and columns {2 tx, 2 tx + 1,
// 32 + 2 tx, 33 + 2 tx} in registers (16-byte loads, a warp reads two 256-byte
// row segments per instruction), forms their row and column products with v
// (6 FMAs per entry) and the 16 partial sums of every output meet in shared
// memory (fixed order).
constexpr int TT = 256;           // threads of cg_tile
constexpr int RP = CT * 3 + 1;    // row stride of the partial-sum buffer (bank spread)
// Two consecutive entries of a row: 16-byte loads of FP64, 8-byte loads of
// the FP32 copy (half the bytes of the pass).
template <typename T> struct Pair;
template <> struct Pair<double> { using V = double2; };
template <> struct Pair<float> { using V = float2; };
template <typename T>
__device__ __forceinline__ typename Pair<T>::V load_pair(const T* A, size_t o) {
  return *reinterpret_cast<const typename Pair<T>::V*>(A + o);
}
// TA = double: the FP64 pass (FP64 products and sums).  TA = float: the pass
// of the mixed-precision block-CG, products and the per-tile sums of 64
// terms in FP32 (at 2x the FP64 rate: the FP32 pass would otherwise stay
// bound by its 12 FP64 FMAs per entry, not by its halved bytes), the 16
// partial sums of each output added in FP64.  A tile's sums carry a relative
// error of a few 1e-7, below what either phase of that solve resolves.
template <typename TA>
__global__ void __launch_bounds__(TT, sizeof(TA) == 4 ? 4 : 3) cg_tile_kernel(CgArgs a, const TA* Abase,
                                                                            const double* in) {
  using TC = TA;
  __shared__ __align__(16) TC xI[CT * 3], xJ[CT * 3];
  __shared__ TC buf[16 * RP];
  const int ntiles = a.nt * (a.nt + 1) / 2;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  const int n = a.n;
  const long long items = (long long)ntiles * a.batch;
  for (long long item = blockIdx.x; item < items; item += gridDim.x) {
    const int f = (int)(item / ntiles);
    if (stopped(a, f)) {
      // skip to this CTA's first item of the next frequency (uniform over the CTA)
      const long long next = (long long)(f + 1) * ntiles;
      item += (next - item - 1) / gridDim.x * gridDim.x;
      continue;
    }
    int ti, tj;
    cg_tri((int)(item % ntiles), &ti, &tj);
    const bool diag = ti == tj;
    const TA* A = Abase + (size_t)f * a.a_stride;
    const double* x = in + (size_t)f * a.ystride;
    // the 16 entries (pair loads; rows start 16-byte aligned, ld a multiple
    // of 32; an entry beyond n or above the diagonal reads as zero)
    TC t[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = ty + 16 * i, gr = ti * CT + r;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int c = 2 * tx + 32 * h, gc = tj * CT + c;
        typename Pair<TC>::V v;
        v.x = v.y = (TC)0;
        if (gr < n && gc < n && (!diag || c <= r)) v = load_pair(A, (size_t)gr * a.ld + gc);
        t[i][2 * h] = v.x;
        t[i][2 * h + 1] = (gc + 1 < n && (!diag || c + 1 <= r)) ? v.y : (TC)0;
      }
    }
    __syncthreads();   // the previous item's reads of xI / xJ / buf are done
    for (int idx = tid; idx < CT * 3; idx += TT) {
      const int gi = ti * CT + idx / 3, gj = tj * CT + idx / 3;
      xI[idx] = (TC)(gi < n ? x[(size_t)ti * CT * 3 + idx] : 0.0);
      xJ[idx] = (TC)(gj < n ? x[(size_t)tj * CT * 3 + idx] : 0.0);
    }
    __syncthreads();
    TC rs[4][3], cs[4][3];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int q = 0; q < 3; ++q) rs[k][q] = cs[k][q] = (TC)0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = ty + 16 * i;
      TC xi[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) xi[q] = xI[3 * r + q];
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int c = 2 * tx + 32 * (j >> 1) + (j & 1);
        const TC e = t[i][j];
        const TC ec = (!diag || c < r) ? e : (TC)0;   // the diagonal counts once (row side)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          rs[i][q] += e * xJ[3 * c + q];
          cs[j][q] += ec * xi[q];
        }
      }
    }
    double* pr = a.partial + (size_t)f * a.nt * a.nt * CT * 3;
    // row sums: the 16 column groups of each row
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int q = 0; q < 3; ++q) buf[tx * RP + 3 * (ty + 16 * i) + q] = rs[i][q];
    __syncthreads();
    double y = 0.0;
    if (tid < CT * 3) {
#pragma unroll
      for (int k = 0; k < 16; ++k) y += (double)buf[k * RP + tid];
    }
    __syncthreads();
    // column sums: the 16 row groups of each column
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = 2 * tx + 32 * (j >> 1) + (j & 1);
#pragma unroll
      for (int q = 0; q < 3; ++q) buf[ty * RP + 3 * c + q] = cs[j][q];
    }
    __syncthreads();
    if (tid < CT * 3) {
      double z = 0.0;
#pragma unroll
      for (int k = 0; k < 16; ++k) z += (double)buf[k * RP + tid];
      if (!diag) {
        pr[((size_t)ti * a.nt + tj) * CT * 3 + tid] = y;
        pr[((size_t)tj * a.nt + ti) * CT * 3 + tid] = z;
      } else {
        pr[((size_t)ti * a.nt + ti) * CT * 3 + tid] = y + z;
      }
    }
  }
}

// Row sums y = (A v) of 64-row block I.  init: R = B - y.  Otherwise Q = y and
// the block's partial of P^T Q goes to red[f][I].
__global__ void __launch_bounds__(192) cg_rows_kernel(CgArgs a, int init) {
  const int I = blockIdx.x, f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double sm[kRed * 32];
  const int tid = threadIdx.x;
  const int r = tid / 3, q = tid % 3;
  const int gr = I * CT + r;
  const double* pr = a.partial + (size_t)f * a.nt * a.nt * CT * 3 + (size_t)I * a.nt * CT * 3 + tid;
  double y = 0.0;
  for (int J = 0; J < a.nt; ++J) y += pr[(size_t)J * CT * 3];
  const bool live = gr < a.n;
  const size_t o = (size_t)f * a.ystride + (size_t)gr * 3;
  if (init) {
    if (live) a.R[o + q] = ((gr % 3) == q ? 1.0 : 0.0) - y;
    return;
  }
  if (live) a.Q[o + q] = y;
  double vals[kRed];
#pragma unroll
  for (int k = 0; k < kRed; ++k) vals[k] = 0.0;
  if (live) {
    // thread (row, q) adds P[row][c] Q[row][q] to entry (c, q)
#pragma unroll
    for (int c = 0; c < 3; ++c) vals[3 * c + q] = a.P[o + c] * y;
  }
  cta_record(vals, sm, a.red + ((size_t)f * a.nt + I) * kRed);
}

// One thread per (atom, rhs column): loads the atom's 3x3 block of v.
__device__ __forceinline__ void load_block(const double* v, size_t base, int i, double* out) {
#pragma unroll
  for (int k = 0; k < 9; ++k) out[k] = v[base + (size_t)9 * i + k];
}

// Shared memory of the per-tile preconditioner step.
struct TileSmem {
  double Ms[CT][CT + 1];   // M^-1 of the tile
  double Rs[CT][3], Zs[CT][3];
  double red[kRed * 32];
};

// Thread (r, q) of a 192-thread CTA on 64-row tile I of frequency f holds
// R(64 I + r, q) in rv (0 beyond n): Z = M^-1 R on the tile (written to a.Z,
// and to a.P when also_p), then the CTA's partials of Z^T R and R^T R.
__device__ void tile_precondition(const CgArgs& a, int f, int I, double rv, bool also_p, TileSmem& S) {
  const int tid = threadIdx.x, r = tid / 3, q = tid % 3;
  const double* Mg = a.Minv + ((size_t)f * a.nt + I) * CT * CT;
  for (int e = tid; e < CT * CT / 2; e += blockDim.x) {
    const double2 v = reinterpret_cast<const double2*>(Mg)[e];
    const int rr = (2 * e) / CT, cc = (2 * e) % CT;
    S.Ms[rr][cc] = v.x;
    S.Ms[rr][cc + 1] = v.y;
  }
  S.Rs[r][q] = rv;
  __syncthreads();
  double z0 = 0.0, z1 = 0.0;   // two accumulation chains
#pragma unroll 8
  for (int k = 0; k < CT; k += 2) {
    z0 += S.Ms[r][k] * S.Rs[k][q];
    z1 += S.Ms[r][k + 1] * S.Rs[k + 1][q];
  }
  const double z = z0 + z1;
  S.Zs[r][q] = z;
  const int gr = I * CT + r;
  if (gr < a.n) {
    const size_t o = (size_t)f * a.ystride + (size_t)gr * 3 + q;
    a.Z[o] = z;
    if (also_p) a.P[o] = z;
  }
  __syncthreads();
  double vals[kRed];
#pragma unroll
  for (int k = 0; k < kRed; ++k) vals[k] = 0.0;
  // (Z^T R)(c, q) = sum_rows Z[row][c] R[row][q]
#pragma unroll
  for (int c = 0; c < 3; ++c) vals[3 * c + q] = S.Zs[r][c] * rv;
  vals[9] = rv * rv;
  cta_record(vals, S.red, a.red2 + ((size_t)f * a.nt + I) * kRed);
}

// init: Z = M^-1 R, P = Z on one 64-row tile; partials of Z^T R and R^T R.
__global__ void __launch_bounds__(192) cg_init_tiles_kernel(CgArgs a) {
  const int I = blockIdx.x, f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ TileSmem S;
  const int r = threadIdx.x / 3, q = threadIdx.x % 3, gr = I * CT + r;
  const double rv = gr < a.n ? a.R[(size_t)f * a.ystride + (size_t)gr * 3 + q] : 0.0;
  tile_precondition(a, f, I, rv, true, S);
}

// Between the phases: frequencies stopped as converged (1) or broken down
// (2) run again, negative curvature (3) stays; the first phase's iteration
// count is kept in kCgPhase1Iters.  Must run before any kernel that tests
// the stop flag in the restart.
__global__ void cg_reopen_kernel(CgArgs a) {
  const int f = blockIdx.x * blockDim.x + threadIdx.x;
  if (f >= a.batch) return;
  double* st = a.state + f * kCgState;
  st[kCgPhase1Iters] = st[1];
  if (st[0] == 1.0 || st[0] == 2.0) st[0] = 0.0;
}

// init: Z^T R and R^T R into the state; stop when already converged.
__global__ void cg_init_final_kernel(CgArgs a, int nb) {
  const int f = blockIdx.x;
  __shared__ double tot[kRed];
  if (stopped(a, f)) return;
  sum_records(a.red2 + (size_t)f * nb * kRed, nb, tot);
  if (threadIdx.x == 0) {
    double* st = a.state + f * kCgState;
    for (int k = 0; k < 9; ++k) st[kZR0 + k] = tot[k];
    st[kRR] = tot[9];
    st[1] = 0.0;
    if (tot[9] <= a.tol2) st[0] = 1.0;
  }
}

// alpha = (P^T Q)^-1 (Z^T R); X += P alpha; R -= Q alpha on one 64-row
// tile; Z = M^-1 R; partials of Z^T R (new) and R^T R into red2.
__global__ void __launch_bounds__(192) cg_update_kernel(CgArgs a, int it) {
  const int I = blockIdx.x, f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double tot[kRed];
  __shared__ double s_alpha[9];
  __shared__ int s_indef;
  __shared__ TileSmem S;
  sum_records(a.red + (size_t)f * a.nt * kRed, a.nt, tot);
  if (threadIdx.x == 0) {
    const double* zr = a.state + f * kCgState + kZR0 + 9 * (it & 1);
    double pq[9], ipq[9], al[9];
    for (int k = 0; k < 9; ++k) pq[k] = tot[k];
    // P^T A P with a negative direction: A is not positive definite (the
    // reference's unchecked PDPOTRF info, UTILS.f90:469).  Every CTA sees the
    // same sums and stops; CTA 0 records it and ends this frequency's solve.
    s_indef = negative_curvature(pq) ? 1 : 0;
    if (s_indef && I == 0) {
      double* st = a.state + f * kCgState;
      st[kCgIndefinite] = 1.0;
      st[0] = 3.0;
    }
    if (inv3(pq, ipq)) {
      mul3(ipq, zr, al);
    } else {
      for (int k = 0; k < 9; ++k) al[k] = 0.0;
    }
    for (int k = 0; k < 9; ++k) s_alpha[k] = al[k];
  }
  __syncthreads();
  if (s_indef) return;
  const int r = threadIdx.x / 3, q = threadIdx.x % 3, gr = I * CT + r;
  double rv = 0.0;
  if (gr < a.n) {
    const size_t o = (size_t)f * a.ystride + (size_t)gr * 3;
    double x = a.X[o + q], rr = a.R[o + q];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      x += a.P[o + c] * s_alpha[3 * c + q];
      rr -= a.Q[o + c] * s_alpha[3 * c + q];
    }
    a.X[o + q] = x;
    a.R[o + q] = rr;
    rv = rr;
  }
  tile_precondition(a, f, I, rv, false, S);
}

// beta = (Z^T R)_old^-1 (Z^T R)_new; P = Z + P beta; convergence test.
__global__ void __launch_bounds__(AT) cg_dir_kernel(CgArgs a, int it) {
  const int f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double tot[kRed];
  __shared__ double s_beta[9];
  __shared__ int s_done;
  sum_records(a.red2 + (size_t)f * a.nt * kRed, a.nt, tot);   // one record per 64-row tile
  double* st = a.state + f * kCgState;
  if (threadIdx.x == 0) {
    const double* zr_old = st + kZR0 + 9 * (it & 1);
    double zo[9], izo[9], zn[9], be[9];
    for (int k = 0; k < 9; ++k) {
      zo[k] = zr_old[k];
      zn[k] = tot[k];
    }
    int done = 0;
    if (tot[9] <= a.tol2) {
      done = 1;
    } else if (!inv3(zo, izo)) {
      done = 2;
    } else {
      mul3(izo, zn, be);
      for (int k = 0; k < 9; ++k) s_beta[k] = be[k];
    }
    s_done = done;
    if (blockIdx.x == 0) {
      double* zr_new = st + kZR0 + 9 * ((it + 1) & 1);
      for (int k = 0; k < 9; ++k) zr_new[k] = zn[k];
      st[kRR] = tot[9];
      st[1] = (double)(it + 1);
    }
  }
  __syncthreads();
  if (s_done) {
    // every CTA reads the old flag at entry; CTA 0 raises it after its own
    // update, so no CTA of this launch sees it change
    __syncthreads();
    if (blockIdx.x == 0 && threadIdx.x == 0) st[0] = (double)s_done;
    return;
  }
  const int i = blockIdx.x * AT + threadIdx.x;
  if (i < a.N) {
    const size_t base = (size_t)f * a.ystride;
    double Z[9], P[9], t[9];
    load_block(a.Z, base, i, Z);
    load_block(a.P, base, i, P);
    mul3(P, s_beta, t);
#pragma unroll
    for (int k = 0; k < 9; ++k) a.P[base + 9 * (size_t)i + k] = Z[k] + t[k];
  }
}

}  // namespace

size_t cg_minv_doubles(int n, int batch) {
  const int nt = (n + CT - 1) / CT;
  return (size_t)batch * nt * CT * CT;
}

// CTAs of the grid-stride tile launch: every resident slot of the device.
template <typename TA>
int cg_tile_grid() {
  static int grid = 0;
  if (grid == 0) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, cg_tile_kernel<TA>, TT, 0);
    grid = (sms > 0 ? sms : 148) * (per_sm > 0 ? per_sm : 1);
  }
  return grid;
}

size_t cg_partial_doubles(int n, int batch) {
  const int nt = (n + CT - 1) / CT;
  return (size_t)batch * nt * nt * CT * 3;
}

size_t cg_red_doubles(int n, int batch) {
  const int nt = (n + CT - 1) / CT;
  const int nb = (n / 3 + AT - 1) / AT;
  return (size_t)batch * (nt > nb ? nt : nb) * kRed;
}

void launch_cg_setup(const CgArgs& a, cudaStream_t s) {
  const long long items = (long long)a.nt * (a.nt + 1) / 2 * a.batch;
  const int tgrid = (int)std::min<long long>(cg_tile_grid<double>(), items);
  cudaMemsetAsync(a.state, 0, sizeof(double) * kCgState * a.batch, s);
  cg_tile_inv_kernel<<<dim3(a.nt, a.batch), 256, 0, s>>>(a);
  cg_tile_kernel<double><<<tgrid, TT, 0, s>>>(a, a.A, a.X);
  cg_rows_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a, 1);
  cg_init_tiles_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a);
  cg_init_final_kernel<<<a.batch, 32, 0, s>>>(a, a.nt);
}

void launch_cg_restart(const CgArgs& a, cudaStream_t s) {
  const long long items = (long long)a.nt * (a.nt + 1) / 2 * a.batch;
  const int tgrid = (int)std::min<long long>(cg_tile_grid<double>(), items);
  cg_reopen_kernel<<<(a.batch + 31) / 32, 32, 0, s>>>(a);
  cg_tile_kernel<double><<<tgrid, TT, 0, s>>>(a, a.A, a.X);
  cg_rows_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a, 1);
  cg_init_tiles_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a);
  cg_init_final_kernel<<<a.batch, 32, 0, s>>>(a, a.nt);
}

void launch_cg_iteration(const CgArgs& a, int it, cudaStream_t s, bool fp32) {
  const int nb = (a.N + AT - 1) / AT;
  const long long items = (long long)a.nt * (a.nt + 1) / 2 * a.batch;
  const int tgrid = (int)std::min<long long>(cg_tile_grid<double>(), items);
  if (fp32 && a.A32)
    cg_tile_kernel<float><<<(int)std::min<long long>(cg_tile_grid<float>(), items), TT, 0, s>>>(a, a.A32, a.P);
  else
    cg_tile_kernel<double><<<tgrid, TT, 0, s>>>(a, a.A, a.P);
  cg_rows_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a, 0);
  cg_update_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a, it);
  cg_dir_kernel<<<dim3(nb, a.batch), AT, 0, s>>>(a, it);
}

}  // namespace mbd
