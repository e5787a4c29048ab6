// Block conjugate gradients for the relay system of every frequency at once:
// A(iw_f) X_f = B with B = [I3; ...; I3] (3N x 3), A lower-stored FP64 --
// the solve of get_screened_alpha (UTILS.f90:469-473) by iteration instead of
// PDPOTRF/PDPOTRS, for the MIXED_LEARNED mode.
//
// Preconditioner M^-1: the exact inverses of the 3x3 diagonal blocks of A
// (block Jacobi).  Iteration (O'Leary's block CG, 3 right-hand sides, one
// recurrence per frequency):
//   Q = A P;  alpha = (P^T Q)^-1 (Z^T R);  X += P alpha;  R -= Q alpha
//   Z = M^-1 R;  beta = (Z_old^T R_old)^-1 (Z^T R);  P = Z + P beta
// Four launches per iteration, all frequencies at once (grid.y = f):
//   cg_tile    tile partials of A P (64 x 64 lower tiles serve both triangles)
//   cg_rows    Q = sum of the partials of each 64-row block; partials of P^T Q
//   cg_update  alpha; X, R, Z of 64 atoms per CTA; partials of Z^T R, R^T R
//   cg_dir     beta; P; convergence test ||R||_F^2 <= tol2, after which every
//              later launch returns at once for that frequency
// The 3x3 sums are added in one fixed order by every CTA, so all CTAs of a
// launch take the same decisions.
#include <cuda_runtime.h>

#include "kernels.h"

namespace mbd {
namespace {

constexpr int CT = 64;       // tile edge (rows)
constexpr int AT = 64;       // atoms per CTA in the per-atom kernels
constexpr int kRed = 10;     // per-CTA partial sums: a 3x3 matrix and one scalar
// state[f][kCgState]: [0] stop (0 run, 1 converged, 2 breakdown), [1] iterations,
// [2..10] Z^T R (even iterations), [11..19] Z^T R (odd), [20] R^T R
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

// Dinv[f][i] = inverse of the diagonal 3x3 block of atom i.
__global__ void __launch_bounds__(256) cg_jacobi_kernel(CgArgs a) {
  const int f = blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.N) return;
  const double* A = a.A + (size_t)f * a.a_stride;
  double m[9], inv[9];
#pragma unroll
  for (int r = 0; r < 3; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const int rr = 3 * i + (r > c ? r : c), cc = 3 * i + (r > c ? c : r);
      m[3 * r + c] = A[(size_t)rr * a.ld + cc];
    }
  if (!inv3(m, inv)) {
#pragma unroll
    for (int q = 0; q < 9; ++q) inv[q] = (q % 4 == 0) ? 1.0 : 0.0;
  }
  double* out = a.Dinv + ((size_t)f * a.N + i) * 9;
#pragma unroll
  for (int q = 0; q < 9; ++q) out[q] = inv[q];
}

// partial[f][I][J][64 x 3] = A_IJ v_J, and A_IJ^T v_I into [J][I] (I > J).
__global__ void __launch_bounds__(192) cg_tile_kernel(CgArgs a, const double* in) {
  const int f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double Ts[CT][CT + 1];
  __shared__ double xI[CT][3], xJ[CT][3];
  int ti, tj;
  cg_tri(blockIdx.x, &ti, &tj);
  const double* A = a.A + (size_t)f * a.a_stride;
  const double* x = in + (size_t)f * a.ystride;
  const int tid = threadIdx.x;
  const bool diag = ti == tj;
  const int n = a.n;
  // 16-byte loads (rows start 16-byte aligned: ld is a multiple of 32; the
  // second element of a pair may lie in the row padding, masked below)
  for (int idx = tid; idx < CT * CT / 2; idx += blockDim.x) {
    const int r = idx / (CT / 2), c = 2 * (idx % (CT / 2));
    const int gr = ti * CT + r, gc = tj * CT + c;
    double2 v = make_double2(0.0, 0.0);
    if (gr < n && gc < n && (!diag || c <= r)) v = *reinterpret_cast<const double2*>(A + (size_t)gr * a.ld + gc);
    Ts[r][c] = v.x;
    Ts[r][c + 1] = (gc + 1 < n && (!diag || c + 1 <= r)) ? v.y : 0.0;
  }
  for (int idx = tid; idx < CT * 3; idx += blockDim.x) {
    const int r = idx / 3, q = idx % 3;
    const int gi = ti * CT + r, gj = tj * CT + r;
    xI[r][q] = gi < n ? x[(size_t)gi * 3 + q] : 0.0;
    xJ[r][q] = gj < n ? x[(size_t)gj * 3 + q] : 0.0;
  }
  __syncthreads();
  const int r = tid / 3, q = tid % 3;
  double rs = 0.0, cs = 0.0;
#pragma unroll 8
  for (int c = 0; c < CT; ++c) rs += Ts[r][c] * xJ[c][q];
  if (!diag) {
#pragma unroll 8
    for (int c = 0; c < CT; ++c) cs += Ts[c][r] * xI[c][q];
  } else {
    for (int c = r + 1; c < CT; ++c) cs += Ts[c][r] * xI[c][q];
  }
  double* pr = a.partial + (size_t)f * a.nt * a.nt * CT * 3;
  if (!diag) {
    pr[((size_t)ti * a.nt + tj) * CT * 3 + tid] = rs;
    pr[((size_t)tj * a.nt + ti) * CT * 3 + tid] = cs;
  } else {
    pr[((size_t)ti * a.nt + ti) * CT * 3 + tid] = rs + cs;
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

// init: Z = M^-1 R, P = Z; partials of Z^T R and R^T R into red2.
__global__ void __launch_bounds__(AT) cg_init_atoms_kernel(CgArgs a) {
  const int f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double sm[kRed * 32];
  const int i = blockIdx.x * AT + threadIdx.x;
  double vals[kRed];
#pragma unroll
  for (int k = 0; k < kRed; ++k) vals[k] = 0.0;
  if (i < a.N) {
    const size_t base = (size_t)f * a.ystride;
    double R[9], D[9], Z[9];
    load_block(a.R, base, i, R);
    load_block(a.Dinv, (size_t)f * a.N * 9, i, D);
    mul3(D, R, Z);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      a.Z[base + 9 * (size_t)i + k] = Z[k];
      a.P[base + 9 * (size_t)i + k] = Z[k];
    }
    // (Z^T R)(c, d) = sum_rows Z[row][c] R[row][d]
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = 0; d < 3; ++d) vals[3 * c + d] = Z[c] * R[d] + Z[3 + c] * R[3 + d] + Z[6 + c] * R[6 + d];
#pragma unroll
    for (int k = 0; k < 9; ++k) vals[9] += R[k] * R[k];
  }
  cta_record(vals, sm, a.red2 + ((size_t)f * gridDim.x + blockIdx.x) * kRed);
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

// alpha = (P^T Q)^-1 (Z^T R); X += P alpha; R -= Q alpha; Z = M^-1 R;
// partials of Z^T R (new) and R^T R into red2.
__global__ void __launch_bounds__(AT) cg_update_kernel(CgArgs a, int it) {
  const int f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double tot[kRed];
  __shared__ double sm[kRed * 32];
  __shared__ double s_alpha[9];
  sum_records(a.red + (size_t)f * a.nt * kRed, a.nt, tot);
  if (threadIdx.x == 0) {
    const double* zr = a.state + f * kCgState + kZR0 + 9 * (it & 1);
    double pq[9], ipq[9], al[9];
    for (int k = 0; k < 9; ++k) pq[k] = tot[k];
    if (inv3(pq, ipq)) {
      mul3(ipq, zr, al);
    } else {
      for (int k = 0; k < 9; ++k) al[k] = 0.0;
    }
    for (int k = 0; k < 9; ++k) s_alpha[k] = al[k];
  }
  __syncthreads();
  const int i = blockIdx.x * AT + threadIdx.x;
  double vals[kRed];
#pragma unroll
  for (int k = 0; k < kRed; ++k) vals[k] = 0.0;
  if (i < a.N) {
    const size_t base = (size_t)f * a.ystride;
    double X[9], R[9], P[9], Q[9], D[9], Z[9], t[9];
    load_block(a.X, base, i, X);
    load_block(a.R, base, i, R);
    load_block(a.P, base, i, P);
    load_block(a.Q, base, i, Q);
    load_block(a.Dinv, (size_t)f * a.N * 9, i, D);
    mul3(P, s_alpha, t);
#pragma unroll
    for (int k = 0; k < 9; ++k) X[k] += t[k];
    mul3(Q, s_alpha, t);
#pragma unroll
    for (int k = 0; k < 9; ++k) R[k] -= t[k];
    mul3(D, R, Z);
#pragma unroll
    for (int k = 0; k < 9; ++k) {
      a.X[base + 9 * (size_t)i + k] = X[k];
      a.R[base + 9 * (size_t)i + k] = R[k];
      a.Z[base + 9 * (size_t)i + k] = Z[k];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int d = 0; d < 3; ++d) vals[3 * c + d] = Z[c] * R[d] + Z[3 + c] * R[3 + d] + Z[6 + c] * R[6 + d];
#pragma unroll
    for (int k = 0; k < 9; ++k) vals[9] += R[k] * R[k];
  }
  cta_record(vals, sm, a.red2 + ((size_t)f * gridDim.x + blockIdx.x) * kRed);
}

// beta = (Z^T R)_old^-1 (Z^T R)_new; P = Z + P beta; convergence test.
__global__ void __launch_bounds__(AT) cg_dir_kernel(CgArgs a, int it) {
  const int f = blockIdx.y;
  if (stopped(a, f)) return;
  __shared__ double tot[kRed];
  __shared__ double s_beta[9];
  __shared__ int s_done;
  sum_records(a.red2 + (size_t)f * gridDim.x * kRed, gridDim.x, tot);
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
  const int nb = (a.N + AT - 1) / AT;
  cudaMemsetAsync(a.state, 0, sizeof(double) * kCgState * a.batch, s);
  cg_jacobi_kernel<<<dim3((a.N + 255) / 256, a.batch), 256, 0, s>>>(a);
  cg_tile_kernel<<<dim3(a.nt * (a.nt + 1) / 2, a.batch), 192, 0, s>>>(a, a.X);
  cg_rows_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a, 1);
  cg_init_atoms_kernel<<<dim3(nb, a.batch), AT, 0, s>>>(a);
  cg_init_final_kernel<<<a.batch, 32, 0, s>>>(a, nb);
}

void launch_cg_iteration(const CgArgs& a, int it, cudaStream_t s) {
  const int nb = (a.N + AT - 1) / AT;
  cg_tile_kernel<<<dim3(a.nt * (a.nt + 1) / 2, a.batch), 192, 0, s>>>(a, a.P);
  cg_rows_kernel<<<dim3(a.nt, a.batch), 192, 0, s>>>(a, 0);
  cg_update_kernel<<<dim3(nb, a.batch), AT, 0, s>>>(a, it);
  cg_dir_kernel<<<dim3(nb, a.batch), AT, 0, s>>>(a, it);
}

}  // namespace mbd
