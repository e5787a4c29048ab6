// FP64 eigenvalues of the CFDM Hamiltonian and the MBD energy
// (PDSYEV('N','L') at UTILS.f90:835, energy at UTILS.f90:839-867).
//
// 1. tridiag_kernel: Householder reduction of the row-major lower matrix to
//    tridiagonal (d, e), blocked in panels of 32 columns as LAPACK's
//    DSYTRD/DLATRD: per column, a symmetric matrix-vector product over the
//    trailing matrix (64x64 tiles spread over the group's CTAs), the panel
//    corrections, and the next column's update; per panel, a rank-64 update
//    A22 -= V W^T + W V^T.  The whole reduction is ONE cooperative launch:
//    the CTAs of a group meet at bounded global-memory barriers (three per
//    column), so no launch gaps separate the ~3n dependent steps.
// 2. bisect_kernel: every eigenvalue by bisection on a division-free Sturm
//    count (three-term determinant recurrence with power-of-two rescaling).
// 3. energy_kernel: E = 0.5 sum_{lambda>=0} sqrt(lambda)/n_SL - 0.5 sum 3 omega
//    with compensated (TwoSum) summation; NIMAG = #lambda<0.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int T = kTrdTile;   // 64
constexpr int P = kTrdNB;     // 32 panel width
constexpr int THREADS = 512;
constexpr long long kSpinCycles = 4000000000LL;   // ~2 s at 2 GHz, then give up

struct GroupWS {
  unsigned* bar;   // [0] arrivals, [1] generation
  double* W;       // [nmax][P]
  double* V;       // [nmax][P]
  double* Wpre;    // [nmax]
  double* Pb;      // [nt][nt][T]
  double* dotp;    // [G][2P]
  double* scal;    // [G][4]
};

__host__ __device__ inline size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

__host__ __device__ inline size_t ws_layout(int nmax, int G, GroupWS* w, char* base) {
  const int nt = (nmax + T - 1) / T;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    size_t o = off;
    off = align_up(off + bytes);
    return o;
  };
  size_t o_bar = take(256);
  size_t o_W = take(sizeof(double) * (size_t)nmax * P);
  size_t o_V = take(sizeof(double) * (size_t)nmax * P);
  size_t o_Wp = take(sizeof(double) * (size_t)nmax);
  size_t o_Pb = take(sizeof(double) * (size_t)nt * nt * T);
  size_t o_dp = take(sizeof(double) * (size_t)G * 2 * P);
  size_t o_sc = take(sizeof(double) * (size_t)G * 4);
  if (w) {
    w->bar = reinterpret_cast<unsigned*>(base + o_bar);
    w->W = reinterpret_cast<double*>(base + o_W);
    w->V = reinterpret_cast<double*>(base + o_V);
    w->Wpre = reinterpret_cast<double*>(base + o_Wp);
    w->Pb = reinterpret_cast<double*>(base + o_Pb);
    w->dotp = reinterpret_cast<double*>(base + o_dp);
    w->scal = reinterpret_cast<double*>(base + o_sc);
  }
  return off;
}

__device__ __forceinline__ double ldg_cg(const double* p) { return __ldcg(p); }

// Bounded barrier among the G CTAs of one group.  Returns false (and sets
// *err) when the wait runs out or another CTA already failed.
__device__ bool group_sync(unsigned* bar, int G, unsigned& gen, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned target = gen + 1;
    __threadfence();
    const unsigned arrived = atomicAdd(&bar[0], 1u);
    if (arrived == (unsigned)G - 1) {
      atomicExch(&bar[0], 0u);
      __threadfence();
      atomicExch(&bar[1], target);
    } else {
      const long long t0 = clock64();
      while (*(volatile unsigned*)&bar[1] != target) {
        if (*(volatile int*)err != 0 || clock64() - t0 > kSpinCycles) {
          ok = 0;
          atomicCAS(err, 0, MBD_ERR_TIMEOUT);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    gen = target;
    s_ok = ok && (*(volatile int*)err == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

struct Refl {
  double tau, scale, beta;
};

// v(r) of the reflector of column c (v(c+1) = 1, v(r>c+1) = A[r][c]*scale, else 0).
__device__ __forceinline__ double vval(const double* A, int ld, int n, int c, double scale, int r) {
  if (r == c + 1) return 1.0;
  if (r > c + 1 && r < n) return ldg_cg(A + (size_t)r * ld + c) * scale;
  return 0.0;
}

__device__ double block_sum(double v, double* red) {
  // red: >= THREADS/32 doubles
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0) {
    for (int w = 0; w < THREADS / 32; ++w) s += red[w];
    red[0] = s;
  }
  __syncthreads();
  s = red[0];
  __syncthreads();
  return s;
}

__device__ __forceinline__ void tri_index(int t, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

struct Smem {
  double vI[T], vJ[T], rows[T];
  double red[THREADS / 32 * T];   // 16 x 64 column partials
  double t1[P], t2[P], wc[P], vc[P];
  double small[THREADS / 32];
};

// y contributions of the trailing tiles for column c.
__device__ void symv_tiles(const double* A, int ld, int n, int c, double scale, const GroupWS& w,
                           int nt, int g, int G, Smem& sm) {
  const int I0 = (c + 1) / T;
  const int mt = nt - I0;
  const int ntile = mt * (mt + 1) / 2;
  const int tid = threadIdx.x;
  const int row = tid / 8, cg = tid % 8, warp = tid / 32, lane = tid % 32;
  for (int t = g; t < ntile; t += G) {
    int ti, tj;
    tri_index(t, &ti, &tj);
    const int I = I0 + ti, J = I0 + tj;
    __syncthreads();
    if (tid < T) sm.vI[tid] = vval(A, ld, n, c, scale, I * T + tid);
    else if (tid < 2 * T) sm.vJ[tid - T] = vval(A, ld, n, c, scale, J * T + tid - T);
    __syncthreads();
    const int r = I * T + row;
    double a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int col = cg + 8 * q;
      const int s = J * T + col;
      const bool ok = r < n && s < n && (I != J || col <= row);
      a[q] = ok ? ldg_cg(A + (size_t)r * ld + s) : 0.0;
    }
    double rs = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) rs += a[q] * sm.vJ[cg + 8 * q];
    rs += __shfl_xor_sync(0xffffffffu, rs, 1);
    rs += __shfl_xor_sync(0xffffffffu, rs, 2);
    rs += __shfl_xor_sync(0xffffffffu, rs, 4);
    const double vr = sm.vI[row];
    double cp[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int col = cg + 8 * q;
      cp[q] = (I != J || col < row) ? a[q] * vr : 0.0;
      cp[q] += __shfl_xor_sync(0xffffffffu, cp[q], 8);
      cp[q] += __shfl_xor_sync(0xffffffffu, cp[q], 16);
    }
    if (lane < 8) {
#pragma unroll
      for (int q = 0; q < 8; ++q) sm.red[warp * T + lane + 8 * q] = cp[q];
    }
    if (cg == 0) sm.rows[row] = rs;
    __syncthreads();
    if (tid < T) {
      double cs = 0.0;
#pragma unroll
      for (int wv = 0; wv < THREADS / 32; ++wv) cs += sm.red[wv * T + tid];
      if (I != J) {
        w.Pb[((size_t)I * nt + J) * T + tid] = sm.rows[tid];
        w.Pb[((size_t)J * nt + I) * T + tid] = cs;
      } else {
        w.Pb[((size_t)I * nt + I) * T + tid] = sm.rows[tid] + cs;
      }
    }
  }
}

// A22 -= V W^T + W V^T over rows/cols >= q0 (end of a panel).
__device__ void syr2k_tiles(double* A, int ld, int n, int q0, const GroupWS& w, int nt, int g, int G,
                            double* dyn) {
  double* Vr = dyn;                 // [T][P+1]
  double* Wr = dyn + T * (P + 1);
  double* Vs = dyn + 2 * T * (P + 1);
  double* Ws = dyn + 3 * T * (P + 1);
  const int I0 = q0 / T;
  const int mt = nt - I0;
  const int ntile = mt * (mt + 1) / 2;
  const int tid = threadIdx.x;
  const int row = tid / 8, cg = tid % 8;
  for (int t = g; t < ntile; t += G) {
    int ti, tj;
    tri_index(t, &ti, &tj);
    const int I = I0 + ti, J = I0 + tj;
    __syncthreads();
    for (int idx = tid; idx < T * P; idx += THREADS) {
      const int rr = idx / P, k = idx % P;
      const int ri = I * T + rr, sj = J * T + rr;
      Vr[rr * (P + 1) + k] = ri < n ? ldg_cg(w.V + (size_t)ri * P + k) : 0.0;
      Wr[rr * (P + 1) + k] = ri < n ? ldg_cg(w.W + (size_t)ri * P + k) : 0.0;
      Vs[rr * (P + 1) + k] = sj < n ? ldg_cg(w.V + (size_t)sj * P + k) : 0.0;
      Ws[rr * (P + 1) + k] = sj < n ? ldg_cg(w.W + (size_t)sj * P + k) : 0.0;
    }
    __syncthreads();
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int k = 0; k < P; ++k) {
      const double vr = Vr[row * (P + 1) + k], wr = Wr[row * (P + 1) + k];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int col = cg + 8 * q;
        acc[q] += vr * Ws[col * (P + 1) + k] + wr * Vs[col * (P + 1) + k];
      }
    }
    const int r = I * T + row;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int s = J * T + cg + 8 * q;
      if (r < n && s <= r && s >= q0 && r >= q0) {
        double* p = A + (size_t)r * ld + s;
        *p = ldg_cg(p) - acc[q];
      }
    }
  }
}

__device__ bool tridiag_one(const TridiagJob& job, const GroupWS& w, int g, int G, unsigned& gen,
                            int* err, Smem& sm, double* dyn) {
  double* A = job.A;
  const int n = job.n, ld = job.ld;
  const int nt = (n + T - 1) / T;
  const int tid = threadIdx.x;
  if (n == 1) {
    if (g == 0 && tid == 0) job.d[0] = A[0];
    return group_sync(w.bar, G, gen, err);
  }
  // norm partials of column 0 below the subdiagonal; d[0]
  {
    double s = 0.0;
    for (int X = 0; X < nt; ++X) {
      if (X % G != g) continue;
      const int r = X * T + (tid % T);
      if (tid < T && r >= 2 && r < n) {
        const double x = ldg_cg(A + (size_t)r * ld);
        s += x * x;
      }
    }
    s = block_sum(s, sm.small);
    if (tid == 0) w.scal[g * 4 + 0] = s;
    if (g == 0 && tid == 0) job.d[0] = ldg_cg(A);
  }
  if (!group_sync(w.bar, G, gen, err)) return false;

  for (int c = 0; c <= n - 2; ++c) {
    const int p = c - c % P, j = c - p;
    const int c1 = c + 1;
    const int I0 = c1 / T;
    // ---------------- phase 1: reflector, SYMV, panel dots ----------------
    __shared__ Refl rf;
    if (tid == 0) {
      const double alpha = ldg_cg(A + (size_t)c1 * ld + c);
      double xn2 = 0.0;
      for (int q = 0; q < G; ++q) xn2 += ldg_cg(w.scal + q * 4 + 0);
      Refl r;
      if (xn2 == 0.0) {
        r.tau = 0.0;
        r.scale = 0.0;
        r.beta = alpha;
      } else {
        const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
        r.tau = (beta - alpha) / beta;
        r.scale = 1.0 / (alpha - beta);
        r.beta = beta;
      }
      rf = r;
      if (g == 0) job.e[c] = r.beta;
    }
    __syncthreads();
    const Refl r = rf;
    if (r.tau != 0.0) {
      symv_tiles(A, ld, n, c, r.scale, w, nt, g, G, sm);
      // partial dots t1 = W^T v, t2 = V^T v over own row blocks (k < j)
      if (j > 0) {
        const int warp = tid / 32, lane = tid % 32;
        for (int k2 = warp; k2 < 2 * j; k2 += THREADS / 32) {
          const int k = k2 % j;
          const double* M = (k2 < j) ? w.W : w.V;
          double s = 0.0;
          for (int X = I0; X < nt; ++X) {
            if (X % G != g) continue;
            for (int rr = lane; rr < T; rr += 32) {
              const int row = X * T + rr;
              if (row >= c1 && row < n) s += ldg_cg(M + (size_t)row * P + k) * vval(A, ld, n, c, r.scale, row);
            }
          }
          for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
          if (lane == 0) w.dotp[(size_t)g * 2 * P + (k2 < j ? k : P + k)] = s;
        }
      }
    }
    // V column j for own rows
    for (int X = 0; X < nt; ++X) {
      if (X % G != g) continue;
      const int row = X * T + (tid % T);
      if (tid < T && row < n) w.V[(size_t)row * P + j] = vval(A, ld, n, c, r.scale, row);
    }
    if (!group_sync(w.bar, G, gen, err)) return false;

    // ---------------- phase 2: w_pre = tau (y - V t1 - W t2), dot(w_pre, v) ----------------
    {
      if (r.tau != 0.0 && tid < 2 * j) {
        const int k = tid % j;
        const int off = (tid < j) ? k : P + k;
        double s = 0.0;
        for (int q = 0; q < G; ++q) s += ldg_cg(w.dotp + (size_t)q * 2 * P + off);
        if (tid < j) sm.t1[k] = s; else sm.t2[k] = s;
      }
      __syncthreads();
      double dp = 0.0;
      const int rr = tid / 8, part = tid % 8;
      for (int X = I0; X < nt; ++X) {
        if (X % G != g) continue;
        const int row = X * T + rr;
        double y = 0.0;
        if (r.tau != 0.0 && row >= c1 && row < n) {
          for (int J = I0 + part; J < nt; J += 8) y += ldg_cg(w.Pb + ((size_t)X * nt + J) * T + rr);
          for (int k = part; k < j; k += 8)
            y -= ldg_cg(w.V + (size_t)row * P + k) * sm.t1[k] + ldg_cg(w.W + (size_t)row * P + k) * sm.t2[k];
        }
        y += __shfl_xor_sync(0xffffffffu, y, 1);
        y += __shfl_xor_sync(0xffffffffu, y, 2);
        y += __shfl_xor_sync(0xffffffffu, y, 4);
        if (part == 0 && row >= c1 && row < n) {
          const double wp = r.tau * y;
          w.Wpre[row] = wp;
          dp += wp * vval(A, ld, n, c, r.scale, row);
        }
      }
      dp = block_sum(dp, sm.small);
      if (tid == 0) w.scal[g * 4 + 1] = dp;
    }
    if (!group_sync(w.bar, G, gen, err)) return false;

    // ---------------- phase 3: finalize W column, update next column ----------------
    double alpha2 = 0.0;
    if (r.tau != 0.0) {
      double s = 0.0;
      for (int q = 0; q < G; ++q) s += ldg_cg(w.scal + q * 4 + 1);
      alpha2 = -0.5 * r.tau * s;
    }
    for (int X = 0; X < nt; ++X) {
      if (X % G != g) continue;
      const int row = X * T + (tid % T);
      if (tid < T && row < n) {
        const double wv = (row >= c1) ? ldg_cg(w.Wpre + row) + alpha2 * vval(A, ld, n, c, r.scale, row) : 0.0;
        w.W[(size_t)row * P + j] = (r.tau != 0.0) ? wv : 0.0;
      }
    }
    if (j + 1 == P && c1 < n) {
      if (!group_sync(w.bar, G, gen, err)) return false;
      syr2k_tiles(A, ld, n, c1, w, nt, g, G, dyn);
      if (!group_sync(w.bar, G, gen, err)) return false;
    } else if (c1 < n) {
      // A[r][c1] -= sum_{k<=j} V[r][k] W[c1][k] + W[r][k] V[c1][k]
      if (tid <= j) {
        double wc = ldg_cg(w.W + (size_t)c1 * P + tid);
        if (tid == j) wc = (r.tau != 0.0) ? ldg_cg(w.Wpre + c1) + alpha2 : 0.0;   // v(c1) = 1
        sm.wc[tid] = wc;
        sm.vc[tid] = ldg_cg(w.V + (size_t)c1 * P + tid);
      }
      __syncthreads();
      const int rr = tid / 8, part = tid % 8;
      for (int X = I0; X < nt; ++X) {
        if (X % G != g) continue;
        const int row = X * T + rr;
        double s = 0.0;
        if (row >= c1 && row < n) {
          for (int k = part; k <= j; k += 8) {
            double wrk;
            if (k == j) wrk = (r.tau != 0.0) ? ldg_cg(w.Wpre + row) + alpha2 * vval(A, ld, n, c, r.scale, row) : 0.0;
            else wrk = ldg_cg(w.W + (size_t)row * P + k);
            s += ldg_cg(w.V + (size_t)row * P + k) * sm.wc[k] + wrk * sm.vc[k];
          }
        }
        s += __shfl_xor_sync(0xffffffffu, s, 1);
        s += __shfl_xor_sync(0xffffffffu, s, 2);
        s += __shfl_xor_sync(0xffffffffu, s, 4);
        if (part == 0 && row >= c1 && row < n) {
          double* pa = A + (size_t)row * ld + c1;
          *pa = ldg_cg(pa) - s;
        }
      }
      __syncthreads();
    }
    // norm partials of the updated column c1 (rows >= c1+2) and d[c1]
    if (c1 < n) {
      double s = 0.0;
      for (int X = I0; X < nt; ++X) {
        if (X % G != g) continue;
        const int row = X * T + (tid % T);
        if (tid < T && row >= c1 + 2 && row < n) {
          const double x = ldg_cg(A + (size_t)row * ld + c1);
          s += x * x;
        }
        if (tid < T && row == c1) job.d[c1] = ldg_cg(A + (size_t)row * ld + c1);
      }
      s = block_sum(s, sm.small);
      if (tid == 0) w.scal[g * 4 + 0] = s;
    }
    if (!group_sync(w.bar, G, gen, err)) return false;
  }
  return true;
}

__global__ void __launch_bounds__(THREADS, 1) tridiag_kernel(const TridiagJob* jobs, int n_jobs, int G,
                                                             char* ws, size_t ws_bytes, int nmax,
                                                             int* err) {
  extern __shared__ double dyn[];
  __shared__ Smem sm;
  const int group = blockIdx.x / G, g = blockIdx.x % G;
  const int ngroups = gridDim.x / G;
  GroupWS w;
  ws_layout(nmax, G, &w, ws + (size_t)group * ws_bytes);
  unsigned gen = 0;
  for (int jb = group; jb < n_jobs; jb += ngroups) {
    const TridiagJob job = jobs[jb];
    if (!tridiag_one(job, w, g, G, gen, err, sm, dyn)) return;
  }
}

// ---------------------------------------------------------------------------
// Number of eigenvalues of the symmetric tridiagonal (d, e) below x.
__device__ int sturm_count(const double* d, const double* e, int n, double x) {
  const double big = 0x1p500, small = 0x1p-500;
  double pm = 1.0;
  double p = d[0] - x;
  bool neg = (p < 0.0) || (p == 0.0);  // zero takes the sign opposite to its predecessor
  int cnt = neg ? 1 : 0;
  for (int i = 1; i < n; ++i) {
    const double ei = e[i - 1];
    double pn = fma(d[i] - x, p, -(ei * ei) * pm);
    const bool nn = (pn == 0.0) ? !neg : (pn < 0.0);
    cnt += (nn != neg);
    neg = nn;
    pm = p;
    p = pn;
    const double ap = fabs(p);
    if (ap > big) {
      p *= small;
      pm *= small;
    } else if (ap < small && ap != 0.0) {
      p *= big;
      pm *= big;
    }
  }
  return cnt;
}

__global__ void bisect_kernel(const double* d, const double* e, int n, double* ev) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  double lo = 1e308, hi = -1e308;
  for (int i = 0; i < n; ++i) {
    const double rad = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i < n - 1 ? fabs(e[i]) : 0.0);
    lo = fmin(lo, d[i] - rad);
    hi = fmax(hi, d[i] + rad);
  }
  const double tn = fmax(fabs(lo), fabs(hi));
  lo -= 4.0 * 2.2e-16 * tn + 1e-300;
  hi += 4.0 * 2.2e-16 * tn + 1e-300;
  // invariant: count(lo) <= k < count(hi)
  for (int it = 0; it < 128; ++it) {
    const double mid = 0.5 * (lo + hi);
    if (mid <= lo || mid >= hi) break;
    if (sturm_count(d, e, n, mid) > k) hi = mid; else lo = mid;
    if (hi - lo <= 2.0 * 1.1102230246251565e-16 * fmax(fabs(lo), fabs(hi))) break;
  }
  ev[k] = 0.5 * (lo + hi);
}

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& err) {
  s = a + b;
  const double bb = s - a;
  err = (a - (s - bb)) + (b - bb);
}

__global__ void __launch_bounds__(1024) energy_kernel(const double* ev, int n, int nsl, const double* scalars,
                                                      double* out) {
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

}  // namespace

size_t tridiag_workspace_bytes(int n, int group_ctas) { return ws_layout(n, group_ctas, nullptr, nullptr); }

constexpr size_t kTridiagDynSmem = 4 * T * (P + 1) * sizeof(double);

int tridiag_max_ctas_per_sm() {
  int nb = 0;
  cudaFuncSetAttribute(tridiag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTridiagDynSmem);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, tridiag_kernel, THREADS, kTridiagDynSmem);
  return nb;
}

cudaError_t launch_tridiag(const TridiagJob* jobs_dev, int n_jobs, int groups, int group_ctas,
                           void* workspace, size_t ws_bytes_per_group, int nmax, int* err_flag,
                           cudaStream_t s) {
  for (int gi = 0; gi < groups; ++gi) {
    cudaError_t e = cudaMemsetAsync(static_cast<char*>(workspace) + (size_t)gi * ws_bytes_per_group, 0, 256, s);
    if (e != cudaSuccess) return e;
  }
  int G = group_ctas;
  char* ws = static_cast<char*>(workspace);
  void* args[] = {(void*)&jobs_dev, (void*)&n_jobs, (void*)&G, (void*)&ws, (void*)&ws_bytes_per_group,
                  (void*)&nmax, (void*)&err_flag};
  return cudaLaunchCooperativeKernel((const void*)tridiag_kernel, dim3(groups * group_ctas), dim3(THREADS),
                                     args, kTridiagDynSmem, s);
}

void launch_tridiag_eigenvalues(const double* d, const double* e, int n, double* ev, cudaStream_t s) {
  bisect_kernel<<<(n + 63) / 64, 64, 0, s>>>(d, e, n, ev);
}

void launch_energy(const double* ev, int n, int nsl, const double* scalars, double* out, cudaStream_t s) {
  energy_kernel<<<1, 1024, 0, s>>>(ev, n, nsl, scalars, out);
}

}  // namespace mbd
