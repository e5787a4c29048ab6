// Householder tridiagonalisation of the CFDM Hamiltonian in FP64 (the
// reduction half of PDSYEV('N','L') at UTILS.f90:835), blocked in panels of
// 32 columns as LAPACK's DSYTRD/DLATRD.
//
// The whole reduction is ONE cooperative launch.  The CTAs of a group meet at
// bounded global-memory barriers, two per column:
//   A  reflector of column c from the previous phase's norm partials;
//      y = A22 v over the trailing lower triangle, one 64x64 tile per warp
//      (8 rows of 16-byte loads in flight, no CTA-wide syncs); the partial
//      sums land in Pb[I][J][0..63] so a row's total is a coalesced read;
//      v^T A22 v and the panel dots W^T v, V^T v on the side.
//   B  one thread per row: w = tau (y - V (W^T v) - W (V^T v)) + alpha2 v with
//      alpha2 = -tau^2/2 (v^T A22 v - 2 (W^T v).(V^T v)), all from phase-A
//      sums; store w and v; update column c+1 with the panel (at a panel end:
//      A22 -= V W^T + W V^T); norm of the new column for the next reflector.
// Cross-CTA sums are laid out [item][cta] and reduced by whole warps.
#include <cuda_runtime.h>

#include "kernels.h"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int T = kTrdTile;   // 64
constexpr int P = kTrdNB;     // 32 panel width
constexpr int THREADS = 512;
constexpr int NWARP = THREADS / 32;
constexpr long long kSpinCycles = 4000000000LL;   // ~2 s at 2 GHz, then give up

struct GroupWS {
  unsigned* bar;   // [0] arrivals, [1] generation
  double* W;       // [P][nmax]
  double* V;       // [P][nmax]
  double* col0;    // [nmax] contiguous copy of the current column (double-buffered)
  double* col1;
  double* Pb;      // [nt][nt][T] y partials of tile (I,J) for row block I
  double* dotp;    // [2P][G]
  double* scal;    // [4][G]: [0] norm partial, [1] v^T A v partial
  int nmax;
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
  size_t o_c0 = take(sizeof(double) * (size_t)nmax);
  size_t o_c1 = take(sizeof(double) * (size_t)nmax);
  size_t o_Pb = take(sizeof(double) * (size_t)nt * nt * T);
  size_t o_dp = take(sizeof(double) * (size_t)G * 2 * P);
  size_t o_sc = take(sizeof(double) * (size_t)G * 4);
  if (w) {
    w->bar = reinterpret_cast<unsigned*>(base + o_bar);
    w->W = reinterpret_cast<double*>(base + o_W);
    w->V = reinterpret_cast<double*>(base + o_V);
    w->col0 = reinterpret_cast<double*>(base + o_c0);
    w->col1 = reinterpret_cast<double*>(base + o_c1);
    w->Pb = reinterpret_cast<double*>(base + o_Pb);
    w->dotp = reinterpret_cast<double*>(base + o_dp);
    w->scal = reinterpret_cast<double*>(base + o_sc);
    w->nmax = nmax;
  }
  return off;
}

__device__ __forceinline__ double ldg_cg(const double* p) { return __ldcg(p); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Sum of G consecutive doubles by one warp.
__device__ __forceinline__ double warp_sum_g(const double* p, int G) {
  double s = 0.0;
  for (int q = threadIdx.x % 32; q < G; q += 32) s += ldg_cg(p + q);
  return warp_sum(s);
}

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
        __nanosleep(20);
      }
    }
    __threadfence();
    gen = target;
    s_ok = ok && (*(volatile int*)err == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ __forceinline__ void tri_index(int t, int* ti, int* tj) {
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

struct Refl {
  double tau, scale, beta;
};

// Householder vector of column c: v(c1) = 1, v(r > c1) = col[r] * scale, 0 otherwise.
struct VecV {
  const double* col;
  double scale;
  int c1, n;
  __device__ __forceinline__ double operator()(int r) const {
    if (r == c1) return 1.0;
    if (r > c1 && r < n) return ldg_cg(col + r) * scale;
    return 0.0;
  }
};

struct Smem {
  double t1[P], t2[P], wc[P + 1], vc[P + 1];
  double small[NWARP];
  double vav_all;
  double s_alpha2;
  Refl rf;
};

__device__ double block_sum(double v, Smem& sm) {
  v = warp_sum(v);
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  __syncthreads();
  if (lane == 0) sm.small[warp] = v;
  __syncthreads();
  double s = 0.0;
#pragma unroll
  for (int q = 0; q < NWARP; ++q) s += sm.small[q];
  __syncthreads();
  return s;
}

// Phase A, SYMV part: every warp of the group takes 64x64 lower tiles of the
// trailing matrix in turn.  Returns this warp's share of v^T A v.
__device__ double symv_tiles_warp(const double* A, int ld, int n, int c1, const VecV& v, double* Pb,
                                  int nt, int gw, int WG) {
  const int lane = threadIdx.x % 32;
  const int I0 = c1 / T;
  const int mt = nt - I0;
  const int ntile = mt * (mt + 1) / 2;
  double vav = 0.0;
  for (int t = gw; t < ntile; t += WG) {
    int ti, tj;
    tri_index(t, &ti, &tj);
    const int I = I0 + ti, J = I0 + tj;
    const bool diag = (I == J);
    const int s0 = J * T + 2 * lane;
    const double vj0 = v(s0), vj1 = v(s0 + 1);
    const double vi_lo = v(I * T + lane), vi_hi = v(I * T + 32 + lane);
    double row_lo = 0.0, row_hi = 0.0, cx = 0.0, cy = 0.0;
#pragma unroll 1
    for (int rb = 0; rb < T; rb += 16) {
      double2 a[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int row = I * T + rb + u;
        a[u] = make_double2(0.0, 0.0);
        if (row < n && s0 < n) {
          const double2 q = __ldcg(reinterpret_cast<const double2*>(A + (size_t)row * ld + s0));
          a[u].x = q.x;
          a[u].y = (s0 + 1 < n) ? q.y : 0.0;
        }
      }
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        const int r = rb + u;
        double ax = a[u].x, ay = a[u].y;
        double bx = ax, by = ay;               // column-part values
        if (diag) {                            // lower triangle of the diagonal tile only
          const int sx = 2 * lane, sy = 2 * lane + 1;
          if (sx > r) ax = 0.0;
          if (sy > r) ay = 0.0;
          if (sx >= r) bx = 0.0;
          if (sy >= r) by = 0.0;
        }
        const double rp = warp_sum(ax * vj0 + ay * vj1);
        if (lane == (r & 31)) {
          if (r < 32) row_lo = rp; else row_hi = rp;
        }
        const double vir = __shfl_sync(0xffffffffu, r < 32 ? vi_lo : vi_hi, r & 31);
        cx += bx * vir;
        cy += by * vir;
      }
    }
    double* pr = Pb + ((size_t)I * nt + J) * T;
    if (!diag) {
      pr[lane] = row_lo;
      pr[32 + lane] = row_hi;
      double* pc = Pb + ((size_t)J * nt + I) * T;
      *reinterpret_cast<double2*>(pc + 2 * lane) = make_double2(cx, cy);
      vav += vi_lo * row_lo + vi_hi * row_hi + vj0 * cx + vj1 * cy;
    } else {
      // column sum of row k lives in lane k/2, component k%2
      const double ox = __shfl_sync(0xffffffffu, cx, lane / 2), oy = __shfl_sync(0xffffffffu, cy, lane / 2);
      const double ox2 = __shfl_sync(0xffffffffu, cx, 16 + lane / 2);
      const double oy2 = __shfl_sync(0xffffffffu, cy, 16 + lane / 2);
      const double comb_lo = row_lo + ((lane & 1) ? oy : ox);
      const double comb_hi = row_hi + ((lane & 1) ? oy2 : ox2);
      pr[lane] = comb_lo;
      pr[32 + lane] = comb_hi;
      vav += vi_lo * comb_lo + vi_hi * comb_hi;
    }
  }
  return warp_sum(vav);
}

// A22 -= V W^T + W V^T over rows/cols >= q0 (end of a panel); one 64x64 tile per CTA step.
__device__ void syr2k_tiles(double* A, int ld, int n, int q0, const GroupWS& w, int g, int G, double* dyn) {
  double* Vr = dyn;                 // [T][P+1]
  double* Wr = dyn + T * (P + 1);
  double* Vs = dyn + 2 * T * (P + 1);
  double* Ws = dyn + 3 * T * (P + 1);
  const int nt = (n + T - 1) / T;
  const int I0 = q0 / T;
  const int mt = nt - I0;
  const int ntile = mt * (mt + 1) / 2;
  const int tid = threadIdx.x;
  const int row = tid / 8, cg = tid % 8;
  const size_t nm = (size_t)w.nmax;
  for (int t = g; t < ntile; t += G) {
    int ti, tj;
    tri_index(t, &ti, &tj);
    const int I = I0 + ti, J = I0 + tj;
    __syncthreads();
    for (int idx = tid; idx < T * P; idx += THREADS) {
      const int k = idx / T, rr = idx % T;
      const int ri = I * T + rr, sj = J * T + rr;
      Vr[rr * (P + 1) + k] = ri < n ? ldg_cg(w.V + k * nm + ri) : 0.0;
      Wr[rr * (P + 1) + k] = ri < n ? ldg_cg(w.W + k * nm + ri) : 0.0;
      Vs[rr * (P + 1) + k] = sj < n ? ldg_cg(w.V + k * nm + sj) : 0.0;
      Ws[rr * (P + 1) + k] = sj < n ? ldg_cg(w.W + k * nm + sj) : 0.0;
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

// Rows of [lo, n) owned by CTA g of G (contiguous chunks).
__device__ __forceinline__ void chunk_rows(int lo, int n, int g, int G, int* rs, int* re) {
  const int m = n - lo;
  const int ch = (m + G - 1) / G;
  *rs = min(n, lo + g * ch);
  *re = min(n, lo + (g + 1) * ch);
}

__device__ bool tridiag_one(const TridiagJob& job, const GroupWS& w, int g, int G, unsigned& gen,
                            int* err, Smem& sm, double* dyn) {
  double* A = job.A;
  const int n = job.n, ld = job.ld;
  const int nt = (n + T - 1) / T;
  const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
  const int gw = g * NWARP + warp, WG = G * NWARP;
  const size_t nm = (size_t)w.nmax;
  if (n == 1) {
    if (g == 0 && tid == 0) job.d[0] = ldg_cg(A);
    return group_sync(w.bar, G, gen, err);
  }
  double* col_cur = w.col0;
  double* col_nxt = w.col1;
  // column 0: contiguous copy, norm partial of rows >= 2, d[0]
  {
    int rs, re;
    chunk_rows(0, n, g, G, &rs, &re);
    double s = 0.0;
    for (int r = rs + tid; r < re; r += THREADS) {
      const double x = ldg_cg(A + (size_t)r * ld);
      col_cur[r] = x;
      if (r >= 2) s += x * x;
    }
    s = block_sum(s, sm);
    if (tid == 0) w.scal[0 * G + g] = s;
    if (g == 0 && tid == 0) job.d[0] = ldg_cg(A);
  }
  if (!group_sync(w.bar, G, gen, err)) return false;

  for (int c = 0; c <= n - 2; ++c) {
    const int p = c - c % P, j = c - p;
    const int c1 = c + 1;
    const int I0 = c1 / T;
    // ---------------- phase A: reflector, SYMV, v^T A v, panel dots ----------------
    if (warp == 0) {
      const double xn2 = warp_sum_g(w.scal + 0 * G, G);
      if (lane == 0) {
        const double alpha = ldg_cg(col_cur + c1);
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
        sm.rf = r;
        if (g == 0) job.e[c] = r.beta;
      }
    }
    __syncthreads();
    const Refl rf = sm.rf;
    const VecV v{col_cur, rf.scale, c1, n};
    int rs, re;
    chunk_rows(c1, n, g, G, &rs, &re);
    double vav = 0.0;
    if (rf.tau != 0.0) {
      vav = symv_tiles_warp(A, ld, n, c1, v, w.Pb, nt, gw, WG);
      // W^T v (items 0..j-1) and V^T v (items P..P+j-1) over own rows, one warp per item
      for (int it = warp; it < 2 * j; it += NWARP) {
        const int k = it % j;
        const double* M = (it < j ? w.W : w.V) + k * nm;
        double s = 0.0;
        for (int r = rs + lane; r < re; r += 32) s += ldg_cg(M + r) * v(r);
        s = warp_sum(s);
        if (lane == 0) w.dotp[(size_t)(it < j ? k : P + k) * G + g] = s;
      }
    }
    if (lane == 0) sm.small[warp] = vav;
    __syncthreads();
    if (tid == 0) {
      double s = 0.0;
      for (int q = 0; q < NWARP; ++q) s += sm.small[q];
      w.scal[1 * G + g] = s;
    }
    if (!group_sync(w.bar, G, gen, err)) return false;

    // ---------------- phase B: w, column update, next norm ----------------
    if (rf.tau != 0.0) {
      for (int it = warp; it <= 2 * j; it += NWARP) {
        if (it == 2 * j) {
          const double s = warp_sum_g(w.scal + 1 * G, G);
          if (lane == 0) sm.vav_all = s;
        } else {
          const int k = it % j;
          const double s = warp_sum_g(w.dotp + (size_t)(it < j ? k : P + k) * G, G);
          if (lane == 0) {
            if (it < j) sm.t1[k] = s; else sm.t2[k] = s;
          }
        }
      }
    }
    __syncthreads();
    if (tid == 0) {
      double alpha2 = 0.0;
      if (rf.tau != 0.0) {
        double s12 = 0.0;
        for (int k = 0; k < j; ++k) s12 += sm.t1[k] * sm.t2[k];
        alpha2 = -0.5 * rf.tau * (rf.tau * (sm.vav_all - 2.0 * s12));
      }
      sm.s_alpha2 = alpha2;
    }
    __syncthreads();
    const double alpha2 = sm.s_alpha2;
    const bool panel_end = (j + 1 == P);
    if (!panel_end) {
      // w(c1), and W[c1][k], V[c1][k] for the update of column c1
      if (warp == 0) {
        double wc1 = 0.0;
        if (rf.tau != 0.0) {
          const int X = c1 / T;
          double y = 0.0;
          for (int J = I0 + lane; J < nt; J += 32) y += ldg_cg(w.Pb + ((size_t)X * nt + J) * T + (c1 % T));
          if (lane < j) y -= ldg_cg(w.V + lane * nm + c1) * sm.t1[lane] + ldg_cg(w.W + lane * nm + c1) * sm.t2[lane];
          y = warp_sum(y);
          wc1 = rf.tau * y + alpha2;          // v(c1) = 1
        }
        if (lane < j) {
          sm.wc[lane] = ldg_cg(w.W + lane * nm + c1);
          sm.vc[lane] = ldg_cg(w.V + lane * nm + c1);
        }
        if (lane == 0) {
          sm.wc[j] = wc1;
          sm.vc[j] = 1.0;
        }
      }
      __syncthreads();
    }
    double nrm = 0.0;
    // 8 threads per row: part p sums J = I0+p, I0+p+8, ... and k = p, p+8, ...
    // so every load of a row is independent of the others.
    constexpr int RPT = 8;
    const int part = tid % RPT;
    for (int rbase = rs; rbase < re; rbase += THREADS / RPT) {
      const int r = rbase + tid / RPT;
      const bool live = r < re;
      const double vr = live ? v(r) : 0.0;
      double y = 0.0, corr = 0.0, upd = 0.0;
      if (live) {
        if (rf.tau != 0.0) {
          const double* pb = w.Pb + (size_t)(r / T) * nt * T + (r % T);
#pragma unroll 4
          for (int J = I0 + part; J < nt; J += RPT) y += ldg_cg(pb + (size_t)J * T);
        }
        for (int k = part; k < j; k += RPT) {
          const double vk = ldg_cg(w.V + k * nm + r), wk = ldg_cg(w.W + k * nm + r);
          corr += vk * sm.t1[k] + wk * sm.t2[k];
          upd += vk * sm.wc[k] + wk * sm.vc[k];
        }
      }
#pragma unroll
      for (int o = 1; o < RPT; o <<= 1) {
        y += __shfl_xor_sync(0xffffffffu, y, o);
        corr += __shfl_xor_sync(0xffffffffu, corr, o);
        upd += __shfl_xor_sync(0xffffffffu, upd, o);
      }
      if (!live || part != 0) continue;
      const double wr = (rf.tau != 0.0) ? rf.tau * (y - corr) + alpha2 * vr : 0.0;
      w.W[j * nm + r] = wr;
      w.V[j * nm + r] = vr;
      if (!panel_end) {
        // A[r][c1] -= sum_{k<=j} V[r][k] W[c1][k] + W[r][k] V[c1][k]
        const double s = upd + vr * sm.wc[j] + wr * sm.vc[j];
        double* pa = A + (size_t)r * ld + c1;
        const double x = ldg_cg(pa) - s;
        *pa = x;
        col_nxt[r] = x;
        if (r == c1) job.d[c1] = x;
        if (r >= c1 + 2) nrm += x * x;
      }
    }
    if (panel_end) {
      if (!group_sync(w.bar, G, gen, err)) return false;
      syr2k_tiles(A, ld, n, c1, w, g, G, dyn);
      if (!group_sync(w.bar, G, gen, err)) return false;
      for (int r = rs + tid; r < re; r += THREADS) {
        const double x = ldg_cg(A + (size_t)r * ld + c1);
        col_nxt[r] = x;
        if (r == c1) job.d[c1] = x;
        if (r >= c1 + 2) nrm += x * x;
      }
    }
    nrm = block_sum(nrm, sm);
    if (tid == 0) w.scal[0 * G + g] = nrm;
    if (!group_sync(w.bar, G, gen, err)) return false;
    double* tmp = col_cur;
    col_cur = col_nxt;
    col_nxt = tmp;
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

}  // namespace mbd
