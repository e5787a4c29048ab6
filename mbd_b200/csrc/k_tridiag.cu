// Householder tridiagonalisation of the CFDM Hamiltonian in FP64 (the
// reduction half of PDSYEV('N','L') at UTILS.f90:835), blocked in panels of
// 32 columns as LAPACK's DSYTRD/DLATRD.
//
// The whole reduction is ONE cooperative launch.  The CTAs of a group meet at
// bounded global-memory barriers, two per column, and every phase issues all
// of its global loads before it first needs one, so a column costs about two
// dependent memory round trips plus two barriers:
//   A  reflector of column c from the previous phase's norm partials;
//      y = A22 v over the trailing lower triangle: 64x64 tiles, four warps per
//      tile (16 rows each, all 16 rows of 16-byte loads in flight), four tiles
//      per CTA per round; partial sums land in Pb[I][J][0..63] so a row's total
//      is a coalesced read; v^T A22 v and the panel dots W^T v, V^T v aside.
//   B  8 threads per row: w = tau (y - V (W^T v) - W (V^T v)) + alpha2 v with
//      alpha2 = -tau^2/2 (v^T A22 v - 2 (W^T v).(V^T v)), all from phase-A
//      sums; store w and v; update column c+1 with the panel (at a panel end:
//      A22 -= V W^T + W V^T); norm of the new column for the next reflector.
// Cross-CTA sums are laid out [item][cta] and reduced by whole warps.
#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "wait_limit.cuh"
#include "../../include/mbd_b200.h"

namespace mbd {
namespace {

constexpr int T = kTrdTile;   // 64
constexpr int P = kTrdNB;     // 32 panel width
constexpr int THREADS = 512;
constexpr int NWARP = THREADS / 32;
constexpr int SLOTS = 2;      // tiles per CTA per round (8 warps x 8 rows each)
constexpr int TILE_DBL = SLOTS * T * T;   // doubles of one staging buffer (64 KB)
constexpr int kMaxG = kTridiagMaxGroup;   // largest group (CTAs) the cross-CTA reductions unroll for

struct GroupWS {
  unsigned* bar;   // [0] arrivals, [1] generation
  double* W;       // [P][nmax]
  double* V;       // [P][nmax]
  double* col0;    // [nmax] contiguous copy of the current column (double-buffered)
  double* col1;
  double* Pb;      // [nt][nt][T] y partials of tile (I,J) for row block I
  double* dotp;    // [2P+1][G] panel dots and v^T A v
  double* scal;    // [G] norm partials
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
  size_t o_c0 = take(sizeof(double) * (size_t)(nmax + T));
  size_t o_c1 = take(sizeof(double) * (size_t)(nmax + T));
  size_t o_Pb = take(sizeof(double) * (size_t)nt * nt * T);
  size_t o_dp = take(sizeof(double) * (size_t)G * (2 * P + 1));
  size_t o_sc = take(sizeof(double) * (size_t)G);
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

// Bounded barrier among the G CTAs of one group (acquire-release atomics,
// no separate fences).  Returns false (and sets *err) when the wait runs out
// or another CTA already failed.
__device__ bool group_sync(unsigned* bar, int G, unsigned& gen, int* err) {
  __shared__ int s_ok;
  __syncthreads();
  if (G == 1) return true;
  if (threadIdx.x == 0) {
    int ok = 1;
    const unsigned target = gen + 1;
    unsigned arrived;
    asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], 1;" : "=r"(arrived) : "l"(bar) : "memory");
    if (arrived == (unsigned)G - 1) {
      asm volatile("st.relaxed.gpu.u32 [%0], 0;" ::"l"(bar) : "memory");
      asm volatile("st.release.gpu.u32 [%0], %1;" ::"l"(bar + 1), "r"(target) : "memory");
    } else {
      const long long lim = wait_limit_cycles();
      const long long t0 = clock64();
      while (true) {
        unsigned cur;
        asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(bar + 1) : "memory");
        if (cur == target) break;
        if (*(volatile int*)err != 0 || clock64() - t0 > lim) {
          ok = 0;
          atomicCAS(err, 0, MBD_ERR_TIMEOUT);
          break;
        }
      }
    }
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

// v(r) of column c's reflector from the stored column value x = col[r].
__device__ __forceinline__ double vfun(int r, double x, int c1, int n, double scale) {
  if (r == c1) return 1.0;
  if (r > c1 && r < n) return x * scale;
  return 0.0;
}

struct Smem {
  double red[SLOTS][8][T];   // column partials per warp octet
  double rows[SLOTS][T];     // row sums
  double item[64];           // cross-CTA sums: W^T v, V^T v, v^T A v
  double t1[P], t2[P], wc[P + 1], vc[P + 1];
  double small[NWARP];
  double vav_all, alpha2, wc1, yc1;
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
  __syncthreads();
}

// Rows of [lo, n) owned by CTA g of G (contiguous chunks).
__device__ __forceinline__ void chunk_rows(int lo, int n, int g, int G, int* rs, int* re) {
  const int m = n - lo;
  const int ch = (m + G - 1) / G;
  *rs = min(n, lo + g * ch);
  *re = min(n, lo + (g + 1) * ch);
}

// One warp's 8-row strip of a 64x64 tile, staged in shared memory by
// cp.async (16 bytes per lane per row, zero-filled outside the matrix), plus
// the column values behind v that the compute step needs.
struct Strip {
  double xj0, xj1, xr, xk;   // v's column values at cols s0, s0+1, row (lane<8), combine column (tid<128)
  int I, J;
  bool live;
};

__device__ __forceinline__ void cp_async16(double* dst, const double* src, int bytes) {
  const uint32_t d = static_cast<uint32_t>(__cvta_generic_to_shared(dst));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void tile_of(int t, int ntile, int I0, int* I, int* J, bool* live) {
  *live = t < ntile;
  *I = *J = I0;
  if (*live) {
    int ti, tj;
    tri_index(t, &ti, &tj);
    *I = I0 + ti;
    *J = I0 + tj;
  }
}

// Issue the copies of round `round` into `buf` and load the column values.
__device__ __forceinline__ void issue_round(Strip& st, const double* A, int ld, int n, const double* col, int round,
                                            int g, int G, int ntile, int I0, double* buf, int warp, int lane,
                                            int tid) {
  const int sl = warp / 8, oct = warp % 8;
  const int t = round * SLOTS * G + SLOTS * g + sl;
  tile_of(t, ntile, I0, &st.I, &st.J, &st.live);
  const int s0 = st.J * T + 2 * lane;
  const int bytes = (!st.live || s0 >= n) ? 0 : (s0 + 1 < n ? 16 : 8);
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int rt = 8 * oct + u;               // row within the tile
    const int row = st.I * T + rt;
    const bool ok = bytes > 0 && row < n;
    cp_async16(buf + ((size_t)sl * T + rt) * T + 2 * lane, ok ? A + (size_t)row * ld + s0 : A, ok ? bytes : 0);
  }
  asm volatile("cp.async.commit_group;" ::: "memory");
  st.xj0 = (bytes > 0) ? ldg_cg(col + s0) : 0.0;
  st.xj1 = (bytes == 16) ? ldg_cg(col + s0 + 1) : 0.0;
  const int rr = st.I * T + 8 * oct + (lane & 7);
  st.xr = (st.live && rr < n) ? ldg_cg(col + rr) : 0.0;
  st.xk = 0.0;
  if (tid < SLOTS * T) {
    int I, J;
    bool lv;
    tile_of(round * SLOTS * G + SLOTS * g + tid / T, ntile, I0, &I, &J, &lv);
    const int sk = J * T + tid % T;
    st.xk = (lv && sk < n) ? ldg_cg(col + sk) : 0.0;
  }
}

// Row sums (into sm.rows) and column partials (into sm.red) of this warp's
// staged strip; returns this lane's share of v^T A v from the rows.
__device__ __forceinline__ double strip_compute(const Strip& st, const double* buf, int warp, int lane, int c1,
                                                int n, double scale, Smem& sm) {
  const int sl = warp / 8, oct = warp % 8;
  const bool diag = st.I == st.J;
  const int s0 = st.J * T + 2 * lane;
  const double vj0 = vfun(s0, st.xj0, c1, n, scale), vj1 = vfun(s0 + 1, st.xj1, c1, n, scale);
  const double vr = vfun(st.I * T + 8 * oct + (lane & 7), st.xr, c1, n, scale);
  double rs = 0.0, cx = 0.0, cy = 0.0;
#pragma unroll
  for (int u = 0; u < 8; ++u) {
    const int r = 8 * oct + u;   // row within the tile
    const double2 a = *reinterpret_cast<const double2*>(buf + ((size_t)sl * T + r) * T + 2 * lane);
    double ax = a.x, ay = a.y;
    double bx = ax, by = ay;
    if (diag) {
      const int sx = 2 * lane, sy = 2 * lane + 1;
      if (sx > r) ax = 0.0;
      if (sy > r) ay = 0.0;
      if (sx >= r) bx = 0.0;
      if (sy >= r) by = 0.0;
    }
    const double rp = warp_sum(ax * vj0 + ay * vj1);
    if (lane == u) rs = rp;
    const double vu = __shfl_sync(0xffffffffu, vr, u);
    cx += bx * vu;
    cy += by * vu;
  }
  sm.red[sl][oct][2 * lane] = st.live ? cx : 0.0;
  sm.red[sl][oct][2 * lane + 1] = st.live ? cy : 0.0;
  if (lane < 8) sm.rows[sl][8 * oct + lane] = st.live ? rs : 0.0;
  return (st.live && lane < 8) ? vr * rs : 0.0;
}

__device__ bool tridiag_one(const TridiagJob& job, const GroupWS& w, int g, int G, unsigned& gen,
                            int* err, Smem& sm, double* dyn) {
  double* A = job.A;
  const int n = job.n, ld = job.ld;
  const int nt = (n + T - 1) / T;
  const int tid = threadIdx.x, lane = tid % 32, warp = tid / 32;
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
    if (tid == 0) w.scal[g] = s;
    if (g == 0 && tid == 0) job.d[0] = ldg_cg(A);
  }
  if (!group_sync(w.bar, G, gen, err)) return false;

  for (int c = 0; c <= n - 2; ++c) {
    const int p = c - c % P, j = c - p;
    const int c1 = c + 1;
    const int I0 = c1 / T;
    const int mt = nt - I0;
    const int ntile = mt * (mt + 1) / 2;
    int rs, re;
    chunk_rows(c1, n, g, G, &rs, &re);
    // ================= phase A =================
    // loads first: norm partials + alpha (warp 0), the first round of tiles,
    // and the panel-dot operands of this CTA's rows
    double nrm_part = 0.0, alpha = 0.0;
    if (warp == 0) {
      double v[kMaxG / 32];
#pragma unroll
      for (int u = 0; u < kMaxG / 32; ++u) v[u] = (lane + 32 * u < G) ? ldg_cg(w.scal + lane + 32 * u) : 0.0;
      alpha = ldg_cg(col_cur + c1);
#pragma unroll
      for (int u = 0; u < kMaxG / 32; ++u) nrm_part += v[u];
    }
    Strip st;
    issue_round(st, A, ld, n, col_cur, 0, g, G, ntile, I0, dyn, warp, lane, tid);
    // panel dots: item it = warp (and warp+16, ...) over rows r = rs + lane (+32 ...)
    double dx[2] = {0.0, 0.0}, dm[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
    {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = rs + lane + 32 * h;
        if (r < re) {
          dx[h] = ldg_cg(col_cur + r);
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int it = warp + NWARP * q;
            if (it < 2 * j) {
              const int k = it % j;
              dm[h][q] = ldg_cg((it < j ? w.W : w.V) + k * nm + r);
            }
          }
        }
      }
    }
    if (warp == 0) {
      const double xn2 = warp_sum(nrm_part);
      if (lane == 0) {
        Refl rfl;
        if (xn2 == 0.0) {
          rfl.tau = 0.0;
          rfl.scale = 0.0;
          rfl.beta = alpha;
        } else {
          const double beta = -copysign(sqrt(alpha * alpha + xn2), alpha);
          rfl.tau = (beta - alpha) / beta;
          rfl.scale = 1.0 / (alpha - beta);
          rfl.beta = beta;
        }
        sm.rf = rfl;
        if (g == 0) job.e[c] = rfl.beta;
        if (g == 0 && job.tau) job.tau[c] = rfl.tau;
      }
    }
    __syncthreads();
    const Refl rf = sm.rf;
    double vav = 0.0;
    if (rf.tau != 0.0) {
      // dots over this CTA's rows (more than 64 rows: remaining rows loaded here)
      double acc[4] = {0, 0, 0, 0};
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = rs + lane + 32 * h;
        const double vr = (r < re) ? vfun(r, dx[h], c1, n, rf.scale) : 0.0;
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[q] += dm[h][q] * vr;
      }
      for (int r = rs + lane + 64; r < re; r += 32) {
        const double vr = vfun(r, ldg_cg(col_cur + r), c1, n, rf.scale);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int it = warp + NWARP * q;
          if (it < 2 * j) acc[q] += ldg_cg((it < j ? w.W : w.V) + (it % j) * nm + r) * vr;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int it = warp + NWARP * q;
        const double s = warp_sum(acc[q]);
        if (it < 2 * j && lane == 0) w.dotp[(size_t)(it < j ? it : P + it - j) * G + g] = s;
      }
      // SYMV rounds: SLOTS tiles per CTA per round, the next round's copies
      // in flight while the current one is reduced
      for (int round = 0;; ++round) {
        const bool has_next = (round + 1) * SLOTS * G + SLOTS * g < ntile;   // uniform across the CTA
        Strip nx;
        if (has_next) {
          issue_round(nx, A, ld, n, col_cur, round + 1, g, G, ntile, I0, dyn + ((round + 1) & 1) * TILE_DBL, warp,
                      lane, tid);
          asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
          asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncwarp();
        vav += strip_compute(st, dyn + (round & 1) * TILE_DBL, warp, lane, c1, n, rf.scale, sm);
        __syncthreads();
        if (tid < SLOTS * T) {
          const int sl = tid / T, k = tid % T;
          int I, J;
          bool lv;
          tile_of(round * SLOTS * G + SLOTS * g + sl, ntile, I0, &I, &J, &lv);
          if (lv) {
            double cs = 0.0;
#pragma unroll
            for (int o = 0; o < 8; ++o) cs += sm.red[sl][o][k];
            const int sk = J * T + k;
            const double vk = (sk < n) ? vfun(sk, st.xk, c1, n, rf.scale) : 0.0;
            if (I != J) {
              w.Pb[((size_t)I * nt + J) * T + k] = sm.rows[sl][k];
              w.Pb[((size_t)J * nt + I) * T + k] = cs;
            } else {
              w.Pb[((size_t)I * nt + I) * T + k] = sm.rows[sl][k] + cs;
            }
            vav += vk * cs;
          }
        }
        __syncthreads();
        if (!has_next) break;
        st = nx;
      }
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    vav = block_sum(vav, sm);
    if (tid == 0) w.dotp[(size_t)(2 * P) * G + g] = vav;
    if (!group_sync(w.bar, G, gen, err)) return false;

    // ================= phase B =================
    const bool panel_end = (j + 1 == P);
    constexpr int RPT = 8;
    const int part = tid % RPT;
    const int r = rs + tid / RPT;          // chunk <= 64 rows handled in one pass below
    // loads: per-row y partials, panel rows, A[r][c1], x(r)
    double y = 0.0, vk[4] = {0, 0, 0, 0}, wk[4] = {0, 0, 0, 0}, arc = 0.0, xr = 0.0;
    const bool live = r < re;
    if (live) {
      if (rf.tau != 0.0) {
        const double* pb = w.Pb + (size_t)(r / T) * nt * T + (r % T);
        double v[12];   // independent loads for up to 96 tile columns; the rest in a loop
#pragma unroll
        for (int u = 0; u < 12; ++u) {
          const int J = I0 + part + RPT * u;
          v[u] = (J < nt) ? ldg_cg(pb + (size_t)J * T) : 0.0;
        }
        for (int J = I0 + part + RPT * 12; J < nt; J += RPT) y += ldg_cg(pb + (size_t)J * T);
#pragma unroll
        for (int u = 0; u < 12; ++u) y += v[u];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = part + RPT * q;
        if (k < j) {
          vk[q] = ldg_cg(w.V + k * nm + r);
          wk[q] = ldg_cg(w.W + k * nm + r);
        }
      }
      if (!panel_end && part == 0) arc = ldg_cg(A + (size_t)r * ld + c1);
      xr = ldg_cg(col_cur + r);
    }
    // cross-CTA sums: items 0..2j-1 (t1, t2) and 2P (v^T A v); row c1 for w(c1)
    // (8 threads per item, every load independent: one round trip)
    if (rf.tau != 0.0) {
      const int it = tid / 8, ip = tid % 8;
      double s = 0.0;
      if (it <= 2 * j) {
        const int src = (it == 2 * j) ? 2 * P : (it < j ? it : P + it - j);
        const double* dp = w.dotp + (size_t)src * G;
        double v[kMaxG / 8];
#pragma unroll
        for (int u = 0; u < kMaxG / 8; ++u) {
          const int q = ip + 8 * u;
          v[u] = (q < G) ? ldg_cg(dp + q) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kMaxG / 8; ++u) s += v[u];
      }
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      s += __shfl_xor_sync(0xffffffffu, s, 4);
      if (ip == 0 && it <= 2 * j) {
        if (it == 2 * j) sm.vav_all = s;
        else if (it < j) sm.t1[it] = s;
        else sm.t2[it - j] = s;
      }
    }
    if (warp == NWARP - 1 && !panel_end) {
      double yc = 0.0;
      if (rf.tau != 0.0)
        for (int J = I0 + lane; J < nt; J += 32) yc += ldg_cg(w.Pb + ((size_t)(c1 / T) * nt + J) * T + (c1 % T));
      yc = warp_sum(yc);
      if (lane < j) {
        sm.wc[lane] = ldg_cg(w.W + lane * nm + c1);
        sm.vc[lane] = ldg_cg(w.V + lane * nm + c1);
      }
      if (lane == 0) sm.yc1 = yc;
    }
    __syncthreads();
    if (warp == 0) {
      double alpha2 = 0.0, wc1 = 0.0;
      if (rf.tau != 0.0) {
        const double s12 = warp_sum(lane < j ? sm.t1[lane] * sm.t2[lane] : 0.0);
        alpha2 = -0.5 * rf.tau * (rf.tau * (sm.vav_all - 2.0 * s12));
        if (!panel_end) {
          const double corr =
              warp_sum(lane < j ? sm.vc[lane] * sm.t1[lane] + sm.wc[lane] * sm.t2[lane] : 0.0);
          wc1 = rf.tau * (sm.yc1 - corr) + alpha2;      // v(c1) = 1
        }
      }
      if (lane == 0) {
        sm.alpha2 = alpha2;
        if (!panel_end) {
          sm.wc[j] = wc1;
          sm.vc[j] = 1.0;
        }
      }
    }
    __syncthreads();
    const double alpha2 = sm.alpha2;
    double nrm = 0.0;
    {
      double corr = 0.0, upd = 0.0;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int k = part + RPT * q;
        if (k < j) {
          corr += vk[q] * sm.t1[k] + wk[q] * sm.t2[k];
          if (!panel_end) upd += vk[q] * sm.wc[k] + wk[q] * sm.vc[k];
        }
      }
#pragma unroll
      for (int o = 1; o < RPT; o <<= 1) {
        y += __shfl_xor_sync(0xffffffffu, y, o);
        corr += __shfl_xor_sync(0xffffffffu, corr, o);
        upd += __shfl_xor_sync(0xffffffffu, upd, o);
      }
      if (live && part == 0) {
        const double vr = vfun(r, xr, c1, n, rf.scale);
        const double wr = (rf.tau != 0.0) ? rf.tau * (y - corr) + alpha2 * vr : 0.0;
        w.W[j * nm + r] = wr;
        w.V[j * nm + r] = vr;
        if (job.vsave) job.vsave[(size_t)c * job.ldv + r] = vr;
        if (!panel_end) {
          const double x = arc - (upd + vr * sm.wc[j] + wr * sm.vc[j]);
          A[(size_t)r * ld + c1] = x;
          col_nxt[r] = x;
          if (r == c1) job.d[c1] = x;
          if (r >= c1 + 2) nrm += x * x;
        }
      }
    }
    // chunks of more than 64 rows (very large n): the same steps, loads in place
    for (int r2 = rs + THREADS / RPT + tid / RPT; r2 - tid / RPT < re; r2 += THREADS / RPT) {
      const bool lv = r2 < re;
      double y2 = 0.0, corr = 0.0, upd = 0.0;
      if (lv) {
        if (rf.tau != 0.0) {
          const double* pb = w.Pb + (size_t)(r2 / T) * nt * T + (r2 % T);
          for (int J = I0 + part; J < nt; J += RPT) y2 += ldg_cg(pb + (size_t)J * T);
        }
        for (int k = part; k < j; k += RPT) {
          const double a1 = ldg_cg(w.V + k * nm + r2), a2 = ldg_cg(w.W + k * nm + r2);
          corr += a1 * sm.t1[k] + a2 * sm.t2[k];
          if (!panel_end) upd += a1 * sm.wc[k] + a2 * sm.vc[k];
        }
      }
#pragma unroll
      for (int o = 1; o < RPT; o <<= 1) {
        y2 += __shfl_xor_sync(0xffffffffu, y2, o);
        corr += __shfl_xor_sync(0xffffffffu, corr, o);
        upd += __shfl_xor_sync(0xffffffffu, upd, o);
      }
      if (lv && part == 0) {
        const double vr = vfun(r2, ldg_cg(col_cur + r2), c1, n, rf.scale);
        const double wr = (rf.tau != 0.0) ? rf.tau * (y2 - corr) + alpha2 * vr : 0.0;
        w.W[j * nm + r2] = wr;
        w.V[j * nm + r2] = vr;
        if (job.vsave) job.vsave[(size_t)c * job.ldv + r2] = vr;
        if (!panel_end) {
          const double x = ldg_cg(A + (size_t)r2 * ld + c1) - (upd + vr * sm.wc[j] + wr * sm.vc[j]);
          A[(size_t)r2 * ld + c1] = x;
          col_nxt[r2] = x;
          if (r2 == c1) job.d[c1] = x;
          if (r2 >= c1 + 2) nrm += x * x;
        }
      }
    }
    if (panel_end) {
      if (!group_sync(w.bar, G, gen, err)) return false;
      syr2k_tiles(A, ld, n, c1, w, g, G, dyn);
      if (!group_sync(w.bar, G, gen, err)) return false;
      for (int r2 = rs + tid; r2 < re; r2 += THREADS) {
        const double x = ldg_cg(A + (size_t)r2 * ld + c1);
        col_nxt[r2] = x;
        if (r2 == c1) job.d[c1] = x;
        if (r2 >= c1 + 2) nrm += x * x;
      }
    }
    nrm = block_sum(nrm, sm);
    if (tid == 0) w.scal[g] = nrm;
    if (!group_sync(w.bar, G, gen, err)) return false;
    double* tmp = col_cur;
    col_cur = col_nxt;
    col_nxt = tmp;
  }
  return true;
}

// groups == nullptr: gridDim.x / G_uniform equal groups of G_uniform CTAs,
// group k reducing jobs k, k + groups, ... with workspace ws + k * ws_bytes.
// Otherwise groups[0..n_groups) (ascending first_cta) partition the grid:
// the CTAs [first_cta, first_cta + G) reduce jobs [job_begin, job_end) one
// after another with workspace ws + ws_offset.
__global__ void __launch_bounds__(THREADS, 1) tridiag_kernel(const TridiagJob* jobs, int n_jobs,
                                                             const TridiagGroup* groups, int n_groups,
                                                             int G_uniform, char* ws, size_t ws_bytes, int nmax,
                                                             int* err) {
  extern __shared__ double dyn[];
  __shared__ Smem sm;
  __shared__ int s_grp;
  unsigned gen = 0;
  GroupWS w;
  if (groups == nullptr) {
    const int G = G_uniform;
    const int group = blockIdx.x / G, g = blockIdx.x % G;
    const int ngroups = gridDim.x / G;
    ws_layout(nmax, G, &w, ws + (size_t)group * ws_bytes);
    for (int jb = group; jb < n_jobs; jb += ngroups) {
      const TridiagJob job = jobs[jb];
      if (!tridiag_one(job, w, g, G, gen, err, sm, dyn)) return;
    }
    return;
  }
  if (threadIdx.x == 0) {
    int lo = 0, hi = n_groups - 1;   // last group with first_cta <= blockIdx.x
    while (lo < hi) {
      const int mid = (lo + hi + 1) / 2;
      if (groups[mid].first_cta <= (int)blockIdx.x) lo = mid;
      else hi = mid - 1;
    }
    s_grp = lo;
  }
  __syncthreads();
  const TridiagGroup gr = groups[s_grp];
  const int g = (int)blockIdx.x - gr.first_cta;
  if (g < 0 || g >= gr.G) return;   // CTAs beyond the table (none when the launch matches it)
  ws_layout(gr.nmax, gr.G, &w, ws + gr.ws_offset);
  for (int jb = gr.job_begin; jb < gr.job_end; ++jb) {
    const TridiagJob job = jobs[jb];
    if (!tridiag_one(job, w, g, gr.G, gen, err, sm, dyn)) return;
  }
}

// Zeroes the barrier words of every group before a table launch.
__global__ void reset_group_bars(const TridiagGroup* groups, int n_groups, char* ws) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n_groups) {
    unsigned* bar = reinterpret_cast<unsigned*>(ws + groups[i].ws_offset);
    bar[0] = 0u;
    bar[1] = 0u;
  }
}

}  // namespace

size_t tridiag_workspace_bytes(int n, int group_ctas) { return ws_layout(n, group_ctas, nullptr, nullptr); }

// two SYMV staging buffers (128 KB); the panel-end SYR2K reuses the same space
constexpr size_t kTridiagDynSmem = 2 * TILE_DBL * sizeof(double);
static_assert(kTridiagDynSmem >= 4 * T * (P + 1) * sizeof(double), "SYR2K tiles must fit the staging space");

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
  const TridiagGroup* no_table = nullptr;
  int zero = 0;
  void* args[] = {(void*)&jobs_dev, (void*)&n_jobs, (void*)&no_table, (void*)&zero, (void*)&G, (void*)&ws,
                  (void*)&ws_bytes_per_group, (void*)&nmax, (void*)&err_flag};
  return cudaLaunchCooperativeKernel((const void*)tridiag_kernel, dim3(groups * group_ctas), dim3(THREADS),
                                     args, kTridiagDynSmem, s);
}

cudaError_t launch_tridiag_groups(const TridiagJob* jobs_dev, const TridiagGroup* groups_dev, int n_groups,
                                  int total_ctas, void* workspace, int* err_flag, cudaStream_t s) {
  if (n_groups < 1 || total_ctas < 1) return cudaSuccess;
  char* ws = static_cast<char*>(workspace);
  reset_group_bars<<<(n_groups + 255) / 256, 256, 0, s>>>(groups_dev, n_groups, ws);
  int n_jobs = 0, G = 0, nmax = 0;
  size_t wsb = 0;
  void* args[] = {(void*)&jobs_dev, (void*)&n_jobs, (void*)&groups_dev, (void*)&n_groups, (void*)&G, (void*)&ws,
                  (void*)&wsb, (void*)&nmax, (void*)&err_flag};
  return cudaLaunchCooperativeKernel((const void*)tridiag_kernel, dim3(total_ctas), dim3(THREADS), args,
                                     kTridiagDynSmem, s);
}

MBD_WAIT_LIMIT_SETTER(set_wait_limit_tridiag)

}  // namespace mbd
