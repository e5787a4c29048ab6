// C ABI of the engine (include/mbd_b200.h): context, upload / compute /
// download, and the orchestration of the kernels for one batch of
// geometries.  Replaces MBD_at_rsSCS (UTILS.f90:153-349) and the BLACS /
// MPI plumbing around it (UTILS.f90:97-149, 499-529) with one GPU.
//
// A batch runs in two parts.  The relay and CFDM stages of each geometry
// (UTILS.f90:239-315 and 745-807) run on one of up to kMaxSlots relay slots,
// each a CUDA stream with its own workspace, so the stages of different
// geometries overlap on the GPU.  Every geometry keeps its own CFDM
// Hamiltonian.  Then one cooperative launch reduces all Hamiltonians to
// tridiagonal form with CTA groups planned on the host (plan_tridiag), and
// one launch each computes all eigenvalues and all energies.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <numeric>
#include <vector>

#include "kernels.h"
#include "mbd_internal.h"
#include "tc3.h"

#include "context.h"


namespace mbd {
namespace {

// Symmetric 3x3 eigenvalues from the upper triangle (DSYEV('V','U'), UTILS.f90:273),
// cyclic Jacobi in FP64, ascending.
void sym3_eigenvalues_upper(const double* M, double out[3]) {
  double a[3][3];
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c) a[r][c] = (r <= c) ? M[3 * r + c] : M[3 * c + r];
  for (int sweep = 0; sweep < 50; ++sweep) {
    double off = std::fabs(a[0][1]) + std::fabs(a[0][2]) + std::fabs(a[1][2]);
    if (off == 0.0) break;
    for (int p = 0; p < 2; ++p)
      for (int q = p + 1; q < 3; ++q) {
        if (a[p][q] == 0.0) continue;
        double theta = (a[q][q] - a[p][p]) / (2.0 * a[p][q]);
        double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < 3; ++k) {
          double akp = a[k][p], akq = a[k][q];
          a[k][p] = c * akp - s * akq;
          a[k][q] = s * akp + c * akq;
        }
        for (int k = 0; k < 3; ++k) {
          double apk = a[p][k], aqk = a[q][k];
          a[p][k] = c * apk - s * aqk;
          a[q][k] = s * apk + c * aqk;
        }
      }
  }
  out[0] = a[0][0];
  out[1] = a[1][1];
  out[2] = a[2][2];
  std::sort(out, out + 3);
}

int upload_geometry(mbd_ctx* ctx, const mbd_geom& g, GeomDev* gd) {
  int st = build_plan(g, &gd->plan);
  if (st != MBD_OK) return st;
  const GeomPlan& p = gd->plan;
  const int N = p.N;
  const int nshift_s = (int)p.scs_shifts.size() / 3, nshift_c = (int)p.cfdm_shifts.size() / 3;
  const int ndiff = (int)p.diff_is_zero.size();
  const int nplace = (int)p.place_rc.size();
  // inputs
  size_t off = 0;
  std::vector<size_t> offs;
  auto add = [&](size_t b) { offs.push_back(off); off += b; };
  add(bytes_of<double>(3 * N));             // coords
  add(bytes_of<double>(N));                 // alpha0
  add(bytes_of<double>(N));                 // c6free
  add(bytes_of<double>(N));                 // r0
  add(bytes_of<double>(N));                 // hirsh
  add(bytes_of<double>(3 * nshift_s));
  add(bytes_of<double>(3 * nshift_c));
  add(bytes_of<double>(3 * ndiff));
  add(bytes_of<int>(ndiff));
  add(bytes_of<int>(ndiff + 1));
  add(bytes_of<int>(nplace));
  add(bytes_of<int>(nplace));
  MBD_CUDA(gd->inputs.reserve(off));
  char* base = gd->inputs.as<char>();
  std::vector<char> host(off, 0);
  auto put = [&](int idx, const void* src, size_t b) { std::memcpy(host.data() + offs[idx], src, b); };
  put(0, p.coords.data(), sizeof(double) * 3 * N);
  put(1, p.alpha0.data(), sizeof(double) * N);
  put(2, p.c6free.data(), sizeof(double) * N);
  put(3, p.r0.data(), sizeof(double) * N);
  put(4, p.hirsh.data(), sizeof(double) * N);
  put(5, p.scs_shifts.data(), sizeof(double) * 3 * nshift_s);
  put(6, p.cfdm_shifts.data(), sizeof(double) * 3 * nshift_c);
  put(7, p.diff_shift.data(), sizeof(double) * 3 * ndiff);
  put(8, p.diff_is_zero.data(), sizeof(int) * ndiff);
  put(9, p.place_offset.data(), sizeof(int) * (ndiff + 1));
  put(10, p.place_rc.data(), sizeof(int) * nplace);
  put(11, p.place_cc.data(), sizeof(int) * nplace);
  MBD_CUDA(cudaMemcpyAsync(base, host.data(), off, cudaMemcpyHostToDevice, ctx->stream));
  ctx->h2d_bytes += (double)off;
  gd->coords = reinterpret_cast<const double*>(base + offs[0]);
  gd->alpha0 = reinterpret_cast<const double*>(base + offs[1]);
  gd->c6free = reinterpret_cast<const double*>(base + offs[2]);
  gd->r0 = reinterpret_cast<const double*>(base + offs[3]);
  gd->hirsh = reinterpret_cast<const double*>(base + offs[4]);
  gd->scs_shifts = reinterpret_cast<const double*>(base + offs[5]);
  gd->cfdm_shifts = reinterpret_cast<const double*>(base + offs[6]);
  gd->diff_shift = reinterpret_cast<const double*>(base + offs[7]);
  gd->diff_is_zero = reinterpret_cast<const int*>(base + offs[8]);
  gd->place_offset = reinterpret_cast<const int*>(base + offs[9]);
  gd->place_rc = reinterpret_cast<const int*>(base + offs[10]);
  gd->place_cc = reinterpret_cast<const int*>(base + offs[11]);
  // results
  off = 0;
  offs.clear();
  add(bytes_of<double>(21 * N));   // 0 alpha_w
  add(bytes_of<double>(21 * N));   // 1 sgm
  add(bytes_of<double>(N));        // 2 rvdw_iso
  add(bytes_of<double>(21 * N));   // 3 alpha_iw
  add(bytes_of<double>(21 * 9));   // 4 molpol
  add(bytes_of<double>(N));        // 5 c6_eff
  add(bytes_of<double>(N));        // 6 alpha_eff
  add(bytes_of<double>(N));        // 7 omega
  add(bytes_of<double>(N));        // 8 rvdw_eff
  add(bytes_of<double>(8));        // 9 scalars
  add(bytes_of<double>(8));        // 10 energy
  add(bytes_of<double>(p.nH));     // 11 d
  add(bytes_of<double>(p.nH));     // 12 e
  add(bytes_of<double>(2 * (size_t)p.nH));   // 13 ev (+ e^2 scratch of the bisection)
  add(bytes_of<int>(32));          // 14 info
  add(bytes_of<double>(32));       // 15 rnorm2 (squared refinement residual per frequency)
  add(bytes_of<double>(kNFreq * kCgState));   // 16 block-CG state
  MBD_CUDA(gd->results.reserve(off));
  base = gd->results.as<char>();
  MBD_CUDA(cudaMemsetAsync(base, 0, off, ctx->stream));
  gd->alpha_w = reinterpret_cast<double*>(base + offs[0]);
  gd->sgm = reinterpret_cast<double*>(base + offs[1]);
  gd->rvdw_iso = reinterpret_cast<double*>(base + offs[2]);
  gd->alpha_iw = reinterpret_cast<double*>(base + offs[3]);
  gd->molpol = reinterpret_cast<double*>(base + offs[4]);
  gd->c6_eff = reinterpret_cast<double*>(base + offs[5]);
  gd->alpha_eff = reinterpret_cast<double*>(base + offs[6]);
  gd->omega = reinterpret_cast<double*>(base + offs[7]);
  gd->rvdw_eff = reinterpret_cast<double*>(base + offs[8]);
  gd->scalars = reinterpret_cast<double*>(base + offs[9]);
  gd->energy = reinterpret_cast<double*>(base + offs[10]);
  gd->d = reinterpret_cast<double*>(base + offs[11]);
  gd->e = reinterpret_cast<double*>(base + offs[12]);
  gd->ev = reinterpret_cast<double*>(base + offs[13]);
  gd->info = reinterpret_cast<int*>(base + offs[14]);
  gd->rnorm2 = reinterpret_cast<double*>(base + offs[15]);
  gd->cgstate = reinterpret_cast<double*>(base + offs[16]);
  gd->n_edges = -1;   // the learned-mode graph of the new geometry is built on first use
  return MBD_OK;
}

int tridiag_group_ctas(const mbd_ctx* ctx, int n) {
  const int nt = (n + kTrdTile - 1) / kTrdTile;
  const int tiles = nt * (nt + 1) / 2;
  return std::max(1, std::min(std::min(ctx->num_sms * ctx->trd_ctas_per_sm, tiles), kTridiagMaxGroup));
}

// ---- plan of the grouped tridiagonal reduction ----------------------------
// Time model of reducing one n x n matrix with a group of G CTAs, in
// microseconds per column: a fixed part (reflector, cross-CTA sums, and two
// group barriers when G > 1) plus the SYMV over the trailing triangle, whose
// average size per column is n^2/6 elements, shared by min(G, tiles) CTAs.
// Coefficients fitted to B200 runs of the kernel at n = 1500, 3000, 6000.
double trd_col_us(int n, int G) {
  const int nt = (n + kTrdTile - 1) / kTrdTile;
  const int ge = std::max(1, std::min(G, nt * (nt + 1) / 2));
  return (G == 1 ? 7.0 : 12.0) + 9.1e-5 * (double)n * (double)n / ge;
}
double trd_us(int n, int G) { return n < 2 ? 1.0 : (double)n * trd_col_us(n, G); }

struct TrdPlan {
  std::vector<std::vector<int>> bins;   // job indices per group, descending n
  std::vector<int> G;
  double makespan_us = 0.0;
};

// Partitions `ctas` co-resident CTAs into groups and the jobs (matrix sizes)
// among them to minimise the modelled makespan: for B = min(jobs, ctas),
// B/2, ..., 1 groups, longest-first assignment of the jobs at one CTA per
// group, then the spare CTAs go one at a time to the slowest group while that
// shortens it.  The best B wins.
TrdPlan plan_tridiag(const std::vector<int>& sizes, int ctas) {
  TrdPlan best;
  const int J = (int)sizes.size();
  if (J == 0 || ctas < 1) return best;
  std::vector<int> idx(J);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return sizes[a] > sizes[b]; });
  best.makespan_us = 1e300;
  for (int B = std::min(J, ctas); B >= 1; B = (B == 1) ? 0 : std::max(1, B / 2)) {
    TrdPlan p;
    p.bins.assign(B, {});
    p.G.assign(B, 1);
    std::vector<double> load(B, 0.0);
    for (int j : idx) {
      const int b = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      p.bins[b].push_back(j);
      load[b] += trd_us(sizes[j], 1);
    }
    auto bin_time = [&](int b, int g) {
      double t = 0.0;
      for (int j : p.bins[b]) t += trd_us(sizes[j], g);
      return t;
    };
    int spare = ctas - B;
    while (spare > 0) {
      const int b = (int)(std::max_element(load.begin(), load.end()) - load.begin());
      if (p.G[b] >= kTridiagMaxGroup) break;
      const double t2 = bin_time(b, p.G[b] + 1);
      if (!(t2 < load[b])) break;
      p.G[b] += 1;
      load[b] = t2;
      --spare;
    }
    p.makespan_us = *std::max_element(load.begin(), load.end());
    if (p.makespan_us < best.makespan_us) best = p;
  }
  return best;
}

// ---- relay stages of one geometry (on its slot's stream) ------------------

// Mixed relay solve: FP32 copy factorised with 3xTF32 tcgen05 GEMMs (128-wide
// panels), FP64 iterative refinement against the FP64 matrices.  Leaves the
// refined solution X (n x 3 per frequency) at the start of slot.mixv.
int relay_mixed(mbd_ctx* ctx, GeomDev* gd, RelaySlot& sl, size_t mstride, cudaEvent_t ev_factor) {
  const GeomPlan& p = gd->plan;
  cudaStream_t s = sl.stream;
  const int n = p.n;
  const int npad = round_up(n, kMixNB);
  BatchMat32 m32{sl.relay32.as<float>(), mstride, p.ld, n, kNFreq};
  float* phi = sl.p_hi.as<float>();
  float* plo = sl.p_lo.as<float>();
  float* lhi = sl.l_hi.as<float>();
  float* llo = sl.l_lo.as<float>();
  const size_t pb = (size_t)npad * kMixNB;   // elements per matrix of the panel / Linv buffers
  Tc3Maps trsm_maps, syrk_maps;
  // panel operands/outputs cover rows [0, n) (TMA zero-fills beyond), the
  // diagonal inverses [0, npad), the output matrix is the n x n FP32 relay copy
  bool ok = make_tc3_map(&trsm_maps.a_hi, phi, n, kMixNB, kMixNB, pb, kNFreq) &&
            make_tc3_map(&trsm_maps.a_lo, plo, n, kMixNB, kMixNB, pb, kNFreq) &&
            make_tc3_map(&trsm_maps.b_hi, lhi, npad, kMixNB, kMixNB, pb, kNFreq) &&
            make_tc3_map(&trsm_maps.b_lo, llo, npad, kMixNB, kMixNB, pb, kNFreq) &&
            make_tc3_map(&trsm_maps.c, m32.A, n, n, p.ld, mstride, kNFreq);
  if (!ok) return MBD_ERR_DEVICE;
  trsm_maps.c_hi = trsm_maps.a_hi;
  trsm_maps.c_lo = trsm_maps.a_lo;
  syrk_maps.a_hi = trsm_maps.a_hi;
  syrk_maps.a_lo = trsm_maps.a_lo;
  syrk_maps.b_hi = trsm_maps.a_hi;
  syrk_maps.b_lo = trsm_maps.a_lo;
  syrk_maps.c = trsm_maps.c;
  syrk_maps.c_hi = trsm_maps.a_hi;
  syrk_maps.c_lo = trsm_maps.a_lo;
  for (int k0 = 0; k0 < n; k0 += kMixNB) {
    launch_potrf_diag_f32(m32, k0, lhi, llo, pb, gd->info, s);
    ctx->launches += 1;
    const int rows = n - k0 - kMixNB;
    if (rows <= 0) continue;
    launch_split(m32.A, mstride, p.ld, k0 + kMixNB, k0, rows, kMixNB, phi, plo, pb, kMixNB, kNFreq, s);
    const int mt = (rows + 127) / 128;
    Tc3Params tp{};
    tp.mode = TC3_STORE_SPLIT;
    tp.batch = kNFreq;
    tp.a_row0 = k0 + kMixNB;
    tp.b_row0 = k0;
    tp.m_rows = rows;
    tp.n_cols = kMixNB;
    tp.k = kMixNB;
    tp.n_tiles_n = 1;
    tp.C = m32.A;
    tp.c_bstride = mstride;
    tp.c_ld = p.ld;
    tp.c_row0 = k0 + kMixNB;
    tp.c_col0 = k0;
    tp.out_hi = phi;
    tp.out_lo = plo;
    tp.o_bstride = pb;
    tp.o_ld = kMixNB;
    tp.err = ctx->err_flag;
    launch_tc3_gemm(trsm_maps, tp, mt, s);
    Tc3Params sp = tp;
    sp.mode = TC3_SYRK_LOWER;
    sp.b_row0 = k0 + kMixNB;
    sp.n_cols = rows;
    sp.c_col0 = k0 + kMixNB;
    sp.out_hi = sp.out_lo = nullptr;
    launch_tc3_gemm(syrk_maps, sp, mt * (mt + 1) / 2, s);
    ctx->launches += 3;
  }
  record_timing(ctx, ev_factor, s);
  // FP64 iterative refinement: X = 0, R = B; repeat D = (LL^T)^-1 R, X += D, R = B - A X
  const size_t ystride = (size_t)n * 3;
  double* X = sl.mixv.as<double>();
  double* R = X + kNFreq * ystride;
  double* Z = R + kNFreq * ystride;
  double* D = Z + kNFreq * ystride;
  MBD_CUDA(cudaMemsetAsync(X, 0, sizeof(double) * kNFreq * ystride, s));
  launch_init_rhs(R, ystride, n, kNFreq, s);
  ctx->launches += 1;
  const int nblk = (n + kMixNB - 1) / kMixNB;
  for (int it = 0; it < kRefineIters; ++it) {
    launch_solve_f32(m32, lhi, llo, pb, R, Z, D, ystride, sl.solve_sync.as<int>(), ++sl.solve_epoch,
                     ctx->err_flag, s);
    launch_relay_residual(sl.relay64.as<double>(), mstride, p.ld, n, kNFreq, X, D, R, ystride,
                          sl.res_ws.as<double>(), gd->rnorm2, s);
    ctx->launches += 2 * nblk + 4;
  }
  return MBD_OK;
}

}  // namespace

void drop_graphs(mbd_ctx* ctx, bool keep_first) {
  for (int m = 0; m < 3; ++m) {
    cudaGraphExec_t& g = ctx->graph[m];
    cudaGraphExec_t& prev = ctx->graph_prev[m];
    if (g && keep_first && ctx->graph_first[m]) {
      if (prev) cudaGraphExecDestroy(prev);
      prev = g;
    } else if (g) {
      cudaGraphExecDestroy(g);
    }
    g = nullptr;
    ctx->graph_first[m] = false;
    if (!keep_first && prev) {
      cudaGraphExecDestroy(prev);
      prev = nullptr;
      ctx->graph_sig[m].clear();
    }
  }
  // the next compute of each mode launches directly again (and reads back
  // the CG iterations), the one after it captures
  for (auto& gd : ctx->geoms) gd->cg_iters_seen = gd->cg_iters_seen1 = 0;
  for (int& k : ctx->mode_runs) k = 0;
}

int band_to_tridiag_single(mbd_ctx* ctx, double* Br, int n, double* d, double* e, DevBuf& scratch, cudaStream_t s) {
  const int C = (ctx->cluster_chase && !ctx->test_stall_wait && n <= sb2st_cluster_max_n() &&
                 tuned_chase_c(ctx, n) != kChaseFlag)
                    ? sb2st_cluster_size(n, 1, ctx->num_sms, tuned_chase_c(ctx, n)) : 0;
  if (C > 0) {
    const BandJob job{Br, n, d, e};
    MBD_CUDA(scratch.reserve(bytes_of<BandJob>(1)));
    MBD_CUDA(cudaMemcpyAsync(scratch.p, &job, sizeof(job), cudaMemcpyHostToDevice, s));
    MBD_CUDA(cudaStreamSynchronize(s));   // the pageable source must outlive the copy
    MBD_CUDA(launch_sb2st_cluster(scratch.as<BandJob>(), 1, n, C, s));
    ctx->launches += 1;
    return MBD_OK;
  }
  std::vector<SweepItem> items;
  for (int i = 0; i + 3 <= n; ++i) items.push_back(SweepItem{0, i, i - 1, 0});
  const BandJob job{Br, n, d, e};
  const size_t b_job = bytes_of<BandJob>(1), b_it = bytes_of<SweepItem>(std::max<size_t>(items.size(), 1));
  const size_t b_pr = bytes_of<int>(2 * std::max<size_t>(items.size(), 1));
  MBD_CUDA(scratch.reserve(b_job + b_it + b_pr));
  char* base = scratch.as<char>();
  std::vector<char> host(b_job + b_it, 0);
  std::memcpy(host.data(), &job, sizeof(job));
  std::memcpy(host.data() + b_job, items.data(), sizeof(SweepItem) * items.size());
  MBD_CUDA(cudaMemcpyAsync(base, host.data(), host.size(), cudaMemcpyHostToDevice, s));
  MBD_CUDA(cudaStreamSynchronize(s));   // the pageable source must outlive the copy
  MBD_CUDA(launch_sb2st(reinterpret_cast<BandJob*>(base), 1, reinterpret_cast<SweepItem*>(base + b_job),
                        (int)items.size(), reinterpret_cast<int*>(base + b_job + b_it), ctx->err_flag,
                        ctx->num_sms, n, n / (2 * kBand) + 1, -1, s));
  ctx->launches += 3;
  return MBD_OK;
}

// Relay and CFDM stages of geometry gi on its slot's stream: per-atom
// frequency table, relay tensors, relay factorisation and solve (plain or
// mixed), screened polarizabilities and C6, CFDM Hamiltonian into gd->hmat.
int run_front(mbd_ctx* ctx, GeomDev* gd, int gi, int mode, bool relay_only) {
  NvtxRange nvtx("mbd_b200 enqueue geometry");
  const GeomPlan& p = gd->plan;
  RelaySlot& sl = *ctx->slots[gd->slot];
  cudaStream_t s = sl.stream;
  const int N = p.N, n = p.n;
  cudaEvent_t* ev = ctx->events.data() + (size_t)gi * kGeomEvents;
  auto mark = [&](int k) { record_timing(ctx, ev[k], s); };
  const bool mixed = mode == MBD_MODE_MIXED;
  const bool learned = mode == MBD_MODE_MIXED_LEARNED;
  mark(0);
  // 1. per-atom frequency table
  AtomDev ad{gd->coords, gd->alpha0, gd->c6free, gd->r0, gd->hirsh, gd->alpha_w, gd->sgm, gd->rvdw_iso};
  launch_atom_freq(ad, N, s);
  ctx->launches += 1;
  MBD_CUDA(cudaMemsetAsync(gd->info, 0, sizeof(int) * 32, s));
  mark(1);
  // 2. relay matrices (21, FP64; plus an FP32 copy in mixed mode)
  const size_t mstride = (size_t)n * p.ld;
  RelayBuildArgs rb{N, p.ld, mstride, gd->coords, gd->alpha_w, gd->sgm, gd->rvdw_iso, gd->scs_shifts,
                    (int)p.scs_shifts.size() / 3, p.beta, p.scs_eval_cut, sl.relay64.as<double>(),
                    (mixed || (learned && ctx->cg_fp32)) ? sl.relay32.as<float>() : nullptr};
  rb.f32_math = (mixed || learned) && ctx->f32_tensor_build;
  launch_relay_build(rb, s);
  ctx->launches += 1;
  mark(2);
  const size_t ystride = (size_t)n * 3;
  double* Xv = nullptr;
  if (mixed) {
    int st = relay_mixed(ctx, gd, sl, mstride, ev[3]);
    if (st != MBD_OK) return st;
    Xv = sl.mixv.as<double>();
  } else if (learned) {
    // network warm start (stage 3), block-CG (stage 4)
    int st = relay_learned(ctx, gd, sl, mstride, ev[3], &Xv);
    if (st != MBD_OK) return st;
  } else {
    // 3. blocked Cholesky, batched over the 21 frequencies
    BatchMat bm{sl.relay64.as<double>(), mstride, p.ld, n, kNFreq};
    const int nblk = (n + kCholNB - 1) / kCholNB;
    const size_t lstride = (size_t)nblk * kCholNB * kCholNB;
    double* Linv = sl.linv.as<double>();
    for (int k0 = 0; k0 < n; k0 += kCholNB) {
      launch_potrf_diag_f64(bm, k0, Linv, lstride, gd->info, s);
      launch_trsm_panel_f64(bm, k0, Linv, lstride, s);
      launch_syrk_lower_f64(bm, k0, s);
      ctx->launches += (k0 + kCholNB < n) ? 3 : 1;
    }
    mark(3);
    // 4. solve X = A^-1 [I;..;I]
    double* Wv = sl.rhs.as<double>();
    double* Zv = Wv + kNFreq * ystride;
    Xv = Zv + kNFreq * ystride;
    launch_init_rhs(Wv, ystride, n, kNFreq, s);
    for (int k0 = 0; k0 < n; k0 += kCholNB) launch_trsv_fwd_step(bm, k0, Linv, lstride, Wv, Zv, ystride, s);
    for (int k0 = (nblk - 1) * kCholNB; k0 >= 0; k0 -= kCholNB)
      launch_trsv_bwd_step(bm, k0, Linv, lstride, Zv, Xv, ystride, s);
    ctx->launches += 1 + 2 * nblk;
  }
  EpilogueArgs ea{N, Xv, ystride, gd->alpha_iw, gd->molpol, gd->alpha0, gd->c6free, gd->r0,
                  gd->c6_eff, gd->alpha_eff, gd->omega, gd->rvdw_eff, gd->scalars};
  launch_relay_epilogue(ea, s);
  launch_relay_post(ea, ctx->weights_dev, s);
  ctx->launches += 2;
  mark(4);
  if (relay_only) {
    mark(5);
    mark(6);
    return cuda_status(cudaGetLastError());
  }
  // 5. CFDM Hamiltonian (lower blocks; the rest of the matrix is never read)
  CfdmBuildArgs cb{N, p.nsl, p.ldH, gd->coords, gd->omega, gd->alpha_eff, gd->rvdw_eff, gd->cfdm_shifts,
                   (int)p.cfdm_shifts.size() / 3, gd->diff_shift, gd->diff_is_zero, gd->place_offset,
                   gd->place_rc, gd->place_cc, (int)p.diff_is_zero.size(), p.beta, p.cfdm_cut,
                   gd->hmat.as<double>()};
  launch_cfdm_build(cb, s);
  ctx->launches += 1;
  mark(5);
  // 6. dense -> band (stage 1 of the two-stage tridiagonalisation)
  if (two_stage(ctx, p.nH)) {
    MBD_CUDA(launch_sy2sb(gd->hmat.as<double>(), p.ldH, p.nH, sl.trd_ws.as<double>(), gd->band.as<double>(),
                          ctx->num_sms, s, tuned_rows(ctx, p.nH), tuned_panel_qr(ctx, p.nH),
                          lookahead_for(ctx, sl.la)));
    ctx->launches += sy2sb_launches(p.nH);
  }
  mark(6);
  return cuda_status(cudaGetLastError());
}

namespace {

// Eigen stages of one geometry on stream s with its own launches (the
// residual-gate fallback of download; run_front has reduced a two-stage
// geometry's Hamiltonian to its band already).
int run_tail_single(mbd_ctx* ctx, GeomDev* gd, cudaStream_t s) {
  const GeomPlan& p = gd->plan;
  if (two_stage(ctx, p.nH)) {
    int st = band_to_tridiag_single(ctx, gd->band.as<double>(), p.nH, gd->d, gd->e, ctx->fb_ws, s);
    if (st != MBD_OK) return st;
  } else {
    TridiagJob job{gd->hmat.as<double>(), p.nH, p.ldH, gd->d, gd->e};
    MBD_CUDA(cudaMemcpyAsync(ctx->job_dev, &job, sizeof(job), cudaMemcpyHostToDevice, s));
    const int G = tridiag_group_ctas(ctx, p.nH);
    const size_t wsb = tridiag_workspace_bytes(p.nH, G);
    MBD_CUDA(ctx->fb_ws.reserve(wsb));
    MBD_CUDA(launch_tridiag(ctx->job_dev, 1, 1, G, ctx->fb_ws.p, wsb, p.nH, ctx->err_flag, s));
    ctx->launches += 1;
  }
  launch_tridiag_eigenvalues(gd->d, gd->e, p.nH, gd->ev, s);
  launch_energy(gd->ev, p.nH, p.nsl, gd->scalars, gd->energy, s);
  ctx->launches += 2;
  return cuda_status(cudaGetLastError());
}

// ---- workspaces and the batch plan ----------------------------------------

size_t plain_bytes(const GeomPlan& p, size_t* relay, size_t* linv, size_t* rhs) {
  const int nblk = (p.n + kCholNB - 1) / kCholNB;
  *relay = sizeof(double) * (size_t)kNFreq * p.n * p.ld;
  *linv = sizeof(double) * (size_t)kNFreq * nblk * kCholNB * kCholNB;
  *rhs = sizeof(double) * 3 * (size_t)kNFreq * p.n * 3;
  return *relay + *linv + *rhs;
}

size_t mixed_bytes(const GeomPlan& p, size_t* r32, size_t* pan, size_t* vec, size_t* res, size_t* sync) {
  *r32 = sizeof(float) * (size_t)kNFreq * p.n * p.ld;
  *pan = sizeof(float) * (size_t)kNFreq * round_up(p.n, kMixNB) * kMixNB;
  *vec = sizeof(double) * 4 * (size_t)kNFreq * p.n * 3;
  *res = sizeof(double) * relay_residual_ws_doubles(p.n, kNFreq);
  *sync = sizeof(int) * solve_sync_ints(p.n, kNFreq);
  return *r32 + 4 * *pan + *vec + *res + *sync;
}

// Assigns the geometries to relay slots (longest first onto the least loaded
// slot, load = (3N)^3), with as many slots as fit in the device memory share.
int plan_slots(mbd_ctx* ctx) {
  const int ng = (int)ctx->order.size();
  size_t free_b = 0, total_b = 0;
  MBD_CUDA(cudaMemGetInfo(&free_b, &total_b));
  size_t held = 0;
  for (auto& s : ctx->slots) held += s->held();
  const double budget = kSlotMemoryShare * (double)(free_b + held);
  int S = std::max(1, std::min(kMaxSlots, ng));
  std::vector<int> slot_of(ctx->geoms.size(), 0);
  for (; S >= 1; --S) {
    std::vector<double> load(S, 0.0);
    std::vector<size_t> need(S, 0);
    for (int g : ctx->order) {
      const GeomPlan& p = ctx->geoms[g]->plan;
      const int s = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      slot_of[g] = s;
      load[s] += std::pow((double)p.n, 3.0);
      size_t a, b, c, d, e, f, h;
      need[s] = std::max(need[s], plain_bytes(p, &a, &b, &c) + mixed_bytes(p, &d, &e, &f, &h, &a));
    }
    double total = 0.0;
    for (size_t x : need) total += (double)x;
    if (total <= budget || S == 1) break;
  }
  for (int g : ctx->order) ctx->geoms[g]->slot = slot_of[g];
  while ((int)ctx->slots.size() < S) {
    std::unique_ptr<RelaySlot> sl(new RelaySlot());
    // slot 0 takes the batch's largest geometry (longest first), whose
    // stages set the batch's length: its stream runs at the device's highest
    // priority, so the block scheduler serves its kernels before the other
    // slots' (MBD_B200_PRIORITY=0: all at the default priority)
    int least = 0, greatest = 0;
    MBD_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    const int prio = (ctx->priorities && ctx->slots.empty()) ? greatest : least;
    MBD_CUDA(cudaStreamCreateWithPriority(&sl->stream, cudaStreamNonBlocking, prio));
    MBD_CUDA(cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming));
    MBD_CUDA(create_lookahead(&sl->la));
    ctx->slots.push_back(std::move(sl));
  }
  ctx->n_slots = S;
  return MBD_OK;
}

// Plain-path slot buffers, per-geometry Hamiltonians, the tridiagonal plan and
// the device job tables of the uploaded batch.
int prepare_batch(mbd_ctx* ctx, bool eigen) {
  drop_graphs(ctx, true);
  ctx->order.clear();
  for (size_t g = 0; g < ctx->geoms.size(); ++g)
    if (ctx->geoms[g]->status_host == MBD_OK) ctx->order.push_back((int)g);
  // Tridiagonalisation path.  Measured on B200 (mixed mode, one geometry,
  // reduction + eigenvalues, one-stage vs two-stage): n = 300: 7.6 vs 3.7 ms,
  // n = 1050: 15.0 vs 14.2, n = 1500: 22.4 vs 20.9, n = 3000: 54.8 vs 47.3;
  // a batch of 8 geometries n = 270 .. 1800: step 50.3 vs 38.6 ms.  So every
  // matrix the two-stage reduction can take goes through it; larger ones
  // (n above the panel cluster's rows) take the one-stage grouped launch.
  ctx->two_stage_batch = ctx->two_stage_force != 0;
  std::stable_sort(ctx->order.begin(), ctx->order.end(),
                   [&](int a, int b) { return ctx->geoms[a]->plan.n > ctx->geoms[b]->plan.n; });
  for (int g : ctx->order) {
    const GeomPlan& p = ctx->geoms[g]->plan;
    if (!eigen) continue;
    MBD_CUDA(ctx->geoms[g]->hmat.reserve(sizeof(double) * (size_t)p.nH * p.ldH));
    if (two_stage(ctx, p.nH)) MBD_CUDA(ctx->geoms[g]->band.reserve(sizeof(double) * (size_t)p.nH * kBandLd));
  }
  const size_t nev = ctx->geoms.size() * kGeomEvents;
  while (ctx->events.size() < nev) {
    cudaEvent_t e;
    MBD_CUDA(cudaEventCreate(&e));
    ctx->events.push_back(e);
  }
  if (ctx->order.empty()) {
    ctx->n_slots = 0;
    ctx->n_trd_groups = ctx->trd_total_ctas = ctx->n_eig_jobs = ctx->n_eig_batch = 0;
    return MBD_OK;
  }
  int st = plan_slots(ctx);
  if (st != MBD_OK) return st;
  for (int s = 0; s < ctx->n_slots; ++s) {
    size_t relay = 0, linv = 0, rhs = 0;
    for (int g : ctx->order) {
      if (ctx->geoms[g]->slot != s) continue;
      size_t a, b, c;
      plain_bytes(ctx->geoms[g]->plan, &a, &b, &c);
      relay = std::max(relay, a);
      linv = std::max(linv, b);
      rhs = std::max(rhs, c);
    }
    RelaySlot& sl = *ctx->slots[s];
    MBD_CUDA(sl.relay64.reserve(relay));
    MBD_CUDA(sl.linv.reserve(linv));
    MBD_CUDA(sl.rhs.reserve(rhs));
    if (eigen) {
      size_t tw = 0;
      for (int g : ctx->order)
        if (ctx->geoms[g]->slot == s && two_stage(ctx, ctx->geoms[g]->plan.nH))
          tw = std::max(tw, sizeof(double) * sy2sb_workspace_doubles(ctx->geoms[g]->plan.nH));
      MBD_CUDA(sl.trd_ws.reserve(tw));
    }
  }
  if (!eigen) {
    ctx->n_trd_groups = ctx->trd_total_ctas = ctx->n_eig_jobs = ctx->n_eig_batch = 0;
    return MBD_OK;
  }
  // one-stage tridiagonal plan for the matrices too large for the two-stage path
  std::vector<int> sizes, one_stage;
  for (int g : ctx->order)
    if (!two_stage(ctx, ctx->geoms[g]->plan.nH)) {
      sizes.push_back(ctx->geoms[g]->plan.nH);
      one_stage.push_back(g);
    }
  const TrdPlan tp = plan_tridiag(sizes, ctx->num_sms * ctx->trd_ctas_per_sm);
  std::vector<TridiagJob> jobs;
  std::vector<TridiagGroup> groups;
  size_t ws_off = 0;
  int cta = 0;
  for (size_t b = 0; b < tp.bins.size(); ++b) {
    TridiagGroup gr{};
    gr.first_cta = cta;
    gr.G = tp.G[b];
    gr.job_begin = (int)jobs.size();
    gr.nmax = 1;
    for (int j : tp.bins[b]) {
      GeomDev* gd = ctx->geoms[one_stage[j]].get();
      const GeomPlan& p = gd->plan;
      jobs.push_back(TridiagJob{gd->hmat.as<double>(), p.nH, p.ldH, gd->d, gd->e});
      gr.nmax = std::max(gr.nmax, p.nH);
    }
    gr.job_end = (int)jobs.size();
    gr.ws_offset = ws_off;
    ws_off += (tridiag_workspace_bytes(gr.nmax, gr.G) + 255) & ~size_t(255);
    cta += gr.G;
    groups.push_back(gr);
  }
  ctx->n_trd_groups = (int)groups.size();
  ctx->trd_total_ctas = cta;
  ctx->trd_est_ms = tp.makespan_us / 1000.0;
  MBD_CUDA(ctx->tridiag_ws.reserve(ws_off));
  // eigenvalue jobs: the batched launch first, then matrices too large for it
  std::vector<EigJob> eig;
  ctx->eig_single.clear();
  ctx->eig_batch_max_n = 0;
  for (int pass = 0; pass < 2; ++pass)
    for (int g : ctx->order) {
      GeomDev* gd = ctx->geoms[g].get();
      const GeomPlan& p = gd->plan;
      const bool fits = p.nH <= kEigBatchMaxN;
      if (fits != (pass == 0)) continue;
      eig.push_back(EigJob{gd->d, gd->e, gd->ev, gd->scalars, gd->energy, p.nH, p.nsl});
      if (fits) ctx->eig_batch_max_n = std::max(ctx->eig_batch_max_n, p.nH);
      else ctx->eig_single.push_back(g);
    }
  ctx->n_eig_jobs = (int)eig.size();
  ctx->n_eig_batch = ctx->n_eig_jobs - (int)ctx->eig_single.size();
  // band -> tridiagonal: one job per two-stage matrix, (job, sweep) items
  // ordered by sweep then job, each pointing at its job's previous sweep
  // (the bands that fit a cluster's shared memory first, largest first; the
  // flag-synchronised chase takes the rest, and all of them while the
  // failure-detection stall is on: its waits are the ones that can run out)
  std::vector<BandJob> bjobs, fjobs;
  // one chase kernel per batch (the two launches would run one after the
  // other): the one tuned for the batch's largest band, whose chase sets the
  // launch's length
  int big = 0;
  for (int g : ctx->order)
    if (two_stage(ctx, ctx->geoms[g]->plan.nH)) big = std::max(big, ctx->geoms[g]->plan.nH);
  const bool cluster_ok = ctx->cluster_chase && !ctx->test_stall_wait && big > 0 &&
                          big <= sb2st_cluster_max_n() && tuned_chase_c(ctx, big) != kChaseFlag;
  const int cap = cluster_ok ? sb2st_cluster_max_n() : 0;
  ctx->band_max_n = ctx->band_cluster_max_n = 0;
  for (int g : ctx->order) {
    GeomDev* gd = ctx->geoms[g].get();
    if (!two_stage(ctx, gd->plan.nH)) continue;
    const BandJob bj{gd->band.as<double>(), gd->plan.nH, gd->d, gd->e};
    if (bj.n <= cap) {
      bjobs.push_back(bj);
      ctx->band_cluster_max_n = std::max(ctx->band_cluster_max_n, bj.n);
    } else {
      fjobs.push_back(bj);
      ctx->band_max_n = std::max(ctx->band_max_n, bj.n);
    }
  }
  std::stable_sort(bjobs.begin(), bjobs.end(), [](const BandJob& a, const BandJob& b) { return a.n > b.n; });
  ctx->n_band_cluster = (int)bjobs.size();
  ctx->band_cluster_C = sb2st_cluster_size(ctx->band_cluster_max_n, ctx->n_band_cluster, ctx->num_sms,
                                           tuned_chase_c(ctx, ctx->band_cluster_max_n));
  if (ctx->n_band_cluster > 0 && ctx->band_cluster_C < 1) {   // no cluster fits after all
    fjobs.insert(fjobs.begin(), bjobs.begin(), bjobs.end());
    for (const BandJob& bj : bjobs) ctx->band_max_n = std::max(ctx->band_max_n, bj.n);
    bjobs.clear();
    ctx->n_band_cluster = 0;
  }
  std::vector<SweepItem> items;
  {
    std::vector<int> last(fjobs.size(), -1);
    for (int i = 0; i + 3 <= ctx->band_max_n; ++i)
      for (size_t j = 0; j < fjobs.size(); ++j) {
        if (i + 3 > fjobs[j].n) continue;
        items.push_back(SweepItem{(int)j, i, last[j], 0});
        last[j] = (int)items.size() - 1;
      }
  }
  bjobs.insert(bjobs.end(), fjobs.begin(), fjobs.end());
  ctx->n_band_jobs = (int)bjobs.size();
  ctx->sweeps_in_flight = 0;
  for (const BandJob& bj : fjobs) ctx->sweeps_in_flight += bj.n / (2 * kBand) + 1;
  ctx->n_sweep_items = (int)items.size();
  MBD_CUDA(ctx->sweep_progress.reserve(2 * sizeof(int) * std::max<size_t>(items.size(), 1)));
  const size_t b_jobs = bytes_of<TridiagJob>(jobs.size());
  const size_t b_groups = bytes_of<TridiagGroup>(groups.size());
  const size_t b_eig = bytes_of<EigJob>(eig.size());
  const size_t b_bj = bytes_of<BandJob>(bjobs.size());
  const size_t b_it = bytes_of<SweepItem>(items.size());
  MBD_CUDA(ctx->tables.reserve(b_jobs + b_groups + b_eig + b_bj + b_it));
  char* base = ctx->tables.as<char>();
  ctx->trd_jobs = reinterpret_cast<TridiagJob*>(base);
  ctx->trd_groups = reinterpret_cast<TridiagGroup*>(base + b_jobs);
  ctx->eig_jobs = reinterpret_cast<EigJob*>(base + b_jobs + b_groups);
  ctx->band_jobs = reinterpret_cast<BandJob*>(base + b_jobs + b_groups + b_eig);
  ctx->sweep_items = reinterpret_cast<SweepItem*>(base + b_jobs + b_groups + b_eig + b_bj);
  std::vector<char> host(b_jobs + b_groups + b_eig + b_bj + b_it, 0);
  std::memcpy(host.data(), jobs.data(), sizeof(TridiagJob) * jobs.size());
  std::memcpy(host.data() + b_jobs, groups.data(), sizeof(TridiagGroup) * groups.size());
  std::memcpy(host.data() + b_jobs + b_groups, eig.data(), sizeof(EigJob) * eig.size());
  std::memcpy(host.data() + b_jobs + b_groups + b_eig, bjobs.data(), sizeof(BandJob) * bjobs.size());
  std::memcpy(host.data() + b_jobs + b_groups + b_eig + b_bj, items.data(), sizeof(SweepItem) * items.size());
  MBD_CUDA(h2d_ordered(ctx, base, host.data(), host.size()));
  ctx->h2d_bytes += (double)host.size();
  return MBD_OK;
}

// Buffers only the mixed modes use (allocated on first use).
int reserve_mixed(mbd_ctx* ctx) {
  for (int s = 0; s < ctx->n_slots; ++s) {
    size_t r32 = 0, pan = 0, vec = 0, res = 0, sync = 0;
    for (int g : ctx->order) {
      if (ctx->geoms[g]->slot != s) continue;
      size_t a, b, c, d, e;
      mixed_bytes(ctx->geoms[g]->plan, &a, &b, &c, &d, &e);
      r32 = std::max(r32, a);
      pan = std::max(pan, b);
      vec = std::max(vec, c);
      res = std::max(res, d);
      sync = std::max(sync, e);
    }
    RelaySlot& sl = *ctx->slots[s];
    bool moved = false;
    auto grow = [&](DevBuf& b, size_t bytes) {
      const bool re = bytes > b.bytes;
      moved = moved || re;
      return b.reserve(bytes);
    };
    MBD_CUDA(grow(sl.relay32, r32));
    MBD_CUDA(grow(sl.p_hi, pan));
    MBD_CUDA(grow(sl.p_lo, pan));
    MBD_CUDA(grow(sl.l_hi, pan));
    MBD_CUDA(grow(sl.l_lo, pan));
    MBD_CUDA(grow(sl.mixv, vec));
    MBD_CUDA(grow(sl.res_ws, res));
    MBD_CUDA(grow(sl.solve_sync, sync));
    if (moved) drop_graphs(ctx, true);
  }
  return MBD_OK;
}

// Enqueues the whole batch (relay stages on the slots' streams, then the
// batch-wide eigen stages on the context stream).  Stream-capture safe: no
// allocation, no host-side copies, and the mixed solve's progress flags are
// cleared and its epochs restarted on every run.
int enqueue_batch(mbd_ctx* ctx, int mode) {
  cudaStream_t s = ctx->stream;
  ctx->launches = 0;
  MBD_CUDA(cudaMemsetAsync(ctx->err_flag, 0, sizeof(int), s));
  record_timing(ctx, ctx->bev[0], s);
  if (ctx->order.empty()) {
    for (int k = 1; k < 5; ++k) record_timing(ctx, ctx->bev[k], s);
    return cuda_status(cudaGetLastError());
  }
  // relay and CFDM stages, geometries spread over the slots' streams
  MBD_CUDA(cudaEventRecord(ctx->fork_ev, s));
  for (int k = 0; k < ctx->n_slots; ++k) {
    RelaySlot& sl = *ctx->slots[k];
    MBD_CUDA(cudaStreamWaitEvent(sl.stream, ctx->fork_ev, 0));
    if (mode == MBD_MODE_MIXED) {
      MBD_CUDA(cudaMemsetAsync(sl.solve_sync.p, 0, sl.solve_sync.bytes, sl.stream));
      sl.solve_epoch = 0;
    }
  }
  for (int g : ctx->order) {
    int st = run_front(ctx, ctx->geoms[g].get(), g, mode);
    if (st != MBD_OK) return st;
  }
  for (int k = 0; k < ctx->n_slots; ++k) {
    MBD_CUDA(cudaEventRecord(ctx->slots[k]->done, ctx->slots[k]->stream));
    MBD_CUDA(cudaStreamWaitEvent(s, ctx->slots[k]->done, 0));
  }
  record_timing(ctx, ctx->bev[1], s);
  // bands -> tridiagonal in one persistent launch; matrices too large for the
  // two-stage path in one grouped one-stage launch
  if (ctx->n_trd_groups > 0) {
    MBD_CUDA(launch_tridiag_groups(ctx->trd_jobs, ctx->trd_groups, ctx->n_trd_groups, ctx->trd_total_ctas,
                                   ctx->tridiag_ws.p, ctx->err_flag, s));
    ctx->launches += 2;
  }
  record_timing(ctx, ctx->bev[4], s);
  if (ctx->n_band_cluster > 0) {
    MBD_CUDA(launch_sb2st_cluster(ctx->band_jobs, ctx->n_band_cluster, ctx->band_cluster_max_n,
                                  ctx->band_cluster_C, s));
    ctx->launches += 1;
  }
  if (ctx->n_band_jobs > ctx->n_band_cluster) {
    MBD_CUDA(launch_sb2st(ctx->band_jobs + ctx->n_band_cluster, ctx->n_band_jobs - ctx->n_band_cluster,
                          ctx->sweep_items, ctx->n_sweep_items, ctx->sweep_progress.as<int>(), ctx->err_flag,
                          ctx->num_sms, ctx->band_max_n, ctx->sweeps_in_flight, ctx->test_stall_wait ? 0 : -1, s));
    ctx->launches += 3;
  }
  record_timing(ctx, ctx->bev[2], s);
  // eigenvalues and energies
  launch_eigen_batch(ctx->eig_jobs, ctx->n_eig_batch, ctx->eig_batch_max_n, s);
  ctx->launches += ctx->n_eig_batch > 0 ? 1 : 0;
  for (int g : ctx->eig_single) {
    GeomDev* gd = ctx->geoms[g].get();
    launch_tridiag_eigenvalues(gd->d, gd->e, gd->plan.nH, gd->ev, s);
    ctx->launches += 2;
  }
  launch_energy_batch(ctx->eig_jobs, ctx->n_eig_jobs, s);
  ctx->launches += 1;
  record_timing(ctx, ctx->bev[3], s);
  return cuda_status(cudaGetLastError());
}

// Captures enqueue_batch into a graph for `mode`; false when capture is not
// possible (the caller then enqueues directly).  first: the batch's first
// compute in the mode (the full CG schedule); its graph updates the one kept
// from an earlier batch when the launch sequences match (same kernels and
// dependencies: cudaGraphExecUpdate then rewrites only the launch arguments,
// far cheaper than instantiating), else it is instantiated.
bool capture_batch(mbd_ctx* ctx, int mode, bool first) {
  NvtxRange nvtx(first ? "mbd_b200 capture first compute" : "mbd_b200 capture");
  cudaGraph_t graph = nullptr;
  if (cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  ctx->capturing = true;
  const int st = enqueue_batch(ctx, mode);
  ctx->capturing = false;
  const cudaError_t ec = cudaStreamEndCapture(ctx->stream, &graph);
  cudaGraphExec_t exec = nullptr;
  bool ok = st == MBD_OK && ec == cudaSuccess && graph;
  if (ok && first && ctx->graph_prev[mode]) {
    cudaGraphExecUpdateResultInfo info{};
    const cudaError_t eu = cudaGraphExecUpdate(ctx->graph_prev[mode], graph, &info);
    ctx->graph_update_result = (int)info.result;
    ctx->graph_update_node = -1;
    cudaGraphNodeType nt;
    if (info.errorNode && cudaGraphNodeGetType(info.errorNode, &nt) == cudaSuccess) ctx->graph_update_node = (int)nt;
    if (eu == cudaSuccess) {
      exec = ctx->graph_prev[mode];
      ctx->graph_updates += 1;
    } else {
      cudaGetLastError();
      cudaGraphExecDestroy(ctx->graph_prev[mode]);
    }
    ctx->graph_prev[mode] = nullptr;
  }
  if (ok && !exec)
    ok = cudaGraphInstantiate(&exec, graph, ctx->priorities ? cudaGraphInstantiateFlagUseNodePriority : 0) ==
         cudaSuccess;
  if (graph) cudaGraphDestroy(graph);
  if (!ok) {
    if (exec) cudaGraphExecDestroy(exec);
    cudaGetLastError();
    return false;
  }
  ctx->graph[mode] = exec;
  ctx->graph_first[mode] = first;
  ctx->graph_launches[mode] = ctx->launches;
  return true;
}

// What fixes a batch's launch sequence in `mode`, as far as the host knows
// it before enqueueing: the geometries' sizes, image counts, slots and
// reduction paths.  A first compute is captured only when this matches the
// batch whose graph is kept (or the batch before it), so batches of changing
// shape keep launching kernel by kernel instead of instantiating every time.
std::vector<long long> batch_signature(const mbd_ctx* ctx, int mode) {
  std::vector<long long> sig{mode, ctx->n_slots, (long long)ctx->order.size(), ctx->two_stage_batch ? 1 : 0};
  for (int g : ctx->order) {
    const GeomDev& gd = *ctx->geoms[g];
    const GeomPlan& p = gd.plan;
    sig.insert(sig.end(), {p.N, p.nsl, p.nH, gd.slot, (long long)p.scs_shifts.size(),
                           (long long)p.cfdm_shifts.size(), (long long)p.diff_shift.size(),
                           two_stage(ctx, p.nH) ? 1 : 0});
  }
  return sig;
}

}  // namespace
}  // namespace mbd

using namespace mbd;

extern "C" {

int mbd_rsscs_create(mbd_ctx** out, int device) {
  if (!out) return MBD_ERR_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return MBD_ERR_DEVICE;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return MBD_ERR_DEVICE;
  if (prop.major != 10) return MBD_ERR_DEVICE;   // sm_100a only
  if (!prop.cooperativeLaunch) return MBD_ERR_DEVICE;
  std::unique_ptr<mbd_ctx> ctx(new mbd_ctx());
  ctx->device = device;
  MBD_CUDA(cudaSetDevice(device));
  ctx->num_sms = prop.multiProcessorCount;
  MBD_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  for (auto& e : ctx->bev) MBD_CUDA(cudaEventCreate(&e));
  MBD_CUDA(cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming));
  MBD_CUDA(create_lookahead(&ctx->la_ctx));
  {
    const char* ng = std::getenv("MBD_B200_NO_GRAPHS");
    ctx->use_graphs = !(ng && ng[0] && ng[0] != '0');
    const char* gu = std::getenv("MBD_B200_GRAPH_UPDATE");
    ctx->graph_update = gu && gu[0] == '1';
    // the band -> tridiagonal chase of size classes the autotuner has not
    // timed: flag-synchronised (measured faster at every size on B200);
    // MBD_B200_CLUSTER_CHASE=1 makes it the cluster-resident one, =0 rules
    // the cluster-resident chase out even where the autotuner picks it
    // the learned mode's block-CG runs its matrix passes on an FP32 copy of
    // the relay matrices in two phases with an FP64 restart between them
    // (measured on B200 for the 2000-atom cluster: relay solve 15.7 ms
    // against 17.4 ms for the one-phase FP64 passes) wherever the copy (50 %
    // more relay memory) fits in half the free device memory;
    // MBD_B200_CG_FP32=1 always, =0 never
    const char* cf = std::getenv("MBD_B200_CG_FP32");
    ctx->cg_fp32_mode = (cf && cf[0] == '1') ? 1 : ((cf && cf[0] == '0') ? 0 : -1);
    const char* cc = std::getenv("MBD_B200_CLUSTER_CHASE");
    ctx->cluster_chase = !(cc && cc[0] == '0');
    if (cc && cc[0] == '1')
      for (TuneChoice& t : ctx->tune) t.chase_c = 0;
    const char* pq = std::getenv("MBD_B200_PANEL_QR");
    ctx->panel_qr_default = (pq && std::strcmp(pq, "tsqr") == 0) ? 1 : 0;
    // the dense -> band reduction's look-ahead: each panel's QR beside the
    // previous panel's trailing update (MBD_B200_LOOKAHEAD=0: one stream)
    const char* la = std::getenv("MBD_B200_LOOKAHEAD");
    ctx->lookahead = !(la && la[0] == '0');
    // stream priorities (the largest geometry's slot, the look-ahead QR),
    // kept by captured graphs (MBD_B200_PRIORITY=0: default priority everywhere)
    const char* pr = std::getenv("MBD_B200_PRIORITY");
    ctx->priorities = !(pr && pr[0] == '0');
  }
  MBD_CUDA(init_device_constants());
  MBD_CUDA(init_chol_attributes());
  MBD_CUDA(init_eigval_attributes());
  MBD_CUDA(init_tc3_attributes());
  MBD_CUDA(init_mixed_attributes());
  MBD_CUDA(init_sy2sb_attributes());
  {
    // reduction path (prepare_batch): MBD_B200_TWO_STAGE=0 forces the
    // one-stage path; otherwise two-stage wherever it applies
    const char* ts = std::getenv("MBD_B200_TWO_STAGE");
    ctx->two_stage_max_n = sy2sb_max_n();
    ctx->two_stage_force = (ts && ts[0] == '1') ? 1 : ((ts && ts[0] == '0') ? 0 : -1);
  }
  MBD_CUDA(init_sb2st_attributes());
  ctx->trd_ctas_per_sm = std::max(1, tridiag_max_ctas_per_sm());
  MBD_CUDA(ctx->misc.reserve(4096));
  char* m = ctx->misc.as<char>();
  ctx->weights_dev = reinterpret_cast<double*>(m);
  ctx->err_flag = reinterpret_cast<int*>(m + 256);
  ctx->job_dev = reinterpret_cast<TridiagJob*>(m + 512);
  ctx->omega_dev = reinterpret_cast<double*>(m + 1024);
  ctx->loss_dev = reinterpret_cast<double*>(m + 1280);
  MBD_CUDA(h2d_ordered(ctx.get(), ctx->omega_dev, kCasimirOmega, sizeof(double) * kNFreq));
  MBD_CUDA(h2d_ordered(ctx.get(), ctx->weights_dev, kCasimirWeight, sizeof(double) * kNFreq));
  MBD_CUDA(zero_ordered(ctx.get(), ctx->err_flag, sizeof(int)));
  *out = ctx.release();
  return MBD_OK;
}

void mbd_rsscs_destroy(mbd_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  for (auto e : ctx->events) cudaEventDestroy(e);
  drop_graphs(ctx);
  for (auto e : ctx->bev)
    if (e) cudaEventDestroy(e);
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->la_ctx.ready) cudaEventDestroy(ctx->la_ctx.ready);
  if (ctx->la_ctx.done) cudaEventDestroy(ctx->la_ctx.done);
  if (ctx->la_ctx.aux) cudaStreamDestroy(ctx->la_ctx.aux);
  ctx->geoms.clear();
  ctx->slots.clear();
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

int mbd_rsscs_upload(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms) {
  NvtxRange nvtx("mbd_b200 upload");
  if (!ctx || n_geom < 1 || !geoms) return MBD_ERR_ARG;
  return upload_batch(ctx, n_geom, geoms, true);
}

}  // extern "C"

namespace mbd {

// Uploads a batch; eigen = false prepares only the relay stages (training
// batches: no CFDM Hamiltonians, no eigen plan, not computable).
int upload_batch(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, bool eigen) {
  MBD_CUDA(cudaSetDevice(ctx->device));
  // buffers of the previous batch may still be in use by its kernels
  MBD_CUDA(cudaDeviceSynchronize());
  ctx->have_batch = false;
  ctx->h2d_bytes = 0;
  while ((int)ctx->geoms.size() < n_geom) ctx->geoms.emplace_back(new GeomDev());
  ctx->geoms.resize(n_geom);
  int first = MBD_OK;
  for (int g = 0; g < n_geom; ++g) {
    int st = upload_geometry(ctx, geoms[g], ctx->geoms[g].get());
    ctx->geoms[g]->status_host = st;
    if (st != MBD_OK && first == MBD_OK) first = st;
    if (st == MBD_ERR_OUT_OF_MEMORY || st == MBD_ERR_DEVICE) return st;
  }
  int st = prepare_batch(ctx, eigen);
  if (st != MBD_OK) return st;
  ctx->have_batch = eigen;
  return first;
}

}  // namespace mbd

extern "C" {

int mbd_rsscs_compute(mbd_ctx* ctx, int mode) {
  static const char* const kRange[3] = {"mbd_b200 compute plain", "mbd_b200 compute mixed",
                                        "mbd_b200 compute mixed_learned"};
  NvtxRange nvtx(mode >= 0 && mode < 3 ? kRange[mode] : "mbd_b200 compute");
  if (!ctx || !ctx->have_batch) return MBD_ERR_ARG;
  if (mode != MBD_MODE_PLAIN_FP64 && mode != MBD_MODE_MIXED && mode != MBD_MODE_MIXED_LEARNED) return MBD_ERR_ARG;
  if (mode == MBD_MODE_MIXED_LEARNED && ctx->use_net && !ctx->have_net) return MBD_ERR_NO_NETWORK;
  MBD_CUDA(cudaSetDevice(ctx->device));
  if (mode == MBD_MODE_MIXED) {
    int st = reserve_mixed(ctx);
    if (st != MBD_OK) return st;
  } else if (mode == MBD_MODE_MIXED_LEARNED) {
    int st = reserve_learned(ctx);
    if (st != MBD_OK) return st;
  }
  ctx->last_mode = mode;
  // From the second compute of a batch in a mode on, capture the batch into a
  // CUDA graph once and replay it; a batch computed once (energy_batch, an
  // upload per call) is launched directly and does not pay for the capture.
  //   A context that uploads batch after batch of one shape (a trajectory,
  // the same structures re-submitted) runs each batch's first compute as a
  // graph as well: captured, then written into the graph kept from the
  // previous batch with cudaGraphExecUpdate, which costs a fraction of the
  // gaps between kernels launched one by one.  The learned mode's graph of
  // a first compute runs the full CG schedule; its second compute captures
  // the iterations seen instead and the first graph is kept for the next
  // batch.
  const bool repeat = ctx->mode_runs[mode]++ > 0;
  if (ctx->use_graphs && repeat && ctx->graph[mode] && ctx->graph_first[mode] &&
      mode == MBD_MODE_MIXED_LEARNED) {
    if (ctx->graph_prev[mode]) cudaGraphExecDestroy(ctx->graph_prev[mode]);
    ctx->graph_prev[mode] = ctx->graph[mode];
    ctx->graph[mode] = nullptr;
    ctx->graph_first[mode] = false;
  }
  if (ctx->use_graphs && !ctx->graph[mode]) {
    if (repeat) {
      if (!capture_batch(ctx, mode, false)) ctx->use_graphs = false;
    } else if (ctx->graph_update) {
      std::vector<long long> sig = batch_signature(ctx, mode);
      const bool same = sig == ctx->graph_sig[mode] || sig == ctx->last_sig[mode];
      ctx->last_sig[mode] = sig;
      // a failed capture launches directly below
      if (same && capture_batch(ctx, mode, true)) ctx->graph_sig[mode] = std::move(sig);
    }
  }
  if (ctx->use_graphs && ctx->graph[mode]) {
    ctx->launches = ctx->graph_launches[mode];
    ctx->graph_kind = repeat ? 1 : 2;
    return cuda_status(cudaGraphLaunch(ctx->graph[mode], ctx->stream));
  }
  ctx->graph_kind = 0;
  return enqueue_batch(ctx, mode);
}

int mbd_rsscs_download(mbd_ctx* ctx, mbd_result* out) {
  NvtxRange nvtx("mbd_b200 download");
  if (!ctx || !ctx->have_batch || !out) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  // Every geometry's results in one pass into page-locked memory: the block
  // alpha_iw .. energy and the block info .. CG state of its results buffer,
  // queued behind the batch on the context stream, one synchronisation.
  struct Range {
    const char* lo;
    size_t bytes, at;
  };
  auto range = [](const void* a, const void* b_end) {
    const char* lo = static_cast<const char*>(a);
    return Range{lo, (size_t)(static_cast<const char*>(b_end) - lo), 0};
  };
  std::vector<Range> r1(ctx->geoms.size()), r2(ctx->geoms.size());
  size_t stage = 256;
  for (size_t g = 0; g < ctx->geoms.size(); ++g) {
    const GeomDev* gd = ctx->geoms[g].get();
    if (gd->status_host != MBD_OK) continue;
    r1[g] = range(gd->alpha_iw, gd->energy + 8);
    r2[g] = range(gd->info, gd->cgstate + (size_t)kNFreq * kCgState);
    r1[g].at = stage;
    stage += (r1[g].bytes + 255) & ~size_t(255);
    r2[g].at = stage;
    stage += (r2[g].bytes + 255) & ~size_t(255);
  }
  MBD_CUDA(ctx->staging.reserve(stage));
  char* hs = ctx->staging.as<char>();
  MBD_CUDA(cudaMemcpyAsync(hs, ctx->err_flag, sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  ctx->d2h_bytes = sizeof(int);
  auto fetch = [&](size_t g, cudaStream_t s) -> cudaError_t {
    for (const Range* r : {&r1[g], &r2[g]}) {
      cudaError_t e = cudaMemcpyAsync(hs + r->at, r->lo, r->bytes, cudaMemcpyDeviceToHost, s);
      if (e != cudaSuccess) return e;
      ctx->d2h_bytes += (double)r->bytes;
    }
    return cudaSuccess;
  };
  for (size_t g = 0; g < ctx->geoms.size(); ++g)
    if (ctx->geoms[g]->status_host == MBD_OK) MBD_CUDA(fetch(g, ctx->stream));
  MBD_CUDA(cudaStreamSynchronize(ctx->stream));
  int err = 0;
  std::memcpy(&err, hs, sizeof(int));
  // host copy of a device array inside geometry g's two blocks
  auto host = [&](size_t g, const void* dev) -> const char* {
    const char* d = static_cast<const char*>(dev);
    const Range& r = (d >= r1[g].lo && d < r1[g].lo + r1[g].bytes) ? r1[g] : r2[g];
    return hs + r.at + (d - r.lo);
  };
  // stage timings: relay/CFDM stages summed over geometries (they overlap on
  // the slots' streams), the batch-wide stages and the total from batch events
  for (int k = 0; k < Stage::kCount; ++k) ctx->last_ms[k] = 0.0;
  auto elapsed = [](cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    return cudaEventElapsedTime(&ms, a, b) == cudaSuccess ? (double)ms : 0.0;
  };
  ctx->last_ms[Stage::kTotal] = elapsed(ctx->bev[0], ctx->bev[3]);
  ctx->last_ms[Stage::kTridiag] = elapsed(ctx->bev[1], ctx->bev[2]);
  ctx->last_band_ms = 0.0;
  ctx->last_chase_ms = ctx->last_ms[Stage::kTridiag];
  ctx->last_onestage_ms = elapsed(ctx->bev[1], ctx->bev[4]);
  ctx->last_sb2st_ms = elapsed(ctx->bev[4], ctx->bev[2]);
  ctx->last_ms[Stage::kEig] = elapsed(ctx->bev[2], ctx->bev[3]);
  for (int g : ctx->order) {
    cudaEvent_t* evs = ctx->events.data() + (size_t)g * kGeomEvents;
    for (int k = 1; k < kGeomEvents; ++k) ctx->last_ms[k] += elapsed(evs[k - 1], evs[k]);   // [6]: dense -> band
    ctx->last_band_ms += elapsed(evs[5], evs[6]);
  }
  int first = MBD_OK;
  for (size_t g = 0; g < ctx->geoms.size(); ++g) {
    GeomDev* gd = ctx->geoms[g].get();
    const GeomPlan& p = gd->plan;
    mbd_result& r = out[g];
    r.status = gd->status_host;
    for (int k = 0; k < 3; ++k) r.supercell[k] = p.sl[k];
    r.refine_iters = 0;
    for (int k = 0; k < 3; ++k) r.err_est[k] = 0.0;
    if (gd->status_host != MBD_OK) {
      r.energy_Ha = std::nan("");
      r.c6_mol = std::nan("");
      r.nimag = 0;
      if (first == MBD_OK) first = r.status;
      continue;
    }
    const int N = p.N;
    if (ctx->last_mode != MBD_MODE_PLAIN_FP64) {
      // residual gate of the mixed relay solve; a miss re-runs this geometry
      // with the direct FP64 solve (the plain path) before reading results
      const double* rn = reinterpret_cast<const double*>(host(g, gd->rnorm2));
      double worst = 0.0;
      for (int f = 0; f < 21; ++f) worst = std::max(worst, std::sqrt(rn[f] / (3.0 * N)));
      r.err_est[0] = r.err_est[1] = r.err_est[2] = worst;
      r.refine_iters = kRefineIters;
      if (ctx->last_mode == MBD_MODE_MIXED_LEARNED) {
        const double* cs = reinterpret_cast<const double*>(host(g, gd->cgstate));
        double most = 0.0, most1 = 0.0;
        bool indefinite = false;
        for (int f = 0; f < kNFreq; ++f) {
          most = std::max(most, cs[(size_t)f * kCgState + 1]);
          if (ctx->cg_fp32) most1 = std::max(most1, cs[(size_t)f * kCgState + kCgPhase1Iters]);
          indefinite = indefinite || cs[(size_t)f * kCgState + kCgIndefinite] != 0.0;
        }
        // iterations of both phases (the mixed-precision form) or of the one
        r.refine_iters = (int)(most1 + most);
        // a negative curvature proves the relay matrix indefinite: the direct
        // solve below then reports it (MBD_ERR_RELAY_NOT_SPD)
        if (indefinite) worst = std::numeric_limits<double>::infinity();
        const bool ok = worst <= ctx->residual_gate;
        gd->cg_iters_seen = ok ? (int)most : 0;
        gd->cg_iters_seen1 = ok ? (int)most1 : 0;
      }
      if (!(worst <= ctx->residual_gate)) {
        int st = run_front(ctx, gd, (int)g, MBD_MODE_PLAIN_FP64);
        if (st == MBD_OK) st = run_tail_single(ctx, gd, ctx->slots[gd->slot]->stream);
        if (st != MBD_OK) return st;
        const cudaStream_t ss = ctx->slots[gd->slot]->stream;
        MBD_CUDA(fetch(g, ss));   // the re-run's results replace the staged ones
        MBD_CUDA(cudaStreamSynchronize(ss));
        r.refine_iters = -1;
      }
    }
    const double* aiw = reinterpret_cast<const double*>(host(g, gd->alpha_iw));
    const double* molpol = reinterpret_cast<const double*>(host(g, gd->molpol));
    const double* scal = reinterpret_cast<const double*>(host(g, gd->scalars));
    const double* en = reinterpret_cast<const double*>(host(g, gd->energy));
    const int* info = reinterpret_cast<const int*>(host(g, gd->info));
    int status = MBD_OK;
    for (int f = 0; f < 21; ++f)
      if (info[f] != 0) status = MBD_ERR_RELAY_NOT_SPD;
    if (status == MBD_OK && scal[2] > 0.0) status = MBD_ERR_NONPOSITIVE_ALPHA;
    if (status == MBD_OK && err != 0) status = err;
    r.status = status;
    r.c6_mol = scal[0];
    if (status == MBD_OK) {
      r.energy_Ha = en[0];
      r.nimag = (int)en[2];
    } else {
      r.energy_Ha = std::nan("");
      r.nimag = 0;
    }
    // per-atom results back in the caller's atom order
    const std::vector<int>& pm = gd->plan.perm;
    if (r.alpha_iw)   // column-major alpha(f, i): element (f, i) at f + 21 i
      for (int q = 0; q < N; ++q)
        for (int f = 0; f < 21; ++f) r.alpha_iw[f + 21 * (size_t)pm[q]] = aiw[(size_t)f * N + q];
    if (r.alpha_eff) {
      const double* a = reinterpret_cast<const double*>(host(g, gd->alpha_eff));
      for (int q = 0; q < N; ++q) r.alpha_eff[pm[q]] = a[q];
    }
    if (r.c6_eff) {
      const double* c = reinterpret_cast<const double*>(host(g, gd->c6_eff));
      for (int q = 0; q < N; ++q) r.c6_eff[pm[q]] = c[q];
    }
    if (r.molpol_eig)
      for (int f = 0; f < 21; ++f) {
        double e3[3];
        sym3_eigenvalues_upper(molpol + 9 * f, e3);
        for (int k = 0; k < 3; ++k) r.molpol_eig[f + 21 * k] = e3[k];
      }
    if (status != MBD_OK && first == MBD_OK) first = status;
  }
  return first;
}

int mbd_rsscs_energy_batch(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, int mode, mbd_result* out) {
  if (!ctx || !geoms || !out || n_geom < 1) return MBD_ERR_ARG;
  int st = mbd_rsscs_upload(ctx, n_geom, geoms);
  if (st == MBD_ERR_OUT_OF_MEMORY || st == MBD_ERR_DEVICE || st == MBD_ERR_ARG) {
    for (int g = 0; g < n_geom; ++g) out[g].status = st;
    return st;
  }
  int cs = mbd_rsscs_compute(ctx, mode);
  if (cs != MBD_OK) {
    for (int g = 0; g < n_geom; ++g) out[g].status = cs;
    return cs;
  }
  return mbd_rsscs_download(ctx, out);
}

int mbd_rsscs_energy(mbd_ctx* ctx, const mbd_geom* geom, int mode, mbd_result* out) {
  if (!out) return MBD_ERR_ARG;
  int st = mbd_rsscs_energy_batch(ctx, 1, geom, mode, out);
  out->status = out->status ? out->status : st;
  return out->status;
}

int mbd_rsscs_eigvalsh(mbd_ctx* ctx, const double* H, int n, int ld, double* w) {
  NvtxRange nvtx("mbd_b200 eigvalsh");
  if (!ctx || !H || !w || n < 1 || ld < n) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  const int ldp = round_up(n, 32);
  MBD_CUDA(ctx->eig_a.reserve(sizeof(double) * (size_t)n * ldp));
  MBD_CUDA(ctx->eig_vec.reserve(sizeof(double) * 4 * (size_t)n));   // d, e, ev (2n)
  double* A = ctx->eig_a.as<double>();
  double* d = ctx->eig_vec.as<double>();
  double* e = d + n;
  double* ev = e + n;
  MBD_CUDA(cudaMemcpy2DAsync(A, sizeof(double) * ldp, H, sizeof(double) * ld, sizeof(double) * n, n,
                             cudaMemcpyHostToDevice, s));
  MBD_CUDA(cudaMemsetAsync(ctx->err_flag, 0, sizeof(int), s));
  if (n <= ctx->two_stage_max_n) {
    const size_t wsd = sy2sb_workspace_doubles(n);
    MBD_CUDA(ctx->eig_ws.reserve(sizeof(double) * (wsd + (size_t)n * kBandLd)));
    double* ws = ctx->eig_ws.as<double>();
    double* band = ws + wsd;
    MBD_CUDA(launch_sy2sb(A, ldp, n, ws, band, ctx->num_sms, s, tuned_rows(ctx, n), tuned_panel_qr(ctx, n),
                          lookahead_for(ctx, ctx->la_ctx)));
    int st = band_to_tridiag_single(ctx, band, n, d, e, ctx->fb_ws, s);
    if (st != MBD_OK) return st;
  } else {
    const int G = tridiag_group_ctas(ctx, n);
    const size_t wsb = tridiag_workspace_bytes(n, G);
    MBD_CUDA(ctx->eig_ws.reserve(wsb));
    TridiagJob job{A, n, ldp, d, e};
    MBD_CUDA(cudaMemcpyAsync(ctx->job_dev, &job, sizeof(job), cudaMemcpyHostToDevice, s));
    MBD_CUDA(launch_tridiag(ctx->job_dev, 1, 1, G, ctx->eig_ws.p, wsb, n, ctx->err_flag, s));
  }
  launch_tridiag_eigenvalues(d, e, n, ev, s);
  MBD_CUDA(cudaMemcpyAsync(w, ev, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaStreamSynchronize(s));
  int err = 0;
  MBD_CUDA(cudaMemcpy(&err, ctx->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
  return err ? err : MBD_OK;
}

int mbd_rsscs_eigh(mbd_ctx* ctx, const double* H, int n, int ld, double* w, double* Z, int ldz) {
  NvtxRange nvtx("mbd_b200 eigh");
  if (!ctx || !H || !w || !Z || n < 1 || ld < n || ldz < n) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  constexpr int NBW = 128;   // reflectors per compact-WY block of the back-transformation
  const size_t ldp = round_up(n, 32);
  const size_t nn = (size_t)n * ldp;
  const int G = tridiag_group_ctas(ctx, n);
  const size_t wsb = tridiag_workspace_bytes(n, G);
  MBD_CUDA(ctx->eig_ws.reserve(wsb));
  // A, V (reflectors), X, X2 (vectors), Gram; scratch; W, W2 (NBW x n);
  // S, T (NBW x NBW); tau, d, e, ev (2n); the deviation word
  size_t off = 0;
  std::vector<size_t> o;
  auto add = [&](size_t doubles) { o.push_back(off); off += (doubles + 31) & ~size_t(31); };
  add(nn);
  add(nn);
  add(nn);
  add(nn);
  add((size_t)n * n);
  add(eigh_scratch_doubles(n));
  add((size_t)NBW * n);
  add((size_t)NBW * n);
  add((size_t)NBW * NBW);
  add((size_t)NBW * NBW);
  add(n);
  add(n);
  add(n);
  add(2 * (size_t)n);
  add(4);
  MBD_CUDA(ctx->eigh_buf.reserve(sizeof(double) * off));
  double* base = ctx->eigh_buf.as<double>();
  double* A = base + o[0];
  double* V = base + o[1];
  double* X = base + o[2];
  double* X2 = base + o[3];
  double* Gm = base + o[4];
  double* scratch = base + o[5];
  double* W = base + o[6];
  double* W2 = base + o[7];
  double* Sg = base + o[8];
  double* Tb = base + o[9];
  double* tau = base + o[10];
  double* d = base + o[11];
  double* e = base + o[12];
  double* ev = base + o[13];
  unsigned long long* dev = reinterpret_cast<unsigned long long*>(base + o[14]);
  MBD_CUDA(cudaMemcpy2DAsync(A, sizeof(double) * ldp, H, sizeof(double) * ld, sizeof(double) * n, n,
                             cudaMemcpyHostToDevice, s));
  MBD_CUDA(cudaMemsetAsync(V, 0, sizeof(double) * nn, s));
  MBD_CUDA(cudaMemsetAsync(tau, 0, sizeof(double) * n, s));
  MBD_CUDA(cudaMemsetAsync(e, 0, sizeof(double) * n, s));
  MBD_CUDA(cudaMemsetAsync(ctx->err_flag, 0, sizeof(int), s));
  // A = Q T Q^T, the reflectors of Q kept
  TridiagJob job{A, n, (int)ldp, d, e};
  job.vsave = V;
  job.tau = tau;
  job.ldv = ldp;
  MBD_CUDA(cudaMemcpyAsync(ctx->job_dev, &job, sizeof(job), cudaMemcpyHostToDevice, s));
  MBD_CUDA(launch_tridiag(ctx->job_dev, 1, 1, G, ctx->eig_ws.p, wsb, n, ctx->err_flag, s));
  launch_tridiag_eigenvalues(d, e, n, ev, s);
  double ends[2];
  MBD_CUDA(cudaMemcpyAsync(&ends[0], ev, sizeof(double), cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaMemcpyAsync(&ends[1], ev + n - 1, sizeof(double), cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaStreamSynchronize(s));
  int err = 0;
  MBD_CUDA(cudaMemcpy(&err, ctx->err_flag, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) return err;
  const double tnorm = std::max(std::fabs(ends[0]), std::fabs(ends[1]));
  // the tridiagonal's eigenvectors, then Newton-Schulz to orthonormality
  launch_tri_vectors(d, e, ev, n, tnorm, X, ldp, scratch, s);
  // a step maps a deviation dv of X^T X from I to about 3/4 dv^2: after one
  // from dv <= ns_one the product is not formed again to check it
  const double ns_tol = 1e-15 * std::max(10.0, 4.0 * std::sqrt((double)n));
  const double ns_one = std::sqrt(ns_tol);
  for (int step = 0; step < 4; ++step) {
    dgemm_rm(true, false, n, n, n, 1.0, X, ldp, X, ldp, 0.0, Gm, n, s);   // X^T X
    MBD_CUDA(cudaMemsetAsync(dev, 0, sizeof(unsigned long long), s));
    launch_ns_prepare(Gm, n, dev, s);
    unsigned long long bits = 0;
    MBD_CUDA(cudaMemcpyAsync(&bits, dev, sizeof(bits), cudaMemcpyDeviceToHost, s));
    MBD_CUDA(cudaStreamSynchronize(s));
    double dv;
    std::memcpy(&dv, &bits, sizeof(dv));
    if (!(dv > ns_tol)) break;
    dgemm_rm(false, false, n, n, n, 1.0, X, ldp, Gm, n, 0.0, X2, ldp, s);   // X (3I - X^T X) / 2
    std::swap(X, X2);
    if (dv <= ns_one) break;
  }
  // X <- Q X: blocks of reflectors c0 .. c0 + kb - 1 (rows c0 + 1 .. n - 1),
  // the last block first; V^T of a block is row-major (kb x m) at
  // V + c0 * ldp + c0 + 1
  const int nr = n - 1;
  for (int c0 = nr > 0 ? ((nr - 1) / NBW) * NBW : -1; c0 >= 0; c0 -= NBW) {
    const int kb = std::min(NBW, nr - c0);
    const int m = n - c0 - 1;
    const double* Vt = V + (size_t)c0 * ldp + c0 + 1;
    double* Xs = X + (size_t)(c0 + 1) * ldp;
    dgemm_rm(false, true, kb, kb, m, 1.0, Vt, ldp, Vt, ldp, 0.0, Sg, NBW, s);    // S = V^T V
    launch_wy_t(Sg, tau + c0, kb, NBW, Tb, s);
    dgemm_rm(false, false, kb, n, m, 1.0, Vt, ldp, Xs, ldp, 0.0, W, n, s);       // W = V^T X
    dgemm_rm(false, false, kb, n, kb, 1.0, Tb, NBW, W, n, 0.0, W2, n, s);        // W2 = T W
    dgemm_rm(true, false, m, n, kb, -1.0, Vt, ldp, W2, n, 1.0, Xs, ldp, s);      // X -= V W2
  }
  MBD_CUDA(cudaGetLastError());
  MBD_CUDA(cudaMemcpyAsync(w, ev, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaMemcpy2DAsync(Z, sizeof(double) * ldz, X, sizeof(double) * ldp, sizeof(double) * n, n,
                             cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaStreamSynchronize(s));
  return MBD_OK;
}

int mbd_rsscs_element_z(const char* symbol) { return element_z(symbol); }

int mbd_rsscs_frequency_grid(double* omega, double* weight, int n) {
  if (!omega || n < kNFreq) return MBD_ERR_ARG;
  for (int f = 0; f < kNFreq; ++f) {
    omega[f] = kCasimirOmega[f];
    if (weight) weight[f] = kCasimirWeight[f];
  }
  return MBD_OK;
}

int mbd_rsscs_vdw_params(int z, double* alpha0, double* c6, double* r0) {
  VdwParam v;
  if (!vdw_param(z, &v)) return MBD_ERR_UNKNOWN_ELEMENT;
  if (alpha0) *alpha0 = v.alpha0;
  if (c6) *c6 = v.c6;
  if (r0) *r0 = v.r0;
  return MBD_OK;
}

const char* mbd_rsscs_strerror(int code) {
  switch (code) {
    case MBD_OK: return "ok";
    case MBD_ERR_ARG: return "invalid argument";
    case MBD_ERR_UNKNOWN_ELEMENT: return "VdW parameters not defined for atom";
    case MBD_ERR_RELAY_NOT_SPD: return "relay matrix is not positive definite (Cholesky failed)";
    case MBD_ERR_NONPOSITIVE_ALPHA: return "screened polarizability alpha_eff <= 0; R_vdW_eff undefined";
    case MBD_ERR_EIGENSOLVER: return "diagonalization of CFDM hamiltonian failed";
    case MBD_ERR_DEVICE: return "CUDA device error or no sm_100 device";
    case MBD_ERR_TIMEOUT: return "a bounded device-side wait timed out";
    case MBD_ERR_OUT_OF_MEMORY: return "out of device memory";
    case MBD_ERR_REFINEMENT: return "mixed-precision refinement missed the residual gate; FP64 fallback used";
    case MBD_ERR_NOT_BUILT: return "mode not available in this build";
    case MBD_ERR_TOO_LARGE: return "matrix larger than the fixed scratch of the allocation-free entry point";
    case MBD_ERR_NO_NETWORK: return "MIXED_LEARNED needs a trained or loaded network (or the network switched off)";
    default: return "unknown error";
  }
}

int mbd_rsscs_last_stats(mbd_ctx* ctx, double* out, int n) {
  if (!ctx || !out || n < 3) return MBD_ERR_ARG;
  out[0] = ctx->launches;
  out[1] = ctx->h2d_bytes;
  out[2] = ctx->d2h_bytes;
  if (n >= 4) out[3] = ctx->graph_kind;
  if (n >= 5) {
    double edges = 0.0;
    for (const auto& gd : ctx->geoms) edges += std::max(gd->n_edges, 0);
    out[4] = edges;
  }
  if (n >= 6) out[5] = ctx->graph_updates;
  if (n >= 7) out[6] = ctx->graph_update_result;
  if (n >= 8) out[7] = ctx->graph_update_node;
  return MBD_OK;
}

void* mbd_rsscs_stream(mbd_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int mbd_rsscs_set_option(mbd_ctx* ctx, int option, double value) {
  if (!ctx) return MBD_ERR_ARG;
  switch (option) {
    case MBD_OPT_RESIDUAL_GATE:
      if (!(value >= 0.0)) return MBD_ERR_ARG;
      ctx->residual_gate = value;
      return MBD_OK;
    case MBD_OPT_WAIT_LIMIT_S: {
      if (!(value > 0.0 && value <= 60.0)) return MBD_ERR_ARG;
      // clock64 counts SM cycles: seconds x the device's maximum SM clock
      int khz = 0;
      MBD_CUDA(cudaSetDevice(ctx->device));
      MBD_CUDA(cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, ctx->device));
      const long long cycles = std::max(1LL, (long long)(value * 1e3 * (double)khz));
      MBD_CUDA(cudaDeviceSynchronize());   // no launch of this device reads the limit meanwhile
      MBD_CUDA(set_wait_limit_sb2st(cycles));
      MBD_CUDA(set_wait_limit_tridiag(cycles));
      MBD_CUDA(set_wait_limit_mixed(cycles));
      MBD_CUDA(set_wait_limit_tc3(cycles));
      ctx->wait_limit_s = value;
      return MBD_OK;
    }
    case MBD_OPT_FP32_TENSOR_BUILD: {
      const int on = value != 0.0;
      if (on != ctx->f32_tensor_build) {
        MBD_CUDA(cudaSetDevice(ctx->device));
        MBD_CUDA(cudaDeviceSynchronize());
        drop_graphs(ctx);   // the captured launches carry the old setting
      }
      ctx->f32_tensor_build = on;
      return MBD_OK;
    }
    case MBD_OPT_TEST_STALL_WAIT: {
      const int on = value != 0.0;
      if (on != ctx->test_stall_wait) {
        MBD_CUDA(cudaSetDevice(ctx->device));
        MBD_CUDA(cudaDeviceSynchronize());
        drop_graphs(ctx);   // the captured launches carry the old setting
      }
      ctx->test_stall_wait = on;
      return MBD_OK;
    }
    default:
      return MBD_ERR_ARG;
  }
}

int mbd_rsscs_autotune(mbd_ctx* ctx, int max_n) {
  NvtxRange nvtx("mbd_b200 autotune");
  if (!ctx || max_n < 1) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  MBD_CUDA(cudaDeviceSynchronize());
  return autotune(ctx, max_n);
}

int mbd_rsscs_tuning(mbd_ctx* ctx, double* out, int n) {
  if (!ctx || !out || n < 8 * kTuneClasses) return MBD_ERR_ARG;
  int filled = 0;
  for (int k = 0; k < kTuneClasses; ++k) {
    const TuneChoice& t = ctx->tune[k];
    double* o = out + 8 * k;
    o[0] = t.n;
    o[1] = t.rows;
    o[2] = t.chase_c;
    o[3] = t.sy2sb_ms;
    o[4] = t.chase_ms;
    o[5] = t.panel_qr;
    o[6] = t.flag_chase_ms;
    o[7] = t.cluster_chase_ms;
    if (t.n > 0) filled = k + 1;
  }
  return filled;
}

int mbd_rsscs_get_option(mbd_ctx* ctx, int option, double* value) {
  if (!ctx || !value) return MBD_ERR_ARG;
  switch (option) {
    case MBD_OPT_RESIDUAL_GATE: *value = ctx->residual_gate; return MBD_OK;
    case MBD_OPT_WAIT_LIMIT_S: *value = ctx->wait_limit_s; return MBD_OK;
    case MBD_OPT_TEST_STALL_WAIT: *value = ctx->test_stall_wait; return MBD_OK;
    case MBD_OPT_FP32_TENSOR_BUILD: *value = ctx->f32_tensor_build; return MBD_OK;
    default: return MBD_ERR_ARG;
  }
}

int mbd_rsscs_last_timings(mbd_ctx* ctx, double* ms, int n) {
  if (!ctx || !ms || n < Stage::kCount) return MBD_ERR_ARG;
  for (int k = 0; k < Stage::kCount; ++k) ms[k] = ctx->last_ms[k];
  if (n >= Stage::kCount + 2) {
    ms[Stage::kCount] = ctx->last_band_ms;        // dense -> band, summed over geometries
    ms[Stage::kCount + 1] = ctx->last_chase_ms;   // band (or dense, one-stage) -> tridiagonal, batch-wide
  }
  if (n >= Stage::kCount + 4) {
    ms[Stage::kCount + 2] = ctx->last_onestage_ms;   // the grouped one-stage launch alone
    ms[Stage::kCount + 3] = ctx->last_sb2st_ms;      // the bulge-chasing launch alone
  }
  return MBD_OK;
}

}  // extern "C"
