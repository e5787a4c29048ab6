// MIXED_LEARNED relay solve and the training of its network.
//
// The relay system A(iw) X = [I3; ...; I3] of every frequency (the solve of
// get_screened_alpha, UTILS.f90:469-473) is solved by block conjugate
// gradients (k_cg.cu) started from a network's prediction of each atom's 3x3
// screened-polarizability block X_i (k_gnn.cu).  The network is trained here,
// on the GPU, on relay solutions that the plain direct solve produces for a
// training set of geometries.  A frequency whose final residual misses the
// gate is re-solved directly at download (the plain path), as in MIXED.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "context.h"
#include "tc3.h"

namespace mbd {
namespace {

constexpr int kCgMaxIters = 64;
constexpr int kCgSlack = 4;       // iterations a captured graph adds to the count last seen
constexpr double kCgTol = 3e-11;   // relative residual the iteration stops at (gate: 1e-10)
// Mixed-precision form (the matrix passes on the FP32 copy of the relay
// matrices): phase 1 from the warm start to a relative residual of
// kCgTol1, a restart from the true FP64 residual, phase 2 to kCgTol.  Each
// phase's FP32 passes perturb only the correction it computes: phase 2 starts
// from a residual ~1e-5 of B, and the FP32 rounding of the matrix (~6e-8
// relative) then leaves ~1e-12 in the final residual, far below the gate.
constexpr int kCgPhaseMaxIters = 40;
constexpr double kCgTol1 = 1e-5;

// Image range and bounding box of the network's neighbour lists (within the
// cut-off, including periodic images along non-vacuum axes: an atom may meet
// another atom, or itself, through several images).  The lists are
// symmetric: edge (i, j + t) implies (j, i - t).
GraphBox graph_box(const GeomPlan& p) {
  GraphBox b{};
  const double rc = kGnnCutoffBohr;
  for (int k = 0; k < 9; ++k) b.lat[k] = p.lat[k];
  if (p.n_periodic != 0) {
    // images up to the cut-off plus a cell: widths from |a_k| lower-bound nothing,
    // so use the perpendicular width V / |a_i x a_j|
    const double* a = p.lat;
    auto cross = [](const double* u, const double* v, double* w) {
      w[0] = u[1] * v[2] - u[2] * v[1];
      w[1] = u[2] * v[0] - u[0] * v[2];
      w[2] = u[0] * v[1] - u[1] * v[0];
    };
    double c12[3], c20[3], c01[3];
    cross(a + 3, a + 6, c12);
    cross(a + 6, a + 0, c20);
    cross(a + 0, a + 3, c01);
    const double vol = std::fabs(a[0] * c12[0] + a[1] * c12[1] + a[2] * c12[2]);
    const double* cs[3] = {c12, c20, c01};
    for (int k = 0; k < 3; ++k) {
      if (p.vac[k]) continue;
      const double area = std::sqrt(cs[k][0] * cs[k][0] + cs[k][1] * cs[k][1] + cs[k][2] * cs[k][2]);
      const double width = vol > 0.0 ? vol / area : 0.0;
      b.rng[k] = width > 0.0 ? (int)std::ceil(rc / width) + 1 : 0;
    }
  }
  for (int c = 0; c < 3; ++c) {
    b.lo[c] = 1e300;
    b.hi[c] = -1e300;
  }
  for (int i = 0; i < p.N; ++i)
    for (int c = 0; c < 3; ++c) {
      b.lo[c] = std::min(b.lo[c], p.coords[3 * i + c]);
      b.hi[c] = std::max(b.hi[c], p.coords[3 * i + c]);
    }
  b.pad = rc + 1e-6;   // far above the rounding of |coordinates| <= 1e6 bohr
  b.rc2 = rc * rc;
  return b;
}

// The network graphs of `todo`, built on the GPU: every geometry's edge
// counts and offsets, one synchronisation to size the graph buffers, then the
// lists.  Device copy of a graph: [off | nbr | src | species] ints,
// [dvec | efeat | eproj] floats.
int build_graphs(mbd_ctx* ctx, const std::vector<GeomDev*>& todo, cudaStream_t s) {
  NvtxRange nvtx("mbd_b200 network neighbour lists");
  if (todo.empty()) return MBD_OK;
  const size_t K = todo.size();
  auto pad64 = [](size_t k) { return (k + 63) & ~size_t(63); };
  size_t total = pad64(K);
  for (GeomDev* gd : todo) total += pad64((size_t)gd->plan.N + 1);
  MBD_CUDA(ctx->graph_scan.reserve(sizeof(int) * total));
  int* Ed = ctx->graph_scan.as<int>();
  std::vector<int*> offs(K);
  std::vector<GraphBox> boxes(K);
  size_t o = pad64(K);
  for (size_t k = 0; k < K; ++k) {
    GeomDev* gd = todo[k];
    offs[k] = Ed + o;
    o += pad64((size_t)gd->plan.N + 1);
    boxes[k] = graph_box(gd->plan);
    gnn_graph_count(gd->coords, gd->plan.N, boxes[k], offs[k], s);
    gnn_graph_scan(offs[k], gd->plan.N, Ed + k, s);
  }
  std::vector<int> Eh(K);
  MBD_CUDA(cudaMemcpyAsync(Eh.data(), Ed, sizeof(int) * K, cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaStreamSynchronize(s));
  for (size_t k = 0; k < K; ++k) {
    GeomDev* gd = todo[k];
    const GeomPlan& p = gd->plan;
    const int N = p.N, E = Eh[k];
    if (E < 0) return MBD_ERR_DEVICE;
    const size_t b_off = bytes_of<int>(N + 1), b_e = bytes_of<int>(std::max(E, 1)), b_sp = bytes_of<int>(N);
    const size_t b_dv = bytes_of<float>(3 * (size_t)std::max(E, 1)), b_ef = bytes_of<float>(kGnnRbf * (size_t)std::max(E, 1));
    const size_t b_ep = bytes_of<float>(6 * (size_t)std::max(E, 1));
    MBD_CUDA(gd->graph.reserve(b_off + 2 * b_e + b_sp + b_dv + b_ef + b_ep));
    char* base = gd->graph.as<char>();
    int* off = reinterpret_cast<int*>(base);
    int* nbr = reinterpret_cast<int*>(base + b_off);
    int* src = reinterpret_cast<int*>(base + b_off + b_e);
    int* species = reinterpret_cast<int*>(base + b_off + 2 * b_e);
    float* dv = reinterpret_cast<float*>(base + b_off + 2 * b_e + b_sp);
    float* ef = reinterpret_cast<float*>(base + b_off + 2 * b_e + b_sp + b_dv);
    float* ep = reinterpret_cast<float*>(base + b_off + 2 * b_e + b_sp + b_dv + b_ef);
    MBD_CUDA(cudaMemcpyAsync(species, p.species.data(), sizeof(int) * N, cudaMemcpyHostToDevice, s));
    ctx->h2d_bytes += (double)sizeof(int) * N;
    gnn_graph_fill(gd->coords, N, boxes[k], offs[k], off, nbr, src, dv, s);
    gnn_edges(dv, E, ef, ep, s);
    ctx->launches += 3 + (E > 0 ? 1 : 0);
    GnnGraph& g = gd->gnn;
    g.N = N;
    g.F = kNFreq;
    g.E = E;
    g.off = off;
    g.nbr = nbr;
    g.src = src;
    g.efeat = ef;
    g.eproj = ep;
    g.x = nullptr;
    gd->n_edges = E;
  }
  return cuda_status(cudaGetLastError());
}

const int* graph_species(const GeomDev* gd) {
  const int N = gd->plan.N;
  const int E = std::max(gd->n_edges, 1);
  return reinterpret_cast<const int*>(gd->graph.as<char>() + bytes_of<int>(N + 1) + 2 * bytes_of<int>(E));
}

size_t cg_doubles(const GeomPlan& p) {
  const size_t ys = (size_t)p.n * 3;
  return cg_minv_doubles(p.n, kNFreq) + 5 * kNFreq * ys + cg_partial_doubles(p.n, kNFreq) +
         2 * cg_red_doubles(p.n, kNFreq) + 64;
}

// Deterministic parameter initialisation (splitmix64 + Box-Muller): weights
// N(0, 1/fan_in), readout vectors zero, wg N(0, 0.01), biases zero.
void init_params(std::vector<float>& P, uint64_t seed) {
  P.assign(kGnnParams, 0.0f);
  uint64_t st = seed * 0x9E3779B97F4A7C15ull + 1;
  auto next = [&]() {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return ((z >> 11) + 0.5) * (1.0 / 9007199254740992.0);
  };
  auto normal = [&]() { return std::sqrt(-2.0 * std::log(next())) * std::cos(2.0 * kPi * next()); };
  auto fill = [&](int off, int rows, int cols, double sd) {
    for (int k = 0; k < rows * cols; ++k) P[off + k] = (float)(normal() * sd);
  };
  fill(kGnnOffW0, kGnnHidden, kGnnIn, std::sqrt(1.0 / kGnnIn));
  for (int l = 0; l < kGnnLayers; ++l) {
    fill(kGnnOffWf(l), kGnnHidden, kGnnRbf, std::sqrt(1.0 / kGnnRbf));
    fill(kGnnOffWu(l), kGnnHidden, kGnnHidden, std::sqrt(1.0 / kGnnHidden));
  }
  fill(kGnnOffWg, 1, kGnnRbf, 0.1);
}

int reserve_params(mbd_ctx* ctx) {
  const size_t b = sizeof(float) * kGnnParams;
  if (ctx->gnn_params.bytes < b) {
    MBD_CUDA(ctx->gnn_params.reserve(b));
    MBD_CUDA(ctx->gnn_grad.reserve(b));
    MBD_CUDA(ctx->gnn_m1.reserve(b));
    MBD_CUDA(ctx->gnn_m2.reserve(b));
  }
  return MBD_OK;
}

}  // namespace

// Per-slot CG and network buffers and every geometry's graph.
int reserve_learned(mbd_ctx* ctx) {
  {
    std::vector<GeomDev*> todo;
    for (int g : ctx->order)
      if (ctx->geoms[g]->n_edges < 0) todo.push_back(ctx->geoms[g].get());
    int st = build_graphs(ctx, todo, ctx->stream);
    if (st != MBD_OK) return st;
  }
  bool moved = false;
  {
    // the FP32 copy of the relay matrices for the two-phase block-CG: per
    // slot n x ld x 21 floats of its largest geometry
    bool fp32 = ctx->cg_fp32_mode == 1;
    if (ctx->cg_fp32_mode < 0) {
      size_t need = 0, held = 0, free_b = 0, total_b = 0;
      for (int s = 0; s < ctx->n_slots; ++s) {
        size_t r32 = 0;
        for (int g : ctx->order)
          if (ctx->geoms[g]->slot == s)
            r32 = std::max(r32, sizeof(float) * (size_t)kNFreq * ctx->geoms[g]->plan.n * ctx->geoms[g]->plan.ld);
        need += r32;
        held += ctx->slots[s]->relay32.bytes;
      }
      MBD_CUDA(cudaMemGetInfo(&free_b, &total_b));
      fp32 = (double)need <= 0.5 * (double)(free_b + held);
    }
    moved = fp32 != ctx->cg_fp32;   // the captured launches carry the choice
    ctx->cg_fp32 = fp32;
  }
  for (int s = 0; s < ctx->n_slots; ++s) {
    size_t cg = 0, gw = 0, res = 0;
    for (int g : ctx->order) {
      GeomDev* gd = ctx->geoms[g].get();
      if (gd->slot != s) continue;
      const GeomPlan& p = gd->plan;
      cg = std::max(cg, sizeof(double) * cg_doubles(p));
      gw = std::max(gw, sizeof(float) * (gnn_work_floats(p.N, kNFreq, gd->n_edges, false) +
                                         (size_t)kNFreq * p.N * kGnnIn + 64));
      res = std::max(res, sizeof(double) * relay_residual_ws_doubles(p.n, kNFreq));
    }
    RelaySlot& sl = *ctx->slots[s];
    moved = moved || cg > sl.cg.bytes || gw > sl.gnn.bytes || res > sl.res_ws.bytes;
    MBD_CUDA(sl.cg.reserve(cg));
    MBD_CUDA(sl.gnn.reserve(gw));
    MBD_CUDA(sl.res_ws.reserve(res));
    if (ctx->cg_fp32) {
      // the FP32 copy of the relay matrices the mixed-precision passes read
      size_t r32 = 0;
      for (int g : ctx->order)
        if (ctx->geoms[g]->slot == s) r32 = std::max(r32, sizeof(float) * (size_t)kNFreq * ctx->geoms[g]->plan.n *
                                                              ctx->geoms[g]->plan.ld);
      moved = moved || r32 > sl.relay32.bytes;
      MBD_CUDA(sl.relay32.reserve(r32));
    }
  }
  if (moved) drop_graphs(ctx);
  return MBD_OK;
}

// Learned relay solve of one geometry on its slot's stream; *X_out = the
// solution (n x 3 per frequency) in the slot's CG buffer.
int relay_learned(mbd_ctx* ctx, GeomDev* gd, RelaySlot& sl, size_t mstride, cudaEvent_t ev_net, double** X_out) {
  const GeomPlan& p = gd->plan;
  cudaStream_t s = sl.stream;
  const int n = p.n, N = p.N;
  const size_t ys = (size_t)n * 3;
  double* base = sl.cg.as<double>();
  CgArgs a{};
  a.A = sl.relay64.as<double>();
  a.A32 = ctx->cg_fp32 ? sl.relay32.as<float>() : nullptr;
  a.a_stride = mstride;
  a.ld = p.ld;
  a.n = n;
  a.N = N;
  a.nt = (n + 63) / 64;
  a.batch = kNFreq;
  a.Minv = base;   // first: its 16-byte loads need the buffer's alignment
  a.X = a.Minv + cg_minv_doubles(n, kNFreq);
  a.R = a.X + kNFreq * ys;
  a.Z = a.R + kNFreq * ys;
  a.P = a.Z + kNFreq * ys;
  a.Q = a.P + kNFreq * ys;
  a.ystride = ys;
  a.partial = a.Q + kNFreq * ys;
  a.red = a.partial + cg_partial_doubles(n, kNFreq);
  a.red2 = a.red + cg_red_doubles(n, kNFreq);
  a.state = gd->cgstate;
  a.tol2 = kCgTol * kCgTol * 3.0 * N;
  // start: the network's prediction, or zero
  if (ctx->use_net) {
    float* w = sl.gnn.as<float>();
    float* x = w;
    float* work = w + (((size_t)kNFreq * N * kGnnIn + 63) & ~size_t(63));
    gnn_features(graph_species(gd), gd->hirsh, gd->alpha_w, ctx->omega_dev, N, kNFreq, x, s);
    GnnGraph g = gd->gnn;
    g.x = x;
    const GnnWork wk = gnn_work_layout(work, N, kNFreq, gd->n_edges, false);
    ctx->launches += 1 + gnn_forward(ctx->gnn_params.as<float>(), g, wk, s);
    gnn_warmstart(wk.S, gd->alpha_w, N, kNFreq, a.X, ys, s);
    ctx->launches += 1;
  } else {
    MBD_CUDA(cudaMemsetAsync(a.X, 0, sizeof(double) * kNFreq * ys, s));
  }
  record_timing(ctx, ev_net, s);
  // the full schedule, or in a captured graph the iterations this geometry
  // took on its last compute plus a margin
  // MBD_B200_CG_PREDICT=0: captured graphs keep the full schedule too
  static const bool predict = [] {
    const char* e = std::getenv("MBD_B200_CG_PREDICT");
    return !(e && e[0] == '0');
  }();
  auto sched = [&](int seen, int cap) {
    return (predict && ctx->capturing && seen > 0) ? std::min(cap, seen + kCgSlack) : cap;
  };
  if (a.A32) {
    const double tol2 = a.tol2;
    a.tol2 = kCgTol1 * kCgTol1 * 3.0 * N;
    launch_cg_setup(a, s);
    const int it1 = sched(gd->cg_iters_seen1, kCgPhaseMaxIters);
    for (int it = 0; it < it1; ++it) launch_cg_iteration(a, it, s, true);
    a.tol2 = tol2;
    launch_cg_restart(a, s);
    const int it2 = sched(gd->cg_iters_seen, kCgPhaseMaxIters);
    for (int it = 0; it < it2; ++it) launch_cg_iteration(a, it, s, true);
    ctx->launches += 5 + 5 + 4 * (it1 + it2);
  } else {
    launch_cg_setup(a, s);
    const int iters = sched(gd->cg_iters_seen, kCgMaxIters);
    for (int it = 0; it < iters; ++it) launch_cg_iteration(a, it, s);
    ctx->launches += 5 + 4 * iters;
  }
  // the gate's residual, recomputed from X: R = B - A X
  launch_relay_residual(sl.relay64.as<double>(), mstride, p.ld, n, kNFreq, a.X, nullptr, a.R, ys,
                        sl.res_ws.as<double>(), gd->rnorm2, s);
  ctx->launches += 3;
  *X_out = a.X;
  return cuda_status(cudaGetLastError());
}

}  // namespace mbd

using namespace mbd;

extern "C" {

int mbd_rsscs_learned_param_count(void) { return kGnnParams; }

int mbd_rsscs_learned_set_params(mbd_ctx* ctx, const float* params, int n) {
  if (!ctx || !params || n != kGnnParams) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  int st = reserve_params(ctx);
  if (st != MBD_OK) return st;
  MBD_CUDA(h2d_ordered(ctx, ctx->gnn_params.p, params, sizeof(float) * kGnnParams));
  drop_graphs(ctx);
  ctx->have_net = true;
  return MBD_OK;
}

int mbd_rsscs_learned_get_params(mbd_ctx* ctx, float* params, int n) {
  if (!ctx || !params || n != kGnnParams) return MBD_ERR_ARG;
  if (!ctx->have_net) return MBD_ERR_NO_NETWORK;
  MBD_CUDA(cudaSetDevice(ctx->device));
  MBD_CUDA(cudaMemcpy(params, ctx->gnn_params.p, sizeof(float) * kGnnParams, cudaMemcpyDeviceToHost));
  return MBD_OK;
}

int mbd_rsscs_learned_use_network(mbd_ctx* ctx, int on) {
  if (!ctx) return MBD_ERR_ARG;
  if (ctx->use_net != (on != 0)) drop_graphs(ctx);
  ctx->use_net = on != 0;
  return MBD_OK;
}

int mbd_rsscs_learned_train(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, int epochs, double lr, int seed,
                            double* epoch_loss) {
  NvtxRange nvtx("mbd_b200 learned train");
  if (!ctx || !geoms || n_geom < 1 || epochs < 1 || !(lr > 0.0)) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  int st = upload_batch(ctx, n_geom, geoms, false);
  if (st == MBD_ERR_OUT_OF_MEMORY || st == MBD_ERR_DEVICE || st == MBD_ERR_ARG) return st;
  if (ctx->order.empty()) return st != MBD_OK ? st : MBD_ERR_ARG;
  st = reserve_learned(ctx);
  if (st != MBD_OK) return st;
  st = reserve_params(ctx);
  if (st != MBD_OK) return st;
  // training targets: direct FP64 relay solutions of every geometry
  size_t work = 0;
  for (int g : ctx->order) {
    GeomDev* gd = ctx->geoms[g].get();
    const GeomPlan& p = gd->plan;
    MBD_CUDA(gd->train.reserve(sizeof(float) * (size_t)kNFreq * p.N * (kGnnIn + 9) + 256));
    work = std::max(work, gnn_work_floats(p.N, kNFreq, gd->n_edges, true));
  }
  MBD_CUDA(ctx->gnn_train_work.reserve(sizeof(float) * work));
  MBD_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->launches = 0;
  for (int g : ctx->order) {
    GeomDev* gd = ctx->geoms[g].get();
    const GeomPlan& p = gd->plan;
    RelaySlot& sl = *ctx->slots[gd->slot];
    st = run_front(ctx, gd, g, MBD_MODE_PLAIN_FP64, true);
    if (st != MBD_OK) return st;
    const size_t ys = (size_t)p.n * 3;
    const double* X = sl.rhs.as<double>() + 2 * kNFreq * ys;
    float* x = gd->train.as<float>();
    float* St = x + (size_t)kNFreq * p.N * kGnnIn;
    gnn_features(graph_species(gd), gd->hirsh, gd->alpha_w, ctx->omega_dev, p.N, kNFreq, x, sl.stream);
    gnn_targets(X, ys, gd->alpha_w, p.N, kNFreq, St, sl.stream);
  }
  MBD_CUDA(cudaDeviceSynchronize());
  {
    int info_bad = 0;
    for (int g : ctx->order) {
      int info[32];
      MBD_CUDA(cudaMemcpy(info, ctx->geoms[g]->info, sizeof(info), cudaMemcpyDeviceToHost));
      for (int f = 0; f < kNFreq; ++f) info_bad |= info[f] != 0;
    }
    if (info_bad) return MBD_ERR_RELAY_NOT_SPD;
  }
  // Adam over the geometries (one geometry = one step), shuffled every epoch
  std::vector<float> P0;
  init_params(P0, (uint64_t)seed);
  cudaStream_t s = ctx->stream;
  float* P = ctx->gnn_params.as<float>();
  float* G = ctx->gnn_grad.as<float>();
  MBD_CUDA(h2d_ordered(ctx, P, P0.data(), sizeof(float) * kGnnParams));
  MBD_CUDA(zero_ordered(ctx, G, sizeof(float) * kGnnParams));
  MBD_CUDA(zero_ordered(ctx, ctx->gnn_m1.p, sizeof(float) * kGnnParams));
  MBD_CUDA(zero_ordered(ctx, ctx->gnn_m2.p, sizeof(float) * kGnnParams));
  std::vector<int> order = ctx->order;
  uint64_t rs = (uint64_t)seed * 6364136223846793005ull + 1442695040888963407ull;
  int step = 0;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int k = (int)order.size() - 1; k > 0; --k) {
      rs = rs * 6364136223846793005ull + 1442695040888963407ull;
      std::swap(order[k], order[(int)((rs >> 33) % (uint64_t)(k + 1))]);
    }
    MBD_CUDA(cudaMemsetAsync(ctx->loss_dev, 0, sizeof(double), s));
    for (int g : order) {
      GeomDev* gd = ctx->geoms[g].get();
      const GeomPlan& p = gd->plan;
      GnnGraph gg = gd->gnn;
      gg.x = gd->train.as<float>();
      GnnWork w = gnn_work_layout(ctx->gnn_train_work.as<float>(), p.N, kNFreq, gd->n_edges, true);
      w.S_true = gd->train.as<float>() + (size_t)kNFreq * p.N * kGnnIn;
      gnn_forward(P, gg, w, s);
      gnn_loss_backward(P, gg, w, G, ctx->loss_dev, s);
      gnn_adam(P, G, ctx->gnn_m1.as<float>(), ctx->gnn_m2.as<float>(), ++step, (float)lr, s);
    }
    double loss = 0.0;
    MBD_CUDA(cudaMemcpyAsync(&loss, ctx->loss_dev, sizeof(double), cudaMemcpyDeviceToHost, s));
    MBD_CUDA(cudaStreamSynchronize(s));
    if (epoch_loss) epoch_loss[ep] = loss / (double)order.size();
    if (!std::isfinite(loss)) {
      ctx->have_net = false;
      return MBD_ERR_NO_NETWORK;   // training diverged: no usable network
    }
  }
  ctx->have_net = true;
  drop_graphs(ctx);
  return MBD_OK;
}

// Forward pass, loss and gradient of the network on caller-given inputs
// (host arrays; a check of the kernels against a CPU restatement).  Leaves
// the context's own network untouched.
int mbd_rsscs_learned_eval(mbd_ctx* ctx, const float* params, int n_atoms, int n_freq, const int* off,
                           const int* nbr, const float* dvec, const float* x, const float* S_true, float* S_pred,
                           float* grad, double* loss) {
  if (!ctx || !params || n_atoms < 1 || n_freq < 1 || !off || !x || !S_pred) return MBD_ERR_ARG;
  MBD_CUDA(cudaSetDevice(ctx->device));
  const int N = n_atoms, F = n_freq, E = off[N];
  if (E < 0 || (E > 0 && (!nbr || !dvec))) return MBD_ERR_ARG;
  std::vector<int> src(std::max(E, 1), 0);
  for (int i = 0; i < N; ++i)
    for (int e = off[i]; e < off[i + 1]; ++e) {
      if (e < 0 || e >= E || nbr[e] < 0 || nbr[e] >= N) return MBD_ERR_ARG;
      src[e] = i;
    }
  const size_t M = (size_t)N * F;
  const int Ep = std::max(E, 1);
  const size_t fl = kGnnParams + kGnnParams + M * kGnnIn + 9 * M + (size_t)Ep * (3 + kGnnRbf + 6) +
                    gnn_work_floats(N, F, E, true) + 1024;
  const size_t il = (size_t)(N + 1) + 2 * (size_t)Ep + 64;
  MBD_CUDA(ctx->gnn_eval.reserve(sizeof(float) * fl + sizeof(int) * il + 4096));
  float* f = ctx->gnn_eval.as<float>();
  auto takef = [&](size_t k) {
    float* q = f;
    f += (k + 63) & ~size_t(63);
    return q;
  };
  float* P = takef(kGnnParams);
  float* G = takef(kGnnParams);
  float* xd = takef(M * kGnnIn);
  float* St = takef(9 * M);
  float* dv = takef(3 * (size_t)Ep);
  float* ef = takef(kGnnRbf * (size_t)Ep);
  float* epj = takef(6 * (size_t)Ep);
  float* work = takef(gnn_work_floats(N, F, E, true));
  int* ib = reinterpret_cast<int*>(f);
  int* d_off = ib;
  int* d_nbr = ib + ((N + 1 + 63) & ~63);
  int* d_src = d_nbr + ((Ep + 63) & ~63);
  double* d_loss = ctx->loss_dev;
  cudaStream_t s = ctx->stream;
  MBD_CUDA(cudaMemcpyAsync(P, params, sizeof(float) * kGnnParams, cudaMemcpyHostToDevice, s));
  MBD_CUDA(cudaMemsetAsync(G, 0, sizeof(float) * kGnnParams, s));
  MBD_CUDA(cudaMemcpyAsync(xd, x, sizeof(float) * M * kGnnIn, cudaMemcpyHostToDevice, s));
  MBD_CUDA(cudaMemcpyAsync(d_off, off, sizeof(int) * (N + 1), cudaMemcpyHostToDevice, s));
  if (E > 0) {
    MBD_CUDA(cudaMemcpyAsync(d_nbr, nbr, sizeof(int) * E, cudaMemcpyHostToDevice, s));
    MBD_CUDA(cudaMemcpyAsync(d_src, src.data(), sizeof(int) * E, cudaMemcpyHostToDevice, s));
    MBD_CUDA(cudaMemcpyAsync(dv, dvec, sizeof(float) * 3 * E, cudaMemcpyHostToDevice, s));
  }
  gnn_edges(dv, E, ef, epj, s);
  GnnGraph g{N, F, E, d_off, d_nbr, d_src, ef, epj, xd};
  GnnWork w = gnn_work_layout(work, N, F, E, true);
  w.S_true = St;
  gnn_forward(P, g, w, s);
  if (S_true && grad) {
    MBD_CUDA(cudaMemcpyAsync(St, S_true, sizeof(float) * 9 * M, cudaMemcpyHostToDevice, s));
    MBD_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(double), s));
    gnn_loss_backward(P, g, w, G, d_loss, s);
    MBD_CUDA(cudaMemcpyAsync(grad, G, sizeof(float) * kGnnParams, cudaMemcpyDeviceToHost, s));
    if (loss) MBD_CUDA(cudaMemcpyAsync(loss, d_loss, sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  MBD_CUDA(cudaMemcpyAsync(S_pred, w.S, sizeof(float) * 9 * M, cudaMemcpyDeviceToHost, s));
  MBD_CUDA(cudaStreamSynchronize(s));
  return cuda_status(cudaGetLastError());
}

}  // extern "C"
