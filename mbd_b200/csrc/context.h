// Context and per-geometry device state shared by the C ABI (api.cpp) and
// the learned relay path (learn.cpp).
#pragma once

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <memory>
#include <vector>

#include "gnn.h"
#include "kernels.h"
#include "mbd_internal.h"

namespace mbd {

// NVTX range over one scope of host code (upload, compute, capture, the
// enqueue of one geometry, download, ...): a profiler that records NVTX shows
// where the host time of a call goes; without one the calls return at once
// (NVTX v3 is header-only and loads a tool's library only when one is
// attached).
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Refinement sweeps of the mixed relay solve and the residual gate
// ||B - A X||_F / ||B||_F that accepts its result.
constexpr int kRefineIters = 4;
constexpr double kResidualGate = 1e-10;
// Relay slots (streams with private relay workspaces) of one context.
constexpr int kMaxSlots = 8;
// Share of free device memory the relay slots of one batch may plan for.
constexpr double kSlotMemoryShare = 0.7;

// Raw device allocation owned by the context (grow-only).
struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t reserve(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMalloc(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

// Page-locked host memory (the download's staging area).
struct HostBuf {
  void* p = nullptr;
  size_t bytes = 0;
  ~HostBuf() {
    if (p) cudaFreeHost(p);
  }
  cudaError_t reserve(size_t b) {
    if (b <= bytes) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&p, b);
    if (e == cudaSuccess) bytes = b;
    return e;
  }
  template <class T>
  T* as() const { return static_cast<T*>(p); }
};

// Per-geometry device state that must survive until download.
struct GeomDev {
  GeomPlan plan;
  DevBuf inputs;     // coords, alpha0, c6free, r0, hirsh, shifts, diff data
  DevBuf results;    // alpha_w, sgm, rvdw_iso, alpha_iw, molpol, c6_eff, alpha_eff, omega, rvdw_eff, scalars, energy, info, d, e, ev
  DevBuf hmat;       // CFDM Hamiltonian (nH x ldH, lower blocks), reduced in place
  DevBuf band;       // two-stage reduction: the band, nH x kBandLd
  // offsets into inputs (doubles unless noted)
  const double *coords, *alpha0, *c6free, *r0, *hirsh, *scs_shifts, *cfdm_shifts, *diff_shift;
  const int *diff_is_zero, *place_offset, *place_rc, *place_cc;
  // results
  double *alpha_w, *sgm, *rvdw_iso, *alpha_iw, *molpol, *c6_eff, *alpha_eff, *omega, *rvdw_eff;
  double *scalars, *energy, *d, *e, *ev, *rnorm2;
  double* cgstate;   // [21][kCgState] block-CG recurrence state (MIXED_LEARNED)
  int* info;
  int status_host = MBD_OK;
  int slot = 0;      // relay slot running this geometry's relay and CFDM stages
  // learned warm start: neighbour graph (built on first use), training data
  DevBuf graph;      // off, nbr, src, species (int); dvec, efeat, eproj (float)
  int n_edges = -1;  // -1 until the graph is built
  // Block-CG iterations (max over frequencies) of this geometry's last
  // MIXED_LEARNED compute, as read back by download; 0: unknown.  A captured
  // graph runs this many iterations plus a margin instead of the full
  // schedule (the same inputs and network converge identically; a miss
  // would still be caught by the residual gate).  Forgotten with the graphs.
  int cg_iters_seen = 0;    // block-CG iterations of the last compute (the second phase when two-phase)
  int cg_iters_seen1 = 0;   // the first phase's (mixed-precision block-CG)
  GnnGraph gnn{};    // device views into `graph` (x set per use)
  DevBuf train;      // x [21N][8] and S_true [21N][9] of a training batch
};

// One relay slot: a stream and the relay workspaces of the geometries it runs
// (sized for the largest of them).
struct RelaySlot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  Sy2sbLookAhead la{};   // the dense -> band look-ahead's stream and events
  DevBuf relay64, linv, rhs;                                  // plain FP64 path
  DevBuf relay32, p_hi, p_lo, l_hi, l_lo, mixv, res_ws, solve_sync;   // mixed path
  DevBuf cg, gnn;                                             // learned path: CG vectors, network work
  DevBuf trd_ws;                                              // dense -> band workspace
  int solve_epoch = 0;
  ~RelaySlot() {
    if (done) cudaEventDestroy(done);
    if (la.ready) cudaEventDestroy(la.ready);
    if (la.done) cudaEventDestroy(la.done);
    if (la.aux) cudaStreamDestroy(la.aux);
    if (stream) cudaStreamDestroy(stream);
  }
  size_t held() const {
    return relay64.bytes + linv.bytes + rhs.bytes + relay32.bytes + p_hi.bytes + p_lo.bytes + l_hi.bytes +
           l_lo.bytes + mixv.bytes + res_ws.bytes + solve_sync.bytes + cg.bytes + gnn.bytes + trd_ws.bytes;
  }
};

// Autotuned launch shapes of the eigen stages per size class n <= 512 * 2^k
// (tune.cu); 0 = not tuned (the defaults apply).
constexpr int kTuneClasses = 8;
struct TuneChoice {
  int n = 0;            // size the class was timed at
  int rows = 0;         // panel-QR rows per CTA of the dense -> band reduction
  int panel_qr = -1;    // panel QR: 0 per-column Householder, 1 TSQR (-1: not tuned)
  int chase_c = -1;     // band -> tridiagonal: CTAs of the cluster-resident chase
                        // (0: its default size), or kChaseFlag (-1): the flag-synchronised chase
  double sy2sb_ms = 0.0, chase_ms = 0.0;   // the chosen candidates' times
  double flag_chase_ms = 0.0, cluster_chase_ms = 0.0;   // the best of each chase kernel
};
constexpr int kChaseFlag = -1;

struct Stage {
  enum { kTotal = 0, kSetup, kBuild, kFactor, kSolve, kCfdm, kTridiag, kEig, kCount };
};
// Events per geometry: start, then the ends of setup, build, factor, solve,
// CFDM build and dense -> band reduction.
constexpr int kGeomEvents = 7;



}  // namespace mbd

struct mbd_ctx {
  int device = 0;
  int num_sms = 0;
  int trd_ctas_per_sm = 1;
  cudaStream_t stream = nullptr;             // batch stream: tridiagonal reduction, eigenvalues, energies
  std::vector<std::unique_ptr<mbd::GeomDev>> geoms;
  std::vector<std::unique_ptr<mbd::RelaySlot>> slots;
  int n_slots = 0;                           // slots in use for the current batch
  mbd::DevBuf tridiag_ws, tables, misc, fb_ws;
  mbd::HostBuf staging;   // download: every geometry's results in one pass
  mbd::Sy2sbLookAhead la_ctx{};   // look-ahead stream and events of the context-stream reductions
  bool lookahead = true;     // dense -> band look-ahead (MBD_B200_LOOKAHEAD=0: off)
  bool priorities = true;    // stream and graph-node priorities (MBD_B200_PRIORITY=0: off)
  // standalone eigenvalue call: matrix, (d, e, eigenvalues, scratch), workspace
  mbd::DevBuf eig_a, eig_vec, eig_ws;
  mbd::DevBuf eigh_buf;   // mbd_rsscs_eigh: matrix, reflectors, vectors, Gram, scratch
  // batch plan (device tables in `tables`)
  mbd::TridiagJob* trd_jobs = nullptr;
  mbd::TridiagGroup* trd_groups = nullptr;
  mbd::EigJob* eig_jobs = nullptr;
  mbd::BandJob* band_jobs = nullptr;
  mbd::SweepItem* sweep_items = nullptr;
  mbd::DevBuf sweep_progress;
  int n_band_jobs = 0, n_sweep_items = 0, band_max_n = 0;
  // band jobs [0, n_band_cluster) run in the cluster-resident chase (cluster
  // size band_cluster_C, largest n band_cluster_max_n), the rest in the
  // flag-synchronised one
  int n_band_cluster = 0, band_cluster_C = 0, band_cluster_max_n = 0;
  bool cluster_chase = true;                 // MBD_B200_CLUSTER_CHASE=0 turns the cluster-resident chase off
  long long sweeps_in_flight = 0;
  int n_trd_groups = 0, trd_total_ctas = 0, n_eig_jobs = 0, n_eig_batch = 0, eig_batch_max_n = 0;
  double trd_est_ms = 0.0;
  std::vector<int> order;                    // geometries that run, descending relay size
  std::vector<int> eig_single;               // geometries whose eigenvalues need their own launch
  double* weights_dev = nullptr;
  double* omega_dev = nullptr;               // the 21 imaginary frequencies
  // learned warm start: network parameters, Adam state, training work
  mbd::DevBuf gnn_params, gnn_grad, gnn_m1, gnn_m2, gnn_train_work, gnn_eval;
  mbd::DevBuf graph_scan;   // edge counts / offsets of the network graphs being built
  bool have_net = false;
  bool use_net = true;
  double* loss_dev = nullptr;
  int* err_flag = nullptr;
  mbd::TridiagJob* job_dev = nullptr;
  std::vector<cudaEvent_t> events;           // kGeomEvents per geometry
  // start, relay done, tridiag done, end, one-stage launch done
  cudaEvent_t bev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t fork_ev = nullptr;             // releases the slot streams at the start of a compute
  // one captured graph of mbd_rsscs_compute per mode, valid until the next
  // upload or workspace reallocation
  cudaGraphExec_t graph[3] = {nullptr, nullptr, nullptr};
  double graph_launches[3] = {0, 0, 0};
  // graph[mode] was captured at the batch's first compute (full CG schedule)
  bool graph_first[3] = {false, false, false};
  // a first-compute graph of an earlier batch, kept so that the next batch's
  // first compute can update it (cudaGraphExecUpdate) instead of launching
  // kernel by kernel or instantiating anew
  cudaGraphExec_t graph_prev[3] = {nullptr, nullptr, nullptr};
  // batch_signature of the batch whose first-compute graph is kept, and of
  // the last batch computed for the first time, per mode
  std::vector<long long> graph_sig[3], last_sig[3];
  double graph_updates = 0;                  // first-compute graphs written by cudaGraphExecUpdate
  // the last update's cudaGraphExecUpdateResult and, where it names one, the
  // cudaGraphNodeType of the node it refused (-1 none)
  int graph_update_result = 0, graph_update_node = -1;
  bool use_graphs = true;
  bool graph_update = false;                 // MBD_B200_GRAPH_UPDATE=1: first computes of repeated shapes as graphs
  // how the last compute ran: 0 kernel by kernel, 1 replay of the batch's
  // graph, 2 a graph captured at the batch's first compute (updated from an
  // earlier batch's where the launch sequence matched)
  int graph_kind = 0;
  int two_stage_max_n = 0;                   // largest matrix the two-stage reduction takes on this device
  bool two_stage_batch = false;              // two-stage reduction for the matrices it can take
  int two_stage_force = -1;                  // 1 / 0: forced on / off; -1: policy
  bool capturing = false;
  int mode_runs[3] = {0, 0, 0};              // computes of the uploaded batch, per mode
  double last_ms[mbd::Stage::kCount] = {0};
  double last_band_ms = 0.0, last_chase_ms = 0.0;
  double last_onestage_ms = 0.0, last_sb2st_ms = 0.0;   // the two batch-wide launches of last_chase_ms
  double launches = 0, h2d_bytes = 0, d2h_bytes = 0;
  int last_mode = 0;
  bool have_batch = false;
  // options (mbd_rsscs_set_option)
  double residual_gate = mbd::kResidualGate;   // accepted ||B - A X||_F / ||B||_F of the fast relay solves
  double wait_limit_s = 2.0;                   // bounded device waits (per device)
  int test_stall_wait = 0;                     // 1: the bulge-chasing launch's first wait runs out
  int f32_tensor_build = 0;                    // 1: mixed modes build the relay tensors in FP32 arithmetic
  bool cg_fp32 = false;                        // learned mode: block-CG matrix passes on the FP32 copy (this batch)
  int cg_fp32_mode = -1;                       // 1 always, 0 never, -1 where the copy fits (reserve_learned)
  mbd::TuneChoice tune[mbd::kTuneClasses];     // mbd_rsscs_autotune
  int panel_qr_default = 0;                    // MBD_B200_PANEL_QR=tsqr: 1
};

namespace mbd {

inline int cuda_status(cudaError_t e) {
  if (e == cudaSuccess) return MBD_OK;
  if (e == cudaErrorMemoryAllocation) return MBD_ERR_OUT_OF_MEMORY;
  return MBD_ERR_DEVICE;
}

#define MBD_CUDA(x)                                \
  do {                                             \
    cudaError_t _e = (x);                          \
    if (_e != cudaSuccess) return ::mbd::cuda_status(_e); \
  } while (0)

template <class T>
size_t bytes_of(size_t n) {
  return ((n * sizeof(T)) + 255) & ~size_t(255);
}

// Records a timing event; inside a stream capture it becomes an event-record
// node of the graph, so the event is recorded again on every replay.
inline void record_timing(const mbd_ctx* ctx, cudaEvent_t ev, cudaStream_t s) {
  cudaEventRecordWithFlags(ev, s, ctx->capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
}

// Host-to-device copy ordered with the context's streams: a plain
// cudaMemcpy / cudaMemset runs on the legacy default stream, which the
// context's non-blocking streams do not wait for, and may return before a
// copy from pageable memory has landed.
inline cudaError_t h2d_ordered(const mbd_ctx* ctx, void* dst, const void* src, size_t bytes) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(ctx->stream);
}
inline cudaError_t zero_ordered(const mbd_ctx* ctx, void* dst, size_t bytes) {
  cudaError_t e = cudaMemsetAsync(dst, 0, bytes, ctx->stream);
  return e != cudaSuccess ? e : cudaStreamSynchronize(ctx->stream);
}

// Look-ahead streams: an auxiliary stream at the device's highest priority
// and its two events.
inline cudaError_t create_lookahead(Sy2sbLookAhead* la) {
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&la->aux, cudaStreamNonBlocking, greatest);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&la->ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&la->done, cudaEventDisableTiming);
  la->priority = greatest;
  return e;
}
inline const Sy2sbLookAhead* lookahead_for(const mbd_ctx* ctx, const Sy2sbLookAhead& la) {
  return ctx->lookahead && la.aux ? &la : nullptr;
}

// tune.cu
int tune_class(int n);
int autotune(mbd_ctx* ctx, int max_n);
inline int tuned_rows(const mbd_ctx* ctx, int n) { return ctx->tune[tune_class(n)].rows; }
inline int tuned_panel_qr(const mbd_ctx* ctx, int n) {
  const int q = ctx->tune[tune_class(n)].panel_qr;
  return q >= 0 ? q : ctx->panel_qr_default;
}
inline int tuned_chase_c(const mbd_ctx* ctx, int n) { return ctx->tune[tune_class(n)].chase_c; }
// api.cpp
// Destroys the captured graphs (they hold the launch arguments of the
// uploaded batch and its buffers).  keep_first: a graph captured at a first
// compute is kept for the next batch's first compute to update.
void drop_graphs(mbd_ctx* ctx, bool keep_first = false);
int run_front(mbd_ctx* ctx, GeomDev* gd, int gi, int mode, bool relay_only = false);
int upload_batch(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, bool eigen);
// learn.cpp
int reserve_learned(mbd_ctx* ctx);
// Band -> tridiagonal (d, e) of one band with its own tables in `scratch`
// (grown as needed), on stream s.
int band_to_tridiag_single(mbd_ctx* ctx, double* Br, int n, double* d, double* e, DevBuf& scratch, cudaStream_t s);
int relay_learned(mbd_ctx* ctx, GeomDev* gd, RelaySlot& sl, size_t mstride, cudaEvent_t ev_net, double** X_out);

// Matrices reduced by the two-stage path (the rest by the one-stage kernel).
inline bool two_stage(const mbd_ctx* ctx, int n) {
  return ctx->two_stage_batch && n <= ctx->two_stage_max_n;
}

}  // namespace mbd
