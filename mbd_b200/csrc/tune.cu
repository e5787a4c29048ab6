// Autotuner of the eigen stages' launch shapes (no counterpart in the
// reference, whose ScaLAPACK block sizes are fixed at UTILS.f90:451-452,
// 813-831).
//
// For each size class (n <= 512 * 2^k) up to the largest Hamiltonian a
// caller announces, it times on a synthetic symmetric matrix of the class's
// size, generated on the device:
//   * the dense -> band reduction with each panel-QR algorithm (Householder
//     with one cluster exchange per column, or TSQR with Householder
//     reconstruction) and rows-per-CTA target (48 .. 384: the target sets how
//     many CTAs share a panel's QR cluster, trading exchange latency against
//     per-CTA work);
//   * the band -> tridiagonal chase: the flag-synchronised kernel (each
//     sweep waits for its predecessor's progress flag in global memory)
//     against the cluster-resident kernel (lock-step wavefront steps) with
//     each cluster size from the smallest that holds the band to the widest
//     allowed (more CTAs: fewer tasks per CTA and step, a wider barrier);
// each candidate twice, keeping the faster run, and stores the fastest choice
// per class in the context.  Later computes and eigenvalue calls of the
// context use them.  A choice only regroups sums (cluster partials), so the
// results of a context stay deterministic once tuned.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "context.h"
#include "kernels.h"

namespace mbd {
namespace {

__device__ __forceinline__ unsigned mix32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Lower triangle of a symmetric matrix with entries uniform in [-1, 1)
// (hash of the position), diagonal shifted by 4.
__global__ void fill_sym_kernel(double* A, int n, int ld, unsigned seed) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long long)n * ld) return;
  const int r = (int)(idx / ld), c = (int)(idx % ld);
  if (c > r) return;
  const unsigned h = mix32((unsigned)r * 0x9e3779b9u ^ mix32((unsigned)c + seed));
  A[idx] = (double)h * (2.0 / 4294967296.0) - 1.0 + (r == c ? 4.0 : 0.0);
}

struct Buf {
  void* p = nullptr;
  ~Buf() {
    if (p) cudaFree(p);
  }
};

}  // namespace

int tune_class(int n) {
  int k = 0;
  while (k < kTuneClasses - 1 && (512 << k) < n) ++k;
  return k;
}

int autotune(mbd_ctx* ctx, int max_n) {
  max_n = std::min(max_n, ctx->two_stage_max_n);
  if (max_n < 64) return MBD_OK;
  cudaStream_t s = ctx->stream;
  cudaEvent_t e0, e1;
  MBD_CUDA(cudaEventCreate(&e0));
  MBD_CUDA(cudaEventCreate(&e1));
  int status = MBD_OK;
  const int kmax = tune_class(max_n);
  for (int k = 0; k <= kmax && status == MBD_OK; ++k) {
    const int n = std::min(max_n, 512 << k);
    const int ld = (n + 31) / 32 * 32;
    const size_t mat = sizeof(double) * (size_t)n * ld;
    Buf a0, a, ws, band, de, job;
    auto fail = [&](cudaError_t e) {
      if (e != cudaSuccess && status == MBD_OK) status = cuda_status(e);
      return e != cudaSuccess;
    };
    if (fail(cudaMalloc(&a0.p, mat)) || fail(cudaMalloc(&a.p, mat)) ||
        fail(cudaMalloc(&ws.p, sizeof(double) * sy2sb_workspace_doubles(n))) ||
        fail(cudaMalloc(&band.p, sizeof(double) * (size_t)n * kBandLd)) ||
        fail(cudaMalloc(&de.p, sizeof(double) * 2 * (size_t)n)) || fail(cudaMalloc(&job.p, sizeof(BandJob))))
      break;
    const long long cells = (long long)n * ld;
    fill_sym_kernel<<<(unsigned)((cells + 255) / 256), 256, 0, s>>>(static_cast<double*>(a0.p), n, ld,
                                                                     0x5eedu + (unsigned)k);
    TuneChoice tc;
    tc.n = n;
    // dense -> band: panel QR algorithm and rows per CTA
    double best = 1e30;
    const int cand[][2] = {{0, 48}, {0, 96}, {0, 192}, {0, 384}, {1, 96}, {1, 192}, {1, 384}};
    for (const auto& cq : cand) {
      double t = 1e30;
      for (int rep = 0; rep < 2; ++rep) {
        if (fail(cudaMemcpyAsync(a.p, a0.p, mat, cudaMemcpyDeviceToDevice, s)) || fail(cudaEventRecord(e0, s)) ||
            fail(launch_sy2sb(static_cast<double*>(a.p), ld, n, static_cast<double*>(ws.p),
                              static_cast<double*>(band.p), ctx->num_sms, s, cq[1], cq[0],
                              lookahead_for(ctx, ctx->la_ctx))) ||
            fail(cudaEventRecord(e1, s)) || fail(cudaEventSynchronize(e1)))
          break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        t = std::min(t, (double)ms);
      }
      if (status != MBD_OK) break;
      if (t < best) {
        best = t;
        tc.panel_qr = cq[0];
        tc.rows = cq[1];
      }
    }
    tc.sy2sb_ms = best;
    // band -> tridiagonal: the flag-synchronised chase (which works on the
    // band in place, so every run starts from a saved copy) against the
    // cluster-resident chase at each cluster size (which leaves the band in
    // global memory untouched)
    double* d = static_cast<double*>(de.p);
    const BandJob bj{static_cast<double*>(band.p), n, d, d + n};
    const size_t band_bytes = sizeof(double) * (size_t)n * kBandLd;
    std::vector<SweepItem> items;
    for (int i = 0; i + 3 <= n; ++i) items.push_back(SweepItem{0, i, i - 1, 0});
    Buf band0, items_d, prog;
    if (status != MBD_OK || fail(cudaMalloc(&band0.p, band_bytes)) ||
        fail(cudaMalloc(&items_d.p, sizeof(SweepItem) * std::max<size_t>(1, items.size()))) ||
        fail(cudaMalloc(&prog.p, 2 * sizeof(int) * std::max<size_t>(1, items.size()))) ||
        fail(cudaMemcpyAsync(band0.p, band.p, band_bytes, cudaMemcpyDeviceToDevice, s)) ||
        fail(cudaMemcpyAsync(items_d.p, items.data(), sizeof(SweepItem) * items.size(), cudaMemcpyHostToDevice, s)) ||
        fail(cudaMemcpyAsync(job.p, &bj, sizeof(bj), cudaMemcpyHostToDevice, s)) || fail(cudaStreamSynchronize(s)))
      break;
    {
      double t = 1e30;
      for (int rep = 0; rep < 2; ++rep) {
        if (fail(cudaMemcpyAsync(band.p, band0.p, band_bytes, cudaMemcpyDeviceToDevice, s)) ||
            fail(cudaEventRecord(e0, s)) ||
            fail(launch_sb2st(static_cast<const BandJob*>(job.p), 1, static_cast<const SweepItem*>(items_d.p),
                              (int)items.size(), static_cast<int*>(prog.p), ctx->err_flag, ctx->num_sms, n,
                              n / (2 * kBand) + 1, -1, s)) ||
            fail(cudaEventRecord(e1, s)) || fail(cudaEventSynchronize(e1)))
          break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        t = std::min(t, (double)ms);
      }
      if (status != MBD_OK) break;
      tc.flag_chase_ms = t;
      tc.chase_c = kChaseFlag;
      tc.chase_ms = t;
      if (fail(cudaMemcpyAsync(band.p, band0.p, band_bytes, cudaMemcpyDeviceToDevice, s))) break;
    }
    const int cmin = sb2st_cluster_min(n);
    const int chi = sb2st_cluster_size(n, 1, ctx->num_sms, 0);   // 0: no cluster holds this band
    if (status == MBD_OK && chi > 0) {
      std::vector<int> cands;
      const int step = std::max(1, (chi - cmin + 3) / 4);
      for (int c = cmin; c <= chi; c += step) cands.push_back(c);
      if (cands.back() != chi) cands.push_back(chi);
      best = 1e30;
      for (int c : cands) {
        double t = 1e30;
        for (int rep = 0; rep < 2; ++rep) {
          if (fail(cudaEventRecord(e0, s)) ||
              fail(launch_sb2st_cluster(static_cast<const BandJob*>(job.p), 1, n, c, s)) ||
              fail(cudaEventRecord(e1, s)) || fail(cudaEventSynchronize(e1)))
            break;
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          t = std::min(t, (double)ms);
        }
        if (status != MBD_OK) break;
        if (t < best) best = t;
        if (t < tc.chase_ms) {
          tc.chase_ms = t;
          tc.chase_c = c;
        }
      }
      tc.cluster_chase_ms = best < 1e30 ? best : 0.0;
    }
    if (status == MBD_OK) ctx->tune[k] = tc;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (status != MBD_OK) return status;
  // the captured graphs and the batch's chase plan used the old choices
  drop_graphs(ctx);
  if (ctx->n_band_cluster > 0)
    ctx->band_cluster_C = sb2st_cluster_size(ctx->band_cluster_max_n, ctx->n_band_cluster, ctx->num_sms,
                                             ctx->tune[tune_class(ctx->band_cluster_max_n)].chase_c);
  return MBD_OK;
}

}  // namespace mbd
