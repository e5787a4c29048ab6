// Learned relay warm start: the message-passing network's sizes, parameter
// layout and launch interfaces (device pointers only).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace mbd {

constexpr int kGnnHidden = 64;
constexpr int kGnnRbf = 16;
constexpr int kGnnIn = 8;
constexpr int kGnnLayers = 3;
constexpr float kGnnCutoffBohr = 5.0f / 0.52917721f;   // 5 Angstrom

// Flat FP32 parameter vector: W0[64][8] b0[64], per layer Wf[64][16]
// Wu[64][64] bu[64], then ws[64] bs wa[64] ca wg[16].
constexpr int kGnnOffW0 = 0;
constexpr int kGnnOffB0 = kGnnOffW0 + kGnnHidden * kGnnIn;
constexpr int kGnnLayerSize = kGnnHidden * kGnnRbf + kGnnHidden * kGnnHidden + kGnnHidden;
__host__ __device__ constexpr int kGnnOffWf(int l) { return kGnnOffB0 + kGnnHidden + l * kGnnLayerSize; }
__host__ __device__ constexpr int kGnnOffWu(int l) { return kGnnOffWf(l) + kGnnHidden * kGnnRbf; }
__host__ __device__ constexpr int kGnnOffBu(int l) { return kGnnOffWu(l) + kGnnHidden * kGnnHidden; }
constexpr int kGnnOffWs = kGnnOffWf(kGnnLayers);
constexpr int kGnnOffBs = kGnnOffWs + kGnnHidden;
constexpr int kGnnOffWa = kGnnOffBs + 1;
constexpr int kGnnOffCa = kGnnOffWa + kGnnHidden;
constexpr int kGnnOffWg = kGnnOffCa + 1;
constexpr int kGnnParams = kGnnOffWg + kGnnRbf;
static_assert(kGnnParams == 16274, "parameter layout");

// One geometry's graph, F frequency copies of N atoms (node f * N + i).
struct GnnGraph {
  int N, F, E;
  const int* off;          // [N + 1] CSR offsets
  const int* nbr;          // [E] neighbour atom
  const int* src;          // [E] owning atom
  const float* efeat;      // [E][16] radial features
  const float* eproj;      // [E][6] u u^T - I/3: xx yy zz xy xz yz
  const float* x;          // [F * N][8] node inputs
};

struct GnnWork {
  float* pre0;
  float* h[kGnnLayers + 1];
  float* m[kGnnLayers];
  float* u[kGnnLayers];
  float* filt;             // [3][E][64]
  float* g;                // [E]
  float *s, *a;            // [M]
  float* S;                // [M][9] prediction
  // training only
  float *dS, *dh, *dh2, *du, *dm, *ds, *da, *dfilt, *cw, *S_true;
};

// Radius graph of one geometry (the network's neighbour lists): edges
// (i, j, t) for the images t = n0 a0 + n1 a1 + n2 a2, |n_k| <= rng[k], with
// 1e-12 <= |x_j + t - x_i|^2 < rc2, CSR by i, each list in (image, j) order.
struct GraphBox {
  double lat[9];         // lattice vectors a_k = lat[3k .. 3k+2], bohr
  int rng[3];            // image range per axis (0 along vacuum axes and for clusters)
  double lo[3], hi[3];   // bounding box of the atoms
  double pad;            // the cut-off plus a rounding margin (image pruning)
  double rc2;            // squared cut-off, bohr^2
};
// cnt[i] = edges of atom i
void gnn_graph_count(const double* x, int N, const GraphBox& b, int* cnt, cudaStream_t s);
// cnt[0..N) -> CSR offsets in place, cnt[N] = *E = the edge count
void gnn_graph_scan(int* cnt_off, int N, int* E, cudaStream_t s);
// the lists at the offsets off_in (copied to off[0..N])
void gnn_graph_fill(const double* x, int N, const GraphBox& b, const int* off_in, int* off, int* nbr, int* src,
                    float* dvec, cudaStream_t s);

size_t gnn_work_floats(int N, int F, int E, bool train);
GnnWork gnn_work_layout(float* base, int N, int F, int E, bool train);
void gnn_edges(const float* dvec, int E, float* efeat, float* eproj, cudaStream_t s);
void gnn_features(const int* species, const double* hirsh, const double* alpha_w, const double* omega, int N, int F,
                  float* x, cudaStream_t s);
// Forward pass into w.S; returns the number of launches.
int gnn_forward(const float* P, const GnnGraph& g, const GnnWork& w, cudaStream_t s);
// Loss against w.S_true (added to *loss) and its gradient added to G.
int gnn_loss_backward(const float* P, const GnnGraph& g, const GnnWork& w, float* G, double* loss, cudaStream_t s);
// Adam step `step` (from 1) with learning rate lr; zeroes G.
void gnn_adam(float* P, float* G, float* m1, float* m2, int step, float lr, cudaStream_t s);
// X (FP64, [F][3N][3], row stride ystride per frequency) = alpha_w * S.
void gnn_warmstart(const float* S, const double* alpha_w, int N, int F, double* X, size_t ystride, cudaStream_t s);
// S_true = X / alpha_w (training targets from a direct relay solve).
void gnn_targets(const double* X, size_t ystride, const double* alpha_w, int N, int F, float* St, cudaStream_t s);

}  // namespace mbd
