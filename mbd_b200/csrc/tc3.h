// Interfaces of the tensor-core (tcgen05, 3xTF32) relay factorisation used by
// the mixed mode.  Separate from kernels.h because CUtensorMap needs <cuda.h>.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstddef>

namespace mbd {

enum { TC3_SYRK_LOWER = 0, TC3_STORE_SPLIT = 1 };

// Tensor maps of the two operands, each split into its TF32 head (hi) and
// FP32 remainder (lo); all 3-D [batch][rows][K] FP32, 32x128 box, 128B swizzle.
struct Tc3Maps {
  CUtensorMap a_hi, a_lo, b_hi, b_lo;
  CUtensorMap c;              // output matrix (TMA reduce-add / store target)
  CUtensorMap c_hi, c_lo;     // TC3_STORE_SPLIT: hi/lo copies of the output
};

struct Tc3Params {
  int mode;          // TC3_SYRK_LOWER: C[lower] -= A B^T ; TC3_STORE_SPLIT: C = A B^T and hi/lo of C
  int batch;
  int a_row0, b_row0;  // first operand row of tile (0,0) in the A / B maps
  int m_rows, n_cols;  // extent of the C region
  int k;             // inner dimension, multiple of 32
  int n_tiles_n;     // tiles along N (TC3_STORE_SPLIT)
  float* C;
  size_t c_bstride;
  int c_ld, c_row0, c_col0;
  float* out_hi;     // TC3_STORE_SPLIT: hi/lo copies of C at [b][c_row0 + r][c]
  float* out_lo;
  size_t o_bstride;
  int o_ld;
  int* err;
};

bool make_tc3_map(CUtensorMap* map, const float* base, int rows, int cols, int ld, size_t bstride, int batch);
cudaError_t init_tc3_attributes();
// tiles: number of 128x128 C tiles (lower-triangle count for TC3_SYRK_LOWER).
void launch_tc3_gemm(const Tc3Maps& maps, const Tc3Params& p, int tiles, cudaStream_t s);
void launch_split(const float* A, size_t a_bstride, int a_ld, int r0, int c0, int rows, int cols, float* hi,
                  float* lo, size_t o_bstride, int o_ld, int batch, cudaStream_t s);

// ---- mixed-mode relay pieces (k_mixed.cu) ----
constexpr int kMixNB = 128;
struct BatchMat32 {
  float* A;
  size_t stride;
  int ld, n, batch;
};
// Factor the 128x128 diagonal block at k0 in FP32, store L_kk into A and the
// hi/lo split of L_kk^-1 at rows [k0, k0+128) of Linv_hi / Linv_lo ([b][n_pad][128]).
void launch_potrf_diag_f32(const BatchMat32& m, int k0, float* linv_hi, float* linv_lo, size_t l_bstride,
                           int* info, cudaStream_t s);
// Solve L L^T D = R with the FP32 factor (FP64 right-hand sides and
// accumulation) in two sync-free launches.  Z: n x 3 work array per matrix.
// sync: solve_sync_ints(n, batch) ints, zeroed once at allocation; epoch must
// grow by one per call on the same sync array.
size_t solve_sync_ints(int n, int batch);
void launch_solve_f32(const BatchMat32& m, const float* linv_hi, const float* linv_lo, size_t l_bstride,
                      double* R, double* Z, double* D, size_t ystride, int* sync, int epoch, int* err,
                      cudaStream_t s);
// R = B - A64 X for the lower-stored FP64 relay matrices (B = stacked identities),
// and X += D first when D != null.  partial: workspace of relay_residual_ws_doubles().
cudaError_t init_mixed_attributes();
size_t relay_residual_ws_doubles(int n, int batch);
void launch_relay_residual(const double* A64, size_t a_stride, int ld, int n, int batch, double* X, const double* D,
                           double* R, size_t ystride, double* partial, double* rnorm2, cudaStream_t s);

}  // namespace mbd
