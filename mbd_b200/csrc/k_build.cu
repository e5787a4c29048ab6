// Dipole-tensor builders for the relay matrix (K1) and the CFDM Hamiltonian
// (K5), plus the per-atom frequency table.
//
// Layout: every matrix is row-major with a padded leading dimension; only
// atom blocks (i >= j) are written (the lower triangle, as the reference's
// fill at UTILS.f90:427-431 / 799-803).  One thread owns one atom pair
// (i, j); consecutive threads take consecutive j, so the three 24-byte rows
// of the 3x3 blocks of a warp form contiguous 768-byte runs, which the relay
// builder writes with 16-byte vector stores.
#include <cuda_runtime.h>

#include "kernels.h"
#include "mbd_internal.h"

namespace mbd {

__constant__ double c_omega[21];

namespace {

constexpr double kPiD = 3.14159265358979323846;
constexpr double kOtdD = 0.33333333333333333333;

__global__ void atom_freq_kernel(AtomDev a, int N) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double h = a.hirsh[i], a0 = a.alpha0[i], c6 = a.c6free[i];
  // get_alpha_and_sgm, UTILS.f90:1172-1179
  const double w_p = (4.0 / 3.0) * c6 / (a0 * a0);
  const double s2p = sqrt(2.0 / kPiD);
  for (int f = 0; f < 21; ++f) {
    const double w = c_omega[f];
    const double a_w = (h * a0) / (1.0 + (w * w) / (w_p * w_p));
    a.alpha_w[f * N + i] = a_w;
    a.sgm[f * N + i] = pow((a_w / 3.0) * s2p, kOtdD);
  }
  a.rvdw_iso[i] = pow(h, kOtdD) * a.r0[i];   // UTILS.f90:254
}

// Rows of the folded lower-triangle grid: grid row p holds atom rows p and
// N - 1 - p, whose column blocks (of kBuildThreads atoms) together number
// about N / kBuildThreads + 1, so nearly every CTA has pairs j <= i to build.
constexpr int kBuildThreads = 128;

__device__ __forceinline__ bool folded_row(int N, int* i, int* j0) {
  const int p = blockIdx.y, q = N - 1 - p;
  const int nb_p = p / kBuildThreads + 1;
  int jb = blockIdx.x;
  if (jb < nb_p) {
    *i = p;
  } else {
    jb -= nb_p;
    if (q == p || jb >= q / kBuildThreads + 1) return false;
    *i = q;
  }
  *j0 = jb * kBuildThreads;
  return true;
}

// Value type of the tensor arithmetic: FP64, or FP32 from FP64 displacements
// (the image set is always selected in FP64: r <= cut exactly as
// UTILS.f90:574,623 test it).
template <bool F32>
struct TensorMath;
template <>
struct TensorMath<false> {
  using T = double;
  static __device__ __forceinline__ double exp_(double x) { return exp(x); }
  static __device__ __forceinline__ double erf_(double x) { return erf(x); }
};
template <>
struct TensorMath<true> {
  using T = float;
  static __device__ __forceinline__ float exp_(float x) { return expf(x); }
  static __device__ __forceinline__ float erf_(float x) { return erff(x); }
};

// One thread: pair (i, j) of the folded grid, frequencies [f0, f0+FCH) (blockIdx.z).
// gaussian_dipole_tensor (UTILS.f90:637-696) summed over translations
// (scs_offdiag_block 591-633, scs_diag_block 543-587).  The 3x3 blocks of a
// warp's 32 consecutive pairs go out through shared memory as whole block
// rows: 96 contiguous doubles (FP64, double2 stores) or floats (FP32, float4
// stores) per matrix row.
template <int FCH, bool F32>
__global__ void __launch_bounds__(kBuildThreads) relay_build_kernel(RelayBuildArgs a) {
  using M = TensorMath<F32>;
  using T = typename M::T;
  __shared__ __align__(16) double stage[kBuildThreads / 32][3 * 96];
  int i, j0;
  if (!folded_row(a.N, &i, &j0)) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int j = j0 + threadIdx.x;
  const int jw = j0 + warp * 32;               // the warp's first pair
  if (jw > i || jw >= a.N) return;             // whole warps only: none of its pairs exists
  const bool valid = j <= i && j < a.N;
  const int f0 = blockIdx.z * FCH;
  const int N = a.N;
  const int jj = valid ? j : jw;               // a lane past the end computes a dummy pair
  const bool diag = (i == jj);
  const double xi = a.coords[3 * i], yi = a.coords[3 * i + 1], zi = a.coords[3 * i + 2];
  const double d0x = xi - a.coords[3 * jj], d0y = yi - a.coords[3 * jj + 1], d0z = zi - a.coords[3 * jj + 2];
  const double rv12 = diag ? 2.0 * a.rvdw_iso[i] : a.rvdw_iso[i] + a.rvdw_iso[jj];
  const T inv_brv = (T)(1.0 / (a.beta * rv12));
  const T c4pi = (T)sqrt(4.0 / kPiD), c16pi = (T)sqrt(16.0 / kPiD);

  T sg[FCH];
#pragma unroll
  for (int q = 0; q < FCH; ++q) {
    const int f = f0 + q;
    const double si = a.sgm[f * N + i];
    if (diag) {
      sg[q] = (T)si;                                     // UTILS.f90:571 (sigma_i, not sqrt(2) sigma_i)
    } else {
      const double sj = a.sgm[f * N + jj];
      sg[q] = (T)sqrt(si * si + sj * sj);                // UTILS.f90:620
    }
  }
  T acc[FCH][6];
#pragma unroll
  for (int q = 0; q < FCH; ++q)
#pragma unroll
    for (int c = 0; c < 6; ++c) acc[q][c] = (T)0;

  for (int s = diag ? 1 : 0; s < a.n_shifts; ++s) {
    const double dxd = d0x + a.shifts[3 * s], dyd = d0y + a.shifts[3 * s + 1], dzd = d0z + a.shifts[3 * s + 2];
    const double r2d = dxd * dxd + dyd * dyd + dzd * dzd;
    if (!(sqrt(r2d) <= a.cut)) continue;
    const T dx = (T)dxd, dy = (T)dyd, dz = (T)dzd;
    const T r2 = (T)r2d;
    const T r = F32 ? (T)sqrt(r2d) : sqrt(r2);
    // frequency-independent parts: Fermi damping 1 - 1/(1+exp(-6(r/(beta R)-1)))
    const T damp = (T)1 - ((T)1 / ((T)1 + M::exp_((T)-6 * (r * inv_brv - (T)1))));
    const T inv_r5 = (T)1 / (r2 * r2 * r);
    const T xx = dx * dx, xy = dx * dy, xz = dx * dz, yy = dy * dy, yz = dy * dz, zz = dz * dz;
#pragma unroll
    for (int q = 0; q < FCH; ++q) {
      const T ratio = r / sg[q];
      const T ex = M::exp_(-(ratio * ratio));
      const T zeta_l = (M::erf_(ratio) - (c4pi * ratio * ex)) * inv_r5;
      const T zeta_r = (c16pi * ex) / (sg[q] * sg[q] * sg[q] * r2);
      // -(3 dd - r^2 I) zeta_l + dd zeta_r, damped
      const T ca = (zeta_r - (T)3 * zeta_l) * damp;
      const T cb = (r2 * zeta_l) * damp;
      acc[q][0] += ca * xx + cb;
      acc[q][1] += ca * xy;
      acc[q][2] += ca * xz;
      acc[q][3] += ca * yy + cb;
      acc[q][4] += ca * yz;
      acc[q][5] += ca * zz + cb;
    }
  }
  const bool full = __all_sync(0xffffffffu, valid);   // all 32 pairs of the warp exist
  double* st = stage[warp];
#pragma unroll
  for (int q = 0; q < FCH; ++q) {
    const int f = f0 + q;
    double t[6];
#pragma unroll
    for (int c = 0; c < 6; ++c) t[c] = (double)acc[q][c];
    if (diag) {
      const double inv = 1.0 / a.alpha_w[f * N + i];    // UTILS.f90:583-585
      t[0] += inv;
      t[3] += inv;
      t[5] += inv;
    }
    const double b9[9] = {t[0], t[1], t[2], t[1], t[3], t[4], t[2], t[4], t[5]};
    const size_t base = (size_t)f * a.mat_stride + (size_t)(3 * i) * a.ld + 3 * jw;
    if (full) {
      // the warp's three block rows, 96 consecutive values each
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) st[r * 96 + 3 * lane + c] = b9[3 * r + c];
      __syncwarp();
#pragma unroll
      for (int r = 0; r < 3; ++r) {
        if (a.A64) {
          double2* dst = reinterpret_cast<double2*>(a.A64 + base + (size_t)r * a.ld);
          const double2* src = reinterpret_cast<const double2*>(st + r * 96);
          dst[lane] = src[lane];
          if (lane < 16) dst[32 + lane] = src[32 + lane];
        }
        if (a.A32 && lane < 24) {
          float4 v;
          v.x = (float)st[r * 96 + 4 * lane];
          v.y = (float)st[r * 96 + 4 * lane + 1];
          v.z = (float)st[r * 96 + 4 * lane + 2];
          v.w = (float)st[r * 96 + 4 * lane + 3];
          reinterpret_cast<float4*>(a.A32 + base + (size_t)r * a.ld)[lane] = v;
        }
      }
      __syncwarp();
    } else if (valid) {
      const size_t pb = base + 3 * (size_t)(j - jw);
#pragma unroll
      for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          if (a.A64) a.A64[pb + (size_t)r * a.ld + c] = b9[3 * r + c];
          if (a.A32) a.A32[pb + (size_t)r * a.ld + c] = (float)b9[3 * r + c];
        }
    }
  }
}

// One thread: atom pair (r = blockIdx.y, c), cell difference blockIdx.z.
// lr_bare_dipole_tensor (UTILS.f90:1098-1153) summed over supercell images
// (cfdm_diag_block 998-1043 / cfdm_offdiag_block 1047-1094), then placed at
// every (row cell, col cell) with that difference (supercell_*_block 883-994).
__global__ void __launch_bounds__(128) cfdm_build_kernel(CfdmBuildArgs a) {
  const int r = blockIdx.y;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c > r || c >= a.N) return;
  const int di = blockIdx.z;
  const bool same_atom = (r == c);
  const bool self = same_atom && a.diff_is_zero[di];
  const double d0x = a.coords[3 * r] - a.coords[3 * c] + a.diff_shift[3 * di];
  const double d0y = a.coords[3 * r + 1] - a.coords[3 * c + 1] + a.diff_shift[3 * di + 1];
  const double d0z = a.coords[3 * r + 2] - a.coords[3 * c + 2] + a.diff_shift[3 * di + 2];
  const double rv12 = same_atom ? 2.0 * a.rvdw_eff[r] : a.rvdw_eff[r] + a.rvdw_eff[c];
  const double inv_brv = 1.0 / (a.beta * rv12);
  const double wr = a.omega[r], wc = a.omega[c];
  // UTILS.f90:1028 (same atom, same cell) and 1086 (all other blocks)
  const double pref = self ? wr * wr * a.alpha_eff[r] : wr * wc * sqrt(a.alpha_eff[r] * a.alpha_eff[c]);
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int s = self ? 1 : 0; s < a.n_shifts; ++s) {
    const double dx = d0x + a.shifts[3 * s], dy = d0y + a.shifts[3 * s + 1], dz = d0z + a.shifts[3 * s + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double rr = sqrt(r2);
    if (!(rr <= a.cut)) continue;
    const double fermi = 1.0 / (1.0 + exp(-6.0 * (rr * inv_brv - 1.0)));
    const double s5 = fermi / (r2 * r2 * rr);
    const double ca = -3.0 * s5, cb = r2 * s5;   // (r^2 I - 3 dd)/r^5 * fermi
    acc[0] += ca * dx * dx + cb;
    acc[1] += ca * dx * dy;
    acc[2] += ca * dx * dz;
    acc[3] += ca * dy * dy + cb;
    acc[4] += ca * dy * dz;
    acc[5] += ca * dz * dz + cb;
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) acc[k] *= pref;
  if (self) {                                       // UTILS.f90:1039-1041
    acc[0] += wr * wr;
    acc[3] += wr * wr;
    acc[5] += wr * wr;
  }
  const double t[9] = {acc[0], acc[1], acc[2], acc[1], acc[3], acc[4], acc[2], acc[4], acc[5]};
  const int w3 = 3 * a.nsl;
  for (int p = a.place_offset[di]; p < a.place_offset[di + 1]; ++p) {
    const size_t row0 = (size_t)r * w3 + 3 * a.place_rc[p];
    const size_t col0 = (size_t)c * w3 + 3 * a.place_cc[p];
#pragma unroll
    for (int u = 0; u < 3; ++u)
#pragma unroll
      for (int v = 0; v < 3; ++v) a.H[(row0 + u) * a.ldH + col0 + v] = t[3 * u + v];
  }
}

}  // namespace

cudaError_t init_device_constants() {
  return cudaMemcpyToSymbol(c_omega, kCasimirOmega, sizeof(double) * 21);
}

void launch_atom_freq(const AtomDev& a, int N, cudaStream_t s) {
  atom_freq_kernel<<<(N + 127) / 128, 128, 0, s>>>(a, N);
}

void launch_relay_build(const RelayBuildArgs& a, cudaStream_t s) {
  constexpr int FCH = 7;
  // folded rows p and N - 1 - p: at most (N - 1) / 128 + 2 column blocks
  dim3 grid((a.N - 1) / kBuildThreads + 2, (a.N + 1) / 2, 21 / FCH);
  if (a.f32_math)
    relay_build_kernel<FCH, true><<<grid, kBuildThreads, 0, s>>>(a);
  else
    relay_build_kernel<FCH, false><<<grid, kBuildThreads, 0, s>>>(a);
}

void launch_cfdm_build(const CfdmBuildArgs& a, cudaStream_t s) {
  dim3 grid((a.N + 127) / 128, a.N, a.n_diff);
  cfdm_build_kernel<<<grid, 128, 0, s>>>(a);
}

}  // namespace mbd
