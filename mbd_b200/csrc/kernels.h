// Kernel launch interfaces (device pointers only).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace mbd {

// ---- per-atom, per-frequency data (get_alpha_and_sgm, UTILS.f90:1157-1184) ----
struct AtomDev {
  const double* coords;    // [3N]
  const double* alpha0;    // [N]
  const double* c6free;    // [N]
  const double* r0;        // [N]
  const double* hirsh;     // [N]
  double* alpha_w;         // [21][N] free-atom alpha(iw), scaled by Hirshfeld ratio
  double* sgm;             // [21][N] dipole spread sigma(iw)
  double* rvdw_iso;        // [N]     h^(1/3) R0
};
void launch_atom_freq(const AtomDev& a, int N, cudaStream_t s);
// Copies the frequency grid to constant memory of the current device.
cudaError_t init_device_constants();

// ---- relay tensor build (get_screened_alpha UTILS.f90:415-441) ----
struct RelayBuildArgs {
  int N, ld;
  size_t mat_stride;       // elements between consecutive frequency matrices
  const double* coords;
  const double* alpha_w;   // [21][N]
  const double* sgm;       // [21][N]
  const double* rvdw_iso;  // [N]
  const double* shifts;    // [3*n_shifts], zero shift first
  int n_shifts;
  double beta;
  double cut;              // min(scs cut-off, damping radius), bohr
  double* A64;             // 21 matrices, row-major lower (may be null)
  float* A32;              // 21 matrices, row-major lower (may be null)
  int f32_math = 0;        // 1: tensor arithmetic in FP32 from FP64 displacements
};
void launch_relay_build(const RelayBuildArgs& a, cudaStream_t s);

// ---- CFDM Hamiltonian build (get_mbd_rSCS UTILS.f90:787-807) ----
struct CfdmBuildArgs {
  int N, nsl, ldH;
  const double* coords;
  const double* omega;     // [N] screened characteristic frequency
  const double* alpha_eff; // [N]
  const double* rvdw_eff;  // [N]
  const double* shifts;    // [3*n_shifts] supercell image translations, zero first
  int n_shifts;
  const double* diff_shift;   // [3*n_diff]
  const int* diff_is_zero;    // [n_diff]
  const int* place_offset;    // [n_diff+1]
  const int* place_rc;
  const int* place_cc;
  int n_diff;
  double beta;
  double cut;
  double* H;
};
void launch_cfdm_build(const CfdmBuildArgs& a, cudaStream_t s);

// ---- relay factorisation / solve, FP64 (PDPOTRF/PDPOTRS UTILS.f90:469-473) ----
constexpr int kCholNB = 64;
struct BatchMat {
  double* A;               // batch of row-major lower matrices
  size_t stride;           // elements between matrices
  int ld, n, batch;
};
// Linv: per matrix, ceil(n/64) blocks of 64x64 inverses of the diagonal factor blocks.
void launch_potrf_diag_f64(const BatchMat& m, int k0, double* Linv, size_t linv_stride, int* info,
                           cudaStream_t s);
void launch_trsm_panel_f64(const BatchMat& m, int k0, const double* Linv, size_t linv_stride,
                           cudaStream_t s);
void launch_syrk_lower_f64(const BatchMat& m, int k0, cudaStream_t s);
// Y (n x 3 per matrix, row-major, stride ystride) := stacked identities [I;I;..;I].
void launch_init_rhs(double* Y, size_t ystride, int n, int batch, cudaStream_t s);
// Forward step: reads W at block k0, writes Z at block k0, updates W below it.
void launch_trsv_fwd_step(const BatchMat& m, int k0, const double* Linv, size_t linv_stride, double* W,
                          double* Z, size_t ystride, cudaStream_t s);
// Backward step: reads Zw at block k0, writes X at block k0, updates Zw above it.
void launch_trsv_bwd_step(const BatchMat& m, int k0, const double* Linv, size_t linv_stride, double* Zw,
                          double* X, size_t ystride, cudaStream_t s);
cudaError_t init_chol_attributes();

// ---- epilogues (UTILS.f90:479-495, 272-315, 731-741) ----
struct EpilogueArgs {
  int N;
  const double* X;         // [21][3N][3] relay solutions
  size_t xstride;
  double* alpha_iw;        // [21][N]
  double* molpol;          // [21][9] row-major 3x3
  // post
  const double* alpha0;
  const double* c6free;
  const double* r0;
  double* c6_eff;          // [N]
  double* alpha_eff;       // [N]
  double* omega;           // [N]
  double* rvdw_eff;        // [N]
  double* scalars;         // [0] c6_mol, [1] sum 3*omega, [2] #alpha_eff <= 0
};
void launch_relay_epilogue(const EpilogueArgs& a, cudaStream_t s);
void launch_relay_post(const EpilogueArgs& a, const double* weights_dev, cudaStream_t s);

// ---- eigensolver (PDSYEV('N','L') UTILS.f90:835, energy UTILS.f90:839-867) ----
struct TridiagJob {
  double* A;               // row-major lower, overwritten
  int n, ld;
  double* d;               // [n]
  double* e;               // [n-1]
  // optional (eigenvectors): reflector c = 0..n-2, H_c = I - tau[c] v v^T with
  // v(r) at vsave[c * ldv + r] for r >= c + 1 (v(c + 1) = 1); rows r <= c of
  // each reflector are left as the caller set them (zero)
  double* vsave = nullptr;
  double* tau = nullptr;
  size_t ldv = 0;
};
constexpr int kTrdTile = 64;
constexpr int kTrdNB = 32;
constexpr int kTridiagMaxGroup = 160;   // CTAs per group the kernel's reductions are sized for
size_t tridiag_workspace_bytes(int n, int group_ctas);
// Reduces each job's matrix to tridiagonal form with `groups` groups of
// `group_ctas` co-resident CTAs (cooperative launch).  Returns a cudaError.
// nmax: the largest n among the jobs (sizes each group's workspace layout).
cudaError_t launch_tridiag(const TridiagJob* jobs_dev, int n_jobs, int groups, int group_ctas,
                           void* workspace, size_t ws_bytes_per_group, int nmax, int* err_flag,
                           cudaStream_t s);
// One CTA group of a table launch: CTAs [first_cta, first_cta + G) reduce
// jobs [job_begin, job_end) in order; workspace at ws_offset, laid out for
// nmax (tridiag_workspace_bytes(nmax, G) bytes).
struct TridiagGroup {
  int first_cta, G;
  int job_begin, job_end;
  int nmax, pad;
  size_t ws_offset;
};
// Groups of different sizes in one cooperative launch of total_ctas CTAs
// (groups ascending in first_cta, covering [0, total_ctas)); zeroes their
// barrier words first.  Returns a cudaError.
cudaError_t launch_tridiag_groups(const TridiagJob* jobs_dev, const TridiagGroup* groups_dev, int n_groups,
                                  int total_ctas, void* workspace, int* err_flag, cudaStream_t s);
int tridiag_max_ctas_per_sm();

// Eigenvalues of (d, e) by multisection; writes ev[0..n) ascending and uses
// ev[n..2n) as scratch (ev must hold 2n doubles).
void launch_tridiag_eigenvalues(const double* d, const double* e, int n, double* ev, cudaStream_t s);
void launch_tridiag_eigenvalues_scratch(const double* d, const double* e, int n, double* ev, double* e2,
                                        cudaStream_t s);
cudaError_t init_eigval_attributes();
// ---- eigenvectors (k_eigvec.cu) ----
// C (M x N, row-major) = alpha op(A) op(B) + beta C on FP64 MMA; op(A)(i, k) =
// ta ? A[k * lda + i] : A[i * lda + k], op(B)(k, j) = tb ? B[j * ldb + k] :
// B[k * ldb + j]; beta == 0 does not read C.
void dgemm_rm(bool ta, bool tb, int M, int N, int K, double alpha, const double* A, size_t lda, const double* B,
              size_t ldb, double beta, double* C, size_t ldc, cudaStream_t s);
// doubles of the scratch launch_tri_vectors needs
size_t eigh_scratch_doubles(int n);
// Eigenvectors of the tridiagonal (d, e) for its ascending eigenvalues ev into
// the columns of Z (row-major, Z[i * ldz + k] = component i of vector k);
// tnorm = max |ev| sets the cluster tolerance and the pivot floor.
void launch_tri_vectors(const double* d, const double* e, const double* ev, int n, double tnorm, double* Z, size_t ldz,
                        double* scratch, cudaStream_t s);
// G (n x n) <- 3/2 I - G/2, *dev = max |G - I| as bits (atomic max; zero it first)
void launch_ns_prepare(double* G, int n, unsigned long long* dev, cudaStream_t s);
// T (nb x nb row-major upper) of I - V T V^T = H_0 ... H_{kb-1} from S = V^T V (ld nb)
void launch_wy_t(const double* S, const double* tau, int kb, int nb, double* T, cudaStream_t s);
// energy = 0.5*sum_{ev>=0} sqrt(ev)/nsl - 0.5*sum_nonint; out[0]=E, out[1]=sum sqrt, out[2]=nimag
void launch_energy(const double* ev, int n, int nsl, const double* scalars, double* out,
                   cudaStream_t s);
// ---- two-stage tridiagonalisation (PDSYEV('N','L') reduction, UTILS.f90:835) ----
constexpr int kBand = 32;                    // half-bandwidth of the intermediate band
constexpr int kBandLd = 2 * kBand + 1;       // band row: A(r, r - d), d = 0..2 kBand (room for bulges)
constexpr int kPanelMaxRowsPerCta = 1152;    // panel rows one CTA keeps (384 in registers, the rest in shared memory)
constexpr int kPanelRowsTarget = 96;         // fewer rows per CTA while the cluster can grow
constexpr int kPanelMaxCluster = 16;         // CTAs of the panel-QR cluster
constexpr int kSymmMaxSplit = 16;
struct PanelArgs {
  double* A;
  int ld;
  int row0, col0;          // panel = A[row0 .. row0 + m)[col0 .. col0 + kBand)
  int m;
  int rows_per_cta;
  double* V;               // [m][kBand] out: Householder vectors, unit lower trapezoidal
  double* T;               // [kBand][kBand] out: compact-WY factor
  double* tau;             // [kBand] out
};
cudaError_t init_sy2sb_attributes();
int sy2sb_max_n();
int sy2sb_max_cluster();
size_t sy2sb_workspace_doubles(int n);
// Dense (lower, row-major, ld) -> band: A is overwritten; Br[n][kBandLd]
// receives the band (diagonal d = 0..kBand, zero beyond).  ws: workspace.
// rows_per_cta: panel rows per CTA the QR cluster aims at (0: default);
// panel_qr: 0 Householder QR with one cluster exchange per column,
// 1 TSQR with Householder reconstruction (k_tsqr.cu) where it applies.
// la (optional): look-ahead -- each panel's update first applies to the next
// panel's columns, whose QR then runs on la->aux (at la->priority) beside the
// rest of the update; ready/done order the two streams.
struct Sy2sbLookAhead {
  cudaStream_t aux;
  cudaEvent_t ready, done;
  int priority;
};
cudaError_t launch_sy2sb(double* A, int ld, int n, double* ws, double* Br, int num_sms, cudaStream_t s,
                         int rows_per_cta = 0, int panel_qr = 0, const Sy2sbLookAhead* la = nullptr);
// TSQR panel QR (k_tsqr.cu): rows per CTA in [32, tsqr_max_rows_per_cta()], C <= 16.
cudaError_t init_tsqr_attributes();
int tsqr_max_rows_per_cta();
cudaError_t launch_tsqr_panel(const PanelArgs& pa, int C, cudaStream_t s);
int sy2sb_launches(int n);
// Band -> tridiagonal for a batch of bands in one persistent cooperative
// launch (bulge chasing, one warp per task of a sweep).
struct BandJob {
  double* Br;              // [n][kBandLd], overwritten
  int n;
  double* d;               // [n] diagonal out
  double* e;               // [n-1] subdiagonal out
};
// items: (job, sweep) pairs ordered by sweep then job; pred[t] = the item of
// the same job's previous sweep or -1; progress[n_items] zeroed by the launch.
struct SweepItem {
  int job, sweep, pred, pad;
};
// sweeps_in_flight: sum over jobs of n / (2 kBand), the concurrency the
// sweep pipeline offers (sizes the worker count).
// stall_item >= 0 makes that item's first wait target a count no sweep
// reaches, so the bounded wait runs out (failure-detection tests only).
// progress: 2 * n_items ints (two published task counts per sweep item).
cudaError_t launch_sb2st(const BandJob* jobs, int n_jobs, const SweepItem* items, int n_items, int* progress,
                         int* err, int num_sms, int max_n, long long sweeps_in_flight, int stall_item,
                         cudaStream_t s);
cudaError_t init_sb2st_attributes();
// The same chase with each band held in the distributed shared memory of one
// thread-block cluster (k_sb2st_cluster.cu): largest n it takes on this
// device (0 when clusters of this kernel cannot run), the cluster size for a
// batch (0: none fits), and the launch (jobs with n <= max_n; writes d, e).
int sb2st_cluster_max_n();
// want_c > 0: the (autotuned) cluster size to use when it is allowed
int sb2st_cluster_size(int max_n, int n_jobs, int num_sms, int want_c = 0);
// smallest and largest cluster size the chase may use for a band of n rows
int sb2st_cluster_min(int n);
int sb2st_cluster_cmax();
cudaError_t launch_sb2st_cluster(const BandJob* jobs, int n_jobs, int max_n, int C, cudaStream_t s);

// ---- block-CG relay solve of the MIXED_LEARNED mode (UTILS.f90:469-473) ----
constexpr int kCgState = 24;   // per-frequency recurrence state (doubles)
constexpr int kCgIndefinite = 21;   // state slot: 1 when a search direction found p^T A p < 0
struct CgArgs {
  const double* A;         // 21 relay matrices, row-major lower FP64
  const float* A32;        // the same matrices rounded to FP32 (same strides), or null
  size_t a_stride;
  int ld, n, N, nt;        // n = 3N, nt = ceil(n / 64)
  int batch;               // frequencies
  double *X, *R, *Z, *P, *Q;   // [batch][n][3]; X holds the start on entry
  size_t ystride;          // n * 3
  double* Minv;            // [batch][nt][64][64] inverses of the 64 x 64 diagonal tiles
  double* partial;         // cg_partial_doubles
  double* red;             // cg_red_doubles (row-block partials)
  double* red2;            // cg_red_doubles (atom-block partials)
  double* state;           // [batch][kCgState]: [0] stop flag, [1] iterations
  double tol2;             // stop when ||R||_F^2 <= tol2
};
size_t cg_partial_doubles(int n, int batch);
size_t cg_minv_doubles(int n, int batch);
size_t cg_red_doubles(int n, int batch);
constexpr int kCgPhase1Iters = 22;   // state slot: iterations of the first (FP32-pass) phase
// Tile inverses, R = B - A X, Z, P and Z^T R for every frequency.
void launch_cg_setup(const CgArgs& a, cudaStream_t s);
// One iteration (iteration index it = 0, 1, ...); a converged frequency
// skips it.  fp32: the matrix pass reads A32 instead of A (FP64 vectors and
// sums either way).
void launch_cg_iteration(const CgArgs& a, int it, cudaStream_t s, bool fp32 = false);
// Restart between the two phases of the mixed-precision solve: the true
// residual R = B - A X from the FP64 matrix, Z = M^-1 R, P = Z, Z^T R; the
// frequencies the first phase stopped (converged or broke down) run again,
// those shown indefinite stay stopped; the first phase's iteration count
// moves to state slot kCgPhase1Iters.
void launch_cg_restart(const CgArgs& a, cudaStream_t s);

// Many tridiagonal eigenproblems and energies in one launch each.
struct EigJob {
  const double* d;
  const double* e;
  double* ev;              // [n]
  const double* scalars;   // relay scalars ([1] = sum of 3 omega)
  double* out;             // energy outputs as launch_energy
  int n, nsl;
};
constexpr int kEigBatchMaxN = 12800;    // d and e^2 staged in shared memory
// jobs with n <= kEigBatchMaxN only; max_n the largest n among them.
void launch_eigen_batch(const EigJob* jobs_dev, int n_jobs, int max_n, cudaStream_t s);
void launch_energy_batch(const EigJob* jobs_dev, int n_jobs, cudaStream_t s);

// Limit (SM clock cycles) of the bounded device-side waits of each
// translation unit that has them (wait_limit.cuh); per device.
cudaError_t set_wait_limit_sb2st(long long cycles);
cudaError_t set_wait_limit_tridiag(long long cycles);
cudaError_t set_wait_limit_mixed(long long cycles);
cudaError_t set_wait_limit_tc3(long long cycles);

}  // namespace mbd
