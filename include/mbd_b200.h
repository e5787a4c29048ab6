/*
 * mbd_b200.h -- C ABI of the B200-native MBD@rsSCS engine.
 *
 * Drop-in for the pmbd.x hot path of 000Justin000/MBD.  The reference enters
 * its physics through one in-process seam, MBD_rsSCS.f90:218-221
 *     CALL init_blacs(); CALL MBD_at_rsSCS(ene_mbd_rsSCS)
 * where MBD_at_rsSCS (UTILS.f90:153-349) reads module globals (coords,
 * atom_name, hirshfeld_volume, lattice_vector, cut-offs, vacuum axes, flag_xc)
 * and leaves the energy, alpha_eff, C6_eff and coupled_atom_pol behind.  The
 * calls below take the same data explicitly.  Every pointer is HOST memory
 * owned by the caller (except those of mbd_rsscs_eigvalsh_noalloc, which are
 * device pointers), arrays follow Fortran column-major order, atoms keep the
 * caller's order in every result, and every argument type maps to
 * iso_c_binding (c_int, c_double, c_ptr, c_char).
 *
 * Threading: one context per host thread.  A context owns its device
 * buffers, streams and kernels' workspaces.
 */
#ifndef MBD_B200_H
#define MBD_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (replace the reference's STOP / ignored INFO) ---------- */
enum {
    MBD_OK = 0,
    MBD_ERR_ARG = 1,              /* bad argument (null pointer, n_atoms < 1, ...) */
    MBD_ERR_UNKNOWN_ELEMENT = 2,  /* get_vdw_param 'case default' STOP, UTILS.f90:1693-1699 */
    MBD_ERR_RELAY_NOT_SPD = 3,    /* PDPOTRF info > 0, never checked at UTILS.f90:469 */
    MBD_ERR_NONPOSITIVE_ALPHA = 4,/* screened alpha_eff <= 0: (alpha/alpha0)^(1/3) undefined, UTILS.f90:737 */
    MBD_ERR_EIGENSOLVER = 5,      /* PDSYEV info != 0, UTILS.f90:845,864-866 */
    MBD_ERR_DEVICE = 6,           /* CUDA runtime error / no sm_100 device */
    MBD_ERR_TIMEOUT = 7,          /* a bounded device-side wait ran out */
    MBD_ERR_OUT_OF_MEMORY = 8,
    MBD_ERR_REFINEMENT = 9,       /* mixed mode: refinement did not reach the residual gate
                                     (informational: the direct FP64 fallback then ran) */
    MBD_ERR_NOT_BUILT = 10,       /* requested mode is not available in this build */
    MBD_ERR_TOO_LARGE = 11,       /* mbd_rsscs_eigvalsh_noalloc: n > MBD_NOALLOC_MAX_N */
    MBD_ERR_NO_NETWORK = 12       /* MIXED_LEARNED without a trained or loaded network */
};

/* ---- compute modes ------------------------------------------------------- */
enum {
    MBD_MODE_PLAIN_FP64 = 0,      /* FP64 tensor build, FP64 Cholesky, FP64 eigensolve */
    MBD_MODE_MIXED = 1,           /* FP32 relay copy factorised on tcgen05 tensor cores
                                     (3xTF32), FP64 iterative refinement to 1e-10 */
    MBD_MODE_MIXED_LEARNED = 2    /* relay solved by block-CG (FP64, preconditioned by the
                                     inverses of the 64x64 diagonal tiles of the relay
                                     matrix) started from a message-passing network's
                                     prediction of every atom's screened-polarizability
                                     block; direct FP64 fallback on a residual miss */
};

#define MBD_N_FREQ 21             /* omega = 0 plus 20 Gauss-Legendre points, UTILS.f90:1188-1211 */

typedef struct mbd_ctx mbd_ctx;

/* One geometry plus its settings (the module globals of UTILS.f90:18-49). */
typedef struct {
    int n_atoms;
    const int* z;                 /* [n_atoms] atomic numbers (get_vdw_param's atom_name) */
    const double* coords_bohr;    /* [3*n_atoms] column-major coords(3,N), bohr (after MBD_rsSCS.f90:211) */
    const double* hirshfeld;      /* [n_atoms] Hirshfeld volume ratios */
    int n_periodic;               /* 0 = cluster, >0 = periodic (MBD_rsSCS.f90:83) */
    const double* lattice_bohr;   /* [9] column-major lattice_vector(3,3), columns = vectors, bohr;
                                     ignored when n_periodic == 0 (may be NULL) */
    double scs_cut_A;             /* mbd_scs_dip_cutoff, Angstrom (default 120) */
    double cfdm_cut_A;            /* mbd_cfdm_dip_cutoff, Angstrom (default 100) */
    double sc_cut_A;              /* mbd_supercell_cutoff, Angstrom (default 25) */
    int vacuum[3];                /* mbd_scs_vacuum_axis, 0/1 */
    int xc;                       /* flag_xc: 1 PBE, 2 PBE0, 3 HSE, other -> beta = 1 */
} mbd_geom;

/* Results of one geometry.  Array pointers are caller-owned and may be NULL
 * (that output is then skipped). */
typedef struct {
    double energy_Ha;             /* MBD@rsSCS energy, UTILS.f90:858 */
    double c6_mol;                /* system C6, UTILS.f90:288 */
    int nimag;                    /* number of negative CFDM eigenvalues, UTILS.f90:850-863 */
    int status;                   /* MBD_OK or an error code for this geometry */
    int supercell[3];             /* supercell multiplicities, UTILS.f90:1252-1283 */
    int refine_iters;             /* mixed modes: refinement / CG iterations taken (max over freqs) */
    double err_est[3];            /* [0] max relative relay residual ||b-Ax||/||b|| over freqs (FP64),
                                     [1] estimated relative error of alpha_eff,
                                     [2] estimated relative error of C6 */
    double* alpha_eff;            /* [n_atoms] screened static polarizability, UTILS.f90:263 */
    double* c6_eff;               /* [n_atoms] screened C6, UTILS.f90:313 */
    double* alpha_iw;             /* [21*n_atoms] column-major alpha(f,i); row f=0 is alpha_eff,
                                     rows 1..20 are coupled_atom_pol(1:20,:) of UTILS.f90:265 */
    double* molpol_eig;           /* [21*3] column-major eig(f,k) of the molecular polarizability
                                     tensor (DSYEV('V','U'), UTILS.f90:273) */
} mbd_result;

/* Create a context on CUDA device `device`.  Replaces start_mpi/init_blacs
 * (UTILS.f90:97-135): there is no process grid.  Returns MBD_OK or
 * MBD_ERR_DEVICE when the device is not an sm_100 GPU. */
int mbd_rsscs_create(mbd_ctx** ctx, int device);

/* Destroy a context and free its device memory. */
void mbd_rsscs_destroy(mbd_ctx* ctx);

/* One geometry, host buffers in and out: MBD_at_rsSCS (UTILS.f90:153-349).
 * Returns the same code as out->status. */
int mbd_rsscs_energy(mbd_ctx* ctx, const mbd_geom* geom, int mode, mbd_result* out);

/* Many geometries of uneven size in one call (no reference counterpart: the
 * reference handles one geometry per process launch, MBD_rsSCS.f90:1-239).
 * Returns MBD_OK when every geometry succeeded, else the first failing code;
 * per-geometry codes are in out[g].status. */
int mbd_rsscs_energy_batch(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, int mode,
                           mbd_result* out);

/* Split form of mbd_rsscs_energy_batch for callers that keep inputs resident:
 *   upload   copies the geometries to device memory and prepares the work;
 *   compute  runs every kernel on the resident inputs (no host<->device copy);
 *   download copies results into the mbd_result array.
 * The three calls together equal mbd_rsscs_energy_batch. */
int mbd_rsscs_upload(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms);
int mbd_rsscs_compute(mbd_ctx* ctx, int mode);
int mbd_rsscs_download(mbd_ctx* ctx, mbd_result* out);

/* All eigenvalues of a real symmetric n x n matrix in FP64, ascending: the
 * CFDM eigenvalue step on its own (PDSYEV('N','L') at UTILS.f90:835), for
 * callers that build their own Hamiltonian.  H is HOST memory holding the
 * lower triangle in C row-major order, H(i,j) for j <= i at H[i*ld + j]
 * (for a Fortran column-major array that is its upper triangle, UPLO='U');
 * the rest of H is not read.  w (host) receives n eigenvalues.  Device
 * buffers come from (and stay with) the context. */
int mbd_rsscs_eigvalsh(mbd_ctx* ctx, const double* H, int n, int ld, double* w);

/* Eigenvalues and eigenvectors of a real symmetric n x n matrix in FP64: the
 * PDSYEV call of UTILS.f90:835 with JOBZ = 'V' (the reference passes 'N' and
 * discards the eigenvector matrix it allocates at UTILS.f90:771).  H as for
 * mbd_rsscs_eigvalsh (HOST, lower triangle in C row-major order, H(i,j) for
 * j <= i at H[i*ld + j]).  w (host, n) receives the eigenvalues ascending;
 * Z (host, row-major, ldz >= n) the orthonormal eigenvectors as columns:
 * Z[i*ldz + k] is component i of the eigenvector of w[k] (for a Fortran
 * caller, Z's rows are the eigenvectors).  The sign of each vector, and the
 * basis inside a degenerate eigenspace, are the engine's choice. */
int mbd_rsscs_eigh(mbd_ctx* ctx, const double* H, int n, int ld, double* w, double* Z, int ldz);

/* mbd_rsscs_eigvalsh for callers that must not allocate device memory.
 * (No counterpart in the reference: pmbd.x lets ScaLAPACK allocate its work
 * arrays.)  Meant for hosts that own the GPU's memory through their own pool
 * or arena, or run this step where cudaMalloc's implicit synchronisation and
 * latency are not acceptable.  It calls no cudaMalloc/cudaFree and needs no
 * context: all scratch lives in one fixed 4 MiB device array inside the
 * library, which every GPU that loads the library keeps until exit.
 *   H      DEVICE pointer, 16-byte aligned, lower triangle in C row-major
 *          order (H(i,j), j <= i, at H[i*ld + j]); ld even, ld >= n.
 *          OVERWRITTEN by the reduction.
 *   w      DEVICE pointer, n doubles: eigenvalues in ascending order.
 *   stream cudaStream_t (NULL = legacy default stream); the call returns
 *          after the work on it has finished.
 * n must not exceed MBD_NOALLOC_MAX_N (else MBD_ERR_TOO_LARGE).  Every call
 * synchronises `stream` (it reads the kernels' error flag back before it
 * returns), so no call may be made while a stream is being captured.  Calls
 * share the scratch: calls that overlap on the GPU (other streams or
 * threads, same device) race. */
#define MBD_NOALLOC_MAX_N 2048
int mbd_rsscs_eigvalsh_noalloc(double* H, int n, int ld, double* w, void* stream);

/* Fortran-friendly helpers. */
int mbd_rsscs_element_z(const char* symbol);   /* "C" -> 6; 0 if no vdW parameters (UTILS.f90:1336-1701) */
/* The 21 imaginary frequencies (Hartree; omega = 0 first) and Casimir-Polder
 * weights the engine integrates with: gauss_legendre_grid (UTILS.f90:1188-1211,
 * REAL*4 literals widened to double), as the report prints them
 * (UTILS.f90:278).  weight may be NULL; n must be >= MBD_N_FREQ. */
int mbd_rsscs_frequency_grid(double* omega, double* weight, int n);
const char* mbd_rsscs_strerror(int code);
/* Free-atom table entry: alpha0, C6, R0 as the reference stores them
 * (REAL*4 literals widened to double).  Returns MBD_ERR_UNKNOWN_ELEMENT for
 * elements without parameters. */
int mbd_rsscs_vdw_params(int z, double* alpha0, double* c6, double* r0);

/* Device time in milliseconds of the last mbd_rsscs_compute, per stage:
 * [0] total, [1] atom/frequency setup, [2] relay tensor build, [3] relay
 * factorisation, [4] relay solve/refinement + epilogue, [5] CFDM build,
 * [6] tridiagonal reduction, [7] eigenvalues + energy.  Stages [1]-[5] run
 * per geometry, several geometries at once on separate streams, and are
 * summed over the geometries (their sum can exceed [0]).  [6] is the sum over
 * geometries of the dense -> band reduction (also per geometry, on the same
 * streams) plus the batch-wide band -> tridiagonal launch; [7] is batch-wide.
 * With n >= 10 also [8] the dense -> band part of [6] and [9] the rest;
 * with n >= 12 also [10] the one-stage (dense -> tridiagonal) launch of the
 * matrices that skip the band and [11] the band -> tridiagonal launch, the
 * two batch-wide launches [9] is made of.  n must be >= 8. */
int mbd_rsscs_last_timings(mbd_ctx* ctx, double* ms, int n);

/* Counters of the last upload/compute/download: [0] kernel launches issued
 * by mbd_rsscs_compute, [1] host->device bytes copied by mbd_rsscs_upload,
 * [2] device->host bytes copied by mbd_rsscs_download, [3] (n >= 4) how the
 * last compute ran: 1 replay of the batch's captured CUDA graph, 0 the
 * kernels launched one by one, 2 the batch's first compute in the mode as a
 * graph.  The first compute of an uploaded batch launches directly (with
 * MBD_B200_GRAPH_UPDATE=1 set, not when the context's previous batch had the
 * same shape: then it is captured and written into the graph kept from that
 * batch by cudaGraphExecUpdate, or instantiated where the update is
 * refused); the second compute captures the graph if needed and replays it
 * from then on; a change of network, option or device buffers starts over,
 * [4] (n >= 5) the edges of the MIXED_LEARNED network's neighbour lists over
 * the batch's geometries (pairs within 5 A, periodic images included, both
 * directions; 0 until a learned compute or training has built them),
 * [5] (n >= 6) first-compute graphs this context has written by
 * cudaGraphExecUpdate since it was created, [6] (n >= 7) the last such
 * update's cudaGraphExecUpdateResult (0 success), [7] (n >= 8) the
 * cudaGraphNodeType of the node a refused update names (-1 none).
 * n must be >= 3. */
int mbd_rsscs_last_stats(mbd_ctx* ctx, double* out, int n);

/* The CUDA stream (cudaStream_t) every kernel of this context runs on, so a
 * caller can record its own events around mbd_rsscs_compute. */
void* mbd_rsscs_stream(mbd_ctx* ctx);

/* ---- options --------------------------------------------------------------
 * (No counterpart in the reference, which ignores PDPOTRF's info at
 * UTILS.f90:469 and has no device waits.)  Failure handling of the engine:
 *   MBD_OPT_RESIDUAL_GATE    relative relay residual ||B - A X||_F / ||B||_F
 *                            that the MIXED and MIXED_LEARNED solves must reach
 *                            at every frequency for their result to be used
 *                            (default 1e-10).  A geometry that misses it is
 *                            recomputed with the direct FP64 solve, and its
 *                            mbd_result.refine_iters is -1.  0 sends every
 *                            geometry to that fallback.
 *   MBD_OPT_WAIT_LIMIT_S     seconds a bounded device-side wait (flag polls,
 *                            group barriers, mbarrier waits) may spin before
 *                            the launch gives up and the compute reports
 *                            MBD_ERR_TIMEOUT (default 2; 0 < value <= 60).
 *                            Per device: shared by every context on it.
 *   MBD_OPT_TEST_STALL_WAIT  1: the batch's band -> tridiagonal launch makes
 *                            its first sweep wait for a count that no sweep
 *                            reaches, so that its bounded wait runs out and the
 *                            compute reports MBD_ERR_TIMEOUT; the context stays
 *                            usable.  For testing failure detection; 0 (the
 *                            default) turns it off.
 *   MBD_OPT_FP32_TENSOR_BUILD 1: MIXED and MIXED_LEARNED build the short-range
 *                            dipole tensors of the relay matrices in FP32
 *                            arithmetic from FP64 pair displacements (the
 *                            image set is still selected in FP64); the FP64
 *                            refinement then solves that FP32-valued system.
 *                            0 (the default): FP64 arithmetic in every mode.
 * set_option returns MBD_ERR_ARG for an unknown option or a value out of range. */
enum {
    MBD_OPT_RESIDUAL_GATE = 1,
    MBD_OPT_WAIT_LIMIT_S = 2,
    MBD_OPT_TEST_STALL_WAIT = 3,
    MBD_OPT_FP32_TENSOR_BUILD = 4
};
int mbd_rsscs_set_option(mbd_ctx* ctx, int option, double value);
int mbd_rsscs_get_option(mbd_ctx* ctx, int option, double* value);

/* ---- autotuner -------------------------------------------------------------
 * (No counterpart in the reference, whose ScaLAPACK block sizes are fixed,
 * UTILS.f90:451-452, 813-831.)  Times the eigen stages' launch shapes on
 * synthetic symmetric matrices generated on the device, for every size class
 * n <= 512 * 2^k up to max_n (the largest Hamiltonian dimension 3 N n_SL the
 * caller will compute): the dense -> band panel QR (per-column Householder or
 * TSQR with Householder reconstruction) and its rows per CTA (48 .. 384), and
 * the band -> tridiagonal chase (flag-synchronised, or cluster-resident at
 * each cluster size); keeps the fastest per class in the context for its
 * later computes and eigenvalue calls.  Allocates and frees its own test
 * matrices; takes a few seconds up to n = 6000.  Call it before upload (a
 * batch uploaded before keeps working: its captured graphs are dropped).
 * mbd_rsscs_tuning writes, per class k = 0 .. 7, out[8k .. 8k+7] = {size
 * timed, panel rows per CTA, chase (cluster CTAs, or -1: flag-synchronised),
 * dense -> band ms, chase ms, panel QR (0 Householder, 1 TSQR, -1 not tuned),
 * flag-synchronised chase ms, best cluster-resident chase ms} (n >= 64) and
 * returns the number of classes up to the last tuned one. */
int mbd_rsscs_autotune(mbd_ctx* ctx, int max_n);
int mbd_rsscs_tuning(mbd_ctx* ctx, double* out, int n);

/* ---- learned warm start of MBD_MODE_MIXED_LEARNED -----------------------
 * (No counterpart in the reference, which solves the relay system directly
 * at UTILS.f90:469-473.)  A message-passing network (3 layers, 64 hidden,
 * FP32; atoms within 5 A are neighbours) predicts each atom's 3x3 block
 * X_i = sum_j (A^-1)_ij of the relay solution for every frequency; block
 * conjugate gradients start from it.  The context owns the network. */

/* Number of FP32 network parameters (the layout of *_params). */
int mbd_rsscs_learned_param_count(void);

/* Trains the network on the GPU: uploads the geometries (REPLACING the
 * context's uploaded batch), solves their relay systems with the plain FP64
 * direct solve, and runs `epochs` passes of Adam (learning rate lr, one
 * geometry per step, order shuffled with `seed`) on the mean squared error of
 * the predicted blocks X_i / alpha_i.  epoch_loss (may be NULL) receives the
 * mean loss of each epoch. */
int mbd_rsscs_learned_train(mbd_ctx* ctx, int n_geom, const mbd_geom* geoms, int epochs, double lr,
                            int seed, double* epoch_loss);

/* Copy the parameters out of / into the context (n = param_count). */
int mbd_rsscs_learned_get_params(mbd_ctx* ctx, float* params, int n);
int mbd_rsscs_learned_set_params(mbd_ctx* ctx, const float* params, int n);

/* on = 0: MIXED_LEARNED starts block-CG from zero (the method without the
 * network); on = 1 (default): from the network's prediction. */
int mbd_rsscs_learned_use_network(mbd_ctx* ctx, int on);

/* The network's kernels on caller-given inputs, for checking them against a
 * CPU restatement: n_atoms atoms, n_freq frequency copies, CSR neighbour lists
 * off[n_atoms + 1] / nbr[off[n_atoms]] with displacement vectors dvec (bohr,
 * 3 per edge, r_nbr - r_atom), node inputs x[n_freq * n_atoms][8].  Writes the
 * predicted blocks S_pred[n_freq * n_atoms][9]; with S_true and grad given,
 * also the loss (mean over nodes of ||S - S_true||_F^2) and its gradient
 * with respect to params.  Host pointers; the context's network is not used. */
int mbd_rsscs_learned_eval(mbd_ctx* ctx, const float* params, int n_atoms, int n_freq, const int* off,
                           const int* nbr, const float* dvec, const float* x, const float* S_true,
                           float* S_pred, float* grad, double* loss);

#ifdef __cplusplus
}
#endif
#endif /* MBD_B200_H */
