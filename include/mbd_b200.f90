! mbd_b200.f90 -- Fortran 2003 binding of the C ABI in mbd_b200.h.
!
! For a Fortran host such as pmbd.x: USE mbd_b200_c and call the engine in
! place of the physics entered at MBD_rsSCS.f90:218-221 (CALL init_blacs();
! CALL MBD_at_rsSCS(ene)).  The derived types are BIND(C) copies of mbd_geom
! and mbd_result, component for component, so the host fills them with
! C_LOC of its own arrays (coords(3,N), lattice_vector(3,3), alpha_iw(21,N),
! molpol_eig(21,3) keep their Fortran layout) and passes them by reference.
! Link with -L<repo>/mbd_b200 -lmbd_b200.  No Fortran compiler is present
! where this library is built, so this file is not compiled here; the names
! it binds are checked against the library's exports by the CPU tests.
MODULE mbd_b200_c
  USE, INTRINSIC :: iso_c_binding
  IMPLICIT NONE

  ! status codes (MBD_OK and MBD_ERR_* of mbd_b200.h)
  INTEGER(c_int), PARAMETER :: MBD_OK = 0, MBD_ERR_ARG = 1, MBD_ERR_UNKNOWN_ELEMENT = 2, &
                               MBD_ERR_RELAY_NOT_SPD = 3, MBD_ERR_NONPOSITIVE_ALPHA = 4, &
                               MBD_ERR_EIGENSOLVER = 5, MBD_ERR_DEVICE = 6, MBD_ERR_TIMEOUT = 7, &
                               MBD_ERR_OUT_OF_MEMORY = 8, MBD_ERR_REFINEMENT = 9, &
                               MBD_ERR_NOT_BUILT = 10, MBD_ERR_TOO_LARGE = 11, &
                               MBD_ERR_NO_NETWORK = 12
  ! compute modes
  INTEGER(c_int), PARAMETER :: MBD_MODE_PLAIN_FP64 = 0, MBD_MODE_MIXED = 1, &
                               MBD_MODE_MIXED_LEARNED = 2
  INTEGER(c_int), PARAMETER :: MBD_N_FREQ = 21
  ! options of mbd_rsscs_set_option / mbd_rsscs_get_option
  INTEGER(c_int), PARAMETER :: MBD_OPT_RESIDUAL_GATE = 1, MBD_OPT_WAIT_LIMIT_S = 2, &
                               MBD_OPT_TEST_STALL_WAIT = 3, MBD_OPT_FP32_TENSOR_BUILD = 4

  ! one geometry and its settings (the module globals of UTILS.f90:18-49)
  TYPE, BIND(C) :: mbd_geom
    INTEGER(c_int) :: n_atoms
    TYPE(c_ptr)    :: z             ! INTEGER(c_int) z(n_atoms): atomic numbers
    TYPE(c_ptr)    :: coords_bohr   ! REAL(c_double) coords(3,n_atoms), bohr
    TYPE(c_ptr)    :: hirshfeld     ! REAL(c_double) hirshfeld_volume(n_atoms)
    INTEGER(c_int) :: n_periodic
    TYPE(c_ptr)    :: lattice_bohr  ! REAL(c_double) lattice_vector(3,3), columns = vectors
    REAL(c_double) :: scs_cut_A, cfdm_cut_A, sc_cut_A   ! Angstrom, as in setting.in
    INTEGER(c_int) :: vacuum(3)     ! mbd_scs_vacuum_axis as 0/1
    INTEGER(c_int) :: xc            ! flag_xc
  END TYPE mbd_geom

  ! the results of one geometry; array pointers may be C_NULL_PTR
  TYPE, BIND(C) :: mbd_result
    REAL(c_double) :: energy_Ha, c6_mol
    INTEGER(c_int) :: nimag, status, supercell(3), refine_iters
    REAL(c_double) :: err_est(3)
    TYPE(c_ptr)    :: alpha_eff     ! REAL(c_double) alpha_eff(n_atoms)
    TYPE(c_ptr)    :: c6_eff        ! REAL(c_double) C6_eff(n_atoms)
    TYPE(c_ptr)    :: alpha_iw      ! REAL(c_double) alpha_iw(21,n_atoms)
    TYPE(c_ptr)    :: molpol_eig    ! REAL(c_double) molpol_eig(21,3)
  END TYPE mbd_result

  INTERFACE
    INTEGER(c_int) FUNCTION mbd_rsscs_create(ctx, device) BIND(C, NAME='mbd_rsscs_create')
      IMPORT :: c_int, c_ptr
      TYPE(c_ptr), INTENT(OUT) :: ctx
      INTEGER(c_int), VALUE :: device
    END FUNCTION mbd_rsscs_create

    SUBROUTINE mbd_rsscs_destroy(ctx) BIND(C, NAME='mbd_rsscs_destroy')
      IMPORT :: c_ptr
      TYPE(c_ptr), VALUE :: ctx
    END SUBROUTINE mbd_rsscs_destroy

    INTEGER(c_int) FUNCTION mbd_rsscs_energy(ctx, geom, mode, res) BIND(C, NAME='mbd_rsscs_energy')
      IMPORT :: c_int, c_ptr, mbd_geom, mbd_result
      TYPE(c_ptr), VALUE :: ctx
      TYPE(mbd_geom), INTENT(IN) :: geom
      INTEGER(c_int), VALUE :: mode
      TYPE(mbd_result), INTENT(INOUT) :: res
    END FUNCTION mbd_rsscs_energy

    INTEGER(c_int) FUNCTION mbd_rsscs_energy_batch(ctx, n_geom, geoms, mode, res) &
        BIND(C, NAME='mbd_rsscs_energy_batch')
      IMPORT :: c_int, c_ptr, mbd_geom, mbd_result
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: n_geom
      TYPE(mbd_geom), INTENT(IN) :: geoms(*)
      INTEGER(c_int), VALUE :: mode
      TYPE(mbd_result), INTENT(INOUT) :: res(*)
    END FUNCTION mbd_rsscs_energy_batch

    INTEGER(c_int) FUNCTION mbd_rsscs_upload(ctx, n_geom, geoms) BIND(C, NAME='mbd_rsscs_upload')
      IMPORT :: c_int, c_ptr, mbd_geom
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: n_geom
      TYPE(mbd_geom), INTENT(IN) :: geoms(*)
    END FUNCTION mbd_rsscs_upload

    INTEGER(c_int) FUNCTION mbd_rsscs_compute(ctx, mode) BIND(C, NAME='mbd_rsscs_compute')
      IMPORT :: c_int, c_ptr
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: mode
    END FUNCTION mbd_rsscs_compute

    INTEGER(c_int) FUNCTION mbd_rsscs_download(ctx, res) BIND(C, NAME='mbd_rsscs_download')
      IMPORT :: c_int, c_ptr, mbd_result
      TYPE(c_ptr), VALUE :: ctx
      TYPE(mbd_result), INTENT(INOUT) :: res(*)
    END FUNCTION mbd_rsscs_download

    ! h: the lower triangle in C row-major order, i.e. a Fortran h(ld,n)'s
    ! upper triangle (UPLO = 'U'); w(n) ascending
    INTEGER(c_int) FUNCTION mbd_rsscs_eigvalsh(ctx, h, n, ld, w) BIND(C, NAME='mbd_rsscs_eigvalsh')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_double), INTENT(IN) :: h(*)
      INTEGER(c_int), VALUE :: n, ld
      REAL(c_double), INTENT(OUT) :: w(*)
    END FUNCTION mbd_rsscs_eigvalsh

    ! as mbd_rsscs_eigvalsh, plus the eigenvectors as the rows of a Fortran
    ! z(ldz,n) (the columns of the C row-major array)
    INTEGER(c_int) FUNCTION mbd_rsscs_eigh(ctx, h, n, ld, w, z, ldz) BIND(C, NAME='mbd_rsscs_eigh')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_double), INTENT(IN) :: h(*)
      INTEGER(c_int), VALUE :: n, ld
      REAL(c_double), INTENT(OUT) :: w(*), z(*)
      INTEGER(c_int), VALUE :: ldz
    END FUNCTION mbd_rsscs_eigh

    ! device pointers (h, w) and a cudaStream_t (C_NULL_PTR: the legacy stream)
    INTEGER(c_int) FUNCTION mbd_rsscs_eigvalsh_noalloc(h, n, ld, w, stream) &
        BIND(C, NAME='mbd_rsscs_eigvalsh_noalloc')
      IMPORT :: c_int, c_ptr
      TYPE(c_ptr), VALUE :: h
      INTEGER(c_int), VALUE :: n, ld
      TYPE(c_ptr), VALUE :: w, stream
    END FUNCTION mbd_rsscs_eigvalsh_noalloc

    INTEGER(c_int) FUNCTION mbd_rsscs_element_z(symbol) BIND(C, NAME='mbd_rsscs_element_z')
      IMPORT :: c_int, c_char
      CHARACTER(KIND=c_char), INTENT(IN) :: symbol(*)   ! NUL-terminated
    END FUNCTION mbd_rsscs_element_z

    INTEGER(c_int) FUNCTION mbd_rsscs_frequency_grid(omega, weight, n) &
        BIND(C, NAME='mbd_rsscs_frequency_grid')
      IMPORT :: c_int, c_double
      REAL(c_double), INTENT(OUT) :: omega(*), weight(*)
      INTEGER(c_int), VALUE :: n
    END FUNCTION mbd_rsscs_frequency_grid

    TYPE(c_ptr) FUNCTION mbd_rsscs_strerror(code) BIND(C, NAME='mbd_rsscs_strerror')
      IMPORT :: c_int, c_ptr
      INTEGER(c_int), VALUE :: code
    END FUNCTION mbd_rsscs_strerror

    INTEGER(c_int) FUNCTION mbd_rsscs_vdw_params(z, alpha0, c6, r0) BIND(C, NAME='mbd_rsscs_vdw_params')
      IMPORT :: c_int, c_double
      INTEGER(c_int), VALUE :: z
      REAL(c_double), INTENT(OUT) :: alpha0, c6, r0
    END FUNCTION mbd_rsscs_vdw_params

    INTEGER(c_int) FUNCTION mbd_rsscs_set_option(ctx, option, val) BIND(C, NAME='mbd_rsscs_set_option')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: option
      REAL(c_double), VALUE :: val
    END FUNCTION mbd_rsscs_set_option

    INTEGER(c_int) FUNCTION mbd_rsscs_get_option(ctx, option, val) BIND(C, NAME='mbd_rsscs_get_option')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: option
      REAL(c_double), INTENT(OUT) :: val
    END FUNCTION mbd_rsscs_get_option

    INTEGER(c_int) FUNCTION mbd_rsscs_last_timings(ctx, ms, n) BIND(C, NAME='mbd_rsscs_last_timings')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_double), INTENT(OUT) :: ms(*)
      INTEGER(c_int), VALUE :: n
    END FUNCTION mbd_rsscs_last_timings

    ! counters of the last upload / compute / download (launches, bytes,
    ! graph kind, network edges, graph updates): stats(n), n >= 3
    INTEGER(c_int) FUNCTION mbd_rsscs_last_stats(ctx, stats, n) BIND(C, NAME='mbd_rsscs_last_stats')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_double), INTENT(OUT) :: stats(*)
      INTEGER(c_int), VALUE :: n
    END FUNCTION mbd_rsscs_last_stats

    INTEGER(c_int) FUNCTION mbd_rsscs_autotune(ctx, max_n) BIND(C, NAME='mbd_rsscs_autotune')
      IMPORT :: c_int, c_ptr
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: max_n
    END FUNCTION mbd_rsscs_autotune

    ! the autotuner's choices, 8 values per size class: tuning(n), n >= 64
    INTEGER(c_int) FUNCTION mbd_rsscs_tuning(ctx, tuning, n) BIND(C, NAME='mbd_rsscs_tuning')
      IMPORT :: c_int, c_ptr, c_double
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_double), INTENT(OUT) :: tuning(*)
      INTEGER(c_int), VALUE :: n
    END FUNCTION mbd_rsscs_tuning

    INTEGER(c_int) FUNCTION mbd_rsscs_learned_param_count() BIND(C, NAME='mbd_rsscs_learned_param_count')
      IMPORT :: c_int
    END FUNCTION mbd_rsscs_learned_param_count

    INTEGER(c_int) FUNCTION mbd_rsscs_learned_train(ctx, n_geom, geoms, epochs, lr, seed, epoch_loss) &
        BIND(C, NAME='mbd_rsscs_learned_train')
      IMPORT :: c_int, c_ptr, c_double, mbd_geom
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: n_geom
      TYPE(mbd_geom), INTENT(IN) :: geoms(*)
      INTEGER(c_int), VALUE :: epochs
      REAL(c_double), VALUE :: lr
      INTEGER(c_int), VALUE :: seed
      REAL(c_double), INTENT(OUT) :: epoch_loss(*)
    END FUNCTION mbd_rsscs_learned_train

    INTEGER(c_int) FUNCTION mbd_rsscs_learned_get_params(ctx, params, n) &
        BIND(C, NAME='mbd_rsscs_learned_get_params')
      IMPORT :: c_int, c_ptr, c_float
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_float), INTENT(OUT) :: params(*)
      INTEGER(c_int), VALUE :: n
    END FUNCTION mbd_rsscs_learned_get_params

    INTEGER(c_int) FUNCTION mbd_rsscs_learned_set_params(ctx, params, n) &
        BIND(C, NAME='mbd_rsscs_learned_set_params')
      IMPORT :: c_int, c_ptr, c_float
      TYPE(c_ptr), VALUE :: ctx
      REAL(c_float), INTENT(IN) :: params(*)
      INTEGER(c_int), VALUE :: n
    END FUNCTION mbd_rsscs_learned_set_params

    INTEGER(c_int) FUNCTION mbd_rsscs_learned_use_network(ctx, on) BIND(C, NAME='mbd_rsscs_learned_use_network')
      IMPORT :: c_int, c_ptr
      TYPE(c_ptr), VALUE :: ctx
      INTEGER(c_int), VALUE :: on
    END FUNCTION mbd_rsscs_learned_use_network

    INTEGER(c_size_t) FUNCTION c_strlen(s) BIND(C, NAME='strlen')
      IMPORT :: c_size_t, c_ptr
      TYPE(c_ptr), VALUE :: s
    END FUNCTION c_strlen
  END INTERFACE

CONTAINS

  ! atomic number of an element symbol as written in geometry.in
  ! (get_vdw_param's atom_name, UTILS.f90:1336-1701); 0 when unknown
  INTEGER(c_int) FUNCTION mbd_element_z(symbol)
    CHARACTER(LEN=*), INTENT(IN) :: symbol
    mbd_element_z = mbd_rsscs_element_z(TRIM(ADJUSTL(symbol)) // c_null_char)
  END FUNCTION mbd_element_z

  ! the message of a status code as a Fortran string
  FUNCTION mbd_strerror(code) RESULT(msg)
    INTEGER(c_int), INTENT(IN) :: code
    CHARACTER(LEN=:), ALLOCATABLE :: msg
    TYPE(c_ptr) :: p
    CHARACTER(KIND=c_char), POINTER :: chars(:)
    INTEGER :: n, i
    p = mbd_rsscs_strerror(code)
    n = INT(c_strlen(p))
    CALL c_f_pointer(p, chars, [n])
    ALLOCATE(CHARACTER(LEN=n) :: msg)
    DO i = 1, n
      msg(i:i) = chars(i)
    END DO
  END FUNCTION mbd_strerror

END MODULE mbd_b200_c
