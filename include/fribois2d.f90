! fribois2d.f90 -- ISO_C_BINDING interface to the C ABI in fribois2d.h.
!
! What a FRiBoIS2D maintainer adds to the reference to replace fluid_tsch
! (src/fluid_tsch.F90:4) and rigid (src/rigid.F90:4), and the set-up calls
! of src/main.F90:51-62, with one GPU.  Every function returns an integer
! status (FB_OK = 0) where the reference calls stopcase/MPI_ABORT.  Fields are
! the reference's column-major A(j,k), j = 1..n2 contiguous, k = 0..n3.
! Strings passed in must end with c_null_char.  Link with
!   -L<repo>/fribois2d_b200 -lfribois2d -Wl,-rpath,<repo>/fribois2d_b200
module fribois2d_gpu
  use iso_c_binding
  implicit none

  ! status codes
  integer(c_int), parameter :: FB_OK = 0, FB_ERR_CFL = 1, FB_ERR_MLS = 2, FB_ERR_MARKER_OUT = 3, &
       FB_ERR_INPUT = 4, FB_ERR_CUDA = 5, FB_ERR_STATE = 6, FB_ERR_UNSUPPORTED = 7, &
       FB_ERR_NUMERIC = 8, FB_ERR_TIMEOUT = 9
  ! array ids (fb_get_array / fb_set_array / fb_host_array)
  integer(c_int), parameter :: FB_Q2 = 0, FB_Q3 = 1, FB_PR = 2, FB_DPH = 3, FB_RHS2 = 7, FB_RHS3 = 8, &
       FB_RU2 = 9, FB_RU3 = 10
  integer(c_int), parameter :: FB_QB2S = 20, FB_QB2N = 21, FB_DQB2S = 22, FB_DQB2N = 23, FB_QB3S = 24, &
       FB_QB3N = 25, FB_DQB3S = 26, FB_DQB3N = 27, FB_DQ2X2O = 28, FB_DQ3X2O = 29
  integer(c_int), parameter :: FB_RC = 40, FB_RM = 41, FB_ZZ = 42, FB_ZM = 43, FB_UDX2C = 48, &
       FB_UDX2M = 49, FB_UDX3C = 50, FB_UDX3M = 51, FB_AMPHJ = 64, FB_ACPHJ = 65, FB_APPHJ = 66, &
       FB_AMPHK = 67, FB_ACPHK = 68, FB_APPHK = 69, FB_WR = 80, FB_ZMM = 81, FB_ZMMT = 82
  integer(c_int), parameter :: FB_LMCC = 90, FB_LMVEL = 91, FB_LMACC = 92, FB_LMNOR = 93, FB_LMA = 94, &
       FB_VERT = 95, FB_PHI = 96, FB_CL = 97, FB_PRESS = 98, FB_TAU = 99, FB_BCERRV = 100, &
       FB_BCERRW = 101, FB_RIGID = 110, FB_SCALARS = 111, FB_FORCES = 112, FB_HMN = 113
  integer(c_int), parameter :: FB_LMIND = 0, FB_EULINS = 1
  integer(c_int), parameter :: FB_HIST_COLS = 31
  ! stage ids (fb_stage), one per reference subroutine
  integer(c_int), parameter :: FB_ST_CFL = 0, FB_ST_BOUCDQ = 1, FB_ST_NL_RHS = 2, FB_ST_LGRDIST = 6, &
       FB_ST_FORCING = 7, FB_ST_HELSOLVE = 8, FB_ST_DIVG = 9, FB_ST_PHCALC = 10, FB_ST_UPDVP = 11, &
       FB_ST_PRSUBMEAN = 13, FB_ST_CHECKBCS = 15, FB_ST_LOADS = 16, FB_ST_RIGID = 17
  integer(c_int), parameter :: FB_TK_GEMM_FWD = 100, FB_TK_POISSON_TRI = 101, FB_TK_GEMM_BWD = 102, &
       FB_TK_TF32X3_GEMM = 103, FB_TK_I8_SPLIT = 104, FB_TK_I8X8_GEMM = 105
  ! options without a counterpart in the reference
  integer(c_int), parameter :: FB_BATCH_GROUPED = 0, FB_BATCH_GRAPH = 1
  integer(c_int), parameter :: FB_COUPLING_LOOSE = 0, FB_COUPLING_STRONG = 1, FB_COUPLING_LEARNED = 2
  integer(c_int), parameter :: FB_POISSON_FP64 = 0, FB_POISSON_TF32X3 = 1, FB_POISSON_INT8X8 = 2
  integer(c_int), parameter :: FB_NOALLOC_MAX_ROWS = 8192

  interface
    ! ---- set-up and the main loop body (main.F90:51-97)
    integer(c_int) function fb_create(input_dir, device, ctx) bind(C, name="fb_create")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: input_dir
      integer(c_int), value :: device
      type(c_ptr), intent(out) :: ctx
    end function
    integer(c_int) function fb_destroy(ctx) bind(C, name="fb_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function fb_fluid_tsch(ctx, ns) bind(C, name="fb_fluid_tsch")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: ns
    end function
    integer(c_int) function fb_rigid(ctx, ns, forcecomp) bind(C, name="fb_rigid")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ns
      real(c_double), dimension(8), intent(out) :: forcecomp
    end function
    integer(c_int) function fb_advance(ctx, ns0, nsteps, hist) bind(C, name="fb_advance")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ns0, nsteps
      real(c_double), dimension(*), intent(out) :: hist
    end function
    integer(c_int) function fb_get_loads(ctx, press, tau) bind(C, name="fb_get_loads")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(out) :: press, tau
    end function
    integer(c_int) function fb_set_markers(ctx, lmcc, lmvel, lmacc, lmnor) bind(C, name="fb_set_markers")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(in) :: lmcc, lmvel, lmacc, lmnor
    end function
    integer(c_int) function fb_get_markers(ctx, lmcc, lmvel, lmacc, lmnor) bind(C, name="fb_get_markers")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(out) :: lmcc, lmvel, lmacc, lmnor
    end function
    integer(c_int) function fb_step_markers(ctx, ns, lmcc, lmvel, lmacc, lmnor, forcecomp) &
        bind(C, name="fb_step_markers")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: ns
      real(c_double), dimension(*), intent(inout) :: lmcc, lmvel, lmacc, lmnor
      real(c_double), dimension(8), intent(out) :: forcecomp
    end function
    integer(c_int) function fb_last_history(ctx, row) bind(C, name="fb_last_history")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(*), intent(out) :: row
    end function
    integer(c_int) function fb_set_report(ctx, on) bind(C, name="fb_set_report")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: on
    end function

    ! ---- batches of independent cases
    integer(c_int) function fb_batch_create(ctxs, n, batch) bind(C, name="fb_batch_create")
      import :: c_int, c_ptr
      type(c_ptr), dimension(*), intent(in) :: ctxs
      integer(c_int), value :: n
      type(c_ptr), intent(out) :: batch
    end function
    integer(c_int) function fb_batch_create_mode(ctxs, n, mode, batch) bind(C, name="fb_batch_create_mode")
      import :: c_int, c_ptr
      type(c_ptr), dimension(*), intent(in) :: ctxs
      integer(c_int), value :: n, mode
      type(c_ptr), intent(out) :: batch
    end function
    integer(c_int) function fb_batch_advance(batch, nsteps) bind(C, name="fb_batch_advance")
      import :: c_int, c_ptr
      type(c_ptr), value :: batch
      integer(c_int), value :: nsteps
    end function
    integer(c_int) function fb_batch_last_ms(batch, ms) bind(C, name="fb_batch_last_ms")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: batch
      real(c_double), intent(out) :: ms
    end function
    integer(c_int) function fb_batch_info(batch, info) bind(C, name="fb_batch_info")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: batch
      integer(c_int32_t), dimension(3), intent(out) :: info
    end function
    integer(c_int) function fb_batch_destroy(batch) bind(C, name="fb_batch_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: batch
    end function

    ! ---- strong coupling and the learned predictor
    integer(c_int) function fb_set_coupling(ctx, mode, tol, max_iter) bind(C, name="fb_set_coupling")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: mode
      real(c_double), value :: tol
      integer(c_int), value :: max_iter
    end function
    integer(c_int) function fb_set_predictor(ctx, mlp, norm) bind(C, name="fb_set_predictor")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx, mlp
      real(c_float), dimension(*), intent(in) :: norm
    end function
    integer(c_int) function fb_coupling_stats(ctx, out) bind(C, name="fb_coupling_stats")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), dimension(4), intent(out) :: out
    end function
    integer(c_int) function fb_coupling_samples(ctx, x, t, cap, n) bind(C, name="fb_coupling_samples")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: ctx
      real(c_float), dimension(*), intent(out) :: x, t
      integer(c_int), value :: cap
      integer(c_int), intent(out) :: n
    end function
    integer(c_int) function fb_mlp_create(device, n_in, n_out, seed, mlp) bind(C, name="fb_mlp_create")
      import :: c_int, c_ptr, c_int64_t
      integer(c_int), value :: device, n_in, n_out
      integer(c_int64_t), value :: seed
      type(c_ptr), intent(out) :: mlp
    end function
    integer(c_int) function fb_mlp_destroy(mlp) bind(C, name="fb_mlp_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: mlp
    end function
    integer(c_int) function fb_mlp_params(mlp, n) bind(C, name="fb_mlp_params")
      import :: c_int, c_ptr
      type(c_ptr), value :: mlp
      integer(c_int), intent(out) :: n
    end function
    integer(c_int) function fb_mlp_get(mlp, params) bind(C, name="fb_mlp_get")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: mlp
      real(c_float), dimension(*), intent(out) :: params
    end function
    integer(c_int) function fb_mlp_set(mlp, params) bind(C, name="fb_mlp_set")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: mlp
      real(c_float), dimension(*), intent(in) :: params
    end function
    integer(c_int) function fb_mlp_predict(mlp, x, n, y) bind(C, name="fb_mlp_predict")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: mlp
      real(c_float), dimension(*), intent(in) :: x
      integer(c_int), value :: n
      real(c_float), dimension(*), intent(out) :: y
    end function
    integer(c_int) function fb_mlp_grad(mlp, x, t, n, grad, loss) bind(C, name="fb_mlp_grad")
      import :: c_int, c_ptr, c_float
      type(c_ptr), value :: mlp
      real(c_float), dimension(*), intent(in) :: x, t
      integer(c_int), value :: n
      real(c_float), dimension(*), intent(out) :: grad
      real(c_float), intent(out) :: loss
    end function
    integer(c_int) function fb_mlp_train(mlp, x, t, n, epochs, batch, lr, seed, loss) bind(C, name="fb_mlp_train")
      import :: c_int, c_ptr, c_float, c_int64_t
      type(c_ptr), value :: mlp
      real(c_float), dimension(*), intent(in) :: x, t
      integer(c_int), value :: n, epochs, batch
      real(c_float), value :: lr
      integer(c_int64_t), value :: seed
      real(c_float), dimension(*), intent(out) :: loss
    end function

    ! ---- checkpoint / restart (mpi_routines.F90:532-806, iobcs.F90:114-205)
    integer(c_int) function fb_write_restart(ctx, dir) bind(C, name="fb_write_restart")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), dimension(*), intent(in) :: dir
    end function
    integer(c_int) function fb_read_restart(ctx, dir) bind(C, name="fb_read_restart")
      import :: c_int, c_ptr, c_char
      type(c_ptr), value :: ctx
      character(kind=c_char), dimension(*), intent(in) :: dir
    end function

    ! ---- state access
    integer(c_int) function fb_get_dims(ctx, dims) bind(C, name="fb_get_dims")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), dimension(8), intent(out) :: dims
    end function
    integer(c_int) function fb_get_array(ctx, id, host, n) bind(C, name="fb_get_array")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: id
      real(c_double), dimension(*), intent(out) :: host
      integer(c_int64_t), value :: n
    end function
    integer(c_int) function fb_set_array(ctx, id, host, n) bind(C, name="fb_set_array")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: id
      real(c_double), dimension(*), intent(in) :: host
      integer(c_int64_t), value :: n
    end function
    integer(c_int) function fb_get_iarray(ctx, id, host, n) bind(C, name="fb_get_iarray")
      import :: c_int, c_ptr, c_int32_t, c_int64_t
      type(c_ptr), value :: ctx
      integer(c_int), value :: id
      integer(c_int32_t), dimension(*), intent(out) :: host
      integer(c_int64_t), value :: n
    end function
    integer(c_int) function fb_synchronize(ctx) bind(C, name="fb_synchronize")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function fb_set_substep(ctx, ns, n) bind(C, name="fb_set_substep")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: ns, n
    end function
    integer(c_int) function fb_stage(ctx, stage, n) bind(C, name="fb_stage")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: stage, n
    end function

    ! ---- timing
    integer(c_int) function fb_last_advance_ms(ctx, ms) bind(C, name="fb_last_advance_ms")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: ms
    end function
    integer(c_int) function fb_time_stage(ctx, stage, n, reps, ms) bind(C, name="fb_time_stage")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: stage, n, reps
      real(c_double), intent(out) :: ms
    end function
    integer(c_int) function fb_kernel_count(ctx, per_step) bind(C, name="fb_kernel_count")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), intent(out) :: per_step
    end function

    ! ---- Poisson transform forms and the tile autotuner
    integer(c_int) function fb_set_poisson(ctx, mode) bind(C, name="fb_set_poisson")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: mode
    end function
    integer(c_int) function fb_set_refinement(ctx, sweeps) bind(C, name="fb_set_refinement")
      import :: c_int, c_ptr
      type(c_ptr), value :: ctx
      integer(c_int), value :: sweeps
    end function
    integer(c_int) function fb_gemm_i8x8(device, m, n, k, a, b, c) bind(C, name="fb_gemm_i8x8")
      import :: c_int, c_double
      integer(c_int), value :: device, m, n, k
      real(c_double), dimension(*), intent(in) :: a, b
      real(c_double), dimension(*), intent(out) :: c
    end function
    integer(c_int) function fb_gemm_tf32x3(device, m, n, k, bn, a, b, c) bind(C, name="fb_gemm_tf32x3")
      import :: c_int, c_double
      integer(c_int), value :: device, m, n, k, bn
      real(c_double), dimension(*), intent(in) :: a, b
      real(c_double), dimension(*), intent(out) :: c
    end function
    integer(c_int) function fb_autotune(ctx, choice) bind(C, name="fb_autotune")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: ctx
      integer(c_int32_t), dimension(2), intent(out) :: choice
    end function

    ! ---- host-only set-up (no GPU)
    integer(c_int) function fb_host_create(input_dir, h) bind(C, name="fb_host_create")
      import :: c_int, c_char, c_ptr
      character(kind=c_char), dimension(*), intent(in) :: input_dir
      type(c_ptr), intent(out) :: h
    end function
    integer(c_int) function fb_host_destroy(h) bind(C, name="fb_host_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function
    integer(c_int) function fb_host_dims(h, dims) bind(C, name="fb_host_dims")
      import :: c_int, c_ptr, c_int32_t
      type(c_ptr), value :: h
      integer(c_int32_t), dimension(8), intent(out) :: dims
    end function
    integer(c_int) function fb_host_array(h, id, out, n) bind(C, name="fb_host_array")
      import :: c_int, c_ptr, c_double, c_int64_t
      type(c_ptr), value :: h
      integer(c_int), value :: id
      real(c_double), dimension(*), intent(out) :: out
      integer(c_int64_t), value :: n
    end function
    integer(c_int) function fb_eigen_tridiag(n, am, ac, ap, wr, zmm, zmmt) bind(C, name="fb_eigen_tridiag")
      import :: c_int, c_double
      integer(c_int), value :: n
      real(c_double), dimension(*), intent(in) :: am, ac, ap
      real(c_double), dimension(*), intent(out) :: wr, zmm, zmmt
    end function

    ! ---- CFL number from the caller's device arrays, nothing allocated
    !      (q2 .. udx3m and out are device addresses, e.g. c_loc of CUDA
    !      Fortran device arrays or OpenACC host_data use_device)
    integer(c_int) function fb_cfl_noalloc(q2, q3, pitch, n2, n3, rc, zz, udx2m, udx3m, dt, rext2, alx3, &
                                           out, stream) bind(C, name="fb_cfl_noalloc")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: q2, q3
      integer(c_int), value :: pitch, n2, n3
      type(c_ptr), value :: rc, zz, udx2m, udx3m
      real(c_double), value :: dt, rext2, alx3
      type(c_ptr), value :: out, stream
    end function

    ! ---- messages (C strings; convert with c_f_pointer)
    type(c_ptr) function fb_status_string(st) bind(C, name="fb_status_string")
      import :: c_int, c_ptr
      integer(c_int), value :: st
    end function
    type(c_ptr) function fb_version() bind(C, name="fb_version")
      import :: c_ptr
    end function
  end interface
end module fribois2d_gpu
