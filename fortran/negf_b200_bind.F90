! Uncompiled on this image (no Fortran compiler here): the iso_c_binding
! module a libNEGF build links against libnegf_b200.so with.  Every
! interface mirrors one declaration of include/negf_b200.h; arrays are passed
! as assumed-size actual arguments (by reference), scalars by value.
module negf_b200_bind
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: NEGF_B200_OK = 0, NEGF_B200_ERR_SINGULAR = 1, NEGF_B200_ERR_NOT_CONVERGED = 2, &
      NEGF_B200_ERR_NONFINITE = 3, NEGF_B200_ERR_NOMEM = 4, NEGF_B200_ERR_BAD_ARG = 5, NEGF_B200_ERR_CUDA = 6, &
      NEGF_B200_ERR_TIMEOUT = 7, NEGF_B200_ERR_ADMISSION = 8, NEGF_B200_ERR_NO_GPU = 9, &
      NEGF_B200_ERR_SCBA_NOT_CONVERGED = 10

  ! negf_b200_device: pointers to column-major complex128 block families
  type, bind(C) :: negf_b200_device
    integer(c_int32_t) :: nbl
    type(c_ptr) :: pl_size, h_diag, h_upper, h_lower, s_diag, s_upper, s_lower
    integer(c_int32_t) :: ncont
    type(c_ptr) :: cblk, lead_size, lead_h00, lead_h01, lead_s00, lead_s01, hmc, smc
    type(c_ptr) :: surf_size, lead_hs, lead_ss
  end type

  ! negf_b200_options
  type, bind(C) :: negf_b200_options
    real(c_double) :: sgf_tol
    integer(c_int32_t) :: sgf_max_iter
    real(c_double) :: eps_drop
    real(c_double) :: scba_tol
    integer(c_int32_t) :: scba_niter
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: ctas_per_sm
    real(c_double) :: scba_mix
    integer(c_int32_t) :: scba_rule
    integer(c_int32_t) :: schedule
  end type

  interface
    subroutine negf_b200_default_options(o) bind(C, name='negf_b200_default_options')
      import; type(negf_b200_options) :: o
    end subroutine
    function negf_b200_version() bind(C, name='negf_b200_version')
      import; type(c_ptr) :: negf_b200_version
    end function
    integer(c_int) function negf_b200_ctx_create(dev, ctx) bind(C, name='negf_b200_ctx_create')
      import; integer(c_int32_t), value :: dev; type(c_ptr) :: ctx
    end function
    integer(c_int) function negf_b200_ctx_destroy(ctx) bind(C, name='negf_b200_ctx_destroy')
      import; type(c_ptr), value :: ctx
    end function
    integer(c_int) function negf_b200_set_options(ctx, o) bind(C, name='negf_b200_set_options')
      import; type(c_ptr), value :: ctx; type(negf_b200_options) :: o
    end function
    function negf_b200_last_error(ctx) bind(C, name='negf_b200_last_error')
      import; type(c_ptr), value :: ctx; type(c_ptr) :: negf_b200_last_error
    end function
    integer(c_int) function negf_b200_launch_count(ctx, count) bind(C, name='negf_b200_launch_count')
      import; type(c_ptr), value :: ctx; integer(c_int64_t) :: count
    end function
    integer(c_int) function negf_b200_upload_device(ctx, d, id) bind(C, name='negf_b200_upload_device')
      import; type(c_ptr), value :: ctx; type(negf_b200_device) :: d; integer(c_int32_t) :: id
    end function
    integer(c_int) function negf_b200_release_device(ctx, id) bind(C, name='negf_b200_release_device')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: id
    end function
    integer(c_int) function negf_b200_transmission(ctx, npts, ids, E, eta, ni, nf, T, ncyc, st) &
        bind(C, name='negf_b200_transmission')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: npts, ni, nf
      integer(c_int32_t) :: ids(*), ncyc(*), st(*); real(c_double) :: E(*), T(*); real(c_double), value :: eta
    end function
    integer(c_int) function negf_b200_transmission_dos(ctx, npts, ids, E, eta, dos_delta, ni, nf, T, dos, ncyc, st) &
        bind(C, name='negf_b200_transmission_dos')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: npts, ni, nf
      integer(c_int32_t) :: ids(*), ncyc(*), st(*); real(c_double) :: E(*), T(*), dos(*)
      real(c_double), value :: eta, dos_delta
    end function
    integer(c_int) function negf_b200_meir_wingreen(ctx, npts, ids, E, eta, frm, cpl, curr, lcurr, ldens, &
        it, err, ncyc, st) bind(C, name='negf_b200_meir_wingreen')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: npts; real(c_double), value :: eta
      integer(c_int32_t) :: ids(*), it(*), ncyc(*), st(*)
      real(c_double) :: E(*), frm(*), cpl(*), curr(*), lcurr(*), ldens(*), err(*)
    end function
    integer(c_int) function negf_b200_transmissions(ctx, npts, ids, E, eta, dos_delta, npairs, ni, nf, T, ledos, &
        ncyc, st) bind(C, name='negf_b200_transmissions')
      import; type(c_ptr), value :: ctx, ledos; integer(c_int32_t), value :: npts, npairs
      integer(c_int32_t) :: ids(*), ni(*), nf(*), ncyc(*), st(*); real(c_double) :: E(*), T(*)
      real(c_double), value :: eta, dos_delta
    end function
    integer(c_int) function negf_b200_set_tun_proj(ctx, id, nidx, idx) bind(C, name='negf_b200_set_tun_proj')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: id, nidx; integer(c_int32_t) :: idx(*)
    end function
    integer(c_int) function negf_b200_set_dos_proj(ctx, id, nsets, ptr, idx) bind(C, name='negf_b200_set_dos_proj')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: id, nsets
      integer(c_int32_t) :: ptr(*), idx(*)
    end function
    integer(c_int) function negf_b200_set_sgf_cache(ctx, mode, bytes) bind(C, name='negf_b200_set_sgf_cache')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: mode; integer(c_size_t), value :: bytes
    end function
    integer(c_int) function negf_b200_sgf_cache_save(ctx, path, n) bind(C, name='negf_b200_sgf_cache_save')
      import; type(c_ptr), value :: ctx; character(kind=c_char) :: path(*); integer(c_int64_t) :: n
    end function
    integer(c_int) function negf_b200_sgf_cache_load(ctx, path, n) bind(C, name='negf_b200_sgf_cache_load')
      import; type(c_ptr), value :: ctx; character(kind=c_char) :: path(*); integer(c_int64_t) :: n
    end function
    integer(c_int) function negf_b200_upload_csr(ctx, nrow, nnz, rowpnt, colind, hval, sval, npl, plend, &
        ncont, cblk, surfstart, surfend, contend, id) bind(C, name='negf_b200_upload_csr')
      import; type(c_ptr), value :: ctx, sval     ! sval: c_loc(S%nzval), or c_null_ptr for set_S_id
      integer(c_int32_t), value :: nrow, nnz, npl, ncont
      integer(c_int32_t) :: rowpnt(*), colind(*), plend(*), cblk(*), surfstart(*), surfend(*), contend(*), id
      complex(c_double_complex) :: hval(*)
    end function
    integer(c_int) function negf_b200_density(ctx, id, npts, ere, eim, w, rd, ru, rl, rdc, rcd, ncyc, st) &
        bind(C, name='negf_b200_density')
      import; type(c_ptr), value :: ctx, rdc, rcd; integer(c_int32_t), value :: id, npts
      real(c_double) :: ere(*), eim(*); complex(c_double_complex) :: w(*), rd(*), ru(*), rl(*)
      integer(c_int32_t) :: ncyc(*), st(*)
    end function
    integer(c_int) function negf_b200_density_neq(ctx, id, npts, E, eta, w, frm, cpl, rd, ru, rl, rdc, rcd, &
        ncyc, st) bind(C, name='negf_b200_density_neq')
      import; type(c_ptr), value :: ctx, cpl, rdc, rcd; integer(c_int32_t), value :: id, npts
      real(c_double), value :: eta; real(c_double) :: E(*), frm(*)
      complex(c_double_complex) :: w(*), rd(*), ru(*), rl(*); integer(c_int32_t) :: ncyc(*), st(*)
    end function
    integer(c_int) function negf_b200_device_bytes(ctx, id, bytes) bind(C, name='negf_b200_device_bytes')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: id; integer(c_size_t) :: bytes
    end function
    integer(c_int) function negf_b200_set_tracing(ctx, enable) bind(C, name='negf_b200_set_tracing')
      import; type(c_ptr), value :: ctx; integer(c_int32_t), value :: enable
    end function
    integer(c_int) function negf_b200_get_trace(ctx, cycles) bind(C, name='negf_b200_get_trace')
      import; type(c_ptr), value :: ctx; integer(c_int64_t) :: cycles(*)
    end function
    integer(c_int) function negf_b200_set_workspace_limit(ctx, bytes) bind(C, name='negf_b200_set_workspace_limit')
      import; type(c_ptr), value :: ctx; integer(c_size_t), value :: bytes
    end function
    integer(c_int) function negf_b200_sgf_cache_stats(ctx, hits, misses, entries, used) &
        bind(C, name='negf_b200_sgf_cache_stats')
      import; type(c_ptr), value :: ctx; integer(c_int64_t) :: hits, misses, entries; integer(c_size_t) :: used
    end function
    ! the same solves on device buffers and a caller stream (c_ptr device addresses)
    integer(c_int) function negf_b200_transmission_dev(ctx, npts, ids, E, eta, ni, nf, T, ncyc, st, s) &
        bind(C, name='negf_b200_transmission_dev')
      import; type(c_ptr), value :: ctx, ids, E, T, ncyc, st, s; integer(c_int32_t), value :: npts, ni, nf
      real(c_double), value :: eta
    end function
    integer(c_int) function negf_b200_transmission_dos_dev(ctx, npts, ids, E, eta, dos_delta, ni, nf, T, dos, &
        dos_stride, ncyc, st, s) bind(C, name='negf_b200_transmission_dos_dev')
      import; type(c_ptr), value :: ctx, ids, E, T, dos, ncyc, st, s; integer(c_int32_t), value :: npts, ni, nf
      real(c_double), value :: eta, dos_delta; integer(c_int64_t), value :: dos_stride
    end function
    integer(c_int) function negf_b200_meir_wingreen_dev(ctx, npts, ids, E, eta, frm, cpl, curr, lcurr, ldens, &
        it, err, ncyc, st, cont_stride, layer_stride, s) bind(C, name='negf_b200_meir_wingreen_dev')
      import; type(c_ptr), value :: ctx, ids, E, frm, cpl, curr, lcurr, ldens, it, err, ncyc, st, s
      integer(c_int32_t), value :: npts, cont_stride, layer_stride; real(c_double), value :: eta
    end function
    ! device-pointer primitives: pointers are device addresses (c_ptr), stream c_null_ptr = default
    integer(c_int) function negf_b200_zgemm_batched(b, m, n, k, alpha, A, sA, B_, sB, beta, C, sC, dagger, s) &
        bind(C, name='negf_b200_zgemm_batched')
      import; integer(c_int32_t), value :: b, m, n, k, dagger; integer(c_int64_t), value :: sA, sB, sC
      real(c_double) :: alpha(2), beta(2); type(c_ptr), value :: A, B_, C, s
    end function
    integer(c_size_t) function negf_b200_zinv_work_bytes(b, n) bind(C, name='negf_b200_zinv_work_bytes')
      import; integer(c_int32_t), value :: b, n
    end function
    integer(c_int) function negf_b200_zinv_batched(b, n, A, X, info, work, s) bind(C, name='negf_b200_zinv_batched')
      import; integer(c_int32_t), value :: b, n; type(c_ptr), value :: A, X, info, work, s
    end function
    integer(c_size_t) function negf_b200_decimation_work_bytes(b, n) bind(C, name='negf_b200_decimation_work_bytes')
      import; integer(c_int32_t), value :: b, n
    end function
    integer(c_int) function negf_b200_decimation_batched(b, n, Ao, Bo, Co, Go, ncyc, tol, maxit, work, s) &
        bind(C, name='negf_b200_decimation_batched')
      import; integer(c_int32_t), value :: b, n, maxit; real(c_double), value :: tol
      type(c_ptr), value :: Ao, Bo, Co, Go, ncyc, work, s
    end function
    integer(c_int) function negf_b200_decimation_noalloc(b, n, Ao, Bo, Co, Go, ncyc, tol, maxit, s) &
        bind(C, name='negf_b200_decimation_noalloc')
      import; integer(c_int32_t), value :: b, n, maxit; real(c_double), value :: tol
      type(c_ptr), value :: Ao, Bo, Co, Go, ncyc, s
    end function
    integer(c_size_t) function negf_b200_zgemm_i8_work_bytes(b, m, n, k, slices) &
        bind(C, name='negf_b200_zgemm_i8_work_bytes')
      import; integer(c_int32_t), value :: b, m, n, k, slices
    end function
    integer(c_int) function negf_b200_zgemm_batched_i8(b, m, n, k, alpha, A, sA, B_, sB, beta, C, sC, slices, &
        work, status, s) bind(C, name='negf_b200_zgemm_batched_i8')
      import; integer(c_int32_t), value :: b, m, n, k, slices; integer(c_int64_t), value :: sA, sB, sC
      real(c_double) :: alpha(2), beta(2); type(c_ptr), value :: A, B_, C, work, status, s
    end function

    ! CUDA runtime calls the shims below stage blocks with
    integer(c_int) function cudaMalloc(p, n) bind(C, name='cudaMalloc')
      import; type(c_ptr) :: p; integer(c_size_t), value :: n
    end function
    integer(c_int) function cudaFree(p) bind(C, name='cudaFree')
      import; type(c_ptr), value :: p
    end function
    integer(c_int) function cudaMemcpy(dst, src, n, kind) bind(C, name='cudaMemcpy')
      import; type(c_ptr), value :: dst, src; integer(c_size_t), value :: n; integer(c_int), value :: kind
    end function
  end interface

  integer(c_int), parameter :: cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2
end module negf_b200_bind
