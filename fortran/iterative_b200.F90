! Uncompiled on this image (no Fortran compiler here).
!
! The B200 backend for libNEGF's RGF seam: a module with the public names of
! iterative_gpu (src/iterative_gpu.F90:44-50), so that src/iterative.F90:38-43
! can `use iterative_b200` in its place, plus decimation_b200 for the
! contact-side seam decimation_gpu (src/contselfenergy.F90:347-379).
!
! This is the per-point, per-block seam: every block product goes to
! negf_b200_zgemm_batched and every block inverse to negf_b200_zinv_batched
! (batch 1), the blocks being staged through device buffers around each call.
! It keeps libNEGF's own energy loop unchanged.  The fast path replaces that
! loop instead: one negf_b200_transmission / _transmission_dos /
! _meir_wingreen call over all of a rank's (E, k) points, with the device
! description resident in HBM (INTEGRATION.md, "Where the calls go").
!
! The lesser sweep (calculate_Gn_tridiag_blocks) of this seam is the CPU
! backend's: its B200 counterpart is the batched negf_b200_meir_wingreen, which
! runs the whole elastic SCBA point by point on the device.
module iterative_b200
  use iso_c_binding
  use ln_precision, only : dp, EPS, SGFACC
  use mat_def, only : z_DNS, create, destroy
  use lib_param, only : Tnegf, intarray
  use ln_structure, only : TStruct_Info
  use iterative_cpu, only : cpu_Gn_tridiag_blocks => calculate_Gn_tridiag_blocks
  use negf_b200_bind
  use, intrinsic :: ieee_arithmetic
  implicit none
  private

  public :: calculate_gsmr_blocks
  public :: calculate_Gr_tridiag_blocks
  public :: calculate_Gn_tridiag_blocks
  public :: calculate_single_transmission_2_contacts
  public :: calculate_single_transmission_N_contacts
  public :: check_convergence_trid
  public :: check_convergence_vec
  public :: decimation_b200

  complex(dp), parameter :: one = (1.0_dp, 0.0_dp), mone = (-1.0_dp, 0.0_dp), imag = (0.0_dp, 1.0_dp)

contains

  ! ---------------------------------------------------------------- staging
  function dev_put(A) result(p)
    type(z_DNS), intent(in), target :: A
    type(c_ptr) :: p
    integer(c_size_t) :: nb
    nb = int(16, c_size_t) * int(max(A%nrow * A%ncol, 1), c_size_t)
    if (cudaMalloc(p, nb) /= 0) error stop 'iterative_b200: cudaMalloc failed'
    if (A%nrow * A%ncol > 0) then
      if (cudaMemcpy(p, c_loc(A%val), nb, cudaMemcpyHostToDevice) /= 0) error stop 'iterative_b200: upload failed'
    end if
  end function

  subroutine dev_get(p, A)
    type(c_ptr), intent(in) :: p
    type(z_DNS), intent(inout), target :: A
    integer(c_size_t) :: nb
    nb = int(16, c_size_t) * int(A%nrow * A%ncol, c_size_t)
    if (nb > 0) then
      if (cudaMemcpy(c_loc(A%val), p, nb, cudaMemcpyDeviceToHost) /= 0) error stop 'iterative_b200: download failed'
    end if
    if (cudaFree(p) /= 0) error stop 'iterative_b200: cudaFree failed'
  end subroutine

  subroutine dev_drop(p)
    type(c_ptr), intent(in) :: p
    if (cudaFree(p) /= 0) error stop 'iterative_b200: cudaFree failed'
  end subroutine

  ! C = s A B if C is not allocated, else C = C + s A B: the rule of
  ! prealloc_mult (src/sparsekit_drv.F90:1896-2081), on the FP64 tensor cores
  subroutine mult(A, B, C, s)
    type(z_DNS), intent(in) :: A, B
    type(z_DNS), intent(inout) :: C
    complex(dp), intent(in), optional :: s
    real(c_double) :: alpha(2), beta(2)
    type(c_ptr) :: pa, pb, pc
    complex(dp) :: sc
    sc = one
    if (present(s)) sc = s
    alpha = [real(sc, dp), aimag(sc)]
    if (allocated(C%val)) then
      beta = [1.0_dp, 0.0_dp]
    else
      call create(C, A%nrow, B%ncol)
      C%val = (0.0_dp, 0.0_dp)
      beta = [0.0_dp, 0.0_dp]
    end if
    pa = dev_put(A); pb = dev_put(B); pc = dev_put(C)
    if (negf_b200_zgemm_batched(1_c_int32_t, int(A%nrow, c_int32_t), int(B%ncol, c_int32_t), &
        int(A%ncol, c_int32_t), alpha, pa, 0_c_int64_t, pb, 0_c_int64_t, beta, pc, 0_c_int64_t, &
        0_c_int32_t, c_null_ptr) /= NEGF_B200_OK) error stop 'iterative_b200: block product failed'
    call dev_drop(pa); call dev_drop(pb)
    call dev_get(pc, C)
  end subroutine

  ! X = A^-1 (zinv, src/inversions.F90:807-839): Gauss-Jordan with the izamax
  ! pivot rule on the device; a zero pivot stops as zgetrf's info > 0 does
  subroutine inv(A, X)
    type(z_DNS), intent(in) :: A
    type(z_DNS), intent(inout) :: X
    type(c_ptr) :: pa, px, pinfo, pw
    integer(c_int32_t), target :: info(1)
    integer(c_size_t) :: wb
    call create(X, A%nrow, A%ncol)
    pa = dev_put(A); px = dev_put(X)
    if (cudaMalloc(pinfo, int(4, c_size_t)) /= 0) error stop 'iterative_b200: cudaMalloc failed'
    wb = max(negf_b200_zinv_work_bytes(1_c_int32_t, int(A%nrow, c_int32_t)), int(16, c_size_t))
    if (cudaMalloc(pw, wb) /= 0) error stop 'iterative_b200: cudaMalloc failed'
    if (negf_b200_zinv_batched(1_c_int32_t, int(A%nrow, c_int32_t), pa, px, pinfo, pw, c_null_ptr) &
        /= NEGF_B200_OK) error stop 'iterative_b200: block inversion failed'
    if (cudaMemcpy(c_loc(info), pinfo, int(4, c_size_t), cudaMemcpyDeviceToHost) /= 0) error stop 'download failed'
    call dev_drop(pa); call dev_drop(pinfo); call dev_drop(pw)
    call dev_get(px, X)
    if (info(1) /= 0) error stop 'iterative_b200: singular block (zero pivot)'
  end subroutine

  ! i (S - S^dag)  (zspectral, src/sparsekit_drv.F90:2870-2890)
  subroutine spectral(S, G)
    type(z_DNS), intent(in) :: S
    type(z_DNS), intent(inout) :: G
    call create(G, S%nrow, S%ncol)
    G%val = imag * (S%val - conjg(transpose(S%val)))
  end subroutine

  ! ---------------------------------------------------------------- the seam
  ! gsmr(sbl) = ESH(sbl,sbl)^-1, gsmr(i) = [ESH(i,i) - ESH(i,i+1) gsmr(i+1) ESH(i+1,i)]^-1
  ! for i = sbl-1 .. ebl (src/iterative_cpu.F90:51-124)
  subroutine calculate_gsmr_blocks(negf, ESH, sbl, ebl, gsmr, keep_gsmr)
    type(Tnegf), intent(in) :: negf
    type(z_DNS), dimension(:,:), intent(in) :: ESH
    integer, intent(in) :: sbl, ebl
    type(z_DNS), dimension(:), intent(inout) :: gsmr
    logical, intent(in), optional :: keep_gsmr
    type(z_DNS) :: w1, w2
    integer :: i
    logical :: keep
    if (sbl < ebl) return
    if (size(ESH, 1) == 1) return
    keep = .true.
    if (present(keep_gsmr)) keep = keep_gsmr
    call inv(ESH(sbl, sbl), gsmr(sbl))
    do i = sbl - 1, ebl, -1
      call mult(ESH(i, i + 1), gsmr(i + 1), w1, mone)
      if (.not. keep) call destroy(gsmr(i + 1))
      w2 = ESH(i, i)
      call mult(w1, ESH(i + 1, i), w2)
      call inv(w2, gsmr(i))
      call destroy(w1); call destroy(w2)
    end do
  end subroutine

  ! Gr(1,1) = [ESH(1,1) - ESH(1,2) gsmr(2) ESH(2,1)]^-1 (sbl = 1, no ebl), or
  ! the forward sweep i = sbl .. ebl (src/iterative_cpu.F90:134-224):
  ! Gr(i,i-1) = -gsmr(i) ESH(i,i-1) Gr(i-1,i-1), Gr(i-1,i) = -Gr(i-1,i-1) ESH(i-1,i) gsmr(i),
  ! Gr(i,i) = gsmr(i) - Gr(i,i-1) ESH(i-1,i) gsmr(i)
  subroutine calculate_Gr_tridiag_blocks(negf, ESH, gsmr, Gr, sbl, ebl)
    type(Tnegf), intent(in) :: negf
    type(z_DNS), dimension(:,:), intent(in) :: ESH
    type(z_DNS), dimension(:), intent(in) :: gsmr
    type(z_DNS), dimension(:,:), intent(inout) :: Gr
    integer, intent(in) :: sbl
    integer, intent(in), optional :: ebl
    type(z_DNS) :: w1, w2, w3
    integer :: i, nbl
    nbl = size(ESH, 1)
    if (.not. present(ebl)) then
      if (nbl == 1) then
        call inv(ESH(sbl, sbl), Gr(sbl, sbl))
        return
      end if
      w1 = ESH(sbl, sbl)
      if (sbl + 1 <= nbl) then
        call mult(ESH(sbl, sbl + 1), gsmr(sbl + 1), w2)
        call mult(w2, ESH(sbl + 1, sbl), w1, mone)
        call destroy(w2)
      end if
      call inv(w1, Gr(sbl, sbl))
      call destroy(w1)
      return
    end if
    do i = sbl, ebl
      call mult(gsmr(i), ESH(i, i - 1), w1)
      call mult(w1, Gr(i - 1, i - 1), Gr(i, i - 1), mone)
      call destroy(w1)
      call mult(ESH(i - 1, i), gsmr(i), w2)
      call mult(Gr(i - 1, i - 1), w2, Gr(i - 1, i), mone)
      w3 = gsmr(i)
      call mult(Gr(i, i - 1), w2, w3, mone)
      Gr(i, i) = w3
      call destroy(w2); call destroy(w3)
    end do
  end subroutine

  ! The lesser sweep of the CPU backend (see the module header)
  subroutine calculate_Gn_tridiag_blocks(negf, ESH, SelfEneR, frm, ref, struct, gsmr, Gr, Gn)
    type(Tnegf), intent(in) :: negf
    type(z_DNS), dimension(:,:), intent(in) :: ESH
    type(z_DNS), dimension(:), intent(in) :: SelfEneR
    real(dp), dimension(:), intent(in) :: frm
    integer, intent(in) :: ref
    type(TStruct_Info), intent(in) :: struct
    type(z_DNS), dimension(:), intent(in) :: gsmr
    type(z_DNS), dimension(:,:), intent(in) :: Gr
    type(z_DNS), dimension(:,:), intent(inout) :: Gn
    call cpu_Gn_tridiag_blocks(negf, ESH, SelfEneR, frm, ref, struct, gsmr, Gr, Gn)
  end subroutine

  ! diagonal entries of block bl selected by tun_proj (global 1-based orbital
  ! indices; none given = the whole block), as get_tun_mask
  subroutine block_mask(ESH, bl, tun_proj, mask)
    type(z_DNS), dimension(:,:), intent(in) :: ESH
    integer, intent(in) :: bl
    type(intarray), intent(in) :: tun_proj
    logical, allocatable, intent(out) :: mask(:)
    integer :: k, i0, ind
    allocate(mask(ESH(bl, bl)%nrow))
    if (.not. allocated(tun_proj%indexes)) then
      mask = .true.
      return
    end if
    mask = .false.
    i0 = 0
    do k = 1, bl - 1
      i0 = i0 + ESH(k, k)%nrow
    end do
    do k = 1, size(tun_proj%indexes)
      ind = tun_proj%indexes(k) - i0
      if (ind >= 1 .and. ind <= ESH(bl, bl)%nrow) mask(ind) = .true.
    end do
  end subroutine

  ! T = |Re Tr_mask[Gam1 i(G - G^dag) - Gam1 G Gam1 G^dag]|, ct1 = the contact on
  ! the smaller block (src/iterative_cpu.F90:399-470)
  subroutine calculate_single_transmission_2_contacts(negf, ni, nf, ESH, SelfEneR, cblk, tun_proj, Gr, TUN)
    type(Tnegf), intent(in) :: negf
    integer, intent(in) :: ni, nf
    type(z_DNS), dimension(:,:), intent(in) :: ESH
    type(z_DNS), dimension(:), intent(in) :: SelfEneR
    integer, dimension(:), intent(in) :: cblk
    type(intarray), intent(in) :: tun_proj
    type(z_DNS), dimension(:,:), intent(in) :: Gr
    real(dp), intent(out) :: TUN
    type(z_DNS) :: gam, ga, w1, w2, w3, aa, w4
    logical, allocatable :: mask(:)
    integer :: ct1, bl1, k
    complex(dp) :: tr
    ct1 = nf
    if (cblk(ni) < cblk(nf)) ct1 = ni
    bl1 = cblk(ct1)
    call spectral(SelfEneR(ct1), gam)
    call create(ga, Gr(bl1, bl1)%ncol, Gr(bl1, bl1)%nrow)
    ga%val = conjg(transpose(Gr(bl1, bl1)%val))
    call mult(gam, Gr(bl1, bl1), w1)
    call mult(w1, gam, w2)
    call mult(w2, ga, w3)
    call create(aa, ga%nrow, ga%ncol)
    aa%val = imag * (Gr(bl1, bl1)%val - ga%val)
    call mult(gam, aa, w4)
    call block_mask(ESH, bl1, tun_proj, mask)
    tr = (0.0_dp, 0.0_dp)
    do k = 1, size(mask)
      if (mask(k)) tr = tr + w4%val(k, k) - w3%val(k, k)
    end do
    TUN = abs(real(tr, dp))
    call destroy(gam); call destroy(ga); call destroy(w1); call destroy(w2); call destroy(w3)
    call destroy(aa); call destroy(w4)
  end subroutine

  ! Column sweep Gr(i,bl1) = -gsmr(i) ESH(i,i-1) Gr(i-1,bl1) up to bl2 (stops
  ! with T = EPS^2 when a column block falls below EPS), then
  ! T = |Re Tr_mask[Gam2 G21 Gam1 G21^dag]| (src/iterative_cpu.F90:477-583)
  subroutine calculate_single_transmission_N_contacts(negf, ni, nf, ESH, SelfEneR, cblk, tun_proj, gsmr, Gr, TUN)
    type(Tnegf), intent(in) :: negf
    integer, intent(in) :: ni, nf
    type(z_DNS), dimension(:,:), intent(in) :: ESH
    type(z_DNS), dimension(:), intent(in) :: SelfEneR
    integer, dimension(:), intent(in) :: cblk
    type(intarray), intent(in) :: tun_proj
    type(z_DNS), dimension(:), intent(in) :: gsmr
    type(z_DNS), dimension(:,:), intent(inout) :: Gr
    real(dp), intent(out) :: TUN
    type(z_DNS) :: col_prev, col, w1, gam1, gam2, w2, w3, ga, trs
    logical, allocatable :: mask(:)
    integer :: ct1, ct2, bl1, bl2, i, k
    complex(dp) :: tr
    if (cblk(ni) < cblk(nf)) then
      ct1 = ni; ct2 = nf
    else
      ct1 = nf; ct2 = ni
    end if
    bl1 = cblk(ct1); bl2 = cblk(ct2)
    if (bl2 == bl1) then
      col = Gr(bl1, bl1)
    else
      col = Gr(bl1 + 1, bl1)
      do i = bl1 + 2, bl2
        if (maxval(abs(col%val)) < EPS) then
          TUN = EPS * EPS
          call destroy(col)
          return
        end if
        col_prev = col
        call destroy(col)
        call mult(gsmr(i), ESH(i, i - 1), w1, mone)
        call mult(w1, col_prev, col)
        call destroy(w1); call destroy(col_prev)
      end do
    end if
    call spectral(SelfEneR(ct1), gam1)
    call spectral(SelfEneR(ct2), gam2)
    call mult(gam2, col, w2)
    call mult(w2, gam1, w3)
    call create(ga, col%ncol, col%nrow)
    ga%val = conjg(transpose(col%val))
    call mult(w3, ga, trs)
    call block_mask(ESH, bl2, tun_proj, mask)
    tr = (0.0_dp, 0.0_dp)
    do k = 1, size(mask)
      if (mask(k)) tr = tr + trs%val(k, k)
    end do
    TUN = abs(real(tr, dp))
    call destroy(col); call destroy(gam1); call destroy(gam2); call destroy(w2); call destroy(w3)
    call destroy(ga); call destroy(trs)
  end subroutine

  ! NaN scan of the tridiagonal blocks (the host side of the reference's checksum)
  subroutine check_convergence_trid(negf, T, nome, gpu)
    type(Tnegf), intent(in) :: negf
    type(z_DNS), dimension(:,:), intent(in) :: T
    character(3), intent(in) :: nome
    logical, intent(in) :: gpu
    integer :: i, j, nbl
    nbl = size(T, 1)
    do i = 1, nbl
      do j = max(1, i - 1), min(nbl, i + 1)
        if (allocated(T(i, j)%val)) then
          if (ieee_is_nan(sum(abs(T(i, j)%val)))) write(*, *) nome, '(', i, j, ') has NaN'
        end if
      end do
    end do
  end subroutine

  subroutine check_convergence_vec(negf, T, nome, gpu)
    type(Tnegf), intent(in) :: negf
    type(z_DNS), dimension(:), intent(in) :: T
    character(3), intent(in) :: nome
    logical, intent(in) :: gpu
    integer :: i
    do i = 1, size(T)
      if (allocated(T(i)%val)) then
        if (ieee_is_nan(sum(abs(T(i)%val)))) write(*, *) nome, '(', i, ') has NaN'
      end if
    end do
  end subroutine

  ! decimation_gpu (src/contselfenergy.F90:347-379) on the B200 decimation:
  ! the CPU convergence rule (max|C1| <= SGFACC on two consecutive
  ! iterations, at most 300), the surface GF in Go_out, ncyc as the reference
  ! reports it.  tf32 has no counterpart (the decimation is FP64).
  subroutine decimation_b200(negf, Go_out, Ao_in, Bo_in, Co_in, n, tf32, ncyc)
    type(Tnegf), intent(in) :: negf
    integer, intent(in) :: n
    complex(dp), dimension(n, n), intent(out), target :: Go_out
    complex(dp), dimension(n, n), intent(in), target :: Ao_in, Bo_in, Co_in
    logical, intent(in) :: tf32
    integer, intent(out) :: ncyc
    type(c_ptr) :: pa, pb, pc, pg, pn, pw
    integer(c_size_t) :: nb, wb
    integer(c_int32_t), target :: nc(1)
    integer(c_int) :: st
    nb = int(16, c_size_t) * int(n, c_size_t) * int(n, c_size_t)
    if (cudaMalloc(pa, nb) /= 0 .or. cudaMalloc(pb, nb) /= 0 .or. cudaMalloc(pc, nb) /= 0 .or. &
        cudaMalloc(pg, nb) /= 0 .or. cudaMalloc(pn, int(4, c_size_t)) /= 0) error stop 'decimation_b200: cudaMalloc'
    wb = negf_b200_decimation_work_bytes(1_c_int32_t, int(n, c_int32_t))
    if (cudaMalloc(pw, wb) /= 0) error stop 'decimation_b200: cudaMalloc'
    if (cudaMemcpy(pa, c_loc(Ao_in), nb, cudaMemcpyHostToDevice) /= 0 .or. &
        cudaMemcpy(pb, c_loc(Bo_in), nb, cudaMemcpyHostToDevice) /= 0 .or. &
        cudaMemcpy(pc, c_loc(Co_in), nb, cudaMemcpyHostToDevice) /= 0) error stop 'decimation_b200: upload'
    st = negf_b200_decimation_batched(1_c_int32_t, int(n, c_int32_t), pa, pb, pc, pg, pn, real(SGFACC, c_double), &
                                      300_c_int32_t, pw, c_null_ptr)
    if (st /= NEGF_B200_OK) error stop 'decimation_b200: decimation failed'
    if (cudaMemcpy(c_loc(Go_out), pg, nb, cudaMemcpyDeviceToHost) /= 0 .or. &
        cudaMemcpy(c_loc(nc), pn, int(4, c_size_t), cudaMemcpyDeviceToHost) /= 0) error stop 'decimation_b200: download'
    ncyc = nc(1)
    call dev_drop(pa); call dev_drop(pb); call dev_drop(pc); call dev_drop(pg); call dev_drop(pn); call dev_drop(pw)
  end subroutine

end module iterative_b200
