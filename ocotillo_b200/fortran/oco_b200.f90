! oco_b200.f90 -- Fortran 2003 binding (ISO_C_BINDING) of the B200 engine's C ABI, include/oco.h.
!
! A Fortran driver (the reference's flux_feautrier.f90) uses this module to replace its xy/lambda
! loop (source/flux_feautrier.f90:160-228) by one call per processor block:
!
!   use OcoB200
!   rc = oco_create(ctx, 0_c_int)
!   rc = oco_set_wavelengths(ctx, waves_angstrom, int(nw, c_int32_t))   ! pre_calc_opacity_quantities
!   prm = oco_params(nxloc, nyloc, nz, nw, dz, sigma_grey, fully_ionized_T, lgrey_int, &
!                    OCO_FORM_PLAIN, OCO_LAYOUT_REFERENCE, 0)
!   rc = oco_solve_block(ctx, prm, rho3d, temp3d, U, absorp_coeff, V, c_null_ptr, c_null_ptr)
!
! Arrays keep the reference's shapes: rho3d, temp3d (nz,nyloc,nxloc); U (mz,nyloc,nxloc,nw);
! absorp_coeff, V (nz,nyloc,nxloc,nw).  Link with -loco_b200.  Every function returns 0 or a
! negative OCO_E* code; oco_last_error(ctx) points to the message (a C string).
module OcoB200
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: OCO_OK = 0, OCO_EINVAL = -1, OCO_ENOMEM = -2, OCO_EZEROPIVOT = -3
  integer(c_int), parameter :: OCO_EGREY = -4, OCO_ECUDA = -5, OCO_ETIMEDOUT = -6, OCO_ENOWAVES = -11
  integer(c_int32_t), parameter :: OCO_FORM_PLAIN = 0, OCO_FORM_STABLE = 1, OCO_FORM_MIXED = 2
  integer(c_int32_t), parameter :: OCO_LAYOUT_REFERENCE = 0, OCO_LAYOUT_LAMBDA_FASTEST = 1

  ! struct oco_params
  type, bind(C) :: oco_params
     integer(c_int32_t) :: nx, ny, nz, nw
     real(c_double)     :: dz
     real(c_double)     :: sigma_grey
     real(c_double)     :: fully_ionized_T
     integer(c_int32_t) :: lgrey
     integer(c_int32_t) :: form
     integer(c_int32_t) :: layout
     integer(c_int32_t) :: reserved
  end type oco_params

  interface
     integer(c_int) function oco_abi_version() bind(C, name="oco_abi_version")
       import :: c_int
     end function oco_abi_version

     integer(c_int) function oco_create(ctx, device) bind(C, name="oco_create")
       import :: c_int, c_ptr
       type(c_ptr), intent(out) :: ctx
       integer(c_int), value :: device
     end function oco_create

     subroutine oco_destroy(ctx) bind(C, name="oco_destroy")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end subroutine oco_destroy

     type(c_ptr) function oco_last_error(ctx) bind(C, name="oco_last_error")
       import :: c_ptr
       type(c_ptr), value :: ctx
     end function oco_last_error

     integer(c_int) function oco_calc_wavelength(w1, w0, nw, wa) bind(C, name="oco_calc_wavelength")
       import :: c_int, c_int32_t, c_double
       real(c_double), value :: w1, w0
       integer(c_int32_t), value :: nw
       real(c_double) :: wa(*)
     end function oco_calc_wavelength

     integer(c_int) function oco_set_wavelengths(ctx, wa, nw) bind(C, name="oco_set_wavelengths")
       import :: c_int, c_int32_t, c_double, c_ptr
       type(c_ptr), value :: ctx
       real(c_double), intent(in) :: wa(*)
       integer(c_int32_t), value :: nw
     end function oco_set_wavelengths

     integer(c_int) function oco_solve_block(ctx, p, rho, T, U, kappa, V, Vtop, Vbot) bind(C, name="oco_solve_block")
       import :: c_int, c_double, c_ptr, oco_params
       type(c_ptr), value :: ctx
       type(oco_params), intent(in) :: p
       real(c_double), intent(in) :: rho(*), T(*)
       real(c_double) :: U(*), kappa(*), V(*)
       type(c_ptr), value :: Vtop, Vbot
     end function oco_solve_block

     integer(c_int) function oco_solve_block_device(ctx, p, rho, T, U, kappa, V, Vtop, Vbot, stream) &
          bind(C, name="oco_solve_block_device")
       import :: c_int, c_ptr, oco_params
       type(c_ptr), value :: ctx
       type(oco_params), intent(in) :: p
       type(c_ptr), value :: rho, T, U, kappa, V, Vtop, Vbot, stream
     end function oco_solve_block_device

     integer(c_int) function oco_synchronize(ctx) bind(C, name="oco_synchronize")
       import :: c_int, c_ptr
       type(c_ptr), value :: ctx
     end function oco_synchronize

     integer(c_int) function oco_set_mixed_repair(ctx, cond_max) bind(C, name="oco_set_mixed_repair")
       import :: c_int, c_double, c_ptr
       type(c_ptr), value :: ctx
       real(c_double), value :: cond_max
     end function oco_set_mixed_repair

     integer(c_int) function oco_mixed_repairs(ctx, items) bind(C, name="oco_mixed_repairs")
       import :: c_int, c_int64_t, c_ptr
       type(c_ptr), value :: ctx
       integer(c_int64_t), intent(out) :: items
     end function oco_mixed_repairs

     integer(c_int) function oco_run_deck(deck_dir, snapshot, out_dir, form, device, write_binary) &
          bind(C, name="oco_run_deck")
       import :: c_int, c_int32_t, c_char
       character(kind=c_char), intent(in) :: deck_dir(*), snapshot(*), out_dir(*)
       integer(c_int32_t), value :: form, device, write_binary
     end function oco_run_deck
  end interface
end module OcoB200
