! soap_turbo_desc_b200 -- Fortran front end of libsoapb200.so.
!
! Keeps the argument lists of soap_turbo's get_soap (src/soap_turbo.f90:139-169),
! soap_contract (:1723-1730) and get_soap_central_hessian (:1151-1160), so a
! caller switches by changing
!   use soap_turbo_desc      ->      use soap_turbo_desc_b200
! and linking libsoapb200.so.  The arrays cross the C ABI as base addresses plus
! the extents the assumed-shape descriptors carry; LOGICAL masks become bytes;
! the basis and scaling-mode strings become NUL-terminated C strings.  Non-zero
! status codes print the library's message and stop, as the reference does on
! bad input.
!
! Behavioural notes for callers of the reference:
!  * soap and soap_cart_der are intent(inout) with the reference's meaning: a
!    compressed soap is added into (src/soap_turbo.f90:798-802), the self
!    columns of soap_cart_der are accumulated into (:888-892); callers pass
!    both zeroed, as for the reference.
!  * soap_cart_der is written only when do_derivatives and not contract, and
!    then in FP64 like the reference.  With contract, call soap_contract.
module soap_turbo_desc_b200

  use, intrinsic :: iso_c_binding
  use, intrinsic :: iso_fortran_env, only: real64

  implicit none
  private

  integer, parameter :: dp = real64

  public :: get_soap, soap_contract, get_soap_central_hessian, soap_b200_set_legacy_filter_seed, &
            soap_b200_set_precision, soap_b200_set_hessian_enabled

  interface
    function soapb_get_soap(n_sites, n_neigh, n_species, species, max_mult, species_multiplicity, &
                            n_atom_pairs, mask, rjs, thetas, phis, alpha_max, l_max, rcut_hard, &
                            rcut_soft, nf, global_scaling, atom_sigma_r, atom_sigma_r_scaling, &
                            atom_sigma_t, atom_sigma_t_scaling, amplitude_scaling, &
                            radial_enhancement, central_weight, basis, scaling_mode, do_timing, &
                            do_derivatives, compress_soap, compress_P_nonzero, compress_P_i, &
                            compress_P_j, compress_P_el, soap, n_soap, soap_cart_der, contract) &
                            result(rc) bind(C, name="soapb_get_soap")
      import :: c_int, c_int8_t, c_double, c_char, c_ptr
      integer(c_int), value :: n_sites, n_species, max_mult, n_atom_pairs, l_max
      integer(c_int), intent(in) :: n_neigh(*), species(*), species_multiplicity(*), alpha_max(*)
      integer(c_int8_t), intent(in) :: mask(*)
      real(c_double), intent(in) :: rjs(*), thetas(*), phis(*)
      real(c_double), intent(in) :: rcut_hard(*), rcut_soft(*), nf(*), global_scaling(*)
      real(c_double), intent(in) :: atom_sigma_r(*), atom_sigma_r_scaling(*)
      real(c_double), intent(in) :: atom_sigma_t(*), atom_sigma_t_scaling(*)
      real(c_double), intent(in) :: amplitude_scaling(*), central_weight(*)
      integer(c_int), value :: radial_enhancement
      character(kind=c_char), intent(in) :: basis(*), scaling_mode(*)
      integer(c_int), value :: do_timing, do_derivatives, compress_soap, compress_P_nonzero
      integer(c_int), intent(in) :: compress_P_i(*), compress_P_j(*)
      real(c_double), intent(in) :: compress_P_el(*)
      real(c_double), intent(inout) :: soap(*)
      integer(c_int), value :: n_soap
      type(c_ptr), value :: soap_cart_der
      integer(c_int), value :: contract
      integer(c_int) :: rc
    end function

    function soapb_soap_contract(soap, G, sgn, pair, n_sites, n_soap, n_atom_pairs) result(rc) &
                                 bind(C, name="soapb_soap_contract")
      import :: c_int, c_double
      real(c_double), intent(in) :: soap(*), G(*)
      real(c_double), value :: sgn
      real(c_double), intent(out) :: pair(*)
      integer(c_int), value :: n_sites, n_soap, n_atom_pairs
      integer(c_int) :: rc
    end function

    function soapb_get_soap_central_hessian(n_sites, n_neigh, n_atom_pairs, n_species, mask, rjs, thetas, &
                                            phis, l_max, rcut_hard, atom_sigma_t, atom_sigma_t_scaling, &
                                            compress_soap, compress_P_nonzero, compress_P_i, compress_P_j, &
                                            compress_P_el, soap, n_soap, n_vec, vecs, hess) result(rc) &
                                            bind(C, name="soapb_get_soap_central_hessian")
      import :: c_int, c_double, c_int8_t
      integer(c_int), value :: n_sites, n_atom_pairs, n_species, l_max, compress_soap, compress_P_nonzero
      integer(c_int), value :: n_soap, n_vec
      integer(c_int), intent(in) :: n_neigh(*), compress_P_i(*), compress_P_j(*)
      integer(c_int8_t), intent(in) :: mask(*)
      real(c_double), intent(in) :: rjs(*), thetas(*), phis(*), rcut_hard(*), atom_sigma_t(*)
      real(c_double), intent(in) :: atom_sigma_t_scaling(*), compress_P_el(*), soap(*), vecs(*)
      real(c_double), intent(out) :: hess(*)
      integer(c_int) :: rc
    end function

    function soapb_set_soap_hessian_enabled(enabled) result(rc) bind(C, name="soapb_set_soap_hessian_enabled")
      import :: c_int
      integer(c_int), value :: enabled
      integer(c_int) :: rc
    end function

    function soapb_set_legacy_filter_seed(legacy) result(rc) bind(C, name="soapb_set_legacy_filter_seed")
      import :: c_int
      integer(c_int), value :: legacy
      integer(c_int) :: rc
    end function

    function soapb_set_precision(precision) result(rc) bind(C, name="soapb_set_precision")
      import :: c_int
      integer(c_int), value :: precision
      integer(c_int) :: rc
    end function

    function soapb_last_error() result(msg) bind(C, name="soapb_last_error")
      import :: c_ptr
      type(c_ptr) :: msg
    end function

    function c_strlen(s) result(n) bind(C, name="strlen")
      import :: c_ptr, c_size_t
      type(c_ptr), value :: s
      integer(c_size_t) :: n
    end function
  end interface

contains

  subroutine check(rc)
    integer(c_int), intent(in) :: rc
    character(kind=c_char), pointer :: chars(:)
    character(len=:), allocatable :: msg
    type(c_ptr) :: p
    integer :: i, n
    if( rc == 0 ) return
    p = soapb_last_error()
    n = int(c_strlen(p))
    call c_f_pointer(p, chars, [n])
    allocate( character(len=n) :: msg )
    do i = 1, n
      msg(i:i) = chars(i)
    end do
    write(*,*) "ERROR: soap_turbo_b200: ", msg
    stop
  end subroutine

  subroutine get_soap(n_sites, n_neigh, n_species, species, species_multiplicity, n_atom_pairs, mask, rjs, &
                      thetas, phis, alpha_max, l_max, rcut_hard, rcut_soft, nf, global_scaling, atom_sigma_r, &
                      atom_sigma_r_scaling, atom_sigma_t, atom_sigma_t_scaling, &
                      amplitude_scaling, radial_enhancement, central_weight, basis, scaling_mode, do_timing, &
                      do_derivatives, compress_soap, compress_P_nonzero, compress_P_i, compress_P_j, &
                      compress_P_el, soap, soap_cart_der, contract)
    implicit none
    real(dp), intent(in) :: rjs(:), thetas(:), phis(:)
    real(dp), intent(in) :: amplitude_scaling(:), atom_sigma_r_scaling(:), atom_sigma_t(:), atom_sigma_t_scaling(:)
    real(dp), intent(in) :: central_weight(:), atom_sigma_r(:), global_scaling(:)
    real(dp), intent(in) :: nf(:), rcut_hard(:), rcut_soft(:)
    real(dp), intent(in) :: compress_P_el(:)
    integer, intent(in) :: n_species, radial_enhancement, species(:,:), species_multiplicity(:)
    integer, intent(in) :: n_sites, n_neigh(:), l_max, n_atom_pairs, alpha_max(:), compress_P_nonzero, &
                           compress_P_i(:), compress_P_j(:)
    logical, intent(in) :: do_derivatives, do_timing, mask(:,:), compress_soap
    character(*), intent(in) :: basis, scaling_mode
    logical, intent(in), optional :: contract
    real(dp), intent(inout), target, contiguous :: soap(:,:), soap_cart_der(:,:,:)

    integer(c_int8_t), allocatable :: mask8(:,:)
    logical :: do_contract
    type(c_ptr) :: cart
    integer(c_int) :: rc

    do_contract = .false.
    if( present(contract) ) do_contract = contract .and. do_derivatives
    allocate( mask8(size(mask,1), size(mask,2)) )
    mask8 = merge(1_c_int8_t, 0_c_int8_t, mask)
    cart = c_null_ptr
    if( do_derivatives .and. .not. do_contract ) cart = c_loc(soap_cart_der)
    rc = soapb_get_soap(int(n_sites, c_int), n_neigh, int(n_species, c_int), species, &
                        int(size(species, 1), c_int), species_multiplicity, int(n_atom_pairs, c_int), &
                        mask8, rjs, thetas, phis, alpha_max, int(l_max, c_int), rcut_hard, rcut_soft, &
                        nf, global_scaling, atom_sigma_r, atom_sigma_r_scaling, atom_sigma_t, &
                        atom_sigma_t_scaling, amplitude_scaling, int(radial_enhancement, c_int), &
                        central_weight, trim(adjustl(basis))//c_null_char, &
                        trim(adjustl(scaling_mode))//c_null_char, merge(1_c_int, 0_c_int, do_timing), &
                        merge(1_c_int, 0_c_int, do_derivatives), merge(1_c_int, 0_c_int, compress_soap), &
                        int(compress_P_nonzero, c_int), compress_P_i, compress_P_j, compress_P_el, soap, &
                        int(size(soap, 1), c_int), cart, merge(1_c_int, 0_c_int, do_contract))
    deallocate( mask8 )
    call check(rc)
  end subroutine get_soap

  subroutine soap_contract(soap, G, sgn, pair)
    implicit none
    real(dp), intent(in) :: soap(:,:)
    real(dp), intent(in) :: G(:,:)
    real(dp), intent(in) :: sgn
    real(dp), intent(out) :: pair(:,:)
    integer(c_int) :: rc
    rc = soapb_soap_contract(soap, G, real(sgn, c_double), pair, int(size(soap, 2), c_int), &
                             int(size(soap, 1), c_int), int(size(pair, 2), c_int))
    call check(rc)
  end subroutine soap_contract

  ! get_soap_central_hessian (src/soap_turbo.f90:1151-1160): after get_soap with
  ! do_derivatives on the same batch, with soap_b200_set_hessian_enabled(.true.)
  ! called before that get_soap.  hess(1:3, 1:3, 1:n_vec, 1:n_atom_pairs).
  subroutine get_soap_central_hessian(n_sites, n_neigh, n_atom_pairs, n_species, mask, rjs, thetas, phis, &
                                      l_max, rcut_hard, atom_sigma_t, atom_sigma_t_scaling, compress_soap, &
                                      compress_P_nonzero, compress_P_i, compress_P_j, compress_P_el, soap, &
                                      n_vec, vecs, hess)
    implicit none
    integer, intent(in) :: n_sites, n_neigh(:), n_atom_pairs, n_species, l_max, n_vec
    integer, intent(in) :: compress_P_nonzero, compress_P_i(:), compress_P_j(:)
    logical, intent(in) :: mask(:,:), compress_soap
    real(dp), intent(in) :: rjs(:), thetas(:), phis(:), rcut_hard(:)
    real(dp), intent(in) :: atom_sigma_t(:), atom_sigma_t_scaling(:), compress_P_el(:)
    real(dp), intent(in) :: soap(:,:), vecs(:,:,:)
    real(dp), intent(out) :: hess(:,:,:,:)

    integer(c_int8_t), allocatable :: mask8(:,:)
    integer(c_int) :: rc

    allocate( mask8(size(mask,1), size(mask,2)) )
    mask8 = merge(1_c_int8_t, 0_c_int8_t, mask)
    rc = soapb_get_soap_central_hessian(int(n_sites, c_int), n_neigh, int(n_atom_pairs, c_int), &
                                        int(n_species, c_int), mask8, rjs, thetas, phis, int(l_max, c_int), &
                                        rcut_hard, atom_sigma_t, atom_sigma_t_scaling, &
                                        merge(1_c_int, 0_c_int, compress_soap), int(compress_P_nonzero, c_int), &
                                        compress_P_i, compress_P_j, compress_P_el, soap, &
                                        int(size(soap, 1), c_int), int(n_vec, c_int), vecs, hess)
    deallocate( mask8 )
    call check(rc)
  end subroutine get_soap_central_hessian

  ! The reference's module flag soap_turbo_desc::soap_hessian_enabled
  ! (src/soap_turbo.f90:76), default .false.
  subroutine soap_b200_set_hessian_enabled(enabled)
    logical, intent(in) :: enabled
    call check(soapb_set_soap_hessian_enabled(merge(1_c_int, 0_c_int, enabled)))
  end subroutine

  ! The reference's module flag soap_turbo_radial::legacy_filter_seed
  ! (src/soap_turbo_radial.f90:67), default .true.
  subroutine soap_b200_set_legacy_filter_seed(legacy)
    logical, intent(in) :: legacy
    call check(soapb_set_legacy_filter_seed(merge(1_c_int, 0_c_int, legacy)))
  end subroutine

  ! 0: mixed precision (default), 1: plain FP64
  subroutine soap_b200_set_precision(precision)
    integer, intent(in) :: precision
    call check(soapb_set_precision(int(precision, c_int)))
  end subroutine

end module soap_turbo_desc_b200
