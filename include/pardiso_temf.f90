! Drop-in replacement for the reference's module pardiso_multi_real_mpi
! (src/FETD_UTILITY.f90:826-1028): the same module name, the same five public
! subroutines with the same argument lists, so adap_euler and its call sites
! (src/FETD_FWD.f90:1304-1307,1331,1361,1420,1431,1446-1447) compile unchanged.
! Underneath, every call goes to libtemf_b200.so through the temf_b200
! interface module (temf_b200.f90).
!
! The library factors on the GPU with an analysis of the mesh, so the context
! must know the mesh before the first pardiso_direct_1: mesh_process creates it
! (temf_create, temf_set_mesh, temf_set_media, temf_analyse, temf_assemble)
! and hands it over once with pardiso_use_context.  The CSR passed to
! pardiso_direct_1 must then carry the step-matrix pattern of that mesh (the
! pattern mkl_add_3 produces), which the library checks.
!
! Error behaviour follows the reference:
!   pardiso_alloc     stops on max_matrix < 1;
!   pardiso_direct_1  stops with "matrix error!" when the CSR structure is
!                     invalid (pardiso_checker), and prints the reference's
!                     warning when the matrix is not positive definite and was
!                     factored in indefinite mode (mtype -2) instead;
!   pardiso_direct_2/3 stop on any solver error.
! Only rank 0 calls the library; the module keeps no MPI state.
module pardiso_multi_real_mpi
  use iso_c_binding
  use temf_b200
  implicit none
  private
  type(c_ptr), save :: ctx = c_null_ptr
  integer, save :: maxfct = 0
  public :: pardiso_use_context, pardiso_alloc, pardiso_direct_1, pardiso_direct_2, pardiso_direct_3, &
            pardiso_dealloc
contains

  subroutine pardiso_use_context(context)
    ! the library context of the mesh (set up by mesh_process)
    type(c_ptr), intent(in) :: context
    ctx = context
  end subroutine pardiso_use_context

  subroutine stop_on(status, what)
    integer(c_int), intent(in) :: status
    character(len=*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    integer :: k
    if (status >= 0) return
    call c_f_pointer(temf_last_error(ctx), msg, [512])
    k = 0
    do while (k < 512)
      if (msg(k + 1) == c_null_char) exit
      k = k + 1
    end do
    print *, 'ERROR - ', what, ': ', msg(1:k)
    stop
  end subroutine stop_on

  subroutine pardiso_alloc(max_matrix)
    integer, intent(in) :: max_matrix
    if (max_matrix < 1) stop "maximum number of matrix error, stop!"
    if (.not. c_associated(ctx)) stop "pardiso_alloc: no library context (call pardiso_use_context first)"
    maxfct = max_matrix
    call stop_on(temf_pardiso_alloc(ctx, int(max_matrix, c_int)), 'pardiso_alloc')
  end subroutine pardiso_alloc

  subroutine pardiso_direct_1(num_m, symm, n_in, nnz_in, ia, ja, va, log)
    integer, intent(in) :: num_m
    logical, intent(in) :: symm
    integer, intent(in) :: n_in, nnz_in
    integer, allocatable, intent(in) :: ia(:), ja(:)
    real(8), allocatable, intent(in) :: va(:)
    logical, optional, intent(in) :: log
    integer(c_int) :: status, ok
    character(kind=c_char) :: msg(256)
    status = temf_pardiso_checker(merge(1_c_int, 0_c_int, symm), int(n_in, c_int), int(nnz_in, c_int), ia, ja, &
                                  ok, msg, 256_c_int)
    if (status /= TEMF_OK .or. ok /= 1) stop "matrix error!"
    status = temf_pardiso_direct_1(ctx, int(num_m, c_int), merge(1_c_int, 0_c_int, symm), int(n_in, c_int), &
                                   int(nnz_in, c_int), ia, ja, va)
    call stop_on(status, 'The following error was detected during analysis step of pardiso solver')
    if (status > 0 .and. .not. present(log)) print *, 'WARNING - SYSTEM MATRIX IS INDEFINITE, CHANGE TO INDEFINITE MODE.'
  end subroutine pardiso_direct_1

  subroutine pardiso_direct_2(num_m, b_in, x_out, ia, ja, va)
    integer, intent(in) :: num_m
    real(8), allocatable :: b_in(:), x_out(:)
    integer, allocatable, intent(in) :: ia(:), ja(:)
    real(8), allocatable, intent(in) :: va(:)
    ! the factor lives on the device: ia/ja/va are not read again
    call stop_on(temf_pardiso_direct_2(ctx, int(num_m, c_int), b_in, x_out), &
                 'The following error was detected during solve step of pardiso solver')
  end subroutine pardiso_direct_2

  subroutine pardiso_direct_3(num_m)
    integer, intent(in) :: num_m
    call stop_on(temf_pardiso_direct_3(ctx, int(num_m, c_int)), &
                 'The following error was detected during terminal step of pardiso solver')
  end subroutine pardiso_direct_3

  subroutine pardiso_dealloc
    if (c_associated(ctx)) call stop_on(temf_pardiso_dealloc(ctx), 'pardiso_dealloc')
    maxfct = 0
  end subroutine pardiso_dealloc

end module pardiso_multi_real_mpi
