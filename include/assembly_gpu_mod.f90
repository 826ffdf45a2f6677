! Fortran 2003 binding of the B200 hot path (source only: no Fortran compiler is
! available where this library is built, so this file is not compiled here).
!
! A QUADESTH build replaces `use assembly_mod`, `use solver_mod` and the stress
! routines of `stress_mod` in main.f90 with `use assembly_gpu_mod` (keeping
! `use stress_mod, only: output_boundary_stresses, output_internal_points,
! deallocate_stress_data` for the writers).  The subroutines
! below keep the reference's names and arguments and work on the same data_mod
! globals:
!   precompute_element_geometry  (assembly_mod.f90:28)
!   ghmat8                       (assembly_mod.f90:53)   A stays in GPU memory
!   solve_linear_system          (solver_mod.f90:17)     same stop message on info /= 0
!   reorganize_solution          (io_mod.f90:148)
!   compute_boundary_stresses    (stress_mod.f90:365)
!   compute_internal_points      (stress_mod.f90:511)
! Link with -L<dir> -lbem3d_b200 -Wl,-rpath,<dir> and the CUDA runtime.

module bem3d_b200
  use, intrinsic :: iso_c_binding
  implicit none

  integer(c_int), parameter :: BEM_PREC_FP64 = 0, BEM_PREC_FP32_IR = 1, BEM_PREC_BF16_IR = 2
  integer(c_int), parameter :: BEM_ASM_FP64 = 0, BEM_ASM_FP32_FAR = 1

  interface
    integer(c_int) function bem_ctx_create(ctx, device) bind(C, name="bem_ctx_create")
      import :: c_ptr, c_int
      type(c_ptr), intent(out) :: ctx
      integer(c_int), value :: device
    end function
    integer(c_int) function bem_ctx_destroy(ctx) bind(C, name="bem_ctx_destroy")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    type(c_ptr) function bem_last_error(ctx) bind(C, name="bem_last_error")
      import :: c_ptr
      type(c_ptr), value :: ctx
    end function
    integer(c_int) function bem_set_mesh(ctx, n, ne, x, y, z, nconec, kconec) bind(C, name="bem_set_mesh")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n, ne
      real(c_double), intent(in) :: x(*), y(*), z(*)
      integer(c_int), intent(in) :: nconec(*), kconec(9, *)
    end function
    integer(c_int) function bem_set_material(ctx, mu, nu) bind(C, name="bem_set_material")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), value :: mu, nu
    end function
    integer(c_int) function bem_set_bc(ctx, kode, bc) bind(C, name="bem_set_bc")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), intent(in) :: kode(*)
      real(c_double), intent(in) :: bc(27, *)
    end function
    integer(c_int) function bem_precompute_geometry(ctx) bind(C, name="bem_precompute_geometry")
      import :: c_ptr, c_int
      type(c_ptr), value :: ctx
    end function
    ! A as a pointer (c_null_ptr keeps A in GPU memory), FI as the host array
    integer(c_int) function bem_ghmat8(ctx, prec, A, lda, FI) bind(C, name="bem_ghmat8")
      import :: c_ptr, c_int, c_int64_t, c_double
      type(c_ptr), value :: ctx, A
      integer(c_int), value :: prec
      integer(c_int64_t), value :: lda
      real(c_double), intent(out) :: FI(*)
    end function
    integer(c_int) function bem_solve(ctx, prec, tol, maxit, FI, info, stats) bind(C, name="bem_solve")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx, stats
      integer(c_int), value :: prec, maxit
      real(c_double), value :: tol
      real(c_double), intent(inout) :: FI(*)
      integer(c_int), intent(out) :: info
    end function
    integer(c_int) function bem_dgesv(ctx, n, nrhs, A, lda, ipiv, B, ldb, info) bind(C, name="bem_dgesv")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: n, nrhs, lda, ldb
      real(c_double), intent(inout) :: A(lda, *), B(ldb, *)
      integer(c_int), intent(out) :: ipiv(*), info
    end function
    integer(c_int) function bem_reorganize(ctx, FI, DFI) bind(C, name="bem_reorganize")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: FI(*), DFI(27, *)
    end function
    integer(c_int) function bem_boundary_stresses(ctx, se, sn, pr, vm) bind(C, name="bem_boundary_stresses")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      real(c_double), intent(out) :: se(6, 9, *), sn(6, *), pr(3, *), vm(*)
    end function
    integer(c_int) function bem_internal_points(ctx, l, cx, cy, cz, u, s, p, vm, flags) &
        bind(C, name="bem_internal_points")
      import :: c_ptr, c_int, c_double
      type(c_ptr), value :: ctx
      integer(c_int), value :: l, flags
      real(c_double), intent(in) :: cx(*), cy(*), cz(*)
      real(c_double), intent(out) :: u(3, *), s(6, *), p(3, *), vm(*)
    end function
  end interface
end module bem3d_b200

module assembly_gpu_mod
  use, intrinsic :: iso_c_binding
  use data_mod
  use stress_mod, only: sigma_elem, sigma_node, sigma_principal, sigma_vm, &
                        u_int, sigma_int, sigma_int_prin, sigma_int_vm
  use bem3d_b200
  implicit none

  type(c_ptr), save :: gpu_ctx = c_null_ptr
  integer(c_int), save :: gpu_device = 0                 ! CUDA device of the context
  integer(c_int), save :: gpu_precision = BEM_PREC_FP32_IR
  real(c_double), save :: gpu_tolerance = 1.0e-15_c_double
  integer(c_int), save :: gpu_max_iter = 60

contains

  subroutine gpu_check(rc, what)
    integer(c_int), intent(in) :: rc
    character(len=*), intent(in) :: what
    character(kind=c_char), pointer :: msg(:)
    integer :: i
    if (rc >= 0) return
    write(*, '(A, A, A, I4)') ' *** GPU error in ', what, ': status ', rc
    call c_f_pointer(bem_last_error(gpu_ctx), msg, [512])
    do i = 1, 512
      if (msg(i) == c_null_char) exit
      write(*, '(A)', advance='no') msg(i)
    end do
    write(*, *)
    stop 'GPU failure in the B200 hot path.'
  end subroutine gpu_check

  subroutine precompute_element_geometry()
    if (.not. c_associated(gpu_ctx)) call gpu_check(bem_ctx_create(gpu_ctx, gpu_device), 'bem_ctx_create')
    call gpu_check(bem_set_mesh(gpu_ctx, n, ne, x, y, z, nconec, kconec), 'bem_set_mesh')
    call gpu_check(bem_set_material(gpu_ctx, rge, xnu), 'bem_set_material')
    call gpu_check(bem_set_bc(gpu_ctx, kode, bc), 'bem_set_bc')
    call gpu_check(bem_precompute_geometry(gpu_ctx), 'bem_precompute_geometry')
  end subroutine precompute_element_geometry

  ! A is assembled and kept in GPU memory (43.5 GB at 73,734 DOF); FI comes back.
  subroutine ghmat8()
    call gpu_check(bem_ghmat8(gpu_ctx, BEM_ASM_FP64, c_null_ptr, 0_c_int64_t, FI), 'bem_ghmat8')
  end subroutine ghmat8

  ! The system is the one ghmat8 left on the GPU; A_mat is not touched (main.f90
  ! passes the module's A, which a GPU build need not allocate at full size).
  subroutine solve_linear_system(A_mat, B_vec, n_size)
    integer, intent(in) :: n_size
    real(dp), intent(inout) :: A_mat(:, :)
    real(dp), intent(inout) :: B_vec(n_size)
    integer(c_int) :: info
    call gpu_check(bem_solve(gpu_ctx, gpu_precision, gpu_tolerance, gpu_max_iter, B_vec, info, c_null_ptr), &
                   'bem_solve')
    if (info /= 0) then
      write(*, '(A, I6)') ' *** ERROR in LAPACK DGESV: info = ', info
      stop 'Solver failure: Singular matrix or bad arguments in LAPACK DGESV.'
    end if
  end subroutine solve_linear_system

  subroutine reorganize_solution()
    call gpu_check(bem_reorganize(gpu_ctx, FI, DFI), 'bem_reorganize')
  end subroutine reorganize_solution

  subroutine compute_boundary_stresses()
    if (allocated(sigma_elem)) deallocate(sigma_elem)
    if (allocated(sigma_node)) deallocate(sigma_node, sigma_principal, sigma_vm)
    allocate(sigma_elem(6, 9, ne), sigma_node(6, n), sigma_principal(3, n), sigma_vm(n))
    call gpu_check(bem_boundary_stresses(gpu_ctx, sigma_elem, sigma_node, sigma_principal, sigma_vm), &
                   'bem_boundary_stresses')
  end subroutine compute_boundary_stresses

  subroutine compute_internal_points()
    integer :: ip
    if (l <= 0) return
    if (allocated(u_int)) deallocate(u_int, sigma_int, sigma_int_prin, sigma_int_vm)
    allocate(u_int(3, l), sigma_int(6, l), sigma_int_prin(3, l), sigma_int_vm(l))
    call gpu_check(bem_internal_points(gpu_ctx, l, cx, cy, cz, u_int, sigma_int, sigma_int_prin, &
                                       sigma_int_vm, 0_c_int), 'bem_internal_points')
    do ip = 1, l
      dsol(3*ip - 2) = u_int(1, ip)
      dsol(3*ip - 1) = u_int(2, ip)
      dsol(3*ip) = u_int(3, ip)
    end do
  end subroutine compute_internal_points

  subroutine release_gpu()
    integer(c_int) :: rc
    if (c_associated(gpu_ctx)) rc = bem_ctx_destroy(gpu_ctx)
    gpu_ctx = c_null_ptr
  end subroutine release_gpu

end module assembly_gpu_mod
