! iso_c_binding interfaces to libsubfv_b200.so (declarations: include/subfv.h), for the
! reference's Fortran callers (subfvlagrange, subfvns). Written for gfortran with the
! reference's own build; this image has no Fortran compiler, so the file is not compiled
! or tested here (the C-ABI it binds is tested from Python ctypes).
!
! Ids in subfv_mesh_desc are the reference's 1-based ids; host arrays keep the
! reference's layouts (sol(5, n_elems), vp(3, n_vert), grad(3, 5, n_elems),
! diag(5, 5, n_elems), column-major), so they are passed as they are.
module subfv_c
  use, intrinsic :: iso_c_binding
  implicit none
  private

  public :: subfv_mesh_desc, subfv_ns_cfg, subfv_error
  public :: subfv_mesh_create, subfv_mesh_destroy, subfv_mesh_set_coords, subfv_mesh_get_geometry
  public :: subfv_compute_geometry_mesh, subfv_compute_rhs_lagrange, subfv_compute_dt, subfv_move_mesh
  public :: subfv_compute_euler_flux, subfv_compute_cell_grad_from_nodal_grad, subfv_flux_limiting
  public :: subfv_add_timedisc_and_solve
  public :: subfv_bcsr_create, subfv_bcsr_destroy, subfv_bcsr_set_values, subfv_bcsr_matmul, subfv_bcsr_diag
  public :: subfv_bcsr_gmres_diag, subfv_bcsr_gmres

  integer(c_int), parameter, public :: SUBFV_ERR_MESH_CHECK = 1, SUBFV_ERR_NONFINITE = 2, &
    SUBFV_ERR_NEG_DENSITY = 4, SUBFV_ERR_BAD_OMEGA = 8, SUBFV_ERR_GMRES = 16, SUBFV_ERR_INDEX = 32

  ! mesh_type (mesh_module.F90:76-89) flattened: per-entity lists as offsets + values
  type, bind(c) :: subfv_mesh_desc
    integer(c_int32_t) :: n_vert, n_elems, n_faces, n_sub_faces, n_sub_elems, b2d
    type(c_ptr) :: vert_coord, elem_kind, elem_vert_off, elem_vert, elem_sub_elem
    type(c_ptr) :: elem_face_off, elem_face, face_vert_off, face_vert, face_sub_face
    type(c_ptr) :: face_left, face_right, sub_face_vert, sub_face_face
    type(c_ptr) :: sub_face_left_sub_elem, sub_face_right_sub_elem, sub_face_loc
    type(c_ptr) :: sub_elem_elem, sub_elem_vert, sub_elem_loc
    type(c_ptr) :: sub_elem_sub_face_off, sub_elem_sub_face
    type(c_ptr) :: vert_sub_face_off, vert_sub_face, vert_sub_elem_off, vert_sub_elem
    type(c_ptr) :: vert_is_bound, vert_elem_off, vert_elem
  end type subfv_mesh_desc

  ! the namelist entries of ns_global_data_module.F90 the residual path reads
  type, bind(c) :: subfv_ns_cfg
    integer(c_int32_t) :: scheme, second_order, method, bc_style, boundary_2d
    integer(c_int32_t) :: exclude_bound_vert, local_time_step, n_bc
    integer(c_int32_t) :: bc_type(16)
    real(c_double)     :: bc_val(5, 16)
    real(c_double)     :: cfl, tmax
    integer(c_int32_t) :: precision
    integer(c_int32_t) :: activate_diffusion, use_sutherland
    real(c_double)     :: mu_p, mu0, T0, Cv_p
    integer(c_int32_t) :: bc_type_V(16)
    real(c_double)     :: bc_val_V(3, 16)
    integer(c_int32_t) :: bc_type_T(16)
    real(c_double)     :: bc_val_T(16)
    real(c_double)     :: prandtl           ! 0: the reference's Prandtl = 0.71
  end type subfv_ns_cfg

  interface
    function subfv_last_error() bind(c, name="subfv_last_error") result(p)
      import :: c_ptr
      type(c_ptr) :: p
    end function subfv_last_error

    integer(c_int) function subfv_mesh_create(desc, h) bind(c, name="subfv_mesh_create")
      import :: c_int, c_ptr, subfv_mesh_desc
      type(subfv_mesh_desc), intent(in) :: desc
      type(c_ptr), intent(out) :: h
    end function subfv_mesh_create
    integer(c_int) function subfv_mesh_destroy(h) bind(c, name="subfv_mesh_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function subfv_mesh_destroy
    integer(c_int) function subfv_mesh_set_coords(h, coord) bind(c, name="subfv_mesh_set_coords")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: coord(*)
    end function subfv_mesh_set_coords
    integer(c_int) function subfv_mesh_get_geometry(h, name, out) bind(c, name="subfv_mesh_get_geometry")
      import :: c_int, c_ptr, c_double, c_char
      type(c_ptr), value :: h
      character(kind=c_char), intent(in) :: name(*)
      real(c_double), intent(out) :: out(*)
    end function subfv_mesh_get_geometry

    ! compute_geometry_mesh (mesh_geometry_module.F90:16) + check_mesh
    integer(c_int) function subfv_compute_geometry_mesh(h) bind(c, name="subfv_compute_geometry_mesh")
      import :: c_int, c_ptr
      type(c_ptr), value :: h
    end function subfv_compute_geometry_mesh
    ! compute_rhs_lagrange (lagrange_module.F90:14)
    integer(c_int) function subfv_compute_rhs_lagrange(h, sol, vp, rhs, b2d, mass) &
        bind(c, name="subfv_compute_rhs_lagrange")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: sol(*), mass(*)
      real(c_double), intent(inout) :: vp(*), rhs(*)
      integer(c_int), value :: b2d
    end function subfv_compute_rhs_lagrange
    ! compute_dt (lagrange_module.F90:240)
    integer(c_int) function subfv_compute_dt(h, sol, cfl, vp, dt) bind(c, name="subfv_compute_dt")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: sol(*), vp(*)
      real(c_double), value :: cfl
      real(c_double), intent(out) :: dt
    end function subfv_compute_dt
    ! move_mesh (lagrange_module.F90:772)
    integer(c_int) function subfv_move_mesh(h, vp, dt) bind(c, name="subfv_move_mesh")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: vp(*)
      real(c_double), value :: dt
    end function subfv_move_mesh

    ! compute_euler_flux (ns_euler_module.F90:151)
    integer(c_int) function subfv_compute_euler_flux(h, cfg, sol, rhs, grad, sum_lambda, second_order, vp) &
        bind(c, name="subfv_compute_euler_flux")
      import :: c_int, c_ptr, c_double, subfv_ns_cfg
      type(c_ptr), value :: h
      type(subfv_ns_cfg), intent(in) :: cfg
      real(c_double), intent(in) :: sol(*), grad(*)
      real(c_double), intent(out) :: rhs(*), sum_lambda(*), vp(*)
      integer(c_int), value :: second_order
    end function subfv_compute_euler_flux
    ! compute_cell_grad_from_nodal_grad (ns_euler_recon_module.F90:8)
    integer(c_int) function subfv_compute_cell_grad_from_nodal_grad(h, cfg, sol, grad, nodal_grad) &
        bind(c, name="subfv_compute_cell_grad_from_nodal_grad")
      import :: c_int, c_ptr, c_double, subfv_ns_cfg
      type(c_ptr), value :: h
      type(subfv_ns_cfg), intent(in) :: cfg
      real(c_double), intent(in) :: sol(*)
      real(c_double), intent(out) :: grad(*), nodal_grad(*)
    end function subfv_compute_cell_grad_from_nodal_grad
    ! flux_limiting (ns_euler_recon_module.F90:560)
    integer(c_int) function subfv_flux_limiting(h, sol, rhs, rhs_o2, sum_lambda, cfl) &
        bind(c, name="subfv_flux_limiting")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(in) :: sol(*), rhs_o2(*), sum_lambda(*)
      real(c_double), intent(inout) :: rhs(*)
      real(c_double), value :: cfl
    end function subfv_flux_limiting
    ! add_timedisc_and_solve (ns_euler_module.F90:521), one process, global time step
    integer(c_int) function subfv_add_timedisc_and_solve(h, sol, rhs, diag, sum_lambda, delta_sol, res, res_vect, &
        a1, a2, cfl, t, tmax, dt) bind(c, name="subfv_add_timedisc_and_solve")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: h
      real(c_double), intent(inout) :: sol(*), rhs(*), diag(*), sum_lambda(*)
      real(c_double), intent(out) :: delta_sol(*), res, res_vect(5), dt
      real(c_double), value :: a1, a2, cfl, t, tmax
    end function subfv_add_timedisc_and_solve

    ! bcsr_matrix_type and its routines (sparse_bcsr_linear_module.F90)
    integer(c_int) function subfv_bcsr_create(m, bs, row, col, v, a) bind(c, name="subfv_bcsr_create")
      import :: c_int, c_ptr, c_double, c_int32_t
      integer(c_int), value :: m, bs
      integer(c_int32_t), intent(in) :: row(*), col(*)
      real(c_double), intent(in) :: v(*)
      type(c_ptr), intent(out) :: a
    end function subfv_bcsr_create
    integer(c_int) function subfv_bcsr_destroy(a) bind(c, name="subfv_bcsr_destroy")
      import :: c_int, c_ptr
      type(c_ptr), value :: a
    end function subfv_bcsr_destroy
    integer(c_int) function subfv_bcsr_set_values(a, v) bind(c, name="subfv_bcsr_set_values")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: a
      real(c_double), intent(in) :: v(*)
    end function subfv_bcsr_set_values
    integer(c_int) function subfv_bcsr_matmul(a, x, y) bind(c, name="subfv_bcsr_matmul")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: a
      real(c_double), intent(in) :: x(*)
      real(c_double), intent(out) :: y(*)
    end function subfv_bcsr_matmul
    integer(c_int) function subfv_bcsr_diag(a, x, b) bind(c, name="subfv_bcsr_diag")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: a
      real(c_double), intent(out) :: x(*)
      real(c_double), intent(in) :: b(*)
    end function subfv_bcsr_diag
    integer(c_int) function subfv_bcsr_gmres_diag(a, x, b, tol, m, conv, restarts, rho) &
        bind(c, name="subfv_bcsr_gmres_diag")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: a
      real(c_double), intent(inout) :: x(*)
      real(c_double), intent(in) :: b(*)
      real(c_double), value :: tol
      integer(c_int), value :: m
      integer(c_int), intent(out) :: conv, restarts
      real(c_double), intent(out) :: rho
    end function subfv_bcsr_gmres_diag
    integer(c_int) function subfv_bcsr_gmres(a, x, b, tol, m, conv, restarts, rho) bind(c, name="subfv_bcsr_gmres")
      import :: c_int, c_ptr, c_double
      type(c_ptr), value :: a
      real(c_double), intent(inout) :: x(*)
      real(c_double), intent(in) :: b(*)
      real(c_double), value :: tol
      integer(c_int), value :: m
      integer(c_int), intent(out) :: conv, restarts
      real(c_double), intent(out) :: rho
    end function subfv_bcsr_gmres
  end interface

contains

  ! the library's last error message as a Fortran string
  function subfv_error() result(msg)
    character(len=:), allocatable :: msg
    character(kind=c_char), pointer :: s(:)
    type(c_ptr) :: p
    integer :: n
    p = subfv_last_error()
    msg = ''
    if (.not. c_associated(p)) return
    call c_f_pointer(p, s, [4096])
    n = 0
    do while (n < 4096)
      if (s(n + 1) == c_null_char) exit
      n = n + 1
    end do
    allocate(character(len=n) :: msg)
    msg = transfer(s(1:n), msg)
  end function subfv_error
end module subfv_c
