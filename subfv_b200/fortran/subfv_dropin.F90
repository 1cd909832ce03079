! Drop-in bodies for the reference's hot-path module procedures, for a build of
! vdelmas/subfv that links libsubfv_b200.so. Each reference procedure keeps its name and
! arguments and calls the dropin_* routine of the same name here, e.g. in
! src/lagrange/lagrange_module.F90:
!
!   subroutine compute_rhs_lagrange(mesh, sol, vp, dt, rhs, n_bc, bc_type, bc_val, b2d, mass)
!     use subfv_dropin, only: dropin_compute_rhs_lagrange
!     ...same declarations as the reference...
!     call dropin_compute_rhs_lagrange(mesh, sol, vp, rhs, b2d, mass)
!   end subroutine compute_rhs_lagrange
!
! so subfvlagrange and subfvns keep their loops. The mesh is flattened once into
! subfv_mesh_desc (1-based ids, as mesh_type holds them) and its device handle is cached
! for the process's one mesh. A positive status maps to the reference's print + error stop;
! a negative one is an API or CUDA error. One process (num_procs = 1): the library does not
! use the MPI decomposition.
!
! Written for gfortran with the reference's own build (it uses mesh_module,
! precision_module, ns_global_data_module and sparse_bcsr_linear_module); this image has no
! Fortran compiler, so the file is not compiled or tested here.
module subfv_dropin
  use, intrinsic :: iso_c_binding
  use precision_module
  use mesh_module
  use subfv_c
  implicit none
  private

  public :: subfv_handle, subfv_release, dropin_ns_cfg
  public :: dropin_compute_geometry_mesh, dropin_compute_rhs_lagrange, dropin_compute_dt, dropin_move_mesh
  public :: dropin_compute_euler_flux, dropin_compute_cell_grad_from_nodal_grad, dropin_flux_limiting
  public :: dropin_add_timedisc_and_solve, dropin_bcsr_matmul, dropin_bcsr_gmres_diag

  type(c_ptr), save :: g_mesh = c_null_ptr
  integer(ENTIER), save :: g_n_vert = -1, g_n_elems = -1

  ! the flattened mesh (kept until subfv_mesh_create has copied it)
  integer(c_int32_t), allocatable, target, save :: f_elem_kind(:), f_elem_vert_off(:), f_elem_vert(:), &
    f_elem_sub_elem(:), f_elem_face_off(:), f_elem_face(:), f_face_vert_off(:), f_face_vert(:), &
    f_face_sub_face(:), f_face_left(:), f_face_right(:), f_sf_vert(:), f_sf_face(:), f_sf_lse(:), f_sf_rse(:), &
    f_sf_loc(:), f_se_elem(:), f_se_vert(:), f_se_loc(:), f_se_sf_off(:), f_se_sf(:), f_v_sf_off(:), f_v_sf(:), &
    f_v_se_off(:), f_v_se(:), f_v_bound(:), f_v_el_off(:), f_v_el(:)
  real(c_double), allocatable, target, save :: f_coord(:, :)

contains

  subroutine stop_on(ierr, what)
    integer(c_int), intent(in) :: ierr
    character(len=*), intent(in) :: what
    if (ierr < 0) then
      print *, 'subfv_b200: ', what, ': ', subfv_error()
      error stop
    end if
  end subroutine stop_on

  ! offsets (0-based starts, n+1 entries) of per-entity lists of the given lengths
  subroutine offsets(len, off)
    integer(ENTIER), intent(in) :: len(:)
    integer(c_int32_t), allocatable, intent(out) :: off(:)
    integer :: i
    allocate(off(size(len) + 1))
    off(1) = 0
    do i = 1, size(len)
      off(i + 1) = off(i) + len(i)
    end do
  end subroutine offsets

  ! The device handle of the mesh, created on first use (after build_mesh and
  ! compute_geometry_mesh have filled mesh_type).
  function subfv_handle(mesh, b2d) result(h)
    type(mesh_type), intent(in) :: mesh
    logical, intent(in) :: b2d
    type(c_ptr) :: h
    type(subfv_mesh_desc) :: d
    integer(ENTIER) :: i, j, k
    integer(ENTIER), allocatable :: len(:)
    integer(c_int) :: ierr

    if (c_associated(g_mesh) .and. g_n_vert == mesh%n_vert .and. g_n_elems == mesh%n_elems) then
      h = g_mesh
      return
    end if
    call subfv_release()

    allocate(f_coord(3, mesh%n_vert))
    do i = 1, mesh%n_vert
      f_coord(:, i) = mesh%vert(i)%coord
    end do
    ! cells: vertices (and their subcells, same offsets), faces
    allocate(f_elem_kind(mesh%n_elems), len(mesh%n_elems))
    do i = 1, mesh%n_elems
      f_elem_kind(i) = mesh%elem(i)%elem_kind
      len(i) = mesh%elem(i)%n_vert
    end do
    call offsets(len, f_elem_vert_off)
    allocate(f_elem_vert(f_elem_vert_off(mesh%n_elems + 1)), f_elem_sub_elem(f_elem_vert_off(mesh%n_elems + 1)))
    do i = 1, mesh%n_elems
      k = f_elem_vert_off(i)
      f_elem_vert(k + 1:k + len(i)) = mesh%elem(i)%vert(1:len(i))
      f_elem_sub_elem(k + 1:k + len(i)) = mesh%elem(i)%sub_elem(1:len(i))
      len(i) = mesh%elem(i)%n_faces
    end do
    call offsets(len, f_elem_face_off)
    allocate(f_elem_face(f_elem_face_off(mesh%n_elems + 1)))
    do i = 1, mesh%n_elems
      k = f_elem_face_off(i)
      f_elem_face(k + 1:k + len(i)) = mesh%elem(i)%face(1:len(i))
    end do
    deallocate(len)
    ! faces: vertices and subfaces (same offsets), neighbours
    allocate(len(mesh%n_faces), f_face_left(mesh%n_faces), f_face_right(mesh%n_faces))
    do i = 1, mesh%n_faces
      len(i) = mesh%face(i)%n_vert
      f_face_left(i) = mesh%face(i)%left_neigh
      f_face_right(i) = mesh%face(i)%right_neigh
    end do
    call offsets(len, f_face_vert_off)
    allocate(f_face_vert(f_face_vert_off(mesh%n_faces + 1)), f_face_sub_face(f_face_vert_off(mesh%n_faces + 1)))
    do i = 1, mesh%n_faces
      k = f_face_vert_off(i)
      f_face_vert(k + 1:k + len(i)) = mesh%face(i)%vert(1:len(i))
      f_face_sub_face(k + 1:k + len(i)) = mesh%face(i)%sub_face(1:len(i))
    end do
    deallocate(len)
    ! subfaces
    allocate(f_sf_vert(mesh%n_sub_faces), f_sf_face(mesh%n_sub_faces), f_sf_lse(mesh%n_sub_faces), &
      f_sf_rse(mesh%n_sub_faces), f_sf_loc(mesh%n_sub_faces))
    do i = 1, mesh%n_sub_faces
      f_sf_vert(i) = mesh%sub_face(i)%mesh_vert
      f_sf_face(i) = mesh%sub_face(i)%mesh_face
      f_sf_lse(i) = mesh%sub_face(i)%left_sub_elem_neigh
      f_sf_rse(i) = mesh%sub_face(i)%right_sub_elem_neigh
      f_sf_loc(i) = mesh%sub_face(i)%id_loc_around_node
    end do
    ! subcells
    allocate(len(mesh%n_sub_elems), f_se_elem(mesh%n_sub_elems), f_se_vert(mesh%n_sub_elems), &
      f_se_loc(mesh%n_sub_elems))
    do i = 1, mesh%n_sub_elems
      len(i) = mesh%sub_elem(i)%n_sub_faces
      f_se_elem(i) = mesh%sub_elem(i)%mesh_elem
      f_se_vert(i) = mesh%sub_elem(i)%mesh_vert
      f_se_loc(i) = mesh%sub_elem(i)%id_loc_around_node
    end do
    call offsets(len, f_se_sf_off)
    allocate(f_se_sf(f_se_sf_off(mesh%n_sub_elems + 1)))
    do i = 1, mesh%n_sub_elems
      k = f_se_sf_off(i)
      f_se_sf(k + 1:k + len(i)) = mesh%sub_elem(i)%sub_face(1:len(i))
    end do
    deallocate(len)
    ! vertices: subfaces, subcells and cells around, boundary flag
    allocate(len(mesh%n_vert), f_v_bound(mesh%n_vert))
    do i = 1, mesh%n_vert
      len(i) = mesh%vert(i)%n_sub_faces_neigh
      f_v_bound(i) = merge(1, 0, mesh%vert(i)%is_bound)
    end do
    call offsets(len, f_v_sf_off)
    allocate(f_v_sf(f_v_sf_off(mesh%n_vert + 1)))
    do i = 1, mesh%n_vert
      k = f_v_sf_off(i)
      f_v_sf(k + 1:k + len(i)) = mesh%vert(i)%sub_face_neigh(1:len(i))
      len(i) = mesh%vert(i)%n_sub_elems_neigh
    end do
    call offsets(len, f_v_se_off)
    allocate(f_v_se(f_v_se_off(mesh%n_vert + 1)))
    do i = 1, mesh%n_vert
      k = f_v_se_off(i)
      f_v_se(k + 1:k + len(i)) = mesh%vert(i)%sub_elem_neigh(1:len(i))
      len(i) = mesh%vert(i)%n_elems_neigh
    end do
    call offsets(len, f_v_el_off)
    allocate(f_v_el(f_v_el_off(mesh%n_vert + 1)))
    do i = 1, mesh%n_vert
      k = f_v_el_off(i)
      do j = 1, len(i)
        f_v_el(k + j) = mesh%vert(i)%elem_neigh(j)
      end do
    end do
    deallocate(len)

    d%n_vert = mesh%n_vert
    d%n_elems = mesh%n_elems
    d%n_faces = mesh%n_faces
    d%n_sub_faces = mesh%n_sub_faces
    d%n_sub_elems = mesh%n_sub_elems
    d%b2d = merge(1, 0, b2d)
    d%vert_coord = c_loc(f_coord)
    d%elem_kind = c_loc(f_elem_kind)
    d%elem_vert_off = c_loc(f_elem_vert_off)
    d%elem_vert = c_loc(f_elem_vert)
    d%elem_sub_elem = c_loc(f_elem_sub_elem)
    d%elem_face_off = c_loc(f_elem_face_off)
    d%elem_face = c_loc(f_elem_face)
    d%face_vert_off = c_loc(f_face_vert_off)
    d%face_vert = c_loc(f_face_vert)
    d%face_sub_face = c_loc(f_face_sub_face)
    d%face_left = c_loc(f_face_left)
    d%face_right = c_loc(f_face_right)
    d%sub_face_vert = c_loc(f_sf_vert)
    d%sub_face_face = c_loc(f_sf_face)
    d%sub_face_left_sub_elem = c_loc(f_sf_lse)
    d%sub_face_right_sub_elem = c_loc(f_sf_rse)
    d%sub_face_loc = c_loc(f_sf_loc)
    d%sub_elem_elem = c_loc(f_se_elem)
    d%sub_elem_vert = c_loc(f_se_vert)
    d%sub_elem_loc = c_loc(f_se_loc)
    d%sub_elem_sub_face_off = c_loc(f_se_sf_off)
    d%sub_elem_sub_face = c_loc(f_se_sf)
    d%vert_sub_face_off = c_loc(f_v_sf_off)
    d%vert_sub_face = c_loc(f_v_sf)
    d%vert_sub_elem_off = c_loc(f_v_se_off)
    d%vert_sub_elem = c_loc(f_v_se)
    d%vert_is_bound = c_loc(f_v_bound)
    d%vert_elem_off = c_loc(f_v_el_off)
    d%vert_elem = c_loc(f_v_el)
    ierr = subfv_mesh_create(d, g_mesh)
    call stop_on(ierr, 'subfv_mesh_create')
    g_n_vert = mesh%n_vert
    g_n_elems = mesh%n_elems
    call free_flat()
    h = g_mesh
  end function subfv_handle

  subroutine free_flat()
    if (allocated(f_coord)) deallocate(f_coord)
    if (allocated(f_elem_kind)) deallocate(f_elem_kind, f_elem_vert_off, f_elem_vert, f_elem_sub_elem, &
      f_elem_face_off, f_elem_face)
    if (allocated(f_face_vert_off)) deallocate(f_face_vert_off, f_face_vert, f_face_sub_face, f_face_left, &
      f_face_right)
    if (allocated(f_sf_vert)) deallocate(f_sf_vert, f_sf_face, f_sf_lse, f_sf_rse, f_sf_loc)
    if (allocated(f_se_elem)) deallocate(f_se_elem, f_se_vert, f_se_loc, f_se_sf_off, f_se_sf)
    if (allocated(f_v_sf_off)) deallocate(f_v_sf_off, f_v_sf, f_v_se_off, f_v_se, f_v_bound, f_v_el_off, f_v_el)
  end subroutine free_flat

  subroutine subfv_release()
    integer(c_int) :: ierr
    if (c_associated(g_mesh)) then
      ierr = subfv_mesh_destroy(g_mesh)
      g_mesh = c_null_ptr
    end if
    g_n_vert = -1
    g_n_elems = -1
  end subroutine subfv_release

  ! ------------------------------------------------------------------ subfvlagrange
  ! compute_geometry_mesh (mesh_geometry_module.F90:16-57) and check_mesh (:374-411) on the
  ! device from mesh%vert%coord; the results are copied back into mesh_type for the rest
  ! of the reference (output, initial state).
  subroutine dropin_compute_geometry_mesh(mesh, use_sub_entities, b2d)
    type(mesh_type), intent(inout) :: mesh
    logical, intent(in) :: use_sub_entities, b2d
    type(c_ptr) :: h
    real(c_double), allocatable :: c(:, :), s(:), v3(:, :)
    integer(c_int) :: ierr
    integer(ENTIER) :: i
    h = subfv_handle(mesh, b2d)
    allocate(c(3, mesh%n_vert))
    do i = 1, mesh%n_vert
      c(:, i) = mesh%vert(i)%coord
    end do
    call stop_on(subfv_mesh_set_coords(h, c), 'subfv_mesh_set_coords')
    ierr = subfv_compute_geometry_mesh(h)
    call stop_on(ierr, 'subfv_compute_geometry_mesh')
    if (iand(ierr, SUBFV_ERR_MESH_CHECK) /= 0) then
      print *, "MESH GEOMETRY IS NOT OK"
      error stop
    end if
    allocate(s(max(mesh%n_vert, mesh%n_elems, mesh%n_faces, mesh%n_sub_faces, mesh%n_sub_elems)))
    allocate(v3(3, max(mesh%n_elems, mesh%n_faces, mesh%n_sub_faces)))
    call stop_on(subfv_mesh_get_geometry(h, c_char_"vert_volume"//c_null_char, s), 'get_geometry')
    do i = 1, mesh%n_vert
      mesh%vert(i)%volume = s(i)
    end do
    call stop_on(subfv_mesh_get_geometry(h, c_char_"elem_volume"//c_null_char, s), 'get_geometry')
    call stop_on(subfv_mesh_get_geometry(h, c_char_"elem_coord"//c_null_char, v3), 'get_geometry')
    do i = 1, mesh%n_elems
      mesh%elem(i)%volume = s(i)
      mesh%elem(i)%coord = v3(:, i)
    end do
    call stop_on(subfv_mesh_get_geometry(h, c_char_"face_area"//c_null_char, s), 'get_geometry')
    do i = 1, mesh%n_faces
      mesh%face(i)%area = s(i)
    end do
    call stop_on(subfv_mesh_get_geometry(h, c_char_"face_norm"//c_null_char, v3), 'get_geometry')
    do i = 1, mesh%n_faces
      mesh%face(i)%norm = v3(:, i)
    end do
    call stop_on(subfv_mesh_get_geometry(h, c_char_"face_coord"//c_null_char, v3), 'get_geometry')
    do i = 1, mesh%n_faces
      mesh%face(i)%coord = v3(:, i)
    end do
    if (use_sub_entities) then
      call stop_on(subfv_mesh_get_geometry(h, c_char_"sub_face_area"//c_null_char, s), 'get_geometry')
      call stop_on(subfv_mesh_get_geometry(h, c_char_"sub_face_norm"//c_null_char, v3), 'get_geometry')
      do i = 1, mesh%n_sub_faces
        mesh%sub_face(i)%area = s(i)
        mesh%sub_face(i)%norm = v3(:, i)
      end do
      call stop_on(subfv_mesh_get_geometry(h, c_char_"sub_elem_volume"//c_null_char, s), 'get_geometry')
      do i = 1, mesh%n_sub_elems
        mesh%sub_elem(i)%volume = s(i)
      end do
    end if
  end subroutine dropin_compute_geometry_mesh

  ! compute_rhs_lagrange (lagrange_module.F90:14-147), scheme "classic"
  subroutine dropin_compute_rhs_lagrange(mesh, sol, vp, rhs, b2d, mass)
    type(mesh_type), intent(in) :: mesh
    real(DOUBLE), intent(in) :: sol(5, mesh%n_elems), mass(mesh%n_elems)
    real(DOUBLE), intent(inout) :: vp(3, mesh%n_vert), rhs(5, mesh%n_elems)
    logical, intent(in) :: b2d
    call stop_on(subfv_compute_rhs_lagrange(subfv_handle(mesh, b2d), sol, vp, rhs, merge(1, 0, b2d), mass), &
      'subfv_compute_rhs_lagrange')
  end subroutine dropin_compute_rhs_lagrange

  ! compute_dt (lagrange_module.F90:240-283)
  subroutine dropin_compute_dt(mesh, sol, dt, cfl, vp, b2d)
    type(mesh_type), intent(in) :: mesh
    real(DOUBLE), intent(in) :: sol(5, mesh%n_elems), vp(3, mesh%n_vert), cfl
    real(DOUBLE), intent(inout) :: dt
    logical, intent(in) :: b2d
    integer(c_int) :: ierr
    ierr = subfv_compute_dt(subfv_handle(mesh, b2d), sol, cfl, vp, dt)
    call stop_on(ierr, 'subfv_compute_dt')
    if (ierr > 0) then
      print *, "compute_dt: non-finite time step"
      error stop
    end if
  end subroutine dropin_compute_dt

  ! move_mesh (lagrange_module.F90:772-784): the device copy and mesh%vert%coord, with the
  ! same arithmetic, so both stay equal
  subroutine dropin_move_mesh(mesh, vp, dt, b2d)
    type(mesh_type), intent(inout) :: mesh
    real(DOUBLE), intent(in) :: vp(3, mesh%n_vert), dt
    logical, intent(in) :: b2d
    integer(ENTIER) :: i
    call stop_on(subfv_move_mesh(subfv_handle(mesh, b2d), vp, dt), 'subfv_move_mesh')
    do i = 1, mesh%n_vert
      mesh%vert(i)%coord = mesh%vert(i)%coord + dt*vp(:, i)
    end do
  end subroutine dropin_move_mesh

  ! ------------------------------------------------------------------ subfvns
  ! the namelist entries the residual path reads (ns_global_data_module.F90), after
  ! read_input_parameters / init_flags
  function dropin_ns_cfg() result(c)
    use ns_global_data_module, only: scheme_id, second_order, method, bc_style, boundary_2d, &
      exclude_bound_vert, local_time_step, n_bc, bc_euler_id, bc_val, cfl, tmax, activate_diffusion, &
      use_sutherland, mu_p, mu0, T0, Cv_p, bc_V_id, bc_val_V, bc_T_id, bc_val_T, Prandtl
    type(subfv_ns_cfg) :: c
    integer :: i
    c%scheme = scheme_id
    c%second_order = merge(1, 0, second_order)
    c%method = method
    c%bc_style = bc_style
    c%boundary_2d = merge(1, 0, boundary_2d)
    c%exclude_bound_vert = merge(1, 0, exclude_bound_vert)
    c%local_time_step = merge(1, 0, local_time_step)
    c%n_bc = n_bc
    c%bc_type = 0
    c%bc_val = 0.0_c_double
    c%bc_type_V = 0
    c%bc_val_V = 0.0_c_double
    c%bc_type_T = 0
    c%bc_val_T = 0.0_c_double
    do i = 1, n_bc
      c%bc_type(i) = bc_euler_id(i)
      c%bc_val(:, i) = bc_val(:, i)
      if (allocated(bc_V_id)) c%bc_type_V(i) = bc_V_id(i)
      if (allocated(bc_T_id)) c%bc_type_T(i) = bc_T_id(i)
      c%bc_val_V(:, i) = bc_val_V(:, i)
      c%bc_val_T(i) = bc_val_T(i)
    end do
    c%cfl = cfl
    c%tmax = tmax
    c%precision = 0
    c%activate_diffusion = merge(1, 0, activate_diffusion)
    c%use_sutherland = merge(1, 0, use_sutherland)
    c%mu_p = mu_p
    c%mu0 = mu0
    c%T0 = T0
    c%Cv_p = Cv_p
    c%prandtl = Prandtl
  end function dropin_ns_cfg

  ! compute_euler_flux (ns_euler_module.F90:151-339); h_p and mat_h_p belong to the ZB
  ! schemes and are not read
  subroutine dropin_compute_euler_flux(mesh, sol, rhs, grad, sum_lambda, second_order, vp)
    use ns_global_data_module, only: boundary_2d
    type(mesh_type), intent(in) :: mesh
    real(DOUBLE), intent(in) :: sol(5, mesh%n_elems), grad(3, 5, mesh%n_elems)
    real(DOUBLE), intent(inout) :: rhs(5, mesh%n_elems), sum_lambda(mesh%n_elems), vp(3, mesh%n_vert)
    logical, intent(in) :: second_order
    integer(c_int) :: ierr
    ierr = subfv_compute_euler_flux(subfv_handle(mesh, boundary_2d), dropin_ns_cfg(), sol, rhs, grad, sum_lambda, &
      merge(1, 0, second_order), vp)
    call stop_on(ierr, 'subfv_compute_euler_flux')
    if (iand(ierr, SUBFV_ERR_NEG_DENSITY) /= 0) then
      print *, "Negative density in multi_point"
      error stop
    end if
  end subroutine dropin_compute_euler_flux

  ! compute_cell_grad_from_nodal_grad (ns_euler_recon_module.F90:8-59)
  subroutine dropin_compute_cell_grad_from_nodal_grad(mesh, sol, grad, all_nodal_grad, method)
    use ns_global_data_module, only: boundary_2d
    type(mesh_type), intent(in) :: mesh
    real(DOUBLE), intent(in) :: sol(5, mesh%n_elems)
    real(DOUBLE), intent(inout) :: grad(3, 5, mesh%n_elems), all_nodal_grad(3, 5, mesh%n_vert)
    integer(ENTIER), intent(in) :: method
    type(subfv_ns_cfg) :: c
    c = dropin_ns_cfg()
    c%method = method
    call stop_on(subfv_compute_cell_grad_from_nodal_grad(subfv_handle(mesh, boundary_2d), c, sol, grad, &
      all_nodal_grad), 'subfv_compute_cell_grad_from_nodal_grad')
  end subroutine dropin_compute_cell_grad_from_nodal_grad

  ! flux_limiting (ns_euler_recon_module.F90:560-601)
  subroutine dropin_flux_limiting(mesh, sol, rhs, rhs_o2, sum_lambda, cfl)
    use ns_global_data_module, only: boundary_2d
    type(mesh_type), intent(in) :: mesh
    real(DOUBLE), intent(in) :: sol(5, mesh%n_elems), rhs_o2(5, mesh%n_elems), sum_lambda(mesh%n_elems), cfl
    real(DOUBLE), intent(inout) :: rhs(5, mesh%n_elems)
    call stop_on(subfv_flux_limiting(subfv_handle(mesh, boundary_2d), sol, rhs, rhs_o2, sum_lambda, cfl), &
      'subfv_flux_limiting')
  end subroutine dropin_flux_limiting

  ! add_timedisc_and_solve (ns_euler_module.F90:521-609), one process, global time step
  subroutine dropin_add_timedisc_and_solve(mesh, sol, rhs, diag, sum_lambda, delta_sol, res, res_vect, a1, a2, &
      cfl, t, dt)
    use ns_global_data_module, only: boundary_2d, tmax, local_time_step
    type(mesh_type), intent(in) :: mesh
    real(DOUBLE), intent(inout) :: sol(5, mesh%n_elems), rhs(5, mesh%n_elems), diag(5, 5, mesh%n_elems)
    real(DOUBLE), intent(inout) :: sum_lambda(mesh%n_elems), delta_sol(5, mesh%n_elems)
    real(DOUBLE), intent(inout) :: res, res_vect(5), dt
    real(DOUBLE), intent(in) :: a1, a2, cfl, t
    integer(c_int) :: ierr
    if (local_time_step) then
      print *, "subfv_b200: local_time_step is not provided"
      error stop
    end if
    ierr = subfv_add_timedisc_and_solve(subfv_handle(mesh, boundary_2d), sol, rhs, diag, sum_lambda, delta_sol, &
      res, res_vect, a1, a2, cfl, t, tmax, dt)
    call stop_on(ierr, 'subfv_add_timedisc_and_solve')
    if (iand(ierr, SUBFV_ERR_BAD_OMEGA) /= 0) then
      print *, "BAD OMEGA"
      error stop
    end if
  end subroutine dropin_add_timedisc_and_solve

  ! ------------------------------------------------------------------ linear algebra
  ! y = bcsr_matmul(A, x) (sparse_bcsr_linear_module.F90:13-29), one device copy of A
  ! per call
  function dropin_bcsr_matmul(A, x) result(y)
    use sparse_bcsr_linear_module, only: bcsr_matrix_type
    type(bcsr_matrix_type), intent(in) :: A
    real(DOUBLE), intent(in) :: x(A%blc_size*A%n)
    real(DOUBLE) :: y(A%blc_size*A%m)
    type(c_ptr) :: d
    integer(c_int) :: ierr
    call stop_on(subfv_bcsr_create(A%m, A%blc_size, A%row, A%col, A%v, d), 'subfv_bcsr_create')
    call stop_on(subfv_bcsr_matmul(d, x, y), 'subfv_bcsr_matmul')
    ierr = subfv_bcsr_destroy(d)
  end function dropin_bcsr_matmul

  ! bcsr_gmres_diag(A, x, b, tol, m, conv, ...) (:1592-1691)
  subroutine dropin_bcsr_gmres_diag(A, x, b, tol, m, conv)
    use sparse_bcsr_linear_module, only: bcsr_matrix_type
    type(bcsr_matrix_type), intent(in) :: A
    real(DOUBLE), intent(inout) :: x(A%blc_size*A%m)
    real(DOUBLE), intent(in) :: b(A%blc_size*A%m), tol
    integer(ENTIER), intent(in) :: m
    logical, intent(out) :: conv
    type(c_ptr) :: d
    integer(c_int) :: ierr, cv, restarts
    real(c_double) :: rho
    call stop_on(subfv_bcsr_create(A%m, A%blc_size, A%row, A%col, A%v, d), 'subfv_bcsr_create')
    ierr = subfv_bcsr_gmres_diag(d, x, b, tol, m, cv, restarts, rho)
    call stop_on(ierr, 'subfv_bcsr_gmres_diag')
    conv = cv /= 0
    ierr = subfv_bcsr_destroy(d)
  end subroutine dropin_bcsr_gmres_diag
end module subfv_dropin
