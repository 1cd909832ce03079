/* subfv_b200: C-ABI of the B200-native subface finite-volume residual path and its
 * implicit linear solve.
 *
 * The entry points mirror the reference's Fortran module procedures so that a thin
 * iso_c_binding shim can route subfvlagrange / subfvns through them unchanged. All
 * host arrays use the reference's layouts: sol(5, n_elems) and rhs(5, n_elems) are
 * column-major (five values per cell, cell after cell), vp(3, n_vert) likewise,
 * vertex coordinates (3, n_vert). Ids inside descriptors are 1-based like the
 * reference's.
 *
 * Return codes: 0 = OK; > 0 = numerical fault bits (SUBFV_ERR_*); < 0 = API or CUDA
 * error, text in subfv_last_error(). Handles are not thread-safe; each mesh owns one
 * CUDA stream and every call is synchronous unless its name ends in _async.
 */
#ifndef SUBFV_B200_H
#define SUBFV_B200_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SUBFV_ERR_MESH_CHECK 1   /* check_mesh failed: mesh_geometry_module.F90:403-408 */
#define SUBFV_ERR_NONFINITE 2    /* non-finite state, volume or time step */
#define SUBFV_ERR_NEG_DENSITY 4  /* negative density / specific volume: ns_euler_rs_module.F90:257-266 */
#define SUBFV_ERR_BAD_OMEGA 8    /* positivity limiter omega <= 1e-6: ns_euler_module.F90:595-598 */
#define SUBFV_ERR_GMRES 16       /* a Krylov solve did not converge: sparse_bcsr_linear_module.F90:1614,1686,1164 */
#define SUBFV_ERR_INDEX 32       /* an index outside its array */

const char* subfv_last_error(void);
int subfv_version(void);
/* FP64 issue-rate probe (no counterpart in the reference): times fused multiply-adds
 * in eight independent chains per thread over the whole current device and returns the
 * achieved TFLOP/s (2 flops per FMA), the denominator of the FP64 fraction reported
 * for FP64-bound kernels. iters in [1, 2^20]; ~4096 takes a few milliseconds. */
int subfv_probe_fp64_fma(int iters, double* tflops, double* ms);
/* Check of the geometry kernels' exact division by 3 and by 6 (a reciprocal multiply
 * with one FMA remainder correction; no counterpart in the reference): counts, over the
 * n host doubles x, the quotients x/3 and x/6 that differ in any bit from CUDA's
 * division. */
int subfv_probe_div_const(const double* x, int64_t n, int64_t* mismatches);

/* ---------------------------------------------------------------------------------
 * Topology: build_mesh (src/mesh/mesh_connectivity_module.F90:12-59) on the host,
 * from volume elements as the MSH2 reader produces them
 * (src/mesh/mesh_reading_module.F90:989-1324). Numbering is identical to the
 * reference's (BFS vertices, first-touch cells and faces, vertex-ordered subfaces).
 * Arrays are fetched by name (the mesh_type component they flatten, e.g.
 * "face_left", "vert_sub_face_off"). */
typedef struct subfv_topology subfv_topology;
int subfv_topology_build(int n_vert, const double* coords, int n_elems, const int32_t* elem_kind,
                         const int32_t* elem_vert_off, const int32_t* elem_vert, int n_bfaces,
                         const int32_t* bface_off, const int32_t* bface_vert, const int32_t* bface_tag,
                         int b2d, int periodic, subfv_topology** out);
/* The same with a choice of vertex order: renumber 0 is the reference's breadth-first
 * order (subfv_topology_build); 1 orders the vertices along a Hilbert curve (the 2-D
 * curve of (x, y) for slabs, b2d, else the 3-D curve; ties by input id), and cells,
 * faces and subfaces then follow the reference's rules over that order. Results on a
 * renumbered mesh differ from the breadth-first mesh's only in the order of sums. */
int subfv_topology_build_ex(int n_vert, const double* coords, int n_elems, const int32_t* elem_kind,
                            const int32_t* elem_vert_off, const int32_t* elem_vert, int n_bfaces,
                            const int32_t* bface_off, const int32_t* bface_vert, const int32_t* bface_tag,
                            int b2d, int periodic, int renumber, subfv_topology** out);
int64_t subfv_topology_array_len(const subfv_topology* t, const char* name);
int subfv_topology_array_get(const subfv_topology* t, const char* name, int32_t* out);
int subfv_topology_coords(const subfv_topology* t, double* coords_out);
void subfv_topology_destroy(subfv_topology* t);

/* ---- mesh and solution files (host) ----
   read_mesh_msh (mesh_reading_module.F90:154-205) for one process: gmsh ASCII MSH 2 or 4,
   volumes of types 4-7 (tet, hex, prism, pyramid) and boundary faces of types 2-3 whose
   tag is the 1-based index of the bc_names entry naming their physical group (0 when
   none). MSH 2 takes node ids as the nodes' order; MSH 4 keeps the nodes the volumes use,
   numbered in their order in $Nodes (:771-900). The arrays feed subfv_topology_build. */
typedef struct subfv_msh subfv_msh;
int subfv_msh_read(const char* path, int n_bc, const char* const* bc_names, subfv_msh** out);
/* sizes: n_vert, n_elems, len(elem_vert), n_boundary_faces, len(bface_vert) */
int subfv_msh_sizes(const subfv_msh* m, int64_t* sizes);
int subfv_msh_get(const subfv_msh* m, double* coords, int32_t* elem_kind, int32_t* elem_vert_off,
                  int32_t* elem_vert, int32_t* bface_off, int32_t* bface_vert, int32_t* bface_tag);
void subfv_msh_destroy(subfv_msh* m);
/* write_sol_vtu (ns_io_module.F90:403-884): ASCII VTU, polyhedral cells with their faces,
   Nodal_Velocity (vp, may be NULL) and the cell fields Centroid (elem_coord, may be NULL),
   Tag, MPI_Color, Density, Momentum, Energy, Velocity, Pressure, Internal_energy, H, Mach,
   Temperature (Cv_p), mu (when mu >= 0) and Residual (norm2 of delta, may be NULL);
   sol (5, n_elems) conservative */
int subfv_write_sol_vtu(const char* path, const subfv_topology* t, const double* sol, const double* delta,
                        const double* vp, const double* elem_coord, double Cv_p, double mu);
/* write_sol_vtu_lag (lagrange_io_module.F90:26-289): the same mesh part, point data Vp
   (3, n_vert) and Pp (nodal pressure, may be NULL), cell data Centroid / Rxy / R
   (elem_coord, may be NULL), Tag, MPI_Color, Density (1 / tau), Velocity, Pressure and
   Internal_energy of the Lagrangian state sol (tau, u, v, w, E) */
int subfv_write_sol_vtu_lag(const char* path, const subfv_topology* t, const double* sol, const double* vp,
                            const double* pp, const double* elem_coord);
/* restart_from_vtu_file (ns_io_module.F90:1333-1382): Density, Momentum and Energy (per
   unit mass) of a VTU written above, into sol (5, n_elems) */
int subfv_restart_from_vtu(const char* path, int64_t n_elems, double* sol);

/* ---------------------------------------------------------------------------------
 * Device mesh. subfv_mesh_desc flattens mesh_type (src/mesh/mesh_module.F90:76-89);
 * the Fortran shim fills it from its mesh after build_mesh. */
typedef struct subfv_mesh_desc {
  int32_t n_vert, n_elems, n_faces, n_sub_faces, n_sub_elems;
  int32_t b2d;
  const double* vert_coord;             /* (3, n_vert) */
  const int32_t* elem_kind;             /* (n_elems) */
  const int32_t* elem_vert_off;         /* (n_elems+1); also offsets of elem%sub_elem */
  const int32_t* elem_vert;             /* elem%vert */
  const int32_t* elem_sub_elem;         /* elem%sub_elem */
  const int32_t* elem_face_off;         /* (n_elems+1) */
  const int32_t* elem_face;             /* elem%face */
  const int32_t* face_vert_off;         /* (n_faces+1); also offsets of face%sub_face */
  const int32_t* face_vert;             /* face%vert */
  const int32_t* face_sub_face;         /* face%sub_face */
  const int32_t* face_left;             /* face%left_neigh */
  const int32_t* face_right;            /* face%right_neigh: >0 cell, 0 wall, <0 -bc tag */
  const int32_t* sub_face_vert;         /* sub_face%mesh_vert */
  const int32_t* sub_face_face;         /* sub_face%mesh_face */
  const int32_t* sub_face_left_sub_elem;  /* sub_face%left_sub_elem_neigh */
  const int32_t* sub_face_right_sub_elem; /* sub_face%right_sub_elem_neigh (0 none) */
  const int32_t* sub_face_loc;          /* sub_face%id_loc_around_node */
  const int32_t* sub_elem_elem;         /* sub_elem%mesh_elem */
  const int32_t* sub_elem_vert;         /* sub_elem%mesh_vert */
  const int32_t* sub_elem_loc;          /* sub_elem%id_loc_around_node */
  const int32_t* sub_elem_sub_face_off; /* (n_sub_elems+1) */
  const int32_t* sub_elem_sub_face;     /* sub_elem%sub_face */
  const int32_t* vert_sub_face_off;     /* (n_vert+1) */
  const int32_t* vert_sub_face;         /* vert%sub_face_neigh */
  const int32_t* vert_sub_elem_off;     /* (n_vert+1) */
  const int32_t* vert_sub_elem;         /* vert%sub_elem_neigh */
  const int32_t* vert_is_bound;         /* vert%is_bound (0/1) */
  const int32_t* vert_elem_off;         /* (n_vert+1), or NULL when no second-order NS is run */
  const int32_t* vert_elem;             /* vert%elem_neigh */
} subfv_mesh_desc;

typedef struct subfv_mesh subfv_mesh;
int subfv_mesh_create(const subfv_mesh_desc* desc, subfv_mesh** out);
int subfv_mesh_create_from_topology(const subfv_topology* t, int b2d, subfv_mesh** out);
int subfv_mesh_destroy(subfv_mesh* m);
int64_t subfv_mesh_device_bytes(const subfv_mesh* m);
int subfv_mesh_set_coords(subfv_mesh* m, const double* vert_coord);
int subfv_mesh_get_coords(subfv_mesh* m, double* vert_coord);
/* name: vert_volume, face_coord, face_norm, face_area, sub_face_norm, sub_face_area,
 * elem_coord, elem_volume, sub_elem_volume (reference layouts); vert_is_bound as 0/1 doubles */
int subfv_mesh_get_geometry(subfv_mesh* m, const char* name, double* out);

/* compute_geometry_mesh(mesh, .true., b2d) — src/mesh/mesh_geometry_module.F90:16-57.
 * Returns SUBFV_ERR_MESH_CHECK where the reference would print and error stop. */
int subfv_compute_geometry_mesh(subfv_mesh* m);

/* ---------------------------------------------------------------------------------
 * Lagrangian hydro (subfvlagrange), scheme "classic". */

/* compute_rhs_lagrange(mesh, sol, vp, dt, rhs, n_bc, bc_type, bc_val, b2d, mass) —
 * src/lagrange/lagrange_module.F90:14-147. sol/rhs (5, n_elems), vp (3, n_vert). */
int subfv_compute_rhs_lagrange(subfv_mesh* m, const double* sol, double* vp, double* rhs,
                               int b2d, const double* mass);
/* compute_rhs_lagrange_sidil(mesh, sol, vp, dt, rhs, n_bc, bc_type, bc_val, b2d, mass,
 * method, b2d_h) — lagrange_module.F90:149-223 with compute_nodal_velocity_sidil,
 * compute_nodal_pressure_sidil and compute_length (:538-711): scheme "sidil", FP64.
 * method_length 0..4; b2d_h is unused by the reference. A negative nodal pressure (the
 * reference's error stop) sets SUBFV_ERR_NEG_DENSITY in the returned status. */
int subfv_compute_rhs_lagrange_sidil(subfv_mesh* m, const double* sol, double* vp, double* rhs, int b2d,
                                     const double* mass, int method_length);
/* compute_dt(mesh, sol, dt, cfl, vp, me, num_procs) — lagrange_module.F90:240-283 */
int subfv_compute_dt(subfv_mesh* m, const double* sol, double cfl, const double* vp, double* dt);
/* No counterpart in the reference. compute_dt for callers that cannot allocate device
 * memory when they call (all device memory reserved at start-up, or an allocator owned
 * by a host application): d_sol (5, n_elems), d_vp (3, n_vert) and d_dt (one double)
 * are device buffers the caller owns; nothing is allocated or freed. Scratch is a
 * static 128 KiB device array (one minimum per 256 cells), so meshes above 4,194,304
 * cells are rejected (-4). The first call on a device looks up that array's device
 * address (and, under lazy module loading, loads the module that holds it): make it at
 * start-up, before device memory is reserved and before any stream capture. Calls
 * share the array: do not let two calls overlap on the GPU. Runs on the mesh's stream,
 * on the mesh's device whichever device is current, and returns after it finishes; the
 * mesh's stream does not wait for the caller's, so d_sol and d_vp must be complete
 * before the call. The result and the status (SUBFV_ERR_NONFINITE on a negative or NaN
 * CFL term) equal subfv_compute_dt's. */
int subfv_compute_dt_noalloc(subfv_mesh* m, const double* d_sol, const double* d_vp, double cfl, double* d_dt);
/* move_mesh(mesh, vp, dt) — lagrange_module.F90:772-784 */
int subfv_move_mesh(subfv_mesh* m, const double* vp, double dt);

/* Device-resident time loop of lagrange_main.F90:89-127: state, mass and mesh stay in
 * HBM; each step = rhs, CFL reduction, mesh motion, geometry, update. The step loop
 * is replayed from a captured CUDA graph. precision 0: plain FP64 (bit-identical to the
 * reference's arithmetic); 1: the per-face wave speeds in FP32, the nodal 3x3 solve,
 * star pressures, fluxes, positions, volumes and sums in FP64 (totals conserved to
 * FP64 rounding). */
typedef struct subfv_lag_state subfv_lag_state;
int subfv_lag_state_create(subfv_mesh* m, const double* sol, const double* mass, double cfl,
                           double t0, double t_max, int precision, subfv_lag_state** out);
int subfv_lag_state_destroy(subfv_lag_state* s);
/* The state's scheme (lagrange_main.F90:91-100): 0 "classic" (default), 1 "sidil" with
 * method_length 0..4 (FP64 whatever the state's precision). */
int subfv_lag_state_set_scheme(subfv_lag_state* s, int scheme, int method_length);
/* run n_steps (stops early once t >= t_max); returns status bits */
int subfv_lag_advance(subfv_lag_state* s, int n_steps, int* steps_done, double* t);
/* captures the graph the time loop replays (done by the first advance otherwise); the
   state does not move */
int subfv_lag_prepare(subfv_lag_state* s);
int subfv_lag_advance_async(subfv_lag_state* s, int n_steps);
int subfv_lag_sync(subfv_lag_state* s, int* steps_done, double* t);
int subfv_lag_get_sol(subfv_lag_state* s, double* sol);
int subfv_lag_set_sol(subfv_lag_state* s, const double* sol);
int subfv_lag_get_vp(subfv_lag_state* s, double* vp);
int subfv_lag_last_dt(subfv_lag_state* s, double* dt);
/* one step through host buffers: uploads sol, advances one step, downloads sol */
int subfv_lag_step_host(subfv_lag_state* s, double* sol_inout);
/* Runs n_steps steps launched one kernel at a time with CUDA events between kernels on
 * the mesh's stream; kernel_ms[0..6] receives the summed milliseconds of each kernel in
 * step order: face wave speeds, node, cell, finalize, move, face geometry, cell
 * geometry + update. */
int subfv_lag_profile_steps(subfv_lag_state* s, int n_steps, double* kernel_ms);

/* The CUDA stream (cudaStream_t) all work of this mesh is launched on. */
void* subfv_mesh_stream(subfv_mesh* m);

/* ---------------------------------------------------------------------------------
 * Explicit Euler (subfvns): compute_euler_flux with the multi-point nodal solver or the
 * two-wave subface flux, second-order reconstruction with limiters, flux limiting and
 * add_timedisc_and_solve, first order or the two-stage scheme of ns_main.F90:83-107.
 * Conservative state sol(5, n_elems) = (rho, rho u, rho v, rho w, E). */
typedef struct subfv_ns_cfg {
  int32_t scheme;             /* 1 multi_point, 2 multi_point_iso, 3 three_wave, 4 two_wave,
                                 5 modified_three_wave, 6 multi_point_pressure,
                                 8 multi_point_pressure_ph (ns_global_data_module.F90:67-73) */
  int32_t second_order;       /* 0 / 1 */
  int32_t method;             /* cell gradient: 0 or 1 (none), 2-6 (compute_cell_grad_method_2..6,
                                 ns_euler_recon_module.F90:166-320) */
  int32_t bc_style;           /* 0, 1, 2 */
  int32_t boundary_2d;        /* one-cell slab: z-faces are walls */
  int32_t exclude_bound_vert; /* boundary vertices use two_wave */
  int32_t local_time_step;    /* must be 0 (global time step) */
  int32_t n_bc;               /* boundary tags in use (<= 16) */
  int32_t bc_type[16];        /* per tag (ns_global_data_module.F90:53-61): 1 wall, 2 adherence
                                 wall, 3 freestream, 4 outflow supersonic, 5 pondered inflow,
                                 6 double-Mach inflow/outflow, 7 double-Mach bottom, 8 / 9
                                 potential flow 2-D / 3-D; others are rejected */
  double bc_val[16][5];       /* per tag: primitive (rho, u, v, w, p) */
  double cfl, tmax;
  int32_t precision;          /* 0 plain FP64; 1 FP32 wave-speed bounds of the nodal solver;
                                 2 also FP32 flux, reconstruction and limiter arithmetic
                                 (nodal 3x3 systems, the flux's pressure-jump term and all
                                 sums FP64 in both, so totals are conserved to FP64
                                 rounding) */
  /* Navier-Stokes diffusion (namelist entries of ns_global_data_module.F90:10-46, 111):
     momentum and heat assembled point-implicitly into the cells' 5x5 blocks, always FP64.
     Explicit time loop and residual entry point only, on meshes without periodic faces. */
  int32_t activate_diffusion;
  int32_t use_sutherland;     /* mu from Sutherland's law (mu0, T0, C0 = 110.4), else mu_p */
  double mu_p, mu0, T0, Cv_p; /* reference defaults 1.329e-5, 1.716e-5, 273.15, 720.19471 */
  int32_t bc_type_V[16];      /* per tag: 0 or 1 neumann, 2 dirichlet (velocity bc_val_V) */
  double bc_val_V[16][3];
  int32_t bc_type_T[16];      /* per tag: 0 or 1 neumann, 2 dirichlet (temperature bc_val_T) */
  double bc_val_T[16];
  double prandtl;             /* kappa = mu Cv_p gamma / prandtl; 0 stands for the reference's
                                 parameter Prandtl = 0.71 (ns_global_data_module.F90:10) */
} subfv_ns_cfg;

/* compute_rhs_ns (ns_main.F90:130-179, no diffusion): one residual evaluation.
 * rhs (5, n_elems), sum_lambda (n_elems, first-order pass), vp (3, n_vert) of the last
 * pass, cell_grad (3, 5, n_elems) or NULL. Host arrays. */
int subfv_compute_rhs_ns(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs,
                         double* sum_lambda, double* vp, double* cell_grad);

/* The procedures compute_rhs_ns and ns_main's loop call, one at a time, so a shim can
 * keep ns_main.F90:83-107 as it is. Host arrays in the reference's layouts; each call
 * uploads its inputs, runs on the mesh's stream and downloads its outputs.
 *
 * compute_euler_flux(mesh, sol, rhs, grad, sum_lambda, second_order, vp, h_p, mat_h_p) —
 * ns_euler_module.F90:151-339 with the subface scheme of cfg (h_p and mat_h_p belong to
 * the ZB schemes, which are not provided). sol (5, n_elems) and, when second_order, the
 * cell gradients grad (3, 5, n_elems) in; rhs (5, n_elems), sum_lambda (n_elems, started
 * at 1e-12) and vp (3, n_vert, the multi-point nodal velocities; may be NULL) out. */
int subfv_compute_euler_flux(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs,
                             const double* grad, double* sum_lambda, int second_order, double* vp);
/* compute_cell_grad_from_nodal_grad(mesh, sol, grad, all_nodal_grad, method) —
 * ns_euler_recon_module.F90:8-59, method = cfg->method (the nodal least-squares
 * gradients, then the cell gradient of the method with the physical slope limiter and the
 * relaxed maximum principle). sol (5, n_elems) in; grad (3, 5, n_elems) and nodal_grad
 * (3, 5, n_vert; may be NULL) out. */
int subfv_compute_cell_grad_from_nodal_grad(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol,
                                            double* grad, double* nodal_grad);
/* flux_limiting(mesh, sol, rhs, rhs_o2, sum_lambda, cfl) — ns_euler_recon_module.F90:560-601:
 * rhs (5, n_elems) in and out, sol and rhs_o2 (5, n_elems) and sum_lambda (n_elems) in. */
int subfv_flux_limiting(subfv_mesh* m, const double* sol, double* rhs, const double* rhs_o2,
                        const double* sum_lambda, double cfl);
/* add_timedisc_and_solve(mesh, sol, rhs, diag, sum_lambda, delta_sol, res, res_vect,
 * num_procs, me, a1, a2, cfl, t, dt) — ns_euler_module.F90:521-609 on one process with
 * the global time step (tmax, the namelist's, is an argument). In and out: sol (5,
 * n_elems), rhs (5, n_elems; + a1 V/dt sol on return), diag (5, 5, n_elems column-major
 * per cell; the LU factors of diag + a1 V/dt I on return, as dgetrf leaves them; NULL
 * stands for zero blocks), sum_lambda (zeroed). Out: delta_sol (5, n_elems), *res (the
 * sum of norm2(delta) in cell order), res_vect (5), *dt. Returns SUBFV_ERR_BAD_OMEGA,
 * with sol not advanced, where the reference prints "BAD OMEGA" and stops. */
int subfv_add_timedisc_and_solve(subfv_mesh* m, double* sol, double* rhs, double* diag, double* sum_lambda,
                                 double* delta_sol, double* res, double* res_vect, double a1, double a2,
                                 double cfl, double t, double tmax, double* dt);

typedef struct subfv_ns_state subfv_ns_state;
/* compute_rhs_ns with the diffusion blocks: mat_diag (5, 5, n_elems), column-major per
   cell, as ns_main.F90:130-179 leaves it for add_timedisc_and_solve (may be NULL) */
int subfv_compute_rhs_ns_ex(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double* rhs,
                            double* sum_lambda, double* vp, double* cell_grad, double* mat_diag);
int subfv_ns_state_create(subfv_mesh* m, const subfv_ns_cfg* cfg, const double* sol, double t0,
                          subfv_ns_state** out);
int subfv_ns_state_destroy(subfv_ns_state* s);
/* n_steps iterations of ns_main.F90:83-107 (stops once t >= tmax); status bits */
/* captures the graph the time loop replays (done by the first advance otherwise): set-up
   that a caller may take out of its timed region; the state does not move */
int subfv_ns_prepare(subfv_ns_state* s);
int subfv_ns_advance(subfv_ns_state* s, int n_steps, int* steps_done, double* t);
int subfv_ns_advance_async(subfv_ns_state* s, int n_steps);
int subfv_ns_sync(subfv_ns_state* s, int* steps_done, double* t);
int subfv_ns_get_sol(subfv_ns_state* s, double* sol);
/* Node kernel layout: 0 one thread per vertex (the default from 32,768 vertices up), 1 a
 * group of lanes per vertex (8, 16 or 32 as the mesh needs, one per subface) with the
 * per-vertex sums formed in shared memory (the default on smaller meshes); 8, 16 or 32:
 * a group of at least that many lanes. With a group layout the second-order cell
 * gradient also runs a group of 8 lanes per cell (one per vertex) when no cell has more
 * than 8 vertices. Results are bit-identical in every layout. */
int subfv_ns_state_set_node_kernel(subfv_ns_state* s, int lanes);
/* res = sum of |delta|_2 and res_vect(5) of the last add_timedisc_and_solve call */
int subfv_ns_residuals(subfv_ns_state* s, double* res, double* res_vect, double* dt);
/* No counterpart in the reference (its NS path is point-implicit only). One backward
 * Euler step U += dU with (V/dt I - d rhs/dU) dU = rhs(U): rhs the first-order two-wave
 * residual, its Jacobian assembled exactly with the wave speeds frozen, solved by
 * block-Jacobi GMRES(krylov) to |r| < rel_tol |rhs| (or FP64 iterative refinement around
 * an FP32-matrix GMRES when refine_fp32); dt = cfl_implicit * min V / sum_lambda. With
 * activate_diffusion the viscous and heat terms join the residual and their
 * point-implicit blocks mat_diag (the reference's add_timedisc_and_solve solves
 * (mat_diag + V/dt I) U^{n+1} = rhs + V/dt U^n) join the diagonal blocks, the right-hand
 * side being rhs - mat_diag U. */
typedef struct subfv_implicit_stats {
  double dt, b_norm, res_norm;
  int32_t conv, restarts, outer;
  double ms_assemble, ms_solve, ms_update;
  int64_t nnz_blocks;
} subfv_implicit_stats;
int subfv_ns_implicit_step(subfv_ns_state* s, double cfl_implicit, int krylov, double rel_tol, int refine_fp32,
                           subfv_implicit_stats* stats);
/* The same with the preconditioner chosen: 1 block Jacobi (bcsr_gmres_diag, 40
 * restarts), 2 the coloured LU-SGS (bcsr_gmres_parallel_lusgs, 20 restarts; the cells
 * are coloured greedily in order, once per mesh). */
int subfv_ns_implicit_step_ex(subfv_ns_state* s, double cfl_implicit, int krylov, double rel_tol, int refine_fp32,
                              int precond, subfv_implicit_stats* out);
/* The assembled matrix at the state's current U for a given dt (bcsr_matrix_type layout,
 * 1-based row/col, blocks column-major); returns the number of blocks. */
int subfv_ns_be_jacobian(subfv_ns_state* s, double dt, int32_t* row, int32_t* col, double* v, int64_t cap);
/* Gresho vortex of ns_euler_exact_sol_module.F90:7-44 at the cell centroids, as
 * conservative variables (init_sol with init_gresho, ns_euler_module.F90:49-53). */
int subfv_ns_init_gresho(subfv_mesh* m, double mach, double* sol);

/* ---------------------------------------------------------------------------------
 * Batched and served explicit Euler. No counterpart in the reference, whose
 * ns_main.F90:83-107 loop advances one mesh per process: here many independent problems
 * (each its own mesh, initial state and end time, one shared subfv_ns_cfg) are advanced
 * together in shared persistent launches with the step loop captured in a CUDA graph.
 * Each problem's result is bit-identical to the same problem run alone through
 * subfv_ns_state. Problems may join (subfv_ns_batch_add) and leave
 * (subfv_ns_batch_remove) between calls while earlier steps are still running. */
#define SUBFV_BATCH_FULL (-3) /* no free slot or the HBM budget is exhausted: retry later */
typedef struct subfv_ns_batch subfv_ns_batch;
/* capacity: the most problems in flight; budget_bytes: the device bytes that admitted
 * problems (their meshes plus their state) may hold. */
int subfv_ns_batch_create(const subfv_ns_cfg* cfg, int capacity, int64_t budget_bytes, subfv_ns_batch** out);
int subfv_ns_batch_destroy(subfv_ns_batch* b);
/* Device bytes of the per-problem state batch b allocates for a problem on mesh m. */
int64_t subfv_ns_batch_state_bytes(const subfv_ns_batch* b, const subfv_mesh* m);
int64_t subfv_ns_batch_free_bytes(const subfv_ns_batch* b);
int subfv_ns_batch_size(const subfv_ns_batch* b, int* n_live, int64_t* used_bytes);
/* Admit a problem: mesh (with geometry computed), sol (5, n_elems) conservative, start
 * time t0 and end time tmax. take_mesh != 0 hands the mesh over: the batch destroys it
 * when the problem is removed. Returns SUBFV_BATCH_FULL when it cannot be admitted now. */
int subfv_ns_batch_add(subfv_ns_batch* b, subfv_mesh* m, int take_mesh, const double* sol, double t0, double tmax,
                       int* slot);
int subfv_ns_batch_remove(subfv_ns_batch* b, int slot);
/* Enqueue n_steps steps of every problem (finished problems are skipped on the device)
 * and a snapshot of every problem's time, step count, done flag and status. Returns
 * without waiting. */
int subfv_ns_batch_advance(subfv_ns_batch* b, int n_steps);
/* subfv_ns_batch_advance timed on the device (CUDA events around the enqueued steps,
 * including the snapshot copy); waits for the end of the steps. */
int subfv_ns_batch_time_steps(subfv_ns_batch* b, int n_steps, double* ms);
/* Take the oldest outstanding snapshot: wait != 0 blocks for it; wait == 0 returns 1 if
 * it is not complete yet. */
int subfv_ns_batch_poll(subfv_ns_batch* b, int wait);
/* Wait for everything enqueued and take a snapshot of the state after it. */
int subfv_ns_batch_sync(subfv_ns_batch* b);
/* From the latest snapshot taken: returns 1 (and t0, 0 steps) while no snapshot taken
 * covers the problem yet. */
int subfv_ns_batch_slot_info(const subfv_ns_batch* b, int slot, double* t, int64_t* steps, int* done,
                             unsigned* status);
/* Copy a problem's state to the host (waits for the queued steps unless the latest
 * snapshot shows the problem finished). */
int subfv_ns_batch_get_sol(subfv_ns_batch* b, int slot, double* sol);
/* Launch shape: block_v threads (one per vertex) per block of the vertex kernels (64,
 * 128 or 256), and the persistent grid sizes of the vertex and cell kernels. Results do
 * not depend on it. */
int subfv_ns_batch_set_launch(subfv_ns_batch* b, int block_v, int grid_v, int grid_c);
/* Node kernel layout of the batch, as subfv_ns_state_set_node_kernel. */
int subfv_ns_batch_set_node_kernel(subfv_ns_batch* b, int lanes);

/* ---------------------------------------------------------------------------------
 * Batched and served Lagrangian hydro. No counterpart in the reference (one mesh per
 * lagrange_main.F90 process): many independent problems, each its own mesh (moved by its
 * steps), initial state, mass, CFL number and end time, advanced together in shared
 * launches; each result is bit-identical to the same problem run alone through
 * subfv_lag_state. Calls and semantics as for subfv_ns_batch_*. */
typedef struct subfv_lag_batch subfv_lag_batch;
int subfv_lag_batch_create(int precision, int capacity, int64_t budget_bytes, subfv_lag_batch** out);
int subfv_lag_batch_destroy(subfv_lag_batch* b);
int64_t subfv_lag_batch_state_bytes(const subfv_lag_batch* b, const subfv_mesh* m);
int64_t subfv_lag_batch_free_bytes(const subfv_lag_batch* b);
int subfv_lag_batch_size(const subfv_lag_batch* b, int* n_live, int64_t* used_bytes);
/* sol (5, n_elems), mass (n_elems) as for subfv_lag_state_create; returns
 * SUBFV_BATCH_FULL when the problem cannot be admitted now. */
int subfv_lag_batch_add(subfv_lag_batch* b, subfv_mesh* m, int take_mesh, const double* sol, const double* mass,
                        double cfl, double t0, double t_max, int* slot);
int subfv_lag_batch_remove(subfv_lag_batch* b, int slot);
int subfv_lag_batch_advance(subfv_lag_batch* b, int n_steps);
int subfv_lag_batch_time_steps(subfv_lag_batch* b, int n_steps, double* ms);
int subfv_lag_batch_poll(subfv_lag_batch* b, int wait);
int subfv_lag_batch_sync(subfv_lag_batch* b);
int subfv_lag_batch_slot_info(const subfv_lag_batch* b, int slot, double* t, int64_t* steps, int* done,
                              unsigned* status);
int subfv_lag_batch_get_sol(subfv_lag_batch* b, int slot, double* sol);
/* persistent grid size of every batched kernel; results do not depend on it */
int subfv_lag_batch_set_grid(subfv_lag_batch* b, int grid);

/* ---------------------------------------------------------------------------------
 * Block-CSR linear algebra (src/linear_algebra/sparse_bcsr_linear_module.F90).
 * bcsr_matrix_type layout: m block rows, row(m+1) and col(nnz) 1-based, values
 * v(bs, bs, nnz) column-major blocks. Vectors have bs*m entries (host arrays). */
typedef struct subfv_bcsr subfv_bcsr;
int subfv_bcsr_create(int m, int bs, const int32_t* row, const int32_t* col, const double* v,
                      subfv_bcsr** out);
int subfv_bcsr_destroy(subfv_bcsr* A);
int subfv_bcsr_set_values(subfv_bcsr* A, const double* v);
/* y = bcsr_matmul(A, x) — :13-29 */
int subfv_bcsr_matmul(subfv_bcsr* A, const double* x, double* y);
/* bcsr_diag(A, x, b): x = D^-1 b with a no-pivot LU per diagonal block — :1414-1436 */
int subfv_bcsr_diag(subfv_bcsr* A, double* x, const double* b);
/* bcsr_gmres_diag(A, x, b, tol, m, conv, ...) — :1592-1691: restarted GMRES(m),
 * right block-Jacobi preconditioning, absolute tol, 40 restarts. Returns
 * SUBFV_ERR_GMRES when not converged (the reference's conv = .false.). */
int subfv_bcsr_gmres_diag(subfv_bcsr* A, double* x, const double* b, double tol, int m, int* conv,
                          int* restarts, double* rho);
/* Colouring for the parallel LU-SGS preconditioner: colour (1..n_color_sets) of each
 * block row, as bcsr_parallel_lusgs takes it (color, with color_set the rows of each
 * colour; the order of rows inside a set does not change the result). */
int subfv_bcsr_set_colors(subfv_bcsr* A, int n_color_sets, const int32_t* color);
/* bcsr_parallel_lusgs(A, x, b, n_color_sets, color_set, color) — :1438-1502:
 * x = (U+D)^-1 D (L+D)^-1 b, the sweeps ordered by colour set */
int subfv_bcsr_parallel_lusgs(subfv_bcsr* A, double* x, const double* b);
/* bcsr_gmres_parallel_lusgs — :885-993 with modifiedArnoldi_parallel_lusgs (:583-611):
 * restarted GMRES(m) right-preconditioned by the coloured LU-SGS, 20 restarts,
 * absolute tol; conv from the final true residual as the reference sets it */
int subfv_bcsr_gmres_parallel_lusgs(subfv_bcsr* A, double* x, const double* b, double tol, int m, int* conv,
                                    int* restarts, double* rho);
/* bcsr_pcgm(A, x, b, tol) — :1110-1169: conjugate gradients from the initial guess in
 * x, preconditioned by lu_solve (partial pivoting) on each diagonal block (the
 * reference hard-codes 3x3 blocks; any supported block size works here). Returns
 * SUBFV_ERR_GMRES where the reference stops on non-convergence, SUBFV_ERR_NONFINITE on
 * a singular diagonal block. */
int subfv_bcsr_pcgm(subfv_bcsr* A, double* x, const double* b, double tol, int* iters, double* res);
/* bcsr_gmres — :194-290: unpreconditioned, 20 restarts */
int subfv_bcsr_gmres(subfv_bcsr* A, double* x, const double* b, double tol, int m, int* conv,
                     int* restarts, double* rho);
/* Any of the above (precond 1 block Jacobi, 2 coloured LU-SGS, 0 none); H_first (m+1, m)
 * receives the first Arnoldi Hessenberg. */
int subfv_bcsr_gmres_ex(subfv_bcsr* A, double* x, const double* b, double tol, int m, int precond,
                        int* conv, int* restarts, double* rho, double* H_first);
/* No counterpart in the reference: FP64 iterative refinement around block-Jacobi GMRES(m)
 * whose SpMV reads an FP32 copy of the matrix; stops at |b - A x| < rel_tol |b|. */
int subfv_bcsr_gmres_refine(subfv_bcsr* A, double* x, const double* b, double rel_tol, int m, int* conv,
                            int* outer, double* rho);
/* Device time of one SpMV (FP64 or FP32 matrix), averaged over n_iter launches. */
int subfv_bcsr_profile_spmv(subfv_bcsr* A, int n_iter, int fp32, double* ms_per_spmv);

#ifdef __cplusplus
}
#endif
#endif
