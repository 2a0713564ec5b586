/* wdg_b200.h -- C ABI of the B200 (sm_100a) wave hot path.
 *
 * Every entry point replaces one operator of the reference waveDG library
 * (arotem3/waveDG) on the 2D, Gauss-Lobatto, approximate-quadrature path; the
 * reference interface each one stands in for is cited beside it
 * (path:line within the reference project).  Layouts are the reference's,
 * column-major with the first index fastest:
 *
 *   state / RHS   u(d, i, j, el)        d = (p, u_x, u_y), i, j < n    (docs/docs.md:55-61)
 *   face traces   uf(i, d, side, edge)                                (wavedg/FaceProlongator.hpp:43)
 *
 * Conventions
 *   - Every function returns 0 (WDG_OK) or a negative WDG_ERR_* code; the
 *     message of the last failure on the calling thread is wdg_last_error().
 *   - Array arguments may be host or device memory; the library asks the CUDA
 *     runtime which.  Host arrays are staged through the handle's device
 *     buffers and the call returns when the result is back on the host.
 *     Device arrays are used in place and the call is asynchronous on the
 *     handle's stream (wdg_wave_set_stream; default: the legacy default
 *     stream); wdg_wave_sync() waits and reports device-side errors.
 *   - Like the reference's operators, a handle is not re-entrant: calls on one
 *     handle must not overlap.  Distinct handles are independent.
 *   - Operator "action" entry points ACCUMULATE into their output, as the
 *     reference's do (source/Div.cpp:174, source/FaceProlongator.cpp:667);
 *     callers zero the output first, exactly as the reference examples do.
 *
 * Boundary codes, one per boundary edge in the mesh's boundary-edge order
 * (the order of Mesh2D::edge(i, FaceType::BOUNDARY)):
 *   0 absorbing / outflow   exterior u_e = t (t.u) + n (p + n.u)/2, p_e = n.u_e
 *                           (the formula wavedg/WaveEquation.hpp:77-84 intends;
 *                           the reference evaluates p_e before u_e)
 *   1 reflecting            wavedg/WaveEquation.hpp:64-69
 *   2 Dirichlet p = 0       mirror state p_e = -p, u_e = u (README.md:6 names
 *                           it; the reference has no 2D implementation)
 */
#ifndef WDG_B200_H
#define WDG_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define WDG_OK 0
#define WDG_ERR_ARG -1         /* invalid argument (sizes, codes, null pointers) */
#define WDG_ERR_CUDA -2        /* a CUDA runtime call failed */
#define WDG_ERR_ALLOC -3       /* device or host allocation failed */
#define WDG_ERR_TIMEOUT -4     /* a bounded device-side wait expired */
#define WDG_ERR_UNSUPPORTED -5 /* degree / precision / feature not built */
#define WDG_ERR_NOT_CONVERGED -6

#define WDG_INTERIOR 0 /* dg::FaceType::INTERIOR (wavedg/Edge.hpp:11-22) */
#define WDG_BOUNDARY 1 /* dg::FaceType::BOUNDARY */

#define WDG_FP64 0 /* state, stepping and reductions in double */
#define WDG_FP32 1 /* state and stepping in float; WaveHoltz filter, residual, norms and energy in double */

typedef struct wdg_mesh wdg_mesh;
typedef struct wdg_wave wdg_wave;
typedef struct wdg_waveholtz wdg_waveholtz;

const char *wdg_last_error(void);
int wdg_version(void);
/* n_colloc values this build has kernels for: writes up to cap entries, returns the count */
int wdg_supported_degrees(int *n_colloc, int cap);

/* ------------------------------------------------------------------ mesh */
/* dg::Mesh2D::from_vertices (source/Mesh2D.cpp:5-92): xy (2, n_vert), quads (4, n_elem)
 * counter-clockwise corners.  Same edge numbering as the reference (edges in order of first
 * appearance over elements and sides 0..3), with 64-bit vertex-pair keys. */
int wdg_mesh_from_vertices(int n_vert, const double *xy, int n_elem, const int *quads, wdg_mesh **out);
/* dg::Mesh2D::uniform_rect (source/Mesh2D.cpp:130-163) */
int wdg_mesh_uniform_rect(int nx, double ax, double bx, int ny, double ay, double by, wdg_mesh **out);
/* dg::Mesh2D::from_file (source/Mesh2D.cpp:94-128): dir/info.txt "n_points n_elements",
 * dir/coordinates.txt one "x y" per point, dir/elements.txt four 0-based point indices per
 * element; then as wdg_mesh_from_vertices.  Missing or short files are errors. */
int wdg_mesh_from_file(const char *dir, wdg_mesh **out);
/* Adopt the tables of an existing dg::Mesh2D (what a C++ drop-in reads through the reference's
 * public API): corners (2, 4, n_elem) = QuadElement::corner(c) (wavedg/Element.hpp:123-126);
 * per edge (el0, s0, el1, s1, delta) = Edge::{elements, sides, delta} (wavedg/Edge.hpp:37-49),
 * in Mesh2D::edge(i, type) order; boundary rows ignore el1, s1, delta. */
int wdg_mesh_from_tables(int n_elem, const double *corners, int n_interior, const int *interior_edges,
                         int n_boundary, const int *boundary_edges, wdg_mesh **out);
void wdg_mesh_destroy(wdg_mesh *mesh);
int wdg_mesh_n_elem(const wdg_mesh *mesh);
int wdg_mesh_n_edges(const wdg_mesh *mesh, int face_type);               /* Mesh2D::n_edges(type) */
int wdg_mesh_edges(const wdg_mesh *mesh, int face_type, int *out);        /* (el0, s0, el1, s1, delta) rows */
int wdg_mesh_min_h(const wdg_mesh *mesh, double *h);                      /* Mesh2D::min_h (source/Mesh2D.cpp:751-767) */
int wdg_mesh_boundary_midpoints(const wdg_mesh *mesh, double *xy);         /* edge_metrics(1-pt rule, BOUNDARY).physical_coordinates() */

/* ------------------------------------------------------------------ snapshots */
/* dg::to_file (examples/examples.hpp:14-19): n doubles as raw native-order bytes; u on the
 * host or on the GPU.  wdg_read_raw reads such a file back (its size must be 8 n bytes). */
int wdg_write_raw(const char *fname, long long n, const double *u);
int wdg_read_raw(const char *fname, long long n, double *u);

/* QuadratureRule::gauss_lobatto (source/QuadratureRule.cpp:32-97) and
 * lagrange_basis_deriv at the nodes (source/lagrange_interpolation.cpp:33-50):
 * D (n, n), D[l + n*j] = phi_j'(x_l).  D may be NULL. */
int wdg_gauss_lobatto(int n, double *x, double *w, double *D);

/* ----------------------------------------------------- discretisation */
/* One GPU-resident discretisation of the wave system on `mesh` with n_colloc GLL nodes per
 * direction: WaveEquation(mesh, basis, approx_quad=true) (source/WaveEquation.cpp:5-30),
 * WaveBC(mesh, bc, basis, true) (:70-105) and MassMatrix<true>(mesh, basis)
 * (source/MassMatrix.cpp:6-28).  bc: one code per boundary edge (NULL = all 0).
 * device: CUDA ordinal (-1 = current device). */
int wdg_wave_create(const wdg_mesh *mesh, int n_colloc, const int *bc, int precision, int device, wdg_wave **out);
void wdg_wave_destroy(wdg_wave *wave);
int wdg_wave_info(const wdg_wave *wave, int *n_colloc, int *n_elem, long long *ndof, int *precision);
int wdg_wave_set_stream(wdg_wave *wave, void *cuda_stream);
int wdg_wave_sync(wdg_wave *wave);
/* elements per thread block of the fused kernels (a multiple of 4; 0 = built-in default) */
int wdg_wave_set_tile(wdg_wave *wave, int elems_per_block);
int wdg_wave_get_tile(const wdg_wave *wave, int *elems_per_block);
/* upper bound on the persistent CTAs of the fused kernels (0 = one full wave of resident CTAs);
 * lowering it makes each CTA walk more tiles (used by the tuner and the pipeline tests) */
int wdg_wave_set_max_ctas(wdg_wave *wave, int max_ctas);
/* depth of the bulk-copy pipeline of the fused kernels: 2, 3 or 4 tiles staged (0 = default);
 * the tile shrinks if needed to fit shared memory */
int wdg_wave_set_stages(wdg_wave *wave, int stages);
/* fused-kernel family: 0 warp per element (nodes on lanes; n^2 <= 32 keeps them in registers),
 * 1 tiled (element tiles staged in shared memory by a TMA bulk-copy pipeline), -1 default */
int wdg_wave_set_kernel(wdg_wave *wave, int family);
int wdg_wave_get_launch(const wdg_wave *wave, int *family, int *elems_per_block, int *stages, int *max_ctas);
/* the project's autotuner: times `steps` RK4 steps (dt = 0, state unchanged) for the warp
 * kernel and every (elements per block, pipeline depth) of the tiled kernel that fits, and
 * keeps the fastest for this handle */
int wdg_wave_autotune(wdg_wave *wave, int steps, float *best_ms_per_step);
/* Mesh2D::element_metrics(basis).physical_coordinates(): xy (2, n, n, n_elem) */
int wdg_wave_node_coords(wdg_wave *wave, double *xy);
/* Failure detection (no counterpart in the reference, which has no device-side waits): every
 * wait of the fused stage kernels on a copy completion gives up after `seconds` (default 2),
 * records it in the handle's device error word and lets the kernel finish; the next
 * synchronising call returns WDG_ERR_TIMEOUT and clears the word, and the handle stays usable. */
int wdg_wave_set_wait_limit(wdg_wave *wave, double seconds);
/* Test hooks (no counterpart in the reference) that exercise that failure detection without
 * faulting the GPU.  wdg_test_skip_chunk: in the first stage launch of the next RK4 call that
 * takes the warp-specialised kernel, every CTA leaves its chunk number `chunk` unloaded (-1:
 * none), so the waits on that chunk run out.  wdg_test_set_partner: overwrites the fused
 * kernels' partner offset of (elem, side) (returns the previous value in *previous); an offset
 * outside the state makes the kernels skip that trace and report WDG_ERR_ARG ("neighbour
 * index outside the mesh") instead of reading out of bounds. */
int wdg_test_skip_chunk(wdg_wave *wave, int chunk);
int wdg_test_set_partner(wdg_wave *wave, int elem, int side, int offset, int *previous);

/* ---- Operator::action drop-ins, FP64, accumulate (y += A x) ---- */
int wdg_div_action(wdg_wave *wave, const double *u, double *du);   /* Div<true>::action (source/Div.cpp:131-196) */
int wdg_wave_action(wdg_wave *wave, const double *u, double *du);  /* WaveEquation::action (source/WaveEquation.cpp:54-68) */
int wdg_wavebc_action(wdg_wave *wave, const double *u, double *du); /* WaveBC::action (source/WaveEquation.cpp:190-215) */
/* LobattoFaceProlongator::action, n_var = 3 (source/FaceProlongator.cpp:565-590, 628-648):
 * uf (n, 3, 2, n_edges(face_type)) is overwritten (boundary: side 1 zeroed). */
int wdg_face_prolong(wdg_wave *wave, int face_type, const double *u, double *uf);
/* LobattoFaceProlongator::t (source/FaceProlongator.cpp:650-714): u += P^T uf */
int wdg_face_prolong_t(wdg_wave *wave, int face_type, const double *uf, double *u);
/* EdgeFlux<true>::action with the upwind defaults a = -1, b = -1/2 (source/EdgeFlux.cpp:289-373):
 * fb side 0 <- flux, side 1 <- -flux; fb may equal ub. */
int wdg_edge_flux(wdg_wave *wave, int face_type, const double *ub, double *fb);
/* apply_bc_2d (source/WaveEquation.cpp:144-167): side 1 of boundary traces <- exterior state */
int wdg_apply_bc(wdg_wave *wave, double *uB);
/* MassMatrix<true>::action / ::inv (source/MassMatrix.cpp:55-82) */
int wdg_mass_action(wdg_wave *wave, int n_var, const double *x, double *y);
int wdg_mass_inv(wdg_wave *wave, int n_var, double *x);

/* ---- fused hot path ---- */
/* The examples' time derivative (examples/wave2d.cpp:164-177 without its forcing callback;
 * source/WaveHoltz.cpp:57-68): dudt = M^{-1} (A u + B u + s F).  F may be NULL.  One kernel. */
int wdg_rhs(wdg_wave *wave, const double *u, double *dudt, const double *F, double s);
/* nsteps of ode::RungeKutta4::step (wavedg/ode.hpp:66-93) on dudt = M^{-1}(A + B) u, in place;
 * t advances by dt per step.  One fused kernel per RK stage. */
int wdg_rk4_steps(wdg_wave *wave, double *u, double dt, double *t, int nsteps);

/* ---- linear advection, constant coefficients (the generic conservation-law path) ---- */
/* Advection<true>(n_var, mesh, basis, a, true) (wavedg/Advection.hpp:17-142),
 * AdvectionHomogeneousBC<true> (:144-273, u = 0 outside) and MassMatrix<true> for n_var <= 8
 * variables; a = (A_0, A_1) with a(d, c, k) = a[d + n_var (c + n_var k)], both symmetric.
 * Arrays u(d, i, j, el) with n_var fields; FP64. */
typedef struct wdg_advect wdg_advect;
int wdg_advect_create(const wdg_mesh *mesh, int n_colloc, int n_var, const double *a, int device, wdg_advect **out);
void wdg_advect_destroy(wdg_advect *adv);
int wdg_advect_action(wdg_advect *adv, const double *u, double *du);    /* Advection::action, du += */
int wdg_advect_bc_action(wdg_advect *adv, const double *u, double *du); /* AdvectionHomogeneousBC::action, du += */
/* dudt = M^{-1} (A u + B u) and nsteps of ode::RungeKutta4 on it */
int wdg_advect_rhs(wdg_advect *adv, const double *u, double *dudt);
int wdg_advect_rk4_steps(wdg_advect *adv, double *u, double dt, double *t, int nsteps);

/* ---- linear advection with a spatially varying coefficient ---- */
/* Advection<AQ> and AdvectionHomogeneousBC<AQ> with constant_coefficient = false
 * (wavedg/Advection.hpp:59-273) and MassMatrix<AQ> on a basis of basis_type (Gauss-Lobatto, or
 * Gauss-Legendre as examples/advec2d.cpp uses, with LegendreFaceProlongator's traces): a is the host array
 * a(k, l, comp, i, j, el) = a[k + n_var (l + n_var (comp + 2 (i + n (j + n el))))], A^comp_{k,l}
 * at node (i, j) of element el (the reference's layout); approx_quad selects Div<true> /
 * EdgeFlux<true> (1) or Div<false> / EdgeFlux<false> on their default Gauss-Legendre rules with
 * MassMatrix<false> (0, the setting of examples/advec2d.cpp).  The flux matrices come from an
 * eigen-decomposition of n.A at every face point: n_var = 1, or n.A symmetric (n_var <= 8;
 * WDG_ERR_UNSUPPORTED otherwise).  FP64. */
typedef struct wdg_vadvect wdg_vadvect;
#define WDG_GAUSS_LEGENDRE 0 /* QuadratureRule::GaussLegendre (wavedg/QuadratureRule.hpp:26-30) */
#define WDG_GAUSS_LOBATTO 1  /* QuadratureRule::GaussLobatto */
int wdg_vadvect_create(const wdg_mesh *mesh, int n_colloc, int basis_type, int n_var, const double *a,
                       int approx_quad, int device, wdg_vadvect **out);
void wdg_vadvect_destroy(wdg_vadvect *adv);
int wdg_vadvect_set_stream(wdg_vadvect *adv, void *cuda_stream);
int wdg_vadvect_sync(wdg_vadvect *adv);
int wdg_vadvect_action(wdg_vadvect *adv, const double *u, double *du);    /* Advection::action, du += */
int wdg_vadvect_bc_action(wdg_vadvect *adv, const double *u, double *du); /* AdvectionHomogeneousBC::action, du += */
/* dudt = M^{-1} (Advection + AdvectionHomogeneousBC) u, and nsteps of ode::RungeKutta4 (method 0)
 * or ode::SSPRK3 (method 1, the stepper of examples/advec2d.cpp) on u in place */
int wdg_vadvect_rhs(wdg_vadvect *adv, const double *u, double *dudt);
int wdg_vadvect_steps(wdg_vadvect *adv, int method, double *u, double dt, double *t, int nsteps);

/* ---- set-up operators on either basis type ---- */
/* MassMatrix<AQ> (source/MassMatrix.cpp:6-227; approx_quad 1: diag(w_i w_j det J), 0: the exact
 * element matrices on the (n + 1)-point rule) and LinearFunctional2D (wavedg/LinearFunctional.hpp:
 * 61-202, its default n-point Gauss-Legendre rule) on a basis of basis_type, FP64: what
 * examples/advec2d.cpp uses to project its coefficient, c = M^{-1} (f, phi), on a
 * Gauss-Legendre basis. */
typedef struct wdg_massmatrix wdg_massmatrix;
int wdg_massmatrix_create(const wdg_mesh *mesh, int n_colloc, int basis_type, int approx_quad, int device,
                          wdg_massmatrix **out);
void wdg_massmatrix_destroy(wdg_massmatrix *m);
int wdg_massmatrix_set_stream(wdg_massmatrix *m, void *cuda_stream);
int wdg_massmatrix_action(wdg_massmatrix *m, int n_var, const double *x, double *y); /* y = M x (y may be x) */
int wdg_massmatrix_inv(wdg_massmatrix *m, int n_var, double *x);                     /* x = M^{-1} x */
/* the points the load vector samples f at: (x, y) of point k + n (l + n el), host array (2, n, n, nel) */
int wdg_massmatrix_points(const wdg_massmatrix *m, double *xy);
/* F(d, i, j, el) = (f_d, phi_ij) from fq(d, point), f at those points (host); F host or device */
int wdg_massmatrix_load(wdg_massmatrix *m, int n_var, const double *fq, double *F);

/* ---- nonlinear conservation law: the compressible Euler system of examples/cl2d.cpp ---- */
/* State u(d, i, j, el), d = density, x-momentum, y-momentum, energy; gamma = 1.4; FP64.
 * The operators of the example with approx_quad = true on GLL nodes: DivF2D<true>
 * (wavedg/DivF.hpp:74-260) with its physical flux F(u) (cl2d.cpp:67-90), EdgeFluxF2D<true>
 * (wavedg/EdgeFluxF.hpp:65-180) with its local Lax-Friedrichs numerical flux
 * 1/2 n.(F(uL) + F(uR)) + 1/2 max(|v| + c) (uL - uR) (cl2d.cpp:92-120), MassMatrix<true>. */
typedef struct wdg_claw wdg_claw;
int wdg_euler_create(const wdg_mesh *mesh, int n_colloc, int device, wdg_claw **out);
/* The same system with approx_quad = false, as examples/cl2d.cpp ships: DivF2D<false>
 * (wavedg/DivF.hpp:262-394) and EdgeFluxF2D<false> (wavedg/EdgeFluxF.hpp:182-254) on their
 * default 2n-point Gauss-Legendre rules (source/DivF.cpp:59, source/EdgeFluxF.cpp:55), the
 * face traces interpolated to the face rule, and MassMatrix<false>'s dense inverse.  The
 * entry points below serve both kinds of handle. */
int wdg_euler_create_exact(const wdg_mesh *mesh, int n_colloc, int device, wdg_claw **out);
void wdg_claw_destroy(wdg_claw *claw);
int wdg_claw_set_stream(wdg_claw *claw, void *cuda_stream);
int wdg_claw_sync(wdg_claw *claw);
/* DivF2D::action: divF += (F(u), grad v) */
int wdg_claw_div(wdg_claw *claw, const double *u, double *divF);
/* EdgeFluxF2D::action on nodal face traces uB (n, 4, 2, n_edges(face_type)): fB(side 0) =
 * sum_i P(i, k) w_i |E|/2 fh(n, side 0, side 1) (P the identity with approx_quad = true),
 * fB(side 1) = -fB(side 0), n the outward normal of the edge's first element; fB may be uB */
int wdg_claw_flux(wdg_claw *claw, int face_type, const double *uB, double *fB);
/* the time derivative of examples/cl2d.cpp:171-220: dudt = M^{-1} (DivF(u) - interior faces -
 * boundary faces with exterior state = interior state), one fused launch */
int wdg_claw_rhs(wdg_claw *claw, const double *u, double *dudt);
/* nsteps of ode::RungeKutta4 (method 0, wavedg/ode.hpp:66-93) or ode::SSPRK3 (method 1,
 * wavedg/ode.hpp:145-186, the stepper of cl2d.cpp) on u in place, one fused launch per stage */
int wdg_claw_steps(wdg_claw *claw, int method, double *u, double dt, double *t, int nsteps);

/* ---- domain decomposition (one rank's share of a mesh) ---- */
/* The fused kernels' partner table of `mesh` (what Mesh2D::distribute and FaceVector need to
 * know, source/Mesh2D.cpp:384-592): per element side the DOF offset of the neighbour node that
 * faces face node 0 (fbase, 4 per element, -1 on the boundary) and per element four bytes
 * (stride code in bits 0-1: +3, -3, +3n, -3n per face node; boundary code bits 3-4; boundary bit 7).
 * Host only. */
int wdg_mesh_partner_table(const wdg_mesh *mesh, int n_colloc, const int *bc, int *fbase, unsigned *fcode);
/* A discretisation of the local elements of a decomposed mesh: `mesh` holds this rank's
 * elements, so the sides it shares with other ranks are boundary sides of `mesh`; the n_halo
 * sides (halo_elem[j], halo_side[j]) read their neighbour trace from halo slot j instead,
 * n x 3 values (face-node order of this side) stored after the elements in every state
 * buffer.  For RK stepping (wdg_rk4_stage) and the resident-state calls only. */
int wdg_wave_create_halo(const wdg_mesh *mesh, int n_colloc, const int *bc, int precision, int device, int n_halo,
                         const int *halo_elem, const int *halo_side, wdg_wave **out);
int wdg_halo_info(const wdg_wave *wave, long long *elements_values, long long *halo_values);
/* out[3 j + f] = state buffer `buffer` (0 resident, 1, 2 the RK rotation) at idx[j] + f, f < 3:
 * the traces another rank's halo needs (idx, out: device arrays; the handle's precision) */
int wdg_halo_gather(wdg_wave *wave, int buffer, const int *idx, int count, void *out);
/* halo values [offset, offset + count) of state buffer `buffer` <- src (device or host) */
int wdg_halo_put(wdg_wave *wave, int buffer, long long offset, const void *src, long long count);
/* RK4 stage `stage` (0..4) of ode::RungeKutta4::step on the resident state: reads buffer
 * 0, 1, 2, 1, 2 and writes 1, 2, 1, 2, 0; the stage's input halo must be filled first */
int wdg_rk4_stage(wdg_wave *wave, int stage, double dt);
/* wdg_rk4_stage of the step that starts at time t, with the terms WaveHoltz adds
 * (source/WaveHoltz.cpp:55-121): F (device, the handle's precision, NULL for none) enters the
 * RHS as F * (-sin(omega (t + c_stage dt)) / omega); at stage 4, acc (device FP64, NULL for
 * none) accumulates acc_c * (the new state), the period filter's term of this step. */
int wdg_rk4_stage_forced(wdg_wave *wave, int stage, double dt, double t, const void *F, double omega, double *acc,
                         double acc_c);
/* wdg_rk4_stage_forced over elements [el_begin, el_end) only (el_begin a multiple of 4): a
 * stage split into the elements that read no halo trace and the rest lets the halo exchange
 * run beside the first part (needs the warp-specialised kernel; WDG_ERR_UNSUPPORTED otherwise) */
int wdg_rk4_stage_elems(wdg_wave *wave, int stage, double dt, double t, const void *F, double omega, double *acc,
                        double acc_c, int el_begin, int el_end);
/* Mesh2D::distribute's element -> rank maps, computed on the host without MPI
 * (source/Mesh2D.cpp:233-382): method 0 recursive coordinate bisection (rcb), 1 reverse
 * Cuthill-McKee blocks (rcm).  e2p: n_elem ranks in [0, n_parts).  The rcb principal axis takes
 * the mean of y from y and cuts a part with zero covariance across its axis of larger
 * variance (the reference averages x for both means and divides by the covariance). */
int wdg_mesh_partition(const wdg_mesh *mesh, int n_parts, int method, int *e2p);

/* ---- exact quadrature (approx_quad = false), FP64 ---- */
/* WaveEquation(mesh, basis, false) (source/WaveEquation.cpp:5-30: Div<false>, EdgeFlux<false>),
 * WaveBC(mesh, bc, basis, false) (:70-105) and MassMatrix<false>(mesh, basis)
 * (source/MassMatrix.cpp:84-230), with the reference's default Gauss-Legendre rules for
 * bilinear elements: Div 1 + ((n-2) + (n-1) + 1)/2 points per direction, EdgeFlux and
 * MassMatrix 1 + (2(n-1) + 2)/2.  Arrays and semantics as the collocation entry points. */
typedef struct wdg_waveq wdg_waveq;
int wdg_waveq_create(const wdg_mesh *mesh, int n_colloc, const int *bc, int device, wdg_waveq **out);
void wdg_waveq_destroy(wdg_waveq *wave);
int wdg_waveq_rules(const wdg_waveq *wave, int *n_div, int *n_face, int *n_mass);
/* the collocation handle it shares geometry, prolongation and staging with (owned by `wave`) */
int wdg_waveq_wave(const wdg_waveq *wave, wdg_wave **collocation);
int wdg_waveq_div_action(wdg_waveq *wave, const double *u, double *du);    /* Div<false>::action (Div.cpp:469-588, 658-673), du += */
int wdg_waveq_wave_action(wdg_waveq *wave, const double *u, double *du);   /* WaveEquation::action, du += */
int wdg_waveq_wavebc_action(wdg_waveq *wave, const double *u, double *du); /* WaveBC::action, du += */
/* EdgeFlux<false>::action (EdgeFlux.cpp:548-640): fb side 0 <- flux, side 1 <- -flux; fb may equal ub */
int wdg_waveq_edge_flux(wdg_waveq *wave, int face_type, const double *ub, double *fb);
/* MassMatrix<false>::action (y = L L^T x) / ::inv (x <- L^-T L^-1 x) (MassMatrix.cpp:194-230) */
int wdg_waveq_mass_action(wdg_waveq *wave, int n_var, const double *x, double *y);
int wdg_waveq_mass_inv(wdg_waveq *wave, int n_var, double *x);
/* dudt = M^{-1} (A u + B u + s F), F may be NULL; and nsteps of ode::RungeKutta4 on it */
int wdg_waveq_rhs(wdg_waveq *wave, const double *u, double *dudt, const double *F, double s);
int wdg_waveq_rk4_steps(wdg_waveq *wave, double *u, double dt, double *t, int nsteps);

/* ---- resident state (stays on the GPU in the handle's precision) ---- */
int wdg_state_upload(wdg_wave *wave, const double *u);
int wdg_state_download(wdg_wave *wave, double *u);
/* device pointer of the resident state (double* for WDG_FP64, float* for WDG_FP32) */
int wdg_state_device_ptr(wdg_wave *wave, void **ptr);
/* like wdg_rk4_steps on the resident state; asynchronous */
int wdg_state_rk4_steps(wdg_wave *wave, double dt, double *t, int nsteps);
/* discrete energy 1/2 sum_i m_i |q_i|^2 of the resident state, accumulated in FP64 */
int wdg_state_energy(wdg_wave *wave, double *energy);

/* ---- LinearFunctional2D (wavedg/LinearFunctional.hpp:61-74, 136-202) ---- */
/* physical coordinates of the n-point Gauss-Legendre quadrature points: xy (2, n, n, n_elem) */
int wdg_quad_points(wdg_wave *wave, double *xy);
/* F = (f, phi) from f sampled at those points: fq (n_var, n, n, n_elem) -> F (n_var, n, n, n_elem) */
int wdg_linear_functional(wdg_wave *wave, int n_var, const double *fq, double *F);
/* (f, phi) for f = scale * sum_k amp_k exp(-|x - c_k|^2 / (2 sigma_k^2)) in component comp
 * (others 0), evaluated on the GPU; mass_inv != 0 returns M^{-1} (f, phi). */
int wdg_load_gaussians(wdg_wave *wave, int n_src, const double *cx, const double *cy, const double *sigma,
                       const double *amp, double scale, int comp, int mass_inv, double *F);

/* wdg_load_gaussians for callers that cannot allocate device memory (no counterpart in the
 * reference).  wdg_load_gaussians grows a device buffer for its source table on first use; some
 * callers cannot let a library do that once they run: loops whose memory is fixed before they start
 * (a cudaMalloc there could fail, and it synchronises the device, stalling a real-time loop), and
 * hosts whose own allocator has reserved the GPU's memory.  This entry point gives the same load
 * vector but stages the table in a fixed 32 KiB array that belongs to the library image (held on
 * every GPU that loads the library until the process exits).  Nothing is allocated: at most 1024
 * sources per call (more return WDG_ERR_ARG), and F must be device memory.
 * The first call on a device looks up the array's device address (once per device, cached for the
 * life of the process); make that first call before any stream capture.  The cached address dies
 * with the device's context: after cudaDeviceReset this entry point must not be called again in
 * the process.  All calls share the one table and it keeps the last call's sources, so calls that
 * overlap on the GPU (different streams or threads) race.  Asynchronous on the handle's stream:
 * cx..amp in pageable host memory are copied before the call returns; in pinned host or device
 * memory they are read when the stream reaches the copy and must stay valid and unchanged until
 * then. */
int wdg_load_gaussians_noalloc(wdg_wave *wave, int n_src, const double *cx, const double *cy,
                               const double *sigma, const double *amp, double scale, int comp, int mass_inv,
                               double *F);

/* ---- norms (source/linalg.cpp:102-131), FP64 on the GPU ---- */
int wdg_norm(wdg_wave *wave, const double *x, double *result);
int wdg_error(wdg_wave *wave, const double *x, const double *y, double *result);

/* ------------------------------------------------------------ WaveHoltz */
/* dg::WaveHoltz(omega, mesh, basis, bc, approx_quad=true) (source/WaveHoltz.cpp:5-30) on a
 * discretisation: T = 2 pi / omega, dt = 0.5 min_h / n^2, nt = ceil(T / dt), dt = T / nt. */
int wdg_waveholtz_create(wdg_wave *wave, double omega, wdg_waveholtz **out);
/* WaveHoltz(omega, mesh, basis, bc, approx_quad = false): the same iteration over the exact-
 * quadrature operators of `exact` (which must outlive the handle); every wdg_waveholtz_* call
 * below works on it, FP64. */
int wdg_waveholtz_create_exact(wdg_waveq *exact, double omega, wdg_waveholtz **out);
void wdg_waveholtz_destroy(wdg_waveholtz *wh);
int wdg_waveholtz_params(const wdg_waveholtz *wh, double *T, double *dt, int *nt);
/* WaveHoltz::pi0 (source/WaveHoltz.cpp:55-89): w = Pi(0) for load vector F */
int wdg_waveholtz_pi0(wdg_waveholtz *wh, double *w, const double *F);
/* WaveHoltz::S (source/WaveHoltz.cpp:91-121), in place */
int wdg_waveholtz_S(wdg_waveholtz *wh, double *w);
/* WaveHoltz::postprocess (source/WaveHoltz.cpp:123-145): H (2, n_points) */
int wdg_waveholtz_postprocess(wdg_waveholtz *wh, double *H, const double *w);
/* The fixed-point loop of examples/waveholtz2d.cpp:137-185: pi0 = Pi(0)(F); from the initial
 * guess in W iterate W <- S W + pi0 until ||W - W_prev|| / ||pi0|| < tol or maxit.
 * Returns WDG_OK or WDG_ERR_NOT_CONVERGED; *iters and *residual are always written. */
int wdg_waveholtz_solve(wdg_waveholtz *wh, const double *F, double tol, int maxit, double *W, int *iters,
                        double *residual);

/* ------------------------------------------------------ batched WaveHoltz */
/* Up to 64 independent WaveHoltz solves, each on its own discretisation (mesh, degree) with
 * its own omega, advanced together: per RK stage one persistent kernel launch per degree
 * over a work list of (solve, chunk of elements), the degrees' launches concurrent, blocks
 * of steps replayed as a CUDA graph.  Per solve,
 * T, dt and nt follow WaveHoltz::WaveHoltz (source/WaveHoltz.cpp:24-29), and the iteration is
 * the fixed-point loop of examples/waveholtz2d.cpp:165-185 with its residual
 * ||W - W_prev|| / ||pi0|| (each iteration runs one forced period from W, which equals
 * S W + pi0).  All discretisations must share device and precision (WDG_FP32 steps in FP32
 * with the filter, iterate and residual in FP64); a discretisation may appear once per batch
 * and must not be stepped elsewhere while the batch solves. */
typedef struct wdg_whbatch wdg_whbatch;
int wdg_whbatch_create(int n_solves, wdg_wave *const *waves, const double *omegas, wdg_whbatch **out);
void wdg_whbatch_destroy(wdg_whbatch *batch);
int wdg_whbatch_params(const wdg_whbatch *batch, int solve, double *T, double *dt, int *nt);
/* chunk = rounds x (4 warps x floor(32 / n) elements) per solve; ring = chunk slots (2..6) */
int wdg_whbatch_set_launch(wdg_whbatch *batch, int rounds, int ring);
/* grid: CTAs of one launch of an RK stage without the filter, summed over the degree groups */
int wdg_whbatch_get_launch(const wdg_whbatch *batch, int *rounds, int *ring, int *grid);
/* times `steps` batch steps of every launch shape that fits and keeps the fastest */
int wdg_whbatch_autotune(wdg_whbatch *batch, int steps, float *best_ms_per_step);
/* F[s], W[s]: FP64 arrays (host or device) of solve s.  warm (nullable): warm[s] != 0 starts
 * solve s from W[s] (one extra period from zero then gives |pi0|), else from zero.
 * pi0_norm (nullable, in/out): a warm-started solve with pi0_norm[s] > 0 takes that value as
 * |pi0| and skips the extra period (e.g. the norm an FP32 batch of the same problems measured);
 * on return pi0_norm[s] holds the |pi0| that scaled solve s's residual.  A solve stops at
 * residual < tol (status 0), after maxit iterations (1), or when stall_limit > 0 updates in a
 * row bring no new smallest residual (2: the stepping precision's floor).
 * W[s] receives the last iterate; iters, residuals, status (nullable) get one entry per solve.
 * Runs after the work already queued on the solves' streams (device inputs written there are
 * complete before they are read) and returns when the results are written. */
int wdg_whbatch_solve(wdg_whbatch *batch, const double *const *F, double tol, int maxit, int stall_limit,
                      double *const *W, const int *warm, double *pi0_norm, int *iters, double *residuals,
                      int *status);

#ifdef __cplusplus
}
#endif

#endif /* WDG_B200_H */
