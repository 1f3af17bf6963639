/*
 * edge_b200.h — C ABI of libedgeb200.so, the sm_100a implementation of the
 * EDGE flow-map solver's per-step hot path.
 *
 * The reference (pfm-gatech/EDGE-Flow-Maps) is Python + Taichi; its "FFI" for
 * this path is the set of Taichi kernels and solver methods the run_*.py
 * drivers call.  Each entry point below names the reference function (file
 * and lines inside that project) that it replaces; the Python modules under
 * edge-flow-maps_b200/sim keep the reference's names and arguments and call
 * these through ctypes.
 *
 * Conventions
 *  - All pointers are device pointers (cudaMalloc'd or torch-owned); the
 *    library never frees caller memory.  Solver workspaces live in an opaque
 *    handle (edge_mgpcg_create / edge_mgpcg_destroy).
 *  - Fields are float32, row-major (i, j, k) with k fastest.  vec3 / vec4
 *    fields store their components last (the order of Taichi's to_numpy()).
 *    vec4 dye fields must be 16-byte aligned.
 *  - Face grids of an (nx, ny, nz) cell grid: u_x (nx+1, ny, nz),
 *    u_y (nx, ny+1, nz), u_z (nx, ny, nz+1).
 *  - `stream` is a cudaStream_t (0 = legacy default stream).  Calls are
 *    asynchronous unless stated otherwise.
 *  - Return value: 0 on success, a positive cudaError_t on a CUDA error, or a
 *    negative EDGE_E* code.  No call aborts the process.
 */
#ifndef EDGE_B200_H
#define EDGE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define EDGE_OK 0
#define EDGE_EINVAL (-1)     /* bad sizes, null pointer, unsupported option */
#define EDGE_EALIGN (-2)     /* misaligned pointer (vec4 fields need 16 B) */
#define EDGE_ENOCONV (-3)    /* solver stopped at max_iters without converging */
#define EDGE_ENAN (-4)       /* non-finite residual */
#define EDGE_ESTALL (-5)     /* residual stalled (flexible PCG fallback taken) */
#define EDGE_ESTATE (-6)     /* call order / handle state error */

/* Hermite variants (sim/hermite.py) */
#define EDGE_HERMITE_FD 0    /* interp_(grad_)hermite_fd_unroll, hermite.py:65-295 (ED4) */
#define EDGE_HERMITE_GARM 1  /* interp_(grad_)hermite_garm_fd_unroll, hermite.py:299-456 (EDGE) */
#define EDGE_HERMITE_FULL 2  /* interp_(grad_)hermite, hermite.py:460-607 (ED8) */

/* ---- library ---------------------------------------------------------- */
int edge_version(void);
const char *edge_error_string(int code);

/* ---- point samplers (util/taichi_utils.py, sim/hermite.py) ------------- */
/* interp_u_MAC / interp_u_MAC_grad, taichi_utils.py:322-341, at n points
 * pts (n x 3): v (n x 3), vg (n x 3, value of the grad variant), g (n x 3 x 3,
 * rows = grad u_x, grad u_y, grad u_z). */
int edge_points_mac(int nx, int ny, int nz, float dx, const float *ux, const float *uy, const float *uz,
                    const float *pts, int n, float *v, float *vg, float *g, void *stream);
/* interp_1 and sample_min_max_1 on a 4-channel cell field,
 * taichi_utils.py:172-227 */
int edge_points_dye(int nx, int ny, int nz, float dx, const float *smoke, const float *pts, int n, float *lin,
                    float *mn, float *mx, void *stream);
/* the Hermite interpolants of all three components of psi at n points:
 * val (value-only function), gval/grad (grad function), hermite.py:65-607.
 * dT may be NULL for EDGE_HERMITE_FD; d2T is only read by EDGE_HERMITE_FULL. */
int edge_points_hermite(int variant, int nx, int ny, int nz, float dx, const float *psi, const float *Tx,
                        const float *Ty, const float *Tz, const float *dTx, const float *dTy, const float *dTz,
                        const float *d2Tx, const float *d2Ty, const float *d2Tz, const float *pts, int n,
                        float *val, float *gval, float *grad, void *stream);

/* ---- map state -------------------------------------------------------- */
/* reset_to_identity_1/2/3, hermite.py:642-700: psi = X, T = I, dT = 0,
 * d2T = 0 (the dT and d2T pointers may be NULL). */
int edge_reset_cells(int nx, int ny, int nz, float dx, float *psi, float *Tx, float *Ty, float *Tz, float *dTx,
                     float *dTy, float *dTz, float *d2Tx, float *d2Ty, float *d2Tz, void *stream);
/* reset_to_identity, run_edge.py:306-320: phi_a = X_a, F_a = e_a on the faces */
int edge_reset_faces(int nx, int ny, int nz, float dx, float *phix, float *phiy, float *phiz, float *Fx,
                     float *Fy, float *Fz, void *stream);

/* ---- flow-map marches -------------------------------------------------- */
/* advect_psi_garm_ed4_fusion_unroll, hermite.py:1426-1521 (EDGE): one RK4
 * step (-dt) of the cell centre and 4 epsilon points with Jacobians, composed
 * with the accumulated map (psi, T, dT); results to the o* buffers, which
 * must not alias the inputs.  If `identity` is non-zero the accumulated map
 * is taken to be the identity (the step right after a reinitialisation) and
 * psi/T/dT are not read. */
int edge_march_edge(int nx, int ny, int nz, float dx, float dt, float epsilon, const float *ux, const float *uy,
                    const float *uz, const float *psi, const float *Tx, const float *Ty, const float *Tz,
                    const float *dTx, const float *dTy, const float *dTz, float *opsi, float *oTx, float *oTy,
                    float *oTz, float *odTx, float *odTy, float *odTz, int identity, void *stream);
/* advect_ps_hermite_ed4_fd_unroll, hermite.py:1375-1395 (ED4) */
int edge_march_ed4(int nx, int ny, int nz, float dx, float dt, float epsilon, const float *ux, const float *uy,
                   const float *uz, const float *psi, const float *Tx, const float *Ty, const float *Tz, float *opsi,
                   float *oTx, float *oTy, float *oTz, void *stream);
/* advect_ps_hermite_ed8, hermite.py:1290-1338 (ED8) */
int edge_march_ed8(int nx, int ny, int nz, float dx, float dt, float epsilon, const float *ux, const float *uy,
                   const float *uz, const float *psi, const float *Tx, const float *Ty, const float *Tz,
                   const float *dTx, const float *dTy, const float *dTz, const float *d2Tx, const float *d2Ty,
                   const float *d2Tz, float *opsi, float *oTx, float *oTy, float *oTz, float *odTx, float *odTy,
                   float *odTz, float *od2Tx, float *od2Ty, float *od2Tz, void *stream);
/* advect_ps_garm, hermite.py:1398-1424 (GE, run_ge.py:220-230): each cell
 * centre marched back by RK4 with its Jacobian from the identity, composed
 * with the accumulated map (psi, T, dT, d2T) by the full stored-derivative
 * Hermite; dT and d2T of the new map by edge_calc_fd_3_from_grad.  Outputs
 * must not alias the inputs. */
int edge_march_ge(int nx, int ny, int nz, float dx, float dt, const float *ux, const float *uy, const float *uz,
                  const float *psi, const float *Tx, const float *Ty, const float *Tz, const float *dTx,
                  const float *dTy, const float *dTz, const float *d2Tx, const float *d2Ty, const float *d2Tz,
                  float *opsi, float *oTx, float *oTy, float *oTz, float *odTx, float *odTy, float *odTz,
                  float *od2Tx, float *od2Ty, float *od2Tz, void *stream);
/* calc_fd_3_from_grad, hermite.py:1180-1256: dT_c = (psi_c,yz, psi_c,xz,
 * psi_c,xy) from central differences of the gradient rows T_c and d2T_c =
 * psi_c,xyz from central differences of dT_c, neighbour indices clamped to
 * the grid.  dT must not alias T. */
int edge_calc_fd_3_from_grad(int nx, int ny, int nz, float dx, const float *Tx, const float *Ty, const float *Tz,
                             float *dTx, float *dTy, float *dTz, float *d2Tx, float *d2Ty, float *d2Tz,
                             void *stream);
/* Hermite psi and Jacobian column a at every face of grid a:
 *  - EDGE_HERMITE_FULL: split_psi_hermite, run_ed8.py:191-224
 *  - EDGE_HERMITE_GARM / _FD: the face evaluations shared by map_u_psi
 *    (run_edge.py:377-417, run_ed4.py:219-260) and split_to_mac
 *    (run_edge.py:430-440, run_ed4.py:279-289).
 * fpsi* / fcol* are vec3 face fields. */
int edge_face_map(int variant, int nx, int ny, int nz, float dx, const float *psi, const float *Tx, const float *Ty,
                  const float *Tz, const float *dTx, const float *dTy, const float *dTz, const float *d2Tx,
                  const float *d2Ty, const float *d2Tz, float *fpsix, float *fpsiy, float *fpsiz, float *fcolx,
                  float *fcoly, float *fcolz, void *stream);
/* The backward map in the packed layout the device driver keeps: 8 float4
 * planes of n = nx*ny*nz cells (plane q at packed + 4*q*n floats) for every
 * variant (edge_packed_planes): 0 psi, 1-3 the columns d psi/dx, d psi/dy,
 * d psi/dz, 4-6 the mixed derivatives (psi_yz, psi_xz, psi_xy) per
 * component, 7 psi_xyz.  ED8 keeps all eight as state; EDGE keeps 0-6 and
 * plane 7 holds the finite-difference triple-derivative coefficient the
 * reference re-derives from planes 4-6 at every Hermite evaluation; ED4 keeps
 * 0-3 and planes 4-7 hold the finite-difference coefficients derived from
 * planes 1-3.  pack and the marches fill the derived planes.  pack/unpack
 * convert from/to the reference layout (psi, T_c rows, dT_c, d2T_c as above;
 * no reference counterpart). */
int edge_packed_planes(int variant);
int edge_map_pack(int variant, int nx, int ny, int nz, const float *psi, const float *Tx, const float *Ty,
                  const float *Tz, const float *dTx, const float *dTy, const float *dTz, const float *d2Tx,
                  const float *d2Ty, const float *d2Tz, float *packed, void *stream);
int edge_map_unpack(int variant, int nx, int ny, int nz, const float *packed, float *psi, float *Tx, float *Ty,
                    float *Tz, float *dTx, float *dTy, float *dTz, float *d2Tx, float *d2Ty, float *d2Tz,
                    void *stream);
/* The EDGE / ED4 / ED8 marches (hermite.py:1426-1521, 1375-1395, 1290-1338)
 * on packed maps: in_packed is the accumulated map, out_packed receives the
 * new one (must not alias).  flags (EDGE only):
 *   EDGE_MARCH_IDENTITY     compose with the identity map, in_packed is not
 *                           read (the step right after a reinitialisation);
 *   EDGE_MARCH_F64_COMPOSE  accumulate each entry of the composed Jacobian
 *                           T_old(psi_step) T_step (hermite.py:960-980, float32
 *                           in the reference) in float64, rounded once. */
#define EDGE_MARCH_IDENTITY 1
#define EDGE_MARCH_F64_COMPOSE 2
int edge_march_packed(int variant, int nx, int ny, int nz, float dx, float dt, float epsilon, const float *ux,
                      const float *uy, const float *uz, const float *in_packed, float *out_packed, int flags,
                      void *stream);
/* edge_march_ge on packed maps (the ED8 planes 0-7); out_packed must not
 * alias in_packed. */
int edge_march_ge_packed(int nx, int ny, int nz, float dx, float dt, const float *ux, const float *uy,
                         const float *uz, const float *in_packed, float *out_packed, void *stream);
/* edge_face_map on a packed map */
int edge_face_map_packed(int variant, int nx, int ny, int nz, float dx, const float *packed, float *fpsix,
                         float *fpsiy, float *fpsiz, float *fcolx, float *fcoly, float *fcolz, void *stream);
/* forward map on the faces, advance_map x3, run_edge.py:330-357 (in place) */
int edge_advance_map(int nx, int ny, int nz, float dx, float dt, const float *ux, const float *uy, const float *uz,
                     float *phix, float *phiy, float *phiz, float *Fx, float *Fy, float *Fz, void *stream);
/* EFM backward map on the faces, backtrack_psi_grid(curr_step),
 * run_efm.py:179-186 (with reset_to_identity 153-167, march_no_neural 170-176,
 * advance_map 194-215): from the identity, advance_map with -dts[s] through
 * the cached velocities s = curr_step, ..., 0, all in one launch.
 * u?_cache and dts are HOST arrays of curr_step + 1 entries (device field
 * pointers and float step sizes); slot curr_step is the current velocity, as
 * the reference copies it there first.  curr_step < 64. */
int edge_efm_backtrack(int nx, int ny, int nz, float dx, int curr_step, const float *const *ux_cache,
                       const float *const *uy_cache, const float *const *uz_cache, const float *dts, float *psix,
                       float *psiy, float *psiz, float *Tx, float *Ty, float *Tz, void *stream);

/* ---- velocity / dye transport ------------------------------------------ */
/* advect_u_semi_lagrangian, hermite.py:1578-1621 (dt as passed; the driver
 * passes 0.5*dt).  u1 must not alias u0. */
int edge_advect_u_sl(int nx, int ny, int nz, float dx, float dt, const float *ux0, const float *uy0,
                     const float *uz0, float *ux1, float *uy1, float *uz1, void *stream);
/* Pull a face velocity back through face maps (position pos_a, Jacobian
 * column col_a): out_a = col_a . u0(pos_a).  This is map_u
 * (run_edge.py:361-373, pos = phi, col = F) and, with the face_map outputs,
 * map_u_psi (run_edge.py:377-417).  Fused BFECC options (NULL = off):
 *   init_*: out = scale * (out - init)         (run_edge.py:675-682)
 *   sub_*:  out = sub - out                      (run_edge.py:685-687) */
int edge_pullback_u(int nx, int ny, int nz, float dx, const float *ux0, const float *uy0, const float *uz0,
                    const float *posx, const float *posy, const float *posz, const float *colx, const float *coly,
                    const float *colz, const float *initx, const float *inity, const float *initz, float scale,
                    const float *subx, const float *suby, const float *subz, float *ux1, float *uy1, float *uz1,
                    void *stream);
/* map_u_psi computed directly from the cell map (no face buffers),
 * run_edge.py:377-417 (EDGE_HERMITE_GARM) / run_ed4.py:219-260 (_FD) */
int edge_map_u_psi(int variant, int nx, int ny, int nz, float dx, const float *ux0, const float *uy0,
                   const float *uz0, float *ux1, float *uy1, float *uz1, const float *psi, const float *Tx,
                   const float *Ty, const float *Tz, const float *dTx, const float *dTy, const float *dTz,
                   void *stream);
/* Dye pullback through a face map pos_a (cell centre = mean of its six face
 * positions): out = interp_1(smoke0, centre).  This is map_smoke
 * (run_edge.py:421-427, pos = phi) and, with face_map outputs, map_smoke_psi
 * (run_edge.py:444-466).  Fused options (NULL = off), applied in order:
 *   init:     out = scale * (out - init)        (run_edge.py:678-682)
 *   sub:      out = sub - out                   (run_edge.py:688)
 *   clampsrc: out = clamp(out, min/max of clampsrc's 8 corners at the centre)
 *             (clamp_smoke(_psi), run_edge.py:470-505)
 * If `inplace_clamp` is non-zero the kernel instead clamps out's own value
 * (clamp_smoke semantics: smoke1 = clamp(smoke1, ...)). */
int edge_pullback_dye(int nx, int ny, int nz, float dx, const float *smoke0, const float *posx, const float *posy,
                      const float *posz, const float *init, float scale, const float *sub, const float *clampsrc,
                      int inplace_clamp, float *out, void *stream);
/* map_smoke_psi / clamp_smoke_psi computed directly from the cell map,
 * run_edge.py:444-505, run_ed4.py:293-336.  mode 0: out = map; mode 1:
 * out = clamp(out, minmax(smoke0)). */
int edge_smoke_psi(int variant, int mode, int nx, int ny, int nz, float dx, const float *smoke0, float *out,
                   const float *psi, const float *Tx, const float *Ty, const float *Tz, const float *dTx,
                   const float *dTy, const float *dTz, void *stream);
/* clamp_u on all three face grids, run_edge.py:509-519:
 * u2 = clamp(u, min/max of u1's six neighbours) */
int edge_clamp_u(int nx, int ny, int nz, const float *ux, const float *uy, const float *uz, const float *u1x,
                 const float *u1y, const float *u1z, float *u2x, float *u2y, float *u2z, void *stream);
/* calc_max_speed, run_edge.py:296-303: max |u_centre| (>= 1e-3) into
 * out_max (one float, device memory) */
int edge_max_speed(int nx, int ny, int nz, const float *ux, const float *uy, const float *uz, float *out_max,
                   void *stream);
/* The driver's dt rule (run_edge.py:595-614) on the device: reads
 * max_speed, updates the double state sub_t (and frame bookkeeping) and writes
 * dt (float) and dt/2 (float).  state: double[4] = {sub_t, frame_idx,
 * output_frame, last dt}. */
int edge_compute_dt(const float *max_speed, float cfl, float dx, double visualize_dt, double *state, float *dt,
                    float *half_dt, void *stream);
/* add_fields / scale_field, taichi_utils.py:6-15: dest = f1 + a*f2 (f2 may
 * be NULL: dest = a*f1) over n floats */
int edge_axpy(long long n, const float *f1, const float *f2, float a, float *dest, void *stream);
/* copy_from over n floats */
int edge_copy(long long n, const float *src, float *dst, void *stream);

/* ---- pressure projection (sim/mgpcg.py, sim/mgpcg_solid.py) ------------ */
/* MGPCG_3 / MGPCG_Solid_3 constructors, mgpcg.py:364-371, mgpcg_solid.py:313-324.
 * bt: boundary_types as int[6] = {x-, x+, y-, y+, z-, z+} (2 = wall).
 * mask / bvel (device, int32 cells / vec3 cells) select the solid solver;
 * both NULL for the plain one.  precision: 0 = float32 V-cycle (the
 * reference), 1 = mixed with bf16 smoother storage, 2 = mixed with fp16
 * smoother storage (the V-cycle runs on the residual times a power of two
 * that brings its RMS near 1); both keep float32 residuals and arithmetic
 * and float64 dot products. */
int edge_mgpcg_create(void **handle, int nx, int ny, int nz, int base_level, const int *bt, const int *mask,
                      const float *bvel, int precision);
int edge_mgpcg_destroy(void *handle);
/* Poisson (mgpcg.py:440-445), Poisson_with_buffer (mgpcg.py:481-486; f* non-
 * NULL) and MGPCG_Solid_3.Poisson (mgpcg_solid.py:418-427), in place on u.
 * max_iters < 0 uses the reference's (400 plain, 100 solid).  The whole
 * solve runs on the stream without host synchronisation (CUDA graph with a
 * device-side while loop); read the outcome with edge_mgpcg_result. */
int edge_mgpcg_poisson(void *handle, float *ux, float *uy, float *uz, float *fx, float *fy, float *fz,
                       double abs_tol, double rel_tol, int max_iters, void *stream);
/* Solve A x = b (A: the solver's 7-point operator) from x = 0 with the same
 * MGPCG loop; b is not modified. */
int edge_mgpcg_solve(void *handle, const float *b, float *x, double abs_tol, double rel_tol, int max_iters,
                     void *stream);
/* Outcome of the last solve (synchronises the stream): iters as the reference
 * prints it, final r.r, status (0 converged, EDGE_ENOCONV, EDGE_ENAN). */
int edge_mgpcg_result(void *handle, int *iters, double *rTr, int *status, void *stream);
/* One V-cycle z = M^-1 r (apply_preconditioner, mgpcg.py:177-195) and
 * Ap = A p (compute_Ap, mgpcg.py:112-117), for testing. */
int edge_mgpcg_vcycle(void *handle, const float *r, float *z, void *stream);
int edge_mgpcg_apply_A(void *handle, const float *p, float *Ap, void *stream);
/* The same operator in float64 (no reference counterpart): the FP64
 * reference solve that the precision study measures errors against. */
int edge_mgpcg_apply_A_f64(void *handle, const double *p, double *Ap, void *stream);
/* Stepwise solve with a replaceable coarse solver (no reference counterpart;
 * the learned preconditioner's path).  The V-cycle's levels lc..L-1 normally
 * run in one shared-memory block (the coarse group); these calls let the
 * caller replace that group by its own solver of the level-lc residual
 * equation.  EDGE_ESTATE when the whole grid fits the coarse group (lc = 0).
 *   coarse_shape: lc and its cell dims (int[3]);
 *   solve_begin:  set-up of solve(b) up to the first V-cycle's coarse level;
 *   coarse_get_r: the level-lc residual as a float32 cell array;
 *   coarse_set_z: the level-lc correction from a float32 cell array, or
 *   coarse_default: the built-in coarse group;
 *   solve_iter:   the rest of that V-cycle, one CG iteration and the next
 *                 V-cycle's descent (nothing once the solve has ended);
 *   solve_end:    the solution into x.
 * edge_mgpcg_result reports the status between iterations.  One coarse step
 * per solve_iter, starting after solve_begin: the V-cycles and CG updates are
 * those of edge_mgpcg_solve. */
int edge_mgpcg_coarse_shape(void *handle, int *level, int *dims);
int edge_mgpcg_solve_begin(void *handle, const float *b, double abs_tol, double rel_tol, int max_iters,
                           void *stream);
int edge_mgpcg_coarse_get_r(void *handle, float *dense, void *stream);
int edge_mgpcg_coarse_set_z(void *handle, const float *dense, void *stream);
int edge_mgpcg_coarse_default(void *handle, void *stream);
int edge_mgpcg_solve_iter(void *handle, void *stream);
int edge_mgpcg_solve_end(void *handle, const float *b, float *x, void *stream);
/* The same for the projection (edge_mgpcg_poisson): poisson_begin applies
 * the walls / solid velocities and forms the divergence, poisson_end
 * subtracts the pressure gradient (and writes -grad p into f*, each may be
 * NULL, as Poisson_with_buffer does). */
int edge_mgpcg_poisson_begin(void *handle, float *ux, float *uy, float *uz, double abs_tol, double rel_tol,
                             int max_iters, void *stream);
int edge_mgpcg_poisson_end(void *handle, float *ux, float *uy, float *uz, float *fx, float *fy, float *fz,
                           void *stream);
/* Restart the CG recursion of a stepwise solve: the next iteration takes
 * p = z (beta = 0), e.g. after the caller changes its coarse solver. */
int edge_mgpcg_restart(void *handle, void *stream);
/* Iterations, r.r and whether the CG loop still runs (1) or has ended (0);
 * synchronises the stream. */
int edge_mgpcg_progress(void *handle, int *iters, double *rTr, int *running, void *stream);
/* Iterative refinement of a mixed-precision solve (no reference counterpart):
 * r = b - A x with b, x (device float64, cell layout) and the arithmetic in
 * float64, r written as float32 (the right-hand side of the next inner solve),
 * and sums[0] = sum r^2, sums[1] = sum b^2 over fluid cells (device float64,
 * block-ordered sums); then x += d for the inner solve's correction d. */
int edge_mgpcg_refine_residual(void *handle, const double *b, const double *x, float *r, double *sums,
                               void *stream);
int edge_mgpcg_refine_update(void *handle, double *x, const float *d, void *stream);
/* Copy the divergence (u_div) or pressure (p) of the last Poisson call. */
int edge_mgpcg_get(void *handle, int which, float *dst, void *stream);
/* Number of multigrid levels (mgpcg.py:34). */
int edge_mgpcg_levels(void *handle);
/* Kernels this solver has executed since creation, counted on the device
 * (the CG loop's length is decided there); synchronises the stream.  No
 * reference counterpart: launch accounting for benchmarks. */
int edge_mgpcg_kernel_count(void *handle, long long *count, void *stream);

/* The plain (wall-bounded, no solid mask) Poisson projection of
 * edge_mgpcg_poisson for callers that cannot allocate device memory while
 * they run, e.g. code hosted inside a runtime that owns the device heap or a
 * graph-replaying engine that forbids cudaMalloc after warm-up.  It has no
 * counterpart in the reference.  It allocates nothing: its scratch is a set
 * of file-scope __device__ arrays sized for at most 262144 cells (64^3),
 * about 8 MB held by every GPU that loads the library until the process
 * exits; larger grids return EDGE_EINVAL.  The first call on a device looks
 * up the arrays' device addresses (with that device current) and should come
 * before any stream capture.  All calls share the arrays, so calls that
 * overlap on the GPU (other streams, other threads) race; the call returns
 * after the solve (it reads the loop state each iteration) with iters, r.r
 * and status as edge_mgpcg_result reports them (each may be NULL). */
int edge_mgpcg_poisson_noalloc(int nx, int ny, int nz, int base_level, const int *bt, float *ux, float *uy,
                               float *uz, double abs_tol, double rel_tol, int max_iters, int *iters, double *rTr,
                               int *status, void *stream);

/* ---- measurement ---------------------------------------------------------- */
/* FP32 FMA throughput probe (no reference counterpart): `blocks` blocks of
 * 256 threads run `iters` x 128 dependent-chain FMAs each; *flops receives
 * the floating-point operations enqueued.  Time it with events on `stream`.
 * `out` is a device float that is never written for these inputs. */
int edge_fma_peak(int blocks, int iters, float *out, double *flops, void *stream);

/* ---- learned preconditioner (no reference counterpart) ------------------------
 * A 3-D U-Net whose 16-64 channel 3x3x3 convolutions run on the tensor cores
 * (tcgen05, BF16 operands, FP32 accumulation in TMEM).  Activation tensors
 * are "padded chunked" bf16: interior grid X x Y x Z with a zero voxel of
 * padding on each side, channels in chunks of 8, each chunk *chunk_voxels
 * voxels long (guards included); a tensor of C channels holds
 * C/8 * chunk_voxels * 8 bf16 values and starts zeroed.  Calls that can give
 * up a bounded wait set the device int *err to 1. */
/* One-CTA tcgen05 GEMM D = A B^T (layout self-test).  mode 0: M = 128, A is
 * 128 x K, B is N x K; mode 1: M = 64, A is K x 64, B is K x N.  D is M x N
 * row-major FP32; 16 <= N, K <= 256, multiples of 16. */
int edge_tc_selftest(int mode, int N, int K, const void *A, const void *B, float *D, int *err, void *stream);
int edge_unet_geometry(int X, int Y, int Z, long long *chunk_voxels);
/* y = act(conv3(x0; w0) [+ conv3(x1; w1)] + bias): 3x3x3 zero-padded
 * cross-correlation, tap t = 9(dx+1) + 3(dy+1) + (dz+1) reading x[v+(dx,dy,dz)].
 * cin0, cin1, cout in {16, 32, 64}; w packed by edge_unet_pack_weights;
 * flags bit 0: ReLU, bit 1: add the result to y; x1 and bias may be NULL. */
int edge_unet_conv(int X, int Y, int Z, const void *x0, const void *w0, int cin0, const void *x1, const void *w1,
                   int cin1, int cout, const float *bias, int flags, void *y, int *err, void *stream);
/* dw[co][ci][27] (float32) = sum over voxels of d[v][co] x[v+off(t)][ci] on
 * the tensor cores; partial holds nsplit * 27 * cout * cin floats. */
int edge_unet_wgrad(int X, int Y, int Z, const void *d, int cout, const void *x, int cin, float *partial,
                    int nsplit, float *dw, int *err, void *stream);
/* First layer (1 -> 16, ReLU) of r (float32 X x Y x Z) times *scale, and last
 * layer (16 -> 1, divided by *scale), on the SIMT cores; w [16][27] float
 * (bf16-rounded values). */
int edge_unet_conv_first(int X, int Y, int Z, const float *r, const float *scale, const float *w, const float *bias,
                         void *y, void *stream);
int edge_unet_conv_last(int X, int Y, int Z, const void *f, const float *w, const float *bias, const float *scale,
                        float *z, void *stream);
/* Backward of the first layer (weight gradient dw [16][27] from its
 * pre-activation gradient d) and of the last (data gradient df and weight
 * gradient dw [16][27] from dzn, the gradient of the output times *scale);
 * partial holds 27 * nblk * 16 floats. */
int edge_unet_first_bwd(int X, int Y, int Z, const void *d, const float *r, const float *scale, float *partial,
                        int nblk, float *dw, void *stream);
int edge_unet_last_bwd(int X, int Y, int Z, const float *dzn, const float *w, const void *f, void *df,
                       float *partial, int nblk, float *dw, void *stream);
/* out[c] = sum over voxels of d[v][c] (bias gradients); partial holds
 * channels * nblk floats. */
int edge_unet_chan_sum(int X, int Y, int Z, int channels, const void *d, float *partial, int nblk, float *out,
                       void *stream);
/* out = dy where y > 0, else 0 (whole tensors). */
int edge_unet_relu_bwd(int X, int Y, int Z, int channels, const void *dy, const void *y, void *out, void *stream);
/* 2x2x2 mean pooling fine -> coarse and its backward (dfine = dcoarse/8,
 * added when accum); nearest 2x upsampling coarse -> fine and its backward
 * (sum of the 8 children).  X, Y, Z: the fine grid. */
int edge_unet_pool(int X, int Y, int Z, int channels, const void *fine, void *coarse, void *stream);
int edge_unet_pool_bwd(int X, int Y, int Z, int channels, const void *dcoarse, void *dfine, int accum, void *stream);
int edge_unet_upsample(int X, int Y, int Z, int channels, const void *coarse, void *fine, void *stream);
int edge_unet_up_bwd(int X, int Y, int Z, int channels, const void *dfine, void *dcoarse, void *stream);
/* float32 weights [cout][cin][27] -> packed bf16 [27][cin/8][cout][8]; with
 * transpose != 0 the data-gradient form [27][cout/8][cin][8] of w[co][ci][26-t]. */
int edge_unet_pack_weights(const float *w, int cout, int cin, int transpose, void *out, void *stream);
/* *scale = 1 / rms(r) over n values (the network's input normalisation).
 * work: device scratch of 1024 doubles + 8 bytes, zeroed before its first use
 * (the call leaves it ready for the next). */
int edge_unet_input_scale(const float *r, long long n, void *work, float *scale, void *stream);
/* Training loss on the scaled problem, d = (z - target) * scale:
 * stats[0] = mean(d), stats[1] = mean((d - mean d)^2); dzn = 2 (d - mean d) / n. */
int edge_unet_loss(const float *z, const float *target, const float *scale, long long n, double *stats, float *dzn,
                   void *stream);
/* One Adam step on n float32 parameters (step counts from 1). */
int edge_unet_adam(long long n, float *p, const float *g, float *m, float *v, float lr, float b1, float b2, float eps,
                   int step, void *stream);

/* ---- laden particles (sim/lp.py) ---------------------------------------- */
/* update_particles_acc, lp.py:6-29 (acc zeroed for all nmax particles) */
int edge_lp_acc(int nx, int ny, int nz, float dx, const float *ux, const float *uy, const float *uz,
                const float *vel, const float *pos, float *acc, int num, int nmax, float dt, float St,
                float gravity, void *stream);
/* update_particles_velocity, lp.py:32-70 */
int edge_lp_velocity(const float *acc, float *vel, const float *pos, float dt, float dx, int num, float Lx,
                     float Ly, float Lz, void *stream);
/* calculate_velocity_diff, lp.py:73-97 */
int edge_lp_vel_diff(int nx, int ny, int nz, float dx, const float *ux, const float *uy, const float *uz,
                     const float *vel, float *vdiff, const float *pos, int num, float St, float density_ratio,
                     float epiral_radius_ratio, void *stream);
/* laden_particles_back_with_computing_particle, lp.py:100-156 (P2G drag
 * scatter; drag fields are zeroed first) */
int edge_lp_p2g(int nx, int ny, int nz, float dx, float *dragx, float *dragy, float *dragz, const float *vdiff,
                const float *pos, const float *rad, int num, float laden_radius, float Lx, float Ly, float Lz,
                void *stream);
/* calc_max_particle_speed, run_edge.py:256-261: max |v| (>= 1e-3) of the
 * first num particles into out (one float, device memory) */
int edge_lp_max_speed(const float *vel, int num, float *out, void *stream);
/* update_particles_position, lp.py:158-181 */
int edge_lp_position(const float *vel, float *pos, float dt, int num, float Lx, float Ly, float Lz, void *stream);
/* calculate_viscous_force, lp.py:183-219, on all three face grids */
int edge_lp_viscous(int nx, int ny, int nz, float dx, float Re, const float *ux, const float *uy, const float *uz,
                    float *visx, float *visy, float *visz, void *stream);

/* ---- initial conditions (sim/init_conditions.py, util/taichi_utils.py) -- */
/* add_vortex_ring_and_smoke, init_conditions.py:11-36: accumulates into u
 * (vec3 cells) and smoke (vec4 cells); c, ex, ey, color are host float[3]. */
int edge_add_vortex_ring(int nx, int ny, int nz, float dx, float w, float rad, float delta, const float *c,
                         const float *ex, const float *ey, float *u, float *smoke, const float *color,
                         int num_samples, void *stream);
/* emit_smoke_delta, init_conditions.py:177-232: cells within `radius` of one
 * of k <= 16 emitter centres (host float[k][3]) take its colour (host
 * float[k][4]); later emitters win. */
int edge_emit_smoke(int nx, int ny, int nz, float dx, const float *centers, const float *colors, int k,
                    float radius, float *smoke, void *stream);
/* clamp_smoke_density, init_conditions.py:234-243: x = min(x, hi) over n floats */
int edge_clamp_max(long long n, float hi, float *x, void *stream);
/* split_central_vector, taichi_utils.py:103-116 */
int edge_split_central_vector(int nx, int ny, int nz, const float *vc, float *ux, float *uy, float *uz,
                              void *stream);
/* get_central_vector, taichi_utils.py:95-100: vc (nx,ny,nz,3) = face averages */
int edge_get_central_vector(int nx, int ny, int nz, const float *ux, const float *uy, const float *uz, float *vc,
                            void *stream);
/* curl, taichi_utils.py:69-92: cf = curl of the cell vec3 field vf (both
 * (nx,ny,nz,3)), central differences with clamped neighbour indices */
int edge_curl(int nx, int ny, int nz, float dx, const float *vf, float *cf, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* EDGE_B200_H */
