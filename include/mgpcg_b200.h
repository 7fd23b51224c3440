/*
 * mgpcg_b200.h - C ABI of the B200-native MGPCG Poisson solver.
 *
 * This is the boundary a host binding (ctypes, cffi, a C/C++ simulator) links
 * against.  Signatures use plain C types: integers, float/double scalars,
 * void pointers to device memory and an opaque plan handle.  A cudaStream_t
 * is passed as `void*`.  Nothing here allocates device memory: the caller
 * allocates one workspace of mg_plan_workspace_bytes() and every field of the
 * solver lives at a fixed offset inside it (mg_plan_field()).
 *
 * Each entry point names the reference interface it replaces
 * (file:line in g1n0st/taichi-ferrofluid).
 *
 * Return value of every `int` function: MG_OK (0) or a negative MG_E* code.
 */
#ifndef MGPCG_B200_H
#define MGPCG_B200_H

#include <stdint.h>

#if defined(__GNUC__)
#define MG_API __attribute__((visibility("default")))
#else
#define MG_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- labels: utils.py:4-6 --------------------------------------------- */
#define MG_FLUID 0
#define MG_AIR 1
#define MG_SOLID 2

/* ---- status codes -------------------------------------------------------- */
#define MG_OK 0
#define MG_E_BADARG (-1)    /* invalid size, level count, pointer or field id */
#define MG_E_CUDA (-2)      /* a CUDA runtime call failed (see mg_last_error) */
#define MG_E_UNBOUND (-3)   /* the plan has no workspace bound */
#define MG_E_TOO_BIG (-4)   /* a size exceeds a fixed capacity of the call */

/* solve outcome, written to mg_solve_stats_t.status */
#define MG_SOLVE_CONVERGED 0
#define MG_SOLVE_MAX_ITERS 1   /* stopped at max_iters (the reference is silent) */
#define MG_SOLVE_NONFINITE 2   /* a reduction produced NaN/Inf (H3: zero Adiag) */
#define MG_SOLVE_BAD_OPERATOR 3 /* a declared operator form (mg_plan_prepare_declared*) was wrong */
#define MG_SOLVE_TIMEOUT 4      /* a bounded wait on a TMA copy ran out (the sweep left its chunk) */

/* V-cycle grid storage type */
#define MG_STORE_F32 0
#define MG_STORE_F16 1
#define MG_STORE_BF16 2

/* field ids for mg_plan_field() */
#define MG_FIELD_B 0        /* level 0, f32: right-hand side       (mgpcg.py:21) */
#define MG_FIELD_X 1        /* level 0, f32: solution              (mgpcg.py:39) */
#define MG_FIELD_P 2        /* level 0, f32: CG direction          (mgpcg.py:40) */
#define MG_FIELD_AP 3       /* level 0, f32: A p                   (mgpcg.py:41) */
#define MG_FIELD_R 4        /* per level: residual r[l]; level 0 is f32, coarser
                               levels use the storage type          (mgpcg.py:23) */
#define MG_FIELD_Z 5        /* per level, storage type: z[l]        (mgpcg.py:25) */
#define MG_FIELD_TYPE 6     /* per level, int8: grid_type[l]        (mgpcg.py:29) */
#define MG_FIELD_ADIAG 7    /* per level, f32: Adiag[l]             (mgpcg.py:33) */
#define MG_FIELD_AX 8       /* per level, f32, component k: Ax[l][k] stored as
                               `dim` contiguous planes (SoA)        (mgpcg.py:35) */

/* Problem description: MGPCGPoissonSolver.__init__ (mgpcg.py:6-44). */
typedef struct mg_plan_desc {
  int32_t dim;          /* 2 or 3 */
  int32_t res[3];       /* level-0 shape; res[2] ignored when dim == 2 */
  int32_t levels;       /* n_mg_levels (>= 1); every res[k] % 2^(levels-1) == 0 */
  int32_t pre_post;     /* pre_and_post_smoothing */
  int32_t bottom;       /* bottom_smoothing (half of it in each colour order) */
  int32_t storage;      /* MG_STORE_*: type of the V-cycle grids */
  int32_t refresh_every;/* recompute r = b - A x every N iterations (0: never) */
  int32_t flags;        /* MG_PLAN_* bits */
} mg_plan_desc_t;

/* plan flags */
#define MG_PLAN_STORED 1  /* always use the stored-coefficient kernels, one launch
                             per reference kernel (no fused V-cycle) */
#define MG_PLAN_DIRECT 2  /* launch the PCG iterations from a host loop instead
                             of the CUDA graph: the same kernels in the same
                             order, one 4-byte device->host read and stream
                             synchronisation per iteration, so mg_pcg_solve_async
                             returns only when the solve has finished.  For
                             profilers that do not follow conditional graph
                             nodes; slower than the default. */

/* Solve parameters: MGPCGPoissonSolver.solve (mgpcg.py:150-155). */
typedef struct mg_solve_params {
  int32_t max_iters;    /* -1: no limit */
  int32_t warm_start;   /* 0: x = 0, r = b (reference); 1: r = b - A x for the given x */
  double rel_tol;       /* on squared norms: stop when r.r < max(abs_tol, rel_tol * b.b) */
  double abs_tol;
  double eps;           /* added to the denominators of alpha and beta */
} mg_solve_params_t;

/* Outcome of one solve (the reference returns nothing; see H5). */
typedef struct mg_solve_stats {
  int32_t status;       /* MG_SOLVE_* */
  int32_t iters;        /* the reference's `iter` counter at exit */
  double rTr0;          /* initial r.r */
  double rTr;           /* final r.r (recursive residual) */
  double bTb;           /* b.b; the tolerance is max(abs_tol, rel_tol * b.b),
                           which equals the reference's r0.r0 for a cold start */
} mg_solve_stats_t;

typedef struct mg_plan mg_plan_t;

/* ---- plan ----------------------------------------------------------------- */

/* MGPCGPoissonSolver.__init__ (mgpcg.py:6-44): validates the description and
 * lays out every field; allocates host memory only. */
MG_API int mg_plan_create(const mg_plan_desc_t* desc, mg_plan_t** out);
MG_API int mg_plan_destroy(mg_plan_t* plan);

/* Bytes of device memory the caller must provide (256-byte aligned). */
MG_API int64_t mg_plan_workspace_bytes(const mg_plan_t* plan);

/* Offset and size in bytes of a field inside the workspace (mgpcg.py:21-44). */
MG_API int mg_plan_field(const mg_plan_t* plan, int32_t field, int32_t level, int32_t component,
                  int64_t* offset, int64_t* nbytes);

/* Binds the workspace base pointer (device memory on the current device). */
MG_API int mg_plan_bind(mg_plan_t* plan, void* workspace);

/* ---- setup: MGPCGPoissonSolver.initialize / reinitialize ------------------ */

/* initialize() (mgpcg.py:63-77): zeroes every field. */
MG_API int mg_initialize(mg_plan_t* plan, void* stream);

/* grid_type[0].copy_from(cell_type) (mgpcg.py:81): int32 labels -> int8. */
MG_API int mg_set_cell_type(mg_plan_t* plan, const int32_t* cell_type, void* stream);

/* init_gridtype(grid_type[l-1], grid_type[l]) (mgpcg.py:46-60, :86). */
MG_API int mg_init_gridtype(mg_plan_t* plan, int32_t level, void* stream);

/* grid_type[l].fill(FLUID) for every level (mgpcg.py:93). */
MG_API int mg_fill_fluid(mg_plan_t* plan, void* stream);

/* PressureProjectStrategy.build_b_kernel (pressure_project.py:15-39).
 * vel[k] is the MAC face velocity of axis k, shape res + e_k (f32);
 * phi is the level set at cell centres (f32).  ghost != 0 selects the ghost
 * fluid method; gfm_clamp is the cap on (phi_i - phi_j) / phi_i (1e3 in the
 * reference). */
MG_API int mg_build_pressure_b(mg_plan_t* plan, const float* vel0, const float* vel1, const float* vel2,
                        const float* phi, float p0, float scale_A, float scale_b, int32_t ghost,
                        float gfm_clamp, void* stream);

/* PressureProjectStrategy.build_A_kernel(level) (pressure_project.py:45-64). */
MG_API int mg_build_pressure_A(mg_plan_t* plan, int32_t level, const float* phi, float scale_A,
                        int32_t ghost, float gfm_clamp, void* stream);

/* b[I] += c * src[I] (or += c when src is NULL) on level-0 FLUID cells:
 * PressureProjectWithVolumeControlStrategy.add_c (volume_control.py:33-37),
 * and the extra smooth source term of the precision workload. */
MG_API int mg_add_rhs(mg_plan_t* plan, const float* src, float c, void* stream);

/* Magnetic potential Strategy of the 3D ferrofluid substep: the solve of
 * FerrofluidSimulator.update_potential_function (ferrofluid_simulator.py:77-87,
 * potential_function.py:19-55) in the benchmark's form: permeability
 * mu = 1 + chi (chi at cell centres), face coefficient = harmonic mean of mu
 * over dx^2, rhs = -div(mu H) for a constant external field H, Neumann at the
 * domain boundary, psi pinned to 0 at cell `pin`.  Use with
 * full_reinitialize (every label FLUID).  mg_build_psi_A builds level 0. */
MG_API int mg_build_psi_b(mg_plan_t* plan, const float* chi, float H0, float H1, float H2, float dx,
                          int32_t pin0, int32_t pin1, int32_t pin2, void* stream);
MG_API int mg_build_psi_A(mg_plan_t* plan, const float* chi, float dx, int32_t pin0, int32_t pin1,
                          int32_t pin2, void* stream);

/* Galerkin coarse operator of `level` from level-1: A_c = scale * P^T A P for
 * the reference's piecewise-constant prolongation and child-sum restriction
 * (mgpcg.py:111-123); scale must be a power of two (exact in f32).  scale 1/2
 * over-corrects the piecewise-constant coarse correction by 2, which the
 * magnetic potential Strategy uses (8 PCG iterations instead of 38 at 128^3).  The reference's whole-domain Strategies rebuild each
 * level from the fine fields instead (mgpcg.py:89-94, potential_function.py:
 * 41-55); this is the coarse-level rule of the magnetic potential Strategy
 * above. */
MG_API int mg_galerkin_coarsen(mg_plan_t* plan, int32_t level, float scale, void* stream);

/* The same operator rediscretised on coarse level `level` (>= 1), as the
 * reference's potential Strategy builds its coarse levels
 * (potential_function.py:39-55: the coefficient field re-sampled per level,
 * spacing dx * 2^level): chi_level (the level's shape, written) = the mean of
 * the 2^dim children of chi_fine (the finer level's chi), then face
 * coefficients mu(I, J) / (dx 2^level)^2 and the pin's coarse cell pinned.
 * Call per level in increasing order, each with the previous level's chi. */
MG_API int mg_build_psi_A_level(mg_plan_t* plan, int32_t level, const float* chi_fine, float* chi_level, float dx,
                                int32_t pin0, int32_t pin1, int32_t pin2, void* stream);

/* ---- the reference's other Strategies (all f32, all on `stream`) ----------
 * Fields are dense row-major device arrays, last axis fastest: cell fields
 * have the plan's level-0 shape res, MAC face fields of axis k have shape
 * res + e_k.  Python-side constants the reference folds in double (1/dt,
 * sigma dt / dx^2, 1/dx) are taken as double and folded here the same way. */

/* MagneticForceStrategy.build_b_kernel (magnetic_force.py:17-38): the
 * pressure right-hand side with the magnetic pressure on AIR faces,
 * scale_A (p0 + coef |H|^2) with H interpolated from the MAC field H at the
 * AIR cell centre (FerrofluidSimulator.H_interp, ferrofluid_simulator.py:
 * 64-69) and coef = k mu0 / 2.  Use with mg_build_pressure_A (the Strategy
 * inherits build_A from PressureProjectStrategy). */
MG_API int mg_build_magnetic_b(mg_plan_t* plan, const float* vel0, const float* vel1, const float* vel2,
                               const float* H0, const float* H1, const float* H2, float p0, float scale_A,
                               float scale_b, float coef, void* stream);

/* PotentialFunctionStrategy (potential_function.py:19-55), the reference's
 * own form of the magnetic potential solve: whole domain, negative-definite A
 * with face coefficients (1 + chi)/dx from chi sampled at the faces, the
 * origin cell pinned (Adiag = 1/dx, b = 0), faces tested against the fine
 * resolution on every level.  H_ext is the MAC external field.  Use with
 * full_reinitialize; mg_build_potential_A builds one level. */
MG_API int mg_build_potential_b(mg_plan_t* plan, const float* chi, const float* Hext0, const float* Hext1,
                                const float* Hext2, void* stream);
MG_API int mg_build_potential_A(mg_plan_t* plan, int32_t level, const float* chi, double dx, void* stream);

/* The field updates around the potential solve of the ferrofluid substep:
 * mg_update_susceptibility: update_magnetic_susceptibility
 * (ferrofluid_simulator.py:71-75), chi = k (1 - theta(phi)), eps the level
 * set's half width; mg_update_magnetic_field: update_magnetic_field
 * (ferrofluid_simulator.py:89-97), H = H_ext - grad psi on the MAC faces
 * (H = H_ext on the domain faces); psi NULL reads the plan's x. */
MG_API int mg_update_susceptibility(mg_plan_t* plan, const float* phi, double k, float eps, float* chi,
                                    void* stream);
MG_API int mg_update_magnetic_field(mg_plan_t* plan, const float* psi, const float* Hext0, const float* Hext1,
                                    const float* Hext2, float dx, float* H0, float* H1, float* H2, void* stream);

/* PressureProjectWithVolumeControlStrategy (volume_control.py:7-51).
 * mg_level_set_volume: calc_volume (volume_control.py:22-31), the smoothed
 * fluid volume sum over cells of the mean of theta(-phi) over the 2^d cell
 * corners, summed in FP64 into the device double *out.  eps is the level
 * set's interface half width (level_set.py:22, 5 dx).
 * mg_volume_control: one build_b step after mg_build_pressure_b: the volume,
 * the PI controller on the device and b += c on FLUID cells, with no host
 * synchronisation.  state is 8 device doubles: [0] step, [1] vol_0, [2] y,
 * [3] last volume, [4] last c, [5] k_p, [6] k_i, [7] dt; the caller sets
 * [0..4] = 0 and [5..7] (k_p = 2.3 / (25 dt), k_i = (k_p / 4)^2 in the
 * reference). */
MG_API int mg_level_set_volume(mg_plan_t* plan, const float* phi, float eps, double* out, void* stream);
MG_API int mg_volume_control(mg_plan_t* plan, const float* phi, float eps, double* state, void* stream);

/* SurfaceTension (surface_tension.py:98-153) and SurfaceTensionStrategy
 * (surface_tension.py:10-95) for velocity axis d: mg_calc_surface_normal
 * writes n (dim planes of the cell grid, n[k * cells + i]) = normalised
 * gradient of phi at the cell shifted half a cell off axis d; mg_calc_curvature
 * writes kappa = div n; the builders write b and one level of A of the
 * implicit surface tension solve for u_d (whole domain, use with
 * full_reinitialize).  eps is the level set's half width (5 dx). */
MG_API int mg_calc_surface_normal(mg_plan_t* plan, int32_t d, const float* phi, float dx, float* n,
                                  void* stream);
MG_API int mg_calc_curvature(mg_plan_t* plan, const float* n, float dx, float* kappa, void* stream);
MG_API int mg_build_surface_tension_b(mg_plan_t* plan, int32_t d, const float* u_d, const float* phi,
                                      const float* n, const float* kappa, double sigma, double dt, double dx,
                                      double eps, void* stream);
MG_API int mg_build_surface_tension_A(mg_plan_t* plan, int32_t level, int32_t d, const float* phi,
                                      double sigma, double dt, double dx, double eps, void* stream);

/* ---- the step before the solve: labels and level set ----------------------
 * Plan-free: the grid is (dim, res).  phi and cell_type are dense row-major
 * device arrays of shape res (float32 / int32, the simulator's fields).
 * mg_level_set_shape: LevelSet.initialize_with_aabb (level_set.py:40-59;
 * sphere = 0, box [a, b]) or initialize_with_sphere (level_set.py:61-64;
 * sphere != 0, centre a, radius b[0]): phi = the shape's signed distance at
 * the cell centres (I + 0.5) dx; combine != 0 keeps min(phi, distance)
 * instead, the union of several shapes.
 * mg_apply_markers: FluidSimulator.apply_markers (fluid_simulator.py:151-159),
 * non-SOLID cells AIR, then FLUID where phi <= 0 (strict != 0: phi < 0).
 * mg_init_boundary: FluidSimulator.init_boundary (fluid_simulator.py:337-341),
 * SOLID on the outermost ring. */
MG_API int mg_level_set_shape(int32_t dim, const int32_t* res, float* phi, float dx, int32_t sphere,
                              const float* a, const float* b, int32_t combine, void* stream);
MG_API int mg_apply_markers(int32_t dim, const int32_t* res, int32_t* cell_type, const float* phi, int32_t strict,
                            void* stream);
MG_API int mg_init_boundary(int32_t dim, const int32_t* res, int32_t* cell_type, void* stream);

/* FastSweepingLevelSet.redistance (level_set.py:260-334): valid = -1 and
 * target_surface (level_set.py:66-86: cells beside a sign change get the
 * interpolated distance to it, valid 0), then repeat_times rounds of the fast
 * sweeping propagation (each round: forward and backward sweeps along the
 * last axis, then along each slower axis; upwind Eikonal update of
 * level_set.py:88-112), then phi = phi_temp.  phi_temp (float32) and valid
 * (int32) are caller scratch of shape res.  The lines of a sweep run in
 * parallel and read each other's cells while they change, as the
 * reference's do, so the propagated values can differ in the last bits from
 * run to run.  Every axis needs at least 2 cells. */
MG_API int mg_level_set_redistance(int32_t dim, const int32_t* res, float* phi, float* phi_temp, int32_t* valid,
                                   double dx, int32_t repeat_times, void* stream);

/* FastSweepingLevelSet.propagate (level_set.py:283-327) alone: the sweeps of
 * mg_level_set_redistance on the caller's phi_temp (updated where valid is
 * -1), with phi giving the sign. */
MG_API int mg_level_set_propagate(int32_t dim, const int32_t* res, const float* phi, float* phi_temp,
                                  const int32_t* valid, double dx, int32_t repeat_times, void* stream);

/* FastSweepingLevelSet.build_from_markers (level_set.py:381-392), its first
 * part: phi = 1e20, valid = -1, LevelSet.distance_to_markers
 * (level_set.py:114-122: the cell of each marker - coordinates / dx
 * truncated toward zero - takes the distance to its centre when smaller,
 * valid = the marker's index), then markers_propagate (level_set.py:336-379:
 * repeat_times rounds of 2 dim line sweeps; a cell takes the distance to the
 * marker of its neighbour one step ahead when smaller).  markers: n_markers x
 * dim float32 positions (device).  Where the reference's parallel loop races
 * between markers of one cell, the cell keeps the smallest distance and,
 * among equal ones, the smallest index; a neighbour without a marker is
 * skipped (the reference reads markers[-1] there); markers with non-finite
 * coordinates are ignored. */
MG_API int mg_level_set_markers_distance(int32_t dim, const int32_t* res, float* phi, int32_t* valid,
                                         const float* markers, int32_t n_markers, double dx, int32_t repeat_times,
                                         void* stream);

/* LevelSet.target_minus (level_set.py:124-146) after valid.fill(-1): phi -=
 * 0.99 dx (the marker radius); cells beside a sign change with phi <= 0 and
 * cells with phi > 0 are known (valid 0, phi_temp = phi), the other cells get
 * phi_temp = -1 for mg_level_set_propagate. */
MG_API int mg_level_set_target_minus(int32_t dim, const int32_t* res, float* phi, float* phi_temp, int32_t* valid,
                                     double dx, void* stream);

/* LevelSet.smoothing (level_set.py:148-163): out = min(mean of the in-range
 * axis neighbours of in, in); out and in are different arrays of shape res. */
MG_API int mg_level_set_smooth(int32_t dim, const int32_t* res, float* out, const float* in, void* stream);

/* ---- the velocity steps around the projection (plan-free) ----------------
 * Velocity components vel0..2 are MAC face arrays of shape res + e_k; cell
 * arrays have shape res.
 * mg_advect_quantity: FluidSimulator.advect_quantity (fluid_simulator.py:
 * 216-236): every face of every component (and, if phi_out is not NULL, the
 * level set) is traced back through the velocity with the midpoint rule and
 * sampled from its source (utils.sample) into the *_out arrays, which must not
 * alias the inputs; update_quantity is the caller's copy back.
 * mg_extrapolate_velocity: FluidSimulator.extrap_velocity for one axis
 * (fluid_simulator.py:244-272): faces beside a FLUID cell are valid, then
 * `iterations` rounds (10 in the reference) give each invalid face with valid
 * neighbours in its 3^d box their mean.  u_tmp, valid, valid_tmp are caller
 * scratch of the face shape; a neighbour outside the face array is invalid.
 * mg_enforce_boundary: FluidSimulator.enforce_boundary (fluid_simulator.py:
 * 168-174): zero velocity on both faces of every SOLID cell.
 * mg_add_gravity: FluidSimulator.add_gravity (fluid_simulator.py:160-166):
 * u_k += g_k dt for every nonzero component g_k. */
MG_API int mg_advect_quantity(int32_t dim, const int32_t* res, const float* vel0, const float* vel1,
                              const float* vel2, const float* phi, float* phi_out, float* vel0_out, float* vel1_out,
                              float* vel2_out, float dx, float dt, void* stream);
MG_API int mg_extrapolate_velocity(int32_t dim, const int32_t* res, int32_t axis, float* vel, float* vel_tmp,
                                   int32_t* valid, int32_t* valid_tmp, const int32_t* cell_type, int32_t iterations,
                                   void* stream);
MG_API int mg_enforce_boundary(int32_t dim, const int32_t* res, float* vel0, float* vel1, float* vel2,
                               const int32_t* cell_type, void* stream);
MG_API int mg_add_gravity(int32_t dim, const int32_t* res, float* vel0, float* vel1, float* vel2, double g0,
                          double g1, double g2, float dt, void* stream);

/* ---- the step after the solve ---------------------------------------------
 * FluidSimulator.apply_pressure (fluid_simulator.py:193-214): the ghost-fluid
 * pressure-gradient update of the MAC velocity, u_k[I] -= scale (p[I] -
 * p[I - e_k]) with p0 (times the clamped ghost-fluid factor) on AIR sides
 * and u = 0 on faces touching SOLID or the domain edge.  pressure NULL reads
 * the plan's x (the solution stays on the device); cell_type (int32, the
 * simulator's labels) NULL reads the plan's level-0 labels.
 * scale = dt / (rho dx).
 * mg_apply_magnetic_force: FerrofluidSimulator.apply_magnetic_force
 * (ferrofluid_simulator.py:115-137), the same update with the AIR-side
 * pressure p0 + coef |H|^2 and no ghost-fluid factor. */
MG_API int mg_apply_pressure(mg_plan_t* plan, float* vel0, float* vel1, float* vel2, const float* pressure,
                             const int32_t* cell_type, const float* phi, float scale, float p0, int32_t ghost,
                             float gfm_clamp, void* stream);
MG_API int mg_apply_magnetic_force(mg_plan_t* plan, float* vel0, float* vel1, float* vel2,
                                   const float* pressure, const int32_t* cell_type, const float* H0,
                                   const float* H1, const float* H2, float scale, float p0, float coef,
                                   void* stream);

/* Prepares the V-cycle operator after the Strategy has written A:
 * detects whether every level's off-diagonals are the uniform label-derived
 * value (the pressure Strategy's form) and, for 16-bit storage, writes the
 * scaled 16-bit coefficient copies.  Called by mg_pcg_solve when A changed;
 * callable explicitly to separate setup from solve time. */
MG_API int mg_plan_prepare(mg_plan_t* plan, void* stream);
/* Prepare without synchronizing: the caller declares that every level is
 * label-uniform with off-diagonal magnitude offdiag[l] (what the pressure
 * Strategy builds, pressure_project.py:56-58).  A device kernel verifies the
 * declaration during the solve; a wrong one ends the solve with status
 * MG_SOLVE_BAD_OPERATOR.  No reference counterpart (the reference has no
 * operator forms). */
MG_API int mg_plan_prepare_declared(mg_plan_t* plan, const float* offdiag, void* stream);
/* Prepare without synchronizing for a whole-domain operator: the caller
 * declares that every cell of every level is FLUID with a nonzero diagonal
 * and the couplings are stored (what the potential Strategies build with
 * full_reinitialize, mgpcg.py:89-94, potential_function.py:6-60).  Verified
 * on the device like mg_plan_prepare_declared; a wrong declaration ends the
 * solve with MG_SOLVE_BAD_OPERATOR. */
MG_API int mg_plan_prepare_declared_whole(mg_plan_t* plan, void* stream);

/* The whole per-request pressure path in one call, enqueued on `stream` with
 * no host synchronization: initialize, cell_type, PressureProjectStrategy
 * build_b / build_A on every level, declared prepare, then the solve
 * (mgpcg.py:79-87 followed by :150-209).  With params->warm_start the x held
 * in the workspace is the initial guess (initialize then keeps x).  Read the
 * outcome with mg_pcg_stats after the stream completes. */
MG_API int mg_pressure_solve_async(mg_plan_t* plan, const int32_t* cell_type, const float* vel0,
                                   const float* vel1, const float* vel2, const float* phi, float p0,
                                   float scale_A, float scale_b, int32_t ghost, float gfm_clamp,
                                   const mg_solve_params_t* params, void* stream);

/* Reports the operator form chosen per level: 1 = label-uniform (fused
 * V-cycle), 2 = whole-domain stored coefficients (every cell FLUID with a
 * nonzero diagonal; fused V-cycle reading the stored couplings), 0 = stored
 * coefficients with the per-kernel V-cycle. */
MG_API int mg_plan_operator_form(const mg_plan_t* plan, int32_t level, int32_t* form);

/* The autotuner's choice per streamed level of a fused V-cycle: bit l set =
 * level l runs the per-kernel sweeps / restriction / prolongation, clear =
 * the streamed kernel.  The whole-domain stored form is timed both ways when
 * a shape is first prepared (the choice is cached per shape); the
 * label-uniform form always streams.  set != 0 forces *bits (after the plan
 * is prepared; valid until the next prepare); *bits returns the choice and
 * *streamed (if not NULL) the number of streamed levels.  The environment
 * variable MGPCG_SPLIT=<bits> replaces the timing for every plan (for
 * profilers, which serialise the trial launches). */
MG_API int mg_plan_split(mg_plan_t* plan, int32_t set, uint32_t* bits, int32_t* streamed);

/* Planes per pipeline step of the streamed sweep (no reference counterpart: a
 * B200 launch shape of the same arithmetic): bit 2l set = level l's PRE sweep
 * (pre-smoothing + restriction) steps one plane at a time, bit 2l+1 the same
 * for its POST sweep; clear = two planes.  3D label-uniform float32 plans
 * time both per level and direction when a shape is first prepared (cached
 * per shape); levels whose chunks are 2 planes run as one step either way.
 * Both shapes give bit-identical values.  set != 0 forces *bits (after the
 * plan is prepared; valid until the next prepare); *bits returns the choice.
 * MGPCG_STEP1=<bits> replaces the timing for every plan (for profilers; with
 * MGPCG_GRID unset, every grid is sized for the blocks that fit). */
MG_API int mg_plan_steps(mg_plan_t* plan, int32_t set, uint32_t* bits);

/* Grid of the streamed sweep (no reference counterpart: a B200 launch shape
 * of the same arithmetic): bits 2l..2l+1 = the blocks per SM, beyond those
 * that fit its shared memory, that level l's grid is sized for (0..3; more
 * blocks, shorter chunks of planes).  Every fused plan times 0, 1 and 2 per
 * pipelined level when a shape is first prepared (cached per shape), before
 * the planes per step.  All grids give bit-identical V-cycles.  set != 0
 * forces *bits (after the plan is prepared; valid until the next prepare);
 * *bits returns the choice.  MGPCG_GRID=<bits> replaces the timing for every
 * plan (for profilers; with MGPCG_STEP1 unset, one plane per step is off). */
MG_API int mg_plan_grid(mg_plan_t* plan, int32_t set, uint32_t* bits);

/* Kernel of each streamed level's sweeps (no reference counterpart: a B200
 * implementation choice for the same arithmetic, mgpcg.py:104-123): bits
 * 2l..2l+1 = 0 for the shared-memory ring kernel, 1..3 for the
 * column-register kernel (TMA-staged planes, z in registers) with a tile of
 * 32x16, 32x32 or 64x16 columns.  The column kernel runs 3D label-uniform
 * plans with pre_post 2 whose fastest extent is a multiple of 16 bytes.
 * Every prepared shape times both kernels, every tile and grid per level when
 * first prepared (cached per shape).  All choices give bit-identical
 * V-cycles.  set != 0 forces *bits (after the plan is prepared; valid until
 * the next prepare; MG_E_BADARG where a level cannot run the column kernel);
 * *bits returns the choice.  MGPCG_COL=<bits> replaces the timing for every
 * plan (for profilers). */
MG_API int mg_plan_sweep_kernel(mg_plan_t* plan, int32_t set, uint32_t* bits);

/* The cluster-resident V-cycle (no reference counterpart: a B200 launch shape
 * of mgpcg.py:125-148 with the same float32 values): for a label-uniform
 * float32 3D plan whose levels [first_level, L) halve exactly, those levels run
 * as ONE launch of one thread-block cluster (up to 16 CTAs), each CTA holding
 * its brick of every level in shared memory and reading its neighbours'
 * through distributed shared memory; the levels above stay streamed.  When a
 * shape is first prepared the V-cycle is timed streamed and with the cluster
 * from each feasible level in 1024- and in 512-thread CTAs, and the fastest
 * kept (cached per shape); MGPCG_RESIDENT=<level> (the first feasible start
 * level from there; MGPCG_RES_THREADS=512 for 512-thread CTAs) or
 * MGPCG_RESIDENT=off replaces the timing.  set != 0 forces *on and, when
 * *on and first_level != NULL and *first_level >= 0, the level the cluster
 * starts at (after the plan is prepared; valid until the next prepare; fails
 * when that level, or any, allows no bricks); *on returns the choice and
 * *first_level (if not NULL) the cluster's first level, -1 when there is none. */
MG_API int mg_plan_resident(mg_plan_t* plan, int32_t set, int32_t* on, int32_t* first_level);

/* ---- the reference's per-kernel operations (for parity tests) ------------ */

MG_API int mg_smooth(mg_plan_t* plan, int32_t level, int32_t phase, void* stream);   /* mgpcg.py:104-109 */
MG_API int mg_restrict(mg_plan_t* plan, int32_t level, void* stream);                /* mgpcg.py:111-118 */
MG_API int mg_prolongate(mg_plan_t* plan, int32_t level, void* stream);              /* mgpcg.py:120-123 */
MG_API int mg_v_cycle(mg_plan_t* plan, void* stream);                                /* mgpcg.py:125-148 */
MG_API int mg_compute_Ap(mg_plan_t* plan, void* stream);                             /* mgpcg.py:218-224 */
/* reduce(a, b) (mgpcg.py:211-216) over level-0 FLUID cells, FP64 sum, written
 * to *out_host after a stream synchronize. a, b are MG_FIELD_* of level 0. */
MG_API int mg_reduce(mg_plan_t* plan, int32_t field_a, int32_t field_b, double* out_host, void* stream);

/* ---- solve ------------------------------------------------------------------ */

/* solve(max_iters, verbose, rel_tol, abs_tol, eps) (mgpcg.py:150-209).
 * The whole PCG loop runs on the device inside one CUDA graph (a while node);
 * scalars alpha, beta and the norms are FP64 on the device.  Blocks until done
 * and writes the outcome to *stats. */
MG_API int mg_pcg_solve(mg_plan_t* plan, const mg_solve_params_t* params, mg_solve_stats_t* stats,
                 void* stream);

/* Same solve without the final synchronize: enqueue on `stream`; read the
 * outcome later with mg_pcg_stats() after the stream has completed. */
MG_API int mg_pcg_solve_async(mg_plan_t* plan, const mg_solve_params_t* params, void* stream);
MG_API int mg_pcg_stats(mg_plan_t* plan, mg_solve_stats_t* stats, void* stream);

/* ---- measurement --------------------------------------------------------------- */

/* Kernel launches the solve graph makes: `prologue` once per solve, `body`
 * once per PCG iteration after the first (no reference counterpart). */
MG_API int mg_plan_launch_counts(mg_plan_t* plan, int32_t* prologue, int32_t* body);

/* Launches one stage of the solve pipeline once on `stream`, on whatever the
 * fields hold, so a caller can time it with events (no reference counterpart;
 * the reference's closest tool is ti.kernel_profiler, fluid_simulator.py:16).
 * stage: 0 = level-`level` pre-smoothing (+ restriction), 1 = level-`level`
 * post-smoothing (+ prolongation), 2 = the coarse solve, 3 = the CG step
 * p/Ap/alpha, 4 = the CG step x/r/r.r, 5 = one whole V-cycle, 6 = the
 * cluster-resident part of the V-cycle (mg_plan_resident). */
MG_API int mg_launch_stage(mg_plan_t* plan, int32_t stage, int32_t level, void* stream);

/* ---- batched solves ------------------------------------------------------------------ */

/* The system half of mg_pressure_solve_async: initialize (keeping x when
 * warm_start), labels, build_b, build_A per level, coarse labels and the
 * declared operator form, enqueued on `stream` with no host synchronisation
 * (mgpcg.py:63-94 with pressure_project.py:15-70).  mg_pcg_solve_async or a
 * batch solve then runs the PCG loop. */
MG_API int mg_pressure_setup_async(mg_plan_t* plan, const int32_t* cell_type, const float* v0, const float* v1,
                                   const float* v2, const float* phi, float p0, float scale_A, float scale_b,
                                   int32_t ghost_fluid, float gfm_clamp, int32_t warm_start, void* stream);

/* A batch: many plans' PCG loops advanced together, ONE kernel launch per
 * V-cycle stage (the sweeps of one level depth, the coarse blocks) and per CG
 * step for every instance, each launch driven by a table of (instance, block)
 * entries; every instance keeps its own reductions, alpha, beta, iteration
 * count and convergence test on the device, and the whole loop is one CUDA
 * graph that runs while any instance is unconverged.  No reference
 * counterpart: the reference solves one system per call (mgpcg.py:150-209).
 * Every plan must be bound and prepared in the label-uniform fused form
 * (mg_pressure_setup_async), with pre_post 2 and one storage type; each
 * instance's arithmetic is that of its own solve (the same blocks; the level
 * sweeps use the tiled ring kernel).  The batch's tables live in a workspace
 * the caller allocates (mg_batch_workspace_bytes) and binds. */
typedef struct mg_batch mg_batch_t;
MG_API int mg_batch_create(mg_plan_t* const* plans, int32_t n, mg_batch_t** out);
MG_API void mg_batch_destroy(mg_batch_t* batch);
MG_API int64_t mg_batch_workspace_bytes(const mg_batch_t* batch);
/* Uploads the tables into `workspace` (256-byte aligned) and builds the graph. */
MG_API int mg_batch_bind(mg_batch_t* batch, void* workspace, void* stream);
/* Solves every instance (its b, A as last set up; warm_start keeps each x);
 * MG_E_BADARG if an instance's plan was prepared to another shape since
 * mg_batch_create.  Results and mg_pcg_stats stay per plan. */
MG_API int mg_batch_solve_async(mg_batch_t* batch, const mg_solve_params_t* params, void* stream);
/* Kernels one batch launches before its loop and per loop pass. */
MG_API int mg_batch_launch_counts(const mg_batch_t* batch, int32_t* prologue, int32_t* body);

/* ---- allocation-free variant ------------------------------------------------------ */

/* Sum of a[i] * b[i] over the n cells with grid_type[i] == MG_FLUID, in FP64,
 * written to the DEVICE location *out (enqueued on `stream`, no synchronize).
 * No counterpart in the reference: it is the reference's reduce
 * (mgpcg.py:211-216) for callers that cannot allocate device memory - a host
 * whose engine owns every byte of device memory, a real-time step loop where
 * cudaMalloc/cudaFree would synchronise the device, or code without a solver
 * plan.  It allocates nothing: its scratch (64 KB of FP64 partial sums and a
 * counter) is a static array inside the library, held by every GPU that loads
 * it.  Each call looks that array up (cudaGetSymbolAddress) except while its
 * stream is being captured, when the address kept from an earlier call on the
 * device is used: the first call on a device must come before any stream
 * capture (else MG_E_CUDA).  n must be at most 33,554,432
 * (else MG_E_TOO_BIG).  Calls share the array: calls that overlap on the GPU
 * race; order them on one stream. */
MG_API int mg_reduce_static(const int8_t* grid_type, const float* a, const float* b, int64_t n, double* out,
                            void* stream);

/* Last CUDA error string recorded by this library (thread-local). */
MG_API const char* mg_last_error(void);

/* Library version (major * 10000 + minor * 100 + patch). */
MG_API int32_t mg_version(void);

#ifdef __cplusplus
}
#endif

#endif /* MGPCG_B200_H */
