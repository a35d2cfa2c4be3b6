/* hfgrid.h -- C ABI of the B200-native grid half of the hybrid fluid step.
 *
 * libhfgrid.so replaces, for one GPU, the grid solver of the reference engine
 * junwei-jiang/Hybrid-Fluid-Simulation (MPhysics/).  Two layers are exported:
 *
 *   hfg_solver_*  a handle-based mirror of CGridFluidSolver
 *                 (MPhysics/GridFluidSolver.h:17-137): same construction,
 *                 setters, update()/updateWithoutPressure()/solvePressure()
 *                 split and getters, with host buffers in and out;
 *   hfg_op_*      one entry point per reference "Invoker" stage of the step
 *                 (device pointers + a CUDA stream), the operator API the
 *                 parity tests drive.
 *
 * The reference-compatible MPhysicsAPI exports live in mphysics.h.
 *
 * Every function returns HFG_OK (0) or a negative status; hfg_last_error()
 * gives the message of the last failure on the calling thread.  No C++
 * exception crosses this boundary.  Arrays follow the reference layout:
 * cell-centred (nx*ny*nz, x fastest), face-centred X (nx+1)*ny*nz,
 * Y nx*(ny+1)*nz, Z nx*ny*(nz+1); particles as xyz triples; FP32 values,
 * uint8 cell markers (0 air, 1 fluid, 2 solid).
 */
#ifndef HFGRID_H
#define HFGRID_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define HFG_API __attribute__((visibility("default")))

enum {
  HFG_OK = 0,
  HFG_ERR_INVALID = -1,      /* bad argument */
  HFG_ERR_CUDA = -2,         /* CUDA runtime error */
  HFG_ERR_NOMEM = -3,        /* device allocation failed */
  HFG_ERR_STATE = -4,        /* call not valid in the solver's state */
  HFG_ERR_NOT_CONVERGED = -5,/* CG hit its iteration cap (stats still valid) */
  HFG_ERR_UNSUPPORTED = -6,
  HFG_ERR_TIMEOUT = -7
};

/* Advection solvers (GridFluidSolver.cpp:90-158). */
enum { HFG_ADV_SEMI_LAGRANGIAN = 0, HFG_ADV_PIC = 1, HFG_ADV_FLIP = 2, HFG_ADV_MIX_PIC_FLIP = 3 };
/* EAdvectionAccuracy (MPhysics/EnumType.h:12-17). */
enum { HFG_RK1 = 0, HFG_RK2 = 1, HFG_RK3 = 2 };
/* EPGTransferAlgorithm (MPhysics/EnumType.h:19-26). */
enum { HFG_P2GSUM = 0, HFG_G2PNEAREST = 1, HFG_LINEAR = 2, HFG_QUADRATIC = 3, HFG_CUBIC = 4 };
/* CG preconditioners: identity is the reference's "InvDia" (PressureSolver.cpp:12-15). */
enum { HFG_PRECOND_IDENTITY = 0, HFG_PRECOND_JACOBI = 1, HFG_PRECOND_MG = 2 };
/* CG stopping rules: the reference's sqrt(||r||_2) < tol (CuMatrixFreePCG.cpp:28,51),
 * or the relative ||r||_2 / ||b||_2 < tol. */
enum { HFG_TOL_REFERENCE = 0, HFG_TOL_RELATIVE = 1 };
/* ESamplingAlgorithm (EnumType.h:3-10) */
enum {
  HFG_SAMPLE_TRILINEAR = 0,
  HFG_SAMPLE_CATMULLROM = 1,
  HFG_SAMPLE_MONOCATMULLROM = 2,
  HFG_SAMPLE_CUBICBRIDSON = 3,
  HFG_SAMPLE_CLAMPCUBICBRIDSON = 4
};

typedef struct hfg_solver_s* hfg_solver_t;

typedef struct {
  int precond;            /* HFG_PRECOND_* (default identity) */
  int tol_mode;           /* HFG_TOL_* (default reference) */
  double tol;             /* default 1e-3 (CuMatrixFreePCG.h:28) */
  long long max_iter;     /* <0: N cells (PressureSolver.cpp:150-151) */
  int clamp_mode;         /* 1: clamp the first min(N,P) particles like the
                             reference launch (EulerParticlesTool.cu:880);
                             0: clamp every particle */
  int advect_scalars;     /* 1: also carry the colour / fluid-domain fields */
  int extrapolation_layers; /* default 1000 (GridFluidSolver.cpp:176) */
  int mg_levels;          /* multigrid levels for HFG_PRECOND_MG (0 = auto) */
  int mg_smooth;          /* smoothing sweeps per level (0 = default) */
  int mg_half;            /* multigrid storage: 0 FP32 on every level; 1 (default)
                             the coarse levels store their right-hand sides and
                             iterates in BF16; 2 as 1, and level 0's smoothing
                             iterates in BF16 too (grids with the marching
                             level-0 sweeps), the last sweep's output, which the
                             CG reads, staying FP32.  Arithmetic is FP32 on every
                             level and the CG's dot products FP64. */
  int report_divergence;  /* 1: measure the divergence residual of every projection
                             and recompute the solve's residual ||b - A x|| in FP64 */
  int sampling;           /* HFG_SAMPLE_* of the semi-Lagrangian advection (setSamplingAlg,
                             AdvectionSolver.cpp:21-24; default trilinear) */
  int pressure_fp64;      /* 1: accumulate the pressure iterate in FP64 and take the
                             gradient's differences in FP64 (the reference keeps
                             it in FP32, which bounds the divergence of the
                             projected field near 1e-4 of ||b|| on large grids) */
  int autotune;           /* 1: on the first Jacobi / identity solve of a grid size,
                             time the CG kernels at every candidate z-chunk length
                             and keep the fastest for that size (process wide;
                             hfg_tune_save / hfg_tune_load keep it across runs).
                             The reference's fixed launch shape is
                             EulerSolverTool.cu:650-656. */
  int sort_interval;      /* k > 0: at the start of every k-th particle step
                             after the first, reorder the particles by cell
                             (stable counting sort; velocities and carried
                             values follow), so that the substeps and the P2G
                             scatter keep touching neighbouring entries as the
                             flow mixes.  0 (default): the seeding order is
                             kept, as the reference keeps it.  The order of
                             hfg_solver_get_particles follows the sort.  Under
                             clamp_mode 1 with more particles than cells, the
                             first N particles (those the boundary fix
                             reaches) and the others are sorted each within
                             their own index range, so the fix reaches the
                             same particles. */
} hfg_options_t;

typedef struct {
  long long cg_iterations;
  double cg_residual;       /* final ||r||_2 (FP64 reduction on the GPU) */
  double cg_rhs_norm;       /* ||b||_2 */
  int cg_converged;
  int substeps;             /* CFL substeps of the last particle advection */
  int extrapolation_layers; /* deepest layer filled by the last extrapolation */
  double sim_time;
  long long num_particles;
  long long fluid_cells;
  float stage_ms[8];        /* boundaries, advection, forces, markers, rhs,
                               cg, gradient, extrapolation (when timing on) */
  double divergence_l2;     /* with report_divergence: ||b(u)||_2 over the fluid
                               cells after the projection (b as the RHS: -div u
                               plus the solid-face terms, 1/s) */
  double divergence_max;    /* max |b(u)| over the fluid cells after the projection */
  double cg_true_residual;  /* with report_divergence: ||b - A x||_2 of the last solve,
                               recomputed in FP64 on the GPU after it (-1 otherwise) */
  float particle_ms[3];     /* when timing on: device time of the particle transfers of
                               the advection stage: G2P, the substep launches (summed
                               over their chunks), P2G with its normalisation */
} hfg_stats_t;

/* ---- library ---------------------------------------------------------- */
HFG_API int hfg_init(int device);
HFG_API const char* hfg_last_error(void);
/* Self-test of the bounded waits every TMA-fed and cooperative kernel uses
 * (no reference counterpart): an mbarrier wait of wait_ms on bytes no copy
 * delivers, and a grid barrier missing one arrival (its own 1 s limit), both
 * on the current device.  Each must give up and report it (*..._timed_out =
 * 1), leaving the context usable; no fault is involved. */
HFG_API int hfg_selftest_bounded_waits(int wait_ms, int* mbarrier_timed_out, int* grid_barrier_timed_out);
/* Failure injection on the host (no reference counterpart): the after-th
 * device allocation of the library from now on fails as cudaMalloc would
 * (HFG_ERR_NOMEM), without calling it.  0 disarms. */
HFG_API int hfg_test_inject_alloc_failure(int after);
/* The launch shapes measured by the autotuner (option autotune), as a text
 * file of "cg<0 direction | 1 update> px ny nz zchunk" lines; loading adds to
 * the table and sets *entries.  No reference counterpart. */
HFG_API int hfg_tune_save(const char* path);
HFG_API int hfg_tune_load(const char* path, int* entries);
HFG_API const char* hfg_version(void);
HFG_API void hfg_default_options(hfg_options_t* o);

/* ---- CGridFluidSolver mirror ----------------------------------------- */
/* CGridFluidSolver(dt, res, origin, spacing)  GridFluidSolver.cpp:32-41,161-196 */
HFG_API int hfg_solver_create(float dt, const int res[3], const float origin[3], const float spacing[3],
                              hfg_solver_t* out);
HFG_API int hfg_solver_destroy(hfg_solver_t s);
/* addSolidBoundary / generateSolidSDFFromCLDGrid(.., vel)  GridFluidSolver.cpp:203-206,557-562 */
HFG_API int hfg_solver_add_solid_boundary(hfg_solver_t s, const float* sdf, const float vel[3]);
/* Velocity of boundary `index` from the next step on (translation += -dt*vel
 * per step, Boundary.cpp:124-127); the per-frame rigid-boundary update of the
 * reference viewer loop (MPhysics.cpp:52-65 transformRigidBoundary). */
HFG_API int hfg_solver_set_boundary_velocity(hfg_solver_t s, int index, const float vel[3]);
/* addExternalForce  GridFluidSolver.cpp:198-201 */
HFG_API int hfg_solver_add_external_force(hfg_solver_t s, const float force[3]);
/* setVelocityField / setFluidDomainField / setColorField  GridFluidSolver.cpp:208-229 */
HFG_API int hfg_solver_set_velocity_field(hfg_solver_t s, const float* x, const float* y, const float* z);
HFG_API int hfg_solver_set_fluid_domain_field(hfg_solver_t s, const float* d);
HFG_API int hfg_solver_set_color_field(hfg_solver_t s, const float* x, const float* y, const float* z);
/* generateFluidDomainFromBBox  GridFluidSolver.cpp:551-555 */
HFG_API int hfg_solver_generate_fluid_domain_from_bbox(hfg_solver_t s, const float mn[3], const float mx[3]);
/* setAdvectionSolver (SemiLagrangian / PIC / FLIP / MixPICAndFLIP)  GridFluidSolver.cpp:90-158 */
HFG_API int hfg_solver_set_advection(hfg_solver_t s, int kind, int accuracy, int transfer_alg, float cfl,
                                     float mixing);
/* CEulerParticles::generateParticlesInFluid with a seeded counter-based stream
 * in place of rand()  EulerParticles.cpp:140-179 */
HFG_API int hfg_solver_seed_particles(hfg_solver_t s, int per_cell, unsigned long long seed);
/* CEulerParticles::setParticlesPos / setParticlesVel (host arrays of 3n)  EulerParticles.cpp:125-133 */
HFG_API int hfg_solver_set_particles(hfg_solver_t s, const float* pos, const float* vel, long long n);
HFG_API int hfg_solver_set_options(hfg_solver_t s, const hfg_options_t* o);
HFG_API int hfg_solver_enable_timing(hfg_solver_t s, int on);
/* update / updateWithoutPressure / solvePressure  GridFluidSolver.cpp:336-357 */
HFG_API int hfg_solver_update(hfg_solver_t s);
HFG_API int hfg_solver_update_steps(hfg_solver_t s, int steps);
HFG_API int hfg_solver_update_without_pressure(hfg_solver_t s);
HFG_API int hfg_solver_solve_pressure(hfg_solver_t s);
/* getVelocityField (which=0) / getVelocityFieldBeforePressure (which=1)  GridFluidSolver.cpp:302-324 */
HFG_API int hfg_solver_get_velocity_field(hfg_solver_t s, int which, float* x, float* y, float* z);
HFG_API int hfg_solver_get_fluid_domain_field(hfg_solver_t s, float* d);
HFG_API int hfg_solver_get_color_field(hfg_solver_t s, float* x, float* y, float* z);
/* getPressureSolver()->getMarkers() / getConstVectorx()  PressureSolver.h:25-31 */
HFG_API int hfg_solver_get_markers(hfg_solver_t s, uint8_t* markers);
HFG_API int hfg_solver_get_pressure(hfg_solver_t s, float* p);
/* getSolidSDFField (the total solid marker field)  GridFluidSolver.cpp:292-295 */
HFG_API int hfg_solver_get_solid_sdf(hfg_solver_t s, float* sdf);
HFG_API int hfg_solver_get_solid_vel_field(hfg_solver_t s, float* x, float* y, float* z);
/* generateCurFluidSDF + getFluidSDFField: the layered fluid SDF of the current
 * fluid-domain field (GridFluidSolver.cpp:571-591, EulerSolverTool.cu:324-406) */
HFG_API int hfg_solver_get_fluid_sdf(hfg_solver_t s, float* sdf);
/* generateCurFluidDensity + getFluidDensityField (N floats: 1 fluid, 0.2 at the
 * surface, 0 elsewhere)  GridFluidSolver.cpp:297-300,593-613 */
HFG_API int hfg_solver_get_fluid_density(hfg_solver_t s, float* density);
/* mixVelFieldWithOthers  GridFluidSolver.cpp:615-642: blends another face
 * velocity field into the buffer the step in progress writes (call it between
 * hfg_solver_update_without_pressure and hfg_solver_solve_pressure), weighted by
 * the two cell densities.  DEVICE pointers, like the reference's fields. */
HFG_API int hfg_solver_mix_vel_field_with_others(hfg_solver_t s, const float* vx, const float* vy, const float* vz,
                                                 const float* others_density, const float* fluid_density);
/* transferFluidVelField2Particles  GridFluidSolver.cpp:644-670: G2P from the
 * current velocity field; DEVICE pointers (pos, vel: 3n floats). */
HFG_API int hfg_solver_transfer_vel_to_particles(hfg_solver_t s, const float* pos, long long n, int alg, float* vel);
HFG_API long long hfg_solver_num_particles(hfg_solver_t s);
HFG_API int hfg_solver_get_particles(hfg_solver_t s, float* pos, float* vel);
/* Reorder the particles by cell now: stable (particles of one cell keep
 * their relative order), velocities and carried values follow; under
 * clamp_mode 1 with more particles than cells the first N and the rest are
 * sorted each within its own range (see sort_interval).  No reference
 * counterpart (the reference keeps the seeding order). */
HFG_API int hfg_solver_sort_particles(hfg_solver_t s);
/* Host mirror of the particles (an extension; the reference's viewer calls
 * copyEulerParticlesPos/VelToCPU after every update, MPhysicsAPI.h).  While a
 * mirror is set, every update also copies the particle positions and
 * velocities into pos and vel (HOST buffers of 3 * capacity floats, either may
 * be NULL), as the step leaves them: each copy runs on a second stream from
 * the point where the step is done with that array (the velocities after the
 * grid-to-particle update, the positions after the substeps), overlapped with
 * the rest of the step; the update returns after both have landed.  Buffers allocated with
 * cudaHostAlloc or registered with cudaHostRegister let the copy overlap; other
 * host memory is copied correctly but not overlapped.  An update with more
 * particles than capacity fails with HFG_ERR_INVALID.  pos = vel = NULL
 * removes the mirror. */
HFG_API int hfg_solver_set_particle_mirror(hfg_solver_t s, float* pos, float* vel, long long capacity);
HFG_API int hfg_solver_get_stats(hfg_solver_t s, hfg_stats_t* st);
HFG_API int hfg_solver_get_grid(hfg_solver_t s, int res[3], float origin[3], float spacing[3]);
/* The CUDA stream every kernel of this solver runs on (cudaStream_t). */
HFG_API void* hfg_solver_stream(hfg_solver_t s);
/* Launches of this library's kernels since creation (counted on the host). */
HFG_API long long hfg_solver_launch_count(hfg_solver_t s);
HFG_API int hfg_solver_synchronize(hfg_solver_t s);
/* Times `iters` back-to-back CG iterations (both kernels, no host round trip)
 * on the system of the last pressure solve with CUDA events on the solver's
 * stream; writes the mean milliseconds per iteration.  Overwrites the pressure
 * of the last step (the next update recomputes it). */
HFG_API int hfg_solver_time_cg(hfg_solver_t s, int iters, float* ms_per_iter);

/* ---- operators (device pointers, asynchronous on `stream` unless noted) -- */
/* buildFluidMarkersInvoker(solidSDF, particles)  EulerParticlesTool.cu:366-411 */
HFG_API int hfg_op_markers_from_particles(const int res[3], const float origin[3], const float spacing[3],
                                          const float* solid_sdf, const float* pos, long long n, uint8_t* markers,
                                          void* stream);
/* statisticalFluidDensity counts  EulerParticlesTool.cu:27-46,413-441 */
HFG_API int hfg_op_bin_counts(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                              long long n, unsigned int* counts, void* stream);
/* buildFluidMarkersInvoker(solidSDF, fluidSDF)  EulerSolverTool.cu:629-648 */
HFG_API int hfg_op_markers_from_sdf(const int res[3], const float* solid_sdf, const float* fluid_sdf,
                                    uint8_t* markers, void* stream);
/* buildPressureFdmMatrixAInvoker  EulerSolverTool.cu:650-664 ([diag,+x,+y,+z] per cell) */
HFG_API int hfg_op_build_matrix_a(const int res[3], const float spacing[3], float dt, const uint8_t* markers,
                                  float* A, void* stream);
/* fdmMatrixVectorMulInvoker  EulerSolverTool.cu:706-720 */
HFG_API int hfg_op_apply_a(const int res[3], const float spacing[3], float dt, const uint8_t* markers,
                           const float* x, float* y, void* stream);
/* divergence + buildPressureVectorbInvoker  PressureSolver.cpp:223-227 */
HFG_API int hfg_op_build_rhs(const int res[3], const float spacing[3], const float* vx, const float* vy,
                             const float* vz, const float* svx, const float* svy, const float* svz,
                             const uint8_t* markers, float* b, void* stream);
/* the projection of CPressureSolver::solvePressure after the markers
 * (PressureSolver.cpp:210-233): RHS, CG, pressure gradient in place on v.
 * Blocks until the solve finishes; stats (3 doubles: iterations, ||r||, ||b||) optional. */
HFG_API int hfg_op_project(const int res[3], const float spacing[3], float dt, const uint8_t* markers, float* vx,
                           float* vy, float* vz, const float* svx, const float* svy, const float* svz, int precond,
                           int tol_mode, double tol, long long max_iter, float* p, double* stats, void* stream);
/* extrapolatingDataInvoker on a face-centred field  EulerSolverTool.cu:904-969 (blocks) */
HFG_API int hfg_op_extrapolate_fc(const int res[3], float* vx, float* vy, float* vz, int layers, void* stream);
/* extrapolatingDataInvoker on one cell-centred scalar field  EulerSolverTool.cu:812-842 (blocks) */
HFG_API int hfg_op_extrapolate_cc(const int res[3], float* f, int layers, void* stream);
/* sampleFaceCenteredVectorFieldInvoker at n points (trilinear)  FieldMathTool.cu:894-1002 */
HFG_API int hfg_op_sample_fc(const int res[3], const float origin[3], const float spacing[3], const float* vx,
                             const float* vy, const float* vz, const float* pos, long long n, float* out,
                             void* stream);
/* sampleCellCenteredScalarFieldInvoker at n points (trilinear)  FieldMathTool.cu:526-573 */
HFG_API int hfg_op_sample_cc(const int res[3], const float origin[3], const float spacing[3], const float* f,
                             const float* pos, long long n, float* out, void* stream);
/* sampleCellCenteredScalarFieldInvoker with an ESamplingAlgorithm (HFG_SAMPLE_*)
 * FieldMathTool.cu:470-573 (cubic kernels :106-173, EulerMathTool.cu:134-240) */
HFG_API int hfg_op_sample_cc_ex(const int res[3], const float origin[3], const float spacing[3], const float* f,
                                const float* pos, long long n, int sampling, float* out, void* stream);
/* sampleFaceCenteredVectorFieldInvoker with an ESamplingAlgorithm; out 3n floats
 * FieldMathTool.cu:783-1128 */
HFG_API int hfg_op_sample_fc_ex(const int res[3], const float origin[3], const float spacing[3], const float* vx,
                                const float* vy, const float* vz, const float* pos, long long n, int sampling,
                                float* out, void* stream);
/* tranferFCVField2ParticlesInvoker  EulerParticlesTool.cu:805-868 */
HFG_API int hfg_op_g2p_fc(const int res[3], const float origin[3], const float spacing[3], const float* vx,
                          const float* vy, const float* vz, const float* pos, long long n, int alg, float* out,
                          void* stream);
/* tranferCCSField2ParticlesInvoker  EulerParticlesTool.cu:713-741 */
HFG_API int hfg_op_g2p_cc(const int res[3], const float origin[3], const float spacing[3], const float* f,
                          const float* pos, long long n, int alg, float* out, void* stream);
/* tranferParticles2FCVFieldInvoker (normalised)  EulerParticlesTool.cu:601-711; weights optional */
HFG_API int hfg_op_p2g_fc(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                          const float* vel, long long n, int alg, float* vx, float* vy, float* vz, float* wx,
                          float* wy, float* wz, void* stream);
/* tranferParticles2CCSFieldInvoker  EulerParticlesTool.cu:443-496 */
HFG_API int hfg_op_p2g_cc(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                          const float* val, long long n, int alg, int normalize, float* f, float* w, void* stream);
/* CEulerParticles::advectParticlesInVelField  EulerParticles.cpp:231-325 (blocks; returns substeps) */
HFG_API int hfg_op_advect_particles(const int res[3], const float origin[3], const float spacing[3],
                                    const float* vx, const float* vy, const float* vz, float* pos, long long n,
                                    float dt, float cfl, int accuracy, int clamp_mode, int* substeps, void* stream);
/* CSemiLagrangian::advect (face-centred)  SemiLagrangian.cpp:169-186 */
HFG_API int hfg_op_sl_advect_fc(const int res[3], const float origin[3], const float spacing[3], const float* ix,
                                const float* iy, const float* iz, const float* vx, const float* vy, const float* vz,
                                float dt, int accuracy, float* ox, float* oy, float* oz, void* stream);
/* CSemiLagrangian::advect (cell-centred scalar)  SemiLagrangian.cpp:135-150 */
HFG_API int hfg_op_sl_advect_cc(const int res[3], const float origin[3], const float spacing[3], const float* in,
                                const float* vx, const float* vy, const float* vz, float dt, int accuracy, float* out,
                                void* stream);
/* CSemiLagrangian::advect with the advection's ESamplingAlgorithm for every
 * back-trace and final sample  SemiLagrangian.cpp:135-347 */
HFG_API int hfg_op_sl_advect_fc_ex(const int res[3], const float origin[3], const float spacing[3], const float* ix,
                                   const float* iy, const float* iz, const float* vx, const float* vy,
                                   const float* vz, float dt, int accuracy, int sampling, float* ox, float* oy,
                                   float* oz, void* stream);
HFG_API int hfg_op_sl_advect_cc_ex(const int res[3], const float origin[3], const float spacing[3], const float* in,
                                   const float* vx, const float* vy, const float* vz, float dt, int accuracy,
                                   int sampling, float* out, void* stream);
/* buildFluidSDFInvoker  EulerSolverTool.cu:760-785 (layers = the reference's
 * vExtrapolationDistance; blocks) */
HFG_API int hfg_op_build_fluid_sdf(const int res[3], const float* domain, float* sdf, int layers, void* stream);
/* mixFieldWithDensityInvoker (cell grid of n entries / face grids of res):
 * b := (wa a + wb b) / (wa + wb) where wa + wb > FLT_EPSILON, in place
 * HybridSimulatorMixFieldWithDensity.cu:6-265 */
HFG_API int hfg_op_mix_field_with_density_cc(long long n, const float* a, float* b, const float* wa, const float* wb,
                                             void* stream);
HFG_API int hfg_op_mix_field_with_density_fc(const int res[3], const float* ax, const float* ay, const float* az,
                                             float* bx, float* by, float* bz, const float* wa, const float* wb,
                                             void* stream);
/* mixParitcleVelWithPICAndFLIPInvoker  HybridSimulatorMixParitcleVelWithPICAndFLIP.cu:5-88 */
HFG_API int hfg_op_mix_particle_vel_pic_flip(const float* pic, const float* flip, const float* dist, long long n,
                                             float cell, float g_rate, float gf_rate, float f_rate, float p_rate,
                                             float* predict, void* stream);
/* buildFluidDensityInvoker  EulerSolverTool.cu:408-448,787-810; solid_sdf < 0 inside solids */
HFG_API int hfg_op_build_fluid_density(const int res[3], const float* domain, const float* solid_sdf, float* out,
                                       void* stream);
/* buildFluidOutsideSDFInvoker / buildFluidInsideSDFInvoker of the hybrid
 * coupler  HybridSimulatorBuildSDF.cu:4-146,177-238: the distance in cells
 * from the surface cells (density 0.2) into the air (outside) or the fluid
 * (inside) of a fluid density field (hfg_op_build_fluid_density), grown over
 * `distance` sweeps as the reference's invokers do (it passes 1000); solids
 * (solid_sdf < 0) and the other side hold 0, cells no sweep reaches UNKNOWN
 * (FLT_MAX), negative values end as 0.  distance 0 only clamps `out`'s
 * negative values to 0.  0 <= distance <= 100000.  Blocks (one host read per
 * sweep). */
HFG_API int hfg_op_build_fluid_outside_sdf(const int res[3], const float* density, const float* solid_sdf, float* out,
                                           int distance, void* stream);
HFG_API int hfg_op_build_fluid_inside_sdf(const int res[3], const float* density, const float* solid_sdf, float* out,
                                          int distance, void* stream);
/* buildMixedFluidOutsideSDFInvoker  HybridSimulatorBuildSDF.cu:139-175,240-266:
 * at a cell of grid density 0.2, 0.5 - mixed density (negative -> 0);
 * elsewhere grid_outside_sdf */
HFG_API int hfg_op_build_mixed_fluid_outside_sdf(const int res[3], const float* grid_density,
                                                 const float* mixed_density, const float* grid_outside_sdf,
                                                 float* out, void* stream);
/* generateFluidDomainFromBBoxInvoker  EulerSolverTool.cu:989-1013 */
HFG_API int hfg_op_fluid_domain_from_bbox(const int res[3], const float origin[3], const float spacing[3],
                                          const float mn[3], const float mx[3], float* out, void* stream);
/* particle seeding (see hfg_solver_seed_particles); pos may be NULL to count only (blocks) */
HFG_API int hfg_op_seed_particles(const int res[3], const float origin[3], const float spacing[3],
                                  const float* fluid_sdf, const float* solid_sdf, int per_cell,
                                  unsigned long long seed, float* pos, long long capacity, long long* count,
                                  void* stream);

/* ---- analytic solids and the scene server -------------------------------
 * Neither has a counterpart in the reference, whose solids come from meshes
 * voxelised by a D3D11 compute shader (BoundaryHelper.cpp:48-121) and whose
 * simulators step one after another in one thread (MPhysics.cpp:19-25). */

enum { HFG_SOLID_WALLS = 0, HFG_SOLID_SPHERE = 1, HFG_SOLID_BOX = 2 };
/* addSolidBoundary with the SDF evaluated on the device at the cell centres
 * (FP64, stored FP32): walls = everything outside the inner box
 * [origin + h, origin + (n - 1) h]; sphere params (cx, cy, cz, r); box params
 * (cx, cy, cz, sx, sy, sz) with full side lengths. */
HFG_API int hfg_solver_add_analytic_solid(hfg_solver_t s, int type, const double params[6], const float vel[3]);

/* A seeded dam break on the unit cube: walls, up to 4 static spheres, fluid
 * in the cells whose centre lies below fluid_max on every axis, per_cell
 * particles per fluid cell, PIC/FLIP mix, `steps` calls of update(). */
typedef struct {
  int res[3];
  float dt;
  float fluid_max[3];
  int n_spheres;
  float spheres[4][4];    /* centre x, y, z and radius */
  int per_cell;
  unsigned long long seed;
  float cfl;
  float mixing;           /* MixingCoefficient (PIC weight) */
  int steps;
  int keep_particles;     /* keep the final positions for hfg_server_particles */
  hfg_options_t options;
} hfg_scene_desc_t;

typedef struct {
  int status;             /* 0 queued, 1 running, 2 done, negative: the HFG_ERR_* it failed with */
  int steps_done;
  long long cells, particles, footprint_bytes;
  double queue_ms;        /* submission -> admission */
  double run_ms;          /* admission -> completion */
  double step_ms_p50, step_ms_max;
  hfg_stats_t last;       /* statistics of the last step */
} hfg_request_info_t;

typedef struct {
  long long submitted, completed, failed, rejected;
  double step_ms_p50, step_ms_p99;        /* over every step of every completed request */
  double request_ms_p50, request_ms_p99;  /* submission -> completion */
  double cell_steps;                      /* sum over completed requests of cells x steps */
  double wall_s;                          /* first submission -> last completion */
  long long peak_bytes, budget_bytes;
  int peak_running, slots;
} hfg_server_stats_t;

typedef struct hfg_server_s* hfg_server_t;

/* Device bytes a scene of this size holds while resident (the admission
 * estimate of the server); host-only arithmetic. */
HFG_API int hfg_scene_bytes(const int res[3], long long particles, int boundaries, int precond, long long* bytes);
/* Upper bound of the particles a dam-break description seeds (fluid cells of
 * the bbox, before solids are removed, x per_cell); host-only. */
HFG_API int hfg_scene_particles_bound(const hfg_scene_desc_t* d, long long* particles);

/* Continuous-batching server: `slots` worker threads on `device`, each owning
 * the scene it runs (grids and particles resident on the device for all of
 * its steps) on its own stream, so the steps of different scenes overlap on
 * the GPU.  A queued request is admitted as soon as a slot is free and its
 * footprint fits the remaining byte budget; smaller requests may pass a head
 * that does not fit, unless the head has waited longer than 1 s.  A request
 * whose footprint exceeds the whole budget is rejected at submission. */
HFG_API int hfg_server_create(int device, int slots, long long budget_bytes, hfg_server_t* out);
HFG_API int hfg_server_submit(hfg_server_t srv, const hfg_scene_desc_t* desc, long long* id);
HFG_API int hfg_server_info(hfg_server_t srv, long long id, hfg_request_info_t* info);  /* non-blocking */
HFG_API int hfg_server_wait(hfg_server_t srv, long long id, hfg_request_info_t* info);  /* until done */
/* per-step latencies (ms) of a request; returns the count written */
HFG_API int hfg_server_step_times(hfg_server_t srv, long long id, double* ms, int capacity);
/* final particle positions (3n floats) of a done request with keep_particles */
HFG_API int hfg_server_particles(hfg_server_t srv, long long id, float* pos, long long capacity);
HFG_API int hfg_server_drain(hfg_server_t srv);  /* waits until every submitted request is done */
HFG_API int hfg_server_stats(hfg_server_t srv, hfg_server_stats_t* st);
HFG_API int hfg_server_destroy(hfg_server_t srv);  /* drains first */

/* Batched lockstep stepping (no reference counterpart; the reference steps
 * its simulators one after another, MPhysics.cpp:19-25): n dam-break scenes
 * (their `steps` field is ignored) stay resident on `device` and advance
 * together.  Per step the CFL substeps of all scenes run in one launch per
 * substep (each scene keeping its own CFL state), the launches of a step
 * replayed from a CUDA graph; the other stages run on the scenes' own
 * streams, issued by `threads` host threads.  A scene's results are those it
 * has alone, up to the order of the P2G float atomics. */
typedef struct hfg_batch_s* hfg_batch_t;
HFG_API int hfg_batch_create(int device, const hfg_scene_desc_t* scenes, int n, int threads, hfg_batch_t* out);
/* `steps` steps of every scene; ms (optional) receives each step's host wall time */
HFG_API int hfg_batch_step(hfg_batch_t b, int steps, double* ms);
HFG_API int hfg_batch_scene_stats(hfg_batch_t b, int scene, hfg_stats_t* st);
HFG_API int hfg_batch_particles(hfg_batch_t b, int scene, float* pos, long long capacity);
HFG_API int hfg_batch_destroy(hfg_batch_t b);

/* hfg_op_p2g_fc without any device allocation.  This entry point has no
 * counterpart in the reference.  It is for callers that may not allocate
 * device memory at call time (a fixed-memory real-time loop, or a host whose
 * own allocator reserves the whole device and forbids other allocations): the
 * accumulators live in one 8 MiB array inside libhfgrid.so instead of coming
 * from the stream-ordered allocator.
 *   - Limit: the three face grids together hold at most 1,048,576 faces
 *     ((nx+1)ny nz + nx(ny+1)nz + nx ny(nz+1); 64^3 cells fit).  Larger grids
 *     return HFG_ERR_INVALID with a message; use hfg_op_p2g_fc for them.
 *   - Every call, on every stream and thread of the process, uses the same
 *     array on a device: calls that overlap in time on one device race and
 *     give wrong results.  Serialise them.  Each call zeroes the accumulators
 *     it uses before scattering, so nothing has to be cleared in advance.
 *   - Every call looks up the array's address on the caller's current
 *     device.  With lazy module loading (the CUDA 12 default) the first call
 *     on a device loads the library's device code there, which reserves the
 *     8 MiB array and the code itself.  Make that first call before any
 *     stream capture begins, and before the host's own allocator reserves
 *     the rest of the device's memory.
 * Arguments, results and blocking behaviour are those of hfg_op_p2g_fc. */
HFG_API int hfg_op_p2g_fc_static(const int res[3], const float origin[3], const float spacing[3], const float* pos,
                                 const float* vel, long long n, int alg, float* vx, float* vy, float* vz, float* wx,
                                 float* wy, float* wz, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* HFGRID_H */
