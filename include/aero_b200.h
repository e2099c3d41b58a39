/*
 * aero_b200.h -- C ABI of the aero_b200 lattice Boltzmann engine (sm_100a).
 *
 * The engine replaces the per-step hot path of the Aero wind-tunnel solver:
 * the body of Solver._step / Solver3D._step (aero/lbm/solver.py:276-464,
 * aero/lbm/solver3d.py:325-541) and the kernels it calls.  Plain C types
 * only; every function returns AERO_OK (0) or a negative AERO_ERR_* code and
 * leaves a message for aero_last_error().
 *
 * Memory ownership: the caller allocates ONE device workspace of
 * aero_workspace_size() bytes (e.g. a torch uint8 tensor) and binds it; the
 * library never allocates or frees device memory for a lattice.  Bulk state
 * I/O (populations, outlet state, scalar) goes through caller-owned DEVICE
 * buffers in the reference layout.  Calls are ordered on the caller's CUDA
 * stream (a cudaStream_t passed as void*; NULL = legacy default stream).
 * A handle is not thread-safe: one host thread per handle.
 */
#ifndef AERO_B200_H
#define AERO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define AERO_ABI_VERSION 3

#if defined(__GNUC__)
#define AERO_API __attribute__((visibility("default")))
#else
#define AERO_API
#endif

enum {
  AERO_OK = 0,
  AERO_ERR_INVALID = -1,     /* bad argument or parameter combination */
  AERO_ERR_CUDA = -2,        /* a CUDA call failed */
  AERO_ERR_STATE = -3,       /* call out of order (e.g. step before bind) */
  AERO_ERR_UNSUPPORTED = -4, /* option outside the engine (IBM, SEM inlet, ...) */
  AERO_ERR_CAPACITY = -5     /* a fixed capacity is exceeded: force history full (read it
                                first), or a link list too long for a fixed scratch */
};

enum { AERO_STORE_F32 = 0, AERO_STORE_F64 = 1, AERO_STORE_F16 = 2, AERO_STORE_BF16 = 3 };
enum { AERO_BGK = 0, AERO_TRT = 1, AERO_MRT = 2 };
enum { AERO_INLET_NONE = 0, AERO_INLET_VELOCITY = 1, AERO_INLET_PRESSURE = 2 };
enum { AERO_OUTLET_NONE = 0, AERO_OUTLET_CONVECTIVE = 1, AERO_OUTLET_ZEROGRADIENT = 2, AERO_OUTLET_PRESSURE = 3 };
enum { AERO_WALL_NONE = 0, AERO_WALL_SLIP = 1, AERO_WALL_NOSLIP = 2, AERO_WALL_MOVING = 3 };
enum { AERO_LES_SMAGORINSKY = 0, AERO_LES_WALE = 1 };

/* Solver options.  Field meanings follow the keyword arguments of the
 * reference constructors (aero/lbm/solver.py:75-116,
 * aero/lbm/solver3d.py:71-119). */
typedef struct AeroParams {
  int32_t abi_version;      /* AERO_ABI_VERSION */
  int32_t dims;             /* 2 = D2Q9, 3 = D3Q19 */
  int32_t nx, ny, nz;       /* nz = 1 in 2D */
  int32_t storage;          /* AERO_STORE_* */
  int32_t collision;        /* AERO_BGK / AERO_TRT / AERO_MRT */
  int32_t inlet_bc;         /* AERO_INLET_* */
  int32_t outlet_bc;        /* AERO_OUTLET_* */
  int32_t wall_bc;          /* AERO_WALL_* */
  int32_t streamwise_open;  /* 1: inlet/outlet active; 0: streamwise periodic (3D) */
  int32_t les;              /* Smagorinsky/WALE eddy viscosity (ignored by MRT, as in the reference) */
  int32_t les_model;        /* AERO_LES_* */
  int32_t van_driest;       /* damp the LES constant with |phi| (needs phi) */
  int32_t bouzidi;          /* interpolated bounce-back with per-link q */
  int32_t thermal;          /* passive scalar lattice */
  int32_t buoyancy;         /* Boussinesq forcing of the flow by the scalar */
  int32_t scalar_reduced;   /* 0: D2Q9/D3Q19 scalar (reference); 1: D2Q5/D3Q7 */
  int32_t sponge_thickness; /* outlet sponge planes (0 = off) */
  int32_t hist_capacity;    /* steps of force history kept on the device (0 = 4096) */
  double omega, u0, rho0, rho_in, rho_out;
  double inlet_perturbation, trt_lambda, sponge_strength;
  double les_cs, van_driest_A;
  double wall_velocity_top, wall_velocity_bottom;
  double body_force[3];     /* (fx, fy, fz); 3D only */
  double alpha_T, T_hot, T_cold, g_gravity, beta, T_ref;
  double center[3];         /* moment reference point (x, y, z): mean solid cell */
  int32_t recycling;        /* 3D streamwise "recycling": the inlet plane is the rescaled
                               equilibrium of plane x = nx-2 (needs streamwise_open = 0) */
  int32_t inflow_field;     /* velocity inlet driven by per-step fields uploaded with
                               aero_set_inflow: 1 = synthetic inflow (transverse velocities),
                               2 = SEM fluctuations (u', v', w'; 3D) */
  int32_t inflow_ring;      /* steps of inflow fields held on the device (0 = 64) */
  int32_t layout;           /* AERO_LAYOUT_AB: two population buffers; AERO_LAYOUT_AA: one buffer
                               updated in place (AA pattern; half the population memory) */
} AeroParams;

enum { AERO_LAYOUT_AB = 0, AERO_LAYOUT_AA = 1 };

typedef struct AeroLattice AeroLattice;

/* Number of per-step force values returned by aero_read_forces. Layout of one
 * step: Fx Fy Fz | pressure Fx Fy Fz | viscous Fx Fy Fz | Mx My Mz, raw
 * lattice units (forces.py:15-127, forces3d.py:8-131). */
#define AERO_FORCE_VALUES 12

/* Creates a handle and validates the options.  Replaces the option handling
 * and backend selection of Solver.__init__ (solver.py:143-203,
 * solver3d.py:136-221). */
AERO_API int aero_create(const AeroParams *params, AeroLattice **out);

/* Geometry on the host: solid (nz*ny*nx bytes, 1 = solid), the surface link
 * list (n_links rows of [i, (z,) y, x] int32, as built by
 * build_surface_links(_3d), boundary.py:232-280, boundary3d.py:279-329) with
 * its q values (float32), and phi (float64 per cell, only read when
 * van_driest is set; may be NULL).  Must precede aero_workspace_size. */
AERO_API int aero_set_geometry(AeroLattice *lat, const uint8_t *solid, const int32_t *links, const float *q,
                      int64_t n_links, const double *phi);

/* Device bytes the lattice needs; the caller allocates them. */
AERO_API int aero_workspace_size(const AeroLattice *lat, uint64_t *bytes);

/* Binds the caller's device workspace (256-byte aligned) and uploads the
 * geometry tables.  Replaces the array set-up of solver.py:205-257. */
AERO_API int aero_bind_workspace(AeroLattice *lat, void *device_ptr, uint64_t bytes, void *stream);

/* Sets the solver state from caller DEVICE buffers in the reference layout:
 * f (Q, nz, ny, nx) float64, f_outlet_prev (Q, [nz,] ny) float64 (NULL keeps
 * the current one), g (Qg, nz, ny, nx) float64 (thermal only, NULL keeps),
 * and the number of steps already taken.  Replaces the initial-state code of
 * solver.py:218-227 / solver3d.py:239-247 and load_checkpoint
 * (solver.py:688-709). */
AERO_API int aero_set_state(AeroLattice *lat, const double *f, const double *f_outlet_prev, const double *g,
                   int64_t step_count, void *stream);

/* Sets the state to the equilibrium of macroscopic fields, built on the
 * device: f = feq(rho, u) at every cell (solids included, as the
 * reference's initial state, solver.py:218-227 / solver3d.py:239-247, and
 * as a caller's `s.f = compute_feq(...)` assignment), the convective outlet
 * state = the x = nx-1 column of that f, and the scalar g_i = w_i T.  rho,
 * ux, uy, uz, T are caller DEVICE arrays of nz*ny*nx float64 values in the
 * reference's (z, y, x) order, or NULL for the uniform value (rho0, u0, 0,
 * 0, T_ref); uz only in 3D, T only with a scalar.  feq is evaluated in FP64
 * with the operations of compute_feq(_3d) (d2q9.py:66-89,
 * d3q19.py:105-129), so the state equals aero_set_state of the same f.
 * Moves one field per cell where aero_set_state moves Q populations. */
AERO_API int aero_set_equilibrium(AeroLattice *lat, const double *rho, const double *ux, const double *uy,
                                  const double *uz, const double *T, int64_t step_count, void *stream);

/* Writes the current state into caller DEVICE buffers (same layouts; any
 * pointer may be NULL).  The state is the reference's self.f after the last
 * step. */
AERO_API int aero_get_state(AeroLattice *lat, double *f, double *f_outlet_prev, double *g, void *stream);

/* Advances n_steps steps (Solver._step, solver.py:276-464; Solver3D._step,
 * solver3d.py:325-541), forces included.  Asynchronous on the stream. */
AERO_API int aero_step(AeroLattice *lat, int64_t n_steps, void *stream);

/* Copies the force values of the steps taken since the previous read into
 * host memory (max_steps * AERO_FORCE_VALUES doubles) and synchronises the
 * stream.  *n_out receives the number of steps copied. */
AERO_API int aero_read_forces(AeroLattice *lat, double *out, int64_t max_steps, int64_t *n_out, void *stream);

/* Force profile of the last step: 3 doubles (fx, fy, fz) per y row (2D,
 * force_profile_2d, forces.py:142-162) or per z plane (3D,
 * spanwise_force_profile_3d, forces3d.py:148-171); host memory, synchronous. */
AERO_API int aero_read_profile(AeroLattice *lat, double *out, void *stream);

/* Status flags raised on the device since creation (bit 0: a cell had a
 * non-finite or non-positive density; the test of check_stability,
 * diagnostics.py:32-71.  Bit 1: a bounded device-side wait gave up, so a
 * step's output is incomplete; no counterpart in the reference).
 * Synchronous. */
AERO_API int aero_status(AeroLattice *lat, uint32_t *status, void *stream);

/* The first step (1-based, as counted by step_count) whose state had a
 * non-finite or non-positive density, or -1 if none has.  Synchronous. */
AERO_API int aero_first_bad_step(AeroLattice *lat, int64_t *step, void *stream);

/* Which step kernel aero_step launches (no counterpart in the reference):
 * *tiled = 0 for the default kernel, in which each cell gathers its pulled
 * populations from global memory; 1 for the row-tiled kernel, in which each
 * block stages the source rows of its tile in shared memory with bulk async
 * copies (selected by AERO_B200_TILES=1 in the environment at bind time,
 * where rows fit a tile and start 16-byte aligned), with the rows per tile
 * and the persistent grid size.  Valid after binding. */
AERO_API int aero_step_plan(const AeroLattice *lat, int32_t *tiled, int32_t *tile_rows, int32_t *blocks);

/* Step kernel choice for an autotuner (no counterpart in the reference):
 * 0, 1, 2 = the per-cell-gather kernel with blocks of 128x1, 256x1 or 32x4
 * cells (x by y); 3 = the row-tiled kernel (AERO_ERR_UNSUPPORTED where rows
 * do not fit it); 4 = two cells per thread on packed FP32 arithmetic (D3Q19
 * BGK/TRT/MRT, FP32/FP16/BF16 storage, even nx, no body force or scalar
 * lattice; else AERO_ERR_UNSUPPORTED); 5 = four cells per thread with one
 * 8-byte load per direction (D3Q19 BGK/TRT/MRT, FP16/BF16 storage, nx a
 * multiple of 4, no body force or scalar lattice; else AERO_ERR_UNSUPPORTED);
 * 6 = the D3Q19 BGK/TRT step with the LES velocity stencil staged in shared
 * memory, no separate moments pass (lattices with LES; else
 * AERO_ERR_UNSUPPORTED).  Results are the same for every choice up to FP
 * rounding of the compiled variant.  Takes effect at the next aero_step. */
AERO_API int aero_set_step_kernel(AeroLattice *lat, int32_t kernel);
AERO_API int aero_get_step_kernel(const AeroLattice *lat, int32_t *kernel);

/* Persistent runs (no counterpart in the reference; on by default): a
 * lattice of at most 2^19 cells in the two-buffer layout, stepped by the
 * per-cell kernel with no pass before the step (no BGK/TRT LES, no recycling
 * inlet), takes all steps of an aero_step call of two or more steps in one
 * cooperative launch, its force finalisation overlapping the next step.  The
 * results equal those of per-step launches bit for bit.  A bounded device
 * barrier that gives up sets status bit 1 (aero_status).  enable = 0 keeps
 * per-step launches (graphs).  Not used while the stream is capturing. */
AERO_API int aero_set_persistent(AeroLattice *lat, int32_t enable);
/* 1 when the lattice's next aero_step call of two or more steps runs
 * persistently (enabled and the lattice qualifies), else 0. */
AERO_API int aero_get_persistent(const AeroLattice *lat, int32_t *active);

/* Which compiled kernel set the lattice steps with (no counterpart in the
 * reference): 0 = the generic kernels, which read the feature word at run
 * time; otherwise a set compiled for one feature word and wall type, whose
 * other features' branches are removed: 1 = the thermal channel (D3Q19 TRT
 * + WALE, body force, D3Q7 scalar with buoyancy, obstacle, no-slip walls,
 * streamwise periodic; FP32 / FP16 / BF16 storage); 2, 3 = the open wind
 * tunnel in 2D, 3D (velocity inlet, outlet, obstacle with mid-link
 * bounce-back, slip walls; BGK / TRT / MRT; FP32); 4, 5 = the same with
 * Smagorinsky LES (BGK / TRT).  Batch classes keep their members' set.
 * Results agree with the generic kernels' up to FP rounding of the compiled
 * variant.  AERO_B200_GENERIC_KERNELS=1 in the environment at
 * aero_bind_workspace keeps the generic set. */
AERO_API int aero_kernel_variant(const AeroLattice *lat, int32_t *variant);

/* Inlet fields of steps first_step .. first_step+n_steps-1 for a lattice
 * with inflow_field set: `fields` (host) holds n_steps blocks of planes of
 * nz*ny doubles, (z, y) order.  Synthetic inflow: uy in 2D, uy then uz in
 * 3D; the inlet is the Zou-He velocity-field inlet of
 * apply_inlet_velocity_field(_3d) (boundary.py:48-65, boundary3d.py:71-93)
 * with ux = u0, as the reference's synthetic inflow calls it
 * (solver.py:386-392, solver3d.py:436-445).  SEM: u', v', w'; the inlet is
 * apply_inlet_sem_3d (boundary3d.py:96-137, solver3d.py:433-438).  The device holds inflow_ring
 * steps: first_step must not precede the next step to run, and the fields
 * must not reach beyond inflow_ring steps past it; aero_step refuses steps
 * whose fields are missing.  Synchronous. */
AERO_API int aero_set_inflow(AeroLattice *lat, const double *fields, int64_t first_step, int64_t n_steps,
                             void *stream);

/* Steps taken (host mirror of the reference's step_count). */
AERO_API int aero_step_count(const AeroLattice *lat, int64_t *steps);

/* Releases the handle (never the caller's workspace). */
AERO_API int aero_destroy(AeroLattice *lat);

/* Message of the last failed call on this thread. */
AERO_API const char *aero_last_error(void);

/* FP64 MRT operator f_post = A f + B feq of the reference basis
 * (mrt2d.py:36-77, mrt3d.py:46-135): A, B are Q x Q row-major.  Exposed so a
 * caller can check the engine's operator. */
AERO_API int aero_mrt_operator(int32_t dims, double omega, double *A, double *B);

/* Runs the engine's collision arithmetic (the device code compiled for the
 * host, FP64) on n cells: f_in / f_out are (Q, n) absolute populations,
 * solid may be NULL.  Lets a caller check the collision operators on a CPU
 * (kernels.py:42-92, kernels_trt.py:125-174, kernels3d_mrt.py:24-82). */
AERO_API int aero_collide_host(const AeroParams *params, const double *f_in, double *f_out,
                               const uint8_t *solid, int64_t n);

/* Number of lattice directions and scalar directions for the options. */
AERO_API int aero_lattice_q(const AeroParams *params, int32_t *q, int32_t *q_scalar);

AERO_API int aero_abi_version(void);

/* Per-kernel timing of aero_step (no counterpart in the reference, which
 * has no GPU path): while enabled, aero_step launches each step without
 * CUDA graphs and brackets the fused step kernel and the force kernels with
 * CUDA events on the caller's stream.  aero_kernel_times synchronises the
 * stream, returns the summed event times in milliseconds and the number of
 * steps timed, and resets the sums. */
AERO_API int aero_enable_timing(AeroLattice *lat, int32_t on);
AERO_API int aero_kernel_times(AeroLattice *lat, double *step_ms, double *forces_ms, int64_t *steps,
                               void *stream);

/* Momentum-exchange forces for callers that cannot allocate GPU memory.
 * No counterpart in the reference (its force sums run on host arrays).
 * Real-time loops whose device memory is fixed in advance, and host
 * frameworks that only lend out buffers they own and forbid a library to
 * allocate behind their back, cannot call cudaMalloc (or a caching
 * allocator); this entry point allocates nothing.  Given device arrays
 * f_pre and f_post (Q, nz, ny, nx) float64 and the link list (n_links rows
 * of [i, (z,) y, x] int32), it writes the AERO_FORCE_VALUES sums of
 * forces.py / forces3d.py to out (device, 12 doubles) and, if profile is not
 * NULL, the per-row (2D) / per-plane (3D) force profile (device, 3 doubles per
 * row/plane).  center is a HOST pointer to (x, y, z).  Its per-link scratch is
 * a fixed 4 MiB array in the library's device image, so n_links is limited to
 * 32768 (larger lists return AERO_ERR_CAPACITY).  Every call shares that
 * array: calls that overlap on the GPU race.  Each call made outside stream
 * capture looks the array's address up (cudaGetSymbolAddress) with its
 * device current; a call on a capturing stream reuses the address found by
 * an earlier call on that device, so make the first call on a device before
 * any stream capture (otherwise AERO_ERR_STATE).  A row whose direction is
 * outside 1..Q-1 or whose cell is outside the grid (the reference raises
 * IndexError there) makes every output value NaN.  The profile is summed
 * by one block per row/plane, each thread over a fixed stride of the link
 * list and the block in a fixed order (deterministic); the blocks run in
 * parallel, each one pass over the list. */
AERO_API int aero_link_forces_static(int32_t dims, int32_t nx, int32_t ny, int32_t nz, const double *f_pre,
                                     const double *f_post, const int32_t *links, int64_t n_links,
                                     const double *center, double *out, double *profile, void *stream);

/* ---- Batches: many lattices advanced together -------------------------
 * No counterpart in the reference, which advances one Solver at a time from
 * Python (Solver.run, solver.py:517-570).  A batch steps all its member
 * lattices with one launch per lattice class (dimensions, storage,
 * collision) and step kernel, replayed as CUDA graphs; lattices of any size,
 * geometry and parameters mix.  Members keep their own device state, force
 * history and read functions (aero_read_forces, aero_get_state, ...); while a
 * member, a lattice is advanced only by aero_batch_step (aero_step,
 * aero_set_state and aero_destroy on it return AERO_ERR_STATE) and its force
 * history is a rolling window of its ring: unread steps older than the ring
 * are dropped.  The caller allocates the batch's device workspace, as for a
 * lattice.  Not thread-safe: one host thread per batch and its members. */
typedef struct AeroBatch AeroBatch;

/* A batch for up to max_members lattices. */
AERO_API int aero_batch_create(int32_t max_members, AeroBatch **out);
/* Device bytes of the batch's plan; the caller allocates them. */
AERO_API int aero_batch_workspace_size(const AeroBatch *batch, uint64_t *bytes);
/* Binds the caller's device workspace (256-byte aligned). */
AERO_API int aero_batch_bind_workspace(AeroBatch *batch, void *device_ptr, uint64_t bytes);
/* Adds a bound lattice whose state is set.  cd_norm is the drag
 * normalisation used by aero_batch_converge: Cd = Fx / cd_norm (the
 * reference's 0.5 rho0 u0^2 D in 2D, forces.py:78-103, and 0.5 rho0 u0^2 D^2
 * in 3D, forces3d.py:70-101).  A lattice of at least 2^20 cells steps on
 * its own kernels as a branch of the batch step; only such a lattice may be
 * in the AA layout (AERO_ERR_UNSUPPORTED otherwise): each aero_batch_step
 * then collides the state it stored and ends on a state-storing step, as
 * aero_step does.  A lattice with a recycling inlet joins (its plane-mean
 * pass runs before each step, as in aero_step); one with synthetic inflow
 * or an SEM inlet joins, and aero_batch_step needs its inflow fields for
 * all the call's steps on the device first (aero_set_inflow;
 * AERO_ERR_STATE otherwise). */
AERO_API int aero_batch_add(AeroBatch *batch, AeroLattice *lat, double cd_norm);
/* Removes a member; it can then be stepped, read or destroyed on its own. */
AERO_API int aero_batch_remove(AeroBatch *batch, AeroLattice *lat);
AERO_API int aero_batch_size(const AeroBatch *batch, int32_t *n);
/* Advances every member n_steps steps, forces included.  Asynchronous. */
AERO_API int aero_batch_step(AeroBatch *batch, int64_t n_steps, void *stream);
/* Rolling drag convergence of every member on the device, by the rule of
 * analyze_convergence (diagnostics.py:87-120): over the last `window`
 * steps, ratio = std(Cd) / mean|Cd|, converged when ratio < tol (or mean|Cd|
 * < 1e-12).  out (host) receives AERO_CONVERGE_VALUES doubles per member, in
 * the order the members joined: ratio, mean|Cd|, std, converged (0/1),
 * steps taken, the member's status word (aero_status), mean Cd; ratio is
 * +inf and converged 0 while fewer than `window` steps are in the ring.
 * Synchronous. */
#define AERO_CONVERGE_VALUES 7
AERO_API int aero_batch_converge(AeroBatch *batch, int32_t window, double tol, double *out, void *stream);
/* Releases the batch (members stay valid and leave it). */
AERO_API int aero_batch_destroy(AeroBatch *batch);

/* sizeof(AeroParams), so bindings can check their struct layout. */
AERO_API int aero_params_size(void);

/* Like aero_get_state for f only, restricted to the planes z0 .. z0+nzs-1:
 * f receives (Q, nzs, ny, nx) float64 in caller DEVICE memory.  Lets a
 * caller inspect one plane of a large lattice (the 3D stability check reads
 * the mid plane, solver3d.py:608-615). */
AERO_API int aero_get_state_slab(AeroLattice *lat, int32_t z0, int32_t nzs, double *f, void *stream);

/* Density and velocity of the current state, computed on the device without
 * materialising f: out (caller DEVICE memory) receives 1 + dims planes of
 * nz*ny*nx doubles, rho, ux, uy (, uz).  Replaces compute_macroscopic(_3d)
 * (d2q9.py:44-63, d3q19.py:80-102) on self.f, as Solver.run's result uses it
 * (solver.py:603-632, solver3d.py:654-723).  Asynchronous. */
AERO_API int aero_get_macroscopic(AeroLattice *lat, double *out, void *stream);

/* FP64 statistics of the current state over the planes z0 .. z0+nzs-1 (2D:
 * z0 = 0, nzs = 1), reduced on the device in a fixed order.  out (HOST)
 * receives AERO_FIELD_STATS doubles:
 *   0 NaN populations, 1 cells with rho <= 0, 2 max sqrt(ux^2 + uy^2),
 *   3 sum of rho, 4 cells, 5 sum of the scalar T = sum_i g_i (0 without a
 *   scalar), 6 sum of -dT/dy at the y = 0 row, 7 columns in that sum,
 *   8 sum of -dT/dy at the y = ny-1 row, 9 columns in that sum.
 * Values 0-4 are what check_stability (diagnostics.py:32-71) tests on the
 * field (solver.py:522-531 on the whole 2D field, solver3d.py:608-615 on
 * the mid plane); 3 and 5 are the global mass and scalar totals.  The wall
 * gradients (the reference computes no Nusselt number) are second-order
 * one-sided differences of T at the Dirichlet rows, over the (x, z) columns
 * whose two cells next to the wall are fluid: the Nusselt number is
 * (sum / columns) (ny - 1) / (T_hot - T_cold).  Synchronous. */
#define AERO_FIELD_STATS 10
AERO_API int aero_field_stats(AeroLattice *lat, int32_t z0, int32_t nzs, double *out, void *stream);

/* ---- Surface links built on the device --------------------------------
 * Replaces build_surface_links (boundary.py:232-280) and
 * build_surface_links_3d (boundary3d.py:279-329) for geometry that already
 * lives on the GPU.  Same list, entry for entry: rows [i, (z,) y, x] int32
 * for every fluid cell whose neighbour in direction i (1..Q-1, the index
 * clipped to the grid) is solid, direction-major, cells in C order within a
 * direction; q = clip(float32(phi), 1e-4, 1) when phi is given, else 0.5.
 * dims 2 (nz = 1, D2Q9) or 3 (D3Q19).  The caller provides the scratch:
 * aero_surface_links_scratch_size gives its bytes (8-byte aligned). */
AERO_API int aero_surface_links_scratch_size(int32_t dims, int32_t nx, int32_t ny, int32_t nz, uint64_t *bytes);
/* solid (nz*ny*nx bytes, nonzero = solid), phi (float64 per cell or NULL),
 * links (capacity rows of dims+1 int32) and q (capacity floats) are DEVICE
 * arrays.  Counts the links, writes the count to *n_links (host), then writes
 * the list; when the count exceeds capacity nothing is written and the call
 * returns AERO_ERR_CAPACITY with *n_links set, so a caller can size the
 * output from a first call with capacity 0.  Synchronises the stream once
 * (to read the count). */
AERO_API int aero_surface_links_device(int32_t dims, int32_t nx, int32_t ny, int32_t nz, const uint8_t *solid,
                                       const double *phi, void *scratch, uint64_t scratch_size, int32_t *links,
                                       float *q, int64_t capacity, int64_t *n_links, void *stream);

#ifdef __cplusplus
}
#endif
#endif
