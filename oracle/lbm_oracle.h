/*
 * lbm_oracle.h -- parity oracle (TEST INFRASTRUCTURE ONLY).
 *
 * FP64 CPU restatement of the Aero LBM step (aero/lbm/solver.py:276-464,
 * aero/lbm/solver3d.py:325-541).  Used by tests/ and by bench.py's CPU
 * baseline; never by the aero_b200 product path.
 */
#ifndef AERO_LBM_ORACLE_H
#define AERO_LBM_ORACLE_H
#include <stdint.h>

enum { ORACLE_BGK = 0, ORACLE_TRT = 1, ORACLE_MRT = 2 };
enum { ORACLE_LES_SMAGORINSKY = 0, ORACLE_LES_WALE = 1 };
enum { ORACLE_WALL_NONE = 0, ORACLE_WALL_SLIP = 1, ORACLE_WALL_NOSLIP = 2, ORACLE_WALL_MOVING = 3 };
enum { ORACLE_INLET_NONE = 0, ORACLE_INLET_VELOCITY = 1, ORACLE_INLET_PRESSURE = 2 };
enum {
  ORACLE_OUTLET_NONE = 0,
  ORACLE_OUTLET_CONVECTIVE = 1,
  ORACLE_OUTLET_ZEROGRAD = 2,
  ORACLE_OUTLET_PRESSURE = 3
};
enum { ORACLE_STREAM_OPEN = 0, ORACLE_STREAM_PERIODIC = 1, ORACLE_STREAM_RECYCLING = 2 };

typedef struct OracleLattice {
  int32_t dims, nx, ny, nz;
  int32_t collision, les, les_model, van_driest, bouzidi, ibm_enabled;
  int32_t wall_bc, inlet_bc, outlet_bc, streamwise_bc, sponge_thickness;
  int32_t thermal, buoyancy, scalar_reduced;
  int64_t step_count;
  int64_t n_links;
  double omega, u0, rho_in, rho_out, inlet_perturbation, trt_lambda;
  double sponge_strength, les_cs, van_driest_A;
  double wall_velocity_top, wall_velocity_bottom;
  double body_force[3];
  double omega_T, T_hot, T_cold, g_gravity, beta, T_ref;
  double center[3]; /* moment reference point (x, y, z) */
  /* caller-owned arrays */
  double *f;             /* (Q, nz, ny, nx) state, updated in place */
  double *g;             /* (Qg, nz, ny, nx) scalar state or NULL */
  double *f_outlet_prev; /* (Q, [nz,] ny) convective-outlet state */
  const uint8_t *solid;  /* (nz, ny, nx) */
  const double *phi;     /* (nz, ny, nx) or NULL */
  const int32_t *links;  /* (n_links, 3|4) */
  const float *q_vals;   /* (n_links,) */
  const double *mrt_M, *mrt_Minv, *mrt_s;
  double *work_a, *work_b, *work_om, *work_g;
  /* synthetic inflow of the step about to run: (dims-1, nz, ny) transverse
   * inlet velocities (uy; 3D then uz), or NULL for the uniform inlet */
  const double *inflow;
  /* SEM fluctuations of the step about to run: (3, nz, ny) u', v', w'
   * (3D), or NULL; takes precedence over `inflow` */
  const double *sem;
} OracleLattice;

int oracle_step(OracleLattice *s, double *out_forces, double *out_profile);
int oracle_collide_only(OracleLattice *s, double *f_post);
int oracle_omega_field(OracleLattice *s, double *om);
int oracle_abi_version(void);

#endif
