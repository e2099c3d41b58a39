/*
 * lbm_oracle.c -- FP64 CPU restatement of the Aero lattice Boltzmann step.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle: the tests and the
 * CPU-baseline leg of bench.py call it to check (and time) the CUDA engine.  It
 * is never linked into, loaded by, or used as a fallback for the product path
 * in aero_b200/.
 *
 * It restates, in plain C with OpenMP loops, the per-step update of the
 * reference solver in exactly the reference's order:
 *   aero/lbm/solver.py:276-464   (Solver._step, D2Q9)
 *   aero/lbm/solver3d.py:325-541 (Solver3D._step, D3Q19)
 * Every array has the reference layout: C-contiguous float64 (Q, Nz, Ny, Nx)
 * with Nz = 1 in 2D.  Each function cites the reference lines it follows.
 *
 * Pinned against golden vectors produced by importing the reference itself
 * (tests/golden/make_golden.py); see tests/test_oracle_golden.py.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "lbm_oracle.h"

/* ------------------------------------------------------------------------ */
/* Lattice tables: aero/lbm/d2q9.py:18-38, aero/lbm/d3q19.py:37-73          */
/* ------------------------------------------------------------------------ */
static const int E2[9][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1},
                             {1, 1}, {-1, 1}, {-1, -1}, {1, -1}};
static const int OPP2[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
static const int E3[19][3] = {
    {0, 0, 0},  {1, 0, 0},   {-1, 0, 0}, {0, 1, 0},  {0, -1, 0},
    {0, 0, 1},  {0, 0, -1},  {1, 1, 0},  {-1, 1, 0}, {1, -1, 0},
    {-1, -1, 0}, {1, 0, 1},  {-1, 0, 1}, {1, 0, -1}, {-1, 0, -1},
    {0, 1, 1},  {0, -1, 1},  {0, 1, -1}, {0, -1, -1}};
static const int OPP3[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};

/* D2Q5 / D3Q7 scalar lattices (speed-mode scalar; not in the reference). */
static const int E2Q5[5][2] = {{0, 0}, {1, 0}, {0, 1}, {-1, 0}, {0, -1}};
static const int E3Q7[7][3] = {{0, 0, 0}, {1, 0, 0}, {-1, 0, 0}, {0, 1, 0},
                               {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};

typedef struct {
  int Q;
  int ex[19], ey[19], ez[19], opp[19];
  double w[19];
} Lat;

static void lat_init(Lat *L, int dims) {
  memset(L, 0, sizeof(*L));
  if (dims == 2) {
    L->Q = 9;
    for (int i = 0; i < 9; i++) {
      L->ex[i] = E2[i][0];
      L->ey[i] = E2[i][1];
      L->opp[i] = OPP2[i];
      L->w[i] = i == 0 ? 4.0 / 9.0 : (i < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
    }
  } else {
    L->Q = 19;
    for (int i = 0; i < 19; i++) {
      L->ex[i] = E3[i][0];
      L->ey[i] = E3[i][1];
      L->ez[i] = E3[i][2];
      L->opp[i] = OPP3[i];
      L->w[i] = i == 0 ? 1.0 / 3.0 : (i < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
    }
  }
}

/* Scalar lattice: the flow lattice in parity mode (aero/lbm/thermal.py uses
 * D2Q9/D3Q19), or D2Q5/D3Q7 in reduced mode. */
static void scalar_lat_init(Lat *L, int dims, int reduced) {
  if (!reduced) {
    lat_init(L, dims);
    return;
  }
  memset(L, 0, sizeof(*L));
  if (dims == 2) {
    L->Q = 5;
    for (int i = 0; i < 5; i++) {
      L->ex[i] = E2Q5[i][0];
      L->ey[i] = E2Q5[i][1];
      L->w[i] = i == 0 ? 1.0 / 3.0 : 1.0 / 6.0;
    }
  } else {
    L->Q = 7;
    for (int i = 0; i < 7; i++) {
      L->ex[i] = E3Q7[i][0];
      L->ey[i] = E3Q7[i][1];
      L->ez[i] = E3Q7[i][2];
      L->w[i] = i == 0 ? 1.0 / 4.0 : 1.0 / 8.0;
    }
  }
}

#define IDX(i, z, y, x) ((((int64_t)(i) * nz + (z)) * ny + (y)) * nx + (x))
#define CIDX(z, y, x) ((((int64_t)(z)) * ny + (y)) * nx + (x))

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int wrapi(int v, int n) {
  int r = v % n;
  return r < 0 ? r + n : r;
}

/* feq: aero/lbm/d2q9.py:66-89, aero/lbm/d3q19.py:105-129 */
static inline double feq_i(const Lat *L, int i, double rho, double ux, double uy, double uz) {
  double usq = ux * ux + uy * uy + uz * uz;
  double eu = L->ex[i] * ux + L->ey[i] * uy + L->ez[i] * uz;
  return L->w[i] * rho * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * usq);
}

/* compute_macroscopic(_3d): aero/lbm/d2q9.py:44-63, d3q19.py:80-102 */
static inline void moments(const Lat *L, const double *f, int64_t cs, int64_t c, double *rho,
                           double *ux, double *uy, double *uz) {
  double r = 0, mx = 0, my = 0, mz = 0;
  for (int i = 0; i < L->Q; i++) {
    double fi = f[i * cs + c];
    r += fi;
    mx += L->ex[i] * fi;
    my += L->ey[i] * fi;
    mz += L->ez[i] * fi;
  }
  double inv = r > 0.0 ? 1.0 / r : 0.0;
  *rho = r;
  *ux = inv * mx;
  *uy = inv * my;
  *uz = inv * mz;
}

/* ------------------------------------------------------------------------ */
/* LES omega field: aero/lbm/les.py:24-78 (strain), :177-262 (WALE),        */
/* :265-266 (omega_from_nu), :273-344 (build_omega_field_2d/3d)             */
/* ------------------------------------------------------------------------ */
static void build_omega_field(const OracleLattice *s, const Lat *L, const double *f, double *om) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int64_t cs = (int64_t)nx * ny * nz;
  double *u = (double *)malloc(sizeof(double) * 3 * cs);
  const double base_nu = (1.0 / s->omega - 0.5) / 3.0; /* physics.py:27-29 */
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < cs; c++) {
    double rho, ux, uy, uz;
    moments(L, f, cs, c, &rho, &ux, &uy, &uz);
    u[c] = ux;
    u[cs + c] = uy;
    u[2 * cs + c] = uz;
  }
  const double *UX = u, *UY = u + cs, *UZ = u + 2 * cs;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < cs; c++) {
    int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((int64_t)nx * ny));
    double nu_sgs = 0.0;
    int interior = x >= 1 && x <= nx - 2 && y >= 1 && y <= ny - 2;
    if (s->dims == 3) interior = interior && z >= 1 && z <= nz - 2;
    double cs_eff = s->les_cs;
    if (s->van_driest && s->phi) {
      double yw = fabs(s->phi[c]);
      double d = 1.0 - exp(-yw / s->van_driest_A);
      cs_eff = s->les_cs * d * d;
    }
    if (interior && !s->solid[c]) {
      double g[3][3] = {{0}};
      g[0][0] = 0.5 * (UX[c + 1] - UX[c - 1]);
      g[0][1] = 0.5 * (UX[c + nx] - UX[c - nx]);
      g[1][0] = 0.5 * (UY[c + 1] - UY[c - 1]);
      g[1][1] = 0.5 * (UY[c + nx] - UY[c - nx]);
      if (s->dims == 3) {
        int64_t sz = (int64_t)nx * ny;
        g[0][2] = 0.5 * (UX[c + sz] - UX[c - sz]);
        g[1][2] = 0.5 * (UY[c + sz] - UY[c - sz]);
        g[2][0] = 0.5 * (UZ[c + 1] - UZ[c - 1]);
        g[2][1] = 0.5 * (UZ[c + nx] - UZ[c - nx]);
        g[2][2] = 0.5 * (UZ[c + sz] - UZ[c - sz]);
      }
      if (s->les_model == ORACLE_LES_WALE) {
        int d = s->dims;
        double s_sq = 0, sd_sq = 0, gsq[3][3] = {{0}}, tr = 0;
        for (int a = 0; a < d; a++)
          for (int b = 0; b < d; b++) {
            double sab = 0.5 * (g[a][b] + g[b][a]);
            s_sq += sab * sab;
            for (int k = 0; k < d; k++) gsq[a][b] += g[a][k] * g[k][b];
          }
        for (int a = 0; a < d; a++) tr += gsq[a][a];
        tr /= (double)d; /* 2D: 0.5*trace (les.py:207); 3D: trace/3 (les.py:257) */
        for (int a = 0; a < d; a++)
          for (int b = 0; b < d; b++) {
            double sdab = 0.5 * (gsq[a][b] + gsq[b][a]) - (a == b ? tr : 0.0);
            sd_sq += sdab * sdab;
          }
        double num = pow(sd_sq, 1.5);
        double den = pow(s_sq, 2.5) + pow(sd_sq, 1.25) + 1e-30;
        nu_sgs = (cs_eff * cs_eff) * num / den;
      } else {
        double s11 = g[0][0], s22 = g[1][1], s33 = g[2][2];
        double s12 = 0.5 * (g[0][1] + g[1][0]);
        double s13 = 0.5 * (g[0][2] + g[2][0]);
        double s23 = 0.5 * (g[1][2] + g[2][1]);
        double smag;
        if (s->dims == 2)
          smag = sqrt(2.0 * (s11 * s11 + s22 * s22 + 2.0 * s12 * s12));
        else
          smag = sqrt(2.0 * (s11 * s11 + s22 * s22 + s33 * s33) +
                      4.0 * (s12 * s12 + s13 * s13 + s23 * s23));
        nu_sgs = cs_eff * cs_eff * smag;
      }
    }
    double nu_eff = s->solid[c] ? base_nu : base_nu + nu_sgs;
    om[c] = 1.0 / (3.0 * nu_eff + 0.5);
  }
  free(u);
}

/* ------------------------------------------------------------------------ */
/* Collision: BGK aero/lbm/kernels.py:42-92, kernels3d.py:24-61;            */
/* TRT kernels_trt.py:125-174 + trt2d.py:8-18; MRT kernels_mrt.py:190-241,  */
/* kernels3d_mrt.py:24-82 (f_post = Minv (m - s (m - m_eq)))                */
/* ------------------------------------------------------------------------ */
static void collide(const OracleLattice *s, const Lat *L, const double *f, double *fp,
                    const double *om_field) {
  const int nx = s->nx, ny = s->ny, nz = s->nz, Q = L->Q;
  const int64_t cs = (int64_t)nx * ny * nz;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < cs; c++) {
    double rho, ux, uy, uz, feq[19], fc[19];
    moments(L, f, cs, c, &rho, &ux, &uy, &uz);
    if (s->solid[c]) ux = uy = uz = 0.0;
    for (int i = 0; i < Q; i++) {
      feq[i] = feq_i(L, i, rho, ux, uy, uz);
      fc[i] = f[i * cs + c];
    }
    if (s->collision == ORACLE_MRT) {
      double m[19], meq[19], mp[19];
      for (int a = 0; a < Q; a++) {
        double acc = 0, acq = 0;
        for (int b = 0; b < Q; b++) {
          acc += s->mrt_M[a * Q + b] * fc[b];
          acq += s->mrt_M[a * Q + b] * feq[b];
        }
        m[a] = acc;
        meq[a] = acq;
      }
      for (int a = 0; a < Q; a++) mp[a] = m[a] - s->mrt_s[a] * (m[a] - meq[a]);
      for (int i = 0; i < Q; i++) {
        double acc = 0;
        for (int a = 0; a < Q; a++) acc += s->mrt_Minv[i * Q + a] * mp[a];
        fp[i * cs + c] = acc;
      }
    } else if (s->collision == ORACLE_TRT) {
      double om = om_field ? om_field[c] : s->omega;
      double tau = 1.0 / om, lam = s->trt_lambda;
      double tp = lam * tau + (1.0 - lam);
      double tm = (tp * tau - 0.5) / (tp - 0.5);
      double sm = 1.0 / tm;
      for (int i = 0; i < Q; i++) {
        int j = L->opp[i];
        double fpl = 0.5 * (fc[i] + fc[j]), fmi = 0.5 * (fc[i] - fc[j]);
        double epl = 0.5 * (feq[i] + feq[j]), emi = 0.5 * (feq[i] - feq[j]);
        fp[i * cs + c] = feq[i] + (1.0 - om) * (fpl - epl) + (1.0 - sm) * (fmi - emi);
      }
    } else {
      double om = om_field ? om_field[c] : s->omega;
      for (int i = 0; i < Q; i++) fp[i * cs + c] = (1.0 - om) * fc[i] + om * feq[i];
    }
  }
}

/* Push stream with periodic wrap: kernels.py:94-114, kernels3d.py:63-80 */
static void stream(const OracleLattice *s, const Lat *L, const double *src, double *dst) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++)
        for (int i = 0; i < L->Q; i++) {
          int zn = wrapi(z + L->ez[i], nz), yn = wrapi(y + L->ey[i], ny), xn = wrapi(x + L->ex[i], nx);
          dst[IDX(i, zn, yn, xn)] = src[IDX(i, z, y, x)];
        }
}

/* Uniform Guo body force on fluid cells, post-stream: ibm_guo.py:263-301 */
static void body_force(const OracleLattice *s, const Lat *L, double *f) {
  const double fx = s->body_force[0], fy = s->body_force[1], fz = s->body_force[2];
  if (fabs(fx) < 1e-16 && fabs(fy) < 1e-16 && fabs(fz) < 1e-16) return;
  const int64_t cs = (int64_t)s->nx * s->ny * s->nz;
  const double cs2 = 1.0 / 3.0, coeff = 1.0 - 0.5 / (1.0 / s->omega);
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < cs; c++) {
    if (s->solid[c]) continue;
    double rho, ux, uy, uz;
    moments(L, f, cs, c, &rho, &ux, &uy, &uz);
    if (rho <= 0.0) continue;
    double uf = ux * fx + uy * fy + uz * fz;
    for (int i = 0; i < L->Q; i++) {
      double eu = L->ex[i] * ux + L->ey[i] * uy + L->ez[i] * uz;
      double ef = L->ex[i] * fx + L->ey[i] * fy + L->ez[i] * fz;
      double term = (ef - uf) / cs2 + (eu * ef) / (cs2 * cs2);
      f[i * cs + c] += coeff * L->w[i] * rho * term;
    }
  }
}

/* Mid-link and Bouzidi bounce-back over the link list:
 * boundary.py:283-352, boundary3d.py:333-393 */
static void bounce_back(const OracleLattice *s, const Lat *L, double *f, const double *fpre) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int lw = s->dims == 3 ? 4 : 3;
  for (int64_t k = 0; k < s->n_links; k++) {
    const int32_t *lk = s->links + k * lw;
    int i = lk[0], z = s->dims == 3 ? lk[1] : 0, y = lk[lw - 2], x = lk[lw - 1];
    int o = L->opp[i];
    if (!s->bouzidi) {
      f[IDX(o, z, y, x)] = fpre[IDX(i, z, y, x)];
      continue;
    }
    double q = (double)s->q_vals[k];
    if (q < 0.5) {
      f[IDX(o, z, y, x)] = 2.0 * q * fpre[IDX(i, z, y, x)] + (1.0 - 2.0 * q) * fpre[IDX(o, z, y, x)];
    } else {
      int zn = clampi(z + L->ez[o], 0, nz - 1), yn = clampi(y + L->ey[o], 0, ny - 1),
          xn = clampi(x + L->ex[o], 0, nx - 1);
      double inv2q = 1.0 / (2.0 * q);
      f[IDX(o, z, y, x)] = inv2q * fpre[IDX(i, z, y, x)] + (1.0 - inv2q) * fpre[IDX(i, zn, yn, xn)];
    }
  }
}

/* 2D inlet/outlet: boundary.py:15-45 (Zou-He velocity + sin perturbation),
 * :116-136 (Zou-He pressure in), :139-159 (pressure out), :68-75 (zero
 * gradient), :78-113 (convective). */
static void inlet_outlet_2d(OracleLattice *s, double *f) {
  const int nx = s->nx, ny = s->ny, nz = 1;
  const double u0 = s->u0;
  if (s->inlet_bc == ORACLE_INLET_VELOCITY && s->inflow) {
    /* per-row field inlet, boundary.py:48-65, with ux = u0 (solver.py:386-392) */
    for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, 0, y, 0)]
      double den = 1.0 - u0 > 1e-8 ? 1.0 - u0 : 1e-8;
      double rho_in = ((F(0) + F(2) + F(4)) + 2.0 * (F(3) + F(6) + F(7))) / den;
      double cy = rho_in * s->inflow[y];
      F(1) = F(3) + (2.0 / 3.0) * rho_in * u0;
      F(5) = F(7) - 0.5 * cy + (1.0 / 6.0) * rho_in * u0;
      F(8) = F(6) + 0.5 * cy + (1.0 / 6.0) * rho_in * u0;
#undef F
    }
  } else if (s->inlet_bc == ORACLE_INLET_VELOCITY) {
    const int64_t step = s->step_count + 1;
    for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, 0, y, 0)]
      double rho_in = ((F(0) + F(2) + F(4)) + 2.0 * (F(3) + F(6) + F(7))) / (1.0 - u0);
      F(1) = F(3) + (2.0 / 3.0) * rho_in * u0;
      F(5) = F(7) - 0.5 * (F(2) - F(4)) + (1.0 / 6.0) * rho_in * u0;
      F(8) = F(6) + 0.5 * (F(2) - F(4)) + (1.0 / 6.0) * rho_in * u0;
      if (s->inlet_perturbation > 0.0) {
        double uy = s->inlet_perturbation * u0 *
                    sin(2.0 * M_PI * y / (double)(ny > 1 ? ny : 1) + 0.17 * (double)step);
        F(2) += uy * 0.25;
        F(4) -= uy * 0.25;
        F(5) += uy * 0.15;
        F(8) -= uy * 0.15;
      }
#undef F
    }
  } else if (s->inlet_bc == ORACLE_INLET_PRESSURE) {
    const double rin = s->rho_in;
    for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, 0, y, 0)]
      double ux = 1.0 - (F(0) + F(2) + F(4) + 2.0 * (F(3) + F(6) + F(7))) / rin;
      F(1) = F(3) + (2.0 / 3.0) * rin * ux;
      F(5) = F(7) - 0.5 * (F(2) - F(4)) + (1.0 / 6.0) * rin * ux;
      F(8) = F(6) + 0.5 * (F(2) - F(4)) + (1.0 / 6.0) * rin * ux;
#undef F
    }
  }
  if (s->outlet_bc == ORACLE_OUTLET_CONVECTIVE) {
    double u = u0 < 0.0 ? 0.0 : (u0 > 1.0 ? 1.0 : u0);
    for (int i = 0; i < 9; i++)
      for (int y = 0; y < ny; y++) {
        double nv = (1.0 - u) * s->f_outlet_prev[(int64_t)i * ny + y] + u * f[IDX(i, 0, y, nx - 2)];
        f[IDX(i, 0, y, nx - 1)] = nv;
        s->f_outlet_prev[(int64_t)i * ny + y] = nv;
      }
  } else if (s->outlet_bc == ORACLE_OUTLET_PRESSURE) {
    const double ro = s->rho_out;
    for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, 0, y, nx - 1)]
      double ux = -1.0 + (F(0) + F(2) + F(4) + 2.0 * (F(1) + F(5) + F(8))) / ro;
      F(3) = F(1) - (2.0 / 3.0) * ro * ux;
      F(7) = F(5) + 0.5 * (F(2) - F(4)) - (1.0 / 6.0) * ro * ux;
      F(6) = F(8) - 0.5 * (F(2) - F(4)) - (1.0 / 6.0) * ro * ux;
#undef F
    }
  } else if (s->outlet_bc == ORACLE_OUTLET_ZEROGRAD) {
    for (int i = 0; i < 9; i++)
      for (int y = 0; y < ny; y++) f[IDX(i, 0, y, nx - 1)] = f[IDX(i, 0, y, nx - 2)];
  }
}

/* 3D inlet/outlet: boundary3d.py:24-68 (Zou-He, uz perturbation as called
 * from solver3d.py:447-452), :144-146 (zero gradient), :149-164 (convective).
 * Streamwise "periodic" is a no-op (boundary3d.py:167-169). */
static void inlet_outlet_3d(OracleLattice *s, double *f) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const double u0 = s->u0;
  if (s->streamwise_bc == ORACLE_STREAM_RECYCLING) {
    /* boundary3d.py:172-198: macroscopic state of plane x = nx-2, its mean ux
     * over the plane, then the inlet plane = feq(rho, scale * u) */
    const int64_t plane = (int64_t)nz * ny;
    double *rho = malloc(sizeof(double) * plane * 4);
    double *ux = rho + plane, *uy = ux + plane, *uz = uy + plane;
    double sum = 0.0;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
        const int64_t r = (int64_t)z * ny + y;
        double m = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
        for (int i = 0; i < 19; i++) {
          double v = f[IDX(i, z, y, nx - 2)];
          m += v;
          jx += E3[i][0] * v;
          jy += E3[i][1] * v;
          jz += E3[i][2] * v;
        }
        double inv = m > 0.0 ? 1.0 / m : 0.0;
        rho[r] = m;
        ux[r] = inv * jx;
        uy[r] = inv * jy;
        uz[r] = inv * jz;
      }
    for (int64_t r = 0; r < plane; r++) sum += ux[r];
    const double mean = sum / (double)plane;
    const double scale = fabs(mean) < 1e-12 ? 1.0 : u0 / mean;
    Lat L;
    lat_init(&L, 3);
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
        const int64_t r = (int64_t)z * ny + y;
        for (int i = 0; i < 19; i++)
          f[IDX(i, z, y, 0)] = feq_i(&L, i, rho[r], ux[r] * scale, uy[r] * scale, uz[r] * scale);
      }
    free(rho);
    return;
  }
  if (s->streamwise_bc != ORACLE_STREAM_OPEN) return;
  if (s->inlet_bc == ORACLE_INLET_VELOCITY && s->sem) {
    /* apply_inlet_sem_3d, boundary3d.py:96-137 */
    const int64_t plane = (int64_t)nz * ny;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, z, y, 0)]
        const int64_t r = (int64_t)z * ny + y;
        double ux = u0 + s->sem[r];
        double den = 1.0 - ux > 1e-10 ? 1.0 - ux : 1e-10;
        double Fm = F(2) + F(8) + F(10) + F(12) + F(14);
        double Fn = F(0) + F(3) + F(4) + F(5) + F(6) + F(15) + F(16) + F(17) + F(18);
        double rho_in = (2.0 * Fm + Fn) / den;
        double cy = F(3) - F(4) + F(15) - F(16) + F(17) - F(18) - rho_in * s->sem[plane + r];
        double cz = F(5) - F(6) + F(15) + F(16) - F(17) - F(18) - rho_in * s->sem[2 * plane + r];
        F(1) = F(2) + (1.0 / 3.0) * rho_in * ux;
        F(7) = F(10) + (1.0 / 6.0) * rho_in * ux - 0.5 * cy;
        F(9) = F(8) + (1.0 / 6.0) * rho_in * ux + 0.5 * cy;
        F(11) = F(14) + (1.0 / 6.0) * rho_in * ux - 0.5 * cz;
        F(13) = F(12) + (1.0 / 6.0) * rho_in * ux + 0.5 * cz;
#undef F
      }
  } else if (s->inlet_bc == ORACLE_INLET_VELOCITY && s->inflow) {
    /* per-cell field inlet, boundary3d.py:71-93, ux = u0 (solver3d.py:436-445) */
    const int64_t plane = (int64_t)nz * ny;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, z, y, 0)]
        const int64_t r = (int64_t)z * ny + y;
        double Fm = F(2) + F(8) + F(10) + F(12) + F(14);
        double Fn = F(0) + F(3) + F(4) + F(5) + F(6) + F(15) + F(16) + F(17) + F(18);
        double den = 1.0 - u0 > 1e-8 ? 1.0 - u0 : 1e-8;
        double rho_in = (2.0 * Fm + Fn) / den;
        double cy = rho_in * s->inflow[r], cz = rho_in * s->inflow[plane + r];
        F(1) = F(2) + (1.0 / 3.0) * rho_in * u0;
        F(7) = F(10) + (1.0 / 6.0) * rho_in * u0 - 0.5 * cy;
        F(9) = F(8) + (1.0 / 6.0) * rho_in * u0 + 0.5 * cy;
        F(11) = F(14) + (1.0 / 6.0) * rho_in * u0 - 0.5 * cz;
        F(13) = F(12) + (1.0 / 6.0) * rho_in * u0 + 0.5 * cz;
#undef F
      }
  } else if (s->inlet_bc == ORACLE_INLET_VELOCITY) {
    const int64_t step = s->step_count + 1;
#pragma omp parallel for collapse(2)
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
#define F(i) f[IDX(i, z, y, 0)]
        double Fm = F(2) + F(8) + F(10) + F(12) + F(14);
        double Fn = F(0) + F(3) + F(4) + F(5) + F(6) + F(15) + F(16) + F(17) + F(18);
        double rho_in = (2.0 * Fm + Fn) / (1.0 - u0);
        double cy = F(3) - F(4) + F(15) - F(16) + F(17) - F(18);
        double cz = F(5) - F(6) + F(15) + F(16) - F(17) - F(18);
        if (s->inlet_perturbation > 0.0) {
          double uz = s->inlet_perturbation * u0 *
                      sin(2.0 * M_PI * z / (double)(nz > 1 ? nz : 1) + 0.17 * (double)step);
          cz = cz + rho_in * uz;
        }
        F(1) = F(2) + (1.0 / 3.0) * rho_in * u0;
        F(7) = F(10) + (1.0 / 6.0) * rho_in * u0 - 0.5 * cy;
        F(9) = F(8) + (1.0 / 6.0) * rho_in * u0 + 0.5 * cy;
        F(11) = F(14) + (1.0 / 6.0) * rho_in * u0 - 0.5 * cz;
        F(13) = F(12) + (1.0 / 6.0) * rho_in * u0 + 0.5 * cz;
#undef F
      }
  }
  if (s->outlet_bc == ORACLE_OUTLET_CONVECTIVE) {
    double u = u0 < 0.0 ? 0.0 : (u0 > 1.0 ? 1.0 : u0);
    for (int i = 0; i < 19; i++)
      for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++) {
          int64_t pi = ((int64_t)i * nz + z) * ny + y;
          double nv = (1.0 - u) * s->f_outlet_prev[pi] + u * f[IDX(i, z, y, nx - 2)];
          f[IDX(i, z, y, nx - 1)] = nv;
          s->f_outlet_prev[pi] = nv;
        }
  } else {
    for (int i = 0; i < 19; i++)
      for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++) f[IDX(i, z, y, nx - 1)] = f[IDX(i, z, y, nx - 2)];
  }
}

/* Sponge: sponge.py:8-21 (sigma ramp), :24-70 (relaxation to feq(rho,u0)) */
static void sponge(const OracleLattice *s, const Lat *L, double *f) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int T = s->sponge_thickness;
  if (T <= 0 || s->sponge_strength <= 0.0) return;
  int start = nx - T > 0 ? nx - T : 0;
  for (int x = start; x < nx; x++) {
    double frac = (double)(x - start + 1) / (double)(T > 1 ? T : 1);
    double sg = s->sponge_strength * frac * frac;
    if (sg <= 0.0) continue;
    for (int z = 0; z < nz; z++)
      for (int y = 0; y < ny; y++) {
        double rho = 0;
        for (int i = 0; i < L->Q; i++) rho += f[IDX(i, z, y, x)];
        for (int i = 0; i < L->Q; i++) {
          double feq = feq_i(L, i, rho, s->u0, 0.0, 0.0);
          f[IDX(i, z, y, x)] = (1.0 - sg) * f[IDX(i, z, y, x)] + sg * feq;
        }
      }
  }
}

/* Walls: 2D boundary.py:162-226; 3D boundary3d.py:205-271 */
static void walls(const OracleLattice *s, const Lat *L, double *f) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  if (s->wall_bc == ORACLE_WALL_NONE) return;
  const double ub = s->wall_velocity_bottom, ut = s->wall_velocity_top;
  for (int z = 0; z < nz; z++)
    for (int x = 0; x < nx; x++) {
      const int yb = 0, yt = ny - 1;
#define B(i) f[IDX(i, z, yb, x)]
#define T(i) f[IDX(i, z, yt, x)]
      if (s->dims == 2) {
        if (s->wall_bc == ORACLE_WALL_SLIP) {
          B(2) = B(4); B(5) = B(8); B(6) = B(7);
          T(4) = T(2); T(8) = T(5); T(7) = T(6);
        } else if (s->wall_bc == ORACLE_WALL_NOSLIP) {
          B(2) = B(4); B(5) = B(7); B(6) = B(8);
          T(4) = T(2); T(7) = T(5); T(8) = T(6);
        } else {
          double rb = 0, rt = 0;
          for (int i = 0; i < 9; i++) { rb += B(i); rt += T(i); }
          rb = rb > 1e-12 ? rb : 1e-12;
          rt = rt > 1e-12 ? rt : 1e-12;
          B(2) = B(4);
          B(5) = B(7) + 6.0 * (1.0 / 36.0) * rb * ub;
          B(6) = B(8) - 6.0 * (1.0 / 36.0) * rb * ub;
          T(4) = T(2);
          T(7) = T(5) - 6.0 * (1.0 / 36.0) * rt * ut;
          T(8) = T(6) + 6.0 * (1.0 / 36.0) * rt * ut;
        }
      } else {
        if (s->wall_bc == ORACLE_WALL_SLIP) {
          B(3) = B(4); B(7) = B(9); B(8) = B(10); B(15) = B(16); B(17) = B(18);
          T(4) = T(3); T(9) = T(7); T(10) = T(8); T(16) = T(15); T(18) = T(17);
        } else if (s->wall_bc == ORACLE_WALL_NOSLIP) {
          B(3) = B(4); B(7) = B(10); B(8) = B(9); B(15) = B(18); B(17) = B(16);
          T(4) = T(3); T(10) = T(7); T(9) = T(8); T(18) = T(15); T(16) = T(17);
        } else {
          double rb = 0, rt = 0;
          for (int i = 0; i < 19; i++) { rb += B(i); rt += T(i); }
          rb = rb > 1e-12 ? rb : 1e-12;
          rt = rt > 1e-12 ? rt : 1e-12;
          B(3) = B(4);
          B(7) = B(10) + 6.0 * (1.0 / 36.0) * rb * ub;
          B(8) = B(9) - 6.0 * (1.0 / 36.0) * rb * ub;
          B(15) = B(18);
          B(17) = B(16);
          T(4) = T(3);
          T(10) = T(7) - 6.0 * (1.0 / 36.0) * rt * ut;
          T(9) = T(8) + 6.0 * (1.0 / 36.0) * rt * ut;
          T(18) = T(15);
          T(16) = T(17);
        }
      }
#undef B
#undef T
    }
  (void)L;
}

/* Scalar step: thermal.py:47-124 (2D), :149-222 (3D); order as in
 * solver.py:427-443 and solver3d.py:481-503. */
static void thermal(OracleLattice *s, const Lat *L, double *f) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int64_t cs = (int64_t)nx * ny * nz;
  Lat G;
  scalar_lat_init(&G, s->dims, s->scalar_reduced);
  const int Qg = G.Q;
  double *gp = s->work_g;
#pragma omp parallel for schedule(static)
  for (int64_t c = 0; c < cs; c++) {
    double rho, ux, uy, uz;
    moments(L, f, cs, c, &rho, &ux, &uy, &uz);
    double T = 0;
    for (int i = 0; i < Qg; i++) T += s->g[i * cs + c];
    if (s->buoyancy) {
      double buoy = s->g_gravity * s->beta * (T - s->T_ref);
      for (int i = 0; i < L->Q; i++) f[i * cs + c] += L->w[i] * 3.0 * rho * buoy * (double)L->ey[i];
    }
    const double oT = s->omega_T;
    for (int i = 0; i < Qg; i++) {
      double gi = s->g[i * cs + c];
      if (s->solid[c]) {
        gp[i * cs + c] = G.w[i] * T;
      } else {
        double eu = G.ex[i] * ux + G.ey[i] * uy + G.ez[i] * uz;
        double cs2inv = s->scalar_reduced && s->dims == 3 ? 4.0 : 3.0;
        double geq = G.w[i] * T * (1.0 + cs2inv * eu);
        gp[i * cs + c] = gi - oT * (gi - geq);
      }
    }
  }
  /* stream (periodic push) then Dirichlet rows y=0 (hot), y=Ny-1 (cold) */
#pragma omp parallel for collapse(2) schedule(static)
  for (int z = 0; z < nz; z++)
    for (int y = 0; y < ny; y++)
      for (int x = 0; x < nx; x++)
        for (int i = 0; i < Qg; i++) {
          int zn = wrapi(z + G.ez[i], nz), yn = wrapi(y + G.ey[i], ny), xn = wrapi(x + G.ex[i], nx);
          s->g[IDX(i, zn, yn, xn)] = gp[IDX(i, z, y, x)];
        }
  for (int i = 0; i < Qg; i++)
    for (int z = 0; z < nz; z++)
      for (int x = 0; x < nx; x++) {
        s->g[IDX(i, z, 0, x)] = G.w[i] * s->T_hot;
        s->g[IDX(i, z, ny - 1, x)] = G.w[i] * s->T_cold;
      }
}

/* Forces: forces.py:15-162, forces3d.py:8-171.  out[0..2] = F (x,y,z),
 * out[3..5] = pressure part, out[6..8] = viscous part, out[9..11] = moment
 * (Mx, My, Mz) about (cx, cy, cz).  profile[3*k + d] = force component d
 * summed over links whose y (2D) / z (3D) index is k. */
static void forces(const OracleLattice *s, const Lat *L, const double *fpre, const double *f,
                   double *out, double *profile) {
  const int nx = s->nx, ny = s->ny, nz = s->nz;
  const int64_t cs = (int64_t)nx * ny * nz;
  const int lw = s->dims == 3 ? 4 : 3;
  const int nprof = s->dims == 3 ? nz : ny;
  for (int k = 0; k < 12; k++) out[k] = 0.0;
  if (profile)
    for (int k = 0; k < 3 * nprof; k++) profile[k] = 0.0;
  for (int64_t k = 0; k < s->n_links; k++) {
    const int32_t *lk = s->links + k * lw;
    int i = lk[0], z = s->dims == 3 ? lk[1] : 0, y = lk[lw - 2], x = lk[lw - 1];
    int o = L->opp[i];
    int64_t c = CIDX(z, y, x);
    double fo = fpre[i * cs + c], fin = f[o * cs + c];
    double mom = fo + fin;
    double e[3] = {(double)L->ex[i], (double)L->ey[i], (double)L->ez[i]};
    double rho, ux, uy, uz;
    moments(L, fpre, cs, c, &rho, &ux, &uy, &uz);
    double eo = feq_i(L, i, rho, ux, uy, uz), ei = feq_i(L, o, rho, ux, uy, uz);
    double mp = eo + ei, mv = (fo - eo) + (fin - ei);
    double r[3] = {x - s->center[0], y - s->center[1], z - s->center[2]};
    double df[3] = {e[0] * mom, e[1] * mom, e[2] * mom};
    for (int d = 0; d < 3; d++) {
      out[d] += df[d];
      out[3 + d] += e[d] * mp;
      out[6 + d] += e[d] * mv;
    }
    out[9] += r[1] * df[2] - r[2] * df[1];
    out[10] += r[2] * df[0] - r[0] * df[2];
    out[11] += r[0] * df[1] - r[1] * df[0];
    if (profile) {
      int b = s->dims == 3 ? z : y;
      for (int d = 0; d < 3; d++) profile[3 * b + d] += df[d];
    }
  }
}

/* ------------------------------------------------------------------------ */
int oracle_step(OracleLattice *s, double *out_forces, double *out_profile) {
  Lat L;
  lat_init(&L, s->dims);
  if ((s->dims == 2 && s->nz != 1) || s->nx < 3 || s->ny < 2) return -1;
  if (s->ibm_enabled) return -2; /* IBM forcing is outside the hot path */
  const int64_t n = (int64_t)L.Q * s->nx * s->ny * s->nz;
  double *fp = s->work_a, *fs = s->work_b;
  /* 1. LES omega field from the pre-collision state (solver.py:289-295) */
  const double *om = NULL;
  if (s->les) {
    build_omega_field(s, &L, s->f, s->work_om);
    om = s->work_om;
  }
  /* 2. collision (MRT ignores the LES field: solver.py:298-300) */
  collide(s, &L, s->f, fp, s->collision == ORACLE_MRT ? NULL : om);
  /* 3-4. f_pre = f_post; push stream */
  stream(s, &L, fp, fs);
  /* 5. body force (3D only, solver3d.py:411-423) */
  if (s->dims == 3) body_force(s, &L, fs);
  /* 6. obstacle bounce-back */
  bounce_back(s, &L, fs, fp);
  /* 7-8. inlet / outlet */
  if (s->dims == 2)
    inlet_outlet_2d(s, fs);
  else
    inlet_outlet_3d(s, fs);
  /* 9. sponge */
  sponge(s, &L, fs);
  /* 10. walls */
  walls(s, &L, fs);
  /* 11. scalar */
  if (s->thermal) thermal(s, &L, fs);
  /* 12. commit */
  memcpy(s->f, fs, sizeof(double) * n);
  s->step_count += 1;
  /* 13. forces from f_pre and the new state */
  if (out_forces) forces(s, &L, fp, s->f, out_forces, out_profile);
  return 0;
}

int oracle_collide_only(OracleLattice *s, double *f_post) {
  /* Post-collision populations of the current state (test helper). */
  Lat L;
  lat_init(&L, s->dims);
  const double *om = NULL;
  if (s->les) {
    build_omega_field(s, &L, s->f, s->work_om);
    om = s->work_om;
  }
  collide(s, &L, s->f, f_post, s->collision == ORACLE_MRT ? NULL : om);
  return 0;
}

int oracle_omega_field(OracleLattice *s, double *om) {
  Lat L;
  lat_init(&L, s->dims);
  build_omega_field(s, &L, s->f, om);
  return 0;
}

int oracle_abi_version(void) { return 1; }
