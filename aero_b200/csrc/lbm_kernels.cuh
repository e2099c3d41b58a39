// lbm_kernels.cuh -- sm_100a kernels of the aero_b200 lattice Boltzmann engine.
//
// Stored state.  The population buffers hold POST-COLLISION populations P of
// the current step, as deviations from the rest weights (lbm_store.cuh), in
// SoA planes (Q, Nz, Ny, Nx) with a padded plane stride.  One fused pull
// kernel (k_step) then performs the rest of the reference step and the
// collision of the next one:
//
//   gather P at x - e_i (periodic)                 solver.py:351-353 (push stream)
//   uniform body force on fluid cells (3D)          solver3d.py:411-423
//   mid-link / Bouzidi bounce-back at link cells    solver.py:379-383
//   inlet (x = 0), outlet (x = Nx-1)                solver.py:385-407, solver3d.py:432-461
//   sponge relaxation                               solver.py:409-413
//   slip / no-slip / moving walls (y rows)          solver.py:415-424
//   Boussinesq buoyancy + scalar collide/push       solver.py:427-443
//   LES omega, then BGK / TRT / MRT collision       solver.py:287-345 (next step)
//
// Every step of that chain is cell-local once the gather is done, except the
// outlet copy (which reads the column x = Nx-2 after bounce-back): an outlet
// cell simply evaluates the chain for its x = Nx-2 neighbour.  The momentum-
// exchange forces of the step (forces.py:15-162, forces3d.py:8-171) need the
// pre-stream P and the post-BC state at link cells; k_step has both in
// registers at every link cell and writes that cell's twelve sums to a slot
// of lc_contrib, and k_finalize (launched after k_step) adds the slots in a
// fixed order in FP64.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "lbm_lattice.cuh"
#include "lbm_params.h"
#include "lbm_store.cuh"

// Kernel variants.  Every translation unit that includes the kernels compiles
// them into the inline namespace AERO_KNS (aero::gen by default), so a unit
// that fixes the feature word at compile time (AERO_FIXED_FEAT: the features
// of one lattice configuration, branches of the others removed) produces
// kernels of its own names beside the generic ones.
#ifndef AERO_KNS
#define AERO_KNS gen
#endif
#ifdef AERO_FIXED_FEAT
#define FEAT_OF(p) ((uint32_t)(AERO_FIXED_FEAT))
#else
#define FEAT_OF(p) ((p).feat)
#endif
#ifdef AERO_FIXED_WALL
#define WALL_OF(p) ((int32_t)(AERO_FIXED_WALL))
#else
#define WALL_OF(p) ((p).wall)
#endif

namespace aero {
inline namespace AERO_KNS {

#ifndef AERO_STEP_BLOCK
#define AERO_STEP_BLOCK 128
#endif
#ifndef AERO_STEP_MINB
#define AERO_STEP_MINB 8
#endif
constexpr int kStepBlock = AERO_STEP_BLOCK;  // threads along x per block
constexpr int kStepMinBlocks = AERO_STEP_MINB;  // resident blocks per SM the step kernel is built for
constexpr int kFinalizeBlock = 256;
constexpr int kFinalizeMaxBlocks = 64;

__device__ __forceinline__ int wrap_n(int v, int n) { return v < 0 ? v + n : (v >= n ? v - n : v); }
__device__ __forceinline__ int clamp_n(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }

// Cell indices are 32-bit (the host limits a lattice to fewer than 2^31
// cells); direction planes are addressed through warp-uniform base pointers.
template <class Real>
__device__ __forceinline__ uint32_t cell_index(const StepParams<Real> &p, int x, int y, int z) {
  return ((uint32_t)z * (uint32_t)p.ny + (uint32_t)y) * (uint32_t)p.nx + (uint32_t)x;
}

// Element offset of direction i at cell c: every population access is the
// buffer base plus one 32-bit offset (the host keeps Q * cs below 2^32), so
// the address costs one add and one wide multiply-add.
template <class Real>
__device__ __forceinline__ uint32_t elem(const StepParams<Real> &p, int i, uint32_t c) {
  return (uint32_t)i * (uint32_t)p.cs + c;
}

// (x, y, z) of cell index c in C order, in 32-bit arithmetic (a lattice has
// fewer than 2^31 cells; 64-bit division costs several times as many
// instructions).
__device__ __forceinline__ void cell_xyz(uint32_t c, uint32_t nx, uint32_t ny, int &x, int &y, int &z) {
  const uint32_t row = c / nx;
  const uint32_t zz = row / ny;
  x = (int)(c - row * nx);
  y = (int)(row - zz * ny);
  z = (int)zz;
}

// Link-cell slot of cell (x, y, z), or -1 when the cell has no link.
template <class Real>
__device__ __forceinline__ int64_t link_slot(const StepParams<Real> &p, int x, int y, int z) {
  const int64_t word = ((int64_t)z * p.ny + y) * p.nwx + (x >> 5);
  const uint32_t bits = __ldg(p.lbits + word);
  const int lane = x & 31;
  if (!((bits >> lane) & 1u)) return -1;
  return (int64_t)__ldg(p.loff + word) + __popc(bits & ((1u << lane) - 1u));
}

template <class Real> __device__ __forceinline__ Real sqrt_(Real v);
template <> __device__ __forceinline__ float sqrt_(float v) { return sqrtf(v); }
template <> __device__ __forceinline__ double sqrt_(double v) { return sqrt(v); }

// --------------------------------------------------------------------------
// Inlet / outlet / wall formulas in deviation form.  With f_i = w_i + d_i
// every reference formula keeps its shape because the weights cancel in
// pairs (w_i = w_opp(i) = w_mirror(i)) and the weighted sums used for the
// Zou-He densities total exactly 1.
// --------------------------------------------------------------------------

// Zou-He velocity inlet at x = 0.  2D: boundary.py:15-45; 3D: boundary3d.py:24-68
// (the 3D solver passes the perturbation as uz_amp, solver3d.py:447-452).
template <class L, class Real>
__device__ __forceinline__ void inlet_velocity(const StepParams<Real> &p, Real (&d)[L::Q], int y, int z,
                                               int64_t step_now) {
  const Real u0 = p.u0;
  if constexpr (L::DIMS == 2) {
    const Real rho_in = (Real(1) + (d[0] + d[2] + d[4]) + Real(2) * (d[3] + d[6] + d[7])) / (Real(1) - u0);
    d[1] = d[3] + Real(2.0 / 3.0) * rho_in * u0;
    d[5] = d[7] - Real(0.5) * (d[2] - d[4]) + Real(1.0 / 6.0) * rho_in * u0;
    d[8] = d[6] + Real(0.5) * (d[2] - d[4]) + Real(1.0 / 6.0) * rho_in * u0;
    if (p.pert_amp > Real(0)) {
      const double ph = 2.0 * 3.14159265358979323846 * (double)y / (double)(p.ny > 1 ? p.ny : 1) +
                        0.17 * (double)(step_now + 1);
      const Real uy = p.pert_amp * u0 * (Real)sin(ph);
      d[2] += uy * Real(0.25);
      d[4] -= uy * Real(0.25);
      d[5] += uy * Real(0.15);
      d[8] -= uy * Real(0.15);
    }
  } else {
    const Real Fm = d[2] + d[8] + d[10] + d[12] + d[14];
    const Real Fn = d[0] + d[3] + d[4] + d[5] + d[6] + d[15] + d[16] + d[17] + d[18];
    const Real rho_in = (Real(1) + Real(2) * Fm + Fn) / (Real(1) - u0);
    const Real cy = d[3] - d[4] + d[15] - d[16] + d[17] - d[18];
    Real cz = d[5] - d[6] + d[15] + d[16] - d[17] - d[18];
    if (p.pert_amp > Real(0)) {
      const double ph = 2.0 * 3.14159265358979323846 * (double)z / (double)(p.nz > 1 ? p.nz : 1) +
                        0.17 * (double)(step_now + 1);
      cz = cz + rho_in * (p.pert_amp * u0 * (Real)sin(ph));
    }
    const Real r6 = Real(1.0 / 6.0) * rho_in * u0;
    d[1] = d[2] + Real(1.0 / 3.0) * rho_in * u0;
    d[7] = d[10] + r6 - Real(0.5) * cy;
    d[9] = d[8] + r6 + Real(0.5) * cy;
    d[11] = d[14] + r6 - Real(0.5) * cz;
    d[13] = d[12] + r6 + Real(0.5) * cz;
  }
}

// Zou-He velocity inlet with per-row target velocities (ux = u0, transverse
// components from the inflow ring slot of this step): 2D boundary.py:48-65,
// 3D boundary3d.py:71-93, as the synthetic inflow calls them
// (solver.py:386-392, solver3d.py:436-445).  Unlike the uniform inlet these
// carry no transverse correction from the incoming populations.
// With FEAT_INFLOW_SEM (3D) the slot holds the SEM fluctuations (u', v', w')
// and the inlet is apply_inlet_sem_3d (boundary3d.py:96-137): ux = u0 + u',
// the uniform inlet's transverse corrections minus rho (v', w').
template <class L, class Real>
__device__ __forceinline__ void inlet_velocity_field(const StepParams<Real> &p, Real (&d)[L::Q], int y, int z,
                                                     int64_t step_now) {
  const int64_t plane = (int64_t)p.nz * p.ny;
  if constexpr (L::DIMS == 3) {
    if (FEAT_OF(p) & FEAT_INFLOW_SEM) {
      const Real *slot = p.inflow + (step_now % p.inflow_ring) * 3 * plane;
      const int64_t r = (int64_t)z * p.ny + y;
      const Real ux = p.u0 + slot[r];
      const Real den = Real(1) - ux > Real(1e-10) ? Real(1) - ux : Real(1e-10);
      const Real Fm = d[2] + d[8] + d[10] + d[12] + d[14];
      const Real Fn = d[0] + d[3] + d[4] + d[5] + d[6] + d[15] + d[16] + d[17] + d[18];
      const Real rho_in = (Real(1) + Real(2) * Fm + Fn) / den;
      const Real cy = (d[3] - d[4] + d[15] - d[16] + d[17] - d[18]) - rho_in * slot[plane + r];
      const Real cz = (d[5] - d[6] + d[15] + d[16] - d[17] - d[18]) - rho_in * slot[2 * plane + r];
      const Real r6 = Real(1.0 / 6.0) * rho_in * ux;
      d[1] = d[2] + Real(1.0 / 3.0) * rho_in * ux;
      d[7] = d[10] + r6 - Real(0.5) * cy;
      d[9] = d[8] + r6 + Real(0.5) * cy;
      d[11] = d[14] + r6 - Real(0.5) * cz;
      d[13] = d[12] + r6 + Real(0.5) * cz;
      return;
    }
  }
  const Real *slot = p.inflow + (step_now % p.inflow_ring) * (L::DIMS - 1) * plane;
  const int64_t r = (int64_t)z * p.ny + y;
  const Real ux = p.u0;
  const Real den = Real(1) - ux > Real(1e-8) ? Real(1) - ux : Real(1e-8);
  if constexpr (L::DIMS == 2) {
    const Real rho_in = (Real(1) + (d[0] + d[2] + d[4]) + Real(2) * (d[3] + d[6] + d[7])) / den;
    const Real cy = rho_in * slot[r];
    d[1] = d[3] + Real(2.0 / 3.0) * rho_in * ux;
    d[5] = d[7] - Real(0.5) * cy + Real(1.0 / 6.0) * rho_in * ux;
    d[8] = d[6] + Real(0.5) * cy + Real(1.0 / 6.0) * rho_in * ux;
  } else {
    const Real Fm = d[2] + d[8] + d[10] + d[12] + d[14];
    const Real Fn = d[0] + d[3] + d[4] + d[5] + d[6] + d[15] + d[16] + d[17] + d[18];
    const Real rho_in = (Real(1) + Real(2) * Fm + Fn) / den;
    const Real cy = rho_in * slot[r], cz = rho_in * slot[plane + r];
    const Real r6 = Real(1.0 / 6.0) * rho_in * ux;
    d[1] = d[2] + Real(1.0 / 3.0) * rho_in * ux;
    d[7] = d[10] + r6 - Real(0.5) * cy;
    d[9] = d[8] + r6 + Real(0.5) * cy;
    d[11] = d[14] + r6 - Real(0.5) * cz;
    d[13] = d[12] + r6 + Real(0.5) * cz;
  }
}

// Zou-He pressure inlet (2D): boundary.py:116-136
template <class Real>
__device__ __forceinline__ void inlet_pressure_2d(const StepParams<Real> &p, Real (&d)[9]) {
  const Real rin = p.rho_in;
  const Real ux = Real(1) - (Real(1) + (d[0] + d[2] + d[4]) + Real(2) * (d[3] + d[6] + d[7])) / rin;
  d[1] = d[3] + Real(2.0 / 3.0) * rin * ux;
  d[5] = d[7] - Real(0.5) * (d[2] - d[4]) + Real(1.0 / 6.0) * rin * ux;
  d[8] = d[6] + Real(0.5) * (d[2] - d[4]) + Real(1.0 / 6.0) * rin * ux;
}

// Zou-He pressure outlet (2D): boundary.py:139-159
template <class Real>
__device__ __forceinline__ void outlet_pressure_2d(const StepParams<Real> &p, Real (&d)[9]) {
  const Real ro = p.rho_out;
  const Real ux = Real(-1) + (Real(1) + (d[0] + d[2] + d[4]) + Real(2) * (d[1] + d[5] + d[8])) / ro;
  d[3] = d[1] - Real(2.0 / 3.0) * ro * ux;
  d[7] = d[5] + Real(0.5) * (d[2] - d[4]) - Real(1.0 / 6.0) * ro * ux;
  d[6] = d[8] - Real(0.5) * (d[2] - d[4]) - Real(1.0 / 6.0) * ro * ux;
}

template <class L, class Real>
__device__ __forceinline__ Real sum_dev(const Real (&d)[L::Q]) {
  Real s = Real(0);
  static_for<L::Q>([&](auto ic) { s += d[decltype(ic)::value]; });
  return s;
}

// Walls on the y = 0 / y = Ny-1 rows.  2D: boundary.py:162-226;
// 3D: boundary3d.py:205-271.
template <class L, class Real>
__device__ __forceinline__ void walls(const StepParams<Real> &p, Real (&d)[L::Q], bool bottom) {
  const Real k6 = Real(6.0 * (1.0 / 36.0));
  if constexpr (L::DIMS == 2) {
    if (WALL_OF(p) == WALL_SLIP) {
      if (bottom) { d[2] = d[4]; d[5] = d[8]; d[6] = d[7]; }
      else        { d[4] = d[2]; d[8] = d[5]; d[7] = d[6]; }
    } else if (WALL_OF(p) == WALL_NOSLIP) {
      if (bottom) { d[2] = d[4]; d[5] = d[7]; d[6] = d[8]; }
      else        { d[4] = d[2]; d[7] = d[5]; d[8] = d[6]; }
    } else {
      Real r = Real(1) + sum_dev<L>(d);
      r = r > Real(1e-12) ? r : Real(1e-12);
      if (bottom) {
        const Real m = k6 * r * p.wall_u_bottom;
        d[2] = d[4]; d[5] = d[7] + m; d[6] = d[8] - m;
      } else {
        const Real m = k6 * r * p.wall_u_top;
        d[4] = d[2]; d[7] = d[5] - m; d[8] = d[6] + m;
      }
    }
  } else {
    if (WALL_OF(p) == WALL_SLIP) {
      if (bottom) { d[3] = d[4]; d[7] = d[9]; d[8] = d[10]; d[15] = d[16]; d[17] = d[18]; }
      else        { d[4] = d[3]; d[9] = d[7]; d[10] = d[8]; d[16] = d[15]; d[18] = d[17]; }
    } else if (WALL_OF(p) == WALL_NOSLIP) {
      if (bottom) { d[3] = d[4]; d[7] = d[10]; d[8] = d[9]; d[15] = d[18]; d[17] = d[16]; }
      else        { d[4] = d[3]; d[10] = d[7]; d[9] = d[8]; d[18] = d[15]; d[16] = d[17]; }
    } else {
      Real r = Real(1) + sum_dev<L>(d);
      r = r > Real(1e-12) ? r : Real(1e-12);
      if (bottom) {
        const Real m = k6 * r * p.wall_u_bottom;
        d[3] = d[4]; d[7] = d[10] + m; d[8] = d[9] - m; d[15] = d[18]; d[17] = d[16];
      } else {
        const Real m = k6 * r * p.wall_u_top;
        d[4] = d[3]; d[10] = d[7] - m; d[9] = d[8] + m; d[18] = d[15]; d[16] = d[17];
      }
    }
  }
}

// --------------------------------------------------------------------------
// State of one cell after stream and every boundary condition of the
// reference step, evaluated from the post-collision buffer P.
// --------------------------------------------------------------------------

// Pull gather of row (y, z) straight from the population buffer: direction
// i of cell x reads P_i at (x - ex, y - ey, z - ez) with periodic wrap.
template <class L, class S, class Real>
struct GlobalGather {
  const StepParams<Real> &p;
  int y, z;
  __device__ __forceinline__ void operator()(int x, Real (&d)[L::Q]) const {
    using SO = StoreOps<S>;
    const S *P = static_cast<const S *>(p.P);
    // per axis only three source coordinates occur, so each source index is
    // one 3-way add
    const uint32_t nx = p.nx, nxy = (uint32_t)p.nx * (uint32_t)p.ny;
    const uint32_t xs_p = x == 0 ? nx - 1 : x - 1;            // ex = +1
    const uint32_t xs_m = x == p.nx - 1 ? 0 : x + 1;          // ex = -1
    const uint32_t ry_0 = (uint32_t)y * nx;
    const uint32_t ry_p = (y == 0 ? p.ny - 1 : y - 1) * nx;   // ey = +1
    const uint32_t ry_m = (y == p.ny - 1 ? 0 : y + 1) * nx;   // ey = -1
    uint32_t pz_0 = 0, pz_p = 0, pz_m = 0;
    if constexpr (L::DIMS == 3) {
      pz_0 = (uint32_t)z * nxy;
      pz_p = (z == 0 ? p.nz - 1 : z - 1) * nxy;
      pz_m = (z == p.nz - 1 ? 0 : z + 1) * nxy;
    }
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int ex = Dir<L, i>::x, ey = Dir<L, i>::y, ez = Dir<L, i>::z;
      const uint32_t src = (ex > 0 ? xs_p : (ex < 0 ? xs_m : (uint32_t)x)) +
                           (ey > 0 ? ry_p : (ey < 0 ? ry_m : ry_0)) +
                           (ez > 0 ? pz_p : (ez < 0 ? pz_m : pz_0));
      d[i] = SO::template load<i, L>(P, elem(p, i, src));
    });
  }
  // flag byte of cell x of the row
  __device__ __forceinline__ uint32_t flags(int x) const { return p.flags[cell_index(p, x, y, z)]; }
  // convective outlet state of the row, direction i
  __device__ __forceinline__ Real prev(int i) const { return p.prev[((int64_t)z * p.ny + y) * L::QP + i]; }
  // pre-stream population I of cell c (link cell slot `slot`)
  template <int I>
  __device__ __forceinline__ Real pre(uint32_t c, int64_t slot) const {
    (void)slot;
    return StoreOps<S>::template load<I, L>(static_cast<const S *>(p.P), elem(p, I, c));
  }
  // pre-stream population I of cell (xn, yn, zn) (the clipped neighbour of a
  // Bouzidi link with q >= 1/2)
  template <int I>
  __device__ __forceinline__ Real nbr(int xn, int yn, int zn, int64_t slot) const {
    (void)slot;
    return StoreOps<S>::template load<I, L>(static_cast<const S *>(p.P), elem(p, I, cell_index(p, xn, yn, zn)));
  }
  // stores the post-collision population I of cell x (index c) of the row
  template <int I>
  __device__ __forceinline__ void put(int x, uint32_t c, Real v) const {
    (void)x;
    StoreOps<S>::template store<I, L>(static_cast<S *>(p.Pn), elem(p, I, c), v);
  }
  static constexpr bool kAA = false;
};

// Element offset of the value V_I of cell (x, y, z) (index c) in the AA
// layout `layout`: plane opp(I) at c (layout 0), or plane I at the periodic
// neighbour x + e_I (layout 1).
template <class L, int I, class Real>
__device__ __forceinline__ uint32_t aa_own(const StepParams<Real> &p, int layout, int x, int y, int z, uint32_t c) {
  constexpr int o = L::opp[I];
  if (layout == 0) return elem(p, o, c);
  constexpr int ex = Dir<L, I>::x, ey = Dir<L, I>::y, ez = Dir<L, I>::z;
  const int xn = ex ? wrap_n(x + ex, p.nx) : x;
  const int yn = ey ? wrap_n(y + ey, p.ny) : y;
  const int zn = (L::DIMS == 3 && ez) ? wrap_n(z + ez, p.nz) : z;
  return elem(p, I, cell_index(p, xn, yn, zn));
}

// Population access of a step in the AA layout (one buffer, p.P == p.Pn).
// A step reading layout 0 gathers V_i(x - e_i) from plane opp(i) at the
// source cell and writes its result V'_i(x) to plane i at x + e_i (layout
// 1); a step reading layout 1 gathers from plane i at x itself and writes to
// plane opp(i) at x (layout 0).  Either way a cell writes exactly the slots
// it read, so the update is race-free in place.  The reads that cross cells
// within a step -- the pre-stream values of link cells (bounce-back and
// forces) and the pulled populations of plane nx-2 (which the outlet and
// recycling cells re-evaluate) -- come from the staging area k_aa_stage
// fills before the step.  RL is the layout the step reads when the kernel is
// compiled for one (0 or 1), or -1 for p.aa_layout at run time.
template <class L, class S, class Real, int RL = -1>
struct AAGather {
  const StepParams<Real> &p;
  int y, z;
  // the step kernel (one read layout compiled in): its outlet column may take
  // the state of x = nx-2 by warp shuffles (p.aa_shfl_out)
  static constexpr bool kStep = RL >= 0;
  __device__ __forceinline__ int layout() const { return RL >= 0 ? RL : p.aa_layout; }
  __device__ __forceinline__ void operator()(int x, Real (&d)[L::Q]) const {
    if (x == p.nx - 2 && p.stage_out) {
      const int64_t plane = (int64_t)p.ny * p.nz;
      const Real *so = static_cast<const Real *>(p.stage_out) + (int64_t)z * p.ny + y;
      static_for<L::Q>([&](auto ic) { d[decltype(ic)::value] = so[decltype(ic)::value * plane]; });
      return;
    }
    raw(x, d);
  }
  // the pulled population I of cell x straight from the buffer
  template <int I>
  __device__ __forceinline__ Real raw_one(int x) const {
    using SO = StoreOps<S>;
    const S *A = static_cast<const S *>(p.P);
    if (layout() == 1) return SO::template load<I, L>(A, elem(p, I, cell_index(p, x, y, z)));
    constexpr int ex = Dir<L, I>::x, ey = Dir<L, I>::y, ez = Dir<L, I>::z;
    constexpr int o = L::opp[I];
    const int xs = ex ? wrap_n(x - ex, p.nx) : x;
    const int ys = ey ? wrap_n(y - ey, p.ny) : y;
    const int zs = (L::DIMS == 3 && ez) ? wrap_n(z - ez, p.nz) : z;
    return SO::template load<I, L>(A, elem(p, o, cell_index(p, xs, ys, zs)));
  }
  // the pulled populations of cell x straight from the buffer
  __device__ __forceinline__ void raw(int x, Real (&d)[L::Q]) const {
    using SO = StoreOps<S>;
    const S *A = static_cast<const S *>(p.P);
    if (layout() == 1) {
      const uint32_t c = cell_index(p, x, y, z);
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        d[i] = SO::template load<i, L>(A, elem(p, i, c));
      });
      return;
    }
    const uint32_t nx = p.nx, nxy = (uint32_t)p.nx * (uint32_t)p.ny;
    const uint32_t xs_p = x == 0 ? nx - 1 : x - 1;
    const uint32_t xs_m = x == p.nx - 1 ? 0 : x + 1;
    const uint32_t ry_0 = (uint32_t)y * nx;
    const uint32_t ry_p = (y == 0 ? p.ny - 1 : y - 1) * nx;
    const uint32_t ry_m = (y == p.ny - 1 ? 0 : y + 1) * nx;
    uint32_t pz_0 = 0, pz_p = 0, pz_m = 0;
    if constexpr (L::DIMS == 3) {
      pz_0 = (uint32_t)z * nxy;
      pz_p = (z == 0 ? p.nz - 1 : z - 1) * nxy;
      pz_m = (z == p.nz - 1 ? 0 : z + 1) * nxy;
    }
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int ex = Dir<L, i>::x, ey = Dir<L, i>::y, ez = Dir<L, i>::z;
      const uint32_t src = (ex > 0 ? xs_p : (ex < 0 ? xs_m : (uint32_t)x)) +
                           (ey > 0 ? ry_p : (ey < 0 ? ry_m : ry_0)) +
                           (ez > 0 ? pz_p : (ez < 0 ? pz_m : pz_0));
      constexpr int o = L::opp[i];
      d[i] = SO::template load<i, L>(A, elem(p, o, src));
    });
  }
  __device__ __forceinline__ uint32_t flags(int x) const { return p.flags[cell_index(p, x, y, z)]; }
  __device__ __forceinline__ Real prev(int i) const { return p.prev[((int64_t)z * p.ny + y) * L::QP + i]; }
  template <int I>
  __device__ __forceinline__ Real pre(uint32_t c, int64_t slot) const {
    (void)c;
    return static_cast<const Real *>(p.stage_link)[slot * L::Q + I];
  }
  template <int I>
  __device__ __forceinline__ Real nbr(int xn, int yn, int zn, int64_t slot) const {
    (void)xn;
    (void)yn;
    (void)zn;
    return static_cast<const Real *>(p.stage_nb)[slot * L::Q + I];
  }
  template <int I>
  __device__ __forceinline__ void put(int x, uint32_t c, Real v) const {
    // layout 0 read -> write layout 1 (plane I at x + e_I); 1 -> 0 (plane opp(I) at x)
    StoreOps<S>::template store<I, L>(static_cast<S *>(p.Pn), aa_own<L, I>(p, 1 - layout(), x, y, z, c), v);
  }
  static constexpr bool kAA = true;
};

// Value V_I of cell (x, y, z) (index c) of a buffer that holds a state or
// a post-collision set stored per cell: plane I at c with two buffers, its
// AA slot in layout p.aa_layout in the AA layout.  Used where a kernel reads
// or writes a cell's own values only (the collision of a set state, the
// readers of the state, the initial state, the AA staging).
template <class L, int I, class Real>
__device__ __forceinline__ uint32_t own_elem(const StepParams<Real> &p, int x, int y, int z, uint32_t c) {
  return p.aa ? aa_own<L, I>(p, p.aa_layout, x, y, z, c) : elem(p, I, c);
}
template <class L, class S, int I, class Real>
__device__ __forceinline__ Real own_value(const StepParams<Real> &p, int x, int y, int z, uint32_t c) {
  return StoreOps<S>::template load<I, L>(static_cast<const S *>(p.P), own_elem<L, I>(p, x, y, z, c));
}

// Pull gather from a shared-memory tile: slab i (CAP elements) holds, for
// every row of the tile, the whole source row of direction i, i.e. row
// (y - ey, z - ez) with the y/z wrap already resolved when the tile was
// loaded, so only the x shift (periodic within the row) is left.  `row` is
// the tile-local offset of the cell's row (local row * nx).
// The stage also holds the tile's flag bytes (`fl` points at the row's first
// cell) and, for a convective outlet, the row's outlet state (`pv`).
template <class L, class S, class Real, int CAP>
struct SmemGather {
  const S *tile;
  uint32_t row;
  int nx;
  const uint8_t *fl;
  const Real *pv;
  const StepParams<Real> *pp;
  __device__ __forceinline__ uint32_t flags(int x) const { return fl[x]; }
  __device__ __forceinline__ Real prev(int i) const { return pv[i]; }
  template <int I>
  __device__ __forceinline__ Real pre(uint32_t c, int64_t slot) const {
    (void)slot;
    return StoreOps<S>::template load<I, L>(static_cast<const S *>(pp->P), elem(*pp, I, c));
  }
  template <int I>
  __device__ __forceinline__ Real nbr(int xn, int yn, int zn, int64_t slot) const {
    (void)slot;
    return StoreOps<S>::template load<I, L>(static_cast<const S *>(pp->P), elem(*pp, I, cell_index(*pp, xn, yn, zn)));
  }
  template <int I>
  __device__ __forceinline__ void put(int x, uint32_t c, Real v) const {
    (void)x;
    StoreOps<S>::template store<I, L>(static_cast<S *>(pp->Pn), elem(*pp, I, c), v);
  }
  static constexpr bool kAA = false;
  __device__ __forceinline__ void operator()(int x, Real (&d)[L::Q]) const {
    using SO = StoreOps<S>;
    const uint32_t o_0 = row + (uint32_t)x;
    const uint32_t o_p = row + (uint32_t)(x == 0 ? nx - 1 : x - 1);   // ex = +1
    const uint32_t o_m = row + (uint32_t)(x == nx - 1 ? 0 : x + 1);   // ex = -1
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      constexpr int ex = Dir<L, i>::x;
      const uint32_t o = ex > 0 ? o_p : (ex < 0 ? o_m : o_0);
      d[i] = SO::template lds<i, L>(tile + i * CAP, o);
    });
  }
};

// gather + body force + obstacle bounce-back + inlet (everything the
// reference applies before the outlet copy reads column Nx-2).
template <class L, class S, class Real, class Gather>
__device__ __forceinline__ void partial_state(const StepParams<Real> &p, int x, int y, int z, int64_t step_now,
                                              Real (&d)[L::Q], const Gather &gather) {
  gather(x, d);
  const uint32_t c = cell_index(p, x, y, z);
  if constexpr (L::DIMS == 3) {
    // Guo-style uniform body force on fluid cells (ibm_guo.py:263-301)
    if ((FEAT_OF(p) & FEAT_BODY_FORCE) && !(gather.flags(x) & FLAG_SOLID)) {
      Real drho = 0, jx = 0, jy = 0, jz = 0;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        drho += d[i];
        if (Dir<L, i>::x) jx += Dir<L, i>::x * d[i];
        if (Dir<L, i>::y) jy += Dir<L, i>::y * d[i];
        if (Dir<L, i>::z) jz += Dir<L, i>::z * d[i];
      });
      const Real rho = Real(1) + drho;
      if (rho > Real(0)) {
        const Real ux = jx / rho, uy = jy / rho, uz = jz / rho;
        const Real uf = ux * p.bf_x + uy * p.bf_y + uz * p.bf_z;
        static_for<L::Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          const Real eu = Dir<L, i>::x * ux + Dir<L, i>::y * uy + Dir<L, i>::z * uz;
          const Real ef = Dir<L, i>::x * p.bf_x + Dir<L, i>::y * p.bf_y + Dir<L, i>::z * p.bf_z;
          const Real term = (ef - uf) * Real(3) + (eu * ef) * Real(9);
          d[i] += p.bf_coeff * Real(Dir<L, i>::w) * rho * term;
        });
      }
    }
  }
  // obstacle bounce-back (boundary.py:283-352, boundary3d.py:333-393)
  if ((FEAT_OF(p) & FEAT_OBSTACLE_BB) && (gather.flags(x) & FLAG_LINK)) {
    const int64_t slot = link_slot(p, x, y, z);
    if (slot >= 0) {
      const uint32_t mask = __ldg(p.lc_mask + slot);
      const bool bouzidi = FEAT_OF(p) & FEAT_BOUZIDI;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (i > 0) {
          if ((mask >> i) & 1u) {
            constexpr int o = L::opp[i];
            const Real fi = gather.template pre<i>(c, slot);
            if (!bouzidi) {
              d[o] = fi;
            } else {
              const Real q = (Real)__ldg(p.lc_q + slot * L::Q + i);
              if (q < Real(0.5)) {
                const Real fo = gather.template pre<o>(c, slot);
                d[o] = Real(2) * q * fi + (Real(1) - Real(2) * q) * fo;
              } else {
                const int xn = clamp_n(x + Dir<L, o>::x, p.nx);
                const int yn = clamp_n(y + Dir<L, o>::y, p.ny);
                const int zn = L::DIMS == 3 ? clamp_n(z + Dir<L, o>::z, p.nz) : 0;
                const Real fn = gather.template nbr<i>(xn, yn, zn, slot);
                const Real inv2q = Real(1) / (Real(2) * q);
                d[o] = inv2q * fi + (Real(1) - inv2q) * fn;
              }
            }
          }
        }
      });
    }
  }
  if ((FEAT_OF(p) & FEAT_OPEN) && x == 0) {
    if (p.inlet == INLET_VELOCITY) {
      if (FEAT_OF(p) & FEAT_INFLOW_FIELD)
        inlet_velocity_field<L>(p, d, y, z, step_now);
      else
        inlet_velocity<L>(p, d, y, z, step_now);
    } else if constexpr (L::DIMS == 2) {
      if (p.inlet == INLET_PRESSURE) inlet_pressure_2d(p, d);
    }
  }
}

// Thermal outputs of the state evaluation.
template <class Real>
struct ScalarCtx {
  Real T;       // sum of the current scalar populations at the cell
  Real u[3];    // flow velocity before buoyancy (drives the scalar collision)
  // moments (rho - 1, j) of the final state, buoyancy included: buoyancy
  // adds rho g beta (T - T_ref) to j_y and nothing to rho, so the collision
  // need not sum the populations again
  Real m[4];
  bool m_set = false;
};

// Full post-BC state.  When prev_out is non-null the convective outlet writes
// its advanced state there (only the step kernels do).
template <class L, class S, class Real, class Gather>
__device__ __forceinline__ void full_state(const StepParams<Real> &p, int x, int y, int z, int64_t step_now,
                                           Real (&d)[L::Q], Real *prev_out, ScalarCtx<Real> *sc,
                                           const Gather &gather) {
  const bool open = FEAT_OF(p) & FEAT_OPEN;
  const bool copy_out =
      open && x == p.nx - 1 && (p.outlet == OUTLET_CONVECTIVE || p.outlet == OUTLET_ZEROGRAD);
  bool shfl = false;
  if constexpr (Gather::kAA) shfl = Gather::kStep && p.aa_shfl_out;
  partial_state<L, S, Real>(p, copy_out && !shfl ? p.nx - 2 : x, y, z, step_now, d, gather);
  if constexpr (Gather::kAA) {
    // In place, the x = nx-2 thread overwrites the slots it read, so the
    // outlet thread takes that cell's post-boundary state from its lane
    // instead of re-reading them.  Warp-uniform: the warp holding x = nx-1,
    // whose lanes 0 .. (nx-1) mod 32 have cells (warps cover 32 consecutive
    // x of one row).
    if (shfl && (x | 31) >= p.nx - 1) {
      const int last = (p.nx - 1) & 31;
      const unsigned lanes = last == 31 ? 0xffffffffu : (2u << last) - 1u;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const Real v = __shfl_up_sync(lanes, d[i], 1);
        if (copy_out) d[i] = v;
      });
    }
  }
  if (copy_out) {
    if (p.outlet == OUTLET_CONVECTIVE) {
      // boundary.py:78-113, boundary3d.py:149-164
      Real u = p.u0 < Real(0) ? Real(0) : (p.u0 > Real(1) ? Real(1) : p.u0);
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        d[i] = (Real(1) - u) * gather.prev(i) + u * d[i];
        if (prev_out) prev_out[((int64_t)z * p.ny + y) * L::QP + i] = d[i];
      });
    }
  } else if constexpr (L::DIMS == 2) {
    if (open && x == p.nx - 1 && p.outlet == OUTLET_PRESSURE) outlet_pressure_2d(p, d);
  }
  if constexpr (L::DIMS == 3) {
    // recycling inlet (boundary3d.py:172-198, applied after bounce-back as in
    // solver3d.py:460-461): the inlet plane takes the equilibrium of the
    // x = nx-2 cell's post-bounce-back state with its velocity scaled so that
    // the plane's mean ux becomes u0
    if ((FEAT_OF(p) & FEAT_RECYCLE) && x == 0) {
      Real r[L::Q];
      partial_state<L, S, Real>(p, p.nx - 2, y, z, step_now, r, gather);
      Real drho = 0, jx = 0, jy = 0, jz = 0;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        drho += r[i];
        if (Dir<L, i>::x) jx += Dir<L, i>::x * r[i];
        if (Dir<L, i>::y) jy += Dir<L, i>::y * r[i];
        if (Dir<L, i>::z) jz += Dir<L, i>::z * r[i];
      });
      const Real rho = Real(1) + drho;
      const Real inv = rho > Real(0) ? Real(1) / rho : Real(0);
      const double mean = *p.recycle_mean;
      const Real scale = fabs(mean) < 1e-12 ? Real(1) : (Real)((double)p.u0 / mean);
      const Real ux = jx * inv * scale, uy = jy * inv * scale, uz = jz * inv * scale;
      const Real usq = ux * ux + uy * uy + uz * uz;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const Real eu = Dir<L, i>::x * ux + Dir<L, i>::y * uy + Dir<L, i>::z * uz;
        d[i] = Real(Dir<L, i>::w) * (drho + rho * (Real(3) * eu + Real(4.5) * eu * eu - Real(1.5) * usq));
      });
    }
  }
  // sponge (sponge.py:8-70)
  if ((FEAT_OF(p) & FEAT_SPONGE) && x >= p.sponge_start) {
    const double frac = (double)(x - p.sponge_start + 1) / (double)(p.sponge_thickness > 1 ? p.sponge_thickness : 1);
    const Real sg = (Real)((double)p.sponge_sigma_max * frac * frac);
    if (sg > Real(0)) {
      const Real drho = sum_dev<L>(d);
      const Real rho = Real(1) + drho;
      const Real u0 = p.u0, usq = u0 * u0;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        const Real eu = Dir<L, i>::x * u0;
        const Real deq = Real(Dir<L, i>::w) * (drho + rho * (Real(3) * eu + Real(4.5) * eu * eu - Real(1.5) * usq));
        d[i] = (Real(1) - sg) * d[i] + sg * deq;
      });
    }
  }
  if (WALL_OF(p) != WALL_NONE) {
    if (y == 0) walls<L>(p, d, true);
    if (y == p.ny - 1) walls<L>(p, d, false);
  }
  if (FEAT_OF(p) & FEAT_THERMAL) {
    // thermal.py:103-124 / :206-222 with the order of solver.py:432-439
    const uint32_t c = cell_index(p, x, y, z);
    Real T = 0;
    if (FEAT_OF(p) & FEAT_SCALAR_REDUCED) {
      using G = typename ScalarReduced<L>::Lat;
      static_for<G::Q>([&](auto ic) { T += p.g[elem(p, decltype(ic)::value, c)]; });
    } else {
      static_for<L::Q>([&](auto ic) { T += p.g[elem(p, decltype(ic)::value, c)]; });
    }
    Real drho = 0, jx = 0, jy = 0, jz = 0;
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      drho += d[i];
      if (Dir<L, i>::x) jx += Dir<L, i>::x * d[i];
      if (Dir<L, i>::y) jy += Dir<L, i>::y * d[i];
      if (Dir<L, i>::z) jz += Dir<L, i>::z * d[i];
    });
    const Real rho = Real(1) + drho;
    if (sc) {
      const Real inv = rho > Real(0) ? Real(1) / rho : Real(0);
      sc->T = T;
      sc->u[0] = jx * inv;
      sc->u[1] = jy * inv;
      sc->u[2] = jz * inv;
    }
    Real jy_final = jy;
    if (FEAT_OF(p) & FEAT_BUOYANCY) {
      const Real buoy = p.gbeta * (T - p.T_ref);
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        if constexpr (Dir<L, i>::y != 0) d[i] += Real(Dir<L, i>::w) * Real(3) * rho * buoy * Real(Dir<L, i>::y);
      });
      jy_final += rho * buoy;
    }
    if (sc) {
      sc->m[0] = drho;
      sc->m[1] = jx;
      sc->m[2] = jy_final;
      sc->m[3] = jz;
      sc->m_set = true;
    }
  }
}

template <class L, class S, class Real>
__device__ __forceinline__ void full_state(const StepParams<Real> &p, int x, int y, int z, int64_t step_now,
                                           Real (&d)[L::Q], Real *prev_out, ScalarCtx<Real> *sc) {
  full_state<L, S, Real>(p, x, y, z, step_now, d, prev_out, sc, GlobalGather<L, S, Real>{p, y, z});
}

// --------------------------------------------------------------------------
// LES relaxation rate (les.py:24-78, :177-266, :273-344).
// --------------------------------------------------------------------------
// The eddy-viscosity model on the velocity gradient g[a][b] = d u_a / d x_b
// (central differences, halved), then omega = 1 / (3 (nu0 + nu_t) + 1/2).
template <class L, class Real>
__device__ __forceinline__ Real les_rate_from_gradient(const StepParams<Real> &p, const Real (&g)[3][3],
                                                       uint32_t c) {
  Real nu_t;
  Real cs2 = p.les_cs2;
  if (FEAT_OF(p) & FEAT_LES_CS_FIELD) {
    const Real cc = p.cs_cell[c];
    cs2 = cc * cc;
  }
  constexpr int D = L::DIMS;
  if (FEAT_OF(p) & FEAT_LES_WALE) {
    Real s_sq = 0, sd_sq = 0, gsq[3][3], tr = 0;
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        const Real sab = Real(0.5) * (g[a][b] + g[b][a]);
        s_sq += sab * sab;
        Real acc = 0;
#pragma unroll
        for (int k = 0; k < D; k++) acc += g[a][k] * g[k][b];
        gsq[a][b] = acc;
      }
#pragma unroll
    for (int a = 0; a < D; a++) tr += gsq[a][a];
    tr = tr / Real(D);
#pragma unroll
    for (int a = 0; a < D; a++)
#pragma unroll
      for (int b = 0; b < D; b++) {
        const Real sd = Real(0.5) * (gsq[a][b] + gsq[b][a]) - (a == b ? tr : Real(0));
        sd_sq += sd * sd;
      }
    // pow(sd, 1.5) / (pow(s, 2.5) + pow(sd, 1.25) + 1e-30) via square roots
    const Real r_sd = sqrt_(sd_sq), r_s = sqrt_(s_sq);
    const Real num = sd_sq * r_sd;
    const Real den = s_sq * s_sq * r_s + sd_sq * sqrt_(r_sd) + Real(1e-30);
    nu_t = cs2 * num / den;
  } else {
    const Real s11 = g[0][0], s22 = g[1][1], s33 = g[2][2];
    const Real s12 = Real(0.5) * (g[0][1] + g[1][0]);
    const Real s13 = Real(0.5) * (g[0][2] + g[2][0]);
    const Real s23 = Real(0.5) * (g[1][2] + g[2][1]);
    Real smag;
    if constexpr (D == 2)
      smag = sqrt_(Real(2) * (s11 * s11 + s22 * s22 + Real(2) * s12 * s12));
    else
      smag = sqrt_(Real(2) * (s11 * s11 + s22 * s22 + s33 * s33) +
                    Real(4) * (s12 * s12 + s13 * s13 + s23 * s23));
    nu_t = cs2 * smag;
  }
  return Real(1) / (Real(3) * (p.base_nu + nu_t) + Real(0.5));
}

// Whether the LES rate applies at (x, y, z): interior cells (the edge planes
// keep nu_t = 0, les.py:55-57, no periodic wrap) that are not solid.
template <class L, class Real>
__device__ __forceinline__ bool les_interior(const StepParams<Real> &p, int x, int y, int z) {
  bool interior = x >= 1 && x <= p.nx - 2 && y >= 1 && y <= p.ny - 2;
  if constexpr (L::DIMS == 3) interior = interior && z >= 1 && z <= p.nz - 2;
  return interior;
}

// LES relaxation rate from the velocity side buffer (les.py:24-78,
// :177-266, :273-344).  Edge planes and solid cells keep the base rate.
template <class L, class Real>
__device__ __forceinline__ Real les_omega(const StepParams<Real> &p, int x, int y, int z, uint32_t c, bool solid) {
  if (!les_interior<L>(p, x, y, z) || solid) return Real(1) / (Real(3) * p.base_nu + Real(0.5));
  const Real *UX = p.U, *UY = p.U + p.cs, *UZ = p.U + 2 * p.cs;
  const uint32_t sx = 1, sy = p.nx;
  Real g[3][3];
  g[0][0] = Real(0.5) * (UX[c + sx] - UX[c - sx]);
  g[0][1] = Real(0.5) * (UX[c + sy] - UX[c - sy]);
  g[1][0] = Real(0.5) * (UY[c + sx] - UY[c - sx]);
  g[1][1] = Real(0.5) * (UY[c + sy] - UY[c - sy]);
  g[0][2] = g[1][2] = g[2][0] = g[2][1] = g[2][2] = Real(0);
  if constexpr (L::DIMS == 3) {
    const uint32_t sz = (uint32_t)p.nx * (uint32_t)p.ny;
    g[0][2] = Real(0.5) * (UX[c + sz] - UX[c - sz]);
    g[1][2] = Real(0.5) * (UY[c + sz] - UY[c - sz]);
    g[2][0] = Real(0.5) * (UZ[c + sx] - UZ[c - sx]);
    g[2][1] = Real(0.5) * (UZ[c + sy] - UZ[c - sy]);
    g[2][2] = Real(0.5) * (UZ[c + sz] - UZ[c - sz]);
  }
  return les_rate_from_gradient<L>(p, g, c);
}

// --------------------------------------------------------------------------
// Collision (deviation form).  BGK: kernels.py:42-92; TRT: kernels_trt.py:
// 125-174 with trt2d.py:8-18; MRT: kernels_mrt.py:190-241,
// kernels3d_mrt.py:24-82.  Solid cells relax toward feq(rho, 0).
// --------------------------------------------------------------------------
// D3Q19 MRT in the cubic-symmetry-adapted basis.  The reference operator
// (dense M19 / pseudo-inverse, see lbm_mrt.cpp) commutes with the lattice's
// cubic symmetry, so in coordinates built from sums and differences of
// populations it splits into: a 3x3 block on the scalars (rest, face sum,
// edge sum), one 2x2 block shared by both components of the face/edge
// doublets, the scalar 1 - omega on the three shear-type edge differences, a
// 2x2 block shared by the x, y, z momentum-like pairs, and zero on the three
// remaining odd edge combinations (the directions the rank-16 basis projects
// out).  The host derives the block entries from the dense operator and
// checks that nothing outside them is non-zero.
// 1 / rho for rho > 0, else 0 (the reference's guard in compute_macroscopic)
template <class Real>
AERO_HD Real pos_recip(Real rho) {
  return rho > Real(0) ? Real(1) / rho : Real(0);
}

// The operator on the values V of one cell (V = Real), or of two cells at
// once (V = F2, lbm_pair.cuh: every operation one packed FP32 instruction).
template <class Real, class V>
AERO_HD V mrt3_core(const Mrt3Adapted<Real> &m, V (&d)[19], bool solid) {
  // pair sums (even) and differences (odd)
  const V X = d[1] + d[2], Y = d[3] + d[4], Z = d[5] + d[6];
  const V p710 = d[7] + d[10], p89 = d[8] + d[9], p1114 = d[11] + d[14], p1213 = d[12] + d[13];
  const V p1518 = d[15] + d[18], p1617 = d[16] + d[17];
  const V t1 = d[1] - d[2], t2 = d[3] - d[4], t3 = d[5] - d[6];
  const V q710 = d[7] - d[10], q89 = d[8] - d[9], q1114 = d[11] - d[14], q1213 = d[12] - d[13];
  const V q1518 = d[15] - d[18], q1617 = d[16] - d[17];
  // even adapted coordinates
  const V Pxy = p710 + p89, Pxz = p1114 + p1213, Pyz = p1518 + p1617;
  const V g0 = d[0], g1 = X + Y + Z, g2 = Pxy + Pxz + Pyz;
  const V g3 = Real(2) * X - Y - Z, g4 = Y - Z;
  const V g5 = Real(2) * Pyz - Pxz - Pxy, g6 = Pxz - Pxy;
  const V g7 = p710 - p89, g8 = p1114 - p1213, g9 = p1518 - p1617;
  // odd adapted coordinates (momentum-like edge sums)
  const V Wx = (q710 - q89) + (q1114 - q1213);
  const V Wy = (q710 + q89) + (q1518 - q1617);
  const V Wz = (q1114 + q1213) + (q1518 + q1617);
  // moments
  const V drho = g0 + g1 + g2;
  const V jx = t1 + Wx, jy = t2 + Wy, jz = t3 + Wz;
  const V rho = Real(1) + drho;
  const V inv = pos_recip(rho);
  V ux = jx * inv, uy = jy * inv, uz = jz * inv;
  if (solid) ux = uy = uz = V(Real(0));
  const V rux = rho * ux, ruy = rho * uy, ruz = rho * uz;
  const V kxx = rux * ux, kyy = ruy * uy, kzz = ruz * uz;
  const V ru2 = kxx + kyy + kzz;
  const V mE1 = Real(2) * kxx - kyy - kzz, mE2 = kyy - kzz;
  // blocks
  const V h0 = m.a1[0] * g0 + m.a1[1] * g1 + m.a1[2] * g2 + m.ca1[0] * drho + m.ca1[1] * ru2;
  const V h1 = m.a1[3] * g0 + m.a1[4] * g1 + m.a1[5] * g2 + m.ca1[2] * drho + m.ca1[3] * ru2;
  const V h2 = m.a1[6] * g0 + m.a1[7] * g1 + m.a1[8] * g2 + m.ca1[4] * drho + m.ca1[5] * ru2;
  const V h3 = m.e[0] * g3 + m.e[1] * g5 + m.ce[0] * mE1;
  const V h5 = m.e[2] * g3 + m.e[3] * g5 + m.ce[1] * mE1;
  const V h4 = m.e[0] * g4 + m.e[1] * g6 + m.ce[0] * mE2;
  const V h6 = m.e[2] * g4 + m.e[3] * g6 + m.ce[1] * mE2;
  const V h7 = m.t2 * g7 + m.ct2 * (rux * uy);
  const V h8 = m.t2 * g8 + m.ct2 * (rux * uz);
  const V h9 = m.t2 * g9 + m.ct2 * (ruy * uz);
  const V vx = m.v[0] * t1 + m.v[1] * Wx + m.cv[0] * rux;
  const V Vx = m.v[2] * t1 + m.v[3] * Wx + m.cv[1] * rux;
  const V vy = m.v[0] * t2 + m.v[1] * Wy + m.cv[0] * ruy;
  const V Vy = m.v[2] * t2 + m.v[3] * Wy + m.cv[1] * ruy;
  const V vz = m.v[0] * t3 + m.v[1] * Wz + m.cv[0] * ruz;
  const V Vz = m.v[2] * t3 + m.v[3] * Wz + m.cv[1] * ruz;
  // back to populations
  const V Xn = (h1 + h3) * Real(1.0 / 3.0);
  const V Yn = Real(0.5) * (h1 - Xn + h4), Zn = Real(0.5) * (h1 - Xn - h4);
  const V Pyzn = (h2 + h5) * Real(1.0 / 3.0);
  const V Pxzn = Real(0.5) * (h2 - Pyzn + h6), Pxyn = Real(0.5) * (h2 - Pyzn - h6);
  const V p710n = Real(0.5) * (Pxyn + h7), p89n = Real(0.5) * (Pxyn - h7);
  const V p1114n = Real(0.5) * (Pxzn + h8), p1213n = Real(0.5) * (Pxzn - h8);
  const V p1518n = Real(0.5) * (Pyzn + h9), p1617n = Real(0.5) * (Pyzn - h9);
  const V q710n = Real(0.25) * (Vx + Vy), q89n = Real(0.25) * (Vy - Vx);
  const V q1114n = Real(0.25) * (Vx + Vz), q1213n = Real(0.25) * (Vz - Vx);
  const V q1518n = Real(0.25) * (Vy + Vz), q1617n = Real(0.25) * (Vz - Vy);
  d[0] = h0;
  d[1] = Real(0.5) * (Xn + vx);
  d[2] = Real(0.5) * (Xn - vx);
  d[3] = Real(0.5) * (Yn + vy);
  d[4] = Real(0.5) * (Yn - vy);
  d[5] = Real(0.5) * (Zn + vz);
  d[6] = Real(0.5) * (Zn - vz);
  d[7] = Real(0.5) * (p710n + q710n);
  d[10] = Real(0.5) * (p710n - q710n);
  d[8] = Real(0.5) * (p89n + q89n);
  d[9] = Real(0.5) * (p89n - q89n);
  d[11] = Real(0.5) * (p1114n + q1114n);
  d[14] = Real(0.5) * (p1114n - q1114n);
  d[12] = Real(0.5) * (p1213n + q1213n);
  d[13] = Real(0.5) * (p1213n - q1213n);
  d[15] = Real(0.5) * (p1518n + q1518n);
  d[18] = Real(0.5) * (p1518n - q1518n);
  d[16] = Real(0.5) * (p1617n + q1617n);
  d[17] = Real(0.5) * (p1617n - q1617n);
  return rho;
}

template <class Real>
AERO_HD Real mrt3_adapted(const StepParams<Real> &p, Real (&d)[19], bool solid, Real drho_in) {
  (void)drho_in;
  return mrt3_core<Real, Real>(p.mrt3, d, solid);
}

template <class L, class Real, int COLL>
AERO_HD Real collide(const StepParams<Real> &p, Real (&d)[L::Q], bool solid, Real om, bool per_cell_omega,
                     const Real *mom = nullptr) {
  if constexpr (COLL == COLL_MRT && L::DIMS == 3) {
    (void)om;
    (void)per_cell_omega;
    (void)mom;
    return mrt3_adapted<Real>(p, d, solid, Real(0));
  }
  // moments of d: given (the state evaluation's, buoyancy included) or summed
  Real drho = 0, jx = 0, jy = 0, jz = 0;
  if (mom) {
    drho = mom[0];
    jx = mom[1];
    jy = mom[2];
    jz = mom[3];
  } else {
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      drho += d[i];
      if (Dir<L, i>::x) jx += Dir<L, i>::x * d[i];
      if (Dir<L, i>::y) jy += Dir<L, i>::y * d[i];
      if (Dir<L, i>::z) jz += Dir<L, i>::z * d[i];
    });
  }
  const Real rho = Real(1) + drho;
  const Real inv = rho > Real(0) ? Real(1) / rho : Real(0);
  Real ux = jx * inv, uy = jy * inv, uz = jz * inv;
  if (solid) ux = uy = uz = Real(0);
  if constexpr (COLL == COLL_MRT) {
    // D2Q9: dense blocks in the pair basis (see lbm_mrt.cpp)
    constexpr int NE = L::NP + 1, NO = L::NP, KE = 4, KO = 2;
    Real s[NE], t[NO], me[KE], mo[KO];
    s[0] = d[0];
    static_for<NO>([&](auto pc) {
      constexpr int k = decltype(pc)::value;
      constexpr int i = L::pair[k], o = L::opp[L::pair[k]];
      s[k + 1] = d[i] + d[o];
      t[k] = d[i] - d[o];
    });
    const Real rux = rho * ux, ruy = rho * uy;
    me[0] = drho;
    me[1] = rux * ux;
    me[2] = ruy * uy;
    me[3] = rux * uy;
    mo[0] = rux;
    mo[1] = ruy;
    Real sp[NE], tp[NO];
#pragma unroll
    for (int r = 0; r < NE; r++) {
      Real acc = 0;
#pragma unroll
      for (int k = 0; k < KE; k++) acc += p.mrt.Ce[r * 7 + k] * me[k];
#pragma unroll
      for (int k = 0; k < NE; k++) acc += p.mrt.Ae[r * 10 + k] * s[k];
      sp[r] = acc;
    }
#pragma unroll
    for (int r = 0; r < NO; r++) {
      Real acc = 0;
#pragma unroll
      for (int k = 0; k < KO; k++) acc += p.mrt.Co[r * 3 + k] * mo[k];
#pragma unroll
      for (int k = 0; k < NO; k++) acc += p.mrt.Ao[r * 9 + k] * t[k];
      tp[r] = acc;
    }
    // rows 1.. of the even block and the odd block carry the factor 1/2 of
    // f_i = (s + t) / 2, f_opp = (s - t) / 2 (folded in on the host)
    d[0] = sp[0];
    static_for<NO>([&](auto pc) {
      constexpr int k = decltype(pc)::value;
      constexpr int i = L::pair[k], o = L::opp[L::pair[k]];
      d[i] = sp[k + 1] + tp[k];
      d[o] = sp[k + 1] - tp[k];
    });
    (void)om;
    (void)per_cell_omega;
  } else {
    // BGK / TRT.  The equilibrium of an opposite pair (i, o) splits into an
    // even part w (drho + rho (4.5 (e.u)^2 - 1.5 u^2)), shared by both, and an
    // odd part 3 w rho (e.u), taken with opposite signs (the reference's
    // w rho (1 + 3 e.u + 4.5 (e.u)^2 - 1.5 u^2) in deviation form); each part
    // is evaluated once per pair.  The update is applied as a correction to d
    // (d + omega (feq - d)), which keeps the FP32 rounding small.
    const Real usq = ux * ux + uy * uy + uz * uz;
    const Real u15 = Real(1.5) * usq;
    const Real deq0 = Real(Dir<L, 0>::w) * (drho - rho * u15);
    if constexpr (COLL == COLL_TRT) {
      Real sm = p.trt_sminus;
      if (per_cell_omega) {
        const Real tau = Real(1) / om, lam = p.trt_lambda;
        const Real tp = lam * tau + (Real(1) - lam);
        const Real tm = (tp * tau - Real(0.5)) / (tp - Real(0.5));
        sm = Real(1) / tm;
      }
      d[0] = d[0] + om * (deq0 - d[0]);  // the rest population is even
      static_for<L::NP>([&](auto pc) {
        constexpr int k = decltype(pc)::value;
        constexpr int i = L::pair[k], o = L::opp[L::pair[k]];
        const Real eu = Dir<L, i>::x * ux + Dir<L, i>::y * uy + Dir<L, i>::z * uz;
        const Real ep = Real(Dir<L, i>::w) * (drho + rho * (Real(4.5) * eu * eu - u15));
        const Real em = Real(Dir<L, i>::w) * (Real(3) * rho * eu);
        const Real fp = Real(0.5) * (d[i] + d[o]), fm = Real(0.5) * (d[i] - d[o]);
        const Real a = om * (ep - fp), b = sm * (em - fm);
        d[i] = d[i] + (a + b);
        d[o] = d[o] + (a - b);
      });
    } else {
      d[0] = d[0] + om * (deq0 - d[0]);
      static_for<L::NP>([&](auto pc) {
        constexpr int k = decltype(pc)::value;
        constexpr int i = L::pair[k], o = L::opp[L::pair[k]];
        const Real eu = Dir<L, i>::x * ux + Dir<L, i>::y * uy + Dir<L, i>::z * uz;
        const Real ep = Real(Dir<L, i>::w) * (drho + rho * (Real(4.5) * eu * eu - u15));
        const Real em = Real(Dir<L, i>::w) * (Real(3) * rho * eu);
        d[i] = d[i] + om * ((ep + em) - d[i]);
        d[o] = d[o] + om * ((ep - em) - d[o]);
      });
    }
    (void)per_cell_omega;
  }
  return rho;
}

// Scalar lattice collision + push (thermal.py:47-100, :149-203).  Rows y = 0
// and y = Ny-1 are Dirichlet rows: every population there is overwritten by
// w_i T_wall, so pushes into them are skipped and the row's own thread writes
// them.
template <class L, class G, class Real>
__device__ __forceinline__ void scalar_step(const StepParams<Real> &p, int x, int y, int z, uint32_t c, bool solid,
                                            const ScalarCtx<Real> &sc, Real cs2inv) {
  const Real oT = p.omega_T, T = sc.T;
  static_for<G::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const Real gi = p.g[elem(p, i, c)];
    Real gp;
    if (solid) {
      gp = Real(Dir<G, i>::w) * T;
    } else {
      const Real eu = Dir<G, i>::x * sc.u[0] + Dir<G, i>::y * sc.u[1] + Dir<G, i>::z * sc.u[2];
      const Real geq = Real(Dir<G, i>::w) * T * (Real(1) + cs2inv * eu);
      gp = gi - oT * (gi - geq);
    }
    const int xd = wrap_n(x + Dir<G, i>::x, p.nx);
    const int yd = wrap_n(y + Dir<G, i>::y, p.ny);
    const int zd = L::DIMS == 3 ? wrap_n(z + Dir<G, i>::z, p.nz) : 0;
    if (yd != 0 && yd != p.ny - 1) p.gn[elem(p, i, cell_index(p, xd, yd, zd))] = gp;
  });
  if (y == 0 || y == p.ny - 1) {
    const Real Tw = y == 0 ? p.T_hot : p.T_cold;
    static_for<G::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      p.gn[elem(p, i, c)] = Real(Dir<G, i>::w) * Tw;
    });
  }
}

// --------------------------------------------------------------------------
// Kernels
// --------------------------------------------------------------------------

// Momentum-exchange force, pressure/viscous split and moment contributions
// of the links of one cell (forces.py:15-127, forces3d.py:8-131): for each
// link i, f_pre[i] + f_post[opp i] with f_pre = P at the cell and f_post = its
// post-BC state d; the split uses feq of the f_pre moments at the cell.  The
// rest-weight part of every term (2 w_i e_i, and r x 2 w_i e_i) is constant
// and added once per step by k_finalize, so only deviations are summed here.
template <class L, class S, class Real, class Gather>
__device__ __forceinline__ void link_cell_forces(const StepParams<Real> &p, int x, int y, int z, uint32_t c,
                                                 int64_t slot, const Real (&d)[L::Q], const Gather &gather) {
  Real drho = 0, jx = 0, jy = 0, jz = 0;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const Real v = gather.template pre<i>(c, slot);
    drho += v;
    if (Dir<L, i>::x) jx += Dir<L, i>::x * v;
    if (Dir<L, i>::y) jy += Dir<L, i>::y * v;
    if (Dir<L, i>::z) jz += Dir<L, i>::z * v;
  });
  const Real rho = Real(1) + drho;
  const Real inv = rho > Real(0) ? Real(1) / rho : Real(0);
  const Real ux = jx * inv, uy = jy * inv, uz = jz * inv, usq = ux * ux + uy * uy + uz * uz;
  const uint32_t mask = __ldg(p.lc_mask + slot);
  const Real rx = Real(x - p.center[0]), ry = Real(y - p.center[1]), rz = Real(z - p.center[2]);
  Real acc[12];
#pragma unroll
  for (int j = 0; j < 12; j++) acc[j] = Real(0);
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    if constexpr (i > 0) {
      if ((mask >> i) & 1u) {
        constexpr int o = L::opp[i];
        constexpr Real ex = Dir<L, i>::x, ey = Dir<L, i>::y, ez = Dir<L, i>::z;
        const Real fi = gather.template pre<i>(c, slot);
        const Real eui = ex * ux + ey * uy + ez * uz;
        const Real quad = Real(4.5) * eui * eui - Real(1.5) * usq;
        const Real deq_i = Real(Dir<L, i>::w) * (drho + rho * (Real(3) * eui + quad));
        const Real deq_o = Real(Dir<L, o>::w) * (drho + rho * (Real(-3) * eui + quad));
        const Real din = d[o];
        const Real mom = fi + din;
        const Real mp = deq_i + deq_o;
        const Real mv = (fi - deq_i) + (din - deq_o);
        acc[0] += ex * mom;
        acc[1] += ey * mom;
        acc[2] += ez * mom;
        acc[3] += ex * mp;
        acc[4] += ey * mp;
        acc[5] += ez * mp;
        acc[6] += ex * mv;
        acc[7] += ey * mv;
        acc[8] += ez * mv;
        acc[9] += (ry * ez - rz * ey) * mom;
        acc[10] += (rz * ex - rx * ez) * mom;
        acc[11] += (rx * ey - ry * ex) * mom;
      }
    }
  });
#pragma unroll
  for (int j = 0; j < 12; j++) p.lc_contrib[j * p.n_lc + slot] = (double)acc[j];
}

// Divergence guard (diagnostics.py:32-71): non-finite or non-positive rho of
// the state; one lane per warp reports, and only until it is recorded.
template <class Real>
__device__ __forceinline__ void guard_bad(const StepParams<Real> &p, bool bad, int64_t step_now) {
  const unsigned badm = __ballot_sync(__activemask(), bad);
  if (bad && (threadIdx.x & 31) == __ffs(badm) - 1) {
    if (!(*(volatile uint32_t *)p.status & STATUS_NONFINITE_OR_NONPOSITIVE_RHO))
      atomicOr(p.status, STATUS_NONFINITE_OR_NONPOSITIVE_RHO);
    if (*(volatile unsigned long long *)p.first_bad_step > (unsigned long long)(step_now + 1))
      atomicMin(p.first_bad_step, (unsigned long long)(step_now + 1));
  }
}

template <class Real>
__device__ __forceinline__ void guard_rho(const StepParams<Real> &p, Real rho, int64_t step_now) {
  guard_bad(p, !(rho > Real(0)) || !isfinite(rho), step_now);
}

// The part of a cell's step that follows its post-BC state d: link-cell
// forces, scalar step, collision at rate om (per-cell rate when `les`),
// divergence guard, P_{n+1} stored through the access functor.  In the AA
// layout's state-storing step the state itself is stored, uncollided.
template <class L, class S, int COLL, class Gather>
__device__ __forceinline__ void finish_cell(const StepParams<typename StoreOps<S>::Real> &p, int x, int y, int z,
                                            uint32_t c, uint32_t fl, int64_t step_now,
                                            typename StoreOps<S>::Real (&d)[L::Q],
                                            const ScalarCtx<typename StoreOps<S>::Real> &sc,
                                            typename StoreOps<S>::Real om, bool les, const Gather &gather) {
  using Real = typename StoreOps<S>::Real;
  const bool solid = fl & FLAG_SOLID;
  if ((FEAT_OF(p) & FEAT_OBSTACLE_BB) && (fl & FLAG_LINK)) {
    const int64_t slot = link_slot(p, x, y, z);
    if (slot >= 0) link_cell_forces<L, S, Real>(p, x, y, z, c, slot, d, gather);
  }
  if (FEAT_OF(p) & FEAT_THERMAL) {
    if (FEAT_OF(p) & FEAT_SCALAR_REDUCED) {
      using G = typename ScalarReduced<L>::Lat;
      scalar_step<L, G>(p, x, y, z, c, solid, sc, Real(G::cs2inv));
    } else {
      scalar_step<L, L>(p, x, y, z, c, solid, sc, Real(3));
    }
  }
  // the last step of an AA call stores the state itself (uncollided)
  const Real rho = Gather::kAA && p.aa_store_state ? Real(1) + sum_dev<L>(d)
                                                   : collide<L, Real, COLL>(p, d, solid, om, les,
                                                                            sc.m_set ? sc.m : nullptr);
  guard_rho(p, rho, step_now);
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    gather.template put<i>(x, c, d[i]);
  });
}

// One regular step of cell (x, y, z): state of step n from P_n (gathered by
// `gather`), link-cell forces, scalar step, collision, P_{n+1} stored.
template <class L, class S, int COLL, class Gather>
__device__ __forceinline__ void step_cell(const StepParams<typename StoreOps<S>::Real> &p, int x, int y, int z,
                                          int64_t step_now, const Gather &gather) {
  using Real = typename StoreOps<S>::Real;
  const uint32_t c = cell_index(p, x, y, z);
  const uint32_t fl = gather.flags(x);
  const bool solid = fl & FLAG_SOLID;
  Real d[L::Q];
  ScalarCtx<Real> sc;
  full_state<L, S, Real>(p, x, y, z, step_now, d, p.prevn, &sc, gather);
  Real om = p.omega;
  const bool les = (COLL != COLL_MRT) && (FEAT_OF(p) & FEAT_LES);
  if (les) om = les_omega<L>(p, x, y, z, c, solid);
  finish_cell<L, S, COLL>(p, x, y, z, c, fl, step_now, d, sc, om, les, gather);
}

// One full step: state of step n from P_n, scalar step, collision -> P_{n+1}.
// FROM_STATE: P holds a state (deviations) to be collided as is (used after
// the host sets f, and to start from an initial state).
// Block shapes of the per-cell kernel: BX threads along x times BY rows
// (y).  Every shape keeps 64 registers per thread: 8 blocks of 128 threads,
// 4 of 256 (4-byte arithmetic; FP64 takes half the blocks).
template <int BX, int BY>
struct StepShape {
  static constexpr int threads = BX * BY;
  static constexpr int min_blocks4 = kStepMinBlocks * 128 / (BX * BY);
};

// The AA variant keeps one block per SM less (72 registers instead of 64 for
// 4-byte arithmetic): its address arithmetic for the shifted stores would
// otherwise spill.
constexpr int kStepAAMinBlocks = 7;
template <class L, class S, int COLL, bool FROM_STATE, int BX = kStepBlock, int BY = 1, bool AA = false, int RL = -1>
__global__ void __launch_bounds__(BX *BY, AA ? (sizeof(typename StoreOps<S>::Real) == 4 ? kStepAAMinBlocks
                                                                                        : kStepAAMinBlocks / 2)
                                             : (sizeof(typename StoreOps<S>::Real) == 4 ? StepShape<BX, BY>::min_blocks4
                                                                                        : StepShape<BX, BY>::min_blocks4 / 2))
    k_step(const StepParams<typename StoreOps<S>::Real> p) {
  using Real = typename StoreOps<S>::Real;
  using SO = StoreOps<S>;
  const int x = blockIdx.x * BX + threadIdx.x;
  const int y = BY == 1 ? (int)blockIdx.y : (int)(blockIdx.y * BY + threadIdx.y), z = blockIdx.z;
  // the AA outlet shuffle needs warps of 32 consecutive x of one row
  static_assert(!AA || (BY == 1 && BX % 32 == 0), "the AA step kernel runs full-warp row segments");
  if (x >= p.nx || y >= p.ny) return;
  if constexpr (FROM_STATE) {
    // the collision of a state the host set: each cell reads and writes its
    // own values only (in place in the AA layout)
    const uint32_t c = cell_index(p, x, y, z);
    const bool solid = p.flags[c] & FLAG_SOLID;
    Real d[L::Q];
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = own_value<L, S, i>(p, x, y, z, c);
    });
    Real om = p.omega;
    const bool les = (COLL != COLL_MRT) && (FEAT_OF(p) & FEAT_LES);
    if (les) om = les_omega<L>(p, x, y, z, c, solid);
    collide<L, Real, COLL>(p, d, solid, om, les);
    S *Pn = static_cast<S *>(p.Pn);
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      SO::template store<i, L>(Pn, own_elem<L, i>(p, x, y, z, c), d[i]);
    });
  } else if constexpr (AA) {
    step_cell<L, S, COLL>(p, x, y, z, *p.step, AAGather<L, S, Real, RL>{p, y, z});
  } else {
    step_cell<L, S, COLL>(p, x, y, z, *p.step, GlobalGather<L, S, Real>{p, y, z});
  }
}

// --------------------------------------------------------------------------
// Row-tiled step.  A tile is `tile_rows` consecutive y rows of one z plane
// (whole x rows).  For direction i the cells of a tile pull from the source
// rows (y - ey, z - ez), which are contiguous in plane i of P (one run, or
// two when the y range wraps), so one thread of the block brings them into
// a shared-memory slab with bulk async copies (cp.async.bulk, completion
// counted in bytes on an mbarrier).  Blocks are persistent, walk the tiles
// with a grid stride and keep two stages: the next tile's rows are in
// flight while the current tile is computed.  Every element of P is read
// from HBM once per step and the gather costs no global-load latency in the
// issue path.  The host uses this kernel when a row fits a slab
// (nx <= TileCfg::cap) and rows start 16-byte aligned (nx * sizeof(S) a
// multiple of 16, P 16-byte aligned); otherwise it launches k_step.  With
// NS stages the block keeps NS - 1 tiles in flight while it computes one.
// --------------------------------------------------------------------------
// Tile shape: one cell per thread, so a slab holds `threads` cells and a row
// of up to that many cells fits one tile (at most kMaxTileRows rows).  A
// stage holds Q population slabs, the tile's flag bytes (copied from a
// 16-byte-aligned superset of the tile's cells, hence cap + 32 bytes) and
// the rows' convective outlet state (kMaxTileRows x QP values).  Every block
// gets the same shared-memory budget (two blocks per SM fit), spent on as
// many stages (two to four) as it holds.
#ifndef AERO_TILE_BLOCK_SMEM
#define AERO_TILE_BLOCK_SMEM 100352
#endif
constexpr uint64_t kWaitNs = 1000000000ull;  // a stage not complete after 1 s is declared lost
constexpr int kMaxTileRows = 16;

template <class L, class S>
struct TileCfg {
  using Real = typename StoreOps<S>::Real;
  static constexpr int threads = sizeof(S) == 8 ? 256 : 512;
  static constexpr int min_blocks = 2;
  static constexpr int cap = threads;  // cells per slab
  static constexpr int stage_elems = L::Q * cap;
  static constexpr int pop_bytes = stage_elems * (int)sizeof(S);
  static constexpr int flag_bytes = cap + 32;
  static constexpr int prev_bytes = kMaxTileRows * L::QP * (int)sizeof(Real);
  static constexpr int stage_bytes = pop_bytes + flag_bytes + prev_bytes;
  static constexpr int stages_fit = AERO_TILE_BLOCK_SMEM / stage_bytes;
  static constexpr int stages = stages_fit > 4 ? 4 : (stages_fit < 2 ? 2 : stages_fit);
  static constexpr int smem_bytes = stages * stage_bytes + 8 * stages;  // stages + one mbarrier per stage
  static_assert(pop_bytes % 16 == 0 && flag_bytes % 16 == 0 && prev_bytes % 16 == 0, "16-byte stage parts");
};

__device__ __forceinline__ uint32_t smem_addr(const void *ptr) {
  return (uint32_t)__cvta_generic_to_shared(ptr);
}
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred pw;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 pw, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, pw;\n\t}"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// Bounded wait: false when the phase did not complete within kWaitNs.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    for (int k = 0; k < 64; ++k)
      if (mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kWaitNs) return false;
  }
}
// Generic-proxy accesses to shared memory before async-proxy writes to it.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
// Bulk copy global -> shared (no multicast), completion counted on bar.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

struct TileCoord {
  int z, y0, rows;
};

template <class Real>
__device__ __forceinline__ TileCoord tile_coord(const StepParams<Real> &p, int tile) {
  TileCoord t;
  t.z = tile / p.tiles_per_plane;
  t.y0 = (tile - t.z * p.tiles_per_plane) * p.tile_rows;
  t.rows = p.ny - t.y0 < p.tile_rows ? p.ny - t.y0 : p.tile_rows;
  return t;
}

// Byte offset of the tile's first cell in its flag copy (the copy starts at
// the 16-byte boundary at or below that cell).
template <class Real>
__device__ __forceinline__ uint32_t tile_flag_skew(const StepParams<Real> &p, const TileCoord &t) {
  return (uint32_t)((((int64_t)t.z * p.ny + t.y0) * p.nx) & 15);
}

// Issued by one thread: the source rows of every direction of a tile, its
// flag bytes and (convective outlet) its rows' outlet state into one stage.
// The byte count announced on the barrier is exactly what the copies
// deliver.  Every copy starts and ends on a 16-byte boundary: rows because
// nx * sizeof(S) and the plane stride are multiples of 16, flags because
// the copy is widened to 16-byte boundaries (the flag buffer has slack past
// the last cell), outlet rows because QP * sizeof(Real) is.
template <class L, class S, class Real>
__device__ __forceinline__ void issue_tile(const StepParams<Real> &p, int tile, unsigned char *stage,
                                           uint64_t *bar) {
  using Cfg = TileCfg<L, S>;
  constexpr int CAP = Cfg::cap;
  const TileCoord t = tile_coord(p, tile);
  const uint32_t row_bytes = (uint32_t)p.nx * (uint32_t)sizeof(S);
  const int64_t c0 = ((int64_t)t.z * p.ny + t.y0) * p.nx;  // first cell of the tile
  const int64_t fa = c0 & ~(int64_t)15;
  const uint32_t fbytes = (uint32_t)(((c0 + (int64_t)t.rows * p.nx + 15) & ~(int64_t)15) - fa);
  const bool conv = (FEAT_OF(p) & FEAT_OPEN) && p.outlet == OUTLET_CONVECTIVE;
  const uint32_t pbytes = conv ? (uint32_t)t.rows * (uint32_t)(L::QP * sizeof(Real)) : 0u;
  mbar_arrive_expect_tx(bar, (uint32_t)L::Q * (uint32_t)t.rows * row_bytes + fbytes + pbytes + p.tile_extra_tx);
  const char *P = static_cast<const char *>(p.P);
  S *slab0 = reinterpret_cast<S *>(stage);
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ey = Dir<L, i>::y, ez = Dir<L, i>::z;
    const int zs = L::DIMS == 3 ? wrap_n(t.z - ez, p.nz) : 0;
    const int ys = wrap_n(t.y0 - ey, p.ny);               // first source row
    const int n1 = p.ny - ys < t.rows ? p.ny - ys : t.rows;  // rows before the y wrap
    char *dst = reinterpret_cast<char *>(slab0 + i * CAP);
    const int64_t base = (int64_t)i * p.cs + (int64_t)zs * p.ny * p.nx;
    bulk_g2s(dst, P + (base + (int64_t)ys * p.nx) * (int64_t)sizeof(S), (uint32_t)n1 * row_bytes, bar);
    if (n1 < t.rows)
      bulk_g2s(dst + (size_t)n1 * row_bytes, P + base * (int64_t)sizeof(S), (uint32_t)(t.rows - n1) * row_bytes,
               bar);
  });
  bulk_g2s(stage + Cfg::pop_bytes, p.flags + fa, fbytes, bar);
  if (conv)
    bulk_g2s(stage + Cfg::pop_bytes + Cfg::flag_bytes, p.prev + ((int64_t)t.z * p.ny + t.y0) * L::QP, pbytes, bar);
}

// Warps never wait for one another: each one waits only for the stage it
// needs to be full, computes its cells of the tile, and counts itself done
// with the stage on a shared-memory counter; the warp that completes the
// count refills the stage with the tile NS tiles ahead.  A slow warp (inlet,
// outlet or link cells) therefore delays only the refill of one stage, not
// the other warps, which may run up to NS - 1 tiles ahead.
template <class L, class S, int COLL>
__global__ void __launch_bounds__(TileCfg<L, S>::threads, TileCfg<L, S>::min_blocks)
    k_step_tiled(const StepParams<typename StoreOps<S>::Real> p) {
  using Real = typename StoreOps<S>::Real;
  using Cfg = TileCfg<L, S>;
  constexpr int NS = Cfg::stages;
  constexpr int NW = Cfg::threads / 32;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  unsigned char *stage0 = smem_raw;
  uint64_t *bar = reinterpret_cast<uint64_t *>(smem_raw + NS * Cfg::stage_bytes);
  __shared__ uint32_t done[NS];  // warps finished with each stage (monotonic)
  const int tid = threadIdx.x, lane = tid & 31;
  const int G = gridDim.x, nt = p.ntiles;
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) {
      mbar_init(&bar[k], 1);
      done[k] = 0;
    }
    mbar_init_fence();
  }
  __syncthreads();
  if (tid == 0) {
#pragma unroll
    for (int k = 0; k < NS; k++) {
      const int tk = blockIdx.x + k * G;
      if (tk < nt) issue_tile<L, S>(p, tk, stage0 + k * Cfg::stage_bytes, &bar[k]);
    }
  }
  const int64_t step_now = *p.step;
  int tile = blockIdx.x;
  for (int it = 0; tile < nt; ++it, tile += G) {
    const int s = it % NS;
    const uint32_t use = (uint32_t)(it / NS);
    if (!mbar_wait(&bar[s], use & 1u)) {
      // the stage never completed: report and stop this warp; the stage is
      // not refilled, so the other warps stop at their next wait.  Copies
      // still in flight are waited for (bounded again) so that none lands
      // after the block has exited.
      if (lane == 0) atomicOr(p.status, STATUS_WAIT_TIMEOUT);
      for (int k = 1; k < NS; k++) {
        const int jt = it + k;
        if (tile + k * G < nt) mbar_wait(&bar[jt % NS], (uint32_t)(jt / NS) & 1u);
      }
      return;
    }
    const unsigned char *sb = stage0 + s * Cfg::stage_bytes;
    const S *st = reinterpret_cast<const S *>(sb);
    const TileCoord t = tile_coord(p, tile);
    const uint8_t *fl = sb + Cfg::pop_bytes + tile_flag_skew(p, t);
    const Real *pv = reinterpret_cast<const Real *>(sb + Cfg::pop_bytes + Cfg::flag_bytes);
    const int ncell = t.rows * p.nx;
    int r = 0, x = tid;
    while (x >= p.nx) { x -= p.nx; ++r; }
    for (int k = tid; k < ncell; k += Cfg::threads) {
      const uint32_t row = (uint32_t)(r * p.nx);
      step_cell<L, S, COLL>(p, x, t.y0 + r, t.z, step_now,
                            SmemGather<L, S, Real, Cfg::cap>{st, row, p.nx, fl + row, pv + r * L::QP, &p});
      x += Cfg::threads;
      while (x >= p.nx) { x -= p.nx; ++r; }
    }
    // this warp's reads of stage s are complete (their values have been
    // used); the last warp to get here refills the stage
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      const uint32_t before = atomicAdd(&done[s], 1u);
      if (before == (use + 1) * NW - 1 && tile + NS * G < nt) {
        fence_proxy_async_smem();
        issue_tile<L, S>(p, tile + NS * G, stage0 + s * Cfg::stage_bytes, &bar[s]);
      }
    }
  }
}

// LES side pass: velocity of the current state (les.py:288 / :325 use
// compute_macroscopic of the pre-collision state, solids not zeroed).
template <class L, class S, bool FROM_STATE, bool AA = false>
__device__ __forceinline__ void moments_cell(const StepParams<typename StoreOps<S>::Real> &p, int x, int y, int z) {
  using Real = typename StoreOps<S>::Real;
  const uint32_t c = cell_index(p, x, y, z);
  Real d[L::Q];
  if constexpr (FROM_STATE) {
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = own_value<L, S, i>(p, x, y, z, c);
    });
  } else if constexpr (AA) {
    full_state<L, S, Real>(p, x, y, z, *p.step, d, nullptr, nullptr, AAGather<L, S, Real>{p, y, z});
  } else {
    // A fluid cell that no boundary rule touches (no link, not a wall row,
    // not an inlet / outlet column, not in the sponge) ends its chain as the
    // pulled populations plus the body-force and buoyancy terms, whose
    // moments are known in closed form: the Guo term adds bf_coeff rho F to
    // j and nothing to rho (the lattice's odd moments of third order vanish);
    // buoyancy adds rho g beta (T - T_ref) to j_y.  Such a cell needs one sum
    // of its pulled populations instead of the whole chain.
    const uint32_t fl = p.flags[c];
    const bool open = FEAT_OF(p) & FEAT_OPEN;
    const bool plain = !(fl & (FLAG_SOLID | FLAG_LINK)) && !(WALL_OF(p) != WALL_NONE && (y == 0 || y == p.ny - 1)) &&
                       !(open && (x == 0 || x == p.nx - 1)) && !((FEAT_OF(p) & FEAT_RECYCLE) && x == 0) &&
                       !((FEAT_OF(p) & FEAT_SPONGE) && x >= p.sponge_start);
    if (plain) {
      GlobalGather<L, S, Real>{p, y, z}(x, d);
      Real drho = 0, jx = 0, jy = 0, jz = 0;
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        drho += d[i];
        if (Dir<L, i>::x) jx += Dir<L, i>::x * d[i];
        if (Dir<L, i>::y) jy += Dir<L, i>::y * d[i];
        if (Dir<L, i>::z) jz += Dir<L, i>::z * d[i];
      });
      const Real rho = Real(1) + drho;
      if constexpr (L::DIMS == 3) {
        if ((FEAT_OF(p) & FEAT_BODY_FORCE) && rho > Real(0)) {
          jx += p.bf_coeff * rho * p.bf_x;
          jy += p.bf_coeff * rho * p.bf_y;
          jz += p.bf_coeff * rho * p.bf_z;
        }
      }
      if ((FEAT_OF(p) & FEAT_THERMAL) && (FEAT_OF(p) & FEAT_BUOYANCY)) {
        Real T = 0;
        if (FEAT_OF(p) & FEAT_SCALAR_REDUCED) {
          using G = typename ScalarReduced<L>::Lat;
          static_for<G::Q>([&](auto ic) { T += p.g[elem(p, decltype(ic)::value, c)]; });
        } else {
          static_for<L::Q>([&](auto ic) { T += p.g[elem(p, decltype(ic)::value, c)]; });
        }
        jy += rho * (p.gbeta * (T - p.T_ref));
      }
      const Real inv = rho > Real(0) ? Real(1) / rho : Real(0);
      p.Uw[c] = jx * inv;
      p.Uw[p.cs + c] = jy * inv;
      p.Uw[2 * p.cs + c] = jz * inv;
      return;
    }
    full_state<L, S, Real>(p, x, y, z, *p.step, d, nullptr, nullptr);
  }
  Real drho = 0, jx = 0, jy = 0, jz = 0;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    drho += d[i];
    if (Dir<L, i>::x) jx += Dir<L, i>::x * d[i];
    if (Dir<L, i>::y) jy += Dir<L, i>::y * d[i];
    if (Dir<L, i>::z) jz += Dir<L, i>::z * d[i];
  });
  const Real rho = Real(1) + drho;
  const Real inv = rho > Real(0) ? Real(1) / rho : Real(0);
  p.Uw[c] = jx * inv;
  p.Uw[p.cs + c] = jy * inv;
  p.Uw[2 * p.cs + c] = jz * inv;
}

template <class L, class S, bool FROM_STATE, bool AA = false>
__global__ void __launch_bounds__(kStepBlock) k_moments(const StepParams<typename StoreOps<S>::Real> p) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= p.nx) return;
  moments_cell<L, S, FROM_STATE, AA>(p, x, (int)blockIdx.y, (int)blockIdx.z);
}

// AA layout, before each step: the pre-stream populations of every link
// cell, the clipped-neighbour values of its Bouzidi links with q >= 1/2, and
// the pulled populations of plane x = nx-2 (where an outlet or the
// recycling inlet re-evaluates it), copied out of the buffer the step is
// about to update in place.  Block row blockIdx.y is the direction; along x,
// threads [0, n_lc) take link cells and the rest the (y, z) rows of plane
// nx-2.  One load and one store per thread, the direction uniform in a block,
// so the few link cells still spread over the whole GPU and no warp runs the
// directions one after another.
constexpr int kStageBlock = 256;

template <class L, class S>
__global__ void __launch_bounds__(kStageBlock) k_aa_stage(const StepParams<typename StoreOps<S>::Real> p) {
  using Real = typename StoreOps<S>::Real;
  const int dir = blockIdx.y;
  const int64_t k = (int64_t)blockIdx.x * kStageBlock + threadIdx.x;
  if (k < p.n_lc) {
    // cell indices are below 2^31
    const uint32_t c = (uint32_t)p.lc_cell[k];
    const uint32_t row = c / (uint32_t)p.nx;
    const int x = (int)(c - row * (uint32_t)p.nx);
    const int z = (int)(row / (uint32_t)p.ny), y = (int)(row - (uint32_t)z * (uint32_t)p.ny);
    const int64_t t = k * L::Q + dir;
    const bool bouzidi = FEAT_OF(p) & FEAT_BOUZIDI;
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      if (dir != i) return;
      static_cast<Real *>(p.stage_link)[t] = own_value<L, S, i>(p, x, y, z, c);
      if constexpr (i > 0) {
        if (bouzidi && ((__ldg(p.lc_mask + k) >> i) & 1u) && __ldg(p.lc_q + t) >= 0.5f) {
          constexpr int o = L::opp[i];
          const int xn = clamp_n(x + Dir<L, o>::x, p.nx);
          const int yn = clamp_n(y + Dir<L, o>::y, p.ny);
          const int zn = L::DIMS == 3 ? clamp_n(z + Dir<L, o>::z, p.nz) : 0;
          static_cast<Real *>(p.stage_nb)[t] = own_value<L, S, i>(p, xn, yn, zn, cell_index(p, xn, yn, zn));
        }
      }
    });
    return;
  }
  // plane x = nx-2, direction-major: a warp's stores are contiguous
  const int64_t plane = (int64_t)p.ny * p.nz;
  const int64_t r = k - p.n_lc;
  if (!p.stage_out || r >= plane) return;
  const int y = (int)(r % p.ny), z = (int)(r / p.ny);
  Real *so = static_cast<Real *>(p.stage_out) + r;
  const AAGather<L, S, Real> g{p, y, z};
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    if (dir == i) so[i * plane] = g.template raw_one<i>(p.nx - 2);
  });
}

// Mean ux of the recycle plane x = nx-2 of the current step's post-bounce-
// back state (boundary3d.py:186-188: compute_macroscopic_3d, 0 where rho <=
// 0, mean over every cell of the plane).  One thread per (z, y) row; blocks
// sum in a fixed order, the last block adds the block sums in block order.
constexpr int kRecycleBlock = 256;

template <class L, class S, bool AA = false>
__global__ void __launch_bounds__(kRecycleBlock) k_recycle_mean(const StepParams<typename StoreOps<S>::Real> p) {
  using Real = typename StoreOps<S>::Real;
  __shared__ double red[kRecycleBlock / 32];
  __shared__ bool last;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int64_t k = (int64_t)blockIdx.x * kRecycleBlock + t;
  const int64_t plane = (int64_t)p.ny * p.nz;
  double v = 0.0;
  if (k < plane) {
    const int y = (int)(k % p.ny), z = (int)(k / p.ny);
    Real d[L::Q];
    if constexpr (AA)
      partial_state<L, S, Real>(p, p.nx - 2, y, z, *p.step, d, AAGather<L, S, Real>{p, y, z});
    else
      partial_state<L, S, Real>(p, p.nx - 2, y, z, *p.step, d, GlobalGather<L, S, Real>{p, y, z});
    Real drho = 0, jx = 0;
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      drho += d[i];
      if (Dir<L, i>::x) jx += Dir<L, i>::x * d[i];
    });
    const Real rho = Real(1) + drho;
    v = rho > Real(0) ? (double)(jx * (Real(1) / rho)) : 0.0;
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (t == 0) {
    double b = 0.0;
    for (int w = 0; w < kRecycleBlock / 32; w++) b += red[w];
    p.recycle_partial[blockIdx.x] = b;
    __threadfence();
    last = atomicAdd(p.recycle_ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && t == 0) {
    __threadfence();
    double sum = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) sum += __ldcg(p.recycle_partial + b);
    *p.recycle_mean = sum / (double)plane;
    *p.recycle_ticket = 0u;
  }
}

// Sums the per-link-cell contributions plus the constant rest-weight part
// into the device history ring, sums the profile segments when this step's
// profile is the one that can be read, then advances the step counter.
// Block b adds link cells [b * fin_chunk, (b + 1) * fin_chunk) in a fixed
// order and stores 12 partial sums; the block that finishes last adds the
// partials in block order, so the result does not depend on block timing.
// Block `bid` of `nblocks` finalisation blocks of one lattice.
// Finalisation block `bid`: the fixed-order FP64 sums of its chunk of the
// link cells' force terms into fin_partial[bid].  Ends on a block barrier,
// so a block may call it for several chunks in turn.
template <class Real>
__device__ __forceinline__ void finalize_partial(const StepParams<Real> &p, int bid) {
  __shared__ double sm[12][kFinalizeBlock / 32];
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  const int64_t n = p.n_lc;
  const int64_t k0 = (int64_t)bid * p.fin_chunk;
  const int64_t k1 = k0 + p.fin_chunk < n ? k0 + p.fin_chunk : n;
  double a[12];
#pragma unroll
  for (int j = 0; j < 12; j++) a[j] = 0.0;
  for (int64_t k = k0 + t; k < k1; k += kFinalizeBlock) {
#pragma unroll
    for (int j = 0; j < 12; j++) a[j] += __ldcg(p.lc_contrib + j * n + k);
  }
#pragma unroll
  for (int j = 0; j < 12; j++) {
    double v = a[j];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (lane == 0) sm[j][wid] = v;
  }
  __syncthreads();
  if (t < 12) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < kFinalizeBlock / 32; w++) v += sm[t][w];
    p.fin_partial[bid * 12 + t] = v;
    __threadfence();
  }
  __syncthreads();
}

// The step's totals from the nblocks partials (in block order) plus the
// rest-weight part, into the history ring; the force profile on the step the
// call asked for; then the device step counter advances.
template <class Real>
__device__ __forceinline__ void finalize_total(const StepParams<Real> &p, int nblocks) {
  const int t = threadIdx.x;
  const int64_t n = p.n_lc;
  const int64_t step = *p.step;
  const int64_t slot = (step - *p.hist_base) % p.hist_cap;
  if (t < 12) {
    double v = p.force_const[t];
    for (int b = 0; b < nblocks; b++) v += __ldcg(p.fin_partial + b * 12 + t);
    p.hist[slot * 12 + t] = v;
  }
  if (p.want_profile && step + 1 == *p.profile_step) {
    for (int b = t; b < p.nprof; b += kFinalizeBlock) {
      double a0 = p.prof_const[b * 3 + 0], a1 = p.prof_const[b * 3 + 1], a2 = p.prof_const[b * 3 + 2];
      for (int k = p.prof_off[b]; k < p.prof_off[b + 1]; k++) {
        a0 += __ldcg(p.lc_contrib + k);
        a1 += __ldcg(p.lc_contrib + n + k);
        a2 += __ldcg(p.lc_contrib + 2 * n + k);
      }
      p.prof_out[b * 3 + 0] = a0;
      p.prof_out[b * 3 + 1] = a1;
      p.prof_out[b * 3 + 2] = a2;
    }
  }
  __syncthreads();
  if (t == 0) {
    *p.fin_ticket = 0u;
    *p.step = step + 1;
  }
}

template <class Real>
__device__ __forceinline__ void finalize_block(const StepParams<Real> &p, int bid, int nblocks) {
  __shared__ bool last;
  finalize_partial(p, bid);
  if (threadIdx.x == 0) last = atomicAdd(p.fin_ticket, 1u) == (unsigned)nblocks - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  finalize_total(p, nblocks);
}

template <class Real>
__global__ void __launch_bounds__(kFinalizeBlock) k_finalize(const StepParams<Real> p) {
  finalize_block(p, (int)blockIdx.x, (int)gridDim.x);
}

// --------------------------------------------------------------------------
// Batched stepping: many lattices of one class (lattice, storage format,
// collision) advance in one launch.  Member m owns blocks [first[m],
// first[m + 1]) of the grid (blocks of consecutive cells, or finalisation
// blocks); each block copies its member's parameters into shared
// memory, then runs the same per-cell code.  The parameter arrays live in
// device memory, so a captured launch stays valid while the members advance.
// --------------------------------------------------------------------------
// Member owning block b: the last m with first[m] <= b (first[0] = 0).
// Up to 1024 members the search takes two dependent loads: every lane of
// the first warp tests one of 32 evenly spaced entries, then one entry of
// the chosen stretch; larger batches bisect.  The result is broadcast
// through shared memory, so the caller must reach this with the whole block.
__device__ __forceinline__ int find_member(const int64_t *__restrict__ first, int n, int64_t b) {
  __shared__ int found;
  if (n <= 1024) {
    if (threadIdx.x < 32) {
      const int lane = threadIdx.x;
      const int S = (n + 31) >> 5;  // stretch length, <= 32
      const int c0 = lane * S;
      const unsigned coarse = __ballot_sync(0xffffffffu, c0 < n && __ldg(first + c0) <= b);
      const int c = (31 - __clz(coarse)) * S;  // start of the stretch holding b (bit 0 is always set)
      const int f = c + lane;
      const unsigned fine = __ballot_sync(0xffffffffu, lane < S && f < n && __ldg(first + f) <= b);
      if (lane == 0) found = c + (31 - __clz(fine));
    }
  } else if (threadIdx.x == 0) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(first + mid) <= b) lo = mid; else hi = mid - 1;
    }
    found = lo;
  }
  __syncthreads();
  return found;
}

template <class Real>
__device__ __forceinline__ void params_to_smem(StepParams<Real> &dst, const StepParams<Real> *src) {
  static_assert(sizeof(StepParams<Real>) % 8 == 0, "parameter block in 8-byte words");
  constexpr int W = (int)(sizeof(StepParams<Real>) / 8);
  uint64_t *d = reinterpret_cast<uint64_t *>(&dst);
  const uint64_t *s = reinterpret_cast<const uint64_t *>(src);
  for (int k = threadIdx.x; k < W; k += blockDim.x) d[k] = __ldg(s + k);
  __syncthreads();
}

// A block of a batched cell kernel covers batch_rows * kStepBlock
// consecutive cells of its member in C order (batch_rows passes of one cell
// per thread): kBatchRows for large members, so the member lookup and the
// parameter copy are paid once per kBatchRows passes, and 1 for members below
// kBatchSmallCells, so a few small members still spread over the whole GPU.
// Cells rather than x segments: rows of 96 or 160 cells would leave a quarter
// or more of a 128-thread block idle.
constexpr int kBatchRows = 4;
constexpr int64_t kBatchSmallCells = 1 << 16;

template <class L, class S, int COLL>
__global__ void __launch_bounds__(kStepBlock, sizeof(typename StoreOps<S>::Real) == 4 ? kStepMinBlocks : 4)
    k_step_batch(const StepParams<typename StoreOps<S>::Real> *__restrict__ params,
                 const int64_t *__restrict__ first, int nmembers) {
  using Real = typename StoreOps<S>::Real;
  __shared__ StepParams<Real> sp;
  const int m = find_member(first, nmembers, blockIdx.x);
  params_to_smem(sp, params + m);
  // block b takes cells [b, b + 1) * R * kStepBlock of the member in C order
  // (R = batch_rows passes of kStepBlock consecutive cells), so rows shorter
  // or longer than a block leave no thread idle but in the member's last block
  const int64_t b = (int64_t)blockIdx.x - __ldg(first + m);
  const int64_t step_now = *sp.step;
  const int R = sp.batch_rows;
  for (int k = 0; k < R; ++k) {
    const int64_t c = (b * R + k) * kStepBlock + threadIdx.x;
    if (c >= sp.ncells) return;
    int x, y, z;
    cell_xyz((uint32_t)c, (uint32_t)sp.nx, (uint32_t)sp.ny, x, y, z);
    step_cell<L, S, COLL>(sp, x, y, z, step_now, GlobalGather<L, S, Real>{sp, y, z});
  }
}

template <class L, class S>
__global__ void __launch_bounds__(kStepBlock) k_moments_batch(const StepParams<typename StoreOps<S>::Real> *__restrict__ params,
                                                              const int64_t *__restrict__ first, int nmembers) {
  using Real = typename StoreOps<S>::Real;
  __shared__ StepParams<Real> sp;
  const int m = find_member(first, nmembers, blockIdx.x);
  params_to_smem(sp, params + m);
  // the cell blocks of k_step_batch
  const int64_t b = (int64_t)blockIdx.x - __ldg(first + m);
  const int R = sp.batch_rows;
  for (int k = 0; k < R; ++k) {
    const int64_t c = (b * R + k) * kStepBlock + threadIdx.x;
    if (c >= sp.ncells) return;
    int x, y, z;
    cell_xyz((uint32_t)c, (uint32_t)sp.nx, (uint32_t)sp.ny, x, y, z);
    moments_cell<L, S, false>(sp, x, y, z);
  }
}

template <class Real>
__global__ void __launch_bounds__(kFinalizeBlock) k_finalize_batch(const StepParams<Real> *__restrict__ params,
                                                                   const int64_t *__restrict__ first, int nmembers) {
  __shared__ StepParams<Real> sp;
  const int m = find_member(first, nmembers, blockIdx.x);
  params_to_smem(sp, params + m);
  finalize_block(sp, (int)((int64_t)blockIdx.x - __ldg(first + m)), sp.fin_blocks);
}

// State of the step that produced P (f as the reference stores it), written
// as absolute FP64 populations (Q, planes, ny, nx) for the planes z0 ..
// z0 + gridDim.z - 1.  step_delta selects the step index the inlet
// perturbation phase uses.  RAW: P already holds a state.
template <class L, class S, bool RAW>
__global__ void __launch_bounds__(kStepBlock) k_state_out(const StepParams<typename StoreOps<S>::Real> p,
                                                          double *out, int step_delta, int z0, int64_t out_plane) {
  using Real = typename StoreOps<S>::Real;
  using SO = StoreOps<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z + z0;
  if (x >= p.nx) return;
  const uint32_t c = cell_index(p, x, y, z);
  Real d[L::Q];
  if constexpr (RAW) {
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = own_value<L, S, i>(p, x, y, z, c);
    });
  } else {
    full_state<L, S, Real>(p, x, y, z, *p.step + step_delta, d, nullptr, nullptr);
  }
  const int64_t oc = (int64_t)c - (int64_t)z0 * p.ny * p.nx;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    out[(int64_t)i * out_plane + oc] = Dir<L, i>::w + (double)d[i];
  });
}

// Density and velocity of the state (compute_macroscopic(_3d), d2q9.py:44-63,
// d3q19.py:80-102) straight from the population buffers: out holds planes
// rho, ux, uy[, uz] of out_plane cells each (z0 .. z0 + gridDim.z - 1), FP64,
// with f_i = w_i + d_i summed in direction order and u = (sum e_i f_i) / rho
// taken as (1 / rho) * sum, 0 where rho <= 0, as the reference writes it.
template <class L, class S, bool RAW>
__global__ void __launch_bounds__(kStepBlock) k_macro_out(const StepParams<typename StoreOps<S>::Real> p,
                                                          double *out, int step_delta, int z0, int64_t out_plane) {
  using Real = typename StoreOps<S>::Real;
  using SO = StoreOps<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z + z0;
  if (x >= p.nx) return;
  const uint32_t c = cell_index(p, x, y, z);
  Real d[L::Q];
  if constexpr (RAW) {
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = own_value<L, S, i>(p, x, y, z, c);
    });
  } else {
    full_state<L, S, Real>(p, x, y, z, *p.step + step_delta, d, nullptr, nullptr);
  }
  double rho = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const double f = Dir<L, i>::w + (double)d[i];
    rho += f;
    jx += (double)Dir<L, i>::x * f;
    jy += (double)Dir<L, i>::y * f;
    if constexpr (L::DIMS == 3) jz += (double)Dir<L, i>::z * f;
  });
  const double inv = rho > 0.0 ? 1.0 / rho : 0.0;
  const int64_t oc = (int64_t)c - (int64_t)z0 * p.ny * p.nx;
  out[oc] = rho;
  out[out_plane + oc] = inv * jx;
  out[2 * out_plane + oc] = inv * jy;
  if constexpr (L::DIMS == 3) out[3 * out_plane + oc] = inv * jz;
}

// --------------------------------------------------------------------------
// Field statistics of the current state, summed in FP64 on the device: the
// global mass and scalar totals, the quantities check_stability tests
// (diagnostics.py:32-71: NaN populations, rho <= 0, max |(ux, uy)|, mean
// rho) and the wall heat-flux sums of the Nusselt number, over the planes
// z0 .. z0 + nzs - 1.  A fixed grid of kStatsBlocks blocks strides over the
// cells; each block stores its partial values and the block that finishes
// last combines the partials in block order, so every figure is the same
// from run to run.
//
// Nusselt number (the reference computes none): at the Dirichlet rows y = 0
// (T_hot) and y = ny-1 (T_cold), the wall-normal gradient of T = sum_i g_i
// by the second-order one-sided difference, for every (x, z) column whose
// two cells next to the wall are fluid; Nu = mean(-dT/dy) (ny - 1) /
// (T_hot - T_cold), which is 1 for pure conduction between the rows.
// --------------------------------------------------------------------------
constexpr int kStatsBlocks = 296;
constexpr int kStatsBlock = 256;
constexpr int kStatsValues = 10;  // see aero_field_stats in aero_b200.h for the order

template <class L, class S, bool RAW>
__global__ void __launch_bounds__(kStatsBlock)
    k_field_stats(const StepParams<typename StoreOps<S>::Real> p, const typename StoreOps<S>::Real *gcur, int z0,
                  int nzs, int step_delta, double *partial, uint32_t *ticket, double *out) {
  using Real = typename StoreOps<S>::Real;
  using SO = StoreOps<S>;
  __shared__ double red[kStatsValues][kStatsBlock / 32];
  __shared__ bool last;
  const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
  double a[kStatsValues];
#pragma unroll
  for (int k = 0; k < kStatsValues; k++) a[k] = 0.0;
  const int64_t plane = (int64_t)p.nx * p.ny;
  const int64_t n = plane * nzs;
  const bool thermal = (FEAT_OF(p) & FEAT_THERMAL) && gcur != nullptr;
  const int Qg = (FEAT_OF(p) & FEAT_SCALAR_REDUCED) ? ScalarReduced<L>::Lat::Q : L::Q;
  auto Tcell = [&](int x, int y, int z) {
    const uint32_t cc = cell_index(p, x, y, z);
    double T = 0.0;
    for (int i = 0; i < Qg; i++) T += (double)gcur[elem(p, i, cc)];
    return T;
  };
  for (int64_t k = (int64_t)blockIdx.x * kStatsBlock + t; k < n; k += (int64_t)kStatsBlocks * kStatsBlock) {
    const int z = z0 + (int)(k / plane);
    const int64_t r = k - (int64_t)(z - z0) * plane;
    const int y = (int)(r / p.nx), x = (int)(r - (int64_t)y * p.nx);
    const uint32_t c = cell_index(p, x, y, z);
    Real d[L::Q];
    if constexpr (RAW) {
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        d[i] = own_value<L, S, i>(p, x, y, z, c);
      });
    } else {
      full_state<L, S, Real>(p, x, y, z, *p.step + step_delta, d, nullptr, nullptr);
    }
    double rho = 0.0, jx = 0.0, jy = 0.0;
    int nan = 0;
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      nan += isnan(d[i]) ? 1 : 0;
      const double f = Dir<L, i>::w + (double)d[i];
      rho += f;
      jx += (double)Dir<L, i>::x * f;
      jy += (double)Dir<L, i>::y * f;
    });
    const double inv = rho > 0.0 ? 1.0 / rho : 0.0;
    const double ux = inv * jx, uy = inv * jy;
    a[0] += (double)nan;
    a[1] += rho <= 0.0 ? 1.0 : 0.0;
    a[2] = fmax(a[2], sqrt(ux * ux + uy * uy));
    a[3] += rho;
    a[4] += 1.0;
    if (thermal) {
      a[5] += Tcell(x, y, z);
      if (p.ny >= 3 && (y == 0 || y == p.ny - 1)) {
        const int s = y == 0 ? 1 : -1;  // into the fluid
        const bool fluid = !(p.flags[cell_index(p, x, y + s, z)] & FLAG_SOLID) &&
                           !(p.flags[cell_index(p, x, y + 2 * s, z)] & FLAG_SOLID);
        if (fluid) {
          const double T0 = Tcell(x, y, z), T1 = Tcell(x, y + s, z), T2 = Tcell(x, y + 2 * s, z);
          // one-sided d T / d(distance into the fluid), then as -dT/dy
          const double dn = 0.5 * (-3.0 * T0 + 4.0 * T1 - T2);
          const double mdTdy = y == 0 ? -dn : dn;
          a[y == 0 ? 6 : 8] += mdTdy;
          a[y == 0 ? 7 : 9] += 1.0;
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < kStatsValues; k++) {
    double v = a[k];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      const double o = __shfl_down_sync(0xffffffffu, v, off);
      v = k == 2 ? fmax(v, o) : v + o;
    }
    if (lane == 0) red[k][wid] = v;
  }
  __syncthreads();
  if (t < kStatsValues) {
    double v = 0.0;
    for (int w = 0; w < kStatsBlock / 32; w++) v = t == 2 ? fmax(v, red[t][w]) : v + red[t][w];
    partial[blockIdx.x * kStatsValues + t] = v;
    __threadfence();
  }
  __syncthreads();
  if (t == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  if (t < kStatsValues) {
    double v = 0.0;
    for (int b = 0; b < (int)gridDim.x; b++) {
      const double pb = __ldcg(partial + b * kStatsValues + t);
      v = t == 2 ? fmax(v, pb) : v + pb;
    }
    out[t] = v;
  }
  if (t == 0) *ticket = 0u;
}

// --------------------------------------------------------------------------
// Equilibrium state from macroscopic fields, built on the device: the
// reference's initial state f = feq(rho, u) at every cell, solids included
// (solver.py:218-227, solver3d.py:239-247), with the convective outlet state
// = the x = nx-1 column of f and the scalar g_i = w_i T.  Each field is an
// FP64 array of ncells values or, when NULL, the uniform value (rho0, u0,
// 0, 0, T_ref).  feq is evaluated in FP64 with the operations of
// compute_feq(_3d) (d2q9.py:66-89, d3q19.py:105-129) in their order, each
// rounded on its own (no fused multiply-adds), so a state built here equals
// one built from the same fields on the host; the deviation f - w is rounded
// once to the storage format.
// --------------------------------------------------------------------------
template <class L, int I>
__device__ __forceinline__ double feq_exact(double rho, double ux, double uy, double uz, double usq) {
  constexpr double ex = Dir<L, I>::x, ey = Dir<L, I>::y, ez = Dir<L, I>::z;
  double eu = __dadd_rn(ex * ux, ey * uy);  // products with 0 / +-1 are exact
  eu = __dadd_rn(eu, L::DIMS == 3 ? ez * uz : 0.0);
  const double poly = __dsub_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(3.0, eu)), __dmul_rn(__dmul_rn(4.5, eu), eu)),
                                __dmul_rn(1.5, usq));
  return __dmul_rn(__dmul_rn(Dir<L, I>::w, rho), poly);
}

template <class L, class S>
__global__ void __launch_bounds__(kStepBlock) k_init_equilibrium(const StepParams<typename StoreOps<S>::Real> p,
                                                                 EqFields e, S *dst,
                                                                 typename StoreOps<S>::Real *prev_dst,
                                                                 typename StoreOps<S>::Real *g_dst) {
  using Real = typename StoreOps<S>::Real;
  using SO = StoreOps<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= p.nx) return;
  const uint32_t c = cell_index(p, x, y, z);
  const double rho = e.rho ? e.rho[c] : e.rho0;
  const double ux = e.ux ? e.ux[c] : e.u0;
  const double uy = e.uy ? e.uy[c] : 0.0;
  const double uz = (L::DIMS == 3 && e.uz) ? e.uz[c] : 0.0;
  const double usq = __dadd_rn(__dadd_rn(__dmul_rn(ux, ux), __dmul_rn(uy, uy)), __dmul_rn(uz, uz));
  const bool outlet = prev_dst && x == p.nx - 1;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const double dv = __dsub_rn(feq_exact<L, i>(rho, ux, uy, uz, usq), Dir<L, i>::w);
    SO::template store<i, L>(dst, own_elem<L, i>(p, x, y, z, c), (Real)dv);
    if (outlet) prev_dst[((int64_t)z * p.ny + y) * L::QP + i] = (Real)dv;
  });
  if (g_dst) {
    const double T = e.T ? e.T[c] : e.T0;
    if (FEAT_OF(p) & FEAT_SCALAR_REDUCED) {
      using G = typename ScalarReduced<L>::Lat;
      static_for<G::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        g_dst[elem(p, i, c)] = (Real)__dmul_rn(Dir<G, i>::w, T);
      });
    } else {
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        g_dst[elem(p, i, c)] = (Real)__dmul_rn(Dir<L, i>::w, T);
      });
    }
  }
}

// Converts absolute FP64 populations (Q, ncells) into the storage format.
template <class L, class S>
__global__ void __launch_bounds__(kStepBlock) k_load_state(const StepParams<typename StoreOps<S>::Real> p,
                                                           const double *in, S *dst) {
  using Real = typename StoreOps<S>::Real;
  using SO = StoreOps<S>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  if (x >= p.nx) return;
  const uint32_t c = cell_index(p, x, y, z);
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    SO::template store<i, L>(dst, own_elem<L, i>(p, x, y, z, c), (Real)(in[(int64_t)i * p.ncells + c] - Dir<L, i>::w));
  });
}

// --------------------------------------------------------------------------
// Persistent run of a small lattice: one cooperative launch takes all steps
// of an aero_step call, so a lattice whose step is a few microseconds of work
// stops paying a kernel launch and a grid drain per step and per force
// finalisation.  Blocks 1.. take the cells (grid-stride over the cells in C
// order, the per-cell step of k_step), block 0 finalises: after the barrier
// that ends step s it sums step s's link-cell force terms (the chunks and
// order of k_finalize, so the history is the same bit for bit) while the
// other blocks compute step s + 1.  Consecutive steps write their force terms
// to alternate buffers (the parameter sets of the two steps of a pair carry
// the two pointers), and block 0 reaches the barrier of step s + 1 only after
// that finalisation, so step s + 2 cannot overwrite terms still being read.
// The grid barrier is bounded: a block that waits more than kWaitNs sets
// STATUS_WAIT_TIMEOUT and returns, and so do the others at their next wait.
// A launch takes at most kRunMaxSteps steps (the arrival count stays below
// 2^32); the host splits longer calls.
// --------------------------------------------------------------------------
constexpr int kRunBlock = kFinalizeBlock;  // block 0 runs the finalisation code, built for this width
#ifndef AERO_RUN_BLOCKS_PER_SM
#define AERO_RUN_BLOCKS_PER_SM 3
#endif
constexpr int64_t kRunMaxSteps = (int64_t)1 << 20;
constexpr int kRunMinBlocks = 3;  // 85 registers (FP64 arithmetic: 2 blocks, 128)

__device__ __forceinline__ uint32_t ld_acquire_u32(const uint32_t *q) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(q) : "memory");
  return v;
}

// Barrier k of a launch completes when the arrival counter (zeroed by the
// host before the launch) reaches (k + 1) * nblocks: each block adds one
// after a fence over its writes, and waits, reading the counter with acquire
// semantics, until it gets there; the last arrival releases the others with
// its own increment.
__device__ __forceinline__ bool run_barrier(uint32_t *count, uint32_t nblocks, uint32_t k, uint32_t *status) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    const uint32_t target = (k + 1u) * nblocks;
    __threadfence();
    if (atomicAdd(count, 1u) + 1u < target) {
      const uint64_t t0 = global_ns();
      while (ld_acquire_u32(count) < target) {
        __nanosleep(32);
        if (global_ns() - t0 > kWaitNs) {
          ok = 0;
          atomicOr(status, (uint32_t)STATUS_WAIT_TIMEOUT);
          break;
        }
      }
    }
    __threadfence();
    ok_s = ok;
  }
  __syncthreads();
  return ok_s != 0;
}

// pp[0], pp[1]: the parameters of even and odd steps of the call (buffer
// parities cur and 1 - cur, force terms in alternate buffers).  stall_block
// (tests only, else -1): that block leaves before its first barrier, so the
// others' bounded wait runs out.
template <class L, class S, int COLL>
__global__ void __launch_bounds__(kRunBlock, sizeof(typename StoreOps<S>::Real) == 4 ? kRunMinBlocks : 2)
    k_run_small(const StepParams<typename StoreOps<S>::Real> *__restrict__ pp, int64_t nsteps, int stall_block) {
  using Real = typename StoreOps<S>::Real;
  __shared__ StepParams<Real> sp2[2];  // both parameter sets, loaded once
  uint32_t *count = reinterpret_cast<uint32_t *>(pp[0].step + 6);
  const uint32_t nb = gridDim.x;
  // the call's first step; block 0 advances the counter only after the
  // first barrier, which every block reaches after this read
  const int64_t step0 = *pp[0].step;
  const int64_t cstride = (int64_t)(nb - 1) * kRunBlock;
  params_to_smem(sp2[0], pp);
  params_to_smem(sp2[1], pp + 1);
  for (int64_t s = 0; s < nsteps; ++s) {
    const StepParams<Real> &sp = sp2[s & 1];
    if (blockIdx.x != 0) {
      if ((int)blockIdx.x == stall_block) return;
      const int64_t step_now = step0 + s;
      for (int64_t c = (int64_t)(blockIdx.x - 1) * kRunBlock + threadIdx.x; c < sp.ncells; c += cstride) {
        int x, y, z;
        cell_xyz((uint32_t)c, (uint32_t)sp.nx, (uint32_t)sp.ny, x, y, z);
        step_cell<L, S, COLL>(sp, x, y, z, step_now, GlobalGather<L, S, Real>{sp, y, z});
      }
    }
    if (!run_barrier(count, nb, (uint32_t)s, sp.status)) return;
    if (blockIdx.x == 0) {
      for (int b = 0; b < sp.fin_blocks; ++b) finalize_partial(sp, b);
      finalize_total(sp, sp.fin_blocks);
    }
  }
}

}  // namespace AERO_KNS
}  // namespace aero
