// lbm_params.h -- launch parameters shared by the host runtime and the
// sm_100a kernels of the aero_b200 lattice Boltzmann engine.
#pragma once
#include <stdint.h>

namespace aero {

enum Collision : int32_t { COLL_BGK = 0, COLL_TRT = 1, COLL_MRT = 2 };
enum StoreKind : int32_t { STORE_F32 = 0, STORE_F64 = 1, STORE_F16 = 2, STORE_BF16 = 3 };
enum Inlet : int32_t { INLET_NONE = 0, INLET_VELOCITY = 1, INLET_PRESSURE = 2 };
enum Outlet : int32_t { OUTLET_NONE = 0, OUTLET_CONVECTIVE = 1, OUTLET_ZEROGRAD = 2, OUTLET_PRESSURE = 3 };
enum Wall : int32_t { WALL_NONE = 0, WALL_SLIP = 1, WALL_NOSLIP = 2, WALL_MOVING = 3 };

enum Feature : uint32_t {
  FEAT_BOUZIDI = 1u << 0,
  FEAT_BODY_FORCE = 1u << 1,
  FEAT_SPONGE = 1u << 2,
  FEAT_LES = 1u << 3,
  FEAT_LES_WALE = 1u << 4,
  FEAT_LES_CS_FIELD = 1u << 5,  // per-cell Smagorinsky constant (van Driest damping)
  FEAT_THERMAL = 1u << 6,
  FEAT_BUOYANCY = 1u << 7,
  FEAT_SCALAR_REDUCED = 1u << 8,  // D2Q5 / D3Q7 scalar lattice
  FEAT_OPEN = 1u << 9,            // streamwise open: inlet/outlet active
  FEAT_OBSTACLE_BB = 1u << 10,    // obstacle bounce-back active (links present)
  FEAT_INFLOW_FIELD = 1u << 11,   // velocity inlet from per-step transverse fields (synthetic inflow)
  FEAT_RECYCLE = 1u << 12,        // 3D recycling inlet (rescaled equilibrium of plane nx-2)
  FEAT_INFLOW_SEM = 1u << 13,     // with FEAT_INFLOW_FIELD: SEM fluctuations (u', v', w') per step
};

// Per-cell flag byte.
enum CellFlag : uint8_t {
  FLAG_SOLID = 1u << 0,
  FLAG_LINK = 1u << 1,  // the cell has at least one obstacle link
};

// Status bits raised by the kernels (atomicOr into a device word).
enum Status : uint32_t {
  STATUS_NONFINITE_OR_NONPOSITIVE_RHO = 1u << 0,
  STATUS_WAIT_TIMEOUT = 1u << 1,  // a bounded device-side wait gave up (the step's output is incomplete)
};

// MRT operator in the even/odd pair basis (see lbm_mrt.cpp).  For D3Q19:
// even block 10x10, 7 equilibrium moments; odd block 9x9, 3 momenta.
template <class Real>
struct MrtCoeffs {
  Real Ae[10 * 10];
  Real Ce[10 * 7];
  Real Ao[9 * 9];
  Real Co[9 * 3];
};

// D3Q19 MRT blocks in the cubic-symmetry-adapted basis (see lbm_mrt.cpp):
// a1 3x3 (scalars), ca1 3x2 (their equilibrium inputs drho, rho u.u),
// e 2x2 and ce 2x1 (doublets), t2 / ct2 (shear-type edge differences),
// v 2x2 and cv 2x1 (momentum-like pairs).
template <class Real>
struct Mrt3Adapted {
  Real a1[9], ca1[6], e[4], ce[2], t2, ct2, v[4], cv[2];
};

// Everything a kernel needs for one step of one lattice.  Passed by value
// (kernel parameter space), so per-step variation lives in device memory
// (step counter) and the struct can be captured once in a CUDA graph.
template <class Real>
struct StepParams {
  int32_t nx, ny, nz;
  int32_t nwx;          // 32-cell words per x row = ceil(nx / 32)
  int64_t cs;           // population plane stride (cells, padded)
  int64_t ncells;       // nx * ny * nz
  uint32_t feat;
  int32_t inlet, outlet, wall;
  int32_t sponge_start; // first sponge x plane (>= nx when off)
  int32_t sponge_thickness;
  // row tiles of the tiled step kernel: tile_rows y rows of one z plane
  int32_t tile_rows, tiles_per_plane, ntiles;
  int32_t batch_rows;   // rows per block in the batched cell kernels
  int32_t les_chunk;    // planes per block of the fused LES step (k_step_les)
  uint32_t tile_extra_tx;  // bytes announced on a tile stage beyond its copies (0; > 0 only to test
                           // that the bounded stage waits give up)

  // populations (deviation from the rest weights, see Store<>)
  const void *P;        // current post-collision populations (read)
  void *Pn;             // next post-collision populations (written); = P in the AA layout
  // AA layout (one buffer updated in place).  aa_layout 0: value V_i of cell
  // x at plane opp(i), cell x; 1: at plane i, cell x + e_i (x-, y-, z-periodic).
  int32_t aa;             // 1 in the AA layout
  int32_t aa_layout;      // layout of the buffer's contents before this launch
  int32_t aa_store_state; // the step stores its post-boundary state instead of colliding it
  int32_t aa_shfl_out;    // the outlet cells take the state of x = nx-2 from the neighbour lane
  void *stage_link;       // per link cell: its Q pre-stream populations (Real)
  void *stage_nb;         // per link cell: the clipped neighbour's pre-stream value of each Bouzidi
                          // link with q >= 1/2 (Real, Q per link cell)
  void *stage_out;        // the pulled populations of plane x = nx-2, (Q, nz, ny) Real; NULL
                          // without an outlet that re-evaluates that plane
  const uint8_t *flags; // (cells) CellFlag bits; the buffer has 32 bytes of slack past cs
  const uint32_t *lbits;  // per 32-cell word: bit k set when cell k of the word has links
  const int32_t *loff;    // per 32-cell word: index of its first link cell
  const uint32_t *lc_mask;  // per link cell: bit i set when direction i is a link
  const float *lc_q;        // per link cell: q for each direction (Q floats)
  const int64_t *lc_cell;   // per link cell: cell index
  int64_t n_lc;

  const Real *prev;     // convective outlet state (nz, ny, QP), deviations
  Real *prevn;
  const Real *g;        // scalar state (Qg, cells) -- populations, not deviations
  Real *gn;
  const Real *U;        // LES velocities (3, cells) of the current state
  Real *Uw;             // LES velocity side output (written by the moments pass)
  const Real *cs_cell;  // per-cell LES constant (van Driest), optional
  const Real *inflow;   // inflow ring: inflow_ring steps x components x (nz*ny) inlet velocities
  int32_t inflow_ring;
  double *recycle_partial;  // per k_recycle_mean block: sum of ux over its cells
  double *recycle_mean;     // mean ux of the recycle plane of the current step
  uint32_t *recycle_ticket;
  int32_t recycle_blocks;

  // force reduction
  double *lc_contrib;   // 12 x n_lc doubles, component-major: deviation part of each link cell's forces
  double *fin_partial;  // per k_finalize block: 12 partial sums
  uint32_t *fin_ticket; // blocks of k_finalize done (reset by the last one)
  int64_t fin_chunk;    // link cells per k_finalize block
  int32_t fin_blocks;   // k_finalize grid size (<= kFinalizeMaxBlocks)
  const double *force_const;  // 12 doubles: rest-weight part of the forces
  const double *prof_const;   // nprof * 3 doubles: rest-weight part of the profile
  const int32_t *prof_off;  // nprof + 1 segment offsets into the link-cell list
  double *hist;         // force history ring: hist_cap * 12 doubles
  double *prof_out;     // last profile: nprof * 3 doubles
  int32_t nprof;
  int32_t hist_cap;
  int32_t want_profile;
  int64_t *step;        // device step counter (steps completed)
  const int64_t *profile_step;  // the profile is summed only by the step that completes this count
  int64_t *hist_base;   // step index stored in hist slot 0
  uint32_t *status;
  unsigned long long *first_bad_step;  // smallest step whose state had a bad density

  // physics (Real)
  Real omega, u0, rho_in, rho_out, pert_amp, trt_lambda, trt_sminus;
  Real sponge_sigma_max;
  Real base_nu, les_cs2;
  Real wall_u_top, wall_u_bottom;
  Real bf_x, bf_y, bf_z, bf_coeff;
  Real omega_T, T_hot, T_cold, gbeta, T_ref;
  double center[3];
  MrtCoeffs<Real> mrt;      // D2Q9
  Mrt3Adapted<Real> mrt3;   // D3Q19
};

// Macroscopic fields of an equilibrium state (k_init_equilibrium): FP64
// device arrays of ncells values, or NULL for the uniform value.
struct EqFields {
  const double *rho, *ux, *uy, *uz, *T;
  double rho0, u0, T0;
};

// Block layout of one lattice in the two-cells-per-thread batch kernel
// (128-thread blocks).  A row's P pairs (x, x+1), x = 2, 4, .., nx - 4, take
// TP threads (P rounded up to whole warps); a block holds RB rows of them
// (TP <= 128) or a row takes bpr blocks (TP > 128).  The four edge cells of
// a row (x = 0, 1, nx - 2, nx - 1) follow, 32 rows per block.  nx even.
struct PairBatchLayout {
  int P, TP, RB, bpr;
  int64_t rows, pair_blocks, edge_blocks;
};

#if defined(__CUDACC__)
__host__ __device__
#endif
inline PairBatchLayout pair_batch_layout(int nx, int ny, int nz) {
  PairBatchLayout l;
  l.P = nx >= 6 ? (nx - 4) / 2 : 0;
  l.TP = (l.P + 31) / 32 * 32;
  l.RB = (l.TP > 0 && l.TP <= 128) ? 128 / l.TP : 1;
  l.bpr = l.TP > 128 ? (l.TP + 127) / 128 : 1;
  l.rows = (int64_t)ny * nz;
  l.pair_blocks = l.P > 0 ? (l.rows + l.RB - 1) / l.RB * l.bpr : 0;
  l.edge_blocks = (l.rows + 31) / 32;
  return l;
}

}  // namespace aero
