// lbm_les.cuh -- the D3Q19 BGK / TRT step with the LES rate computed from a
// shared-memory velocity stencil, in one kernel.
//
// The LES rate of a cell (les.py:24-78, :219-262, :273-344) needs the
// velocity of the post-boundary state of its six face neighbours, i.e. of
// cells other threads are still evaluating in the same step.  The two-pass
// form runs a moments pass first (a full second gather of every population
// plus a 12-byte velocity side output per cell, which the step kernel reads
// back).  This kernel does it in one pass:
//
//   * A block owns a tile of 32 x kLesRows (x, y) columns and marches along
//     z through a chunk of planes.  Its threads evaluate the post-boundary
//     state (gather, body force, bounce-back, inlet / outlet, sponge,
//     walls, buoyancy: full_state) of the tile's cells and of a one-cell
//     halo around it (the rows above and below, the columns left and
//     right; the stencil has no diagonal neighbours, so no corners), plane
//     by plane, and write each cell's velocity into a ring of four planes
//     in shared memory.  The chunk's first and last planes are also
//     evaluated one plane beyond the chunk, for the z neighbours.
//   * The tile's own cells also park their state (and the scalar inputs) in
//     shared memory, and collide one plane behind the evaluation: once the
//     velocities of planes z-1, z and z+1 are all in shared memory, plane z's
//     cells take their velocity gradient from there, derive the WALE or
//     Smagorinsky rate and finish the step (forces, scalar, collision,
//     store) as the per-cell kernel does.
//
// One barrier per plane separates evaluation from collision; the rings are
// deep enough (four velocity planes, three state planes) that a warp
// evaluating plane z+1 never overwrites what a slower warp still reads.
// The velocities are computed with the moments pass's arithmetic, so the
// results equal the two-pass form's bit for bit.  The halo costs about a
// third more state evaluations than cells (mostly L2 hits); the moments
// pass it replaces cost a whole second gather from HBM.
#pragma once

#include "lbm_kernels.cuh"

namespace aero {
inline namespace AERO_KNS {

constexpr int kLesTileX = 32;                      // one warp per tile row
constexpr int kLesRows = 8;                        // tile rows (y)
constexpr int kLesInnerWarps = kLesRows;           // warps 0..7: the tile's rows
constexpr int kLesWarps = kLesInnerWarps + 3;      // + halo rows y0-1, y0+8, + halo columns
constexpr int kLesThreads = 32 * kLesWarps;        // 352
constexpr int kLesSlots = (kLesTileX + 2) * (kLesRows + 2);  // velocity slots of a plane (halo included)

template <class Real>
struct LesSmem {
  Real u[4][3][kLesSlots];                      // velocity ring: plane z at z & 3
  Real s[3][19][kLesTileX * kLesRows];          // states of the tile's cells: plane z at z % 3
  Real sc[3][4][kLesTileX * kLesRows];          // scalar inputs (T, u before buoyancy)
};

// Shared-memory bytes of the kernel for a storage type (host side).
template <class Real>
constexpr size_t les_smem_bytes() { return sizeof(LesSmem<Real>); }

// The thread's column in the tile: (lx, ly) in [-1, 32] x [-1, kLesRows],
// inner = one of the tile's own cells.  Returns false for idle lanes.
__device__ __forceinline__ bool les_column(int tid, int &lx, int &ly, bool &inner) {
  const int w = tid >> 5, lane = tid & 31;
  inner = w < kLesInnerWarps;
  if (inner) {
    lx = lane;
    ly = w;
    return true;
  }
  if (w == kLesInnerWarps) {  // the row below the tile
    lx = lane;
    ly = -1;
    return true;
  }
  if (w == kLesInnerWarps + 1) {  // the row above
    lx = lane;
    ly = kLesRows;
    return true;
  }
  if (lane < kLesRows) {  // the column left of the tile
    lx = -1;
    ly = lane;
    return true;
  }
  if (lane < 2 * kLesRows) {  // the column right of it
    lx = kLesTileX;
    ly = lane - kLesRows;
    return true;
  }
  return false;
}

__device__ __forceinline__ int les_slot(int lx, int ly) { return (ly + 1) * (kLesTileX + 2) + (lx + 1); }

// grid: x = tiles along x, y = tiles along y, z = chunks of p.les_chunk planes
template <class L, class S, int COLL>
__global__ void __launch_bounds__(kLesThreads, sizeof(typename StoreOps<S>::Real) == 4 ? 2 : 1)
    k_step_les(const StepParams<typename StoreOps<S>::Real> p) {
  static_assert(L::DIMS == 3 && COLL != COLL_MRT, "the fused LES step covers D3Q19 BGK / TRT");
  using Real = typename StoreOps<S>::Real;
  extern __shared__ __align__(16) unsigned char les_smem_raw[];
  LesSmem<Real> &sm = *reinterpret_cast<LesSmem<Real> *>(les_smem_raw);
  const int tid = threadIdx.x;
  int lx = 0, ly = 0;
  bool inner = false;
  const bool has_col = les_column(tid, lx, ly, inner);
  const int x = (int)blockIdx.x * kLesTileX + lx, y = (int)blockIdx.y * kLesRows + ly;
  const bool in_grid = has_col && x >= 0 && x < p.nx && y >= 0 && y < p.ny;
  const int it = inner ? ly * kLesTileX + lx : 0;  // index of an inner cell in the state ring
  const int slot = les_slot(lx, ly);
  const int zc0 = (int)blockIdx.z * p.les_chunk;
  const int zc1 = zc0 + p.les_chunk < p.nz ? zc0 + p.les_chunk : p.nz;
  const int64_t step_now = *p.step;
  for (int zi = zc0 - 1; zi <= zc1; ++zi) {
    // evaluation of plane zi: every column with a cell in the grid
    if (zi >= 0 && zi < p.nz && in_grid) {
      const bool own = inner && zi >= zc0 && zi < zc1;
      Real d[L::Q];
      ScalarCtx<Real> sc;
      const GlobalGather<L, S, Real> gz{p, y, zi};
      full_state<L, S, Real>(p, x, y, zi, step_now, d, own ? p.prevn : nullptr, &sc, gz);
      // the velocity as the moments pass computes it (moments_cell)
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
      const int u = zi & 3;
      sm.u[u][0][slot] = jx * inv;
      sm.u[u][1][slot] = jy * inv;
      sm.u[u][2][slot] = jz * inv;
      if (own) {
        const int k = zi % 3;
        static_for<L::Q>([&](auto ic) {
          constexpr int i = decltype(ic)::value;
          sm.s[k][i][it] = d[i];
        });
        if (FEAT_OF(p) & FEAT_THERMAL) {
          sm.sc[k][0][it] = sc.T;
          sm.sc[k][1][it] = sc.u[0];
          sm.sc[k][2][it] = sc.u[1];
          sm.sc[k][3][it] = sc.u[2];
        }
      }
    }
    __syncthreads();
    // collision of plane zb = zi - 1 by the tile's own cells
    const int zb = zi - 1;
    if (inner && in_grid && zb >= zc0 && zb < zc1) {
      const int k = zb % 3;
      Real d[L::Q];
      static_for<L::Q>([&](auto ic) {
        constexpr int i = decltype(ic)::value;
        d[i] = sm.s[k][i][it];
      });
      ScalarCtx<Real> sc{};
      if (FEAT_OF(p) & FEAT_THERMAL) {
        sc.T = sm.sc[k][0][it];
        sc.u[0] = sm.sc[k][1][it];
        sc.u[1] = sm.sc[k][2][it];
        sc.u[2] = sm.sc[k][3][it];
      }
      const uint32_t c = cell_index(p, x, y, zb);
      const uint32_t flc = p.flags[c];
      Real om;
      if (!les_interior<L>(p, x, y, zb) || (flc & FLAG_SOLID)) {
        om = Real(1) / (Real(3) * p.base_nu + Real(0.5));
      } else {
        // velocity gradient from the ring (planes zb - 1, zb, zb + 1)
        const int um = (zb + 3) & 3, u0 = zb & 3, up = (zb + 1) & 3;
        const int sxm = les_slot(lx - 1, ly), sxp = les_slot(lx + 1, ly);
        const int sym = les_slot(lx, ly - 1), syp = les_slot(lx, ly + 1);
        Real g[3][3];
#pragma unroll
        for (int a = 0; a < 3; a++) {
          g[a][0] = Real(0.5) * (sm.u[u0][a][sxp] - sm.u[u0][a][sxm]);
          g[a][1] = Real(0.5) * (sm.u[u0][a][syp] - sm.u[u0][a][sym]);
          g[a][2] = Real(0.5) * (sm.u[up][a][slot] - sm.u[um][a][slot]);
        }
        om = les_rate_from_gradient<L>(p, g, c);
      }
      finish_cell<L, S, COLL>(p, x, y, zb, c, flc, step_now, d, sc, om, true, GlobalGather<L, S, Real>{p, y, zb});
    }
  }
}

}  // namespace AERO_KNS
}  // namespace aero
