// lbm_quad.cuh -- the D3Q19 step with four cells per thread for 16-bit
// population storage (FP16 / BF16 deviations), single lattices.
//
// With 16-bit storage the step moves half the bytes of FP32 but the two-
// cells-per-thread kernel (lbm_pair.cuh) leaves DRAM two-thirds idle: it is
// bound by memory latency, each thread having 19 loads of 2-4 bytes per
// cell pair in flight.  Here a thread takes the four cells x .. x+3 of a row
// (x a multiple of 4) and reads each direction's source with ONE aligned
// 8-byte load -- the four 16-bit values of the source row at x .. x+3.  The
// directions with e_x = +1 need x-1 .. x+2 and those with e_x = -1 need
// x+1 .. x+4: the missing value comes from the neighbouring lane's load
// through a warp shuffle (the first / last lane of a warp, or of a row,
// loads it itself), and two funnel shifts realign the four values.  Every
// load is issued before any arithmetic, so a thread has 152 bytes in flight
// where the pair kernel has 76.  The realigned words are parked in shared
// memory (each thread reads back only its own), so the two pair updates that
// follow do not hold the raw data in registers: the quad runs as two pairs
// through the pair arithmetic of lbm_pair.cuh (sponge, MRT in the adapted
// basis or BGK / TRT with each cell's LES rate, all on packed FP32
// instructions), and each pair's result is stored as one 4-byte half2 /
// bfloat162 per direction.
//
// Work split: in lattices with an open inlet and outlet the columns 0 .. 3
// and nx-4 .. nx-1 (inlet, outlet and the column the outlet copies) run the
// per-cell chain in edge blocks of their own, as in the pair kernel;
// streamwise periodic lattices have no edge columns and the quads cover
// whole rows, the x wrap taken by the shuffles' edge loads.  A quad that is
// not plain fluid (a flag bit set in any of its cells, or a wall row) runs
// the per-cell chain for its four cells.  Each lane performs the pair
// kernel's operations in the same order, so plain cells get the pair
// kernel's results.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbm_pair.cuh"

namespace aero {
inline namespace AERO_KNS {

// Two cells packed in 32 bits <-> their deviations as F2, with the scales
// and conversions of PairOps (bit-identical values).
template <class S> struct QuadOps;

template <> struct QuadOps<__half> {
  template <int I, class L>
  static __device__ __forceinline__ F2 unpack(uint32_t u) {
    constexpr float s = float(L::w[I] / 64.0);
    return F2(__fmul2_rn(__half22float2(*reinterpret_cast<const __half2 *>(&u)), make_float2(s, s)));
  }
  template <int I, class L>
  static __device__ __forceinline__ uint32_t pack(F2 v) {
    constexpr float s = float(64.0 / L::w[I]);
    const __half2 h = __float22half2_rn(__fmul2_rn(v.v, make_float2(s, s)));
    return *reinterpret_cast<const uint32_t *>(&h);
  }
};

template <> struct QuadOps<__nv_bfloat16> {
  template <int I, class L>
  static __device__ __forceinline__ F2 unpack(uint32_t u) {
    return F2(__bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u)));
  }
  template <int I, class L>
  static __device__ __forceinline__ uint32_t pack(F2 v) {
    const __nv_bfloat162 h = __float22bfloat162_rn(v.v);
    return *reinterpret_cast<const uint32_t *>(&h);
  }
};

// 8 bytes (cells o .. o+3, o a multiple of 4) of a 16-bit direction plane.
__device__ __forceinline__ uint2 ld_quad(const void *p) {
#if AERO_L2_256B
  uint2 v;
  asm("ld.global.nc.L2::256B.v2.b32 {%0, %1}, [%2];" : "=r"(v.x), "=r"(v.y) : "l"(p));
  return v;
#else
  return __ldg(static_cast<const uint2 *>(p));
#endif
}

constexpr int kQuadBlock = 128;  // threads per block
constexpr int kQuadRows = 16;    // rows per group; a group's edge block holds their 8 edge cells each
#ifndef AERO_QUAD_MINB
#define AERO_QUAD_MINB 6
#endif
constexpr int kQuadMinBlocks = AERO_QUAD_MINB;

// Work split.  A row's quads take TP threads (its quad count rounded up to
// whole warps, so a warp never spans two rows and the shuffles stay within a
// row); a block holds RB = 128 / TP rows when TP <= 128, else a row takes
// bpr blocks.  Rows come in groups of kQuadRows: the group's quad blocks,
// then (open lattices) its edge block.  One-dimensional grid.
struct QuadSplit {
  int x0, nquads, TP, RB, bpr, rows, groups, gblocks;
  bool edges;  // open lattices: columns 0..3 and nx-4..nx-1 run per cell in edge blocks
};

template <class Real>
__host__ __device__ __forceinline__ QuadSplit quad_split(const StepParams<Real> &p) {
  QuadSplit q;
  q.edges = (FEAT_OF(p) & (FEAT_OPEN | FEAT_RECYCLE)) != 0;  // inlet / outlet / recycling columns
  q.x0 = q.edges ? 4 : 0;
  q.nquads = q.edges ? (p.nx - 8) / 4 : p.nx / 4;
  q.TP = (q.nquads + 31) / 32 * 32;
  q.RB = q.TP <= kQuadBlock ? kQuadBlock / q.TP : 1;  // 4, 2 or 1: divides kQuadRows
  q.bpr = q.TP <= kQuadBlock ? 1 : (q.TP + kQuadBlock - 1) / kQuadBlock;
  q.rows = p.ny * p.nz;
  q.groups = (q.rows + kQuadRows - 1) / kQuadRows;
  q.gblocks = (kQuadRows / q.RB) * q.bpr + (q.edges ? 1 : 0);
  return q;
}

template <class Real>
inline dim3 quad_grid(const StepParams<Real> &p) {
  const QuadSplit q = quad_split(p);
  return dim3((unsigned)((int64_t)q.groups * q.gblocks), 1, 1);
}

// The plain-quad step: the two pairs of the quad, their 16-bit values read
// back from the block's shared-memory parking area (sq: direction i, half h
// at sq[(i * 2 + h) * kQuadBlock + tid]).
template <class L, class S, int COLL>
__device__ __forceinline__ void quad_step_plain(const StepParams<float> &p, int x, int y, int z, uint32_t c,
                                                int64_t step_now, const uint32_t *sq) {
  using QO = QuadOps<S>;
  S *Pn = static_cast<S *>(p.Pn);
  const bool les = (COLL != COLL_MRT) && (FEAT_OF(p) & FEAT_LES);
  const int tid = threadIdx.x;
#pragma unroll 1
  for (int h = 0; h < 2; h++) {
    const int xp = x + 2 * h;
    F2 d[L::Q];
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = QO::template unpack<i, L>(sq[(i * 2 + h) * kQuadBlock + tid]);
    });
    pair_sponge<L>(p, xp, d);
    F2 rho;
    if constexpr (COLL == COLL_MRT) {
      rho = mrt3_core<float, F2>(p.mrt3, d, false);
    } else {
      F2 om(p.omega);
      if (les)
        om = F2(make_float2(les_omega<L>(p, xp, y, z, c + 2 * h, false),
                            les_omega<L>(p, xp + 1, y, z, c + 2 * h + 1, false)));
      rho = collide_pair_bt<L, COLL>(p, d, om, les);
    }
    guard_bad(p, !(rho.v.x > 0.f) || !isfinite(rho.v.x) || !(rho.v.y > 0.f) || !isfinite(rho.v.y), step_now);
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      *reinterpret_cast<uint32_t *>(Pn + elem(p, i, c + 2 * h)) = QO::template pack<i, L>(d[i]);
    });
  }
}

// One regular step of a D3Q19 lattice with 16-bit storage, four cells per
// thread.  The host offers it for nx a multiple of 4 (>= 12 with an open
// inlet), without body force or scalar lattice.
template <class L, class S, int COLL>
__global__ void __launch_bounds__(kQuadBlock, kQuadMinBlocks) k_step_quad(const StepParams<float> p) {
  static_assert(L::DIMS == 3 && sizeof(S) == 2, "the quad kernel covers D3Q19 with 16-bit storage");
  __shared__ uint32_t sq[L::Q * 2 * kQuadBlock];  // the realigned words of each thread's quad
  const QuadSplit qs = quad_split(p);
  const int64_t step_now = *p.step;
  const int g = (int)(blockIdx.x / (unsigned)qs.gblocks);
  const int k = (int)(blockIdx.x - (unsigned)g * (unsigned)qs.gblocks);
  if (qs.edges && k == qs.gblocks - 1) {
    // edge block: cell e (0..7) of row g * kQuadRows + threadIdx.x / 8
    const int e = threadIdx.x & 7;
    const int r = g * kQuadRows + (int)(threadIdx.x >> 3);
    if (r >= qs.rows) return;
    const int y = r % p.ny, z = r / p.ny;
    step_cell<L, S, COLL>(p, e < 4 ? e : p.nx - 8 + e, y, z, step_now, GlobalGather<L, S, float>{p, y, z});
    return;
  }
  const int slot = k / qs.bpr, part = k - slot * qs.bpr;  // RB-row slot of the group, block of the row
  const int rl = qs.TP <= kQuadBlock ? (int)threadIdx.x / qs.TP : 0;
  const int t = qs.TP <= kQuadBlock ? (int)threadIdx.x - rl * qs.TP : part * kQuadBlock + (int)threadIdx.x;
  const int r = g * kQuadRows + slot * qs.RB + rl;
  if (rl >= qs.RB || r >= qs.rows) return;  // whole warps (TP is a multiple of 32)
  const bool active = t < qs.nquads;
  // inactive lanes at the end of a row take part in the shuffles with the
  // row's last quad as their (unused) data
  const int tq = active ? t : qs.nquads - 1;
  const int x = qs.x0 + 4 * tq, y = r % p.ny, z = r / p.ny;
  const int lane = threadIdx.x & 31;
  // a lane's left / right neighbour holds the adjacent quad of the same row
  // unless it is the first / last lane of the warp or the row
  const bool own_left = lane == 0 || t == 0;
  const bool own_right = lane == 31 || t + 1 >= qs.nquads;
  const S *P = static_cast<const S *>(p.P);
  const uint32_t nx = p.nx, nxy = (uint32_t)p.nx * (uint32_t)p.ny;
  const uint32_t ry_0 = (uint32_t)y * nx;
  const uint32_t ry_p = (y == 0 ? p.ny - 1 : y - 1) * nx;   // ey = +1
  const uint32_t ry_m = (y == p.ny - 1 ? 0 : y + 1) * nx;   // ey = -1
  const uint32_t pz_0 = (uint32_t)z * nxy;
  const uint32_t pz_p = (z == 0 ? p.nz - 1 : z - 1) * nxy;
  const uint32_t pz_m = (z == p.nz - 1 ? 0 : z + 1) * nxy;
  // the element left of x and right of x + 3 in the source row, x-periodic
  const uint32_t xl = x == 0 ? nx - 2 : (uint32_t)x - 2;   // the 4-byte word holding x - 1
  const uint32_t xr = (uint32_t)x + 4 == nx ? 0 : (uint32_t)x + 4;  // the word holding x + 4
  uint2 raw[L::Q];
  uint32_t side[L::Q];
  // all loads first: 19 aligned 8-byte words, plus the edge lanes' 4-byte words
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ex = Dir<L, i>::x, ey = Dir<L, i>::y, ez = Dir<L, i>::z;
    const uint32_t row = (ey > 0 ? ry_p : (ey < 0 ? ry_m : ry_0)) + (ez > 0 ? pz_p : (ez < 0 ? pz_m : pz_0));
    raw[i] = ld_quad(P + elem(p, i, row + (uint32_t)x));
    side[i] = 0u;
    if constexpr (ex > 0) {
      if (own_left) side[i] = ld_pop32(P + elem(p, i, row + xl));
    } else if constexpr (ex < 0) {
      if (own_right) side[i] = ld_pop32(P + elem(p, i, row + xr));
    }
  });
  // realign the shifted directions and park every word in shared memory
  const int tid = threadIdx.x;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ex = Dir<L, i>::x;
    uint32_t lo = raw[i].x, hi = raw[i].y;
    if constexpr (ex > 0) {
      // cells x-1 .. x+2: the high half of the word left of x, then x .. x+2
      const uint32_t nb = __shfl_up_sync(0xffffffffu, raw[i].y, 1);
      const uint32_t left = own_left ? side[i] : nb;
      lo = __funnelshift_r(left, raw[i].x, 16);
      hi = __funnelshift_r(raw[i].x, raw[i].y, 16);
    } else if constexpr (ex < 0) {
      // cells x+1 .. x+4: x+1 .. x+3, then the low half of the word right of x+3
      const uint32_t nb = __shfl_down_sync(0xffffffffu, raw[i].x, 1);
      const uint32_t right = own_right ? side[i] : nb;
      lo = __funnelshift_r(raw[i].x, raw[i].y, 16);
      hi = __funnelshift_r(raw[i].y, right, 16);
    }
    sq[(i * 2 + 0) * kQuadBlock + tid] = lo;
    sq[(i * 2 + 1) * kQuadBlock + tid] = hi;
  });
  if (!active) return;
  const uint32_t c = cell_index(p, x, y, z);
  bool plain = !(WALL_OF(p) != WALL_NONE && (y == 0 || y == p.ny - 1));
  if (plain) plain = *reinterpret_cast<const uint32_t *>(p.flags + c) == 0u;  // the four flag bytes, c % 4 == 0
  if (plain) {
    quad_step_plain<L, S, COLL>(p, x, y, z, c, step_now, sq);
    return;
  }
  const GlobalGather<L, S, float> gather{p, y, z};
#pragma unroll 1
  for (int e = 0; e < 4; e++) step_cell<L, S, COLL>(p, x + e, y, z, step_now, gather);
}

}  // namespace AERO_KNS
}  // namespace aero
