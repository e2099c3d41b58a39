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
// where the pair kernel has 76.  The quad then runs as two pairs through the
// pair arithmetic of lbm_pair.cuh (sponge, MRT in the adapted basis or BGK /
// TRT with each cell's LES rate, all on packed FP32 instructions), and each
// pair's result is stored as one 4-byte half2 / bfloat162 per direction.
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

constexpr int kQuadBlock = 128;  // threads per block: 512 cells along x
constexpr int kQuadRows = 16;    // rows per group; the group's edge block holds their 8 edge cells each
#ifndef AERO_QUAD_MINB
#define AERO_QUAD_MINB 6
#endif
constexpr int kQuadMinBlocks = AERO_QUAD_MINB;

struct QuadSplit {
  int x0, nquads, row_blocks, rows, groups;
  bool edges;  // open lattices: columns 0..3 and nx-4..nx-1 run per cell in edge blocks
};

template <class Real>
__host__ __device__ __forceinline__ QuadSplit quad_split(const StepParams<Real> &p) {
  QuadSplit q;
  q.edges = (p.feat & (FEAT_OPEN | FEAT_RECYCLE)) != 0;  // inlet / outlet / recycling columns
  q.x0 = q.edges ? 4 : 0;
  q.nquads = q.edges ? (p.nx - 8) / 4 : p.nx / 4;
  q.row_blocks = (q.nquads + kQuadBlock - 1) / kQuadBlock;
  q.rows = p.ny * p.nz;
  q.groups = (q.rows + kQuadRows - 1) / kQuadRows;
  return q;
}

template <class Real>
inline dim3 quad_grid(const StepParams<Real> &p) {
  const QuadSplit q = quad_split(p);
  return dim3((unsigned)(q.row_blocks > 0 ? q.row_blocks : 1), (unsigned)(kQuadRows + (q.edges ? 1 : 0)),
              (unsigned)q.groups);
}

// The plain-quad step: per direction, the four source values assembled from
// the lane's 8-byte load and a neighbour's, then the two pairs.
template <class L, class S, int COLL>
__device__ __forceinline__ void quad_step_plain(const StepParams<float> &p, int x, int y, int z, uint32_t c,
                                                int64_t step_now, const uint2 (&raw)[L::Q]) {
  using QO = QuadOps<S>;
  S *Pn = static_cast<S *>(p.Pn);
  const bool les = (COLL != COLL_MRT) && (p.feat & FEAT_LES);
#pragma unroll 1
  for (int h = 0; h < 2; h++) {
    const int xp = x + 2 * h;
    F2 d[L::Q];
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = QO::template unpack<i, L>(h == 0 ? raw[i].x : raw[i].y);
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
// inlet), without body force or scalar lattice.  Grid: x = quad block of a
// row, y = row of a group of kQuadRows rows (y = kQuadRows: the group's edge
// block, x = 0 only), z = group.
template <class L, class S, int COLL>
__global__ void __launch_bounds__(kQuadBlock, kQuadMinBlocks) k_step_quad(const StepParams<float> p) {
  static_assert(L::DIMS == 3 && sizeof(S) == 2, "the quad kernel covers D3Q19 with 16-bit storage");
  const QuadSplit qs = quad_split(p);
  const int64_t step_now = *p.step;
  if (blockIdx.y == kQuadRows) {
    // edge block: cell k (0..7) of row blockIdx.z * kQuadRows + threadIdx.x / 8
    if (blockIdx.x != 0) return;
    const int k = threadIdx.x & 7;
    const int r = (int)(blockIdx.z * kQuadRows + (threadIdx.x >> 3));
    if (r >= qs.rows) return;
    const int y = r % p.ny, z = r / p.ny;
    step_cell<L, S, COLL>(p, k < 4 ? k : p.nx - 8 + k, y, z, step_now, GlobalGather<L, S, float>{p, y, z});
    return;
  }
  const int r = (int)(blockIdx.z * kQuadRows + blockIdx.y);
  if (r >= qs.rows) return;  // whole warps leave together (r is uniform in the block)
  const int t = (int)(blockIdx.x * kQuadBlock + threadIdx.x);
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
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ex = Dir<L, i>::x;
    if constexpr (ex > 0) {
      // cells x-1 .. x+2: the high half of the word left of x, then x .. x+2
      const uint32_t nb = __shfl_up_sync(0xffffffffu, raw[i].y, 1);
      const uint32_t left = own_left ? side[i] : nb;
      const uint32_t lo = __funnelshift_r(left, raw[i].x, 16);
      const uint32_t hi = __funnelshift_r(raw[i].x, raw[i].y, 16);
      raw[i] = make_uint2(lo, hi);
    } else if constexpr (ex < 0) {
      // cells x+1 .. x+4: x+1 .. x+3, then the low half of the word right of x+3
      const uint32_t nb = __shfl_down_sync(0xffffffffu, raw[i].x, 1);
      const uint32_t right = own_right ? side[i] : nb;
      const uint32_t lo = __funnelshift_r(raw[i].x, raw[i].y, 16);
      const uint32_t hi = __funnelshift_r(raw[i].y, right, 16);
      raw[i] = make_uint2(lo, hi);
    }
  });
  if (!active) return;
  const uint32_t c = cell_index(p, x, y, z);
  bool plain = !(p.wall != WALL_NONE && (y == 0 || y == p.ny - 1));
  if (plain) plain = *reinterpret_cast<const uint32_t *>(p.flags + c) == 0u;  // the four flag bytes, c % 4 == 0
  if (plain) {
    quad_step_plain<L, S, COLL>(p, x, y, z, c, step_now, raw);
    return;
  }
  const GlobalGather<L, S, float> gather{p, y, z};
#pragma unroll 1
  for (int k = 0; k < 4; k++) step_cell<L, S, COLL>(p, x + k, y, z, step_now, gather);
}

}  // namespace aero
