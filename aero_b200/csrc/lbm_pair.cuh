// lbm_pair.cuh -- the D3Q19 MRT step with two cells per thread on the packed
// FP32 instructions of sm_100 (FADD2 / FMUL2 / FFMA2).
//
// The per-cell step kernel is issue-bound once populations are 16-bit: its
// collision, conversions and addressing take more instruction slots than the
// halved bytes take DRAM time.  Here a thread takes the cells (x, x+1) of one
// row, x even, in the columns clear of the inlet and the outlet.  When both
// are plain fluid cells -- no flag bit (solid, link), not a wall row -- the
// pair runs through the same sponge and collision (mrt3_core) with every
// value a float2, so each arithmetic step is one instruction for both cells;
// the loads of directions with e_x = 0 and every store move both cells'
// values as one aligned 8-byte (FP32) or 4-byte (16-bit) access.  Other pairs
// run the per-cell step for each cell, and the edge columns run it in blocks
// of their own.  Each lane does the per-cell step's operations in the same
// order; only where the per-cell compile fuses a product into a sum
// differently can the last bit differ.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbm_kernels.cuh"

namespace aero {

struct P2;

// Values of the two cells (x in .x, x+1 in .y).  Sums and products are packed
// instructions rounded to nearest; a product that feeds a sum stays pending
// (P2) and is fused into it, as the per-cell compile fuses them.
struct F2 {
  float2 v;
  F2() = default;
  __device__ __forceinline__ F2(float c) : v(make_float2(c, c)) {}
  __device__ __forceinline__ explicit F2(float2 a) : v(a) {}
  __device__ __forceinline__ F2(const P2 &p);
};

struct P2 {
  F2 a, b;
};

__device__ __forceinline__ F2 neg(F2 a) { return F2(make_float2(-a.v.x, -a.v.y)); }
__device__ __forceinline__ F2::F2(const P2 &p) : v(__fmul2_rn(p.a.v, p.b.v)) {}
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return F2(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return F2(__fadd2_rn(a.v, neg(b).v)); }
__device__ __forceinline__ P2 operator*(F2 a, F2 b) { return P2{a, b}; }
__device__ __forceinline__ F2 operator+(P2 p, F2 c) { return F2(__ffma2_rn(p.a.v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator+(F2 c, P2 p) { return F2(__ffma2_rn(p.a.v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator-(P2 p, F2 c) { return F2(__ffma2_rn(p.a.v, p.b.v, neg(c).v)); }
__device__ __forceinline__ F2 operator-(F2 c, P2 p) { return F2(__ffma2_rn(neg(p.a).v, p.b.v, c.v)); }
__device__ __forceinline__ F2 operator+(P2 p, P2 q) { return F2(__ffma2_rn(q.a.v, q.b.v, F2(p).v)); }
__device__ __forceinline__ F2 operator-(P2 p, P2 q) { return F2(__ffma2_rn(neg(q.a).v, q.b.v, F2(p).v)); }

__device__ __forceinline__ F2 pos_recip(F2 r) {
  return F2(make_float2(pos_recip(r.v.x), pos_recip(r.v.y)));
}

// Pair accesses of one direction plane: `aligned` reads the values of cells o
// and o+1 with one access (o even), `split` with two; store writes both (o
// even).  Conversions and scales are those of StoreOps, lane by lane.
template <class S> struct PairOps;

template <> struct PairOps<float> {
  template <int I, class L>
  static __device__ __forceinline__ F2 aligned(const float *p, uint32_t o) {
    return F2(ld_pop64(p + o));
  }
  template <int I, class L>
  static __device__ __forceinline__ F2 split(const float *p, uint32_t o) {
    return F2(make_float2(ld_pop(p + o), ld_pop(p + o + 1)));
  }
  template <int I, class L>
  static __device__ __forceinline__ void store(float *p, uint32_t o, F2 v) {
    *reinterpret_cast<float2 *>(p + o) = v.v;
  }
};

template <> struct PairOps<__half> {
  template <int I, class L>
  static __device__ __forceinline__ F2 scaled(float2 raw) {
    constexpr float s = float(L::w[I] / 64.0);
    return F2(__fmul2_rn(raw, make_float2(s, s)));
  }
  template <int I, class L>
  static __device__ __forceinline__ F2 aligned(const __half *p, uint32_t o) {
    const unsigned int u = ld_pop32(p + o);
    return scaled<I, L>(__half22float2(*reinterpret_cast<const __half2 *>(&u)));
  }
  template <int I, class L>
  static __device__ __forceinline__ F2 split(const __half *p, uint32_t o) {
    return scaled<I, L>(make_float2(__half2float(__ushort_as_half(ld_pop16(p + o))),
                                    __half2float(__ushort_as_half(ld_pop16(p + o + 1)))));
  }
  template <int I, class L>
  static __device__ __forceinline__ void store(__half *p, uint32_t o, F2 v) {
    constexpr float s = float(64.0 / L::w[I]);
    *reinterpret_cast<__half2 *>(p + o) = __float22half2_rn(__fmul2_rn(v.v, make_float2(s, s)));
  }
};

template <> struct PairOps<__nv_bfloat16> {
  template <int I, class L>
  static __device__ __forceinline__ F2 aligned(const __nv_bfloat16 *p, uint32_t o) {
    const unsigned int u = ld_pop32(p + o);
    return F2(__bfloat1622float2(*reinterpret_cast<const __nv_bfloat162 *>(&u)));
  }
  template <int I, class L>
  static __device__ __forceinline__ F2 split(const __nv_bfloat16 *p, uint32_t o) {
    return F2(make_float2(__bfloat162float(__ushort_as_bfloat16(ld_pop16(p + o))),
                          __bfloat162float(__ushort_as_bfloat16(ld_pop16(p + o + 1)))));
  }
  template <int I, class L>
  static __device__ __forceinline__ void store(__nv_bfloat16 *p, uint32_t o, F2 v) {
    *reinterpret_cast<__nv_bfloat162 *>(p + o) = __float22bfloat162_rn(v.v);
  }
};

// Pull gather of the pair (x, x+1), x even, 2 <= x, x + 1 <= nx - 2: neither
// cell's sources wrap in x; y and z wrap as in GlobalGather.
template <class L, class S>
__device__ __forceinline__ void pair_gather(const StepParams<float> &p, int x, int y, int z, F2 (&d)[L::Q]) {
  using PO = PairOps<S>;
  const S *P = static_cast<const S *>(p.P);
  const uint32_t nx = p.nx, nxy = (uint32_t)p.nx * (uint32_t)p.ny;
  const uint32_t ry_0 = (uint32_t)y * nx;
  const uint32_t ry_p = (y == 0 ? p.ny - 1 : y - 1) * nx;   // ey = +1
  const uint32_t ry_m = (y == p.ny - 1 ? 0 : y + 1) * nx;   // ey = -1
  const uint32_t pz_0 = (uint32_t)z * nxy;
  const uint32_t pz_p = (z == 0 ? p.nz - 1 : z - 1) * nxy;
  const uint32_t pz_m = (z == p.nz - 1 ? 0 : z + 1) * nxy;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ex = Dir<L, i>::x, ey = Dir<L, i>::y, ez = Dir<L, i>::z;
    const uint32_t src = (uint32_t)(x - ex) + (ey > 0 ? ry_p : (ey < 0 ? ry_m : ry_0)) +
                         (ez > 0 ? pz_p : (ez < 0 ? pz_m : pz_0));
    if constexpr (ex == 0)
      d[i] = PO::template aligned<i, L>(P, elem(p, i, src));
    else
      d[i] = PO::template split<i, L>(P, elem(p, i, src));
  });
}

// Outlet sponge on the pair (sponge.py:8-70), as full_state applies it to a
// cell: d <- (1 - s) d + s feq(rho, u0 x) with s = sigma_max frac^2, frac
// the cell's depth into the sponge; lanes outside the sponge keep d.
template <class L>
__device__ __forceinline__ void pair_sponge(const StepParams<float> &p, int x, F2 (&d)[L::Q]) {
  if (!(p.feat & FEAT_SPONGE) || x + 1 < p.sponge_start) return;
  float sgv[2];
#pragma unroll
  for (int k = 0; k < 2; k++) {
    const double frac =
        (double)(x + k - p.sponge_start + 1) / (double)(p.sponge_thickness > 1 ? p.sponge_thickness : 1);
    sgv[k] = x + k >= p.sponge_start ? (float)((double)p.sponge_sigma_max * frac * frac) : 0.f;
  }
  const F2 sg(make_float2(sgv[0], sgv[1]));
  F2 drho(0.f);
  static_for<L::Q>([&](auto ic) { drho = drho + d[decltype(ic)::value]; });
  const F2 rho = F2(1.f) + drho;
  const float u0 = p.u0, usq = u0 * u0;
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    const float eu = Dir<L, i>::x * u0;
    const F2 deq = float(Dir<L, i>::w) * (drho + rho * (3.f * eu + 4.5f * eu * eu - 1.5f * usq));
    const F2 r = (F2(1.f) - sg) * d[i] + sg * deq;
    d[i] = F2(make_float2(sgv[0] > 0.f ? r.v.x : d[i].v.x, sgv[1] > 0.f ? r.v.y : d[i].v.y));
  });
}

// Resident blocks of 128 threads per SM the pair kernel is built for (7: 72
// registers a thread, the most blocks without spills).
#ifndef AERO_PAIR_MINB
#define AERO_PAIR_MINB 7
#endif
constexpr int kPairBlock = 128;     // threads per block: 256 cells along x
constexpr int kPairMinBlocks = AERO_PAIR_MINB;

// Work split of the pair step.  The pairs (x, x+1), x even, of columns
// [2, xb), xb = nx - 2 -- clear of the inlet column and of the outlet column
// with the column it copies -- take two cells per thread; the edge columns 0,
// 1 and [xb, nx) one cell per thread.  Grid: x = pair block of a row, y = row
// of a group of kPairRows rows, z = group; y = kPairRows is the group's edge
// block (x = 0 only), which holds the edge cells of all its rows, so a warp
// of edge cells spans eight rows instead of leaving most of its lanes idle,
// and edge blocks run among pair blocks.
constexpr int kPairRows = kPairBlock / 4;

struct PairSplit {
  int xb, npairs, nedge, row_blocks, rows, groups;  // rows = ny * nz < 2^31
};

template <class Real>
__host__ __device__ __forceinline__ PairSplit pair_split(const StepParams<Real> &p) {
  PairSplit sp;
  sp.xb = (p.nx - 1) & ~1;
  if (sp.xb < 2) sp.xb = 2;
  sp.npairs = (sp.xb - 2) / 2;
  sp.nedge = 2 + (p.nx > sp.xb ? p.nx - sp.xb : 0);  // at most 4 for even nx
  sp.row_blocks = (sp.npairs + kPairBlock - 1) / kPairBlock;
  sp.rows = p.ny * p.nz;
  sp.groups = (sp.rows + kPairRows - 1) / kPairRows;
  return sp;
}

// One regular step of a D3Q19 MRT lattice.  The host offers it for even nx
// and without body force or scalar lattice (which act on every cell); pairs
// that are not plain fluid (solid, link, wall rows) and edge cells run
// step_cell.
template <class L, class S, int COLL>
__global__ void __launch_bounds__(kPairBlock, kPairMinBlocks) k_step_pair(const StepParams<float> p) {
  static_assert(L::DIMS == 3 && COLL == COLL_MRT, "the pair kernel covers the D3Q19 MRT step");
  const PairSplit sp = pair_split(p);
  const int64_t step_now = *p.step;
  if (blockIdx.y == kPairRows) {
    // edge block: cell k of row blockIdx.z * kPairRows + threadIdx.x / 4
    if (blockIdx.x != 0) return;
    const int k = threadIdx.x & 3;
    const int r = (int)(blockIdx.z * kPairRows + (threadIdx.x >> 2));
    if (k >= sp.nedge || r >= sp.rows) return;
    const int y = r % p.ny, z = r / p.ny;
    step_cell<L, S, COLL>(p, k < 2 ? k : sp.xb + (k - 2), y, z, step_now, GlobalGather<L, S, float>{p, y, z});
    return;
  }
  const int r = (int)(blockIdx.z * kPairRows + blockIdx.y);
  const int t = (int)(blockIdx.x * kPairBlock + threadIdx.x);
  if (r >= sp.rows || t >= sp.npairs) return;
  const int x = 2 + 2 * t, y = r % p.ny, z = r / p.ny;
  const uint32_t c = cell_index(p, x, y, z);
  bool plain = !(p.wall != WALL_NONE && (y == 0 || y == p.ny - 1));
  if (plain) plain = *reinterpret_cast<const uint16_t *>(p.flags + c) == 0;  // both flag bytes, c even
  if (plain) {
    F2 d[L::Q];
    pair_gather<L, S>(p, x, y, z, d);
    pair_sponge<L>(p, x, d);
    const F2 rho = mrt3_core<float, F2>(p.mrt3, d, false);
    guard_bad(p, !(rho.v.x > 0.f) || !isfinite(rho.v.x) || !(rho.v.y > 0.f) || !isfinite(rho.v.y), step_now);
    S *Pn = static_cast<S *>(p.Pn);
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      PairOps<S>::template store<i, L>(Pn, elem(p, i, c), d[i]);
    });
    return;
  }
  const GlobalGather<L, S, float> gather{p, y, z};
#pragma unroll 1
  for (int k = 0; k < 2; k++) step_cell<L, S, COLL>(p, x + k, y, z, step_now, gather);
}

template <class Real>
inline dim3 pair_grid(const StepParams<Real> &p) {
  const PairSplit sp = pair_split(p);
  return dim3((unsigned)(sp.row_blocks > 0 ? sp.row_blocks : 1), (unsigned)(kPairRows + 1), (unsigned)sp.groups);
}

}  // namespace aero
