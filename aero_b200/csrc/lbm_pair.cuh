// lbm_pair.cuh -- the D3Q19 step with two cells per thread on the packed FP32
// instructions of sm_100 (FADD2 / FMUL2 / FFMA2), single lattices and batches.
//
// The per-cell step kernel is issue-bound once populations are 16-bit: its
// collision, conversions and addressing take more instruction slots than the
// halved bytes take DRAM time.  Here a thread takes the cells (x, x+1) of one
// row, x even, in the columns clear of the inlet and the outlet.  When both
// are plain fluid cells -- no flag bit (solid, link), not a wall row -- the
// pair runs through the same sponge and collision (mrt3_core for MRT,
// collide_pair_bt for BGK / TRT) with every value a float2, so each
// arithmetic step is one instruction for both cells; the loads of directions
// with e_x = 0 and every store move both cells' values as one aligned 8-byte
// (FP32) or 4-byte (16-bit) access.  Other pairs run the per-cell step for
// each cell, and the edge columns run it in blocks of their own.  Each lane
// does the per-cell step's operations in the same order; only where the
// per-cell compile fuses a product into a sum differently can the last bit
// differ.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <type_traits>

#include "lbm_kernels.cuh"

namespace aero {
inline namespace AERO_KNS {

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
  if (!(FEAT_OF(p) & FEAT_SPONGE) || x + 1 < p.sponge_start) return;
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

// BGK / TRT collision of the pair, the operations of collide() (BGK:
// kernels.py:42-92, TRT: kernels_trt.py:125-174) lane by lane: moments,
// per-direction equilibrium, relaxation as a correction to d.  om is the
// pair's relaxation rate (the base rate, or each cell's LES rate, in which
// case TRT derives each cell's s- from it).  Plain fluid cells: no solid.
template <class L, int COLL>
__device__ __forceinline__ F2 collide_pair_bt(const StepParams<float> &p, F2 (&d)[L::Q], F2 om,
                                              bool per_cell_omega) {
  F2 drho(0.f), jx(0.f), jy(0.f), jz(0.f);
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    drho = drho + d[i];
    if constexpr (Dir<L, i>::x > 0) jx = jx + d[i];
    if constexpr (Dir<L, i>::x < 0) jx = jx - d[i];
    if constexpr (Dir<L, i>::y > 0) jy = jy + d[i];
    if constexpr (Dir<L, i>::y < 0) jy = jy - d[i];
    if constexpr (Dir<L, i>::z > 0) jz = jz + d[i];
    if constexpr (Dir<L, i>::z < 0) jz = jz - d[i];
  });
  const F2 rho = F2(1.f) + drho;
  const F2 inv = pos_recip(rho);
  const F2 ux = jx * inv, uy = jy * inv, uz = jz * inv;
  const F2 usq = ux * ux + uy * uy + uz * uz;
  // equilibrium deviation of direction i, evaluated where it is used (no
  // array of 19 values stays live beside the populations)
  auto deq = [&](auto ic) {
    constexpr int i = decltype(ic)::value;
    constexpr int ex = Dir<L, i>::x, ey = Dir<L, i>::y, ez = Dir<L, i>::z;
    F2 eu(0.f);
    if constexpr (ex > 0) eu = eu + ux;
    if constexpr (ex < 0) eu = eu - ux;
    if constexpr (ey > 0) eu = eu + uy;
    if constexpr (ey < 0) eu = eu - uy;
    if constexpr (ez > 0) eu = eu + uz;
    if constexpr (ez < 0) eu = eu - uz;
    const F2 poly = 3.f * eu + (4.5f * eu) * eu - 1.5f * usq;
    return F2(float(Dir<L, i>::w) * (drho + rho * poly));
  };
  if constexpr (COLL == COLL_TRT) {
    F2 sm(p.trt_sminus);
    if (per_cell_omega) {
      float smv[2];
      const float omv[2] = {om.v.x, om.v.y};
#pragma unroll
      for (int k = 0; k < 2; k++) {
        const float tau = 1.f / omv[k], lam = p.trt_lambda;
        const float tp = lam * tau + (1.f - lam);
        const float tm = (tp * tau - 0.5f) / (tp - 0.5f);
        smv[k] = 1.f / tm;
      }
      sm = F2(make_float2(smv[0], smv[1]));
    }
    d[0] = d[0] + om * (deq(std::integral_constant<int, 0>{}) - d[0]);
    static_for<L::NP>([&](auto pc) {
      constexpr int k = decltype(pc)::value;
      constexpr int i = L::pair[k], o = L::opp[L::pair[k]];
      const F2 qi = deq(std::integral_constant<int, i>{}), qo = deq(std::integral_constant<int, o>{});
      const F2 fp = 0.5f * (d[i] + d[o]), fm = 0.5f * (d[i] - d[o]);
      const F2 ep = 0.5f * (qi + qo), em = 0.5f * (qi - qo);
      const F2 a = om * (ep - fp), b = sm * (em - fm);
      d[i] = d[i] + (a + b);
      d[o] = d[o] + (a - b);
    });
  } else {
    static_for<L::Q>([&](auto ic) {
      constexpr int i = decltype(ic)::value;
      d[i] = d[i] + om * (deq(ic) - d[i]);
    });
  }
  return rho;
}

// The step of a plain pair (x, x+1), x even, c its first cell: gather,
// sponge, collision (MRT in the adapted basis, or BGK / TRT with the LES
// rate of each cell), divergence guard, store.
template <class L, class S, int COLL>
__device__ __forceinline__ void pair_step_plain(const StepParams<float> &p, int x, int y, int z, uint32_t c,
                                                int64_t step_now) {
  F2 d[L::Q];
  pair_gather<L, S>(p, x, y, z, d);
  pair_sponge<L>(p, x, d);
  F2 rho;
  if constexpr (COLL == COLL_MRT) {
    rho = mrt3_core<float, F2>(p.mrt3, d, false);
  } else {
    const bool les = FEAT_OF(p) & FEAT_LES;
    F2 om(p.omega);
    if (les) om = F2(make_float2(les_omega<L>(p, x, y, z, c, false), les_omega<L>(p, x + 1, y, z, c + 1, false)));
    rho = collide_pair_bt<L, COLL>(p, d, om, les);
  }
  guard_bad(p, !(rho.v.x > 0.f) || !isfinite(rho.v.x) || !(rho.v.y > 0.f) || !isfinite(rho.v.y), step_now);
  S *Pn = static_cast<S *>(p.Pn);
  static_for<L::Q>([&](auto ic) {
    constexpr int i = decltype(ic)::value;
    PairOps<S>::template store<i, L>(Pn, elem(p, i, c), d[i]);
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
  static_assert(L::DIMS == 3, "the pair kernel covers the D3Q19 step");
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
  bool plain = !(WALL_OF(p) != WALL_NONE && (y == 0 || y == p.ny - 1));
  if (plain) plain = *reinterpret_cast<const uint16_t *>(p.flags + c) == 0;  // both flag bytes, c even
  if (plain) {
    pair_step_plain<L, S, COLL>(p, x, y, z, c, step_now);
    return;
  }
  const GlobalGather<L, S, float> gather{p, y, z};
#pragma unroll 1
  for (int k = 0; k < 2; k++) step_cell<L, S, COLL>(p, x + k, y, z, step_now, gather);
}

// The batched step (k_step_batch) of a lattice class whose members all take
// the pair layout (pair_batch_layout): D3Q19, even nx >= 6, no body force or
// scalar lattice.  The member's parameters are copied into shared memory as
// in k_step_batch.
template <class L, class S, int COLL>
__global__ void __launch_bounds__(kPairBlock, kPairMinBlocks)
    k_step_batch_pair(const StepParams<float> *__restrict__ params, const int64_t *__restrict__ first,
                      int nmembers) {
  static_assert(L::DIMS == 3, "the pair kernel covers the D3Q19 step");
  __shared__ StepParams<float> sp;
  const int m = find_member(first, nmembers, blockIdx.x);
  params_to_smem(sp, params + m);
  const int64_t b = (int64_t)blockIdx.x - __ldg(first + m);
  const PairBatchLayout lay = pair_batch_layout(sp.nx, sp.ny, sp.nz);
  const int64_t step_now = *sp.step;
  if (b >= lay.pair_blocks) {
    // edge block: cell k of row 32 * e + threadIdx.x / 4
    const int k = threadIdx.x & 3;
    const int64_t r = (b - lay.pair_blocks) * 32 + (threadIdx.x >> 2);
    if (r >= lay.rows) return;
    const uint32_t zz = (uint32_t)r / (uint32_t)sp.ny;  // rows < 2^31
    const int y = (int)((uint32_t)r - zz * (uint32_t)sp.ny), z = (int)zz;
    step_cell<L, S, COLL>(sp, k < 2 ? k : sp.nx - 4 + k, y, z, step_now, GlobalGather<L, S, float>{sp, y, z});
    return;
  }
  const int64_t g = b / lay.bpr;
  const int t = (int)(b - g * lay.bpr) * kPairBlock + (int)threadIdx.x;
  const int rl = lay.TP <= kPairBlock ? t / lay.TP : 0;
  const int k = lay.TP <= kPairBlock ? t - rl * lay.TP : t;
  const int64_t r = g * lay.RB + rl;
  if (rl >= lay.RB || r >= lay.rows || k >= lay.P) return;
  const uint32_t zz = (uint32_t)r / (uint32_t)sp.ny;  // rows < 2^31
  const int x = 2 + 2 * k, y = (int)((uint32_t)r - zz * (uint32_t)sp.ny), z = (int)zz;
  const uint32_t c = cell_index(sp, x, y, z);
  bool plain = !(WALL_OF(sp) != WALL_NONE && (y == 0 || y == sp.ny - 1));
  if (plain) plain = *reinterpret_cast<const uint16_t *>(sp.flags + c) == 0;  // both flag bytes, c even
  if (plain) {
    pair_step_plain<L, S, COLL>(sp, x, y, z, c, step_now);
    return;
  }
  const GlobalGather<L, S, float> gather{sp, y, z};
#pragma unroll 1
  for (int kk = 0; kk < 2; kk++) step_cell<L, S, COLL>(sp, x + kk, y, z, step_now, gather);
}

template <class Real>
inline dim3 pair_grid(const StepParams<Real> &p) {
  const PairSplit sp = pair_split(p);
  return dim3((unsigned)(sp.row_blocks > 0 ? sp.row_blocks : 1), (unsigned)(kPairRows + 1), (unsigned)sp.groups);
}

}  // namespace AERO_KNS
}  // namespace aero
