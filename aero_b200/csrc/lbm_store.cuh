// lbm_store.cuh -- population storage formats.
//
// All formats hold the deviation d_i = f_i - w_i from the rest state
// (rho = 1, u = 0), so that rounding acts on the small part of f only:
//   float / double : d_i as is
//   __half         : d_i * 64 / w_i (keeps near-rest values out of the
//                    FP16 subnormal range; |d_i / w_i| < 1000 before overflow)
//   __nv_bfloat16  : d_i as is (8-bit exponent, no scaling needed)
// Arithmetic is always done in Real (float, or double for double storage).
// load/store take the base of one direction plane (a warp-uniform pointer)
// and a 32-bit cell index, so each access is one wide multiply-add; lds
// reads the same format from a shared-memory tile.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include "lbm_lattice.cuh"

namespace aero {

// Read-only population loads.  With AERO_L2_256B the load asks L2 to fetch
// the whole 256-byte block around a miss (PTX ld.global.nc.L2::256B): a warp
// reads 64-128 contiguous bytes of a direction plane and its neighbour warp
// the next ones, so one DRAM access serves both.
#ifndef AERO_L2_256B
#define AERO_L2_256B 1
#endif
__device__ __forceinline__ float ld_pop(const float *p) {
#if AERO_L2_256B
  float v;
  asm("ld.global.nc.L2::256B.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
#else
  return __ldg(p);
#endif
}
__device__ __forceinline__ double ld_pop(const double *p) { return __ldg(p); }
__device__ __forceinline__ unsigned short ld_pop16(const void *p) {
#if AERO_L2_256B
  unsigned short v;
  asm("ld.global.nc.L2::256B.b16 %0, [%1];" : "=h"(v) : "l"(p));
  return v;
#else
  return __ldg(static_cast<const unsigned short *>(p));
#endif
}
__device__ __forceinline__ unsigned int ld_pop32(const void *p) {
#if AERO_L2_256B
  unsigned int v;
  asm("ld.global.nc.L2::256B.b32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
#else
  return __ldg(static_cast<const unsigned int *>(p));
#endif
}
__device__ __forceinline__ float2 ld_pop64(const float *p) {
#if AERO_L2_256B
  float2 v;
  asm("ld.global.nc.L2::256B.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "l"(p));
  return v;
#else
  return __ldg(reinterpret_cast<const float2 *>(p));
#endif
}

template <class S> struct StoreOps;

template <> struct StoreOps<float> {
  using Real = float;
  template <int I, class L>
  static __device__ __forceinline__ float load(const float *p, uint32_t o) { return ld_pop(p + o); }
  template <int I, class L>
  static __device__ __forceinline__ float lds(const float *p, uint32_t o) { return p[o]; }
  template <int I, class L>
  static __device__ __forceinline__ void store(float *p, uint32_t o, float v) { p[o] = v; }
};

template <> struct StoreOps<double> {
  using Real = double;
  template <int I, class L>
  static __device__ __forceinline__ double load(const double *p, uint32_t o) { return __ldg(p + o); }
  template <int I, class L>
  static __device__ __forceinline__ double lds(const double *p, uint32_t o) { return p[o]; }
  template <int I, class L>
  static __device__ __forceinline__ void store(double *p, uint32_t o, double v) { p[o] = v; }
};

template <> struct StoreOps<__half> {
  using Real = float;
  template <int I, class L>
  static __device__ __forceinline__ float load(const __half *p, uint32_t o) {
    constexpr float s = float(L::w[I] / 64.0);
    return __half2float(__ushort_as_half(ld_pop16(p + o))) * s;
  }
  template <int I, class L>
  static __device__ __forceinline__ float lds(const __half *p, uint32_t o) {
    constexpr float s = float(L::w[I] / 64.0);
    return __half2float(p[o]) * s;
  }
  template <int I, class L>
  static __device__ __forceinline__ void store(__half *p, uint32_t o, float v) {
    constexpr float s = float(64.0 / L::w[I]);
    p[o] = __float2half_rn(v * s);
  }
};

template <> struct StoreOps<__nv_bfloat16> {
  using Real = float;
  template <int I, class L>
  static __device__ __forceinline__ float load(const __nv_bfloat16 *p, uint32_t o) {
    return __bfloat162float(__ushort_as_bfloat16(ld_pop16(p + o)));
  }
  template <int I, class L>
  static __device__ __forceinline__ float lds(const __nv_bfloat16 *p, uint32_t o) {
    return __bfloat162float(p[o]);
  }
  template <int I, class L>
  static __device__ __forceinline__ void store(__nv_bfloat16 *p, uint32_t o, float v) {
    p[o] = __float2bfloat16_rn(v);
  }
};

}  // namespace aero
