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

template <class S> struct StoreOps;

template <> struct StoreOps<float> {
  using Real = float;
  template <int I, class L>
  static __device__ __forceinline__ float load(const float *p, uint32_t o) { return __ldg(p + o); }
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
    return __half2float(__ldg(p + o)) * s;
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
    return __bfloat162float(__ldg(p + o));
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
