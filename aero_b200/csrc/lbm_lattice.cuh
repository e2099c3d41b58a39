// lbm_lattice.cuh -- lattice descriptors and compile-time iteration helpers.
//
// Direction order, weights and opposites follow the reference exactly
// (aero/lbm/d2q9.py:18-38, aero/lbm/d3q19.py:37-73) so that population
// arrays keep the reference (Q, [Nz,] Ny, Nx) layout and meaning.
#pragma once
#include <cstdint>
#include <type_traits>
#include <utility>

namespace aero {

#define AERO_HD __host__ __device__ __forceinline__

// Calls f(std::integral_constant<int, I>{}) for I = 0 .. N-1, so that lattice
// tables are indexed with compile-time constants and fold into immediates.
template <class F, int... I>
AERO_HD void static_for_impl(F &&f, std::integer_sequence<int, I...>) {
  (f(std::integral_constant<int, I>{}), ...);
}
template <int N, class F>
AERO_HD void static_for(F &&f) {
  static_for_impl(f, std::make_integer_sequence<int, N>{});
}

struct D2Q9 {
  static constexpr int Q = 9, DIMS = 2, NP = 4;
  static constexpr int QP = 12;  // Q rounded up to a multiple of 4 (16-byte rows of outlet state)
  static constexpr int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
  static constexpr int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
  static constexpr int ez[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  static constexpr int opp[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
  static constexpr double w[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                                  1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  // representative direction of each +/- pair (pair p = 1..NP)
  static constexpr int pair[4] = {1, 2, 5, 6};
  // specular (y-mirror) partner, used by slip walls
  static constexpr int ymir[9] = {0, 1, 4, 3, 2, 8, 7, 6, 5};
};

struct D3Q19 {
  static constexpr int Q = 19, DIMS = 3, NP = 9;
  static constexpr int QP = 20;  // Q rounded up to a multiple of 4 (16-byte rows of outlet state)
  static constexpr int ex[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
  static constexpr int ey[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
  static constexpr int ez[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
  static constexpr int opp[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
  static constexpr double w[19] = {1.0 / 3.0,  1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0, 1.0 / 18.0,
                                   1.0 / 18.0, 1.0 / 18.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                   1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0,
                                   1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
  static constexpr int pair[9] = {1, 3, 5, 7, 8, 11, 12, 15, 16};
  static constexpr int ymir[19] = {0, 1, 2, 4, 3, 5, 6, 9, 10, 7, 8, 11, 12, 13, 14, 16, 15, 18, 17};
};

// Reduced scalar lattices (speed mode; the reference's scalar uses the flow
// lattice).  D2Q5 with cs^2 = 1/3, D3Q7 with cs^2 = 1/4.
struct D2Q5 {
  static constexpr int Q = 5, DIMS = 2;
  static constexpr int ex[5] = {0, 1, 0, -1, 0};
  static constexpr int ey[5] = {0, 0, 1, 0, -1};
  static constexpr int ez[5] = {0, 0, 0, 0, 0};
  static constexpr double w[5] = {1.0 / 3.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0, 1.0 / 6.0};
  static constexpr double cs2inv = 3.0;
};
struct D3Q7 {
  static constexpr int Q = 7, DIMS = 3;
  static constexpr int ex[7] = {0, 1, -1, 0, 0, 0, 0};
  static constexpr int ey[7] = {0, 0, 0, 1, -1, 0, 0};
  static constexpr int ez[7] = {0, 0, 0, 0, 0, 1, -1};
  static constexpr double w[7] = {0.25, 0.125, 0.125, 0.125, 0.125, 0.125, 0.125};
  static constexpr double cs2inv = 4.0;
};

// Scalar constants of direction I (usable in device code, unlike the arrays).
template <class L, int I>
struct Dir {
  static constexpr int x = L::ex[I];
  static constexpr int y = L::ey[I];
  static constexpr int z = L::ez[I];
  static constexpr double w = L::w[I];
};

// The scalar lattice that goes with a flow lattice.
template <class L> struct ScalarFull;
template <> struct ScalarFull<D2Q9> {
  using Lat = D2Q9;
  static constexpr double cs2inv = 3.0;
};
template <> struct ScalarFull<D3Q19> {
  using Lat = D3Q19;
  static constexpr double cs2inv = 3.0;
};
template <class L> struct ScalarReduced;
template <> struct ScalarReduced<D2Q9> { using Lat = D2Q5; };
template <> struct ScalarReduced<D3Q19> { using Lat = D3Q7; };

}  // namespace aero
