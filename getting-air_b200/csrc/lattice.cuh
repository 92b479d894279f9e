// Lattice velocity sets for D2Q9, D3Q19 and D3Q27, usable from host and
// device code with compile-time indices.
//
// The tables must be the reference's own, bit for bit, because parity is
// defined against them:
//   D2Q9   lattice-2d.mjs:106-162 (order rest, +x,+y,-x,-y, then the four
//          diagonals counter-clockwise; plain correctly rounded f32 weights,
//          WEIGHT_ULP_TWEAK = [0,0,0]), emitted as common_lattice.wgsl:20-37.
//   D3Q19  lattice-3d.mjs:50-210 (rest, face, edge; each velocity followed
//          by its negation so opp[i] = i+1 for odd i, i-1 for even i > 0;
//          f32 weights moved by [1,-4,2] ulps so they sum to exactly 1),
//          emitted as common_d3q19_lattice.wgsl:26-52.
//   D3Q27  the same ordering plus the 8 corners; ulp tweak [-1,1,-1,0],
//          common_d3q27_lattice.wgsl:26-57.
// The oracle derives the same numbers independently from the fractions and
// the tweak rule, and the tests compare both against the literals parsed
// out of the reference's generated WGSL.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define LBM_HD __host__ __device__ __forceinline__
#else
#define LBM_HD inline
#endif

namespace lbm {

template <int Q> struct Lattice;

template <> struct Lattice<9> {
  static constexpr int D = 2;
  static LBM_HD constexpr int ex(int i) {
    constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    return t[i];
  }
  static LBM_HD constexpr int ey(int i) {
    constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    return t[i];
  }
  static LBM_HD constexpr int ez(int) { return 0; }
  static LBM_HD constexpr int opp(int i) {
    constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    return t[i];
  }
  static LBM_HD constexpr float w(int i) {
    return i == 0 ? 0.44444444775581360f
                  : (i < 5 ? 0.11111111193895340f : 0.027777777984738350f);
  }
};

namespace detail {
// Shared D3Q27 ordering; D3Q19 is its first 19 entries.
LBM_HD constexpr int ex27(int i) {
  constexpr int t[27] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1,
                         -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1};
  return t[i];
}
LBM_HD constexpr int ey27(int i) {
  constexpr int t[27] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 0, 0, 0,
                         0, 1, -1, 1, -1, 1, -1, 1, -1, -1, 1, -1, 1};
  return t[i];
}
LBM_HD constexpr int ez27(int i) {
  constexpr int t[27] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1,
                         1, 1, -1, -1, 1, 1, -1, -1, 1, 1, -1, -1, 1};
  return t[i];
}
LBM_HD constexpr int opp27(int i) { return i == 0 ? 0 : ((i & 1) ? i + 1 : i - 1); }
}  // namespace detail

template <> struct Lattice<19> {
  static constexpr int D = 3;
  static LBM_HD constexpr int ex(int i) { return detail::ex27(i); }
  static LBM_HD constexpr int ey(int i) { return detail::ey27(i); }
  static LBM_HD constexpr int ez(int i) { return detail::ez27(i); }
  static LBM_HD constexpr int opp(int i) { return detail::opp27(i); }
  static LBM_HD constexpr float w(int i) {
    return i == 0 ? 0.33333337306976318f
                  : (i < 7 ? 0.055555541068315506f : 0.027777781710028648f);
  }
};

template <> struct Lattice<27> {
  static constexpr int D = 3;
  static LBM_HD constexpr int ex(int i) { return detail::ex27(i); }
  static LBM_HD constexpr int ey(int i) { return detail::ey27(i); }
  static LBM_HD constexpr int ez(int i) { return detail::ez27(i); }
  static LBM_HD constexpr int opp(int i) { return detail::opp27(i); }
  static LBM_HD constexpr float w(int i) {
    return i == 0 ? 0.29629626870155334f
                  : (i < 7 ? 0.074074082076549530f
                           : (i < 19 ? 0.018518516793847084f : 0.0046296296641230583f));
  }
};

}  // namespace lbm
