// lattice.cuh -- compile-time lattice tables for the sm_100a lattice update.
//
// Velocity sets, weights and opposite tables follow the reference ordering so
// that population k here is population k there:
//   D2Q9 / D2Q5   src/LBM/LBM2D/_initialize.py:25-35, opposite table LBM2D/_core.py:35
//   D3Q19 / D3Q7  src/LBM/LBM3D/_initialize.py:25-43, opposite table LBM3D/_core.py:36
// The thermal lattice is the first QT directions of the flow lattice.
//
// MRT moment bases (no reference counterpart; new behaviour):
//   D3Q19  d'Humieres, Ginzburg, Krafczyk, Lallemand & Luo, Phil. Trans. R. Soc. A 360 (2002) 437
//   D2Q9   Lallemand & Luo, Phys. Rev. E 61 (2000) 6546
// Every table entry is a constexpr function of a compile-time index, so the
// fully unrolled kernels fold them into immediates.
#pragma once
#include <cstdint>
#include <utility>

namespace lbm {

template <int N, class F, int... Is>
__host__ __device__ __forceinline__ void static_for_impl(F&& f, std::integer_sequence<int, Is...>) {
  (f(std::integral_constant<int, Is>{}), ...);
}
// Calls f(std::integral_constant<int,0>) ... f(std::integral_constant<int,N-1>).
template <int N, class F>
__host__ __device__ __forceinline__ void static_for(F&& f) {
  static_for_impl<N>(f, std::make_integer_sequence<int, N>{});
}

template <int DIM> struct Lattice;

template <> struct Lattice<2> {
  static constexpr int DIM = 2, Q = 9, QT = 5, NPASS = 2;
  __host__ __device__ static constexpr int ex(int k) {
    constexpr int t[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    return t[k];
  }
  __host__ __device__ static constexpr int ey(int k) {
    constexpr int t[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    return t[k];
  }
  __host__ __device__ static constexpr int ez(int) { return 0; }
  __host__ __device__ static constexpr int opp(int k) {
    constexpr int t[9] = {0, 3, 4, 1, 2, 7, 8, 5, 6};
    return t[k];
  }
  __host__ __device__ static constexpr double w(int k) {
    return k == 0 ? 4.0 / 9.0 : (k < 5 ? 1.0 / 9.0 : 1.0 / 36.0);
  }
  __host__ __device__ static constexpr double wt(int k) { return k == 0 ? 1.0 / 3.0 : 1.0 / 6.0; }
  // thermal equilibrium w T (1 + ta e.u + tb (e.u)^2 - tc u.u)   (LBM2D/_thermal.py:54-61)
  static constexpr double ta = 3.0, tb = 4.5, tc = 1.5;
  // MRT moment polynomial r evaluated at velocity k (Lallemand & Luo 2000)
  __host__ __device__ static constexpr double mrt(int r, int k) {
    const double cx = ex(k), cy = ey(k), c2 = cx * cx + cy * cy;
    switch (r) {
      case 0: return 1;
      case 1: return -4 + 3 * c2;
      case 2: return 4 - 10.5 * c2 + 4.5 * c2 * c2;
      case 3: return cx;
      case 4: return (-5 + 3 * c2) * cx;
      case 5: return cy;
      case 6: return (-5 + 3 * c2) * cy;
      case 7: return cx * cx - cy * cy;
      default: return cx * cy;
    }
  }
  __host__ __device__ static constexpr bool mrt_conserved(int r) { return r == 0 || r == 3 || r == 5; }
  __host__ __device__ static constexpr bool mrt_viscous(int r) { return r == 7 || r == 8; }
};

template <> struct Lattice<3> {
  static constexpr int DIM = 3, Q = 19, QT = 7, NPASS = 3;
  __host__ __device__ static constexpr int ex(int k) {
    constexpr int t[19] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 1, -1, 1, -1, 0, 0, 0, 0};
    return t[k];
  }
  __host__ __device__ static constexpr int ey(int k) {
    constexpr int t[19] = {0, 0, 0, 1, -1, 0, 0, 1, 1, -1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
    return t[k];
  }
  __host__ __device__ static constexpr int ez(int k) {
    constexpr int t[19] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    return t[k];
  }
  __host__ __device__ static constexpr int opp(int k) {
    constexpr int t[19] = {0, 2, 1, 4, 3, 6, 5, 10, 9, 8, 7, 14, 13, 12, 11, 18, 17, 16, 15};
    return t[k];
  }
  __host__ __device__ static constexpr double w(int k) {
    return k == 0 ? 1.0 / 3.0 : (k < 7 ? 1.0 / 18.0 : 1.0 / 36.0);
  }
  __host__ __device__ static constexpr double wt(int k) { return k == 0 ? 1.0 / 4.0 : 1.0 / 8.0; }
  // thermal equilibrium w T (1 + 4 e.u + 8 (e.u)^2 - 2 u.u)   (LBM3D/_thermal.py:54-61)
  static constexpr double ta = 4.0, tb = 8.0, tc = 2.0;
  __host__ __device__ static constexpr double mrt(int r, int k) {
    const double cx = ex(k), cy = ey(k), cz = ez(k);
    const double c2 = cx * cx + cy * cy + cz * cz;
    switch (r) {
      case 0: return 1;
      case 1: return 19 * c2 - 30;
      case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2.0;
      case 3: return cx;
      case 4: return (5 * c2 - 9) * cx;
      case 5: return cy;
      case 6: return (5 * c2 - 9) * cy;
      case 7: return cz;
      case 8: return (5 * c2 - 9) * cz;
      case 9: return 3 * cx * cx - c2;
      case 10: return (3 * c2 - 5) * (3 * cx * cx - c2);
      case 11: return cy * cy - cz * cz;
      case 12: return (3 * c2 - 5) * (cy * cy - cz * cz);
      case 13: return cx * cy;
      case 14: return cy * cz;
      case 15: return cx * cz;
      case 16: return (cy * cy - cz * cz) * cx;
      case 17: return (cz * cz - cx * cx) * cy;
      default: return (cx * cx - cy * cy) * cz;
    }
  }
  __host__ __device__ static constexpr bool mrt_conserved(int r) {
    return r == 0 || r == 3 || r == 5 || r == 7;
  }
  __host__ __device__ static constexpr bool mrt_viscous(int r) {
    return r == 9 || r == 11 || r == 13 || r == 14 || r == 15;
  }
};

// Squared norm of MRT row r (rows are orthogonal, so M^-1 = M^T diag(1/norm)).
template <class L>
__host__ __device__ constexpr double mrt_norm(int r) {
  double s = 0;
  for (int k = 0; k < L::Q; ++k) s += L::mrt(r, k) * L::mrt(r, k);
  return s;
}

// Opposite-direction pairs: pair p = (pk(p), opp(pk(p))) with pk(p) < opp(pk(p)).
// Symmetric and antisymmetric combinations of a pair carry the even and odd
// moments separately, which halves the equilibrium and MRT arithmetic.
template <class L>
__host__ __device__ constexpr int num_pairs() { return (L::Q - 1) / 2; }
template <class L>
__host__ __device__ constexpr int pk(int p) {
  int n = 0;
  for (int k = 1; k < L::Q; ++k)
    if (k < L::opp(k)) {
      if (n == p) return k;
      ++n;
    }
  return -1;
}
template <class L, int QQ>
__host__ __device__ constexpr int pkt(int p) {  // same for the thermal lattice (first QQ directions)
  int n = 0;
  for (int k = 1; k < QQ; ++k)
    if (k < L::opp(k)) {
      if (n == p) return k;
      ++n;
    }
  return -1;
}
// True if MRT row r is even under velocity reversal (M[r][opp k] == M[r][k]).
template <class L>
__host__ __device__ constexpr bool mrt_even(int r) {
  for (int k = 0; k < L::Q; ++k)
    if (L::mrt(r, L::opp(k)) != L::mrt(r, k)) return false;
  return true;
}

}  // namespace lbm
