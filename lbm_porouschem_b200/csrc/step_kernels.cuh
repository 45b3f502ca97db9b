// step_kernels.cuh -- fused pull-scheme lattice update for sm_100a.
//
// One pass of step_bulk<> does, per cell, what the reference does in three
// separate Taichi loops (src/LBM/LBM2D/_evolution.py:16-25):
//   stream (pull form of the push at :67-95, halfway bounce-back at :78-86)
//   -> macro (:118-202: rho, u, T, sources, pyrolysis, flip)
//   -> collision of the NEXT step (:26-66: BGK toward feq, Guo force, thermal
//      BGK with the geq(dS) source).
// Reading post-collision populations of step n and writing those of step n+1
// keeps one read and one write per population per step, the minimum for an
// A/B double buffer.  Cells on active (non-periodic) domain sides are skipped
// here and finished by step_boundary<>, which re-derives the non-equilibrium
// extrapolation (src/LBM/LBM2D/_boundary.py:17-101) from the same input buffer.
//
// Layout in HBM (structure of arrays, x fastest, c = x + nx*(y + ny*z)):
//   f[buf][k][c]   storage type S (float / __half shifted / double), buf = A|B
//   g[buf][k][c]   temperature populations
//   mask[c]        uint8: bit0/bit1 solid at even/odd parity, bit2 reactive
//   alpha[c]       reactive fraction (compute precision; solid cells only, in place)
//   rel[buf][c]    gas release per unit lattice weight (reacting solids)
// Solid cells carry no flow populations: a fluid cell pulling from a solid
// neighbour bounces its own opposite population instead, so the f planes of
// solid cells are neither read nor written (except when a cell flips).
#pragma once
#include <cuda_fp16.h>
#include <math.h>
#include <stdint.h>

#include "lattice.cuh"
#include "lbm_b200.h"

namespace lbm {

// ------------------------------------------------------------------ storage
template <class S> struct Store;
template <> struct Store<float> {
  using C = float;
  __device__ __forceinline__ static C ld(const float* p, size_t i, C) { return p[i]; }
  __device__ __forceinline__ static void st(float* p, size_t i, C v, C) { p[i] = v; }
};
template <> struct Store<double> {
  using C = double;
  __device__ __forceinline__ static C ld(const double* p, size_t i, C) { return p[i]; }
  __device__ __forceinline__ static void st(double* p, size_t i, C v, C) { p[i] = v; }
};
// FP16 storage of the deviation from the rest equilibrium (value - shift),
// FP32 arithmetic.
template <> struct Store<__half> {
  using C = float;
  __device__ __forceinline__ static C ld(const __half* p, size_t i, C shift) {
    return __half2float(p[i]) + shift;
  }
  __device__ __forceinline__ static void st(__half* p, size_t i, C v, C shift) {
    p[i] = __float2half_rn(v - shift);
  }
};

constexpr int kNumDiag = 10;  // partial slots per block (order of lbm_diag fields)
constexpr int kStepPeek = 1 << 8;  // internal flag: recompute outputs, leave the state untouched
constexpr double kGasConstant = 8.314441;  // src/LBM/util/constant.py:17

template <class S>
struct StepParams {
  using C = typename Store<S>::C;
  int nx, ny, nz;
  size_t N;
  const S* fA;
  S* fB;
  const S* gA;
  S* gB;
  uint8_t* mask;
  C* alpha;        // reactive fraction (compute precision), updated in place
  const C* relA;   // gas release per unit lattice weight, read plane
  C* relB;         //   and write plane
  int par;  // step parity: mask bit read this pass
  int eos;
  int half_force;
  int has_force;
  C nu, Fx, Fy, Fz;
  C mrt_sn[19];  // s_r / |M_r|^2 for non-viscous, non-conserved rows
  C itauT_f, itauT_s;
  C rho0, T0;
  C pyA, pyb, pyEa, pyTmin, Tref, Tscale, dtp, heat_norm, gas_coef, alpha_flip;
  int active;  // bit s: side s uses NEE
  const lbm_side_desc* sides;  // device copy
  int flags;   // LBM_STEP_*
  double* partials;    // SoA: partials[i * partial_rows + block]
  int partial_rows;
  int block_offset;
  C* rho_out;
  C* u_out;
  C* T_out;
  float* uprev;
};

// Per-population storage shifts (FP16 deviation storage); zero otherwise.
template <class L, class S, int K>
__device__ __forceinline__ typename Store<S>::C fshift(const StepParams<S>& p) {
  if constexpr (std::is_same<S, __half>::value) return (float)L::w(K) * p.rho0;
  else return 0;
}
template <class L, class S, int K>
__device__ __forceinline__ typename Store<S>::C gshift(const StepParams<S>& p) {
  if constexpr (std::is_same<S, __half>::value) return (float)L::wt(K) * p.T0;
  else return 0;
}

__device__ __forceinline__ int wrapi(int v, int n) { return v < 0 ? n - 1 : (v > n - 1 ? 0 : v); }

// Indices of the 3x3x3 neighbourhood of (x,y,z) with the reference's periodic
// wrap (src/LBM/LBM2D/_evolution.py:205-212): xs[d+1], ys[d+1]*nx, zs[d+1]*nx*ny.
struct Nbhd {
  int xs[3], ro[3], po[3];
  __device__ __forceinline__ Nbhd(int x, int y, int z, int nx, int ny, int nz) {
    xs[0] = wrapi(x - 1, nx); xs[1] = x; xs[2] = wrapi(x + 1, nx);
    ro[0] = wrapi(y - 1, ny) * nx; ro[1] = y * nx; ro[2] = wrapi(y + 1, ny) * nx;
    const int pl = nx * ny;
    po[0] = wrapi(z - 1, nz) * pl; po[1] = z * pl; po[2] = wrapi(z + 1, nz) * pl;
  }
  // cell at offset (dx,dy,dz) in {-1,0,1}^3
  __device__ __forceinline__ int at(int dx, int dy, int dz) const {
    return xs[dx + 1] + ro[dy + 1] + po[dz + 1];
  }
};

template <class C> __device__ __forceinline__ bool finite_(C v) { return isfinite(v); }

template <class L, class S>
struct Kern {
  using C = typename Store<S>::C;
  static constexpr int Q = L::Q, QT = L::QT;
  using P = StepParams<S>;

  __device__ __forceinline__ static bool solid_at(const P& p, int c) {
    return (p.mask[c] >> p.par) & 1;
  }

  // Post-stream flow populations of fluid cell c (pull form of the reference push).
  template <bool PYRO>
  __device__ __forceinline__ static void pull_flow(const P& p, const Nbhd& nb, int c, C F[Q]) {
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if constexpr (k == 0) {
        F[0] = Store<S>::ld(p.fA, c, fshift<L, S, 0>(p));
      } else {
        const int src = nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
        if (solid_at(p, src)) {
          constexpr int o = L::opp(k);
          C v = Store<S>::ld(p.fA, (size_t)o * p.N + c, fshift<L, S, o>(p));
          if constexpr (PYRO) v += (C)p.relA[src] * (C)L::w(k);
          F[k] = v;
        } else {
          F[k] = Store<S>::ld(p.fA, (size_t)k * p.N + src, fshift<L, S, k>(p));
        }
      }
    });
  }

  // Post-stream temperature populations (conjugate mode streams through solids).
  __device__ __forceinline__ static void pull_thermal(const P& p, const Nbhd& nb, int c, C G[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      const int src = (k == 0) ? c : nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
      G[k] = Store<S>::ld(p.gA, (size_t)k * p.N + src, gshift<L, S, k>(p));
    });
  }

  // macro moments, src/LBM/LBM2D/_evolution.py:123-130
  __device__ __forceinline__ static void moments(const P& p, const C F[Q], C& rho, C& ux, C& uy, C& uz) {
    C r = 0, jx = 0, jy = 0, jz = 0;
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      r += F[k];
      if constexpr (L::ex(k) != 0) jx += (C)L::ex(k) * F[k];
      if constexpr (L::ey(k) != 0) jy += (C)L::ey(k) * F[k];
      if constexpr (L::ez(k) != 0) jz += (C)L::ez(k) * F[k];
    });
    if (p.half_force) {
      const C s = p.eos == 0 ? r : (C)1;
      jx += (C)0.5 * p.Fx * s; jy += (C)0.5 * p.Fy * s; jz += (C)0.5 * p.Fz * s;
    }
    if (p.eos == 0) { jx /= r; jy /= r; jz /= r; }
    rho = r; ux = jx; uy = jy; uz = jz;
  }

  // feq9/feq19 with eps = 1 (src/LBM/LBM2D/_evolution.py:213-225)
  template <int k>
  __device__ __forceinline__ static C feq(const P& p, C rho, C ux, C uy, C uz, C usq) {
    constexpr C ie = (C)1 / ((C)1 + (C)1e-12);
    const C eu = (C)L::ex(k) * ux + (C)L::ey(k) * uy + (C)L::ez(k) * uz;
    if (p.eos == 1) return (C)L::w(k) * (rho + (C)3.0 * eu + (C)4.5 * eu * eu * ie - (C)1.5 * usq * ie);
    return (C)L::w(k) * rho * ((C)1.0 + (C)3.0 * eu + (C)4.5 * eu * eu * ie - (C)1.5 * usq * ie);
  }

  // forceTermGuo, src/LBM/LBM2D/_evolution.py:284-298 (eps = 1)
  template <int k>
  __device__ __forceinline__ static C guo(const P& p, C rho, C ux, C uy, C uz, C pre) {
    constexpr C ie = (C)1 / ((C)1 + (C)1e-12);
    const C ex = (C)L::ex(k), ey = (C)L::ey(k), ez = (C)L::ez(k);
    const C t1 = (ex - ux * ie) * p.Fx + (ey - uy * ie) * p.Fy + (ez - uz * ie) * p.Fz;
    const C eu = ex * ux + ey * uy + ez * uz;
    const C eF = ex * p.Fx + ey * p.Fy + ez * p.Fz;
    const C t = pre * (C)L::w(k) * ((C)3.0 * t1 + (C)9.0 * eu * eF * ie);
    return p.eos == 1 ? t : rho * t;
  }

  // Flow collision: BGK (_evolution.py:33) or MRT (new), plus Guo forcing.
  // Writes the post-collision populations over F.
  template <int COLL>
  __device__ __forceinline__ static void collide_flow(const P& p, C F[Q], C rho, C ux, C uy, C uz) {
    const C tau = (C)3 * (p.eos == 0 ? p.nu / rho : p.nu) + (C)0.5;
    const C itau = (C)1 / tau;
    const C usq = ux * ux + uy * uy + uz * uz;
    const C pre = (C)1.0 - (C)1.0 / (C)2.0 / tau;
    if constexpr (COLL == LBM_COLL_BGK) {
      static_for<Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        C v = F[k] - itau * (F[k] - feq<k>(p, rho, ux, uy, uz, usq));
        if (p.has_force) v += guo<k>(p, rho, ux, uy, uz, pre);
        F[k] = v;
      });
    } else {
      C fn[Q];
      static_for<Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        fn[k] = F[k] - feq<k>(p, rho, ux, uy, uz, usq);
      });
      C m[Q];
      static_for<Q>([&](auto rr) {
        constexpr int r = decltype(rr)::value;
        if constexpr (!L::mrt_conserved(r)) {
          C acc = 0;
          static_for<Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            constexpr double mv = L::mrt(r, k);
            if constexpr (mv == 1.0) acc += fn[k];
            else if constexpr (mv == -1.0) acc -= fn[k];
            else if constexpr (mv != 0.0) acc += (C)mv * fn[k];
          });
          constexpr double inv_norm = 1.0 / mrt_norm<L>(r);
          if constexpr (L::mrt_viscous(r)) m[r] = acc * itau * (C)inv_norm;
          else m[r] = acc * p.mrt_sn[r];
        }
      });
      static_for<Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        C acc = 0;
        static_for<Q>([&](auto rr) {
          constexpr int r = decltype(rr)::value;
          if constexpr (!L::mrt_conserved(r)) {
            constexpr double mv = L::mrt(r, k);
            if constexpr (mv == 1.0) acc += m[r];
            else if constexpr (mv == -1.0) acc -= m[r];
            else if constexpr (mv != 0.0) acc += (C)mv * m[r];
          }
        });
        C v = F[k] - acc;
        if (p.has_force) v += guo<k>(p, rho, ux, uy, uz, pre);
        F[k] = v;
      });
    }
  }

  // Thermal collision with source (conjugate): fluid geq = TF.geq (advected),
  // solid geq = w T (TS.geq, LBM2D/_thermal.py:162-166); source wt*dS (:54-58).
  __device__ __forceinline__ static void collide_thermal(const P& p, C G[QT], C T, bool solid, C ux, C uy,
                                                         C uz, C dS) {
    const C itau = solid ? p.itauT_s : p.itauT_f;
    const C usq = ux * ux + uy * uy + uz * uz;
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      C ge;
      if (solid) {
        ge = (C)L::wt(k) * T;
      } else {
        const C eu = (C)L::ex(k) * ux + (C)L::ey(k) * uy + (C)L::ez(k) * uz;
        ge = (C)L::wt(k) * T * ((C)1.0 + (C)L::ta * eu + (C)L::tb * eu * eu - (C)L::tc * usq);
      }
      G[k] = G[k] - itau * (G[k] - ge) + (C)L::wt(k) * dS;
    });
  }

  __device__ __forceinline__ static void store_flow(const P& p, int c, const C F[Q]) {
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      Store<S>::st(p.fB, (size_t)k * p.N + c, F[k], fshift<L, S, k>(p));
    });
  }
  __device__ __forceinline__ static void store_thermal(const P& p, int c, const C G[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      Store<S>::st(p.gB, (size_t)k * p.N + c, G[k], gshift<L, S, k>(p));
    });
  }

  // Is (x,y,z) on an active (NEE) side?  Those cells belong to step_boundary.
  __device__ __forceinline__ static bool on_active_side(const P& p, int x, int y, int z) {
    const int a = p.active;
    return ((a & 1) && x == 0) || ((a & 2) && x == p.nx - 1) || ((a & 4) && y == 0) ||
           ((a & 8) && y == p.ny - 1) || ((a & 16) && z == 0) || ((a & 32) && z == p.nz - 1);
  }
};

// --------------------------------------------------------------- diagnostics
struct DiagAcc {
  double v[kNumDiag];
  __device__ __forceinline__ void clear() {
    for (int i = 0; i < kNumDiag; ++i) v[i] = 0;
    v[3] = 0;       // umax^2
    v[4] = 1e300;   // Tmin
    v[5] = -1e300;  // Tmax
  }
};

// Block reduction with warp shuffles (FP64), one partial row per block.
__device__ __forceinline__ void block_reduce_store(DiagAcc& a, double* out_row, size_t stride) {
  __shared__ double sh[32][kNumDiag];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < kNumDiag; ++i) {
    double v = a.v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double w = __shfl_xor_sync(0xffffffffu, v, o);
      v = (i == 3 || i == 5) ? fmax(v, w) : (i == 4 ? fmin(v, w) : v + w);
    }
    if (lane == 0) sh[warp][i] = v;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int i = 0; i < kNumDiag; ++i) {
      double v = lane < nwarps ? sh[lane][i] : (i == 4 ? 1e300 : (i == 3 || i == 5 ? -1e300 : 0.0));
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double w = __shfl_xor_sync(0xffffffffu, v, o);
        v = (i == 3 || i == 5) ? fmax(v, w) : (i == 4 ? fmin(v, w) : v + w);
      }
      if (lane == 0) out_row[(size_t)i * stride] = v;
    }
  }
}

template <class L, class S>
__device__ __forceinline__ void diag_cell(const StepParams<S>& p, DiagAcc& a, int c, bool fluid,
                                          bool reactive_solid, typename Store<S>::C rho,
                                          typename Store<S>::C ux, typename Store<S>::C uy,
                                          typename Store<S>::C uz, typename Store<S>::C T, bool thermal,
                                          typename Store<S>::C alpha) {
  using C = typename Store<S>::C;
  if (thermal) {
    a.v[1] += (double)T;
    a.v[4] = fmin(a.v[4], (double)T);
    a.v[5] = fmax(a.v[5], (double)T);
    if (!finite_(T)) a.v[6] += 1;
  }
  if (fluid) {
    a.v[0] += (double)rho;
    const double u2 = (double)ux * ux + (double)uy * uy + (double)uz * uz;
    a.v[3] = fmax(a.v[3], u2);
    if (!finite_(rho)) a.v[6] += 1;
    a.v[7] += 1;
    if (p.flags & LBM_STEP_RESIDUAL) {
      const double dx = (double)ux - p.uprev[c], dy = (double)uy - p.uprev[p.N + c],
                   dz = (double)uz - p.uprev[2 * p.N + c];
      a.v[8] += dx * dx + dy * dy + dz * dz;
      a.v[9] += u2;
      p.uprev[c] = (float)ux;
      p.uprev[p.N + c] = (float)uy;
      p.uprev[2 * p.N + c] = (float)uz;
    }
    if (p.flags & LBM_STEP_MACRO) {
      p.rho_out[c] = rho;
      p.u_out[c] = ux;
      p.u_out[p.N + c] = uy;
      p.u_out[2 * p.N + c] = uz;
    }
  } else if (reactive_solid) {
    a.v[2] += (double)alpha;
  }
  if (thermal && (p.flags & LBM_STEP_MACRO)) p.T_out[c] = T;
  (void)sizeof(C);
}

// Mean post-stream (rho, u) over the fluid neighbours of (x,y,z), in direction
// order 1..Q-1; (1, 0) if there are none.  Used when a spent solid cell turns fluid.
template <class L, class S>
__device__ __noinline__ void neighbour_mean(const StepParams<S>& p, int x, int y, int z,
                                            typename Store<S>::C& rb, typename Store<S>::C& ux,
                                            typename Store<S>::C& uy, typename Store<S>::C& uz) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q;
  C rs = 0, us0 = 0, us1 = 0, us2 = 0;
  int n = 0;
  static_for<Q>([&](auto kk) {
    constexpr int q = decltype(kk)::value;
    if constexpr (q > 0) {
      const int xq = wrapi(x + L::ex(q), p.nx), yq = wrapi(y + L::ey(q), p.ny), zq = wrapi(z + L::ez(q), p.nz);
      const int cq = xq + p.nx * (yq + p.ny * zq);
      if (!K::solid_at(p, cq)) {
        const Nbhd nq(xq, yq, zq, p.nx, p.ny, p.nz);
        C Fq[Q], rq, uxq, uyq, uzq;
        K::template pull_flow<true>(p, nq, cq, Fq);
        K::moments(p, Fq, rq, uxq, uyq, uzq);
        rs += rq; us0 += uxq; us1 += uyq; us2 += uzq;
        ++n;
      }
    }
  });
  rb = n ? rs / (C)n : (C)1;
  ux = n ? us0 / (C)n : (C)0;
  uy = n ? us1 / (C)n : (C)0;
  uz = n ? us2 / (C)n : (C)0;
}

// ------------------------------------------------------------------ kernels
// THERM: 0 no temperature, 1 conjugate, 2 conjugate + pyrolysis.
template <class L, class S, int COLL, int THERM>
__global__ void __launch_bounds__(256) step_bulk(const StepParams<S> p) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y, z = blockIdx.z;
  const bool diag = (p.flags & (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) != 0;
  const bool peek = (p.flags & kStepPeek) != 0;
  DiagAcc acc;
  if (diag) acc.clear();

  if (x < p.nx && !K::on_active_side(p, x, y, z)) {
    const int c = x + p.nx * (y + p.ny * z);
    const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
    const uint8_t mk = p.mask[c];
    const bool solid = (mk >> p.par) & 1;
    bool solid_next = solid;
    C G[QT > 0 ? QT : 1];
    C T = 0, dS = 0;
    if constexpr (THERMAL) {
      K::pull_thermal(p, nb, c, G);
      static_for<QT>([&](auto kk) { T += G[decltype(kk)::value]; });
    }
    if (!solid) {
      C F[Q];
      C rho, ux, uy, uz;
      K::template pull_flow<PYRO>(p, nb, c, F);
      K::moments(p, F, rho, ux, uy, uz);
      if (diag) diag_cell<L, S>(p, acc, c, true, false, rho, ux, uy, uz, T, THERMAL, (C)0);
      if (!peek) {
        K::template collide_flow<COLL>(p, F, rho, ux, uy, uz);
        K::store_flow(p, c, F);
        if constexpr (THERMAL) {
          K::collide_thermal(p, G, T, false, ux, uy, uz, (C)0);
          K::store_thermal(p, c, G);
        }
      }
    } else {
      C ux = 0, uy = 0, uz = 0;
      C an = 0;
      const bool reactive = PYRO && (mk & LBM_MASK_REACTIVE);
      if constexpr (PYRO) {
        if (reactive && peek) {
          // Current state: alpha already updated; a cell flipped in the last pass
          // reports the neighbour-mean state it was given.
          an = p.alpha[c];
          if (!((mk >> (p.par ^ 1)) & 1)) {
            solid_next = false;
            C rb;
            neighbour_mean<L, S>(p, x, y, z, rb, ux, uy, uz);
            if (diag) diag_cell<L, S>(p, acc, c, true, false, rb, ux, uy, uz, (C)0, false, (C)0);
          }
        } else if (reactive) {
          // Arrhenius rate at the solid temperature, src/LBM/LBM2D/_chemical.py:198-212
          const C a = (C)p.alpha[c];
          const C TK = T * p.Tscale + p.Tref;
          C kr = 0;
          if (TK > p.pyTmin) {
            const C Te = TK + (C)1e-6;
            kr = p.pyA * exp(-(p.pyEa / Te / (C)kGasConstant));
            if (p.pyb != (C)0) kr *= pow(Te, p.pyb);
          }
          const C da = kr * a * p.dtp;
          const C anC = a - da;
          an = anC;
          p.alpha[c] = an;
          dS = -p.heat_norm * da;
          const C mg = p.gas_coef * da;
          C W = 0;
          static_for<Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            if constexpr (k > 0) {
              if (!K::solid_at(p, nb.at(L::ex(k), L::ey(k), L::ez(k)))) W += (C)L::w(k);
            }
          });
          if (anC < p.alpha_flip) {
            // Spent cell turns fluid at the mean (rho, u) of its fluid neighbours.
            solid_next = false;
            C rb;
            neighbour_mean<L, S>(p, x, y, z, rb, ux, uy, uz);
            C F[Q];
            const C usq = ux * ux + uy * uy + uz * uz;
            static_for<Q>([&](auto kk) {
              constexpr int k = decltype(kk)::value;
              F[k] = K::template feq<k>(p, rb, ux, uy, uz, usq);
            });
            if (diag) diag_cell<L, S>(p, acc, c, true, false, rb, ux, uy, uz, (C)0, false, (C)0);
            K::template collide_flow<COLL>(p, F, rb, ux, uy, uz);
            K::store_flow(p, c, F);
            p.relB[c] = (C)0;
          } else {
            p.relB[c] = W > (C)0 ? mg / W : (C)0;
          }
        }
      }
      if constexpr (THERMAL) {
        if (!peek) {
          K::collide_thermal(p, G, T, solid_next, ux, uy, uz, dS);
          K::store_thermal(p, c, G);
        }
      }
      if (diag) diag_cell<L, S>(p, acc, c, false, solid_next && reactive, 0, 0, 0, 0, T, THERMAL, an);
    }
    // Mask bit for the next parity: written only when it changes.
    if (!peek) {
      const int np = p.par ^ 1;
      const uint8_t want = (uint8_t)((mk & ~(1u << np)) | ((solid_next ? 1u : 0u) << np));
      if (want != mk) p.mask[c] = want;
    }
  }
  if (diag) {
    const int blk = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blk), (size_t)p.partial_rows);
  }
}

// --------------------------------------------------------- boundary kernel
template <class L, class S>
struct MState {
  using C = typename Store<S>::C;
  C F[L::Q];
  C G[L::QT];
  C rho, ux, uy, uz, T;
};

// State of cell (x,y,z) after the first PASS+1 NEE passes (0: x sides,
// 1: y sides, 2: z sides), in the reference's loop order
// (src/LBM/LBM3D/_boundary.py:15-68).  PASS = -1 is the post-stream macro state.
template <class L, class S, bool THERMAL, bool PYRO, int PASS>
__device__ MState<L, S> bc_state(const StepParams<S>& p, int x, int y, int z) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  MState<L, S> s;
  if constexpr (PASS < 0) {
    const int c = x + p.nx * (y + p.ny * z);
    const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
    K::template pull_flow<PYRO>(p, nb, c, s.F);
    K::moments(p, s.F, s.rho, s.ux, s.uy, s.uz);
    s.T = 0;
    if constexpr (THERMAL) {
      K::pull_thermal(p, nb, c, s.G);
      static_for<L::QT>([&](auto kk) { s.T += s.G[decltype(kk)::value]; });
    }
    return s;
  } else {
    s = bc_state<L, S, THERMAL, PYRO, PASS - 1>(p, x, y, z);
    int side = -1, ix = x, iy = y, iz = z;
    if constexpr (PASS == 0) {
      if ((p.active & 1) && x == 0) { side = 0; ix = 1; }
      else if ((p.active & 2) && x == p.nx - 1) { side = 1; ix = p.nx - 2; }
    } else if constexpr (PASS == 1) {
      if ((p.active & 4) && y == 0) { side = 2; iy = 1; }
      else if ((p.active & 8) && y == p.ny - 1) { side = 3; iy = p.ny - 2; }
    } else {
      if ((p.active & 16) && z == 0) { side = 4; iz = 1; }
      else if ((p.active & 32) && z == p.nz - 1) { side = 5; iz = p.nz - 2; }
    }
    if (side < 0) return s;
    const MState<L, S> in = bc_state<L, S, THERMAL, PYRO, PASS - 1>(p, ix, iy, iz);
    const lbm_side_desc& sd = p.sides[side];
    // _boundary.py:54-65 (flow), _scalarField.py:83-92 (scalar)
    if (sd.v_type == LBM_BC_FIXEDVALUE) { s.ux = (C)sd.v[0]; s.uy = (C)sd.v[1]; s.uz = (C)sd.v[2]; }
    else if (sd.v_type == LBM_BC_ZEROGRADIENT) { s.ux = in.ux; s.uy = in.uy; s.uz = in.uz; }
    if (sd.rho_type == LBM_BC_FIXEDVALUE) s.rho = (C)sd.rho;
    else if (sd.rho_type == LBM_BC_ZEROGRADIENT) s.rho = in.rho;
    const C usb = s.ux * s.ux + s.uy * s.uy + s.uz * s.uz;
    const C usi = in.ux * in.ux + in.uy * in.uy + in.uz * in.uz;
    static_for<L::Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      s.F[k] = K::template feq<k>(p, s.rho, s.ux, s.uy, s.uz, usb) +
               (in.F[k] - K::template feq<k>(p, in.rho, in.ux, in.uy, in.uz, usi));
    });
    if constexpr (THERMAL) {
      if (sd.T_type == LBM_BC_FIXEDVALUE) s.T = (C)sd.T;
      else if (sd.T_type == LBM_BC_ZEROGRADIENT) s.T = in.T;
      static_for<L::QT>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        const C eb = (C)L::ex(k) * s.ux + (C)L::ey(k) * s.uy + (C)L::ez(k) * s.uz;
        const C ei = (C)L::ex(k) * in.ux + (C)L::ey(k) * in.uy + (C)L::ez(k) * in.uz;
        const C gb = (C)L::wt(k) * s.T * ((C)1.0 + (C)L::ta * eb + (C)L::tb * eb * eb - (C)L::tc * usb);
        const C gi = (C)L::wt(k) * in.T * ((C)1.0 + (C)L::ta * ei + (C)L::tb * ei * ei - (C)L::tc * usi);
        s.G[k] = gb + (in.G[k] - gi);
      });
    }
    return s;
  }
}

// One thread per boundary cell.  blockIdx.y selects an active face; a cell on
// several active faces is owned by the lowest-numbered one.
template <class L, class S, int COLL, int THERM>
__global__ void __launch_bounds__(128) step_boundary(const StepParams<S> p, int4 faces01, int2 faces2) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  const int fid[6] = {faces01.x, faces01.y, faces01.z, faces01.w, faces2.x, faces2.y};
  const int face = fid[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool diag = (p.flags & (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) != 0;
  DiagAcc acc;
  if (diag) acc.clear();
  int x = 0, y = 0, z = 0;
  bool valid = false;
  if (face == 0 || face == 1) {
    valid = i < p.ny * p.nz;
    x = face == 0 ? 0 : p.nx - 1; y = i % p.ny; z = i / p.ny;
  } else if (face == 2 || face == 3) {
    valid = i < p.nx * p.nz;
    y = face == 2 ? 0 : p.ny - 1; x = i % p.nx; z = i / p.nx;
  } else {
    valid = i < p.nx * p.ny;
    z = face == 4 ? 0 : p.nz - 1; x = i % p.nx; y = i / p.nx;
  }
  if (valid) {
    // ownership: skip if a lower-numbered active face also contains the cell
    for (int f = 0; f < face; ++f) {
      if (!(p.active & (1 << f))) continue;
      const bool on = (f == 0 && x == 0) || (f == 1 && x == p.nx - 1) || (f == 2 && y == 0) ||
                      (f == 3 && y == p.ny - 1) || (f == 4 && z == 0) || (f == 5 && z == p.nz - 1);
      if (on) valid = false;
    }
  }
  if (valid) {
    const int c = x + p.nx * (y + p.ny * z);
    MState<L, S> s = bc_state<L, S, THERMAL, PYRO, L::NPASS - 1>(p, x, y, z);
    if (diag) {
      diag_cell<L, S>(p, acc, c, true, false, s.rho, s.ux, s.uy, s.uz, s.T, THERMAL, (C)0);
    }
    if (!(p.flags & kStepPeek)) {
      K::template collide_flow<COLL>(p, s.F, s.rho, s.ux, s.uy, s.uz);
      K::store_flow(p, c, s.F);
      if constexpr (THERMAL) {
        K::collide_thermal(p, s.G, s.T, false, s.ux, s.uy, s.uz, (C)0);
        K::store_thermal(p, c, s.G);
      }
    }
  }
  if (diag) {
    const int blk = blockIdx.x + gridDim.x * blockIdx.y;
    block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blk), (size_t)p.partial_rows);
  }
}

// ------------------------------------------------------- init / finalize
// Equilibrium initialisation: post-collision state of f = feq(rho,u), g = geq(T,u),
// i.e. what the reference's first collision produces after init_kernel
// (src/LBM/LBM2D/_initialize.py:37-65).
template <class L, class S, int COLL, int THERM>
__global__ void init_equilibrium_kernel(StepParams<S> p, const float* rho_in, const float* u_in,
                                        const float* T_in, const float* alpha_in, int solid_bit) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= p.N) return;
  const uint8_t m0 = p.mask[c];
  const bool solid = (m0 >> solid_bit) & 1;
  p.mask[c] = (uint8_t)((m0 & LBM_MASK_REACTIVE) | (solid ? LBM_MASK_SOLID : 0u));
  const C rho = (C)rho_in[c];
  const C ux = (C)u_in[c], uy = (C)u_in[p.N + c], uz = (C)u_in[2 * p.N + c];
  if (!solid) {
    C F[Q];
    const C usq = ux * ux + uy * uy + uz * uz;
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      F[k] = K::template feq<k>(p, rho, ux, uy, uz, usq);
    });
    K::template collide_flow<COLL>(p, F, rho, ux, uy, uz);
    K::store_flow(p, (int)c, F);
  }
  if constexpr (THERMAL) {
    const C T = (C)T_in[c];
    C G[QT];
    const C z0 = 0;
    static_for<QT>([&](auto kk) { G[decltype(kk)::value] = z0; });
    // geq itself: collide_thermal with itau toward geq from G = geq gives geq.
    const C usq = solid ? (C)0 : ux * ux + uy * uy + uz * uz;
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if (solid) G[k] = (C)L::wt(k) * T;
      else {
        const C eu = (C)L::ex(k) * ux + (C)L::ey(k) * uy + (C)L::ez(k) * uz;
        G[k] = (C)L::wt(k) * T * ((C)1.0 + (C)L::ta * eu + (C)L::tb * eu * eu - (C)L::tc * usq);
      }
    });
    K::store_thermal(p, (int)c, G);
  }
  if constexpr (PYRO) {
    p.alpha[c] = alpha_in ? (C)alpha_in[c] : ((m0 & LBM_MASK_REACTIVE) ? (C)1 : (C)0);
    p.relB[c] = (C)0;
    const_cast<C*>(p.relA)[c] = (C)0;
  }
}

constexpr int kStage1Blocks = 256;  // first-level partial sums of the diagnostics

__device__ __forceinline__ double diag_identity(int i) {
  return i == 4 ? 1e300 : ((i == 3 || i == 5) ? -1e300 : 0.0);
}
__device__ __forceinline__ double diag_combine(int i, double a, double b) {
  return (i == 3 || i == 5) ? fmax(a, b) : (i == 4 ? fmin(a, b) : a + b);
}

// Fixed-shape shared-memory tree over 256 threads; returns the total in thread 0.
__device__ __forceinline__ double block_tree_256(int i, double v, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) sh[threadIdx.x] = diag_combine(i, sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

// Stage 1: block b reduces a contiguous chunk of the per-block partial rows
// (SoA layout partials[i * nrows + row]).  Fixed partition and tree: the
// result does not depend on scheduling.  Launch: kStage1Blocks x 256.
static __global__ void __launch_bounds__(256) reduce_diag_stage1(const double* partials, int nrows,
                                                                 double* stage1) {
  __shared__ double sh[256];
  const int chunk = (nrows + gridDim.x - 1) / gridDim.x;
  const int r0 = blockIdx.x * chunk, r1 = min(nrows, r0 + chunk);
  for (int i = 0; i < kNumDiag; ++i) {
    double v = diag_identity(i);
    for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x)
      v = diag_combine(i, v, partials[(size_t)i * nrows + r]);
    v = block_tree_256(i, v, sh);
    if (threadIdx.x == 0) stage1[i * gridDim.x + blockIdx.x] = v;
  }
}

// Stage 2: one block of 256 threads reduces the stage-1 sums into out[kNumDiag].
static __global__ void __launch_bounds__(256) reduce_diag_stage2(const double* stage1, int n, double* out) {
  __shared__ double sh[256];
  for (int i = 0; i < kNumDiag; ++i) {
    double v = diag_identity(i);
    for (int r = threadIdx.x; r < n; r += blockDim.x) v = diag_combine(i, v, stage1[i * n + r]);
    v = block_tree_256(i, v, sh);
    if (threadIdx.x == 0) out[i] = (i == 3) ? sqrt(v) : v;
  }
}

}  // namespace lbm
