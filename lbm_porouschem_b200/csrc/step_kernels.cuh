// step_kernels.cuh -- fused pull-scheme lattice update for sm_100a.
//
// One pass of step_bulk<> does, per cell, what the reference does in three
// separate Taichi loops (src/LBM/LBM2D/_evolution.py:16-25):
//   stream (pull form of the push at :67-95, halfway bounce-back at :78-86)
//   -> macro (:118-202: rho, u, T, sources, pyrolysis)
//   -> collision of the NEXT step (:26-66: BGK/MRT toward feq, Guo force,
//      thermal BGK with the geq(dS) source).
// Reading post-collision populations of step n and writing those of step n+1
// keeps one read and one write per population per step.  Cells on active
// (non-periodic) domain sides are finished by step_boundary<>, which re-derives
// the non-equilibrium extrapolation (src/LBM/LBM2D/_boundary.py:17-101) from
// the same input buffer; cells that turn fluid are finished by flip_cells<>.
//
// Layout in HBM (structure of arrays, x fastest, c = x + nx*(y + ny*z)):
//   f[buf][k][c]   storage type S (float / __half shifted / double), buf = A|B
//   g[buf][k][c]   temperature populations
//   mask[c]        uint8: bit0/bit1 solid at even/odd parity, bit2 reactive
//   alpha[c]       reactive fraction (compute precision; solid cells, in place)
//   rel[buf][c]    gas release per unit lattice weight (reacting solid cells)
//
// Bounce-back by own slots.  Every cell stores its post-collision populations in its
// own slots f[k][c]; solid cells carry no flow populations (their flow slots are never
// read).  A fluid cell pulls direction k from f[k][c-e_k]; when c-e_k is solid, the
// halfway bounce-back value is the cell's own post-collision population of direction
// opp(k) from the last pass, f[opp k][c].  So every pull is one load whose address
// depends on one link bit, every store goes to the cell's own slots, and a warp's
// stores of a row cover whole sectors when its solid lanes store too (the dense
// kernel stores zeros there).
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
  __device__ __forceinline__ static C ldg(const float* p, size_t i, C) { return __ldg(p + i); }
  __device__ __forceinline__ static void st(float* p, size_t i, C v, C) { p[i] = v; }
  __device__ __forceinline__ static void st_sr(float* p, size_t i, C v, C, uint32_t) { p[i] = v; }
};
template <> struct Store<double> {
  using C = double;
  __device__ __forceinline__ static C ld(const double* p, size_t i, C) { return p[i]; }
  __device__ __forceinline__ static C ldg(const double* p, size_t i, C) { return __ldg(p + i); }
  __device__ __forceinline__ static void st(double* p, size_t i, C v, C) { p[i] = v; }
  __device__ __forceinline__ static void st_sr(double* p, size_t i, C v, C, uint32_t) { p[i] = v; }
};

// 32-bit integer hash ("lowbias32", C. Wellons, 2018: xor-shift / multiply rounds).
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16; x *= 0x7feb352du;
  x ^= x >> 15; x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Stochastic rounding of v to half precision: the neighbour toward zero, h0, or the next
// one away from zero, h1, the latter with probability |v - h0| / |h1 - h0|, so the stored
// value equals v on average.  A change of a slowly varying field smaller than half a unit
// in the last place then survives on average instead of being rounded away at every step
// (round to nearest stalls slow diffusion).  The threshold is a hash of v's own bits and
// a salt per direction: a function of the stored state alone, so every bulk form, a batch,
// a slab decomposition and a resumed run store the same bits.
__device__ __forceinline__ __half half_sr(float v, uint32_t salt) {
  const __half h0 = __float2half_rz(v);
  const float v0 = __half2float(h0);
  if (v0 == v) return h0;
  const __half h1 = __ushort_as_half((unsigned short)(__half_as_ushort(h0) + 1u));
  const float v1 = __half2float(h1);
  const float u = (float)(hash32(__float_as_uint(v) + salt) >> 8) * (1.0f / 16777216.0f);
  return fabsf(v - v0) > u * fabsf(v1 - v0) ? h1 : h0;
}
// FP16 storage of the deviation from the rest equilibrium (value - shift),
// FP32 arithmetic.
template <> struct Store<__half> {
  using C = float;
  __device__ __forceinline__ static C ld(const __half* p, size_t i, C shift) {
    return __half2float(p[i]) + shift;
  }
  __device__ __forceinline__ static C ldg(const __half* p, size_t i, C shift) {
    return __half2float(__ldg(p + i)) + shift;
  }
  // stochastically rounded store (the temperature populations); salt: per direction
  __device__ __forceinline__ static void st_sr(__half* p, size_t i, C v, C shift, uint32_t salt) {
    p[i] = half_sr(v - shift, salt);
  }
  __device__ __forceinline__ static void st(__half* p, size_t i, C v, C shift) {
    p[i] = __float2half_rn(v - shift);
  }
};

constexpr int kNumDiag = 10;              // partial slots per block (order of lbm_diag fields)
// Internal collision codes: LBM_COLL_BGK / LBM_COLL_MRT, plus kCollSutherland when the
// viscosity follows the cell's temperature (LBM_VISC_SUTHERLAND), or plus kCollPorous
// when the lattice has porous cells (lbm_desc.porous)
constexpr int kCollSutherland = 2;
constexpr int kCollPorous = 4;
__host__ __device__ constexpr bool coll_sutherland(int coll) { return (coll & ~1) == kCollSutherland; }
__host__ __device__ constexpr bool coll_porous(int coll) { return (coll & ~1) == kCollPorous; }

// Flow-rate inlet state (LBM_FIELD_INLET, compute precision): slot 0 holds the
// coefficient F/flow0 of the current step; after kInletHead slots come two halves,
// one per step parity, each of 4 planes over the side's cells j = y + ny*z: rho*u_x
// of side cell (0,y,z) and the velocity of cell (1,y,z), as the step before left them.
constexpr int kInletHead = 32;
template <class C>
__host__ __device__ __forceinline__ C* inlet_half(C* base, int half, size_t M) {
  return base + kInletHead + (size_t)half * 4 * M;
}
constexpr int kStepPeek = 1 << 8;         // internal flag: recompute outputs, leave the state untouched
constexpr double kGasConstant = 8.314441; // src/LBM/util/constant.py:17

// Register cap of the FP32/FP16 bulk kernels (FP64 keeps the full budget):
// 128 registers = 4 blocks of 128 threads (16 warps) per SM.  On B200 at 256^3
// (D3Q19-MRT + D3Q7 + pyrolysis), 96 and 80 registers with 5 and 6 blocks per SM
// measured slower: FP32 10.9 and 9.2 GLUPS, FP16 15.8 and 15.1, against 12.3 and 18.0.
#ifndef LBM_BULK_MAXNREG
#define LBM_BULK_MAXNREG 128
#endif
template <class S> struct BulkRegs { static constexpr int v = LBM_BULK_MAXNREG; };
// FP64: 168 registers = 3 blocks per SM (the ordinary MRT step does not spill); at 256^3
// 9.14 GLUPS against 8.22 with the full budget (215 registers, 2 blocks per SM).
#ifndef LBM_BULK_MAXNREG_F64
#define LBM_BULK_MAXNREG_F64 168
#endif
template <> struct BulkRegs<double> { static constexpr int v = LBM_BULK_MAXNREG_F64; };

// Resident 128-thread list-kernel blocks per SM at the register cap (65,536
// registers per SM, allocated 8 per thread at a time): 4 at 128, 3 for FP64 at 168.
inline int list_blocks_per_sm(bool fp64) {
  const int regs = ((fp64 ? BulkRegs<double>::v : BulkRegs<float>::v) + 7) / 8 * 8;
  return 65536 / (128 * regs);
}

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
  int par;         // step parity: mask bit read this pass
  int eos;
  int half_force;
  int has_force;
  C nu, Fx, Fy, Fz;
  C mrt_sn[19];    // s_r / |M_r|^2 for non-viscous, non-conserved rows
  C itauT_f, itauT_s;
  C rho0, T0;
  C pyA, pyb, pyEaR, pyTmin, Tref, Tscale, dtp, heat_norm, gas_coef, alpha_flip;  // pyEaR = Ea/R
  // collision codes kCollSutherland + BGK/MRT (properties that follow the cell's
  // temperature): the Sutherland viscosity (suth set), and per phase (bit 0 fluid, 1 solid of
  // tprop) the derived thermal diffusivity k(T) / rho / c(T) * dt / dx^2 (lbm_desc.tprop)
  int suth;
  C suthA, suthTs;
  int tprop;
  C tp_cond[2][5], tp_lo[2][5], tp_hi[2][5], tp_Tmid[2], tp_mul[2], tp_Tsc[2], tp_Tref[2];
  C tp_rhos, tp_dt, tp_dx2, tp_lat, tp_prandtl;
  const C* poro;   // porous cells (collision codes kCollPorous + BGK/MRT): solid fraction,
  const C* darcy;  //   Darcy and Forchheimer coefficients per cell, and the model
  const C* forch;  //   (LBM_PORO_*)
  int poro_model;
  // porous cells with two temperature fields (THERM 4): TS populations of the porous cells
  // (read and write halves), per cell h*a, rhos and emissivity*a_r (3 planes), the solid
  // temperature mapping, heat capacities, sigma/dx, T_ambient^4 and the radiation switch
  const S* gsA;
  S* gsB;
  const C* xheat;
  C Trs, Tss, cap_f, cap_s, sig_dx, Tamb4;
  int radiation;
  int fp16_nearest;  // FP16 storage: temperature populations rounded to nearest (else stochastically)
  int nebb;          // the active sides use NEBB (Zou-He, 2D, no temperature field)
  int inward_only;   // bit s: a cell on side s alone stores only the populations that point
                     // into the domain (the only ones any later pull reads there)
  int active;      // bit s: side s uses NEE
  const lbm_side_desc* sides;  // device copy
  int flags;       // LBM_STEP_* | kStepPeek
  int adiabatic;   // two-field temperature (pull_thermal<>'s run-time form)
  double* partials;    // SoA: partials[i * partial_rows + block]
  int partial_rows;
  int block_offset;
  C* rho_out;
  C* u_out;
  C* T_out;
  float* uprev;
  C* inlet;        // flow-rate inlet state (LBM_FIELD_INLET), null without one
  int* err;        // bit 0: a bounded wait gave up; bit 1: the fluid list overflowed
  unsigned wait_spins;  // tries of a bounded mbarrier wait (dense kernel) before it gives up
  // cell lists (step_list<>): entry cell index / neighbour-solid bits, the entry
  // of each cell (-1: none) and the list header (kLh* slots)
  uint32_t* ent_c;
  uint32_t* ent_b;
  int* pos;
  int* lhdr;
  int* flips;      // [2][N]: cells that turned fluid on a pass of parity 0 / 1
  // x-face records (lbm SCRATCH): post-stream populations F[Q] then G[QT] of the cells at
  // x = 1 (side 0) and x = nx - 2 (side 1), plane-major [side][value][y + ny z]; written by
  // the bulk kernels, read by step_boundary; null: the boundary kernel pulls them itself
  C* face;
  int face_sides;  // bit s: side s records
  uint32_t nx_mul; // c / nx = umulhi(c, nx_mul) >> nx_shr (exact for every 32-bit c)
  int nx_shr;
};

// Division by the run-time constant nx with a multiply-high (Granlund & Montgomery, PLDI
// 1994): m = ceil(2^(32+l) / d) - 2^32 with l = ceil(log2 d), then
// q = (umulhi(n, m) + ((n - umulhi(n, m)) >> 1)) >> (l - 1) for every 32-bit n.
inline void fastdiv_init(uint32_t d, uint32_t& m, int& l) {
  l = 0;
  while ((1ull << l) < d) ++l;
  m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
}
__device__ __forceinline__ uint32_t fastdiv(uint32_t n, uint32_t m, int l) {
  const uint32_t t = __umulhi(n, m);
  return l == 0 ? n : (t + ((n - t) >> 1)) >> (l - 1);
}

// Cell-list entries (step_list<>): bit k (1..Q-1) of the bit word is set if
// c + e_k is solid; kEntReactive marks a reactive cell, kEntDead an entry whose
// cell has left the list.
constexpr uint32_t kEntReactive = 1u << 24;
constexpr uint32_t kEntDead = 1u << 31;
constexpr uint32_t kEntPad = 0xffffffffu;  // cell index of a padding entry

// List header slots (int32).
enum : int {
  kLhFi = 0,      // end of the fluid interior segment
  kLhFg = 1,      // begin of the fluid general segment (multiple of 32)
  kLhFe = 2,      // end of the fluid list (grows when cells turn fluid)
  kLhSb = 3,      // begin of the solid list = capacity of the fluid list
  kLhSi = 4,      // end of the solid interior segment
  kLhSg = 5,      // begin of the solid general segment
  kLhSe = 6,      // end of the solid list
  kLhFlip0 = 8,   // cells that turned fluid on a pass of parity 0 / 1 (flip lists)
  kLhFlip1 = 9,
  kLhSlots = 16
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
// wrap (src/LBM/LBM2D/_evolution.py:205-212).
struct Nbhd {
  int xs[3], ro[3], po[3];
  Nbhd() = default;
  __device__ __forceinline__ Nbhd(int x, int y, int z, int nx, int ny, int nz) {
    xs[0] = wrapi(x - 1, nx); xs[1] = x; xs[2] = wrapi(x + 1, nx);
    ro[0] = wrapi(y - 1, ny) * nx; ro[1] = y * nx; ro[2] = wrapi(y + 1, ny) * nx;
    const int pl = nx * ny;
    po[0] = wrapi(z - 1, nz) * pl; po[1] = z * pl; po[2] = wrapi(z + 1, nz) * pl;
  }
  // Cell c away from every periodic edge: neighbours are plain offsets.
  __device__ __forceinline__ static Nbhd interior(int c, int nx, int pl) {
    Nbhd n;
    n.xs[0] = c - 1; n.xs[1] = c; n.xs[2] = c + 1;
    n.ro[0] = -nx; n.ro[1] = 0; n.ro[2] = nx;
    n.po[0] = -pl; n.po[1] = 0; n.po[2] = pl;
    return n;
  }
  __device__ __forceinline__ int at(int dx, int dy, int dz) const {
    return xs[dx + 1] + ro[dy + 1] + po[dz + 1];
  }
};

template <class C> __device__ __forceinline__ bool finite_(C v) { return isfinite(v); }

template <class L, class S>
struct Kern {
  using C = typename Store<S>::C;
  using P = StepParams<S>;
  static constexpr int Q = L::Q, QT = L::QT, NP = num_pairs<L>();

  __device__ __forceinline__ static bool solid_bit(const P& p, int c, int bit) {
    return (p.mask[c] >> bit) & 1;
  }

  // bit k (1..Q-1) set if the neighbour c + e_k is solid at mask parity `bit`.
  __device__ __forceinline__ static uint32_t neighbour_bits(const P& p, const Nbhd& nb, int bit) {
    uint32_t b = 0;
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if constexpr (k > 0) b |= (uint32_t)((p.mask[nb.at(L::ex(k), L::ey(k), L::ez(k))] >> bit) & 1) << k;
    });
    return b;
  }

  // Post-stream flow populations of fluid cell c.  Pull direction k comes from
  // c - e_k = c + e_opp(k) (bit opp(k) of nbits set if that cell is solid): the
  // neighbour's slot f[k][c-e_k], or at a solid neighbour the halfway bounce-back,
  // c's own slot f[opp k][c] (same FP16 shift: w(k) = w(opp k)), plus the gas a
  // reacting solid neighbour released along that link.
  template <bool PYRO>
  __device__ __forceinline__ static void pull_flow(const P& p, const Nbhd& nb, int c, uint32_t nbits, C F[Q]) {
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if constexpr (k == 0) {
        F[0] = Store<S>::ldg(p.fA, c, fshift<L, S, 0>(p));
      } else {
        const int src = nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
        const bool bb = (nbits >> L::opp(k)) & 1;
        const size_t idx = bb ? (size_t)L::opp(k) * p.N + c : (size_t)k * p.N + src;
        C v = Store<S>::ldg(p.fA, idx, fshift<L, S, k>(p));
        if constexpr (PYRO) {
          if (bb) v += p.relA[src] * (C)L::w(k);
        }
        F[k] = v;
      }
    });
  }

  // Post-stream temperature populations.  Conjugate mode streams through solids.  In
  // the two-field mode (the reference's TF / TS, which never exchange heat across a
  // binary mask, src/LBM/LBM2D/_evolution.py:67-95) a link to a cell of the other phase
  // is adiabatic: the population bounces back, i.e. comes from c's own slot of the
  // opposite direction.  ADIA selects that at compile time, RT tests p.adiabatic at run
  // time instead (the ordinary step of the list kernel; fewer registers there).
  // nbits: bit j set if c + e_j is solid; solid: c itself.
  template <bool ADIA = false, bool RT = false>
  __device__ __forceinline__ static void pull_thermal(const P& p, const Nbhd& nb, int c, uint32_t nbits,
                                                      bool solid, C G[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if constexpr (k == 0) {
        G[0] = Store<S>::ldg(p.gA, c, gshift<L, S, 0>(p));
      } else {
        size_t idx = (size_t)k * p.N + nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
        if constexpr (ADIA || RT) {
          if ((ADIA || p.adiabatic) && ((nbits >> L::opp(k)) & 1) != (uint32_t)solid)
            idx = (size_t)L::opp(k) * p.N + c;
        }
        G[k] = Store<S>::ldg(p.gA, idx, gshift<L, S, k>(p));
      }
    });
  }

  // Two fields with porous cells (THERM 4).  A cell's first temperature field (in G) is
  // TF where the cell is fluid or porous and TS in a pure-solid cell.  TF crosses to fluid
  // and porous neighbours and bounces back at pure-solid ones; TS of a pure-solid cell
  // crosses to solid neighbours and to porous ones (whose TS is in GS) and bounces back at
  // pure-fluid ones (src/LBM/LBM2D/_evolution.py:69-100).
  __device__ __forceinline__ static void pull_thermal_ph(const P& p, const Nbhd& nb, int c, uint32_t nbits,
                                                         bool solid, C G[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if constexpr (k == 0) {
        G[0] = Store<S>::ldg(p.gA, c, gshift<L, S, 0>(p));
      } else {
        const int n = nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
        const S* src = p.gA;
        size_t idx = (size_t)k * p.N + n;
        if (((nbits >> L::opp(k)) & 1) != (uint32_t)solid) {
          if (solid && p.poro[n] > (C)0) src = p.gsA;
          else idx = (size_t)L::opp(k) * p.N + c;
        }
        G[k] = Store<S>::ldg(src, idx, gshift<L, S, k>(p));
      }
    });
  }
  // TS of a porous cell: from the G of pure-solid neighbours, the GS of porous ones, and
  // its own slot of the opposite direction at pure-fluid ones.
  __device__ __forceinline__ static void pull_ts(const P& p, const Nbhd& nb, int c, uint32_t nbits, C GS[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if constexpr (k == 0) {
        GS[0] = Store<S>::ldg(p.gsA, c, gshift<L, S, 0>(p));
      } else {
        const int n = nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
        const S* src = p.gsA;
        size_t idx = (size_t)k * p.N + n;
        if ((nbits >> L::opp(k)) & 1) src = p.gA;
        else if (!(p.poro[n] > (C)0)) idx = (size_t)L::opp(k) * p.N + c;
        GS[k] = Store<S>::ldg(src, idx, gshift<L, S, k>(p));
      }
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
    if (p.eos == 0) {
      const C ir = (C)1 / r;
      jx *= ir; jy *= ir; jz *= ir;
    }
    rho = r; ux = jx; uy = jy; uz = jz;
  }

  // 1/(eps + 1e-12) of a fluid cell (eps = 1 - solid = 1), src/LBM/LBM2D/_evolution.py:216
  __host__ __device__ static constexpr C kie() { return (C)1 / ((C)1 + (C)1e-12); }

  // feq9/feq19 (src/LBM/LBM2D/_evolution.py:213-225; ie = 1/(eps + 1e-12), eps = 1 - solid)
  // split into the part even under e -> -e (ev) and the odd part (od): feq_k = ev + od,
  // feq_opp(k) = ev - od.
  template <int k>
  __device__ __forceinline__ static void feq_pair(const P& p, C rho, C ux, C uy, C uz, C usq, C& ev, C& od,
                                                  C ie = kie()) {
    const C eu = (C)L::ex(k) * ux + (C)L::ey(k) * uy + (C)L::ez(k) * uz;
    const C w = (C)L::w(k);
    if (p.eos == 1) {
      ev = w * (rho + (C)4.5 * eu * eu * ie - (C)1.5 * usq * ie);
      od = w * ((C)3.0 * eu);
    } else {
      ev = w * rho * ((C)1.0 + (C)4.5 * eu * eu * ie - (C)1.5 * usq * ie);
      od = w * rho * ((C)3.0 * eu);
    }
  }
  __device__ __forceinline__ static C feq_rest(const P& p, C rho, C usq, C ie = kie()) {
    const C w = (C)L::w(0);
    return p.eos == 1 ? w * (rho - (C)1.5 * usq * ie) : w * rho * ((C)1.0 - (C)1.5 * usq * ie);
  }
  // Full equilibrium set of (rho, u) in F.
  __device__ __forceinline__ static void feq_all(const P& p, C rho, C ux, C uy, C uz, C F[Q], C ie = kie()) {
    const C usq = ux * ux + uy * uy + uz * uz;
    F[0] = feq_rest(p, rho, usq, ie);
    static_for<NP>([&](auto pp) {
      constexpr int k = pk<L>(decltype(pp)::value), o = L::opp(k);
      C ev, od;
      feq_pair<k>(p, rho, ux, uy, uz, usq, ev, od, ie);
      F[k] = ev + od;
      F[o] = ev - od;
    });
  }

  // What drives one cell's collision besides its moments: ie = 1/(eps + 1e-12) of the
  // equilibrium and the force of forceTermGuo (src/LBM/LBM2D/_evolution.py:254-261: the
  // volume force, plus the Darcy drag in a porous cell).
  struct Drive {
    C ie, Fx, Fy, Fz;
    bool force;
  };
  __device__ __forceinline__ static Drive plain_drive(const P& p) { return Drive{kie(), p.Fx, p.Fy, p.Fz, p.has_force != 0}; }

  // A porous cell's drive: eps = 1 - solid and the drag of its model added to the volume
  // force (darcy_force, src/LBM/LBM2D/_evolution.py:262-283; the 3D solver takes the lattice
  // viscosity there instead of the kinetic one, LBM3D/_evolution.py:262-278).  s: solid
  // fraction (0 < s < 1), velocity and density of the cell.
  __device__ __forceinline__ static Drive porous_drive(const P& p, int c, C s, C rho, C ux, C uy, C uz) {
    const C eps = (C)1 - s;
    const C nu = L::DIM == 2 && p.eos == 0 ? p.nu / rho : p.nu;
    const C v = sqrt(ux * ux + uy * uy + uz * uz);
    C a;
    if (p.poro_model == LBM_PORO_ERGUN) {
      const C perm = eps * eps * eps / (((C)1.000001 - eps) * ((C)1.000001 - eps));
      const C beta = (C)1.75 / sqrt((C)150 * eps * perm);
      a = -nu / perm * eps - beta * v;
    } else if (p.poro_model == LBM_PORO_DARCY) {
      a = -eps * nu * p.darcy[c];
    } else {
      a = -eps * nu * p.darcy[c] - eps * p.forch[c] * v;
    }
    return Drive{(C)1 / (eps + (C)1e-12), p.Fx + a * ux, p.Fy + a * uy, p.Fz + a * uz, true};
  }

  // macro's velocity correction of a porous cell (src/LBM/LBM2D/_evolution.py:131-151) at
  // its new density, then its drive.  Returns the plain drive for a cell that is not porous.
  __device__ __forceinline__ static Drive porous_cell(const P& p, int c, C rho, C& ux, C& uy, C& uz) {
    const C s = p.poro[c];
    if (s == (C)0 || s == (C)1) return plain_drive(p);
    const C eps = (C)1 - s;
    const C nu = p.eos == 0 ? p.nu / rho : p.nu;  // kinetic_viscosity(i)
    C div;
    if (p.poro_model == LBM_PORO_DARCY) {
      div = (C)1 + eps * nu * p.darcy[c] / (C)2;
    } else {
      C Dc, Fc;
      if (p.poro_model == LBM_PORO_ERGUN) {
        const C perm = eps * eps * eps / (((C)1.000001 - eps) * ((C)1.000001 - eps));
        Dc = (C)1 / perm;
        Fc = (C)1.75 / sqrt((C)150 * eps * eps * eps);
      } else {
        Dc = p.darcy[c];
        Fc = p.forch[c];
      }
      const C c0 = (C)0.5 * ((C)1 + eps * nu / (C)2 * Dc);
      const C c1 = (C)0.5 * eps * Fc;
      const C v = sqrt(ux * ux + uy * uy + uz * uz);
      div = c0 + sqrt(c0 * c0 + c1 * v);
    }
    const C idv = (C)1 / div;
    ux *= idv; uy *= idv; uz *= idv;
    return porous_drive(p, c, s, rho, ux, uy, uz);
  }

  // forceTermGuo, src/LBM/LBM2D/_evolution.py:284-298, force and ie of the drive
  template <int k>
  __device__ __forceinline__ static C guo(const P& p, C rho, C ux, C uy, C uz, C pre, const Drive& d) {
    const C ie = d.ie;
    const C ex = (C)L::ex(k), ey = (C)L::ey(k), ez = (C)L::ez(k);
    const C t1 = (ex - ux * ie) * d.Fx + (ey - uy * ie) * d.Fy + (ez - uz * ie) * d.Fz;
    const C eu = ex * ux + ey * uy + ez * uz;
    const C eF = ex * d.Fx + ey * d.Fy + ez * d.Fz;
    const C t = pre * (C)L::w(k) * ((C)3.0 * t1 + (C)9.0 * eu * eF * ie);
    return p.eos == 1 ? t : rho * t;
  }

  // Flow collision (BGK: _evolution.py:33; MRT: new) plus Guo forcing; writes
  // the post-collision populations over F.  Works on opposite-direction pairs.
  template <int COLL>
  __device__ __forceinline__ static void collide_flow(const P& p, C F[Q], C rho, C ux, C uy, C uz, C T = (C)0) {
    collide_flow_d<COLL>(p, F, rho, ux, uy, uz, T, plain_drive(p));
  }
  template <int COLL>
  __device__ __forceinline__ static void collide_flow_d(const P& p, C F[Q], C rho, C ux, C uy, C uz, C T,
                                                        const Drive& dr) {
    C nu = p.nu;
    if constexpr (coll_sutherland(COLL)) {
      if (p.suth) {
        // Sutherland, src/LBM/LBM2D/_evolution.py:232-234, at the cell's temperature in kelvin
        const C TK = T * p.Tscale + p.Tref;
        nu = p.suthA * TK * sqrt(TK) / (TK + p.suthTs);
      }
    }
    const C tau = (C)3 * (p.eos == 0 ? nu / rho : nu) + (C)0.5;
    const C itau = (C)1 / tau;
    const C usq = ux * ux + uy * uy + uz * uz;
    const C fe0 = feq_rest(p, rho, usq, dr.ie);
    if constexpr ((COLL & 1) == LBM_COLL_BGK) {
      F[0] = F[0] - itau * (F[0] - fe0);
      static_for<NP>([&](auto pp) {
        constexpr int k = pk<L>(decltype(pp)::value), o = L::opp(k);
        C ev, od;
        feq_pair<k>(p, rho, ux, uy, uz, usq, ev, od, dr.ie);
        F[k] = F[k] - itau * (F[k] - (ev + od));
        F[o] = F[o] - itau * (F[o] - (ev - od));
      });
    } else {
      // non-equilibrium parts in pair form: Sn = fneq_k + fneq_o, Dn = fneq_k - fneq_o
      const C n0 = F[0] - fe0;
      C Sn[NP], Dn[NP];
      static_for<NP>([&](auto pp) {
        constexpr int q = decltype(pp)::value;
        constexpr int k = pk<L>(q), o = L::opp(k);
        C ev, od;
        feq_pair<k>(p, rho, ux, uy, uz, usq, ev, od, dr.ie);
        const C a = F[k] - (ev + od), b = F[o] - (ev - od);
        Sn[q] = a + b;
        Dn[q] = a - b;
      });
      // forward transform of the non-conserved moments, scaled by s_r/|M_r|^2
      C mt[Q];
      static_for<Q>([&](auto rr) {
        constexpr int r = decltype(rr)::value;
        if constexpr (!L::mrt_conserved(r)) {
          constexpr bool even = mrt_even<L>(r);
          C acc = 0;
          if constexpr (even && L::mrt(r, 0) != 0.0) acc = (C)L::mrt(r, 0) * n0;
          static_for<NP>([&](auto pp) {
            constexpr int q = decltype(pp)::value;
            constexpr double mv = L::mrt(r, pk<L>(q));
            const C v = even ? Sn[q] : Dn[q];
            if constexpr (mv == 1.0) acc += v;
            else if constexpr (mv == -1.0) acc -= v;
            else if constexpr (mv != 0.0) acc += (C)mv * v;
          });
          constexpr double inv_norm = 1.0 / mrt_norm<L>(r);
          if constexpr (L::mrt_viscous(r)) mt[r] = acc * itau * (C)inv_norm;
          else mt[r] = acc * p.mrt_sn[r];
        }
      });
      // back transform: even part E (same for k and opp), odd part O (opposite sign)
      {
        C e0 = 0;
        static_for<Q>([&](auto rr) {
          constexpr int r = decltype(rr)::value;
          if constexpr (!L::mrt_conserved(r) && mrt_even<L>(r) && L::mrt(r, 0) != 0.0)
            e0 += (C)L::mrt(r, 0) * mt[r];
        });
        F[0] -= e0;
      }
      static_for<NP>([&](auto pp) {
        constexpr int k = pk<L>(decltype(pp)::value), o = L::opp(k);
        C E = 0, O = 0;
        static_for<Q>([&](auto rr) {
          constexpr int r = decltype(rr)::value;
          if constexpr (!L::mrt_conserved(r)) {
            constexpr double mv = L::mrt(r, k);
            C& a = mrt_even<L>(r) ? E : O;
            if constexpr (mv == 1.0) a += mt[r];
            else if constexpr (mv == -1.0) a -= mt[r];
            else if constexpr (mv != 0.0) a += (C)mv * mt[r];
          }
        });
        F[k] -= E + O;
        F[o] -= E - O;
      });
    }
    if (dr.force) {
      const C pre = (C)1.0 - (C)1.0 / (C)2.0 / tau;
      static_for<Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        F[k] += guo<k>(p, rho, ux, uy, uz, pre, dr);
      });
    }
  }

  // Thermal relaxation rate of a cell: its phase's constant, or where the phase's bit of
  // tprop is set (collision codes kCollSutherland + BGK/MRT) the derived diffusivity at
  // the cell's temperature, TF/TS.coefDiff with DERIVED (src/LBM/LBM2D/_thermal.py:62-71,
  // :167-174), conductivity and capacity in the nested form of :79, :93, :97-99 / :182, :196,
  // :200-202, and
  // tau = 3 D + 1/2 (2D) or 4 D + 1/2 (3D) (_scalarField.py:56-58 of LBM2D / LBM3D).
  template <int COLL>
  __device__ __forceinline__ static C itau_thermal(const P& p, bool fluid, C T, C rho) {
    if constexpr (coll_sutherland(COLL)) {
      if (fluid && ((p.tprop >> 2) & 1)) {
        // PRANDTL: kinetic_viscosity / Pr, src/LBM/LBM2D/_thermal.py:67-68, _evolution.py:227-246
        C nu = p.nu;
        if (p.suth) {
          const C TK = T * p.Tscale + p.Tref;
          nu = p.suthA * TK * sqrt(TK) / (TK + p.suthTs);
        }
        if (p.eos == 0) nu = nu / rho;
        return (C)1 / (p.tp_lat * (nu / p.tp_prandtl) + (C)0.5);
      }
      const int ph = fluid ? 0 : 1;
      if ((p.tprop >> ph) & 1) {
        const C Tp = T * p.tp_Tsc[ph] + p.tp_Tref[ph];
        const C k = nested5(p.tp_cond[ph], Tp);
        const C cm = (Tp < p.tp_Tmid[ph] ? nested5(p.tp_lo[ph], Tp) : nested5(p.tp_hi[ph], Tp)) * p.tp_mul[ph];
        const C D = k / (fluid ? rho : p.tp_rhos) / cm * p.tp_dt / p.tp_dx2;
        return (C)1 / (p.tp_lat * D + (C)0.5);
      }
    }
    return fluid ? p.itauT_f : p.itauT_s;
  }
  // c0 + T (c1 + T (c2 T + T (c3 + T c4))), the reference's evaluation order
  __device__ __forceinline__ static C nested5(const C* c, C T) {
    return c[0] + T * (c[1] + T * (c[2] * T + T * (c[3] + T * c[4])));
  }

  // Thermal collision with source, one code path for fluid and solid cells:
  // fluid geq = TF.geq (advected), solid geq = w T (TS.geq, LBM2D/_thermal.py:162-166),
  // i.e. the fluid form with u = 0; source wt*dS (_evolution.py:54-58).
  // USRC: the source enters as TF.geq(k, dS) with the cell's velocity (the two-field
  // exchange source of a fluid or porous cell, src/LBM/LBM2D/_evolution.py:54-56), else as
  // w dS (the pyrolysis heat sink of a solid cell, where u = 0 makes the two equal)
  template <bool USRC = false>
  __device__ __forceinline__ static void collide_thermal(const P& p, C G[QT], C T, C itau, C ux, C uy, C uz,
                                                         C dS) {
    const C usq = ux * ux + uy * uy + uz * uz;
    {
      const C ge = (C)L::wt(0) * T * ((C)1.0 - (C)L::tc * usq);
      const C src = USRC ? (C)L::wt(0) * dS * ((C)1.0 - (C)L::tc * usq) : (C)L::wt(0) * dS;
      G[0] = G[0] - itau * (G[0] - ge) + src;
    }
    static_for<(QT - 1) / 2>([&](auto pp) {
      constexpr int k = pkt<L, QT>(decltype(pp)::value), o = L::opp(k);
      const C eu = (C)L::ex(k) * ux + (C)L::ey(k) * uy + (C)L::ez(k) * uz;
      const C wT = (C)L::wt(k) * T;
      const C ev = wT * ((C)1.0 + (C)L::tb * eu * eu - (C)L::tc * usq);
      const C od = wT * ((C)L::ta * eu);
      if constexpr (USRC) {
        const C wd = (C)L::wt(k) * dS;
        const C sev = wd * ((C)1.0 + (C)L::tb * eu * eu - (C)L::tc * usq);
        const C sod = wd * ((C)L::ta * eu);
        G[k] = G[k] - itau * (G[k] - (ev + od)) + (sev + sod);
        G[o] = G[o] - itau * (G[o] - (ev - od)) + (sev - sod);
      } else {
        const C src = (C)L::wt(k) * dS;
        G[k] = G[k] - itau * (G[k] - (ev + od)) + src;
        G[o] = G[o] - itau * (G[o] - (ev - od)) + src;
      }
    });
  }
  // TS collision of a porous cell: towards w T_s with the source w dS_s (TS.geq,
  // src/LBM/LBM2D/_thermal.py:162-166; _evolution.py:39-41, :56-57)
  __device__ __forceinline__ static void collide_ts(const P& p, C GS[QT], C Ts, C dSs) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      const C w = (C)L::wt(k);
      GS[k] = GS[k] - p.itauT_s * (GS[k] - w * Ts) + w * dSs;
    });
  }
  // geq of (T, u) itself (initialisation).
  __device__ __forceinline__ static void geq_all(C T, C ux, C uy, C uz, C G[QT]) {
    const C usq = ux * ux + uy * uy + uz * uz;
    G[0] = (C)L::wt(0) * T * ((C)1.0 - (C)L::tc * usq);
    static_for<(QT - 1) / 2>([&](auto pp) {
      constexpr int k = pkt<L, QT>(decltype(pp)::value), o = L::opp(k);
      const C eu = (C)L::ex(k) * ux + (C)L::ey(k) * uy + (C)L::ez(k) * uz;
      const C wT = (C)L::wt(k) * T;
      const C ev = wT * ((C)1.0 + (C)L::tb * eu * eu - (C)L::tc * usq);
      const C od = wT * ((C)L::ta * eu);
      G[k] = ev + od;
      G[o] = ev - od;
    });
  }

  // Store post-collision flow populations in the cell's own slots.
  __device__ __forceinline__ static void store_flow(const P& p, int c, const C F[Q]) {
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      Store<S>::st(p.fB, (size_t)k * p.N + c, F[k], fshift<L, S, k>(p));
    });
  }
  // Post-collision TS populations of porous cell c, in its own slots.
  __device__ __forceinline__ static void store_ts(const P& p, int c, const C GS[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if (p.fp16_nearest) Store<S>::st(p.gsB, (size_t)k * p.N + c, GS[k], gshift<L, S, k>(p));
      else Store<S>::st_sr(p.gsB, (size_t)k * p.N + c, GS[k], gshift<L, S, k>(p), 0x9e3779b9u * (k + 1));
    });
  }
  // Post-collision temperature populations of cell c, in its own slots (the adiabatic
  // links of the two-field mode are resolved by the pull).
  __device__ __forceinline__ static void store_thermal(const P& p, int c, const C G[QT]) {
    static_for<QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if (p.fp16_nearest) Store<S>::st(p.gB, (size_t)k * p.N + c, G[k], gshift<L, S, k>(p));
      else Store<S>::st_sr(p.gB, (size_t)k * p.N + c, G[k], gshift<L, S, k>(p), 0x9e3779b9u * (k + 1));
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
// Per-thread diagnostics: FP64 sums (mass, energy, solid reactive fraction,
// residual numerator and denominator), max |u|^2 / min T / max T in the compute
// type C, integer counts.  The block partial rows are FP64 in lbm_diag order.
template <class C>
struct DiagAcc {
  double mass, energy, alpha, res_num, res_den;
  C u2max, Tmin, Tmax;
  unsigned nonfinite, nfluid;
  __device__ __forceinline__ void clear() {
    mass = energy = alpha = res_num = res_den = 0;
    u2max = 0;
    Tmin = (C)3.0e38;
    Tmax = (C)-3.0e38;
    nonfinite = nfluid = 0;
  }
  // add another accumulator (a cell's contribution) into this one
  __device__ __forceinline__ void merge(const DiagAcc& b) {
    mass += b.mass; energy += b.energy; alpha += b.alpha; res_num += b.res_num; res_den += b.res_den;
    u2max = fmax(u2max, b.u2max); Tmin = fmin(Tmin, b.Tmin); Tmax = fmax(Tmax, b.Tmax);
    nonfinite += b.nonfinite; nfluid += b.nfluid;
  }
  __device__ __forceinline__ double get(int i) const {
    switch (i) {
      case 0: return mass;
      case 1: return energy;
      case 2: return alpha;
      case 3: return (double)u2max;
      case 4: return Tmin <= (C)-3.0e38 || Tmin >= (C)3.0e38 ? (Tmin > 0 ? 1e300 : -1e300) : (double)Tmin;
      case 5: return Tmax <= (C)-3.0e38 || Tmax >= (C)3.0e38 ? (Tmax > 0 ? 1e300 : -1e300) : (double)Tmax;
      case 6: return (double)nonfinite;
      case 7: return (double)nfluid;
      case 8: return res_num;
      default: return res_den;
    }
  }
};

// Per-thread accumulators in shared memory, one array per field (consecutive
// threads hit consecutive banks).
template <class C, int T>
struct DiagSmem {
  double mass[T], energy[T], alpha[T], res_num[T], res_den[T];
  C u2max[T], Tmin[T], Tmax[T];
  unsigned nonfinite[T], nfluid[T];
  __device__ __forceinline__ void clear(int t) {
    mass[t] = energy[t] = alpha[t] = res_num[t] = res_den[t] = 0;
    u2max[t] = 0; Tmin[t] = (C)3.0e38; Tmax[t] = (C)-3.0e38;
    nonfinite[t] = nfluid[t] = 0;
  }
  __device__ __forceinline__ void merge(int t, const DiagAcc<C>& b) {
    mass[t] += b.mass; energy[t] += b.energy; alpha[t] += b.alpha; res_num[t] += b.res_num; res_den[t] += b.res_den;
    u2max[t] = fmax(u2max[t], b.u2max); Tmin[t] = fmin(Tmin[t], b.Tmin); Tmax[t] = fmax(Tmax[t], b.Tmax);
    nonfinite[t] += b.nonfinite; nfluid[t] += b.nfluid;
  }
  __device__ __forceinline__ DiagAcc<C> load(int t) const {
    DiagAcc<C> a;
    a.mass = mass[t]; a.energy = energy[t]; a.alpha = alpha[t]; a.res_num = res_num[t]; a.res_den = res_den[t];
    a.u2max = u2max[t]; a.Tmin = Tmin[t]; a.Tmax = Tmax[t]; a.nonfinite = nonfinite[t]; a.nfluid = nfluid[t];
    return a;
  }
};

// Block reduction with warp shuffles (FP64), one partial row per block.
template <class C>
__device__ __forceinline__ void block_reduce_store(const DiagAcc<C>& a, double* out_row, size_t stride) {
  __shared__ double sh[32][kNumDiag];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nwarps = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int i = 0; i < kNumDiag; ++i) {
    double v = a.get(i);
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

// Flow part of one cell's diagnostics (and macro/residual outputs).
template <class S>
__device__ __forceinline__ void diag_flow(const StepParams<S>& p, DiagAcc<typename Store<S>::C>& a, int c,
                                          typename Store<S>::C rho, typename Store<S>::C ux,
                                          typename Store<S>::C uy, typename Store<S>::C uz) {
  using C = typename Store<S>::C;
  a.mass += (double)rho;
  // in double with explicit roundings: no contraction choice of the kernel at hand changes it
  // (FP64 velocities would otherwise round differently in the tile, list and dense forms)
  const double u2 = __dadd_rn(__dadd_rn(__dmul_rn((double)ux, (double)ux), __dmul_rn((double)uy, (double)uy)),
                              __dmul_rn((double)uz, (double)uz));
  a.u2max = fmax(a.u2max, (C)u2);
  if (!finite_(rho)) a.nonfinite += 1;
  a.nfluid += 1;
  if (p.flags & LBM_STEP_RESIDUAL) {
    const double dx = (double)ux - p.uprev[c], dy = (double)uy - p.uprev[p.N + c],
                 dz = (double)uz - p.uprev[2 * p.N + c];
    a.res_num += dx * dx + dy * dy + dz * dz;
    a.res_den += (double)ux * ux + (double)uy * uy + (double)uz * uz;
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
}
// Temperature part (every cell).
template <class S>
__device__ __forceinline__ void diag_thermal(const StepParams<S>& p, DiagAcc<typename Store<S>::C>& a, int c,
                                             typename Store<S>::C T) {
  a.energy += (double)T;
  a.Tmin = fmin(a.Tmin, T);
  a.Tmax = fmax(a.Tmax, T);
  if (!finite_(T)) a.nonfinite += 1;
  if (p.flags & LBM_STEP_MACRO) p.T_out[c] = T;
}

// Mean post-stream (rho, u) over the fluid neighbours of (x,y,z) at the pass
// parity, in direction order 1..Q-1; (1, 0) if there are none.  Used when a
// spent solid cell turns fluid.
template <class L, class S>
__device__ __noinline__ void neighbour_mean(const StepParams<S>& p, int x, int y, int z,
                                            typename Store<S>::C& rb, typename Store<S>::C& ux,
                                            typename Store<S>::C& uy, typename Store<S>::C& uz) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q;
  C rs = 0, us0 = 0, us1 = 0, us2 = 0;
  int n = 0;
  for (int q = 1; q < Q; ++q) {
    int dx = 0, dy = 0, dz = 0;
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      if (k == q) { dx = L::ex(k); dy = L::ey(k); dz = L::ez(k); }
    });
    const int xq = wrapi(x + dx, p.nx), yq = wrapi(y + dy, p.ny), zq = wrapi(z + dz, p.nz);
    const int cq = xq + p.nx * (yq + p.ny * zq);
    if (K::solid_bit(p, cq, p.par)) continue;
    const Nbhd nq(xq, yq, zq, p.nx, p.ny, p.nz);
    const uint32_t nbq = K::neighbour_bits(p, nq, p.par);
    C Fq[Q], rq, uxq, uyq, uzq;
    K::template pull_flow<true>(p, nq, cq, nbq, Fq);
    K::moments(p, Fq, rq, uxq, uyq, uzq);
    rs += rq; us0 += uxq; us1 += uyq; us2 += uzq;
    ++n;
  }
  rb = n ? rs / (C)n : (C)1;
  ux = n ? us0 / (C)n : (C)0;
  uy = n ? us1 / (C)n : (C)0;
  uz = n ? us2 / (C)n : (C)0;
}

// ------------------------------------------------------------------ kernels
// THERM: 0 no temperature, 1 conjugate, 2 conjugate + pyrolysis, 3 two-field
// (adiabatic fluid-solid links), 4 two-field with porous cells (TF and TS in a porous cell,
// exchanging heat there).

// x-face record of cell c (post-stream F, and G with the temperature field) if it sits at
// x = 1 or x = nx - 2 next to an active x side: step_boundary<> extrapolates that side from
// it.  The bulk kernels update only cells off the active sides, so a record exists for a
// face cell exactly when its inner cell is not on another active side (face_record).
template <class L, class S, bool THERMAL>
__device__ __forceinline__ void record_face(const StepParams<S>& p, int c, const typename Store<S>::C* F,
                                            const typename Store<S>::C* G) {
  const uint32_t j = fastdiv((uint32_t)c, p.nx_mul, p.nx_shr);  // y + ny z
  const int x = c - (int)j * p.nx;
  const int side = (x == 1 && (p.face_sides & 1)) ? 0 : ((x == p.nx - 2 && (p.face_sides & 2)) ? 1 : -1);
  if (side < 0) return;
  constexpr int FV = L::Q + (THERMAL ? L::QT : 0);
  const size_t M = (size_t)p.ny * p.nz;
  typename Store<S>::C* o = p.face + (size_t)side * FV * M + j;
  static_for<L::Q>([&](auto kk) { o[(size_t)decltype(kk)::value * M] = F[decltype(kk)::value]; });
  if constexpr (THERMAL)
    static_for<L::QT>([&](auto kk) { o[(size_t)(L::Q + decltype(kk)::value) * M] = G[decltype(kk)::value]; });
}
template <class L, class S>
__device__ __forceinline__ bool face_record(const StepParams<S>& p, int x, int y, int z) {
  if (!p.face) return false;
  if (!((x == 1 && (p.face_sides & 1)) || (x == p.nx - 2 && (p.face_sides & 2)))) return false;
  return !Kern<L, S>::on_active_side(p, x, y, z);
}

// The TS field of porous cell c and the heat its two fields exchange (THERM 4): pulls and
// sums TS, computes the exchange dH = h a (T_f,phys - T_s,phys) dt and the surface
// radiation q = e sigma a_r/dx (T_amb^4 - T_s,phys^4) as the reference's macro does
// (src/LBM/LBM2D/_evolution.py:186-202, _thermal.py:213-220), collides and stores TS with
// its source, and returns TF's source -dH/(c_f rho T_scale).  Tf: the cell's TF, rho its
// density.
template <class L, class S>
__device__ __forceinline__ typename Store<S>::C porous_heat(const StepParams<S>& p, const Nbhd& nb, int c,
                                                            uint32_t nbits, typename Store<S>::C Tf,
                                                            typename Store<S>::C rho, bool peek) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  C GS[L::QT];
  K::pull_ts(p, nb, c, nbits, GS);
  C Ts = 0;
  static_for<L::QT>([&](auto kk) { Ts += GS[decltype(kk)::value]; });
  if (p.flags & LBM_STEP_MACRO) p.T_out[p.N + c] = Ts;  // second plane of the macro temperature
  const C TsP = Ts * p.Tss + p.Trs;
  const C dH = p.xheat[c] * ((Tf * p.Tscale + p.Tref) - TsP) * p.dtp;
  const C rs = p.xheat[p.N + c];
  C dSs = dH / p.cap_s / rs / p.Tss;
  if (p.radiation) {
    const C T2 = TsP * TsP;
    const C q = p.xheat[2 * p.N + c] * p.sig_dx * (p.Tamb4 - T2 * T2);
    dSs += q * p.dtp / p.cap_s / rs / p.Tss;
  }
  if (!peek) {
    K::collide_ts(p, GS, Ts, dSs);
    K::store_ts(p, c, GS);
  }
  return -dH / p.cap_f / rho / p.Tscale;
}

// Where cell_update<> takes its post-stream populations from: straight from the
// input buffers in HBM (this source), or from copies staged in shared memory
// (StagedPull in list_kernel.cuh).
template <class L, class S>
struct GlobalPull {
  using C = typename Store<S>::C;
  template <bool PYRO>
  __device__ __forceinline__ void flow(const StepParams<S>& p, const Nbhd& nb, int c, uint32_t nbits,
                                       C F[L::Q]) const {
    Kern<L, S>::template pull_flow<PYRO>(p, nb, c, nbits, F);
  }
  template <bool ADIA, bool RT>
  __device__ __forceinline__ void thermal(const StepParams<S>& p, const Nbhd& nb, int c, uint32_t nbits, bool solid,
                                          C G[L::QT]) const {
    Kern<L, S>::template pull_thermal<ADIA, RT>(p, nb, c, nbits, solid, G);
  }
  __device__ __forceinline__ C alpha(const StepParams<S>& p, int c) const { return p.alpha[c]; }
};
//
// One cell of the fused update (shared by the tile and the cell-list bulk
// kernels): temperature pull, flow pull/moments/collision/store for fluid cells,
// Arrhenius pyrolysis for reactive solid cells, temperature collision/store and
// the diagnostics.  nbits: bit k set if c + e_k is solid at this parity.  mk is
// the mask byte (read only by a peek pass over a reactive cell).  Returns whether
// the cell is solid at the next parity.
template <class L, class S, int COLL, int THERM, class Src = GlobalPull<L, S>, bool RT = false>
__device__ __forceinline__ bool cell_update(const StepParams<S>& p, DiagAcc<typename Store<S>::C>& acc, bool diag, bool peek, int c,
                                            const Nbhd& nb, uint32_t nbits, bool solid, bool reactive,
                                            uint8_t mk, const Src& src = Src()) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2, PHEAT = THERM == 4;
  C G[QT > 0 ? QT : 1];
  C T = 0, dS = 0, rho = 0, ux = 0, uy = 0, uz = 0;
  if constexpr (THERMAL) {
    if constexpr (PHEAT) K::pull_thermal_ph(p, nb, c, nbits, solid, G);
    else src.template thermal<THERM == 3, RT>(p, nb, c, nbits, solid, G);
    static_for<QT>([&](auto kk) { T += G[decltype(kk)::value]; });
  }
  bool solid_next = solid;
  bool flipping = false;
  if (!solid) {
    C F[Q];
    src.template flow<PYRO>(p, nb, c, nbits, F);
    if (p.face) record_face<L, S, THERMAL>(p, c, F, G);
    K::moments(p, F, rho, ux, uy, uz);
    typename K::Drive dr = K::plain_drive(p);
    if constexpr (coll_porous(COLL)) dr = K::porous_cell(p, c, rho, ux, uy, uz);
    if constexpr (PHEAT) {
      if (p.poro[c] > (C)0) dS = porous_heat<L, S>(p, nb, c, nbits, T, rho, peek);
    }
    if (!peek) {
      K::template collide_flow_d<COLL>(p, F, rho, ux, uy, uz, T, dr);
      K::store_flow(p, c, F);
    }
    if (diag) diag_flow(p, acc, c, rho, ux, uy, uz);  // after the store: fewer live registers
  } else if constexpr (PYRO) {
    if (reactive) {
      if (peek) {
        // current state: a cell that turned fluid on the last pass is fluid now;
        // flip_cells<> reports its flow state
        if (!((mk >> (p.par ^ 1)) & 1)) solid_next = false;
      } else {
        // Arrhenius rate at the solid temperature, src/LBM/LBM2D/_chemical.py:198-212
        const C a = src.alpha(p, c);
        const C TK = T * p.Tscale + p.Tref;
        C kr = 0;
        if (TK > p.pyTmin) {
          const C Te = TK + (C)1e-6;
          kr = p.pyA * exp(-(p.pyEaR / Te));
          if (p.pyb != (C)0) kr *= pow(Te, p.pyb);
        }
        const C da = kr * a * p.dtp;
        const C an = a - da;
        p.alpha[c] = an;
        dS = -p.heat_norm * da;
        if (an < p.alpha_flip) {
          // turns fluid: flip_cells<> finishes it after this pass and finds the
          // heat source here
          solid_next = false;
          flipping = true;
          p.relB[c] = dS;
        } else {
          C W = 0;
          static_for<Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            if constexpr (k > 0) {
              if (!((nbits >> k) & 1)) W += (C)L::w(k);
            }
          });
          p.relB[c] = W > (C)0 ? p.gas_coef * da / W : (C)0;
        }
      }
    }
  }
  if constexpr (THERMAL) {
    if (!peek && !flipping) {
      const bool fl = !solid;
      K::template collide_thermal<PHEAT>(p, G, T, K::template itau_thermal<COLL>(p, fl, T, rho), fl ? ux : (C)0,
                                         fl ? uy : (C)0, fl ? uz : (C)0, dS);
      K::store_thermal(p, c, G);
    }
    if (diag) diag_thermal(p, acc, c, T);
  }
  if (PYRO && diag && solid_next && reactive) acc.alpha += (double)p.alpha[c];
  return solid_next;
}

// Tile form of the bulk update: one block per run of blockDim.x cells of an x row
// (blockDim.x a multiple of 32, at most 256); register cap BulkRegs<S>.
template <class L, class S, int COLL, int THERM>
__global__ void __maxnreg__(BulkRegs<S>::v) step_bulk(const __grid_constant__ StepParams<S> p) {
  using K = Kern<L, S>;
  const int y = blockIdx.y, z = blockIdx.z;
  const bool diag = (p.flags & (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) != 0;
  const bool peek = (p.flags & kStepPeek) != 0;
  DiagAcc<typename Store<S>::C> acc;
  if (diag) acc.clear();

  // Rank the tile's cells fluid first, then solid, then cells this kernel skips
  // (past nx or on an active side), so that warps run one branch instead of both.
  __shared__ uint8_t s_rank_cell[256];
  __shared__ uint8_t s_mask[256];
  __shared__ int s_count[2][8];
  int x, cell_kind;  // 0 fluid, 1 solid, 2 skipped
  uint8_t mk;
  {
    const int xt = blockIdx.x * blockDim.x + threadIdx.x;
    const bool ok = xt < p.nx && !K::on_active_side(p, xt, y, z);
    const uint8_t mt = ok ? p.mask[xt + p.nx * (y + p.ny * z)] : (uint8_t)0;
    const int kind = !ok ? 2 : (((mt >> p.par) & 1) ? 1 : 0);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const unsigned bf = __ballot_sync(0xffffffffu, kind == 0), bs = __ballot_sync(0xffffffffu, kind == 1);
    if (lane == 0) { s_count[0][warp] = __popc(bf); s_count[1][warp] = __popc(bs); }
    s_mask[threadIdx.x] = mt;
    __syncthreads();
    int nf = 0, ns = 0, pf = 0, ps = 0, pk_ = 0;
    for (int w = 0; w < nw; ++w) {
      if (w < warp) { pf += s_count[0][w]; ps += s_count[1][w]; pk_ += 32 - s_count[0][w] - s_count[1][w]; }
      nf += s_count[0][w]; ns += s_count[1][w];
    }
    const unsigned lt = (1u << lane) - 1u;
    int rank;
    if (kind == 0) rank = pf + __popc(bf & lt);
    else if (kind == 1) rank = nf + ps + __popc(bs & lt);
    else rank = nf + ns + pk_ + __popc(~(bf | bs) & lt);
    s_rank_cell[rank] = (uint8_t)threadIdx.x;
    __syncthreads();
    const int t = s_rank_cell[threadIdx.x];
    x = blockIdx.x * blockDim.x + t;
    mk = s_mask[t];
    cell_kind = (int)threadIdx.x < nf ? 0 : ((int)threadIdx.x < nf + ns ? 1 : 2);
  }

  if (cell_kind != 2) {
    const int c = x + p.nx * (y + p.ny * z);
    const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
    const bool solid = cell_kind == 1;
    const uint32_t nbits = K::neighbour_bits(p, nb, p.par);
    const bool solid_next = cell_update<L, S, COLL, THERM>(p, acc, diag, peek, c, nb, nbits, solid,
                                                          (mk & LBM_MASK_REACTIVE) != 0, mk);
    // mask bit for the next parity: written only when it changes
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

// Cell-list upkeep for cell c turning fluid (nbn: its neighbour bits at the
// next parity): its solid entry dies, a fluid entry is appended, and the bit
// that points at c is cleared in the entries of its neighbours.  Neighbours that
// turn fluid on the same pass build their entries from the next-parity mask, so
// the order of these updates does not matter.
template <class L, class S>
__device__ __forceinline__ void list_turn_fluid(const StepParams<S>& p, int c, const Nbhd& nb, uint32_t nbn) {
  const int old = p.pos[c];
  if (old >= 0) atomicOr(&p.ent_b[old], kEntDead);
  const int idx = atomicAdd(&p.lhdr[kLhFe], 1);
  if (idx >= p.lhdr[kLhSb]) {  // cannot happen: the fluid list has room for every listed cell
    if (p.err) atomicOr(p.err, 2);
    return;
  }
  p.ent_c[idx] = (uint32_t)c;
  p.ent_b[idx] = nbn;
  p.pos[c] = idx;
  static_for<L::Q>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    if constexpr (k > 0) {
      const int n = nb.at(-L::ex(k), -L::ey(k), -L::ez(k));  // n + e_k = c
      const int pn = p.pos[n];
      if (pn >= 0) atomicAnd(&p.ent_b[pn], ~(1u << k));
    }
  });
}

// Cells that turned fluid on this pass (mask bit par solid, bit par^1 fluid).
// Runs after step_bulk and step_boundary, over the whole mask (in a peek pass it
// only reports the flow state of cells that turned fluid on the last pass):
//  1. X takes the mean post-stream (rho, u) of its fluid neighbours, collides
//     from that equilibrium and stores in its own slots, which its fluid
//     neighbours pull from on the next pass (their own post-collision values are
//     already in their own slots, where X pulls them from);
//  2. its temperature populations collide as fluid with the heat source that
//     step_bulk left in rel[B][X].
template <class L, class S, int COLL, int THERM>
__device__ __forceinline__ void flip_one(const StepParams<S>& p, DiagAcc<typename Store<S>::C>& acc, bool diag,
                                         bool peek, size_t c0) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1;
  const int np = p.par ^ 1;
  const uint8_t mk = p.mask[c0];
  if (!(((mk >> p.par) & 1) && !((mk >> np) & 1))) return;
  const int c = (int)c0;
  const int x = c % p.nx, y = (c / p.nx) % p.ny, z = c / (p.nx * p.ny);
  const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
  C rb, ux, uy, uz;
  neighbour_mean<L, S>(p, x, y, z, rb, ux, uy, uz);
  if (peek) {
    // recomputing the current state: report the state the cell was given
    if (diag) diag_flow(p, acc, c, rb, ux, uy, uz);
    return;
  }
  // temperature first: the collision's viscosity may depend on it (the pull reads the
  // input half, which the flow store below does not touch)
  C G[QT > 0 ? QT : 1];
  C T = 0;
  if constexpr (THERMAL) {
    K::pull_thermal(p, nb, c, 0u, true, G);  // conjugate field only (pyrolysis)
    static_for<QT>([&](auto kk) { T += G[decltype(kk)::value]; });
  }
  {
    C F[Q];
    K::feq_all(p, rb, ux, uy, uz, F);
    K::template collide_flow<COLL>(p, F, rb, ux, uy, uz, T);
    K::store_flow(p, c, F);
    if (p.ent_c) list_turn_fluid<L>(p, c, nb, K::neighbour_bits(p, nb, np));
  }
  if constexpr (THERMAL) {
    // the cell is fluid now: its last heat source enters as TF.geq(k, dS) with its velocity
    // (src/LBM/LBM2D/_evolution.py:54-56)
    const C dS = p.relB[c];
    p.relB[c] = (C)0;
    K::template collide_thermal<true>(p, G, T, K::template itau_thermal<COLL>(p, true, T, rb), ux, uy, uz, dS);
    K::store_thermal(p, c, G);
  }
  if (diag) diag_flow(p, acc, c, rb, ux, uy, uz);
}

template <class L, class S, int COLL, int THERM>
__global__ void __launch_bounds__(256) flip_cells(const __grid_constant__ StepParams<S> p) {
  const bool diag = (p.flags & (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) != 0;
  DiagAcc<typename Store<S>::C> acc;
  if (diag) acc.clear();
  const int np = p.par ^ 1;
  const bool peek = (p.flags & kStepPeek) != 0;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  // with cell lists the bulk pass listed the cells that turned fluid; otherwise
  // the whole mask is scanned
  const bool listed = p.lhdr != nullptr;
  const size_t n = listed ? (size_t)p.lhdr[kLhFlip0 + p.par] : p.N;
  if (listed && !peek && blockIdx.x == 0 && threadIdx.x == 0) p.lhdr[kLhFlip0 + np] = 0;  // for the next pass
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const size_t c0 = listed ? (size_t)p.flips[(size_t)p.par * p.N + i] : i;
    flip_one<L, S, COLL, THERM>(p, acc, diag, peek, c0);
  }
  if (diag) block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blockIdx.x), (size_t)p.partial_rows);
}

// ------------------------------------------------------ flow-rate inlet
// Coefficient F/flow0 of this step (src/LBM/LBM2D/_boundary.py:324-329): flow0 sums
// rho*u_x over the side cells as the previous step left them (half p.par).  One block;
// FP64 sum in a fixed order.
template <class S>
__global__ void __launch_bounds__(1024) inlet_flow_coef(const __grid_constant__ StepParams<S> p) {
  using C = typename Store<S>::C;
  const size_t M = (size_t)p.ny * p.nz;
  const C* m = inlet_half(p.inlet, p.par, M);
  double acc = 0.0;
  for (size_t j = threadIdx.x; j < M; j += blockDim.x) acc += (double)m[j];
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ double part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < (blockDim.x >> 5) ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) p.inlet[0] = (C)(p.sides[0].v[0] / acc);
  }
}

// Controller start (src/LBM/LBM2D/_initialize.py:67-73): both reads of the first
// step see the uniform inlet velocity v0 = F/ny/nz, with the initial density of the
// side cells.  Half 0 (the first step's parity).  One block.
template <class C>
__global__ void __launch_bounds__(1024) inlet_seed(C* inlet, const float* rho, int nx, int ny, int nz, double F) {
  const size_t M = (size_t)ny * nz;
  const C v0 = (C)(F / ny / nz);
  C* h = inlet_half(inlet, 0, M);
  for (size_t j = threadIdx.x; j < M; j += blockDim.x) {
    h[j] = (C)rho[(size_t)nx * j] * v0;
    h[M + j] = v0;
    h[2 * M + j] = (C)0;
    h[3 * M + j] = (C)0;
  }
  if (threadIdx.x == 0) inlet[0] = (C)1;
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
// With needT false the temperature part (G, T) is left unset.
//
// NEE replaces every population of a side cell from its inner neighbour's; of
// the side cell's own state only what its side's types keep (PERIODIC) is used.
// So the own state is computed only for such a side: at an inlet or outlet the
// cell pulls nothing of its own, which halves its loads and drops the sectors it
// would pull across the periodic wrap.
template <class L, class S, bool THERMAL, bool PYRO, int PASS>
__device__ __forceinline__ MState<L, S> bc_state(const StepParams<S>& p, int x, int y, int z, bool needT) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  MState<L, S> s;
  if constexpr (PASS < 0) {
    const int c = x + p.nx * (y + p.ny * z);
    if (face_record<L, S>(p, x, y, z)) {
      // recorded by the bulk kernel of this pass: coalesced reads
      constexpr int FV = L::Q + (THERMAL ? L::QT : 0);
      const size_t M = (size_t)p.ny * p.nz;
      const C* o = p.face + (size_t)(x == 1 ? 0 : 1) * FV * M + (size_t)y + (size_t)p.ny * z;
      static_for<L::Q>([&](auto kk) { s.F[decltype(kk)::value] = o[(size_t)decltype(kk)::value * M]; });
      K::moments(p, s.F, s.rho, s.ux, s.uy, s.uz);
      s.T = 0;
      if constexpr (THERMAL) {
        if (needT) {
          static_for<L::QT>([&](auto kk) { s.G[decltype(kk)::value] = o[(size_t)(L::Q + decltype(kk)::value) * M]; });
          static_for<L::QT>([&](auto kk) { s.T += s.G[decltype(kk)::value]; });
        }
      }
      return s;
    }
    const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
    const uint32_t nbits = K::neighbour_bits(p, nb, p.par);
    K::template pull_flow<PYRO>(p, nb, c, nbits, s.F);
    K::moments(p, s.F, s.rho, s.ux, s.uy, s.uz);
    s.T = 0;
    if constexpr (THERMAL) {
      if (needT) {
        // side cells and the inner cells NEE reads are fluid
        K::template pull_thermal<false, true>(p, nb, c, nbits, false, s.G);
        static_for<L::QT>([&](auto kk) { s.T += s.G[decltype(kk)::value]; });
      }
    }
    return s;
  } else {
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
    if (side < 0) return bc_state<L, S, THERMAL, PYRO, PASS - 1>(p, x, y, z, needT);
    const lbm_side_desc& sd = p.sides[side];
    const bool ownT = THERMAL && needT && sd.T_type == LBM_BC_PERIODIC;
    if (sd.v_type == LBM_BC_PERIODIC || sd.rho_type == LBM_BC_PERIODIC || ownT) {
      s = bc_state<L, S, THERMAL, PYRO, PASS - 1>(p, x, y, z, ownT);
    } else {
      s.rho = s.ux = s.uy = s.uz = s.T = (C)0;  // all set below (F and G entirely)
    }
    const MState<L, S> in = bc_state<L, S, THERMAL, PYRO, PASS - 1>(p, ix, iy, iz, needT);
    // _boundary.py:54-65 (flow), _scalarField.py:83-92 (scalar)
    if (sd.v_type == LBM_BC_FIXEDVALUE) { s.ux = (C)sd.v[0]; s.uy = (C)sd.v[1]; s.uz = (C)sd.v[2]; }
    else if (sd.v_type == LBM_BC_ZEROGRADIENT) { s.ux = in.ux; s.uy = in.uy; s.uz = in.uz; }
    else if (sd.v_type == LBM_BC_FLOWRATE) {
      // side 0 only: (a*F/flow0 + 1 - a) * u(1,y,z) of the previous step, a = 0.01
      // (src/LBM/LBM2D/_boundary.py:330-332)
      const size_t M = (size_t)p.ny * p.nz, j = (size_t)y + (size_t)p.ny * z;
      const C* w = inlet_half(p.inlet, p.par, M) + M;
      const C a = (C)0.01;
      const C gain = a * p.inlet[0] + (C)1 - a;
      s.ux = gain * w[j]; s.uy = gain * w[M + j]; s.uz = gain * w[2 * M + j];
    }
    if (sd.rho_type == LBM_BC_FIXEDVALUE) s.rho = (C)sd.rho;
    else if (sd.rho_type == LBM_BC_ZEROGRADIENT) s.rho = in.rho;
    const C usb = s.ux * s.ux + s.uy * s.uy + s.uz * s.uz;
    const C usi = in.ux * in.ux + in.uy * in.uy + in.uz * in.uz;
    if (sd.active == LBM_SIDE_ES) {
      // equilibrium scheme (src/LBM/LBM2D/_boundary.py:269-315): feq of the side's state
      s.F[0] = K::feq_rest(p, s.rho, usb);
      static_for<num_pairs<L>()>([&](auto pp) {
        constexpr int k = pk<L>(decltype(pp)::value), o = L::opp(k);
        C evb, odb;
        K::template feq_pair<k>(p, s.rho, s.ux, s.uy, s.uz, usb, evb, odb);
        s.F[k] = evb + odb;
        s.F[o] = evb - odb;
      });
    } else {
      s.F[0] = K::feq_rest(p, s.rho, usb) + (in.F[0] - K::feq_rest(p, in.rho, usi));
      static_for<num_pairs<L>()>([&](auto pp) {
        constexpr int k = pk<L>(decltype(pp)::value), o = L::opp(k);
        C evb, odb, evi, odi;
        K::template feq_pair<k>(p, s.rho, s.ux, s.uy, s.uz, usb, evb, odb);
        K::template feq_pair<k>(p, in.rho, in.ux, in.uy, in.uz, usi, evi, odi);
        s.F[k] = (evb + odb) + (in.F[k] - (evi + odi));
        s.F[o] = (evb - odb) + (in.F[o] - (evi - odi));
      });
    }
    if (THERMAL && needT) {
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

// Non-equilibrium bounce-back (Zou & He 1997) on the post-stream D2Q9 populations of a cell
// of side `side` (BC_MODEL.NEBB, src/LBM/LBM2D/_boundary.py:103-226): the populations that
// enter from outside are rebuilt from the known ones so that the cell takes the side's
// velocity (v_type fixed: wall or inlet) or density (rho_type fixed: outlet, the normal
// velocity then follows from the known populations; tangential velocity 0).  Every side in
// the Zou-He form (the reference's side-1 wall, side-1 inlet and side-2/3 inlet and outlet
// branches do otherwise; the oracle's ref_quirk_nebb restates them).
template <class C>
__device__ __forceinline__ void zou_he(int side, const lbm_side_desc& sd, C F[9]) {
  const bool vel = sd.v_type == LBM_BC_FIXEDVALUE, pres = sd.rho_type == LBM_BC_FIXEDVALUE;
  if (!vel && !pres) return;
  const C u = (C)sd.v[0], v = (C)sd.v[1], c23 = (C)(2.0 / 3.0), c16 = (C)(1.0 / 6.0), h = (C)0.5;
  C rho, w;
  switch (side) {
    case 0:  // x = 0: 1, 5, 8 enter
      if (vel) {
        rho = (F[0] + F[2] + F[4] + 2 * (F[3] + F[6] + F[7])) / ((C)1 - u);
        F[1] = F[3] + c23 * rho * u;
        F[5] = F[7] + h * (F[4] - F[2]) + c16 * rho * u + h * rho * v;
        F[8] = F[6] + h * (F[2] - F[4]) + c16 * rho * u - h * rho * v;
      } else {
        rho = (C)sd.rho;
        w = (C)1 - (F[0] + F[2] + F[4] + 2 * (F[3] + F[6] + F[7])) / rho;
        F[1] = F[3] + c23 * rho * w;
        F[5] = F[7] + h * (F[4] - F[2]) + c16 * rho * w;
        F[8] = F[6] + h * (F[2] - F[4]) + c16 * rho * w;
      }
      break;
    case 1:  // x = nx-1: 3, 6, 7 enter
      if (vel) {
        rho = (F[0] + F[2] + F[4] + 2 * (F[1] + F[5] + F[8])) / ((C)1 + u);
        F[3] = F[1] - c23 * rho * u;
        F[6] = F[8] + h * (F[4] - F[2]) - c16 * rho * u + h * rho * v;
        F[7] = F[5] + h * (F[2] - F[4]) - c16 * rho * u - h * rho * v;
      } else {
        rho = (C)sd.rho;
        w = (C)-1 + (2 * (F[1] + F[5] + F[8]) + F[0] + F[2] + F[4]) / rho;
        F[3] = F[1] - c23 * rho * w;
        F[6] = F[8] + h * (F[4] - F[2]) - c16 * rho * w;
        F[7] = F[5] + h * (F[2] - F[4]) - c16 * rho * w;
      }
      break;
    case 2:  // y = 0: 2, 5, 6 enter
      if (vel) {
        rho = (F[0] + F[1] + F[3] + 2 * (F[4] + F[7] + F[8])) / ((C)1 - v);
        F[2] = F[4] + c23 * rho * v;
        F[5] = F[7] + h * (F[3] - F[1]) + h * rho * u + c16 * rho * v;
        F[6] = F[8] + h * (F[1] - F[3]) - h * rho * u + c16 * rho * v;
      } else {
        rho = (C)sd.rho;
        w = (C)1 - (F[0] + F[1] + F[3] + 2 * (F[4] + F[7] + F[8])) / rho;
        F[2] = F[4] + c23 * rho * w;
        F[5] = F[7] + h * (F[3] - F[1]) + c16 * rho * w;
        F[6] = F[8] + h * (F[1] - F[3]) + c16 * rho * w;
      }
      break;
    default:  // y = ny-1: 4, 7, 8 enter
      if (vel) {
        rho = (F[0] + F[1] + F[3] + 2 * (F[2] + F[5] + F[6])) / ((C)1 + v);
        F[4] = F[2] - c23 * rho * v;
        F[7] = F[5] + h * (F[1] - F[3]) - h * rho * u - c16 * rho * v;
        F[8] = F[6] + h * (F[3] - F[1]) + h * rho * u - c16 * rho * v;
      } else {
        rho = (C)sd.rho;
        w = (C)-1 + (F[0] + F[1] + F[3] + 2 * (F[2] + F[5] + F[6])) / rho;
        F[4] = F[2] - c23 * rho * w;
        F[7] = F[5] + h * (F[1] - F[3]) - c16 * rho * w;
        F[8] = F[6] + h * (F[3] - F[1]) - c16 * rho * w;
      }
      break;
  }
}

// A cell on a NEBB side (2D, no temperature field): its own post-stream populations (the
// ones that enter from outside came across the periodic wrap, as the reference streams),
// Zou-He for the side that treats it -- an x side on rows 1 .. ny-2, a y side on every
// column (Boundary_condition_NEBB's two loops) -- then macro and the collision.
template <class L, class S, int COLL, int THERM>
__device__ __forceinline__ void nebb_boundary_cell(const StepParams<S>& p, int x, int y, int c,
                                                   DiagAcc<typename Store<S>::C>& acc, bool diag) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  if constexpr (L::DIM == 2 && THERM == 0) {
    const Nbhd nb(x, y, 0, p.nx, p.ny, 1);
    const uint32_t nbits = K::neighbour_bits(p, nb, p.par);
    C F[L::Q];
    K::template pull_flow<false>(p, nb, c, nbits, F);
    int side = -1;
    if (y >= 1 && y <= p.ny - 2 && x == 0 && (p.active & 1)) side = 0;
    else if (y >= 1 && y <= p.ny - 2 && x == p.nx - 1 && (p.active & 2)) side = 1;
    else if (y == 0 && (p.active & 4)) side = 2;
    else if (y == p.ny - 1 && (p.active & 8)) side = 3;
    if (side >= 0) zou_he<C>(side, p.sides[side], F);
    C rho, ux, uy, uz;
    K::moments(p, F, rho, ux, uy, uz);
    if (diag) diag_flow(p, acc, c, rho, ux, uy, uz);
    if (!(p.flags & kStepPeek)) {
      K::template collide_flow<COLL>(p, F, rho, ux, uy, uz);
      K::store_flow(p, c, F);
    }
  }
}

// Boundary cell i of face `face` (a cell on several active faces is owned by the
// lowest-numbered one): NEE state, collision, store.
template <class L, class S, int COLL, int THERM>
__device__ __forceinline__ void boundary_cell(const StepParams<S>& p, int face, int i,
                                              DiagAcc<typename Store<S>::C>& acc, bool diag) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
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
    for (int f = 0; f < face; ++f) {
      if (!(p.active & (1 << f))) continue;
      const bool on = (f == 0 && x == 0) || (f == 1 && x == p.nx - 1) || (f == 2 && y == 0) ||
                      (f == 3 && y == p.ny - 1) || (f == 4 && z == 0) || (f == 5 && z == p.nz - 1);
      if (on) valid = false;
    }
  }
  if (!valid) return;
  const int c = x + p.nx * (y + p.ny * z);
  if (p.nebb) {
    nebb_boundary_cell<L, S, COLL, THERM>(p, x, y, c, acc, diag);
    return;
  }
  MState<L, S> s = bc_state<L, S, THERMAL, PYRO, L::NPASS - 1>(p, x, y, z, THERMAL);
  if (p.inlet && x <= 1 && !(p.flags & kStepPeek)) {
    // flow-rate inlet: record what the next step's controller reads (final values)
    const size_t M = (size_t)p.ny * p.nz, j = (size_t)y + (size_t)p.ny * z;
    C* o = inlet_half(p.inlet, p.par ^ 1, M);
    if (x == 0) {
      o[j] = s.rho * s.ux;
      // cell (1,y,z) behind it: its post-stream state when no side owns it
      const bool owned = ((p.active & 2) && p.nx == 2) || ((p.active & 4) && y == 0) ||
                         ((p.active & 8) && y == p.ny - 1) || ((p.active & 16) && z == 0) ||
                         ((p.active & 32) && z == p.nz - 1);
      if (!owned) {
        const MState<L, S> b = bc_state<L, S, THERMAL, PYRO, -1>(p, 1, y, z, false);
        o[M + j] = b.ux; o[2 * M + j] = b.uy; o[3 * M + j] = b.uz;
      }
    } else {
      o[M + j] = s.ux; o[2 * M + j] = s.uy; o[3 * M + j] = s.uz;
    }
  }
  if (diag) {
    diag_flow(p, acc, c, s.rho, s.ux, s.uy, s.uz);
    if (THERMAL) diag_thermal(p, acc, c, s.T);
  }
  if (!(p.flags & kStepPeek)) {
    K::template collide_flow<COLL>(p, s.F, s.rho, s.ux, s.uy, s.uz, s.T);
    if constexpr (THERMAL)
      K::collide_thermal(p, s.G, s.T, K::template itau_thermal<COLL>(p, true, s.T, s.rho), s.ux, s.uy, s.uz, (C)0);
    // A cell on one side whose pair keeps no quantity of its own (no PERIODIC type) is read
    // afterwards only by the pulls of its inner neighbours, along the directions pointing
    // into the domain (the side cells extrapolate from their inner cells, their own slots
    // serve no bounce-back since the two outer layers are fluid); its other slots would be
    // dead stores, each a lone 4-byte write to a sector of its own.
    const int on = ((x == 0) ? 1 : 0) | ((x == p.nx - 1) ? 2 : 0) | ((y == 0) ? 4 : 0) | ((y == p.ny - 1) ? 8 : 0) |
                   ((L::DIM == 3 && z == 0) ? 16 : 0) | ((L::DIM == 3 && z == p.nz - 1) ? 32 : 0);
    const int act = on & p.active;
    const int sd = (act && !(act & (act - 1)) && (p.inward_only & act)) ? __ffs(act) - 1 : -1;
    if (sd < 0) {
      K::store_flow(p, c, s.F);
      if constexpr (THERMAL) K::store_thermal(p, c, s.G);
    } else {
      const int ax = sd >> 1, dir = (sd & 1) ? -1 : 1;
      static_for<L::Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        const int e = ax == 0 ? L::ex(k) : (ax == 1 ? L::ey(k) : L::ez(k));
        if (e == dir) Store<S>::st(p.fB, (size_t)k * p.N + c, s.F[k], fshift<L, S, k>(p));
      });
      if constexpr (THERMAL) {
        static_for<L::QT>([&](auto kk) {
          constexpr int k = decltype(kk)::value;
          const int e = ax == 0 ? L::ex(k) : (ax == 1 ? L::ey(k) : L::ez(k));
          if (e == dir) {
            if (p.fp16_nearest) Store<S>::st(p.gB, (size_t)k * p.N + c, s.G[k], gshift<L, S, k>(p));
            else Store<S>::st_sr(p.gB, (size_t)k * p.N + c, s.G[k], gshift<L, S, k>(p), 0x9e3779b9u * (k + 1));
          }
        });
      }
    }
  }
}

// One thread per boundary cell; blockIdx.y selects an active face.
template <class L, class S, int COLL, int THERM>
__global__ void __launch_bounds__(128) step_boundary(const __grid_constant__ StepParams<S> p, int4 faces01,
                                                      int2 faces2) {
  const int fid[6] = {faces01.x, faces01.y, faces01.z, faces01.w, faces2.x, faces2.y};
  const int face = fid[blockIdx.y];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool diag = (p.flags & (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) != 0;
  DiagAcc<typename Store<S>::C> acc;
  if (diag) acc.clear();
  boundary_cell<L, S, COLL, THERM>(p, face, i, acc, diag);
  if (diag) {
    const int blk = blockIdx.x + gridDim.x * blockIdx.y;
    block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blk), (size_t)p.partial_rows);
  }
}

// ------------------------------------------------------- init / finalize
// Equilibrium initialisation: post-collision state of f = feq(rho,u), g = geq(T,u),
// i.e. what the reference's first collision produces after init_kernel
// (src/LBM/LBM2D/_initialize.py:37-65).  Writes the B side of `p` (the buffer the
// first pass reads), own slots; `solid_bit` selects the input mask bit.
template <class L, class S, int COLL, int THERM>
__global__ void init_equilibrium_kernel(const __grid_constant__ StepParams<S> p, const float* rho_in,
                                        const float* u_in,
                                        const float* T_in, const float* alpha_in, int solid_bit) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  const size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (c >= p.N) return;
  const uint8_t m0 = p.mask[c];
  const bool solid = (m0 >> solid_bit) & 1;
  const int x = (int)(c % p.nx);
  const C rho = (C)rho_in[c];
  C ux = (C)u_in[c], uy = (C)u_in[p.N + c], uz = (C)u_in[2 * p.N + c];
  if (p.inlet && x <= 1) {
    // flow-rate inlet: the columns x = 0 and 1 start at the inlet velocity v0 = F/ny/nz,
    // which the reference writes into their macro velocity for its first collision
    // (src/LBM/LBM2D/_initialize.py:69-74); without it the first profile is zero
    ux = (C)(p.sides[0].v[0] / p.ny / p.nz);
    uy = uz = (C)0;
  }
  if (!solid) {
    C F[Q];
    typename K::Drive dr = K::plain_drive(p);
    if constexpr (coll_porous(COLL)) {
      // the reference's first collision: eps-equilibrium and drag at the initial velocity
      const C s = p.poro[c];
      if (s != (C)0 && s != (C)1) dr = K::porous_drive(p, (int)c, s, rho, ux, uy, uz);
    }
    K::feq_all(p, rho, ux, uy, uz, F, dr.ie);
    K::template collide_flow_d<COLL>(p, F, rho, ux, uy, uz, T_in ? (C)T_in[c] : (C)0, dr);
    K::store_flow(p, (int)c, F);
  }
  if constexpr (THERMAL) {
    C G[QT];
    if (solid) K::geq_all((C)T_in[c], (C)0, (C)0, (C)0, G);
    else K::geq_all((C)T_in[c], ux, uy, uz, G);
    K::store_thermal(p, (int)c, G);
  }
  if constexpr (THERM == 4) {
    // TS of a porous cell: w T_s, its temperature the second half of T_in
    if (!solid && p.poro[c] > (C)0) {
      C GS[QT];
      K::geq_all((C)T_in[p.N + c], (C)0, (C)0, (C)0, GS);
      K::store_ts(p, (int)c, GS);
    }
  }
  if constexpr (PYRO) {
    p.alpha[c] = alpha_in ? (C)alpha_in[c] : ((m0 & LBM_MASK_REACTIVE) ? (C)1 : (C)0);
    p.relB[c] = (C)0;
    const_cast<C*>(p.relA)[c] = (C)0;
  }
  p.mask[c] = (uint8_t)((m0 & LBM_MASK_REACTIVE) | (solid ? LBM_MASK_SOLID : 0u));
}

constexpr int kStage1Blocks = 256;  // first-level partial sums of the diagnostics

__device__ __forceinline__ double diag_identity(int i) {
  return i == 4 ? 1e300 : ((i == 3 || i == 5) ? -1e300 : 0.0);
}
__device__ __forceinline__ double diag_combine(int i, double a, double b) {
  return (i == 3 || i == 5) ? fmax(a, b) : (i == 4 ? fmin(a, b) : a + b);
}

// Fixed-shape shared-memory tree over 256 threads; returns the total in every thread.
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

// Both stages in one block of 1024 threads, for up to kSingleReduceRows partial rows (the
// cell-list form at any size: its rows are the persistent blocks and the boundary blocks):
// thread t combines rows t, t + 1024, ... in order, every field at once, then a fixed tree
// per field.  Deterministic; one launch instead of two.
constexpr int kSingleReduceRows = 8192;
static __global__ void __launch_bounds__(1024) reduce_diag_single(const double* partials, int nrows, double* out) {
  __shared__ double sh[1024];
  double v[kNumDiag];
#pragma unroll
  for (int i = 0; i < kNumDiag; ++i) v[i] = diag_identity(i);
  for (int r = threadIdx.x; r < nrows; r += blockDim.x) {
#pragma unroll
    for (int i = 0; i < kNumDiag; ++i) v[i] = diag_combine(i, v[i], partials[(size_t)i * nrows + r]);
  }
  for (int i = 0; i < kNumDiag; ++i) {
    sh[threadIdx.x] = v[i];
    __syncthreads();
    for (int st = 512; st > 0; st >>= 1) {
      if ((int)threadIdx.x < st) sh[threadIdx.x] = diag_combine(i, sh[threadIdx.x], sh[threadIdx.x + st]);
      __syncthreads();
    }
    if (threadIdx.x == 0) out[i] = (i == 3) ? sqrt(sh[0]) : sh[0];
    __syncthreads();
  }
}

}  // namespace lbm
