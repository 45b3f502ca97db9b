// dense_kernel.cuh -- 3D bulk update over dense tiles whose inputs the Tensor Memory
// Accelerator stages in shared memory (sm_100a).
//
// The lattice is cut into tiles of 32 (x) x kDTY (y) x kDTZ (z) cells.  A persistent grid
// walks the tiles; for each tile one thread issues, on an mbarrier, the TMA box loads of
// everything the tile's cells read:
//   - per flow direction k, plane k of the input half over the tile shifted by -e_k (the
//     neighbours c - e_k), extended by one layer in y / z towards the tile so that it also
//     holds the tile's own slots of that plane (halfway bounce-back reads a cell's own
//     slot of the opposite direction); x-moving directions take a box 16 bytes wider on
//     each side, since a box must start on a 16-byte boundary in x;
//   - per temperature direction, its plane over the shifted tile;
//   - the mask bytes, and with pyrolysis the gas release of the input half, over the tile
//     and its one-cell halo; the reactive fractions of the tile.
// Boxes of the next tile are in flight while the current one is updated from shared
// memory (two stages).
//
// Every input of the tile is in shared memory, so any thread can update any cell: the
// cells of a tile are ranked fluid first, then reacting solid, then inert solid (cells on
// active sides last, they belong to step_boundary<>), and warps take 32-cell slices of
// that order, so a warp runs one branch of the update instead of all of them.  The
// per-cell arithmetic is cell_update<> (the one the tile and cell-list kernels run), fed
// by DensePull.  Every cell writes all its slots: the (never read) flow slots of solid
// cells get zeros, so that with the other stores of the same tile every 32-byte sector of
// the output is written whole and none is left for the L2 to complete from DRAM.
//
// Tiles that touch a periodic domain edge (their pulls wrap around) are updated with
// global-memory pulls (GlobalPull) instead; at 256^3 with periodic y and z that is about
// 5 % of the tiles.
//
// Every mbarrier wait is bounded (p.wait_spins tries of about a microsecond each): on
// timeout the block records bit 0 in p.err, its warps stop, and one thread waits (with a
// long, fixed bound) for the copies the block issued before it ends; lbm_read_diag then
// reports LBM_ERR_TIMEOUT.
#pragma once
#include <cuda.h>

#include "step_kernels.cuh"

namespace lbm {

constexpr int kDTX = 32, kDTY = 4, kDTZ = 2, kDThreads = kDTX * kDTY * kDTZ;
constexpr unsigned kDrainSpins = 1u << 24;     // bound of the wait for copies in flight on abort
constexpr unsigned kDefaultWaitSpins = 1u << 22;

// Tensor maps of the dense kernel, built by the host over the bound buffers.  Flow
// populations as a 4-D tensor (x, y, z, plane = half * Q + k), one map per box shape
// f[wide << 2 | (ey != 0) << 1 | (ez != 0)]; temperature the same with QT (unextended
// boxes); the mask as (x, y, z) bytes; gas release as (x, y, z, half); reactive
// fraction as (x, y, z).
struct DenseMaps {
  CUtensorMap f[8];
  CUtensorMap g_wide, g_narrow, mask, rel, alpha;
};

template <class L, class S, bool THERMAL, bool PYRO>
struct DenseLayout {
  using C = typename Store<S>::C;
  static constexpr int H = 16 / (int)sizeof(S);  // x halo of a wide population box, elements
  static constexpr int BXW = kDTX + 2 * H, BXN = kDTX;
  static constexpr int HC = 16 / (int)sizeof(C);  // the same for compute-precision fields
  static constexpr int RX = kDTX + 2 * HC;
  static constexpr int MX = 64, MH = 16, MY = kDTY + 2, MZ = kDTZ + 2;  // mask / rel halo box
  static constexpr int QT = THERMAL ? L::QT : 0;
  __host__ __device__ static constexpr int iabs(int v) { return v < 0 ? -v : v; }
  __host__ __device__ static constexpr bool wide(int k) { return L::ex(k) != 0; }
  __host__ __device__ static constexpr int bx(int k) { return wide(k) ? BXW : BXN; }
  // flow box of direction k: extents and origin offset from the tile origin
  __host__ __device__ static constexpr int fby(int k) { return kDTY + iabs(L::ey(k)); }
  __host__ __device__ static constexpr int fbz(int k) { return kDTZ + iabs(L::ez(k)); }
  __host__ __device__ static constexpr int foy(int k) { return L::ey(k) > 0 ? -L::ey(k) : 0; }
  __host__ __device__ static constexpr int foz(int k) { return L::ez(k) > 0 ? -L::ez(k) : 0; }
  __host__ __device__ static constexpr int fmap(int k) {
    return (wide(k) ? 4 : 0) | (L::ey(k) != 0 ? 2 : 0) | (L::ez(k) != 0 ? 1 : 0);
  }
  __host__ __device__ static constexpr int f_bytes(int k) { return bx(k) * fby(k) * fbz(k) * (int)sizeof(S); }
  __host__ __device__ static constexpr int g_bytes(int k) { return bx(k) * kDTY * kDTZ * (int)sizeof(S); }
  __host__ __device__ static constexpr int rup(int b) { return (b + 127) / 128 * 128; }
  __host__ __device__ static constexpr int f_off(int k) {
    int o = 0;
    for (int j = 0; j < k; ++j) o += rup(f_bytes(j));
    return o;
  }
  __host__ __device__ static constexpr int g_off(int k) {
    int o = f_off(L::Q);
    for (int j = 0; j < k; ++j) o += rup(g_bytes(j));
    return o;
  }
  static constexpr int M_OFF = g_off(QT);
  static constexpr int M_BYTES = MX * MY * MZ;
  static constexpr int R_OFF = M_OFF + rup(M_BYTES);
  static constexpr int R_BYTES = PYRO ? RX * MY * MZ * (int)sizeof(C) : 0;
  static constexpr int A_OFF = R_OFF + rup(R_BYTES);
  static constexpr int A_BYTES = PYRO ? kDTX * kDTY * kDTZ * (int)sizeof(C) : 0;
  static constexpr int STAGE = A_OFF + rup(A_BYTES);
  // bytes the TMA writes per tile (a box counts whole, its out-of-bounds part too)
  __host__ __device__ static constexpr unsigned tx_bytes() {
    unsigned b = (unsigned)(M_BYTES + R_BYTES + A_BYTES);
    for (int k = 0; k < L::Q; ++k) b += (unsigned)f_bytes(k);
    for (int k = 0; k < QT; ++k) b += (unsigned)g_bytes(k);
    return b;
  }
  // element index, in flow box k, of the cell at tile position (tx, ty, tz) + (dx, dy, dz)
  __host__ __device__ static constexpr int fidx(int k, int tx, int ty, int tz, int dx, int dy, int dz) {
    return ((tz + dz - foz(k)) * fby(k) + (ty + dy - foy(k))) * bx(k) + tx + dx + (wide(k) ? H : 0);
  }
};

// CTAs per SM of step_dense: two stages of one tile each fit twice per SM in FP32 and
// FP16; FP64 (255 registers) once.
template <class S> struct DenseCTAs { static constexpr int v = 2; };
template <> struct DenseCTAs<double> { static constexpr int v = 1; };

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void dmbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void dmbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// One bounded try (the hardware may suspend the thread up to about a microsecond).
__device__ __forceinline__ bool dmbar_try_wait(uint64_t* bar, unsigned phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool dmbar_wait_bounded(uint64_t* bar, unsigned phase, unsigned spins) {
  for (unsigned i = 0; i < spins; ++i)
    if (dmbar_try_wait(bar, phase)) return true;
  return false;
}
__device__ __forceinline__ void dfence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void dfence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// TMA tile loads global -> shared, completion counted on `bar` (no multicast).
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_addr(bar))
      : "memory");
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_addr(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_addr(bar))
      : "memory");
}

// Post-stream populations of one cell of a staged tile; (tx, ty, tz): its position in
// the tile.  Everything comes from the stage in shared memory.
template <class L, class S, bool THERMAL, bool PYRO>
struct DensePull {
  using C = typename Store<S>::C;
  using LY = DenseLayout<L, S, THERMAL, PYRO>;
  const unsigned char* stage;
  int tx, ty, tz;
  template <bool PY>
  __device__ __forceinline__ void flow(const StepParams<S>& p, const Nbhd&, int, uint32_t nbits, C F[L::Q]) const {
    const S* sf = reinterpret_cast<const S*>(stage);
    static_for<L::Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      constexpr int fk = LY::f_off(k) / (int)sizeof(S);
      if constexpr (k == 0) {
        F[0] = Store<S>::ld(sf + fk, LY::fidx(0, tx, ty, tz, 0, 0, 0), fshift<L, S, 0>(p));
      } else {
        constexpr int o = L::opp(k);
        constexpr int fo = LY::f_off(o) / (int)sizeof(S);
        // c - e_k fluid: its slot of plane k; solid: the cell's own slot of plane opp(k)
        const bool bb = (nbits >> o) & 1;
        const int i = bb ? fo + LY::fidx(o, tx, ty, tz, 0, 0, 0)
                         : fk + LY::fidx(k, tx, ty, tz, -L::ex(k), -L::ey(k), -L::ez(k));
        C v = Store<S>::ld(sf, i, fshift<L, S, k>(p));
        if constexpr (PY) {
          if (bb) {
            const C* sr = reinterpret_cast<const C*>(stage + LY::R_OFF);
            v += sr[((tz + 1 - L::ez(k)) * LY::MY + ty + 1 - L::ey(k)) * LY::RX + LY::HC + tx - L::ex(k)] * (C)L::w(k);
          }
        }
        F[k] = v;
      }
    });
  }
  template <bool ADIA, bool RT>
  __device__ __forceinline__ void thermal(const StepParams<S>& p, const Nbhd&, int, uint32_t, bool, C G[L::QT]) const {
    static_assert(!ADIA, "the dense kernel runs the conjugate temperature field only");
    const S* sg = reinterpret_cast<const S*>(stage);
    static_for<L::QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      constexpr int gk = LY::g_off(k) / (int)sizeof(S);
      const int i = LY::wide(k) ? (tz * kDTY + ty) * LY::BXW + tx + LY::H - L::ex(k) : (tz * kDTY + ty) * LY::BXN + tx;
      G[k] = Store<S>::ld(sg + gk, i, gshift<L, S, k>(p));
    });
  }
  __device__ __forceinline__ C alpha(const StepParams<S>& p, int c) const {
    if constexpr (PYRO) return reinterpret_cast<const C*>(stage + LY::A_OFF)[(tz * kDTY + ty) * kDTX + tx];
    else return p.alpha[c];
  }
};

// MODE 0: ordinary step; 1: a step that also writes diagnostics / macro fields; 2: a
// peek pass (recompute the outputs of the last pass).  THERM 0, 1 or 2 (the two-field
// temperature mode runs on the other forms).
//
// Warps do not wait for one another.  Each warp, once a stage's boxes have landed, ranks
// the tile's cells itself (from the staged mask) and then takes 32-cell slices of the
// ranked tile from a shared counter until none is left, so warps that drew cheap solid
// slices take more of them.  A warp done with a tile releases its stage; the last one to
// release it issues the loads of the tile two ahead into it.  The two stages thus let a
// fast warp run up to one tile ahead of the slowest.
template <class L, class S, int COLL, int THERM, int MODE>
__global__ void __launch_bounds__(kDThreads, DenseCTAs<S>::v)
    step_dense(const __grid_constant__ StepParams<S> p, const __grid_constant__ DenseMaps maps) {
  static_assert(L::DIM == 3 && THERM != 3, "step_dense: 3D, conjugate temperature or none");
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  constexpr int Q = L::Q;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  using LY = DenseLayout<L, S, THERMAL, PYRO>;
  using DP = DensePull<L, S, THERMAL, PYRO>;
  constexpr bool diag = MODE >= 1, peek = MODE == 2;
  constexpr int NW = kDThreads / 32;
  extern __shared__ __align__(128) unsigned char dsm[];
  __shared__ __align__(8) uint64_t bar[2];
  __shared__ int s_next[2], s_done[2], s_issued[2];
  __shared__ volatile int s_abort;
  __shared__ uint8_t s_order[NW][kDThreads];  // each warp's copy of the tile's rank order
  __shared__ DiagSmem<C, MODE >= 1 ? kDThreads : 1> s_acc;
  if (diag) s_acc.clear(threadIdx.x);

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ntx = p.nx / kDTX, nty = p.ny / kDTY, ntz = p.nz / kDTZ;
  const int ntiles = ntx * nty * ntz;
  const int np = p.par ^ 1;
  const int G = (int)gridDim.x;

  auto tile_origin = [&](int t, int& x0, int& y0, int& z0) {
    x0 = (t % ntx) * kDTX;
    y0 = ((t / ntx) % nty) * kDTY;
    z0 = (t / (ntx * nty)) * kDTZ;
  };
  // one thread: the boxes of tile t into stage st (after the stage's counters are reset;
  // the arrive below releases those stores to the warps that see the phase complete)
  auto issue = [&](int t, int st) {
    int x0, y0, z0;
    tile_origin(t, x0, y0, z0);
    unsigned char* base = dsm + st * LY::STAGE;
    s_issued[st] += 1;
    dmbar_expect_tx(&bar[st], LY::tx_bytes());
    static_for<Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      tma_load_4d(base + LY::f_off(k), &maps.f[LY::fmap(k)], LY::wide(k) ? x0 - LY::H : x0, y0 + LY::foy(k),
                  z0 + LY::foz(k), p.par * Q + k, &bar[st]);
    });
    if constexpr (THERMAL) {
      static_for<L::QT>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        tma_load_4d(base + LY::g_off(k), LY::wide(k) ? &maps.g_wide : &maps.g_narrow,
                    LY::wide(k) ? x0 - LY::H : x0, y0 - L::ey(k), z0 - L::ez(k), p.par * L::QT + k, &bar[st]);
      });
    }
    tma_load_3d(base + LY::M_OFF, &maps.mask, x0 - LY::MH, y0 - 1, z0 - 1, &bar[st]);
    if constexpr (PYRO) {
      tma_load_4d(base + LY::R_OFF, &maps.rel, x0 - LY::HC, y0 - 1, z0 - 1, p.par, &bar[st]);
      tma_load_3d(base + LY::A_OFF, &maps.alpha, x0, y0, z0, &bar[st]);
    }
  };

  if (threadIdx.x == 0) {
    dmbar_init(&bar[0], 1);
    dmbar_init(&bar[1], 1);
    dfence_mbar_init();
    s_next[0] = s_next[1] = s_done[0] = s_done[1] = s_issued[0] = s_issued[1] = 0;
    s_abort = 0;
    if ((int)blockIdx.x < ntiles) issue(blockIdx.x, 0);
    if ((int)blockIdx.x + G < ntiles) issue(blockIdx.x + G, 1);
  }
  __syncthreads();

  uint8_t* order = s_order[warp];
  int it = 0;
  for (int t = blockIdx.x; t < ntiles; t += G, ++it) {
    const int st = it & 1;
    const unsigned ph = (unsigned)((it >> 1) & 1);
    // ---- wait for the stage (bounded; another warp's timeout ends this one's wait too)
    bool ok = false;
    for (unsigned i = 0; i < p.wait_spins && !s_abort; ++i)
      if (dmbar_try_wait(&bar[st], ph)) { ok = true; break; }
    ok = __all_sync(0xffffffffu, ok);
    if (!ok) {
      if (lane == 0) {
        s_abort = 1;
        if (p.err) atomicOr(p.err, 1);
      }
      break;
    }
    int x0, y0, z0;
    tile_origin(t, x0, y0, z0);
    const int a = p.active;
    // pulls of this tile wrap around a periodic edge: global-memory pulls
    const bool edge = (x0 == 0 && !(a & 1)) || (x0 + kDTX == p.nx && !(a & 2)) || (y0 == 0 && !(a & 4)) ||
                      (y0 + kDTY == p.ny && !(a & 8)) || (z0 == 0 && !(a & 16)) || (z0 + kDTZ == p.nz && !(a & 32));
    const unsigned char* sbase = dsm + st * LY::STAGE;
    const uint8_t* smask = sbase + LY::M_OFF;

    // ---- rank the tile's 256 cells: fluid, reacting solid, inert solid, skipped (cells
    // on active sides).  Lane l classifies cells 8l .. 8l+7 (one 8-byte mask load).
    {
      const int row = lane >> 2, xb = (lane & 3) * 8;  // row = ty + kDTY * tz
      const int ty = row % kDTY, tz = row / kDTY;
      const uint2 m8 = *reinterpret_cast<const uint2*>(smask + ((tz + 1) * LY::MY + ty + 1) * LY::MX + LY::MH + xb);
      unsigned long long packed = 0;  // 16-bit count per class (a tile has 256 cells)
      uint32_t cls2 = 0;              // 2-bit class per cell
      for (int e = 0; e < 8; ++e) {
        const uint32_t mk = ((e < 4 ? m8.x : m8.y) >> (8 * (e & 3))) & 0xffu;
        const bool skip = K::on_active_side(p, x0 + xb + e, y0 + ty, z0 + tz);
        const bool solid = (mk >> p.par) & 1;
        const int cls = skip ? 3 : (!solid ? 0 : ((PYRO && (mk & LBM_MASK_REACTIVE)) ? 1 : 2));
        cls2 |= (uint32_t)cls << (2 * e);
        packed += 1ull << (16 * cls);
      }
      // exclusive scan of the packed counts over the lanes, and the class totals
      unsigned long long incl = packed;
      for (int o = 1; o < 32; o <<= 1) {
        const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += v;
      }
      const unsigned long long tot = __shfl_sync(0xffffffffu, incl, 31);
      unsigned long long excl = incl - packed;
      const int t0 = (int)(tot & 0xffffu), t1 = (int)((tot >> 16) & 0xffffu), t2 = (int)((tot >> 32) & 0xffffu);
      const int cbase[4] = {0, t0, t0 + t1, t0 + t1 + t2};
      for (int e = 0; e < 8; ++e) {
        const int cls = (cls2 >> (2 * e)) & 3;
        const int r = cbase[cls] + (int)((excl >> (16 * cls)) & 0xffffu);
        excl += 1ull << (16 * cls);
        order[r] = (uint8_t)(row * 32 + xb + e);
      }
      __syncwarp();
    }

    // ---- take 32-cell slices of the ranked tile until none is left
    while (true) {
      int j = 0;
      if (lane == 0) j = atomicAdd(&s_next[st], 1);
      j = __shfl_sync(0xffffffffu, j, 0);
      if (j >= NW) break;
      const int tc = order[32 * j + lane];
      const int tx = tc & 31, ty = (tc >> 5) % kDTY, tz = (tc >> 5) / kDTY;
      const int x = x0 + tx, y = y0 + ty, z = z0 + tz;
      const int mc = ((tz + 1) * LY::MY + ty + 1) * LY::MX + LY::MH + tx;
      const uint8_t mk = smask[mc];
      if (!K::on_active_side(p, x, y, z)) {
        const int c = x + p.nx * (y + p.ny * z);
        const bool solid = (mk >> p.par) & 1;
        const bool reactive = (mk & LBM_MASK_REACTIVE) != 0;
        DiagAcc<C> cacc;
        if (diag) cacc.clear();
        bool solid_next;
        if (!edge) {
          uint32_t nbits = 0;
          static_for<Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            if constexpr (k > 0)
              nbits |= (uint32_t)((smask[mc + (L::ez(k) * LY::MY + L::ey(k)) * LY::MX + L::ex(k)] >> p.par) & 1) << k;
          });
          const DP src{sbase, tx, ty, tz};
          const Nbhd nb{};
          solid_next = cell_update<L, S, COLL, THERM, DP>(p, cacc, diag, peek, c, nb, nbits, solid, reactive, mk, src);
        } else {
          const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
          const uint32_t nbits = K::neighbour_bits(p, nb, p.par);
          solid_next = cell_update<L, S, COLL, THERM>(p, cacc, diag, peek, c, nb, nbits, solid, reactive, mk);
        }
        if (diag) s_acc.merge(threadIdx.x, cacc);
        if (!peek) {
          if (solid) {
            // the (never read) flow slots of a solid cell get zeros, so that with the rest
            // of the tile's stores every sector of the output is written whole
            static_for<Q>([&](auto kk) { p.fB[(size_t)decltype(kk)::value * p.N + c] = S{}; });
            if (!solid_next) {
              // turns fluid: clear the solid bit of the next parity, list it for flip_cells<>
              p.mask[c] = (uint8_t)(mk & ~(1u << np));
              const int fi = atomicAdd(&p.lhdr[kLhFlip0 + p.par], 1);
              p.flips[(size_t)p.par * p.N + fi] = c;
            }
          } else if ((mk >> np) & 1) {
            // a cell that turned fluid on the last pass still has its old solid bit
            p.mask[c] = (uint8_t)(mk & ~(1u << np));
          }
        }
      }
    }

    // ---- release the stage; the last warp refills it with the tile two ahead
    __syncwarp();
    if (lane == 0) {
      __threadfence_block();
      if (atomicAdd(&s_done[st], 1) == NW - 1) {
        s_done[st] = 0;
        s_next[st] = 0;
        const int t2 = t + 2 * G;
        if (t2 < ntiles && !s_abort) {
          dfence_proxy_async();
          issue(t2, st);
        }
      }
    }
  }
  __syncthreads();
  if (s_abort && threadIdx.x == 0) {
    // let every copy this block issued land before the block ends
    for (int st = 0; st < 2; ++st)
      if (s_issued[st] > 0) dmbar_wait_bounded(&bar[st], (unsigned)((s_issued[st] - 1) & 1), kDrainSpins);
  }
  if (diag) {
    const DiagAcc<C> acc = s_acc.load(threadIdx.x);
    block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blockIdx.x), (size_t)p.partial_rows);
  }
  __syncthreads();
}

}  // namespace lbm
