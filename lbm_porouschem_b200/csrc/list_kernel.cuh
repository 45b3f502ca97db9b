// list_kernel.cuh -- cell-list form of the bulk lattice update.
//
// A porous lattice is mostly solid or mostly fluid in long runs, and fluid and
// solid cells do very different amounts of work (19 + 7 populations against 7
// plus the reaction).  The tile kernel (step_bulk<>) sorts each x-run of cells
// into fluid-first order, but a block still holds both kinds, its solid warps
// finish early and their slots idle until the block retires, and the sort costs
// a dependent mask load and two block barriers per tile.
//
// Here the cells are listed once, when the lattice is initialised, in four
// segments, each padded to a multiple of 32 entries so that a warp never mixes
// them:
//   [fluid interior | fluid general | (room for cells that turn fluid)]
//   [solid interior | solid general]
// "interior" cells are away from every periodic edge (neighbours are plain index
// offsets); "general" cells wrap.  An entry is the cell index and a bit word:
// bit k (1..Q-1) set if c + e_k is solid, bit 24 reactive, bit 31 dead.  Cells on
// active (NEE) sides are not listed: step_boundary<> updates them.  Without a
// temperature field solid cells have no work and are not listed either.
//
// step_list<> is a persistent kernel: each warp walks chunks of 32 entries
// (fluid and solid chunks interleaved in proportion, strided over all warps so
// that every block gets the same mix), loading the next chunk's entry while it
// updates the current one.  The per-cell arithmetic is cell_update<>, shared with the tile
// kernel, so both forms give the same fields bit for bit.
//
// A cell that turns fluid (flip_cells<>) marks its solid entry dead, appends a
// fluid entry at the end of the fluid list (general segment) and clears the bit
// that points at it in the entries of its neighbours.
#pragma once
#include "step_kernels.cuh"

namespace lbm {

constexpr int kListChunk = 2048;  // cells per block of the list build

// Which list segment cell c belongs to: 0 fluid interior, 1 fluid general,
// 2 solid interior, 3 solid general, 4 none.
template <class L>
__device__ __forceinline__ int list_class(const uint8_t* mask, int c, int nx, int ny, int nz, int active,
                                          int par, bool thermal) {
  const int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
  const bool side = ((active & 1) && x == 0) || ((active & 2) && x == nx - 1) || ((active & 4) && y == 0) ||
                    ((active & 8) && y == ny - 1) || ((active & 16) && z == 0) || ((active & 32) && z == nz - 1);
  if (side) return 4;
  const bool solid = (mask[c] >> par) & 1;
  if (solid && !thermal) return 4;
  bool edge = x == 0 || x == nx - 1 || y == 0 || y == ny - 1;
  if (L::DIM == 3) edge = edge || z == 0 || z == nz - 1;
  return (solid ? 2 : 0) + (edge ? 1 : 0);
}

// Entry bit word of cell c at mask parity par.
template <class L>
__device__ __forceinline__ uint32_t list_bits(const uint8_t* mask, int c, int nx, int ny, int nz, int par) {
  const int x = c % nx, y = (c / nx) % ny, z = c / (nx * ny);
  const Nbhd nb(x, y, z, nx, ny, nz);
  uint32_t b = 0;
  static_for<L::Q>([&](auto kk) {
    constexpr int k = decltype(kk)::value;
    if constexpr (k > 0) b |= (uint32_t)((mask[nb.at(L::ex(k), L::ey(k), L::ez(k))] >> par) & 1) << k;
  });
  if (mask[c] & LBM_MASK_REACTIVE) b |= kEntReactive;
  return b;
}

struct ListBuild {
  const uint8_t* mask;
  int nx, ny, nz, active, par;
  int thermal;
  size_t N;
  int nbb;          // build blocks (kListChunk cells each)
  int* blk;         // [4][nbb] counts, then offsets
  int* hdr;
  uint32_t* ent_c;
  uint32_t* ent_b;
  int* pos;
  int solid_base;
};

template <class L>
__global__ void __launch_bounds__(256) list_count(const __grid_constant__ ListBuild a) {
  __shared__ int sc[4];
  if (threadIdx.x < 4) sc[threadIdx.x] = 0;
  __syncthreads();
  int cnt[4] = {0, 0, 0, 0};
  const size_t c0 = (size_t)blockIdx.x * kListChunk;
  for (int r = 0; r < kListChunk / 256; ++r) {
    const size_t c = c0 + (size_t)r * 256 + threadIdx.x;
    if (c < a.N) {
      const int k = list_class<L>(a.mask, (int)c, a.nx, a.ny, a.nz, a.active, a.par, a.thermal != 0);
      if (k < 4) ++cnt[k];
    }
  }
  for (int k = 0; k < 4; ++k) {
    int v = cnt[k];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sc[k], v);
  }
  __syncthreads();
  if (threadIdx.x < 4) a.blk[threadIdx.x * a.nbb + blockIdx.x] = sc[threadIdx.x];
}

// Exclusive block-wide scan of one int per thread (blockDim.x = 1024).
__device__ __forceinline__ int block_scan_1024(int v, int& total) {
  __shared__ int ws[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) ws[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int s = ws[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    ws[lane] = s;
  }
  __syncthreads();
  total = ws[31];
  const int before = warp > 0 ? ws[warp - 1] : 0;
  __syncthreads();
  return before + x - v;
}

// One block of 1024 threads: block offsets of every class and the list header.
template <class L>
__global__ void __launch_bounds__(1024) list_scan(const __grid_constant__ ListBuild a) {
  __shared__ int totals[4];
  for (int k = 0; k < 4; ++k) {
    int run = 0;
    for (int b0 = 0; b0 < a.nbb; b0 += 1024) {
      const int b = b0 + (int)threadIdx.x;
      const int v = b < a.nbb ? a.blk[k * a.nbb + b] : 0;
      int tot;
      const int ex = block_scan_1024(v, tot);
      if (b < a.nbb) a.blk[k * a.nbb + b] = run + ex;
      run += tot;
    }
    if (threadIdx.x == 0) totals[k] = run;
    __syncthreads();
  }
  const int fg = (totals[0] + 31) / 32 * 32;
  const int sb = a.solid_base;
  const int sg = sb + (totals[2] + 31) / 32 * 32;
  const int base[4] = {0, fg, sb, sg};
  for (int k = 1; k < 4; ++k)
    for (int b = threadIdx.x; b < a.nbb; b += 1024) a.blk[k * a.nbb + b] += base[k];
  if (threadIdx.x == 0) {
    for (int i = 0; i < kLhSlots; ++i) a.hdr[i] = 0;
    a.hdr[kLhFi] = totals[0];
    a.hdr[kLhFg] = fg;
    a.hdr[kLhFe] = fg + totals[1];
    a.hdr[kLhSb] = sb;
    a.hdr[kLhSi] = sb + totals[2];
    a.hdr[kLhSg] = sg;
    a.hdr[kLhSe] = sg + totals[3];
  }
}

// Entries in cell order within each class (deterministic).
template <class L>
__global__ void __launch_bounds__(256) list_scatter(const __grid_constant__ ListBuild a) {
  __shared__ int run[4];
  __shared__ int wc[4][8];
  if (threadIdx.x < 4) run[threadIdx.x] = a.blk[threadIdx.x * a.nbb + blockIdx.x];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t c0 = (size_t)blockIdx.x * kListChunk;
  for (int r = 0; r < kListChunk / 256; ++r) {
    const size_t c = c0 + (size_t)r * 256 + threadIdx.x;
    const int k = c < a.N ? list_class<L>(a.mask, (int)c, a.nx, a.ny, a.nz, a.active, a.par, a.thermal != 0) : 4;
    unsigned bal[4];
    for (int q = 0; q < 4; ++q) bal[q] = __ballot_sync(0xffffffffu, k == q);
    __syncthreads();  // run[] from the previous round is final
    if (lane == 0)
      for (int q = 0; q < 4; ++q) wc[q][warp] = __popc(bal[q]);
    __syncthreads();
    if (k < 4) {
      int off = run[k];
      for (int w = 0; w < warp; ++w) off += wc[k][w];
      off += __popc(bal[k] & ((1u << lane) - 1u));
      a.ent_c[off] = (uint32_t)c;
      a.ent_b[off] = list_bits<L>(a.mask, (int)c, a.nx, a.ny, a.nz, a.par);
      a.pos[c] = off;
    }
    __syncthreads();
    if (threadIdx.x < 4) {
      int t = 0;
      for (int w = 0; w < 8; ++w) t += wc[threadIdx.x][w];
      run[threadIdx.x] += t;
    }
  }
}

// ---------------------------------------------------------------- step_list
// Thread-private asynchronous copies (cp.async, 4 or 8 bytes) of the next
// chunk's pulled populations into shared memory.  A thread reads back only the
// copies it issued itself, so cp.async.wait_group is the only synchronisation.
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
// Copies `bytes` (0 or 4) of a 4-byte element and zero-fills the rest.
__device__ __forceinline__ void cp_async4_zfill(void* smem, const void* gmem, unsigned bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async8_zfill(void* smem, const void* gmem, unsigned bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// FP32 and FP64 populations can be staged; FP16 elements (2 bytes) are below the
// smallest asynchronous copy and are pulled from HBM directly.
template <class S> struct Staged { static constexpr bool value = !std::is_same<S, __half>::value; };
template <class L, class S> struct ListStaged { static constexpr bool value = L::DIM == 2 && Staged<S>::value; };

// Post-stream populations from this thread's staging slots: element k of a
// stage sits at base[k * stride] (stride = threads per block, so that the
// threads of a warp read consecutive words).  Per stage and thread: f[Q] | g[QT] |
// rel[Q] (gas release of the solid neighbour c - e_k, zero where that neighbour
// is fluid) | alpha (reactive fraction of a solid cell).  The copies take the
// bounce-back slots (the cell's own slot of the opposite direction) where the link
// needs them, so the staged values are the post-stream populations themselves.
template <class L, class S>
struct StagedPull {
  using C = typename Store<S>::C;
  const S* sf;
  int stride;
  static constexpr int kG = L::Q, kR = L::Q + L::QT, kA = 2 * L::Q + L::QT, kElems = 2 * L::Q + L::QT + 1;
  template <bool PYRO>
  __device__ __forceinline__ void flow(const StepParams<S>&, const Nbhd&, int, uint32_t nbits, C F[L::Q]) const {
    static_for<L::Q>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      C v = (C)sf[k * stride];
      if constexpr (PYRO && k > 0) {
        if ((nbits >> L::opp(k)) & 1) v += (C)sf[(kR + k) * stride] * (C)L::w(k);
      }
      F[k] = v;
    });
  }
  // the copies already resolved the adiabatic links of the two-field mode
  template <bool ADIA, bool RT>
  __device__ __forceinline__ void thermal(const StepParams<S>&, const Nbhd&, int, uint32_t, bool, C G[L::QT]) const {
    static_for<L::QT>([&](auto kk) {
      constexpr int k = decltype(kk)::value;
      G[k] = (C)sf[(kG + k) * stride];
    });
  }
  __device__ __forceinline__ C alpha(const StepParams<S>&, int) const { return (C)sf[kA * stride]; }
};

// Chunk j of the walk: fluid and solid chunks interleaved in proportion
// (Bresenham), so that both kinds of cell of a region are updated at about the
// same time and the sectors they share are moved once.  With q, r the quotient
// and remainder of j * cf / total, chunk j is fluid chunk q if r + cf >= total,
// else solid chunk j - q.  A warp visits j, j + nw, j + 2 nw, ..., so q and r
// advance by constant steps and no division is needed after the first.
struct ChunkCursor {
  int j, q, r;          // chunk, quotient, remainder
  int cf, total, sb;
  int dq, dr, step;     // (step * cf) = dq * total + dr
  __device__ __forceinline__ void init(int j0, int nw, int cf_, int total_, int sb_) {
    j = j0; cf = cf_; total = total_; sb = sb_; step = nw;
    const long long a = (long long)j0 * cf_, d = (long long)nw * cf_;
    q = total_ > 0 ? (int)(a / total_) : 0;
    r = total_ > 0 ? (int)(a - (long long)q * total_) : 0;
    dq = total_ > 0 ? (int)(d / total_) : 0;
    dr = total_ > 0 ? (int)(d - (long long)dq * total_) : 0;
  }
  // first entry of the chunk, bit 31 set for a fluid chunk
  __device__ __forceinline__ uint32_t mapped() const {
    const bool fluid = r + cf >= total;
    return fluid ? ((uint32_t)(q << 5) | 0x80000000u) : (uint32_t)(sb + ((j - q) << 5));
  }
  __device__ __forceinline__ void next() {
    j += step; q += dq; r += dr;
    if (r >= total) { r -= total; ++q; }
  }
};

// Persistent bulk update over the cell lists; 128 threads per block, dynamic
// shared memory list_smem_bytes<>().  MODE 0: an ordinary step; 1: a step that
// also writes diagnostics / macro fields; 2: a peek pass (recompute the outputs
// of the last pass).  Each mode carries only the code it runs.  The pulls are
// staged in shared memory in 2D; in 3D direct loads measured faster (D3Q19 +
// D3Q7 + pyrolysis at 256^3: 11.2 against 9.6 GLUPS in FP32).
template <class L, class S, int COLL, int THERM, int MODE>
__global__ void __maxnreg__(BulkRegs<S>::v) step_list(const __grid_constant__ StepParams<S> p) {
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  // the two fields with porous cells (THERM 4) pull directly
  constexpr bool STAGE = ListStaged<L, S>::value && THERM != 4;
  using SP = StagedPull<L, S>;
  extern __shared__ __align__(16) unsigned char list_smem[];
  // modes 1 and 2 run only with an output flag set (lbm_step, lbm_compute_macro)
  constexpr bool diag = MODE >= 1;
  constexpr bool peek = MODE == 2;
  using C = typename Store<S>::C;
  // per-thread diagnostics live in shared memory between cells (MODE >= 1), so
  // that no accumulator occupies registers through the loop
  __shared__ DiagSmem<C, MODE >= 1 ? 128 : 1> s_acc;
  if (diag) s_acc.clear(threadIdx.x);
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int fg = p.lhdr[kLhFg], fe = p.lhdr[kLhFe];
  const int sb = p.lhdr[kLhSb], sg = p.lhdr[kLhSg], se = p.lhdr[kLhSe];
  const int cf = (fe + 31) >> 5, cs = (se - sb + 31) >> 5;
  const int total = cf + cs;
  ChunkCursor cur;
  cur.init(gw, nw, cf, total, sb);
  const int np = p.par ^ 1;
  const int pl = p.nx * p.ny;
  const int stride = blockDim.x;
  S* stage0 = reinterpret_cast<S*>(list_smem) + threadIdx.x;
  const int stage_elems = SP::kElems * stride;

  // entry of the cursor's chunk for this lane (padding beyond the list ends), then
  // advance the cursor
  auto fetch = [&](uint32_t& ec, uint32_t& eb, uint32_t& mb) {
    ec = kEntPad;
    eb = kEntDead;
    mb = 0;
    if (cur.j < total) {
      mb = cur.mapped();
      const bool fl = (mb >> 31) != 0;
      const int i = (int)(mb & 0x7fffffffu) + lane;
      if (i < (fl ? fe : se)) { ec = p.ent_c[i]; eb = p.ent_b[i]; }
    }
    cur.next();
  };
  auto nbhd = [&](int c, bool interior) {
    if (interior) return Nbhd::interior(c, p.nx, pl);
    return Nbhd(c % p.nx, (c / p.nx) % p.ny, c / pl, p.nx, p.ny, p.nz);
  };
  // copies of chunk j's pulled populations into stage st
  auto issue = [&](uint32_t ec, uint32_t eb, uint32_t mb, int st) {
    if constexpr (STAGE) {
      if (ec != kEntPad && (peek || !(eb & kEntDead))) {
        const bool fl = (mb >> 31) != 0;
        const int base = (int)(mb & 0x7fffffffu);
        const int c = (int)ec;
        const Nbhd nb = nbhd(c, base < (fl ? fg : sg));
        S* sf = stage0 + st * stage_elems;
        // neighbour-solid bits of the pass being run: the entry's, or for a peek pass
        // (which recomputes the last pass before flip_cells<> updated the entries) the
        // mask's at that parity
        const uint32_t bits = peek ? Kern<L, S>::neighbour_bits(p, nb, p.par) : (eb & ~(kEntReactive | kEntDead));
        if (fl) {
          static_for<Q>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            const int src = k == 0 ? c : nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
            const bool bb = k > 0 && ((bits >> L::opp(k)) & 1);
            const S* g = bb ? p.fA + (size_t)L::opp(k) * p.N + c : p.fA + (size_t)k * p.N + src;
            if constexpr (sizeof(S) == 8) cp_async8(sf + k * stride, g); else cp_async4(sf + k * stride, g);
            if constexpr (PYRO && k > 0) {
              // gas released by a solid neighbour c - e_k (zero where it is fluid)
              const unsigned nbytes = bb ? (unsigned)sizeof(S) : 0u;
              const S* r = (const S*)p.relA + src;
              if constexpr (sizeof(S) == 8) cp_async8_zfill(sf + (SP::kR + k) * stride, r, nbytes);
              else cp_async4_zfill(sf + (SP::kR + k) * stride, r, nbytes);
            }
          });
        } else if constexpr (PYRO) {
          if (eb & kEntReactive) {
            const S* a = (const S*)p.alpha + c;
            if constexpr (sizeof(S) == 8) cp_async8(sf + SP::kA * stride, a); else cp_async4(sf + SP::kA * stride, a);
          }
        }
        if constexpr (THERMAL) {
          S* sgp = sf + SP::kG * stride;
          const bool adia = THERM == 3 || p.adiabatic;  // two-field: links across phases bounce
          static_for<QT>([&](auto kk) {
            constexpr int k = decltype(kk)::value;
            const int src = k == 0 ? c : nb.at(-L::ex(k), -L::ey(k), -L::ez(k));
            const bool bb = k > 0 && adia && ((bits >> L::opp(k)) & 1) != (uint32_t)!fl;
            const S* g = bb ? p.gA + (size_t)L::opp(k) * p.N + c : p.gA + (size_t)k * p.N + src;
            if constexpr (sizeof(S) == 8) cp_async8(sgp + k * stride, g); else cp_async4(sgp + k * stride, g);
          });
        }
      }
      cp_async_commit();
    }
  };

  uint32_t ec0, eb0, mb0, ec1, eb1, mb1;
  fetch(ec0, eb0, mb0);
  fetch(ec1, eb1, mb1);
  issue(ec0, eb0, mb0, 0);
  int st = 0;
  for (int j = gw; j < total; j += nw) {
    issue(ec1, eb1, mb1, st ^ 1);  // next chunk's populations, in flight while this one is updated
    uint32_t ec2, eb2, mb2;
    fetch(ec2, eb2, mb2);
    if constexpr (STAGE) cp_async_wait_prev();
    const bool fluid_chunk = (mb0 >> 31) != 0;
    const int base = (int)(mb0 & 0x7fffffffu);
    const bool interior = base < (fluid_chunk ? fg : sg);  // uniform per chunk
    bool act = ec0 != kEntPad;
    uint8_t mk = 0;
    const int c = (int)ec0;
    if (act) {
      if (peek) {
        // recomputing the last pass: classify by the mask at that parity, so a
        // cell that turned fluid on it reports through its (dead) solid entry
        mk = p.mask[c];
        act = fluid_chunk ? !((mk >> p.par) & 1) : ((mk >> p.par) & 1);
      } else if (eb0 & kEntDead) {
        act = false;
      }
    }
    if (act) {
      const Nbhd nb = nbhd(c, interior);
      const bool solid = !fluid_chunk;
      // a peek pass recomputes the last pass as it ran, before flip_cells<> updated
      // the entries: its neighbour bits come from the mask at that parity
      const uint32_t nbits = peek ? Kern<L, S>::neighbour_bits(p, nb, p.par) : (eb0 & ~(kEntReactive | kEntDead));
      const bool reactive = (eb0 & kEntReactive) != 0;
      bool solid_next;
      DiagAcc<C> cacc;  // this cell's contribution
      if (diag) cacc.clear();
      if constexpr (STAGE) {
        const SP src{stage0 + st * stage_elems, stride};
        solid_next = cell_update<L, S, COLL, THERM>(p, cacc, diag, peek, c, nb, nbits, solid, reactive, mk, src);
      } else {
        // the ordinary step takes pull_thermal<>'s run-time form (fewer spills)
        solid_next = cell_update<L, S, COLL, THERM, GlobalPull<L, S>, MODE == 0>(p, cacc, diag, peek, c, nb, nbits,
                                                                                 solid, reactive, mk);
      }
      if (diag) s_acc.merge(threadIdx.x, cacc);
      if (!peek) {
        if (solid && !solid_next) {
          // turns fluid: clear the solid bit of the next parity, list it for flip_cells<>
          const uint8_t m = p.mask[c];
          p.mask[c] = (uint8_t)(m & ~(1u << np));
          const int fi = atomicAdd(&p.lhdr[kLhFlip0 + p.par], 1);
          p.flips[(size_t)p.par * p.N + fi] = c;
        } else if (!solid && !interior) {
          // a cell that turned fluid on the last pass still has its old solid bit
          const uint8_t m = p.mask[c];
          if ((m >> np) & 1) p.mask[c] = (uint8_t)(m & ~(1u << np));
        }
      }
    }
    ec0 = ec1; eb0 = eb1; mb0 = mb1;
    ec1 = ec2; eb1 = eb2; mb1 = mb2;
    st ^= 1;
  }
  if constexpr (STAGE) cp_async_wait_all();
  if (diag) {
    const DiagAcc<C> acc = s_acc.load(threadIdx.x);
    block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blockIdx.x), (size_t)p.partial_rows);
  }
}

// Dynamic shared memory of step_list<> per block of `threads` (two stages).
template <class L, class S, int THERM>
constexpr size_t list_smem_bytes(int threads) {
  return ListStaged<L, S>::value && THERM != 4 ? (size_t)2 * StagedPull<L, S>::kElems * threads * sizeof(S) : 0;
}

}  // namespace lbm
