// staged_kernel.cuh -- step_bulk with shared-memory staging of the source rows.
//
// Same per-cell update as step_bulk<> (step_kernels.cuh), but the inputs of a
// tile of TILE consecutive x cells -- for every population k the source row
// (y - ey_k, z - ez_k) of plane k with its x halo, and the 3x3 (3D) or 1x3 (2D)
// neighbourhood rows of the mask -- are brought into shared memory by 1-D bulk
// asynchronous copies (cp.async.bulk, completion counted on an mbarrier), one
// copy per thread, STAGES tiles ahead.  A persistent grid walks the
// tiles; while the block computes tile j from shared memory the copies of tiles
// j+1 .. j+STAGES-1 are in flight, so the memory latency is hidden without
// holding the loads in registers.  Results go straight from registers to the
// output buffer (mirror stores as in step_bulk).
//
// Requires nx % TILE == 0 (every row start and halo piece is 16-byte aligned);
// other shapes use step_bulk.  Every mbarrier wait is bounded: on timeout the
// block records an error in p.err, drains its outstanding copies (also bounded)
// and stops.
#pragma once
#include "step_kernels.cuh"

namespace lbm {

constexpr int kStagedTile = 128;
constexpr int kStagedStages = 3;
constexpr unsigned kWaitSpins = 1u << 22;  // ~ seconds with the suspend hint

template <class L, class S, int TILE>
struct StagedLayout {
  static constexpr int HALO = 16 / (int)sizeof(S);        // elements per 16-byte halo piece
  static constexpr int ROWF = TILE + 2 * HALO;            // elements per staged population row
  static constexpr int NZR = L::DIM == 3 ? 3 : 1;          // mask rows along z
  static constexpr int NMASK = 3 * NZR;                    // mask rows staged
  static constexpr int ROWM = TILE + 32;                   // bytes per mask row (16-byte halos)
  static constexpr size_t POP_BYTES = (size_t)(L::Q + L::QT) * ROWF * sizeof(S);
  static constexpr size_t STAGE_BYTES = (POP_BYTES + (size_t)NMASK * ROWM + 127) / 128 * 128;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, 1000;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
// 1-D bulk copy global -> shared, completion counted on `bar` (no multicast).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

template <class L, class S, int TILE, bool THERMAL>
struct StagedTile {
  using LY = StagedLayout<L, S, TILE>;
  static constexpr int Q = L::Q, QT = THERMAL ? L::QT : 0;
  // copies per tile: one main piece per staged row, one halo piece per row with ex != 0,
  // three pieces per mask row
  __host__ __device__ static constexpr int halos(int n) {
    int h = 0;
    for (int k = 0; k < n; ++k) h += L::ex(k) != 0;
    return h;
  }
  static constexpr int NHF = halos(L::Q), NHG = THERMAL ? halos(L::QT) : 0;
  static constexpr int NCOPY = Q + NHF + QT + NHG + 3 * LY::NMASK;

  // tile index -> (x0, y, z)
  __device__ __forceinline__ static void coords(const StepParams<S>& p, int t, int& x0, int& y, int& z) {
    const int nxb = p.nx / TILE;
    x0 = (t % nxb) * TILE;
    y = (t / nxb) % p.ny;
    z = t / (nxb * p.ny);
  }
  // Bytes one tile brings in (the mbarrier's expected transaction count).
  __host__ __device__ static constexpr unsigned tile_bytes() {
    unsigned b = 0;
    for (int k = 0; k < L::Q; ++k) b += (unsigned)((L::ex(k) == 0 ? TILE : TILE + LY::HALO) * sizeof(S));
    if (THERMAL)
      for (int k = 0; k < L::QT; ++k) b += (unsigned)((L::ex(k) == 0 ? TILE : TILE + LY::HALO) * sizeof(S));
    return b + (unsigned)(LY::NMASK * (TILE + 32));
  }
  // direction of the n-th row with ex != 0 among the first `rows` directions
  __device__ __forceinline__ static int nth_halo_dir(int n, int rows) {
    int k = 0, seen = -1;
    bool found = false;
    static_for<L::Q>([&](auto qq) {
      constexpr int q = decltype(qq)::value;
      if (!found && q < rows) {
        if constexpr (L::ex(q) != 0) ++seen;
        if (seen == n) { k = q; found = true; }
      }
    });
    return k;
  }
  __device__ __forceinline__ static void dir(int k, int& ex, int& ey, int& ez) {
    ex = ey = ez = 0;
    static_for<L::Q>([&](auto kk) {
      constexpr int q = decltype(kk)::value;
      if (q == k) { ex = L::ex(q); ey = L::ey(q); ez = L::ez(q); }
    });
  }
  // Issue copy `ci` (0 <= ci < NCOPY) of tile t into stage buffer `st`.
  // Staged population row j holds x = x0 - HALO + j; mask row byte j holds x = x0 - 16 + j.
  __device__ __forceinline__ static void issue_one(const StepParams<S>& p, int t, int ci, unsigned char* st,
                                                   uint64_t* bar) {
    constexpr int H = LY::HALO;
    int x0, y, z;
    coords(p, t, x0, y, z);
    const size_t plane = (size_t)p.nx * p.ny;
    if (ci < Q + NHF + QT + NHG) {
      const bool is_g = ci >= Q + NHF;
      const int c2 = is_g ? ci - (Q + NHF) : ci;
      const int nrow = is_g ? QT : Q;
      const bool halo = c2 >= nrow;
      const int k = halo ? nth_halo_dir(c2 - nrow, nrow) : c2;
      int ex, ey, ez;
      dir(k, ex, ey, ez);
      const S* pl = (is_g ? p.gA : p.fA) + (size_t)k * p.N;
      const size_t ro = (size_t)wrapi(y - ey, p.ny) * p.nx + (size_t)wrapi(z - ez, p.nz) * plane;
      S* row = (S*)st + (size_t)((is_g ? Q : 0) + k) * LY::ROWF;
      if (!halo) {
        bulk_g2s(row + H, pl + ro + x0, TILE * sizeof(S), bar);
      } else if (ex == 1) {  // left halo [x0-H, x0), wrapped
        bulk_g2s(row, pl + ro + (x0 == 0 ? p.nx - H : x0 - H), H * sizeof(S), bar);
      } else {  // right halo [x0+TILE, x0+TILE+H), wrapped
        bulk_g2s(row + H + TILE, pl + ro + (x0 + TILE == p.nx ? 0 : x0 + TILE), H * sizeof(S), bar);
      }
    } else {
      const int m = ci - (Q + NHF + QT + NHG);
      const int r = m / 3, piece = m % 3;
      const int dy = r % 3 - 1, dz = LY::NZR == 3 ? r / 3 - 1 : 0;
      const size_t ro = (size_t)wrapi(y + dy, p.ny) * p.nx + (size_t)wrapi(z + dz, p.nz) * plane;
      unsigned char* d = st + LY::POP_BYTES + (size_t)r * LY::ROWM;
      if (piece == 0) bulk_g2s(d, p.mask + ro + (x0 == 0 ? p.nx - 16 : x0 - 16), 16, bar);
      else if (piece == 1) bulk_g2s(d + 16, p.mask + ro + x0, TILE, bar);
      else bulk_g2s(d + 16 + TILE, p.mask + ro + (x0 + TILE == p.nx ? 0 : x0 + TILE), 16, bar);
    }
  }
};

// Bounded wait on a stage barrier; false on timeout.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase) {
  for (unsigned it = 0; it < kWaitSpins; ++it)
    if (mbar_try_wait(bar, phase)) return true;
  return false;
}

template <class L, class S, int COLL, int THERM, int TILE, int STAGES>
__global__ void __launch_bounds__(TILE, (std::is_same<S, double>::value ? 1 : 4))
    step_bulk_staged(const __grid_constant__ StepParams<S> p) {
  using K = Kern<L, S>;
  using C = typename Store<S>::C;
  using LY = StagedLayout<L, S, TILE>;
  using TL = StagedTile<L, S, TILE, (THERM >= 1)>;
  constexpr int Q = L::Q, QT = L::QT;
  constexpr bool THERMAL = THERM >= 1, PYRO = THERM == 2;
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ uint64_t bars[STAGES];
  __shared__ uint8_t s_rank_cell[TILE];
  __shared__ int s_count[2][TILE / 32];
  __shared__ int s_abort;

  const bool diag = (p.flags & (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) != 0;
  const bool peek = (p.flags & kStepPeek) != 0;
  DiagAcc<typename Store<S>::C> acc;
  if (diag) acc.clear();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ntiles = (p.nx / TILE) * p.ny * p.nz;
  const int nmine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  static_assert(TL::NCOPY <= TILE, "one copy per thread");
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) mbar_init(&bars[s], 1);
    fence_mbar_init();
    s_abort = 0;
    // arm the barriers of the first STAGES tiles
    for (int j = 0; j < STAGES && j < nmine; ++j) mbar_expect_tx(&bars[j], TL::tile_bytes());
  }
  __syncthreads();
  if ((int)threadIdx.x < TL::NCOPY)
    for (int j = 0; j < STAGES && j < nmine; ++j)
      TL::issue_one(p, blockIdx.x + j * gridDim.x, threadIdx.x, smem + (size_t)j * LY::STAGE_BYTES, &bars[j]);

  int done = 0;  // tiles whose copies completed and were consumed
  for (int j = 0; j < nmine; ++j) {
    const int st = j % STAGES;
    const unsigned phase = (unsigned)((j / STAGES) & 1);
    if (!mbar_wait_bounded(&bars[st], phase)) atomicExch(&s_abort, 1);
    __syncthreads();
    if (s_abort) break;
    ++done;
    // this stage's next use is tile j + STAGES: arm its barrier now (its copies
    // are issued after every thread has finished reading tile j)
    if (threadIdx.x == 0 && j + STAGES < nmine) mbar_expect_tx(&bars[st], TL::tile_bytes());

    const unsigned char* sb = smem + (size_t)st * LY::STAGE_BYTES;
    const S* fs = (const S*)sb;
    const S* gs = fs + (size_t)Q * LY::ROWF;
    const unsigned char* ms = sb + LY::POP_BYTES;
    const unsigned char* mrow0 = ms + (size_t)(LY::NZR == 3 ? 4 : 1) * LY::ROWM;  // (dy, dz) = (0, 0)
    int x0, y, z;
    TL::coords(p, blockIdx.x + j * gridDim.x, x0, y, z);

    // per-tile fluid-first ordering (as in step_bulk)
    int i, cell_kind;
    {
      const int it = threadIdx.x;
      const int xt = x0 + it;
      const bool ok = !K::on_active_side(p, xt, y, z);
      const uint8_t mt = mrow0[16 + it];
      const int kind = !ok ? 2 : (((mt >> p.par) & 1) ? 1 : 0);
      const unsigned bf = __ballot_sync(0xffffffffu, kind == 0), bs = __ballot_sync(0xffffffffu, kind == 1);
      if (lane == 0) { s_count[0][warp] = __popc(bf); s_count[1][warp] = __popc(bs); }
      __syncthreads();
      int nf = 0, ns = 0, pf = 0, ps = 0, pk_ = 0;
      for (int w = 0; w < TILE / 32; ++w) {
        if (w < warp) { pf += s_count[0][w]; ps += s_count[1][w]; pk_ += 32 - s_count[0][w] - s_count[1][w]; }
        nf += s_count[0][w]; ns += s_count[1][w];
      }
      const unsigned lt = (1u << lane) - 1u;
      int rank;
      if (kind == 0) rank = pf + __popc(bf & lt);
      else if (kind == 1) rank = nf + ps + __popc(bs & lt);
      else rank = nf + ns + pk_ + __popc(~(bf | bs) & lt);
      s_rank_cell[rank] = (uint8_t)it;
      __syncthreads();
      i = s_rank_cell[threadIdx.x];
      cell_kind = (int)threadIdx.x < nf ? 0 : ((int)threadIdx.x < nf + ns ? 1 : 2);
    }

    if (cell_kind != 2) {
      const int x = x0 + i;
      const int c = x + p.nx * (y + p.ny * z);
      const Nbhd nb(x, y, z, p.nx, p.ny, p.nz);
      const uint8_t mk = mrow0[16 + i];
      const bool solid = cell_kind == 1;
      // neighbour solidity bits from the staged mask rows
      uint32_t nbits = 0;
      static_for<Q>([&](auto kk) {
        constexpr int k = decltype(kk)::value;
        if constexpr (k > 0) {
          constexpr int r = (L::ey(k) + 1) + 3 * (LY::NZR == 3 ? L::ez(k) + 1 : 0);
          nbits |= (uint32_t)((ms[(size_t)r * LY::ROWM + 16 + i + L::ex(k)] >> p.par) & 1) << k;
        }
      });
      C G[QT > 0 ? QT : 1];
      C T = 0, dS = 0, rho = 0, ux = 0, uy = 0, uz = 0;
      if constexpr (THERMAL) {
        static_for<QT>([&](auto kk) {
          constexpr int k = decltype(kk)::value;
          G[k] = Store<S>::ld(gs, (size_t)k * LY::ROWF + LY::HALO + i - L::ex(k), gshift<L, S, k>(p));
          T += G[k];
        });
      }
      bool solid_next = solid;
      bool flipping = false;
      if (!solid) {
        C F[Q];
        static_for<Q>([&](auto kk) {
          constexpr int k = decltype(kk)::value;
          C v = Store<S>::ld(fs, (size_t)k * LY::ROWF + LY::HALO + i - L::ex(k), fshift<L, S, k>(p));
          if constexpr (PYRO && k > 0) {
            if ((nbits >> L::opp(k)) & 1) v += p.relA[nb.at(-L::ex(k), -L::ey(k), -L::ez(k))] * (C)L::w(k);
          }
          F[k] = v;
        });
        K::moments(p, F, rho, ux, uy, uz);
        if (diag) diag_flow(p, acc, c, rho, ux, uy, uz);
        if (!peek) {
          K::template collide_flow<COLL>(p, F, rho, ux, uy, uz, T);
          K::store_flow(p, nb, c, nbits, F);
        }
      } else if constexpr (PYRO) {
        if (mk & LBM_MASK_REACTIVE) {
          if (peek) {
            if (!((mk >> (p.par ^ 1)) & 1)) solid_next = false;
          } else {
            const C a = p.alpha[c];
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
          K::collide_thermal(p, G, T, fl ? p.itauT_f : p.itauT_s, fl ? ux : (C)0, fl ? uy : (C)0,
                             fl ? uz : (C)0, dS);
          K::template store_thermal<THERM == 3>(p, nb, c, G, nbits, solid);
        }
        if (diag) diag_thermal(p, acc, c, T);
      }
      if (PYRO && diag && solid_next && (mk & LBM_MASK_REACTIVE)) acc.alpha += (double)p.alpha[c];
      if (!peek) {
        const int np = p.par ^ 1;
        const uint8_t want = (uint8_t)((mk & ~(1u << np)) | ((solid_next ? 1u : 0u) << np));
        if (want != mk) p.mask[c] = want;
      }
    }
    __syncthreads();  // every thread is done with stage st: refill it with tile j + STAGES
    if ((int)threadIdx.x < TL::NCOPY && j + STAGES < nmine) {
      fence_proxy_async_smem();
      TL::issue_one(p, blockIdx.x + (j + STAGES) * gridDim.x, threadIdx.x, smem + (size_t)st * LY::STAGE_BYTES,
                    &bars[st]);
    }
  }

  if (s_abort) {
    // drain this block's copies still in flight (tiles done .. done+STAGES-1, bounded)
    for (int j = done; j < nmine && j < done + STAGES; ++j)
      mbar_wait_bounded(&bars[j % STAGES], (unsigned)((j / STAGES) & 1));
    if (threadIdx.x == 0 && p.err) atomicExch(p.err, 1);
  }
  if (diag) block_reduce_store(acc, p.partials + (size_t)(p.block_offset + blockIdx.x), (size_t)p.partial_rows);
}

}  // namespace lbm
