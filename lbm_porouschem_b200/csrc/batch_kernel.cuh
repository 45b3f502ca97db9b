// batch_kernel.cuh -- many lattices of uneven sizes in one persistent launch.
//
// A parameter sweep runs dozens of independent lattices (different geometries,
// sizes, relaxation times, boundary values).  Stepping them one launch sequence
// at a time leaves most of the GPU idle on the small ones and pays three launches
// per lattice per step.  A batch steps them all with three launches per step:
//   step_list_batch     every bulk cell of every lattice, over a chunk table of
//                       (lattice, fluid/solid, interior/general, first entry);
//   step_boundary_batch the NEE faces, over a block table (lattice, face, block);
//   flip_cells_batch    the flip lists, one grid row per lattice.
// Each lattice keeps its own buffers and cell lists; the batch adds only the
// tables and a copy of every lattice's kernel parameters for both step parities.
// The per-cell arithmetic is that of the single-lattice kernels (cell_update,
// boundary_cell, flip_one), so a batch step gives the same bits as stepping the
// lattices one by one.  A batch step issues no host synchronisation and no
// allocation, so a sequence of them can be captured in a CUDA graph.
#pragma once
#include "list_kernel.cuh"

namespace lbm {

template <class S>
struct BatchArgs {
  const StepParams<S>* params;  // [lattice][parity]
  const int2* chunks;           // x: lattice << 2 | fluid << 1 | interior, y: first entry
  int nchunks;
  const int4* bc;               // x: lattice, y: face, z: block within the face
  int nbc;
  int par;
};

// Copy one lattice's parameters into shared memory; thread t of nt copying threads.
template <class S>
__device__ __forceinline__ void copy_params(StepParams<S>& dst, const StepParams<S>& src, int t, int nt) {
  static_assert(sizeof(StepParams<S>) % 4 == 0, "parameter block is copied in words");
  constexpr int W = (int)(sizeof(StepParams<S>) / 4);
  const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
  uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
  for (int i = t; i < W; i += nt) d[i] = s[i];
}

// Bulk update of every lattice of the batch (ordinary steps: no diagnostics).
// 128 threads per block; each warp keeps the parameters of the lattice of its
// current chunk in shared memory.
template <class L, class S, int COLL, int THERM>
__global__ void __maxnreg__(BulkRegs<S>::v) step_list_batch(const __grid_constant__ BatchArgs<S> a) {
  using C = typename Store<S>::C;
  __shared__ StepParams<S> sp[4];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int np = a.par ^ 1;
  DiagAcc<C> none;
  int cur = -1;
  int2 ch = gw < a.nchunks ? a.chunks[gw] : make_int2(0, 0);
  for (int j = gw; j < a.nchunks; j += nw) {
    const int2 next = j + nw < a.nchunks ? a.chunks[j + nw] : make_int2(0, 0);  // in flight meanwhile
    const int inst = ch.x >> 2;
    if (inst != cur) {  // uniform per warp
      __syncwarp();
      copy_params(sp[warp], a.params[2 * inst + a.par], lane, 32);
      __syncwarp();
      cur = inst;
    }
    const StepParams<S>& p = sp[warp];
    const bool fluid = (ch.x & 2) != 0, interior = (ch.x & 1) != 0;
    const int i = ch.y + lane;
    const int end = fluid ? p.lhdr[kLhFe] : p.lhdr[kLhSe];
    uint32_t ec = kEntPad, eb = kEntDead;
    if (i < end) { ec = p.ent_c[i]; eb = p.ent_b[i]; }
    if (ec != kEntPad && !(eb & kEntDead)) {
      const int c = (int)ec;
      const int pl = p.nx * p.ny;
      const Nbhd nb = interior ? Nbhd::interior(c, p.nx, pl)
                               : Nbhd(c % p.nx, (c / p.nx) % p.ny, c / pl, p.nx, p.ny, p.nz);
      const bool solid = !fluid;
      const bool solid_next = cell_update<L, S, COLL, THERM>(p, none, false, false, c, nb,
                                                            eb & ~(kEntReactive | kEntDead), solid,
                                                            (eb & kEntReactive) != 0, 0);
      if (solid && !solid_next) {
        const uint8_t m = p.mask[c];
        p.mask[c] = (uint8_t)(m & ~(1u << np));
        const int fi = atomicAdd(&p.lhdr[kLhFlip0 + p.par], 1);
        p.flips[(size_t)p.par * p.N + fi] = c;
      } else if (!solid && !interior) {
        const uint8_t m = p.mask[c];
        if ((m >> np) & 1) p.mask[c] = (uint8_t)(m & ~(1u << np));
      }
    }
    ch = next;
  }
}

// NEE faces of every lattice: block b updates block bc[b].z of face bc[b].y of
// lattice bc[b].x (128 cells).
template <class L, class S, int COLL, int THERM>
__global__ void __launch_bounds__(128) step_boundary_batch(const __grid_constant__ BatchArgs<S> a) {
  __shared__ StepParams<S> sp;
  const int4 b = a.bc[blockIdx.x];
  copy_params(sp, a.params[2 * b.x + a.par], threadIdx.x, blockDim.x);
  __syncthreads();
  DiagAcc<typename Store<S>::C> none;
  boundary_cell<L, S, COLL, THERM>(sp, b.y, b.z * blockDim.x + threadIdx.x, none, false);
}

// Cells that turned fluid, lattice blockIdx.y.
template <class L, class S, int COLL, int THERM>
__global__ void __launch_bounds__(256) flip_cells_batch(const __grid_constant__ BatchArgs<S> a) {
  __shared__ StepParams<S> sp;
  copy_params(sp, a.params[2 * blockIdx.y + a.par], threadIdx.x, blockDim.x);
  __syncthreads();
  const StepParams<S>& p = sp;
  const int n = p.lhdr[kLhFlip0 + p.par];
  if (blockIdx.x == 0 && threadIdx.x == 0) p.lhdr[kLhFlip0 + (p.par ^ 1)] = 0;  // for the next pass
  DiagAcc<typename Store<S>::C> none;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    flip_one<L, S, COLL, THERM>(p, none, false, false, (size_t)p.flips[(size_t)p.par * p.N + i]);
}

}  // namespace lbm
