// Step, batch and init launchers, instantiated per lattice and storage precision
// by the inst_*.cu translation units (split so that the kernels compile in
// parallel).
#pragma once
#include <atomic>

#include "capi_internal.cuh"

namespace lbm {
namespace capi {

// Collision code of the kernels: LBM_COLL_*, plus kCollSutherland with properties that
// follow the cell's temperature (the Sutherland viscosity, derived thermal diffusivities;
// thermal modes only: THERM 1-3), or plus kCollPorous with porous cells (no temperature
// field, THERM 0, or two fields exchanging heat in them, THERM 4)
constexpr int kSB = kCollSutherland + LBM_COLL_BGK, kSM = kCollSutherland + LBM_COLL_MRT;
constexpr int kPB = kCollPorous + LBM_COLL_BGK, kPM = kCollPorous + LBM_COLL_MRT;
inline int collision_code(const lbm_desc& d) {
  return d.collision + ((d.viscosity == LBM_VISC_SUTHERLAND || d.tprop) ? kCollSutherland : 0) +
         (d.porous != LBM_PORO_NONE ? kCollPorous : 0);
}
// Temperature code of the kernels (THERM): 0 none, 1 conjugate, 2 conjugate + pyrolysis,
// 3 two fields, 4 two fields with porous cells
inline int therm_code(const lbm_desc& d) {
  if (!d.thermal) return 0;
  if (d.pyro) return 2;
  if (d.thermal == LBM_THERMAL_TWOFIELD) return d.porous != LBM_PORO_NONE ? 4 : 3;
  return 1;
}

// Dynamic shared memory above the 48 KB default is a per-device attribute of a kernel:
// opt in once per device ordinal (one bit per device in `done`, which each call site keeps
// per kernel instantiation), again after a failure; the launch that follows then reports
// the error through cudaGetLastError.
template <class K>
inline void opt_in_smem(std::atomic<unsigned long long>& done, K* kernel, int bytes) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes) == cudaSuccess && bit)
    done.fetch_or(bit, std::memory_order_acq_rel);
}

template <class Lt, class S, int COLL, int THERM, int MODE>
static void launch_list(const Launch& L, const StepParams<S>& p, cudaStream_t st) {
  constexpr size_t smem = list_smem_bytes<Lt, S, THERM>(128);
  if (smem > 0) {
    // opt in above the 48 KB default: with the static reduction buffer the total can
    // pass it even when the stages alone do not
    static std::atomic<unsigned long long> done{0};
    opt_in_smem(done, step_list<Lt, S, COLL, THERM, MODE>, (int)smem);
  }
  step_list<Lt, S, COLL, THERM, MODE><<<L.bulk_blocks, 128, smem, st>>>(p);
}

// Second stream for the boundary kernel (list form with active sides), made on the
// device current at the first step; on failure the step stays on one stream.
inline void ensure_side_stream(lbm_handle* h) {
  if (h->side_tried) return;
  h->side_tried = true;
  if (!((h->L.list || h->L.dense) && h->L.nfaces > 0)) return;
  if (cudaStreamCreateWithFlags(&h->side, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming) != cudaSuccess) {
    cudaGetLastError();
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->side) cudaStreamDestroy(h->side);
    h->side = nullptr;
    h->ev_fork = h->ev_join = nullptr;
  }
}

template <class Lt, class S, int COLL, int THERM, int MODE>
static void launch_dense(lbm_handle* h, const StepParams<S>& p, cudaStream_t st) {
  if constexpr (Lt::DIM == 3 && THERM != 3) {
    static std::atomic<unsigned long long> done{0};
    opt_in_smem(done, step_dense<Lt, S, COLL, THERM, MODE>, h->L.dense_smem);
    step_dense<Lt, S, COLL, THERM, MODE><<<h->L.bulk_blocks, kDThreads, h->L.dense_smem, st>>>(p, h->maps);
  }
}

template <class Lt, class S, int COLL, int THERM>
static void launch_step(lbm_handle* h, StepParams<S> p, cudaStream_t st) {
  const Launch& L = h->L;
  ensure_side_stream(h);
  // flow-rate inlet: this step's coefficient, before the kernels that read it (a
  // recompute of the last step reuses the one it had)
  if (p.inlet && !(p.flags & kStepPeek)) inlet_flow_coef<S><<<1, 1024, 0, st>>>(p);
  // list form: the boundary kernel is independent of the list kernel (both read the
  // input half only and write disjoint slots, partial rows apart), so it runs on the
  // second stream and its blocks take the SMs that the persistent list kernel's blocks
  // leave as they finish; flip_cells waits for both
  // (with x-face records the boundary kernel reads what the bulk kernel writes: it follows it)
  const bool fork = (L.list || L.dense) && L.nfaces > 0 && h->side != nullptr && !p.face;
  if (fork) {
    cudaEventRecord(h->ev_fork, st);
    cudaStreamWaitEvent(h->side, h->ev_fork, 0);
  }
  if (L.dense) {
    if (p.flags & kStepPeek) launch_dense<Lt, S, COLL, THERM, 2>(h, p, st);
    else if (p.flags) launch_dense<Lt, S, COLL, THERM, 1>(h, p, st);
    else launch_dense<Lt, S, COLL, THERM, 0>(h, p, st);
  } else if (L.list) {
    if (p.flags & kStepPeek) launch_list<Lt, S, COLL, THERM, 2>(L, p, st);
    else if (p.flags) launch_list<Lt, S, COLL, THERM, 1>(L, p, st);
    else launch_list<Lt, S, COLL, THERM, 0>(L, p, st);
  } else {
    step_bulk<Lt, S, COLL, THERM><<<L.grid, L.block, 0, st>>>(p);
  }
  if (L.nfaces > 0) {
    p.block_offset = L.bulk_blocks;  // one partial row per bulk block, then the boundary blocks
    const int4 f01 = make_int4(L.faces[0], L.faces[1], L.faces[2], L.faces[3]);
    const int2 f2 = make_int2(L.faces[4], L.faces[5]);
    step_boundary<Lt, S, COLL, THERM><<<L.bc_grid, L.bc_threads, 0, fork ? h->side : st>>>(p, f01, f2);
  }
  if (fork) {
    cudaEventRecord(h->ev_join, h->side);
    cudaStreamWaitEvent(st, h->ev_join, 0);
  }
  if constexpr (THERM == 2) {
    // after the boundary kernel: the flipped cells' new populations go in after every
    // other store of the pass
    p.block_offset = L.bulk_blocks + L.bc_blocks;
    flip_cells<Lt, S, COLL, THERM><<<L.flip_blocks, 256, 0, st>>>(p);
  }
}

template <class Lt, class S>
int dispatch_step(lbm_handle* h, StepParams<S> p, cudaStream_t st) {
  const int coll = collision_code(h->d);
  const int therm = therm_code(h->d);
  if (h->L.dense) {
    const char* why = dense_unsupported(h->d);
    if (why) return fail(LBM_ERR_ARG, why);
    const int rc = encode_dense_maps<S>(h);
    if (rc) return rc;
  }
#define LBM_CASE(C_, T_) \
  if (coll == C_ && therm == T_) { launch_step<Lt, S, C_, T_>(h, p, st); return LBM_OK; }
  LBM_CASE(LBM_COLL_BGK, 0) LBM_CASE(LBM_COLL_BGK, 1) LBM_CASE(LBM_COLL_BGK, 2) LBM_CASE(LBM_COLL_BGK, 3)
  LBM_CASE(LBM_COLL_MRT, 0) LBM_CASE(LBM_COLL_MRT, 1) LBM_CASE(LBM_COLL_MRT, 2) LBM_CASE(LBM_COLL_MRT, 3)
  LBM_CASE(kSB, 1) LBM_CASE(kSB, 2) LBM_CASE(kSB, 3) LBM_CASE(kSM, 1) LBM_CASE(kSM, 2) LBM_CASE(kSM, 3)
  LBM_CASE(kPB, 0) LBM_CASE(kPM, 0) LBM_CASE(kPB, 4) LBM_CASE(kPM, 4)
#undef LBM_CASE
  return fail(LBM_ERR_ARG, "unsupported collision/thermal combination");
}

template <class Lt, class S, int COLL, int THERM>
static void launch_batch(lbm_batch* b, cudaStream_t st) {
  BatchArgs<S> a;
  a.params = (const StepParams<S>*)b->params;
  a.chunks = b->chunks;
  a.nchunks = b->nchunks;
  a.bc = b->bc;
  a.nbc = b->nbc;
  a.par = (int)(b->hs[0]->step & 1);
  step_list_batch<Lt, S, COLL, THERM><<<b->list_blocks, 128, 0, st>>>(a);
  if (b->nbc > 0) step_boundary_batch<Lt, S, COLL, THERM><<<b->nbc, 128, 0, st>>>(a);
  if constexpr (THERM == 2) flip_cells_batch<Lt, S, COLL, THERM><<<dim3(b->flip_blocks, (unsigned)b->hs.size()), 256, 0, st>>>(a);
}

template <class Lt, class S>
int dispatch_batch(lbm_batch* b, cudaStream_t st) {
  const lbm_desc& d = b->hs[0]->d;
  const int coll = collision_code(d);
  const int therm = therm_code(d);
#define LBM_CASE(C_, T_) \
  if (coll == C_ && therm == T_) { launch_batch<Lt, S, C_, T_>(b, st); return LBM_OK; }
  LBM_CASE(LBM_COLL_BGK, 0) LBM_CASE(LBM_COLL_BGK, 1) LBM_CASE(LBM_COLL_BGK, 2) LBM_CASE(LBM_COLL_BGK, 3)
  LBM_CASE(LBM_COLL_MRT, 0) LBM_CASE(LBM_COLL_MRT, 1) LBM_CASE(LBM_COLL_MRT, 2) LBM_CASE(LBM_COLL_MRT, 3)
  LBM_CASE(kSB, 1) LBM_CASE(kSB, 2) LBM_CASE(kSB, 3) LBM_CASE(kSM, 1) LBM_CASE(kSM, 2) LBM_CASE(kSM, 3)
  LBM_CASE(kPB, 0) LBM_CASE(kPM, 0)
#undef LBM_CASE
  return fail(LBM_ERR_ARG, "unsupported collision/thermal combination");
}

template <class Lt, class S>
int dispatch_init(lbm_handle* h, StepParams<S> p, const float* rho, const float* u, const float* T,
                  const float* alpha, int solid_bit, cudaStream_t st) {
  const int coll = collision_code(h->d);
  const int therm = therm_code(h->d);
  const int bs = 256;
  const unsigned nb = (unsigned)((h->N + bs - 1) / bs);
#define LBM_CASE(C_, T_)                                                                       \
  if (coll == C_ && therm == T_) {                                                             \
    init_equilibrium_kernel<Lt, S, C_, T_><<<nb, bs, 0, st>>>(p, rho, u, T, alpha, solid_bit); \
    return LBM_OK;                                                                             \
  }
  LBM_CASE(LBM_COLL_BGK, 0) LBM_CASE(LBM_COLL_BGK, 1) LBM_CASE(LBM_COLL_BGK, 2) LBM_CASE(LBM_COLL_BGK, 3)
  LBM_CASE(LBM_COLL_MRT, 0) LBM_CASE(LBM_COLL_MRT, 1) LBM_CASE(LBM_COLL_MRT, 2) LBM_CASE(LBM_COLL_MRT, 3)
  LBM_CASE(kSB, 1) LBM_CASE(kSB, 2) LBM_CASE(kSB, 3) LBM_CASE(kSM, 1) LBM_CASE(kSM, 2) LBM_CASE(kSM, 3)
  LBM_CASE(kPB, 0) LBM_CASE(kPM, 0) LBM_CASE(kPB, 4) LBM_CASE(kPM, 4)
#undef LBM_CASE
  return fail(LBM_ERR_ARG, "unsupported collision/thermal combination");
}

}  // namespace capi
}  // namespace lbm
