// capi_internal.cuh -- handle layout and launch templates shared by the C-ABI
// translation unit and the per-(lattice, precision) instantiation units.
#pragma once
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "batch_kernel.cuh"
#include "dense_kernel.cuh"
#include "list_kernel.cuh"
#include "step_kernels.cuh"

namespace lbm {
namespace capi {

int fail(int code, const std::string& msg);

#define LBM_CUDA_TRY(expr)                                                         \
  do {                                                                             \
    cudaError_t e__ = (expr);                                                      \
    if (e__ != cudaSuccess)                                                        \
      return ::lbm::capi::fail(LBM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e__)); \
  } while (0)

constexpr int kCtrlBytes = 6 * (int)sizeof(lbm_side_desc);

inline size_t storage_bytes(int prec) { return prec == LBM_PREC_FP16 ? 2 : (prec == LBM_PREC_FP64 ? 8 : 4); }
inline size_t compute_bytes(int prec) { return prec == LBM_PREC_FP64 ? 8 : 4; }
inline int lat_q(int dim) { return dim == 2 ? 9 : 19; }
inline int lat_qt(int dim) { return dim == 2 ? 5 : 7; }
// Flow-rate inlet (side 0 of velocity type LBM_BC_FLOWRATE) and the element count of
// its state in LBM_FIELD_INLET (compute precision).
inline bool has_flowrate(const lbm_desc& d) { return d.side[0].active && d.side[0].v_type == LBM_BC_FLOWRATE; }
// porous cells with two temperature fields: TS of the porous cells in LBM_FIELD_GS
inline bool porous_heat(const lbm_desc& d) { return d.porous != LBM_PORO_NONE && d.thermal == LBM_THERMAL_TWOFIELD; }
inline size_t inlet_elems(const lbm_desc& d) { return kInletHead + 2 * 4 * (size_t)d.ny * d.nz; }

struct Launch {
  int tx;             // threads per block along x (bulk kernel)
  dim3 grid, block;   // bulk
  int nfaces;         // active faces
  int faces[6];
  int bc_threads;
  dim3 bc_grid;
  int bulk_blocks, bc_blocks;
  int flip_blocks;    // grid of flip_cells (pyrolysis only), 256 threads each
  bool list;          // bulk update by step_list (persistent grid of bulk_blocks x 128)
  bool dense;         // bulk update by step_dense (persistent grid of bulk_blocks x kDThreads)
  int dense_smem;     // its dynamic shared memory (two stages)
  size_t N;
  // x-face records: with an active x side the bulk kernel leaves the post-stream state of
  // the cells at x = 1 / nx - 2 (the ones NEE extrapolates from) in SCRATCH, face-major,
  // and the boundary kernel reads it there: face_cells = ny * nz records of face_vals
  // values (Q + QT) per side, compute precision
  size_t face_cells;
  int face_vals;
  size_t face_elem;   // bytes per value
  int list_base;      // first entry of the solid list (capacity of the fluid list)
  size_t list_cap;    // entries in both lists
  int list_nbb;       // blocks of the list build
};

// Streaming multiprocessors of the current device (148 on B200; also the value
// used when no device is visible, e.g. when only sizes are being computed).
inline int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return 148;
  }
  return n;
}

// Shared memory of one stage of step_dense for this lattice's storage and physics.
template <class S>
inline int dense_stage_bytes_t(const lbm_desc& d) {
  const bool th = d.thermal != LBM_THERMAL_NONE, py = d.pyro != 0;
  if (th && py) return DenseLayout<Lattice<3>, S, true, true>::STAGE;
  if (th) return DenseLayout<Lattice<3>, S, true, false>::STAGE;
  return DenseLayout<Lattice<3>, S, false, false>::STAGE;
}
inline int dense_stage_bytes(const lbm_desc& d) {
  return d.precision == LBM_PREC_FP16 ? dense_stage_bytes_t<__half>(d)
                                      : (d.precision == LBM_PREC_FP64 ? dense_stage_bytes_t<double>(d)
                                                                       : dense_stage_bytes_t<float>(d));
}

inline Launch plan(const lbm_desc& d, int tx) {
  Launch L{};
  L.tx = tx;
  L.block = dim3(tx, 1, 1);
  L.grid = dim3((d.nx + tx - 1) / tx, d.ny, d.nz);
  L.bulk_blocks = (int)(L.grid.x * L.grid.y * L.grid.z);
  L.nfaces = 0;
  int maxcells = 0;
  for (int s = 0; s < 6; ++s) {
    if (!d.side[s].active) continue;
    L.faces[L.nfaces++] = s;
    const int cells = s < 2 ? d.ny * d.nz : (s < 4 ? d.nx * d.nz : d.nx * d.ny);
    if (cells > maxcells) maxcells = cells;
  }
  for (int s = L.nfaces; s < 6; ++s) L.faces[s] = -1;
  L.bc_threads = 128;
  L.bc_grid = dim3((maxcells + L.bc_threads - 1) / L.bc_threads, L.nfaces > 0 ? L.nfaces : 1, 1);
  L.bc_blocks = L.nfaces > 0 ? (int)(L.bc_grid.x * L.bc_grid.y) : 0;
  L.flip_blocks = d.pyro ? 2 * 148 : 0;
  // cell-list bulk kernel from 65536 cells up (below, its start-up round trips
  // outweigh what it saves); LBM_BULK=tile / list forces either form
  const char* b = getenv("LBM_BULK");
  L.N = (size_t)d.nx * d.ny * d.nz;
  // the descriptor's bulk_form wins over LBM_BULK
  const bool force_tile = d.bulk_form == 1 || (d.bulk_form == 0 && b && std::strcmp(b, "tile") == 0);
  const bool force_list = d.bulk_form == 2 || (d.bulk_form == 0 && b && std::strcmp(b, "list") == 0);
  const bool force_dense = d.bulk_form == 3 || (d.bulk_form == 0 && b && std::strcmp(b, "dense") == 0);
  L.list = !force_tile && !force_dense && (force_list || L.N >= 65536);
  // x-face records for NEE / ES x sides (a NEBB side reads only its own cell)
  const bool xface = (d.side[0].active || d.side[1].active) && d.nx >= 4 &&
                     d.side[0].active != LBM_SIDE_NEBB && d.side[1].active != LBM_SIDE_NEBB;
  L.face_cells = xface ? (size_t)d.ny * d.nz : 0;
  L.face_vals = lat_q(d.dim) + (d.thermal ? lat_qt(d.dim) : 0);
  L.face_elem = compute_bytes(d.precision);
  L.dense = force_dense;
  L.list_base = (int)((L.N + 64 + 31) / 32 * 32);
  L.list_cap = 2 * (size_t)L.list_base;
  L.list_nbb = (int)((L.N + kListChunk - 1) / kListChunk);
  if (L.list) {
    const int per_sm = list_blocks_per_sm(d.precision == LBM_PREC_FP64);  // 128-thread blocks at the register cap
    const long chunks = (long)(L.N / 32) + 8;
    L.bulk_blocks = (int)std::max<long>(1, std::min<long>((chunks + 3) / 4, (long)sm_count() * per_sm));
  }
  if (L.dense) {
    const long ntiles = (long)(d.nx / kDTX) * (d.ny / kDTY) * (d.nz / kDTZ);
    const int per_sm = d.precision == LBM_PREC_FP64 ? DenseCTAs<double>::v : DenseCTAs<float>::v;
    L.bulk_blocks = (int)std::max<long>(1, std::min<long>(ntiles, (long)sm_count() * per_sm));
    L.dense_smem = 2 * dense_stage_bytes(d);
  }
  return L;
}

// Why the dense form cannot run this lattice (nullptr: it can).
inline const char* dense_unsupported(const lbm_desc& d) {
  if (d.dim != 3) return "the dense bulk form is 3D only";
  if (d.nx % kDTX || d.ny % kDTY || d.nz % kDTZ) return "the dense bulk form needs nx % 32 == 0, ny % 4 == 0, nz % 2 == 0";
  if (d.thermal == LBM_THERMAL_TWOFIELD) return "the dense bulk form runs the conjugate temperature field only";
  return nullptr;
}

// Threads per block along x for the bulk kernel.  LBM_BLOCK_X (32..256, a
// multiple of 32) overrides the default for launch-shape sweeps.
inline int default_tx(const lbm_desc& d) {
  if (const char* e = getenv("LBM_BLOCK_X")) {
    const int v = atoi(e);
    if (v >= 32 && v <= 256 && v % 32 == 0) return v;
  }
  if (d.dim == 2) return d.nx >= 64 ? 64 : 32;
  return d.nx >= 128 ? 128 : (d.nx >= 64 ? 64 : 32);
}

}  // namespace capi
}  // namespace lbm

struct lbm_handle {
  lbm_desc d;
  size_t N;
  void* ptr[LBM_NUM_FIELDS];
  size_t bytes[LBM_NUM_FIELDS];
  int64_t step;
  lbm::capi::Launch L;
  bool diag_valid;
  bool initialised;  // lbm_init_equilibrium ran (state and cell lists exist)
  // list form with active sides: the boundary kernel runs on a second stream beside
  // the list kernel (created at the first step; null: one stream)
  cudaStream_t side = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  bool side_tried = false;
  // dense form: tensor maps over the bound F / G / MASK buffers (rebuilt when a buffer
  // is rebound) and the bound of its mbarrier waits
  lbm::DenseMaps maps{};
  const void* maps_for[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  uint32_t wait_spins = lbm::kDefaultWaitSpins;
  int device = 0;  // the CUDA device current at lbm_create: every call runs its work there
};

// Makes the handle's device current for the scope of an entry point and restores the
// caller's device afterwards (a call made with another device current still works on
// the device whose memory the handle's buffers are).
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {  // dev < 0: leave the current device alone
    if (dev < 0) return;
    if (cudaGetDevice(&prev) != cudaSuccess) { prev = -1; cudaGetLastError(); return; }
    if (prev != dev && cudaSetDevice(dev) != cudaSuccess) cudaGetLastError();
    if (prev == dev) prev = -1;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// A batch of lattices stepped together (batch_kernel.cuh).  Its device tables
// live in a caller-owned buffer: parameters [n][2] | chunk table | boundary
// block table.
struct lbm_batch {
  std::vector<lbm_handle*> hs;
  void* scratch;
  size_t bytes;
  void* params;
  int2* chunks;
  int nchunks;
  int4* bc;
  int nbc;
  int list_blocks;   // persistent grid of step_list_batch (128 threads each)
  int flip_blocks;   // flip_cells_batch blocks per lattice
};

namespace lbm {
namespace capi {

// Scratch layout: partials [kNumDiag][rows] | stage-1 sums [kNumDiag][kStage1Blocks] |
// final [kNumDiag] | (256-byte aligned) device copy of the 6 side records.
inline int partial_rows(const Launch& L) { return L.bulk_blocks + L.bc_blocks + L.flip_blocks; }
inline size_t scratch_diag_doubles(const Launch& L) {
  return (size_t)kNumDiag * (partial_rows(L) + kStage1Blocks + 1);
}
// Cell lists (step_list): header | build blocks [4][nbb] | ent_c | ent_b | pos | flips[2][N],
// 256-byte aligned after the error flag.
inline size_t list_offset(const Launch& L) {
  return ((scratch_diag_doubles(L) * sizeof(double) + 255) / 256 * 256 + kCtrlBytes + 16 + 255) / 256 * 256;
}
inline size_t list_bytes(const Launch& L) {
  if (L.dense) return (size_t)kLhSlots * 4 + 2 * L.N * 4;  // header | flip lists [2][N]
  if (!L.list) return 0;
  return (size_t)kLhSlots * 4 + (size_t)4 * L.list_nbb * 4 + 2 * L.list_cap * 4 + L.N * 4 + 2 * L.N * 4;
}
inline size_t scratch_base_bytes(const Launch& L) {
  if (L.list || L.dense) return list_offset(L) + list_bytes(L);
  return (scratch_diag_doubles(L) * sizeof(double) + 255) / 256 * 256 + kCtrlBytes + 16;
}
inline size_t face_offset(const Launch& L) { return (scratch_base_bytes(L) + 255) / 256 * 256; }
inline size_t scratch_bytes(const Launch& L) {
  if (!L.face_cells) return scratch_base_bytes(L);
  return face_offset(L) + 2 * (size_t)L.face_vals * L.face_cells * L.face_elem;
}
inline double* scratch_partials(lbm_handle* h) { return (double*)h->ptr[LBM_FIELD_SCRATCH]; }
inline double* scratch_stage1(lbm_handle* h) {
  return scratch_partials(h) + (size_t)kNumDiag * partial_rows(h->L);
}
inline double* scratch_final(lbm_handle* h) { return scratch_stage1(h) + (size_t)kNumDiag * kStage1Blocks; }
inline lbm_side_desc* scratch_sides(lbm_handle* h) {
  const size_t off = (scratch_diag_doubles(h->L) * sizeof(double) + 255) / 256 * 256;
  return (lbm_side_desc*)((char*)h->ptr[LBM_FIELD_SCRATCH] + off);
}
// Kernel error flags after the side records: bit 0 a bounded wait timed out,
// bit 1 the fluid list overflowed.
inline int* scratch_err(lbm_handle* h) { return (int*)(scratch_sides(h) + 6); }
inline int* scratch_lhdr(lbm_handle* h) { return (int*)((char*)h->ptr[LBM_FIELD_SCRATCH] + list_offset(h->L)); }
inline int* scratch_lblk(lbm_handle* h) { return scratch_lhdr(h) + kLhSlots; }
inline uint32_t* scratch_ent_c(lbm_handle* h) { return (uint32_t*)(scratch_lblk(h) + 4 * (size_t)h->L.list_nbb); }
inline uint32_t* scratch_ent_b(lbm_handle* h) { return scratch_ent_c(h) + h->L.list_cap; }
inline int* scratch_pos(lbm_handle* h) { return (int*)(scratch_ent_b(h) + h->L.list_cap); }
inline int* scratch_flips(lbm_handle* h) {
  return h->L.dense ? scratch_lhdr(h) + kLhSlots : scratch_pos(h) + h->N;
}
// Two-stage deterministic reduction of the block partials into scratch_final().
inline void launch_reduce(lbm_handle* h, cudaStream_t st) {
  const int rows = partial_rows(h->L);
  if (rows <= kSingleReduceRows) {
    reduce_diag_single<<<1, 1024, 0, st>>>(scratch_partials(h), rows, scratch_final(h));
    return;
  }
  reduce_diag_stage1<<<kStage1Blocks, 256, 0, st>>>(scratch_partials(h), rows, scratch_stage1(h));
  reduce_diag_stage2<<<1, 256, 0, st>>>(scratch_stage1(h), kStage1Blocks, scratch_final(h));
}

template <class S>
StepParams<S> make_params(lbm_handle* h, int buf) {
  using C = typename Store<S>::C;
  const lbm_desc& d = h->d;
  StepParams<S> p{};
  p.nx = d.nx; p.ny = d.ny; p.nz = d.nz; p.N = h->N;
  const int Q = lat_q(d.dim), QT = lat_qt(d.dim);
  S* f = (S*)h->ptr[LBM_FIELD_F];
  S* g = (S*)h->ptr[LBM_FIELD_G];
  p.fA = f + (size_t)buf * Q * h->N;
  p.fB = f + (size_t)(buf ^ 1) * Q * h->N;
  if (g) { p.gA = g + (size_t)buf * QT * h->N; p.gB = g + (size_t)(buf ^ 1) * QT * h->N; }
  p.mask = (uint8_t*)h->ptr[LBM_FIELD_MASK];
  p.alpha = (C*)h->ptr[LBM_FIELD_ALPHA];
  C* rel = (C*)h->ptr[LBM_FIELD_REL];
  if (rel) { p.relA = rel + (size_t)buf * h->N; p.relB = rel + (size_t)(buf ^ 1) * h->N; }
  p.par = buf;
  p.eos = d.eos;
  p.half_force = d.half_force_velocity;
  p.has_force = (d.force[0] != 0 || d.force[1] != 0 || d.force[2] != 0);
  p.nu = (C)d.nu; p.Fx = (C)d.force[0]; p.Fy = (C)d.force[1]; p.Fz = (C)d.force[2];
  for (int r = 0; r < 19; ++r) {
    double n2 = 0;
    if (r < Q) {
      for (int k = 0; k < Q; ++k) {
        const double m = d.dim == 2 ? Lattice<2>::mrt(r, k) : Lattice<3>::mrt(r, k);
        n2 += m * m;
      }
    }
    p.mrt_sn[r] = n2 > 0 ? (C)(d.mrt_s[r] / n2) : (C)0;
  }
  p.itauT_f = d.thermal ? (C)1 / (C)d.tauT_fluid : (C)0;
  p.itauT_s = d.thermal ? (C)1 / (C)d.tauT_solid : (C)0;
  p.rho0 = (C)d.rho0; p.T0 = (C)d.T0;
  p.pyA = (C)d.pyro_A; p.pyb = (C)d.pyro_b; p.pyEaR = (C)(d.pyro_Ea / kGasConstant); p.pyTmin = (C)d.pyro_Tmin;
  p.Tref = (C)d.T_ref; p.Tscale = (C)d.T_scale; p.dtp = (C)d.dt_phys;
  p.heat_norm = (C)d.heat_norm; p.gas_coef = (C)d.gas_coef; p.alpha_flip = (C)d.alpha_flip;
  p.suth = d.viscosity == LBM_VISC_SUTHERLAND;
  p.suthA = (C)d.suth_A; p.suthTs = (C)d.suth_Ts;
  p.tprop = d.tprop;
  for (int ph = 0; ph < 2; ++ph) {
    for (int i = 0; i < 5; ++i) {
      p.tp_cond[ph][i] = (C)d.tp_cond[ph][i];
      p.tp_lo[ph][i] = (C)d.tp_cap_lo[ph][i];
      p.tp_hi[ph][i] = (C)d.tp_cap_hi[ph][i];
    }
    p.tp_Tmid[ph] = (C)d.tp_cap_Tmid[ph];
    p.tp_mul[ph] = (C)d.tp_cap_mul[ph];
  }
  p.tp_Tsc[0] = (C)d.T_scale; p.tp_Tref[0] = (C)d.T_ref;
  p.tp_Tsc[1] = (C)d.Ts_scale; p.tp_Tref[1] = (C)d.Ts_ref;
  p.tp_rhos = (C)d.tp_rhos; p.tp_dt = (C)d.tp_dt; p.tp_dx2 = (C)d.tp_dx2;
  p.tp_lat = (C)(d.dim == 2 ? 3 : 4);
  p.tp_prandtl = (C)d.tp_prandtl;
  p.poro = (const C*)h->ptr[LBM_FIELD_PORO];
  p.darcy = (const C*)h->ptr[LBM_FIELD_DARCY];
  p.forch = (const C*)h->ptr[LBM_FIELD_FORCH];
  p.poro_model = d.porous;
  S* gs = (S*)h->ptr[LBM_FIELD_GS];
  if (gs) { p.gsA = gs + (size_t)buf * QT * h->N; p.gsB = gs + (size_t)(buf ^ 1) * QT * h->N; }
  p.xheat = (const C*)h->ptr[LBM_FIELD_XHEAT];
  p.Trs = (C)d.Ts_ref; p.Tss = (C)d.Ts_scale;
  p.cap_f = (C)d.cap_fluid; p.cap_s = (C)d.cap_solid;
  p.sig_dx = d.dx_phys > 0 ? (C)(5.670374419e-8 / d.dx_phys) : (C)0;  // Stefan-Boltzmann, util/constant.py:20
  p.Tamb4 = (C)(d.T_ambient * d.T_ambient * d.T_ambient * d.T_ambient);
  p.radiation = d.radiation;
  p.fp16_nearest = d.fp16_rounding == LBM_FP16_NEAREST;
  p.nebb = 0;
  for (int s = 0; s < 6; ++s) p.nebb |= d.side[s].active == LBM_SIDE_NEBB;
  // sides whose cells store only their inward populations: NEE / ES sides where neither the
  // side nor its opposite keeps a quantity of its own (a PERIODIC type makes the boundary
  // kernel pull that side's own state, which reads the other slots across the wrap)
  p.inward_only = 0;
  for (int s = 0; s < 6; ++s) {
    const lbm_side_desc& a = d.side[s];
    const lbm_side_desc& b = d.side[s ^ 1];
    auto keeps = [&d](const lbm_side_desc& q) {
      return q.active && (q.v_type == LBM_BC_PERIODIC || q.rho_type == LBM_BC_PERIODIC ||
                          (d.thermal && q.T_type == LBM_BC_PERIODIC));
    };
    const bool ok = (a.active == LBM_SIDE_NEE || a.active == LBM_SIDE_ES) && !keeps(a) && !keeps(b) &&
                    b.active != LBM_SIDE_NEBB;
    if (ok) p.inward_only |= 1 << s;
  }
  p.active = 0;
  for (int s = 0; s < 6; ++s) if (d.side[s].active) p.active |= 1 << s;
  p.sides = h->ptr[LBM_FIELD_SCRATCH] ? scratch_sides(h) : nullptr;
  p.err = h->ptr[LBM_FIELD_SCRATCH] ? scratch_err(h) : nullptr;
  p.flags = 0;
  p.adiabatic = d.thermal == LBM_THERMAL_TWOFIELD;
  p.partials = h->ptr[LBM_FIELD_SCRATCH] ? scratch_partials(h) : nullptr;
  p.partial_rows = partial_rows(h->L);
  p.block_offset = 0;
  p.rho_out = (C*)h->ptr[LBM_FIELD_RHO];
  p.u_out = (C*)h->ptr[LBM_FIELD_U];
  p.T_out = (C*)h->ptr[LBM_FIELD_T];
  p.uprev = (float*)h->ptr[LBM_FIELD_UPREV];
  p.inlet = has_flowrate(d) ? (C*)h->ptr[LBM_FIELD_INLET] : nullptr;
  if (h->L.list && h->ptr[LBM_FIELD_SCRATCH]) {
    p.lhdr = scratch_lhdr(h);
    p.ent_c = scratch_ent_c(h);
    p.ent_b = scratch_ent_b(h);
    p.pos = scratch_pos(h);
    p.flips = scratch_flips(h);
  }
  if (h->L.dense && h->ptr[LBM_FIELD_SCRATCH]) {  // flip lists only
    p.lhdr = scratch_lhdr(h);
    p.flips = scratch_flips(h);
  }
  p.wait_spins = h->wait_spins;
  p.face = nullptr;
  p.face_sides = 0;
  if (h->L.face_cells && h->ptr[LBM_FIELD_SCRATCH]) {
    p.face = (C*)((char*)h->ptr[LBM_FIELD_SCRATCH] + face_offset(h->L));
    p.face_sides = (d.side[0].active ? 1 : 0) | (d.side[1].active ? 2 : 0);
  }
  fastdiv_init((uint32_t)d.nx, p.nx_mul, p.nx_shr);
  return p;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link to libcuda).
inline PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    else
      cudaGetLastError();
  });
  return fn;
}

// Tensor maps of the dense form over the bound buffers (kept until a buffer is rebound).
// Populations: 4-D (x, y, z, plane) with planes = 2 Q (both halves), one flow map per box
// shape (bx, kDTY [+1], kDTZ [+1], 1); mask: 3-D bytes, box (64, kDTY + 2, kDTZ + 2); gas
// release: 4-D (x, y, z, half) of the compute type, box (bx, kDTY + 2, kDTZ + 2, 1);
// reactive fraction: 3-D, box (32, kDTY, kDTZ).  Out-of-bounds box parts read zeros.
template <class S>
int encode_dense_maps(lbm_handle* h) {
  if (h->maps_for[0] == h->ptr[LBM_FIELD_F] && h->maps_for[1] == h->ptr[LBM_FIELD_G] &&
      h->maps_for[2] == h->ptr[LBM_FIELD_MASK] && h->maps_for[3] == h->ptr[LBM_FIELD_REL] &&
      h->maps_for[4] == h->ptr[LBM_FIELD_ALPHA])
    return LBM_OK;
  PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
  if (!enc) return fail(LBM_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const lbm_desc& d = h->d;
  const cuuint64_t nx = (cuuint64_t)d.nx, ny = (cuuint64_t)d.ny, nz = (cuuint64_t)d.nz, es = sizeof(S);
  const CUtensorMapDataType dt = sizeof(S) == 2 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16
                                                : (sizeof(S) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64
                                                                  : CU_TENSOR_MAP_DATA_TYPE_FLOAT32);
  using LY = DenseLayout<Lattice<3>, S, true, true>;
  using C = typename Store<S>::C;
  const CUtensorMapDataType dtc = sizeof(C) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  auto map4 = [&](CUtensorMap* m, CUtensorMapDataType t, cuuint64_t e, void* base, int planes, int bx, int by,
                  int bz) -> CUresult {
    const cuuint64_t dims[4] = {nx, ny, nz, (cuuint64_t)planes};
    const cuuint64_t strides[3] = {nx * e, nx * ny * e, nx * ny * nz * e};
    const cuuint32_t box[4] = {(cuuint32_t)bx, (cuuint32_t)by, (cuuint32_t)bz, 1};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return enc(m, t, 4, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  };
  CUresult r = CUDA_SUCCESS;
  for (int i = 0; i < 8 && r == CUDA_SUCCESS; ++i)  // f[wide << 2 | ey << 1 | ez]
    r = map4(&h->maps.f[i], dt, es, h->ptr[LBM_FIELD_F], 2 * 19, (i & 4) ? LY::BXW : LY::BXN,
             kDTY + ((i >> 1) & 1), kDTZ + (i & 1));
  if (r == CUDA_SUCCESS && h->ptr[LBM_FIELD_G]) {
    r = map4(&h->maps.g_wide, dt, es, h->ptr[LBM_FIELD_G], 2 * 7, LY::BXW, kDTY, kDTZ);
    if (r == CUDA_SUCCESS) r = map4(&h->maps.g_narrow, dt, es, h->ptr[LBM_FIELD_G], 2 * 7, LY::BXN, kDTY, kDTZ);
  }
  if (r == CUDA_SUCCESS && d.pyro && h->ptr[LBM_FIELD_REL] && h->ptr[LBM_FIELD_ALPHA]) {
    r = map4(&h->maps.rel, dtc, sizeof(C), h->ptr[LBM_FIELD_REL], 2, LY::RX, LY::MY, LY::MZ);
    if (r == CUDA_SUCCESS) {
      const cuuint64_t dims[3] = {nx, ny, nz};
      const cuuint64_t strides[2] = {nx * sizeof(C), nx * ny * sizeof(C)};
      const cuuint32_t box[3] = {(cuuint32_t)kDTX, (cuuint32_t)kDTY, (cuuint32_t)kDTZ};
      const cuuint32_t estr[3] = {1, 1, 1};
      r = enc(&h->maps.alpha, dtc, 3, h->ptr[LBM_FIELD_ALPHA], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
  }
  if (r == CUDA_SUCCESS) {
    const cuuint64_t dims[3] = {nx, ny, nz};
    const cuuint64_t strides[2] = {nx, nx * ny};
    const cuuint32_t box[3] = {(cuuint32_t)LY::MX, (cuuint32_t)LY::MY, (cuuint32_t)LY::MZ};
    const cuuint32_t estr[3] = {1, 1, 1};
    r = enc(&h->maps.mask, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, h->ptr[LBM_FIELD_MASK], dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  }
  if (r != CUDA_SUCCESS) {
    for (auto& q : h->maps_for) q = nullptr;
    return fail(LBM_ERR_CUDA, "cuTensorMapEncodeTiled failed with CUresult " + std::to_string((int)r));
  }
  h->maps_for[0] = h->ptr[LBM_FIELD_F];
  h->maps_for[1] = h->ptr[LBM_FIELD_G];
  h->maps_for[2] = h->ptr[LBM_FIELD_MASK];
  h->maps_for[3] = h->ptr[LBM_FIELD_REL];
  h->maps_for[4] = h->ptr[LBM_FIELD_ALPHA];
  return LBM_OK;
}

// Launch one step (bulk + boundary) for handle h; defined per (lattice, storage)
// in the inst_*.cu units.
template <class Lt, class S>
int dispatch_step(lbm_handle* h, StepParams<S> p, cudaStream_t st);
template <class Lt, class S>
int dispatch_init(lbm_handle* h, StepParams<S> p, const float* rho, const float* u, const float* T,
                  const float* alpha, int solid_bit, cudaStream_t st);

template <class Lt, class S>
int dispatch_batch(lbm_batch* b, cudaStream_t st);

#define LBM_EXTERN_INST(LT, ST)                                                                 \
  extern template int dispatch_batch<LT, ST>(lbm_batch*, cudaStream_t);                         \
  extern template int dispatch_step<LT, ST>(lbm_handle*, StepParams<ST>, cudaStream_t);         \
  extern template int dispatch_init<LT, ST>(lbm_handle*, StepParams<ST>, const float*, const float*, \
                                            const float*, const float*, int, cudaStream_t);
LBM_EXTERN_INST(Lattice<2>, float)
LBM_EXTERN_INST(Lattice<3>, float)
LBM_EXTERN_INST(Lattice<2>, __half)
LBM_EXTERN_INST(Lattice<3>, __half)
LBM_EXTERN_INST(Lattice<2>, double)
LBM_EXTERN_INST(Lattice<3>, double)
#undef LBM_EXTERN_INST

}  // namespace capi
}  // namespace lbm
