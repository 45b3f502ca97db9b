// lbm_noalloc.cu -- diagnostics of the current state without any device allocation.
//
// lbm_diag_noalloc() runs the same recompute (peek) pass and the same two-stage
// reduction as lbm_compute_macro(h, LBM_STEP_DIAG) + lbm_read_diag(), but the
// reduction's scratch -- one partial row per block, the stage-1 sums, the final
// values and the device copy of the six side records -- lives in the file-scope
// array below instead of the caller-bound LBM_FIELD_SCRATCH buffer.  It exists
// for callers that cannot allocate device memory at all: a plug-in whose host
// application owns every device allocation through its own pool, or a
// monitoring hook inside a latency-critical time loop where a cudaMalloc (which
// can synchronise the whole device) is not acceptable.  Such a caller still
// binds the lattice state (its inputs) and receives the lbm_diag (its output).
#include <mutex>

#include "capi_internal.cuh"

using namespace lbm;
using namespace lbm::capi;

namespace {

constexpr int kMaxRows = LBM_NOALLOC_MAX_ROWS;
// partial rows [kNumDiag][kMaxRows] | stage-1 [kNumDiag][kStage1Blocks] | final [kNumDiag]
constexpr size_t kStage1Off = (size_t)kNumDiag * kMaxRows;
constexpr size_t kFinalOff = kStage1Off + (size_t)kNumDiag * kStage1Blocks;
constexpr size_t kDiagDoubles = kFinalOff + kNumDiag;

// Held by every GPU that loads this library until the process exits
// (kDiagDoubles * 8 bytes, about 2.6 MB, plus the side records).
static __device__ __align__(256) double g_noalloc_diag[kDiagDoubles];
static __device__ __align__(256) lbm_side_desc g_noalloc_sides[6];
// Kernel error flags of a call whose lattice has no SCRATCH buffer bound (tile form):
// bit 0 a bounded wait gave up, bit 1 the fluid cell list overflowed.
static __device__ __align__(256) int g_noalloc_err[1];

// Device addresses of the three arrays, looked up once per device with that
// device current (in host code the array names are host-side stand-ins, not
// device addresses).
constexpr int kMaxDevices = 64;
std::mutex g_mu;
double* g_diag_dev[kMaxDevices] = {};
lbm_side_desc* g_sides_dev[kMaxDevices] = {};
int* g_err_dev[kMaxDevices] = {};

int device_arrays(double** diag, lbm_side_desc** sides, int** err) {
  int dev = -1;
  LBM_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(LBM_ERR_ARG, "device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_diag_dev[dev]) {
    void* pd = nullptr;
    void* ps = nullptr;
    void* pe = nullptr;
    LBM_CUDA_TRY(cudaGetSymbolAddress(&pd, g_noalloc_diag));
    LBM_CUDA_TRY(cudaGetSymbolAddress(&ps, g_noalloc_sides));
    LBM_CUDA_TRY(cudaGetSymbolAddress(&pe, g_noalloc_err));
    g_diag_dev[dev] = (double*)pd;
    g_sides_dev[dev] = (lbm_side_desc*)ps;
    g_err_dev[dev] = (int*)pe;
  }
  *diag = g_diag_dev[dev];
  *sides = g_sides_dev[dev];
  *err = g_err_dev[dev];
  return LBM_OK;
}

template <class Fn>
int with_types_na(lbm_handle* h, Fn&& fn) {
  const int dim = h->d.dim, prec = h->d.precision;
  if (dim == 2 && prec == LBM_PREC_FP32) return fn(Lattice<2>{}, float{});
  if (dim == 3 && prec == LBM_PREC_FP32) return fn(Lattice<3>{}, float{});
  if (dim == 2 && prec == LBM_PREC_FP16) return fn(Lattice<2>{}, __half{});
  if (dim == 3 && prec == LBM_PREC_FP16) return fn(Lattice<3>{}, __half{});
  if (dim == 2 && prec == LBM_PREC_FP64) return fn(Lattice<2>{}, double{});
  if (dim == 3 && prec == LBM_PREC_FP64) return fn(Lattice<3>{}, double{});
  return fail(LBM_ERR_ARG, "unsupported dim/precision");
}

}  // namespace

extern "C" int32_t lbm_diag_noalloc(lbm_handle* h, lbm_diag* out, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h || !out) return fail(LBM_ERR_ARG, "NULL argument");
  if (h->step < 1) return fail(LBM_ERR_ARG, "no step taken yet: the initial fields are the state");
  const int rows = partial_rows(h->L);
  if (rows > kMaxRows)
    return fail(LBM_ERR_SIZE, "lbm_diag_noalloc: the lattice needs " + std::to_string(rows) +
                                  " partial rows, more than LBM_NOALLOC_MAX_ROWS = " +
                                  std::to_string(kMaxRows) + "; use lbm_compute_macro + lbm_read_diag");
  if (!h->ptr[LBM_FIELD_F] || !h->ptr[LBM_FIELD_MASK] || (h->d.thermal && !h->ptr[LBM_FIELD_G]) ||
      (h->d.pyro && (!h->ptr[LBM_FIELD_ALPHA] || !h->ptr[LBM_FIELD_REL])))
    return fail(LBM_ERR_UNBOUND, "lbm_diag_noalloc needs the lattice state (F, MASK, G, ALPHA, REL) bound");
  if (h->L.list && !h->ptr[LBM_FIELD_SCRATCH])
    return fail(LBM_ERR_UNBOUND, "lbm_diag_noalloc needs SCRATCH bound: it holds the cell lists of the lattice");
  double* diag = nullptr;
  lbm_side_desc* sides = nullptr;
  int* static_err = nullptr;
  int rc = device_arrays(&diag, &sides, &static_err);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  LBM_CUDA_TRY(cudaMemcpyAsync(sides, h->d.side, sizeof(h->d.side), cudaMemcpyHostToDevice, st));
  // Error flags: with SCRATCH bound they are the lattice's own, which also hold what the
  // earlier steps recorded (a state they invalidated stays invalid); without it, this
  // call's flags go to the static word, cleared first.
  int* err = h->ptr[LBM_FIELD_SCRATCH] ? scratch_err(h) : static_err;
  if (err == static_err) LBM_CUDA_TRY(cudaMemsetAsync(static_err, 0, sizeof(int), st));
  const int buf = (int)((h->step - 1) & 1);
  rc = with_types_na(h, [&](auto lat, auto s) -> int {
    using Lt = decltype(lat);
    using S = decltype(s);
    StepParams<S> p = make_params<S>(h, buf);
    p.partials = diag;
    p.partial_rows = rows;
    p.sides = sides;
    p.err = err;
    p.flags = LBM_STEP_DIAG | kStepPeek;
    return dispatch_step<Lt, S>(h, p, st);
  });
  if (rc) return rc;
  // every partial row and stage-1 slot read below is written earlier in this call
  if (rows <= kSingleReduceRows) {   // the same reduction as the allocating path
    reduce_diag_single<<<1, 1024, 0, st>>>(diag, rows, diag + kFinalOff);
  } else {
    reduce_diag_stage1<<<kStage1Blocks, 256, 0, st>>>(diag, rows, diag + kStage1Off);
    reduce_diag_stage2<<<1, 256, 0, st>>>(diag + kStage1Off, kStage1Blocks, diag + kFinalOff);
  }
  LBM_CUDA_TRY(cudaGetLastError());
  double v[kNumDiag];
  int flags = 0;
  LBM_CUDA_TRY(cudaMemcpyAsync(v, diag + kFinalOff, sizeof(v), cudaMemcpyDeviceToHost, st));
  LBM_CUDA_TRY(cudaMemcpyAsync(&flags, err, sizeof(int), cudaMemcpyDeviceToHost, st));
  LBM_CUDA_TRY(cudaStreamSynchronize(st));
  // the same mapping as lbm_read_diag
  if (flags & 1) return fail(LBM_ERR_TIMEOUT, "a staged-load wait in the step kernel timed out; the state is invalid");
  if (flags & 2) return fail(LBM_ERR_CUDA, "the fluid cell list overflowed; the state is invalid");
  out->mass = v[0]; out->energy = v[1]; out->solid_alpha = v[2]; out->umax = v[3];
  out->Tmin = v[4]; out->Tmax = v[5]; out->nonfinite = v[6]; out->nfluid = v[7];
  out->res_num = v[8]; out->res_den = v[9];
  out->step = h->step;
  if (v[6] > 0) return fail(LBM_ERR_NONFINITE, "diagnostics saw NaN/Inf");
  return LBM_OK;
}
