// lbm_capi.cu -- host side of the C ABI declared in include/lbm_b200.h.
//
// Validates descriptors, keeps the caller's device buffers, and launches the
// sm_100a kernels of step_kernels.cuh on the caller's stream.  No allocation
// happens here: every buffer (including the reduction scratch) is bound by the
// caller, sized by lbm_required_bytes().
#include <cmath>
#include <cstddef>
#include "capi_internal.cuh"

using namespace lbm;
using namespace lbm::capi;

namespace lbm {
namespace capi {
thread_local std::string g_err;
int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
}  // namespace capi
}  // namespace lbm

static int validate(const lbm_desc* d) {
  if (!d) return fail(LBM_ERR_ARG, "desc is NULL");
  if (d->struct_size != (int32_t)sizeof(lbm_desc))
    return fail(LBM_ERR_ARG, "desc.struct_size mismatch (ABI drift)");
  if (d->dim != 2 && d->dim != 3) return fail(LBM_ERR_ARG, "dim must be 2 or 3");
  if (d->nx < 3 || d->ny < 3) return fail(LBM_ERR_ARG, "nx and ny must be >= 3");
  if (d->dim == 2 && d->nz != 1) return fail(LBM_ERR_ARG, "nz must be 1 for dim 2");
  if (d->dim == 3 && d->nz < 3) return fail(LBM_ERR_ARG, "nz must be >= 3 for dim 3");
  const double N = (double)d->nx * d->ny * d->nz;
  if (N * lat_q(d->dim) >= 2147483647.0)
    return fail(LBM_ERR_SIZE, "nx*ny*nz*Q must stay below 2^31 (32-bit cell indices)");
  if (d->collision != LBM_COLL_BGK && d->collision != LBM_COLL_MRT)
    return fail(LBM_ERR_ARG, "unknown collision");
  if (d->precision < LBM_PREC_FP32 || d->precision > LBM_PREC_FP64)
    return fail(LBM_ERR_ARG, "unknown precision");
  if (d->bulk_form < 0 || d->bulk_form > 3) return fail(LBM_ERR_ARG, "bulk_form must be 0, 1, 2 or 3");
  if (d->bulk_form == 3) {
    const char* why = dense_unsupported(*d);
    if (why) return fail(LBM_ERR_ARG, why);
  }
  if (d->eos != LBM_EOS_IDEAL_GAS && d->eos != LBM_EOS_INCOMPRESSIBLE)
    return fail(LBM_ERR_ARG, "unknown eos");
  if (d->thermal != LBM_THERMAL_NONE && d->thermal != LBM_THERMAL_CONJUGATE && d->thermal != LBM_THERMAL_TWOFIELD)
    return fail(LBM_ERR_ARG, "unknown thermal mode");
  if (d->pyro && d->thermal != LBM_THERMAL_CONJUGATE)
    return fail(LBM_ERR_ARG, "pyrolysis needs the conjugate thermal field (heat reaches a reacting cell through it)");
  if (!(d->nu > 0)) return fail(LBM_ERR_ARG, "nu must be > 0");
  if (d->viscosity != LBM_VISC_CONSTANT && d->viscosity != LBM_VISC_SUTHERLAND)
    return fail(LBM_ERR_ARG, "unknown viscosity model");
  if (d->viscosity == LBM_VISC_SUTHERLAND && (d->thermal == LBM_THERMAL_NONE || !(d->suth_A > 0)))
    return fail(LBM_ERR_ARG, "Sutherland viscosity needs the temperature field and suth_A > 0");
  if (d->thermal && !(d->tauT_fluid > 0.5 && d->tauT_solid > 0.5))
    return fail(LBM_ERR_ARG, "thermal tau must be > 0.5");
  if (d->porous < LBM_PORO_NONE || d->porous > LBM_PORO_DARCY_FORCHHEIMER)
    return fail(LBM_ERR_ARG, "unknown porous model");
  if (d->porous && (d->thermal == LBM_THERMAL_CONJUGATE || d->viscosity != LBM_VISC_CONSTANT))
    return fail(LBM_ERR_ARG, "porous cells run with constant viscosity, without temperature or with the two-field "
                             "temperature");
  if (d->porous && d->thermal == LBM_THERMAL_TWOFIELD &&
      !(d->cap_fluid > 0 && d->cap_solid > 0 && d->T_scale != 0 && d->Ts_scale != 0 && d->dt_phys > 0 &&
        (!d->radiation || d->dx_phys > 0)))
    return fail(LBM_ERR_ARG, "the heat exchange of porous cells needs cap_fluid, cap_solid, dt_phys > 0, non-zero "
                             "T_scale and Ts_scale, and dx_phys > 0 with radiation");
  if (d->fp16_rounding != LBM_FP16_STOCHASTIC && d->fp16_rounding != LBM_FP16_NEAREST)
    return fail(LBM_ERR_ARG, "fp16_rounding must be LBM_FP16_STOCHASTIC or LBM_FP16_NEAREST");
  if (d->tprop) {
    if ((d->tprop & ~7) || d->thermal == LBM_THERMAL_NONE || d->porous)
      return fail(LBM_ERR_ARG, "temperature-dependent thermal properties (tprop bits 0-2) need the conjugate or "
                               "two-field temperature, without porous cells");
    if ((d->tprop & 4) && ((d->tprop & 1) || !(d->tp_prandtl > 0)))
      return fail(LBM_ERR_ARG, "the fluid's Prandtl diffusivity (tprop bit 2) excludes bit 0 and needs tp_prandtl > 0");
    if (!(d->tp_dt > 0 && d->tp_dx2 > 0) || ((d->tprop & 2) && !(d->tp_rhos > 0)))
      return fail(LBM_ERR_ARG, "tprop needs tp_dt > 0, tp_dx2 > 0 and, for the solid, tp_rhos > 0");
    for (int ph = 0; ph < 2; ++ph) {
      if (!((d->tprop >> ph) & 1)) continue;
      bool ok = std::isfinite(d->tp_cap_Tmid[ph]) && std::isfinite(d->tp_cap_mul[ph]) && d->tp_cap_mul[ph] != 0;
      for (int i = 0; i < 5; ++i)
        ok = ok && std::isfinite(d->tp_cond[ph][i]) && std::isfinite(d->tp_cap_lo[ph][i]) &&
             std::isfinite(d->tp_cap_hi[ph][i]);
      if (!ok) return fail(LBM_ERR_ARG, "tprop coefficients must be finite and tp_cap_mul non-zero");
    }
  }
  if (d->radiation && !(d->porous && d->thermal == LBM_THERMAL_TWOFIELD))
    return fail(LBM_ERR_ARG, "radiation is a source of porous cells in the two-field temperature model");
  int nebb = 0, other = 0;
  for (int s = 0; s < 6; ++s) {
    if (d->side[s].active == LBM_SIDE_NEBB) ++nebb;
    else if (d->side[s].active) ++other;
  }
  if (nebb && (other || d->dim != 2 || d->thermal != LBM_THERMAL_NONE))
    return fail(LBM_ERR_ARG, "NEBB sides: 2D, without the temperature field, every active side NEBB "
                             "(the reference's NEBB exists in 2D only, with one model for all sides)");
  for (int s = 0; s < 6; ++s) {
    const lbm_side_desc& sd = d->side[s];
    if (sd.active < 0 || sd.active > LBM_SIDE_NEBB)
      return fail(LBM_ERR_ARG, "side active must be 0, 1 (NEE), 2 (ES) or 3 (NEBB)");
    if (sd.active == LBM_SIDE_NEBB && sd.v_type == LBM_BC_FLOWRATE)
      return fail(LBM_ERR_ARG, "the flow-rate inlet runs under NEE or ES");
    if (!sd.active) continue;
    if (d->dim == 2 && s >= 4) return fail(LBM_ERR_ARG, "z sides cannot be active in 2D");
    const int types[3] = {sd.v_type, sd.rho_type, sd.T_type};
    for (int i = 0; i < 3; ++i) {
      if (i == 0 && s == 0 && types[i] == LBM_BC_FLOWRATE) continue;
      if (types[i] < LBM_BC_PERIODIC || types[i] > LBM_BC_FIXEDVALUE)
        return fail(LBM_ERR_ARG, types[i] == LBM_BC_FLOWRATE ? "the flow-rate type is for the velocity of side 0 only"
                                                              : "bad side bc type");
    }
  }
  if ((d->side[0].active && d->side[1].active && d->nx < 4) ||
      (d->side[2].active && d->side[3].active && d->ny < 4) ||
      (d->side[4].active && d->side[5].active && d->nz < 4))
    return fail(LBM_ERR_ARG, "two active opposite sides need at least 4 cells between them");
  return LBM_OK;
}

// Sets bit 2 of *flag if a cell on an active (NEE) side, or its inner neighbour,
// is solid or porous: NEE replaces every population of a side cell from the
// post-stream state of the inner neighbour (src/LBM/LBM2D/_boundary.py:54-101), which
// presumes two fluid cells; solid cells here carry no flow populations, and the
// boundary pass takes a cell's moments without the porous velocity correction.
// poro: solid fraction per cell (float, or double when poro_f64), or null.
static __global__ void __launch_bounds__(256) check_sides_kernel(const uint8_t* mask, const void* poro, int poro_f64,
                                                                 int nx, int ny, int nz, int active, size_t N,
                                                                 int* flag) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += stride) {
    const bool porous = poro && (poro_f64 ? ((const double*)poro)[c] != 0.0 : ((const float*)poro)[c] != 0.0f);
    if (!(mask[c] & LBM_MASK_SOLID) && !porous) continue;
    const int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((size_t)nx * ny));
    const bool near = ((active & 1) && x <= 1) || ((active & 2) && x >= nx - 2) || ((active & 4) && y <= 1) ||
                      ((active & 8) && y >= ny - 2) || ((active & 16) && z <= 1) || ((active & 32) && z >= nz - 2);
    if (near) atomicOr(flag, 4);
  }
}

// Both parity bits of every mask byte from bit `bit` (the state a resumed run
// reads first); the reactive bit is kept.
static __global__ void __launch_bounds__(256) normalise_mask_kernel(uint8_t* mask, size_t N, int bit) {
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < N; c += stride) {
    const uint8_t m = mask[c];
    mask[c] = (uint8_t)((m & ~LBM_MASK_SOLID) | (((m >> bit) & 1) ? LBM_MASK_SOLID : 0u));
  }
}

// Side-layer check (check_sides_kernel); synchronises st when a side is active.
static int check_sides(lbm_handle* h, cudaStream_t st) {
  int active = 0;
  for (int s = 0; s < 6; ++s) if (h->d.side[s].active) active |= 1 << s;
  int flag = 0;
  LBM_CUDA_TRY(cudaMemsetAsync(scratch_err(h), 0, sizeof(int), st));
  if (active) {
    check_sides_kernel<<<2 * sm_count(), 256, 0, st>>>((const uint8_t*)h->ptr[LBM_FIELD_MASK],
                                                      h->d.porous ? h->ptr[LBM_FIELD_PORO] : nullptr,
                                                      h->d.precision == LBM_PREC_FP64, h->d.nx, h->d.ny, h->d.nz,
                                                      active, h->N, scratch_err(h));
    LBM_CUDA_TRY(cudaGetLastError());
    LBM_CUDA_TRY(cudaMemcpyAsync(&flag, scratch_err(h), sizeof(int), cudaMemcpyDeviceToHost, st));
    LBM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  if (flag & 4) {
    LBM_CUDA_TRY(cudaMemsetAsync(scratch_err(h), 0, sizeof(int), st));
    return fail(LBM_ERR_ARG,
                "a solid or porous cell lies on an active (NEE) side or next to one; the two outer layers of "
                "an active side must be fluid");
  }
  return LBM_OK;
}

// Cell lists of the step_list kernel from the (normalised) mask; runs after the
// equilibrium initialisation, on the caller's stream.
template <class Lt>
static int build_lists_t(lbm_handle* h, cudaStream_t st) {
  ListBuild a{};
  a.mask = (const uint8_t*)h->ptr[LBM_FIELD_MASK];
  a.nx = h->d.nx; a.ny = h->d.ny; a.nz = h->d.nz;
  a.active = 0;
  for (int s = 0; s < 6; ++s) if (h->d.side[s].active) a.active |= 1 << s;
  a.par = 0;
  a.thermal = h->d.thermal;
  a.N = h->N;
  a.nbb = h->L.list_nbb;
  a.blk = scratch_lblk(h);
  a.hdr = scratch_lhdr(h);
  a.ent_c = scratch_ent_c(h);
  a.ent_b = scratch_ent_b(h);
  a.pos = scratch_pos(h);
  a.solid_base = h->L.list_base;
  // padding entries everywhere (cell index 0xffffffff), no entry for any cell (-1)
  LBM_CUDA_TRY(cudaMemsetAsync(a.ent_c, 0xff, h->L.list_cap * 4, st));
  LBM_CUDA_TRY(cudaMemsetAsync(a.ent_b, 0xff, h->L.list_cap * 4, st));
  LBM_CUDA_TRY(cudaMemsetAsync(a.pos, 0xff, h->N * 4, st));
  list_count<Lt><<<a.nbb, 256, 0, st>>>(a);
  list_scan<Lt><<<1, 1024, 0, st>>>(a);
  list_scatter<Lt><<<a.nbb, 256, 0, st>>>(a);
  LBM_CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}
static int build_lists(lbm_handle* h, cudaStream_t st) {
  if (h->L.dense) {  // flip lists only: both empty
    LBM_CUDA_TRY(cudaMemsetAsync(scratch_lhdr(h), 0, kLhSlots * sizeof(int), st));
    return LBM_OK;
  }
  if (!h->L.list) return LBM_OK;
  return h->d.dim == 2 ? build_lists_t<Lattice<2>>(h, st) : build_lists_t<Lattice<3>>(h, st);
}


extern "C" {

int32_t lbm_abi_version(void) { return LBM_ABI_VERSION; }
const char* lbm_last_error(void) { return g_err.c_str(); }

int32_t lbm_required_bytes(const lbm_desc* d, int32_t field, size_t* bytes) {
  int rc = validate(d);
  if (rc) return rc;
  if (!bytes) return fail(LBM_ERR_ARG, "bytes is NULL");
  const size_t N = (size_t)d->nx * d->ny * d->nz;
  const size_t s = storage_bytes(d->precision), cb = compute_bytes(d->precision);
  switch (field) {
    case LBM_FIELD_F: *bytes = 2 * (size_t)lat_q(d->dim) * N * s; break;
    case LBM_FIELD_G: *bytes = d->thermal ? 2 * (size_t)lat_qt(d->dim) * N * s : 0; break;
    case LBM_FIELD_MASK: *bytes = N; break;
    case LBM_FIELD_ALPHA: *bytes = d->pyro ? N * cb : 0; break;
    case LBM_FIELD_REL: *bytes = d->pyro ? 2 * N * cb : 0; break;
    case LBM_FIELD_RHO: *bytes = N * cb; break;
    case LBM_FIELD_U: *bytes = 3 * N * cb; break;
    case LBM_FIELD_T: *bytes = d->thermal ? (porous_heat(*d) ? 2 : 1) * N * cb : 0; break;
    case LBM_FIELD_UPREV: *bytes = 3 * N * 4; break;
    case LBM_FIELD_INLET: *bytes = has_flowrate(*d) ? inlet_elems(*d) * cb : 0; break;
    case LBM_FIELD_PORO: *bytes = d->porous ? N * cb : 0; break;
    case LBM_FIELD_DARCY: *bytes = d->porous >= LBM_PORO_DARCY ? N * cb : 0; break;
    case LBM_FIELD_FORCH: *bytes = d->porous == LBM_PORO_DARCY_FORCHHEIMER ? N * cb : 0; break;
    case LBM_FIELD_GS: *bytes = porous_heat(*d) ? 2 * (size_t)lat_qt(d->dim) * N * s : 0; break;
    case LBM_FIELD_XHEAT: *bytes = porous_heat(*d) ? 3 * N * cb : 0; break;
    case LBM_FIELD_SCRATCH: {
      const Launch L = plan(*d, default_tx(*d));
      *bytes = scratch_bytes(L);
      break;
    }
    default: return fail(LBM_ERR_ARG, "unknown field id");
  }
  return LBM_OK;
}

int32_t lbm_create(const lbm_desc* d, lbm_handle** out) {
  int rc = validate(d);
  if (rc) return rc;
  if (!out) return fail(LBM_ERR_ARG, "out is NULL");
  lbm_handle* h = new lbm_handle();
  if (cudaGetDevice(&h->device) != cudaSuccess) {
    cudaGetLastError();
    h->device = 0;
  }
  h->d = *d;
  h->N = (size_t)d->nx * d->ny * d->nz;
  for (int i = 0; i < LBM_NUM_FIELDS; ++i) { h->ptr[i] = nullptr; h->bytes[i] = 0; }
  h->step = 0;
  h->L = plan(*d, default_tx(*d));
  h->diag_valid = false;
  h->initialised = false;
  *out = h;
  return LBM_OK;
}

int32_t lbm_destroy(lbm_handle* h) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (h) {
    if (h->ev_fork) cudaEventDestroy(h->ev_fork);
    if (h->ev_join) cudaEventDestroy(h->ev_join);
    if (h->side) cudaStreamDestroy(h->side);
  }
  delete h;
  return LBM_OK;
}

int32_t lbm_bind(lbm_handle* h, int32_t field, void* ptr, size_t bytes) {
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  if (field < 0 || field >= LBM_NUM_FIELDS) return fail(LBM_ERR_ARG, "unknown field id");
  size_t need = 0;
  int rc = lbm_required_bytes(&h->d, field, &need);
  if (rc) return rc;
  if (field == LBM_FIELD_SCRATCH) need = scratch_bytes(h->L);  // the handle's own launch plan
  if (bytes < need)
    return fail(LBM_ERR_ARG, "buffer for field " + std::to_string(field) + " too small: " +
                                 std::to_string(bytes) + " < " + std::to_string(need));
  if (need > 0 && !ptr) return fail(LBM_ERR_ARG, "NULL device pointer");
  if (ptr && ((uintptr_t)ptr % 16) != 0) return fail(LBM_ERR_ARG, "device pointer not 16-byte aligned");
  h->ptr[field] = ptr;
  h->bytes[field] = bytes;
  return LBM_OK;
}

int64_t lbm_step_count(const lbm_handle* h) { return h ? h->step : -1; }

int32_t lbm_set_wait_limit(lbm_handle* h, uint32_t tries) {
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  h->wait_spins = tries;
  return LBM_OK;
}

int32_t lbm_bulk_form(const lbm_handle* h) {
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  return h->L.dense ? 3 : (h->L.list ? 2 : 1);
}

}  // extern "C"

// Calls fn.template operator()<Lattice, Storage>() for the handle's dim/precision.
template <class Fn>
static int with_types(lbm_handle* h, Fn&& fn) {
  const int dim = h->d.dim, prec = h->d.precision;
  if (dim == 2 && prec == LBM_PREC_FP32) return fn(Lattice<2>{}, float{});
  if (dim == 3 && prec == LBM_PREC_FP32) return fn(Lattice<3>{}, float{});
  if (dim == 2 && prec == LBM_PREC_FP16) return fn(Lattice<2>{}, __half{});
  if (dim == 3 && prec == LBM_PREC_FP16) return fn(Lattice<3>{}, __half{});
  if (dim == 2 && prec == LBM_PREC_FP64) return fn(Lattice<2>{}, double{});
  if (dim == 3 && prec == LBM_PREC_FP64) return fn(Lattice<3>{}, double{});
  return fail(LBM_ERR_ARG, "unsupported dim/precision");
}

static int check_bound(lbm_handle* h) {
  const int need[] = {LBM_FIELD_F, LBM_FIELD_MASK, LBM_FIELD_SCRATCH};
  for (int f : need)
    if (!h->ptr[f]) return fail(LBM_ERR_UNBOUND, "field " + std::to_string(f) + " is not bound");
  if (h->d.thermal && !h->ptr[LBM_FIELD_G]) return fail(LBM_ERR_UNBOUND, "field G is not bound");
  if (h->d.pyro && (!h->ptr[LBM_FIELD_ALPHA] || !h->ptr[LBM_FIELD_REL]))
    return fail(LBM_ERR_UNBOUND, "pyrolysis needs ALPHA and REL bound");
  if (has_flowrate(h->d) && !h->ptr[LBM_FIELD_INLET])
    return fail(LBM_ERR_UNBOUND, "a flow-rate inlet needs INLET bound");
  if (h->d.porous && (!h->ptr[LBM_FIELD_PORO] || (h->d.porous >= LBM_PORO_DARCY && !h->ptr[LBM_FIELD_DARCY]) ||
                      (h->d.porous == LBM_PORO_DARCY_FORCHHEIMER && !h->ptr[LBM_FIELD_FORCH])))
    return fail(LBM_ERR_UNBOUND, "porous cells need PORO (and DARCY / FORCH for their models) bound");
  if (porous_heat(h->d) && (!h->ptr[LBM_FIELD_GS] || !h->ptr[LBM_FIELD_XHEAT]))
    return fail(LBM_ERR_UNBOUND, "porous cells with two temperature fields need GS and XHEAT bound");
  return LBM_OK;
}

// ---------------------------------------------------------------- batches
namespace {

size_t params_bytes(const lbm_desc& d) {
  if (d.precision == LBM_PREC_FP64) return sizeof(StepParams<double>);
  if (d.precision == LBM_PREC_FP16) return sizeof(StepParams<__half>);
  return sizeof(StepParams<float>);
}

// Checks the members of a batch and reads their list headers (synchronises st).
int batch_members(lbm_handle* const* hs, int32_t n, cudaStream_t st, std::vector<std::vector<int>>& hdr) {
  if (!hs || n < 1 || !hs[0]) return fail(LBM_ERR_ARG, "a batch needs at least one lattice");
  const lbm_desc& d0 = hs[0]->d;
  for (int i = 0; i < n; ++i) {
    lbm_handle* h = hs[i];
    if (!h) return fail(LBM_ERR_ARG, "batch member " + std::to_string(i) + " is NULL");
    int rc = check_bound(h);
    if (rc) return rc;
    if (!h->initialised) return fail(LBM_ERR_ARG, "batch member " + std::to_string(i) + " is not initialised");
    if (!h->L.list)
      return fail(LBM_ERR_ARG, "batch member " + std::to_string(i) + " does not use cell lists (set bulk_form = 2)");
    if (h->d.dim != d0.dim || h->d.precision != d0.precision || h->d.collision != d0.collision ||
        h->d.thermal != d0.thermal || h->d.pyro != d0.pyro || h->d.viscosity != d0.viscosity ||
        (h->d.tprop != 0) != (d0.tprop != 0))
      return fail(LBM_ERR_ARG, "batch members must share dim, precision, collision, viscosity, thermal, pyro and "
                               "whether tprop is set");
    if (h->device != hs[0]->device) return fail(LBM_ERR_ARG, "batch members must live on one device");
    if ((h->step & 1) != (hs[0]->step & 1)) return fail(LBM_ERR_ARG, "batch members must be at the same step parity");
    if (has_flowrate(h->d)) return fail(LBM_ERR_ARG, "batch members cannot have a flow-rate inlet");
    if (porous_heat(h->d))
      return fail(LBM_ERR_ARG, "batch members cannot have porous cells with two temperature fields");
    for (int j = 0; j < i; ++j)
      if (hs[j] == h) return fail(LBM_ERR_ARG, "a lattice appears twice in the batch");
  }
  hdr.assign(n, std::vector<int>(kLhSlots));
  for (int i = 0; i < n; ++i)
    LBM_CUDA_TRY(cudaMemcpyAsync(hdr[i].data(), scratch_lhdr(hs[i]), kLhSlots * sizeof(int), cudaMemcpyDeviceToHost, st));
  LBM_CUDA_TRY(cudaStreamSynchronize(st));
  return LBM_OK;
}

// Chunk table: per lattice its current fluid and solid chunks interleaved in
// proportion, all lattices in order; then every lattice's room for cells that turn
// fluid (empty until they do).  Boundary block table: (lattice, face, block).
void batch_tables(lbm_handle* const* hs, int32_t n, const std::vector<std::vector<int>>& hdr,
                  std::vector<int2>& chunks, std::vector<int4>& bc) {
  chunks.clear();
  bc.clear();
  std::vector<int2> room;
  for (int i = 0; i < n; ++i) {
    const std::vector<int>& H = hdr[i];
    const int fg = H[kLhFg], fe = H[kLhFe], sb = H[kLhSb], sg = H[kLhSg], se = H[kLhSe];
    const int cf = (fe + 31) / 32, cs = (se - sb + 31) / 32;
    const int cap = std::min(sb, 32 * cf + (se - sb));  // fluid entries the flips can add
    const int cr = (cap + 31) / 32 - cf;
    const long total = (long)cf + cs;
    long fdone = 0;
    for (long j = 0; j < total; ++j) {
      const long f1 = ((j + 1) * cf) / total;
      if (f1 > fdone) {
        const int base = (int)(fdone * 32);
        chunks.push_back(make_int2(i << 2 | 2 | (base < fg ? 1 : 0), base));
        fdone = f1;
      } else {
        const int base = sb + (int)((j - fdone) * 32);
        chunks.push_back(make_int2(i << 2 | (base < sg ? 1 : 0), base));
      }
    }
    for (int r = 0; r < cr; ++r) room.push_back(make_int2(i << 2 | 2, 32 * (cf + r)));
    const lbm_desc& d = hs[i]->d;
    for (int f = 0; f < 6; ++f) {
      if (!d.side[f].active) continue;
      const int cells = f < 2 ? d.ny * d.nz : (f < 4 ? d.nx * d.nz : d.nx * d.ny);
      for (int b = 0; b < (cells + 127) / 128; ++b) bc.push_back(make_int4(i, f, b, 0));
    }
  }
  chunks.insert(chunks.end(), room.begin(), room.end());
}

size_t batch_bytes(lbm_handle* const* hs, int32_t n, size_t nchunks, size_t nbc) {
  const size_t p = ((size_t)n * 2 * params_bytes(hs[0]->d) + 255) / 256 * 256;
  const size_t c = (nchunks * sizeof(int2) + 255) / 256 * 256;
  return p + c + nbc * sizeof(int4) + 256;
}

}  // namespace

extern "C" {

int32_t lbm_set_sides(lbm_handle* h, const lbm_side_desc* host_sides, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h || !host_sides) return fail(LBM_ERR_ARG, "NULL argument");
  if (!h->ptr[LBM_FIELD_SCRATCH]) return fail(LBM_ERR_UNBOUND, "scratch is not bound");
  for (int s = 0; s < 6; ++s) {
    const lbm_side_desc& a = h->d.side[s];
    const lbm_side_desc& b = host_sides[s];
    if (a.active != b.active || a.v_type != b.v_type || a.rho_type != b.rho_type || a.T_type != b.T_type)
      return fail(LBM_ERR_ARG, "lbm_set_sides may change values only, not side types");
  }
  memcpy(h->d.side, host_sides, sizeof(h->d.side));
  LBM_CUDA_TRY(cudaMemcpyAsync(scratch_sides(h), host_sides, kCtrlBytes, cudaMemcpyHostToDevice,
                               (cudaStream_t)stream));
  return LBM_OK;
}

int32_t lbm_init_equilibrium(lbm_handle* h, const float* rho, const float* u, const float* T,
                             const float* alpha, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  int rc = check_bound(h);
  if (rc) return rc;
  if (!rho || !u) return fail(LBM_ERR_ARG, "rho and u are required");
  if (h->d.thermal && !T) return fail(LBM_ERR_ARG, "T is required with the thermal field");
  cudaStream_t st = (cudaStream_t)stream;
  LBM_CUDA_TRY(cudaMemcpyAsync(scratch_sides(h), h->d.side, kCtrlBytes, cudaMemcpyHostToDevice, st));
  const int solid_bit = (int)(h->step & 1);
  rc = with_types(h, [&](auto lat, auto s) -> int {
    using Lt = decltype(lat);
    using S = decltype(s);
    // buf = 1 makes fB/gB/relB the buffers that the first step (parity 0) reads
    StepParams<S> p = make_params<S>(h, 1);
    rc = dispatch_init<Lt, S>(h, p, rho, u, T, alpha, solid_bit, st);
    if (rc == LBM_OK && p.inlet)
      inlet_seed<<<1, 1024, 0, st>>>(p.inlet, rho, p.nx, p.ny, p.nz, h->d.side[0].v[0]);
    return rc;
  });
  if (rc) return rc;
  LBM_CUDA_TRY(cudaGetLastError());
  rc = check_sides(h, st);
  if (rc) return rc;
  rc = build_lists(h, st);
  if (rc) return rc;
  h->initialised = true;
  h->step = 0;
  h->diag_valid = false;
  return LBM_OK;
}

int32_t lbm_resume(lbm_handle* h, int64_t step, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  if (step < 0) return fail(LBM_ERR_ARG, "step must be >= 0");
  int rc = check_bound(h);
  if (rc) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  LBM_CUDA_TRY(cudaMemcpyAsync(scratch_sides(h), h->d.side, kCtrlBytes, cudaMemcpyHostToDevice, st));
  normalise_mask_kernel<<<2 * sm_count(), 256, 0, st>>>((uint8_t*)h->ptr[LBM_FIELD_MASK], h->N, (int)(step & 1));
  LBM_CUDA_TRY(cudaGetLastError());
  rc = check_sides(h, st);
  if (rc) return rc;
  rc = build_lists(h, st);  // both parity bits are equal now, so parity 0 lists the current state
  if (rc) return rc;
  h->initialised = true;
  h->step = step;
  h->diag_valid = false;
  return LBM_OK;
}

int32_t lbm_step(lbm_handle* h, int32_t n, int32_t flags, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  if (n < 0) return fail(LBM_ERR_ARG, "n must be >= 0");
  int rc = check_bound(h);
  if (rc) return rc;
  if ((flags & LBM_STEP_MACRO) && (!h->ptr[LBM_FIELD_RHO] || !h->ptr[LBM_FIELD_U] ||
                                   (h->d.thermal && !h->ptr[LBM_FIELD_T])))
    return fail(LBM_ERR_UNBOUND, "LBM_STEP_MACRO needs RHO, U (and T) bound");
  if ((flags & LBM_STEP_RESIDUAL) && !h->ptr[LBM_FIELD_UPREV])
    return fail(LBM_ERR_UNBOUND, "LBM_STEP_RESIDUAL needs UPREV bound");
  cudaStream_t st = (cudaStream_t)stream;
  for (int i = 0; i < n; ++i) {
    const int buf = (int)(h->step & 1);
    const int fl = (i == n - 1) ? flags : 0;
    rc = with_types(h, [&](auto lat, auto s) -> int {
      using Lt = decltype(lat);
      using S = decltype(s);
      StepParams<S> p = make_params<S>(h, buf);
      p.flags = fl;
      return dispatch_step<Lt, S>(h, p, st);
    });
    if (rc) return rc;
    if (fl) {
      launch_reduce(h, st);
      h->diag_valid = true;
    }
    h->step += 1;
  }
  LBM_CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}

int32_t lbm_compute_macro(lbm_handle* h, int32_t flags, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  if (h->step < 1) return fail(LBM_ERR_ARG, "no step taken yet: the initial fields are the state");
  if (flags & ~(LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL)) return fail(LBM_ERR_ARG, "bad flags");
  if (!flags) return LBM_OK;
  int rc = check_bound(h);
  if (rc) return rc;
  if ((flags & LBM_STEP_MACRO) && (!h->ptr[LBM_FIELD_RHO] || !h->ptr[LBM_FIELD_U] ||
                                   (h->d.thermal && !h->ptr[LBM_FIELD_T])))
    return fail(LBM_ERR_UNBOUND, "LBM_STEP_MACRO needs RHO, U (and T) bound");
  if ((flags & LBM_STEP_RESIDUAL) && !h->ptr[LBM_FIELD_UPREV])
    return fail(LBM_ERR_UNBOUND, "LBM_STEP_RESIDUAL needs UPREV bound");
  cudaStream_t st = (cudaStream_t)stream;
  const int buf = (int)((h->step - 1) & 1);
  rc = with_types(h, [&](auto lat, auto s) -> int {
    using Lt = decltype(lat);
    using S = decltype(s);
    StepParams<S> p = make_params<S>(h, buf);
    p.flags = flags | kStepPeek;
    return dispatch_step<Lt, S>(h, p, st);
  });
  if (rc) return rc;
  launch_reduce(h, st);
  h->diag_valid = true;
  LBM_CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}

int32_t lbm_read_diag(lbm_handle* h, lbm_diag* out, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h || !out) return fail(LBM_ERR_ARG, "NULL argument");
  if (!h->diag_valid) return fail(LBM_ERR_ARG, "no diagnostics: call lbm_step with LBM_STEP_DIAG");
  double v[kNumDiag];
  int err = 0;
  cudaStream_t st = (cudaStream_t)stream;
  LBM_CUDA_TRY(cudaMemcpyAsync(v, scratch_final(h), sizeof(v), cudaMemcpyDeviceToHost, st));
  LBM_CUDA_TRY(cudaMemcpyAsync(&err, scratch_err(h), sizeof(int), cudaMemcpyDeviceToHost, st));
  LBM_CUDA_TRY(cudaStreamSynchronize(st));
  if (err & 1) return fail(LBM_ERR_TIMEOUT, "a staged-load wait in the step kernel timed out; the state is invalid");
  if (err & 2) return fail(LBM_ERR_CUDA, "the fluid cell list overflowed; the state is invalid");
  out->mass = v[0]; out->energy = v[1]; out->solid_alpha = v[2]; out->umax = v[3];
  out->Tmin = v[4]; out->Tmax = v[5]; out->nonfinite = v[6]; out->nfluid = v[7];
  out->res_num = v[8]; out->res_den = v[9];
  out->step = h->step;
  if (v[6] > 0) return fail(LBM_ERR_NONFINITE, "diagnostics saw NaN/Inf");
  return LBM_OK;
}

int32_t lbm_read_diag_async(lbm_handle* h, lbm_diag* out, int32_t* err, void* stream) {
  DeviceScope dev_scope(h ? h->device : -1);
  if (!h || !out || !err) return fail(LBM_ERR_ARG, "NULL argument");
  if (!h->diag_valid) return fail(LBM_ERR_ARG, "no diagnostics: call lbm_step with LBM_STEP_DIAG");
  static_assert(sizeof(double) * kNumDiag == offsetof(lbm_diag, step), "lbm_diag leads with the partial slots");
  cudaStream_t st = (cudaStream_t)stream;
  out->step = h->step;
  LBM_CUDA_TRY(cudaMemcpyAsync(out, scratch_final(h), sizeof(double) * kNumDiag, cudaMemcpyDeviceToHost, st));
  LBM_CUDA_TRY(cudaMemcpyAsync(err, scratch_err(h), sizeof(int32_t), cudaMemcpyDeviceToHost, st));
  return LBM_OK;
}

int32_t lbm_batch_required_bytes(lbm_handle* const* hs, int32_t n, void* stream, size_t* bytes) {
  DeviceScope dev_scope(hs && n > 0 && hs[0] ? hs[0]->device : -1);
  if (!bytes) return fail(LBM_ERR_ARG, "bytes is NULL");
  std::vector<std::vector<int>> hdr;
  int rc = batch_members(hs, n, (cudaStream_t)stream, hdr);
  if (rc) return rc;
  std::vector<int2> chunks;
  std::vector<int4> bc;
  batch_tables(hs, n, hdr, chunks, bc);
  *bytes = batch_bytes(hs, n, chunks.size(), bc.size());
  return LBM_OK;
}

int32_t lbm_batch_create(lbm_handle* const* hs, int32_t n, void* dev_scratch, size_t bytes, void* stream,
                         lbm_batch** out) {
  DeviceScope dev_scope(hs && n > 0 && hs[0] ? hs[0]->device : -1);
  if (!out) return fail(LBM_ERR_ARG, "out is NULL");
  if (!dev_scratch) return fail(LBM_ERR_ARG, "the batch needs a device buffer");
  cudaStream_t st = (cudaStream_t)stream;
  std::vector<std::vector<int>> hdr;
  int rc = batch_members(hs, n, st, hdr);
  if (rc) return rc;
  std::vector<int2> chunks;
  std::vector<int4> bc;
  batch_tables(hs, n, hdr, chunks, bc);
  const size_t need = batch_bytes(hs, n, chunks.size(), bc.size());
  if (bytes < need) return fail(LBM_ERR_SIZE, "batch buffer too small: need " + std::to_string(need) + " bytes");
  if (chunks.size() > (size_t)INT32_MAX || bc.size() > (size_t)INT32_MAX) return fail(LBM_ERR_SIZE, "batch too large");
  lbm_batch* b = new lbm_batch();
  b->hs.assign(hs, hs + n);
  b->scratch = dev_scratch;
  b->bytes = bytes;
  const size_t pb = params_bytes(hs[0]->d);
  char* base = (char*)dev_scratch;
  b->params = base;
  b->chunks = (int2*)(base + ((size_t)n * 2 * pb + 255) / 256 * 256);
  b->nchunks = (int)chunks.size();
  b->bc = (int4*)((char*)b->chunks + (chunks.size() * sizeof(int2) + 255) / 256 * 256);
  b->nbc = (int)bc.size();
  b->list_blocks = (int)std::max<long>(1, std::min<long>(((long)chunks.size() + 3) / 4,
                                                          (long)sm_count() * list_blocks_per_sm(hs[0]->d.precision == LBM_PREC_FP64)));
  b->flip_blocks = 4;
  // parameters of every lattice at both parities, staged on the host
  std::vector<unsigned char> host((size_t)n * 2 * pb);
  rc = with_types(hs[0], [&](auto lat, auto s) -> int {
    using S = decltype(s);
    (void)lat;
    for (int i = 0; i < n; ++i)
      for (int par = 0; par < 2; ++par) {
        StepParams<S> p = make_params<S>(hs[i], par);
        std::memcpy(host.data() + ((size_t)i * 2 + par) * pb, &p, pb);
      }
    return LBM_OK;
  });
  if (rc) { delete b; return rc; }
  cudaError_t e = cudaMemcpyAsync(b->params, host.data(), host.size(), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !chunks.empty())
    e = cudaMemcpyAsync(b->chunks, chunks.data(), chunks.size() * sizeof(int2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess && !bc.empty())
    e = cudaMemcpyAsync(b->bc, bc.data(), bc.size() * sizeof(int4), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // the host staging vectors go out of scope
  if (e != cudaSuccess) {
    delete b;
    return fail(LBM_ERR_CUDA, std::string("batch tables: ") + cudaGetErrorString(e));
  }
  *out = b;
  return LBM_OK;
}

int32_t lbm_batch_step(lbm_batch* b, int32_t n, void* stream) {
  DeviceScope dev_scope(b && !b->hs.empty() ? b->hs[0]->device : -1);
  if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
  if (n < 0) return fail(LBM_ERR_ARG, "n must be >= 0");
  cudaStream_t st = (cudaStream_t)stream;
  for (int i = 0; i < n; ++i) {
    const int rc = with_types(b->hs[0], [&](auto lat, auto s) -> int {
      using Lt = decltype(lat);
      using S = decltype(s);
      return dispatch_batch<Lt, S>(b, st);
    });
    if (rc) return rc;
    for (lbm_handle* h : b->hs) { h->step += 1; h->diag_valid = false; }
  }
  LBM_CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}

int32_t lbm_batch_set_blocks(lbm_batch* b, int32_t blocks_per_sm) {
  if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
  const int cap = list_blocks_per_sm(b->hs[0]->d.precision == LBM_PREC_FP64);  // resident blocks at the register cap
  if (blocks_per_sm < 1 || blocks_per_sm > cap)
    return fail(LBM_ERR_ARG, "blocks_per_sm must be 1.." + std::to_string(cap));
  b->list_blocks = (int)std::max<long>(1, std::min<long>(((long)b->nchunks + 3) / 4, (long)sm_count() * blocks_per_sm));
  return LBM_OK;
}

int32_t lbm_advance(lbm_handle* h, int32_t n) {
  if (!h) return fail(LBM_ERR_ARG, "handle is NULL");
  if (n < 0 || (n & 1)) return fail(LBM_ERR_ARG, "n must be even and >= 0 (a captured sequence keeps the parity)");
  h->step += n;
  h->diag_valid = false;
  return LBM_OK;
}

int32_t lbm_batch_advance(lbm_batch* b, int32_t n) {
  if (!b) return fail(LBM_ERR_ARG, "batch is NULL");
  if (n < 0 || (n & 1)) return fail(LBM_ERR_ARG, "n must be even and >= 0 (a captured sequence keeps the parity)");
  for (lbm_handle* h : b->hs) { h->step += n; h->diag_valid = false; }
  return LBM_OK;
}

int32_t lbm_batch_destroy(lbm_batch* b) {
  DeviceScope dev_scope(b && !b->hs.empty() ? b->hs[0]->device : -1);
  delete b;
  return LBM_OK;
}

}  // extern "C"
