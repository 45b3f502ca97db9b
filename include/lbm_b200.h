/*
 * lbm_b200.h -- C ABI of the sm_100a lattice update of LBM_porousChem.
 *
 * The reference has no FFI: its solver object is the plug-in and its Taichi
 * kernels are methods of the @ti.data_oriented solver class
 * (src/LBM/LBM2D/__init__.py:29-70, src/LBM/LBM3D/__init__.py:11-62), selected
 * by src/LBM/app.py:32-58.  Each entry point below replaces one piece of that
 * class's hot path; the Python host layer (lbm_porouschem_b200.solver) keeps
 * the class surface and calls these through ctypes.
 *
 * Conventions
 *  - Plain C types only; no exceptions cross the ABI.  Every call returns an
 *    int32 status (LBM_OK = 0); lbm_last_error() gives a message for the
 *    calling thread's last failure.
 *  - Device memory is owned by the caller (torch tensors on the Python side)
 *    and handed over with lbm_bind(); sizes come from lbm_required_bytes().
 *  - All GPU work is issued on the caller's stream (a cudaStream_t passed as
 *    void*; NULL = legacy default stream).  One handle per host thread.
 *  - Cell index c = x + nx*(y + ny*z) (x fastest).  A field shaped (nx,ny,nz)
 *    in the reference's numpy convention is this layout in Fortran order.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_ABI_VERSION 1

#if defined(__GNUC__)
#define LBM_API __attribute__((visibility("default")))
#else
#define LBM_API
#endif

/* status codes */
#define LBM_OK 0
#define LBM_ERR_ARG 1        /* bad argument or descriptor */
#define LBM_ERR_UNBOUND 2    /* a required field has no device buffer */
#define LBM_ERR_CUDA 3       /* a CUDA call failed */
#define LBM_ERR_NONFINITE 4  /* diagnostics saw NaN/Inf */
#define LBM_ERR_SIZE 5       /* a size exceeds a fixed limit */
#define LBM_ERR_TIMEOUT 6    /* a bounded wait inside a kernel gave up (state invalid) */

/* descriptor enums */
#define LBM_COLL_BGK 0
#define LBM_COLL_MRT 1
#define LBM_PREC_FP32 0
#define LBM_PREC_FP16 1 /* FP16 storage of f - w*rho0 and g - wt*T0, FP32 arithmetic */
#define LBM_PREC_FP64 2
/* Rounding of the temperature populations in FP16 storage: stochastic (default; a change
 * below half a unit in the last place survives on average, so slow diffusion does not
 * stall) or to nearest (about 12 % faster at 256^3, with a temperature error several times
 * larger over long runs).  The flow populations round to nearest. */
#define LBM_FP16_STOCHASTIC 0
#define LBM_FP16_NEAREST 1
#define LBM_VISC_CONSTANT 0      /* nu (util/flag.py VISCOSITY_MODEL.CONSTANT) */
#define LBM_VISC_SUTHERLAND 1    /* per cell from its temperature; needs the temperature field */

/* Porous cells (lbm_desc.porous): cells whose solid fraction s (LBM_FIELD_PORO) lies
 * between 0 and 1 are porous, eps = 1 - s (src/LBM/util/flag.py PORO_MODEL; set_poro_Darcy /
 * set_poro_Darcy_Forchheimer, src/LBM/LBM2D/_io.py:152-172).  Such a cell relaxes towards
 * the eps-equilibrium (src/LBM/LBM2D/_evolution.py:213-225), feels the drag of its model
 * through the Guo term (:254-298; the 3D solver takes the lattice viscosity there,
 * LBM3D/_evolution.py:262-278) and has its velocity corrected after the moments
 * (:131-151).  Cells with s >= 1 are the solid of the mask; s = 0 is fluid.  Constant
 * viscosity; the two outer cell layers of an active side must have s = 0.  Temperature:
 * none, or LBM_THERMAL_TWOFIELD, where a porous cell carries both fields, TF in
 * LBM_FIELD_G and TS in LBM_FIELD_GS.  TF lives in cells with s < 1 and bounces back at
 * pure-solid neighbours; TS lives in cells with s > 0 and bounces back at pure-fluid
 * neighbours (src/LBM/LBM2D/_evolution.py:30-100).  In a porous cell the two exchange
 * heat, dH = h a (T_f,phys - T_s,phys) dt, TS gaining dH/(c_s rhos Ts_scale) and TF losing
 * dH/(c_f rho T_scale), and with lbm_desc.radiation its surface radiates
 * q = e sigma a_r/dx (T_ambient^4 - T_s,phys^4), TS gaining q dt/(c_s rhos Ts_scale), as
 * sources of the next collision (TF's enters as geq(dS, u), TS's as w dS) (:186-202,
 * src/LBM/LBM2D/_thermal.py:213-220; 3D LBM3D/_evolution.py:179-195).  Per cell
 * (LBM_FIELD_XHEAT): h a, rhos and e a_r. */
#define LBM_PORO_NONE 0
#define LBM_PORO_ERGUN 1              /* SPHERICAL: permeability eps^3/(1.000001-eps)^2, Ergun drag */
#define LBM_PORO_DARCY 2              /* coefficient LBM_FIELD_DARCY per cell */
#define LBM_PORO_DARCY_FORCHHEIMER 3  /* LBM_FIELD_DARCY and LBM_FIELD_FORCH per cell */
#define LBM_EOS_IDEAL_GAS 0      /* util/flag.py:64-67 FLUID_STATE_EQUATION */
#define LBM_EOS_INCOMPRESSIBLE 1
#define LBM_THERMAL_NONE 0
#define LBM_THERMAL_CONJUGATE 1  /* one temperature distribution over fluid and solid */
#define LBM_THERMAL_TWOFIELD 2   /* the reference's TF (fluid) and TS (solid) fields: with a binary
                                    mask they never exchange heat, so fluid-solid links are
                                    adiabatic (src/LBM/LBM2D/_evolution.py:69-95, :197-200) */
#define LBM_BC_PERIODIC 0        /* util/flag.py:89-94 BC */
#define LBM_BC_ZEROGRADIENT 1
#define LBM_BC_FIXEDVALUE 2
/* Velocity type of side 0 (x-) only: the reference's flow-rate inlet BC_FLOW.inlet_flow
 * (src/LBM/LBM2D/_boundary.py:324-333, _initialize.py:67-73).  side[0].v[0] is the
 * target flow rate F (sum of rho*u_x over the side's cells, lattice units).  Before
 * each step, with flow0 = sum of rho*u_x over the side's cells and u1(j) the velocity
 * of the cell behind side cell j (x = 1), both as the previous step left them, side
 * cell j takes the velocity (0.01*F/flow0 + 0.99) * u1(j).  As the reference's
 * init_boundary does, lbm_init_equilibrium gives the columns x = 0 and 1 the velocity
 * (v0, 0, 0), v0 = F/ny/nz, in place of the u plane's (the reference writes it into
 * the macro velocity that its first collision reads; here the populations start at
 * that equilibrium).  The controller's state lives in LBM_FIELD_INLET.  A
 * proportional controller: its steady flux is F only where u(x = 0) = u(x = 1). */
#define LBM_BC_FLOWRATE 3

/* mask byte: bit0/bit1 = solid at even/odd step parity, bit2 = reactive solid */
#define LBM_MASK_SOLID 3u
#define LBM_MASK_REACTIVE 4u

/* One domain side: 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+  (reference side order,
 * src/LBM/LBM3D/_core.py:72).  active = 1 applies non-equilibrium
 * extrapolation (BC_MODEL.NEE, src/LBM/LBM2D/_boundary.py:17-101) on that
 * side; 2 the equilibrium scheme (BC_MODEL.ES, src/LBM/LBM2D/_boundary.py:229-315,
 * LBM3D/_boundary.py:145-274: the side cell's flow populations are feq(rho_b, u_b)
 * alone, its temperature is extrapolated as under NEE); 0 leaves it periodic. */
#define LBM_SIDE_NEE 1
#define LBM_SIDE_ES 2
/* 3: non-equilibrium bounce-back (Zou & He; BC_MODEL.NEBB, src/LBM/LBM2D/_boundary.py:103-226):
 * 2D without the temperature field, every active side NEBB.  A side cell keeps its own
 * post-stream populations and the ones entering from outside are rebuilt so that it takes
 * the side's velocity (v_type fixed) or density (rho_type fixed); an x side treats rows
 * 1 .. ny-2, a y side every column, as the reference's two loops do. */
#define LBM_SIDE_NEBB 3
typedef struct lbm_side_desc {
  int32_t active;
  int32_t v_type;   /* LBM_BC_*, velocity  (set_BC mapping src/LBM/LBM2D/_io.py:385-402) */
  int32_t rho_type; /* LBM_BC_*, density */
  int32_t T_type;   /* LBM_BC_*, temperature distribution (_scalarField.py:83-122) */
  double v[3];
  double rho;
  double T;         /* normalised temperature */
} lbm_side_desc;

typedef struct lbm_desc {
  int32_t struct_size;  /* = sizeof(lbm_desc); guards ABI drift */
  int32_t dim;          /* 2: D2Q9 + D2Q5, 3: D3Q19 + D3Q7 */
  int32_t nx, ny, nz;   /* nz = 1 for dim 2 */
  int32_t collision;    /* LBM_COLL_* */
  int32_t precision;    /* LBM_PREC_* */
  int32_t eos;          /* LBM_EOS_* */
  int32_t thermal;      /* LBM_THERMAL_* */
  int32_t pyro;         /* 1: Arrhenius pyrolysis with solid->fluid flip (needs the conjugate field) */
  int32_t half_force_velocity; /* 1: u includes F/2 (reference: 0) */
  int32_t bulk_form;    /* 0: cell lists from 65536 cells, else tile; 1: tile; 2: cell lists;
                           3: dense TMA-staged tiles (3D; nx % 32, ny % 4, nz % 2 == 0;
                           no two-field temperature) */
  double nu;            /* lattice viscosity visco*dt/dx^2 (_evolution.py:227-249) */
  double force[3];      /* body acceleration in lattice units (Guo forcing) */
  double tauT_fluid;    /* thermal relaxation time in fluid cells */
  double tauT_solid;    /* thermal relaxation time in solid cells */
  double pyro_A, pyro_b, pyro_Ea, pyro_Tmin; /* k = A (T+1e-6)^b exp(-Ea/(R(T+1e-6))), T>Tmin */
  double T_ref, T_scale;  /* T_phys = T*T_scale + T_ref (_scalarField.py:39-42) */
  double dt_phys;         /* seconds per lattice step */
  double heat_norm;       /* dH/(c_s T_scale): normalised temperature drop per unit dalpha */
  double gas_coef;        /* (1 - char_yield)*rho_s: gas mass released per unit dalpha */
  double alpha_flip;      /* reactive fraction below which a solid cell turns fluid */
  double mrt_s[19];       /* MRT rates per moment; viscous moments use 1/tau(rho) */
  double rho0, T0;        /* FP16 storage shift references */
  lbm_side_desc side[6];
  int32_t viscosity;      /* LBM_VISC_* */
  int32_t porous;         /* LBM_PORO_* */
  double suth_A, suth_Ts; /* LBM_VISC_SUTHERLAND: lattice viscosity suth_A T^1.5/(T + suth_Ts) of the
                             cell's temperature T in kelvin (T_ref + T_scale*T); suth_A = As*dt/dx^2
                             of set_viscosity_sutherland(As, Ts) (src/LBM/LBM2D/_evolution.py:228-235) */
  /* porous cells with two temperature fields (see LBM_PORO_*): */
  double Ts_ref, Ts_scale;     /* solid temperature T_s,phys = T_s*Ts_scale + Ts_ref (set_solid_Trange) */
  double cap_fluid, cap_solid; /* constant mass heat capacities c_f, c_s (TF.cm, TS.cm), J/(kg K) */
  double dx_phys;              /* cell size (m), for the radiating surface per volume a_r/dx */
  double T_ambient;            /* K (TS.Tambient, set_radiation) */
  int32_t radiation;           /* 1: surface radiation (RADIATION_MODEL.SURFACE_UNIFORM) */
  int32_t fp16_rounding;       /* LBM_PREC_FP16: LBM_FP16_STOCHASTIC (0) or LBM_FP16_NEAREST */
  /* Temperature-dependent thermal properties, THERMAL_DIFF_MODEL.DERIVED
   * (src/LBM/LBM2D/_thermal.py:62-107 fluid, :167-210 solid).  Bit p of tprop (p = 0
   * fluid, 1 solid) replaces the phase's constant tauT_fluid / tauT_solid by a per-cell
   * rate: D = k(T) / rho / c(T) * dt / dx^2 at the cell's temperature in kelvin
   * (T*T_scale + T_ref for the fluid, T*Ts_scale + Ts_ref for the solid), rho the cell's
   * lattice density for the fluid and tp_rhos for the solid, and tau = 3 D + 1/2 (2D) or
   * 4 D + 1/2 (3D).  k and c are the reference's nested form of five coefficients,
   * c0 + T (c1 + T (c2 T + T (c3 + T c4))) (a constant is {c0, 0, 0, 0, 0}; the solid
   * conductivity takes c4 = 0); c uses tp_cap_lo below tp_cap_Tmid and tp_cap_hi from it on
   * (NASA7 ranges; equal arrays for one polynomial), times tp_cap_mul (the gas constant for
   * a fluid NASA7 capacity, else 1).  Bit 2 instead of bit 0 selects the fluid's
   * THERMAL_DIFF_MODEL.PRANDTL: D = kinetic_viscosity / tp_prandtl, the cell's lattice
   * viscosity (constant or Sutherland) divided by its density under LBM_EOS_IDEAL_GAS
   * (src/LBM/LBM2D/_thermal.py:62-71, _evolution.py:227-246).  Temperature fields
   * THERMAL_CONJUGATE / TWO_FIELD only, without porous cells. */
  int32_t tprop;
  double tp_cond[2][5], tp_cap_lo[2][5], tp_cap_hi[2][5];
  double tp_cap_Tmid[2], tp_cap_mul[2];
  double tp_rhos;         /* solid density of the derived solid diffusivity (uniform) */
  double tp_dt, tp_dx2;   /* dt and dx^2 of the physical units */
  double tp_prandtl;      /* tprop bit 2: the fluid's Prandtl number */
} lbm_desc;

/* Diagnostics (FP64 accumulation).  No reference counterpart except umax,
 * Tmin, Tmax (src/LBM/LBM2D/_io.py:538-588). */
typedef struct lbm_diag {
  double mass;        /* sum rho over fluid cells */
  double energy;      /* sum T over all cells (normalised) */
  double solid_alpha; /* sum of reactive fraction over reactive solid cells */
  double umax;        /* max |u| over fluid cells */
  double Tmin, Tmax;  /* over all cells */
  double nonfinite;   /* count of NaN/Inf in rho or T */
  double nfluid;      /* fluid cell count */
  double res_num;     /* sum |u - u_prev|^2 over fluid cells (residual numerator) */
  double res_den;     /* sum |u|^2 over fluid cells */
  int64_t step;       /* lattice steps taken since lbm_init_equilibrium */
} lbm_diag;

/* Bindable fields (lbm_bind / lbm_required_bytes). */
#define LBM_FIELD_F 0       /* flow populations, 2 x Q planes (A/B), storage precision */
#define LBM_FIELD_G 1       /* temperature populations, 2 x QT planes */
#define LBM_FIELD_MASK 2    /* uint8 per cell */
#define LBM_FIELD_ALPHA 3   /* reactive fraction per cell (compute precision) */
#define LBM_FIELD_REL 4     /* gas release per cell, 2 planes (compute precision) */
#define LBM_FIELD_RHO 5     /* macro outputs: rho (compute precision) */
#define LBM_FIELD_U 6       /* 3 planes */
#define LBM_FIELD_T 7       /* 1 plane; 2 with porous cells and two temperature fields (TS of the porous cells) */
#define LBM_FIELD_UPREV 8   /* 3 float32 planes, residual reference */
#define LBM_FIELD_SCRATCH 9 /* reduction partials, control block, cell lists of the bulk update */
#define LBM_FIELD_INLET 10  /* flow-rate inlet state (side 0 of type LBM_BC_FLOWRATE, else 0 bytes):
                               the step's coefficient F/flow0, then per step parity the
                               rho*u_x of each side cell and the velocity behind it
                               (compute precision); part of a checkpoint */
#define LBM_FIELD_PORO 11   /* solid fraction per cell (compute precision), with lbm_desc.porous */
#define LBM_FIELD_DARCY 12  /* Darcy coefficient per cell (LBM_PORO_DARCY, _DARCY_FORCHHEIMER) */
#define LBM_FIELD_FORCH 13  /* Forchheimer coefficient per cell (LBM_PORO_DARCY_FORCHHEIMER) */
#define LBM_FIELD_GS 14     /* TS populations of porous cells, 2 x QT planes (two fields with porous cells) */
#define LBM_FIELD_XHEAT 15  /* 3 planes (compute precision): h*a, rhos, emissivity*a_r per cell */
#define LBM_NUM_FIELDS 16

/* lbm_step flags */
#define LBM_STEP_DIAG 1      /* reduce diagnostics on the last step */
#define LBM_STEP_MACRO 2     /* write rho/u/T planes on the last step */
#define LBM_STEP_RESIDUAL 4  /* residual vs UPREV on the last step, then UPREV = u */

typedef struct lbm_handle lbm_handle;

LBM_API int32_t lbm_abi_version(void);
LBM_API const char* lbm_last_error(void);

/* Bytes the caller must allocate for field `field` under `desc`.
 * Replaces the Taichi field declarations of src/LBM/LBM2D/_core.py:45-49
 * (3D: src/LBM/LBM3D/_core.py:46-50). */
LBM_API int32_t lbm_required_bytes(const lbm_desc* desc, int32_t field, size_t* bytes);

/* Validate `desc` and create a handle.  Replaces LBM2D_BASE.__init__
 * (src/LBM/LBM2D/_core.py:11-101) minus the field allocation.  The handle belongs to the
 * CUDA device current here: every later call on it makes that device current for its
 * duration and restores the caller's afterwards (bind buffers of that device; the members
 * of a batch share one device). */
LBM_API int32_t lbm_create(const lbm_desc* desc, lbm_handle** out);
LBM_API int32_t lbm_destroy(lbm_handle* h);

/* Hand a caller-owned device buffer to the handle. */
LBM_API int32_t lbm_bind(lbm_handle* h, int32_t field, void* dev_ptr, size_t bytes);

/* Replace the per-side boundary values (v, rho, T) without re-creating the
 * handle; `host_sides` points to 6 lbm_side_desc in host memory (pinned for an
 * asynchronous copy).  Replaces set_v_BC_value / set_rho_BC_value /
 * set_TF_BC_value (src/LBM/LBM2D/_io.py:413-458) between steps. */
LBM_API int32_t lbm_set_sides(lbm_handle* h, const lbm_side_desc* host_sides, void* stream);

/* Equilibrium initialisation from device planes rho[N], u[3N], T[N] (T may be
 * NULL without thermal), alpha[N] (NULL: 1 on reactive cells), all float32.  With
 * porous cells and two temperature fields T holds 2N values: the temperature of the
 * cell's first field (TF where s < 1, TS in pure-solid cells), then TS of the porous
 * cells (init_kernel sets TS.g = w TS.S in every cell, _initialize.py:62-63).
 * Compute precision is float32 for FP32/FP16 storage and float64 for FP64.  The solid mask must be bound first.  Replaces init_simulation /
 * init_kernel (src/LBM/LBM2D/_initialize.py:16-65, LBM3D/_initialize.py:17-77).
 * Resets the step counter and builds the cell lists of the bulk update (in
 * SCRATCH).  Synchronises `stream` once when a side is active: a solid cell on
 * an active side or next to one fails with LBM_ERR_ARG (NEE extrapolates from
 * the inner neighbour, so the two outer layers of an active side must be fluid). */
LBM_API int32_t lbm_init_equilibrium(lbm_handle* h, const float* rho, const float* u, const float* T,
                             const float* alpha, void* stream);

/* Continue from a saved state instead of initialising (checkpoint / resume).
 * The caller has filled the bound buffers with the state saved before step
 * `step` was taken: the half of F and of G that step reads (half step & 1 of the
 * A/B pair), MASK, ALPHA, the REL plane step & 1, and UPREV.  Sets the step
 * counter, makes both parity bits of every mask byte equal to bit step & 1 (so a
 * cell that turned fluid on the last saved pass is fluid for both), checks the
 * side layers as lbm_init_equilibrium does (and synchronises `stream` once when a
 * side is active) and rebuilds the cell lists.  Stepping on from here gives the
 * same fields, bit for bit, as the run that saved the state.  No reference
 * counterpart: the reference's export_snapshot is a reserved no-op
 * (src/LBM/LBM2D/_io.py:589-598) and it has no restart. */
LBM_API int32_t lbm_resume(lbm_handle* h, int64_t step, void* stream);

/* Advance n lattice steps.  Replaces step() / step_kernel()
 * (src/LBM/LBM2D/_evolution.py:12-25, src/LBM/LBM3D/_evolution.py:11-25). */
LBM_API int32_t lbm_step(lbm_handle* h, int32_t n, int32_t flags, void* stream);

/* Recompute, without advancing or modifying the lattice, the outputs that
 * `flags` (LBM_STEP_DIAG | LBM_STEP_MACRO | LBM_STEP_RESIDUAL) ask for, for the
 * state after the last step (rho/u/T planes, diagnostics).  Needs at least one
 * step since lbm_init_equilibrium.  Replaces the field reads behind
 * export_VTK_pyvista / log_info (src/LBM/LBM2D/_io.py:580-683). */
LBM_API int32_t lbm_compute_macro(lbm_handle* h, int32_t flags, void* stream);

/* Copy the diagnostics reduced by the last LBM_STEP_DIAG step into *out
 * (synchronises `stream`).  Replaces get_max_v / get_min_T / get_max_T
 * (src/LBM/LBM2D/_io.py:538-579) and adds mass, energy, residual and the
 * solid-mass integral.  Returns LBM_ERR_NONFINITE if NaN/Inf was seen. */
LBM_API int32_t lbm_read_diag(lbm_handle* h, lbm_diag* out, void* stream);

/* The same copy without waiting (replaces the same reference reads, for a driver loop that
 * keeps the GPU busy while it reads the previous step's values): enqueues on `stream` the
 * copy of the last LBM_STEP_DIAG step's diagnostics into *pinned_out and of the step
 * kernels' error flags into *pinned_err (both in page-locked host memory), sets
 * pinned_out->step, and returns.  Once the stream has passed the copy (an event recorded
 * after the call), *pinned_err bit 0 set means a bounded wait gave up (LBM_ERR_TIMEOUT),
 * bit 1 that the fluid list overflowed, and pinned_out->nonfinite > 0 that NaN/Inf was
 * seen, as lbm_read_diag reports them.  A later step with LBM_STEP_DIAG overwrites the
 * device values only after the copy (stream order). */
LBM_API int32_t lbm_read_diag_async(lbm_handle* h, lbm_diag* pinned_out, int32_t* pinned_err, void* stream);

/* Lattice steps taken since lbm_init_equilibrium (tLattice counter,
 * src/LBM/LBM2D/_evolution.py:15). */
LBM_API int64_t lbm_step_count(const lbm_handle* h);

/* Bulk form the handle runs (1 tile, 2 cell lists, 3 dense TMA-staged tiles), decided
 * by lbm_create from bulk_form, LBM_BULK and the lattice size.  No reference
 * counterpart (Taichi picks its own loop schedule). */
LBM_API int32_t lbm_bulk_form(const lbm_handle* h);

/* Failure detection (no reference counterpart: Taichi kernels have no error status).
 * The dense bulk form waits on an mbarrier for each staged tile; a wait gives up after
 * `tries` tries of about a microsecond each (default 4194304, i.e. seconds), records
 * the timeout for lbm_read_diag (LBM_ERR_TIMEOUT: the state is invalid), lets the copies
 * it issued land and ends the block.  0 gives up at the first wait: a test of that path. */
LBM_API int32_t lbm_set_wait_limit(lbm_handle* h, uint32_t tries);

/* Count n steps (n even) that a replay of a CUDA graph captured around
 * lbm_step(h, n, flags, stream) took: capturing runs no kernel but moves the
 * step counter by n, so the first replay brings the state level with the
 * counter and every later replay is followed by lbm_advance(h, n).  No
 * reference counterpart (the reference launches two Taichi kernels per step). */
LBM_API int32_t lbm_advance(lbm_handle* h, int32_t n);

/* Batches: many initialised lattices (same dim, precision, collision, thermal and
 * pyrolysis settings; sizes, geometries and parameters free; each created with
 * bulk_form = 2) stepped together by one persistent launch per kernel, for
 * parameter sweeps.  The reference runs one case per `lbm` process
 * (src/LBM/app.py:16-680); a batch replaces a loop of step() calls over many
 * solver objects.  The batch's tables live in a caller-owned device buffer of
 * lbm_batch_required_bytes() bytes.  Both calls read the lattices' list headers
 * and synchronise `stream`.  After lbm_batch_create, a lattice of the batch must
 * not be re-initialised or stepped on its own while the batch is used. */
typedef struct lbm_batch lbm_batch;
LBM_API int32_t lbm_batch_required_bytes(lbm_handle* const* handles, int32_t n, void* stream, size_t* bytes);
LBM_API int32_t lbm_batch_create(lbm_handle* const* handles, int32_t n, void* dev_buffer, size_t bytes,
                                 void* stream, lbm_batch** out);
/* Advance every lattice of the batch n steps (no diagnostics).  Issues no host
 * synchronisation and no allocation, so it can be captured in a CUDA graph; after
 * replaying a captured sequence of n steps call lbm_batch_advance(b, n) to move
 * the step counters (n even: a sequence keeps the step parity it was captured at). */
LBM_API int32_t lbm_batch_step(lbm_batch* b, int32_t n, void* stream);
LBM_API int32_t lbm_batch_advance(lbm_batch* b, int32_t n);
/* Persistent grid of the batch's bulk kernel: blocks of 128 threads per SM (1-4;
 * 1-2 in FP64; default the most that stay resident).  For launch-shape tuning. */
LBM_API int32_t lbm_batch_set_blocks(lbm_batch* b, int32_t blocks_per_sm);
LBM_API int32_t lbm_batch_destroy(lbm_batch* b);

/* No counterpart in the reference.  The diagnostics of the current state (the
 * values lbm_compute_macro(h, LBM_STEP_DIAG, ...) + lbm_read_diag return),
 * computed without any device allocation, for callers that cannot allocate
 * device memory: e.g. a plug-in whose host application owns every device
 * allocation through its own pool, or a hook inside a latency-critical time
 * loop where a cudaMalloc, which may synchronise the device, is not allowed.
 * The lattice state must be bound (with the cell-list bulk update, the lists
 * in LBM_FIELD_SCRATCH are part of it; the tile form needs no SCRATCH).  The
 * reduction's scratch is a static device array held by every GPU that loads
 * the library until exit (about 2.6 MB): lattices whose launch plan needs more
 * than LBM_NOALLOC_MAX_ROWS partial rows (one per thread block: four per SM
 * plus the boundary blocks in list form, one per row tile in tile form, e.g.
 * about 128^3 cells) are rejected with LBM_ERR_SIZE.  The first call on
 * a device looks up the array's device address (make it before any stream
 * capture).  All calls share the array and each call rewrites every value it
 * reads, so calls that overlap on the GPU (different streams or handles at
 * the same time) race.  Synchronises `stream`. */
#define LBM_NOALLOC_MAX_ROWS 32768
LBM_API int32_t lbm_diag_noalloc(lbm_handle* h, lbm_diag* out, void* stream);

/* ------------------------------------------------------ geometry: STL meshes
 * Replace StlReader.voxel_stl (src/LBM/GEO/STL.py:147-268, called by
 * load_stl, src/LBM/LBM2D/_io.py:489-495) after the mesh has been read and
 * scaled / rotated / translated on the host.  The reference voxelises with
 * pyvista and samples the voxels onto the grid; here a cell is solid when its
 * centre ((i+0.5)dx, (j+0.5)dx, (k+0.5)dx; the 2D lattice is the plane z = 0)
 * lies inside the closed mesh, by ray parity along x. */

/* Bytes of the work buffer lbm_voxelise_stl needs (dim 2: nz = 1). */
LBM_API int32_t lbm_stl_work_bytes(int32_t nx, int32_t ny, int32_t nz, int32_t dim, size_t* bytes);

/* triangles: device float32 [ntri][3 vertices][x, y, z] in the lattice's physical
 * units (cell size dx).  Writes solid[c] (uint8 0/1) and, if `surface` is not
 * NULL, surface[c] (float32): the reference's surface weight of a solid cell from
 * its solid face neighbours (3D 6..0 solid: 0, 1, 1.414, 2, 3, 4, 6; 2D 4..0: 0,
 * 1, 1.414, 2, 4), counted on a grid padded by one cell as the reference's is;
 * 0 for fluid cells.  Cell c = x + nx*(y + ny*z).  `work` (device,
 * lbm_stl_work_bytes) holds the toggle bits and the padded voxels. */
LBM_API int32_t lbm_voxelise_stl(const float* triangles, int64_t ntri, int32_t nx, int32_t ny, int32_t nz,
                                 int32_t dim, double dx, void* work, size_t work_bytes, uint8_t* solid,
                                 float* surface, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
