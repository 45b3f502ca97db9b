/*
 * lbm_oracle.c -- CPU restatement of LBM_porousChem's per-timestep lattice update.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path: the
 * tests, the smoke entry and the bench's CPU-baseline leg call it.  Nothing in
 * the product links or executes it.
 *
 * PARITY PINNED against the reference's own code: tests/golden/ref_*.npz hold outputs
 * of the unmodified reference solver modules (src/LBM/LBM2D, src/LBM/LBM3D) run on
 * small lattices through a sequential NumPy stand-in for Taichi (the reference's Taichi
 * 1.7.4 is not installable here), in float64; tests/test_oracle_vs_reference.py checks
 * this file's FP64 build against them to 1e-12 (it agrees bit for bit) on periodic, NEE,
 * ES and NEE-on-periodic sides, 2D and 3D, flow and two-field temperature.  Where the
 * reference has no behaviour (body force, conjugate heat, pyrolysis with cell flip, MRT,
 * reductions) this file defines it, pinned by analytic known answers (Poiseuille, mass
 * conservation, equilibrium fixed point, the single-cell Arrhenius ODE) in
 * tests/test_oracle_physics.py.
 *
 * Structure mirrors the reference's push scheme:
 *   step():  collision_source_streaming (push, halfway bounce-back)
 *            -> macro (moments, sources, pyrolysis, flips)
 *            -> non-equilibrium-extrapolation boundaries (NEE)
 *   src/LBM/LBM2D/_evolution.py:12-25   (step / step_kernel)
 *   src/LBM/LBM2D/_evolution.py:26-115  (collision_source_streaming)
 *   src/LBM/LBM2D/_evolution.py:118-202 (macro)
 *   src/LBM/LBM2D/_boundary.py:17-101   (Boundary_condition_NEE, flow sides)
 *   src/LBM/LBM2D/_scalarField.py:83-122 (scalar NEE)
 *   3D twins: src/LBM/LBM3D/_evolution.py:11-195, LBM3D/_boundary.py:15-142,
 *             LBM3D/_scalarField.py:83-140.
 *
 * Build twice: -DREAL=float (FP32 oracle) and -DREAL=double (FP64 oracle).
 * Cell index: c = x + nx*(y + ny*z).  Distribution storage: f[c*Q + k].
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef REAL
#define REAL double
#endif

/* ---------------------------------------------------------------- lattices */
/* D2Q9 / D2Q5: src/LBM/LBM2D/_initialize.py:25-35, opposite table _core.py:35 */
static const int E9[9][3] = {{0,0,0},{1,0,0},{0,1,0},{-1,0,0},{0,-1,0},
                             {1,1,0},{-1,1,0},{-1,-1,0},{1,-1,0}};
static const int OPP9[9] = {0,3,4,1,2,7,8,5,6};
/* D3Q19 / D3Q7: src/LBM/LBM3D/_initialize.py:25-43, opposite table _core.py:36 */
static const int E19[19][3] = {{0,0,0},{1,0,0},{-1,0,0},{0,1,0},{0,-1,0},{0,0,1},{0,0,-1},
                               {1,1,0},{-1,1,0},{1,-1,0},{-1,-1,0},
                               {1,0,1},{-1,0,1},{1,0,-1},{-1,0,-1},
                               {0,1,1},{0,-1,1},{0,1,-1},{0,-1,-1}};
static const int OPP19[19] = {0,2,1,4,3,6,5,10,9,8,7,14,13,12,11,18,17,16,15};

/* ------------------------------------------------------------------ config */
enum { ORC_BC_PERIODIC = 0, ORC_BC_ZEROGRAD = 1, ORC_BC_FIXED = 2,
       ORC_BC_FLOWRATE = 3 /* velocity of side 0 only: BC_FLOW.inlet_flow, v[0] = flow rate */ };

typedef struct orc_side {
    int active;      /* 1: NEE on this side (reference BC_MODEL.NEE), 2: ES (BC_MODEL.ES),
                      * 3: NEBB (BC_MODEL.NEBB, 2D) */
    int v_type;      /* ORC_BC_* for velocity  (LBM2D/_io.py:385-402 set_BC mapping) */
    int rho_type;    /* ORC_BC_* for density */
    int T_type;      /* ORC_BC_* for the temperature distribution */
    double v[3];
    double rho;
    double T;
} orc_side;

typedef struct orc_cfg {
    int dim, nx, ny, nz;
    int collision;           /* 0 BGK, 1 MRT */
    int eos;                 /* 0 IDEAL_GAS (tau = 3 nu/rho + 1/2), 1 INCOMPRESSIBLE */
    double nu;               /* lattice viscosity (visco*dt/dx^2), _evolution.py:227-249 */
    double force[3];         /* body acceleration (new; reference volume_force = 0) */
    int half_force_velocity; /* 1: u = (sum e f + F/2)/rho.  Reference: 0 (_evolution.py:123-130) */
    int thermal;             /* 0 none, 1 conjugate single field, 2 two fields (TF / TS) */
    double tauT_fluid, tauT_solid;
    int pyro;
    double pyro_A, pyro_b, pyro_Ea, pyro_Tmin;  /* Arrhenius, LBM2D/_chemical.py:198-212 */
    double T_ref, T_scale;   /* T_phys = T*T_scale + T_ref, _scalarField.py:39-42 */
    double dt_phys;          /* seconds per lattice step */
    double heat_norm;        /* dH/(c_s*T_scale): normalised temperature drop per unit dalpha */
    double gas_coef;         /* (1-char_yield)*rho_s: gas mass released per unit dalpha */
    double alpha_flip;       /* reactive fraction below which a solid cell turns fluid */
    double mrt_s[19];        /* MRT relaxation rates per moment (viscous ones overwritten by 1/tau) */
    orc_side side[6];        /* 0 x-, 1 x+, 2 y-, 3 y+, 4 z-, 5 z+ */
    int visc_model;          /* 0 constant nu, 1 Sutherland: nu = suth_A T^1.5/(T + suth_Ts), T in K */
    double suth_A, suth_Ts;  /* suth_A = As*dt/dx^2 (LBM2D/_evolution.py:228-235) */
    int ref_quirk_frozen_solid_T; /* two fields only: the reference's macro skips pure-solid
                              * cells (LBM2D/_evolution.py:119), so their TS.S never changes and
                              * TS.g keeps its own post-collision values instead of the streamed
                              * ones (collision :96-100 writes TS.g in place).  1 reproduces that. */
    int poro_model;          /* porous cells (0 < solid < 1, src/LBM/util/flag.py PORO_MODEL): 0 none,
                              * 1 SPHERICAL (Ergun from the porosity), 2 DARCY, 3 DARCYFORCHHEIMER */
    /* Two fields with porous cells: a porous cell carries both TF and TS, which exchange
     * heat there (src/LBM/LBM2D/_evolution.py:186-202, LBM3D/_evolution.py:179-195) */
    double Ts_ref, Ts_scale; /* TS.v_ref, TS.v_scale (set_solid_Trange, LBM2D/_io.py:253-256) */
    double cap_fluid, cap_solid; /* TF.cm, TS.cm: constant capacity_m (LBM2D/_thermal.py:86-88, :189-191) */
    double dx_phys;          /* cell size: radiation per volume a/dx (_thermal.py:213-220) */
    int radiation;           /* 1: RADIATION_MODEL.SURFACE_UNIFORM (set_radiation, _io.py:259-271) */
    double T_ambient;        /* TS.Tambient (K) */
    int ref_quirk_nebb;      /* NEBB sides: 1 reproduces the reference's branches as written
                              * (LBM2D/_boundary.py:145-226): side 0 outlet with the velocity's
                              * sign flipped, side 1 wall rebuilding the populations that point
                              * out of the domain, side 1 inlet and the inlets / outlets of
                              * sides 2 and 3 leaving the populations as streamed; 0 the
                              * Zou-He construction on every side */
    int tprop;               /* bit 0 fluid, bit 1 solid: THERMAL_DIFF_MODEL.DERIVED, the phase's
                              * diffusivity k(T)/rho/c(T)*dt/dx^2 at the cell's temperature
                              * (LBM2D/_thermal.py:62-107, :167-210) instead of tauT_fluid/solid */
    double tp_cond[2][5], tp_cap_lo[2][5], tp_cap_hi[2][5]; /* nested-form coefficients per phase */
    double tp_cap_Tmid[2], tp_cap_mul[2]; /* NASA7 switch temperature (K), R for a fluid NASA7 */
    double tp_rhos, tp_dt, tp_dx2;        /* solid density, dt, dx^2 */
    double tp_prandtl;       /* tprop bit 2: the fluid's THERMAL_DIFF_MODEL.PRANDTL,
                              * D = kinetic_viscosity(i)/Pr (LBM2D/_thermal.py:67-68) */
} orc_cfg;

#define ORC_SIGMA 5.670374419e-8   /* Stefan-Boltzmann constant, src/LBM/util/constant.py:20 */

/* mask bits */
#define ORC_SOLID 1u
#define ORC_REACTIVE 4u

typedef struct orc {
    orc_cfg c;
    int Q, QT;
    long N;
    int e[19][3];
    int opp[19];
    REAL w[19], wt[7];
    REAL ta, tb, tc;          /* thermal equilibrium coefficients (3,4.5,1.5) / (4,8,2) */
    double M[19][19];         /* MRT moment matrix (rows orthogonal) */
    double Mn[19];            /* squared row norms */
    int visc_row[19];         /* 1 if the moment relaxes with 1/tau */
    int cons_row[19];         /* 1 if the moment is conserved (rho, j): never relaxed */
    REAL *f, *F, *g, *G;
    REAL *rho, *u, *T, *dS, *alpha, *rel;
    REAL *sfrac, *cdarcy, *cforch;  /* solid fraction, Darcy and Forchheimer coefficients per cell */
    /* two fields with porous cells (NULL otherwise): TS populations of porous cells
     * (pure-solid cells keep theirs in g/G), their temperature and source, and the
     * per-cell exchangeCoef, exchangeSurface, rhos, emissivity, radiation_surface */
    REAL *gs, *Gs, *Ts, *dSs, *xh, *xa, *rhos, *emis, *rsurf;
    uint8_t *mask, *mask_next;
    /* flow-rate inlet on side 0, per side cell j = y + ny*z: what the reference's
     * updateBC_kernel reads (rho*u_x at x = 0, u at x = 1, 3 per cell) and the
     * inlet velocity profile it writes (v_bc_profile[0], 3 per cell) */
    REAL *inl_m, *inl_w, *inl_prof;
} orc;

/* ------------------------------------------------------------ MRT basis */
/* D3Q19 moment basis of d'Humieres, Ginzburg, Krafczyk, Lallemand & Luo,
 * Phil. Trans. R. Soc. A 360 (2002) 437: rho, e, eps, jx, qx, jy, qy, jz, qz,
 * 3pxx, 3pixx, pww, piww, pxy, pyz, pxz, mx, my, mz.  D2Q9 basis of Lallemand &
 * Luo, Phys. Rev. E 61 (2000) 6546: rho, e, eps, jx, qx, jy, qy, pxx, pxy.  The
 * reference has no MRT; this is new behaviour. */
static double mrt_poly(int dim, int r, int cx, int cy, int cz) {
    double c2 = cx*cx + cy*cy + cz*cz;
    if (dim == 2) {
        switch (r) {
        case 0: return 1;
        case 1: return -4 + 3*c2;
        case 2: return 4 - 10.5*c2 + 4.5*c2*c2;
        case 3: return cx;
        case 4: return (-5 + 3*c2)*cx;
        case 5: return cy;
        case 6: return (-5 + 3*c2)*cy;
        case 7: return cx*cx - cy*cy;
        case 8: return cx*cy;
        }
        return 0;
    }
    switch (r) {
    case 0: return 1;
    case 1: return 19*c2 - 30;
    case 2: return (21*c2*c2 - 53*c2 + 24)/2.0;
    case 3: return cx;
    case 4: return (5*c2 - 9)*cx;
    case 5: return cy;
    case 6: return (5*c2 - 9)*cy;
    case 7: return cz;
    case 8: return (5*c2 - 9)*cz;
    case 9: return 3*cx*cx - c2;
    case 10: return (3*c2 - 5)*(3*cx*cx - c2);
    case 11: return cy*cy - cz*cz;
    case 12: return (3*c2 - 5)*(cy*cy - cz*cz);
    case 13: return cx*cy;
    case 14: return cy*cz;
    case 15: return cx*cz;
    case 16: return (cy*cy - cz*cz)*cx;
    case 17: return (cz*cz - cx*cx)*cy;
    case 18: return (cx*cx - cy*cy)*cz;
    }
    return 0;
}

/* ---------------------------------------------------------------- helpers */
static inline long cidx(const orc* o, int x, int y, int z) {
    return (long)x + (long)o->c.nx * ((long)y + (long)o->c.ny * z);
}
/* src/LBM/LBM2D/_evolution.py:205-212 periodic_index (3D: LBM3D/_evolution.py:200-210) */
static inline int wrap(int v, int n) { return v < 0 ? n - 1 : (v > n - 1 ? 0 : v); }
static inline long nbr(const orc* o, long c, int k, int sign) {
    int nx = o->c.nx, ny = o->c.ny;
    int x = (int)(c % nx), y = (int)((c / nx) % ny), z = (int)(c / ((long)nx * ny));
    x = wrap(x + sign*o->e[k][0], o->c.nx);
    y = wrap(y + sign*o->e[k][1], o->c.ny);
    z = wrap(z + sign*o->e[k][2], o->c.nz);
    return cidx(o, x, y, z);
}
static inline int is_solid(const uint8_t* m, long c) { return (m[c] & ORC_SOLID) != 0; }

/* feq9 / feq19: src/LBM/LBM2D/_evolution.py:213-225, with eps = 1 - solid (1 in a fluid
 * cell, 0 < eps < 1 in a porous one) */
static inline REAL feq_e(const orc* o, int k, REAL rho, const REAL* u, REAL eps0) {
    REAL eu = (REAL)o->e[k][0]*u[0] + (REAL)o->e[k][1]*u[1] + (REAL)o->e[k][2]*u[2];
    REAL uv = u[0]*u[0] + u[1]*u[1] + u[2]*u[2];
    REAL eps = eps0 + (REAL)1e-12;
    if (o->c.eos == 1)
        return o->w[k]*(rho + (REAL)3.0*eu + (REAL)4.5*eu*eu/eps - (REAL)1.5*uv/eps);
    return o->w[k]*rho*((REAL)1.0 + (REAL)3.0*eu + (REAL)4.5*eu*eu/eps - (REAL)1.5*uv/eps);
}
static inline REAL feq(const orc* o, int k, REAL rho, const REAL* u) { return feq_e(o, k, rho, u, (REAL)1.0); }
/* eps = 1 - solid of a cell, src/LBM/LBM2D/_evolution.py:119 */
static inline REAL eps_of(const orc* o, long c) { return (REAL)1.0 - o->sfrac[c]; }
static inline int is_porous(const orc* o, long c) {
    return o->c.poro_model != 0 && o->sfrac[c] != 0 && o->sfrac[c] != 1;
}
/* porous cells carry a TS field of their own (two fields with porous cells) */
static inline int porous_ts(const orc* o, long c) { return o->gs != NULL && is_porous(o, c); }
/* TemperatureFluid.geq5 / geq7: src/LBM/LBM2D/_thermal.py:54-61, LBM3D/_thermal.py:54-61 */
static inline REAL geq_fluid(const orc* o, int k, REAL T, const REAL* u) {
    REAL eu = (REAL)o->e[k][0]*u[0] + (REAL)o->e[k][1]*u[1] + (REAL)o->e[k][2]*u[2];
    REAL uv = u[0]*u[0] + u[1]*u[1] + u[2]*u[2];
    return o->wt[k]*T*((REAL)1.0 + o->ta*eu + o->tb*eu*eu - o->tc*uv);
}
/* viscosity(i) in lattice units: constant or Sutherland at the fluid temperature GetTF(i)
 * = T_ref + T_scale*T (src/LBM/LBM2D/_evolution.py:227-235, :304-307) */
static inline REAL visc_lu(const orc* o, REAL T) {
    REAL nu = (REAL)o->c.nu;
    if (o->c.visc_model == 1) {
        REAL TK = T*(REAL)o->c.T_scale + (REAL)o->c.T_ref;
        nu = (REAL)o->c.suth_A*(REAL)pow(TK, 1.5)/(TK + (REAL)o->c.suth_Ts);
    }
    return nu;
}
/* kinetic_viscosity(i): IDEAL_GAS divides by rho (:236-240) */
static inline REAL visc_kin(const orc* o, REAL rho, REAL T) {
    REAL nu = visc_lu(o, T);
    if (o->c.eos == 0) nu = nu / rho;
    return nu;
}
/* tau = 3 kinetic_viscosity + 1/2 (:241-249) */
static inline REAL tau_flow(const orc* o, REAL rho, REAL T) { return (REAL)3*visc_kin(o, rho, T) + (REAL)0.5; }

/* darcy_force(i) of a porous cell, src/LBM/LBM2D/_evolution.py:262-283: SPHERICAL (Ergun
 * with perm = eps^3/(1.000001-eps)^2, :250-253), DARCY, DARCYFORCHHEIMER.  The 2D solver
 * uses kinetic_viscosity(i); the 3D one uses viscosity(i) (LBM3D/_evolution.py:262-278). */
static void darcy_force(const orc* o, long c, REAL rho, const REAL* u, REAL T, REAL* F) {
    REAL eps = eps_of(o, c);
    REAL nu = o->c.dim == 2 ? visc_kin(o, rho, T) : visc_lu(o, T);
    REAL v = (REAL)sqrt((double)(u[0]*u[0] + u[1]*u[1] + u[2]*u[2]));
    REAL a = 0;
    if (o->c.poro_model == 1) {
        REAL perm = (REAL)pow((double)eps, 3.0)/(REAL)pow((double)((REAL)1.000001 - eps), 2.0)*(REAL)1;
        REAL beta = (REAL)1.75/(REAL)sqrt((double)((REAL)150*eps*perm));
        a = -nu/perm*eps - beta*v;
    } else if (o->c.poro_model == 2) {
        a = -eps*nu*o->cdarcy[c];
    } else if (o->c.poro_model == 3) {
        a = -eps*nu*o->cdarcy[c] - eps*o->cforch[c]*v;
    }
    for (int d = 0; d < 3; ++d) F[d] = a*u[d];
}

/* macro's porous velocity correction, src/LBM/LBM2D/_evolution.py:131-151 (3D: :130-149),
 * at the cell's new rho */
static void porous_correct(const orc* o, long c, REAL rho, REAL T, REAL* u) {
    REAL eps = eps_of(o, c);
    REAL nu = visc_kin(o, rho, T);
    REAL div;
    if (o->c.poro_model == 2) {
        div = (REAL)1 + eps*nu*o->cdarcy[c]/(REAL)2;
    } else {
        REAL Dc, Fc;
        if (o->c.poro_model == 1) {
            REAL perm = (REAL)pow((double)eps, 3.0)/(REAL)pow((double)((REAL)1.000001 - eps), 2.0)*(REAL)1;
            Dc = (REAL)1.0/perm;
            Fc = (REAL)1.75/(REAL)sqrt((double)((REAL)150*(REAL)pow((double)eps, 3.0)));
        } else {
            Dc = o->cdarcy[c];
            Fc = o->cforch[c];
        }
        REAL c0 = (REAL)0.5*((REAL)1 + eps*nu/(REAL)2*Dc);
        REAL c1 = (REAL)0.5*eps*Fc;
        REAL v = (REAL)sqrt((double)(u[0]*u[0] + u[1]*u[1] + u[2]*u[2]));
        div = c0 + (REAL)sqrt((double)((REAL)pow((double)c0, 2.0) + c1*v));
    }
    for (int d = 0; d < 3; ++d) u[d] /= div;
}
/* forceTermGuo: src/LBM/LBM2D/_evolution.py:284-298, force F (volume + darcy) and eps */
static inline REAL guo(const orc* o, int k, REAL rho, const REAL* u, REAL tau, const REAL* Fv, REAL eps0) {
    REAL Fx = Fv[0], Fy = Fv[1], Fz = Fv[2];
    if (Fx == 0 && Fy == 0 && Fz == 0) return 0;
    REAL eps = eps0 + (REAL)1e-12;
    REAL ex = (REAL)o->e[k][0], ey = (REAL)o->e[k][1], ez = (REAL)o->e[k][2];
    REAL t1 = (ex - u[0]/eps)*Fx + (ey - u[1]/eps)*Fy + (ez - u[2]/eps)*Fz;
    REAL eu = ex*u[0] + ey*u[1] + ez*u[2];
    REAL eF = ex*Fx + ey*Fy + ez*Fz;
    REAL pre = (REAL)1.0 - (REAL)1.0/(REAL)2.0/tau;
    if (o->c.eos == 1)
        return pre*o->w[k]*((REAL)3.0*t1 + (REAL)9.0*eu*eF/eps);
    return pre*rho*o->w[k]*((REAL)3.0*t1 + (REAL)9.0*eu*eF/eps);
}

/* Post-collision flow populations of fluid cell c (BGK: _evolution.py:33; MRT new).  A
 * porous cell (0 < solid < 1) relaxes towards its eps-equilibrium and adds the Guo term of
 * its Darcy force (force(i) = volume_force + darcy_force, :254-261). */
static void collide_flow(const orc* o, long c, const REAL* fin, REAL rho, const REAL* u, REAL T, REAL* fout) {
    int Q = o->Q;
    REAL tau = tau_flow(o, rho, T);
    REAL eps = 1;
    REAL Fv[3] = {(REAL)o->c.force[0], (REAL)o->c.force[1], (REAL)o->c.force[2]};
    if (c >= 0 && is_porous(o, c)) {
        REAL Fd[3];
        eps = eps_of(o, c);
        darcy_force(o, c, rho, u, T, Fd);
        for (int d = 0; d < 3; ++d) Fv[d] = (REAL)0 + Fv[d] + Fd[d];
    }
    REAL fe[19];
    for (int k = 0; k < Q; ++k) fe[k] = feq_e(o, k, rho, u, eps);
    if (o->c.collision == 0) {
        for (int k = 0; k < Q; ++k)
            fout[k] = fin[k] - (REAL)1/tau*(fin[k] - fe[k]) + guo(o, k, rho, u, tau, Fv, eps);
        return;
    }
    REAL mneq[19];
    for (int r = 0; r < Q; ++r) {
        if (o->cons_row[r]) { mneq[r] = 0; continue; }
        REAL s = o->visc_row[r] ? (REAL)1/tau : (REAL)o->c.mrt_s[r];
        REAL acc = 0;
        for (int k = 0; k < Q; ++k) acc += (REAL)o->M[r][k]*(fin[k] - fe[k]);
        mneq[r] = s*acc/(REAL)o->Mn[r];
    }
    for (int k = 0; k < Q; ++k) {
        REAL acc = 0;
        for (int r = 0; r < Q; ++r) if (!o->cons_row[r]) acc += (REAL)o->M[r][k]*mneq[r];
        fout[k] = fin[k] - acc + guo(o, k, rho, u, tau, Fv, eps);
    }
}

/* ------------------------------------------------------------- lifecycle */
orc* orc_create(const orc_cfg* cfg) {
    orc* o = (orc*)calloc(1, sizeof(orc));
    o->c = *cfg;
    if (o->c.dim == 2) o->c.nz = 1;
    o->N = (long)o->c.nx * o->c.ny * o->c.nz;
    if (o->c.dim == 2) {
        o->Q = 9; o->QT = 5;
        for (int k = 0; k < 9; ++k) { memcpy(o->e[k], E9[k], sizeof(E9[k])); o->opp[k] = OPP9[k]; }
        o->w[0] = (REAL)(4.0/9.0);
        for (int k = 1; k < 5; ++k) o->w[k] = (REAL)(1.0/9.0);
        for (int k = 5; k < 9; ++k) o->w[k] = (REAL)(1.0/36.0);
        o->wt[0] = (REAL)(1.0/3.0);
        for (int k = 1; k < 5; ++k) o->wt[k] = (REAL)(1.0/6.0);
        o->ta = 3.0; o->tb = 4.5; o->tc = 1.5;
    } else {
        o->Q = 19; o->QT = 7;
        for (int k = 0; k < 19; ++k) { memcpy(o->e[k], E19[k], sizeof(E19[k])); o->opp[k] = OPP19[k]; }
        o->w[0] = (REAL)(1.0/3.0);
        for (int k = 1; k < 7; ++k) o->w[k] = (REAL)(1.0/18.0);
        for (int k = 7; k < 19; ++k) o->w[k] = (REAL)(1.0/36.0);
        o->wt[0] = (REAL)(1.0/4.0);
        for (int k = 1; k < 7; ++k) o->wt[k] = (REAL)(1.0/8.0);
        o->ta = 4.0; o->tb = 8.0; o->tc = 2.0;
    }
    for (int r = 0; r < o->Q; ++r) {
        double n2 = 0;
        for (int k = 0; k < o->Q; ++k) {
            o->M[r][k] = mrt_poly(o->c.dim, r, o->e[k][0], o->e[k][1], o->e[k][2]);
            n2 += o->M[r][k]*o->M[r][k];
        }
        o->Mn[r] = n2;
        o->visc_row[r] = o->c.dim == 2 ? (r == 7 || r == 8)
                                       : (r == 9 || r == 11 || r == 13 || r == 14 || r == 15);
        o->cons_row[r] = o->c.dim == 2 ? (r == 0 || r == 3 || r == 5)
                                       : (r == 0 || r == 3 || r == 5 || r == 7);
    }
    long N = o->N;
    o->f = (REAL*)calloc(N*o->Q, sizeof(REAL));
    o->F = (REAL*)calloc(N*o->Q, sizeof(REAL));
    o->g = (REAL*)calloc(N*o->QT, sizeof(REAL));
    o->G = (REAL*)calloc(N*o->QT, sizeof(REAL));
    o->rho = (REAL*)calloc(N, sizeof(REAL));
    o->u = (REAL*)calloc(3*N, sizeof(REAL));
    o->T = (REAL*)calloc(N, sizeof(REAL));
    o->dS = (REAL*)calloc(N, sizeof(REAL));
    o->alpha = (REAL*)calloc(N, sizeof(REAL));
    o->rel = (REAL*)calloc(N, sizeof(REAL));
    o->mask = (uint8_t*)calloc(N, 1);
    o->sfrac = (REAL*)calloc(N, sizeof(REAL));
    o->cdarcy = (REAL*)calloc(N, sizeof(REAL));
    o->cforch = (REAL*)calloc(N, sizeof(REAL));
    o->mask_next = (uint8_t*)calloc(N, 1);
    if (o->c.thermal == 2 && o->c.poro_model != 0) {
        o->gs = (REAL*)calloc(N*o->QT, sizeof(REAL));
        o->Gs = (REAL*)calloc(N*o->QT, sizeof(REAL));
        o->Ts = (REAL*)calloc(N, sizeof(REAL));
        o->dSs = (REAL*)calloc(N, sizeof(REAL));
        o->xh = (REAL*)calloc(N, sizeof(REAL));
        o->xa = (REAL*)calloc(N, sizeof(REAL));
        o->rhos = (REAL*)calloc(N, sizeof(REAL));
        o->emis = (REAL*)calloc(N, sizeof(REAL));
        o->rsurf = (REAL*)calloc(N, sizeof(REAL));
    }
    long M = (long)o->c.ny * o->c.nz;
    o->inl_m = (REAL*)calloc(M, sizeof(REAL));
    o->inl_w = (REAL*)calloc(3*M, sizeof(REAL));
    o->inl_prof = (REAL*)calloc(3*M, sizeof(REAL));
    return o;
}

void orc_destroy(orc* o) {
    if (!o) return;
    free(o->f); free(o->F); free(o->g); free(o->G); free(o->rho); free(o->u); free(o->T);
    free(o->dS); free(o->alpha); free(o->rel); free(o->mask); free(o->mask_next);
    free(o->sfrac); free(o->cdarcy); free(o->cforch);
    free(o->gs); free(o->Gs); free(o->Ts); free(o->dSs); free(o->xh); free(o->xa); free(o->rhos);
    free(o->emis); free(o->rsurf);
    free(o->inl_m); free(o->inl_w); free(o->inl_prof); free(o);
}

int orc_Q(const orc* o) { return o->Q; }
int orc_QT(const orc* o) { return o->QT; }
double orc_M(const orc* o, int r, int k) { return o->M[r][k]; }

/* Porous cells: solid fraction (0 fluid, 1 solid, between: porous), Darcy and Forchheimer
 * coefficients (set_poro_Darcy / set_poro_Darcy_Forchheimer, src/LBM/LBM2D/_io.py:152-172),
 * planar, any may be NULL.  Call before orc_init. */
void orc_set_porous(orc* o, const double* sfrac, const double* darcy, const double* forch) {
    for (long c = 0; c < o->N; ++c) {
        o->sfrac[c] = sfrac ? (REAL)sfrac[c] : 0;
        o->cdarcy[c] = darcy ? (REAL)darcy[c] : 0;
        o->cforch[c] = forch ? (REAL)forch[c] : 0;
    }
}

/* Heat exchange and radiation inputs of porous cells (two fields): exchangeCoef and
 * exchangeSurface (set_heat_exchange_coef / _surface, LBM2D/_io.py:133-138), rhos
 * (add_rho_solid, :128-132), emissivity and radiation_surface (app.py:564-566); planar,
 * any may be NULL (zero).  Call before orc_init. */
void orc_set_porous_heat(orc* o, const double* h, const double* a, const double* rhos,
                         const double* emis, const double* rsurf) {
    if (!o->gs) return;
    for (long c = 0; c < o->N; ++c) {
        o->xh[c] = h ? (REAL)h[c] : 0;
        o->xa[c] = a ? (REAL)a[c] : 0;
        o->rhos[c] = rhos ? (REAL)rhos[c] : 0;
        o->emis[c] = emis ? (REAL)emis[c] : 0;
        o->rsurf[c] = rsurf ? (REAL)rsurf[c] : 0;
    }
}

/* init_kernel: f = F = feq(rho,u), g = G = geq(T,u)  (src/LBM/LBM2D/_initialize.py:37-65).
 * Inputs are planar: u[d*N + c].  mask bit0 = solid, bit2 = reactive. */
void orc_init(orc* o, const double* rho, const double* u, const double* T,
              const uint8_t* mask, const double* alpha) {
    long N = o->N;
    int fr = o->c.side[0].active && o->c.side[0].v_type == ORC_BC_FLOWRATE;
    REAL v0 = fr ? (REAL)(o->c.side[0].v[0] / o->c.ny / o->c.nz) : 0;
    for (long c = 0; c < N; ++c) {
        o->mask[c] = mask[c] & (ORC_SOLID | ORC_REACTIVE);
        o->rho[c] = (REAL)rho[c];
        for (int d = 0; d < 3; ++d) o->u[c*3 + d] = (REAL)u[d*N + c];
        if (fr && c % o->c.nx <= 1) { o->u[c*3] = v0; o->u[c*3+1] = 0; o->u[c*3+2] = 0; }
        o->T[c] = T ? (REAL)T[c] : 0;
        o->alpha[c] = alpha ? (REAL)alpha[c] : 0;
        o->dS[c] = 0;
        o->rel[c] = 0;
        if (is_solid(o->mask, c)) { o->u[c*3] = o->u[c*3+1] = o->u[c*3+2] = 0; }
        for (int k = 0; k < o->Q; ++k) {
            REAL v = is_solid(o->mask, c) ? 0 : feq_e(o, k, o->rho[c], &o->u[c*3], is_porous(o, c) ? eps_of(o, c) : (REAL)1.0);
            o->f[c*o->Q + k] = v;
            o->F[c*o->Q + k] = v;
        }
        for (int k = 0; k < o->QT; ++k) {
            REAL v = is_solid(o->mask, c) ? o->wt[k]*o->T[c] : geq_fluid(o, k, o->T[c], &o->u[c*3]);
            o->g[c*o->QT + k] = v;
            o->G[c*o->QT + k] = v;
        }
        if (porous_ts(o, c)) {      /* TS.g = TS.G = TS.geq(TS.S) = w T (:62-63), TS.S = T here */
            o->Ts[c] = o->T[c];
            o->dSs[c] = 0;
            for (int k = 0; k < o->QT; ++k) o->gs[c*o->QT + k] = o->Gs[c*o->QT + k] = o->wt[k]*o->T[c];
        }
    }
    /* init_boundary (src/LBM/LBM2D/_initialize.py:67-74): the columns x = 0 and 1 start
     * at the inlet velocity v0 = F/ny/nz and the first controller update reads it.  The
     * reference writes v0 into the macro velocity only (its first collision reads it)
     * and keeps the populations of the initial fields; here the populations start at
     * equilibrium with v0 too. */
    if (fr) {
        for (long j = 0; j < (long)o->c.ny * o->c.nz; ++j) {
            o->inl_m[j] = o->rho[(long)o->c.nx * j] * v0;
            o->inl_w[3*j] = v0; o->inl_w[3*j+1] = 0; o->inl_w[3*j+2] = 0;
        }
    }
}

/* A solid temperature field of its own (TS.S initialised apart from TF.S, app.py:506-509):
 * after orc_init, TS of porous cells and of pure-solid cells (two fields) from Ts, planar. */
void orc_init_solid_T(orc* o, const double* Ts) {
    if (o->c.thermal != 2) return;
    for (long c = 0; c < o->N; ++c) {
        if (porous_ts(o, c)) {
            o->Ts[c] = (REAL)Ts[c];
            for (int k = 0; k < o->QT; ++k) o->gs[c*o->QT + k] = o->Gs[c*o->QT + k] = o->wt[k]*o->Ts[c];
        } else if (is_solid(o->mask, c)) {
            o->T[c] = (REAL)Ts[c];
            for (int k = 0; k < o->QT; ++k) o->g[c*o->QT + k] = o->G[c*o->QT + k] = o->wt[k]*o->T[c];
        }
    }
}

/* --------------------------------------------------------------- the step */

/* c0 + T (c1 + T (c2 T + T (c3 + T c4))): conductivity and capacity_m in the reference's
 * evaluation order (LBM2D/_thermal.py:79, :93, :97-99, :182, :196, :200-202) */
static REAL nested5(const double* c, REAL T) {
    return (REAL)c[0] + T*((REAL)c[1] + T*((REAL)c[2]*T + T*((REAL)c[3] + T*(REAL)c[4])));
}

/* Relaxation time of a cell's temperature populations: the phase's constant, or with the
 * phase's bit of tprop TF.tau / TS.tau with the DERIVED coefDiff, cond(T)/rho/cm(T)*dt/dx**2
 * (LBM2D/_thermal.py:62-71, :167-174; rho the cell's density for the fluid, rhos for the
 * solid), tau = 3 D + 1/2 in 2D and 4 D + 1/2 in 3D (_scalarField.py:56-58 of LBM2D/LBM3D),
 * at the temperature the cell's collision uses (T*v_scale + v_ref of its phase) */
static REAL tau_thermal(const orc* o, long c, int solid) {
    int ph = solid ? 1 : 0;
    if (!solid && (o->c.tprop & 4))
        return (REAL)(o->c.dim == 2 ? 3 : 4)*(visc_kin(o, o->rho[c], o->T[c])/(REAL)o->c.tp_prandtl) + (REAL)0.5;
    if (!((o->c.tprop >> ph) & 1)) return solid ? (REAL)o->c.tauT_solid : (REAL)o->c.tauT_fluid;
    REAL Tp = o->T[c]*(REAL)(ph ? o->c.Ts_scale : o->c.T_scale) + (REAL)(ph ? o->c.Ts_ref : o->c.T_ref);
    REAL k = nested5(o->c.tp_cond[ph], Tp);
    REAL cm = (Tp < (REAL)o->c.tp_cap_Tmid[ph] ? nested5(o->c.tp_cap_lo[ph], Tp)
                                              : nested5(o->c.tp_cap_hi[ph], Tp)) * (REAL)o->c.tp_cap_mul[ph];
    REAL D = k / (ph ? (REAL)o->c.tp_rhos : o->rho[c]) / cm * (REAL)o->c.tp_dt / (REAL)o->c.tp_dx2;
    return (REAL)(o->c.dim == 2 ? 3 : 4)*D + (REAL)0.5;
}

/* collision_source_streaming: src/LBM/LBM2D/_evolution.py:26-115 */
static void collide_stream(orc* o) {
    int Q = o->Q, QT = o->QT;
    long N = o->N;
    #pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c) {
        REAL fo[19], go[7];
        int solid = is_solid(o->mask, c);
        if (!solid) {
            collide_flow(o, c, &o->f[c*Q], o->rho[c], &o->u[c*3], o->T[c], fo);
            for (int k = 0; k < Q; ++k) {
                long ip = nbr(o, c, k, +1);
                if (!is_solid(o->mask, ip)) o->F[ip*Q + k] = fo[k];      /* :69-70 */
                else o->F[c*Q + o->opp[k]] = fo[k];                      /* :78-79 halfway bounce-back */
            }
        }
        if (o->c.thermal >= 1) {
            /* conjugate single field: fluid geq advects (TF.geq), solid geq = w T (TS.geq,
             * LBM2D/_thermal.py:162-166); the source enters as geq(dS) (_evolution.py:54-58).
             * Two fields: TF streams only between fluid cells and TS only between solid
             * cells (_evolution.py:69-95), so a link to the other phase bounces back */
            REAL tauT = tau_thermal(o, c, solid);
            for (int k = 0; k < QT; ++k) {
                REAL gk = o->g[c*QT + k];
                REAL ge = solid ? o->wt[k]*o->T[c] : geq_fluid(o, k, o->T[c], &o->u[c*3]);
                /* TF.geq(k, TF.dS) in fluid cells (with the velocity), TS.geq = w dS in solid */
                REAL src = solid ? o->wt[k]*o->dS[c] : geq_fluid(o, k, o->dS[c], &o->u[c*3]);
                go[k] = gk - (REAL)1/tauT*(gk - ge) + src;
            }
            for (int k = 0; k < QT; ++k) {
                long ip = nbr(o, c, k, +1);
                if (solid && porous_ts(o, ip)) o->Gs[ip*QT + k] = go[k];   /* TS into a porous cell, :109-110 */
                else if (o->c.thermal == 2 && k > 0 && is_solid(o->mask, ip) != solid) o->G[c*QT + o->opp[k]] = go[k];
                else o->G[ip*QT + k] = go[k];
            }
            if (porous_ts(o, c)) {
                /* TS of a porous cell: collide towards w T_s, source w dS_s (:39-41, :56-57);
                 * streams into cells with solid > 0 (porous ones: Gs, pure-solid ones: G) and
                 * bounces back at pure-fluid neighbours (:82-89) */
                REAL gso[7];
                for (int k = 0; k < QT; ++k) {
                    REAL gk = o->gs[c*QT + k];
                    gso[k] = gk - (REAL)1/(REAL)o->c.tauT_solid*(gk - o->wt[k]*o->Ts[c]) + o->wt[k]*o->dSs[c];
                }
                for (int k = 0; k < QT; ++k) {
                    long ip = nbr(o, c, k, +1);
                    if (is_solid(o->mask, ip)) o->G[ip*QT + k] = gso[k];
                    else if (porous_ts(o, ip)) o->Gs[ip*QT + k] = gso[k];
                    else o->Gs[c*QT + o->opp[k]] = gso[k];
                }
            }
            if (solid && o->c.thermal == 2 && o->c.ref_quirk_frozen_solid_T)
                for (int k = 0; k < QT; ++k) o->g[c*QT + k] = go[k];   /* TS.g[i][k] = g, :96-100 */
        }
    }
    /* pyrolysis gas release: a reacting solid cell pushes rel*w_k into each fluid
     * neighbour along e_k (new behaviour; no reference counterpart) */
    if (o->c.pyro) {
        #pragma omp parallel for schedule(static)
        for (long y = 0; y < N; ++y) {
            if (is_solid(o->mask, y)) continue;
            for (int k = 1; k < Q; ++k) {
                long x = nbr(o, y, k, -1);
                if (is_solid(o->mask, x) && o->rel[x] != 0)
                    o->F[y*Q + k] += o->rel[x]*o->w[k];
            }
        }
    }
}

/* macro: src/LBM/LBM2D/_evolution.py:118-202, plus pyrolysis and the cell flip */
static void macro(orc* o) {
    int Q = o->Q, QT = o->QT;
    long N = o->N;
    #pragma omp parallel for schedule(static)
    for (long c = 0; c < N; ++c) {
        o->mask_next[c] = o->mask[c];
        if (!is_solid(o->mask, c)) {
            REAL r = 0, j[3] = {0, 0, 0};
            for (int k = 0; k < Q; ++k) {
                REAL Fk = o->F[c*Q + k];
                o->f[c*Q + k] = Fk;
                r += Fk;
                for (int d = 0; d < 3; ++d) j[d] += (REAL)o->e[k][d]*Fk;
            }
            if (o->c.half_force_velocity)
                for (int d = 0; d < 3; ++d) j[d] += (REAL)0.5*(REAL)o->c.force[d]*(o->c.eos == 0 ? r : (REAL)1);
            if (o->c.eos == 0) for (int d = 0; d < 3; ++d) j[d] /= r;
            if (is_porous(o, c)) porous_correct(o, c, r, o->T[c], j);
            o->rho[c] = r;
            for (int d = 0; d < 3; ++d) o->u[c*3 + d] = j[d];
        }
        if (o->c.thermal >= 1 && !(o->c.thermal == 2 && o->c.ref_quirk_frozen_solid_T && is_solid(o->mask, c))) {
            REAL Tc = 0;
            for (int k = 0; k < QT; ++k) { Tc += o->G[c*QT + k]; o->g[c*QT + k] = o->G[c*QT + k]; }
            o->T[c] = Tc;
            o->dS[c] = 0;
        }
        if (porous_ts(o, c)) {
            /* macro of a porous cell: T_s = sum TS.G, then the exchange with TF and the surface
             * radiation as sources of the next collision (src/LBM/LBM2D/_evolution.py:186-202) */
            REAL Tsc = 0;
            for (int k = 0; k < QT; ++k) { Tsc += o->Gs[c*QT + k]; o->gs[c*QT + k] = o->Gs[c*QT + k]; }
            o->Ts[c] = Tsc;
            o->dSs[c] = 0;
            REAL vsf = (REAL)o->c.T_scale, vrf = (REAL)o->c.T_ref;
            REAL vss = (REAL)o->c.Ts_scale, vrs = (REAL)o->c.Ts_ref;
            REAL cf = (REAL)o->c.cap_fluid, cs = (REAL)o->c.cap_solid, dt = (REAL)o->c.dt_phys;
            REAL Tsp = Tsc*vss + vrs;
            REAL dH = o->xh[c]*o->xa[c]*((o->T[c]*vsf + vrf) - Tsp)*dt;
            o->dSs[c] += dH/cs/o->rhos[c]/vss;
            o->dS[c] += -dH/cf/o->rho[c]/vsf;
            if (o->c.radiation) {
                /* TemperatureSolid.radiation, src/LBM/LBM2D/_thermal.py:213-220 */
                REAL q = o->emis[c]*(REAL)ORC_SIGMA*o->rsurf[c]/(REAL)o->c.dx_phys
                         *((REAL)pow((double)(REAL)o->c.T_ambient, 4.0) - (REAL)pow((double)Tsp, 4.0));
                o->dSs[c] += q*dt/cs/o->rhos[c]/vss;
            }
        }
        o->rel[c] = 0;
        if (o->c.pyro && is_solid(o->mask, c) && (o->mask[c] & ORC_REACTIVE)) {
            /* Arrhenius rate, src/LBM/LBM2D/_chemical.py:198-212 with T = T_s */
            REAL a = o->alpha[c];
            REAL TK = o->T[c]*(REAL)o->c.T_scale + (REAL)o->c.T_ref;
            REAL k = 0;
            if (TK > (REAL)o->c.pyro_Tmin)
                k = (REAL)o->c.pyro_A*(REAL)pow((double)(TK + (REAL)1e-6), o->c.pyro_b)
                    *(REAL)exp(-(double)((REAL)o->c.pyro_Ea/(TK + (REAL)1e-6)/(REAL)8.314441));
            REAL da = k*a*(REAL)o->c.dt_phys;
            REAL an = a - da;
            o->alpha[c] = an;
            o->dS[c] = -(REAL)o->c.heat_norm*da;
            REAL mg = (REAL)o->c.gas_coef*da;
            REAL W = 0;
            for (int q = 1; q < Q; ++q) if (!is_solid(o->mask, nbr(o, c, q, +1))) W += o->w[q];
            o->rel[c] = W > 0 ? mg/W : 0;
            if (an < (REAL)o->c.alpha_flip) o->mask_next[c] = o->mask[c] & ~ORC_SOLID;
        }
    }
    /* cell flip: a spent cell turns fluid at the mean rho,u of its fluid neighbours */
    for (long c = 0; c < N; ++c) {
        if (!(is_solid(o->mask, c) && !is_solid(o->mask_next, c))) continue;
        REAL rs = 0, us[3] = {0, 0, 0};
        int n = 0;
        for (int q = 1; q < Q; ++q) {
            long nb = nbr(o, c, q, +1);
            if (is_solid(o->mask, nb)) continue;
            rs += o->rho[nb];
            for (int d = 0; d < 3; ++d) us[d] += o->u[nb*3 + d];
            ++n;
        }
        REAL rb = n ? rs/(REAL)n : (REAL)1;
        REAL ub[3];
        for (int d = 0; d < 3; ++d) ub[d] = n ? us[d]/(REAL)n : 0;
        o->rho[c] = rb;
        for (int d = 0; d < 3; ++d) o->u[c*3 + d] = ub[d];
        for (int k = 0; k < Q; ++k) o->f[c*Q + k] = feq(o, k, rb, ub);
        o->rel[c] = 0;
    }
    memcpy(o->mask, o->mask_next, (size_t)N);
}

/* Non-equilibrium extrapolation on one boundary cell b with inner neighbour i.
 * Flow: src/LBM/LBM2D/_boundary.py:54-101 (3D: LBM3D/_boundary.py:71-142).
 * Scalar: src/LBM/LBM2D/_scalarField.py:83-122. */
static void nee_cell(orc* o, const orc_side* s, long b, long i, const REAL* prof) {
    int Q = o->Q, QT = o->QT;
    REAL* ub = &o->u[b*3];
    const REAL* ui = &o->u[i*3];
    if (s->v_type == ORC_BC_FIXED) for (int d = 0; d < 3; ++d) ub[d] = (REAL)s->v[d];
    else if (s->v_type == ORC_BC_FLOWRATE) for (int d = 0; d < 3; ++d) ub[d] = prof[d];
    else if (s->v_type == ORC_BC_ZEROGRAD) for (int d = 0; d < 3; ++d) ub[d] = ui[d];
    if (s->rho_type == ORC_BC_FIXED) o->rho[b] = (REAL)s->rho;
    else if (s->rho_type == ORC_BC_ZEROGRAD) o->rho[b] = o->rho[i];
    for (int k = 0; k < Q; ++k)
        o->f[b*Q + k] = s->active == 2   /* ES, src/LBM/LBM2D/_boundary.py:269-315 */
            ? feq(o, k, o->rho[b], ub)
            : feq(o, k, o->rho[b], ub) + (o->f[i*Q + k] - feq(o, k, o->rho[i], ui));
    if (o->c.thermal >= 1) {
        if (s->T_type == ORC_BC_FIXED) o->T[b] = (REAL)s->T;
        else if (s->T_type == ORC_BC_ZEROGRAD) o->T[b] = o->T[i];
        for (int k = 0; k < QT; ++k) {
            o->G[b*QT + k] = geq_fluid(o, k, o->T[b], ub) + (o->G[i*QT + k] - geq_fluid(o, k, o->T[i], ui));
            o->g[b*QT + k] = o->G[b*QT + k];
        }
    }
}

/* Boundary_condition_NEE: x sides first (loop over j,k), then y sides (i,k), then z (i,j).
 * src/LBM/LBM2D/_boundary.py:17-52, LBM3D/_boundary.py:15-68. */
static void nee(orc* o) {
    int nx = o->c.nx, ny = o->c.ny, nz = o->c.nz;
    const orc_side* S = o->c.side;
    for (int z = 0; z < nz; ++z) for (int y = 0; y < ny; ++y) {
        if (S[0].active && S[0].active != 3) nee_cell(o, &S[0], cidx(o, 0, y, z), cidx(o, 1, y, z), &o->inl_prof[3*(y + (long)ny*z)]);
        if (S[1].active && S[1].active != 3) nee_cell(o, &S[1], cidx(o, nx-1, y, z), cidx(o, nx-2, y, z), NULL);
    }
    for (int z = 0; z < nz; ++z) for (int x = 0; x < nx; ++x) {
        if (S[2].active && S[2].active != 3) nee_cell(o, &S[2], cidx(o, x, 0, z), cidx(o, x, 1, z), NULL);
        if (S[3].active && S[3].active != 3) nee_cell(o, &S[3], cidx(o, x, ny-1, z), cidx(o, x, ny-2, z), NULL);
    }
    if (o->c.dim == 3)
        for (int y = 0; y < ny; ++y) for (int x = 0; x < nx; ++x) {
            if (S[4].active) nee_cell(o, &S[4], cidx(o, x, y, 0), cidx(o, x, y, 1), NULL);
            if (S[5].active) nee_cell(o, &S[5], cidx(o, x, y, nz-1), cidx(o, x, y, nz-2), NULL);
        }
}

/* Non-equilibrium bounce-back (Zou & He 1997) on the post-stream F of a D2Q9 side cell,
 * Boundary_condition_flow_NEBB_0..3 (src/LBM/LBM2D/_boundary.py:145-226), before macro:
 * the populations entering from outside are rebuilt from the known ones so that the cell
 * gets the side's velocity (wall / inlet: velocity fixed) or density (outlet).  Velocity
 * order 0 rest, 1 +x, 2 +y, 3 -x, 4 -y, 5 (+,+), 6 (-,+), 7 (-,-), 8 (+,-); the
 * expressions keep the reference's operation order. */
static void nebb_cell(orc* o, int side, long c) {
    REAL* F = &o->F[c*9];
    const orc_side* s = &o->c.side[side];
    const int vel = s->v_type == ORC_BC_FIXED, pres = s->rho_type == ORC_BC_FIXED;
    const int wall = vel && s->v[0] == 0 && s->v[1] == 0;
    const int q = o->c.ref_quirk_nebb;
    const REAL u = (REAL)s->v[0], v = (REAL)s->v[1], r0 = (REAL)s->rho;
    const REAL c23 = (REAL)(2.0/3.0), c16 = (REAL)(1.0/6.0), h = (REAL)0.5;
    REAL rho, w;
    switch (side) {
    case 0:   /* x = 0: F1, F5, F8 unknown */
        if (vel) {
            rho = (F[0]+F[2]+F[4]+2*(F[3]+F[6]+F[7]))/((REAL)1-u);
            F[1] = F[3] + c23*rho*u;
            F[5] = F[7] + h*(F[4]-F[2]) + c16*rho*u + h*rho*v;
            F[8] = F[6] + h*(F[2]-F[4]) + c16*rho*u - h*rho*v;
        } else if (pres) {
            rho = r0;
            w = q ? (REAL)-1 + (2*(F[3]+F[6]+F[7])+F[0]+F[2]+F[4])/rho
                  : (REAL)1 - (F[0]+F[2]+F[4]+2*(F[3]+F[6]+F[7]))/rho;
            F[1] = F[3] + c23*rho*w;
            F[5] = F[7] + h*(F[4]-F[2]) + c16*rho*w;
            F[8] = F[6] + h*(F[2]-F[4]) + c16*rho*w;
        }
        break;
    case 1:   /* x = nx-1: F3, F6, F7 unknown */
        if (vel && q) {
            if (wall) {   /* the reference rebuilds side 0's populations here */
                F[1] = F[3];
                F[5] = F[7] + h*(F[4]-F[2]);
                F[8] = F[6] + h*(F[2]-F[4]);
            }
        } else if (vel) {
            rho = (F[0]+F[2]+F[4]+2*(F[1]+F[5]+F[8]))/((REAL)1+u);
            F[3] = F[1] - c23*rho*u;
            F[6] = F[8] + h*(F[4]-F[2]) - c16*rho*u + h*rho*v;
            F[7] = F[5] + h*(F[2]-F[4]) - c16*rho*u - h*rho*v;
        } else if (pres) {
            rho = r0;
            w = (REAL)-1 + (2*(F[1]+F[5]+F[8])+F[0]+F[2]+F[4])/rho;
            F[3] = F[1] - c23*rho*w;
            F[6] = F[8] + h*(F[4]-F[2]) - c16*rho*w;
            F[7] = F[5] + h*(F[2]-F[4]) - c16*rho*w;
        }
        break;
    case 2:   /* y = 0: F2, F5, F6 unknown */
        if (vel && (wall || !q)) {
            rho = (F[0]+F[1]+F[3]+2*(F[4]+F[7]+F[8]))/((REAL)1-v);
            F[2] = F[4] + c23*rho*v;
            F[5] = F[7] + h*(F[3]-F[1]) + h*rho*u + c16*rho*v;
            F[6] = F[8] + h*(F[1]-F[3]) - h*rho*u + c16*rho*v;
        } else if (pres && !q) {
            rho = r0;
            w = (REAL)1 - (F[0]+F[1]+F[3]+2*(F[4]+F[7]+F[8]))/rho;
            F[2] = F[4] + c23*rho*w;
            F[5] = F[7] + h*(F[3]-F[1]) + c16*rho*w;
            F[6] = F[8] + h*(F[1]-F[3]) + c16*rho*w;
        }
        break;
    case 3:   /* y = ny-1: F4, F7, F8 unknown */
        if (vel && (wall || !q)) {
            rho = (F[0]+F[1]+F[3]+2*(F[2]+F[5]+F[6]))/((REAL)1+v);
            F[4] = F[2] - c23*rho*v;
            F[7] = F[5] + h*(F[1]-F[3]) - h*rho*u - c16*rho*v;
            F[8] = F[6] + h*(F[3]-F[1]) + h*rho*u - c16*rho*v;
        } else if (pres && !q) {
            rho = r0;
            w = (REAL)-1 + (F[0]+F[1]+F[3]+2*(F[2]+F[5]+F[6]))/rho;
            F[4] = F[2] - c23*rho*w;
            F[7] = F[5] + h*(F[1]-F[3]) - c16*rho*w;
            F[8] = F[6] + h*(F[3]-F[1]) - c16*rho*w;
        }
        break;
    }
}

/* Boundary_condition_NEBB (src/LBM/LBM2D/_boundary.py:103-141): the x sides on rows 1 ..
 * ny-2, then the y sides on every column. */
static void nebb(orc* o) {
    const orc_side* S = o->c.side;
    int nx = o->c.nx, ny = o->c.ny;
    for (int y = 1; y < ny - 1; ++y) {
        if (S[0].active == 3 && !is_solid(o->mask, cidx(o, 0, y, 0))) nebb_cell(o, 0, cidx(o, 0, y, 0));
        if (S[1].active == 3 && !is_solid(o->mask, cidx(o, nx-1, y, 0))) nebb_cell(o, 1, cidx(o, nx-1, y, 0));
    }
    for (int x = 0; x < nx; ++x) {
        if (S[2].active == 3 && !is_solid(o->mask, cidx(o, x, 0, 0))) nebb_cell(o, 2, cidx(o, x, 0, 0));
        if (S[3].active == 3 && !is_solid(o->mask, cidx(o, x, ny-1, 0))) nebb_cell(o, 3, cidx(o, x, ny-1, 0));
    }
}

/* Flow-rate inlet, updateBC_kernel (src/LBM/LBM2D/_boundary.py:324-333), run before
 * the step: flow0 = sum of rho*u_x over the side-0 cells, coef = F/flow0, and the
 * profile of side cell j is (a*coef + 1 - a) * u(1,j), a = 0.01, from the fields
 * the previous step left (inl_m, inl_w; flow0 summed in double). */
static void flowrate_update(orc* o) {
    long M = (long)o->c.ny * o->c.nz;
    double flow0 = 0;
    for (long j = 0; j < M; ++j) flow0 += (double)o->inl_m[j];
    REAL coef = (REAL)(o->c.side[0].v[0] / flow0);
    REAL a = (REAL)0.01;
    REAL gain = a*coef + (REAL)1 - a;
    for (long j = 0; j < 3*M; ++j) o->inl_prof[j] = gain*o->inl_w[j];
}

/* What the next update reads: rho*u_x at x = 0 and u at x = 1 after macro and NEE. */
static void flowrate_record(orc* o) {
    for (int z = 0; z < o->c.nz; ++z) for (int y = 0; y < o->c.ny; ++y) {
        long j = y + (long)o->c.ny*z, b = cidx(o, 0, y, z), i = cidx(o, 1, y, z);
        o->inl_m[j] = o->rho[b]*o->u[b*3];
        for (int d = 0; d < 3; ++d) o->inl_w[3*j + d] = o->u[i*3 + d];
    }
}

/* step: src/LBM/LBM2D/_evolution.py:12-25 (updateBC, then step_kernel) */
void orc_step(orc* o, int n) {
    int fr = o->c.side[0].active && o->c.side[0].v_type == ORC_BC_FLOWRATE;
    int nebb_on = 0;
    for (int i = 0; i < 4; ++i) nebb_on |= o->c.side[i].active == 3;
    for (int i = 0; i < n; ++i) {
        if (fr) flowrate_update(o);
        collide_stream(o);
        if (nebb_on) nebb(o);
        macro(o);
        nee(o);
        if (fr) flowrate_record(o);
    }
}

/* Read back macroscopic fields (planar u) and the current mask / reactive fraction. */
void orc_get(const orc* o, double* rho, double* u, double* T, uint8_t* mask, double* alpha) {
    long N = o->N;
    for (long c = 0; c < N; ++c) {
        if (rho) rho[c] = o->rho[c];
        if (u) for (int d = 0; d < 3; ++d) u[d*N + c] = o->u[c*3 + d];
        if (T) T[c] = o->T[c];
        if (mask) mask[c] = o->mask[c];
        if (alpha) alpha[c] = o->alpha[c];
    }
}

/* Solid temperature TS.S of porous cells and, with two fields, of pure-solid cells (0 in
 * pure-fluid cells), and the TS populations of porous cells (planar; 0 elsewhere). */
void orc_get_solid_T(const orc* o, double* Ts, double* gs) {
    long N = o->N;
    for (long c = 0; c < N; ++c) {
        int p = porous_ts(o, c);
        if (Ts) Ts[c] = p ? o->Ts[c] : (o->c.thermal == 2 && is_solid(o->mask, c) ? o->T[c] : 0);
        if (gs) for (int k = 0; k < o->QT; ++k) gs[k*N + c] = p ? o->gs[c*o->QT + k] : 0;
    }
}

/* The oracle's per-cell state that the next step reads (test infrastructure: slab
 * decomposition tests exchange planes of it between ranks), cell-major: id 0 f [N][Q],
 * 1 g [N][QT], 2 rho [N], 3 u [N][3], 4 T [N], 5 dS [N], 6 alpha [N], 7 rel [N],
 * 8 mask [N] (bytes), 9 gs [N][QT], 10 Ts [N], 11 dSs [N].  *n: elements per cell
 * (0 when the array does not exist). */
void* orc_array(orc* o, int id, int* n) {
    int Q = o->Q, QT = o->QT;
    void* p = NULL;
    int m = 0;
    switch (id) {
    case 0: p = o->f; m = Q; break;
    case 1: p = o->g; m = QT; break;
    case 2: p = o->rho; m = 1; break;
    case 3: p = o->u; m = 3; break;
    case 4: p = o->T; m = 1; break;
    case 5: p = o->dS; m = 1; break;
    case 6: p = o->alpha; m = 1; break;
    case 7: p = o->rel; m = 1; break;
    case 8: p = o->mask; m = 1; break;
    case 9: p = o->gs; m = o->gs ? QT : 0; break;
    case 10: p = o->Ts; m = o->Ts ? 1 : 0; break;
    case 11: p = o->dSs; m = o->dSs ? 1 : 0; break;
    }
    *n = p ? m : 0;
    return p;
}

/* Post-stream distributions (f after macro/NEE), planar: out[k*N + c]. */
void orc_get_dist(const orc* o, double* f, double* g) {
    long N = o->N;
    for (long c = 0; c < N; ++c) {
        if (f) for (int k = 0; k < o->Q; ++k) f[k*N + c] = o->f[c*o->Q + k];
        if (g) for (int k = 0; k < o->QT; ++k) g[k*N + c] = o->g[c*o->QT + k];
    }
}

/* Diagnostics over the current state (new: the reference only has max|v|, min/max T,
 * src/LBM/LBM2D/_io.py:565-588).  out: [0] mass (sum rho, fluid), [1] energy (sum T,
 * all cells), [2] reactive solid fraction sum, [3] max |u| (fluid), [4] min T, [5] max T,
 * [6] non-finite count, [7] fluid cell count. */
void orc_diag(const orc* o, double* out) {
    double mass = 0, en = 0, sm = 0, umax2 = 0, tmin = 1e300, tmax = -1e300, nan = 0, nf = 0;
    for (long c = 0; c < o->N; ++c) {
        double T = o->c.thermal ? (double)o->T[c] : 0;
        if (!isfinite(T)) nan += 1;
        en += T;
        if (T < tmin) tmin = T;
        if (T > tmax) tmax = T;
        if (is_solid(o->mask, c)) {
            if (o->mask[c] & ORC_REACTIVE) sm += o->alpha[c];
            continue;
        }
        double r = o->rho[c];
        if (!isfinite(r)) nan += 1;
        mass += r;
        nf += 1;
        double u2 = 0;
        for (int d = 0; d < 3; ++d) u2 += (double)o->u[c*3+d]*(double)o->u[c*3+d];
        if (u2 > umax2) umax2 = u2;
    }
    out[0] = mass; out[1] = en; out[2] = sm; out[3] = sqrt(umax2);
    out[4] = tmin; out[5] = tmax; out[6] = nan; out[7] = nf;
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}
