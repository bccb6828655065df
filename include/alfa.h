/*
 * libalfa: B200 (sm_100a) implementation of the JAX-ALFA per-timestep LES
 * hot path behind a plain C ABI: the FP64 drop-in, and FP32 / mixed-precision
 * forms of the same step (alfa_config.precision).
 *
 * Conventions (identical to the reference's arrays, so no transposes at the
 * boundary):
 *   - every array pointer is a DEVICE pointer unless a comment says "host";
 *   - real 3-D fields are (nx, ny, nz) C-order doubles, z fastest;
 *   - spectra are (nx, ny/2+1, nz) interleaved complex doubles (re, im),
 *     i.e. numpy.fft.rfft2(F, axes=(0, 1)) of such a field;
 *   - padded fields (Dealias1 output) are (mx, my, nz), mx = 1.5 nx;
 *   - the pressure system is (nx, ny/2+1, nz+1) real and imaginary parts;
 *   - 2-D surface planes are (nx, ny); vertical profiles are (nz).
 * All calls are asynchronous on the context's stream (alfa_set_stream) and
 * return 0 or a negative ALFA_E_* code; alfa_last_error() describes it.
 * Nothing here calls exit/abort or traps on the device.
 *
 * Static, configuration-derived reference arguments (kx2, ky2, the pressure
 * wavenumbers, b_thomas, m_thomas, c_pressure, the Rayleigh damping arrays,
 * the ZeRo* scratch arrays) live in the context and are not passed.
 * Reference citations are path:line inside the JAX-ALFA project.
 */
#ifndef ALFA_H
#define ALFA_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ALFA_OK 0
#define ALFA_E_CONFIG (-1)   /* unsupported or inconsistent configuration */
#define ALFA_E_SHAPE (-2)    /* a size or pointer argument is invalid      */
#define ALFA_E_CUDA (-3)     /* a CUDA runtime call or launch failed       */
#define ALFA_E_NUMERIC (-4)  /* non-finite state detected                  */
#define ALFA_E_TIMEOUT (-5)  /* a bounded device wait gave up              */
#define ALFA_E_STATE (-6)    /* call order (e.g. step before init_state)   */
#define ALFA_E_NOALLOC_LIMIT (-7) /* size above a no-allocation entry's limit */

typedef struct alfa_ctx alfa_ctx;

/* Option names and units of the reference's Config.py
 * (src/config/ConfigLoader.py:70-157, examples/NBL_A94/runs/.../Config.py). */
typedef struct alfa_config {
  int nx, ny, nz;
  double l_x, l_y, l_z;          /* m */
  double dt;                     /* s */
  int istep;
  double Ugal;                   /* m/s */
  int optSurfFlux;               /* 0 homogeneous, 1 heterogeneous */
  int optSurfBC;                 /* 0 const flux, 1 flux series, 2 temperature series */
  double z0m, z0T, zTemperature; /* m */
  double SensibleHeatFlux;       /* K m/s */
  double Ug2, Vg2;               /* m/s (optGeoWind = 0) */
  double f_coriolis;             /* 1/s */
  double inversion;              /* K/m */
  int optBuoyancy;               /* 0: /T_0, 1: /<THv> */
  double T_0;                    /* K */
  int optSgs;                    /* 0 static, 1 LASDD-SM, 2 LASDD-WL, 3 LAD-SM, 4 LAD-WL */
  int dynamicSGS_call_time;
  int FGR;                       /* 1: 3/2-rule dealiasing, TFR 2; >= 2: no dealiasing, TFR sqrt(2) */
  double Cs2, Cs2PrRatio;        /* initial coefficients (Cwl, CwlPrRatio for optSgs 2, 4) */
  int optDamping;
  double z_damping, RelaxTime;   /* m, s */
  int optAdvection;
  int optPressureSolver;         /* 1 Thomas, 0 dense (same tridiagonal system) */
  int optGeoWind;                /* 0 constant Ug2, Vg2; 1 time/height-varying series
                                    (alfa_set_geowind_series), ConfigLoader.py:77-82 */
  /* moisture (ConfigLoader.py:100-124, DerivedVars.py:69-75) */
  int optMoisture;               /* 0 dry, 1 specific humidity Q transported */
  int optMoistureSurfBC;         /* 0 constant MoistureFlux, 1 flux series, 2 surface Q series */
  double MoistureFlux;           /* kg/kg m/s */
  double zMoisture;              /* m; reference height of the prescribed-Q flux (0: z0T) */
  double q_inversion;            /* kg/kg/m, Q lapse rate above the domain top */
  /* Storage precision of the context's engine (no counterpart field in the
   * reference's Config.py, whose use_double_precision switch,
   * src/config/ConfigLoader.py:150-151 and src/initialization/Preprocess.py:
   * 112-133, selects FP64 or FP32 for everything):
   *   ALFA_FP64  fields, transforms and arithmetic in FP64 (the drop-in);
   *   ALFA_FP32  fields and transforms in FP32; FP64 kept in the pressure
   *              tridiagonal solve and its zero mode, the plane sums and means,
   *              the beta quintic roots, the surface-layer (MOST) planes, the
   *              profiles and series, and the arithmetic of the pointwise
   *              kernels (values rounded to FP32 where they are stored);
   *   ALFA_MIXED ALFA_FP32 plus the horizontal line transforms on the tensor
   *              cores in split BF16 wherever the autotuner (alfa_autotune)
   *              measures them faster than the FP32 transform.
   * FP32 and mixed contexts serve the whole-step entry points (state as FP64
   * device buffers, converted on import and export); the per-function entry
   * points take FP64 arrays and return ALFA_E_CONFIG on them. */
  int precision;
} alfa_config;

#define ALFA_FP64 0
#define ALFA_FP32 1
#define ALFA_MIXED 2

/* Derived constants (src/config/DerivedVars.py:48-112, Preprocess.py:44-62). */
typedef struct alfa_derived {
  int mx, my, nx_rfft, ny_rfft;
  double z_scale, g_nondim, f_coriolis_nondim, T_0_nondim, inversion_nondim;
  double dx, dy, dz, L, dt_nondim, TFR;
  int cut_explicit[2], cut_level1[2], cut_level2[2];
} alfa_derived;

/* Per-step diagnostics of the whole-step driver (host struct). */
typedef struct alfa_diag {
  int iteration;        /* next iteration number (Main.py loop variable) */
  double CFL, CFLmax;   /* Main.py:534-540 */
  double ustar_rms;     /* sqrt(mean(ustar^2)), Main.py:576 */
  double qz_sfc_avg;    /* non-dimensional surface heat flux */
} alfa_diag;

/* ---- context ----------------------------------------------------------- */
/* Replaces the static initialisation of src/Main.py:46-62 (Wavenumber,
 * ThomasPressureInit / PressureInit) and DerivedVars. */
int alfa_create(const alfa_config* cfg, alfa_ctx** out);
void alfa_destroy(alfa_ctx* ctx);
const char* alfa_last_error(const alfa_ctx* ctx);
int alfa_set_stream(alfa_ctx* ctx, void* cuda_stream);
/* ALFA_FP64, ALFA_FP32 or ALFA_MIXED (no reference counterpart) */
int alfa_get_precision(const alfa_ctx* ctx);
int alfa_get_derived(const alfa_ctx* ctx, alfa_derived* out /* host */);
size_t alfa_workspace_bytes(const alfa_ctx* ctx);

/* ---- src/operations ---------------------------------------------------- */
int alfa_FFT(alfa_ctx*, const double* F, double* F_fft);                 /* FFT.py:44 */
int alfa_FFT_pad(alfa_ctx*, const double* F_pad, double* F_pad_fft);     /* FFT.py:68 */
int alfa_Dealias1(alfa_ctx*, const double* F_fft, double* F_pad);        /* Dealiasing.py:51 */
int alfa_Dealias2(alfa_ctx*, const double* F_pad_fft, double* F);        /* Dealiasing.py:86 */
int alfa_Filtering_Explicit(alfa_ctx*, const double* F_fft, double* F_new,
                            double* F_fft_new);                          /* Filtering.py:50 */
int alfa_Filtering_Level1(alfa_ctx*, const double* F_fft, double* F_hat);  /* Filtering.py:97 */
int alfa_Filtering_Level2(alfa_ctx*, const double* F_fft, double* F_hatd); /* Filtering.py:135 */
/* axis 0: kx2, axis 1: ky2 */
int alfa_Derivxy(alfa_ctx*, const double* F_fft, int axis, double* dFdxy); /* Derivatives.py:161 */
/* out[9] = dudx, dvdx, dwdx, dudy, dvdy, dwdy, dudz, dvdz, dwdz */
int alfa_velocityGradients(alfa_ctx*, const double* u, const double* v, const double* w,
                           const double* u_fft, const double* v_fft, const double* w_fft,
                           const double* ustar, const double* M_sfc_loc, const double* fi2D_m,
                           double* const out[9]);                        /* Derivatives.py:47 */
/* out[3] = dTHdx, dTHdy, dTHdz */
int alfa_potentialTemperatureGradients(alfa_ctx*, const double* TH, const double* ustar,
                                       const double* qz_sfc, const double* fi2D_h,
                                       double* const out[3]);            /* Derivatives.py:107 */
/* out[3] = dQdx, dQdy, dQdz: the theta form with the moisture flux qm_sfc */
int alfa_moistureGradients(alfa_ctx*, const double* Q, const double* ustar,
                           const double* qm_sfc, const double* fi2D_h,
                           double* const out[3]);                    /* Derivatives.py:281 */
int alfa_Derivz_Generic_uvp(alfa_ctx*, const double* F, double* dFdz);  /* Derivatives.py:310 */
int alfa_Derivz_Generic_w(alfa_ctx*, const double* F, double* dFdz);    /* Derivatives.py:340 */

/* ---- src/utilities ----------------------------------------------------- */
int alfa_PlanarMean(alfa_ctx*, const double* F, double* mean_nz);        /* Utilities.py:41 */
/* every (x, y) plane of an (nx, ny, nz) field */
int alfa_Imfilter(alfa_ctx*, const double* F, double* out);              /* Utilities.py:87 */
/* Laguerre roots of nlev quintics from each of the 8 beta guesses, then the
 * beta selection of ComputeBeta1/2: coeffs (6, nlev) = ff, ee, dd, cc, bb, aa */
int alfa_ComputeBeta(alfa_ctx*, const double* coeffs, int nlev, double* beta);
                                         /* DynamicSGS_LASDD_SM.py:53, Utilities.py:123 */

/* ---- src/surface/SurfaceFlux.py:166-443 --------------------------------
 * most_in / most_out: psi2D_m, psi2D_m0, psi2D_h, psi2D_h0, fi2D_m, fi2D_h.
 * qz_sfc_avg is a device scalar; sfc_val is the series value of this step. */
int alfa_SurfaceFlux_HomogeneousConstantFlux(alfa_ctx*, const double* u, const double* v,
    const double* TH, const double* const most_in[6], double* M_sfc_loc, double* ustar,
    double* qz_sfc_avg, double* invOB, double* const most_out[6]);          /* :166 */
int alfa_SurfaceFlux_HeterogeneousConstantFlux(alfa_ctx*, const double* u, const double* v,
    const double* TH, const double* const most_in[6], double* M_sfc_loc, double* ustar,
    double* qz_sfc_avg, double* invOB, double* const most_out[6]);          /* :209 */
int alfa_SurfaceFlux_HomogeneousVaryingFlux(alfa_ctx*, const double* u, const double* v,
    const double* TH, double sfc_val, const double* const most_in[6], double* M_sfc_loc,
    double* ustar, double* qz_sfc_2D, double* qz_sfc_avg, double* invOB,
    double* const most_out[6]);                                              /* :246 */
int alfa_SurfaceFlux_HeterogeneousVaryingFlux(alfa_ctx*, const double* u, const double* v,
    const double* TH, double sfc_val, const double* const most_in[6], double* M_sfc_loc,
    double* ustar, double* qz_sfc_2D, double* qz_sfc_avg, double* invOB,
    double* const most_out[6]);                                              /* :290 */
int alfa_SurfaceFlux_HomogeneousPrescribedTemperature(alfa_ctx*, const double* u,
    const double* v, const double* TH, double sfc_val, const double* const most_in[6],
    double* M_sfc_loc, double* ustar, double* qz_sfc_2D, double* qz_sfc_avg, double* invOB,
    double* const most_out[6]);                                              /* :335 */
int alfa_SurfaceFlux_HeterogeneousPrescribedTemperature(alfa_ctx*, const double* u,
    const double* v, const double* TH, double sfc_val, const double* const most_in[6],
    double* M_sfc_loc, double* ustar, double* qz_sfc_2D, double* qz_sfc_avg, double* invOB,
    double* const most_out[6]);                                              /* :393 */
/* optMoistureSurfBC = 2: the surface moisture flux qm_sfc_2D (nx, ny) from
 * the prescribed surface humidity Q_sfc_t (kg/kg) and psi2D_h, psi2D_h0 of
 * MOSTfunctions (most[2], most[3]; the other four are not read). */
int alfa_SurfaceMoistureFlux_HomogeneousPrescribedQ(alfa_ctx*, const double* Q,
    const double* ustar, double Q_sfc_t, const double* const most[6],
    double* qm_sfc_2D);                                                      /* :452 */
int alfa_SurfaceMoistureFlux_HeterogeneousPrescribedQ(alfa_ctx*, const double* Q,
    const double* ustar, double Q_sfc_t, const double* const most[6],
    double* qm_sfc_2D);                                                      /* :483 */

/* ---- src/pde ------------------------------------------------------------ */
int alfa_Advection(alfa_ctx*, const double* u, const double* v, const double* w,
                   const double* dudy, const double* dudz, const double* dvdx,
                   const double* dvdz, const double* dwdx, const double* dwdy,
                   double* Cx, double* Cy, double* Cz);      /* NSE_AdvectionTerms.py:246 */
int alfa_ScalarAdvection(alfa_ctx*, const double* u, const double* v, const double* w,
                         const double* dsdx, const double* dsdy, const double* dsdz,
                         double* out);                        /* SCL_AdvectionTerms.py:158 */
int alfa_BuoyancyOpt1(alfa_ctx*, const double* TH, const double* H /* Q or NULL */,
                      double* buoyancy); /* NSE_BuoyancyTerms.py:49 */
int alfa_BuoyancyOpt2(alfa_ctx*, const double* TH, const double* H /* Q or NULL */,
                      double* buoyancy); /* NSE_BuoyancyTerms.py:104 */

/* grads[9] as velocityGradients' out.  mom[25] receives DynamicSGS's tuple
 * (DynamicSGS_Main.py:323-331): txx, tyy, tzz, txy, txz, tyz, Cs2_1D_avg1,
 * Cs2_1D_avg2, beta1_1D, Cs2_3D, u_, v_, w_, u_hat, v_hat, w_hat, u_hatd,
 * v_hatd, w_hatd, S_uvp, S_uvp_pad (mx,my,nz; (nx,ny,nz) when FGR > 1), S_w,
 * S_w_pad (as S_uvp_pad),
 * S_uvp_hat, S_uvp_hatd.  Entries 6..9 may be NULL (they duplicate the
 * dedicated outputs).                                  NSE_SGSTerms.py:113 */
int alfa_DivStressDynamicSGS(alfa_ctx*, const double* const grads[9], const double* u,
                             const double* v, const double* w, const double* M_sfc_loc,
                             const double* psi2D_m, const double* psi2D_m0, double* divtx,
                             double* divty, double* divtz, double* Cs2_1D_avg1,
                             double* Cs2_1D_avg2, double* beta1_1D, double* Cs2_3D,
                             double* const mom[25]);
/* mom15 = mom[10..24] of the call above.               SCL_SGSTerms.py:97 */
int alfa_DivFluxDynamicSGS(alfa_ctx*, const double* const mom15[15], const double* TH,
                           const double* dTHdx, const double* dTHdy, const double* dTHdz,
                           const double* qz_sfc, double* qz, double* divq,
                           double* Cs2PrRatio_3D, double* Cs2PrRatio_1D, double* beta2_1D);
/* mom[10] receives StaticSGS's tuple (StaticSGS_Main.py:248-250): txx, tyy,
 * tzz, txy, txz, tyz, S_uvp, S_uvp_pad, S_w, S_w_pad.   NSE_SGSTerms.py:186 */
int alfa_DivStressStaticSGS(alfa_ctx*, const double* const grads[9], const double* Cs2_3D,
                            const double* u, const double* v, const double* M_sfc_loc,
                            const double* psi2D_m, const double* psi2D_m0, double* divtx,
                            double* divty, double* divtz, double* const mom[10]);
/* mom4 = S_uvp, S_uvp_pad, S_w, S_w_pad.              SCL_SGSTerms.py:169 */
int alfa_DivFluxStaticSGS(alfa_ctx*, const double* const mom4[4], const double* Cs2PrRatio_3D,
                          const double* dTHdx, const double* dTHdy, const double* dTHdz,
                          const double* qz_sfc, double* qz, double* divq);

/* Ug, Vg, Uadv, Vadv, THadv are the (nz) profiles the reference broadcasts
 * over (nx, ny, nz) (Main.py:82, 120-122, Initialization.py:163-170). */
int alfa_RHS_Momentum(alfa_ctx*, const double* u, const double* v, const double* w,
                      const double* Ug, const double* Vg, const double* Cx, const double* Cy,
                      const double* Cz, const double* buoyancy, const double* divtx,
                      const double* divty, const double* divtz, const double* Uadv,
                      const double* Vadv, double* RHS_u, double* RHS_v,
                      double* RHS_w);                          /* NSE_AllTerms.py:48 */
int alfa_RHS_Scalar(alfa_ctx*, const double* TH, const double* THAdvectionSum,
                    const double* divq, const double* THadv, double* RHS_TH); /* SCL_AllTerms.py:48 */
/* Qadv: (nz) profile, always added */
int alfa_RHS_Moisture(alfa_ctx*, const double* Q, const double* QAdvectionSum,
                      const double* divqm, const double* Qadv, double* RHS_Q); /* SCL_AllTerms.py:86 */
int alfa_PressureRC(alfa_ctx*, const double* u, const double* v, const double* w,
                    const double* RHS_u, const double* RHS_v, const double* RHS_w,
                    const double* RHS_u_previous, const double* RHS_v_previous,
                    const double* RHS_w_previous, const double* divtz, double* RC_real,
                    double* RC_imag, double* fRz_real);        /* NSE_PressureTerms.py:109 */
int alfa_ThomasPressureSolve(alfa_ctx*, const double* RC_real, const double* RC_imag,
                             const double* fRz_real, double* p, double* dpdx, double* dpdy,
                             double* dpdz);           /* NSE_PressureTerms_Thomas.py:218 */
/* in place allowed (x_new == x) */
int alfa_AB2_uvw(alfa_ctx*, const double* u, const double* v, const double* w,
                 const double* RHS_u, const double* RHS_u_previous, const double* RHS_v,
                 const double* RHS_v_previous, const double* RHS_w,
                 const double* RHS_w_previous, double* u_new, double* v_new,
                 double* w_new);                          /* NSE_TimeAdvancement.py:45 */
int alfa_AB2_TH(alfa_ctx*, const double* TH, const double* RHS_TH,
                const double* RHS_TH_previous, double* TH_new); /* SCL_TimeAdvancement.py:46 */
int alfa_AB2_Q(alfa_ctx*, const double* Q, const double* RHS_Q, const double* RHS_Q_previous,
               double* Q_new);                              /* SCL_TimeAdvancement.py:79 */

/* Main.py:498-500 — RHS_i -= dp/dx_i, in place. */
int alfa_AddPressureGradient(alfa_ctx*, double* RHS_u, double* RHS_v, double* RHS_w,
                             const double* dpdx, const double* dpdy, const double* dpdz);
/* Main.py:534-536 — cfl3 (device) = max|u| dt/dx, max|v| dt/dy, max|w| dt/dz. */
int alfa_CFL(alfa_ctx*, const double* u, const double* v, const double* w, double* cfl3);

/* ---- whole step: the loop body of src/Main.py:156-541 -------------------
 * State is held in the context.  init_state takes non-dimensional fields as
 * Main.py holds them after Initialize_uvw/TH (u without Ugal, TH - T_0).
 * Series (host pointers, copied): Uadv/Vadv/THadv (nrows, nz) non-dimensional
 * (Initialize_AdvForcing), sfc (nrows) non-dimensional (Initialize_SurfaceBC);
 * row iteration-1 is used at each iteration, as in Main.py:179-188, 225. */
int alfa_init_state(alfa_ctx*, const double* u, const double* v, const double* w,
                    const double* TH);
int alfa_set_series(alfa_ctx*, const double* Uadv, const double* Vadv, const double* THadv,
                    const double* sfc, int nrows);
/* optGeoWind = 1: the geostrophic wind series (host, copied), Ug and Vg
 * (nrows, nz) non-dimensional as Initialize_GeoWind_Varying returns them
 * (Initialization.py:163-246); row iteration-1 is the profile of each
 * iteration (Main.py:84-86, 170-174). */
int alfa_set_geowind_series(alfa_ctx*, const double* Ug, const double* Vg, int nrows);
/* optMoisture = 1 (Main.py:71-76): the initial specific humidity Q (device,
 * kg/kg as Initialize_Q loads it; required before the first step), and the
 * moisture series (host, copied): Qadv (nrows, nz) non-dimensional
 * (Initialize_AdvForcing's AdvForcing_Q, or NULL) and msfc (nrows) as
 * Initialize_MoistureSurfaceBC returns it (or NULL); row iteration-1 is used
 * at each iteration (Main.py:186-188, 253-267).  get_moisture copies the
 * current Q out. */
int alfa_init_moisture(alfa_ctx*, const double* Q);
int alfa_set_moisture_series(alfa_ctx*, const double* Qadv, const double* msfc, int nrows);
int alfa_get_moisture(alfa_ctx*, double* Q);
int alfa_step(alfa_ctx*, int nsteps);
int alfa_get_state(alfa_ctx*, double* u, double* v, double* w, double* TH, double* p);
int alfa_get_diag(alfa_ctx*, alfa_diag* out /* host; synchronises the stream */);

/* ---- statistics: src/utilities/Statistics.py:47-328 (ComputeStats) -------
 * Adds one sample to acc (device, ALFA_STATS_LEN(nz) doubles): 31 profiles
 * of nz, in the reference's key order U V W TH dUdz dVdz dTHdz u2 v2 w2 TH2
 * uv uw vw uTH vTH wTH txy txz tyz qz Cs2_1 Cs2_2 Cs2PrRatio Beta1 Beta2 Q
 * dQdz Q2 wQ qHz, then the scalars M_sfc ustar qz_sfc qm_sfc.  Dimensional
 * (u_scale = TH_scale = Q_scale = 1, z from z_scale), Ugal added to U and u,
 * T_0 to TH.  Arguments in the reference's order; a dry sample passes NULL
 * for Q, dQdz, qm_sfc_avg and qHz_q and accumulates zeros in the moisture
 * entries.  Zeroing acc is the reference's ResetFlag = 1; the averages are
 * acc / samples.  M_sfc_loc, ustar: (nx, ny); qz_sfc_avg, qm_sfc_avg: one
 * device double each; profiles: (nz). */
#define ALFA_STATS_NPROF 31
#define ALFA_STATS_LEN(nz) (ALFA_STATS_NPROF * (nz) + 4)
int alfa_ComputeStats(alfa_ctx*, const double* u, const double* v, const double* w,
                      const double* TH, const double* Q, const double* dudz,
                      const double* dvdz, const double* dTHdz, const double* dQdz,
                      const double* M_sfc_loc, const double* ustar,
                      const double* qz_sfc_avg, const double* qm_sfc_avg, const double* txy,
                      const double* txz, const double* tyz, const double* qz,
                      const double* qHz_q, const double* Cs2_1D_avg1,
                      const double* Cs2_1D_avg2, const double* Cs2PrRatio_1D,
                      const double* beta1_1D, const double* beta2_1D, double* acc);
/* The same sample from the context's state after alfa_step (the arguments
 * Main.py:550-558 passes: the new u, v, w, TH, this step's gradients, surface
 * fields, SGS stresses and flux, and the latest coefficient profiles). */
int alfa_stats_sample(alfa_ctx*, double* acc);

/* ---- CUDA-graph step and ensembles (no counterpart in the reference) -----
 * alfa_step_graph: as alfa_step, each step replayed from a captured CUDA
 * graph (one per iteration parity and dynamic/static SGS step, captured on
 * first use; the bootstrap step runs directly).  Needs a non-default stream
 * (alfa_set_stream).  Results equal alfa_step's bit for bit.
 * Ensemble: independent contexts of any grid sizes advanced together; each
 * step of all members is one CUDA graph launch in which every member runs on
 * its own stream.  Members must have state; create gives each member its own
 * stream (restored to the default at destroy).  Members at different
 * iterations or with different dynamic intervals step one by one instead.
 * alfa_ensemble_sync waits for the work issued so far. */
int alfa_step_graph(alfa_ctx*, int nsteps);
typedef struct alfa_ensemble alfa_ensemble;
int alfa_ensemble_create(alfa_ctx* const* members, int n, alfa_ensemble** out);
int alfa_ensemble_step(alfa_ensemble*, int nsteps);
int alfa_ensemble_sync(alfa_ensemble*);
/* Orders later alfa_ensemble_step calls on `stream` (a created
 * cudaStream_t; NULL, which is also the legacy default stream's handle,
 * stops): each call's steps start after the work already queued on it, and
 * work queued on it afterwards starts after the steps, so events recorded on
 * it time them. */
int alfa_ensemble_set_stream(alfa_ensemble*, void* stream);
const char* alfa_ensemble_error(const alfa_ensemble*);
void alfa_ensemble_destroy(alfa_ensemble*);

/* ---- learned SGS coefficient (no counterpart in the reference) ----------
 * A 10 -> 64 -> 64 -> 2 network (tanh) attached to a context predicts Cs^2
 * (and beta) from local strain-rate and scalar-gradient features: log of
 * Delta^2 |S|, the six S_ij / |S|, dtheta/dz, z / Delta and the gradient
 * Richardson number Ri as Ri / (1 + |Ri|).  Hand-written kernels train it (FP32 master weights,
 * Adam) on samples of the dynamic procedure's Cs^2 and beta, and infer it
 * with BF16 weights and FP32 accumulation: alfa_mlp_infer on the CUDA cores
 * with FP32 activations, the learned step with the 64 x 64 hidden layer on
 * the tensor cores (BF16 activations of the first layer).
 * collect: npoints random samples of the context's last step, which must
 *   have run the dynamic procedure, into a ring of `capacity` samples.
 * train: epochs over the collected samples (shuffled), batch, learning rate;
 *   loss_out = last epoch's mean squared error in normalised units.
 * loss_grad: gradient of that loss for n given samples (device X: n x 10,
 *   T: n x 2, norm: 24 floats = means of the 10 features and 2 targets, then
 *   their standard deviations) with the FP32 weights, into grad
 *   (ALFA_MLP_NPARAM floats) and loss (one float).
 * params: W1 (64 x 10), b1, W2 (64 x 64), b2, W3 (2 x 64), b3, FP32.
 * step_learned: steps whose Cs^2 comes from the network (static stresses and
 *   fluxes with it); the first step of a run with no judge step yet, and
 *   then every judge_every-th step, runs the dynamic procedure instead (the
 *   judge) and compares the network's plane-averaged Cs^2 on that state with
 *   the procedure's: last_drift is the relative L2 difference of the two
 *   profiles of that step, window_drift the same for the two profiles
 *   averaged over the last ALFA_MLP_JUDGE_WINDOW judge steps (the
 *   procedure's single-step plane means jump between steps where its
 *   clipping switches on or off, so one step's profile is not a stable
 *   reference).  Once the window is full, a window_drift above tol reverts
 *   to the dynamic procedure for good.  Otherwise each judge step
 *   recalibrates the network per level: its Cs^2 at level z is scaled by
 *   the running ratio of the procedure's plane mean to the network's
 *   (held within [0.1, 10]), so the network supplies the horizontal pattern
 *   and the last judge the level means; then refresh_points samples of the
 *   judge step are collected and the network trains refresh_epochs more
 *   epochs (0, 0: no refresh).  alfa_mlp_infer applies the same scaling. */
#define ALFA_MLP_NPARAM 4994
#define ALFA_MLP_JUDGE_WINDOW 8
typedef struct alfa_mlp alfa_mlp;
typedef struct {
  int steps, learned_steps, judged, reverted, reverted_at;
  double last_drift, max_drift, window_drift, max_window_drift;
} alfa_mlp_report;
int alfa_mlp_create(alfa_ctx*, int capacity, unsigned long long seed, alfa_mlp** out);
void alfa_mlp_destroy(alfa_mlp*);
int alfa_mlp_collect(alfa_mlp*, int npoints);
int alfa_mlp_train(alfa_mlp*, int epochs, int batch, double lr, double* loss_out /* host */);
int alfa_mlp_loss_grad(alfa_mlp*, const float* X, const float* T, const float* norm, int n,
                       float* grad, float* loss);
int alfa_mlp_get_params(alfa_mlp*, float* params, float* norm);
int alfa_mlp_set_params(alfa_mlp*, const float* params, const float* norm);
int alfa_mlp_features(alfa_mlp*, float* X /* N x 10, from the context's last step */);
int alfa_mlp_infer(alfa_mlp*, double* Cs2, double* beta /* may be NULL */);
int alfa_step_learned(alfa_mlp*, int nsteps, int judge_every, double tol, int refresh_points,
                      int refresh_epochs, alfa_mlp_report* report /* host, accumulated */);

/* ---- checkpoint / restart (no counterpart in the reference) --------------
 * Everything alfa_step carries from one iteration to the next: u v w TH p,
 * the previous right-hand sides, the 3-D SGS coefficients, the MOST planes,
 * the coefficient profiles, the iteration counter and CFLmax.  dst / src are
 * device buffers of alfa_checkpoint_doubles(ctx) doubles; a context of the
 * same configuration that loads a checkpoint continues bit for bit as the
 * one that saved it (series set with alfa_set_series are not included). */
size_t alfa_checkpoint_doubles(const alfa_ctx*);
int alfa_save_checkpoint(alfa_ctx*, double* dst);
int alfa_load_checkpoint(alfa_ctx*, const double* src);

/* No counterpart in the reference.  alfa_PlanarMean without a context and
 * without any device allocation, for callers that may not allocate: code
 * running inside another runtime's memory management, such as a JAX/XLA
 * custom call (XLA reserves most of the GPU for its own allocator and gives
 * the call only its buffers) or an application with a fixed device-memory
 * budget.  F is (nx, ny, nz) z-fastest, mean_nz receives the nz plane means;
 * both are the caller's device buffers; the work runs on cuda_stream.
 * Limit: nz <= 2048 (larger returns ALFA_E_NOALLOC_LIMIT before any launch).
 * The partial sums live in a fixed 4 MiB array inside the library, one per
 * device that loads it, kept until the process exits.  The first call on each
 * device looks that array's address up (with the device current), and so
 * does the first call after the device's context was replaced (for example
 * by cudaDeviceReset); make such calls before any stream capture.  All calls
 * on a device share the
 * array: calls that overlap on the GPU (different streams, no ordering)
 * race and must be serialised by the caller. */
int alfa_PlanarMean_noalloc(const double* F, int nx, int ny, int nz, double* mean_nz,
                            void* cuda_stream);

/* Diagnostics with no reference counterpart: the number of kernels this
 * library has launched in this process (all contexts, all streams). */
unsigned long long alfa_launch_count(void);
/* Times `reps` back-to-back launches of one building-block kernel on the
 * context's stream with CUDA events (inputs: the context's state/workspace):
 *   0 y pad pass   (nx,ny,nz) -> (nx,my,nz)        (reads N, writes nx*my*nz)
 *   1 x pad pass   (nx,my,nz) -> (mx,my,nz)        (reads nx*my*nz, writes P)
 *   2 x unpad pass (mx,my,nz) -> (nx,my,nz)        (reads P, writes nx*my*nz)
 *   3 y unpad pass (nx,my,nz) -> (nx,ny,nz)        (reads nx*my*nz, writes N)
 *   4 x derivative line pass                       (reads N, writes N)
 *   5 y-forward real -> half spectrum (2-D path)   (reads N, writes S)
 *   6 x-column: forward FFT + two i*k outputs      (reads S, writes 2 S)
 *   7 y-inverse half spectrum -> real (2-D path)   (reads S, writes N)
 *   8 x derivative of an FP32 field on the tensor cores (alfa_tc_line_apply's
 *     kernel; reads and writes N floats; 3 x 2 nx^2 ny nz issued BF16 flops)
 * (N, P, S: real, padded real and half-spectrum complex field sizes.)
 * ms = average duration of one launch; bytes = its algorithmic HBM bytes. */
int alfa_time_kernel(alfa_ctx*, int which, int reps, double* ms /* host */,
                     double* bytes /* host */);

/* One candidate of the autotuner: a line-pass shape (axis 0 = x, 1 = y;
 * n_in -> n_out points along it; `outputs` outputs, the first with map
 * `map`: 1 truncate, 2 derivative, 3 truncate+derivative, 4 pad, 5 unpad)
 * run with `variant` (0 the default dispatch, 1 the compile-time transform
 * in place of a phase-split pad/unpad, 2/3/4 the runtime-plan transform
 * with radix schedule "largest radix 8" / "largest radix 4" / "default
 * factors in ascending order", 5 the split-BF16 tensor-core pass of an
 * ALFA_MIXED context, 6 the FP32 transform on two-lane elements: two packed
 * columns per thread in paired FP32 instructions, for plain-field inputs
 * with nz a multiple of 4), its average launch time, whether its outputs equal
 * the default's to the precision's round-off of their maximum (1e-12 FP64,
 * 1e-5 FP32, 5e-5 for the tensor-core pass), and whether it was chosen. */
typedef struct alfa_tune_entry {
  int axis, n_in, n_out, outputs, map, variant, chosen, equal;
  double ms;
} alfa_tune_entry;

/* Times every variant of the eight line-pass shapes of a step (y pad, x pad,
 * x unpad, y unpad, x/y derivative, x/y filter + derivative) on a synthetic
 * field, `reps` launches each with CUDA events, and makes the fastest
 * variant whose outputs equal the default's the one later steps use.  Call
 * between steps; model state is not touched (only step scratch), captured
 * step graphs are released.  Writes up to max_out entries to `out` and the
 * number of candidates to *n_out.  Replaces nothing in the reference (JAX
 * picks its FFT plans inside XLA); the choice is the engine's own. */
int alfa_autotune(alfa_ctx*, int reps, alfa_tune_entry* out /* host */, int max_out,
                  int* n_out /* host */);

/* No counterpart in the reference.  Makes `variant` (numbered as in
 * alfa_tune_entry) the one the step uses for the line passes of one of the
 * eight autotuned shapes, without timing: (axis, n_in, n_out, map, outputs)
 * as in alfa_tune_entry.  Variant 5 (tensor cores) needs an ALFA_MIXED
 * context and a shape the GEMM tiles (n_out a multiple of 128, n_in of 32,
 * the pass's columns of 256) and builds the pass's operator here.  Returns
 * ALFA_E_SHAPE when no autotuned shape matches or the variant does not apply
 * to it.  Captured step graphs are released. */
int alfa_set_line_variant(alfa_ctx*, int axis, int n_in, int n_out, int map, int outputs,
                          int variant);

/* ---- split-BF16 tensor-core line pass (FP32; no counterpart in the
 * reference, whose FFT passes run in the run's precision) -----------------
 * Y (n_out, ncols) = scale * M X for X (n_in, ncols) FP32 row-major (the x
 * lines of an (nx, ny, nz) FP32 field: n_in = nx, ncols = ny * nz), M the
 * real operator of line map `map` (1 truncate at `cut`, 2 derivative with the
 * Nyquist mode zeroed, 3 both, 4 the 3/2 pad n -> 3n/2, 5 the unpad 3n/2 ->
 * n; 0 identity) exactly as the FP64 line passes apply it.  Runs as a GEMM
 * on tcgen05 with BF16 hi/lo operand pairs (three products, FP32
 * accumulation in tensor memory): about 1e-5 relative accuracy.  n_out a
 * multiple of 128, ncols of 256, n_in of 32.  Synchronises the stream. */
int alfa_tc_line_apply(alfa_ctx*, int map, int cut, int n_in, int n_out, double scale,
                       long long ncols, const float* X, float* Y);

/* No counterpart in the reference.  The number of mbarrier polls after which
 * a wait of the tensor-core line pass (alfa_tc_line_apply, the split-BF16
 * passes of ALFA_MIXED) gives up; the call then returns ALFA_E_TIMEOUT after
 * waiting (at the full limit) for the products already issued, so the
 * context stays usable.  0 restores the default (2^22 polls). */
int alfa_set_tc_spin_limit(alfa_ctx* ctx, unsigned long long polls);

#ifdef __cplusplus
}
#endif
#endif /* ALFA_H */
