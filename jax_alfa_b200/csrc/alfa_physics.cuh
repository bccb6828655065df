// Physical-space kernels of the LES step (declarations; alfa_physics.cu).
// Fields (nx, ny, nz) are `real`; surface planes (nx, ny), vertical
// profiles, forcing series and the pressure system are double in every
// build, and so is the arithmetic of every kernel here (a field value is
// rounded to `real` only where it is stored).
#pragma once
#include "alfa_internal.cuh"

namespace alfa {
namespace ALFA_PREC {

// ---- reductions over (x, y) planes: deterministic two-level sums -------
// sums[q][z] = sum over the plane of field q (nq fields)
void plane_sums(Engine& e, const real* const* fields, int nq, double* sums);
void plane_means(Engine& e, const real* const* fields, int nq, double* means);

// ---- surface (SurfaceFlux.py) --------------------------------------------
struct SurfaceIO {
  const real* u;
  const real* v;
  const real* TH;
  const double* most_in[6];
  double* M;
  double* ustar;
  double* q2;        // qz_sfc_2D (may be null for constant-flux variants)
  double* qavg;      // device scalar
  double* invOB;
  double* most_out[6];
};
// variant: 0 HomConst, 1 HetConst, 2 HomVary, 3 HetVary, 4 HomPresT, 5 HetPresT
// sfc_series / itp: when given, the surface value is sfc_series[*itp - 1]
// (read on the device, so a captured step replays with the current row)
int surface_flux(Engine& e, int variant, double sfc_val, const SurfaceIO& io,
                 const double* sfc_series = nullptr, const int* itp = nullptr);

// ---- z derivatives (Derivatives.py) --------------------------------------
void derivz_M(Engine& e, const real* u, const real* v, const real* w, const double* ustar,
              const double* M, const double* fi_m, real* dudz, real* dvdz, real* dwdz);
void derivz_TH(Engine& e, const real* TH, const double* ustar, const double* qz,
               const double* fi_h, real* dTHdz);
void derivz_generic(Engine& e, const real* F, int w_nodes, real* out);

// ---- buoyancy ------------------------------------------------------------
// H: the specific humidity (THv = (TH + T_0)(1 + 0.61 H)), or null (dry)
void buoyancy(Engine& e, const real* TH, const real* H, int opt, real* out);

// ---- surface moisture flux (Main.py:253-267, SurfaceFlux.py:447-504) -----
// mode 1: the flux series value; mode 2: from the prescribed surface
// humidity (het: per column, else against the plane mean qbar0 of Q's first
// level).  The series value is series[*itp - 1] when series is given, else
// q_host.
void moisture_surface(Engine& e, int mode, int het, const real* Q, const double* ustar,
                      const double* psi_h, const double* psi_h0, const double* series,
                      const int* itp, double q_host, const double* qbar0, double* qm);

// ---- strains -------------------------------------------------------------
// uvp nodes: S12, S13, S23, |S| (S11, S22, S33 are dudx, dvdy, dwdz)
void strains_uvp(Engine& e, const real* const g[9], real* S12, real* S13, real* S23, real* S);
// |S| at w nodes from the gradients (non-padded)
void smag_w(Engine& e, const real* const g[9], real* Sw);
// |S| of six padded components
void smag6(Engine& e, const real* const s[6], size_t n, real* out);

// ---- LASDD ---------------------------------------------------------------
void wstar(Engine& e, const real* w, real* w_);
void smag6_n(Engine& e, const real* const s[6], real* out);
// Germano terms: 10 plane sums (a1, a2, b1, b2, c1, c2, d1, d2, e1, e2)
struct LasddFields {
  const real* hat[3];    // u_hat v_hat w_hat
  const real* hatd[3];
  const real* ph[6];     // uu_hat .. vw_hat
  const real* pd[6];
  const real* Sh[6];
  const real* Sd[6];
  const real* SSh[6];
  const real* SSd[6];
  const real* S_hat;
  const real* S_hatd;
};
void lasdd_sums(Engine& e, const LasddFields& f, double* sums10);
void lasdd_poly(Engine& e, const double* sums10, int scalar, double* coeffs6);
void compute_beta(Engine& e, const double* coeffs6, int nlev, double* beta);
void lasdd_LM_MM(Engine& e, const LasddFields& f, const double* beta, real* LM, real* MM);
void clip_ratio(Engine& e, const real* num, const real* den, real* out);
void cs2_profiles(Engine& e, const real* Cs2, double* avg1, double* avg2);

struct ScalarLasddFields {
  const real* hat[3];
  const real* hatd[3];
  const real* Th, *Td;
  const real* uTh[3], *uTd[3];
  const real* Gh[3], *Gd[3];
  const real* SGh[3], *SGd[3];
  const real* S_hat, *S_hatd;
};
void scalar_lasdd_sums(Engine& e, const ScalarLasddFields& f, double* sums10);
void scalar_Tup_Tdn(Engine& e, const ScalarLasddFields& f, const double* beta, real* Tup,
                    real* Tdn);

// plane-averaged statistics (Statistics.py:47-328): one sample added to acc
struct StatsIn {
  const real *u, *v, *w, *TH, *dudz, *dvdz, *dTHdz, *txy, *txz, *tyz, *qz;
  const double *M, *ustar, *qz_sfc_avg;  // planes (nx, ny) and one scalar
  const double *cs2_1, *cs2_2, *cs2pr, *beta1, *beta2;  // profiles (nz)
  double Ugal, T0;
  // moisture (null: a dry sample, zeros accumulated): Q, dQdz, qHz_q fields;
  // the surface flux as a device scalar (qm_sfc_avg) or as the plane whose
  // mean it is (qm_plane, used when given)
  const real *Q = nullptr, *dQdz = nullptr, *qHz = nullptr;
  const double *qm_sfc_avg = nullptr, *qm_plane = nullptr;
};
void compute_stats(Engine& e, const StatsIn& a, double* acc);

// Wong-Lilly procedure (optSgs 2, 4)
void lasdd_wl_sums(Engine& e, const LasddFields& f, double* sums4);
void wl_poly(Engine& e, const double* sums4, double* coeffs6);
void lasdd_wl_LM_MM(Engine& e, const LasddFields& f, const double* beta, real* LM, real* MM);
void scalar_lasdd_wl_sums(Engine& e, const ScalarLasddFields& f, double* sums4);
void scalar_wl_Tup_Tdn(Engine& e, const ScalarLasddFields& f, const double* beta, real* Tup,
                       real* Tdn);

// ---- stresses / fluxes / divergence -------------------------------------
void wall_override(Engine& e, const real* u, const real* v, const double* M,
                   const double* psi_m, const double* psi_m0, real* txz, real* tyz);
void set_plane0(Engine& e, const double* plane, real* field);
void divergence_finish(Engine& e, real* div, const real* fz, int w_nodes);

// ---- RHS, pressure, time advance ---------------------------------------
void rhs_momentum(Engine& e, const real* u, const real* v, const real* w,
                  const double* Ug, const double* Vg, const real* Cx, const real* Cy,
                  const real* Cz, const real* b, const real* dx, const real* dy,
                  const real* dz, const double* Uadv, const double* Vadv, const double* ubar,
                  const double* vbar, real* Ru, real* Rv, real* Rw,
                  const int* itp = nullptr, long long rs = 0, const int* gtp = nullptr,
                  long long grs = 0);
// itp / rs: when given, the forcing profiles are row (*itp - 1) of a series
// with row stride rs (read on the device)
void rhs_scalar(Engine& e, const real* TH, const real* adv, const real* divq,
                const double* THadv, const double* THbar, real* R, const int* itp = nullptr,
                long long rs = 0, int always_adv = 0);
// always_adv: add the forcing profile whatever optAdvection is (RHS_Moisture,
// SCL_AllTerms.py:103, adds Qadv unconditionally)
void pressure_rc(Engine& e, const cd* fRx, const cd* fRy, const cd* fRz, const cd* fbot,
                 const cd* ftop, double* RCr, double* RCi, double* fRz_real);
void thomas_solve(Engine& e, const double* RCr, const double* RCi, const double* fRz_real,
                  cd* fp);
void subtract3(Engine& e, real* Ru, real* Rv, real* Rw, const real* a, const real* b,
               const real* c);
void ab2_uvw(Engine& e, const real* u, const real* v, const real* w, const real* Ru,
             const real* Rup, const real* Rv, const real* Rvp, const real* Rw,
             const real* Rwp, real* un, real* vn, real* wn);
void ab2_th(Engine& e, const real* TH, const real* R, const real* Rp, real* out);
// AB2_Q (SCL_TimeAdvancement.py:79-99): the q_inversion top condition
void ab2_q(Engine& e, const real* Q, const real* R, const real* Rp, real* out);
void cfl_max(Engine& e, const real* u, const real* v, const real* w, double* out3);
void copy_planes_z(Engine& e, const real* F, int k0, int k1, real* out2);
void imfilter(Engine& e, const real* F, real* out);
// the plane mean of one field with caller-provided partial-sum storage
// (NOALLOC_RED_BLOCKS x nz doubles)
void plane_mean_with_scratch(const real* F, size_t H, int nz, double* partials, double* mean,
                             cudaStream_t s);

}  // namespace ALFA_PREC
}  // namespace alfa
