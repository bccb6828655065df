// The whole-step driver of one precision build (alfa_step.cu): the model
// state and step workspace, the composite operators the reference's
// functions are made of, and the loop body of the reference's
// src/Main.py:156-541.
#pragma once
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "alfa_iface.cuh"
#include "alfa_internal.cuh"
#include "alfa_physics.cuh"

namespace alfa {
namespace ALFA_PREC {

// ---------------------------------------------------------------------------
// Workspace: named field slots carved from one allocation.  Fields, padded
// fields and spectra are `real`; surface planes, profiles, forcing series and
// the pressure system are double.
// ---------------------------------------------------------------------------
struct Work {
  // model state (whole-step driver)
  real *u, *v, *w, *TH, *p;
  real *RHS[4], *RHSp[4];
  real *Cs2, *Cs2Pr;
  double *most[6], *most_new[6];
  double *M, *ustar, *q2, *invOB, *qz_plane;
  cd *ufft, *vfft, *wfft;
  double* Ug;  // (nz) profiles
  double* Vg;
  double* zero_prof;
  double* series_adv = nullptr;  // (nrows, 3, nz) non-dimensional Uadv, Vadv, THadv
  int series_rows = 0;
  double* series_geo = nullptr;  // (nrows, 2, nz) non-dimensional Ug, Vg (optGeoWind >= 1)
  int geo_rows = 0;
  // moisture (optMoisture >= 1; carved only then)
  real *Q = nullptr, *RHSQ = nullptr, *RHSQp = nullptr;
  real* gQ[3] = {nullptr, nullptr, nullptr};  // dQdx dQdy dQdz
  real *Qadvs = nullptr, *divqm = nullptr, *qzq = nullptr;  // QAdvectionSum, divqm, qHz_q
  double* qm_plane = nullptr;                               // qm_sfc_step (nx, ny)
  double* series_q = nullptr;  // (nrows, nz) non-dimensional Qadv
  int q_rows = 0;
  double* d_msfc = nullptr;  // (nrows) moisture surface series
  int msfc_rows = 0;
  int have_q = 0;
  std::vector<double> sfc_series;  // host
  double* d_sfc = nullptr;         // device copy of sfc_series
  int* d_it;                       // the iteration counter, on the device
  // step temporaries
  real* g[9];
  real* gT[3];
  real *Cx, *Cy, *Cz, *THadv, *buoy;
  real *divt[3], *divq, *qz;
  real* mom[25];
  // internal SGS temporaries
  real *S12, *S13, *S23;
  real *ph[6], *pd[6], *Sh[6], *Sd[6], *SSh[6], *SSd[6];
  real *LM, *MM;
  real *Th, *Td, *uTh[3], *uTd[3], *Gh[3], *Gd[3], *SGh[3], *SGd[3];
  real *qx, *qy;
  real* Pb[10];  // padded fields
  real* Lpad;    // (nx, my, nz): between the two passes of a pad / unpad
  real* L2;      // two N fields: between the passes of filter + derivatives
  // pressure
  double *RCr, *RCi, *fRzr;
  cd *fRx, *fRy, *fRz, *fp, *fb2;
  real* planes2;
  real* dp[3];
  double* prof;  // small profiles scratch
  int iteration = 1;
  int have_state = 0;
  int last_dyn = 0;  // the last step ran the dynamic procedure
  double CFL = 0, CFLmax = 0;
  double* d_cfl;  // 3 maxima
  double* d_qavg;
};

// The swappable buffer pointers of Work: a step exchanges the filtered state
// with its scratch, the MOST planes with their successors and the right-hand
// sides with the previous ones, so the pointer set alternates with the
// iteration's parity.  A captured step graph is valid for one pointer set.
struct StepPtrs {
  real *u, *v, *w, *TH, *Cx, *Cy, *Cz, *THadv;
  double *most[6], *most_new[6];
  real *RHS[4], *RHSp[4];
  real *Q, *Qadvs, *RHSQ, *RHSQp;  // moisture (null when dry)
  static StepPtrs of(const Work& W) {
    StepPtrs p;
    p.u = W.u; p.v = W.v; p.w = W.w; p.TH = W.TH;
    p.Cx = W.Cx; p.Cy = W.Cy; p.Cz = W.Cz; p.THadv = W.THadv;
    for (int i = 0; i < 6; i++) { p.most[i] = W.most[i]; p.most_new[i] = W.most_new[i]; }
    for (int i = 0; i < 4; i++) { p.RHS[i] = W.RHS[i]; p.RHSp[i] = W.RHSp[i]; }
    p.Q = W.Q; p.Qadvs = W.Qadvs; p.RHSQ = W.RHSQ; p.RHSQp = W.RHSQp;
    return p;
  }
  void apply(Work& W) const {
    W.u = u; W.v = v; W.w = w; W.TH = TH;
    W.Cx = Cx; W.Cy = Cy; W.Cz = Cz; W.THadv = THadv;
    for (int i = 0; i < 6; i++) { W.most[i] = most[i]; W.most_new[i] = most_new[i]; }
    for (int i = 0; i < 4; i++) { W.RHS[i] = RHS[i]; W.RHSp[i] = RHSp[i]; }
    W.Q = Q; W.Qadvs = Qadvs; W.RHSQ = RHSQ; W.RHSQp = RHSQp;
  }
  bool operator==(const StepPtrs& o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

struct StepGraph {
  cudaGraphExec_t exec = nullptr;
  StepPtrs before, after;
  unsigned long long kernels = 0;  // kernel launches the graph replays
};

// One simulation: engine, workspace and captured step graphs.
struct Ctx {
  Engine e;
  Work w;
  void* base = nullptr;
  size_t bytes = 0;
  StepGraph graphs[4];  // captured steps by (iteration parity, dynamic SGS step)
  StepPtrs canon{};     // the buffer arrangement as carved; init_state returns to it
  // the learned coefficient (FP64 build): writes the network's Cs^2 field
  std::function<void(real*)> learned;
};

// ---- set-up ---------------------------------------------------------------
void release_graphs(Ctx* c);

// ---- composite operators shared by the per-function C-ABI and the step ----
Loader ld(const Engine& e, int kind, std::initializer_list<const real*> a, double c0 = 0.0,
          double c1 = 0.0, int sub = 0);
void deriv_field_acc(Engine& e, const Loader& L, real* dx, int accx, real* dy, int accy);
void div_stress(Ctx* c, const real* txx, const real* tyy, const real* tzz, const real* txy,
                const real* txz, const real* tyz, real* dtx, real* dty, real* dtz);
void div_flux(Ctx* c, const real* qx, const real* qy, const real* qz, real* divq);
void advection(Ctx* c, const real* u, const real* v, const real* w, const real* uy,
               const real* uz, const real* vx, const real* vz, const real* wx, const real* wy,
               real* Cx, real* Cy, real* Cz);
void scalar_advection(Ctx* c, const real* u, const real* v, const real* w, const real* sx,
                      const real* sy, const real* sz, real* out, bool reuse_uvw);
int dynamic_sgs(Ctx* c, const real* const g[9], const real* u, const real* v, const real* w,
                const double* M, const double* pm, const double* pm0, real* divt[3],
                double* avg1, double* avg2, double* beta1, real* Cs2, real* const mom[25]);
int static_sgs(Ctx* c, const real* const g[9], const real* Cs2, const real* u, const real* v,
               const double* M, const double* pm, const double* pm0, real* divt[3],
               real* const mom10[10]);
void scalar_fluxes(Ctx* c, const real* S_uvp_pad, const real* S_w_pad, const real* r3,
                   const real* gx, const real* gy, const real* gz, const double* qz_sfc,
                   real* qz, real* divq);
int dynamic_sgs_scalar(Ctx* c, const real* const m15[15], const real* TH, const real* gx,
                       const real* gy, const real* gz, const double* qz_sfc, real* qz,
                       real* divq, real* r3, double* r1, double* beta2);
int pressure_rc_fn(Ctx* c, const real* u, const real* v, const real* w, const real* Ru,
                   const real* Rv, const real* Rw, const real* Rup, const real* Rvp,
                   const real* Rwp, const real* divtz, double* RCr, double* RCi, double* fRzr);
int pressure_solve_fn(Ctx* c, const double* RCr, const double* RCi, const double* fRzr, real* p,
                      real* dpdx, real* dpdy, real* dpdz);

}  // namespace ALFA_PREC
}  // namespace alfa
