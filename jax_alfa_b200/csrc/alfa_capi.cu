// The reference-named C-ABI entry points.  A context holds an engine of one
// storage precision (alfa_config.precision): the FP64 build serves every
// entry point; the FP32 build (FP32 and mixed precision) serves the
// whole-step entry points (create, state import/export, stepping,
// diagnostics, statistics, checkpoints, probes, autotuner, ensembles), with
// the state crossing as FP64 device buffers.  The per-function entry points
// take FP64 arrays and need an FP64 context.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <deque>
#include <vector>

#include "alfa_iface.cuh"
#include "alfa_mlp.cuh"
#include "alfa_step.cuh"

using namespace alfa;
using namespace alfa::f64;

namespace alfa {

static std::atomic<unsigned long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
unsigned long long launch_count() { return g_launches.load(); }
void add_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

void raise_smem_limit(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> g(mu);
  size_t& have = done[{dev, kernel}];
  if (have >= bytes) return;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) ==
      cudaSuccess)
    have = bytes;
}

}  // namespace alfa

struct alfa_ctx {
  int precision = ALFA_FP64;
  f64::Ctx* d = nullptr;       // FP64 engine (precision ALFA_FP64)
  alfa::f32::Ctx* f = nullptr;  // FP32 engine (precision ALFA_FP32 or ALFA_MIXED)
  struct alfa_mlp* mlp = nullptr;  // attached learned-coefficient network (FP64 only)
};

struct alfa_mlp {
  alfa_ctx* c = nullptr;
  int cap = 0, count = 0, offset = 0, adam_t = 0;
  unsigned long long seed = 0, draws = 0;
  float *X = nullptr, *T = nullptr, *norm = nullptr, *P = nullptr, *G = nullptr, *M = nullptr,
        *V = nullptr, *loss = nullptr;
  int* perm = nullptr;
  __nv_bfloat16* Pb = nullptr;
  double* scratch = nullptr;  // N: the network's Cs^2 on a judge step
  double* means = nullptr;    // 2 nz plane means
  int trained = 0;
  // the judge's window: the network's and the procedure's plane-mean Cs^2
  // profiles of the last ALFA_MLP_JUDGE_WINDOW judge steps (2 nz each)
  std::deque<std::vector<double>> window;
  // per-level calibration of the network's Cs^2 (nz): the ratio of the
  // procedure's plane mean to the network's at the last judge step
  double* calib = nullptr;
  std::vector<double> calib_h;
};

#define CTX_CHECK(c)                                  \
  do {                                                \
    if (!(c)) return ALFA_E_STATE;                    \
  } while (0)

// the per-function entry points compute on FP64 arrays: FP64 contexts only
#define F64_CHECK(c)                                                                          \
  do {                                                                                        \
    if (!(c)) return ALFA_E_STATE;                                                            \
    if (!(c)->d)                                                                              \
      return alfa::f32::ctx_fail((c)->f,                                                      \
                                 "this entry point takes FP64 arrays: create the context "    \
                                 "with precision ALFA_FP64",                                  \
                                 ALFA_E_CONFIG);                                              \
  } while (0)

// call the whole-step interface function fn of the context's engine
#define DISPATCH(c, fn, ...) ((c)->d ? f64::fn((c)->d, ##__VA_ARGS__) : alfa::f32::fn((c)->f, ##__VA_ARGS__))

static thread_local std::string g_create_error;

static void learned_cs2(alfa_ctx* c, double* Cs2_out);

extern "C" {

int alfa_create(const alfa_config* cfg, alfa_ctx** out) {
  if (!cfg || !out) return ALFA_E_SHAPE;
  *out = nullptr;
  if (cfg->precision != ALFA_FP64 && cfg->precision != ALFA_FP32 && cfg->precision != ALFA_MIXED) {
    g_create_error = "precision must be ALFA_FP64 (0), ALFA_FP32 (1) or ALFA_MIXED (2)";
    return ALFA_E_CONFIG;
  }
  alfa_ctx* c = new alfa_ctx();
  c->precision = cfg->precision;
  const int st = cfg->precision == ALFA_FP64 ? f64::ctx_create(*cfg, &c->d, &g_create_error)
                                             : alfa::f32::ctx_create(*cfg, &c->f, &g_create_error);
  if (st) {
    delete c;
    return st;
  }
  *out = c;
  return ALFA_OK;
}

void alfa_destroy(alfa_ctx* c) {
  if (!c) return;
  if (c->mlp) c->mlp->c = nullptr;  // the network outlives its context only as memory
  if (c->d) f64::ctx_destroy(c->d);
  if (c->f) alfa::f32::ctx_destroy(c->f);
  delete c;
}

// with a null context: the reason of the last failed alfa_create on this thread
const char* alfa_last_error(const alfa_ctx* c) {
  return c ? DISPATCH(c, ctx_error) : g_create_error.c_str();
}

int alfa_set_stream(alfa_ctx* c, void* s) {
  CTX_CHECK(c);
  DISPATCH(c, ctx_set_stream, (cudaStream_t)s);
  return ALFA_OK;
}

size_t alfa_workspace_bytes(const alfa_ctx* c) { return c ? DISPATCH(c, ctx_bytes) : 0; }

int alfa_get_precision(const alfa_ctx* c) { return c ? c->precision : ALFA_E_STATE; }

int alfa_get_derived(const alfa_ctx* c, alfa_derived* o) {
  CTX_CHECK(c);
  if (!o) return ALFA_E_SHAPE;
  DISPATCH(c, ctx_derived, o);
  return ALFA_OK;
}

int alfa_init_state(alfa_ctx* c, const double* u, const double* v, const double* w,
                    const double* TH) {
  CTX_CHECK(c);
  return DISPATCH(c, init_state, u, v, w, TH);
}

int alfa_set_series(alfa_ctx* c, const double* Uadv, const double* Vadv, const double* THadv,
                    const double* sfc, int nrows) {
  CTX_CHECK(c);
  return DISPATCH(c, set_series, Uadv, Vadv, THadv, sfc, nrows);
}

int alfa_set_geowind_series(alfa_ctx* c, const double* Ug, const double* Vg, int nrows) {
  CTX_CHECK(c);
  return DISPATCH(c, set_geowind_series, Ug, Vg, nrows);
}

int alfa_step(alfa_ctx* c, int nsteps) {
  CTX_CHECK(c);
  return DISPATCH(c, step, nsteps, 0);
}

int alfa_step_graph(alfa_ctx* c, int nsteps) {
  CTX_CHECK(c);
  return DISPATCH(c, step_graph, nsteps);
}

int alfa_init_moisture(alfa_ctx* c, const double* Q) {
  CTX_CHECK(c);
  return DISPATCH(c, init_moisture, Q);
}

int alfa_set_moisture_series(alfa_ctx* c, const double* Qadv, const double* msfc, int nrows) {
  CTX_CHECK(c);
  return DISPATCH(c, set_moisture_series, Qadv, msfc, nrows);
}

int alfa_get_moisture(alfa_ctx* c, double* Q) {
  CTX_CHECK(c);
  return DISPATCH(c, get_moisture, Q);
}

int alfa_get_state(alfa_ctx* c, double* u, double* v, double* w, double* TH, double* p) {
  CTX_CHECK(c);
  return DISPATCH(c, get_state, u, v, w, TH, p);
}

int alfa_get_diag(alfa_ctx* c, alfa_diag* o) {
  CTX_CHECK(c);
  if (!o) return ALFA_E_SHAPE;
  return DISPATCH(c, get_diag, o);
}

int alfa_stats_sample(alfa_ctx* c, double* acc) {
  CTX_CHECK(c);
  return DISPATCH(c, stats_sample, acc);
}

size_t alfa_checkpoint_doubles(const alfa_ctx* c) {
  return c ? DISPATCH(c, checkpoint_doubles) : 0;
}

int alfa_save_checkpoint(alfa_ctx* c, double* dst) {
  CTX_CHECK(c);
  return DISPATCH(c, save_checkpoint, dst);
}

int alfa_load_checkpoint(alfa_ctx* c, const double* src) {
  CTX_CHECK(c);
  return DISPATCH(c, load_checkpoint, src);
}

int alfa_time_kernel(alfa_ctx* c, int which, int reps, double* ms, double* bytes) {
  CTX_CHECK(c);
  return DISPATCH(c, time_kernel, which, reps, ms, bytes);
}

int alfa_autotune(alfa_ctx* c, int reps, alfa_tune_entry* out, int max_out, int* n_out) {
  CTX_CHECK(c);
  return DISPATCH(c, autotune, reps, out, max_out, n_out);
}

int alfa_set_line_variant(alfa_ctx* c, int axis, int n_in, int n_out, int map, int outputs,
                          int variant) {
  CTX_CHECK(c);
  return DISPATCH(c, set_line_variant, axis, n_in, n_out, map, outputs, variant);
}

int alfa_tc_line_apply(alfa_ctx* c, int map, int cut, int n_in, int n_out, double scale,
                       long long ncols, const float* X, float* Y) {
  CTX_CHECK(c);
  return DISPATCH(c, tc_line_apply, map, cut, n_in, n_out, scale, ncols, X, Y);
}

int alfa_set_tc_spin_limit(alfa_ctx* c, unsigned long long polls) {
  CTX_CHECK(c);
  DISPATCH(c, ctx_set_tc_spin, polls);
  return ALFA_OK;
}

unsigned long long alfa_launch_count(void) { return g_launches.load(); }

}  // extern "C"

extern "C" {

#define NN(p) \
  if (!(p)) return c->d->e.fail("null pointer argument: " #p, ALFA_E_SHAPE)

int alfa_FFT(alfa_ctx* c, const double* F, double* F_fft) {
  F64_CHECK(c);
  NN(F);
  NN(F_fft);
  op_rfft2(c->d->e, ld_field(c->d->e, F), (cd*)F_fft);
  return check_launch(c->d->e, "FFT");
}

int alfa_FFT_pad(alfa_ctx* c, const double* F_pad, double* F_pad_fft) {
  F64_CHECK(c);
  NN(F_pad);
  NN(F_pad_fft);
  op_rfft2_pad(c->d->e, ld_field(c->d->e, F_pad), (cd*)F_pad_fft);
  return check_launch(c->d->e, "FFT_pad");
}

int alfa_Dealias1(alfa_ctx* c, const double* F_fft, double* F_pad) {
  F64_CHECK(c);
  NN(F_fft);
  NN(F_pad);
  op_pad_spec(c->d->e, (const cd*)F_fft, F_pad);
  return check_launch(c->d->e, "Dealias1");
}

int alfa_Dealias2(alfa_ctx* c, const double* F_pad_fft, double* F) {
  F64_CHECK(c);
  NN(F_pad_fft);
  NN(F);
  op_unpad_spec(c->d->e, (const cd*)F_pad_fft, F);
  return check_launch(c->d->e, "Dealias2");
}

int alfa_Filtering_Explicit(alfa_ctx* c, const double* F_fft, double* F_new, double* F_fft_new) {
  F64_CHECK(c);
  NN(F_fft);
  NN(F_new);
  NN(F_fft_new);
  Engine& e = c->d->e;
  const int cx = e.cut_e[0], cy = e.cut_e[1];
  XOut o[2];
  o[0] = XOut{};
  o[0].kind = XO_SPEC;
  o[0].map = MAP_TRUNC;
  o[0].cx = cx;
  o[0].cy = cy;
  o[0].K = e.nyh;
  o[0].rows = e.nx;
  o[0].dst = (cd*)F_fft_new;
  o[1] = XOut{};
  o[1].kind = XO_INV;
  o[1].map = MAP_TRUNC;
  o[1].cx = cx;
  o[1].cy = cy;
  o[1].K = cy;
  o[1].rows = e.nx;
  o[1].dst = e.T[1];
  o[1].inv = e.pnx;
  launch_x(e, (const cd*)F_fft, 1, e.nx, e.nyh, e.pnx, 2, o, e.nyh);
  launch_y_inv(e, e.T[1], e.nx, cy, e.pny, 1.0 / ((double)e.nx * e.ny), F_new, 0);
  return check_launch(e, "Filtering_Explicit");
}

int alfa_Filtering_Level1(alfa_ctx* c, const double* F_fft, double* F_hat) {
  F64_CHECK(c);
  NN(F_fft);
  NN(F_hat);
  op_filter1_spec(c->d->e, (const cd*)F_fft, 1, F_hat);
  return check_launch(c->d->e, "Filtering_Level1");
}

int alfa_Filtering_Level2(alfa_ctx* c, const double* F_fft, double* F_hatd) {
  F64_CHECK(c);
  NN(F_fft);
  NN(F_hatd);
  op_filter1_spec(c->d->e, (const cd*)F_fft, 2, F_hatd);
  return check_launch(c->d->e, "Filtering_Level2");
}

int alfa_Derivxy(alfa_ctx* c, const double* F_fft, int axis, double* d) {
  F64_CHECK(c);
  NN(F_fft);
  NN(d);
  if (axis != 0 && axis != 1) return c->d->e.fail("axis must be 0 (x) or 1 (y)", ALFA_E_SHAPE);
  op_deriv_spec(c->d->e, (const cd*)F_fft, axis == 0 ? d : nullptr, axis == 1 ? d : nullptr);
  return check_launch(c->d->e, "Derivxy");
}

int alfa_velocityGradients(alfa_ctx* c, const double* u, const double* v, const double* w,
                           const double* u_fft, const double* v_fft, const double* w_fft,
                           const double* ustar, const double* M, const double* fi_m,
                           double* const out[9]) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(u_fft); NN(v_fft); NN(w_fft); NN(ustar); NN(M); NN(fi_m); NN(out);
  for (int i = 0; i < 9; i++) NN(out[i]);
  Engine& e = c->d->e;
  op_deriv_spec(e, (const cd*)u_fft, out[0], out[3]);
  op_deriv_spec(e, (const cd*)v_fft, out[1], out[4]);
  op_deriv_spec(e, (const cd*)w_fft, out[2], out[5]);
  derivz_M(e, u, v, w, ustar, M, fi_m, out[6], out[7], out[8]);
  return check_launch(e, "velocityGradients");
}

int alfa_potentialTemperatureGradients(alfa_ctx* c, const double* TH, const double* ustar,
                                       const double* qz, const double* fi_h, double* const out[3]) {
  F64_CHECK(c);
  NN(TH); NN(ustar); NN(qz); NN(fi_h); NN(out); NN(out[0]); NN(out[1]); NN(out[2]);
  Engine& e = c->d->e;
  deriv_field_acc(e, ld_field(e, TH), out[0], 0, out[1], 0);
  derivz_TH(e, TH, ustar, qz, fi_h, out[2]);
  return check_launch(e, "potentialTemperatureGradients");
}

int alfa_moistureGradients(alfa_ctx* c, const double* Q, const double* ustar, const double* qm,
                           const double* fi_h, double* const out[3]) {
  F64_CHECK(c);
  NN(Q); NN(ustar); NN(qm); NN(fi_h); NN(out); NN(out[0]); NN(out[1]); NN(out[2]);
  Engine& e = c->d->e;
  deriv_field_acc(e, ld_field(e, Q), out[0], 0, out[1], 0);
  derivz_TH(e, Q, ustar, qm, fi_h, out[2]);
  return check_launch(e, "moistureGradients");
}

int alfa_Derivz_Generic_uvp(alfa_ctx* c, const double* F, double* d) {
  F64_CHECK(c);
  NN(F); NN(d);
  derivz_generic(c->d->e, F, 0, d);
  return check_launch(c->d->e, "Derivz_Generic_uvp");
}

int alfa_Derivz_Generic_w(alfa_ctx* c, const double* F, double* d) {
  F64_CHECK(c);
  NN(F); NN(d);
  derivz_generic(c->d->e, F, 1, d);
  return check_launch(c->d->e, "Derivz_Generic_w");
}

int alfa_PlanarMean(alfa_ctx* c, const double* F, double* m) {
  F64_CHECK(c);
  NN(F); NN(m);
  const double* f[1] = {F};
  plane_means(c->d->e, f, 1, m);
  return check_launch(c->d->e, "PlanarMean");
}

int alfa_Imfilter(alfa_ctx* c, const double* F, double* out) {
  F64_CHECK(c);
  NN(F); NN(out);
  imfilter(c->d->e, F, out);
  return check_launch(c->d->e, "Imfilter");
}

int alfa_ComputeBeta(alfa_ctx* c, const double* co, int nlev, double* beta) {
  F64_CHECK(c);
  NN(co); NN(beta);
  if (nlev <= 0) return c->d->e.fail("nlev must be positive", ALFA_E_SHAPE);
  compute_beta(c->d->e, co, nlev, beta);
  return check_launch(c->d->e, "ComputeBeta");
}

static int surf(alfa_ctx* c, int var, double sfc, const double* u, const double* v,
                const double* TH, const double* const mi[6], double* M, double* ustar, double* q2,
                double* qavg, double* invOB, double* const mo[6]) {
  F64_CHECK(c);
  NN(u); NN(v); NN(TH); NN(mi); NN(mo); NN(M); NN(ustar); NN(qavg); NN(invOB);
  for (int i = 0; i < 6; i++) {
    NN(mi[i]);
    NN(mo[i]);
  }
  SurfaceIO io;
  io.u = u;
  io.v = v;
  io.TH = TH;
  for (int i = 0; i < 6; i++) {
    io.most_in[i] = mi[i];
    io.most_out[i] = mo[i];
  }
  io.M = M;
  io.ustar = ustar;
  io.q2 = q2 ? q2 : c->d->w.q2;
  io.qavg = qavg;
  io.invOB = invOB;
  surface_flux(c->d->e, var, sfc, io);
  return check_launch(c->d->e, "SurfaceFlux");
}

int alfa_SurfaceFlux_HomogeneousConstantFlux(alfa_ctx* c, const double* u, const double* v,
    const double* TH, const double* const mi[6], double* M, double* ustar, double* qavg,
    double* invOB, double* const mo[6]) {
  return surf(c, 0, 0.0, u, v, TH, mi, M, ustar, nullptr, qavg, invOB, mo);
}
int alfa_SurfaceFlux_HeterogeneousConstantFlux(alfa_ctx* c, const double* u, const double* v,
    const double* TH, const double* const mi[6], double* M, double* ustar, double* qavg,
    double* invOB, double* const mo[6]) {
  return surf(c, 1, 0.0, u, v, TH, mi, M, ustar, nullptr, qavg, invOB, mo);
}
int alfa_SurfaceFlux_HomogeneousVaryingFlux(alfa_ctx* c, const double* u, const double* v,
    const double* TH, double s, const double* const mi[6], double* M, double* ustar,
    double* q2, double* qavg, double* invOB, double* const mo[6]) {
  return surf(c, 2, s, u, v, TH, mi, M, ustar, q2, qavg, invOB, mo);
}
int alfa_SurfaceFlux_HeterogeneousVaryingFlux(alfa_ctx* c, const double* u, const double* v,
    const double* TH, double s, const double* const mi[6], double* M, double* ustar,
    double* q2, double* qavg, double* invOB, double* const mo[6]) {
  return surf(c, 3, s, u, v, TH, mi, M, ustar, q2, qavg, invOB, mo);
}
int alfa_SurfaceFlux_HomogeneousPrescribedTemperature(alfa_ctx* c, const double* u,
    const double* v, const double* TH, double s, const double* const mi[6], double* M,
    double* ustar, double* q2, double* qavg, double* invOB, double* const mo[6]) {
  return surf(c, 4, s, u, v, TH, mi, M, ustar, q2, qavg, invOB, mo);
}
int alfa_SurfaceFlux_HeterogeneousPrescribedTemperature(alfa_ctx* c, const double* u,
    const double* v, const double* TH, double s, const double* const mi[6], double* M,
    double* ustar, double* q2, double* qavg, double* invOB, double* const mo[6]) {
  return surf(c, 5, s, u, v, TH, mi, M, ustar, q2, qavg, invOB, mo);
}

static int moisture_prescribed(alfa_ctx* c, int het, const double* Q, const double* ustar,
                               double Qs, const double* const most[6], double* qm,
                               const char* name) {
  F64_CHECK(c);
  NN(Q); NN(ustar); NN(most); NN(most[2]); NN(most[3]); NN(qm);
  Engine& e = c->d->e;
  const double* qbar0 = nullptr;
  if (!het) {
    const double* f1[1] = {Q};
    plane_means(e, f1, 1, c->d->w.prof + 44 * e.nz);
    qbar0 = c->d->w.prof + 44 * e.nz;
  }
  moisture_surface(e, 2, het, Q, ustar, most[2], most[3], nullptr, nullptr, Qs, qbar0, qm);
  return check_launch(e, name);
}
int alfa_SurfaceMoistureFlux_HomogeneousPrescribedQ(alfa_ctx* c, const double* Q,
    const double* ustar, double Qs, const double* const most[6], double* qm) {
  return moisture_prescribed(c, 0, Q, ustar, Qs, most, qm,
                             "SurfaceMoistureFlux_HomogeneousPrescribedQ");
}
int alfa_SurfaceMoistureFlux_HeterogeneousPrescribedQ(alfa_ctx* c, const double* Q,
    const double* ustar, double Qs, const double* const most[6], double* qm) {
  return moisture_prescribed(c, 1, Q, ustar, Qs, most, qm,
                             "SurfaceMoistureFlux_HeterogeneousPrescribedQ");
}

int alfa_Advection(alfa_ctx* c, const double* u, const double* v, const double* w,
                   const double* dudy, const double* dudz, const double* dvdx, const double* dvdz,
                   const double* dwdx, const double* dwdy, double* Cx, double* Cy, double* Cz) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(dudy); NN(dudz); NN(dvdx); NN(dvdz); NN(dwdx); NN(dwdy);
  NN(Cx); NN(Cy); NN(Cz);
  advection(c->d, u, v, w, dudy, dudz, dvdx, dvdz, dwdx, dwdy, Cx, Cy, Cz);
  return check_launch(c->d->e, "Advection");
}

int alfa_ScalarAdvection(alfa_ctx* c, const double* u, const double* v, const double* w,
                         const double* sx, const double* sy, const double* sz, double* out) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(sx); NN(sy); NN(sz); NN(out);
  scalar_advection(c->d, u, v, w, sx, sy, sz, out, false);
  return check_launch(c->d->e, "ScalarAdvection");
}

int alfa_BuoyancyOpt1(alfa_ctx* c, const double* TH, const double* H, double* b) {
  F64_CHECK(c);
  NN(TH); NN(b);
  buoyancy(c->d->e, TH, H, 0, b);
  return check_launch(c->d->e, "BuoyancyOpt1");
}

int alfa_BuoyancyOpt2(alfa_ctx* c, const double* TH, const double* H, double* b) {
  F64_CHECK(c);
  NN(TH); NN(b);
  buoyancy(c->d->e, TH, H, 1, b);
  return check_launch(c->d->e, "BuoyancyOpt2");
}

int alfa_DivStressDynamicSGS(alfa_ctx* c, const double* const g[9], const double* u,
                             const double* v, const double* w, const double* M, const double* pm,
                             const double* pm0, double* dtx, double* dty, double* dtz,
                             double* avg1, double* avg2, double* beta1, double* Cs2,
                             double* const mom[25]) {
  F64_CHECK(c);
  NN(g); NN(u); NN(v); NN(w); NN(M); NN(pm); NN(pm0); NN(dtx); NN(dty); NN(dtz);
  NN(avg1); NN(avg2); NN(beta1); NN(Cs2); NN(mom);
  for (int i = 0; i < 9; i++) NN(g[i]);
  for (int i = 0; i < 25; i++)
    if (!(i >= 6 && i <= 9)) NN(mom[i]);
  if (c->d->e.cfg.optSgs < 1 || c->d->e.cfg.optSgs > 4)
    return c->d->e.fail("DivStressDynamicSGS needs optSgs 1-4", ALFA_E_CONFIG);
  double* divt[3] = {dtx, dty, dtz};
  double* m[25];
  for (int i = 0; i < 25; i++) m[i] = mom[i];
  int st = dynamic_sgs(c->d, g, u, v, w, M, pm, pm0, divt, avg1, avg2, beta1, Cs2, m);
  if (st) return st;
  Engine& e = c->d->e;
  if (mom[6]) cudaMemcpyAsync(mom[6], avg1, e.nz * 8, cudaMemcpyDeviceToDevice, e.stream);
  if (mom[7]) cudaMemcpyAsync(mom[7], avg2, e.nz * 8, cudaMemcpyDeviceToDevice, e.stream);
  if (mom[8]) cudaMemcpyAsync(mom[8], beta1, e.nz * 8, cudaMemcpyDeviceToDevice, e.stream);
  if (mom[9]) cudaMemcpyAsync(mom[9], Cs2, e.N() * 8, cudaMemcpyDeviceToDevice, e.stream);
  return check_launch(e, "DivStressDynamicSGS");
}

int alfa_DivFluxDynamicSGS(alfa_ctx* c, const double* const m15[15], const double* TH,
                           const double* gx, const double* gy, const double* gz,
                           const double* qz_sfc, double* qz, double* divq, double* r3,
                           double* r1, double* beta2) {
  F64_CHECK(c);
  NN(m15); NN(TH); NN(gx); NN(gy); NN(gz); NN(qz_sfc); NN(qz); NN(divq); NN(r3); NN(r1);
  NN(beta2);
  for (int i = 0; i < 15; i++) NN(m15[i]);
  if (c->d->e.cfg.optSgs < 1 || c->d->e.cfg.optSgs > 4)
    return c->d->e.fail("DivFluxDynamicSGS needs optSgs 1-4", ALFA_E_CONFIG);
  return dynamic_sgs_scalar(c->d, m15, TH, gx, gy, gz, qz_sfc, qz, divq, r3, r1, beta2);
}

int alfa_DivStressStaticSGS(alfa_ctx* c, const double* const g[9], const double* Cs2,
                            const double* u, const double* v, const double* M, const double* pm,
                            const double* pm0, double* dtx, double* dty, double* dtz,
                            double* const mom10[10]) {
  F64_CHECK(c);
  NN(g); NN(Cs2); NN(u); NN(v); NN(M); NN(pm); NN(pm0); NN(dtx); NN(dty); NN(dtz); NN(mom10);
  for (int i = 0; i < 9; i++) NN(g[i]);
  for (int i = 0; i < 10; i++) NN(mom10[i]);
  double* divt[3] = {dtx, dty, dtz};
  return static_sgs(c->d, g, Cs2, u, v, M, pm, pm0, divt, mom10);
}

int alfa_DivFluxStaticSGS(alfa_ctx* c, const double* const m4[4], const double* r3,
                          const double* gx, const double* gy, const double* gz,
                          const double* qz_sfc, double* qz, double* divq) {
  F64_CHECK(c);
  NN(m4); NN(r3); NN(gx); NN(gy); NN(gz); NN(qz_sfc); NN(qz); NN(divq);
  for (int i = 0; i < 4; i++) NN(m4[i]);
  scalar_fluxes(c->d, m4[1], m4[3], r3, gx, gy, gz, qz_sfc, qz, divq);
  return check_launch(c->d->e, "DivFluxStaticSGS");
}

int alfa_RHS_Momentum(alfa_ctx* c, const double* u, const double* v, const double* w,
                      const double* Ug, const double* Vg, const double* Cx, const double* Cy,
                      const double* Cz, const double* b, const double* dtx, const double* dty,
                      const double* dtz, const double* Uadv, const double* Vadv, double* Ru,
                      double* Rv, double* Rw) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(Ug); NN(Vg); NN(Cx); NN(Cy); NN(Cz); NN(b); NN(dtx); NN(dty); NN(dtz);
  NN(Uadv); NN(Vadv); NN(Ru); NN(Rv); NN(Rw);
  Engine& e = c->d->e;
  double* bars = c->d->w.prof + 40 * e.nz;
  if (e.cfg.optDamping == 1) {
    const double* f2[2] = {u, v};
    plane_means(e, f2, 2, bars);
  }
  rhs_momentum(e, u, v, w, Ug, Vg, Cx, Cy, Cz, b, dtx, dty, dtz, Uadv, Vadv, bars, bars + e.nz,
               Ru, Rv, Rw);
  return check_launch(e, "RHS_Momentum");
}

int alfa_RHS_Scalar(alfa_ctx* c, const double* TH, const double* adv, const double* divq,
                    const double* THadv, double* R) {
  F64_CHECK(c);
  NN(TH); NN(adv); NN(divq); NN(THadv); NN(R);
  Engine& e = c->d->e;
  double* bar = c->d->w.prof + 42 * e.nz;
  if (e.cfg.optDamping == 1) {
    const double* f1[1] = {TH};
    plane_means(e, f1, 1, bar);
  }
  rhs_scalar(e, TH, adv, divq, THadv, bar, R);
  return check_launch(e, "RHS_Scalar");
}

int alfa_RHS_Moisture(alfa_ctx* c, const double* Q, const double* adv, const double* divqm,
                      const double* Qadv, double* R) {
  F64_CHECK(c);
  NN(Q); NN(adv); NN(divqm); NN(Qadv); NN(R);
  Engine& e = c->d->e;
  double* bar = c->d->w.prof + 42 * e.nz;
  if (e.cfg.optDamping == 1) {
    const double* f1[1] = {Q};
    plane_means(e, f1, 1, bar);
  }
  rhs_scalar(e, Q, adv, divqm, Qadv, bar, R, nullptr, 0, 1);
  return check_launch(e, "RHS_Moisture");
}

int alfa_PressureRC(alfa_ctx* c, const double* u, const double* v, const double* w,
                    const double* Ru, const double* Rv, const double* Rw, const double* Rup,
                    const double* Rvp, const double* Rwp, const double* divtz, double* RCr,
                    double* RCi, double* fRzr) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(Ru); NN(Rv); NN(Rw); NN(Rup); NN(Rvp); NN(Rwp); NN(divtz);
  NN(RCr); NN(RCi); NN(fRzr);
  return pressure_rc_fn(c->d, u, v, w, Ru, Rv, Rw, Rup, Rvp, Rwp, divtz, RCr, RCi, fRzr);
}

int alfa_ThomasPressureSolve(alfa_ctx* c, const double* RCr, const double* RCi,
                             const double* fRzr, double* p, double* dpdx, double* dpdy,
                             double* dpdz) {
  F64_CHECK(c);
  NN(RCr); NN(RCi); NN(fRzr); NN(p); NN(dpdx); NN(dpdy); NN(dpdz);
  return pressure_solve_fn(c->d, RCr, RCi, fRzr, p, dpdx, dpdy, dpdz);
}

int alfa_AB2_uvw(alfa_ctx* c, const double* u, const double* v, const double* w,
                 const double* Ru, const double* Rup, const double* Rv, const double* Rvp,
                 const double* Rw, const double* Rwp, double* un, double* vn, double* wn) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(Ru); NN(Rup); NN(Rv); NN(Rvp); NN(Rw); NN(Rwp); NN(un); NN(vn); NN(wn);
  ab2_uvw(c->d->e, u, v, w, Ru, Rup, Rv, Rvp, Rw, Rwp, un, vn, wn);
  return check_launch(c->d->e, "AB2_uvw");
}

int alfa_AddPressureGradient(alfa_ctx* c, double* Ru, double* Rv, double* Rw, const double* dpdx,
                             const double* dpdy, const double* dpdz) {
  F64_CHECK(c);
  NN(Ru); NN(Rv); NN(Rw); NN(dpdx); NN(dpdy); NN(dpdz);
  subtract3(c->d->e, Ru, Rv, Rw, dpdx, dpdy, dpdz);
  return check_launch(c->d->e, "AddPressureGradient");
}

__global__ void k_cfl3(const double* __restrict__ m, double* out, double dt, double dx, double dy,
                       double dz) {
  if (threadIdx.x == 0) {
    out[0] = m[0] * dt / dx;
    out[1] = m[1] * dt / dy;
    out[2] = m[2] * dt / dz;
  }
}

int alfa_CFL(alfa_ctx* c, const double* u, const double* v, const double* w, double* cfl3) {
  F64_CHECK(c);
  NN(u); NN(v); NN(w); NN(cfl3);
  Engine& e = c->d->e;
  cfl_max(e, u, v, w, c->d->w.d_cfl);
  // Main.py:534-536: max|.| * dt_nondim / dx
  ::alfa::note_launch();
  k_cfl3<<<1, 32, 0, e.stream>>>(c->d->w.d_cfl, cfl3, e.dt_nondim, e.dx, e.dy, e.dz);
  return check_launch(e, "CFL");
}


int alfa_AB2_TH(alfa_ctx* c, const double* TH, const double* R, const double* Rp, double* out) {
  F64_CHECK(c);
  NN(TH); NN(R); NN(Rp); NN(out);
  ab2_th(c->d->e, TH, R, Rp, out);
  return check_launch(c->d->e, "AB2_TH");
}

int alfa_AB2_Q(alfa_ctx* c, const double* Q, const double* R, const double* Rp, double* out) {
  F64_CHECK(c);
  NN(Q); NN(R); NN(Rp); NN(out);
  ab2_q(c->d->e, Q, R, Rp, out);
  return check_launch(c->d->e, "AB2_Q");
}

static int compute_stats_checked(alfa_ctx* c, StatsIn& a, double* acc) {
  F64_CHECK(c);
  NN(a.u); NN(a.v); NN(a.w); NN(a.TH); NN(a.dudz); NN(a.dvdz); NN(a.dTHdz); NN(a.M);
  NN(a.ustar); NN(a.qz_sfc_avg); NN(a.txy); NN(a.txz); NN(a.tyz); NN(a.qz); NN(a.cs2_1);
  NN(a.cs2_2); NN(a.cs2pr); NN(a.beta1); NN(a.beta2); NN(acc);
  if (a.Q && (!a.dQdz || !a.qHz))
    return c->d->e.fail("ComputeStats: Q needs dQdz and qHz_q", ALFA_E_SHAPE);
  compute_stats(c->d->e, a, acc);
  return check_launch(c->d->e, "ComputeStats");
}

int alfa_ComputeStats(alfa_ctx* c, const double* u, const double* v, const double* w,
                      const double* TH, const double* Q, const double* dudz, const double* dvdz,
                      const double* dTHdz, const double* dQdz, const double* M_sfc_loc,
                      const double* ustar, const double* qz_sfc_avg, const double* qm_sfc_avg,
                      const double* txy, const double* txz, const double* tyz, const double* qz,
                      const double* qHz_q, const double* Cs2_1D_avg1,
                      const double* Cs2_1D_avg2, const double* Cs2PrRatio_1D,
                      const double* beta1_1D, const double* beta2_1D, double* acc) {
  F64_CHECK(c);
  Engine& e = c->d->e;
  StatsIn a{u, v, w, TH, dudz, dvdz, dTHdz, txy, txz, tyz, qz, M_sfc_loc, ustar, qz_sfc_avg,
            Cs2_1D_avg1, Cs2_1D_avg2, Cs2PrRatio_1D, beta1_1D, beta2_1D, e.cfg.Ugal,
            e.T0_nondim};
  a.Q = Q;
  a.dQdz = dQdz;
  a.qHz = qHz_q;
  a.qm_sfc_avg = qm_sfc_avg;
  return compute_stats_checked(c, a, acc);
}


}  // extern "C"

// ---------------------------------------------------------------------------
// ensemble: independent contexts of one precision stepped together
// ---------------------------------------------------------------------------
struct alfa_ensemble {
  f64::Ens* d = nullptr;
  alfa::f32::Ens* f = nullptr;
  std::string err;
};

extern "C" {

int alfa_ensemble_create(alfa_ctx* const* members, int n, alfa_ensemble** out) {
  if (!members || n < 1 || !out) return ALFA_E_SHAPE;
  for (int i = 0; i < n; i++)
    if (!members[i]) return ALFA_E_STATE;
  const bool fp64 = members[0]->d != nullptr;
  for (int i = 1; i < n; i++)
    if ((members[i]->d != nullptr) != fp64) return ALFA_E_CONFIG;  // one precision per ensemble
  alfa_ensemble* E = new alfa_ensemble();
  int st;
  if (fp64) {
    std::vector<f64::Ctx*> m(n);
    for (int i = 0; i < n; i++) m[i] = members[i]->d;
    st = f64::ens_create(m.data(), n, &E->d);
  } else {
    std::vector<alfa::f32::Ctx*> m(n);
    for (int i = 0; i < n; i++) m[i] = members[i]->f;
    st = alfa::f32::ens_create(m.data(), n, &E->f);
  }
  if (st) {
    delete E;
    return st;
  }
  *out = E;
  return ALFA_OK;
}

int alfa_ensemble_step(alfa_ensemble* E, int nsteps) {
  if (!E) return ALFA_E_STATE;
  return E->d ? f64::ens_step(E->d, nsteps) : alfa::f32::ens_step(E->f, nsteps);
}

int alfa_ensemble_sync(alfa_ensemble* E) {
  if (!E) return ALFA_E_STATE;
  return E->d ? f64::ens_sync(E->d) : alfa::f32::ens_sync(E->f);
}

int alfa_ensemble_set_stream(alfa_ensemble* E, void* stream) {
  if (!E) return ALFA_E_STATE;
  cudaStream_t s = (cudaStream_t)stream;
  return E->d ? f64::ens_set_stream(E->d, s) : alfa::f32::ens_set_stream(E->f, s);
}

const char* alfa_ensemble_error(const alfa_ensemble* E) {
  if (!E) return "";
  return E->d ? f64::ens_error(E->d) : alfa::f32::ens_error(E->f);
}

void alfa_ensemble_destroy(alfa_ensemble* E) {
  if (!E) return;
  if (E->d) f64::ens_destroy(E->d);
  if (E->f) alfa::f32::ens_destroy(E->f);
  delete E;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// learned SGS coefficient (alfa_mlp.cu): data collection, training, the
// learned step with the dynamic procedure as periodic judge
// ---------------------------------------------------------------------------

static MlpFeatIn feat_in(alfa_ctx* c) {
  Engine& e = c->d->e;
  f64::Work& W = c->d->w;
  MlpFeatIn a;
  for (int i = 0; i < 9; i++) a.g[i] = W.g[i];
  a.dTHdz = W.gT[2];
  a.L = e.L;
  a.dz = e.dz;
  a.g_over_T0 = e.g_nondim / e.T0_nondim;
  a.nz = e.nz;
  return a;
}

// the network's Cs^2 for a step (the hidden layer on the tensor cores)
static void learned_cs2(alfa_ctx* c, double* Cs2_out) {
  alfa_mlp* m = c->mlp;
  mlp_infer_tc(c->d->e.stream, c->d->e.sms, feat_in(c), m->Pb, m->norm, c->d->e.N(), m->calib,
               Cs2_out);
}

extern "C" {

void alfa_mlp_destroy(alfa_mlp* m) {
  if (!m) return;
  if (m->c && m->c->mlp == m) {
    m->c->mlp = nullptr;
    m->c->d->learned = nullptr;
  }
  for (void* p : {(void*)m->X, (void*)m->T, (void*)m->norm, (void*)m->P, (void*)m->G,
                  (void*)m->M, (void*)m->V, (void*)m->loss, (void*)m->perm, (void*)m->Pb,
                  (void*)m->scratch, (void*)m->means, (void*)m->calib})
    if (p) cudaFree(p);
  delete m;
}

int alfa_mlp_create(alfa_ctx* c, int capacity, unsigned long long seed, alfa_mlp** out) {
  F64_CHECK(c);
  if (!out || capacity < 64) return c->d->e.fail("mlp_create: bad arguments", ALFA_E_SHAPE);
  alfa_mlp* m = new alfa_mlp();
  m->c = c;
  m->cap = capacity;
  m->seed = seed;
  const size_t N = c->d->e.N();
  bool ok = true;
  auto al = [&](void** p, size_t bytes) {
    if (ok && cudaMalloc(p, bytes) != cudaSuccess) ok = false;
  };
  al((void**)&m->X, (size_t)capacity * MLP_IN * 4);
  al((void**)&m->T, (size_t)capacity * 2 * 4);
  al((void**)&m->norm, 2 * (MLP_IN + 2) * 4);
  al((void**)&m->P, MLP_NPARAM * 4);
  al((void**)&m->G, MLP_NPARAM * 4);
  al((void**)&m->M, MLP_NPARAM * 4);
  al((void**)&m->V, MLP_NPARAM * 4);
  al((void**)&m->loss, 16);
  al((void**)&m->perm, (size_t)capacity * 4);
  al((void**)&m->Pb, MLP_NPARAM * 2);
  al((void**)&m->scratch, N * 8);
  al((void**)&m->means, (size_t)2 * c->d->e.nz * 8);
  al((void**)&m->calib, (size_t)c->d->e.nz * 8);
  if (!ok) {
    alfa_mlp_destroy(m);
    return c->d->e.fail("mlp_create: device allocation failed", ALFA_E_CUDA);
  }
  // Glorot-uniform weights, zero biases (host RNG from the seed)
  std::vector<float> p(MLP_NPARAM, 0.0f);
  unsigned long long x = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&]() {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int rows, int cols) {
    const double a = std::sqrt(6.0 / (rows + cols));
    for (int q = 0; q < rows * cols; q++) p[off + q] = (float)((2.0 * uni() - 1.0) * a);
  };
  const int OW1 = 0, OB1 = MLP_H * MLP_IN, OW2 = OB1 + MLP_H, OB2 = OW2 + MLP_H * MLP_H,
            OW3 = OB2 + MLP_H;
  fill(OW1, MLP_H, MLP_IN);
  fill(OW2, MLP_H, MLP_H);
  fill(OW3, 2, MLP_H);
  std::vector<float> nm(2 * (MLP_IN + 2), 0.0f);
  for (int q = MLP_IN + 2; q < 2 * (MLP_IN + 2); q++) nm[q] = 1.0f;
  m->calib_h.assign(c->d->e.nz, 1.0);
  cudaMemcpy(m->calib, m->calib_h.data(), c->d->e.nz * 8, cudaMemcpyHostToDevice);
  cudaMemcpy(m->P, p.data(), MLP_NPARAM * 4, cudaMemcpyHostToDevice);
  cudaMemcpy(m->norm, nm.data(), nm.size() * 4, cudaMemcpyHostToDevice);
  cudaMemset(m->G, 0, MLP_NPARAM * 4);
  cudaMemset(m->M, 0, MLP_NPARAM * 4);
  cudaMemset(m->V, 0, MLP_NPARAM * 4);
  mlp_to_bf16(c->d->e.stream, m->P, m->Pb);
  c->mlp = m;
  c->d->learned = [c](double* Cs2) { learned_cs2(c, Cs2); };
  *out = m;
  return check_launch(c->d->e, "mlp_create");
}

int alfa_mlp_collect(alfa_mlp* m, int npoints) {
  if (!m || !m->c) return ALFA_E_STATE;
  alfa_ctx* c = m->c;
  if (!c->d->w.last_dyn)
    return c->d->e.fail("mlp_collect: the last step did not run the dynamic procedure", ALFA_E_STATE);
  if (npoints < 1 || npoints > m->cap) return c->d->e.fail("mlp_collect: bad count", ALFA_E_SHAPE);
  const int nz = c->d->e.nz;
  mlp_sample(c->d->e.stream, feat_in(c), c->d->w.Cs2, c->d->w.prof + 20 * nz, c->d->e.N(),
             m->seed + (++m->draws), npoints, m->X, m->T, m->offset, m->cap);
  m->offset = (m->offset + npoints) % m->cap;
  m->count = std::min(m->cap, m->count + npoints);
  return check_launch(c->d->e, "mlp_collect");
}

int alfa_mlp_train(alfa_mlp* m, int epochs, int batch, double lr, double* loss_out) {
  if (!m || !m->c) return ALFA_E_STATE;
  alfa_ctx* c = m->c;
  Engine& e = c->d->e;
  if (m->count < batch || batch < 1 || epochs < 1)
    return e.fail("mlp_train: too few samples for one batch", ALFA_E_SHAPE);
  if (!m->trained) mlp_norm(e.stream, m->X, m->T, m->count, m->norm);
  m->trained = 1;
  std::vector<int> perm(m->count);
  unsigned long long x = m->seed ^ 0x5DEECE66Dull;
  double last = 0.0;
  for (int ep = 0; ep < epochs; ep++) {
    for (int q = 0; q < m->count; q++) perm[q] = q;
    for (int q = m->count - 1; q > 0; q--) {  // Fisher-Yates
      x = x * 6364136223846793005ull + 1442695040888963407ull;
      const int r = (int)((x >> 33) % (unsigned long long)(q + 1));
      std::swap(perm[q], perm[r]);
    }
    cudaMemcpyAsync(m->perm, perm.data(), (size_t)m->count * 4, cudaMemcpyHostToDevice, e.stream);
    cudaMemsetAsync(m->loss, 0, 4, e.stream);
    int nb = 0;
    for (int s0 = 0; s0 + batch <= m->count; s0 += batch, nb++) {
      mlp_grad(e.stream, m->P, m->X, m->T, m->perm, s0, batch, m->count, m->norm, m->G, m->loss);
      mlp_adam(e.stream, m->P, m->G, m->M, m->V, m->Pb, (float)lr, ++m->adam_t);
    }
    float l = 0.0f;
    cudaMemcpyAsync(&l, m->loss, 4, cudaMemcpyDeviceToHost, e.stream);
    if (cudaStreamSynchronize(e.stream) != cudaSuccess) return e.fail("mlp_train failed", ALFA_E_CUDA);
    last = nb ? l / nb : 0.0;
  }
  if (loss_out) *loss_out = last;
  return check_launch(e, "mlp_train");
}

int alfa_mlp_loss_grad(alfa_mlp* m, const float* X, const float* T, const float* norm, int n,
                       float* grad, float* loss) {
  if (!m || !m->c) return ALFA_E_STATE;
  alfa_ctx* c = m->c;
  NN(X); NN(T); NN(norm); NN(grad); NN(loss);
  if (n < 1) return ALFA_E_SHAPE;
  Engine& e = m->c->d->e;
  cudaMemsetAsync(grad, 0, MLP_NPARAM * 4, e.stream);
  cudaMemsetAsync(loss, 0, 4, e.stream);
  mlp_grad(e.stream, m->P, X, T, nullptr, 0, n, n, norm, grad, loss);
  return check_launch(e, "mlp_loss_grad");
}

int alfa_mlp_get_params(alfa_mlp* m, float* P, float* norm) {
  if (!m || !m->c) return ALFA_E_STATE;
  Engine& e = m->c->d->e;
  if (P) cudaMemcpyAsync(P, m->P, MLP_NPARAM * 4, cudaMemcpyDeviceToDevice, e.stream);
  if (norm) cudaMemcpyAsync(norm, m->norm, 2 * (MLP_IN + 2) * 4, cudaMemcpyDeviceToDevice, e.stream);
  return check_launch(e, "mlp_get_params");
}

int alfa_mlp_set_params(alfa_mlp* m, const float* P, const float* norm) {
  if (!m || !m->c) return ALFA_E_STATE;
  Engine& e = m->c->d->e;
  if (P) cudaMemcpyAsync(m->P, P, MLP_NPARAM * 4, cudaMemcpyDeviceToDevice, e.stream);
  if (norm) {
    cudaMemcpyAsync(m->norm, norm, 2 * (MLP_IN + 2) * 4, cudaMemcpyDeviceToDevice, e.stream);
    m->trained = 1;
  }
  mlp_to_bf16(e.stream, m->P, m->Pb);
  return check_launch(e, "mlp_set_params");
}

int alfa_mlp_features(alfa_mlp* m, float* X) {
  if (!m || !m->c) return ALFA_E_STATE;
  alfa_ctx* c = m->c;
  NN(X);
  mlp_features_all(m->c->d->e.stream, feat_in(m->c), m->c->d->e.N(), X);
  return check_launch(m->c->d->e, "mlp_features");
}

int alfa_mlp_infer(alfa_mlp* m, double* Cs2, double* beta) {
  if (!m || !m->c) return ALFA_E_STATE;
  alfa_ctx* c = m->c;
  NN(Cs2);
  mlp_infer(m->c->d->e.stream, m->c->d->e.sms, feat_in(m->c), m->Pb, m->norm, m->c->d->e.N(),
            m->calib, Cs2, beta);
  return check_launch(m->c->d->e, "mlp_infer");
}

int alfa_step_learned(alfa_mlp* m, int nsteps, int judge_every, double tol, int refresh_points,
                      int refresh_epochs, alfa_mlp_report* rep) {
  if (!m || !m->c) return ALFA_E_STATE;
  alfa_ctx* c = m->c;
  Engine& e = c->d->e;
  f64::Work& W = c->d->w;
  if (e.cfg.optSgs < 1 || e.cfg.optSgs > 4)
    return e.fail("step_learned needs a dynamic SGS model (optSgs 1-4)", ALFA_E_CONFIG);
  if (!m->trained) return e.fail("step_learned before mlp_train", ALFA_E_STATE);
  if (judge_every < 1 || !rep) return e.fail("step_learned: bad arguments", ALFA_E_SHAPE);
  const int nz = e.nz;
  for (int s = 0; s < nsteps; s++) {
    const int it = W.iteration;
    const bool judge =
        rep->reverted || rep->judged == 0 || it == e.cfg.istep || it % judge_every == 0;
    int st = f64::step(c->d, 1, judge ? 2 : 1);
    if (st) return st;
    rep->steps++;
    if (!judge) {
      rep->learned_steps++;
      continue;
    }
    if (rep->reverted) continue;
    // judge: the network on the same state against the procedure's Cs^2
    learned_cs2(c, m->scratch);
    const double* f2[2] = {m->scratch, W.Cs2};
    plane_means(e, f2, 2, m->means);
    std::vector<double> h(2 * nz);
    cudaMemcpyAsync(h.data(), m->means, 2 * nz * 8, cudaMemcpyDeviceToHost, e.stream);
    if (cudaStreamSynchronize(e.stream) != cudaSuccess) return e.fail("judge failed", ALFA_E_CUDA);
    double num = 0.0, den = 0.0;  // relative L2 difference of the two profiles
    for (int z = 0; z < nz; z++) {
      num += (h[z] - h[nz + z]) * (h[z] - h[nz + z]);
      den += h[nz + z] * h[nz + z];
    }
    const double drift = den > 0 ? std::sqrt(num / den) : 0.0;
    rep->judged++;
    rep->last_drift = drift;
    rep->max_drift = std::max(rep->max_drift, drift);
    // the windowed drift: relative L2 difference of the two profiles
    // averaged over the last ALFA_MLP_JUDGE_WINDOW judge steps
    m->window.push_back(h);
    if ((int)m->window.size() > ALFA_MLP_JUDGE_WINDOW) m->window.pop_front();
    bool full = (int)m->window.size() == ALFA_MLP_JUDGE_WINDOW;
    if (full) {
      double wn = 0.0, wd = 0.0;
      for (int z = 0; z < nz; z++) {
        double a = 0.0, b = 0.0;
        for (const auto& v : m->window) {
          a += v[z];
          b += v[nz + z];
        }
        wn += (a - b) * (a - b);
        wd += b * b;
      }
      rep->window_drift = wd > 0 ? std::sqrt(wn / wd) : 0.0;
      rep->max_window_drift = std::max(rep->max_window_drift, rep->window_drift);
    }
    if (full && rep->window_drift > tol) {
      rep->reverted = 1;
      rep->reverted_at = it;
      continue;
    }
    // recalibrate the levels to this step's procedure profile (ratios held
    // within [0.1, 10]; levels where either mean is ~0 keep their factor)
    for (int z = 0; z < nz; z++) {
      const double net = h[z], dyn = h[nz + z];
      if (net > 1e-12 && dyn > 1e-12)
        m->calib_h[z] = std::min(10.0, std::max(0.1, m->calib_h[z] * dyn / net));
    }
    cudaMemcpyAsync(m->calib, m->calib_h.data(), nz * 8, cudaMemcpyHostToDevice, e.stream);
    if (refresh_points > 0 && refresh_epochs > 0) {
      // keep learning from the procedure's own fields of this judge step
      st = alfa_mlp_collect(m, std::min(refresh_points, m->cap));
      if (!st && m->count >= 1024) st = alfa_mlp_train(m, refresh_epochs, 1024, 1e-3, nullptr);
      if (st) return st;
    }
  }
  return check_launch(e, "step_learned");
}

}  // extern "C"
