// The whole-step driver of one precision build: engine set-up, the
// workspace, the composite operators behind the reference's functions, the
// loop body of the reference's src/Main.py:156-541, state import/export,
// statistics, checkpoints, kernel probes, the line-pass autotuner and the
// ensemble.  Compiled twice (alfa_prec.cuh): FP64 into alfa::f64, FP32 into
// alfa::f32.  State crosses the interface as FP64 device buffers.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "alfa_step.cuh"

namespace alfa {
namespace ALFA_PREC {

#define NN(p) \
  if (!(p)) return c->e.fail("null pointer argument: " #p, ALFA_E_SHAPE)

// ---------------------------------------------------------------------------
// set-up
// ---------------------------------------------------------------------------
static bool factor_23(int n, int* rad, int* np) {
  int m = n, k = 0;
  const int rs[5] = {16, 8, 4, 3, 2};
  for (int r : rs) {
    while (m % r == 0 && m > 1) {
      if (k >= 8) return false;
      rad[k++] = r;
      m /= r;
    }
  }
  *np = k;
  return m == 1 && n >= 2;
}

// radix schedule r of the autotuner: 0 largest radix 8, 1 largest radix 4,
// 2 the default factors in ascending order
static bool factor_sched(int n, int r, int* rad, int* np) {
  if (r == 2) {
    if (!factor_23(n, rad, np)) return false;
    std::reverse(rad, rad + *np);
    return true;
  }
  const int rs8[4] = {8, 4, 3, 2}, rs4[3] = {4, 3, 2};
  const int* rs = r == 0 ? rs8 : rs4;
  const int nr = r == 0 ? 4 : 3;
  int m = n, k = 0;
  for (int t = 0; t < nr; t++) {
    while (m % rs[t] == 0 && m > 1) {
      if (k >= 8) return false;
      rad[k++] = rs[t];
      m /= rs[t];
    }
  }
  *np = k;
  return m == 1 && n >= 2;
}

static int make_plan(Engine& e, int n, FftPlan* p, int sched = -1) {
  p->n = n;
  if (sched < 0 ? !factor_23(n, p->rad, &p->npass) : !factor_sched(n, sched, p->rad, &p->npass))
    return -1;
  std::vector<cd> tw(n);
  for (int q = 0; q < n; q++) {  // long double, rounded once to the build's precision
    const long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)q / n;
    tw[q] = mkc((real)cosl(a), (real)sinl(a));
  }
  void* d = nullptr;
  if (cudaMalloc(&d, n * sizeof(cd)) != cudaSuccess) return -2;
  cudaMemcpy(d, tw.data(), n * sizeof(cd), cudaMemcpyHostToDevice);
  e.allocs.push_back(d);
  p->tw = (const cd*)d;
  return 0;
}

static double* upload(Engine& e, const std::vector<double>& h) {
  void* d = nullptr;
  if (cudaMalloc(&d, h.size() * sizeof(double) + 8) != cudaSuccess) return nullptr;
  cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
  e.allocs.push_back(d);
  return (double*)d;
}

int check_launch(Engine& e, const char* what) {
  cudaError_t st = cudaGetLastError();
  if (st != cudaSuccess) {
    e.err = std::string(what) + ": " + cudaGetErrorString(st);
    return ALFA_E_CUDA;
  }
  return ALFA_OK;
}

int engine_init(Engine& e, const alfa_config& c) {
  e.cfg = c;
  const double PI = 3.141592653589793;  // jnp.pi
  e.nx = c.nx;
  e.ny = c.ny;
  e.nz = c.nz;
  if (c.nx < 4 || c.ny < 4 || c.nz < 3 || (c.nx % 2) || (c.ny % 2))
    return e.fail("grid must have even nx, ny >= 4 and nz >= 3", ALFA_E_CONFIG);
  if (c.FGR < 1) return e.fail("FGR must be >= 1", ALFA_E_CONFIG);
  if (c.optSgs < 0 || c.optSgs > 4)
    return e.fail("optSgs must be 0 (static), 1 (LASDD-SM), 2 (LASDD-WL), 3 (LAD-SM) or 4 (LAD-WL)",
                  ALFA_E_CONFIG);
  if (c.dynamicSGS_call_time < 1) return e.fail("dynamicSGS_call_time must be >= 1", ALFA_E_CONFIG);
  e.mx = (int)(1.5 * c.nx);
  e.my = (int)(1.5 * c.ny);
  if (c.ny > 512 || c.nx > 1024)
    return e.fail("grid too large for the FFT tiles (ny <= 512, nx <= 1024)", ALFA_E_CONFIG);
  if ((size_t)e.mx * (size_t)e.my * (size_t)(c.nz + 1) >= ((size_t)1 << 32))
    return e.fail("grid too large: 1.5 nx x 1.5 ny x (nz + 1) must stay below 2^32 points",
                  ALFA_E_CONFIG);
  e.nxh = c.nx / 2 + 1;
  e.nyh = c.ny / 2 + 1;
  e.mxh = e.mx / 2 + 1;
  e.myh = e.my / 2 + 1;
  // src/config/DerivedVars.py:48-112 (u_scale = TH_scale = 1)
  e.z_scale = c.l_x / (2 * PI);
  e.g_nondim = 9.81 * e.z_scale / 1.0;
  e.f_nondim = c.f_coriolis * (e.z_scale / 1.0);
  e.T0_nondim = c.T_0 / 1.0;
  e.inversion_nondim = c.inversion * (e.z_scale / 1.0);
  e.qz_sfc_const = c.SensibleHeatFlux * 1.0 / (1.0 * 1.0);
  // moisture: DerivedVars.py:69-75 (Q_scale = 1), SurfaceFlux.py:475-476
  if (c.optMoisture < 0 || c.optMoisture > 1 || c.optMoistureSurfBC < 0 ||
      c.optMoistureSurfBC > 2)
    return e.fail("optMoisture must be 0 or 1 and optMoistureSurfBC 0, 1 or 2", ALFA_E_CONFIG);
  e.q_inversion_nondim = c.q_inversion * (e.z_scale / 1.0);
  e.qm_sfc_const = c.MoistureFlux / (1.0 * 1.0);
  e.dx = 2 * PI / c.nx;
  e.dy = 2 * PI / c.ny;
  e.dz = (c.l_z / e.z_scale) / (c.nz - 1);
  e.idz = 1.0 / e.dz;
  e.log_zq = std::log(0.5 * e.dz * e.z_scale / (c.zMoisture > 0.0 ? c.zMoisture : c.z0T));
  e.L = c.FGR * std::pow(e.dx * e.dy * e.dz, 1.0 / 3.0);
  e.dt_nondim = c.dt * 1.0 / e.z_scale;
  // DerivedVars.py: FGR = 1 -> 3/2-rule dealiasing with TFR = 2; FGR > 1 -> the
  // grid filter removes the aliased band, products are formed in physical
  // space (the *_NoDealias functions) and TFR = sqrt(2)
  e.TFR = (c.FGR == 1) ? 2.0 : std::sqrt(2.0);
  e.optDealias = (c.FGR == 1) ? 1 : 0;
  e.Cs2_init = c.Cs2;
  e.Cs2PrRatio_init = c.Cs2PrRatio;
  e.z_damping_nondim = c.z_damping / e.z_scale;
  e.RelaxTime_nondim = c.RelaxTime * (1.0 / e.z_scale);
  // Filtering.py cut-offs (Python round(): ties to even)
  const double inv2fgr = 1.0 / (2.0 * c.FGR);
  e.cut_e[0] = (int)std::nearbyint(c.nx * inv2fgr);
  e.cut_e[1] = (int)std::nearbyint(c.ny * inv2fgr);
  e.cut_1[0] = (int)std::nearbyint(c.nx / (2 * c.FGR * e.TFR));
  e.cut_1[1] = (int)std::nearbyint(c.ny / (2 * c.FGR * e.TFR));
  e.cut_2[0] = (int)std::nearbyint(c.nx / (2 * c.FGR * e.TFR * e.TFR));
  e.cut_2[1] = (int)std::nearbyint(c.ny / (2 * c.FGR * e.TFR * e.TFR));
  if (e.cut_2[0] < 1 || e.cut_2[1] < 1) return e.fail("grid too small for the test filters", ALFA_E_CONFIG);

  if (make_plan(e, e.nx, &e.pnx) || make_plan(e, e.ny, &e.pny) || make_plan(e, e.mx, &e.pmx) ||
      make_plan(e, e.my, &e.pmy))
    return e.fail("nx and ny must be of the form 2^a 3^b (FFT radices 2, 3, 4, 8, 16)",
                  ALFA_E_CONFIG);
  {  // alternative radix schedules for the autotuner (a schedule with more
     // than 8 passes falls back to the default factors)
    const int lens[4] = {e.nx, e.ny, e.mx, e.my};
    const FftPlan* def[4] = {&e.pnx, &e.pny, &e.pmx, &e.pmy};
    for (int L = 0; L < 4; L++)
      for (int r = 0; r < Engine::N_SCHED; r++)
        if (make_plan(e, lens[L], &e.alt_plans[L][r], r)) e.alt_plans[L][r] = *def[L];
  }

  // wavenumbers (Preprocess.py:89-94): fftfreq / rfftfreq with Nyquist 0
  std::vector<double> kx(c.nx), ky(e.nyh), kr(c.nx);
  for (int i = 0; i < c.nx; i++) {
    kx[i] = (i < c.nx / 2) ? i : i - c.nx;
    kr[i] = kx[i];  // pressure wavenumbers keep the Nyquist (NSE_PressureTerms.py:72-77)
  }
  kx[c.nx / 2] = 0.0;
  for (int j = 0; j < e.nyh; j++) ky[j] = j;
  ky[c.ny / 2] = 0.0;
  e.d_kx = upload(e, kx);
  e.d_ky = upload(e, ky);
  e.d_kr = upload(e, kr);

  // Thomas factors (NSE_PressureTerms_Thomas.py:151-214)
  const int nz = c.nz, N1 = nz + 1;
  const double dz = e.dz;
  std::vector<double> a(N1, 1.0 / (dz * dz)), cc(N1, 1.0 / (dz * dz));
  a[0] = 0;
  a[nz] = -1;
  cc[0] = 1;
  cc[nz] = 0;
  const size_t nm = (size_t)c.nx * e.nyh;
  std::vector<double> bt(nm * N1), mt(nm * N1, 0.0);  // both (nx, nyh, nz+1)
  for (int i = 0; i < c.nx; i++) {
    for (int j = 0; j < e.nyh; j++) {
      const size_t m = (size_t)i * e.nyh + j;
      double* b = &bt[m * N1];
      const double kr2 = kr[i], kc2 = j;
      const double bb = -(kr2 * kr2 + kc2 * kc2 + 2 / (dz * dz));
      for (int k = 0; k < N1; k++) b[k] = bb;
      b[0] = -1;
      b[nz] = 1;
      if (i == 0 && j == 0 && c.optPressureSolver == 1)
        for (int k = 1; k < nz; k++) b[k] = -(1.0 + 2.0 / (dz * dz));
      for (int k = 1; k < N1; k++) {
        const double mk = a[k] / b[k - 1];
        mt[m * N1 + k] = mk;
        b[k] = b[k] - mk * cc[k - 1];
      }
    }
  }
  e.d_b_thomas = upload(e, bt);
  e.d_m_thomas = upload(e, mt);
  e.d_c_p = upload(e, cc);

  // Rayleigh damping profiles (Initialization.py:395-460)
  {
    const double inv = 1.0 / e.RelaxTime_nondim;
    const double ztop = c.l_z / e.z_scale;
    const double thick = ztop - e.z_damping_nondim;
    std::vector<double> r1(nz), r2(nz);
    for (int k = 0; k < nz; k++) {
      const double z1 = k * dz, z2 = (k + 0.5) * dz;
      r1[k] = (z1 >= e.z_damping_nondim && z1 <= ztop)
                  ? 0.5 * inv * (1.0 - std::cos(PI * (z1 - e.z_damping_nondim) / thick))
                  : 0.0;
      r2[k] = (z2 >= e.z_damping_nondim && z2 <= ztop)
                  ? 0.5 * inv * (1.0 - std::cos(PI * (z2 - e.z_damping_nondim) / thick))
                  : 0.0;
    }
    e.d_rd = upload(e, r1);
    e.d_rd_stag = upload(e, r2);
  }
  if (!e.d_kx || !e.d_b_thomas || !e.d_rd) return e.fail("device allocation failed", ALFA_E_CUDA);
  return ALFA_OK;
}

void engine_free(Engine& e) {
  for (void* p : e.allocs) cudaFree(p);
  e.allocs.clear();
}

// carve the workspace: counts first, then pointers
struct Carver {
  char* base;
  size_t off = 0;
  bool dry;
  template <class T>
  T* take(size_t n) {
    off = (off + 255) & ~(size_t)255;
    T* p = dry ? nullptr : (T*)(base + off);
    off += n * sizeof(T);
    return p;
  }
};

static void carve(Ctx* c, Carver& k) {
  Engine& e = c->e;
  Work& w = c->w;
  const size_t N = e.N(), P = e.P(), S = e.S(), H = e.H(), nz = e.nz;
  const size_t R = (size_t)e.nx * e.nyh * (nz + 1);
  w.u = k.take<real>(N);
  w.v = k.take<real>(N);
  w.w = k.take<real>(N);
  w.TH = k.take<real>(N);
  w.p = k.take<real>(N);
  for (int i = 0; i < 4; i++) {
    w.RHS[i] = k.take<real>(N);
    w.RHSp[i] = k.take<real>(N);
  }
  w.Cs2 = k.take<real>(N);
  w.Cs2Pr = k.take<real>(N);
  for (int i = 0; i < 6; i++) {
    w.most[i] = k.take<double>(H);
    w.most_new[i] = k.take<double>(H);
  }
  w.M = k.take<double>(H);
  w.ustar = k.take<double>(H);
  w.q2 = k.take<double>(H);
  w.invOB = k.take<double>(H);
  w.qz_plane = k.take<double>(H);
  w.ufft = k.take<cd>(S);
  w.vfft = k.take<cd>(S);
  w.wfft = k.take<cd>(S);
  w.Ug = k.take<double>(nz);
  w.Vg = k.take<double>(nz);
  w.zero_prof = k.take<double>(nz);
  for (int i = 0; i < 9; i++) w.g[i] = k.take<real>(N);
  for (int i = 0; i < 3; i++) w.gT[i] = k.take<real>(N);
  w.Cx = k.take<real>(N);
  w.Cy = k.take<real>(N);
  w.Cz = k.take<real>(N);
  w.THadv = k.take<real>(N);
  w.buoy = k.take<real>(N);
  for (int i = 0; i < 3; i++) w.divt[i] = k.take<real>(N);
  w.divq = k.take<real>(N);
  w.qz = k.take<real>(N);
  for (int i = 0; i < 25; i++) {
    if (i >= 6 && i <= 9) {
      w.mom[i] = nullptr;
      continue;
    }
    w.mom[i] = (i == 20 || i == 22) ? k.take<real>(P) : k.take<real>(N);
  }
  w.S12 = k.take<real>(N);
  w.S13 = k.take<real>(N);
  w.S23 = k.take<real>(N);
  for (int i = 0; i < 6; i++) {
    w.ph[i] = k.take<real>(N);
    w.pd[i] = k.take<real>(N);
    w.Sh[i] = k.take<real>(N);
    w.Sd[i] = k.take<real>(N);
    w.SSh[i] = k.take<real>(N);
    w.SSd[i] = k.take<real>(N);
  }
  w.LM = k.take<real>(N);
  w.MM = k.take<real>(N);
  w.Th = k.take<real>(N);
  w.Td = k.take<real>(N);
  for (int i = 0; i < 3; i++) {
    w.uTh[i] = k.take<real>(N);
    w.uTd[i] = k.take<real>(N);
    w.Gh[i] = k.take<real>(N);
    w.Gd[i] = k.take<real>(N);
    w.SGh[i] = k.take<real>(N);
    w.SGd[i] = k.take<real>(N);
  }
  w.qx = k.take<real>(N);
  w.qy = k.take<real>(N);
  if (e.cfg.optMoisture >= 1) {
    w.Q = k.take<real>(N);
    w.RHSQ = k.take<real>(N);
    w.RHSQp = k.take<real>(N);
    for (int i = 0; i < 3; i++) w.gQ[i] = k.take<real>(N);
    w.Qadvs = k.take<real>(N);
    w.divqm = k.take<real>(N);
    w.qzq = k.take<real>(N);
    w.qm_plane = k.take<double>(H);
  }
  for (int i = 0; i < 10; i++) w.Pb[i] = k.take<real>(P);
  w.Lpad = k.take<real>((size_t)e.nx * e.my * nz);
  w.L2 = k.take<real>(2 * N);
  w.RCr = k.take<double>(R);
  w.RCi = k.take<double>(R);
  w.fRzr = k.take<double>(S);
  w.fRx = k.take<cd>(S);
  w.fRy = k.take<cd>(S);
  w.fRz = k.take<cd>(S);
  w.fp = k.take<cd>(S);
  w.fb2 = k.take<cd>((size_t)e.nx * e.nyh * 2);
  w.planes2 = k.take<real>(H * 2);
  for (int i = 0; i < 3; i++) w.dp[i] = k.take<real>(N);
  w.prof = k.take<double>(64 * nz + 64);
  w.d_cfl = k.take<double>(4);
  w.d_qavg = k.take<double>(4);
  w.d_it = k.take<int>(64);
  // engine scratch
  e.T_elems = (size_t)e.mx * e.myh * nz;
  for (int i = 0; i < 4; i++) e.T[i] = k.take<cd>(e.T_elems);
  e.red_elems = (size_t)1024 * 18 * nz + 1024;  // 1024 blocks x 18 sums (statistics' pass 1)
  e.red = k.take<double>(e.red_elems);
  e.scal = k.take<double>(64 * nz + 256);
  e.W_elems = N;
  e.W = k.take<real>(N);
  e.mat = k.take<real>(e.P());
  e.stat = k.take<double>((size_t)30 * nz + 64);
#ifdef ALFA_BUILD_FP32
  e.thomas_dm = k.take<double2>(e.S());  // the Thomas forward sweep stays FP64
#endif
}


Loader ld(const Engine& e, int kind, std::initializer_list<const real*> a, double c0, double c1,
          int sub) {
  Loader L{};
  L.kind = kind;
  L.sub = sub;
  L.nz = e.nz;
  int i = 0;
  for (const real* p : a) L.a[i++] = p;
  L.c[0] = c0;
  L.c[1] = c1;
  return L;
}

// Wong-Lilly base model (optSgs 2, 4) instead of Smagorinsky (0, 1, 3)
static bool wong_lilly(const Engine& e) { return e.cfg.optSgs == 2 || e.cfg.optSgs == 4; }
// scale-dependent procedures compute beta; the LAD variants (3, 4) set it to 1
static bool compute_beta_flag(const Engine& e) { return e.cfg.optSgs == 1 || e.cfg.optSgs == 2; }

// Derivxy(FFT(field)) with per-output accumulate flags
void deriv_field_acc(Engine& e, const Loader& L, real* dx, int accx, real* dy,
                            int accy) {
  op2_deriv(e, L, dx, accx, dy, accy);
}

// NSE_SGSTerms.py:55-105
void div_stress(Ctx* c, const real* txx, const real* tyy, const real* tzz,
                       const real* txy, const real* txz, const real* tyz, real* dtx,
                       real* dty, real* dtz) {
  Engine& e = c->e;
  deriv_field_acc(e, ld_field(e, txx), dtx, 0, nullptr, 0);
  deriv_field_acc(e, ld_field(e, txy), dty, 0, dtx, 1);
  deriv_field_acc(e, ld_field(e, tyy), nullptr, 0, dty, 1);
  deriv_field_acc(e, ld_field(e, txz), dtz, 0, nullptr, 0);
  deriv_field_acc(e, ld_field(e, tyz), nullptr, 0, dtz, 1);
  divergence_finish(e, dtx, txz, 1);
  divergence_finish(e, dty, tyz, 1);
  divergence_finish(e, dtz, tzz, 0);
}

// SCL_SGSTerms.py:55-89
void div_flux(Ctx* c, const real* qx, const real* qy, const real* qz,
                     real* divq) {
  Engine& e = c->e;
  deriv_field_acc(e, ld_field(e, qx), divq, 0, nullptr, 0);
  deriv_field_acc(e, ld_field(e, qy), nullptr, 0, divq, 1);
  divergence_finish(e, divq, qz, 1);
}

void advection(Ctx* c, const real* u, const real* v, const real* w,
                      const real* uy, const real* uz, const real* vx, const real* vz,
                      const real* wx, const real* wy, real* Cx, real* Cy, real* Cz) {
  Engine& e = c->e;
  real* const* Pb = c->w.Pb;
  if (!e.optDealias) {  // Advection_NoDealias, NSE_AdvectionTerms.py:163-238
    materialize(e, ld(e, LD_ADV_XY, {v, uy, vx, w, uz, wx}), e.N(), Cx);
    materialize(e, ld(e, LD_ADV_XY, {u, vx, uy, w, vz, wy}), e.N(), Cy);
    materialize(e, ld(e, LD_ADV_Z, {u, v, wx, uz, wy, vz}), e.N(), Cz);
    return;
  }
  const real* src[9] = {u, v, w, uy, uz, vx, vz, wx, wy};
  for (int i = 0; i < 9; i++) op2_pad(e, ld_field(e, src[i]), Pb[i], c->w.Lpad);
  // Pb: 0 up 1 vp 2 wp 3 uy 4 uz 5 vx 6 vz 7 wx 8 wy
  op2_unpad(e, ld(e, LD_ADV_XY, {Pb[1], Pb[3], Pb[5], Pb[2], Pb[4], Pb[7]}), Cx, c->w.Lpad);
  op2_unpad(e, ld(e, LD_ADV_XY, {Pb[0], Pb[5], Pb[3], Pb[2], Pb[6], Pb[8]}), Cy, c->w.Lpad);
  op2_unpad(e, ld(e, LD_ADV_Z, {Pb[0], Pb[1], Pb[7], Pb[4], Pb[8], Pb[6]}), Cz, c->w.Lpad);
}

// SCL_AdvectionTerms.py:57-106; reuse_uvw: Pb[0..2] already hold the padded
// u, v, w of this step (the reference recomputes the identical values)
void scalar_advection(Ctx* c, const real* u, const real* v, const real* w,
                             const real* sx, const real* sy, const real* sz, real* out,
                             bool reuse_uvw) {
  Engine& e = c->e;
  real* const* Pb = c->w.Pb;
  if (!e.optDealias) {  // SCL_AdvectionTerms.py:114-150
    materialize(e, ld(e, LD_SCALAR_ADV, {u, v, w, sx, sy, sz}), e.N(), out);
    return;
  }
  if (!reuse_uvw) {
    op2_pad(e, ld_field(e, u), Pb[0], c->w.Lpad);
    op2_pad(e, ld_field(e, v), Pb[1], c->w.Lpad);
    op2_pad(e, ld_field(e, w), Pb[2], c->w.Lpad);
  }
  op2_pad(e, ld_field(e, sx), Pb[3], c->w.Lpad);
  op2_pad(e, ld_field(e, sy), Pb[4], c->w.Lpad);
  op2_pad(e, ld_field(e, sz), Pb[5], c->w.Lpad);
  op2_unpad(e, ld(e, LD_SCALAR_ADV, {Pb[0], Pb[1], Pb[2], Pb[3], Pb[4], Pb[5]}), out, c->w.Lpad);
}

// Stresses of StressesUVPnodes_Dealias / StressesWnodes_Dealias from the
// strains (uvp padded components in Pb[0..3], |S|_pad), Cs2_pad in Pb[9];
// then the w-node strains are padded into Pb[0..5].
static void sgs_stresses(Ctx* c, const real* const g[9], const real* S_uvp_pad,
                         const real* u, const real* v, const double* M, const double* pm,
                         const double* pm0, real* const t6[6], real* S_w, real* S_w_pad) {
  Engine& e = c->e;
  real* const* Pb = c->w.Pb;
  const bool wl = wong_lilly(e);
  const double cst = -2 * std::pow(e.L, 2.0);
  const double cwl = -2 * std::pow(e.L, 4.0 / 3.0);  // SGSStresses_WL.py:90
  for (int i = 0; i < 4; i++)
    op2_unpad(e, wl ? ld(e, LD_WL_UVP, {Pb[9], Pb[i]}, cwl)
                    : ld(e, LD_STRESS_UVP, {Pb[9], S_uvp_pad, Pb[i]}, cst),
              t6[i], c->w.Lpad);
  Loader Lw = ld(e, LD_W_SXX, {g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8]});
  for (int s = 0; s < 6; s++) {
    Lw.sub = s;
    op2_pad(e, Lw, Pb[s], c->w.Lpad);
  }
  smag_w(e, g, S_w);
  const real* q6[6] = {Pb[0], Pb[1], Pb[2], Pb[3], Pb[4], Pb[5]};
  smag6(e, q6, e.P(), S_w_pad);
  for (int i = 4; i < 6; i++)
    op2_unpad(e, wl ? ld(e, LD_WL_W, {Pb[9], Pb[i]}, cwl)
                    : ld(e, LD_STRESS_W, {Pb[9], S_w_pad, Pb[i]}, cst),
              t6[i], c->w.Lpad);
  wall_override(e, u, v, M, pm, pm0, t6[4], t6[5]);
}

// StressesUVPnodes_NoDealias / StrainsWnodes_NoDealias / StressesWnodes_NoDealias
// (SGSStresses_SM.py:149-178, :251-290; StrainRates.py:307-368): the same
// products in physical space; S_w_pad receives S_w.
static void sgs_stresses_nodealias(Ctx* c, const real* const g[9], const real* Sij[6],
                                   const real* S_uvp, const real* Cs2, const real* u,
                                   const real* v, const double* M, const double* pm,
                                   const double* pm0, real* const t6[6], real* S_w,
                                   real* S_w_pad) {
  Engine& e = c->e;
  real* const* Pb = c->w.Pb;
  const bool wl = wong_lilly(e);
  const double cst = -2 * std::pow(e.L, 2.0);
  const double cwl = -2 * std::pow(e.L, 4.0 / 3.0);
  for (int i = 0; i < 4; i++)
    materialize(e, wl ? ld(e, LD_WL_UVP, {Cs2, Sij[i]}, cwl)
                      : ld(e, LD_STRESS_UVP, {Cs2, S_uvp, Sij[i]}, cst),
                e.N(), t6[i]);
  Loader Lw = ld(e, LD_W_SXX, {g[0], g[1], g[2], g[3], g[4], g[5], g[6], g[7], g[8]});
  Lw.sub = 4;
  materialize(e, Lw, e.N(), Pb[0]);  // S13 on w nodes
  Lw.sub = 5;
  materialize(e, Lw, e.N(), Pb[1]);  // S23 on w nodes
  smag_w(e, g, S_w);
  cudaMemcpyAsync(S_w_pad, S_w, e.N() * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
  for (int i = 0; i < 2; i++)
    materialize(e, wl ? ld(e, LD_WL_W, {Cs2, Pb[i]}, cwl)
                      : ld(e, LD_STRESS_W, {Cs2, S_w, Pb[i]}, cst),
                e.N(), t6[4 + i]);
  wall_override(e, u, v, M, pm, pm0, t6[4], t6[5]);
}

// uvp strains + their padded copies: S11..S33 alias dudx, dvdy, dwdz.
static void uvp_strains_padded(Ctx* c, const real* const g[9], const real* Sij[6],
                               real* S_uvp, real* S_uvp_pad) {
  Engine& e = c->e;
  Work& w = c->w;
  strains_uvp(e, g, w.S12, w.S13, w.S23, S_uvp);
  Sij[0] = g[0];
  Sij[1] = g[4];
  Sij[2] = g[8];
  Sij[3] = w.S12;
  Sij[4] = w.S13;
  Sij[5] = w.S23;
  if (!e.optDealias) {  // StrainsUVPnodes_NoDealias: S_uvp_pad is S_uvp
    cudaMemcpyAsync(S_uvp_pad, S_uvp, e.N() * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
    return;
  }
  for (int i = 0; i < 6; i++) op2_pad(e, ld_field(e, Sij[i]), w.Pb[i], c->w.Lpad);
  const real* p6[6] = {w.Pb[0], w.Pb[1], w.Pb[2], w.Pb[3], w.Pb[4], w.Pb[5]};
  smag6(e, p6, e.P(), S_uvp_pad);
}

__global__ void k_ones_ext(double* p, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 1.0;
}

// DynamicSGS (DynamicSGS_Main.py:85-331, SM, dealiased) + DivStress.
// mom: 25 slots as in alfa.h (6..9 unused here)
int dynamic_sgs(Ctx* c, const real* const g[9], const real* u, const real* v,
                       const real* w, const double* M, const double* pm, const double* pm0,
                       real* divt[3], double* avg1, double* avg2, double* beta1,
                       real* Cs2, real* const mom[25]) {
  Engine& e = c->e;
  Work& W = c->w;
  const real* Sij[6];
  real* S_uvp = mom[19];
  uvp_strains_padded(c, g, Sij, S_uvp, mom[20]);
  // LASDD (DynamicSGS_LASDD_SM.py:178-367)
  real *u_ = mom[10], *v_ = mom[11], *w_ = mom[12];
  if (u_ != u) cudaMemcpyAsync(u_, u, e.N() * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
  if (v_ != v) cudaMemcpyAsync(v_, v, e.N() * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
  wstar(e, w, w_);
  op_filter12(e, ld_field(e, u_), mom[13], mom[16]);
  op_filter12(e, ld_field(e, v_), mom[14], mom[17]);
  op_filter12(e, ld_field(e, w_), mom[15], mom[18]);
  const real* pa[6] = {u_, v_, w_, u_, u_, v_};
  const real* pb[6] = {u_, v_, w_, v_, w_, w_};
  for (int i = 0; i < 6; i++) op_filter12(e, ld(e, LD_MUL, {pa[i], pb[i]}), W.ph[i], W.pd[i]);
  for (int i = 0; i < 6; i++) op_filter12(e, ld_field(e, Sij[i]), W.Sh[i], W.Sd[i]);
  const bool wl = wong_lilly(e);
  if (!wl)  // the Wong-Lilly procedure has no S|S_ij| products
    for (int i = 0; i < 6; i++)
      op_filter12(e, ld(e, LD_MUL, {S_uvp, Sij[i]}), W.SSh[i], W.SSd[i]);
  const real* sh6[6] = {W.Sh[0], W.Sh[1], W.Sh[2], W.Sh[3], W.Sh[4], W.Sh[5]};
  const real* sd6[6] = {W.Sd[0], W.Sd[1], W.Sd[2], W.Sd[3], W.Sd[4], W.Sd[5]};
  smag6_n(e, sh6, mom[23]);
  smag6_n(e, sd6, mom[24]);
  LasddFields f;
  for (int i = 0; i < 3; i++) {
    f.hat[i] = mom[13 + i];
    f.hatd[i] = mom[16 + i];
  }
  for (int i = 0; i < 6; i++) {
    f.ph[i] = W.ph[i];
    f.pd[i] = W.pd[i];
    f.Sh[i] = W.Sh[i];
    f.Sd[i] = W.Sd[i];
    f.SSh[i] = W.SSh[i];
    f.SSd[i] = W.SSd[i];
  }
  f.S_hat = mom[23];
  f.S_hatd = mom[24];
  double* sums = W.prof;
  double* co = W.prof + 10 * e.nz;
  if (compute_beta_flag(e)) {
    if (wl) {  // DynamicSGS_LASDD_WL.py:245-284
      lasdd_wl_sums(e, f, sums);
      wl_poly(e, sums, co);
    } else {
      lasdd_sums(e, f, sums);
      lasdd_poly(e, sums, 0, co);
    }
    compute_beta(e, co, e.nz, beta1);
  } else {
    ::alfa::note_launch(); k_ones_ext<<<1, 256, 0, e.stream>>>(beta1, e.nz);  // LAD: beta = 1 (:321-325)
  }
  if (wl)
    lasdd_wl_LM_MM(e, f, beta1, W.LM, W.MM);
  else
    lasdd_LM_MM(e, f, beta1, W.LM, W.MM);
  clip_ratio(e, W.LM, W.MM, Cs2);
  cs2_profiles(e, Cs2, avg1, avg2);
  // stresses (SGSStresses_SM.py) with Cs2_3D_pad = Dealias1(FFT(Cs2_3D))
  real* t6[6] = {mom[0], mom[1], mom[2], mom[3], mom[4], mom[5]};
  if (e.optDealias) {
    op2_pad(e, ld_field(e, Cs2), W.Pb[9], c->w.Lpad);
    sgs_stresses(c, g, mom[20], u, v, M, pm, pm0, t6, mom[21], mom[22]);
  } else {
    sgs_stresses_nodealias(c, g, Sij, S_uvp, Cs2, u, v, M, pm, pm0, t6, mom[21], mom[22]);
  }
  div_stress(c, mom[0], mom[1], mom[2], mom[3], mom[4], mom[5], divt[0], divt[1], divt[2]);
  return check_launch(e, "DivStressDynamicSGS");
}

// StaticSGS (StaticSGS_Main.py:76-250) + DivStress; mom10 as in alfa.h
int static_sgs(Ctx* c, const real* const g[9], const real* Cs2, const real* u,
                      const real* v, const double* M, const double* pm, const double* pm0,
                      real* divt[3], real* const mom10[10]) {
  Engine& e = c->e;
  Work& W = c->w;
  const real* Sij[6];
  uvp_strains_padded(c, g, Sij, mom10[6], mom10[7]);
  real* t6[6] = {mom10[0], mom10[1], mom10[2], mom10[3], mom10[4], mom10[5]};
  if (e.optDealias) {
    op2_pad(e, ld_field(e, Cs2), W.Pb[9], c->w.Lpad);
    sgs_stresses(c, g, mom10[7], u, v, M, pm, pm0, t6, mom10[8], mom10[9]);
  } else {
    sgs_stresses_nodealias(c, g, Sij, mom10[6], Cs2, u, v, M, pm, pm0, t6, mom10[8], mom10[9]);
  }
  div_stress(c, mom10[0], mom10[1], mom10[2], mom10[3], mom10[4], mom10[5], divt[0], divt[1],
             divt[2]);
  return check_launch(e, "DivStressStaticSGS");
}

// StaticSGSscalar (StaticSGS_Main.py:258-360, dealiased SM) + DivFlux
void scalar_fluxes(Ctx* c, const real* S_uvp_pad, const real* S_w_pad,
                          const real* r3, const real* gx, const real* gy, const real* gz,
                          const double* qz_sfc, real* qz, real* divq) {
  Engine& e = c->e;
  Work& W = c->w;
  const double cst = -2 * std::pow(e.L, 2.0);
  const bool wl = wong_lilly(e);
  const double cwl = -std::pow(e.L, 4.0 / 3.0);  // ScalarSGSFluxes_WL.py:76
  if (!e.optDealias) {  // ScalarFluxes*_NoDealias (ScalarSGSFluxes_SM.py:98-126, :185-222)
    materialize(e, wl ? ld(e, LD_WL_UVP, {r3, gx}, cwl) : ld(e, LD_STRESS_UVP, {r3, S_uvp_pad, gx}, cst),
                e.N(), W.qx);
    materialize(e, wl ? ld(e, LD_WL_UVP, {r3, gy}, cwl) : ld(e, LD_STRESS_UVP, {r3, S_uvp_pad, gy}, cst),
                e.N(), W.qy);
    materialize(e, wl ? ld(e, LD_WL_W, {r3, gz}, cwl) : ld(e, LD_STRESS_W, {r3, S_w_pad, gz}, cst),
                e.N(), qz);
    set_plane0(e, qz_sfc, qz);
    div_flux(c, W.qx, W.qy, qz, divq);
    return;
  }
  op2_pad(e, ld_field(e, gx), W.Pb[0], c->w.Lpad);
  op2_pad(e, ld_field(e, gy), W.Pb[1], c->w.Lpad);
  op2_pad(e, ld_field(e, gz), W.Pb[2], c->w.Lpad);
  op2_pad(e, ld_field(e, r3), W.Pb[3], c->w.Lpad);
  op2_unpad(e, wl ? ld(e, LD_WL_UVP, {W.Pb[3], W.Pb[0]}, cwl)
                  : ld(e, LD_STRESS_UVP, {W.Pb[3], S_uvp_pad, W.Pb[0]}, cst),
            W.qx, c->w.Lpad);
  op2_unpad(e, wl ? ld(e, LD_WL_UVP, {W.Pb[3], W.Pb[1]}, cwl)
                  : ld(e, LD_STRESS_UVP, {W.Pb[3], S_uvp_pad, W.Pb[1]}, cst),
            W.qy, c->w.Lpad);
  op2_unpad(e, wl ? ld(e, LD_WL_W, {W.Pb[3], W.Pb[2]}, cwl)
                  : ld(e, LD_STRESS_W, {W.Pb[3], S_w_pad, W.Pb[2]}, cst),
            qz, c->w.Lpad);
  set_plane0(e, qz_sfc, qz);
  div_flux(c, W.qx, W.qy, qz, divq);
}

// DynamicSGSscalar (DynamicSGS_Main.py:339-478) + DivFlux; m15 = mom[10..24]
int dynamic_sgs_scalar(Ctx* c, const real* const m15[15], const real* TH,
                              const real* gx, const real* gy, const real* gz,
                              const double* qz_sfc, real* qz, real* divq, real* r3,
                              double* r1, double* beta2) {
  Engine& e = c->e;
  Work& W = c->w;
  const real *u_ = m15[0], *v_ = m15[1], *w_ = m15[2];
  const real* S = m15[9];
  op_filter12(e, ld_field(e, TH), W.Th, W.Td);
  const real* uv3[3] = {u_, v_, w_};
  for (int i = 0; i < 3; i++) op_filter12(e, ld(e, LD_MUL, {uv3[i], TH}), W.uTh[i], W.uTd[i]);
  op_filter12(e, ld_field(e, gx), W.Gh[0], W.Gd[0]);
  op_filter12(e, ld_field(e, gy), W.Gh[1], W.Gd[1]);
  op_filter12(e, ld(e, LD_THZ, {gz}), W.Gh[2], W.Gd[2]);
  const bool wl = wong_lilly(e);
  if (!wl) {  // the Wong-Lilly procedure has no |S| grad(theta) products
    op_filter12(e, ld(e, LD_MUL, {S, gx}), W.SGh[0], W.SGd[0]);
    op_filter12(e, ld(e, LD_MUL, {S, gy}), W.SGh[1], W.SGd[1]);
    op_filter12(e, ld(e, LD_MUL_THZ, {S, gz}), W.SGh[2], W.SGd[2]);
  }
  ScalarLasddFields f;
  for (int i = 0; i < 3; i++) {
    f.hat[i] = m15[3 + i];
    f.hatd[i] = m15[6 + i];
    f.uTh[i] = W.uTh[i];
    f.uTd[i] = W.uTd[i];
    f.Gh[i] = W.Gh[i];
    f.Gd[i] = W.Gd[i];
    f.SGh[i] = W.SGh[i];
    f.SGd[i] = W.SGd[i];
  }
  f.Th = W.Th;
  f.Td = W.Td;
  f.S_hat = m15[13];
  f.S_hatd = m15[14];
  double* sums = W.prof;
  double* co = W.prof + 10 * e.nz;
  if (compute_beta_flag(e)) {
    if (wl) {  // DynamicSGS_ScalarLASDD_WL.py:214-252
      scalar_lasdd_wl_sums(e, f, sums);
      wl_poly(e, sums, co);
    } else {
      scalar_lasdd_sums(e, f, sums);
      lasdd_poly(e, sums, 1, co);
    }
    compute_beta(e, co, e.nz, beta2);
  } else {
    ::alfa::note_launch(); k_ones_ext<<<1, 256, 0, e.stream>>>(beta2, e.nz);
  }
  if (wl)
    scalar_wl_Tup_Tdn(e, f, beta2, W.LM, W.MM);
  else
    scalar_Tup_Tdn(e, f, beta2, W.LM, W.MM);
  clip_ratio(e, W.LM, W.MM, r3);
  const real* fr[1] = {r3};
  plane_means(e, fr, 1, r1);
  scalar_fluxes(c, m15[10], m15[12], r3, gx, gy, gz, qz_sfc, qz, divq);
  return check_launch(e, "DivFluxDynamicSGS");
}

// PressureRC (NSE_PressureTerms.py:109-182)
int pressure_rc_fn(Ctx* c, const real* u, const real* v, const real* w,
                          const real* Ru, const real* Rv, const real* Rw, const real* Rup,
                          const real* Rvp, const real* Rwp, const real* divtz, double* RCr,
                          double* RCi, double* fRzr) {
  Engine& e = c->e;
  Work& W = c->w;
  const double c0 = 1.0 / 3.0, c1 = 2.0 / (3.0 * e.dt_nondim);
  op_rfft2(e, ld(e, LD_PRESSURE_R, {Ru, Rup, u}, c0, c1), W.fRx);
  op_rfft2(e, ld(e, LD_PRESSURE_R, {Rv, Rvp, v}, c0, c1), W.fRy);
  op_rfft2(e, ld(e, LD_PRESSURE_R, {Rw, Rwp, w}, c0, c1), W.fRz);
  // rfft2 of the bottom and top planes of divtz, as a 2-level field
  copy_planes_z(e, divtz, 0, e.nz - 1, W.planes2);
  const int nz = e.nz;
  e.nz = 2;
  Loader L2 = ld_field(e, W.planes2);
  op_rfft2(e, L2, W.fb2);
  e.nz = nz;
  pressure_rc(e, W.fRx, W.fRy, W.fRz, W.fb2, nullptr, RCr, RCi, fRzr);
  return check_launch(e, "PressureRC");
}

// ThomasPressureSolve (NSE_PressureTerms_Thomas.py:218-292)
int pressure_solve_fn(Ctx* c, const double* RCr, const double* RCi, const double* fRzr, real* p,
                      real* dpdx, real* dpdy, real* dpdz) {
  Engine& e = c->e;
  Work& W = c->w;
  thomas_solve(e, RCr, RCi, fRzr, W.fp);
  op_irfft2(e, W.fp, p);
  deriv_field_acc(e, ld_field(e, p), dpdx, 0, dpdy, 0);
  derivz_generic(e, p, 0, dpdz);
  return check_launch(e, "ThomasPressureSolve");
}

static int surface_variant(const alfa_config& c) {
  if (c.optSurfBC == 0) return c.optSurfFlux == 0 ? 0 : 1;
  if (c.optSurfBC == 1) return c.optSurfFlux == 0 ? 2 : 3;
  return c.optSurfFlux == 0 ? 4 : 5;
}

// ---------------------------------------------------------------------------
// whole step: src/Main.py:156-541 (dry, constant geostrophic wind)
// ---------------------------------------------------------------------------
__global__ void k_add_int(int* p, int d) { *p += d; }
__global__ void k_set_int(int* p, int v) { *p = v; }

// sgs_mode: 0 the reference's rule (dynamic on the call interval), 1 learned
// (the attached network's Cs^2 with the static stresses), 2 dynamic
static int one_step(Ctx* c, int sgs_mode = 0);


static int one_step(Ctx* c, int sgs_mode) {
  Engine& e = c->e;
  Work& W = c->w;
  const alfa_config& cf = e.cfg;
  const int it = W.iteration;
  const int nz = e.nz;
  const bool moist = cf.optMoisture >= 1;
  if (moist && !W.have_q)
    return e.fail("optMoisture = 1 needs alfa_init_moisture before stepping", ALFA_E_STATE);
  if (moist && cf.optMoistureSurfBC >= 1 && it - 1 >= W.msfc_rows)
    return e.fail("moisture surface series exhausted", ALFA_E_STATE);
  if (it > cf.istep) {
    for (int i = 0; i < 4; i++) std::swap(W.RHSp[i], W.RHS[i]);
    if (moist) std::swap(W.RHSQp, W.RHSQ);
  }
  // Qadv rows (Main.py:186-188): zero unless a Qadv series was given
  const double* Qadvp = W.zero_prof;
  const int* qtp = nullptr;
  if (moist && cf.optAdvection >= 1 && W.series_q) {
    if (it - 1 >= W.q_rows) return e.fail("moisture advection series exhausted", ALFA_E_STATE);
    Qadvp = W.series_q;
    qtp = W.d_it;
  }
  // forcing rows (Main.py:179-188) are selected on the device from the
  // device iteration counter, so a captured step replays with the current row
  const double *Uadv = W.zero_prof, *Vadv = W.zero_prof, *THadv = W.zero_prof;
  const int* itp = nullptr;
  // geostrophic wind rows (Main.py:170-174), selected the same way
  const double *Ugp = W.Ug, *Vgp = W.Vg;
  const int* gtp = nullptr;
  if (cf.optGeoWind >= 1) {
    if (it - 1 >= W.geo_rows) return e.fail("geostrophic wind series exhausted", ALFA_E_STATE);
    Ugp = W.series_geo;
    Vgp = W.series_geo + nz;
    gtp = W.d_it;
  }
  if (cf.optAdvection >= 1) {
    if (it - 1 >= W.series_rows) return e.fail("advection series exhausted", ALFA_E_STATE);
    Uadv = W.series_adv;
    Vadv = W.series_adv + nz;
    THadv = W.series_adv + 2 * nz;
    itp = W.d_it;
  }
  // filtering (Main.py:193-197): the filtered field replaces the state, so
  // filter into the (not yet used) gradient slot and swap the two N-sized
  // buffers; the TH spectrum is discarded as in the reference.
  // The x and y derivatives of the filtered fields (velocityGradients,
  // potentialTemperatureGradients: Derivxy of the filtered spectrum) come
  // out of the same separable passes.  Filtered fields land in buffers
  // that are free until advection, then swap with the state.
  op2_filter_deriv(e, ld_field(e, W.u), W.Cx, W.g[0], W.g[3], W.L2);
  std::swap(W.u, W.Cx);
  op2_filter_deriv(e, ld_field(e, W.v), W.Cy, W.g[1], W.g[4], W.L2);
  std::swap(W.v, W.Cy);
  op2_filter_deriv(e, ld_field(e, W.w), W.Cz, W.g[2], W.g[5], W.L2);
  std::swap(W.w, W.Cz);
  op2_filter_deriv(e, ld_field(e, W.TH), W.THadv, W.gT[0], W.gT[1], W.L2);
  std::swap(W.TH, W.THadv);
  if (moist) {  // Main.py:198-199; moistureGradients' Derivxy from the same passes
    op2_filter_deriv(e, ld_field(e, W.Q), W.Qadvs, W.gQ[0], W.gQ[1], W.L2);
    std::swap(W.Q, W.Qadvs);
  }
  // surface fluxes (Main.py:213-243)
  const int var = surface_variant(cf);
  double sfc = 0.0;
  if (cf.optSurfBC >= 1) {
    if (it - 1 >= (int)W.sfc_series.size()) return e.fail("surface series exhausted", ALFA_E_STATE);
    sfc = W.sfc_series[it - 1];
  }
  const double* sfc_dev = (cf.optSurfBC >= 1) ? W.d_sfc : nullptr;
  SurfaceIO io;
  io.u = W.u;
  io.v = W.v;
  io.TH = W.TH;
  for (int i = 0; i < 6; i++) {
    io.most_in[i] = W.most[i];
    io.most_out[i] = W.most_new[i];
  }
  io.M = W.M;
  io.ustar = W.ustar;
  io.q2 = W.q2;
  io.qavg = W.d_qavg;
  io.invOB = W.invOB;
  surface_flux(e, var, sfc, io, sfc_dev, W.d_it);
  for (int i = 0; i < 6; i++) std::swap(W.most[i], W.most_new[i]);
  const double* qz_step = (var <= 1) ? W.qz_plane : W.q2;
  // surface moisture flux (Main.py:253-267): a constant plane (filled by
  // alfa_init_moisture), the series value, or from the prescribed humidity
  // with this step's ustar and psi functions
  if (moist && cf.optMoistureSurfBC >= 1) {
    const double* qbar0 = nullptr;
    if (cf.optMoistureSurfBC == 2 && cf.optSurfFlux == 0) {
      const real* f1[1] = {W.Q};
      plane_means(e, f1, 1, W.prof + 36 * nz);
      qbar0 = W.prof + 36 * nz;
    }
    moisture_surface(e, cf.optMoistureSurfBC, cf.optSurfFlux != 0, W.Q, W.ustar, W.most[2],
                     W.most[3], W.d_msfc, W.d_it, 0.0, qbar0, W.qm_plane);
  }
  // gradients (Main.py:275-290)
  derivz_M(e, W.u, W.v, W.w, W.ustar, W.M, W.most[4], W.g[6], W.g[7], W.g[8]);
  derivz_TH(e, W.TH, W.ustar, qz_step, W.most[5], W.gT[2]);
  if (moist) derivz_TH(e, W.Q, W.ustar, W.qm_plane, W.most[5], W.gQ[2]);  // Derivatives.py:304
  // advection (Main.py:301-311)
  advection(c, W.u, W.v, W.w, W.g[3], W.g[6], W.g[1], W.g[7], W.g[2], W.g[5], W.Cx, W.Cy, W.Cz);
  scalar_advection(c, W.u, W.v, W.w, W.gT[0], W.gT[1], W.gT[2], W.THadv, true);
  if (moist) scalar_advection(c, W.u, W.v, W.w, W.gQ[0], W.gQ[1], W.gQ[2], W.Qadvs, true);
  // buoyancy (Main.py:323-327), H = Q when moist
  buoyancy(e, W.TH, moist ? W.Q : nullptr, cf.optBuoyancy == 0 ? 0 : 1, W.buoy);
  // SGS (Main.py:333-455)
  const real* g9[9] = {W.g[0], W.g[1], W.g[2], W.g[3], W.g[4], W.g[5], W.g[6], W.g[7], W.g[8]};
  bool dyn = (cf.optSgs >= 1 && cf.optSgs <= 4) &&
             (it == cf.istep || it % cf.dynamicSGS_call_time == 0);
  if (sgs_mode == 1) dyn = false;
  if (sgs_mode == 2) dyn = true;
  W.last_dyn = dyn ? 1 : 0;
  if (sgs_mode == 1) {  // the network replaces the procedure
    if (!c->learned) return e.fail("learned step without an attached network", ALFA_E_STATE);
    c->learned(W.Cs2);
  }
  int st;
  if (dyn) {
    real* mom[25];
    for (int i = 0; i < 25; i++) mom[i] = W.mom[i];
    mom[10] = W.u;  // u_ = u.copy(), v_ = v.copy(): aliases (never written)
    mom[11] = W.v;
    double* beta1 = W.prof + 20 * nz;
    st = dynamic_sgs(c, g9, W.u, W.v, W.w, W.M, W.most[0], W.most[1], W.divt, W.prof + 21 * nz,
                     W.prof + 22 * nz, beta1, W.Cs2, mom);
    if (st) return st;
    const real* m15[15];
    for (int i = 0; i < 15; i++) m15[i] = mom[10 + i];
    st = dynamic_sgs_scalar(c, m15, W.TH, W.gT[0], W.gT[1], W.gT[2], qz_step, W.qz, W.divq,
                            W.Cs2Pr, W.prof + 23 * nz, W.prof + 24 * nz);
    if (st) return st;
    // moisture: the static scalar flux with heat's new Cs2PrRatio and the
    // strains dynamicSGSmomentum[19:23] (Main.py:358-369)
    if (moist)
      scalar_fluxes(c, mom[20], mom[22], W.Cs2Pr, W.gQ[0], W.gQ[1], W.gQ[2], W.qm_plane, W.qzq,
                    W.divqm);
  } else {
    real* m10[10] = {W.mom[0], W.mom[1], W.mom[2], W.mom[3], W.mom[4],
                       W.mom[5], W.mom[19], W.mom[20], W.mom[21], W.mom[22]};
    st = static_sgs(c, g9, W.Cs2, W.u, W.v, W.M, W.most[0], W.most[1], W.divt, m10);
    if (st) return st;
    scalar_fluxes(c, m10[7], m10[9], W.Cs2Pr, W.gT[0], W.gT[1], W.gT[2], qz_step, W.qz, W.divq);
    if (moist)  // Main.py:444-453
      scalar_fluxes(c, m10[7], m10[9], W.Cs2Pr, W.gQ[0], W.gQ[1], W.gQ[2], W.qm_plane, W.qzq,
                    W.divqm);
  }
  // RHS (Main.py:464-473)
  double* bars = W.prof + 30 * nz;
  if (cf.optDamping == 1) {
    const real* f4[4] = {W.u, W.v, W.TH, W.Q};
    plane_means(e, f4, moist ? 4 : 3, bars);
  }
  rhs_momentum(e, W.u, W.v, W.w, Ugp, Vgp, W.Cx, W.Cy, W.Cz, W.buoy, W.divt[0], W.divt[1],
               W.divt[2], Uadv, Vadv, bars, bars + nz, W.RHS[0], W.RHS[1], W.RHS[2], itp,
               3LL * nz, gtp, 2LL * nz);
  rhs_scalar(e, W.TH, W.THadv, W.divq, THadv, bars + 2 * nz, W.RHS[3], itp, 3LL * nz);
  if (moist)  // RHS_Moisture (SCL_AllTerms.py:86-110)
    rhs_scalar(e, W.Q, W.Qadvs, W.divqm, Qadvp, bars + 3 * nz, W.RHSQ, qtp, nz, 1);
  // pressure (Main.py:481-500)
  st = pressure_rc_fn(c, W.u, W.v, W.w, W.RHS[0], W.RHS[1], W.RHS[2], W.RHSp[0], W.RHSp[1],
                      W.RHSp[2], W.divt[2], W.RCr, W.RCi, W.fRzr);
  if (st) return st;
  st = pressure_solve_fn(c, W.RCr, W.RCi, W.fRzr, W.p, W.dp[0], W.dp[1], W.dp[2]);
  if (st) return st;
  subtract3(e, W.RHS[0], W.RHS[1], W.RHS[2], W.dp[0], W.dp[1], W.dp[2]);
  // AB2 bootstrap and advance (Main.py:506-526)
  const real* Rp[4];
  for (int i = 0; i < 4; i++) Rp[i] = (it == cf.istep) ? W.RHS[i] : W.RHSp[i];
  ab2_uvw(e, W.u, W.v, W.w, W.RHS[0], Rp[0], W.RHS[1], Rp[1], W.RHS[2], Rp[2], W.u, W.v, W.w);
  ab2_th(e, W.TH, W.RHS[3], Rp[3], W.TH);
  if (moist) ab2_q(e, W.Q, W.RHSQ, (it == cf.istep) ? W.RHSQ : W.RHSQp, W.Q);
  if (it == cf.istep) {
    for (int i = 0; i < 4; i++)
      cudaMemcpyAsync(W.RHSp[i], W.RHS[i], e.N() * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
    if (moist)
      cudaMemcpyAsync(W.RHSQp, W.RHSQ, e.N() * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
  }
  // CFL (Main.py:534-540): maxima stay on the device, read by alfa_get_diag
  cfl_max(e, W.u, W.v, W.w, W.d_cfl);
  ::alfa::note_launch(); k_add_int<<<1, 1, 0, e.stream>>>(W.d_it, 1);
  W.iteration++;
  return check_launch(e, "step");
}


void release_graphs(Ctx* c) {
  for (StepGraph& g : c->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
  }
}

// One step as a CUDA graph.  The step's launches depend on the host only
// through (a) the buffer pointers, which alternate with the iteration's
// parity, and (b) whether the dynamic SGS procedure runs; the forcing rows
// and the surface value are read on the device from the device iteration
// counter.  So one graph per (parity, dynamic) pair, captured the first time
// it is needed, replays every later step of that kind.  The bootstrap step
// (iteration == istep) runs directly.
static int graph_step(Ctx* c) {
  Engine& e = c->e;
  Work& W = c->w;
  const alfa_config& cf = e.cfg;
  const int it = W.iteration;
  if (it == cf.istep) return one_step(c);
  if (cf.optAdvection >= 1 && it - 1 >= W.series_rows)
    return e.fail("advection series exhausted", ALFA_E_STATE);
  if (cf.optGeoWind >= 1 && it - 1 >= W.geo_rows)
    return e.fail("geostrophic wind series exhausted", ALFA_E_STATE);
  if (cf.optMoisture >= 1 && !W.have_q)
    return e.fail("optMoisture = 1 needs alfa_init_moisture before stepping", ALFA_E_STATE);
  if (cf.optMoisture >= 1 && cf.optMoistureSurfBC >= 1 && it - 1 >= W.msfc_rows)
    return e.fail("moisture surface series exhausted", ALFA_E_STATE);
  if (cf.optMoisture >= 1 && cf.optAdvection >= 1 && W.series_q && it - 1 >= W.q_rows)
    return e.fail("moisture advection series exhausted", ALFA_E_STATE);
  if (cf.optSurfBC >= 1 && it - 1 >= (int)W.sfc_series.size())
    return e.fail("surface series exhausted", ALFA_E_STATE);
  const bool dyn = (cf.optSgs >= 1 && cf.optSgs <= 4) && (it % cf.dynamicSGS_call_time == 0);
  StepGraph& g = c->graphs[(it & 1) * 2 + (dyn ? 1 : 0)];
  const StepPtrs now = StepPtrs::of(W);
  if (!g.exec || !(g.before == now)) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    if (e.stream == 0) return e.fail("graph capture needs a non-default stream", ALFA_E_STATE);
    if (cudaStreamBeginCapture(e.stream, cudaStreamCaptureModeRelaxed) != cudaSuccess)
      return e.fail("cudaStreamBeginCapture failed", ALFA_E_CUDA);
    const unsigned long long l0 = ::alfa::launch_count();
    const int st = one_step(c);
    // capturing counted the step's kernels once; the launch below runs them
    g.kernels = ::alfa::launch_count() - l0;
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e.stream, &graph);
    const StepPtrs after = StepPtrs::of(W);
    now.apply(W);  // nothing ran yet: undo the host side of the captured step
    W.iteration = it;
    if (st || ce != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return st ? st : e.fail("step capture failed", ALFA_E_CUDA);
    }
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      g.exec = nullptr;
      return e.fail("step graph instantiation failed", ALFA_E_CUDA);
    }
    g.before = now;
    g.after = after;
  } else {
    ::alfa::add_launches(g.kernels);  // replayed kernels
  }
  if (cudaGraphLaunch(g.exec, e.stream) != cudaSuccess)
    return e.fail("step graph launch failed", ALFA_E_CUDA);
  g.after.apply(W);
  W.iteration = it + 1;
  return ALFA_OK;
}


// copy n values between an FP64 buffer and a field of the build's precision
template <class S, class D>
__global__ void k_convert(const S* __restrict__ s, D* __restrict__ d, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    d[i] = (D)s[i];
}

static void to_real(Engine& e, const double* s, real* d, size_t n) {
#ifdef ALFA_BUILD_FP32
  ::alfa::note_launch();
  k_convert<double, real><<<4 * e.sms, 256, 0, e.stream>>>(s, d, n);
#else
  cudaMemcpyAsync(d, s, n * sizeof(double), cudaMemcpyDeviceToDevice, e.stream);
#endif
}

static void to_double(Engine& e, const real* s, double* d, size_t n) {
#ifdef ALFA_BUILD_FP32
  ::alfa::note_launch();
  k_convert<real, double><<<4 * e.sms, 256, 0, e.stream>>>(s, d, n);
#else
  cudaMemcpyAsync(d, s, n * sizeof(double), cudaMemcpyDeviceToDevice, e.stream);
#endif
}

__global__ void k_fill(double* p, double v, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = v;
}
template <class T>
__global__ void k_fill_n(T* p, double v, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    p[i] = (T)v;
}

int init_state(Ctx* c, const double* u, const double* v, const double* w,
                    const double* TH) {
  NN(u); NN(v); NN(w); NN(TH);
  Engine& e = c->e;
  Work& W = c->w;
  const size_t N = e.N(), H = e.H();
  // back to the arrangement the buffers were carved in, so that every run
  // from init_state swaps through the same sequence (and replays the same
  // captured step graphs); a humidity field already set moves along
  if (W.Q && W.Q != c->canon.Q)
    cudaMemcpyAsync(c->canon.Q, W.Q, N * sizeof(real), cudaMemcpyDeviceToDevice, e.stream);
  c->canon.apply(W);
  if (W.RHSQ) {
    cudaMemsetAsync(W.RHSQ, 0, N * sizeof(real), e.stream);
    cudaMemsetAsync(W.RHSQp, 0, N * sizeof(real), e.stream);
  }
  to_real(e, u, W.u, N);
  to_real(e, v, W.v, N);
  to_real(e, w, W.w, N);
  to_real(e, TH, W.TH, N);
  for (int i = 0; i < 4; i++) {
    cudaMemsetAsync(W.RHS[i], 0, N * sizeof(real), e.stream);
    cudaMemsetAsync(W.RHSp[i], 0, N * sizeof(real), e.stream);
  }
  for (int i = 0; i < 6; i++) {
    ::alfa::note_launch();
    k_fill_n<<<64, 256, 0, e.stream>>>(W.most[i], i >= 4 ? 1.0 : 0.0, H);
  }
  ::alfa::note_launch(); k_fill_n<<<64, 256, 0, e.stream>>>(W.qz_plane, e.qz_sfc_const, H);
  ::alfa::note_launch(); k_fill_n<<<256, 256, 0, e.stream>>>(W.Cs2, e.Cs2_init, N);
  ::alfa::note_launch(); k_fill_n<<<256, 256, 0, e.stream>>>(W.Cs2Pr, e.Cs2PrRatio_init, N);
  ::alfa::note_launch(); k_fill<<<1, 256, 0, e.stream>>>(W.Ug, e.cfg.Ug2 / 1.0, e.nz);
  ::alfa::note_launch(); k_fill<<<1, 256, 0, e.stream>>>(W.Vg, e.cfg.Vg2 / 1.0, e.nz);
  ::alfa::note_launch(); k_fill<<<1, 256, 0, e.stream>>>(W.zero_prof, 0.0, e.nz);
  W.iteration = e.cfg.istep;
  ::alfa::note_launch(); k_set_int<<<1, 1, 0, e.stream>>>(W.d_it, W.iteration);
  W.have_state = 1;
  W.CFLmax = 0;
  return check_launch(e, "init_state");
}

int set_series(Ctx* c, const double* Uadv, const double* Vadv, const double* THadv,
                    const double* sfc, int nrows) {
  if (nrows < 0) return ALFA_E_SHAPE;
  Engine& e = c->e;
  Work& W = c->w;
  const int nz = e.nz;
  if (W.series_adv) {
    cudaFree(W.series_adv);
    W.series_adv = nullptr;
  }
  W.series_rows = 0;
  if (Uadv || Vadv || THadv) {
    std::vector<double> h((size_t)nrows * 3 * nz, 0.0);
    for (int r = 0; r < nrows; r++)
      for (int k = 0; k < nz; k++) {
        h[((size_t)r * 3 + 0) * nz + k] = Uadv ? Uadv[(size_t)r * nz + k] : 0.0;
        h[((size_t)r * 3 + 1) * nz + k] = Vadv ? Vadv[(size_t)r * nz + k] : 0.0;
        h[((size_t)r * 3 + 2) * nz + k] = THadv ? THadv[(size_t)r * nz + k] : 0.0;
      }
    if (cudaMalloc(&W.series_adv, h.size() * 8 + 8) != cudaSuccess)
      return e.fail("series allocation failed", ALFA_E_CUDA);
    cudaMemcpy(W.series_adv, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
    W.series_rows = nrows;
  }
  W.sfc_series.assign(sfc ? sfc : (const double*)nullptr, sfc ? sfc + nrows : (const double*)nullptr);
  if (W.d_sfc) {
    cudaFree(W.d_sfc);
    W.d_sfc = nullptr;
  }
  if (sfc && nrows > 0) {
    if (cudaMalloc(&W.d_sfc, (size_t)nrows * 8) != cudaSuccess)
      return e.fail("series allocation failed", ALFA_E_CUDA);
    cudaMemcpy(W.d_sfc, sfc, (size_t)nrows * 8, cudaMemcpyHostToDevice);
  }
  release_graphs(c);  // captured steps point at the old series
  return ALFA_OK;
}

int set_geowind_series(Ctx* c, const double* Ug, const double* Vg, int nrows) {
  Engine& e = c->e;
  Work& W = c->w;
  if (nrows < 0 || (nrows > 0 && (!Ug || !Vg)))
    return e.fail("set_geowind_series: bad arguments", ALFA_E_SHAPE);
  const int nz = e.nz;
  if (W.series_geo) {
    cudaFree(W.series_geo);
    W.series_geo = nullptr;
  }
  W.geo_rows = 0;
  if (nrows > 0) {
    std::vector<double> h((size_t)nrows * 2 * nz);
    for (int r = 0; r < nrows; r++)
      for (int k = 0; k < nz; k++) {
        h[((size_t)r * 2 + 0) * nz + k] = Ug[(size_t)r * nz + k];
        h[((size_t)r * 2 + 1) * nz + k] = Vg[(size_t)r * nz + k];
      }
    if (cudaMalloc(&W.series_geo, h.size() * 8) != cudaSuccess)
      return e.fail("series allocation failed", ALFA_E_CUDA);
    cudaMemcpy(W.series_geo, h.data(), h.size() * 8, cudaMemcpyHostToDevice);
    W.geo_rows = nrows;
  }
  release_graphs(c);  // captured steps point at the old series
  return ALFA_OK;
}

int step(Ctx* c, int nsteps, int sgs_mode) {
  if (!c->w.have_state) return c->e.fail("alfa_step before alfa_init_state", ALFA_E_STATE);
  for (int s = 0; s < nsteps; s++) {
    int st = one_step(c, sgs_mode);
    if (st) return st;
  }
  return ALFA_OK;
}

int step_graph(Ctx* c, int nsteps) {
  if (!c->w.have_state) return c->e.fail("alfa_step_graph before alfa_init_state", ALFA_E_STATE);
  for (int s = 0; s < nsteps; s++) {
    int st = graph_step(c);
    if (st) return st;
  }
  return check_launch(c->e, "step_graph");
}

int init_moisture(Ctx* c, const double* Q) {
  NN(Q);
  Engine& e = c->e;
  Work& W = c->w;
  if (e.cfg.optMoisture < 1) return e.fail("alfa_init_moisture with optMoisture = 0", ALFA_E_STATE);
  const size_t N = e.N();
  to_real(e, Q, W.Q, N);
  cudaMemsetAsync(W.RHSQ, 0, N * sizeof(real), e.stream);
  cudaMemsetAsync(W.RHSQp, 0, N * sizeof(real), e.stream);
  // DerivedVars.py:72, the plane every optMoistureSurfBC = 0 step uses
  ::alfa::note_launch(); k_fill_n<<<64, 256, 0, e.stream>>>(W.qm_plane, e.qm_sfc_const, e.H());
  W.have_q = 1;
  return check_launch(e, "init_moisture");
}

int set_moisture_series(Ctx* c, const double* Qadv, const double* msfc, int nrows) {
  Engine& e = c->e;
  Work& W = c->w;
  if (nrows < 0) return e.fail("set_moisture_series: bad arguments", ALFA_E_SHAPE);
  if (W.series_q) cudaFree(W.series_q);
  if (W.d_msfc) cudaFree(W.d_msfc);
  W.series_q = nullptr;
  W.d_msfc = nullptr;
  W.q_rows = W.msfc_rows = 0;
  if (Qadv && nrows > 0) {
    if (cudaMalloc(&W.series_q, (size_t)nrows * e.nz * 8) != cudaSuccess)
      return e.fail("series allocation failed", ALFA_E_CUDA);
    cudaMemcpy(W.series_q, Qadv, (size_t)nrows * e.nz * 8, cudaMemcpyHostToDevice);
    W.q_rows = nrows;
  }
  if (msfc && nrows > 0) {
    if (cudaMalloc(&W.d_msfc, (size_t)nrows * 8) != cudaSuccess)
      return e.fail("series allocation failed", ALFA_E_CUDA);
    cudaMemcpy(W.d_msfc, msfc, (size_t)nrows * 8, cudaMemcpyHostToDevice);
    W.msfc_rows = nrows;
  }
  release_graphs(c);  // captured steps point at the old series
  return ALFA_OK;
}

int get_moisture(Ctx* c, double* Q) {
  NN(Q);
  Engine& e = c->e;
  if (e.cfg.optMoisture < 1) return e.fail("alfa_get_moisture with optMoisture = 0", ALFA_E_STATE);
  to_double(e, c->w.Q, Q, e.N());
  return check_launch(e, "get_moisture");
}

int get_state(Ctx* c, double* u, double* v, double* w, double* TH, double* p) {
  Engine& e = c->e;
  Work& W = c->w;
  const size_t N = e.N();
  if (u) to_double(e, W.u, u, N);
  if (v) to_double(e, W.v, v, N);
  if (w) to_double(e, W.w, w, N);
  if (TH) to_double(e, W.TH, TH, N);
  if (p) to_double(e, W.p, p, N);
  return check_launch(e, "get_state");
}

int get_diag(Ctx* c, alfa_diag* o) {
  if (!o) return ALFA_E_SHAPE;
  Engine& e = c->e;
  Work& W = c->w;
  double m[3] = {0, 0, 0}, q = 0;
  cudaMemcpyAsync(m, W.d_cfl, 3 * 8, cudaMemcpyDeviceToHost, e.stream);
  cudaMemcpyAsync(&q, W.d_qavg, 8, cudaMemcpyDeviceToHost, e.stream);
  std::vector<double> us(e.H());
  cudaMemcpyAsync(us.data(), W.ustar, e.H() * 8, cudaMemcpyDeviceToHost, e.stream);
  int tc_flag = 0;  // a bounded wait of a tensor-core line pass gave up
  if (e.tc_err) {
    cudaMemcpyAsync(&tc_flag, e.tc_err, sizeof(int), cudaMemcpyDeviceToHost, e.stream);
    cudaMemsetAsync(e.tc_err, 0, sizeof(int), e.stream);
  }
  if (cudaStreamSynchronize(e.stream) != cudaSuccess) return e.fail("diag sync failed", ALFA_E_CUDA);
  if (tc_flag)
    return e.fail("a bounded tensor-core wait of a line pass gave up; the step's fields are "
                  "not valid",
                  ALFA_E_TIMEOUT);
  const double cfl = std::max(std::max(m[0] * e.dt_nondim / e.dx, m[1] * e.dt_nondim / e.dy),
                              m[2] * e.dt_nondim / e.dz);
  W.CFL = cfl;
  if (cfl > W.CFLmax) W.CFLmax = cfl;
  double s = 0;
  for (double x : us) s += x * x;
  o->iteration = W.iteration;
  o->CFL = cfl;
  o->CFLmax = W.CFLmax;
  o->ustar_rms = std::sqrt(s / (double)e.H());
  o->qz_sfc_avg = q;
  if (!std::isfinite(cfl)) return e.fail("non-finite velocity", ALFA_E_NUMERIC);
  return ALFA_OK;
}


int stats_sample(Ctx* c, double* acc) {
  Engine& e = c->e;
  Work& W = c->w;
  if (!acc) return e.fail("null pointer argument: acc", ALFA_E_SHAPE);
  if (!W.have_state) return e.fail("alfa_stats_sample before alfa_init_state", ALFA_E_STATE);
  const int nz = e.nz;
  StatsIn a{W.u, W.v, W.w, W.TH, W.g[6], W.g[7], W.gT[2], W.mom[3], W.mom[4], W.mom[5], W.qz,
            W.M, W.ustar, W.d_qavg, W.prof + 21 * nz, W.prof + 22 * nz, W.prof + 23 * nz,
            W.prof + 20 * nz, W.prof + 24 * nz, e.cfg.Ugal, e.T0_nondim};
  if (e.cfg.optMoisture >= 1) {  // Main.py:549-553: Q, dQdz, qm_sfc_avg, qHz_q
    a.Q = W.Q;
    a.dQdz = W.gQ[2];
    a.qHz = W.qzq;
    a.qm_plane = W.qm_plane;
  }
  compute_stats(e, a, acc);
  return check_launch(e, "stats_sample");
}

// checkpoint layout: u v w TH p RHS[4] Cs2 Cs2Pr (N each), Q RHS_Q (N each, when
// optMoisture = 1), most[6] (H each),
// profiles (PROF doubles), then iteration and CFLmax
static size_t ckpt_prof(const Engine& e) { return (size_t)64 * e.nz + 64; }

size_t checkpoint_doubles(const Ctx* c) {
  if (!c) return 0;
  const Engine& e = c->e;
  const size_t nf = e.cfg.optMoisture >= 1 ? 13 : 11;  // + Q, RHS_Q when moist
  return nf * e.N() + 6 * e.H() + ckpt_prof(e) + 2;
}

static int checkpoint_copy(Ctx* c, double* buf, bool save) {
  Engine& e = c->e;
  Work& W = c->w;
  const size_t N = e.N(), H = e.H();
  real* f[11] = {W.u, W.v, W.w, W.TH, W.p, W.RHS[0], W.RHS[1], W.RHS[2], W.RHS[3], W.Cs2,
                 W.Cs2Pr};
  size_t off = 0;
  auto mv = [&](double* dev, size_t n) {
    if (save)
      cudaMemcpyAsync(buf + off, dev, n * 8, cudaMemcpyDeviceToDevice, e.stream);
    else
      cudaMemcpyAsync(dev, buf + off, n * 8, cudaMemcpyDeviceToDevice, e.stream);
    off += n;
  };
  // fields are stored as doubles whatever the build's precision (exact)
  auto mvf = [&](real* dev, size_t n) {
    if (save)
      to_double(e, dev, buf + off, n);
    else
      to_real(e, buf + off, dev, n);
    off += n;
  };
  for (real* p : f) mvf(p, N);
  if (e.cfg.optMoisture >= 1) {
    mvf(W.Q, N);
    mvf(W.RHSQ, N);
  }
  for (int i = 0; i < 6; i++) mv(W.most[i], H);
  mv(W.prof, ckpt_prof(e));
  double tail[2] = {(double)W.iteration, W.CFLmax};
  if (save) {
    cudaMemcpyAsync(buf + off, tail, 2 * 8, cudaMemcpyHostToDevice, e.stream);
  } else {
    cudaMemcpyAsync(tail, buf + off, 2 * 8, cudaMemcpyDeviceToHost, e.stream);
  }
  if (cudaStreamSynchronize(e.stream) != cudaSuccess)
    return e.fail("checkpoint copy failed", ALFA_E_CUDA);
  if (!save) {
    W.iteration = (int)tail[0];
    W.CFLmax = tail[1];
    W.have_state = 1;
    if (e.cfg.optMoisture >= 1) {
      W.have_q = 1;
      ::alfa::note_launch(); k_fill_n<<<64, 256, 0, e.stream>>>(W.qm_plane, e.qm_sfc_const, H);
    }
    ::alfa::note_launch(); k_set_int<<<1, 1, 0, e.stream>>>(W.d_it, W.iteration);
  }
  return ALFA_OK;
}

int save_checkpoint(Ctx* c, double* dst) {
  NN(dst);
  if (!c->w.have_state) return c->e.fail("alfa_save_checkpoint before alfa_init_state", ALFA_E_STATE);
  return checkpoint_copy(c, dst, true);
}

int load_checkpoint(Ctx* c, const double* src) {
  NN(src);
  return checkpoint_copy(c, const_cast<double*>(src), false);
}


int time_kernel(Ctx* c, int which, int reps, double* ms, double* bytes) {
  if (!ms || !bytes || reps < 1 || which < 0 || which > 8)
    return c->e.fail("time_kernel: bad arguments", ALFA_E_SHAPE);
  Engine::TcOp* tcop = nullptr;
  const long long tc_cols = (long long)c->e.ny * c->e.nz;
  if (which == 8) {  // x derivative of an FP32 field on the tensor cores
    const int st = tc_prepare(c->e, LM_DERIV, 0, c->e.nx, c->e.nx, 1.0 / c->e.nx, tc_cols, &tcop);
    if (st) return st;
    cudaMemsetAsync(c->e.tc_err, 0, sizeof(int), c->e.stream);
  }
  Engine& e = c->e;
  Work& W = c->w;
  const double wb = (double)sizeof(real);  // bytes per stored value
  const double N8 = wb * e.N(), Y8 = wb * e.nx * e.my * e.nz, P8 = wb * e.P();
  const double S16 = 2 * wb * e.nx * e.nyh * e.nz;
  auto lo1 = [](int map, real* dst, double scale) {
    LineOut o{};
    o.map = map;
    o.scale = scale;
    o.dst = dst;
    return o;
  };
  XOut o[2];
  for (int i = 0; i < 2; i++) {
    o[i] = XOut{};
    o[i].kind = XO_INV;
    o[i].map = i == 0 ? MAP_DX : MAP_DY;
    o[i].K = e.nyh;
    o[i].rows = e.nx;
    o[i].dst = e.T[1 + i];
    o[i].inv = e.pnx;
  }
  // inputs of the later stages: one pass of each earlier stage
  auto run = [&](int w) {
    switch (w) {
      case 0: {  // y pad pass: (nx, ny, nz) -> (nx, my, nz)
        LineOut q = lo1(LM_PAD, W.Lpad, 1.0 / e.my);
        launch_line(e, 1, ld_field(e, W.u), e.nx, e.ny, e.ny, e.my, 1, &q);
        break;
      }
      case 1: {  // x pad pass: (nx, my, nz) -> (mx, my, nz)
        LineOut q = lo1(LM_PAD, W.Pb[0], 1.0 / e.mx);
        launch_line(e, 0, ld_field(e, W.Lpad), e.nx, e.my, e.nx, e.mx, 1, &q);
        break;
      }
      case 2: {  // x unpad pass: (mx, my, nz) -> (nx, my, nz)
        LineOut q = lo1(LM_UNPAD, W.Lpad, 1.0 / e.nx);
        launch_line(e, 0, ld_field(e, W.Pb[0]), e.mx, e.my, e.mx, e.nx, 1, &q);
        break;
      }
      case 3: {  // y unpad pass: (nx, my, nz) -> (nx, ny, nz)
        LineOut q = lo1(LM_UNPAD, e.W, (9.0 / 4.0) / e.ny);
        launch_line(e, 1, ld_field(e, W.Lpad), e.nx, e.my, e.my, e.ny, 1, &q);
        break;
      }
      case 4: {  // x derivative pass
        LineOut q = lo1(LM_DERIV, e.W, 1.0 / e.nx);
        launch_line(e, 0, ld_field(e, W.u), e.nx, e.ny, e.nx, e.nx, 1, &q);
        break;
      }
      case 5: launch_y_fwd(e, ld_field(e, W.u), e.nx, e.pny, e.nyh, e.T[0]); break;
      case 6: launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, 2, o, e.nyh); break;
      case 8:  // FP32 in and out in two padded-field buffers (P values each)
        tc_launch(e, tcop, tc_cols, reinterpret_cast<const float*>(W.Pb[6]),
                  reinterpret_cast<float*>(W.Pb[7]), nullptr, 1, 0, 0);
        break;
      default: launch_y_inv(e, e.T[1], e.nx, e.nyh, e.pny, 1.0, e.W, 0); break;
    }
  };
  if (which == 1 || which == 2 || which == 3) run(0);
  if (which == 2 || which == 3) run(1);
  if (which == 3) run(2);
  if (which == 6 || which == 7) run(5);
  if (which == 7) run(6);
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  run(which);  // warm
  cudaEventRecord(a, e.stream);
  for (int r = 0; r < reps; r++) run(which);
  cudaEventRecord(b, e.stream);
  cudaEventSynchronize(b);
  float t = 0.f;
  cudaEventElapsedTime(&t, a, b);
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms = (double)t / reps;
  switch (which) {
    case 0: *bytes = N8 + Y8; break;
    case 1: *bytes = Y8 + P8; break;
    case 2: *bytes = P8 + Y8; break;
    case 3: *bytes = Y8 + N8; break;
    case 4: *bytes = 2 * N8; break;
    case 5: *bytes = N8 + S16; break;
    case 6: *bytes = 3 * S16; break;
    case 8: *bytes = 8.0 * e.N(); break;  // N floats in, N floats out
    default: *bytes = S16 + N8; break;
  }
  if (which == 8) {
    int h = 0;
    cudaMemcpyAsync(&h, e.tc_err, sizeof(int), cudaMemcpyDeviceToHost, e.stream);
    cudaStreamSynchronize(e.stream);
    if (h) return e.fail("time_kernel: a bounded tensor-core wait gave up", ALFA_E_TIMEOUT);
  }
  return check_launch(e, "time_kernel");
}

// Deterministic test field for the autotuner: a hash of the index mapped to
// [-1, 1) (no model state is touched).
__global__ void k_fill_hash(real* __restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    unsigned long long h = (i + 1) * 0x9E3779B97F4A7C15ull;
    h ^= h >> 31;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 29;
    x[i] = (real)((double)(h >> 11) * (2.0 / 9007199254740992.0) - 1.0);
  }
}

// out[0] = max |a - b|, out[1] = max |b| (non-negative doubles order like
// their bit patterns, so an integer atomicMax reduces them)
__global__ void k_maxdiff(const real* __restrict__ a, const real* __restrict__ b, size_t n,
                          unsigned long long* out) {
  double d = 0.0, m = 0.0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    d = fmax(d, fabs((double)a[i] - (double)b[i]));
    m = fmax(m, fabs((double)b[i]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    d = fmax(d, __shfl_xor_sync(0xffffffffu, d, o));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, (unsigned long long)__double_as_longlong(d));
    atomicMax(out + 1, (unsigned long long)__double_as_longlong(m));
  }
}

// A variant is a candidate only if its outputs equal the default's to the
// round-off of the build's precision (relative to the output's largest value);
// the split-BF16 tensor-core variant (hi/lo operand pairs, three products,
// about 2^-16 relative per operator entry) to its own accuracy.
static constexpr double kTuneTol = sizeof(real) == 8 ? 1e-12 : 1e-5;
static constexpr double kTcTuneTol = 5e-5;

// the eight line-pass shapes of a step the autotuner times: (X, Y) are the
// input's x and y extents; `in` a synthetic input, `dst` step scratch
struct TuneShape {
  int axis, X, Y, n_in, n_out, nout, map[2];
  const real* in;
  real* dst[2];
  size_t len;
  double scale;
  int cut;
};

static void tune_shapes(Ctx* c, const real* src, TuneShape sh[8]) {
  Engine& e = c->e;
  Work& W = c->w;
  const size_t N = e.N(), Y = (size_t)e.nx * e.my * e.nz, P = e.P();
  const real* Lp = W.Lpad;
  const int nx = e.nx, ny = e.ny, mx = e.mx, my = e.my;
  const TuneShape t[8] = {
      {1, nx, ny, ny, my, 1, {LM_PAD, 0}, src, {W.Lpad, nullptr}, Y, 1.0 / my, 0},
      {0, nx, my, nx, mx, 1, {LM_PAD, 0}, Lp, {W.Pb[0], nullptr}, P, 1.0 / mx, 0},
      {0, mx, my, mx, nx, 1, {LM_UNPAD, 0}, W.Pb[0], {W.Lpad, nullptr}, Y, 1.0 / nx, 0},
      {1, nx, my, my, ny, 1, {LM_UNPAD, 0}, Lp, {e.W, nullptr}, N, (9.0 / 4.0) / ny, 0},
      {0, nx, ny, nx, nx, 1, {LM_DERIV, 0}, src, {e.W, nullptr}, N, 1.0 / nx, 0},
      {1, nx, ny, ny, ny, 1, {LM_DERIV, 0}, src, {e.W, nullptr}, N, 1.0 / ny, 0},
      {0, nx, ny, nx, nx, 2, {LM_TRUNC, LM_TRUNC_DERIV}, src, {W.L2, W.L2 + N}, N, 1.0 / nx,
       e.cut_e[0]},
      {1, nx, ny, ny, ny, 2, {LM_TRUNC, LM_TRUNC_DERIV}, src, {W.L2, W.L2 + N}, N, 1.0 / ny,
       e.cut_e[1]},
  };
  for (int i = 0; i < 8; i++) sh[i] = t[i];
}

// whether a shape's pass can take the phase-split (1) variant's alternative
static bool tune_phase(const TuneShape& sh) {
  return sh.nout == 1 && ((sh.map[0] == LM_PAD && sh.n_in == 256 && sh.n_out == 384) ||
                          (sh.map[0] == LM_UNPAD && sh.n_in == 384 && sh.n_out == 256));
}

// the GEMM columns of a shape's pass on the tensor cores: x lines as one
// (n_in, Y nz) slab, y lines as X slabs of (n_in, nz)
static long long tune_tc_cols(const Engine& e, const TuneShape& sh) {
  return sh.axis == 0 ? (long long)sh.Y * e.nz : (long long)e.nz;
}

#ifdef ALFA_BUILD_FP32
// builds the tensor-core operator of a shape's pass (ALFA_MIXED only)
static int tune_tc_prepare(Engine& e, const TuneShape& sh) {
  Engine::TcOp* op = nullptr;
  return tc_prepare(e, sh.map[0], sh.cut, sh.n_in, sh.n_out, sh.scale, tune_tc_cols(e, sh), &op,
                    sh.nout > 1 ? sh.map[1] : -1, sh.cut, sh.scale);
}
#endif

int set_line_variant(Ctx* c, int axis, int n_in, int n_out, int map, int nout, int variant) {
  Engine& e = c->e;
  if (variant < 0 || variant > CV_VARIANT)
    return e.fail("alfa_set_line_variant: variant must be 0..6", ALFA_E_SHAPE);
  TuneShape shapes[8];
  tune_shapes(c, c->w.Pb[4], shapes);
  for (const TuneShape& sh : shapes) {
    if (sh.axis != axis || sh.n_in != n_in || sh.n_out != n_out || sh.map[0] != map ||
        sh.nout != nout)
      continue;
    if (variant == 1 && !tune_phase(sh))
      return e.fail("alfa_set_line_variant: variant 1 applies to the 256 <-> 384 pad and unpad",
                    ALFA_E_SHAPE);
    if (variant == CV_VARIANT) {
#ifdef ALFA_BUILD_FP32
      LineOut o[2];
      for (int q = 0; q < sh.nout; q++) {
        o[q] = LineOut{};
        o[q].map = sh.map[q];
      }
      if (!cv_line_ok(ld_field(e, sh.in), n_in, n_out, nout, o))
#endif
        return e.fail("alfa_set_line_variant: the two-lane pass needs an FP32 or mixed context, "
                      "nz % 4 == 0 and a pass length it is built for",
                      ALFA_E_SHAPE);
    }
    if (variant == TC_VARIANT) {
#ifdef ALFA_BUILD_FP32
      if (e.cfg.precision != ALFA_MIXED || !tc_shape_ok(n_in, n_out, tune_tc_cols(e, sh)))
        return e.fail("alfa_set_line_variant: the tensor-core pass needs an ALFA_MIXED context "
                      "and n_out % 128 == 0, n_in % 32 == 0, the pass's columns % 256 == 0",
                      ALFA_E_SHAPE);
      const int rc = tune_tc_prepare(e, sh);
      if (rc) return rc;
      cudaMemsetAsync(e.tc_err, 0, sizeof(int), e.stream);
#else
      return e.fail("alfa_set_line_variant: the tensor-core pass needs an ALFA_MIXED context",
                    ALFA_E_SHAPE);
#endif
    }
    e.line_variant[line_key(axis, n_in, n_out, map, nout)] = variant;
    release_graphs(c);  // captured steps hold the old choice
    return check_launch(e, "alfa_set_line_variant");
  }
  return e.fail("alfa_set_line_variant: no autotuned line-pass shape matches", ALFA_E_SHAPE);
}

int autotune(Ctx* c, int reps, alfa_tune_entry* out, int max_out, int* n_out) {
  Engine& e = c->e;
  if (reps < 1 || (max_out > 0 && !out)) return e.fail("autotune: bad arguments", ALFA_E_SHAPE);
  Work& W = c->w;
  const size_t N = e.N();
  real* src = W.Pb[4];
  real* ref[2] = {W.Pb[2], W.Pb[3]};
  unsigned long long* dmax = reinterpret_cast<unsigned long long*>(W.Pb[5]);
  k_fill_hash<<<4 * 148, 256, 0, e.stream>>>(src, N);
  TuneShape shapes[8];
  tune_shapes(c, src, shapes);
  cudaEvent_t ea, eb;
  cudaEventCreate(&ea);
  cudaEventCreate(&eb);
  int n = 0;
  int rc = ALFA_OK;
  for (const TuneShape& sh : shapes) {
    LineOut o[2];
    for (int q = 0; q < sh.nout; q++) {
      o[q] = LineOut{};
      o[q].map = sh.map[q];
      o[q].scale = sh.scale;
      o[q].cut = sh.cut;
      o[q].dst = sh.dst[q];
    }
    const long long key = line_key(sh.axis, sh.n_in, sh.n_out, sh.map[0], sh.nout);
    const bool phase = tune_phase(sh);
    auto run = [&] {
      launch_line(e, sh.axis, ld_field(e, sh.in), sh.X, sh.Y, sh.n_in, sh.n_out, sh.nout, o);
    };
    e.line_variant[key] = 0;
    run();
    for (int q = 0; q < sh.nout; q++)
      cudaMemcpyAsync(ref[q], sh.dst[q], sh.len * sizeof(real), cudaMemcpyDeviceToDevice,
                      e.stream);
    std::vector<int> cand;
    for (int v = 0; v < 2 + Engine::N_SCHED; v++)
      if (v != 1 || phase) cand.push_back(v);
#ifdef ALFA_BUILD_FP32
    {
      const Loader L = ld_field(e, sh.in);
      if (cv_line_ok(L, sh.n_in, sh.n_out, sh.nout, o)) cand.push_back(CV_VARIANT);
    }
    if (e.cfg.precision == ALFA_MIXED) {  // operators are built here, never inside a capture
      if (tc_shape_ok(sh.n_in, sh.n_out, tune_tc_cols(e, sh))) {
        if ((rc = tune_tc_prepare(e, sh)) != ALFA_OK) break;
        cudaMemsetAsync(e.tc_err, 0, sizeof(int), e.stream);
        cand.push_back(TC_VARIANT);
      }
    }
#endif
    int best = -1;
    double best_ms = 0.0;
    const int first = n;
    for (int v : cand) {
      e.line_variant[key] = v;
      run();
      bool same = true;
      for (int q = 0; q < sh.nout; q++) {
        cudaMemsetAsync(dmax, 0, 2 * sizeof(unsigned long long), e.stream);
        k_maxdiff<<<4 * 148, 256, 0, e.stream>>>(sh.dst[q], ref[q], sh.len, dmax);
        unsigned long long h[2] = {0, 0};
        cudaMemcpyAsync(h, dmax, sizeof h, cudaMemcpyDeviceToHost, e.stream);
        cudaStreamSynchronize(e.stream);
        double dd, mm;
        std::memcpy(&dd, &h[0], 8);
        std::memcpy(&mm, &h[1], 8);
        if (!(dd <= (v == TC_VARIANT ? kTcTuneTol : kTuneTol) * mm)) same = false;
      }
      run();  // warm
      cudaEventRecord(ea, e.stream);
      for (int r = 0; r < reps; r++) run();
      cudaEventRecord(eb, e.stream);
      cudaEventSynchronize(eb);
      float t = 0.f;
      cudaEventElapsedTime(&t, ea, eb);
      const double ms = (double)t / reps;
      if (same && (best < 0 || ms < best_ms)) {
        best = v;
        best_ms = ms;
      }
      if (n < max_out) {
        alfa_tune_entry& te = out[n];
        te.axis = sh.axis;
        te.n_in = sh.n_in;
        te.n_out = sh.n_out;
        te.outputs = sh.nout;
        te.map = sh.map[0];
        te.variant = v;
        te.chosen = 0;
        te.equal = same ? 1 : 0;
        te.ms = ms;
      }
      n++;
    }
    if (e.tc_err) {  // a tensor-core candidate whose wait gave up is not chosen
      int h = 0;
      cudaMemcpyAsync(&h, e.tc_err, sizeof(int), cudaMemcpyDeviceToHost, e.stream);
      cudaMemsetAsync(e.tc_err, 0, sizeof(int), e.stream);
      cudaStreamSynchronize(e.stream);
      if (h && best == TC_VARIANT) best = -1;
      if (h)
        for (int i = first; i < n && i < max_out; i++)
          if (out[i].variant == TC_VARIANT) out[i].equal = 0;
    }
    if (best < 0) best = 0;
    e.line_variant[key] = best;
    for (int i = first; i < n && i < max_out; i++) out[i].chosen = out[i].variant == best;
    if ((rc = check_launch(e, "autotune")) != ALFA_OK) break;
  }
  cudaEventDestroy(ea);
  cudaEventDestroy(eb);
  release_graphs(c);  // captured steps hold the old choices
  if (n_out) *n_out = n;
  return rc;
}


struct Ens {
  std::vector<Ctx*> m;
  std::vector<cudaStream_t> own;  // one stream per member
  std::vector<cudaEvent_t> done;  // member i finished its part of the graph
  cudaStream_t master = nullptr;
  cudaEvent_t start = nullptr;
  cudaStream_t user = nullptr;   // the caller's stream the steps are ordered on
  cudaEvent_t fence = nullptr;
  struct G {
    cudaGraphExec_t exec = nullptr;
    std::vector<StepPtrs> before, after;
    unsigned long long kernels = 0;
  } graphs[4];
  std::string err;
};

static void ens_release(Ens* E) {
  for (auto& g : E->graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
  }
}

// one step of every member inside one captured graph (members at the same
// iteration, same istep and dynamic interval); returns nonzero to ask the
// caller for the member-by-member path
static int ens_graph_step(Ens* E) {
  for (size_t i = 0; i < E->m.size(); i++) E->m[i]->e.stream = E->own[i];
  Ctx* c0 = E->m[0];
  const int it = c0->w.iteration;
  const alfa_config& cf0 = c0->e.cfg;
  for (Ctx* c : E->m) {
    const alfa_config& cf = c->e.cfg;
    if (c->w.iteration != it || cf.istep != cf0.istep ||
        cf.dynamicSGS_call_time != cf0.dynamicSGS_call_time ||
        ((cf.optSgs >= 1 && cf.optSgs <= 4) != (cf0.optSgs >= 1 && cf0.optSgs <= 4)))
      return 1;
    if (cf.optAdvection >= 1 && it - 1 >= c->w.series_rows) return 1;
    if (cf.optGeoWind >= 1 && it - 1 >= c->w.geo_rows) return 1;
    if (cf.optMoisture >= 1 &&
        (!c->w.have_q || (cf.optMoistureSurfBC >= 1 && it - 1 >= c->w.msfc_rows) ||
         (cf.optAdvection >= 1 && c->w.series_q && it - 1 >= c->w.q_rows)))
      return 1;
    if (cf.optSurfBC >= 1 && it - 1 >= (int)c->w.sfc_series.size()) return 1;
  }
  if (it == cf0.istep) return 1;
  const bool dyn = (cf0.optSgs >= 1 && cf0.optSgs <= 4) && (it % cf0.dynamicSGS_call_time == 0);
  auto& g = E->graphs[(it & 1) * 2 + (dyn ? 1 : 0)];
  const size_t n = E->m.size();
  std::vector<StepPtrs> now(n);
  for (size_t i = 0; i < n; i++) now[i] = StepPtrs::of(E->m[i]->w);
  bool same = g.exec && g.before.size() == n;
  for (size_t i = 0; same && i < n; i++) same = g.before[i] == now[i];
  if (!same) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    g.exec = nullptr;
    if (cudaStreamBeginCapture(E->master, cudaStreamCaptureModeRelaxed) != cudaSuccess) return 1;
    cudaEventRecord(E->start, E->master);
    int st = 0;
    const unsigned long long l0 = ::alfa::launch_count();
    std::vector<StepPtrs> after(n);
    for (size_t i = 0; i < n; i++) {
      Ctx* c = E->m[i];
      cudaStreamWaitEvent(E->own[i], E->start, 0);
      if (!st) st = one_step(c);
      after[i] = StepPtrs::of(c->w);
      cudaEventRecord(E->done[i], E->own[i]);
      cudaStreamWaitEvent(E->master, E->done[i], 0);
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(E->master, &graph);
    for (size_t i = 0; i < n; i++) {  // nothing ran yet: undo the host side
      now[i].apply(E->m[i]->w);
      E->m[i]->w.iteration = it;
    }
    if (st || ce != cudaSuccess || !graph) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      E->err = st ? E->m[0]->e.err : "ensemble capture failed";
      return st ? st : ALFA_E_CUDA;
    }
    const cudaError_t ie = cudaGraphInstantiate(&g.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie != cudaSuccess) {
      g.exec = nullptr;
      E->err = "ensemble graph instantiation failed";
      return ALFA_E_CUDA;
    }
    g.before = now;
    g.after = after;
    g.kernels = ::alfa::launch_count() - l0;
  } else {
    ::alfa::add_launches(g.kernels);
  }
  if (cudaGraphLaunch(g.exec, E->master) != cudaSuccess) {
    E->err = "ensemble graph launch failed";
    return ALFA_E_CUDA;
  }
  for (size_t i = 0; i < n; i++) {
    g.after[i].apply(E->m[i]->w);
    E->m[i]->w.iteration = it + 1;
  }
  return ALFA_OK;
}

int ens_create(Ctx* const* members, int n, Ens** out) {
  if (!members || n < 1 || !out) return ALFA_E_SHAPE;
  Ens* E = new Ens();
  for (int i = 0; i < n; i++) {
    if (!members[i] || !members[i]->w.have_state) {
      delete E;
      return ALFA_E_STATE;
    }
    E->m.push_back(members[i]);
  }
  bool ok = cudaStreamCreateWithFlags(&E->master, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&E->start, cudaEventDisableTiming) == cudaSuccess;
  E->own.resize(n, nullptr);
  E->done.resize(n, nullptr);
  for (int i = 0; ok && i < n; i++) {
    ok = cudaStreamCreateWithFlags(&E->own[i], cudaStreamNonBlocking) == cudaSuccess &&
         cudaEventCreateWithFlags(&E->done[i], cudaEventDisableTiming) == cudaSuccess;
    if (ok) {
      release_graphs(members[i]);
      members[i]->e.stream = E->own[i];
    }
  }
  if (!ok) {
    ens_destroy(E);
    return ALFA_E_CUDA;
  }
  *out = E;
  return ALFA_OK;
}

static int ens_steps(Ens* E, int nsteps);

int ens_step(Ens* E, int nsteps) {
  if (!E) return ALFA_E_STATE;
  if (E->user) {  // after the work already queued on the caller's stream
    cudaEventRecord(E->fence, E->user);
    cudaStreamWaitEvent(E->master, E->fence, 0);
  }
  const int st = ens_steps(E, nsteps);
  if (E->user) {  // and before the work queued on it next
    cudaEventRecord(E->fence, E->master);
    cudaStreamWaitEvent(E->user, E->fence, 0);
  }
  return st;
}

int ens_set_stream(Ens* E, cudaStream_t s) {
  if (!E) return ALFA_E_STATE;
  if (s && !E->fence &&
      cudaEventCreateWithFlags(&E->fence, cudaEventDisableTiming) != cudaSuccess)
    return ALFA_E_CUDA;
  E->user = s;
  return ALFA_OK;
}

static int ens_steps(Ens* E, int nsteps) {
  for (int s = 0; s < nsteps; s++) {
    int st = ens_graph_step(E);
    if (st == ALFA_OK) continue;
    if (st < 0) return st;
    // member by member (bootstrap step, or members not in lockstep); the
    // master waits for every member so the next graph starts after them
    cudaEventRecord(E->start, E->master);
    for (size_t i = 0; i < E->m.size(); i++) {
      cudaStreamWaitEvent(E->own[i], E->start, 0);
      const int r = graph_step(E->m[i]);
      if (r) {
        E->err = E->m[i]->e.err;
        return r;
      }
      cudaEventRecord(E->done[i], E->own[i]);
      cudaStreamWaitEvent(E->master, E->done[i], 0);
    }
  }
  return ALFA_OK;
}

int ens_sync(Ens* E) {
  if (!E) return ALFA_E_STATE;
  return cudaStreamSynchronize(E->master) == cudaSuccess ? ALFA_OK : ALFA_E_CUDA;
}

const char* ens_error(const Ens* E) { return E ? E->err.c_str() : ""; }

void ens_destroy(Ens* E) {
  if (!E) return;
  if (E->master) cudaStreamSynchronize(E->master);
  ens_release(E);
  for (size_t i = 0; i < E->own.size(); i++) {
    if (E->own[i]) {
      cudaStreamSynchronize(E->own[i]);
      if (i < E->m.size() && E->m[i]->e.stream == E->own[i]) {
        release_graphs(E->m[i]);
        E->m[i]->e.stream = 0;
      }
      cudaStreamDestroy(E->own[i]);
    }
    if (E->done[i]) cudaEventDestroy(E->done[i]);
  }
  if (E->start) cudaEventDestroy(E->start);
  if (E->fence) cudaEventDestroy(E->fence);
  if (E->master) cudaStreamDestroy(E->master);
  delete E;
}



// ---------------------------------------------------------------------------
// context life cycle and accessors (the whole-step interface, alfa_iface.cuh)
// ---------------------------------------------------------------------------
int ctx_create(const alfa_config& cfg, Ctx** out, std::string* err) {
  *out = nullptr;
  Ctx* c = new Ctx();
  cudaGetDevice(&c->e.device);
  int st = engine_init(c->e, cfg);
  if (!st) cudaDeviceGetAttribute(&c->e.sms, cudaDevAttrMultiProcessorCount, c->e.device);
  if (st) {
    if (err) *err = c->e.err;
    engine_free(c->e);
    delete c;
    return st;
  }
  Carver k{nullptr, 0, true};
  carve(c, k);
  c->bytes = k.off + 256;
  if (cudaMalloc(&c->base, c->bytes) != cudaSuccess) {
    cudaGetLastError();
    if (err) *err = "workspace allocation of " + std::to_string(c->bytes) + " bytes failed";
    engine_free(c->e);
    delete c;
    return ALFA_E_CUDA;
  }
  cudaMemset(c->base, 0, c->bytes);
  Carver k2{(char*)c->base, 0, false};
  carve(c, k2);
  c->canon = StepPtrs::of(c->w);
  *out = c;
  return ALFA_OK;
}

void ctx_destroy(Ctx* c) {
  if (!c) return;
  if (c->w.series_adv) cudaFree(c->w.series_adv);
  if (c->w.series_geo) cudaFree(c->w.series_geo);
  if (c->w.series_q) cudaFree(c->w.series_q);
  if (c->w.d_msfc) cudaFree(c->w.d_msfc);
  if (c->w.d_sfc) cudaFree(c->w.d_sfc);
  release_graphs(c);
  cudaFree(c->base);
  engine_free(c->e);
  delete c;
}

const char* ctx_error(const Ctx* c) { return c->e.err.c_str(); }

int ctx_fail(Ctx* c, const std::string& m, int code) { return c->e.fail(m, code); }

void ctx_set_stream(Ctx* c, cudaStream_t s) { c->e.stream = s; }

size_t ctx_bytes(const Ctx* c) { return c->bytes; }

void ctx_derived(const Ctx* c, alfa_derived* o) {
  const Engine& e = c->e;
  o->mx = e.mx;
  o->my = e.my;
  o->nx_rfft = e.nxh;
  o->ny_rfft = e.nyh;
  o->z_scale = e.z_scale;
  o->g_nondim = e.g_nondim;
  o->f_coriolis_nondim = e.f_nondim;
  o->T_0_nondim = e.T0_nondim;
  o->inversion_nondim = e.inversion_nondim;
  o->dx = e.dx;
  o->dy = e.dy;
  o->dz = e.dz;
  o->L = e.L;
  o->dt_nondim = e.dt_nondim;
  o->TFR = e.TFR;
  for (int i = 0; i < 2; i++) {
    o->cut_explicit[i] = e.cut_e[i];
    o->cut_level1[i] = e.cut_1[i];
    o->cut_level2[i] = e.cut_2[i];
  }
}

void ctx_set_tc_spin(Ctx* c, unsigned long long polls) { c->e.tc_spin = polls; }

int tc_line_apply(Ctx* c, int map, int cut, int n_in, int n_out, double scale, long long ncols,
                  const float* X, float* Y) {
  NN(X);
  NN(Y);
  if (map < LM_IDENT || map > LM_UNPAD) return c->e.fail("tc_line_apply: unknown map", ALFA_E_SHAPE);
  return tc_line_apply(c->e, map, cut, n_in, n_out, scale, ncols, X, Y);
}

}  // namespace ALFA_PREC
}  // namespace alfa
