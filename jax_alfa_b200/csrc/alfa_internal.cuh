// Engine state and internal interfaces of libalfa (not part of the C-ABI).
// The enums and the launch counter are shared; the engine, its loaders and
// its operators are declared once per storage precision (alfa_prec.cuh).
#pragma once
#include <cuda_runtime.h>

#include <deque>
#include <map>
#include <string>
#include <vector>

#include "alfa.h"
#include "alfa_fft.cuh"

namespace alfa {

// Partial-sum blocks of the plane mean behind alfa_PlanarMean_noalloc: the
// launch (alfa_physics.cu) and the fixed partial-sum array it fills
// (alfa_noalloc.cu) are both sized by this one constant.
constexpr int NOALLOC_RED_BLOCKS = 256;

// Process-wide count of kernel launches made by this library (every launch
// site calls note_launch(); read through alfa_launch_count()).
void note_launch();
unsigned long long launch_count();
// count n kernels that ran without passing a launch site (graph replays)
void add_launches(unsigned long long n);

// Raise a kernel's dynamic shared-memory limit to at least `bytes` on the
// current device (the attribute call is made once per kernel, device and
// size increase, not on every launch).
void raise_smem_limit(const void* kernel, size_t bytes);

// ---------------------------------------------------------------------------
// Physical-space value producers for the y-forward FFT stage.  Instead of
// materialising a product or a staggered combination as a full field and
// transforming it, the first FFT stage evaluates it while loading its tile.
// Each kind restates one expression of the reference (cited at its use).
// ---------------------------------------------------------------------------
enum LoadKind {
  LD_FIELD = 0,      // a0
  LD_MUL,            // a0 * a1
  LD_MUL3,           // a0 * a1 * a2   (left to right)
  LD_PRESSURE_R,     // a0 - c0*a1 + c1*a2        (PressureRC R_i)
  LD_ADV_XY,         // Cx/Cy rows (advection, padded space)
  LD_ADV_Z,          // Cz rows
  LD_SCALAR_ADV,     // scalar advection rows
  LD_STRESS_UVP,     // -2L^2 Cs2 |S| S_ij, top row 0
  LD_STRESS_W,       // interior -2L^2 stag(Cs2)|S_w| S_i3, rows 0 and top 0
  LD_QZ,             // interior -2L^2 stag(r)|S_w| dTHdz, rows 0 and top 0
  LD_WSTAR,          // w_ of LASDD: staggered w
  LD_UVP_S13,        // S13/S23 on uvp nodes from gradients
  LD_W_SXX,          // w-node strain components from gradients
  LD_THZ,            // THz of ScalarLASDD
  LD_MUL_THZ,        // a0 * THz(a1)
  LD_WL_UVP,         // c0 * a0 * a1, top row 0 (Wong-Lilly stresses / fluxes, uvp nodes)
  LD_WL_W,           // interior c0 * stag(a0) * a1, rows 0 and top 0 (w nodes)
};

// Every kind a tile kernel evaluates (switches expand this list, so a kind
// added above and here is handled everywhere).
#define ALFA_LOADER_KINDS(X)                                                          \
  X(LD_FIELD) X(LD_MUL) X(LD_MUL3) X(LD_PRESSURE_R) X(LD_ADV_XY) X(LD_ADV_Z)           \
  X(LD_SCALAR_ADV) X(LD_STRESS_UVP) X(LD_STRESS_W) X(LD_W_SXX) X(LD_THZ) X(LD_MUL_THZ) \
  X(LD_WL_UVP) X(LD_WL_W)

// Output maps of the x-column stage.
enum SpecMap { MAP_IDENT = 0, MAP_TRUNC, MAP_DX, MAP_DY, MAP_PAD, MAP_UNPAD };
enum XOutKind { XO_SPEC = 0, XO_INV = 1 };

// 1-D line operators (k_line): a transform along x or y of real fields,
// two real z columns packed per complex line.  Maps act on the full packed
// spectrum of length n_in and produce n_out entries.
enum LineMap { LM_IDENT = 0, LM_TRUNC, LM_DERIV, LM_TRUNC_DERIV, LM_PAD, LM_UNPAD };

}  // namespace alfa

namespace alfa {
namespace ALFA_PREC {

// A loader's inputs are fields of the build's precision; its constants and
// the arithmetic of its expression are FP64 (the value is rounded to `real`
// once, where it enters a transform tile or a field).
struct Loader {
  int kind;
  int sub;            // variant selector inside a kind
  int nz;
  const real* a[10];
  double c[4];
};

struct XOut {
  int kind;   // XO_SPEC: write the mapped spectrum column (nx, nyh layout)
              // XO_INV : inverse-transform the mapped column, write T tile
  int map;
  int cx, cy; // truncation cut-offs (MAP_TRUNC)
  int K;      // ky columns held by the destination
  int rows;   // rows of the destination (transform length for XO_INV)
  cd* dst;
  FftPlan inv;
};

struct LineOut {
  int map;
  int cut;          // LM_TRUNC / LM_TRUNC_DERIV: keep k < cut or k >= n - cut + 1
  double scale;     // applied to the inverse transform (1/n_out, times any extra factor)
  int accumulate;   // 1: dst += result
  real* dst;
};

struct Engine;

// ---------------------------------------------------------------------------
// Engine: one configuration, one stream, its constants, tables, workspace.
// ---------------------------------------------------------------------------
struct Engine {
  alfa_config cfg;
  cudaStream_t stream = 0;
  std::string err;
  int device = 0;
  int sms = 148;  // multiprocessors of the device

  // grid
  int nx, ny, nz, mx, my, nxh, nyh, mxh, myh;
  // DerivedVars (src/config/DerivedVars.py:48-112), in the reference's order
  double z_scale, g_nondim, f_nondim, T0_nondim, inversion_nondim, qz_sfc_const;
  // moisture (DerivedVars.py:69-75; SurfaceFlux.py:475-476): q_inversion
  // non-dimensional, the constant surface moisture flux, and
  // log(0.5 dz z_scale / z_ref) of the prescribed-Q flux
  double q_inversion_nondim = 0, qm_sfc_const = 0, log_zq = 0;
  double dx, dy, dz, idz, L, dt_nondim, TFR;
  int optDealias;
  double Cs2_init, Cs2PrRatio_init, z_damping_nondim, RelaxTime_nondim;
  int cut_e[2], cut_1[2], cut_2[2];   // explicit / level-1 / level-2 cut-offs (x, y)

  // device tables
  double* d_kx = nullptr;   // (nx) with Nyquist zeroed
  double* d_ky = nullptr;   // (nyh) with Nyquist zeroed
  double* d_kr = nullptr;   // (nx) pressure x wavenumbers (Nyquist kept)
  double* d_b_thomas = nullptr;  // (nx, nyh, nz+1)
  double* d_m_thomas = nullptr;  // (nx, nyh, nz+1) elimination multipliers, row 0 unused
  double* d_c_p = nullptr;       // (nz+1)
  double* d_rd = nullptr;        // Rayleigh damping profile, full levels (nz)
  double* d_rd_stag = nullptr;   // half levels (nz)
  FftPlan pnx, pny, pmx, pmy;
  std::vector<void*> allocs;

  // workspace (complex tiles and fields)
  cd* T[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t T_elems = 0;
  double* red = nullptr;          // reduction partials (FP64 in every build)
  size_t red_elems = 0;
  double* scal = nullptr;         // small device scalars / profiles
  real* W = nullptr;              // one field of workspace
  size_t W_elems = 0;
  real* mat = nullptr;            // a loader's expression, materialised (P elements)
  double* stat = nullptr;         // statistics scratch (24 nz)
  double2* thomas_dm = nullptr;   // FP32 build: FP64 forward-sweep scratch of the Thomas
                                  // solve (nx, nyh, nz); the FP64 build uses the output

  // Line-pass variants chosen by the autotuner (alfa_autotune), by pass
  // shape (line_key): 0 the default dispatch, 1 the compile-time transform
  // even where a phase-split pad/unpad exists, 2 + r the runtime-plan
  // transform with radix schedule r of alt_plans (largest radix 8, largest
  // radix 4, ascending order).
  std::map<long long, int> line_variant;
  // split-BF16 tensor-core line operators built so far (alfa_tc.cu), and
  // that kernel's error flag
  struct TcOp {
    int map, cut, n_in, n_out;
    double scale;
    int map2, cut2;  // a second map stacked below the first (map2 < 0: none)
    double scale2;
    void *hi, *lo;
  };
  std::deque<TcOp> tc_ops;  // a deque: prepared operators keep their addresses
  int* tc_err = nullptr;
  unsigned long long tc_spin = 0;  // mbarrier polls of the main loop's waits (0: default)
  static constexpr int N_SCHED = 3;
  // the tensor-core (split-BF16) variant of a line pass: ALFA_MIXED contexts
  // only, where the autotuner measured it faster and within its tolerance
  FftPlan alt_plans[4][N_SCHED];  // for nx, ny, mx, my

  size_t N() const { return (size_t)nx * ny * nz; }
  size_t P() const { return (size_t)mx * my * nz; }
  size_t S() const { return (size_t)nx * nyh * nz; }
  size_t H() const { return (size_t)nx * ny; }

  int fail(const std::string& m, int code) {
    err = m;
    return code;
  }
};

int engine_init(Engine& e, const alfa_config& c);
void engine_free(Engine& e);
int check_launch(Engine& e, const char* what);

// spectral building blocks (alfa_spectral.cu)
void launch_y_fwd(Engine& e, const Loader& L, int rows, const FftPlan& p, int K, cd* T);
void launch_x(Engine& e, const cd* src, int in_spec, int rows_in, int Kin, const FftPlan& fwd,
              int nout, const XOut* outs, int Kgrid);
void launch_y_inv(Engine& e, const cd* T, int rows, int K, const FftPlan& p, double scale,
                  real* out, int accumulate);

// 1-D line passes (alfa_spectral.cu).  axis 0: lines along x of a field
// (X, Y, nz); axis 1: lines along y.  X/Y of the input field; the output
// field has n_out in place of the transformed extent.
void launch_line(Engine& e, int axis, const Loader& L, int X, int Y, int n_in, int n_out,
                 int nout, const LineOut* outs);
// the line-pass variant that runs on the tensor cores (after the default, the
// compile-time transform and the N_SCHED runtime radix schedules)
constexpr int TC_VARIANT = 2 + Engine::N_SCHED;
// the FP32 line-pass variant on two-lane elements (two packed columns per
// thread, paired FP32 instructions)
constexpr int CV_VARIANT = TC_VARIANT + 1;
#ifdef ALFA_BUILD_FP32
bool cv_line_ok(const Loader& L, int n_in, int n_out, int nout, const LineOut* outs);
#endif
// the autotuner's key of a line pass
long long line_key(int axis, int n_in, int n_out, int map, int nout);
// Y (n_out, ncols) = M X (X: (n_in, ncols) FP32) for the line map's
// operator M times scale, on the tensor cores in split BF16 (alfa_tc.cu);
// synchronises the stream
int tc_line_apply(Engine& e, int map, int cut, int n_in, int n_out, double scale,
                  long long ncols, const float* X, float* Y);
// the same in parts: the operator (built once, checks the shapes) and one
// asynchronous launch
int tc_prepare(Engine& e, int map, int cut, int n_in, int n_out, double scale, long long ncols,
               Engine::TcOp** out, int map2 = -1, int cut2 = 0, double scale2 = 0.0);
void tc_launch(Engine& e, const Engine::TcOp* op, long long ncols, const float* X, float* Y0,
               float* Y1, int batch, long long xbs, long long ybs);
bool tc_shape_ok(int n_in, int n_out, long long ncols);
// separable spectral operators on real fields
void op2_filter_deriv(Engine& e, const Loader& L, real* f, real* dx, real* dy,
                      real* scratch2);  // explicit filter and its x/y derivatives
void op2_deriv(Engine& e, const Loader& L, real* dx, int accx, real* dy, int accy);
void op2_pad(Engine& e, const Loader& L, real* out_pad, real* scratch);
void op2_unpad(Engine& e, const Loader& L_pad, real* out, real* scratch);
// value of a loader at every point of its n-element domain, written to out
void materialize(Engine& e, const Loader& L, size_t n, real* out);

// composite transforms on regular/padded grids
Loader ld_field(const Engine& e, const real* a);
void op_rfft2(Engine& e, const Loader& L, cd* spec);                       // FFT
void op_filter_explicit(Engine& e, const Loader& L, real* out, cd* spec); // Filtering_Explicit(FFT(.))
void op_filter12(Engine& e, const Loader& L, real* out1, real* out2);   // Level1/Level2 of FFT(.)
void op_deriv_spec(Engine& e, const cd* spec, real* dx, real* dy);      // Derivxy x/y of a spectrum
void op_deriv_field(Engine& e, const Loader& L, real* dx, real* dy);    // Derivxy(FFT(.)) x/y
void op_pad(Engine& e, const Loader& L, real* out_pad);                   // Dealias1(FFT(.))
void op_unpad(Engine& e, const Loader& L_pad, real* out);                 // Dealias2(FFT_pad(.))
void op_irfft2(Engine& e, const cd* spec, real* out);                     // irfft2 of a spectrum
void op_pad_spec(Engine& e, const cd* spec, real* out_pad);               // Dealias1(spec)
void op_unpad_spec(Engine& e, const cd* spec_pad, real* out);             // Dealias2(spec_pad)
void op_rfft2_pad(Engine& e, const Loader& L, cd* spec_pad);                // FFT_pad
void op_filter1_spec(Engine& e, const cd* spec, int level, real* out);    // Filtering_Level1/2(spec)

}  // namespace ALFA_PREC
}  // namespace alfa
