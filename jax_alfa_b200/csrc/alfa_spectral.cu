// Batched 2-D real FFTs over the (x, y) planes of z-fastest fields, and the
// spectral operators of the reference built from them.
//
// A 2-D transform is three tile kernels, each moving one field through HBM
// once, with z runs of 16 (real) or 8 (complex) consecutive levels as the
// contiguous, coalesced dimension:
//   k_y_fwd : real rows -> half-spectrum in y (two real z-columns packed as
//             one complex column, split after the transform); the real
//             input can be an expression of several fields (Loader);
//   k_x     : per (ky, z-run) column: optional forward transform in x, then
//             up to three outputs, each a spectral map (truncation filter,
//             i*k derivative, 3/2-rule pad/unpad) either written as a
//             spectrum or inverse-transformed in x;
//   k_y_inv : half-spectrum in y -> real rows (complex-to-real, imaginary
//             parts of the ky=0 and ky=ny/2 bins ignored, as irfft does).
// Only the ky columns a consumer needs are computed and stored (a level-1
// test filter keeps ky < ny/4, so its tiles hold a quarter of the columns).
#include <cmath>

#include "alfa_internal.cuh"

namespace alfa {

static constexpr int YC = 8;    // complex columns (= 16 real z levels) per y tile
static constexpr int YTHREADS = 128;
static constexpr int XTHREADS = 128;

// ---------------------------------------------------------------------------
// Loader evaluation (value of the real input at linear index i, level z)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double ld_eval(const Loader& L, size_t i, int z) {
  const int nz = L.nz;
  switch (L.kind) {
    case LD_FIELD:
      return L.a[0][i];
    case LD_MUL:
      return L.a[0][i] * L.a[1][i];
    case LD_MUL3:
      return L.a[0][i] * L.a[1][i] * L.a[2][i];
    case LD_PRESSURE_R:  // NSE_PressureTerms.py:140-142
      return L.a[0][i] - L.c[0] * L.a[1][i] + L.c[1] * L.a[2][i];
    case LD_ADV_XY: {  // NSE_AdvectionTerms.py:105-116 (Cx) and :122-132 (Cy)
      const double arg1 = L.a[0][i] * (L.a[1][i] - L.a[2][i]);
      if (z == 0) {
        const double a2n = L.a[3][i + 1] * (L.a[4][i + 1] - L.a[5][i + 1]);
        return arg1 + 0.5 * a2n;
      }
      const double a2 = L.a[3][i] * (L.a[4][i] - L.a[5][i]);
      if (z == nz - 1) return arg1 + a2;
      const double a2n = L.a[3][i + 1] * (L.a[4][i + 1] - L.a[5][i + 1]);
      return arg1 + 0.5 * (a2 + a2n);
    }
    case LD_ADV_Z: {  // NSE_AdvectionTerms.py:137-151
      if (z == 0 || z == nz - 1) return 0.0;
      const double ug = 0.5 * (L.a[0][i - 1] + L.a[0][i]);
      const double vg = 0.5 * (L.a[1][i - 1] + L.a[1][i]);
      const double a1 = ug * (L.a[2][i] - L.a[3][i]);
      const double a2 = vg * (L.a[4][i] - L.a[5][i]);
      return a1 + a2;
    }
    case LD_SCALAR_ADV: {  // SCL_AdvectionTerms.py:89-101
      const double c1 = L.a[0][i] * L.a[3][i] + L.a[1][i] * L.a[4][i];
      const double c2 = L.a[2][i] * L.a[5][i];
      if (z == nz - 1) return c1 + c2;
      const double c2n = L.a[2][i + 1] * L.a[5][i + 1];
      return c1 + 0.5 * (c2 + c2n);
    }
    case LD_STRESS_UVP:  // SGSStresses_SM.py:122-132, ScalarSGSFluxes_SM.py:78-84
      if (z == nz - 1) return 0.0;
      return L.c[0] * L.a[0][i] * L.a[1][i] * L.a[2][i];
    case LD_STRESS_W:  // SGSStresses_SM.py:223-232, ScalarSGSFluxes_SM.py:163-169
      if (z == 0 || z == nz - 1) return 0.0;
      return L.c[0] * (0.5 * (L.a[0][i - 1] + L.a[0][i])) * L.a[1][i] * L.a[2][i];
    case LD_W_SXX: {  // StrainRates.py:250-276: component L.sub of the w-node strain
      const double* const* g = L.a;  // dudx dvdx dwdx dudy dvdy dwdy dudz dvdz dwdz
      auto stag = [&](const double* d) -> double {
        if (z == 0) return d[i];
        if (z == nz - 1) return 0.0;
        return 0.5 * (d[i - 1] + d[i]);
      };
      switch (L.sub) {
        case 0: return stag(g[0]);                                  // S11 = ux
        case 1: return stag(g[4]);                                  // S22 = vy
        case 2: return stag(g[8]);                                  // S33 = wz
        case 3: return 0.5 * (stag(g[3]) + stag(g[1]));             // S12
        case 4: {                                                   // S13
          const double wx = (z == 0) ? 0.5 * (g[2][i] + g[2][i + 1]) : g[2][i];
          return 0.5 * (g[6][i] + wx);
        }
        default: {                                                  // S23
          const double wy = (z == 0) ? 0.5 * (g[5][i] + g[5][i + 1]) : g[5][i];
          return 0.5 * (g[7][i] + wy);
        }
      }
    }
    case LD_THZ: {  // DynamicSGS_ScalarLASDD_SM.py:182-185
      const double* d = L.a[0];
      if (z == 0 || z == nz - 1) return d[i];
      return 0.5 * (d[i] + d[i + 1]);
    }
    case LD_MUL_THZ: {  // S * THz
      const double* d = L.a[1];
      const double t = (z == 0 || z == nz - 1) ? d[i] : 0.5 * (d[i] + d[i + 1]);
      return L.a[0][i] * t;
    }
    default:
      return 0.0;
  }
}

// ---------------------------------------------------------------------------
// k_y_fwd: rows x n(y) x nz real -> T (rows, K, nz) complex, ky < K
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(YTHREADS) k_y_fwd(Loader L, FftPlan p, int K, cd* __restrict__ T) {
  extern __shared__ cd sm[];
  const int n = p.n;
  const int nz = L.nz;
  const int z0 = blockIdx.x * (2 * YC);
  const int row = blockIdx.y;
  cd* b0 = sm;
  cd* b1 = sm + n * YC;
  for (int t = threadIdx.x; t < n * YC; t += blockDim.x) {
    const int y = t / YC, c = t % YC;
    const int z = z0 + 2 * c;
    const size_t base = ((size_t)row * n + y) * nz;
    const double re = (z < nz) ? ld_eval(L, base + z, z) : 0.0;
    const double im = (z + 1 < nz) ? ld_eval(L, base + z + 1, z + 1) : 0.0;
    b0[t] = make_double2(re, im);
  }
  const int r = fft_tile<-1>(b0, b1, p, YC);
  const cd* Z = r ? b1 : b0;
  for (int t = threadIdx.x; t < K * YC; t += blockDim.x) {
    const int k = t / YC, c = t % YC;
    const int z = z0 + 2 * c;
    const cd zk = Z[k * YC + c];
    const cd zn = Z[((n - k) % n) * YC + c];
    const cd A = make_double2(0.5 * (zk.x + zn.x), 0.5 * (zk.y - zn.y));
    const cd B = make_double2(0.5 * (zk.y + zn.y), -0.5 * (zk.x - zn.x));
    const size_t o = ((size_t)row * K + k) * nz + z;
    if (z < nz) T[o] = A;
    if (z + 1 < nz) T[o + 1] = B;
  }
}

// ---------------------------------------------------------------------------
// k_y_inv: T (rows, K, nz), ky < K nonzero -> rows x n(y) x nz real
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(YTHREADS) k_y_inv(const cd* __restrict__ T, int K, FftPlan p,
                                                    int nz, double scale, double* __restrict__ out,
                                                    int accumulate) {
  extern __shared__ cd sm[];
  const int n = p.n;
  const int h = n / 2;
  const int z0 = blockIdx.x * (2 * YC);
  const int row = blockIdx.y;
  cd* b0 = sm;
  cd* b1 = sm + n * YC;
  for (int t = threadIdx.x; t < (h + 1) * YC; t += blockDim.x) {
    const int k = t / YC, c = t % YC;
    const int z = z0 + 2 * c;
    cd A = make_double2(0.0, 0.0), B = make_double2(0.0, 0.0);
    if (k < K) {
      const size_t o = ((size_t)row * K + k) * nz + z;
      if (z < nz) A = T[o];
      if (z + 1 < nz) B = T[o + 1];
    }
    if (k == 0 || k == h) {
      A.y = 0.0;
      B.y = 0.0;
    }
    b0[k * YC + c] = make_double2(A.x - B.y, A.y + B.x);
    if (k > 0 && k < h) b0[(n - k) * YC + c] = make_double2(A.x + B.y, B.x - A.y);
  }
  const int r = fft_tile<+1>(b0, b1, p, YC);
  const cd* Z = r ? b1 : b0;
  for (int t = threadIdx.x; t < n * YC; t += blockDim.x) {
    const int y = t / YC, c = t % YC;
    const int z = z0 + 2 * c;
    const size_t o = ((size_t)row * n + y) * nz + z;
    const cd v = Z[t];
    if (accumulate) {
      if (z < nz) out[o] = out[o] + scale * v.x;
      if (z + 1 < nz) out[o + 1] = out[o + 1] + scale * v.y;
    } else {
      if (z < nz) out[o] = scale * v.x;
      if (z + 1 < nz) out[o + 1] = scale * v.y;
    }
  }
}

// ---------------------------------------------------------------------------
// k_x: per (ky, z run) column program
// ---------------------------------------------------------------------------
struct XArgs {
  const cd* src;
  int in_spec;   // 1: src is already a spectrum column set (no forward FFT)
  int rows_in, Kin, nz, C;
  FftPlan fwd;
  int nout;
  XOut out[3];
  const double* kx;
  const double* ky;
  int nx, mx, maxrows;
};

__device__ __forceinline__ cd map_value(const XArgs& a, const XOut& o, const cd* S, int k,
                                        int ky, int c, int C) {
  switch (o.map) {
    case MAP_IDENT:
      return S[k * C + c];
    case MAP_TRUNC: {
      const bool keep = (k < o.cx || k >= a.nx - o.cx + 1) && ky < o.cy;
      return keep ? S[k * C + c] : make_double2(0.0, 0.0);
    }
    case MAP_DX: {
      const cd v = S[k * C + c];
      const double q = a.kx[k];
      return make_double2(-(q * v.y), q * v.x);
    }
    case MAP_DY: {
      const cd v = S[k * C + c];
      const double q = a.ky[ky];
      return make_double2(-(q * v.y), q * v.x);
    }
    case MAP_PAD: {  // Dealiasing.py:67-73 (rows nx -> mx)
      const int h = a.nx / 2;
      if (k <= h) return S[k * C + c];
      if (k >= a.mx - h) return S[(k - a.mx + a.nx) * C + c];
      return make_double2(0.0, 0.0);
    }
    default: {  // MAP_UNPAD, Dealiasing.py:102-109 (rows mx -> nx)
      const int h = a.nx / 2;
      if (k < h) return S[k * C + c];
      if (k == h) return make_double2(0.0, 0.0);
      return S[(k - a.nx + a.mx) * C + c];
    }
  }
}

__global__ void __launch_bounds__(XTHREADS) k_x(XArgs a) {
  extern __shared__ cd sm[];
  const int C = a.C;
  const int nz = a.nz;
  const int z0 = blockIdx.x * C;
  const int ky = blockIdx.y;
  const int M = a.maxrows * C;
  cd* buf[3] = {sm, sm + M, sm + 2 * M};

  // load the input column set
  for (int t = threadIdx.x; t < a.rows_in * C; t += blockDim.x) {
    const int r = t / C, c = t % C;
    const int z = z0 + c;
    cd v = make_double2(0.0, 0.0);
    if (ky < a.Kin && z < nz) v = a.src[((size_t)r * a.Kin + ky) * nz + z];
    buf[0][t] = v;
  }
  int s = 0;
  if (!a.in_spec) {
    s = fft_tile<-1>(buf[0], buf[1], a.fwd, C);
  } else {
    __syncthreads();
  }
  const cd* S = buf[s];
  cd* f0 = buf[s == 0 ? 1 : 0];
  cd* f1 = buf[2];

  for (int oi = 0; oi < a.nout; oi++) {
    const XOut& o = a.out[oi];
    if (o.kind == XO_SPEC) {
      for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
        const int k = t / C, c = t % C;
        const int z = z0 + c;
        if (z < nz) o.dst[((size_t)k * o.K + ky) * nz + z] = map_value(a, o, S, k, ky, c, C);
      }
      continue;
    }
    if (ky >= o.K) continue;  // column not stored: zero by convention
    for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
      const int k = t / C, c = t % C;
      f0[t] = map_value(a, o, S, k, ky, c, C);
    }
    const int r = fft_tile<+1>(f0, f1, o.inv, C);
    const cd* R = r ? f1 : f0;
    for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
      const int k = t / C, c = t % C;
      const int z = z0 + c;
      if (z < nz) o.dst[((size_t)k * o.K + ky) * nz + z] = R[t];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static void set_smem(const void* f, size_t bytes) {
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

void launch_y_fwd(Engine& e, const Loader& L, int rows, const FftPlan& p, int K, cd* T) {
  const size_t smem = 2 * (size_t)p.n * YC * sizeof(cd);
  set_smem((const void*)k_y_fwd, smem);
  dim3 g((L.nz + 2 * YC - 1) / (2 * YC), rows);
  ::alfa::note_launch(); k_y_fwd<<<g, YTHREADS, smem, e.stream>>>(L, p, K, T);
}

void launch_y_inv(Engine& e, const cd* T, int rows, int K, const FftPlan& p, double scale,
                  double* out, int accumulate) {
  const size_t smem = 2 * (size_t)p.n * YC * sizeof(cd);
  set_smem((const void*)k_y_inv, smem);
  dim3 g((e.nz + 2 * YC - 1) / (2 * YC), rows);
  ::alfa::note_launch(); k_y_inv<<<g, YTHREADS, smem, e.stream>>>(T, K, p, e.nz, scale, out, accumulate);
}

void launch_x(Engine& e, const cd* src, int in_spec, int rows_in, int Kin, const FftPlan& fwd,
              int nout, const XOut* outs, int Kgrid) {
  XArgs a;
  a.src = src;
  a.in_spec = in_spec;
  a.rows_in = rows_in;
  a.Kin = Kin;
  a.nz = e.nz;
  a.fwd = fwd;
  a.nout = nout;
  int maxrows = rows_in;
  for (int i = 0; i < nout; i++) {
    a.out[i] = outs[i];
    if (outs[i].rows > maxrows) maxrows = outs[i].rows;
  }
  a.kx = e.d_kx;
  a.ky = e.d_ky;
  a.nx = e.nx;
  a.mx = e.mx;
  a.maxrows = maxrows;
  a.C = (3 * (size_t)maxrows * 8 * sizeof(cd) <= 100 * 1024) ? 8 : 4;
  const size_t smem = 3 * (size_t)maxrows * a.C * sizeof(cd);
  set_smem((const void*)k_x, smem);
  dim3 g((e.nz + a.C - 1) / a.C, Kgrid);
  ::alfa::note_launch(); k_x<<<g, XTHREADS, smem, e.stream>>>(a);
}

// ---------------------------------------------------------------------------
// composite operators
// ---------------------------------------------------------------------------
Loader ld_field(const Engine& e, const double* a) {
  Loader L{};
  L.kind = LD_FIELD;
  L.nz = e.nz;
  L.a[0] = a;
  return L;
}

static XOut xo_spec(const Engine& e, int map, cd* dst, int cx = 0, int cy = 0) {
  XOut o{};
  o.kind = XO_SPEC;
  o.map = map;
  o.cx = cx;
  o.cy = cy;
  o.K = e.nyh;
  o.rows = e.nx;
  o.dst = dst;
  return o;
}

static XOut xo_inv(int map, cd* dst, int rows, int K, const FftPlan& inv, int cx = 0,
                   int cy = 0) {
  XOut o{};
  o.kind = XO_INV;
  o.map = map;
  o.cx = cx;
  o.cy = cy;
  o.K = K;
  o.rows = rows;
  o.dst = dst;
  o.inv = inv;
  return o;
}

static double inv_scale(int a, int b) { return 1.0 / ((double)a * (double)b); }

// FFT.py:44 — rfft2 over axes (0, 1)
void op_rfft2(Engine& e, const Loader& L, cd* spec) {
  launch_y_fwd(e, L, e.nx, e.pny, e.nyh, e.T[0]);
  XOut o = xo_spec(e, MAP_IDENT, spec);
  launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
}

// FFT.py:68 — rfft2 of a padded field
void op_rfft2_pad(Engine& e, const Loader& L, cd* spec_pad) {
  launch_y_fwd(e, L, e.mx, e.pmy, e.myh, e.T[0]);
  XOut o{};
  o.kind = XO_SPEC;
  o.map = MAP_IDENT;
  o.K = e.myh;
  o.rows = e.mx;
  o.dst = spec_pad;
  launch_x(e, e.T[0], 0, e.mx, e.myh, e.pmx, 1, &o, e.myh);
}

// Filtering.py:50-89 applied to FFT(field)
void op_filter_explicit(Engine& e, const Loader& L, double* out, cd* spec) {
  const int cx = e.cut_e[0], cy = e.cut_e[1];
  launch_y_fwd(e, L, e.nx, e.pny, e.nyh, e.T[0]);
  XOut o[2] = {xo_spec(e, MAP_TRUNC, spec, cx, cy),
               xo_inv(MAP_TRUNC, e.T[1], e.nx, cy, e.pnx, cx, cy)};
  launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, 2, o, e.nyh);
  launch_y_inv(e, e.T[1], e.nx, cy, e.pny, inv_scale(e.nx, e.ny), out, 0);
}

// Filtering_Level1 / Level2 (Filtering.py:97-165) of one FFT(field)
void op_filter12(Engine& e, const Loader& L, double* out1, double* out2) {
  const int c1x = e.cut_1[0], c1y = e.cut_1[1], c2x = e.cut_2[0], c2y = e.cut_2[1];
  const int K = c1y > c2y ? c1y : c2y;
  launch_y_fwd(e, L, e.nx, e.pny, K, e.T[0]);
  XOut o[2] = {xo_inv(MAP_TRUNC, e.T[1], e.nx, c1y, e.pnx, c1x, c1y),
               xo_inv(MAP_TRUNC, e.T[2], e.nx, c2y, e.pnx, c2x, c2y)};
  launch_x(e, e.T[0], 0, e.nx, K, e.pnx, 2, o, K);
  launch_y_inv(e, e.T[1], e.nx, c1y, e.pny, inv_scale(e.nx, e.ny), out1, 0);
  launch_y_inv(e, e.T[2], e.nx, c2y, e.pny, inv_scale(e.nx, e.ny), out2, 0);
}

// one filter level of a given spectrum
void op_filter1_spec(Engine& e, const cd* spec, int level, double* out) {
  const int* cut = level == 1 ? e.cut_1 : e.cut_2;
  XOut o = xo_inv(MAP_TRUNC, e.T[1], e.nx, cut[1], e.pnx, cut[0], cut[1]);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, 1, &o, cut[1]);
  launch_y_inv(e, e.T[1], e.nx, cut[1], e.pny, inv_scale(e.nx, e.ny), out, 0);
}

// Derivxy (Derivatives.py:161-182) in x and/or y of a spectrum
void op_deriv_spec(Engine& e, const cd* spec, double* dx, double* dy) {
  XOut o[2];
  int n = 0;
  if (dx) o[n++] = xo_inv(MAP_DX, e.T[1], e.nx, e.nyh, e.pnx);
  if (dy) o[n++] = xo_inv(MAP_DY, e.T[2], e.nx, e.nyh, e.pnx);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, n, o, e.nyh);
  if (dx) launch_y_inv(e, e.T[1], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), dx, 0);
  if (dy) launch_y_inv(e, e.T[2], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), dy, 0);
}

// Derivxy(FFT(field)) in x and/or y
void op_deriv_field(Engine& e, const Loader& L, double* dx, double* dy) {
  launch_y_fwd(e, L, e.nx, e.pny, e.nyh, e.T[0]);
  XOut o[2];
  int n = 0;
  if (dx) o[n++] = xo_inv(MAP_DX, e.T[1], e.nx, e.nyh, e.pnx);
  if (dy) o[n++] = xo_inv(MAP_DY, e.T[2], e.nx, e.nyh, e.pnx);
  launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, n, o, e.nyh);
  if (dx) launch_y_inv(e, e.T[1], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), dx, 0);
  if (dy) launch_y_inv(e, e.T[2], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), dy, 0);
}

// Dealias1(FFT(field)) (Dealiasing.py:51-78)
void op_pad(Engine& e, const Loader& L, double* out_pad) {
  launch_y_fwd(e, L, e.nx, e.pny, e.nyh, e.T[0]);
  XOut o = xo_inv(MAP_PAD, e.T[1], e.mx, e.nyh, e.pmx);
  launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
  launch_y_inv(e, e.T[1], e.mx, e.nyh, e.pmy, inv_scale(e.mx, e.my), out_pad, 0);
}

// Dealias1(spectrum)
void op_pad_spec(Engine& e, const cd* spec, double* out_pad) {
  XOut o = xo_inv(MAP_PAD, e.T[1], e.mx, e.nyh, e.pmx);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
  launch_y_inv(e, e.T[1], e.mx, e.nyh, e.pmy, inv_scale(e.mx, e.my), out_pad, 0);
}

// Dealias2(FFT_pad(padded field)) (Dealiasing.py:86-114): keeps ky < ny/2,
// drops the x Nyquist row, rescales by 9/4.
void op_unpad(Engine& e, const Loader& L_pad, double* out) {
  const int K = e.nyh - 1;
  launch_y_fwd(e, L_pad, e.mx, e.pmy, K, e.T[0]);
  XOut o = xo_inv(MAP_UNPAD, e.T[1], e.nx, K, e.pnx);
  launch_x(e, e.T[0], 0, e.mx, K, e.pmx, 1, &o, K);
  launch_y_inv(e, e.T[1], e.nx, K, e.pny, (9.0 / 4.0) * inv_scale(e.nx, e.ny), out, 0);
}

// Dealias2(padded spectrum (mx, myh, nz))
void op_unpad_spec(Engine& e, const cd* spec_pad, double* out) {
  const int K = e.nyh - 1;
  XOut o = xo_inv(MAP_UNPAD, e.T[1], e.nx, K, e.pnx);
  launch_x(e, spec_pad, 1, e.mx, e.myh, e.pmx, 1, &o, K);
  launch_y_inv(e, e.T[1], e.nx, K, e.pny, (9.0 / 4.0) * inv_scale(e.nx, e.ny), out, 0);
}

// irfft2(spectrum, s=(nx, ny))
void op_irfft2(Engine& e, const cd* spec, double* out) {
  XOut o = xo_inv(MAP_IDENT, e.T[1], e.nx, e.nyh, e.pnx);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
  launch_y_inv(e, e.T[1], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), out, 0);
}

}  // namespace alfa
