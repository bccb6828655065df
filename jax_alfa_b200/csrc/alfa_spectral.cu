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
//
// Every tile kernel first issues all of a thread's global loads for a batch
// of U elements into registers and only then writes them to shared memory,
// so a thread keeps U loads in flight instead of waiting on each one.
#include <cmath>

#include "alfa_fft_ct.cuh"
#include "alfa_internal.cuh"

namespace alfa {

static constexpr int YC = 8;    // complex columns (= 16 real z levels) per y tile
static constexpr int MAXTHREADS = 384;  // in-place sweeps need C*n/16 threads
static constexpr int U = 8;     // loads in flight per thread

// ---------------------------------------------------------------------------
// Loader evaluation (value of the real input at linear index i, level z);
// the kind is a compile-time constant in the tile kernels.
// ---------------------------------------------------------------------------
template <int KIND>
__device__ __forceinline__ double ldv(const Loader& L, size_t i, int z) {
  const int nz = L.nz;
  if constexpr (KIND == LD_FIELD) {
    return L.a[0][i];
  } else if constexpr (KIND == LD_MUL) {
    return L.a[0][i] * L.a[1][i];
  } else if constexpr (KIND == LD_MUL3) {
    return L.a[0][i] * L.a[1][i] * L.a[2][i];
  } else if constexpr (KIND == LD_PRESSURE_R) {  // NSE_PressureTerms.py:140-142
    return L.a[0][i] - L.c[0] * L.a[1][i] + L.c[1] * L.a[2][i];
  } else if constexpr (KIND == LD_ADV_XY) {  // NSE_AdvectionTerms.py:105-116, :122-132
    const double arg1 = L.a[0][i] * (L.a[1][i] - L.a[2][i]);
    if (z == 0) {
      const double a2n = L.a[3][i + 1] * (L.a[4][i + 1] - L.a[5][i + 1]);
      return arg1 + 0.5 * a2n;
    }
    const double a2 = L.a[3][i] * (L.a[4][i] - L.a[5][i]);
    if (z == nz - 1) return arg1 + a2;
    const double a2n = L.a[3][i + 1] * (L.a[4][i + 1] - L.a[5][i + 1]);
    return arg1 + 0.5 * (a2 + a2n);
  } else if constexpr (KIND == LD_ADV_Z) {  // NSE_AdvectionTerms.py:137-151
    if (z == 0 || z == nz - 1) return 0.0;
    const double ug = 0.5 * (L.a[0][i - 1] + L.a[0][i]);
    const double vg = 0.5 * (L.a[1][i - 1] + L.a[1][i]);
    const double a1 = ug * (L.a[2][i] - L.a[3][i]);
    const double a2 = vg * (L.a[4][i] - L.a[5][i]);
    return a1 + a2;
  } else if constexpr (KIND == LD_SCALAR_ADV) {  // SCL_AdvectionTerms.py:89-101
    const double c1 = L.a[0][i] * L.a[3][i] + L.a[1][i] * L.a[4][i];
    const double c2 = L.a[2][i] * L.a[5][i];
    if (z == nz - 1) return c1 + c2;
    const double c2n = L.a[2][i + 1] * L.a[5][i + 1];
    return c1 + 0.5 * (c2 + c2n);
  } else if constexpr (KIND == LD_STRESS_UVP) {  // SGSStresses_SM.py:122-132
    if (z == nz - 1) return 0.0;
    return L.c[0] * L.a[0][i] * L.a[1][i] * L.a[2][i];
  } else if constexpr (KIND == LD_STRESS_W) {  // SGSStresses_SM.py:223-232
    if (z == 0 || z == nz - 1) return 0.0;
    return L.c[0] * (0.5 * (L.a[0][i - 1] + L.a[0][i])) * L.a[1][i] * L.a[2][i];
  } else if constexpr (KIND == LD_W_SXX) {  // StrainRates.py:250-276, component L.sub
    const double* const* g = L.a;  // dudx dvdx dwdx dudy dvdy dwdy dudz dvdz dwdz
    auto stag = [&](const double* d) -> double {
      if (z == 0) return d[i];
      if (z == nz - 1) return 0.0;
      return 0.5 * (d[i - 1] + d[i]);
    };
    switch (L.sub) {
      case 0: return stag(g[0]);                       // S11 = ux
      case 1: return stag(g[4]);                       // S22 = vy
      case 2: return stag(g[8]);                       // S33 = wz
      case 3: return 0.5 * (stag(g[3]) + stag(g[1]));  // S12
      case 4: {                                        // S13
        const double wx = (z == 0) ? 0.5 * (g[2][i] + g[2][i + 1]) : g[2][i];
        return 0.5 * (g[6][i] + wx);
      }
      default: {                                       // S23
        const double wy = (z == 0) ? 0.5 * (g[5][i] + g[5][i + 1]) : g[5][i];
        return 0.5 * (g[7][i] + wy);
      }
    }
  } else if constexpr (KIND == LD_THZ) {  // DynamicSGS_ScalarLASDD_SM.py:182-185
    const double* d = L.a[0];
    if (z == 0 || z == nz - 1) return d[i];
    return 0.5 * (d[i] + d[i + 1]);
  } else {  // LD_MUL_THZ: S * THz
    const double* d = L.a[1];
    const double t = (z == 0 || z == nz - 1) ? d[i] : 0.5 * (d[i] + d[i + 1]);
    return L.a[0][i] * t;
  }
}

// Load the (n x 16 z) real tile of row `row` into b0 as n x 8 complex
// (z pairs), U elements per thread in flight.
template <int KIND>
__device__ __forceinline__ void y_fwd_load(const Loader& L, int row, int n, int z0, cd* b0) {
  const int nz = L.nz;
  const int total = n * YC;
  const bool vec = (KIND == LD_FIELD) && ((nz & 1) == 0);
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    cd v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      v[u] = make_double2(0.0, 0.0);
      if (t < total) {
        const int y = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t i = ((size_t)row * n + y) * nz + z;
        if (vec && z + 1 < nz) {
          v[u] = __ldg(reinterpret_cast<const double2*>(L.a[0] + i));
        } else {
          if (z < nz) v[u].x = ldv<KIND>(L, i, z);
          if (z + 1 < nz) v[u].y = ldv<KIND>(L, i + 1, z + 1);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < total) b0[t] = v[u];
    }
  }
}

// Transform of an n x C tile: compile-time specialised for the lengths in
// the dispatch tables below (N > 0), the runtime plan otherwise (N == 0).
template <int S, int C, int N, int NT>
__device__ __forceinline__ void tile_fft(cd* buf, const FftPlan& p) {
  if constexpr (N == 0) {
    fft_inplace<S, C>(buf, p);
  } else {
    fft_ct<S, C, N, NT>(buf, p.tw);
  }
}

template <int C, int N>
__host__ __device__ constexpr int tile_threads() {
  return N == 0 ? MAXTHREADS : ct_threads(C, N);
}

// ---------------------------------------------------------------------------
// k_y_fwd: rows x n(y) x nz real -> T (rows, K, nz) complex, ky < K
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(tile_threads<YC, N>(), 1)
    k_y_fwd(Loader L, FftPlan p, int K, cd* __restrict__ T) {
  extern __shared__ cd sm[];
  const int n = (N > 0) ? N : p.n;
  const int nz = L.nz;
  const int z0 = blockIdx.x * (2 * YC);
  const int row = blockIdx.y;
  cd* b0 = sm;
  switch (L.kind) {
    case LD_FIELD: y_fwd_load<LD_FIELD>(L, row, n, z0, b0); break;
    case LD_MUL: y_fwd_load<LD_MUL>(L, row, n, z0, b0); break;
    case LD_MUL3: y_fwd_load<LD_MUL3>(L, row, n, z0, b0); break;
    case LD_PRESSURE_R: y_fwd_load<LD_PRESSURE_R>(L, row, n, z0, b0); break;
    case LD_ADV_XY: y_fwd_load<LD_ADV_XY>(L, row, n, z0, b0); break;
    case LD_ADV_Z: y_fwd_load<LD_ADV_Z>(L, row, n, z0, b0); break;
    case LD_SCALAR_ADV: y_fwd_load<LD_SCALAR_ADV>(L, row, n, z0, b0); break;
    case LD_STRESS_UVP: y_fwd_load<LD_STRESS_UVP>(L, row, n, z0, b0); break;
    case LD_STRESS_W: y_fwd_load<LD_STRESS_W>(L, row, n, z0, b0); break;
    case LD_W_SXX: y_fwd_load<LD_W_SXX>(L, row, n, z0, b0); break;
    case LD_THZ: y_fwd_load<LD_THZ>(L, row, n, z0, b0); break;
    default: y_fwd_load<LD_MUL_THZ>(L, row, n, z0, b0); break;
  }
  tile_fft<-1, YC, N, tile_threads<YC, N>()>(b0, p);
  const cd* Z = b0;
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
template <int N>
__global__ void __launch_bounds__(tile_threads<YC, N>(), 1)
    k_y_inv(const cd* __restrict__ T, int K, FftPlan p, int nz, double scale,
            double* __restrict__ out, int accumulate) {
  extern __shared__ cd sm[];
  const int n = (N > 0) ? N : p.n;
  const int h = n / 2;
  const int z0 = blockIdx.x * (2 * YC);
  const int row = blockIdx.y;
  cd* b0 = sm;
  const int total = (h + 1) * YC;
  const bool pair = (nz & 1) == 0;  // z, z+1 both present whenever z is
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    cd A[U], B[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      A[u] = make_double2(0.0, 0.0);
      B[u] = make_double2(0.0, 0.0);
      const int k = t / YC, c = t % YC;
      const int z = z0 + 2 * c;
      if (t < total && k < K) {
        const size_t o = ((size_t)row * K + k) * nz + z;
        if (pair && z < nz) {
          A[u] = __ldg(T + o);
          B[u] = __ldg(T + o + 1);
        } else {
          if (z < nz) A[u] = T[o];
          if (z + 1 < nz) B[u] = T[o + 1];
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      if (t >= total) continue;
      const int k = t / YC, c = t % YC;
      cd a = A[u], b = B[u];
      if (k == 0 || k == h) {
        a.y = 0.0;
        b.y = 0.0;
      }
      b0[k * YC + c] = make_double2(a.x - b.y, a.y + b.x);
      if (k > 0 && k < h) b0[(n - k) * YC + c] = make_double2(a.x + b.y, b.x - a.y);
    }
  }
  tile_fft<+1, YC, N, tile_threads<YC, N>()>(b0, p);
  const cd* Z = b0;
  if (accumulate) {
    for (int t0 = threadIdx.x; t0 < n * YC; t0 += U * blockDim.x) {
      double2 prev[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int t = t0 + u * blockDim.x;
        const int y = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t o = ((size_t)row * n + y) * nz + z;
        prev[u] = make_double2(0.0, 0.0);
        if (t < n * YC) {
          if (pair && z < nz) {
            prev[u] = *reinterpret_cast<const double2*>(out + o);
          } else {
            if (z < nz) prev[u].x = out[o];
            if (z + 1 < nz) prev[u].y = out[o + 1];
          }
        }
      }
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int t = t0 + u * blockDim.x;
        if (t >= n * YC) continue;
        const int y = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t o = ((size_t)row * n + y) * nz + z;
        const cd v = Z[t];
        const double2 w = make_double2(prev[u].x + scale * v.x, prev[u].y + scale * v.y);
        if (pair && z < nz) {
          *reinterpret_cast<double2*>(out + o) = w;
        } else {
          if (z < nz) out[o] = w.x;
          if (z + 1 < nz) out[o + 1] = w.y;
        }
      }
    }
  } else {
    for (int t = threadIdx.x; t < n * YC; t += blockDim.x) {
      const int y = t / YC, c = t % YC;
      const int z = z0 + 2 * c;
      const size_t o = ((size_t)row * n + y) * nz + z;
      const cd v = Z[t];
      if (pair && z < nz) {
        *reinterpret_cast<double2*>(out + o) = make_double2(scale * v.x, scale * v.y);
      } else {
        if (z < nz) out[o] = scale * v.x;
        if (z + 1 < nz) out[o + 1] = scale * v.y;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// k_x: per (ky, z run) column program
// ---------------------------------------------------------------------------
struct XArgs {
  const cd* src;
  int in_spec;   // 1: src is already a spectrum column set (no forward FFT)
  int rows_in, Kin, nz;
  FftPlan fwd;
  int nout;
  XOut out[3];
  const double* kx;
  const double* ky;
  int nx, mx, maxrows;
};

template <int C>
__device__ __forceinline__ cd map_value(const XArgs& a, const XOut& o, const cd* S, int k, int ky,
                                        int c) {
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

// NI / NO: compile-time forward / inverse lengths (0: runtime plans)
template <int C, int NI, int NO>
__global__ void __launch_bounds__(tile_threads<C, (NI > NO ? NI : NO)>(), 1) k_x(XArgs a) {
  constexpr int NT = tile_threads<C, (NI > NO ? NI : NO)>();
  extern __shared__ cd sm[];
  const int nz = a.nz;
  const int z0 = blockIdx.x * C;
  const int ky = blockIdx.y;
  const int M = a.maxrows * C;
  cd* buf[2] = {sm, sm + M};

  // load the input column set, U loads in flight per thread
  const int total = a.rows_in * C;
  const bool have = ky < a.Kin;
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    cd v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      const int r = t / C, c = t % C;
      const int z = z0 + c;
      v[u] = make_double2(0.0, 0.0);
      if (have && t < total && z < nz) v[u] = __ldg(&a.src[((size_t)r * a.Kin + ky) * nz + z]);
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < total) buf[0][t] = v[u];
    }
  }
  if (!a.in_spec) {
    tile_fft<-1, C, NI, NT>(buf[0], a.fwd);
  } else {
    __syncthreads();
  }
  const cd* S = buf[0];
  cd* f0 = buf[1];

  for (int oi = 0; oi < a.nout; oi++) {
    const XOut& o = a.out[oi];
    if (o.kind == XO_SPEC) {
      for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
        const int k = t / C, c = t % C;
        const int z = z0 + c;
        if (z < nz) o.dst[((size_t)k * o.K + ky) * nz + z] = map_value<C>(a, o, S, k, ky, c);
      }
      continue;
    }
    if (ky >= o.K) continue;  // column not stored: zero by convention
    for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
      const int k = t / C, c = t % C;
      f0[t] = map_value<C>(a, o, S, k, ky, c);
    }
    tile_fft<+1, C, NO, NT>(f0, o.inv);
    const cd* R = f0;
    for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
      const int k = t / C, c = t % C;
      const int z = z0 + c;
      if (z < nz) o.dst[((size_t)k * o.K + ky) * nz + z] = R[t];
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// launchers (dispatch to the specialised lengths)
// ---------------------------------------------------------------------------
static void set_smem(const void* f, size_t bytes) {
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

#define ALFA_Y_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) \
  X(512) X(768)

template <int N>
static void y_fwd_n(Engine& e, const Loader& L, int rows, const FftPlan& p, int K, cd* T) {
  const size_t smem = (size_t)p.n * YC * sizeof(cd);
  set_smem((const void*)k_y_fwd<N>, smem);
  dim3 g((L.nz + 2 * YC - 1) / (2 * YC), rows);
  const int nt = N > 0 ? tile_threads<YC, N>() : inplace_threads(YC, p.n);
  k_y_fwd<N><<<g, nt, smem, e.stream>>>(L, p, K, T);
}

template <int N>
static void y_inv_n(Engine& e, const cd* T, int rows, int K, const FftPlan& p, double scale,
                    double* out, int accumulate) {
  const size_t smem = (size_t)p.n * YC * sizeof(cd);
  set_smem((const void*)k_y_inv<N>, smem);
  dim3 g((e.nz + 2 * YC - 1) / (2 * YC), rows);
  const int nt = N > 0 ? tile_threads<YC, N>() : inplace_threads(YC, p.n);
  k_y_inv<N><<<g, nt, smem, e.stream>>>(T, K, p, e.nz, scale, out, accumulate);
}

void launch_y_fwd(Engine& e, const Loader& L, int rows, const FftPlan& p, int K, cd* T) {
  ::alfa::note_launch();
  switch (p.n) {
#define ALFA_CASE(n) \
  case n: y_fwd_n<n>(e, L, rows, p, K, T); return;
    ALFA_Y_LENGTHS(ALFA_CASE)
#undef ALFA_CASE
    default: y_fwd_n<0>(e, L, rows, p, K, T);
  }
}

void launch_y_inv(Engine& e, const cd* T, int rows, int K, const FftPlan& p, double scale,
                  double* out, int accumulate) {
  ::alfa::note_launch();
  switch (p.n) {
#define ALFA_CASE(n) \
  case n: y_inv_n<n>(e, T, rows, K, p, scale, out, accumulate); return;
    ALFA_Y_LENGTHS(ALFA_CASE)
#undef ALFA_CASE
    default: y_inv_n<0>(e, T, rows, K, p, scale, out, accumulate);
  }
}

template <int C, int NI, int NO>
static void x_n(Engine& e, const XArgs& a, int Kgrid) {
  const size_t smem = 2 * (size_t)a.maxrows * C * sizeof(cd);
  set_smem((const void*)k_x<C, NI, NO>, smem);
  dim3 g((e.nz + C - 1) / C, Kgrid);
  const int nt = (NI > 0) ? tile_threads<C, (NI > NO ? NI : NO)>() : inplace_threads(C, a.maxrows);
  k_x<C, NI, NO><<<g, nt, smem, e.stream>>>(a);
}

// (forward length, inverse length) pairs with a specialised k_x
#define ALFA_X_PAIRS(X) X(16, 16) X(16, 24) X(24, 16) X(24, 24) X(32, 32) X(32, 48) X(48, 32) \
  X(48, 48) X(64, 64) X(64, 96) X(96, 64) X(96, 96) X(128, 128) X(128, 192) X(192, 128)         \
  X(192, 192) X(256, 256) X(256, 384) X(384, 256) X(384, 384)

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
  int ninv = 0;
  bool same_inv = true;
  for (int i = 0; i < nout; i++) {
    a.out[i] = outs[i];
    if (outs[i].rows > maxrows) maxrows = outs[i].rows;
    if (outs[i].kind == XO_INV) {
      if (ninv != 0 && outs[i].inv.n != ninv) same_inv = false;
      ninv = outs[i].inv.n;
    }
  }
  if (ninv == 0) ninv = rows_in;
  a.kx = e.d_kx;
  a.ky = e.d_ky;
  a.nx = e.nx;
  a.mx = e.mx;
  a.maxrows = maxrows;
  ::alfa::note_launch();
  const int ni = in_spec ? ninv : rows_in;  // no forward transform: only the inverse length matters
  if (same_inv) {
#define ALFA_CASE(p, q)                                        \
  if (ni == p && ninv == q) {                                  \
    if ((p > q ? p : q) <= 256) x_n<8, p, q>(e, a, Kgrid);     \
    else x_n<4, p, q>(e, a, Kgrid);                            \
    return;                                                    \
  }
    ALFA_X_PAIRS(ALFA_CASE)
#undef ALFA_CASE
  }
  if (maxrows <= 256) x_n<8, 0, 0>(e, a, Kgrid);
  else x_n<4, 0, 0>(e, a, Kgrid);
}

// ---------------------------------------------------------------------------
// k_line: 1-D spectral operator along x or y on real fields.  A CTA takes one
// line index f (an x row for y lines, a y column for x lines) and 16
// consecutive z levels packed as 8 complex lines, transforms them forward,
// and for each output applies a map to the full packed spectrum, transforms
// back and stores the real pair.  Packing two real lines in one complex
// transform is exact for these maps because each is a real operator
// (Hermitian-symmetric: truncation, i*k with the Nyquist zeroed, the 3/2-rule
// pad with the Nyquist repeated, unpad).
// ---------------------------------------------------------------------------
struct LineArgs {
  Loader L;
  int n_in, n_out;
  long long fs_in, rs_in, fs_out, rs_out;  // line and row strides (elements)
  int nz;
  int nouts;
  LineOut out[3];
  FftPlan pin, pout;
};

template <int KIND>
__device__ __forceinline__ void line_load(const LineArgs& a, long long f, int z0, int n, cd* S) {
  const Loader& L = a.L;
  const int nz = a.nz;
  const int total = n * YC;
  const bool vec = (KIND == LD_FIELD) && ((nz & 1) == 0);
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    cd v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      v[u] = make_double2(0.0, 0.0);
      if (t < total) {
        const int r = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t i = (size_t)(f * a.fs_in + r * a.rs_in) + z;
        if (vec && z + 1 < nz) {
          v[u] = __ldg(reinterpret_cast<const double2*>(L.a[0] + i));
        } else {
          if (z < nz) v[u].x = ldv<KIND>(L, i, z);
          if (z + 1 < nz) v[u].y = ldv<KIND>(L, i + 1, z + 1);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      if (t < total) S[t] = v[u];
    }
  }
}

__device__ __forceinline__ cd line_map(const LineOut& o, const cd* S, int k, int c, int n, int m) {
  auto deriv = [&](cd v) -> cd {
    const int kk = (k < n / 2) ? k : (k == n / 2 ? 0 : k - n);
    const double q = (double)kk;
    return make_double2(-(q * v.y), q * v.x);
  };
  switch (o.map) {
    case LM_IDENT:
      return S[k * YC + c];
    case LM_TRUNC:
      return (k < o.cut || k >= n - o.cut + 1) ? S[k * YC + c] : make_double2(0.0, 0.0);
    case LM_DERIV:
      return deriv(S[k * YC + c]);
    case LM_TRUNC_DERIV:
      return (k < o.cut || k >= n - o.cut + 1) ? deriv(S[k * YC + c]) : make_double2(0.0, 0.0);
    case LM_PAD: {  // n -> m = 3n/2, Nyquist row repeated (Dealiasing.py:67-73)
      const int h = n / 2;
      if (k <= h) return S[k * YC + c];
      if (k >= m - h) return S[(k - m + n) * YC + c];
      return make_double2(0.0, 0.0);
    }
    default: {  // LM_UNPAD: n = 3m/2 -> m, Nyquist dropped (Dealiasing.py:102-109)
      const int h = m / 2;
      if (k < h) return S[k * YC + c];
      if (k == h) return make_double2(0.0, 0.0);
      return S[(k - m + n) * YC + c];
    }
  }
}

template <int NIN, int NOUT>
__global__ void __launch_bounds__(tile_threads<YC, (NIN > NOUT ? NIN : NOUT)>(), 1)
    k_line(LineArgs a) {
  constexpr int NT = tile_threads<YC, (NIN > NOUT ? NIN : NOUT)>();
  extern __shared__ cd sm[];
  const int n = NIN > 0 ? NIN : a.n_in;
  const int m = NOUT > 0 ? NOUT : a.n_out;
  const int nz = a.nz;
  const int z0 = blockIdx.x * (2 * YC);
  const long long f = blockIdx.y;
  cd* S = sm;
  cd* W = sm + n * YC;
  switch (a.L.kind) {
    case LD_FIELD: line_load<LD_FIELD>(a, f, z0, n, S); break;
    case LD_MUL: line_load<LD_MUL>(a, f, z0, n, S); break;
    case LD_MUL3: line_load<LD_MUL3>(a, f, z0, n, S); break;
    case LD_PRESSURE_R: line_load<LD_PRESSURE_R>(a, f, z0, n, S); break;
    case LD_ADV_XY: line_load<LD_ADV_XY>(a, f, z0, n, S); break;
    case LD_ADV_Z: line_load<LD_ADV_Z>(a, f, z0, n, S); break;
    case LD_SCALAR_ADV: line_load<LD_SCALAR_ADV>(a, f, z0, n, S); break;
    case LD_STRESS_UVP: line_load<LD_STRESS_UVP>(a, f, z0, n, S); break;
    case LD_STRESS_W: line_load<LD_STRESS_W>(a, f, z0, n, S); break;
    case LD_W_SXX: line_load<LD_W_SXX>(a, f, z0, n, S); break;
    case LD_THZ: line_load<LD_THZ>(a, f, z0, n, S); break;
    default: line_load<LD_MUL_THZ>(a, f, z0, n, S); break;
  }
  tile_fft<-1, YC, NIN, NT>(S, a.pin);
  const bool pair = (nz & 1) == 0;
  for (int oi = 0; oi < a.nouts; oi++) {
    const LineOut& o = a.out[oi];
    for (int t = threadIdx.x; t < m * YC; t += blockDim.x) {
      const int k = t / YC, c = t % YC;
      W[t] = line_map(o, S, k, c, n, m);
    }
    tile_fft<+1, YC, NOUT, NT>(W, a.pout);
    const double sc = o.scale;
    if (o.accumulate) {
      for (int t0 = threadIdx.x; t0 < m * YC; t0 += U * blockDim.x) {
        double2 prev[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int t = t0 + u * blockDim.x;
          const int r = t / YC, c = t % YC;
          const int z = z0 + 2 * c;
          const size_t i = (size_t)(f * a.fs_out + r * a.rs_out) + z;
          prev[u] = make_double2(0.0, 0.0);
          if (t < m * YC) {
            if (pair && z < nz) {
              prev[u] = *reinterpret_cast<const double2*>(o.dst + i);
            } else {
              if (z < nz) prev[u].x = o.dst[i];
              if (z + 1 < nz) prev[u].y = o.dst[i + 1];
            }
          }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int t = t0 + u * blockDim.x;
          if (t >= m * YC) continue;
          const int r = t / YC, c = t % YC;
          const int z = z0 + 2 * c;
          const size_t i = (size_t)(f * a.fs_out + r * a.rs_out) + z;
          const cd v = W[t];
          const double2 w = make_double2(prev[u].x + sc * v.x, prev[u].y + sc * v.y);
          if (pair && z < nz) {
            *reinterpret_cast<double2*>(o.dst + i) = w;
          } else {
            if (z < nz) o.dst[i] = w.x;
            if (z + 1 < nz) o.dst[i + 1] = w.y;
          }
        }
      }
    } else {
      for (int t = threadIdx.x; t < m * YC; t += blockDim.x) {
        const int r = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t i = (size_t)(f * a.fs_out + r * a.rs_out) + z;
        const cd v = W[t];
        if (pair && z < nz) {
          *reinterpret_cast<double2*>(o.dst + i) = make_double2(sc * v.x, sc * v.y);
        } else {
          if (z < nz) o.dst[i] = sc * v.x;
          if (z + 1 < nz) o.dst[i + 1] = sc * v.y;
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// k_line_rr: k_line for compile-time lengths with register-resident ends.
// The forward transform's first pass takes its inputs straight from global
// memory (every thread issues all of its loads before the first butterfly);
// each output's inverse transform reads its first-pass inputs from the
// forward spectrum through the map, and its last pass stores straight from
// registers.  Shared memory holds the forward spectrum and the inverse's
// intermediate passes only.  GEN: the input is any Loader kind (else a
// plain field, with a leaner register budget).
// ---------------------------------------------------------------------------
template <int C, int NIN, int NOUT>
__host__ __device__ constexpr int line_threads() {
  return ct_threads(C, NIN) > ct_threads(C, NOUT) ? ct_threads(C, NIN) : ct_threads(C, NOUT);
}

// first-pass gather: v[q*R + r] = (x, x') at row j + r*NR of line c
template <int KIND, int C, int N, int NT>
__device__ __forceinline__ void line_gather(const LineArgs& a, long long f, int z0, cd* v) {
  constexpr int R = ct_radix(N);
  constexpr int NR = N / R;
  constexpr int B = NR * C;
  constexpr int MB = (B + NT - 1) / NT;
  const Loader& L = a.L;
  const int nz = a.nz;
  const bool vec = (KIND == LD_FIELD) && ((nz & 1) == 0);
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 2 * c;
    const bool ok = (B % NT == 0 || b < B);
#pragma unroll
    for (int r = 0; r < R; r++) {
      const size_t i = (size_t)(f * a.fs_in + (long long)(j + r * NR) * a.rs_in) + z;
      cd t = make_double2(0.0, 0.0);
      if (ok) {
        if (vec && z + 1 < nz) {
          t = __ldg(reinterpret_cast<const double2*>(L.a[0] + i));
        } else {
          if (z < nz) t.x = ldv<KIND>(L, i, z);
          if (z + 1 < nz) t.y = ldv<KIND>(L, i + 1, z + 1);
        }
      }
      v[q * R + r] = t;
    }
  }
}

// store (or accumulate) v[q*R + r] = value at row j + r*STEP of line c
template <int C, int R, int STEP, int B, int NT>
__device__ __forceinline__ void line_scatter(const LineArgs& a, const LineOut& o, long long f,
                                             int z0, const cd* v) {
  constexpr int MB = (B + NT - 1) / NT;
  const int nz = a.nz;
  const bool pair = (nz & 1) == 0;
  const double sc = o.scale;
  double* __restrict__ dst = o.dst;
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (!(B % NT == 0 || b < B)) continue;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 2 * c;
    if (z >= nz) continue;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const size_t i = (size_t)(f * a.fs_out + (long long)(j + r * STEP) * a.rs_out) + z;
      double2 w = make_double2(sc * v[q * R + r].x, sc * v[q * R + r].y);
      if (pair) {
        double2* p = reinterpret_cast<double2*>(dst + i);
        if (o.accumulate) {
          const double2 pv = *p;
          w.x += pv.x;
          w.y += pv.y;
        }
        *p = w;
      } else {
        if (o.accumulate) {
          w.x += dst[i];
          if (z + 1 < nz) w.y += dst[i + 1];
        }
        dst[i] = w.x;
        if (z + 1 < nz) dst[i + 1] = w.y;
      }
    }
  }
}

template <int NIN, int NOUT, bool GEN>
__global__ void __launch_bounds__(line_threads<YC, NIN, NOUT>())
    k_line_rr(LineArgs a) {
  constexpr int C = YC;
  constexpr int NT = line_threads<C, NIN, NOUT>();
  constexpr int NMAX = NIN > NOUT ? NIN : NOUT;
  extern __shared__ cd sm[];
  cd* S = sm;
  cd* Wb = a.nouts > 1 ? sm + NMAX * C : sm;
  const int z0 = blockIdx.x * (2 * C);
  const long long f = blockIdx.y;
  // forward transform of the NIN-line tile into S
  {
    constexpr int R = ct_radix(NIN);
    constexpr int MB = ct_mb(C, NIN, 1, NT);
    cd v[MB * R];
    if constexpr (GEN) {
      switch (a.L.kind) {
        case LD_FIELD: line_gather<LD_FIELD, C, NIN, NT>(a, f, z0, v); break;
        case LD_MUL: line_gather<LD_MUL, C, NIN, NT>(a, f, z0, v); break;
        case LD_MUL3: line_gather<LD_MUL3, C, NIN, NT>(a, f, z0, v); break;
        case LD_PRESSURE_R: line_gather<LD_PRESSURE_R, C, NIN, NT>(a, f, z0, v); break;
        case LD_ADV_XY: line_gather<LD_ADV_XY, C, NIN, NT>(a, f, z0, v); break;
        case LD_ADV_Z: line_gather<LD_ADV_Z, C, NIN, NT>(a, f, z0, v); break;
        case LD_SCALAR_ADV: line_gather<LD_SCALAR_ADV, C, NIN, NT>(a, f, z0, v); break;
        case LD_STRESS_UVP: line_gather<LD_STRESS_UVP, C, NIN, NT>(a, f, z0, v); break;
        case LD_STRESS_W: line_gather<LD_STRESS_W, C, NIN, NT>(a, f, z0, v); break;
        case LD_W_SXX: line_gather<LD_W_SXX, C, NIN, NT>(a, f, z0, v); break;
        case LD_THZ: line_gather<LD_THZ, C, NIN, NT>(a, f, z0, v); break;
        default: line_gather<LD_MUL_THZ, C, NIN, NT>(a, f, z0, v); break;
      }
    } else {
      line_gather<LD_FIELD, C, NIN, NT>(a, f, z0, v);
    }
    if constexpr (R == NIN) {
      if (threadIdx.x < C) {
        dftR<R, -1>(v);
#pragma unroll
        for (int r = 0; r < R; r++) S[r * C + threadIdx.x] = v[r];
      }
    } else {
      ct_first_reg<-1, C, NIN, NT>(v, S);
      ct_passes<-1, C, NIN, R, NT>(S, a.pin.tw);
    }
    __syncthreads();
  }
  // outputs: map, inverse transform, store
  for (int oi = 0; oi < a.nouts; oi++) {
    const LineOut& o = a.out[oi];
    constexpr int R = ct_radix(NOUT);
    constexpr int NR = NOUT / R;
    constexpr int B = NR * C;
    constexpr int MB = ct_mb(C, NOUT, 1, NT);
    cd v[MB * R];
#pragma unroll
    for (int q = 0; q < MB; q++) {
      const int b = threadIdx.x + q * NT;
      const int c = b % C;
      const int j = b / C;
#pragma unroll
      for (int r = 0; r < R; r++)
        v[q * R + r] = (B % NT == 0 || b < B) ? line_map(o, S, j + r * NR, c, NIN, NOUT)
                                              : make_double2(0.0, 0.0);
    }
    if constexpr (R == NOUT) {
#pragma unroll
      for (int q = 0; q < MB; q++) dftR<R, +1>(v + q * R);
      line_scatter<C, R, 1, C, NT>(a, o, f, z0, v);
    } else {
      __syncthreads();  // Wb may alias S
      ct_first_reg<+1, C, NOUT, NT>(v, Wb);
      ct_mid_passes<+1, C, NOUT, R, NT>(Wb, a.pout.tw);
      __syncthreads();
      constexpr int NSL = ct_last_ns(NOUT);
      constexpr int RL = NOUT / NSL;
      constexpr int ML = ct_mb(C, NOUT, NSL, NT);
      cd u[ML * RL];
      ct_last_reg<+1, C, NOUT, NT>(Wb, a.pout.tw, u);
      line_scatter<C, RL, NSL, NSL * C, NT>(a, o, f, z0, u);
    }
    __syncthreads();
  }
}

template <int NIN, int NOUT>
static void line_n(Engine& e, const LineArgs& a, int F) {
  dim3 g((a.nz + 2 * YC - 1) / (2 * YC), F);
  if constexpr (NIN > 0) {
    const int nmax = NIN > NOUT ? NIN : NOUT;
    const size_t smem = (size_t)(nmax + (a.nouts > 1 ? NOUT : 0)) * YC * sizeof(cd);
    constexpr int nt = line_threads<YC, NIN, NOUT>();
    if (a.L.kind == LD_FIELD) {
      set_smem((const void*)k_line_rr<NIN, NOUT, false>, smem);
      k_line_rr<NIN, NOUT, false><<<g, nt, smem, e.stream>>>(a);
    } else {
      set_smem((const void*)k_line_rr<NIN, NOUT, true>, smem);
      k_line_rr<NIN, NOUT, true><<<g, nt, smem, e.stream>>>(a);
    }
  } else {
    const size_t smem = (size_t)(a.n_in + a.n_out) * YC * sizeof(cd);
    set_smem((const void*)k_line<0, 0>, smem);
    const int nt = inplace_threads(YC, a.n_in > a.n_out ? a.n_in : a.n_out);
    k_line<0, 0><<<g, nt, smem, e.stream>>>(a);
  }
}

static const FftPlan& plan_for(const Engine& e, int n) {
  if (n == e.nx) return e.pnx;
  if (n == e.ny) return e.pny;
  if (n == e.mx) return e.pmx;
  return e.pmy;
}

void launch_line(Engine& e, int axis, const Loader& L, int X, int Y, int n_in, int n_out,
                 int nout, const LineOut* outs) {
  LineArgs a;
  a.L = L;
  a.n_in = n_in;
  a.n_out = n_out;
  a.nz = L.nz;
  const long long nz = L.nz;
  int F;
  if (axis == 0) {  // x lines of (X=n_in, Y, nz) -> (n_out, Y, nz)
    a.fs_in = nz;
    a.rs_in = (long long)Y * nz;
    a.fs_out = nz;
    a.rs_out = (long long)Y * nz;
    F = Y;
  } else {  // y lines of (X, Y=n_in, nz) -> (X, n_out, nz)
    a.fs_in = (long long)n_in * nz;
    a.rs_in = nz;
    a.fs_out = (long long)n_out * nz;
    a.rs_out = nz;
    F = X;
  }
  a.nouts = nout;
  for (int i = 0; i < nout; i++) a.out[i] = outs[i];
  a.pin = plan_for(e, n_in);
  a.pout = plan_for(e, n_out);
  ::alfa::note_launch();
#define ALFA_CASE(p, q)               \
  if (n_in == p && n_out == q) {      \
    line_n<p, q>(e, a, F);            \
    return;                           \
  }
  ALFA_X_PAIRS(ALFA_CASE)
#undef ALFA_CASE
  line_n<0, 0>(e, a, F);
}

static LineOut lo(int map, double* dst, double scale, int cut = 0, int acc = 0) {
  LineOut o;
  o.map = map;
  o.cut = cut;
  o.scale = scale;
  o.accumulate = acc;
  o.dst = dst;
  return o;
}

// Filtering_Explicit followed by Derivxy in x and y (Filtering.py:50-89,
// Derivatives.py:161-182), as separable passes: x pass (filter, and filter +
// d/dx), then y passes.  scratch2: two N-sized fields.
void op2_filter_deriv(Engine& e, const Loader& L, double* f, double* dx, double* dy,
                      double* scratch2) {
  double* sx = scratch2;
  double* sdx = scratch2 + e.N();
  const double ix = 1.0 / e.nx, iy = 1.0 / e.ny;
  LineOut ox[2] = {lo(LM_TRUNC, sx, ix, e.cut_e[0]), lo(LM_TRUNC_DERIV, sdx, ix, e.cut_e[0])};
  launch_line(e, 0, L, e.nx, e.ny, e.nx, e.nx, dx ? 2 : 1, ox);
  LineOut oy[2] = {lo(LM_TRUNC, f, iy, e.cut_e[1]), lo(LM_TRUNC_DERIV, dy, iy, e.cut_e[1])};
  launch_line(e, 1, ld_field(e, sx), e.nx, e.ny, e.ny, e.ny, dy ? 2 : 1, oy);
  if (dx) {
    LineOut od = lo(LM_TRUNC, dx, iy, e.cut_e[1]);
    launch_line(e, 1, ld_field(e, sdx), e.nx, e.ny, e.ny, e.ny, 1, &od);
  }
}

// Derivxy(FFT(field), kx2) and (.., ky2) as one x pass and one y pass
void op2_deriv(Engine& e, const Loader& L, double* dx, int accx, double* dy, int accy) {
  if (dx) {
    LineOut o = lo(LM_DERIV, dx, 1.0 / e.nx, 0, accx);
    launch_line(e, 0, L, e.nx, e.ny, e.nx, e.nx, 1, &o);
  }
  if (dy) {
    LineOut o = lo(LM_DERIV, dy, 1.0 / e.ny, 0, accy);
    launch_line(e, 1, L, e.nx, e.ny, e.ny, e.ny, 1, &o);
  }
}

// Dealias1(FFT(field)): y pad (ny -> my) into scratch (nx, my, nz), then x pad
void op2_pad(Engine& e, const Loader& L, double* out_pad, double* scratch) {
  LineOut oy = lo(LM_PAD, scratch, 1.0 / e.my);
  launch_line(e, 1, L, e.nx, e.ny, e.ny, e.my, 1, &oy);
  LineOut ox = lo(LM_PAD, out_pad, 1.0 / e.mx);
  launch_line(e, 0, ld_field(e, scratch), e.nx, e.my, e.nx, e.mx, 1, &ox);
}

// Dealias2(FFT_pad(padded field)): x unpad (mx -> nx) into scratch
// (nx, my, nz), then y unpad with the 9/4 factor
void op2_unpad(Engine& e, const Loader& L_pad, double* out, double* scratch) {
  LineOut ox = lo(LM_UNPAD, scratch, 1.0 / e.nx);
  launch_line(e, 0, L_pad, e.mx, e.my, e.mx, e.nx, 1, &ox);
  LineOut oy = lo(LM_UNPAD, out, (9.0 / 4.0) * (1.0 / e.ny));
  launch_line(e, 1, ld_field(e, scratch), e.nx, e.my, e.my, e.ny, 1, &oy);
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
