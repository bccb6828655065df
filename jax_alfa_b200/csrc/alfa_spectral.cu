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

#include "alfa_tile.cuh"

namespace alfa {
namespace ALFA_PREC {

// Load the (n x 2 YC z) real tile of row `row` into b0 as n x YC complex
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
      v[u] = mkc(0, 0);
      if (t < total) {
        const int y = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t i = ((size_t)row * n + y) * nz + z;
        if (vec && z + 1 < nz) {
          v[u] = __ldg(reinterpret_cast<const cd*>(L.a[0] + i));
        } else {
          if (z < nz) v[u].x = (real)ldv<KIND>(L, i, z);
          if (z + 1 < nz) v[u].y = (real)ldv<KIND>(L, i + 1, z + 1);
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

// ---------------------------------------------------------------------------
// k_y_fwd: rows x n(y) x nz real -> T (rows, K, nz) complex, ky < K
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(tile_threads<YC, N>(), (N == 256 ? Y_MINBLOCKS : 1))
    k_y_fwd(Loader L, FftPlan p, int K, cd* __restrict__ T) {
  extern __shared__ cd sm[];
  const int n = (N > 0) ? N : p.n;
  const int nz = L.nz;
  const int z0 = blockIdx.x * (2 * YC);
  const int row = blockIdx.y;
  cd* b0 = sm;
  if constexpr (N > 0) {
    // first pass straight from global memory (register-resident start)
    constexpr int NT = tile_threads<YC, N>();
    constexpr int R = ct_radix(N);
    cd v[ct_mb(YC, N, 1, NT) * R];
    const size_t base = (size_t)row * N * nz;
    switch (L.kind) {
#define ALFA_G(K) \
  case K: gather_rows<K, YC, N, NT>(L, nz, base, (size_t)nz, z0, v); break;
      ALFA_LOADER_KINDS(ALFA_G)
#undef ALFA_G
      default: break;
    }
    if constexpr (R == N) {
      if (threadIdx.x < YC) {
        dftR<R, -1>(v);
#pragma unroll
        for (int r = 0; r < R; r++) b0[r * YC + threadIdx.x] = v[r];
      }
    } else {
      ct_first_reg<-1, YC, N, NT>(v, b0);
      ct_passes<-1, YC, N, R, NT>(b0, p.tw);
    }
    __syncthreads();
  } else {
  switch (L.kind) {
#define ALFA_K(K) \
  case K: y_fwd_load<K>(L, row, n, z0, b0); break;
    ALFA_LOADER_KINDS(ALFA_K)
#undef ALFA_K
    default: break;
  }
  tile_fft<-1, YC, N, tile_threads<YC, N>()>(b0, p);
  }
  const cd* Z = b0;
  for (int t = threadIdx.x; t < K * YC; t += blockDim.x) {
    const int k = t / YC, c = t % YC;
    const int z = z0 + 2 * c;
    const cd zk = Z[k * YC + c];
    const cd zn = Z[((n - k) % n) * YC + c];
    const real h = (real)0.5;
    const cd A = mkc(h * (zk.x + zn.x), h * (zk.y - zn.y));
    const cd B = mkc(h * (zk.y + zn.y), -h * (zk.x - zn.x));
    const size_t o = ((size_t)row * K + k) * nz + z;
    if (z < nz) T[o] = A;
    if (z + 1 < nz) T[o + 1] = B;
  }
}

// ---------------------------------------------------------------------------
// k_y_inv: T (rows, K, nz), ky < K nonzero -> rows x n(y) x nz real
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(tile_threads<YC, N>(), (N == 256 ? Y_MINBLOCKS : 1))
    k_y_inv(const cd* __restrict__ T, int K, FftPlan p, int nz, double scale,
            real* __restrict__ out, int accumulate) {
  extern __shared__ cd sm[];
  const int n = (N > 0) ? N : p.n;
  const int h = n / 2;
  const int z0 = blockIdx.x * (2 * YC);
  const int row = blockIdx.y;
  cd* b0 = sm;
  const bool pair = (nz & 1) == 0;  // z, z+1 both present whenever z is
  if constexpr (N > 0) {
    // Hermitian expansion of the two packed columns straight into the first
    // pass's registers; the last pass stores straight from registers
    constexpr int NT = tile_threads<YC, N>();
    constexpr int R = ct_radix(N);
    constexpr int NR = N / R;
    constexpr int B = NR * YC;
    constexpr int MB = ct_mb(YC, N, 1, NT);
    cd v[MB * R];
#pragma unroll
    for (int q = 0; q < MB; q++) {
      const int b = threadIdx.x + q * NT;
      const int c = b % YC;
      const int j = b / YC;
      const int z = z0 + 2 * c;
      const bool ok = (B % NT == 0 || b < B) && z < nz;
#pragma unroll
      for (int r = 0; r < R; r++) {
        const int k = j + r * NR;
        const int src = k <= h ? k : N - k;
        cd a = mkc(0, 0), bb = mkc(0, 0);
        if (ok && src < K) {
          const size_t o = ((size_t)row * K + src) * nz + z;
          a = __ldg(T + o);
          if (pair || z + 1 < nz) bb = __ldg(T + o + 1);
        }
        if (k == 0 || k == h) {
          a.y = 0.0;
          bb.y = 0.0;
        }
        v[q * R + r] = k <= h ? mkc(a.x - bb.y, a.y + bb.x)
                              : mkc(a.x + bb.y, bb.x - a.y);
      }
    }
    const size_t base = (size_t)row * N * nz;
    if constexpr (R == N) {
      if (threadIdx.x < YC) {
        dftR<R, +1>(v);
        const int z = z0 + 2 * threadIdx.x;
#pragma unroll
        for (int r = 0; r < R; r++)
          store_pair2(out, scale, accumulate, base + (size_t)r * nz + z, z, nz, v[r]);
      }
    } else {
      ct_first_reg<+1, YC, N, NT>(v, b0);
      ct_mid_passes<+1, YC, N, R, NT>(b0, p.tw);
      __syncthreads();
      constexpr int NSL = ct_last_ns(N);
      constexpr int RL = N / NSL;
      constexpr int BL = NSL * YC;
      constexpr int ML = ct_mb(YC, N, NSL, NT);
      cd u[ML * RL];
      ct_last_reg<+1, YC, N, NT>(b0, p.tw, u);
#pragma unroll
      for (int q = 0; q < ML; q++) {
        const int b = threadIdx.x + q * NT;
        if (!(BL % NT == 0 || b < BL)) continue;
        const int c = b % YC;
        const int j = b / YC;
        const int z = z0 + 2 * c;
#pragma unroll
        for (int r = 0; r < RL; r++)
          store_pair2(out, scale, accumulate, base + (size_t)(j + r * NSL) * nz + z, z, nz,
                      u[q * RL + r]);
      }
    }
    return;
  }
  const int total = (h + 1) * YC;
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    cd A[U], B[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      A[u] = mkc(0, 0);
      B[u] = mkc(0, 0);
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
      b0[k * YC + c] = mkc(a.x - b.y, a.y + b.x);
      if (k > 0 && k < h) b0[(n - k) * YC + c] = mkc(a.x + b.y, b.x - a.y);
    }
  }
  tile_fft<+1, YC, N, tile_threads<YC, N>()>(b0, p);
  const cd* Z = b0;
  const real sc = (real)scale;
  if (accumulate) {
    for (int t0 = threadIdx.x; t0 < n * YC; t0 += U * blockDim.x) {
      cd prev[U];
#pragma unroll
      for (int u = 0; u < U; u++) {
        const int t = t0 + u * blockDim.x;
        const int y = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t o = ((size_t)row * n + y) * nz + z;
        prev[u] = mkc(0, 0);
        if (t < n * YC) {
          if (pair && z < nz) {
            prev[u] = *reinterpret_cast<const cd*>(out + o);
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
        const cd w = mkc(prev[u].x + sc * v.x, prev[u].y + sc * v.y);
        if (pair && z < nz) {
          *reinterpret_cast<cd*>(out + o) = w;
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
        *reinterpret_cast<cd*>(out + o) = mkc(sc * v.x, sc * v.y);
      } else {
        if (z < nz) out[o] = sc * v.x;
        if (z + 1 < nz) out[o + 1] = sc * v.y;
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
      return keep ? S[k * C + c] : mkc(0, 0);
    }
    case MAP_DX: {
      const cd v = S[k * C + c];
      const real q = (real)a.kx[k];
      return mkc(-(q * v.y), q * v.x);
    }
    case MAP_DY: {
      const cd v = S[k * C + c];
      const real q = (real)a.ky[ky];
      return mkc(-(q * v.y), q * v.x);
    }
    case MAP_PAD: {  // Dealiasing.py:67-73 (rows nx -> mx)
      const int h = a.nx / 2;
      if (k <= h) return S[k * C + c];
      if (k >= a.mx - h) return S[(k - a.mx + a.nx) * C + c];
      return mkc(0, 0);
    }
    default: {  // MAP_UNPAD, Dealiasing.py:102-109 (rows mx -> nx)
      const int h = a.nx / 2;
      if (k < h) return S[k * C + c];
      if (k == h) return mkc(0, 0);
      return S[(k - a.nx + a.mx) * C + c];
    }
  }
}

// NI / NO: compile-time forward / inverse lengths (0: runtime plans)
// two resident CTAs per SM at least (the register budget of the FP32
// build's 256-thread tiles would otherwise leave one)
template <int C, int NI, int NO>
__global__ void __launch_bounds__(tile_threads<C, (NI > NO ? NI : NO)>(), 2) k_x(XArgs a) {
  constexpr int NT = tile_threads<C, (NI > NO ? NI : NO)>();
  extern __shared__ cd sm[];
  const int nz = a.nz;
  const int z0 = blockIdx.x * C;
  const int ky = blockIdx.y;
  const int M = a.maxrows * C;
  cd* buf[2] = {sm, sm + M};

  const bool have = ky < a.Kin;
  if constexpr (NI > 0 && NO > 0) {
    if (!a.in_spec) {
      // forward transform with its first pass straight from global memory
      constexpr int R = ct_radix(NI);
      constexpr int NR = NI / R;
      constexpr int B = NR * C;
      constexpr int MB = ct_mb(C, NI, 1, NT);
      cd v[MB * R];
#pragma unroll
      for (int q = 0; q < MB; q++) {
        const int b = threadIdx.x + q * NT;
        const int c = b % C;
        const int j = b / C;
        const int z = z0 + c;
        const bool ok = have && (B % NT == 0 || b < B) && z < nz;
#pragma unroll
        for (int r = 0; r < R; r++)
          v[q * R + r] = ok ? __ldg(&a.src[((size_t)(j + r * NR) * a.Kin + ky) * nz + z])
                            : mkc(0, 0);
      }
      if constexpr (R == NI) {
        if (threadIdx.x < C) {
          dftR<R, -1>(v);
#pragma unroll
          for (int r = 0; r < R; r++) buf[0][r * C + threadIdx.x] = v[r];
        }
      } else {
        ct_first_reg<-1, C, NI, NT>(v, buf[0]);
        ct_passes<-1, C, NI, R, NT>(buf[0], a.fwd.tw);
      }
      __syncthreads();
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
        // inverse transform: first pass fed through the map, last pass
        // stored straight from registers
        constexpr int RO = ct_radix(NO);
        constexpr int NRO = NO / RO;
        constexpr int BO = NRO * C;
        constexpr int MBO = ct_mb(C, NO, 1, NT);
        cd w[MBO * RO];
#pragma unroll
        for (int q = 0; q < MBO; q++) {
          const int b = threadIdx.x + q * NT;
          const int c = b % C;
          const int j = b / C;
#pragma unroll
          for (int r = 0; r < RO; r++)
            w[q * RO + r] = (BO % NT == 0 || b < BO) ? map_value<C>(a, o, S, j + r * NRO, ky, c)
                                                      : mkc(0, 0);
        }
        if constexpr (RO == NO) {
          if (threadIdx.x < C) {
            dftR<RO, +1>(w);
            const int z = z0 + threadIdx.x;
            if (z < nz) {
#pragma unroll
              for (int r = 0; r < RO; r++) o.dst[((size_t)r * o.K + ky) * nz + z] = w[r];
            }
          }
        } else {
          ct_first_reg<+1, C, NO, NT>(w, f0);
          ct_mid_passes<+1, C, NO, RO, NT>(f0, o.inv.tw);
          __syncthreads();
          constexpr int NSL = ct_last_ns(NO);
          constexpr int RL = NO / NSL;
          constexpr int BL = NSL * C;
          constexpr int ML = ct_mb(C, NO, NSL, NT);
          cd u[ML * RL];
          ct_last_reg<+1, C, NO, NT>(f0, o.inv.tw, u);
#pragma unroll
          for (int q = 0; q < ML; q++) {
            const int b = threadIdx.x + q * NT;
            if (!(BL % NT == 0 || b < BL)) continue;
            const int c = b % C;
            const int j = b / C;
            const int z = z0 + c;
            if (z >= nz) continue;
#pragma unroll
            for (int r = 0; r < RL; r++)
              o.dst[((size_t)(j + r * NSL) * o.K + ky) * nz + z] = u[q * RL + r];
          }
        }
        __syncthreads();
      }
      return;
    }
  }
  // load the input column set, U loads in flight per thread
  const int total = a.rows_in * C;
  for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
    cd v[U];
#pragma unroll
    for (int u = 0; u < U; u++) {
      const int t = t0 + u * blockDim.x;
      const int r = t / C, c = t % C;
      const int z = z0 + c;
      v[u] = mkc(0, 0);
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

#ifdef ALFA_BUILD_FP32
// ---------------------------------------------------------------------------
// k_y_inv_cv: k_y_inv (compile-time length) on two-lane elements: a thread
// takes two packed column pairs, four z levels (two 16-byte spectrum loads,
// one 16-byte store per row), and runs their inverse transforms in paired
// FP32 instructions.  nz a multiple of 4.
// ---------------------------------------------------------------------------
template <int N>
__global__ void __launch_bounds__(ct_threads(tile_cols<cv>(), N))
    k_y_inv_cv(const cd* __restrict__ T, int K, FftPlan p, int nz, double scale,
               real* __restrict__ out, int accumulate) {
  constexpr int C = tile_cols<cv>();
  constexpr int NT = ct_threads(C, N);
  constexpr int R = ct_radix(N);
  constexpr int NR = N / R;
  constexpr int B = NR * C;
  constexpr int MB = ct_mb(C, N, 1, NT);
  constexpr int h = N / 2;
  extern __shared__ __align__(16) unsigned char sm_yinv[];
  cv* b0 = reinterpret_cast<cv*>(sm_yinv);
  const int z0 = blockIdx.x * (4 * C);
  const int row = blockIdx.y;
  // Hermitian expansion of the packed columns (z, z+1) and (z+2, z+3)
  cv v[MB * R];
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 4 * c;
    const bool ok = (B % NT == 0 || b < B) && z < nz;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int k = j + r * NR;
      const int src = k <= h ? k : N - k;
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f), bq = a;  // (a, bb) of lane A, of lane B
      if (ok && src < K) {
        const float4* t = reinterpret_cast<const float4*>(T + ((size_t)row * K + src) * nz + z);
        a = __ldg(t);
        bq = __ldg(t + 1);
      }
      if (k == 0 || k == h) {
        a.y = 0.f;
        a.w = 0.f;
        bq.y = 0.f;
        bq.w = 0.f;
      }
      v[q * R + r] = k <= h ? cv{make_float2(a.x - a.w, bq.x - bq.w),
                                 make_float2(a.y + a.z, bq.y + bq.z)}
                            : cv{make_float2(a.x + a.w, bq.x + bq.w),
                                 make_float2(a.z - a.y, bq.z - bq.y)};
    }
  }
  const size_t base = (size_t)row * N * nz;
  ct_first_reg<+1, C, N, NT>(v, b0);
  ct_mid_passes<+1, C, N, R, NT>(b0, p.tw);
  __syncthreads();
  constexpr int NSL = ct_last_ns(N);
  constexpr int RL = N / NSL;
  constexpr int BL = NSL * C;
  constexpr int ML = ct_mb(C, N, NSL, NT);
  cv u[ML * RL];
  ct_last_reg<+1, C, N, NT>(b0, p.tw, u);
  LineOut o{};
  o.scale = scale;
  o.accumulate = accumulate;
  o.dst = out;
#pragma unroll
  for (int q = 0; q < ML; q++) {
    const int b = threadIdx.x + q * NT;
    if (!(BL % NT == 0 || b < BL)) continue;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 4 * c;
#pragma unroll
    for (int r = 0; r < RL; r++)
      store_elem(o, base + (size_t)(j + r * NSL) * nz + z, z, nz, u[q * RL + r]);
  }
}

// ---------------------------------------------------------------------------
// k_y_fwd_cv: k_y_fwd (compile-time length) on two-lane elements for the
// loaders without z neighbours: four z levels per element, the Hermitian
// split of both packed columns written as two 16-byte stores.  nz a
// multiple of 4.
// ---------------------------------------------------------------------------
template <int N, int KIND>
__global__ void __launch_bounds__(ct_threads(tile_cols<cv>(), N), 5)
    k_y_fwd_cv(Loader L, FftPlan p, int K, cd* __restrict__ T) {
  constexpr int C = tile_cols<cv>();
  constexpr int NT = ct_threads(C, N);
  constexpr int R = ct_radix(N);
  constexpr int NR = N / R;
  constexpr int B = NR * C;
  constexpr int MB = ct_mb(C, N, 1, NT);
  extern __shared__ __align__(16) unsigned char sm_yfwd[];
  cv* b0 = reinterpret_cast<cv*>(sm_yfwd);
  const int nz = L.nz;
  const int z0 = blockIdx.x * (4 * C);
  const int row = blockIdx.y;
  const size_t base = (size_t)row * N * nz;
  cv v[MB * R];
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 4 * c;
    const bool ok = (B % NT == 0 || b < B) && z < nz;
#pragma unroll
    for (int r = 0; r < R; r++)
      v[q * R + r] = ok ? ld_elem_cv<KIND>(L, base + (size_t)(j + r * NR) * nz + z, z, nz)
                        : vzero<cv>();
  }
  ct_first_reg<-1, C, N, NT>(v, b0);
  ct_passes<-1, C, N, R, NT>(b0, p.tw);
  __syncthreads();
  const float2 h = dup2(0.5f);
  for (int t = threadIdx.x; t < K * C; t += blockDim.x) {
    const int k = t / C, c = t % C;
    const int z = z0 + 4 * c;
    if (z >= nz) continue;
    const cv zk = b0[k * C + c];
    const cv zn = b0[((N - k) % N) * C + c];
    const float2 Ar = __fmul2_rn(h, __fadd2_rn(zk.re, zn.re));
    const float2 Ai = __fmul2_rn(h, __fadd2_rn(zk.im, neg2(zn.im)));
    const float2 Br = __fmul2_rn(h, __fadd2_rn(zk.im, zn.im));
    const float2 Bi = neg2(__fmul2_rn(h, __fadd2_rn(zk.re, neg2(zn.re))));
    float4* o = reinterpret_cast<float4*>(T + ((size_t)row * K + k) * nz + z);
    o[0] = make_float4(Ar.x, Ai.x, Br.x, Bi.x);
    o[1] = make_float4(Ar.y, Ai.y, Br.y, Bi.y);
  }
}

template <int N>
static bool y_fwd_cv(Engine& e, const Loader& L, int rows, const FftPlan& p, int K, cd* T) {
  if constexpr (N == 128 || N == 256) {
    if (L.nz % 4 != 0) return false;
    constexpr int C = tile_cols<cv>();
    const size_t smem = (size_t)N * C * sizeof(cv);
    dim3 g((L.nz + 4 * C - 1) / (4 * C), rows);
    switch (L.kind) {
#define ALFA_YF(KD)                                                               \
  case KD:                                                                        \
    set_smem((const void*)k_y_fwd_cv<N, KD>, smem);                               \
    k_y_fwd_cv<N, KD><<<g, ct_threads(C, N), smem, e.stream>>>(L, p, K, T);       \
    return true;
      ALFA_YF(LD_FIELD)
      ALFA_YF(LD_MUL)
      ALFA_YF(LD_PRESSURE_R)
#undef ALFA_YF
      default:
        return false;
    }
  }
  return false;
}

// store a two-lane element as the complex values at z and z+1 of a spectrum
__device__ __forceinline__ void st_cv(cd* p, cv v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.re.x, v.im.x, v.re.y, v.im.y);
}

// map_value on two-lane elements (two consecutive z levels of a spectrum)
template <int C>
__device__ __forceinline__ cv map_value_cv(const XArgs& a, const XOut& o, const cv* S, int k,
                                           int ky, int c) {
  switch (o.map) {
    case MAP_IDENT:
      return S[k * C + c];
    case MAP_TRUNC: {
      const bool keep = (k < o.cx || k >= a.nx - o.cx + 1) && ky < o.cy;
      return keep ? S[k * C + c] : vzero<cv>();
    }
    case MAP_DX:
      return mul_ik(S[k * C + c], (real)a.kx[k]);
    case MAP_DY:
      return mul_ik(S[k * C + c], (real)a.ky[ky]);
    case MAP_PAD: {
      const int h = a.nx / 2;
      if (k <= h) return S[k * C + c];
      if (k >= a.mx - h) return S[(k - a.mx + a.nx) * C + c];
      return vzero<cv>();
    }
    default: {
      const int h = a.nx / 2;
      if (k < h) return S[k * C + c];
      if (k == h) return vzero<cv>();
      return S[(k - a.nx + a.mx) * C + c];
    }
  }
}

// ---------------------------------------------------------------------------
// k_x_cv: the compile-time forward-and-outputs path of k_x on two-lane
// elements (two consecutive z levels of the y half spectrum per element, one
// 16-byte load or store, paired FP32 instructions).  nz even.
// ---------------------------------------------------------------------------
template <int NI, int NO>
__global__ void __launch_bounds__(tile_threads<tile_cols<cv>(), (NI > NO ? NI : NO)>(), 2)
    k_x_cv(XArgs a) {
  constexpr int C = tile_cols<cv>();
  constexpr int NT = tile_threads<C, (NI > NO ? NI : NO)>();
  extern __shared__ __align__(16) unsigned char sm_x[];
  cv* sm = reinterpret_cast<cv*>(sm_x);
  const int nz = a.nz;
  const int z0 = blockIdx.x * (2 * C);
  const int ky = blockIdx.y;
  const int M = a.maxrows * C;
  cv* buf0 = sm;
  cv* f0 = sm + M;
  const bool have = ky < a.Kin;
  {
    constexpr int R = ct_radix(NI);
    constexpr int NR = NI / R;
    constexpr int B = NR * C;
    constexpr int MB = ct_mb(C, NI, 1, NT);
    cv v[MB * R];
#pragma unroll
    for (int q = 0; q < MB; q++) {
      const int b = threadIdx.x + q * NT;
      const int c = b % C;
      const int j = b / C;
      const int z = z0 + 2 * c;
      const bool ok = have && (B % NT == 0 || b < B) && z < nz;
#pragma unroll
      for (int r = 0; r < R; r++)
        v[q * R + r] =
            ok ? ld_cv(reinterpret_cast<const real*>(a.src + ((size_t)(j + r * NR) * a.Kin + ky) *
                                                                  nz + z))
               : vzero<cv>();
    }
    ct_first_reg<-1, C, NI, NT>(v, buf0);
    ct_passes<-1, C, NI, R, NT>(buf0, a.fwd.tw);
    __syncthreads();
  }
  const cv* S = buf0;
  for (int oi = 0; oi < a.nout; oi++) {
    const XOut& o = a.out[oi];
    if (o.kind == XO_SPEC) {
      for (int t = threadIdx.x; t < o.rows * C; t += blockDim.x) {
        const int k = t / C, c = t % C;
        const int z = z0 + 2 * c;
        if (z < nz) st_cv(o.dst + ((size_t)k * o.K + ky) * nz + z, map_value_cv<C>(a, o, S, k, ky, c));
      }
      continue;
    }
    if (ky >= o.K) continue;  // column not stored: zero by convention
    constexpr int RO = ct_radix(NO);
    constexpr int NRO = NO / RO;
    constexpr int BO = NRO * C;
    constexpr int MBO = ct_mb(C, NO, 1, NT);
    cv w[MBO * RO];
#pragma unroll
    for (int q = 0; q < MBO; q++) {
      const int b = threadIdx.x + q * NT;
      const int c = b % C;
      const int j = b / C;
#pragma unroll
      for (int r = 0; r < RO; r++)
        w[q * RO + r] = (BO % NT == 0 || b < BO) ? map_value_cv<C>(a, o, S, j + r * NRO, ky, c)
                                                  : vzero<cv>();
    }
    ct_first_reg<+1, C, NO, NT>(w, f0);
    ct_mid_passes<+1, C, NO, RO, NT>(f0, o.inv.tw);
    __syncthreads();
    constexpr int NSL = ct_last_ns(NO);
    constexpr int RL = NO / NSL;
    constexpr int BL = NSL * C;
    constexpr int ML = ct_mb(C, NO, NSL, NT);
    cv u[ML * RL];
    ct_last_reg<+1, C, NO, NT>(f0, o.inv.tw, u);
#pragma unroll
    for (int q = 0; q < ML; q++) {
      const int b = threadIdx.x + q * NT;
      if (!(BL % NT == 0 || b < BL)) continue;
      const int c = b % C;
      const int j = b / C;
      const int z = z0 + 2 * c;
      if (z >= nz) continue;
#pragma unroll
      for (int r = 0; r < RL; r++)
        st_cv(o.dst + ((size_t)(j + r * NSL) * o.K + ky) * nz + z, u[q * RL + r]);
    }
    __syncthreads();
  }
}

// the two-lane k_x where it is built: plain forward transform from a y half
// spectrum, same-length inverses, nz even
template <int NI, int NO>
static bool x_cv(Engine& e, const XArgs& a, int Kgrid) {
  if constexpr ((NI == 128 || NI == 256) && NO == NI) {
    if (a.in_spec || (e.nz & 1) != 0) return false;
    constexpr int C = tile_cols<cv>();
    const size_t smem = 2 * (size_t)a.maxrows * C * sizeof(cv);
    set_smem((const void*)k_x_cv<NI, NO>, smem);
    dim3 g((e.nz + 2 * C - 1) / (2 * C), Kgrid);
    k_x_cv<NI, NO><<<g, tile_threads<C, NI>(), smem, e.stream>>>(a);
    return true;
  }
  return false;
}

template <int N>
static bool y_inv_cv(Engine& e, const cd* T, int rows, int K, const FftPlan& p, double scale,
                     real* out, int accumulate) {
  if constexpr (N == 128 || N == 256 || N == 384) {
    if (e.nz % 4 != 0 || ct_radix(N) == N) return false;
    constexpr int C = tile_cols<cv>();
    const size_t smem = (size_t)N * C * sizeof(cv);
    set_smem((const void*)k_y_inv_cv<N>, smem);
    dim3 g((e.nz + 4 * C - 1) / (4 * C), rows);
    k_y_inv_cv<N><<<g, ct_threads(C, N), smem, e.stream>>>(T, K, p, e.nz, scale, out,
                                                            accumulate);
    return true;
  }
  return false;
}
#endif

// ---------------------------------------------------------------------------
// launchers (dispatch to the specialised lengths)
// ---------------------------------------------------------------------------
template <int N>
static void y_fwd_n(Engine& e, const Loader& L, int rows, const FftPlan& p, int K, cd* T) {
#ifdef ALFA_BUILD_FP32
  if (y_fwd_cv<N>(e, L, rows, p, K, T)) return;
#endif
  const size_t smem = (size_t)p.n * YC * sizeof(cd);
  set_smem((const void*)k_y_fwd<N>, smem);
  dim3 g((L.nz + 2 * YC - 1) / (2 * YC), rows);
  const int nt = N > 0 ? tile_threads<YC, N>() : inplace_threads(YC, p.n);
  k_y_fwd<N><<<g, nt, smem, e.stream>>>(L, p, K, T);
}

template <int N>
static void y_inv_n(Engine& e, const cd* T, int rows, int K, const FftPlan& p, double scale,
                    real* out, int accumulate) {
#ifdef ALFA_BUILD_FP32
  if (y_inv_cv<N>(e, T, rows, K, p, scale, out, accumulate)) return;
#endif
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
                  real* out, int accumulate) {
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
#ifdef ALFA_BUILD_FP32
  if constexpr (C == YC) {
    if (x_cv<NI, NO>(e, a, Kgrid)) return;
  }
#endif
  const size_t smem = 2 * (size_t)a.maxrows * C * sizeof(cd);
  set_smem((const void*)k_x<C, NI, NO>, smem);
  dim3 g((e.nz + C - 1) / C, Kgrid);
  const int nt = (NI > 0) ? tile_threads<C, (NI > NO ? NI : NO)>() : inplace_threads(C, a.maxrows);
  k_x<C, NI, NO><<<g, nt, smem, e.stream>>>(a);
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
    if ((p > q ? p : q) <= 256) x_n<YC, p, q>(e, a, Kgrid);    \
    else x_n<YC / 2, p, q>(e, a, Kgrid);                       \
    return;                                                    \
  }
    ALFA_X_PAIRS(ALFA_CASE)
#undef ALFA_CASE
  }
  if (maxrows <= 256) x_n<YC, 0, 0>(e, a, Kgrid);
  else x_n<YC / 2, 0, 0>(e, a, Kgrid);
}

// ---------------------------------------------------------------------------
// composite operators
// ---------------------------------------------------------------------------
Loader ld_field(const Engine& e, const real* a) {
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
void op_filter_explicit(Engine& e, const Loader& L, real* out, cd* spec) {
  const int cx = e.cut_e[0], cy = e.cut_e[1];
  launch_y_fwd(e, L, e.nx, e.pny, e.nyh, e.T[0]);
  XOut o[2] = {xo_spec(e, MAP_TRUNC, spec, cx, cy),
               xo_inv(MAP_TRUNC, e.T[1], e.nx, cy, e.pnx, cx, cy)};
  launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, 2, o, e.nyh);
  launch_y_inv(e, e.T[1], e.nx, cy, e.pny, inv_scale(e.nx, e.ny), out, 0);
}

// Filtering_Level1 / Level2 (Filtering.py:97-165) of one FFT(field)
void op_filter12(Engine& e, const Loader& L, real* out1, real* out2) {
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
void op_filter1_spec(Engine& e, const cd* spec, int level, real* out) {
  const int* cut = level == 1 ? e.cut_1 : e.cut_2;
  XOut o = xo_inv(MAP_TRUNC, e.T[1], e.nx, cut[1], e.pnx, cut[0], cut[1]);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, 1, &o, cut[1]);
  launch_y_inv(e, e.T[1], e.nx, cut[1], e.pny, inv_scale(e.nx, e.ny), out, 0);
}

// Derivxy (Derivatives.py:161-182) in x and/or y of a spectrum
void op_deriv_spec(Engine& e, const cd* spec, real* dx, real* dy) {
  XOut o[2];
  int n = 0;
  if (dx) o[n++] = xo_inv(MAP_DX, e.T[1], e.nx, e.nyh, e.pnx);
  if (dy) o[n++] = xo_inv(MAP_DY, e.T[2], e.nx, e.nyh, e.pnx);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, n, o, e.nyh);
  if (dx) launch_y_inv(e, e.T[1], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), dx, 0);
  if (dy) launch_y_inv(e, e.T[2], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), dy, 0);
}

// Derivxy(FFT(field)) in x and/or y
void op_deriv_field(Engine& e, const Loader& L, real* dx, real* dy) {
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
void op_pad(Engine& e, const Loader& L, real* out_pad) {
  launch_y_fwd(e, L, e.nx, e.pny, e.nyh, e.T[0]);
  XOut o = xo_inv(MAP_PAD, e.T[1], e.mx, e.nyh, e.pmx);
  launch_x(e, e.T[0], 0, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
  launch_y_inv(e, e.T[1], e.mx, e.nyh, e.pmy, inv_scale(e.mx, e.my), out_pad, 0);
}

// Dealias1(spectrum)
void op_pad_spec(Engine& e, const cd* spec, real* out_pad) {
  XOut o = xo_inv(MAP_PAD, e.T[1], e.mx, e.nyh, e.pmx);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
  launch_y_inv(e, e.T[1], e.mx, e.nyh, e.pmy, inv_scale(e.mx, e.my), out_pad, 0);
}

// Dealias2(FFT_pad(padded field)) (Dealiasing.py:86-114): keeps ky < ny/2,
// drops the x Nyquist row, rescales by 9/4.
void op_unpad(Engine& e, const Loader& L_pad, real* out) {
  const int K = e.nyh - 1;
  launch_y_fwd(e, L_pad, e.mx, e.pmy, K, e.T[0]);
  XOut o = xo_inv(MAP_UNPAD, e.T[1], e.nx, K, e.pnx);
  launch_x(e, e.T[0], 0, e.mx, K, e.pmx, 1, &o, K);
  launch_y_inv(e, e.T[1], e.nx, K, e.pny, (9.0 / 4.0) * inv_scale(e.nx, e.ny), out, 0);
}

// Dealias2(padded spectrum (mx, myh, nz))
void op_unpad_spec(Engine& e, const cd* spec_pad, real* out) {
  const int K = e.nyh - 1;
  XOut o = xo_inv(MAP_UNPAD, e.T[1], e.nx, K, e.pnx);
  launch_x(e, spec_pad, 1, e.mx, e.myh, e.pmx, 1, &o, K);
  launch_y_inv(e, e.T[1], e.nx, K, e.pny, (9.0 / 4.0) * inv_scale(e.nx, e.ny), out, 0);
}

// irfft2(spectrum, s=(nx, ny))
void op_irfft2(Engine& e, const cd* spec, real* out) {
  XOut o = xo_inv(MAP_IDENT, e.T[1], e.nx, e.nyh, e.pnx);
  launch_x(e, spec, 1, e.nx, e.nyh, e.pnx, 1, &o, e.nyh);
  launch_y_inv(e, e.T[1], e.nx, e.nyh, e.pny, inv_scale(e.nx, e.ny), out, 0);
}

}  // namespace ALFA_PREC
}  // namespace alfa
