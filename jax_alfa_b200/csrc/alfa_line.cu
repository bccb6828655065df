// 1-D line passes along x or y of z-fastest real fields: the separable
// forms of the reference's spectral operators (explicit filter with its
// derivatives, derivatives, 3/2-rule pad and unpad), each a forward
// transform of runs of 2 YC z levels (a 128-byte row segment), a map, and an
// inverse transform.  The FP32 build also has each compile-time pass on
// two-lane elements (cv: two packed columns, four z levels, per thread), a
// variant the autotuner chooses per pass shape.
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "alfa_tile.cuh"

namespace alfa {
namespace ALFA_PREC {

// ---------------------------------------------------------------------------
// k_line: 1-D spectral operator along x or y on real fields.  A CTA takes one
// line index f (an x row for y lines, a y column for x lines) and 2 YC
// consecutive z levels packed as YC complex lines, transforms them forward,
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
      v[u] = mkc(0, 0);
      if (t < total) {
        const int r = t / YC, c = t % YC;
        const int z = z0 + 2 * c;
        const size_t i = (size_t)(f * a.fs_in + r * a.rs_in) + z;
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
      if (t < total) S[t] = v[u];
    }
  }
}

// bin k of output map o applied to the spectrum S (n bins, C elements per
// row) for an m-point output
template <int C = YC, class V = cd>
__device__ __forceinline__ V line_map(const LineOut& o, const V* S, int k, int c, int n, int m) {
  auto deriv = [&](V v) -> V {
    const int kk = (k < n / 2) ? k : (k == n / 2 ? 0 : k - n);
    return mul_ik(v, (real)kk);
  };
  switch (o.map) {
    case LM_IDENT:
      return S[k * C + c];
    case LM_TRUNC:
      return (k < o.cut || k >= n - o.cut + 1) ? S[k * C + c] : vzero<V>();
    case LM_DERIV:
      return deriv(S[k * C + c]);
    case LM_TRUNC_DERIV:
      return (k < o.cut || k >= n - o.cut + 1) ? deriv(S[k * C + c]) : vzero<V>();
    case LM_PAD: {  // n -> m = 3n/2, Nyquist row repeated (Dealiasing.py:67-73)
      const int h = n / 2;
      if (k <= h) return S[k * C + c];
      if (k >= m - h) return S[(k - m + n) * C + c];
      return vzero<V>();
    }
    default: {  // LM_UNPAD: n = 3m/2 -> m, Nyquist dropped (Dealiasing.py:102-109)
      const int h = m / 2;
      if (k < h) return S[k * C + c];
      if (k == h) return vzero<V>();
      return S[(k - m + n) * C + c];
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
#define ALFA_K(K) \
  case K: line_load<K>(a, f, z0, n, S); break;
    ALFA_LOADER_KINDS(ALFA_K)
#undef ALFA_K
    default: break;
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
    const real sc = (real)o.scale;
    if (o.accumulate) {
      for (int t0 = threadIdx.x; t0 < m * YC; t0 += U * blockDim.x) {
        cd prev[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
          const int t = t0 + u * blockDim.x;
          const int r = t / YC, c = t % YC;
          const int z = z0 + 2 * c;
          const size_t i = (size_t)(f * a.fs_out + r * a.rs_out) + z;
          prev[u] = mkc(0, 0);
          if (t < m * YC) {
            if (pair && z < nz) {
              prev[u] = *reinterpret_cast<const cd*>(o.dst + i);
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
          const cd w = mkc(prev[u].x + sc * v.x, prev[u].y + sc * v.y);
          if (pair && z < nz) {
            *reinterpret_cast<cd*>(o.dst + i) = w;
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
          *reinterpret_cast<cd*>(o.dst + i) = mkc(sc * v.x, sc * v.y);
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
// memory (every thread issues all of its loads before the first butterfly)
// and each inverse transform's last pass stores straight from registers.
// Each inverse reads its first-pass inputs from the forward spectrum in
// shared memory through the map.  GEN: the input is any Loader kind (else a
// plain field, with a leaner register budget).  (Keeping the forward
// spectrum in registers for same-length maps, which the n = 16 x 16 layout
// allows, measured slower: the register budget halved the resident CTAs.)
// ---------------------------------------------------------------------------
template <int C, int NIN, int NOUT>
__host__ __device__ constexpr int line_threads() {
  return ct_threads(C, NIN) > ct_threads(C, NOUT) ? ct_threads(C, NIN) : ct_threads(C, NOUT);
}

// first-pass gather: v[q*R + r] = (x, x') at row j + r*NR of line c
template <int KIND, int C, int N, int NT>
__device__ __forceinline__ void line_gather(const LineArgs& a, long long f, int z0, cd* v) {
  gather_rows<KIND, C, N, NT>(a.L, a.nz, (size_t)(f * a.fs_in), (size_t)a.rs_in, z0, v);
}

template <int C, int N, int NT>
__device__ __forceinline__ void line_gather_any(const LineArgs& a, long long f, int z0, cd* v) {
  switch (a.L.kind) {
#define ALFA_K(K) \
  case K: line_gather<K, C, N, NT>(a, f, z0, v); break;
    ALFA_LOADER_KINDS(ALFA_K)
#undef ALFA_K
    default: break;
  }
}

// store (or accumulate) v[q*R + r] = value at row j + r*STEP of line c
template <int C, int R, int STEP, int B, int NT, class V>
__device__ __forceinline__ void line_scatter(const LineArgs& a, const LineOut& o, long long f,
                                             int z0, const V* v) {
  constexpr int MB = (B + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (!(B % NT == 0 || b < B)) continue;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + zp_of<V>() * c;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const size_t i = (size_t)(f * a.fs_out + (long long)(j + r * STEP) * a.rs_out) + z;
      store_elem(o, i, z, a.nz, v[q * R + r]);
    }
  }
}

#ifdef ALFA_BUILD_FP32
// first-pass gather of a plain FP32 field in two-lane elements:
// v[q*R + r] = levels z .. z+3 at row j + r*(N/R) of element column c
template <int C, int N, int NT>
__device__ __forceinline__ void gather_rows_cv(const real* a0, int nz, size_t base, size_t rs,
                                               int z0, cv* v) {
  constexpr int R = ct_radix(N);
  constexpr int NR = N / R;
  constexpr int B = NR * C;
  constexpr int MB = (B + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 4 * c;
    const bool ok = (B % NT == 0 || b < B) && z < nz;
#pragma unroll
    for (int r = 0; r < R; r++)
      v[q * R + r] = ok ? ld_cv(a0 + base + (size_t)(j + r * NR) * rs + z) : vzero<cv>();
  }
}
#endif

// V: cd, or (FP32 build, plain-field input, nz a multiple of 4) the two-lane
// cv, which takes 4 z levels per element and half the threads per tile
template <int NIN, int NOUT, bool GEN, class V = cd>
__global__ void __launch_bounds__(line_threads<tile_cols<V>(), NIN, NOUT>())
    k_line_rr(LineArgs a) {
  constexpr int C = tile_cols<V>();
  constexpr int NT = line_threads<C, NIN, NOUT>();
  constexpr int NMAX = NIN > NOUT ? NIN : NOUT;
  extern __shared__ __align__(16) unsigned char sm_line[];
  V* sm = reinterpret_cast<V*>(sm_line);
  V* S = sm;
  const int z0 = blockIdx.x * (zp_of<V>() * C);
  const long long f = blockIdx.y;
  {
    V* Wb = a.nouts > 1 ? sm + NMAX * C : sm;
    // forward transform of the NIN-line tile into S
    {
      constexpr int R = ct_radix(NIN);
      constexpr int MB = ct_mb(C, NIN, 1, NT);
      V v[MB * R];
      if constexpr (!std::is_same<V, cd>::value) {
#ifdef ALFA_BUILD_FP32
        static_assert(!GEN, "two-lane tiles take plain fields only");
        gather_rows_cv<C, NIN, NT>(a.L.a[0], a.nz, (size_t)(f * a.fs_in), (size_t)a.rs_in, z0, v);
#endif
      } else if constexpr (GEN) {
        line_gather_any<C, NIN, NT>(a, f, z0, v);
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
      V v[MB * R];
#pragma unroll
      for (int q = 0; q < MB; q++) {
        const int b = threadIdx.x + q * NT;
        const int c = b % C;
        const int j = b / C;
#pragma unroll
        for (int r = 0; r < R; r++)
          v[q * R + r] = (B % NT == 0 || b < B)
                             ? line_map<C>(o, (const V*)S, j + r * NR, c, NIN, NOUT)
                             : vzero<V>();
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
        V u[ML * RL];
        ct_last_reg<+1, C, NOUT, NT>(Wb, a.pout.tw, u);
        line_scatter<C, RL, NSL, NSL * C, NT>(a, o, f, z0, u);
      }
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// 3/2-rule pad and unpad by phases.  With n = 2L and m = 3L, output sample
// t = 3s + p (p = 0, 1, 2) of the length-m inverse transform of a padded
// spectrum Y is the length-L inverse transform of the folded spectrum
//   Z_p[q] = sum_{k = q mod L} Y[k] w_m^{kp}.
// The pad spectrum (Y[k] = X[k] for k <= L and k >= 2L, the Nyquist bin X[L]
// repeated at both ends, zero between) folds to
//   Z_p[0] = X[0] + X[L] (w_3^p + w_3^{2p}),
//   Z_p[q] = w_m^{qp} (X[q] + w_3^{2p} X[q + L]),  0 < q < L,
// and the forward transform of a length-m line (decimated the same way into
// F_p = DFT_L of x[3s + p]) truncated to n bins (Nyquist bin zeroed) is
//   X[q] = sum_p w_m^{-qp} F_p[q],
//   X[L + q] = sum_p w_m^{-qp} w_3^{-2p} F_p[q]  (q > 0),  X[L] = 0.
// For n = 256 (= 16 x 16) a thread that ends the length-n forward transform
// holds bins j + 16r (r < 16), i.e. X[q] and X[q + L] for q = j + 16r',
// r' < 8: the folds are thread-local and each length-128 phase transform
// is one radix-8 pass in registers, one shared-memory exchange and one
// radix-16 pass.  The length-m transform and its radix-3 pass disappear.
// ---------------------------------------------------------------------------
template <int N, int C = YC>
__host__ __device__ constexpr bool pad3_ok() {
  return ct_last_ns(N) == ct_radix(N) && ct_radix(N) * ct_radix(N) == N && ct_radix(N) >= 4 &&
         ct_mb(C, N, 1, ct_threads(C, N)) == 1;
}

__device__ __forceinline__ cd cconj(cd a) { return mkc(a.x, -a.y); }

template <int KIND, int C, int N, int NT>
__device__ __forceinline__ void line_gather_sel(const LineArgs& a, long long f, int z0, cd* v) {
  if constexpr (KIND >= 0) line_gather<KIND, C, N, NT>(a, f, z0, v);
  else line_gather_any<C, N, NT>(a, f, z0, v);
}

// KIND: the loader kind, or -1 for any kind (chosen at run time); V as in
// k_line_rr (the two-lane cv for plain fields only)
template <int N, int KIND, class V = cd>
__global__ void __launch_bounds__(ct_threads(tile_cols<V>(), N)) k_pad3(LineArgs a) {
  constexpr int C = tile_cols<V>();
  constexpr int NT = ct_threads(C, N);
  constexpr int R = ct_radix(N);   // both passes of the length-N transform
  constexpr int L = N / 2;
  constexpr int RA = R / 2;        // first radix of the length-L phase transforms
  constexpr int RB = L / RA;       // their second radix (= R)
  static_assert(pad3_ok<N, C>() && RB == R, "pad3 layout");
  extern __shared__ __align__(16) unsigned char sm_pad[];
  V* S = reinterpret_cast<V*>(sm_pad);  // forward exchange, then three phase tiles of L x C
  const int z0 = blockIdx.x * (zp_of<V>() * C);
  const long long f = blockIdx.y;
  const LineOut& o = a.out[0];
  const cd* twN = a.pin.tw;   // exp(-2 pi i q / N)
  const cd* twM = a.pout.tw;  // exp(-2 pi i q / 3L)
  const int c = threadIdx.x % C;
  const int j = threadIdx.x / C;  // 0 .. R-1
  V X[R];
  {
    V v[R];
    if constexpr (!std::is_same<V, cd>::value) {
#ifdef ALFA_BUILD_FP32
      static_assert(KIND == LD_FIELD, "two-lane tiles take plain fields only");
      gather_rows_cv<C, N, NT>(a.L.a[0], a.nz, (size_t)(f * a.fs_in), (size_t)a.rs_in, z0, v);
#endif
    } else {
      line_gather_sel<KIND, C, N, NT>(a, f, z0, v);
    }
    ct_first_reg<-1, C, N, NT>(v, S);
    __syncthreads();
    ct_last_reg<-1, C, N, NT>(S, twN, X);  // X[r] = bin j + R r
  }
  __syncthreads();
  const cd w3a = cconj(__ldg(&twM[2 * L]));  // w_3^{2} (inverse sign)
  const cd w3b = cconj(__ldg(&twM[L]));      // w_3^{4} = w_3
#pragma unroll
  for (int p = 0; p < 3; p++) {
    V z[RA];
#pragma unroll
    for (int r = 0; r < RA; r++) {
      const int k = j + R * r;
      const V lo = X[r], hi = X[r + RA];
      V t;
      if (p == 0) {
        t = (k == 0) ? cadd(lo, cscale(hi, (real)2)) : cadd(lo, hi);
      } else if (k == 0) {
        t = csub(lo, hi);
      } else {
        t = cmul(cadd(lo, cmul(p == 1 ? w3a : w3b, hi)), cconj(__ldg(&twM[k * p])));
      }
      z[r] = t;
    }
    dftR<RA, +1>(z);
    V* P = S + p * L * C;
#pragma unroll
    for (int r = 0; r < RA; r++) P[(j * RA + r) * C + c] = z[r];
  }
  __syncthreads();
  constexpr int BB = 3 * RA * C;
  constexpr int MBB = (BB + NT - 1) / NT;
  const int nz = a.nz;
#pragma unroll
  for (int q = 0; q < MBB; q++) {
    const int b = threadIdx.x + q * NT;
    if (!(BB % NT == 0 || b < BB)) continue;
    const int p = b / (RA * C);
    const int bb = b % (RA * C);
    const int cc = bb % C;
    const int jj = bb / C;  // 0 .. RA-1
    const V* P = S + p * L * C;
    V v[RB];
#pragma unroll
    for (int r = 0; r < RB; r++) v[r] = P[(jj + r * RA) * C + cc];
#pragma unroll
    for (int r = 1; r < RB; r++) v[r] = cmul(v[r], cconj(__ldg(&twM[3 * jj * r])));
    dftR<RB, +1>(v);
    const int z = z0 + zp_of<V>() * cc;
#pragma unroll
    for (int r = 0; r < RB; r++) {
      const int row = 3 * (jj + RA * r) + p;
      const size_t i = (size_t)(f * a.fs_out + (long long)row * a.rs_out) + z;
      store_elem(o, i, z, nz, v[r]);
    }
  }
}

// gather of the unpad phase transforms' first pass: butterfly (p, jj, c),
// v[q*RB + r] = x[3 (jj + RA r) + p] of line c
template <int KIND, int C, int RA, int RB, int NT>
__device__ __forceinline__ void phase_gather(const LineArgs& a, long long f, int z0, cd* v) {
  constexpr int BB = 3 * RA * C;
  constexpr int MBB = (BB + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MBB; q++) {
    const int b = threadIdx.x + q * NT;
    const bool ok = (BB % NT == 0 || b < BB);
    const int p = b / (RA * C);
    const int bb = b % (RA * C);
    const int c = bb % C;
    const int jj = bb / C;
    const int z = z0 + 2 * c;
#pragma unroll
    for (int r = 0; r < RB; r++) {
      const long long row = 3 * (jj + RA * r) + p;
      const size_t i = (size_t)(f * a.fs_in + row * a.rs_in) + z;
      if (KIND != LD_FIELD && (a.nz & 1) == 0)
        v[q * RB + r] = eval_pair<KIND, C>(a.L, i, z, a.nz, c, ok);
      else
        v[q * RB + r] = ok ? load_pair<KIND>(a.L, i, z, a.nz) : mkc(0, 0);
    }
  }
}

#ifdef ALFA_BUILD_FP32
// phase_gather for a plain FP32 field in two-lane elements (4 levels each)
template <int C, int RA, int RB, int NT>
__device__ __forceinline__ void phase_gather_cv(const LineArgs& a, long long f, int z0, cv* v) {
  constexpr int BB = 3 * RA * C;
  constexpr int MBB = (BB + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MBB; q++) {
    const int b = threadIdx.x + q * NT;
    const int p = b / (RA * C);
    const int bb = b % (RA * C);
    const int c = bb % C;
    const int jj = bb / C;
    const int z = z0 + 4 * c;
    const bool ok = (BB % NT == 0 || b < BB) && z < a.nz;
#pragma unroll
    for (int r = 0; r < RB; r++) {
      const long long row = 3 * (jj + RA * r) + p;
      v[q * RB + r] = ok ? ld_cv(a.L.a[0] + (size_t)(f * a.fs_in + row * a.rs_in) + z)
                         : vzero<cv>();
    }
  }
}
#endif

template <int C, int RA, int RB, int NT>
__device__ __forceinline__ void phase_gather_any(const LineArgs& a, long long f, int z0, cd* v) {
  switch (a.L.kind) {
#define ALFA_K(K) \
  case K: phase_gather<K, C, RA, RB, NT>(a, f, z0, v); break;
    ALFA_LOADER_KINDS(ALFA_K)
#undef ALFA_K
    default: break;
  }
}

// three CTAs per SM measured faster than the unconstrained register budget
// (one-lane elements)
template <int N, int KIND, class V = cd>
__global__ void __launch_bounds__(ct_threads(tile_cols<V>(), N),
                                  (std::is_same<V, cd>::value ? 3 : 4))
    k_unpad3(LineArgs a) {
  constexpr int C = tile_cols<V>();
  constexpr int NT = ct_threads(C, N);
  constexpr int R = ct_radix(N);   // both passes of the length-N inverse
  constexpr int L = N / 2;
  constexpr int RA = R / 2;        // last radix of the length-L phase transforms
  constexpr int RB = L / RA;       // their first radix (= R)
  static_assert(pad3_ok<N, C>() && RB == R, "unpad3 layout");
  constexpr int BB = 3 * RA * C;
  constexpr int MBB = (BB + NT - 1) / NT;
  extern __shared__ __align__(16) unsigned char sm_unpad[];
  V* S = reinterpret_cast<V*>(sm_unpad);  // three phase tiles of L x C, then the exchange
  const int z0 = blockIdx.x * (zp_of<V>() * C);
  const long long f = blockIdx.y;
  const LineOut& o = a.out[0];
  const cd* twM = a.pin.tw;   // exp(-2 pi i q / 3L)
  const cd* twN = a.pout.tw;  // exp(-2 pi i q / N)
  {
    V v[MBB * RB];
    if constexpr (!std::is_same<V, cd>::value) {
#ifdef ALFA_BUILD_FP32
      static_assert(KIND == LD_FIELD, "two-lane tiles take plain fields only");
      phase_gather_cv<C, RA, RB, NT>(a, f, z0, v);
#endif
    } else if constexpr (KIND >= 0) {
      phase_gather<KIND, C, RA, RB, NT>(a, f, z0, v);
    } else {
      phase_gather_any<C, RA, RB, NT>(a, f, z0, v);
    }
#pragma unroll
    for (int q = 0; q < MBB; q++) {
      const int b = threadIdx.x + q * NT;
      if (!(BB % NT == 0 || b < BB)) continue;
      const int p = b / (RA * C);
      const int bb = b % (RA * C);
      const int cc = bb % C;
      const int jj = bb / C;
      dftR<RB, -1>(v + q * RB);
      V* P = S + p * L * C;
#pragma unroll
      for (int r = 0; r < RB; r++) P[(jj * RB + r) * C + cc] = v[q * RB + r];
    }
  }
  __syncthreads();
  const int c = threadIdx.x % C;
  const int j = threadIdx.x / C;  // 0 .. R-1
  V out[R];
  {
    V F[3][RA];
#pragma unroll
    for (int p = 0; p < 3; p++) {
      const V* P = S + p * L * C;
#pragma unroll
      for (int r = 0; r < RA; r++) F[p][r] = P[(j + r * RB) * C + c];
#pragma unroll
      for (int r = 1; r < RA; r++) F[p][r] = cmul(F[p][r], __ldg(&twM[3 * j * r]));
      dftR<RA, -1>(F[p]);  // F[p][r] = F_p[j + R r]
    }
    const cd w3a = __ldg(&twM[2 * L]);  // w_3^{-2}
    const cd w3b = __ldg(&twM[L]);      // w_3^{-4} = w_3^{-1}
#pragma unroll
    for (int r = 0; r < RA; r++) {
      const int k = j + R * r;
      const V g0 = F[0][r];
      const V g1 = cmul(F[1][r], __ldg(&twM[k]));
      const V g2 = cmul(F[2][r], __ldg(&twM[2 * k]));
      out[r] = cadd(cadd(g0, g1), g2);
      out[r + RA] = (k == 0) ? vzero<V>()
                             : cadd(cadd(g0, cmul(w3a, g1)), cmul(w3b, g2));
    }
  }
  __syncthreads();  // phase tiles fully read
  ct_first_reg<+1, C, N, NT>(out, S);
  __syncthreads();
  V u[R];
  ct_last_reg<+1, C, N, NT>(S, twN, u);
  line_scatter<C, R, R, R * C, NT>(a, o, f, z0, u);
}

template <int NIN, int NOUT>
static void line_n(Engine& e, const LineArgs& a, int F) {
  dim3 g((a.nz + 2 * YC - 1) / (2 * YC), F);
  if constexpr (NIN > 0) {
    const int nmax = NIN > NOUT ? NIN : NOUT;
    constexpr int nt = line_threads<YC, NIN, NOUT>();
    const size_t smem = (size_t)(nmax + (a.nouts > 1 ? NOUT : 0)) * YC * sizeof(cd);
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

// 3/2-rule pad or unpad by phases, n = N: a plain field (the form op2_pad /
// op2_unpad hand over), or any loader kind through the run-time switch
template <int N, int KIND>
static void pad3_k(Engine& e, const LineArgs& a, dim3 g, size_t smem) {
  set_smem((const void*)k_pad3<N, KIND>, smem);
  k_pad3<N, KIND><<<g, ct_threads(YC, N), smem, e.stream>>>(a);
}

template <int N, int KIND>
static void unpad3_k(Engine& e, const LineArgs& a, dim3 g, size_t smem) {
  set_smem((const void*)k_unpad3<N, KIND>, smem);
  k_unpad3<N, KIND><<<g, ct_threads(YC, N), smem, e.stream>>>(a);
}

template <int N, bool PAD>
static void phase_n(Engine& e, const LineArgs& a, int F) {
  dim3 g((a.nz + 2 * YC - 1) / (2 * YC), F);
  const size_t smem = (size_t)(3 * N / 2) * YC * sizeof(cd);
  const bool field = a.L.kind == LD_FIELD;
  if (PAD) {
    if (field) pad3_k<N, LD_FIELD>(e, a, g, smem);
    else pad3_k<N, -1>(e, a, g, smem);
  } else {
    if (field) unpad3_k<N, LD_FIELD>(e, a, g, smem);
    else unpad3_k<N, -1>(e, a, g, smem);
  }
}

#ifdef ALFA_BUILD_FP32
// The two-lane (cv) kernels: 4 z levels per element, paired FP32
// instructions for two packed columns at once.  Plain-field inputs with nz a
// multiple of 4, the phase-split 256 <-> 384 pad and unpad and the
// same-length compile-time passes of the bench-class grids.
template <int NIN, int NOUT>
static void line_n_cv(Engine& e, const LineArgs& a, int F) {
  constexpr int C = tile_cols<cv>();
  dim3 g((a.nz + 4 * C - 1) / (4 * C), F);
  constexpr int nmax = NIN > NOUT ? NIN : NOUT;
  constexpr int nt = line_threads<C, NIN, NOUT>();
  const size_t smem = (size_t)(nmax + (a.nouts > 1 ? NOUT : 0)) * C * sizeof(cv);
  set_smem((const void*)k_line_rr<NIN, NOUT, false, cv>, smem);
  k_line_rr<NIN, NOUT, false, cv><<<g, nt, smem, e.stream>>>(a);
}

template <int N, bool PAD>
static void phase_n_cv(Engine& e, const LineArgs& a, int F) {
  constexpr int C = tile_cols<cv>();
  dim3 g((a.nz + 4 * C - 1) / (4 * C), F);
  const size_t smem = (size_t)(3 * N / 2) * C * sizeof(cv);
  if (PAD) {
    set_smem((const void*)k_pad3<N, LD_FIELD, cv>, smem);
    k_pad3<N, LD_FIELD, cv><<<g, ct_threads(C, N), smem, e.stream>>>(a);
  } else {
    set_smem((const void*)k_unpad3<N, LD_FIELD, cv>, smem);
    k_unpad3<N, LD_FIELD, cv><<<g, ct_threads(C, N), smem, e.stream>>>(a);
  }
}

#define ALFA_CV_PAIRS(X) X(128, 128) X(192, 192) X(256, 256) X(384, 384)

// whether the pass has a two-lane kernel
bool cv_line_ok(const Loader& L, int n_in, int n_out, int nout, const LineOut* outs) {
  if (L.kind != LD_FIELD || (L.nz & 3) != 0) return false;
  if (nout == 1 && ((outs[0].map == LM_PAD && n_in == 256 && n_out == 384) ||
                    (outs[0].map == LM_UNPAD && n_in == 384 && n_out == 256)))
    return true;
#define ALFA_CASE(p, q) \
  if (n_in == p && n_out == q) return true;
  ALFA_CV_PAIRS(ALFA_CASE)
#undef ALFA_CASE
  return false;
}

static void cv_line(Engine& e, const LineArgs& a, int F, int nout, const LineOut* outs) {
  if (nout == 1 && outs[0].map == LM_PAD && a.n_in == 256 && a.n_out == 384) {
    phase_n_cv<256, true>(e, a, F);
    return;
  }
  if (nout == 1 && outs[0].map == LM_UNPAD && a.n_in == 384 && a.n_out == 256) {
    phase_n_cv<256, false>(e, a, F);
    return;
  }
#define ALFA_CASE(p, q)                  \
  if (a.n_in == p && a.n_out == q) {     \
    line_n_cv<p, q>(e, a, F);            \
    return;                              \
  }
  ALFA_CV_PAIRS(ALFA_CASE)
#undef ALFA_CASE
}
#endif

static const FftPlan& alt_plan_for(const Engine& e, int n, int r) {
  if (n == e.nx) return e.alt_plans[0][r];
  if (n == e.ny) return e.alt_plans[1][r];
  if (n == e.mx) return e.alt_plans[2][r];
  return e.alt_plans[3][r];
}

static const FftPlan& plan_for(const Engine& e, int n) {
  if (n == e.nx) return e.pnx;
  if (n == e.ny) return e.pny;
  if (n == e.mx) return e.pmx;
  return e.pmy;
}

#ifdef ALFA_BUILD_FP32
// The pass as a split-BF16 tensor-core GEMM (alfa_tc.cu) of the stacked
// operators of its outputs: x lines as one (n_in, Y nz) slab, y lines as X
// slabs of (n_in, nz).  Only for a plain-field input, outputs that are
// written (not accumulated) and an operator the autotuner has built already
// (a step being captured into a graph builds nothing); returns false when the
// pass does not qualify.
static bool tc_line(Engine& e, int axis, const Loader& L, int X, int Y, int n_in, int n_out,
                    int nout, const LineOut* outs) {
  if (L.kind != LD_FIELD || nout < 1 || nout > 2) return false;
  for (int q = 0; q < nout; q++)
    if (outs[q].accumulate) return false;
  const long long nz = L.nz;
  const long long ncols = axis == 0 ? (long long)Y * nz : nz;
  if (!tc_shape_ok(n_in, n_out, ncols)) return false;
  const int map2 = nout > 1 ? outs[1].map : -1;
  const Engine::TcOp* op = nullptr;
  for (const auto& o : e.tc_ops)
    if (o.map == outs[0].map && o.cut == outs[0].cut && o.n_in == n_in && o.n_out == n_out &&
        o.scale == outs[0].scale && o.map2 == map2 &&
        (map2 < 0 || (o.cut2 == outs[1].cut && o.scale2 == outs[1].scale)))
      op = &o;
  if (!op || !e.tc_err) return false;
  tc_launch(e, op, ncols, L.a[0], outs[0].dst, nout > 1 ? outs[1].dst : nullptr,
            axis == 0 ? 1 : X, axis == 0 ? 0 : (long long)n_in * nz,
            axis == 0 ? 0 : (long long)n_out * nz);
  return true;
}
#endif

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
  int variant = 0;
  if (!e.line_variant.empty()) {
    auto it = e.line_variant.find(line_key(axis, n_in, n_out, outs[0].map, nout));
    if (it != e.line_variant.end()) variant = it->second;
  }
#ifdef ALFA_BUILD_FP32
  if (variant == TC_VARIANT && tc_line(e, axis, L, X, Y, n_in, n_out, nout, outs)) return;
#endif
  ::alfa::note_launch();
#ifdef ALFA_BUILD_FP32
  if (variant == CV_VARIANT && cv_line_ok(L, n_in, n_out, nout, outs)) {
    cv_line(e, a, F, nout, outs);
    return;
  }
#endif
  if (variant >= 2 && variant < TC_VARIANT) {  // runtime plans, alternative radix schedule
    const int r = variant - 2;
    a.pin = alt_plan_for(e, n_in, r);
    a.pout = alt_plan_for(e, n_out, r);
    line_n<0, 0>(e, a, F);
    return;
  }
  if (variant == 1) goto compile_time;
  if (nout == 1 && outs[0].map == LM_PAD && n_in == 256 && n_out == 384) {
    phase_n<256, true>(e, a, F);
    return;
  }
  if (nout == 1 && outs[0].map == LM_UNPAD && n_in == 384 && n_out == 256) {
    phase_n<256, false>(e, a, F);
    return;
  }
compile_time:
#define ALFA_CASE(p, q)               \
  if (n_in == p && n_out == q) {      \
    line_n<p, q>(e, a, F);            \
    return;                           \
  }
  ALFA_X_PAIRS(ALFA_CASE)
#undef ALFA_CASE
  line_n<0, 0>(e, a, F);
}

long long line_key(int axis, int n_in, int n_out, int map, int nout) {
  const int cls = (map == LM_PAD) ? 1 : (map == LM_UNPAD ? 2 : 0);
  return ((((long long)axis * 8192 + n_in) * 8192 + n_out) * 4 + cls) * 4 + nout;
}

static LineOut lo(int map, real* dst, double scale, int cut = 0, int acc = 0) {
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
void op2_filter_deriv(Engine& e, const Loader& L, real* f, real* dx, real* dy,
                      real* scratch2) {
  real* sx = scratch2;
  real* sdx = scratch2 + e.N();
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
void op2_deriv(Engine& e, const Loader& L, real* dx, int accx, real* dy, int accy) {
  if (dx) {
    LineOut o = lo(LM_DERIV, dx, 1.0 / e.nx, 0, accx);
    launch_line(e, 0, L, e.nx, e.ny, e.nx, e.nx, 1, &o);
  }
  if (dy) {
    LineOut o = lo(LM_DERIV, dy, 1.0 / e.ny, 0, accy);
    launch_line(e, 1, L, e.nx, e.ny, e.ny, e.ny, 1, &o);
  }
}

// Elementwise evaluation of a loader (its kind a template constant): one
// level per thread, stencil neighbours through the cache.  A separate pass
// costs one extra write and read of the domain but keeps the transform
// kernels' gathers to a single 16-byte load per element: gathering several
// inputs per element inside the transform kernel limits the loads a thread
// keeps in flight and measured slower than the two passes.
template <int KIND>
__global__ void __launch_bounds__(256) k_materialize(Loader L, size_t n, real* __restrict__ out) {
  const int nz = L.nz;
#pragma unroll 4
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x)
    out[i] = (real)ldv<KIND>(L, i, zof(i, nz));
}

// 16 bytes of a field: 4 FP32 or 2 FP64 consecutive levels
constexpr int MAT_E = (int)(16 / sizeof(real));
__device__ __forceinline__ void ld16(const real* p, real* v) {
#ifdef ALFA_BUILD_FP32
  const float4 q = __ldg(reinterpret_cast<const float4*>(p));
  v[0] = q.x;
  v[1] = q.y;
  v[2] = q.z;
  v[3] = q.w;
#else
  const double2 q = __ldg(reinterpret_cast<const double2*>(p));
  v[0] = q.x;
  v[1] = q.y;
#endif
}
__device__ __forceinline__ void st16(real* p, const real* v) {
#ifdef ALFA_BUILD_FP32
  *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
#else
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
#endif
}

// Vector form of k_materialize (nz a multiple of MAT_E, 16-byte aligned
// fields): MAT_E consecutive levels of one column per thread, one 16-byte
// load of each input the kind reads plus one scalar load per z-1 / z+MAT_E
// neighbour it needs (only inside the column: ev_kind reads no z-1 value at
// z = 0 and no z+1 value at z = nz-1).  The accessor returns the stored type,
// as ldv's does, so each level's expression has the same operand types (an
// FP32 difference of two inputs stays FP32) and the values equal
// k_materialize's; the scalar form kept 4-byte loads in flight and reached
// 0.36 (FP32) to 0.48 (FP64) of HBM bandwidth.
template <int KIND>
__global__ void __launch_bounds__(256) k_materialize_vec(Loader L, size_t nv,
                                                         real* __restrict__ out) {
  constexpr int E = MAT_E;
  constexpr int NIN = loader_nin(KIND);
  const int nz = L.nz;
  for (size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x; t < nv;
       t += (size_t)gridDim.x * blockDim.x) {
    const size_t i = t * E;
    const int z = zof(i, nz);
    real w[NIN][E + 2];  // levels z-1 .. z+E of each input
#pragma unroll
    for (int k = 0; k < NIN; k++) {
#pragma unroll
      for (int j = 0; j < E + 2; j++) w[k][j] = (real)0;
      const InUse u = loader_use(KIND, L.sub, k);
      if (u.in) {
        ld16(L.a[k] + i, &w[k][1]);
        if (u.m && z > 0) w[k][0] = __ldg(L.a[k] + i - 1);
        if (u.p && z + E < nz) w[k][E + 1] = __ldg(L.a[k] + i + E);
      }
    }
    real r[E];
#pragma unroll
    for (int j = 0; j < E; j++)
      r[j] = (real)ev_kind<KIND>(L, [&](int k, int d) { return w[k][1 + j + d]; }, z + j, nz);
    st16(out + i, r);
  }
}

static bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

void materialize(Engine& e, const Loader& L, size_t n, real* out) {
  bool vec = L.nz % MAT_E == 0 && n % MAT_E == 0 && aligned16(out);
  for (int k = 0; k < 10; k++) vec = vec && aligned16(L.a[k]);
  const size_t items = vec ? n / MAT_E : n;
  const size_t want = (items + 255) / 256;
  const unsigned blocks = (unsigned)(want < (size_t)e.sms * 16 ? want : (size_t)e.sms * 16);
  ::alfa::note_launch();
  switch (L.kind) {
#define ALFA_MAT(K)                                                                 \
  case K:                                                                           \
    if (vec) k_materialize_vec<K><<<blocks, 256, 0, e.stream>>>(L, items, out);     \
    else k_materialize<K><<<blocks, 256, 0, e.stream>>>(L, n, out);                 \
    break;
    ALFA_LOADER_KINDS(ALFA_MAT)
#undef ALFA_MAT
    default: break;
  }
}

// Dealias1(FFT(field)): y pad (ny -> my) into scratch (nx, my, nz), then x
// pad; a non-field loader is first materialised
void op2_pad(Engine& e, const Loader& L0, real* out_pad, real* scratch) {
  Loader L = L0;
  if (L.kind != LD_FIELD) {
    materialize(e, L, e.N(), e.mat);
    L = ld_field(e, e.mat);
  }
  LineOut oy = lo(LM_PAD, scratch, 1.0 / e.my);
  launch_line(e, 1, L, e.nx, e.ny, e.ny, e.my, 1, &oy);
  LineOut ox = lo(LM_PAD, out_pad, 1.0 / e.mx);
  launch_line(e, 0, ld_field(e, scratch), e.nx, e.my, e.nx, e.mx, 1, &ox);
}

// Dealias2(FFT_pad(padded field)): x unpad (mx -> nx) into scratch
// (nx, my, nz), then y unpad with the 9/4 factor; a non-field loader is
// first materialised
void op2_unpad(Engine& e, const Loader& L0, real* out, real* scratch) {
  Loader L = L0;
  LineOut ox = lo(LM_UNPAD, scratch, 1.0 / e.nx);
  if (L.kind != LD_FIELD) {
    materialize(e, L, e.P(), e.mat);
    L = ld_field(e, e.mat);
  }
  launch_line(e, 0, L, e.mx, e.my, e.mx, e.nx, 1, &ox);
  LineOut oy = lo(LM_UNPAD, out, (9.0 / 4.0) * (1.0 / e.ny));
  launch_line(e, 1, ld_field(e, scratch), e.nx, e.my, e.my, e.ny, 1, &oy);
}

}  // namespace ALFA_PREC
}  // namespace alfa
