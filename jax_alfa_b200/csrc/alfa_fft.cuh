// Batched FFT building blocks for sm_100a (complex of `real`: FP64 or FP32,
// alfa_prec.cuh).
//
// A CTA transforms C independent columns at once: a tile of n rows x C
// columns of complex values held in shared memory with the column index
// fastest (element (row, c) at row*C + c), which is exactly the layout of a
// run of C consecutive z levels of a field stored z-fastest (complex doubles in
// the FP64 build, complex floats in the FP32 build).  The transform
// is a mixed-radix Stockham sweep: each pass, every thread takes R elements
// of one column into registers, applies the inter-pass twiddles from a
// per-length table, runs an R-point DFT in registers and writes the R
// results to the other shared-memory buffer (ping-pong, no bit reversal).
// Radices 2, 3, 4, 8 and 16 cover every length 2^a 3^b used by the grids
// (n, 3n/2 for the 3/2-rule padding).
#pragma once
#include "alfa_prec.cuh"

namespace alfa {
namespace ALFA_PREC {

__device__ __forceinline__ cd cadd(cd a, cd b) { return mkc(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ cd csub(cd a, cd b) { return mkc(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ cd cmul(cd a, cd b) {
  return mkc(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ cd cscale(cd a, real s) { return mkc(a.x * s, a.y * s); }
// a * (S i): S = -1 forward (multiply by -i), S = +1 inverse (multiply by +i)
template <int S>
__device__ __forceinline__ cd rot90(cd a) {
  return S < 0 ? mkc(a.y, -a.x) : mkc(-a.y, a.x);
}

// cos(m pi / 8) and sin(m pi / 8) for m = 0..15 (exact roots of unity of
// order 16, correctly rounded to `real`).
__device__ __forceinline__ cd w16(int m, int S) {
  const real c1 = (real)0.92387953251128675613;  // cos(pi/8)
  const real s1 = (real)0.38268343236508977173;  // sin(pi/8)
  const real r2 = (real)0.70710678118654752440;  // sqrt(1/2)
  real c, s;
  switch (m & 15) {
    case 0: c = 1.0; s = 0.0; break;
    case 1: c = c1; s = s1; break;
    case 2: c = r2; s = r2; break;
    case 3: c = s1; s = c1; break;
    case 4: c = 0.0; s = 1.0; break;
    case 5: c = -s1; s = c1; break;
    case 6: c = -r2; s = r2; break;
    case 7: c = -c1; s = s1; break;
    case 8: c = -1.0; s = 0.0; break;
    case 9: c = -c1; s = -s1; break;
    case 10: c = -r2; s = -r2; break;
    case 11: c = -s1; s = -c1; break;
    case 12: c = 0.0; s = -1.0; break;
    case 13: c = s1; s = -c1; break;
    case 14: c = r2; s = -r2; break;
    default: c = c1; s = -s1; break;
  }
  return mkc(c, S * s);
}

#ifdef ALFA_BUILD_FP32
// Two complex values in the same position of two adjacent packed columns
// (lanes A and B: levels z, z+1 and z+2, z+3 of a z-fastest FP32 field),
// held as real and imaginary lane pairs so that every operation of a
// butterfly is one paired FP32 instruction (FADD2 / FMUL2 / FFMA2 on sm_100)
// for both lanes.  The codelets below run unchanged on it.
struct cv {
  float2 re, im;
};
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ cv cadd(cv a, cv b) {
  return cv{__fadd2_rn(a.re, b.re), __fadd2_rn(a.im, b.im)};
}
__device__ __forceinline__ cv csub(cv a, cv b) {
  return cv{__fadd2_rn(a.re, neg2(b.re)), __fadd2_rn(a.im, neg2(b.im))};
}
// a * w, w one complex value for both lanes
__device__ __forceinline__ cv cmul(cv a, cd w) {
  return cv{__ffma2_rn(a.re, dup2(w.x), __fmul2_rn(a.im, dup2(-w.y))),
            __ffma2_rn(a.re, dup2(w.y), __fmul2_rn(a.im, dup2(w.x)))};
}
__device__ __forceinline__ cv cmul(cd w, cv a) { return cmul(a, w); }
__device__ __forceinline__ cv cscale(cv a, real s) {
  return cv{__fmul2_rn(a.re, dup2(s)), __fmul2_rn(a.im, dup2(s))};
}
template <int S>
__device__ __forceinline__ cv rot90(cv a) {
  return S < 0 ? cv{a.im, neg2(a.re)} : cv{neg2(a.im), a.re};
}
#endif

// R-point DFTs in registers over elements of type V: cd (one complex
// value) or, in the FP32 build, cv (two lanes)
template <int S, class V>
__device__ __forceinline__ void dft2(V& a, V& b) {
  V t = a;
  a = cadd(t, b);
  b = csub(t, b);
}

template <int S, class V>
__device__ __forceinline__ void dft3(V& a, V& b, V& c) {
  const real h = (real)0.86602540378443864676;  // sqrt(3)/2
  V t1 = cadd(b, c);
  V t2 = csub(a, cscale(t1, (real)0.5));
  V d = csub(b, c);
  V t3 = rot90<S>(cscale(d, h));
  a = cadd(a, t1);
  b = cadd(t2, t3);
  c = csub(t2, t3);
}

template <int S, class V>
__device__ __forceinline__ void dft4(V& v0, V& v1, V& v2, V& v3) {
  V t0 = cadd(v0, v2), t1 = csub(v0, v2);
  V t2 = cadd(v1, v3), t3 = rot90<S>(csub(v1, v3));
  v0 = cadd(t0, t2);
  v2 = csub(t0, t2);
  v1 = cadd(t1, t3);
  v3 = csub(t1, t3);
}

template <int S, class V>
__device__ __forceinline__ void dft8(V* v) {
  // radix-2 over two 4-point DFTs (even and odd inputs)
  V e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
  V o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
  dft4<S>(e0, e1, e2, e3);
  dft4<S>(o0, o1, o2, o3);
  const real r2 = (real)0.70710678118654752440;
  o1 = cmul(o1, mkc(r2, S * r2));
  o2 = rot90<S>(o2);
  o3 = cmul(o3, mkc(-r2, S * r2));
  v[0] = cadd(e0, o0); v[4] = csub(e0, o0);
  v[1] = cadd(e1, o1); v[5] = csub(e1, o1);
  v[2] = cadd(e2, o2); v[6] = csub(e2, o2);
  v[3] = cadd(e3, o3); v[7] = csub(e3, o3);
}

template <int S, class V>
__device__ __forceinline__ void dft16(V* v) {
  // 4 x 4: inner 4-point DFTs over n2 (stride 4), twiddle W16^(n1 k2),
  // outer 4-point DFTs over n1.
#pragma unroll
  for (int n1 = 0; n1 < 4; n1++) dft4<S>(v[n1], v[n1 + 4], v[n1 + 8], v[n1 + 12]);
#pragma unroll
  for (int n1 = 1; n1 < 4; n1++) {
#pragma unroll
    for (int k2 = 1; k2 < 4; k2++) v[n1 + 4 * k2] = cmul(v[n1 + 4 * k2], w16(n1 * k2, S));
  }
  V o[16];
#pragma unroll
  for (int k2 = 0; k2 < 4; k2++) {
    V a = v[4 * k2], b = v[4 * k2 + 1], c = v[4 * k2 + 2], d = v[4 * k2 + 3];
    dft4<S>(a, b, c, d);
    o[k2] = a; o[k2 + 4] = b; o[k2 + 8] = c; o[k2 + 12] = d;
  }
#pragma unroll
  for (int i = 0; i < 16; i++) v[i] = o[i];
}

template <int R, int S, class V>
__device__ __forceinline__ void dftR(V* v) {
  if (R == 2) dft2<S>(v[0], v[1]);
  else if (R == 3) dft3<S>(v[0], v[1], v[2]);
  else if (R == 4) dft4<S>(v[0], v[1], v[2], v[3]);
  else if (R == 8) dft8<S>(v);
  else dft16<S>(v);
}

// Length-n transform plan: radices of the Stockham passes and the table
// tw[q] = exp(-2 pi i q / n), q = 0..n-1 (computed on the host in long
// double and rounded once).
struct FftPlan {
  int n;
  int npass;
  int rad[8];
  const cd* tw;
};

// One Stockham pass of radix R over C columns (Govindaraju et al., "High
// performance discrete Fourier transforms on graphics processors", SC 2008,
// Stockham formulation).  src/dst are n x C shared-memory tiles.
template <int R, int S, int C>
__device__ __forceinline__ void stockham_pass(const cd* __restrict__ src, cd* __restrict__ dst, int n,
                                              int Ns, const cd* __restrict__ tw) {
  const int nR = n / R;
  const int B = nR * C;
  const int stride = n / (Ns * R);
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const int c = b % C;  // C is a power of two: shifts and masks
    const int j = b / C;
    cd v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = src[(j + r * nR) * C + c];
    const int k = j % Ns;
    if (Ns > 1) {
#pragma unroll
      for (int r = 1; r < R; r++) {
        cd w = __ldg(&tw[k * r * stride]);
        if (S > 0) w.y = -w.y;
        v[r] = cmul(v[r], w);
      }
    }
    dftR<R, S>(v);
    const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
    for (int r = 0; r < R; r++) dst[(idxD + r * Ns) * C + c] = v[r];
  }
}

// Full unnormalised transform of the n x C tile in buf[0]; buf[1] is
// scratch of the same size.  Returns the index (0/1) of the buffer holding
// the result.  S = -1 forward, +1 inverse.  Leaves a __syncthreads() behind.
template <int S, int C>
__device__ int fft_tile(cd* buf0, cd* buf1, const FftPlan& p) {
  cd* src = buf0;
  cd* dst = buf1;
  int Ns = 1;
  for (int i = 0; i < p.npass; i++) {
    __syncthreads();
    switch (p.rad[i]) {
      case 16: stockham_pass<16, S, C>(src, dst, p.n, Ns, p.tw); break;
      case 8: stockham_pass<8, S, C>(src, dst, p.n, Ns, p.tw); break;
      case 4: stockham_pass<4, S, C>(src, dst, p.n, Ns, p.tw); break;
      case 3: stockham_pass<3, S, C>(src, dst, p.n, Ns, p.tw); break;
      default: stockham_pass<2, S, C>(src, dst, p.n, Ns, p.tw); break;
    }
    Ns *= p.rad[i];
    cd* t = src;
    src = dst;
    dst = t;
  }
  __syncthreads();
  return src == buf0 ? 0 : 1;
}

// In-place variant: one n x C tile, no second buffer.  In each pass every
// thread first reads all of its butterflies (at most MB of them, R inputs
// each) into registers, the block synchronises, and only then are the
// results written back over the tile.  With blockDim.x >= C*n/16 a thread
// holds at most 18 complex values in any pass (radix 16: 1 butterfly,
// 8: 2, 4: 4, 3: 6, 2: 8).
// (not inlined: one all-radix body inlined into the pass loop makes the
// register allocator keep every variant's arrays live and spill)
template <int R, int S, int C, int MB>
__device__ __noinline__ void stockham_inplace(cd* __restrict__ buf, int n, int Ns,
                                                 const cd* __restrict__ tw) {
  const int nR = n / R;
  const int B = nR * C;
  const int stride = n / (Ns * R);
  cd v[MB * R];
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * blockDim.x;
    if (b < B) {
      const int c = b % C;
      const int j = b / C;
#pragma unroll
      for (int r = 0; r < R; r++) v[q * R + r] = buf[(j + r * nR) * C + c];
      const int k = j % Ns;
      if (Ns > 1) {
#pragma unroll
        for (int r = 1; r < R; r++) {
          cd w = __ldg(&tw[k * r * stride]);
          if (S > 0) w.y = -w.y;
          v[q * R + r] = cmul(v[q * R + r], w);
        }
      }
      dftR<R, S>(v + q * R);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * blockDim.x;
    if (b < B) {
      const int c = b % C;
      const int j = b / C;
      const int k = j % Ns;
      const int idxD = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) buf[(idxD + r * Ns) * C + c] = v[q * R + r];
    }
  }
}

template <int R, int S, int C>
__device__ __forceinline__ void inplace_pass(cd* buf, int n, int Ns, const cd* tw) {
  const int B = (n / R) * C;
  const int mb = (B + blockDim.x - 1) / blockDim.x;
  if (R == 16) {
    stockham_inplace<R, S, C, 1>(buf, n, Ns, tw);
  } else if (R == 8) {
    if (mb <= 1) stockham_inplace<R, S, C, 1>(buf, n, Ns, tw);
    else stockham_inplace<R, S, C, 2>(buf, n, Ns, tw);
  } else if (R == 4) {
    if (mb <= 2) stockham_inplace<R, S, C, 2>(buf, n, Ns, tw);
    else stockham_inplace<R, S, C, 4>(buf, n, Ns, tw);
  } else if (R == 3) {
    if (mb <= 2) stockham_inplace<R, S, C, 2>(buf, n, Ns, tw);
    else if (mb <= 4) stockham_inplace<R, S, C, 4>(buf, n, Ns, tw);
    else stockham_inplace<R, S, C, 6>(buf, n, Ns, tw);
  } else {
    if (mb <= 2) stockham_inplace<R, S, C, 2>(buf, n, Ns, tw);
    else if (mb <= 4) stockham_inplace<R, S, C, 4>(buf, n, Ns, tw);
    else stockham_inplace<R, S, C, 8>(buf, n, Ns, tw);
  }
}

// Full unnormalised in-place transform of the n x C tile `buf`; requires
// blockDim.x >= ceil(C*n/16).  Leaves a __syncthreads() behind.
template <int S, int C>
__device__ void fft_inplace(cd* buf, const FftPlan& p) {
  int Ns = 1;
  for (int i = 0; i < p.npass; i++) {
    __syncthreads();
    switch (p.rad[i]) {
      case 16: inplace_pass<16, S, C>(buf, p.n, Ns, p.tw); break;
      case 8: inplace_pass<8, S, C>(buf, p.n, Ns, p.tw); break;
      case 4: inplace_pass<4, S, C>(buf, p.n, Ns, p.tw); break;
      case 3: inplace_pass<3, S, C>(buf, p.n, Ns, p.tw); break;
      default: inplace_pass<2, S, C>(buf, p.n, Ns, p.tw); break;
    }
    Ns *= p.rad[i];
  }
  __syncthreads();
}

// threads needed by fft_inplace for lengths up to n_max over C columns
inline int inplace_threads(int C, int n_max) {
  int t = (C * n_max + 15) / 16;
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

}  // namespace ALFA_PREC
}  // namespace alfa
