// Compile-time specialised Stockham FFT over an N x C shared-memory
// tile (the same transform as fft_inplace in alfa_fft.cuh, with the radix
// sequence, thread count and per-thread butterfly count all known to the
// compiler: index arithmetic folds to shifts and constant multiplies, every
// pass is straight-line code, and no pass is a function call).
#pragma once
#include "alfa_fft.cuh"

namespace alfa {
namespace ALFA_PREC {

// radix taken for the remaining length m (the same greedy order as the
// runtime plan: 16, 8, 4, 3, 2)
__host__ __device__ constexpr int ct_radix(int m) {
  return (m % 16 == 0) ? 16 : (m % 8 == 0) ? 8 : (m % 4 == 0) ? 4 : (m % 3 == 0) ? 3 : 2;
}

// threads of a CTA running N x C tiles: one radix-16 butterfly's worth of
// elements (16) per thread, at least two warps
__host__ __device__ constexpr int ct_threads(int C, int N) {
  int t = (C * N + 15) / 16;
  t = (t + 31) / 32 * 32;
  return t < 64 ? 64 : t;
}

// Element type V: cd, or the two-lane cv of the FP32 build (alfa_fft.cuh);
// C counts elements of V per tile row.
template <int R, int S, int C, int N, int NS, int NT, class V>
__device__ __forceinline__ void ct_pass(V* __restrict__ buf, const cd* __restrict__ tw) {
  constexpr int NR = N / R;
  constexpr int B = NR * C;
  constexpr int MB = (B + NT - 1) / NT;
  constexpr int STRIDE = N / (NS * R);
  V v[MB * R];
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (B % NT == 0 || b < B) {
      const int c = b % C;
      const int j = b / C;
#pragma unroll
      for (int r = 0; r < R; r++) v[q * R + r] = buf[(j + r * NR) * C + c];
      if (NS > 1) {
        const int k = j % NS;
#pragma unroll
        for (int r = 1; r < R; r++) {
          cd w = __ldg(&tw[k * r * STRIDE]);
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
    const int b = threadIdx.x + q * NT;
    if (B % NT == 0 || b < B) {
      const int c = b % C;
      const int j = b / C;
      const int k = j % NS;
      const int idxD = (j / NS) * NS * R + k;
#pragma unroll
      for (int r = 0; r < R; r++) buf[(idxD + r * NS) * C + c] = v[q * R + r];
    }
  }
}

template <int S, int C, int N, int NS, int NT, class V>
__device__ __forceinline__ void ct_passes(V* buf, const cd* tw) {
  if constexpr (NS < N) {
    constexpr int R = ct_radix(N / NS);
    __syncthreads();
    ct_pass<R, S, C, N, NS, NT>(buf, tw);
    ct_passes<S, C, N, NS * R, NT>(buf, tw);
  }
}

// Unnormalised in-place transform of the N x C tile; blockDim.x must be NT.
// Leaves a __syncthreads() behind.
template <int S, int C, int N, int NT, class V>
__device__ __forceinline__ void fft_ct(V* buf, const cd* tw) {
  ct_passes<S, C, N, 1, NT>(buf, tw);
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Register-resident ends of the same transform.  The first pass (NS = 1)
// reads x[j + r*N/R] of column c for butterfly b = threadIdx.x + q*NT
// (c = b % C, j = b / C) and the last pass writes X[j + r*NS_last] of the
// same butterfly, so a kernel can load the first pass's inputs straight
// from global memory into registers and store the last pass's outputs
// straight from registers, skipping two trips through shared memory.
// ---------------------------------------------------------------------------

// the remaining-length product NS at which the last pass of length N starts
__host__ __device__ constexpr int ct_last_ns(int N, int NS = 1) {
  return NS * ct_radix(N / NS) >= N ? NS : ct_last_ns(N, NS * ct_radix(N / NS));
}

// butterflies per thread of the pass that starts at NS
__host__ __device__ constexpr int ct_mb(int C, int N, int NS, int NT) {
  return ((N / ct_radix(N / NS)) * C + NT - 1) / NT;
}

// First pass from registers v[q*R + r]; outputs go to buf.  The caller makes
// sure no thread still reads buf.  Requires more than one pass.
template <int S, int C, int N, int NT, class V>
__device__ __forceinline__ void ct_first_reg(V* v, V* __restrict__ buf) {
  constexpr int R = ct_radix(N);
  constexpr int B = (N / R) * C;
  constexpr int MB = (B + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (B % NT == 0 || b < B) {
      const int c = b % C;
      const int j = b / C;
      dftR<R, S>(v + q * R);
#pragma unroll
      for (int r = 0; r < R; r++) buf[(j * R + r) * C + c] = v[q * R + r];
    }
  }
}

// Passes that start at NS, up to but excluding the last one, in buf.
template <int S, int C, int N, int NS, int NT, class V>
__device__ __forceinline__ void ct_mid_passes(V* buf, const cd* tw) {
  if constexpr (NS < ct_last_ns(N)) {
    constexpr int R = ct_radix(N / NS);
    __syncthreads();
    ct_pass<R, S, C, N, NS, NT>(buf, tw);
    ct_mid_passes<S, C, N, NS * R, NT>(buf, tw);
  }
}

// Last pass from buf into registers v[q*R + r] = X[j + r*NS] (the caller
// synchronises before).  Requires more than one pass.
template <int S, int C, int N, int NT, class V>
__device__ __forceinline__ void ct_last_reg(const V* __restrict__ buf, const cd* __restrict__ tw,
                                            V* v) {
  constexpr int NS = ct_last_ns(N);
  constexpr int R = N / NS;
  constexpr int B = NS * C;
  constexpr int MB = (B + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    if (B % NT == 0 || b < B) {
      const int c = b % C;
      const int j = b / C;
#pragma unroll
      for (int r = 0; r < R; r++) v[q * R + r] = buf[(j + r * NS) * C + c];
#pragma unroll
      for (int r = 1; r < R; r++) {
        cd w = __ldg(&tw[j * r]);
        if (S > 0) w.y = -w.y;
        v[q * R + r] = cmul(v[q * R + r], w);
      }
      dftR<R, S>(v + q * R);
    }
  }
}

}  // namespace ALFA_PREC
}  // namespace alfa
