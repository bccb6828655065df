// Tile-kernel building blocks shared by the 2-D transforms
// (alfa_spectral.cu) and the 1-D line passes (alfa_line.cu).
#pragma once
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

static inline void set_smem(const void* f, size_t bytes) {
  cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

#define ALFA_Y_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) \
  X(512) X(768)

// (forward length, inverse length) pairs with a specialised k_x
#define ALFA_X_PAIRS(X) X(16, 16) X(16, 24) X(24, 16) X(24, 24) X(32, 32) X(32, 48) X(48, 32) \
  X(48, 48) X(64, 64) X(64, 96) X(96, 64) X(96, 96) X(128, 128) X(128, 192) X(192, 128)         \
  X(192, 192) X(256, 256) X(256, 384) X(384, 256) X(384, 384)

}  // namespace alfa
