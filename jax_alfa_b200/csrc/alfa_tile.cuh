// Tile-kernel building blocks shared by the 2-D transforms
// (alfa_spectral.cu) and the 1-D line passes (alfa_line.cu).
#pragma once
#include "alfa_fft_ct.cuh"
#include "alfa_internal.cuh"

namespace alfa {
namespace ALFA_PREC {

// Complex columns per tile: one 128-byte row segment (8 complex doubles = 16
// z levels in the FP64 build, 16 complex floats = 32 z levels in the FP32
// build).  The transform kernels are latency bound, so the FP32 build keeps
// the FP64 build's shared-memory tile and bytes in flight per SM (twice the
// threads of half the width) rather than halving them.
static constexpr int YC = (int)(128 / sizeof(cd));
static constexpr int MAXTHREADS = 48 * YC;  // in-place sweeps need C*n/16 threads (n <= 768)
// resident CTAs per SM asked of the 2-D y-transform kernels at n = 256
// (512 threads per SM in both builds)
static constexpr int Y_MINBLOCKS = 512 / (YC * 256 / 16);
static constexpr int U = 8;     // loads in flight per thread

// ---------------------------------------------------------------------------
// Loader evaluation.  ev_kind states each expression once in terms of an
// accessor at(k, d) = input k at level z + d (d = -1, 0, +1); ldv evaluates
// it at one linear index i, eval_pair at the two levels (z, z+1) of a packed
// complex column.  The kind is a compile-time constant in the tile kernels.
// The expressions are evaluated in FP64 whatever the storage precision, except
// where the accessor returns the stored type (ldv and the materialising
// pass): there a sub-expression of inputs alone, such as a difference of two
// FP32 inputs, is computed in FP32 before it meets an FP64 operand.
// ---------------------------------------------------------------------------
template <int KIND, class At>
__device__ __forceinline__ double ev_kind(const Loader& L, const At& at, int z, int nz) {
  if constexpr (KIND == LD_FIELD) {
    return at(0, 0);
  } else if constexpr (KIND == LD_MUL) {
    return at(0, 0) * at(1, 0);
  } else if constexpr (KIND == LD_MUL3) {
    return at(0, 0) * at(1, 0) * at(2, 0);
  } else if constexpr (KIND == LD_PRESSURE_R) {  // NSE_PressureTerms.py:140-142
    return at(0, 0) - L.c[0] * at(1, 0) + L.c[1] * at(2, 0);
  } else if constexpr (KIND == LD_ADV_XY) {  // NSE_AdvectionTerms.py:105-116, :122-132
    const double arg1 = at(0, 0) * (at(1, 0) - at(2, 0));
    if (z == 0) {
      const double a2n = at(3, 1) * (at(4, 1) - at(5, 1));
      return arg1 + 0.5 * a2n;
    }
    const double a2 = at(3, 0) * (at(4, 0) - at(5, 0));
    if (z == nz - 1) return arg1 + a2;
    const double a2n = at(3, 1) * (at(4, 1) - at(5, 1));
    return arg1 + 0.5 * (a2 + a2n);
  } else if constexpr (KIND == LD_ADV_Z) {  // NSE_AdvectionTerms.py:137-151
    if (z == 0 || z == nz - 1) return 0.0;
    const double ug = 0.5 * (at(0, -1) + at(0, 0));
    const double vg = 0.5 * (at(1, -1) + at(1, 0));
    const double a1 = ug * (at(2, 0) - at(3, 0));
    const double a2 = vg * (at(4, 0) - at(5, 0));
    return a1 + a2;
  } else if constexpr (KIND == LD_SCALAR_ADV) {  // SCL_AdvectionTerms.py:89-101
    const double c1 = at(0, 0) * at(3, 0) + at(1, 0) * at(4, 0);
    const double c2 = at(2, 0) * at(5, 0);
    if (z == nz - 1) return c1 + c2;
    const double c2n = at(2, 1) * at(5, 1);
    return c1 + 0.5 * (c2 + c2n);
  } else if constexpr (KIND == LD_STRESS_UVP) {  // SGSStresses_SM.py:122-132
    if (z == nz - 1) return 0.0;
    return L.c[0] * at(0, 0) * at(1, 0) * at(2, 0);
  } else if constexpr (KIND == LD_STRESS_W) {  // SGSStresses_SM.py:223-232
    if (z == 0 || z == nz - 1) return 0.0;
    return L.c[0] * (0.5 * (at(0, -1) + at(0, 0))) * at(1, 0) * at(2, 0);
  } else if constexpr (KIND == LD_W_SXX) {  // StrainRates.py:250-276, component L.sub
    // inputs: dudx dvdx dwdx dudy dvdy dwdy dudz dvdz dwdz
    auto stag = [&](int k) -> double {
      if (z == 0) return at(k, 0);
      if (z == nz - 1) return 0.0;
      return 0.5 * (at(k, -1) + at(k, 0));
    };
    switch (L.sub) {
      case 0: return stag(0);                    // S11 = ux
      case 1: return stag(4);                    // S22 = vy
      case 2: return stag(8);                    // S33 = wz
      case 3: return 0.5 * (stag(3) + stag(1));  // S12
      case 4: {                                  // S13
        const double wx = (z == 0) ? 0.5 * (at(2, 0) + at(2, 1)) : at(2, 0);
        return 0.5 * (at(6, 0) + wx);
      }
      default: {                                 // S23
        const double wy = (z == 0) ? 0.5 * (at(5, 0) + at(5, 1)) : at(5, 0);
        return 0.5 * (at(7, 0) + wy);
      }
    }
  } else if constexpr (KIND == LD_THZ) {  // DynamicSGS_ScalarLASDD_SM.py:182-185
    if (z == 0 || z == nz - 1) return at(0, 0);
    return 0.5 * (at(0, 0) + at(0, 1));
  } else if constexpr (KIND == LD_MUL_THZ) {  // S * THz
    const double t = (z == 0 || z == nz - 1) ? at(1, 0) : 0.5 * (at(1, 0) + at(1, 1));
    return at(0, 0) * t;
  } else if constexpr (KIND == LD_WL_UVP) {  // SGSStresses_WL.py:90-99, ScalarSGSFluxes_WL.py:76-81
    if (z == nz - 1) return 0.0;
    return L.c[0] * at(0, 0) * at(1, 0);
  } else {  // LD_WL_W: SGSStresses_WL.py:175-187, ScalarSGSFluxes_WL.py:149-157
    if (z == 0 || z == nz - 1) return 0.0;
    return L.c[0] * (0.5 * (at(0, -1) + at(0, 0))) * at(1, 0);
  }
}

template <int KIND>
__device__ __forceinline__ double ldv(const Loader& L, size_t i, int z) {
  return ev_kind<KIND>(L, [&](int k, int d) { return L.a[k][i + d]; }, z, L.nz);
}

// Inputs a loader kind has, and for input k whether ev_kind reads it at all
// (in), at level z-1 (m) or at level z+1 (p); `sub` selects the strain
// component of LD_W_SXX and is uniform over a launch.
__host__ __device__ constexpr int loader_nin(int kind) {
  return (kind == LD_FIELD || kind == LD_THZ) ? 1
         : (kind == LD_MUL || kind == LD_MUL_THZ || kind == LD_WL_UVP || kind == LD_WL_W) ? 2
         : (kind == LD_MUL3 || kind == LD_PRESSURE_R || kind == LD_STRESS_UVP ||
            kind == LD_STRESS_W) ? 3
         : (kind == LD_W_SXX) ? 9 : 6;
}
struct InUse {
  bool in, m, p;
};
__host__ __device__ __forceinline__ InUse loader_use(int kind, int sub, int k) {
  if (kind == LD_W_SXX) {
    switch (sub) {
      case 0: return {k == 0, k == 0, false};
      case 1: return {k == 4, k == 4, false};
      case 2: return {k == 8, k == 8, false};
      case 3: return {k == 3 || k == 1, k == 3 || k == 1, false};
      case 4: return {k == 6 || k == 2, false, k == 2};
      default: return {k == 7 || k == 5, false, k == 5};
    }
  }
  const bool m = (kind == LD_ADV_Z && k < 2) || (kind == LD_STRESS_W && k == 0) ||
                 (kind == LD_WL_W && k == 0);
  const bool p = (kind == LD_ADV_XY && k >= 3) ||
                 (kind == LD_SCALAR_ADV && (k == 2 || k == 5)) || kind == LD_THZ ||
                 (kind == LD_MUL_THZ && k == 1);
  return {true, m, p};
}

// Input k around a packed column: levels z-1, z, z+1, z+2.
struct Q4 {
  real m, x, y, p;
};

// One two-value vector load per input for the pair (z, z+1); the z-1 and z+2
// neighbours (NM, NP) come from the adjacent columns of the same row, which
// sit in adjacent lanes (lane % C == column), by warp shuffles, and from a
// scalar load at the tile's edge columns.  Every lane of the warp must call
// it; lanes with ok == false contribute zeros.
template <int C, bool NM, bool NP>
__device__ __forceinline__ Q4 fetch_q4(const real* a, size_t i, int z, int nz, int c, bool ok) {
  Q4 q{0, 0, 0, 0};
  const bool in = ok && z < nz;
  if (in) {
    const cd v = __ldg(reinterpret_cast<const cd*>(a + i));
    q.x = v.x;
    q.y = v.y;
  }
  if constexpr (NM) {
    const real t = __shfl_up_sync(0xffffffffu, q.y, 1);
    q.m = (c == 0) ? ((in && z > 0) ? __ldg(a + i - 1) : (real)0) : t;
  }
  if constexpr (NP) {
    const real t = __shfl_down_sync(0xffffffffu, q.x, 1);
    q.p = (c == C - 1) ? ((in && z + 2 < nz) ? __ldg(a + i + 2) : (real)0) : t;
  }
  return q;
}

// Value pair (z, z+1) of the loader at linear index i of level z (z even,
// nz even).  Warp-collective (see fetch_q4).
template <int KIND, int C>
__device__ __forceinline__ cd eval_pair(const Loader& L, size_t i, int z, int nz, int c,
                                        bool ok) {
  constexpr int NIN = loader_nin(KIND);
  Q4 q[NIN];
  if constexpr (KIND == LD_W_SXX) {
#pragma unroll
    for (int k = 0; k < NIN; k++) q[k] = Q4{0, 0, 0, 0};
    switch (L.sub) {  // uniform over the launch
      case 0: q[0] = fetch_q4<C, true, false>(L.a[0], i, z, nz, c, ok); break;
      case 1: q[4] = fetch_q4<C, true, false>(L.a[4], i, z, nz, c, ok); break;
      case 2: q[8] = fetch_q4<C, true, false>(L.a[8], i, z, nz, c, ok); break;
      case 3:
        q[3] = fetch_q4<C, true, false>(L.a[3], i, z, nz, c, ok);
        q[1] = fetch_q4<C, true, false>(L.a[1], i, z, nz, c, ok);
        break;
      case 4:
        q[6] = fetch_q4<C, false, false>(L.a[6], i, z, nz, c, ok);
        q[2] = fetch_q4<C, false, false>(L.a[2], i, z, nz, c, ok);
        break;
      default:
        q[7] = fetch_q4<C, false, false>(L.a[7], i, z, nz, c, ok);
        q[5] = fetch_q4<C, false, false>(L.a[5], i, z, nz, c, ok);
        break;
    }
  } else {
#pragma unroll
    for (int k = 0; k < NIN; k++) {
      constexpr bool any_m = (KIND == LD_ADV_Z || KIND == LD_STRESS_W || KIND == LD_WL_W);
      constexpr bool any_p = (KIND == LD_ADV_XY || KIND == LD_SCALAR_ADV || KIND == LD_THZ ||
                              KIND == LD_MUL_THZ);
      const bool nm = (KIND == LD_ADV_Z && k < 2) || (KIND == LD_STRESS_W && k == 0) ||
                      (KIND == LD_WL_W && k == 0);
      const bool np = (KIND == LD_ADV_XY && k >= 3) ||
                      (KIND == LD_SCALAR_ADV && (k == 2 || k == 5)) || (KIND == LD_THZ) ||
                      (KIND == LD_MUL_THZ && k == 1);
      if (any_m && nm) q[k] = fetch_q4<C, true, false>(L.a[k], i, z, nz, c, ok);
      else if (any_p && np) q[k] = fetch_q4<C, false, true>(L.a[k], i, z, nz, c, ok);
      else q[k] = fetch_q4<C, false, false>(L.a[k], i, z, nz, c, ok);
    }
  }
  auto at0 = [&](int k, int d) -> double { return d < 0 ? q[k].m : (d == 0 ? q[k].x : q[k].y); };
  auto at1 = [&](int k, int d) -> double { return d < 0 ? q[k].x : (d == 0 ? q[k].y : q[k].p); };
  return mkc((real)ev_kind<KIND>(L, at0, z, nz), (real)ev_kind<KIND>(L, at1, z + 1, nz));
}

// value pair (z, z+1) of the loader at linear index i
template <int KIND>
__device__ __forceinline__ cd load_pair(const Loader& L, size_t i, int z, int nz) {
  cd t = mkc(0, 0);
  if (KIND == LD_FIELD && (nz & 1) == 0) {
    if (z < nz) t = __ldg(reinterpret_cast<const cd*>(L.a[0] + i));
  } else {
    if (z < nz) t.x = (real)ldv<KIND>(L, i, z);
    if (z + 1 < nz) t.y = (real)ldv<KIND>(L, i + 1, z + 1);
  }
  return t;
}

// store (or accumulate) a scaled value pair at linear index i of dst
__device__ __forceinline__ void store_pair2(real* __restrict__ dst, double scale, int accumulate,
                                            size_t i, int z, int nz, cd v) {
  if (z >= nz) return;
  const real s = (real)scale;
  cd w = mkc(s * v.x, s * v.y);
  if ((nz & 1) == 0) {
    cd* p = reinterpret_cast<cd*>(dst + i);
    if (accumulate) {
      const cd pv = *p;
      w.x += pv.x;
      w.y += pv.y;
    }
    *p = w;
  } else {
    if (accumulate) {
      w.x += dst[i];
      if (z + 1 < nz) w.y += dst[i + 1];
    }
    dst[i] = w.x;
    if (z + 1 < nz) dst[i + 1] = w.y;
  }
}

__device__ __forceinline__ void store_pair(const LineOut& o, size_t i, int z, int nz, cd v) {
  store_pair2(o.dst, o.scale, o.accumulate, i, z, nz, v);
}

// Tile elements of type V (cd: one packed complex column, two z levels; cv:
// two packed columns, four z levels): the zero, i q times an element, and
// the store of a scaled element at linear index i (level z) of an output.
template <class V>
__device__ __forceinline__ V vzero();
template <>
__device__ __forceinline__ cd vzero<cd>() { return mkc(0, 0); }
__device__ __forceinline__ cd mul_ik(cd v, real q) { return mkc(-(q * v.y), q * v.x); }
__device__ __forceinline__ void store_elem(const LineOut& o, size_t i, int z, int nz, cd v) {
  store_pair(o, i, z, nz, v);
}
// z levels per element
template <class V>
__host__ __device__ constexpr int zp_of() { return (int)(sizeof(V) / sizeof(real)); }
// elements of type V per tile row: one 128-byte row segment
template <class V>
__host__ __device__ constexpr int tile_cols() { return (int)(128 / sizeof(V)); }

#ifdef ALFA_BUILD_FP32
template <>
__device__ __forceinline__ cv vzero<cv>() { return cv{dup2(0.f), dup2(0.f)}; }
__device__ __forceinline__ cv mul_ik(cv v, real q) {
  return cv{__fmul2_rn(v.im, dup2(-q)), __fmul2_rn(v.re, dup2(q))};
}
// levels z .. z+3 of a plain FP32 field (nz a multiple of 4: an element is
// wholly inside or wholly outside the field)
__device__ __forceinline__ cv ld_cv(const real* p) {
  const float4 q = __ldg(reinterpret_cast<const float4*>(p));
  return cv{make_float2(q.x, q.z), make_float2(q.y, q.w)};
}
// the loader kinds a two-lane kernel evaluates inline: no z neighbours
__host__ __device__ constexpr bool cv_inline_kind(int kind) {
  return kind == LD_FIELD || kind == LD_MUL || kind == LD_MUL3 || kind == LD_PRESSURE_R ||
         kind == LD_STRESS_UVP || kind == LD_WL_UVP;
}

// levels z .. z+3 of such a loader as a two-lane element: one 16-byte load
// per input, each level evaluated by the loader's own FP64 expression (a
// plain field is taken as loaded).  Evaluating the multi-input kinds inside
// a transform kernel is worth it only where the expression is cheap: the
// 3/2-rule unpad with the three-factor stress product inline measured 234 us
// per x pass against 117 + 62 us for the materialising pass and the
// plain-field unpad, so the line passes keep materialising.
template <int KIND>
__device__ __forceinline__ cv ld_elem_cv(const Loader& L, size_t i, int z, int nz) {
  static_assert(cv_inline_kind(KIND), "two-lane loaders: no z neighbours");
  if constexpr (KIND == LD_FIELD) {
    return ld_cv(L.a[0] + i);
  } else {
    constexpr int NI = (KIND == LD_MUL || KIND == LD_WL_UVP) ? 2 : 3;
    float4 q[NI];
#pragma unroll
    for (int k = 0; k < NI; k++) q[k] = __ldg(reinterpret_cast<const float4*>(L.a[k] + i));
    float r[4];
#pragma unroll
    for (int m = 0; m < 4; m++)
      r[m] = (float)ev_kind<KIND>(
          L, [&](int k, int) { return (double)(&q[k].x)[m]; }, z + m, nz);
    return cv{make_float2(r[0], r[2]), make_float2(r[1], r[3])};
  }
}

__device__ __forceinline__ void store_elem(const LineOut& o, size_t i, int z, int nz, cv v) {
  if (z >= nz) return;
  const float s = (float)o.scale;
  float4 w = make_float4(s * v.re.x, s * v.im.x, s * v.re.y, s * v.im.y);
  float4* p = reinterpret_cast<float4*>(o.dst + i);
  if (o.accumulate) {
    const float4 pv = *p;
    w.x += pv.x;
    w.y += pv.y;
    w.z += pv.z;
    w.w += pv.w;
  }
  *p = w;
}
#endif

// First-pass gather of a length-N transform over C packed columns:
// v[q*R + r] = loader pair at row j + r*(N/R) of column c, for butterfly
// b = threadIdx.x + q*NT (c = b % C, j = b / C); element index
// base + row*rs + z.  Warp-collective for non-field kinds (eval_pair).
template <int KIND, int C, int N, int NT>
__device__ __forceinline__ void gather_rows(const Loader& L, int nz, size_t base, size_t rs,
                                            int z0, cd* v) {
  constexpr int R = ct_radix(N);
  constexpr int NR = N / R;
  constexpr int B = NR * C;
  constexpr int MB = (B + NT - 1) / NT;
#pragma unroll
  for (int q = 0; q < MB; q++) {
    const int b = threadIdx.x + q * NT;
    const int c = b % C;
    const int j = b / C;
    const int z = z0 + 2 * c;
    const bool ok = (B % NT == 0 || b < B);
#pragma unroll
    for (int r = 0; r < R; r++) {
      const size_t i = base + (size_t)(j + r * NR) * rs + z;
      if (KIND != LD_FIELD && (nz & 1) == 0)
        v[q * R + r] = eval_pair<KIND, C>(L, i, z, nz, c, ok);
      else
        v[q * R + r] = ok ? load_pair<KIND>(L, i, z, nz) : mkc(0, 0);
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

static inline void set_smem(const void* f, size_t bytes) { raise_smem_limit(f, bytes); }

#define ALFA_Y_LENGTHS(X) X(16) X(24) X(32) X(48) X(64) X(96) X(128) X(192) X(256) X(384) \
  X(512) X(768)

// (forward length, inverse length) pairs with a specialised k_x
#define ALFA_X_PAIRS(X) X(16, 16) X(16, 24) X(24, 16) X(24, 24) X(32, 32) X(32, 48) X(48, 32) \
  X(48, 48) X(64, 64) X(64, 96) X(96, 64) X(96, 96) X(128, 128) X(128, 192) X(192, 128)         \
  X(192, 192) X(256, 256) X(256, 384) X(384, 256) X(384, 384)

}  // namespace ALFA_PREC
}  // namespace alfa
