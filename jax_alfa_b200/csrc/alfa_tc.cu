// Split-BF16 line passes on the 5th-generation tensor cores (tcgen05).
//
// Every separable spectral line pass of the step (truncation, i*k, the 3/2
// pad and unpad) is a real linear operator along one axis: for a slab of
// lines stored as rows of an (n_in, ncols) matrix X (x lines of an (nx, ny,
// nz) field: ncols = ny * nz, contiguous), the pass is Y = M X with M the
// real n_out x n_in matrix of the map.  Here M X runs as a GEMM on tcgen05
// with FP32 accumulation in tensor memory, the operands split into BF16
// pairs (v = v_hi + v_lo, v_hi = bf16(v), v_lo = bf16(v - v_hi)) and three
// products M_hi X_hi + M_hi X_lo + M_lo X_hi, which keeps about 16
// significant bits per product (the dropped M_lo X_lo term and the rounding
// of the lo parts are O(2^-16) relative).
//
// Kernel structure (one CTA = 256 threads = one 128 x 256 output tile):
//   - warp 0 allocates 256 TMEM columns (the FP32 accumulator);
//   - per K chunk of 32: the operator's hi/lo rows are copied to shared
//     memory and X's FP32 columns are split into hi/lo BF16 there, both in
//     the K-major no-swizzle core-matrix layout (8 rows x 16 bytes per core
//     matrix), into one of two stages; one thread issues 2 x 3 tcgen05.mma
//     (M = 128, N = 256, K = 16) and commits them to that stage's mbarrier,
//     which every thread waits on (with an iteration limit) before the
//     stage is rewritten two chunks later, so a chunk's loads overlap the
//     previous chunk's products;
//   - the warps read the accumulator back with tcgen05.ld (32 lanes each)
//     into a shared-memory tile, half the columns at a time, and store whole
//     row segments; the TMEM columns are freed.
// No TMA and no multicast: the operand tiles are written by the threads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "alfa_internal.cuh"

namespace alfa {
namespace ALFA_PREC {

namespace tc {

constexpr int BM = 128;   // output rows per tile (operator rows)
constexpr int BN = 256;   // output columns per tile
constexpr int BK = 32;    // K per staged chunk (two chunks in flight: stages 0 and 1)
constexpr int NT = 256;   // threads
constexpr int TILE_A = BM * BK * 2;  // bytes of one BF16 operator chunk
constexpr int TILE_B = BN * BK * 2;  // bytes of one BF16 input chunk
constexpr int STAGE = 2 * TILE_A + 2 * TILE_B;  // hi and lo of both operands
constexpr int EH = 128;        // epilogue columns per pass (two passes over BN)
constexpr int TROW = EH + 4;   // epilogue tile row stride (floats): conflict-free writes
constexpr int EPI = BM * TROW * 4;  // epilogue tile bytes (reuses the stages)
constexpr int BARS = (EPI > 2 * STAGE ? EPI : 2 * STAGE);  // barriers after both
constexpr int SMEM = BARS + 64;
// mbarrier polls before a wait gives up (the default of the main loop's
// waits; a context can lower it, alfa_set_tc_spin_limit)
constexpr unsigned long long SPIN_LIMIT = 1ull << 22;
// after a wait gave up, the waits for the products still in flight, each of
// SPIN_LIMIT polls, before the accumulator is freed regardless
constexpr int CLEANUP_WAITS = 16;
constexpr int A_UNITS = BM * (BK / 8) / NT;  // 16-byte operator units per thread and chunk
static_assert(NT == 256 && BN == 2 * 4 * 32 && BK / 8 == 4 && BN == 2 * EH,
              "input staging: warp w takes K block w % 4 and column half w / 4, 32 threads x "
              "4 columns; the epilogue runs in two halves");

// byte offset of element (row r, k) in a K-major no-swizzle operand tile of
// `rows` rows: core matrices of 8 rows x 8 BF16 (128 contiguous bytes),
// consecutive along the rows (stride 128 B), K blocks of 8 at stride
// rows/8 * 128 B
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int rows) {
  return (uint32_t)(((k >> 3) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// shared-memory matrix descriptor (sm_100): start address, leading (K)
// byte offset, stride (row-group) byte offset, all >> 4; version 1; no
// swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, SWIZZLE_NONE
}

// instruction descriptor, kind::f16: FP32 accumulator, BF16 A and B, both
// K-major, N = BN, M = BM
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(IDESC), "r"(acc));
}

// false when the limit ran out.  try_wait may suspend the thread for a
// while inside one poll, so a small limit (a test's) polls with the
// non-blocking test_wait instead and gives up as soon as its polls find the
// phase incomplete.
constexpr unsigned long long SMALL_LIMIT = 64;

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity,
                                          unsigned long long limit) {
  for (unsigned long long i = 0; i < limit; i++) {
    uint32_t done;
    if (limit <= SMALL_LIMIT) {
      asm volatile(
          "{\n\t.reg .pred P1;\n\t"
          "mbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t}\n"
          : "=r"(done)
          : "r"(bar), "r"(parity)
          : "memory");
    } else {
      asm volatile(
          "{\n\t.reg .pred P1;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
          "selp.b32 %0, 1, 0, P1;\n\t}\n"
          : "=r"(done)
          : "r"(bar), "r"(parity)
          : "memory");
    }
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ uint32_t pack_bf16(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// one chunk's global loads, all issued before any is used
struct ChunkRegs {
  uint4 ah[A_UNITS], al[A_UNITS];
  float4 xv[8];
};

__device__ __forceinline__ void load_chunk(ChunkRegs& R, const __nv_bfloat16* __restrict__ Mhi,
                                           const __nv_bfloat16* __restrict__ Mlo,
                                           const float* __restrict__ X, int n_in,
                                           long long ncols, int m0, long long n0, int k0,
                                           int tid) {
  // operator: 16-byte units (8 BF16 along K), consecutive threads on
  // consecutive rows
#pragma unroll
  for (int q = 0; q < A_UNITS; q++) {
    const int u = tid + q * NT;
    const size_t g = (size_t)(m0 + u % BM) * n_in + k0 + (u / BM) * 8;
    R.ah[q] = __ldg(reinterpret_cast<const uint4*>(Mhi + g));
    R.al[q] = __ldg(reinterpret_cast<const uint4*>(Mlo + g));
  }
  // input: warp w reads the 8 rows of K block w % 4 in column half w / 4,
  // lane t4 the 4 consecutive columns 4 t4 .. 4 t4 + 3 of that half
  const int w = tid >> 5, t4 = tid & 31;
  const int kbw = w & 3, col = (w >> 2) * 128 + 4 * t4;
#pragma unroll
  for (int j = 0; j < 8; j++)
    R.xv[j] = __ldg(
        reinterpret_cast<const float4*>(X + (size_t)(k0 + kbw * 8 + j) * ncols + n0 + col));
}

// the chunk into a stage: operator units as they are, input columns split
// into hi / lo BF16 units of 8 K values
__device__ __forceinline__ void store_chunk(const ChunkRegs& R, unsigned char* stage, int tid) {
  unsigned char* sAhi = stage;
  unsigned char* sAlo = stage + TILE_A;
  unsigned char* sBhi = stage + 2 * TILE_A;
  unsigned char* sBlo = stage + 2 * TILE_A + TILE_B;
#pragma unroll
  for (int q = 0; q < A_UNITS; q++) {
    const int u = tid + q * NT;
    const uint32_t o = kmajor_off(u % BM, (u / BM) * 8, BM);
    *reinterpret_cast<uint4*>(sAhi + o) = R.ah[q];
    *reinterpret_cast<uint4*>(sAlo + o) = R.al[q];
  }
  const int w = tid >> 5, t4 = tid & 31;
  const int kbw = w & 3, col = (w >> 2) * 128 + 4 * t4;
#pragma unroll
  for (int e4 = 0; e4 < 4; e4++) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 8; j += 2) {
      const float x0 = (&R.xv[j].x)[e4], x1 = (&R.xv[j + 1].x)[e4];
      const __nv_bfloat16 h0 = __float2bfloat16_rn(x0), h1 = __float2bfloat16_rn(x1);
      const __nv_bfloat16 l0 = __float2bfloat16_rn(x0 - __bfloat162float(h0));
      const __nv_bfloat16 l1 = __float2bfloat16_rn(x1 - __bfloat162float(h1));
      h[j / 2] = pack_bf16(h0, h1);
      l[j / 2] = pack_bf16(l0, l1);
    }
    const uint32_t o = kmajor_off(col + e4, kbw * 8, BN);
    *reinterpret_cast<uint4*>(sBhi + o) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(sBlo + o) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

// the three products of one staged chunk (one thread), committed to `bar`
__device__ __forceinline__ void mma_chunk(uint32_t tmem, const unsigned char* stage, bool first,
                                          uint32_t bar) {
  const uint32_t lboA = (BM / 8) * 128, lboB = (BN / 8) * 128, sbo = 128;
  const uint32_t a = smem_u32(stage), b = a + 2 * TILE_A;
#pragma unroll
  for (int ks = 0; ks < BK / 16; ks++) {
    const uint32_t offA = ks * 2 * lboA, offB = ks * 2 * lboB;
    const uint64_t ah = smem_desc(a + offA, lboA, sbo);
    const uint64_t al = smem_desc(a + TILE_A + offA, lboA, sbo);
    const uint64_t bh = smem_desc(b + offB, lboB, sbo);
    const uint64_t bl = smem_desc(b + TILE_B + offB, lboB, sbo);
    mma_bf16(tmem, ah, bh, (first && ks == 0) ? 0u : 1u);
    mma_bf16(tmem, ah, bl, 1u);
    mma_bf16(tmem, al, bh, 1u);
  }
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
      : "memory");
}

// Y[r][c] = sum_k M[r][k] X[k][c] for one 128 x 256 tile (256 TMEM columns); Mhi/Mlo: (n_out,
// n_in) BF16 row-major; X: (n_in, ncols) FP32; Y: (n_out, ncols) FP32.
// Requires n_out % 128 == 0, ncols % 256 == 0, n_in % 32 == 0.  Two stages:
// the loads of chunk ch + 1 are in flight while chunk ch is staged and its
// products run; stage ch % 2 is rewritten once the products of chunk ch - 2
// (the barrier of that stage) have completed.
__global__ void __launch_bounds__(NT, 2)
    k_line_gemm_bf16x3(const __nv_bfloat16* __restrict__ Mhi, const __nv_bfloat16* __restrict__ Mlo,
                       const float* __restrict__ X, float* __restrict__ Y0, float* __restrict__ Y1,
                       int split, int n_in, long long ncols, long long xbs, long long ybs,
                       int* err, unsigned long long spin) {
  // batch blockIdx.z: the slab of lines at X + z xbs; output rows below
  // `split` go to Y0, the others to Y1 (two stacked maps), both + z ybs
  X += (size_t)blockIdx.z * xbs;
  Y0 += (size_t)blockIdx.z * ybs;
  Y1 += (size_t)blockIdx.z * ybs;
  extern __shared__ __align__(1024) unsigned char sm[];
  unsigned char* stages[2] = {sm, sm + STAGE};
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm + BARS);  // bar[0], bar[1]
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm + BARS + 32);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  // blockIdx.x runs over the operator's row tiles: the CTAs that read the
  // same input columns are neighbours, so the second read comes from L2
  const int m0 = blockIdx.x * BM;
  const long long n0 = (long long)blockIdx.y * BN;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar + 1)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  bool ok = true;
  const int nchunks = n_in / BK;
  // two register sets: chunk ch + 1's loads are in flight while chunk ch is
  // converted, stored and multiplied (the loop is unrolled by two so each
  // set stays in registers)
  ChunkRegs R0, R1;
  int committed = -1;  // the last chunk whose products were issued
  load_chunk(R0, Mhi, Mlo, X, n_in, ncols, m0, n0, 0, tid);
  if (nchunks > 1) load_chunk(R1, Mhi, Mlo, X, n_in, ncols, m0, n0, BK, tid);
  auto step = [&](ChunkRegs& R, int ch) {
    const int s = ch & 1;
    bool mine = true;
    if (ch >= 2) {  // stage s still feeds the products of chunk ch - 2
      mine = mbar_wait(smem_u32(bar + s), (uint32_t)(((ch - 2) >> 1) & 1), spin);
      asm volatile("tcgen05.fence::after_thread_sync;");
    }
    store_chunk(R, stages[s], tid);
    // the tensor cores read shared memory through the async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    ok = __syncthreads_and(mine) != 0;  // uniform across the CTA
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (!ok) return;
    if (tid == 0) mma_chunk(tmem, stages[s], ch == 0, smem_u32(bar + s));
    committed = ch;
    if (ch + 2 < nchunks) load_chunk(R, Mhi, Mlo, X, n_in, ncols, m0, n0, (ch + 2) * BK, tid);
  };
  for (int ch = 0; ch < nchunks && ok; ch += 2) {
    step(R0, ch);
    if (ok && ch + 1 < nchunks) step(R1, ch + 1);
  }
  if (ok) {  // the last commit covers every product issued before it
    const int L = nchunks - 1;
    const bool mine = mbar_wait(smem_u32(bar + (L & 1)), (uint32_t)((L >> 1) & 1), spin);
    asm volatile("tcgen05.fence::after_thread_sync;");
    ok = __syncthreads_and(mine) != 0;
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // a wait gave up: wait (bounded, at the full limit) for the products in
    // flight before the accumulator columns are freed; the last commit
    // covers every product issued before it.  Should even that run out, the
    // flag says so (2) and the columns are freed anyway.
    if (committed >= 0) {
      bool done = false;
      for (int k = 0; k < CLEANUP_WAITS && !done; k++)
        done = mbar_wait(smem_u32(bar + (committed & 1)), (uint32_t)((committed >> 1) & 1),
                         SPIN_LIMIT);
      if (!done && tid == 0) atomicExch(err, 2);
    }
  } else {
    // warp w may read accumulator lanes (rows) 32 (w % 4) .. + 31; the tile
    // goes through shared memory (the stages are free now), one half of the
    // columns at a time, so that the global stores are whole 512-byte row
    // segments
    const int r = (warp & 3) * 32 + lane;
    float* T = reinterpret_cast<float*>(sm);
#pragma unroll 1
    for (int h = 0; h < BN / EH; h++) {
      if ((warp >> 2) == h) {
#pragma unroll 1
        for (int c0 = 0; c0 < EH; c0 += 16) {
          uint32_t v[16];
          const uint32_t addr =
              tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(h * EH + c0);
          asm volatile(
              "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
              "%12,%13,%14,%15}, [%16];"
              : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
                "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
                "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
              : "r"(addr));
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
          for (int j = 0; j < 16; j += 4)
            *reinterpret_cast<float4*>(T + r * TROW + c0 + j) =
                make_float4(__uint_as_float(v[j]), __uint_as_float(v[j + 1]),
                            __uint_as_float(v[j + 2]), __uint_as_float(v[j + 3]));
        }
      }
      __syncthreads();
#pragma unroll 4
      for (int it = 0; it < BM / (NT / 32); it++) {
        const int row = it * (NT / 32) + warp;
        const int R = m0 + row;  // a tile's rows all lie below or above split
        float* Yr = R < split ? Y0 + (size_t)R * ncols : Y1 + (size_t)(R - split) * ncols;
        *reinterpret_cast<float4*>(Yr + n0 + h * EH + 4 * lane) =
            *reinterpret_cast<const float4*>(T + row * TROW + 4 * lane);
      }
      __syncthreads();
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}

}  // namespace tc

// ---------------------------------------------------------------------------
// host: the operator matrix of a line map, split into BF16 hi/lo
// ---------------------------------------------------------------------------

// the spectral map of line_map (alfa_line.cu) for output bin k of n_out from
// an n_in-point spectrum: the source bin (or -1) and the multiplier
static void map_bin(int map, int cut, int n_in, int n_out, int k, int* src, double* mul) {
  *src = k;
  *mul = 1.0;
  const int n = n_in;
  switch (map) {
    case LM_IDENT:
      return;
    case LM_TRUNC:
      if (!(k < cut || k >= n - cut + 1)) *src = -1;
      return;
    case LM_DERIV:
    case LM_TRUNC_DERIV: {
      if (map == LM_TRUNC_DERIV && !(k < cut || k >= n - cut + 1)) {
        *src = -1;
        return;
      }
      const int kk = (k < n / 2) ? k : (k == n / 2 ? 0 : k - n);
      *mul = (double)kk;  // times i
      return;
    }
    case LM_PAD: {
      const int h = n / 2, m = n_out;
      if (k <= h) *src = k;
      else if (k >= m - h) *src = k - m + n;
      else *src = -1;
      return;
    }
    default: {  // LM_UNPAD: n_in = m = 3 n_out / 2
      const int h = n_out / 2;
      if (k < h) *src = k;
      else if (k == h) *src = -1;
      else *src = k - n_out + n_in;
      return;
    }
  }
}

// M[j][i] = scale * Re sum_k map(k) e^{+2 pi i k j / n_out} e^{-2 pi i src(k) i / n_in},
// with the angles from per-length tables (long double, rounded once)
static void operator_matrix(int map, int cut, int n_in, int n_out, double scale,
                            std::vector<double>& M) {
  M.assign((size_t)n_out * n_in, 0.0);
  const long double two_pi = 6.283185307179586476925286766559L;
  std::vector<double> co(n_out), so(n_out), ci(n_in), si(n_in);
  for (int t = 0; t < n_out; t++) {
    co[t] = (double)cosl(two_pi * t / n_out);
    so[t] = (double)sinl(two_pi * t / n_out);
  }
  for (int t = 0; t < n_in; t++) {
    ci[t] = (double)cosl(two_pi * t / n_in);
    si[t] = (double)sinl(two_pi * t / n_in);
  }
  const bool deriv = (map == LM_DERIV || map == LM_TRUNC_DERIV);
  for (int k = 0; k < n_out; k++) {
    int src;
    double mul;
    map_bin(map, cut, n_in, n_out, k, &src, &mul);
    if (src < 0 || mul == 0.0) continue;
    for (int j = 0; j < n_out; j++) {
      const int a = (int)((long long)k * j % n_out);
      const double c1 = co[a], s1 = so[a];
      double* row = M.data() + (size_t)j * n_in;
      for (int i = 0; i < n_in; i++) {
        const int b = (int)((long long)src * i % n_in);
        const double c2 = ci[b], s2 = si[b];
        // e^{i(t1 - t2)}: real c1 c2 + s1 s2, imaginary s1 c2 - c1 s2; the
        // derivative multiplies by i k (real part -k * imaginary)
        row[i] += deriv ? -mul * (s1 * c2 - c1 * s2) : (c1 * c2 + s1 * s2);
      }
    }
  }
  for (double& v : M) v *= scale;
}

// whether a line pass of these lengths and column count fits the kernel
bool tc_shape_ok(int n_in, int n_out, long long ncols) {
  return n_out % tc::BM == 0 && ncols % tc::BN == 0 && n_in % tc::BK == 0 && ncols > 0 &&
         n_in > 0;
}

int tc_prepare(Engine& e, int map, int cut, int n_in, int n_out, double scale, long long ncols,
               Engine::TcOp** out, int map2, int cut2, double scale2) {
  if (!tc_shape_ok(n_in, n_out, ncols))
    return e.fail("tc_line_apply: n_out must be a multiple of 128, ncols of 256, n_in of 32",
                  ALFA_E_SHAPE);
  for (int m : {map, map2}) {
    if (m < 0) continue;
    if ((m == LM_PAD && 2 * n_out != 3 * n_in) || (m == LM_UNPAD && 3 * n_out != 2 * n_in) ||
        (m != LM_PAD && m != LM_UNPAD && n_in != n_out))
      return e.fail("tc_line_apply: lengths do not match the map", ALFA_E_SHAPE);
  }
  // operators are built once per context and kept in its engine
  Engine::TcOp* op = nullptr;
  for (auto& o : e.tc_ops)
    if (o.map == map && o.cut == cut && o.n_in == n_in && o.n_out == n_out && o.scale == scale &&
        o.map2 == map2 && (map2 < 0 || (o.cut2 == cut2 && o.scale2 == scale2)))
      op = &o;
  if (!op) {
    std::vector<double> M;
    operator_matrix(map, cut, n_in, n_out, scale, M);
    if (map2 >= 0) {  // a second map stacked below the first
      std::vector<double> M2;
      operator_matrix(map2, cut2, n_in, n_out, scale2, M2);
      M.insert(M.end(), M2.begin(), M2.end());
    }
    std::vector<__nv_bfloat16> hi(M.size()), lo(M.size());
    for (size_t t = 0; t < M.size(); t++) {
      const float f = (float)M[t];
      hi[t] = __float2bfloat16_rn(f);
      lo[t] = __float2bfloat16_rn(f - __bfloat162float(hi[t]));
    }
    Engine::TcOp o{map, cut, n_in, n_out, scale, map2, cut2, scale2, nullptr, nullptr};
    if (cudaMalloc(&o.hi, M.size() * 2) != cudaSuccess) return e.fail("tc: allocation failed", ALFA_E_CUDA);
    e.allocs.push_back(o.hi);
    if (cudaMalloc(&o.lo, M.size() * 2) != cudaSuccess) return e.fail("tc: allocation failed", ALFA_E_CUDA);
    e.allocs.push_back(o.lo);
    cudaMemcpy(o.hi, hi.data(), M.size() * 2, cudaMemcpyHostToDevice);
    cudaMemcpy(o.lo, lo.data(), M.size() * 2, cudaMemcpyHostToDevice);
    e.tc_ops.push_back(o);
    op = &e.tc_ops.back();
  }
  if (!e.tc_err) {
    void* p = nullptr;
    if (cudaMalloc(&p, sizeof(int)) != cudaSuccess)
      return e.fail("tc_line_apply: flag allocation failed", ALFA_E_CUDA);
    e.allocs.push_back(p);
    e.tc_err = (int*)p;
  }
  cudaFuncSetAttribute((const void*)tc::k_line_gemm_bf16x3,
                       cudaFuncAttributeMaxDynamicSharedMemorySize, tc::SMEM);
  *out = op;
  return ALFA_OK;
}

// one launch (asynchronous; a wait that gave up sets e.tc_err): `batch`
// slabs of (n_in, ncols) lines at X + b xbs; the first map's rows to Y0 +
// b ybs, a stacked second map's rows to Y1 + b ybs
void tc_launch(Engine& e, const Engine::TcOp* op, long long ncols, const float* X, float* Y0,
               float* Y1, int batch, long long xbs, long long ybs) {
  const int rows = op->n_out * (op->map2 >= 0 ? 2 : 1);
  dim3 g((unsigned)(rows / tc::BM), (unsigned)(ncols / tc::BN), (unsigned)batch);
  ::alfa::note_launch();
  tc::k_line_gemm_bf16x3<<<g, tc::NT, tc::SMEM, e.stream>>>(
      (const __nv_bfloat16*)op->hi, (const __nv_bfloat16*)op->lo, X, Y0, Y1 ? Y1 : Y0,
      op->n_out, op->n_in, ncols, xbs, ybs, e.tc_err, e.tc_spin ? e.tc_spin : tc::SPIN_LIMIT);
}

int tc_line_apply(Engine& e, int map, int cut, int n_in, int n_out, double scale,
                  long long ncols, const float* X, float* Y) {
  Engine::TcOp* op = nullptr;
  const int st = tc_prepare(e, map, cut, n_in, n_out, scale, ncols, &op);
  if (st) return st;
  cudaMemsetAsync(e.tc_err, 0, sizeof(int), e.stream);
  tc_launch(e, op, ncols, X, Y, nullptr, 1, 0, 0);
  int h = 0;
  cudaMemcpyAsync(&h, e.tc_err, sizeof(int), cudaMemcpyDeviceToHost, e.stream);
  if (cudaStreamSynchronize(e.stream) != cudaSuccess)
    return e.fail("tc_line_apply: kernel failed", ALFA_E_CUDA);
  if (h == 2)
    return e.fail("tc_line_apply: a bounded tensor-core wait gave up and the products in flight "
                  "did not complete within the cleanup limit",
                  ALFA_E_TIMEOUT);
  if (h) return e.fail("tc_line_apply: a bounded tensor-core wait gave up", ALFA_E_TIMEOUT);
  return ALFA_OK;
}

}  // namespace ALFA_PREC
}  // namespace alfa
