// Learned SGS coefficient: a 10 -> 64 -> 64 -> 2 multilayer perceptron
// (tanh hidden layers) that predicts Cs^2 and beta from local resolved-strain
// and scalar-gradient quantities, with its own training (forward, backward,
// Adam) and inference kernels.  No counterpart in the reference: the
// dynamic procedure of the reference (LASDD-SM) produces the training
// targets and judges the network.
//
// Features at a uvp node (FP64 arithmetic, stored as FP32):
//   f0   log(Delta^2 |S| + 1e-12)
//   f1-6 S_ij / |S| for ij = 11, 22, 33, 12, 13, 23 (the normalised strain
//        rate tensor, staggered as StrainsUVPnodes does)
//   f7   dtheta/dz at the node (the THz interpolation of the scalar model)
//   f8   z / Delta
//   f9   local gradient Richardson number Ri = (g/T0) dtheta/dz / (uz^2 + vz^2),
//        mapped to Ri / (1 + |Ri|) (Ri is unbounded where the shear vanishes)
// Targets: the clipped Cs^2 of the dynamic procedure and its beta profile.
// Training keeps FP32 master weights and FP32 accumulation; inference uses
// the weights rounded to BF16, accumulating in FP32.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>

#include "alfa_mlp.cuh"

namespace alfa {

static constexpr int TPB_MLP = 256;
static constexpr int BS = 64;  // samples per training block (one per thread)

__device__ __forceinline__ void mlp_features(const MlpFeatIn& a, size_t i, float* f) {
  const int nz = a.nz;
  const int z = (int)(i % nz);
  const double* const* g = a.g;
  double uz, vz, wx, wy;
  if (z == 0) {
    uz = g[6][i];
    vz = g[7][i];
    wx = 0.5 * g[2][i + 1];
    wy = 0.5 * g[5][i + 1];
  } else if (z == nz - 1) {
    uz = g[6][i];
    vz = g[7][i];
    wx = g[2][i];
    wy = g[5][i];
  } else {
    uz = 0.5 * (g[6][i] + g[6][i + 1]);
    vz = 0.5 * (g[7][i] + g[7][i + 1]);
    wx = 0.5 * (g[2][i] + g[2][i + 1]);
    wy = 0.5 * (g[5][i] + g[5][i + 1]);
  }
  const double s11 = g[0][i], s22 = g[4][i], s33 = g[8][i];
  const double s12 = 0.5 * (g[3][i] + g[1][i]);
  const double s13 = 0.5 * (uz + wx);
  const double s23 = 0.5 * (vz + wy);
  const double S = sqrt(2.0 * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12) +
                               2.0 * (s13 * s13) + 2.0 * (s23 * s23)));
  const double iS = 1.0 / (S + 1e-30);
  const double* T = a.dTHdz;
  const double thz = (z == 0 || z == nz - 1) ? T[i] : 0.5 * (T[i] + T[i + 1]);
  f[0] = (float)log(a.L * a.L * S + 1e-12);
  f[1] = (float)(s11 * iS);
  f[2] = (float)(s22 * iS);
  f[3] = (float)(s33 * iS);
  f[4] = (float)(s12 * iS);
  f[5] = (float)(s13 * iS);
  f[6] = (float)(s23 * iS);
  f[7] = (float)thz;
  f[8] = (float)((z + 0.5) * a.dz / a.L);
  const double ri = a.g_over_T0 * thz / (uz * uz + vz * vz + 1e-12);
  f[9] = (float)(ri / (1.0 + fabs(ri)));
}

// splitmix-style hash -> point index
__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

__global__ void k_mlp_sample(MlpFeatIn a, const double* __restrict__ Cs2,
                             const double* __restrict__ beta, size_t N, unsigned long long seed,
                             int k, float* X, float* T, int offset, int cap) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < k; s += gridDim.x * blockDim.x) {
    const size_t i = (size_t)(mix64(seed * 0x100000001B3ull + (unsigned long long)s) % N);
    const int slot = (offset + s) % cap;
    mlp_features(a, i, X + (size_t)slot * MLP_IN);
    T[(size_t)slot * 2 + 0] = (float)Cs2[i];
    T[(size_t)slot * 2 + 1] = (float)beta[i % a.nz];
  }
}

void mlp_sample(cudaStream_t st, const MlpFeatIn& a, const double* Cs2, const double* beta,
                size_t N, unsigned long long seed, int k, float* X, float* T, int offset,
                int cap) {
  ::alfa::note_launch();
  k_mlp_sample<<<(k + TPB_MLP - 1) / TPB_MLP, TPB_MLP, 0, st>>>(a, Cs2, beta, N, seed, k, X, T,
                                                                offset, cap);
}

// mean and standard deviation of the 10 features and 2 targets over n
// samples (one block per column, FP64 sums)
__global__ void k_mlp_norm(const float* __restrict__ X, const float* __restrict__ T, int n,
                           float* norm) {
  const int col = blockIdx.x;  // 0..11
  __shared__ double s1[256], s2[256];
  double a = 0.0, b = 0.0;
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    const double v = col < MLP_IN ? X[(size_t)r * MLP_IN + col] : T[(size_t)r * 2 + col - MLP_IN];
    a += v;
    b += v * v;
  }
  s1[threadIdx.x] = a;
  s2[threadIdx.x] = b;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double mu = s1[0] / n;
    const double var = s2[0] / n - mu * mu;
    norm[col] = (float)mu;
    norm[MLP_IN + 2 + col] = (float)(var > 1e-20 ? sqrt(var) : 1.0);
  }
}

void mlp_norm(cudaStream_t st, const float* X, const float* T, int n, float* norm) {
  ::alfa::note_launch();
  k_mlp_norm<<<MLP_IN + 2, 256, 0, st>>>(X, T, n, norm);
}

// parameter offsets
static constexpr int OW1 = 0, OB1 = OW1 + MLP_H * MLP_IN, OW2 = OB1 + MLP_H,
                     OB2 = OW2 + MLP_H * MLP_H, OW3 = OB2 + MLP_H, OB3 = OW3 + 2 * MLP_H;
static_assert(OB3 + 2 == MLP_NPARAM, "parameter layout");

// Loss (mean over samples and both outputs of the squared error in
// normalised units) and its gradient, summed into grad (FP32 atomics) and
// loss; samples idx[s0 .. s0+n), features/targets normalised with norm.
__global__ void __launch_bounds__(BS) k_mlp_grad(const float* __restrict__ P,
                                                 const float* __restrict__ X,
                                                 const float* __restrict__ T,
                                                 const int* __restrict__ idx, int s0, int n,
                                                 int total, const float* __restrict__ norm,
                                                 float* grad, float* loss) {
  extern __shared__ float sm[];
  float* W = sm;                           // MLP_NPARAM
  float* H1 = W + MLP_NPARAM;              // [BS][MLP_H + 1]
  float* H2 = H1 + BS * (MLP_H + 1);       // [BS][MLP_H + 1]
  float* XS = H2 + BS * (MLP_H + 1);       // [BS][MLP_IN]
  float* DY = XS + BS * MLP_IN;            // [BS][2]
  const int t = threadIdx.x;
  for (int q = t; q < MLP_NPARAM; q += BS) W[q] = P[q];
  const int s = blockIdx.x * BS + t;
  const bool ok = s < n;
  const int r = ok ? (idx ? idx[(s0 + s) % total] : (s0 + s) % total) : 0;
  const float scale = 1.0f / (2.0f * (float)n);
  float* x = XS + t * MLP_IN;
  for (int f = 0; f < MLP_IN; f++)
    x[f] = ok ? (X[(size_t)r * MLP_IN + f] - norm[f]) / norm[MLP_IN + 2 + f] : 0.0f;
  __syncthreads();
  // forward
  float* h1 = H1 + t * (MLP_H + 1);
  float* h2 = H2 + t * (MLP_H + 1);
  for (int k = 0; k < MLP_H; k++) {
    float acc = W[OB1 + k];
    for (int f = 0; f < MLP_IN; f++) acc += W[OW1 + k * MLP_IN + f] * x[f];
    h1[k] = tanhf(acc);
  }
  for (int k = 0; k < MLP_H; k++) {
    float acc = W[OB2 + k];
    for (int j = 0; j < MLP_H; j++) acc += W[OW2 + k * MLP_H + j] * h1[j];
    h2[k] = tanhf(acc);
  }
  float l = 0.0f;
  for (int o = 0; o < 2; o++) {
    float y = W[OB3 + o];
    for (int k = 0; k < MLP_H; k++) y += W[OW3 + o * MLP_H + k] * h2[k];
    const float tn = ok ? (T[(size_t)r * 2 + o] - norm[MLP_IN + o]) / norm[2 * MLP_IN + 2 + o]
                        : 0.0f;
    const float d = ok ? (y - tn) : 0.0f;
    l += d * d;
    DY[t * 2 + o] = 2.0f * d * scale;
  }
  atomicAdd(loss, l * scale);
  __syncthreads();
  // dW3, db3 (thread t owns hidden unit t)
  if (t < MLP_H) {
    for (int o = 0; o < 2; o++) {
      float a = 0.0f;
      for (int q = 0; q < BS; q++) a += DY[q * 2 + o] * H2[q * (MLP_H + 1) + t];
      atomicAdd(&grad[OW3 + o * MLP_H + t], a);
    }
  }
  if (t < 2) {
    float a = 0.0f;
    for (int q = 0; q < BS; q++) a += DY[q * 2 + t];
    atomicAdd(&grad[OB3 + t], a);
  }
  __syncthreads();
  // dh2 = W3^T dy * (1 - h2^2), in place of h2
  {
    float dh[MLP_H];
    for (int k = 0; k < MLP_H; k++) {
      const float hk = h2[k];
      dh[k] = (W[OW3 + k] * DY[t * 2] + W[OW3 + MLP_H + k] * DY[t * 2 + 1]) * (1.0f - hk * hk);
    }
    for (int k = 0; k < MLP_H; k++) h2[k] = dh[k];
  }
  __syncthreads();
  // dW2 row t: sum_s dh2[s][t] h1[s][j]; db2
  if (t < MLP_H) {
    float b = 0.0f;
    for (int q = 0; q < BS; q++) b += H2[q * (MLP_H + 1) + t];
    atomicAdd(&grad[OB2 + t], b);
    for (int j = 0; j < MLP_H; j++) {
      float a = 0.0f;
      for (int q = 0; q < BS; q++) a += H2[q * (MLP_H + 1) + t] * H1[q * (MLP_H + 1) + j];
      atomicAdd(&grad[OW2 + t * MLP_H + j], a);
    }
  }
  __syncthreads();
  // dh1 = W2^T dh2 * (1 - h1^2), in place of h1
  {
    float dh[MLP_H];
    for (int j = 0; j < MLP_H; j++) {
      float a = 0.0f;
      for (int k = 0; k < MLP_H; k++) a += W[OW2 + k * MLP_H + j] * h2[k];
      const float hj = h1[j];
      dh[j] = a * (1.0f - hj * hj);
    }
    for (int j = 0; j < MLP_H; j++) h1[j] = dh[j];
  }
  __syncthreads();
  // dW1 row t: sum_s dh1[s][t] x[s][f]; db1
  if (t < MLP_H) {
    float b = 0.0f;
    for (int q = 0; q < BS; q++) b += H1[q * (MLP_H + 1) + t];
    atomicAdd(&grad[OB1 + t], b);
    for (int f = 0; f < MLP_IN; f++) {
      float a = 0.0f;
      for (int q = 0; q < BS; q++) a += H1[q * (MLP_H + 1) + t] * XS[q * MLP_IN + f];
      atomicAdd(&grad[OW1 + t * MLP_IN + f], a);
    }
  }
}

size_t mlp_grad_smem() {
  return (size_t)(MLP_NPARAM + 2 * BS * (MLP_H + 1) + BS * MLP_IN + BS * 2) * sizeof(float);
}

void mlp_grad(cudaStream_t st, const float* P, const float* X, const float* T, const int* idx,
              int s0, int n, int total, const float* norm, float* grad, float* loss) {
  const size_t smem = mlp_grad_smem();
  raise_smem_limit((const void*)k_mlp_grad, smem);
  ::alfa::note_launch();
  k_mlp_grad<<<(n + BS - 1) / BS, BS, smem, st>>>(P, X, T, idx, s0, n, total, norm, grad, loss);
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; refreshes the BF16
// inference copy and clears the gradient
__global__ void k_adam(float* P, float* G, float* M, float* V, __nv_bfloat16* Pb, int n,
                       float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    const float g = G[q];
    const float m = b1 * M[q] + (1.0f - b1) * g;
    const float v = b2 * V[q] + (1.0f - b2) * g * g;
    M[q] = m;
    V[q] = v;
    const float p = P[q] - lr * (m / c1) / (sqrtf(v / c2) + eps);
    P[q] = p;
    Pb[q] = __float2bfloat16(p);
    G[q] = 0.0f;
  }
}

void mlp_adam(cudaStream_t st, float* P, float* G, float* M, float* V, __nv_bfloat16* Pb,
              float lr, int t) {
  const float b1 = 0.9f, b2 = 0.999f;
  const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
  ::alfa::note_launch();
  k_adam<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(P, G, M, V, Pb, MLP_NPARAM, lr, b1, b2, 1e-8f,
                                                    c1, c2);
}

__global__ void k_to_bf16(const float* P, __nv_bfloat16* Pb, int n) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x)
    Pb[q] = __float2bfloat16(P[q]);
}

void mlp_to_bf16(cudaStream_t st, const float* P, __nv_bfloat16* Pb) {
  ::alfa::note_launch();
  k_to_bf16<<<(MLP_NPARAM + 255) / 256, 256, 0, st>>>(P, Pb, MLP_NPARAM);
}

// Inference at every uvp node: Cs^2 = clip(y0 s_z, 0, 1) (the dynamic
// procedure's range; s_z the per-level calibration, 1 without one), beta = y1
// (diagnostic), BF16 weights, FP32 accumulation
__global__ void __launch_bounds__(TPB_MLP) k_mlp_infer(MlpFeatIn a,
                                                       const __nv_bfloat16* __restrict__ Pb,
                                                       const float* __restrict__ norm, size_t N,
                                                       const double* __restrict__ level_scale,
                                                       double* Cs2, double* beta) {
  __shared__ float W[MLP_NPARAM];
  __shared__ float nm[2 * (MLP_IN + 2)];
  for (int q = threadIdx.x; q < MLP_NPARAM; q += blockDim.x) W[q] = __bfloat162float(Pb[q]);
  for (int q = threadIdx.x; q < 2 * (MLP_IN + 2); q += blockDim.x) nm[q] = norm[q];
  __syncthreads();
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (size_t)gridDim.x * blockDim.x) {
    float x[MLP_IN];
    mlp_features(a, i, x);
    for (int f = 0; f < MLP_IN; f++) x[f] = (x[f] - nm[f]) / nm[MLP_IN + 2 + f];
    float h1[MLP_H];
#pragma unroll
    for (int k = 0; k < MLP_H; k++) {
      float acc = W[OB1 + k];
#pragma unroll
      for (int f = 0; f < MLP_IN; f++) acc += W[OW1 + k * MLP_IN + f] * x[f];
      h1[k] = tanhf(acc);
    }
    float y0 = W[OB3], y1 = W[OB3 + 1];
    for (int k = 0; k < MLP_H; k++) {
      float acc = W[OB2 + k];
#pragma unroll
      for (int j = 0; j < MLP_H; j++) acc += W[OW2 + k * MLP_H + j] * h1[j];
      const float h = tanhf(acc);
      y0 += W[OW3 + k] * h;
      y1 += W[OW3 + MLP_H + k] * h;
    }
    double c = (double)(y0 * nm[2 * MLP_IN + 2] + nm[MLP_IN]);
    if (level_scale) c *= level_scale[i % a.nz];
    Cs2[i] = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
    if (beta) beta[i] = (double)(y1 * nm[2 * MLP_IN + 3] + nm[MLP_IN + 1]);
  }
}

void mlp_infer(cudaStream_t st, int sms, const MlpFeatIn& a, const __nv_bfloat16* Pb,
               const float* norm, size_t N, const double* level_scale, double* Cs2,
               double* beta) {
  const size_t want = (N + TPB_MLP - 1) / TPB_MLP;
  const unsigned blocks = (unsigned)(want < (size_t)sms * 8 ? want : (size_t)sms * 8);
  ::alfa::note_launch();
  k_mlp_infer<<<blocks, TPB_MLP, 0, st>>>(a, Pb, norm, N, level_scale, Cs2, beta);
}

// ---------------------------------------------------------------------------
// The same inference with the 64 x 64 hidden layer on the tensor cores
// (tcgen05): a CTA of 128 threads takes tiles of 128 points, one point per
// thread.  Each thread computes its point's features and first layer and
// writes the 64 activations, rounded to BF16, as row `tid` of the A operand
// (K-major, no swizzle: core matrices of 8 rows x 16 bytes); the BF16 second-
// layer weights are the B operand (64 outputs x 64 inputs, K-major).  One
// thread issues the four K = 16 MMAs (M = 128, N = 64, FP32 accumulation in
// 64 tensor-memory columns) and commits them to an mbarrier; after the
// (bounded) wait each warp reads its 32 rows back with tcgen05.ld, so every
// thread gets its own point's 64 pre-activations for the tanh and the
// output layer.  Differs from k_mlp_infer by the BF16 rounding of the first
// layer's activations.  A wait that gives up writes NaN for the tile's
// points (a step using them then reports a non-finite state) and waits,
// bounded, for the products in flight before the columns are freed.
// ---------------------------------------------------------------------------
namespace umma {

constexpr int TM = 128;  // points per tile (the MMA's M), threads per CTA
constexpr int TN = MLP_H;  // hidden units (the MMA's N and K)
constexpr int A_BYTES = TM * TN * 2;
constexpr int B_BYTES = TN * TN * 2;
constexpr int F_OFF = A_BYTES + B_BYTES;  // FP32 weights of the other layers
constexpr int NF = MLP_H * MLP_IN + MLP_H + MLP_H + 2 * MLP_H + 2 + 2 * (MLP_IN + 2);
constexpr int BAR_OFF = F_OFF + ((NF * 4 + 15) / 16) * 16;
constexpr int SMEM = BAR_OFF + 32;
constexpr unsigned long long SPIN = 1ull << 22;
constexpr int CLEANUP_WAITS = 16;
// kind::f16 instruction descriptor: FP32 accumulator, BF16 A and B, both
// K-major, N = 64, M = 128
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
// byte offset of element (row r, k) in a K-major no-swizzle tile of `rows` rows
__device__ __forceinline__ uint32_t kmajor_off(int r, int k, int rows) {
  return (uint32_t)(((k >> 3) * (rows >> 3) + (r >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2);
}
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}
// the hardware's single-instruction tanh (tanh.approx.f32, relative error
// ~2^-11): the tensor-core inference rounds the activations to BF16 (2^-9)
// anyway, and the multi-instruction tanhf held the SFU pipe at half its
// throughput
__device__ __forceinline__ float tanh_hw(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ bool bar_wait(uint32_t bar, uint32_t parity,
                                         unsigned long long limit) {
  for (unsigned long long i = 0; i < limit; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}\n"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

}  // namespace umma

__global__ void __launch_bounds__(umma::TM) k_mlp_infer_tc(MlpFeatIn a,
                                                           const __nv_bfloat16* __restrict__ Pb,
                                                           const float* __restrict__ norm,
                                                           size_t N,
                                                           const double* __restrict__ level_scale,
                                                           double* Cs2) {
  using namespace umma;
  extern __shared__ __align__(1024) unsigned char sm_mlp[];
  unsigned char* At = sm_mlp;
  unsigned char* Bt = sm_mlp + A_BYTES;
  float* F = reinterpret_cast<float*>(sm_mlp + F_OFF);
  float* W1 = F;                          // 64 x 10
  float* B1 = W1 + MLP_H * MLP_IN;        // 64
  float* B2 = B1 + MLP_H;                 // 64
  float* W3 = B2 + MLP_H;                 // 2 x 64
  float* B3 = W3 + 2 * MLP_H;             // 2
  float* NM = B3 + 2;                     // 24
  uint64_t* bar = reinterpret_cast<uint64_t*>(sm_mlp + BAR_OFF);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm_mlp + BAR_OFF + 16);
  const int tid = threadIdx.x, warp = tid >> 5;

  for (int q = tid; q < MLP_H * MLP_IN; q += TM) W1[q] = __bfloat162float(Pb[OW1 + q]);
  for (int q = tid; q < MLP_H; q += TM) {
    B1[q] = __bfloat162float(Pb[OB1 + q]);
    B2[q] = __bfloat162float(Pb[OB2 + q]);
  }
  for (int q = tid; q < 2 * MLP_H; q += TM) W3[q] = __bfloat162float(Pb[OW3 + q]);
  if (tid < 2) B3[tid] = __bfloat162float(Pb[OB3 + tid]);
  for (int q = tid; q < 2 * (MLP_IN + 2); q += TM) NM[q] = norm[q];
  // B operand: row n = hidden unit of the second layer, K = its 64 inputs
  for (int q = tid; q < TN * (TN / 8); q += TM) {
    const int n = q / (TN / 8), kb = q % (TN / 8);
    *reinterpret_cast<uint4*>(Bt + kmajor_off(n, kb * 8, TN)) =
        *reinterpret_cast<const uint4*>(Pb + OW2 + n * MLP_H + kb * 8);
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  const uint32_t aA = smem_u32(At), aB = smem_u32(Bt);
  const uint32_t lboA = (TM / 8) * 128, lboB = (TN / 8) * 128, sbo = 128;

  uint32_t phase = 0;
  bool issued = false;  // products of this CTA issued and not yet waited for
  const size_t ntiles = (N + TM - 1) / TM;
  for (size_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const size_t i = tile * TM + tid;
    const bool valid = i < N;
    float x[MLP_IN];
    if (valid) {
      mlp_features(a, i, x);
    } else {
#pragma unroll
      for (int f = 0; f < MLP_IN; f++) x[f] = NM[f];
    }
#pragma unroll
    for (int f = 0; f < MLP_IN; f++) x[f] = (x[f] - NM[f]) / NM[MLP_IN + 2 + f];
    // first layer, written as row tid of A in BF16, 8 K values per 16 bytes
#pragma unroll
    for (int kb = 0; kb < TN / 8; kb++) {
      uint32_t pk[4];
#pragma unroll
      for (int e = 0; e < 4; e++) {
        float h[2];
#pragma unroll
        for (int t = 0; t < 2; t++) {
          const int k = kb * 8 + 2 * e + t;
          float acc = B1[k];
#pragma unroll
          for (int f = 0; f < MLP_IN; f++) acc += W1[k * MLP_IN + f] * x[f];
          h[t] = tanh_hw(acc);
        }
        pk[e] = (uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(h[0])) |
                ((uint32_t)__bfloat16_as_ushort(__float2bfloat16_rn(h[1])) << 16);
      }
      *reinterpret_cast<uint4*>(At + kmajor_off(tid, kb * 8, TM)) =
          make_uint4(pk[0], pk[1], pk[2], pk[3]);
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (tid == 0) {
#pragma unroll
      for (int ks = 0; ks < TN / 16; ks++) {
        const uint64_t da = smem_desc(aA + ks * 2 * lboA, lboA, sbo);
        const uint64_t db = smem_desc(aB + ks * 2 * lboB, lboB, sbo);
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
            "l"(da), "l"(db), "r"(IDESC), "r"(ks > 0 ? 1u : 0u));
      }
      asm volatile(
          "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
              smem_u32(bar))
          : "memory");
    }
    issued = true;
    const bool mine = bar_wait(smem_u32(bar), phase, SPIN);
    asm volatile("tcgen05.fence::after_thread_sync;");
    const bool ok = __syncthreads_and(mine) != 0;
    if (!ok) {
      if (valid) Cs2[i] = __longlong_as_double(0x7FF8000000000000ll);  // NaN: the tile failed
      break;
    }
    issued = false;
    phase ^= 1u;
    // this thread's row of the accumulator, 16 columns at a time (the step
    // uses the Cs^2 output only)
    float y0 = B3[0];
#pragma unroll
    for (int c0 = 0; c0 < TN; c0 += 16) {
      uint32_t v[16];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,"
          "%12,%13,%14,%15}, [%16];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
            "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
            "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
          : "r"(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
      for (int j = 0; j < 16; j++) {
        y0 += W3[c0 + j] * tanh_hw(__uint_as_float(v[j]) + B2[c0 + j]);
      }
    }
    if (valid) {
      double c = (double)(y0 * NM[2 * MLP_IN + 2] + NM[MLP_IN]);
      if (level_scale) c *= level_scale[i % a.nz];
      Cs2[i] = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
    }
    // the A tile and the accumulator are rewritten by the next tile
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
  }
  if (issued) {  // a wait gave up: let the products in flight finish (bounded)
    bool done = false;
    for (int k = 0; k < CLEANUP_WAITS && !done; k++) done = bar_wait(smem_u32(bar), phase, SPIN);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
}

void mlp_infer_tc(cudaStream_t st, int sms, const MlpFeatIn& a, const __nv_bfloat16* Pb,
                  const float* norm, size_t N, const double* level_scale, double* Cs2) {
  static_assert(umma::SMEM <= 48 * 1024, "dynamic shared memory within the default limit");
  const size_t tiles = (N + umma::TM - 1) / umma::TM;
  const unsigned blocks = (unsigned)(tiles < (size_t)sms * 4 ? tiles : (size_t)sms * 4);
  ::alfa::note_launch();
  k_mlp_infer_tc<<<blocks, umma::TM, umma::SMEM, st>>>(a, Pb, norm, N, level_scale, Cs2);
}

// features of every point into X (N x 10), for tests and diagnostics
__global__ void k_mlp_features_all(MlpFeatIn a, size_t N, float* X) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (size_t)gridDim.x * blockDim.x)
    mlp_features(a, i, X + i * MLP_IN);
}

void mlp_features_all(cudaStream_t st, const MlpFeatIn& a, size_t N, float* X) {
  ::alfa::note_launch();
  k_mlp_features_all<<<(unsigned)((N + 255) / 256 < 4096 ? (N + 255) / 256 : 4096), 256, 0, st>>>(
      a, N, X);
}

}  // namespace alfa
