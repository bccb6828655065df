// Physical-space kernels of the LES step.  Each restates a reference
// expression in the reference's evaluation order (cited per kernel); the
// fields are (nx, ny, nz) z-fastest, so z stencils are unit-stride and a
// warp reading consecutive z is coalesced.
#include <cmath>

#include "alfa_physics.cuh"

namespace alfa {
namespace ALFA_PREC {

static constexpr int TPB = 256;

static inline int nblocks(size_t n, int tpb = TPB) {
  size_t b = (n + tpb - 1) / tpb;
  return (int)(b > 148 * 16 ? 148 * 16 : b);
}

// Grid-stride loop over n elements.  (Unrolling it for more loads in flight
// measured slower for the many-input kernels: their register budgets grew and
// their occupancy fell; the few-input in-place AB2 batches two elements
// explicitly instead.)
#define GRID_STRIDE(i, n) \
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (n); \
                               i += (size_t)gridDim.x * blockDim.x)

// ---------------------------------------------------------------------------
// plane reductions: partial sums over blocks of (x, y) rows, then a fixed
// order sum of the partials (deterministic, independent of timing)
// ---------------------------------------------------------------------------
// 1024 blocks of 128 threads: ~28 resident warps per SM for the wide
// LASDD / statistics sums (256 blocks left ~7 per SM and these kernels
// latency-bound); e.red holds RED_BLOCKS x 18 x nz partials
static constexpr int RED_BLOCKS = 1024;
static constexpr int RED_MAXQ = 16;

struct RedArgs {
  const real* f[RED_MAXQ];
  int nq;
};

__global__ void k_plane_partial(RedArgs a, size_t H, int nz, double* __restrict__ part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int q = 0; q < a.nq; q++) {
    for (int z = threadIdx.x; z < nz; z += blockDim.x) {
      double s = 0.0;
      for (size_t r = r0; r < r1; r++) s += a.f[q][r * nz + z];
      part[((size_t)blockIdx.x * a.nq + q) * nz + z] = s;
    }
  }
}

// Sum of the per-block partials in a fixed order (deterministic): thread
// (x, y) of a 32 x 32 block adds partials b = y, y + 32, ... of entry
// t = 32 blockIdx.x + x, then the 32 column sums are added in order of y.
// Launch with finish_grid(nq * nz) blocks of dim3(32, 32).
__global__ void k_partial_finish(const double* __restrict__ part, int nblk, int nq, int nz,
                                 double scale, double* __restrict__ out) {
  __shared__ double sh[32][33];
  const size_t n = (size_t)nq * nz;
  const size_t t = (size_t)blockIdx.x * 32 + threadIdx.x;
  double s = 0.0;
  if (t < n)
    for (int b = threadIdx.y; b < nblk; b += 32) s += part[(size_t)b * n + t];
  sh[threadIdx.y][threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.y == 0 && t < n) {
    double r = 0.0;
    for (int y = 0; y < 32; y++) r += sh[y][threadIdx.x];
    out[t] = r * scale;
  }
}

static inline unsigned finish_grid(size_t n) { return (unsigned)((n + 31) / 32); }

static int red_blocks(const Engine& e) {
  return (int)(e.H() < (size_t)RED_BLOCKS ? e.H() : RED_BLOCKS);
}

void plane_sums(Engine& e, const real* const* fields, int nq, double* sums) {
  RedArgs a{};
  a.nq = nq;
  for (int q = 0; q < nq; q++) a.f[q] = fields[q];
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_plane_partial<<<nb, 128, 0, e.stream>>>(a, e.H(), e.nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)nq * e.nz), dim3(32, 32), 0, e.stream>>>(e.red, nb, nq, e.nz, 1.0,
                                                                       sums);
}

// The plane mean of one field with caller-provided partial-sum storage
// (NOALLOC_RED_BLOCKS x nz doubles); the same kernels as plane_means.
void plane_mean_with_scratch(const real* F, size_t H, int nz, double* partials, double* mean,
                             cudaStream_t s) {
  RedArgs a{};
  a.nq = 1;
  a.f[0] = F;
  const int nb = (int)(H < (size_t)NOALLOC_RED_BLOCKS ? H : NOALLOC_RED_BLOCKS);
  ::alfa::note_launch(); k_plane_partial<<<nb, 128, 0, s>>>(a, H, nz, partials);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)nz), dim3(32, 32), 0, s>>>(
      partials, nb, 1, nz, 1.0 / (double)H, mean);
}

void plane_means(Engine& e, const real* const* fields, int nq, double* means) {
  RedArgs a{};
  a.nq = nq;
  for (int q = 0; q < nq; q++) a.f[q] = fields[q];
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_plane_partial<<<nb, 128, 0, e.stream>>>(a, e.H(), e.nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)nq * e.nz), dim3(32, 32), 0, e.stream>>>(
      e.red, nb, nq, e.nz, 1.0 / (double)e.H(), means);
}

// ---------------------------------------------------------------------------
// surface layer: SurfaceFlux.py:53-443 (one block: three ordered passes
// over the surface plane with block-level reductions in between)
// ---------------------------------------------------------------------------
struct SurfConst {
  double Ugal, T0, vonk_g, log_m, log_h, half_dz, z0m_s, zT_s;
  int variant;
  double sfc_val, qz_const;
  const double* sfc_series;  // non-null: sfc_val is sfc_series[*itp - 1]
  const int* itp;
  size_t H;
  int nz;
};

__device__ double block_sum(double v, double* sh) {
  // fixed-shape tree over the block (deterministic)
  const int t = threadIdx.x;
  sh[t] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (t < s) sh[t] = sh[t] + sh[t + s];
    __syncthreads();
  }
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ void most_fn(double zL, bool stable, double* psi_m, double* psi_h, double* fi_m,
                        double* fi_h) {
  if (stable) {  // MOSTstable, SurfaceFlux.py:53-80
    *psi_m = 5.0 * zL;
    *psi_h = 5.0 * zL;
    *fi_m = 1.0 + *psi_m;
    *fi_h = 1.0 + *psi_h;
  } else {  // MOSTunstable, SurfaceFlux.py:83-112
    const double x = pow(1.0 - 15.0 * zL, 0.25);
    *psi_m = -2.0 * log(0.5 * (1.0 + x)) - log(0.5 * (1.0 + x * x)) + 2.0 * atan(x) -
             3.14159265358979323846 / 2.0;
    *psi_h = -2.0 * log(0.5 * (1.0 + x * x));
    const double ix = 1.0 / x;
    *fi_m = ix;
    *fi_h = ix * ix;
  }
}

struct SurfPtr {
  const real* u;
  const real* v;
  const real* TH;
  const double* mi[6];
  double* M;
  double* ustar;
  double* q2;
  double* qavg;
  double* invOB;
  double* mo[6];
};

__global__ void k_surface(SurfConst c, SurfPtr p) {
  __shared__ double sh[1024];
  if (c.sfc_series) c.sfc_val = c.sfc_series[*c.itp - 1];
  const size_t H = c.H;
  const int nz = c.nz;
  const bool hom = (c.variant == 0 || c.variant == 2 || c.variant == 4);
  // pass 1: plane sums of the local wind speed and first-level theta
  double sM = 0.0, sT = 0.0, sQ = 0.0;
  for (size_t r = threadIdx.x; r < H; r += blockDim.x) {
    const double uu = p.u[r * nz] + c.Ugal;
    const double vv = p.v[r * nz];
    sM += sqrt(uu * uu + vv * vv);
    sT += p.TH[r * nz];
    sQ += c.qz_const;
  }
  const double meanM = block_sum(sM, sh) / (double)H;
  const double meanT = block_sum(sT, sh) / (double)H;
  const double meanQc = block_sum(sQ, sh) / (double)H;
  // pass 2: u*, diagnosed heat flux
  double sq2 = 0.0;
  for (size_t r = threadIdx.x; r < H; r += blockDim.x) {
    double M;
    if (hom) {
      M = meanM;
    } else {
      const double uu = p.u[r * nz] + c.Ugal;
      const double vv = p.v[r * nz];
      M = sqrt(uu * uu + vv * vv);
    }
    const double denom_m = c.log_m + p.mi[0][r] - p.mi[1][r];
    const double us = fmax(0.4 * M / denom_m, 1e-3);
    p.M[r] = M;
    p.ustar[r] = us;
    if (c.variant >= 4) {
      const double th_air = (c.variant == 4) ? meanT : p.TH[r * nz];
      const double denom_h = c.log_h + p.mi[2][r] - p.mi[3][r];
      const double q = (c.variant == 4) ? us * 0.4 * (c.sfc_val - th_air) * 1.0 / denom_h
                                        : us * 0.4 * (c.sfc_val - th_air) / denom_h;
      p.q2[r] = q;
      sq2 += q;
    } else if (c.variant >= 2) {
      p.q2[r] = c.sfc_val * 1.0;
    }
  }
  double qavg;
  if (c.variant >= 4) {
    qavg = block_sum(sq2, sh) / (double)H;
  } else if (c.variant >= 2) {
    qavg = c.sfc_val;
  } else {
    qavg = meanQc;
  }
  __syncthreads();
  if (threadIdx.x == 0) *p.qavg = qavg;
  // pass 3: Obukhov length and the lagged MOST functions
  const bool stable = qavg <= 0.0;
  for (size_t r = threadIdx.x; r < H; r += blockDim.x) {
    double THref;
    if (c.variant == 1 || c.variant == 3) {
      THref = p.TH[r * nz] + c.T0;
    } else {
      THref = (meanT + c.T0) * 1.0;
    }
    const double us = p.ustar[r];
    const double invOB = -(c.vonk_g * qavg) / ((us * us * us) * THref);
    p.invOB[r] = invOB;
    double pm, ph, fm, fh, d0, d1, d2;
    most_fn(c.half_dz * invOB, stable, &pm, &ph, &fm, &fh);
    double pm0, ph0;
    most_fn(c.z0m_s * invOB, stable, &pm0, &d0, &d1, &d2);
    most_fn(c.zT_s * invOB, stable, &d0, &ph0, &d1, &d2);
    p.mo[0][r] = pm;
    p.mo[1][r] = pm0;
    p.mo[2][r] = ph;
    p.mo[3][r] = ph0;
    p.mo[4][r] = fm;
    p.mo[5][r] = fh;
  }
}

int surface_flux(Engine& e, int variant, double sfc_val, const SurfaceIO& io,
                 const double* sfc_series, const int* itp) {
  SurfConst c;
  c.Ugal = e.cfg.Ugal;
  c.T0 = e.T0_nondim;
  c.vonk_g = 0.4 * e.g_nondim;
  c.log_m = std::log(0.5 * e.dz * e.z_scale / e.cfg.z0m);
  const double zref = e.cfg.zTemperature > 0.0 ? e.cfg.zTemperature : e.cfg.z0T;
  c.log_h = std::log(0.5 * e.dz * e.z_scale / zref);
  c.half_dz = 0.5 * e.dz;
  c.z0m_s = e.cfg.z0m / e.z_scale;
  c.zT_s = zref / e.z_scale;
  c.variant = variant;
  c.sfc_val = sfc_val;
  c.sfc_series = sfc_series;
  c.itp = itp;
  c.qz_const = e.qz_sfc_const;
  c.H = e.H();
  c.nz = e.nz;
  SurfPtr p;
  p.u = io.u;
  p.v = io.v;
  p.TH = io.TH;
  for (int i = 0; i < 6; i++) {
    p.mi[i] = io.most_in[i];
    p.mo[i] = io.most_out[i];
  }
  p.M = io.M;
  p.ustar = io.ustar;
  p.q2 = io.q2;
  p.qavg = io.qavg;
  p.invOB = io.invOB;
  ::alfa::note_launch(); k_surface<<<1, 1024, 0, e.stream>>>(c, p);
  return 0;
}

// ---------------------------------------------------------------------------
// vertical derivatives: Derivatives.py:190-362
// ---------------------------------------------------------------------------
__global__ void k_derivz_M(const real* __restrict__ u, const real* __restrict__ v,
                           const real* __restrict__ w, const double* __restrict__ ustar,
                           const double* __restrict__ M, const double* __restrict__ fi,
                           real* __restrict__ dudz, real* __restrict__ dvdz, real* __restrict__ dwdz, size_t n, int nz,
                           double idz, double Ugal, double den_c) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    const size_t r = rof(i, nz);
    if (z == 0) {
      const double den = M[r] * 0.4 * 0.5 * den_c;
      dudz[i] = fi[r] * ustar[r] * (u[i] + Ugal) / den;
      dvdz[i] = fi[r] * ustar[r] * v[i] / den;
    } else if (z < nz - 1) {
      dudz[i] = ((double)u[i] - (double)u[i - 1]) * idz;
      dvdz[i] = ((double)v[i] - (double)v[i - 1]) * idz;
    } else {
      dudz[i] = 0.0;
      dvdz[i] = 0.0;
    }
    dwdz[i] = (z < nz - 1) ? ((double)w[i + 1] - (double)w[i]) * idz : 0.0;
  }
}

void derivz_M(Engine& e, const real* u, const real* v, const real* w, const double* ustar,
              const double* M, const double* fi_m, real* dudz, real* dvdz, real* dwdz) {
  ::alfa::note_launch(); k_derivz_M<<<nblocks(e.N()), TPB, 0, e.stream>>>(u, v, w, ustar, M, fi_m, dudz, dvdz, dwdz,
                                                    e.N(), e.nz, e.idz, e.cfg.Ugal, e.dz);
}

__global__ void k_derivz_TH(const real* __restrict__ T, const double* __restrict__ ustar,
                            const double* __restrict__ qz, const double* __restrict__ fi,
                            real* __restrict__ out, size_t n, int nz, double idz, double den) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    const size_t r = rof(i, nz);
    if (z == 0) {
      out[i] = fi[r] * (-qz[r] / ustar[r]) / den;
    } else {
      out[i] = ((double)T[i] - (double)T[i - 1]) * idz;
    }
  }
}

void derivz_TH(Engine& e, const real* TH, const double* ustar, const double* qz,
               const double* fi_h, real* dTHdz) {
  ::alfa::note_launch(); k_derivz_TH<<<nblocks(e.N()), TPB, 0, e.stream>>>(TH, ustar, qz, fi_h, dTHdz, e.N(), e.nz,
                                                     e.idz, 0.4 * 0.5 * e.dz);
}

__device__ __forceinline__ double dz_generic(const real* F, size_t i, int z, int nz, int w,
                                             double idz) {
  if (w) return (z < nz - 1) ? ((double)F[i + 1] - (double)F[i]) * idz : 0.0;  // Derivz_Generic_w
  return (z > 0) ? ((double)F[i] - (double)F[i - 1]) * idz : 0.0;              // Derivz_Generic_uvp
}

__global__ void k_derivz_generic(const real* __restrict__ F, real* __restrict__ out, size_t n, int nz,
                                 int w, double idz) {
  GRID_STRIDE(i, n) { out[i] = dz_generic(F, i, zof(i, nz), nz, w, idz); }
}

void derivz_generic(Engine& e, const real* F, int w_nodes, real* out) {
  ::alfa::note_launch(); k_derivz_generic<<<nblocks(e.N()), TPB, 0, e.stream>>>(F, out, e.N(), e.nz, w_nodes, e.idz);
}

__global__ void k_div_finish(real* __restrict__ div, const real* __restrict__ f, size_t n, int nz, int w,
                             double idz) {
  GRID_STRIDE(i, n) { div[i] = (double)div[i] + dz_generic(f, i, zof(i, nz), nz, w, idz); }
}

void divergence_finish(Engine& e, real* div, const real* fz, int w_nodes) {
  ::alfa::note_launch(); k_div_finish<<<nblocks(e.N()), TPB, 0, e.stream>>>(div, fz, e.N(), e.nz, w_nodes, e.idz);
}

// ---------------------------------------------------------------------------
// buoyancy: NSE_BuoyancyTerms.py:49-150 (dry, H = 0)
// ---------------------------------------------------------------------------
__device__ __forceinline__ double thv_of(const real* __restrict__ TH,
                                        const real* __restrict__ H, size_t i, double T0) {
  return ((double)TH[i] + T0) * (H ? __dadd_rn(1.0, __dmul_rn(0.61, (double)H[i])) : 1.0);
}

__global__ void k_buoy(const real* __restrict__ TH, const real* __restrict__ H,
                       const double* __restrict__ bar, real* __restrict__ out, size_t n, int nz, double T0,
                       int by_mean, double hg) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    if (z == 0) {
      out[i] = 0.0;
    } else {
      const double b1 = bar[z], b0 = bar[z - 1];
      const double t1 = thv_of(TH, H, i, T0), t0 = thv_of(TH, H, i - 1, T0);
      const double n1 = (t1 - b1) / (by_mean ? b1 : T0);
      const double n0 = (t0 - b0) / (by_mean ? b0 : T0);
      out[i] = hg * (n1 + n0);
    }
  }
}

__global__ void k_thv(const real* __restrict__ TH, const real* __restrict__ H, double T0,
                      real* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) { out[i] = thv_of(TH, H, i, T0); }
}

void buoyancy(Engine& e, const real* TH, const real* H, int opt, real* out) {
  // THv = (TH + T_0)(1 + 0.61 H) and its plane mean
  real* thv = e.W;  // first workspace field
  ::alfa::note_launch(); k_thv<<<nblocks(e.N()), TPB, 0, e.stream>>>(TH, H, e.T0_nondim, thv, e.N());
  const real* f[1] = {thv};
  plane_means(e, f, 1, e.scal);
  ::alfa::note_launch(); k_buoy<<<nblocks(e.N()), TPB, 0, e.stream>>>(TH, H, e.scal, out, e.N(), e.nz,
                                                                      e.T0_nondim, opt,
                                                                      0.5 * e.g_nondim);
}

// surface moisture flux (Main.py:253-267; SurfaceFlux.py:447-504):
// qm = ustar vonk (Q_s - Q_air) / (log(0.5 dz z_scale / z_ref) + psi_h - psi_h0)
__global__ void k_moisture_surface(int mode, int het, const real* __restrict__ Q,
                                   const double* __restrict__ ustar,
                                   const double* __restrict__ psi_h,
                                   const double* __restrict__ psi_h0,
                                   const double* __restrict__ series, const int* itp,
                                   double q_host, const double* __restrict__ qbar0, double log_zq,
                                   double* qm, size_t H, int nz) {
  const double s = series ? series[*itp - 1] : q_host;
  GRID_STRIDE(r, H) {
    if (mode == 1) {
      qm[r] = s;
    } else {
      const double qa = het ? Q[r * nz] : qbar0[0];
      qm[r] = ustar[r] * 0.4 * (s - qa) / (log_zq + psi_h[r] - psi_h0[r]);
    }
  }
}

void moisture_surface(Engine& e, int mode, int het, const real* Q, const double* ustar,
                      const double* psi_h, const double* psi_h0, const double* series,
                      const int* itp, double q_host, const double* qbar0, double* qm) {
  ::alfa::note_launch();
  k_moisture_surface<<<nblocks(e.H()), TPB, 0, e.stream>>>(mode, het, Q, ustar, psi_h, psi_h0,
                                                           series, itp, q_host, qbar0, e.log_zq,
                                                           qm, e.H(), e.nz);
}

// ---------------------------------------------------------------------------
// strain rates: StrainRates.py:56-141 (uvp), 219-299 (w)
// ---------------------------------------------------------------------------
struct G9 {
  const real* g[9];
};

__device__ __forceinline__ double smag_of(double s11, double s22, double s33, double s12,
                                          double s13, double s23) {
  return sqrt(2.0 * (s11 * s11 + s22 * s22 + s33 * s33 + 2.0 * (s12 * s12) +
                     2.0 * (s13 * s13) + 2.0 * (s23 * s23)));
}

__global__ void k_strains_uvp(G9 G, real* __restrict__ S12, real* __restrict__ S13,
                              real* __restrict__ S23, real* __restrict__ S, size_t n,
                              int nz) {
  // g: dudx dvdx dwdx dudy dvdy dwdy dudz dvdz dwdz
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    const real* const* g = G.g;
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
      uz = 0.5 * ((double)g[6][i] + (double)g[6][i + 1]);
      vz = 0.5 * ((double)g[7][i] + (double)g[7][i + 1]);
      wx = 0.5 * ((double)g[2][i] + (double)g[2][i + 1]);
      wy = 0.5 * ((double)g[5][i] + (double)g[5][i + 1]);
    }
    const double s11 = g[0][i], s22 = g[4][i], s33 = g[8][i];
    const double s12 = 0.5 * ((double)g[3][i] + (double)g[1][i]);
    const double s13 = 0.5 * (uz + wx);
    const double s23 = 0.5 * (vz + wy);
    S12[i] = s12;
    S13[i] = s13;
    S23[i] = s23;
    S[i] = smag_of(s11, s22, s33, s12, s13, s23);
  }
}

void strains_uvp(Engine& e, const real* const g[9], real* S12, real* S13, real* S23, real* S) {
  G9 G;
  for (int i = 0; i < 9; i++) G.g[i] = g[i];
  ::alfa::note_launch(); k_strains_uvp<<<nblocks(e.N()), TPB, 0, e.stream>>>(G, S12, S13, S23, S, e.N(), e.nz);
}

__global__ void k_smag_w(G9 G, real* __restrict__ Sw, size_t n, int nz) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    const real* const* g = G.g;
    auto stag = [&](const real* d) -> double {
      if (z == 0) return d[i];
      if (z == nz - 1) return 0.0;
      return 0.5 * ((double)d[i - 1] + (double)d[i]);
    };
    const double s11 = stag(g[0]), s22 = stag(g[4]), s33 = stag(g[8]);
    const double s12 = 0.5 * (stag(g[3]) + stag(g[1]));
    const double wx = (z == 0) ? 0.5 * ((double)g[2][i] + (double)g[2][i + 1]) : (double)g[2][i];
    const double wy = (z == 0) ? 0.5 * ((double)g[5][i] + (double)g[5][i + 1]) : (double)g[5][i];
    const double s13 = 0.5 * ((double)g[6][i] + wx);
    const double s23 = 0.5 * ((double)g[7][i] + wy);
    Sw[i] = smag_of(s11, s22, s33, s12, s13, s23);
  }
}

void smag_w(Engine& e, const real* const g[9], real* Sw) {
  G9 G;
  for (int i = 0; i < 9; i++) G.g[i] = g[i];
  ::alfa::note_launch(); k_smag_w<<<nblocks(e.N()), TPB, 0, e.stream>>>(G, Sw, e.N(), e.nz);
}

struct P6 {
  const real* s[6];
};

__global__ void k_smag6(P6 P, real* __restrict__ out, size_t n) {
  GRID_STRIDE(i, n) {
    out[i] = smag_of(P.s[0][i], P.s[1][i], P.s[2][i], P.s[3][i], P.s[4][i], P.s[5][i]);
  }
}

void smag6(Engine& e, const real* const s[6], size_t n, real* out) {
  P6 P;
  for (int i = 0; i < 6; i++) P.s[i] = s[i];
  ::alfa::note_launch(); k_smag6<<<nblocks(n), TPB, 0, e.stream>>>(P, out, n);
}

void smag6_n(Engine& e, const real* const s[6], real* out) { smag6(e, s, e.N(), out); }

// w_ of DynamicSGS_LASDD_SM.py:180-183
__global__ void k_wstar(const real* __restrict__ w, real* __restrict__ out, size_t n, int nz) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    if (z == 0) out[i] = 0.5 * (double)w[i + 1];
    else if (z == nz - 1) out[i] = w[i - 1];
    else out[i] = 0.5 * ((double)w[i] + (double)w[i + 1]);
  }
}

void wstar(Engine& e, const real* w, real* w_) {
  ::alfa::note_launch(); k_wstar<<<nblocks(e.N()), TPB, 0, e.stream>>>(w, w_, e.N(), e.nz);
}

// ---------------------------------------------------------------------------
// LASDD (DynamicSGS_LASDD_SM.py:250-352): Germano contractions
// ---------------------------------------------------------------------------
struct LasddConst {
  double cA, cB1, cB2, cC, cD1, cD2, cE1, cE2, T1, T2;
};

__device__ __forceinline__ double contract6(const double* A, const double* B) {
  return A[0] * B[0] + A[1] * B[1] + A[2] * B[2] + 2.0 * (A[3] * B[3] + A[4] * B[4] + A[5] * B[5]);
}
__device__ __forceinline__ double sq6(const double* A) {
  return A[0] * A[0] + A[1] * A[1] + A[2] * A[2] + 2.0 * (A[3] * A[3] + A[4] * A[4] + A[5] * A[5]);
}

__device__ __forceinline__ void leonard(const real* const* ph, const real* const* hat, size_t i,
                                        double* Lo) {
  const double u = hat[0][i], v = hat[1][i], w = hat[2][i];
  Lo[0] = (double)ph[0][i] - u * u;
  Lo[1] = (double)ph[1][i] - v * v;
  Lo[2] = (double)ph[2][i] - w * w;
  Lo[3] = (double)ph[3][i] - u * v;
  Lo[4] = (double)ph[4][i] - u * w;
  Lo[5] = (double)ph[5][i] - v * w;
}

__global__ void k_lasdd_partial(LasddFields f, LasddConst c, size_t H, int nz,
                                double* __restrict__ part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double s[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t r = r0; r < r1; r++) {
      const size_t i = r * nz + z;
      double Lm[6], Qm[6], S1[6], S2[6], SS1[6], SS2[6];
      leonard(f.ph, f.hat, i, Lm);
      leonard(f.pd, f.hatd, i, Qm);
#pragma unroll
      for (int q = 0; q < 6; q++) {
        S1[q] = f.Sh[q][i];
        S2[q] = f.Sd[q][i];
        SS1[q] = f.SSh[q][i];
        SS2[q] = f.SSd[q][i];
      }
      const double Sh = f.S_hat[i], Sd = f.S_hatd[i];
      s[0] += c.cA * contract6(Lm, SS1);
      s[1] += c.cA * contract6(Qm, SS2);
      s[2] += c.cB1 * Sh * contract6(Lm, S1);
      s[3] += c.cB2 * Sd * contract6(Qm, S2);
      s[4] += c.cC * sq6(SS1);
      s[5] += c.cC * sq6(SS2);
      s[6] += c.cD1 * (Sh * Sh) * sq6(S1);
      s[7] += c.cD2 * (Sd * Sd) * sq6(S2);
      s[8] += c.cE1 * Sh * contract6(S1, SS1);
      s[9] += c.cE2 * Sd * contract6(S2, SS2);
    }
#pragma unroll
    for (int q = 0; q < 10; q++) part[((size_t)blockIdx.x * 10 + q) * nz + z] = s[q];
  }
}

static LasddConst lasdd_const(const Engine& e) {
  const double L = e.L, T = e.TFR;
  LasddConst c;
  c.cA = 2 * std::pow(L, 2.0);
  c.cB1 = 2 * std::pow(L, 2.0) * std::pow(T, 2.0);
  c.cB2 = 2 * std::pow(L, 2.0) * std::pow(T, 4.0);
  c.cC = std::pow(2 * std::pow(L, 2.0), 2.0);
  c.cD1 = (4 * std::pow(L, 4.0)) * std::pow(T, 4.0);
  c.cD2 = (4 * std::pow(L, 4.0)) * std::pow(T, 8.0);
  c.cE1 = (8 * std::pow(L, 4.0)) * std::pow(T, 2.0);
  c.cE2 = (8 * std::pow(L, 4.0)) * std::pow(T, 4.0);
  c.T1 = 2 * std::pow(L, 2.0);
  c.T2 = 2 * std::pow(T * L, 2.0);
  return c;
}

void lasdd_sums(Engine& e, const LasddFields& f, double* sums10) {
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_lasdd_partial<<<nb, 128, 0, e.stream>>>(f, lasdd_const(e), e.H(), e.nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)10 * e.nz), dim3(32, 32), 0, e.stream>>>(e.red, nb, 10, e.nz,
                                                                       1.0 / (double)e.H(), sums10);
}

// polynomial coefficients per level (ff, ee, dd, cc, bb, aa) from plane means
__global__ void k_poly(const double* __restrict__ m, int nz, int scalar, double* co) {
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    double a1 = m[0 * nz + z], a2 = m[1 * nz + z], b1 = m[2 * nz + z], b2 = m[3 * nz + z];
    double c1 = m[4 * nz + z], c2 = m[5 * nz + z], d1 = m[6 * nz + z], d2 = m[7 * nz + z];
    double e1 = m[8 * nz + z], e2 = m[9 * nz + z];
    double aa, bb, cc, dd, ee, ff;
    if (!scalar) {  // DynamicSGS_LASDD_SM.py:314-319
      aa = a1 * c2 - a2 * c1;
      bb = a2 * e1 - b1 * c2;
      cc = b2 * c1 - a1 * e2 - a2 * d1;
      dd = b1 * e2 - b2 * e1;
      ee = a1 * d2 + b2 * d1;
      ff = -b1 * d2;
    } else {  // DynamicSGS_ScalarLASDD_SM.py:285-290 (slots: a2 b2 c2 d2 e2 a4 b4 c4 d4 e4)
      const double A2 = a1, B2 = a2, C2 = b1, D2 = b2, E2 = c1;
      const double A4 = c2, B4 = d1, C4 = d2, D4 = e1, E4 = e2;
      aa = A2 * C4 - A4 * C2;
      bb = -A4 * D2 + B2 * C4;
      cc = -C2 * B4 + A2 * D4 - A4 * E2;
      dd = B2 * D4 - B4 * D2;
      ee = A2 * E4 - B4 * E2;
      ff = B2 * E4;
    }
    co[0 * nz + z] = ff;
    co[1 * nz + z] = ee;
    co[2 * nz + z] = dd;
    co[3 * nz + z] = cc;
    co[4 * nz + z] = bb;
    co[5 * nz + z] = aa;
  }
}

void lasdd_poly(Engine& e, const double* sums10, int scalar, double* coeffs6) {
  ::alfa::note_launch(); k_poly<<<1, 256, 0, e.stream>>>(sums10, e.nz, scalar, coeffs6);
}

// ---------------------------------------------------------------------------
// Laguerre iteration (Utilities.py:123-241) from 8 guesses per level and the
// beta selection of ComputeBeta1/2: one thread per (level, guess)
// ---------------------------------------------------------------------------
struct cx {
  double r, i;
};
__device__ __forceinline__ cx cxadd(cx a, cx b) { return {a.r + b.r, a.i + b.i}; }
__device__ __forceinline__ cx cxsub(cx a, cx b) { return {a.r - b.r, a.i - b.i}; }
__device__ __forceinline__ cx cxmul(cx a, cx b) { return {a.r * b.r - a.i * b.i, a.r * b.i + a.i * b.r}; }
__device__ __forceinline__ double cxabs(cx a) { return hypot(a.r, a.i); }
// Smith's algorithm for a / b
__device__ cx cxdiv(cx a, cx b) {
  if (fabs(b.r) >= fabs(b.i)) {
    if (b.r == 0.0 && b.i == 0.0) return {a.r / fabs(b.r), a.i / fabs(b.i)};
    const double rat = b.i / b.r;
    const double den = b.r + b.i * rat;
    return {(a.r + a.i * rat) / den, (a.i - a.r * rat) / den};
  }
  const double rat = b.r / b.i;
  const double den = b.i + b.r * rat;
  return {(a.r * rat + a.i) / den, (a.i * rat - a.r) / den};
}
// principal square root
__device__ cx cxsqrt(cx a) {
  if (a.r == 0.0 && a.i == 0.0) return {0.0, a.i};
  const double t = sqrt((fabs(a.r) + hypot(a.r, a.i)) * 0.5);
  if (a.r >= 0.0) return {t, a.i / (2.0 * t)};
  return {fabs(a.i) / (2.0 * t), copysign(t, a.i)};
}

__global__ void k_beta(const double* __restrict__ co, int nlev, double* beta) {
  const double guesses[8] = {0.5, 0.75, 1.0, 1.25, 1.5, 2.0, 3.0, 4.5};
  __shared__ double best[32][8];
  const int lvl_local = threadIdx.x / 8;
  const int g = threadIdx.x % 8;
  const int lvl = blockIdx.x * 32 + lvl_local;
  double val = -INFINITY;
  if (lvl < nlev) {
    double p[6];
#pragma unroll
    for (int j = 0; j < 6; j++) p[j] = co[j * nlev + lvl];
    const int n = 5;
    cx dp[5], d2p[4];
#pragma unroll
    for (int j = 0; j < 5; j++) dp[j] = {p[j] * (double)(n - j), 0.0};
#pragma unroll
    for (int j = 0; j < 4; j++) d2p[j] = {dp[j].r * (double)(n - 1 - j), 0.0};
    cx x = {guesses[g], 0.0};
    bool conv = false;
    const double tol = 1e-6;
    const cx eps = {1e-16, 0.0};
    for (int it = 0; it < 20 && !conv; it++) {
      cx f = {0.0, 0.0}, df = {0.0, 0.0}, d2f = {0.0, 0.0};
      for (int j = 0; j < 6; j++) f = cxadd(cxmul(f, x), cx{p[j], 0.0});
      for (int j = 0; j < 5; j++) df = cxadd(cxmul(df, x), dp[j]);
      for (int j = 0; j < 4; j++) d2f = cxadd(cxmul(d2f, x), d2p[j]);
      const cx fs = (cxabs(f) < 1e-16) ? eps : f;
      const cx G = cxdiv(df, fs);
      const cx G2 = cxmul(G, G);
      const cx Hh = cxsub(G2, cxdiv(d2f, fs));
      const cx inner = cxsub(cx{n * Hh.r, n * Hh.i}, G2);
      const cx disc = {(n - 1) * inner.r, (n - 1) * inner.i};
      const cx sq = cxsqrt(disc);
      const cx d1 = cxadd(G, sq), dd2 = cxsub(G, sq);
      cx den = (cxabs(d1) > cxabs(dd2)) ? d1 : dd2;
      if (cxabs(den) < 1e-16) den = eps;
      const cx xn = cxsub(x, cxdiv(cx{(double)n, 0.0}, den));
      conv = (cxabs(cxsub(xn, x)) < tol * (1.0 + cxabs(x))) || (cxabs(f) < tol);
      x = xn;
    }
    if (conv && fabs(x.i) < 1e-6 && x.r > 0.0 && x.r < 5.0) val = x.r;
  }
  best[lvl_local][g] = val;
  __syncthreads();
  if (g == 0 && lvl < nlev) {
    double m = -INFINITY;
    for (int j = 0; j < 8; j++) m = fmax(m, best[lvl_local][j]);
    beta[lvl] = isinf(m) ? 1.0 : m;
  }
}

void compute_beta(Engine& e, const double* coeffs6, int nlev, double* beta) {
  ::alfa::note_launch(); k_beta<<<(nlev + 31) / 32, 256, 0, e.stream>>>(coeffs6, nlev, beta);
}

__global__ void k_ones(double* p, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = 1.0;
}

__global__ void k_LM_MM(LasddFields f, LasddConst c, const double* __restrict__ beta,
                        real* __restrict__ LM, real* __restrict__ MM, size_t n, int nz) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    double Lm[6], Mm[6];
    leonard(f.ph, f.hat, i, Lm);
    const double b = beta[z];
    const double Sh = f.S_hat[i];
#pragma unroll
    for (int q = 0; q < 6; q++) Mm[q] = c.T1 * (double)f.SSh[q][i] - c.T2 * b * Sh * (double)f.Sh[q][i];
    LM[i] = (Lm[0] * Mm[0] + Lm[1] * Mm[1] + Lm[2] * Mm[2]) +
            2.0 * (Lm[3] * Mm[3] + Lm[4] * Mm[4] + Lm[5] * Mm[5]);
    MM[i] = sq6(Mm);
  }
}

void lasdd_LM_MM(Engine& e, const LasddFields& f, const double* beta, real* LM, real* MM) {
  ::alfa::note_launch(); k_LM_MM<<<nblocks(e.N()), TPB, 0, e.stream>>>(f, lasdd_const(e), beta, LM, MM, e.N(), e.nz);
}

// ---------------------------------------------------------------------------
// Wong-Lilly procedure (DynamicSGS_LASDD_WL.py:127-313,
// DynamicSGS_ScalarLASDD_WL.py:130-275): four plane means a1, a3, a6, a8,
// the quintic mapped from them, then M_ij / T_up, T_dn with the Delta^(4/3)
// scaling.
// ---------------------------------------------------------------------------
__global__ void k_wl_partial(LasddFields f, size_t H, int nz, double* __restrict__ part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double s[4] = {0, 0, 0, 0};
    for (size_t r = r0; r < r1; r++) {
      const size_t i = r * nz + z;
      double Lm[6], Qm[6], S1[6], S2[6];
      leonard(f.ph, f.hat, i, Lm);
      leonard(f.pd, f.hatd, i, Qm);
#pragma unroll
      for (int q = 0; q < 6; q++) {
        S1[q] = f.Sh[q][i];
        S2[q] = f.Sd[q][i];
      }
      s[0] += contract6(Qm, S1);  // a1
      s[1] += sq6(S1);            // a3
      s[2] += contract6(Lm, S1);  // a6
      s[3] += sq6(S2);            // a8
    }
#pragma unroll
    for (int q = 0; q < 4; q++) part[((size_t)blockIdx.x * 4 + q) * nz + z] = s[q];
  }
}

void lasdd_wl_sums(Engine& e, const LasddFields& f, double* sums4) {
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_wl_partial<<<nb, 128, 0, e.stream>>>(f, e.H(), e.nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)4 * e.nz), dim3(32, 32), 0, e.stream>>>(e.red, nb, 4, e.nz,
                                                                       1.0 / (double)e.H(), sums4);
}

struct WLPow {
  double p43, p83, p163;  // TFR^(4/3), TFR^(8/3), TFR^(16/3)
};

static WLPow wl_pow(const Engine& e) {
  return WLPow{std::pow(e.TFR, 4.0 / 3.0), std::pow(e.TFR, 8.0 / 3.0),
               std::pow(e.TFR, 16.0 / 3.0)};
}

// (ff, ee, dd, cc, bb, aa) per level from (a1, a3, a6, a8)
__global__ void k_poly_wl(const double* __restrict__ m, int nz, WLPow P, double* co) {
  for (int z = blockIdx.x * blockDim.x + threadIdx.x; z < nz; z += gridDim.x * blockDim.x) {
    const double a1 = m[0 * nz + z], a3 = m[1 * nz + z], a6 = m[2 * nz + z], a8 = m[3 * nz + z];
    const double a2 = -(P.p83) * a1;
    const double a4 = -2 * P.p43 * a3;
    const double a5 = P.p83 * a3;
    const double a7 = -P.p43 * a6;
    const double a9 = -2 * P.p83 * a8;
    const double a10 = P.p163 * a8;
    co[0 * nz + z] = -a7 * a10;                     // ff
    co[1 * nz + z] = a2 * a5 - a6 * a10;            // ee
    co[2 * nz + z] = a2 * a4 - a7 * a9;             // dd
    co[3 * nz + z] = a2 * a3 + a1 * a5 - a6 * a9;   // cc
    co[4 * nz + z] = a1 * a4 - a7 * a8;             // bb
    co[5 * nz + z] = a1 * a3 - a6 * a8;             // aa
  }
}

void wl_poly(Engine& e, const double* sums4, double* coeffs6) {
  ::alfa::note_launch(); k_poly_wl<<<1, 256, 0, e.stream>>>(sums4, e.nz, wl_pow(e), coeffs6);
}

__global__ void k_LM_MM_wl(LasddFields f, double T1, double T2, const double* __restrict__ beta,
                           real* __restrict__ LM, real* __restrict__ MM, size_t n, int nz) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    double Lm[6], Mm[6];
    leonard(f.ph, f.hat, i, Lm);
    const double b = beta[z];
#pragma unroll
    for (int q = 0; q < 6; q++) Mm[q] = T1 * (double)f.Sh[q][i] - T2 * b * (double)f.Sd[q][i];
    LM[i] = (Lm[0] * Mm[0] + Lm[1] * Mm[1] + Lm[2] * Mm[2]) +
            2.0 * (Lm[3] * Mm[3] + Lm[4] * Mm[4] + Lm[5] * Mm[5]);
    MM[i] = sq6(Mm);
  }
}

void lasdd_wl_LM_MM(Engine& e, const LasddFields& f, const double* beta, real* LM, real* MM) {
  const double T1 = 2 * std::pow(e.L, 4.0 / 3.0);
  const double T2 = 2 * std::pow(e.TFR * e.L, 4.0 / 3.0);
  ::alfa::note_launch(); k_LM_MM_wl<<<nblocks(e.N()), TPB, 0, e.stream>>>(f, T1, T2, beta, LM, MM, e.N(), e.nz);
}

struct WLScalarTerms {
  double a1, a3, a6, a8, b6, c36;
};

__device__ __forceinline__ WLScalarTerms wl_scalar_terms(const ScalarLasddFields& f, size_t i) {
  const double T1 = f.Th[i], T2 = f.Td[i];
  double LT[3], QT[3], G1[3], G2[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    LT[q] = (double)f.uTh[q][i] - (double)f.hat[q][i] * T1;
    QT[q] = (double)f.uTd[q][i] - (double)f.hatd[q][i] * T2;
    G1[q] = f.Gh[q][i];
    G2[q] = f.Gd[q][i];
  }
  WLScalarTerms t;
  t.a1 = QT[0] * G1[0] + QT[1] * G1[1] + QT[2] * G1[2];
  t.a3 = G1[0] * G1[0] + G1[1] * G1[1] + G1[2] * G1[2];
  t.a6 = LT[0] * G1[0] + LT[1] * G1[1] + LT[2] * G1[2];
  t.a8 = G2[0] * G2[0] + G2[1] * G2[1] + G2[2] * G2[2];
  t.b6 = LT[0] * G2[0] + LT[1] * G2[1] + LT[2] * G2[2];
  t.c36 = G1[0] * G2[0] + G1[1] * G2[1] + G1[2] * G2[2];
  return t;
}

__global__ void k_slwl_partial(ScalarLasddFields f, size_t H, int nz, double* part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double s[4] = {0, 0, 0, 0};
    for (size_t r = r0; r < r1; r++) {
      const WLScalarTerms t = wl_scalar_terms(f, r * nz + z);
      s[0] += t.a1;
      s[1] += t.a3;
      s[2] += t.a6;
      s[3] += t.a8;
    }
#pragma unroll
    for (int q = 0; q < 4; q++) part[((size_t)blockIdx.x * 4 + q) * nz + z] = s[q];
  }
}

void scalar_lasdd_wl_sums(Engine& e, const ScalarLasddFields& f, double* sums4) {
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_slwl_partial<<<nb, 128, 0, e.stream>>>(f, e.H(), e.nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)4 * e.nz), dim3(32, 32), 0, e.stream>>>(e.red, nb, 4, e.nz,
                                                                       1.0 / (double)e.H(), sums4);
}

__global__ void k_slwl_TupTdn(ScalarLasddFields f, double L43, double L83, WLPow P,
                              const double* __restrict__ beta, real* __restrict__ Tup,
                              real* __restrict__ Tdn, size_t n,
                              int nz) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    const WLScalarTerms t = wl_scalar_terms(f, i);
    const double b = beta[z];
    Tup[i] = L43 * (t.a6 - P.p43 * b * t.b6);
    Tdn[i] = L83 * (t.a3 - 2 * P.p43 * b * t.c36 + P.p83 * (b * b) * t.a8);
  }
}

void scalar_wl_Tup_Tdn(Engine& e, const ScalarLasddFields& f, const double* beta, real* Tup,
                       real* Tdn) {
  const double L43 = std::pow(e.L, 4.0 / 3.0), L83 = std::pow(e.L, 8.0 / 3.0);
  ::alfa::note_launch(); k_slwl_TupTdn<<<nblocks(e.N()), TPB, 0, e.stream>>>(f, L43, L83, wl_pow(e), beta, Tup, Tdn, e.N(), e.nz);
}

// ---------------------------------------------------------------------------
// Plane-averaged statistics (Statistics.py:47-328), one sample added to the
// accumulator acc[key * nz + z] (profile keys in STATS order) and
// acc[31 * nz + j] (M_sfc, ustar, qz_sfc, qm_sfc).  A dry sample (no Q)
// accumulates zeros in the moisture entries (Q, dQdz, Q2, wQ, qHz, qm_sfc).
// Q_scale = 1 (Statistics.py:166-168, 199-201, 231-256, 275, 289).
// ---------------------------------------------------------------------------
enum StatKey {
  ST_U = 0, ST_V, ST_W, ST_TH, ST_dUdz, ST_dVdz, ST_dTHdz, ST_u2, ST_v2, ST_w2, ST_TH2, ST_uv,
  ST_uw, ST_vw, ST_uTH, ST_vTH, ST_wTH, ST_txy, ST_txz, ST_tyz, ST_qz, ST_Cs2_1, ST_Cs2_2,
  ST_Cs2PrRatio, ST_Beta1, ST_Beta2, ST_Q, ST_dQdz, ST_Q2, ST_wQ, ST_qHz, ST_NPROF = 31
};
static constexpr int ST_NM = 18;  // pass-1 sums
static constexpr int ST_NV = 12;  // pass-2 sums

// pass 1 sums per level: u v w TH dudz dvdz dTHdz txy txz tyz qz u_st v_st TH_st,
// then Q dQdz qHz Q_st
__global__ void k_stats_mean_partial(StatsIn a, size_t H, int nz, double* __restrict__ part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double s[ST_NM] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t r = r0; r < r1; r++) {
      const size_t i = r * nz + z;
      const double u = a.u[i], v = a.v[i], T = a.TH[i];
      s[0] += u;
      s[1] += v;
      s[2] += a.w[i];
      s[3] += T;
      s[4] += a.dudz[i];
      s[5] += a.dvdz[i];
      s[6] += a.dTHdz[i];
      s[7] += a.txy[i];
      s[8] += a.txz[i];
      s[9] += a.tyz[i];
      s[10] += a.qz[i];
      if (z == 0) {
        s[11] += u + a.Ugal;
        s[12] += v;
        s[13] += T;
      } else {
        s[11] += 0.5 * ((double)a.u[i - 1] + u);
        s[12] += 0.5 * ((double)a.v[i - 1] + v);
        s[13] += 0.5 * ((double)a.TH[i - 1] + T);
      }
      if (a.Q) {
        const double q = a.Q[i];
        s[14] += q;
        s[15] += a.dQdz[i];
        s[16] += a.qHz[i];
        s[17] += (z == 0) ? q : 0.5 * ((double)a.Q[i - 1] + q);
      }
    }
#pragma unroll
    for (int q = 0; q < ST_NM; q++) part[((size_t)blockIdx.x * ST_NM + q) * nz + z] = s[q];
  }
}

// pass 2 sums of fluctuation products, with m = the pass-1 plane means
__global__ void k_stats_var_partial(StatsIn a, const double* __restrict__ m, size_t H, int nz,
                                    double* __restrict__ part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  const double Ug = a.Ugal;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    const double mU = m[0 * nz + z] + Ug, mV = m[1 * nz + z], mW = m[2 * nz + z];
    const double mT = m[3 * nz + z];
    const double muS = m[11 * nz + z] + Ug, mvS = m[12 * nz + z], mTS = m[13 * nz + z];
    const double mQ = m[14 * nz + z], mQS = m[17 * nz + z];
    double s[ST_NV] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t r = r0; r < r1; r++) {
      const size_t i = r * nz + z;
      const double u = a.u[i], v = a.v[i], T = a.TH[i];
      const double uf = u + Ug - mU, vf = v - mV, wf = a.w[i] - mW, Tf = T - mT;
      s[0] += uf * uf;
      s[1] += vf * vf;
      s[2] += wf * wf;
      s[3] += Tf * Tf;
      s[4] += uf * vf;
      s[5] += uf * Tf;
      s[6] += vf * Tf;
      double uS, vS, TS;
      if (z == 0) {
        uS = u + Ug;
        vS = v;
        TS = T;
      } else {
        uS = 0.5 * ((double)a.u[i - 1] + u);
        vS = 0.5 * ((double)a.v[i - 1] + v);
        TS = 0.5 * ((double)a.TH[i - 1] + T);
      }
      const double usf = uS + Ug - muS, vsf = vS - mvS, wsf = wf, Tsf = TS - mTS;
      s[7] += usf * wsf;
      s[8] += vsf * wsf;
      s[9] += wsf * Tsf;
      if (a.Q) {
        const double q = a.Q[i];
        const double Qf = q - mQ;
        const double QS = (z == 0) ? q : 0.5 * ((double)a.Q[i - 1] + q);
        s[10] += Qf * Qf;
        s[11] += wsf * (QS - mQS);
      }
    }
#pragma unroll
    for (int q = 0; q < ST_NV; q++) part[((size_t)blockIdx.x * ST_NV + q) * nz + z] = s[q];
  }
}

// surface means (one block) and the accumulation of every entry
__global__ void k_stats_accumulate(StatsIn a, const double* __restrict__ m,
                                   const double* __restrict__ var, size_t H, int nz,
                                   double us_zs, double* acc) {
  __shared__ double red[3][1024];
  double sM = 0.0, sU = 0.0, sQ = 0.0;
  for (size_t r = threadIdx.x; r < H; r += blockDim.x) {
    sM += a.M[r];
    sU += a.ustar[r] * a.ustar[r];
    if (a.qm_plane) sQ += a.qm_plane[r];
  }
  red[0][threadIdx.x] = sM;
  red[1][threadIdx.x] = sU;
  red[2][threadIdx.x] = sQ;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      red[0][threadIdx.x] += red[0][threadIdx.x + w];
      red[1][threadIdx.x] += red[1][threadIdx.x + w];
      red[2][threadIdx.x] += red[2][threadIdx.x + w];
    }
    __syncthreads();
  }
  const double Ug = a.Ugal;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double* A = acc;
    A[ST_U * nz + z] += m[0 * nz + z] + Ug;
    A[ST_V * nz + z] += m[1 * nz + z];
    A[ST_W * nz + z] += m[2 * nz + z];
    A[ST_TH * nz + z] += m[3 * nz + z] + a.T0;
    A[ST_dUdz * nz + z] += m[4 * nz + z] * us_zs;
    A[ST_dVdz * nz + z] += m[5 * nz + z] * us_zs;
    A[ST_dTHdz * nz + z] += m[6 * nz + z] * us_zs;
    A[ST_u2 * nz + z] += var[0 * nz + z];
    A[ST_v2 * nz + z] += var[1 * nz + z];
    A[ST_w2 * nz + z] += var[2 * nz + z];
    A[ST_TH2 * nz + z] += var[3 * nz + z];
    A[ST_uv * nz + z] += var[4 * nz + z];
    A[ST_uTH * nz + z] += var[5 * nz + z];
    A[ST_vTH * nz + z] += var[6 * nz + z];
    A[ST_uw * nz + z] += var[7 * nz + z];
    A[ST_vw * nz + z] += var[8 * nz + z];
    A[ST_wTH * nz + z] += var[9 * nz + z];
    A[ST_txy * nz + z] += m[7 * nz + z];
    A[ST_txz * nz + z] += m[8 * nz + z];
    A[ST_tyz * nz + z] += m[9 * nz + z];
    A[ST_qz * nz + z] += m[10 * nz + z];
    A[ST_Cs2_1 * nz + z] += a.cs2_1[z];
    A[ST_Cs2_2 * nz + z] += a.cs2_2[z];
    A[ST_Cs2PrRatio * nz + z] += a.cs2pr[z];
    A[ST_Beta1 * nz + z] += a.beta1[z];
    A[ST_Beta2 * nz + z] += a.beta2[z];
    if (a.Q) {
      A[ST_Q * nz + z] += m[14 * nz + z];
      A[ST_dQdz * nz + z] += m[15 * nz + z] * us_zs;
      A[ST_Q2 * nz + z] += var[10 * nz + z];
      A[ST_wQ * nz + z] += var[11 * nz + z];
      A[ST_qHz * nz + z] += m[16 * nz + z];
    }
  }
  if (threadIdx.x == 0) {
    double* S = acc + (size_t)ST_NPROF * nz;
    S[0] += red[0][0] / (double)H;
    S[1] += sqrt(red[1][0] / (double)H);
    S[2] += *a.qz_sfc_avg;
    if (a.qm_plane)
      S[3] += red[2][0] / (double)H;
    else if (a.qm_sfc_avg)
      S[3] += *a.qm_sfc_avg;
  }
}

void compute_stats(Engine& e, const StatsIn& a, double* acc) {
  const int nb = red_blocks(e);
  const int nz = e.nz;
  double* m = e.stat;                // ST_NM nz plane means
  double* var = e.stat + ST_NM * nz;  // ST_NV nz
  ::alfa::note_launch(); k_stats_mean_partial<<<nb, 128, 0, e.stream>>>(a, e.H(), nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)ST_NM * nz), dim3(32, 32), 0, e.stream>>>(
      e.red, nb, ST_NM, nz, 1.0 / (double)e.H(), m);
  ::alfa::note_launch(); k_stats_var_partial<<<nb, 128, 0, e.stream>>>(a, m, e.H(), nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)ST_NV * nz), dim3(32, 32), 0, e.stream>>>(
      e.red, nb, ST_NV, nz, 1.0 / (double)e.H(), var);
  // u_scale = TH_scale = 1: dUdz, dVdz, dTHdz scale by 1 / z_scale
  ::alfa::note_launch(); k_stats_accumulate<<<1, 1024, 0, e.stream>>>(a, m, var, e.H(), nz,
                                                                     1.0 / e.z_scale, acc);
}

// 3x3 periodic box mean (Utilities.py:87-115) at (x, y, z).  The periodic
// neighbours are selected, not taken modulo nx / ny (an integer division by
// a run-time divisor per neighbour cost more than the kernel's loads); the
// sum runs in the same order as before.
__device__ __forceinline__ double box9(const real* F, int x, int y, int z, int nx, int ny,
                                       int nz) {
  double s = 0.0;
  const double w = 1.0 / 9.0;
  const int xs[3] = {x == 0 ? nx - 1 : x - 1, x, x == nx - 1 ? 0 : x + 1};
  const int ys[3] = {y == 0 ? ny - 1 : y - 1, y, y == ny - 1 ? 0 : y + 1};
#pragma unroll
  for (int a = 0; a < 3; a++) {
#pragma unroll
    for (int b = 0; b < 3; b++)
      s = s + (double)F[((size_t)xs[a] * ny + ys[b]) * nz + z] * w;
  }
  return s;
}

// The box-filtered kernels run one CTA per (x, y) column (blockIdx.x = y,
// blockIdx.y = x) and loop over its z levels, so the nine neighbour columns'
// offsets are computed once per thread instead of dividing the linear index
// by nz and ny for every element (the index arithmetic was most of these
// kernels' instructions).
static inline dim3 column_grid(const Engine& e) { return dim3((unsigned)e.ny, (unsigned)e.nx); }
static inline int column_threads(int nz) { return nz >= 256 ? 256 : (nz + 31) / 32 * 32; }

__global__ void k_clip_ratio(const real* __restrict__ num, const real* __restrict__ den,
                             real* __restrict__ out, int nx, int ny, int nz) {
  const int y = blockIdx.x, x = blockIdx.y;
  const size_t col = ((size_t)x * ny + y) * nz;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    const double nf = box9(num, x, y, z, nx, ny, nz);
    const double df = box9(den, x, y, z, nx, ny, nz);
    const double q = nf / df;
    const bool bad = (fabs(df) < 1e-10) || (q < 0.0) || (q > 1.0);
    out[col + z] = bad ? 0.0 : q;
  }
}

void clip_ratio(Engine& e, const real* num, const real* den, real* out) {
  ::alfa::note_launch();
  k_clip_ratio<<<column_grid(e), column_threads(e.nz), 0, e.stream>>>(num, den, out, e.nx, e.ny,
                                                                      e.nz);
}

__global__ void k_imfilter(const real* __restrict__ F, real* __restrict__ out, int nx, int ny,
                           int nz) {
  const int y = blockIdx.x, x = blockIdx.y;
  const size_t col = ((size_t)x * ny + y) * nz;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) out[col + z] = box9(F, x, y, z, nx, ny, nz);
}

void imfilter(Engine& e, const real* F, real* out) {
  ::alfa::note_launch();
  k_imfilter<<<column_grid(e), column_threads(e.nz), 0, e.stream>>>(F, out, e.nx, e.ny, e.nz);
}

__global__ void k_cs2_partial(const real* __restrict__ C, size_t H, int nz, double* part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double s0 = 0.0, s1 = 0.0;
    for (size_t r = r0; r < r1; r++) {
      const double c = C[r * nz + z];
      s0 += sqrt(c);
      s1 += c;
    }
    part[((size_t)blockIdx.x * 2 + 0) * nz + z] = s0;
    part[((size_t)blockIdx.x * 2 + 1) * nz + z] = s1;
  }
}

__global__ void k_cs2_finish(const double* __restrict__ m, int nz, double* avg1, double* avg2) {
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    const double a = m[z];
    if (avg1) avg1[z] = a * a;
    if (avg2) avg2[z] = m[nz + z];
  }
}

void cs2_profiles(Engine& e, const real* Cs2, double* avg1, double* avg2) {
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_cs2_partial<<<nb, 128, 0, e.stream>>>(Cs2, e.H(), e.nz, e.red);
  double* m = e.scal + 64;
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)2 * e.nz), dim3(32, 32), 0, e.stream>>>(e.red, nb, 2, e.nz,
                                                                      1.0 / (double)e.H(), m);
  ::alfa::note_launch(); k_cs2_finish<<<1, 256, 0, e.stream>>>(m, e.nz, avg1, avg2);
}

// ---------------------------------------------------------------------------
// Scalar LASDD (DynamicSGS_ScalarLASDD_SM.py:224-307)
// ---------------------------------------------------------------------------
struct SLConst {
  double cL2, cb2, cL4, cd2, ce2, cb4, cd4, ce4;
};

static SLConst sl_const(const Engine& e) {
  const double L = e.L, T = e.TFR;
  SLConst c;
  c.cL2 = std::pow(L, 2.0);
  c.cb2 = -std::pow(L, 2.0) * std::pow(T, 2.0);
  c.cL4 = std::pow(L, 4.0);
  c.cd2 = -2 * std::pow(L, 4.0) * std::pow(T, 2.0);
  c.ce2 = std::pow(L, 4.0) * std::pow(T, 4.0);
  c.cb4 = -std::pow(L, 2.0) * std::pow(T, 4.0);
  c.cd4 = -2 * std::pow(L, 4.0) * std::pow(T, 4.0);
  c.ce4 = std::pow(L, 4.0) * std::pow(T, 8.0);
  return c;
}

struct SLTerms {
  double a, b, c, d, e;
};

__device__ __forceinline__ SLTerms sl_terms(const real* const* uT, const real* const* hat,
                                            const real* Tf, const real* const* SG,
                                            const real* const* G, const real* S, size_t i) {
  const double T = Tf[i], s = S[i];
  double LT[3], sg[3], g[3];
#pragma unroll
  for (int q = 0; q < 3; q++) {
    LT[q] = (double)uT[q][i] - (double)hat[q][i] * T;
    sg[q] = SG[q][i];
    g[q] = G[q][i];
  }
  SLTerms t;
  t.a = LT[0] * sg[0] + LT[1] * sg[1] + LT[2] * sg[2];
  t.b = LT[0] * s * g[0] + LT[1] * s * g[1] + LT[2] * s * g[2];
  t.c = sg[0] * sg[0] + sg[1] * sg[1] + sg[2] * sg[2];
  t.d = sg[0] * s * g[0] + sg[1] * s * g[1] + sg[2] * s * g[2];
  const double p0 = s * g[0], p1 = s * g[1], p2 = s * g[2];
  t.e = p0 * p0 + p1 * p1 + p2 * p2;
  return t;
}

__global__ void k_sl_partial(ScalarLasddFields f, SLConst c, size_t H, int nz, double* part) {
  const size_t rpb = (H + gridDim.x - 1) / gridDim.x;
  const size_t r0 = blockIdx.x * rpb;
  const size_t r1 = (r0 + rpb < H) ? r0 + rpb : H;
  for (int z = threadIdx.x; z < nz; z += blockDim.x) {
    double s[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (size_t r = r0; r < r1; r++) {
      const size_t i = r * nz + z;
      const SLTerms t1 = sl_terms(f.uTh, f.hat, f.Th, f.SGh, f.Gh, f.S_hat, i);
      const SLTerms t2 = sl_terms(f.uTd, f.hatd, f.Td, f.SGd, f.Gd, f.S_hatd, i);
      s[0] += c.cL2 * t1.a;
      s[1] += c.cb2 * t1.b;
      s[2] += c.cL4 * t1.c;
      s[3] += c.cd2 * t1.d;
      s[4] += c.ce2 * t1.e;
      s[5] += c.cL2 * t2.a;
      s[6] += c.cb4 * t2.b;
      s[7] += c.cL4 * t2.c;
      s[8] += c.cd4 * t2.d;
      s[9] += c.ce4 * t2.e;
    }
#pragma unroll
    for (int q = 0; q < 10; q++) part[((size_t)blockIdx.x * 10 + q) * nz + z] = s[q];
  }
}

void scalar_lasdd_sums(Engine& e, const ScalarLasddFields& f, double* sums10) {
  const int nb = red_blocks(e);
  ::alfa::note_launch(); k_sl_partial<<<nb, 128, 0, e.stream>>>(f, sl_const(e), e.H(), e.nz, e.red);
  ::alfa::note_launch(); k_partial_finish<<<finish_grid((size_t)10 * e.nz), dim3(32, 32), 0, e.stream>>>(e.red, nb, 10, e.nz,
                                                                       1.0 / (double)e.H(), sums10);
}

__global__ void k_sl_TupTdn(ScalarLasddFields f, SLConst c, const double* __restrict__ beta,
                            real* __restrict__ Tup, real* __restrict__ Tdn, size_t n, int nz) {
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    const SLTerms t = sl_terms(f.uTh, f.hat, f.Th, f.SGh, f.Gh, f.S_hat, i);
    const double b = beta[z];
    Tup[i] = c.cL2 * t.a + c.cb2 * t.b * b;
    Tdn[i] = c.cL4 * t.c + c.cd2 * t.d * b + c.ce2 * t.e * (b * b);
  }
}

void scalar_Tup_Tdn(Engine& e, const ScalarLasddFields& f, const double* beta, real* Tup,
                    real* Tdn) {
  ::alfa::note_launch(); k_sl_TupTdn<<<nblocks(e.N()), TPB, 0, e.stream>>>(f, sl_const(e), beta, Tup, Tdn, e.N(), e.nz);
}

// ---------------------------------------------------------------------------
// wall stresses (SGSStresses_SM.py:63-90, 238-241) and plane-0 overrides
// ---------------------------------------------------------------------------
__global__ void k_wall(const real* __restrict__ u, const real* __restrict__ v,
                       const double* __restrict__ M, const double* __restrict__ pm,
                       const double* __restrict__ pm0, real* __restrict__ txz,
                       real* __restrict__ tyz, size_t H, int nz,
                       double log_m, double Ugal) {
  GRID_STRIDE(r, H) {
    const double denom = log_m + pm[r] - pm0[r];
    const double us = 0.4 * M[r] / denom;
    const size_t i = r * nz;
    txz[i] = -(us * us) * ((double)u[i] + Ugal) / M[r];
    tyz[i] = -(us * us) * v[i] / M[r];
  }
}

void wall_override(Engine& e, const real* u, const real* v, const double* M,
                   const double* psi_m, const double* psi_m0, real* txz, real* tyz) {
  const double log_m = std::log(0.5 * e.dz * e.z_scale / e.cfg.z0m);
  ::alfa::note_launch(); k_wall<<<nblocks(e.H()), TPB, 0, e.stream>>>(u, v, M, psi_m, psi_m0, txz, tyz, e.H(), e.nz,
                                                log_m, e.cfg.Ugal);
}

__global__ void k_set_plane0(const double* __restrict__ p, real* __restrict__ f, size_t H, int nz) {
  GRID_STRIDE(r, H) { f[r * nz] = p[r]; }
}

void set_plane0(Engine& e, const double* plane, real* field) {
  ::alfa::note_launch(); k_set_plane0<<<nblocks(e.H()), TPB, 0, e.stream>>>(plane, field, e.H(), e.nz);
}

// ---------------------------------------------------------------------------
// RHS assembly: NSE_AllTerms.py:82-102, SCL_AllTerms.py:68-80
// ---------------------------------------------------------------------------
struct RhsM {
  const real *u, *v, *w;
  const double *Ug, *Vg;
  const real *Cx, *Cy, *Cz, *b, *dx, *dy, *dz;
  const double *Uadv, *Vadv, *ubar, *vbar, *rd, *rds;
  real *Ru, *Rv, *Rw;
  double f, Ugal;
  int adv, damp;
  const int* itp;   // non-null: the forcing profiles are row (*itp - 1) of a series
  long long rs;     // row stride of that series
  const int* gtp;   // non-null: Ug, Vg are row (*gtp - 1) of the geostrophic series
  long long grs;    // row stride of that series
};

__global__ void k_rhs_m(RhsM a, size_t n, int nz) {
  const size_t grow = a.gtp ? (size_t)(*a.gtp - 1) * a.grs : 0;
  real* __restrict__ Ru = a.Ru;
  real* __restrict__ Rv = a.Rv;
  real* __restrict__ Rw = a.Rw;
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    double ru = -(double)a.Cx[i] - (double)a.dx[i] - a.f * (a.Vg[grow + z] - (double)a.v[i]);
    double rv = -(double)a.Cy[i] - (double)a.dy[i] + a.f * (a.Ug[grow + z] - a.Ugal - (double)a.u[i]);
    double rw = -(double)a.Cz[i] - (double)a.dz[i] + (double)a.b[i];
    if (a.adv) {
      const size_t row = a.itp ? (size_t)(*a.itp - 1) * a.rs : 0;
      ru = ru + a.Uadv[row + z];
      rv = rv + a.Vadv[row + z];
    }
    if (a.damp) {
      ru = ru - a.rds[z] * ((double)a.u[i] - a.ubar[z]);
      rv = rv - a.rds[z] * ((double)a.v[i] - a.vbar[z]);
      rw = rw - a.rd[z] * (double)a.w[i];
    }
    Ru[i] = ru;
    Rv[i] = rv;
    Rw[i] = rw;
  }
}

void rhs_momentum(Engine& e, const real* u, const real* v, const real* w,
                  const double* Ug, const double* Vg, const real* Cx, const real* Cy,
                  const real* Cz, const real* b, const real* dx, const real* dy,
                  const real* dz, const double* Uadv, const double* Vadv, const double* ubar,
                  const double* vbar, real* Ru, real* Rv, real* Rw, const int* itp,
                  long long rs, const int* gtp, long long grs) {
  RhsM a{u, v, w, Ug, Vg, Cx, Cy, Cz, b, dx, dy, dz, Uadv, Vadv, ubar, vbar, e.d_rd, e.d_rd_stag,
         Ru, Rv, Rw, e.f_nondim, e.cfg.Ugal, e.cfg.optAdvection >= 1, e.cfg.optDamping == 1, itp,
         rs, gtp, grs};
  ::alfa::note_launch(); k_rhs_m<<<nblocks(e.N()), TPB, 0, e.stream>>>(a, e.N(), e.nz);
}

__global__ void k_rhs_s(const real* __restrict__ TH, const real* __restrict__ adv,
                        const real* __restrict__ dq, const double* __restrict__ THadv,
                        const double* __restrict__ bar, const double* __restrict__ rds,
                        real* __restrict__ R,
                        size_t n, int nz, int doadv, int damp, const int* itp, long long rs) {
  const size_t row = (doadv && itp) ? (size_t)(*itp - 1) * rs : 0;
  GRID_STRIDE(i, n) {
    const int z = zof(i, nz);
    double r = -(double)adv[i] - (double)dq[i];
    if (doadv) r = r + THadv[row + z];
    if (damp) r = r - rds[z] * ((double)TH[i] - bar[z]);
    R[i] = r;
  }
}

void rhs_scalar(Engine& e, const real* TH, const real* adv, const real* divq,
                const double* THadv, const double* THbar, real* R, const int* itp,
                long long rs, int always_adv) {
  ::alfa::note_launch(); k_rhs_s<<<nblocks(e.N()), TPB, 0, e.stream>>>(TH, adv, divq, THadv, THbar, e.d_rd_stag, R,
                                                 e.N(), e.nz,
                                                 always_adv || e.cfg.optAdvection >= 1,
                                                 e.cfg.optDamping == 1, itp, rs);
}

// ---------------------------------------------------------------------------
// pressure: NSE_PressureTerms.py:150-182 (RC assembly) and
// NSE_PressureTerms_Thomas.py:246-275 (masked solve + zero mode)
// ---------------------------------------------------------------------------
__global__ void k_rc(const cd* __restrict__ fRx, const cd* __restrict__ fRy,
                     const cd* __restrict__ fRz, const cd* __restrict__ fb2,
                     const double* __restrict__ kr, double* __restrict__ RCr,
                     double* __restrict__ RCi, double* __restrict__ fRzr,
                     int nx, int nyh, int nz, double dz) {
  const size_t n = (size_t)nx * nyh * (nz + 1);
  GRID_STRIDE(t, n) {
    const int k = zof(t, nz + 1);
    const size_t m = rof(t, nz + 1);  // mode (i, j)
    const int j = zof(m, nyh), i = (int)rof(m, nyh);
    if (k == 0) {
      const cd f = fb2[m * 2 + 0];
      RCr[t] = -dz * f.x;
      RCi[t] = -dz * f.y;
    } else if (k == nz) {
      const cd f = fb2[m * 2 + 1];
      RCr[t] = -dz * f.x;
      RCi[t] = -dz * f.y;
    } else {
      const size_t a = m * nz + (k - 1);
      const double q = kr[i], c = (double)j;
      double hr = -q * (double)fRx[a].y;
      hr = hr - c * (double)fRy[a].y;
      double hi = q * (double)fRx[a].x;
      hi = hi + c * (double)fRy[a].x;
      RCr[t] = hr + ((double)fRz[a + 1].x - (double)fRz[a].x) / dz;
      RCi[t] = hi + ((double)fRz[a + 1].y - (double)fRz[a].y) / dz;
    }
    if (k < nz) fRzr[m * nz + k] = fRz[m * nz + k].x;
  }
}

void pressure_rc(Engine& e, const cd* fRx, const cd* fRy, const cd* fRz, const cd* fb2,
                 const cd* /*unused*/, double* RCr, double* RCi, double* fRz_real) {
  ::alfa::note_launch(); k_rc<<<nblocks((size_t)e.nx * e.nyh * (e.nz + 1)), TPB, 0, e.stream>>>(
      fRx, fRy, fRz, fb2, e.d_kr, RCr, RCi, fRz_real, e.nx, e.nyh, e.nz, e.dz);
}

// Forward elimination and back substitution per mode with the factors of
// engine_init, in the reference's order (NSE_PressureTerms_Thomas.py:99-143):
// the solution depends on the order of its operations at ~1e-8 relative in
// the low-wavenumber modes (condition ~(2/dz^2)/k^2), so the recurrences stay
// sequential per mode.  What limited the kernel was memory latency (one
// thread per mode, ~7 warps per SM at 256^3, every row's load waiting on the
// previous row's arithmetic): each thread now issues the loads of RB rows
// (RC, the multipliers and diagonals, all stored mode major, contiguous per
// thread) before it runs them, so RB rows of every thread are in flight.
// The forward sweep's modified right-hand side goes to dm (FP64): the output
// spectrum itself in the FP64 build (each element read before it is
// overwritten), a separate FP64 buffer in the FP32 build.
static constexpr int RB = 8;

__global__ void __launch_bounds__(64) k_thomas(const double* __restrict__ RCr,
                                               const double* __restrict__ RCi,
                                               const double* __restrict__ fRzr,
                                               const double* __restrict__ bt,
                                               const double* __restrict__ mt,
                                               const double* __restrict__ cp, cd* fp,
                                               double2* dm_all, int nx, int nyh, int nz,
                                               double dz) {
  const size_t nm = (size_t)nx * nyh;
  for (size_t m = blockIdx.x * (size_t)blockDim.x + threadIdx.x; m < nm;
       m += (size_t)gridDim.x * blockDim.x) {
    const int j = zof(m, nyh), i = (int)rof(m, nyh);
    const size_t base = m * (nz + 1);
    cd* out = fp + m * nz;
    double2* dm = dm_all + m * nz;
    if (i == 0 && j == 0) {
      // zero mode by direct integration (Thomas.py:271-275)
      const double z0 = RCr[0];
      out[0] = mkc(z0, 0);
      double s = 0.0;
      for (int k = 1; k < nz; k++) {
        s = s + fRzr[k] * dz;
        out[k] = mkc(z0 + s, 0);
      }
      continue;
    }
    if (i == nx / 2 || j == nyh - 1) {  // x- and y-Nyquist rows masked
      for (int k = 0; k < nz; k++) out[k] = mkc(0, 0);
      continue;
    }
    // forward sweep (d_mod of row k in dm[k-1] for k >= 1)
    double dr = RCr[base], di = RCi[base];
    for (int k0 = 1; k0 <= nz; k0 += RB) {
      double rr[RB], ri[RB], mk[RB];
#pragma unroll
      for (int t = 0; t < RB; t++) {
        const int k = k0 + t;
        if (k <= nz) {
          rr[t] = __ldg(RCr + base + k);
          ri[t] = __ldg(RCi + base + k);
          mk[t] = __ldg(mt + base + k);
        }
      }
#pragma unroll
      for (int t = 0; t < RB; t++) {
        const int k = k0 + t;
        if (k <= nz) {
          dr = rr[t] - mk[t] * dr;
          di = ri[t] - mk[t] * di;
          dm[k - 1] = make_double2(dr, di);
        }
      }
    }
    // back substitution, x[k] for k = nz .. 1 (x[0] is not used)
    double xr = dr / bt[base + nz], xi = di / bt[base + nz];
    out[nz - 1] = mkc(xr, xi);
    for (int k1 = nz - 1; k1 >= 1; k1 -= RB) {
      double2 d[RB];
      double b[RB], c[RB];
#pragma unroll
      for (int t = 0; t < RB; t++) {
        const int k = k1 - t;
        if (k >= 1) {
          d[t] = dm[k - 1];
          b[t] = __ldg(bt + base + k);
          c[t] = __ldg(cp + k);
        }
      }
#pragma unroll
      for (int t = 0; t < RB; t++) {
        const int k = k1 - t;
        if (k >= 1) {
          xr = (d[t].x - c[t] * xr) / b[t];
          xi = (d[t].y - c[t] * xi) / b[t];
          out[k - 1] = mkc(xr, xi);
        }
      }
    }
  }
}

void thomas_solve(Engine& e, const double* RCr, const double* RCi, const double* fRz_real, cd* fp) {
  const size_t nm = (size_t)e.nx * e.nyh;
#ifdef ALFA_BUILD_FP32
  double2* dm = e.thomas_dm;
#else
  double2* dm = fp;
#endif
  ::alfa::note_launch();
  k_thomas<<<(unsigned)((nm + 63) / 64), 64, 0, e.stream>>>(RCr, RCi, fRz_real, e.d_b_thomas,
                                                            e.d_m_thomas, e.d_c_p, fp, dm, e.nx,
                                                            e.nyh, e.nz, e.dz);
}

__global__ void k_sub3(real* __restrict__ a, real* __restrict__ b, real* __restrict__ c,
                       const real* __restrict__ x,
                       const real* __restrict__ y, const real* __restrict__ z, size_t n) {
  GRID_STRIDE(i, n) {
    a[i] = a[i] - x[i];
    b[i] = b[i] - y[i];
    c[i] = c[i] - z[i];
  }
}

void subtract3(Engine& e, real* Ru, real* Rv, real* Rw, const real* a, const real* b,
               const real* c) {
  ::alfa::note_launch(); k_sub3<<<nblocks(e.N()), TPB, 0, e.stream>>>(Ru, Rv, Rw, a, b, c, e.N());
}

// ---------------------------------------------------------------------------
// AB2: NSE_TimeAdvancement.py:66-74, SCL_TimeAdvancement.py:64-69.  The
// thread of level nz-2 also writes level nz-1, so in-place update is safe.
// ---------------------------------------------------------------------------
__global__ void k_ab2(const real* u, const real* __restrict__ R, const real* __restrict__ Rp,
                      real* un, size_t n, int nz, double dt, int mode, double top_add) {
  // mode 0: u/v (top copies nz-2), 1: w (top and bottom 0), 2: TH (top = nz-2 + c).
  // u and un may be the same field (the step advances in place), so the two
  // elements a thread takes per iteration are loaded explicitly before either
  // is stored; no element reads what another writes (level nz-1 is only
  // written, by the thread of level nz-2).
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i0 = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i0 < n; i0 += 2 * stride) {
    const size_t i1 = i0 + stride;
    const int z0 = zof(i0, nz), z1 = i1 < n ? zof(i1, nz) : nz - 1;
    double v0 = 0.0, v1 = 0.0;
    if (z0 != nz - 1) v0 = (double)u[i0] + dt * (1.5 * (double)R[i0] - 0.5 * (double)Rp[i0]);
    if (z1 != nz - 1) v1 = (double)u[i1] + dt * (1.5 * (double)R[i1] - 0.5 * (double)Rp[i1]);
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const size_t i = q ? i1 : i0;
      const int z = q ? z1 : z0;
      const double val = q ? v1 : v0;
      if (z == nz - 1) continue;
      if (mode == 1) {
        un[i] = (z == 0) ? 0.0 : val;
        if (z == nz - 2) un[i + 1] = 0.0;
      } else {
        un[i] = val;
        if (z == nz - 2) un[i + 1] = (mode == 2) ? val + top_add : val;
      }
    }
  }
}

void ab2_uvw(Engine& e, const real* u, const real* v, const real* w, const real* Ru,
             const real* Rup, const real* Rv, const real* Rvp, const real* Rw,
             const real* Rwp, real* un, real* vn, real* wn) {
  ::alfa::note_launch(); k_ab2<<<nblocks(e.N()), TPB, 0, e.stream>>>(u, Ru, Rup, un, e.N(), e.nz, e.dt_nondim, 0, 0.0);
  ::alfa::note_launch(); k_ab2<<<nblocks(e.N()), TPB, 0, e.stream>>>(v, Rv, Rvp, vn, e.N(), e.nz, e.dt_nondim, 0, 0.0);
  ::alfa::note_launch(); k_ab2<<<nblocks(e.N()), TPB, 0, e.stream>>>(w, Rw, Rwp, wn, e.N(), e.nz, e.dt_nondim, 1, 0.0);
}

void ab2_th(Engine& e, const real* TH, const real* R, const real* Rp, real* out) {
  ::alfa::note_launch(); k_ab2<<<nblocks(e.N()), TPB, 0, e.stream>>>(TH, R, Rp, out, e.N(), e.nz, e.dt_nondim, 2,
                                               e.inversion_nondim * e.dz);
}

void ab2_q(Engine& e, const real* Q, const real* R, const real* Rp, real* out) {
  ::alfa::note_launch(); k_ab2<<<nblocks(e.N()), TPB, 0, e.stream>>>(Q, R, Rp, out, e.N(), e.nz, e.dt_nondim, 2,
                                               e.q_inversion_nondim * e.dz);
}

// max |u|, |v|, |w| (Main.py:534-537).  The maximum propagates NaN (as the
// reference's jnp.max does; fmax would drop it), so a non-finite state shows
// in the CFL number that alfa_get_diag checks.
__device__ __forceinline__ double nanmax(double m, double a) {
  return (a > m || a != a) ? a : m;
}

__global__ void k_absmax_partial(const real* __restrict__ a, const real* __restrict__ b,
                                 const real* __restrict__ c, size_t n, double* part) {
  __shared__ double sh[3][256];
  double m0 = 0.0, m1 = 0.0, m2 = 0.0;
  GRID_STRIDE(i, n) {
    m0 = nanmax(m0, fabs((double)a[i]));
    m1 = nanmax(m1, fabs((double)b[i]));
    m2 = nanmax(m2, fabs((double)c[i]));
  }
  sh[0][threadIdx.x] = m0;
  sh[1][threadIdx.x] = m1;
  sh[2][threadIdx.x] = m2;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int q = 0; q < 3; q++) sh[q][threadIdx.x] = nanmax(sh[q][threadIdx.x], sh[q][threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int q = 0; q < 3; q++) part[blockIdx.x * 3 + q] = sh[q][0];
}

__global__ void k_absmax_finish(const double* part, int nb, double* out) {
  if (threadIdx.x < 3) {
    double m = 0.0;
    for (int b = 0; b < nb; b++) m = nanmax(m, part[b * 3 + threadIdx.x]);
    out[threadIdx.x] = m;
  }
}

void cfl_max(Engine& e, const real* u, const real* v, const real* w, double* out3) {
  const int nb = 4 * e.sms < 1024 ? 4 * e.sms : 1024;  // e.red holds >= 3 x 1024 partials
  ::alfa::note_launch(); k_absmax_partial<<<nb, 256, 0, e.stream>>>(u, v, w, e.N(), e.red);
  ::alfa::note_launch(); k_absmax_finish<<<1, 32, 0, e.stream>>>(e.red, nb, out3);
}

// copy z-planes k0 and k1 of F into a (nx, ny, 2) field
__global__ void k_planes(const real* __restrict__ F, int k0, int k1, real* __restrict__ out, size_t H,
                         int nz) {
  GRID_STRIDE(r, H) {
    out[r * 2 + 0] = F[r * nz + k0];
    out[r * 2 + 1] = F[r * nz + k1];
  }
}

void copy_planes_z(Engine& e, const real* F, int k0, int k1, real* out2) {
  ::alfa::note_launch(); k_planes<<<nblocks(e.H()), TPB, 0, e.stream>>>(F, k0, k1, out2, e.H(), e.nz);
}

}  // namespace ALFA_PREC
}  // namespace alfa
