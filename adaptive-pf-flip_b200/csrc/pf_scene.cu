// pf_scene.cu -- the synthetic scenes of the benchmark configurations, seeded
// on the device into a context's particle set (pf_seed_scene).
//
// Both scenes put eight particles in every seeded cell, one per 2x2x2
// sub-cell, jittered uniformly inside it by a counter-based generator keyed
// on (seed, cell * 8 + sub-cell, stream): SplitMix64 (Steele, Lea & Flood,
// OOPSLA 2014) of a mixed counter, 53 bits to a double in [0, 1).  Particle p
// is sub-cell p % 8 of the (p / 8)-th seeded cell, cells in x-fastest order.
// Positions are formed in FP64 in a fixed operation order and rounded to FP32
// once, so they equal the host generator's (adaptive-pf-flip_b200/scenes.py)
// bit for bit; so do the phase types, except for a particle within rounding
// of the Rayleigh-Taylor interface (a cosine of the device's libm).  The
// bubble tank's Box-Muller velocities agree to rounding.
//
// The scene layouts follow the reference's initRayleighTaylor / initBubbleTank
// (src/driver/sparse_sim3d_tp.cpp:739-776: interior cells, heavy phase above
// a cos.cos-perturbed interface; water with an air bubble and an empty
// headspace) at the sizes and densities of the benchmark configurations, and
// the dam break of the multires configuration (a water column beside a
// shallow pool, air empty).
#include <cmath>

#include "pf_ctx.h"

namespace {

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform01(unsigned long long seed, unsigned long long key, unsigned stream) {
  const unsigned long long x = (seed * 0x632BE59BD9B4E019ull) ^ (key * 8ull + stream);
  return (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0);
}

__device__ __forceinline__ double normal01(unsigned long long seed, unsigned long long key, unsigned stream) {
  const double u1 = uniform01(seed, key, 2 * stream), u2 = uniform01(seed, key, 2 * stream + 1);
  return sqrt(-2.0 * log1p(-u1)) * cos(2.0 * 3.14159265358979323846 * u2);
}

struct SceneArgs {
  int kind;
  int nx, ny, nz;
  int ci, cj;  // seeded cells along x and y (x-fastest, then y, then z)
  int pi, pj;  // dam break: the pool's cells along x and y, seeded after the column's
  size_t ncol; // dam break: cells of the column
  double dx;
  unsigned long long seed;
  size_t n;
  // Rayleigh-Taylor: interface amplitude; bubble tank: centre, radius, sigma
  double amp, cx, cy, cz, r2, sigma;
};

__global__ void k_seed(SceneArgs a, float* px, float* py, float* pz, float* vx, float* vy, float* vz, float* vol,
                       uint8_t* type) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.n) return;
  size_t c = p >> 3;
  const int s = (int)(p & 7);
  int i, j, k;
  if (a.kind == PF_SCENE_DAM_BREAK && c >= a.ncol) {
    c -= a.ncol;
    i = 1 + a.ci + (int)(c % a.pi);
    j = 1 + (int)((c / a.pi) % a.pj);
    k = 1 + (int)(c / ((size_t)a.pi * a.pj));
  } else {
    i = 1 + (int)(c % a.ci);
    j = 1 + (int)((c / a.ci) % a.cj);
    k = 1 + (int)(c / ((size_t)a.ci * a.cj));
  }
  const unsigned long long cell = (unsigned long long)i + (unsigned long long)a.nx * (j + (unsigned long long)a.ny * k);
  const unsigned long long key = cell * 8ull + s;
  const double ux = uniform01(a.seed, key, 0), uy = uniform01(a.seed, key, 1), uz = uniform01(a.seed, key, 2);
  const double x = __dmul_rn(__dadd_rn(__dadd_rn((double)i, 0.5 * (s & 1)), __dmul_rn(0.5, ux)), a.dx);
  const double y = __dmul_rn(__dadd_rn(__dadd_rn((double)j, 0.5 * ((s >> 1) & 1)), __dmul_rn(0.5, uy)), a.dx);
  const double z = __dmul_rn(__dadd_rn(__dadd_rn((double)k, 0.5 * ((s >> 2) & 1)), __dmul_rn(0.5, uz)), a.dx);
  const float fx = (float)x, fy = (float)y, fz = (float)z;
  px[p] = fx;
  py[p] = fy;
  pz[p] = fz;
  vol[p] = 1.0f;
  const double X = fx, Y = fy, Z = fz;
  if (a.kind == PF_SCENE_DAM_BREAK) {
    type[p] = 0;
    vx[p] = vy[p] = vz[p] = 0.0f;
  } else if (a.kind == PF_SCENE_RAYLEIGH_TAYLOR) {
    const double pi2 = 2.0 * 3.14159265358979323846;
    const double iface = __dadd_rn(0.5, __dmul_rn(__dmul_rn(a.amp, cos(__dmul_rn(pi2, X))), cos(__dmul_rn(pi2, Z))));
    type[p] = Y > iface ? 0 : 1;
    vx[p] = vy[p] = vz[p] = 0.0f;
  } else {
    const double ex = __dsub_rn(X, a.cx), ey = __dsub_rn(Y, a.cy), ez = __dsub_rn(Z, a.cz);
    const double d2 = __dadd_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ey, ey)), __dmul_rn(ez, ez));
    type[p] = d2 < a.r2 ? 1 : 0;
    vx[p] = (float)__dmul_rn(normal01(a.seed + 1, key, 0), a.sigma);
    vy[p] = (float)__dmul_rn(normal01(a.seed + 1, key, 1), a.sigma);
    vz[p] = (float)__dmul_rn(normal01(a.seed + 1, key, 2), a.sigma);
  }
}

}  // namespace

namespace pf {
int take_upload_for(pf_ctx* ctx);
}

extern "C" int pf_seed_scene(pf_ctx* ctx, int scene, unsigned long long seed, size_t* n_out) {
  using namespace pf;
  if (!ctx || (scene != PF_SCENE_RAYLEIGH_TAYLOR && scene != PF_SCENE_BUBBLE_TANK && scene != PF_SCENE_DAM_BREAK))
    return PF_ERR_INVALID;
  const Geom& g = ctx->g;
  if (g.nx < 3 || g.ny < 3 || g.nz < 3) return set_error(ctx, PF_ERR_INVALID, "pf_seed_scene: grid too small");
  cudaSetDevice(ctx->device);
  int rc = take_upload_for(ctx);
  if (rc) return rc;
  SceneArgs a{};
  a.kind = scene;
  a.nx = g.nx;
  a.ny = g.ny;
  a.nz = g.nz;
  a.dx = g.dx;
  a.seed = seed;
  a.ci = g.nx - 2;
  // the last index whose cell centre lies below frac * n (at most n - 2)
  auto last_below = [](double frac, int n) {
    return std::min((int)std::floor(frac * n - 0.5 - 1e-12), n - 2);
  };
  if (scene == PF_SCENE_DAM_BREAK) {
    // water column x < 0.4, y < 0.6, then the pool y < 0.15 beside it
    a.ci = last_below(0.4, g.nx);
    a.cj = last_below(0.6, g.ny);
    a.pi = g.nx - 2 - a.ci;
    a.pj = last_below(0.15, g.ny);
    if (a.ci < 1 || a.cj < 1 || a.pi < 1 || a.pj < 1)
      return set_error(ctx, PF_ERR_INVALID, "pf_seed_scene: grid too small for the dam break");
    a.ncol = (size_t)a.ci * a.cj * (size_t)(g.nz - 2);
  } else if (scene == PF_SCENE_RAYLEIGH_TAYLOR) {
    // heavy (type 0, rho_l) above y = 0.5 + 0.05 cos(2 pi x) cos(2 pi z), light below
    a.cj = g.ny - 2;
    a.amp = 0.05;
  } else {
    // water in the cells whose centre lies below y = 0.7, an air bubble of
    // radius 0.15 at (0.5, 0.3, 0.5), velocities N(0, 0.1^2)
    int jmax = (int)std::floor(0.7 * g.ny - 0.5 - 1e-12);
    if (jmax > g.ny - 2) jmax = g.ny - 2;
    if (jmax < 1) return set_error(ctx, PF_ERR_INVALID, "pf_seed_scene: no water cells");
    a.cj = jmax;
    a.cx = 0.5;
    a.cy = 0.3;
    a.cz = 0.5;
    a.r2 = 0.15 * 0.15;
    a.sigma = 0.1;
  }
  a.n = (size_t)8 * a.ci * a.cj * (size_t)(g.nz - 2);
  if (scene == PF_SCENE_DAM_BREAK) a.n = 8 * (a.ncol + (size_t)a.pi * a.pj * (size_t)(g.nz - 2));
  if (a.n > ctx->cap) return set_error(ctx, PF_ERR_CAPACITY, "pf_seed_scene: more particles than max_particles");
  ctx->np = a.n;
  ctx->bins_valid = false;
  (++ctx->launches), k_seed<<<nblocks(a.n, 256), 256, 0, ctx->stream>>>(a, ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy,
                                                                        ctx->vz, ctx->vol, ctx->type);
  PF_CUDA_TRY(cudaGetLastError());
  if (n_out) *n_out = a.n;
  return PF_OK;
}
