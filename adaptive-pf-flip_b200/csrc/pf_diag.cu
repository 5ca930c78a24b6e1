// pf_diag.cu -- interface diagnostics on the device:
//
//   diagnoseSparseInterface3D  src/driver/interface_diagnostics3d.cpp:363-379
//   (sparseCellPhi, sparseGradient, sparseNormal, sparseCurvature, accumulate,
//    finishStats: the same file, lines 26-66 and 138-208)
//
// Pass 1 writes every cell's phase field phi (the mean of its six faces'
// phi(raw mass), Eq. 7) into a dense FP64 lattice.  Pass 2 visits the fluid
// cells: the gradient of the clamped phi, the curvature as the divergence of
// the six neighbours' normals (computed on the fly from the phi lattice, which
// L2 holds), and per-CTA partial statistics.  Pass 3, one CTA, combines the
// partials in a fixed order.  Every per-cell value rounds exactly as the
// reference's (FP64, _rn intrinsics, no FMA contraction), so counts, minima
// and maxima are exact; the three means are sums in a different order than
// the reference's ascending cell order and agree to rounding.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include "pf_ctx.h"

namespace pf {
namespace {

constexpr int kDiagNT = 256;
constexpr int kDiagBlocks = 8 * 148;

struct PhiK {
  double rmin, den;  // Eq. 7 constants, computed on the host in the reference's order
};

struct DiagPartial {
  int samples, interface, finite, pad;
  double phi_min, phi_max, phi_sum, grad_sum, grad_max, curv_sum, curv_max;
};

struct SurfPartial {
  int applied, finite;
  double dv_sum, dv_max, raw_sum, raw_max, sm_sum, sm_max;
};

struct DiagScratch {
  size_t ncell = 0;
  double* phi = nullptr;         // [ncell]
  DiagPartial* part = nullptr;   // [kDiagBlocks]
  DiagPartial* total = nullptr;  // [1]
  DiagPartial* h_total = nullptr;
  cudaEvent_t copied = nullptr;  // h_total holds the last launch's totals
  bool pending = false;          // ... not yet turned into ctx->diag_last
  // surface tension (allocated on first use)
  float* h = nullptr;        // [ncell][3] FP32 half velocity changes
  uint8_t* ok = nullptr;     // [ncell] cell applies its change
  SurfPartial* spart = nullptr;  // [kDiagBlocks + 1] partial statistics
  int* bad = nullptr;        // first cell with a non-finite change
};

// phiFromRawDensity (src/physics/phasefield.h:11-16)
__device__ __forceinline__ double phi_of_raw(double raw, const PhiK& P) {
  if (raw < P.rmin) return 0.0;
  double e = __dsub_rn(raw, P.rmin);
  if (e < 0.0) e = 0.0;
  const double v = sqrt(__ddiv_rn(e, P.den));
  return 1.0 < v ? 1.0 : v;  // std::min(v, 1.0), NaN included
}

// sparseCellPhi (interface_diagnostics3d.cpp:138-148)
__global__ void k_cell_phi(DevGrid G, PhiK P, double* phi) {
  const Geom& g = G.g;
  const size_t nc = (size_t)g.nx * g.ny * g.nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % g.nx), j = (int)((c / g.nx) % g.ny), k = (int)(c / ((size_t)g.nx * g.ny));
    double s = 0.0;
    s = __dadd_rn(s, phi_of_raw((double)fget(G, PF_MU, i, j, k), P));
    s = __dadd_rn(s, phi_of_raw((double)fget(G, PF_MU, i + 1, j, k), P));
    s = __dadd_rn(s, phi_of_raw((double)fget(G, PF_MV, i, j, k), P));
    s = __dadd_rn(s, phi_of_raw((double)fget(G, PF_MV, i, j + 1, k), P));
    s = __dadd_rn(s, phi_of_raw((double)fget(G, PF_MW, i, j, k), P));
    s = __dadd_rn(s, phi_of_raw((double)fget(G, PF_MW, i, j, k + 1), P));
    phi[c] = __ddiv_rn(s, 6.0);
  }
}

struct Lattice {
  const double* phi;
  int nx, ny, nz;
  double dx;
  __device__ __forceinline__ double at(int i, int j, int k) const {
    return phi[(size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * (size_t)k)];
  }
};

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// sparseGradient (:158-175) at an in-grid cell
__device__ __forceinline__ void gradient(const Lattice& L, int i, int j, int k, double g[3]) {
  const int im = clampi(i - 1, 0, L.nx - 1), ip = clampi(i + 1, 0, L.nx - 1);
  const int jm = clampi(j - 1, 0, L.ny - 1), jp = clampi(j + 1, 0, L.ny - 1);
  const int km = clampi(k - 1, 0, L.nz - 1), kp = clampi(k + 1, 0, L.nz - 1);
  g[0] = __ddiv_rn(__dsub_rn(L.at(ip, j, k), L.at(im, j, k)), __dmul_rn((double)max(1, ip - im), L.dx));
  g[1] = __ddiv_rn(__dsub_rn(L.at(i, jp, k), L.at(i, jm, k)), __dmul_rn((double)max(1, jp - jm), L.dx));
  g[2] = __ddiv_rn(__dsub_rn(L.at(i, j, kp), L.at(i, j, km)), __dmul_rn((double)max(1, kp - km), L.dx));
}

// Vec3::length (src/math/vec3.h:9)
__device__ __forceinline__ double length3(const double v[3]) {
  return sqrt(__dadd_rn(__dadd_rn(__dmul_rn(v[0], v[0]), __dmul_rn(v[1], v[1])), __dmul_rn(v[2], v[2])));
}

// sparseNormal (:177-186): component `a` of the normalised gradient, 0 below 1e-12
__device__ __forceinline__ double normal(const Lattice& L, int i, int j, int k, int a) {
  double g[3];
  gradient(L, i, j, k, g);
  const double mag = length3(g);
  if (mag <= 1e-12 || !isfinite(mag)) return 0.0;
  return __dmul_rn(g[a], __ddiv_rn(1.0, mag));
}

// sparseCurvature (:188-208)
__device__ __forceinline__ double curvature(const Lattice& L, int i, int j, int k) {
  const int im = clampi(i - 1, 0, L.nx - 1), ip = clampi(i + 1, 0, L.nx - 1);
  const int jm = clampi(j - 1, 0, L.ny - 1), jp = clampi(j + 1, 0, L.ny - 1);
  const int km = clampi(k - 1, 0, L.nz - 1), kp = clampi(k + 1, 0, L.nz - 1);
  const double tx = __ddiv_rn(__dsub_rn(normal(L, ip, j, k, 0), normal(L, im, j, k, 0)),
                              __dmul_rn((double)max(1, ip - im), L.dx));
  const double ty = __ddiv_rn(__dsub_rn(normal(L, i, jp, k, 1), normal(L, i, jm, k, 1)),
                              __dmul_rn((double)max(1, jp - jm), L.dx));
  const double tz = __ddiv_rn(__dsub_rn(normal(L, i, j, kp, 2), normal(L, i, j, km, 2)),
                              __dmul_rn((double)max(1, kp - km), L.dx));
  return __dadd_rn(__dadd_rn(tx, ty), tz);
}

__device__ void combine(DiagPartial& a, const DiagPartial& b) {
  if (b.samples) {
    a.phi_min = a.samples ? fmin(a.phi_min, b.phi_min) : b.phi_min;
    a.phi_max = a.samples ? fmax(a.phi_max, b.phi_max) : b.phi_max;
  }
  a.samples += b.samples;
  a.interface += b.interface;
  a.finite &= b.finite;
  a.phi_sum = __dadd_rn(a.phi_sum, b.phi_sum);
  a.grad_sum = __dadd_rn(a.grad_sum, b.grad_sum);
  a.curv_sum = __dadd_rn(a.curv_sum, b.curv_sum);
  a.grad_max = fmax(a.grad_max, b.grad_max);
  a.curv_max = fmax(a.curv_max, b.curv_max);
}

__device__ __forceinline__ DiagPartial empty_partial() {
  DiagPartial p;
  p.samples = p.interface = p.pad = 0;
  p.finite = 1;
  p.phi_min = p.phi_max = p.phi_sum = p.grad_sum = p.grad_max = p.curv_sum = p.curv_max = 0.0;
  return p;
}

// block-wide combine of one partial per thread into part[blockIdx.x] (fixed order)
__device__ void block_combine(DiagPartial mine, DiagPartial* out) {
  __shared__ DiagPartial sp[kDiagNT];
  sp[threadIdx.x] = mine;
  __syncthreads();
  for (int s = kDiagNT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) combine(sp[threadIdx.x], sp[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sp[0];
}

// accumulate (:26-53) over the fluid cells
__global__ void __launch_bounds__(kDiagNT) k_diag_cells(DevGrid G, Lattice L, DiagPartial* part) {
  DiagPartial acc = empty_partial();
  const size_t nc = (size_t)L.nx * L.ny * L.nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(c % L.nx), j = (int)((c / L.nx) % L.ny), k = (int)(c / ((size_t)L.nx * L.ny));
    if (cell_marker(G, i, j, k) != 1) continue;
    const double phi = L.phi[c];
    double g[3];
    gradient(L, i, j, k, g);
    const double gm = length3(g);
    const double cv = curvature(L, i, j, k);
    if (!isfinite(phi) || !isfinite(gm) || !isfinite(cv)) {
      acc.finite = 0;
      continue;
    }
    acc.phi_min = acc.samples ? fmin(acc.phi_min, phi) : phi;
    acc.phi_max = acc.samples ? fmax(acc.phi_max, phi) : phi;
    ++acc.samples;
    acc.phi_sum = __dadd_rn(acc.phi_sum, phi);
    if (!(phi > 0.05 && phi < 0.95)) continue;
    ++acc.interface;
    acc.grad_sum = __dadd_rn(acc.grad_sum, gm);
    acc.grad_max = fmax(acc.grad_max, gm);
    const double ac = fabs(cv);
    acc.curv_sum = __dadd_rn(acc.curv_sum, ac);
    acc.curv_max = fmax(acc.curv_max, ac);
  }
  block_combine(acc, &part[blockIdx.x]);
}

__global__ void __launch_bounds__(kDiagNT) k_diag_total(const DiagPartial* part, int n, DiagPartial* total) {
  DiagPartial acc = empty_partial();
  for (int b = threadIdx.x; b < n; b += blockDim.x) combine(acc, part[b]);
  block_combine(acc, total);
}

// ---- surface tension (interface_diagnostics3d.cpp:405-447) ----------------

__device__ __forceinline__ bool interface_phi(double phi) { return phi > 0.05 && phi < 0.95; }

// sparseSmoothedCurvature (:209-233)
__device__ double smoothed_curvature(const Lattice& L, int i, int j, int k, double raw, int r) {
  if (r <= 0 || !isfinite(raw)) return raw;
  double sum = 0.0;
  int count = 0;
  for (int dz = -r; dz <= r; ++dz)
    for (int dy = -r; dy <= r; ++dy)
      for (int dx = -r; dx <= r; ++dx) {
        const int ni = clampi(i + dx, 0, L.nx - 1), nj = clampi(j + dy, 0, L.ny - 1), nk = clampi(k + dz, 0, L.nz - 1);
        if (!interface_phi(L.at(ni, nj, nk))) continue;
        const double c = curvature(L, ni, nj, nk);
        if (!isfinite(c)) continue;
        sum = __dadd_rn(sum, c);
        ++count;
      }
  return count > 0 ? __ddiv_rn(sum, (double)count) : raw;
}


__device__ void surf_combine(SurfPartial& a, const SurfPartial& b) {
  a.applied += b.applied;
  a.finite &= b.finite;
  a.dv_sum = __dadd_rn(a.dv_sum, b.dv_sum);
  a.raw_sum = __dadd_rn(a.raw_sum, b.raw_sum);
  a.sm_sum = __dadd_rn(a.sm_sum, b.sm_sum);
  a.dv_max = fmax(a.dv_max, b.dv_max);
  a.raw_max = fmax(a.raw_max, b.raw_max);
  a.sm_max = fmax(a.sm_max, b.sm_max);
}

__device__ void surf_block_combine(SurfPartial mine, SurfPartial* out) {
  __shared__ SurfPartial sp[kDiagNT];
  sp[threadIdx.x] = mine;
  __syncthreads();
  for (int s = kDiagNT / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) surf_combine(sp[threadIdx.x], sp[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = sp[0];
}

// Per fluid interface cell with |grad phi| > 1e-5: the limited capillary
// velocity change (limitedDelta, :68-76), its half as the FP32 face
// increments h, and the statistics (accumulateSurfaceStats, :107-126).  A
// cell whose change is not finite lowers `first_bad`: the reference stops
// updating the grid from the first such cell in ascending order on.
__global__ void __launch_bounds__(kDiagNT) k_surface_cells(DevGrid G, Lattice L, double strength, double dt,
                                                         double max_dv, int r, float* h, uint8_t* ok,
                                                         int* first_bad, SurfPartial* part) {
  SurfPartial acc{0, 1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const size_t nc = (size_t)L.nx * L.ny * L.nz;
  for (size_t c = (size_t)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (size_t)gridDim.x * blockDim.x) {
    ok[c] = 0;
    const int i = (int)(c % L.nx), j = (int)((c / L.nx) % L.ny), k = (int)(c / ((size_t)L.nx * L.ny));
    if (cell_marker(G, i, j, k) != 1 || !interface_phi(L.phi[c])) continue;
    double g[3];
    gradient(L, i, j, k, g);
    if (length3(g) <= 1e-5) continue;
    const double raw = curvature(L, i, j, k);
    const double sm = smoothed_curvature(L, i, j, k, raw, r);
    const double s = __dmul_rn(__dmul_rn(-strength, sm), dt);
    double d[3] = {__dmul_rn(g[0], s), __dmul_rn(g[1], s), __dmul_rn(g[2], s)};
    const double m0 = length3(d);
    if (!isfinite(m0)) {
      d[0] = d[1] = d[2] = 0.0;
    } else if (max_dv > 0.0 && m0 > max_dv) {
      const double f = __ddiv_rn(max_dv, m0);
      d[0] = __dmul_rn(d[0], f);
      d[1] = __dmul_rn(d[1], f);
      d[2] = __dmul_rn(d[2], f);
    }
    const double mag = length3(d);
    if (!isfinite(mag) || !isfinite(raw) || !isfinite(sm)) {
      acc.finite = 0;
      atomicMin(first_bad, (int)c);
      continue;
    }
    ++acc.applied;
    acc.dv_sum = __dadd_rn(acc.dv_sum, mag);
    acc.dv_max = fmax(acc.dv_max, mag);
    acc.raw_sum = __dadd_rn(acc.raw_sum, fabs(raw));
    acc.raw_max = fmax(acc.raw_max, fabs(raw));
    acc.sm_sum = __dadd_rn(acc.sm_sum, fabs(sm));
    acc.sm_max = fmax(acc.sm_max, fabs(sm));
    h[3 * c + 0] = (float)__dmul_rn(0.5, d[0]);
    h[3 * c + 1] = (float)__dmul_rn(0.5, d[1]);
    h[3 * c + 2] = (float)__dmul_rn(0.5, d[2]);
    ok[c] = 1;
  }
  surf_block_combine(acc, &part[blockIdx.x]);
}

__global__ void __launch_bounds__(kDiagNT) k_surface_total(const SurfPartial* part, int n, SurfPartial* total) {
  SurfPartial acc{0, 1, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int b = threadIdx.x; b < n; b += blockDim.x) surf_combine(acc, part[b]);
  surf_block_combine(acc, total);
}

// Every face node of u, v, w with mass: the increments of its two cells, the
// lower cell's first (the reference visits cells in ascending order), from the
// cells before the first non-finite one.
__global__ void k_surface_faces(DevGrid G, int nslots, const float* __restrict__ h, const uint8_t* __restrict__ ok,
                                const int* __restrict__ first_bad) {
  const int bad = *first_bad;
  const Geom& g = G.g;
  for (int s = blockIdx.x; s < nslots; s += gridDim.x) {
    const int t = G.slot_tile[s];
    const int tx = t % g.TX, tq = t / g.TX, ty = tq % g.TY, tz = tq / g.TY;
    const int i = tx * 8 + (threadIdx.x & 7), j = ty * 8 + ((threadIdx.x >> 3) & 7), k = tz * 8 + (threadIdx.x >> 6);
    const size_t o = (size_t)s * PF_TV + threadIdx.x;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const int f = PF_U + a;
      if (!in_field(g, f, i, j, k) || !(G.fld[PF_MU + a][o] > 0.0f)) continue;
      const int p[3] = {i, j, k};
      float u = G.fld[f][o];
      bool changed = false;
      for (int side = 0; side < 2; ++side) {  // the cell below the face, then the cell above
        int q[3] = {p[0], p[1], p[2]};
        q[a] -= 1 - side;
        if (q[0] < 0 || q[1] < 0 || q[2] < 0 || q[0] >= g.nx || q[1] >= g.ny || q[2] >= g.nz) continue;
        const size_t c = (size_t)q[0] + (size_t)g.nx * ((size_t)q[1] + (size_t)g.ny * (size_t)q[2]);
        if (!ok[c] || (long long)c >= (long long)bad) continue;
        u = __fadd_rn(u, h[3 * c + a]);
        changed = true;
      }
      if (changed) G.fld[f][o] = u;
    }
  }
}

int scratch(pf_ctx* ctx, DiagScratch** out) {
  DiagScratch* s = static_cast<DiagScratch*>(ctx->idiag);
  if (!s) {
    s = new DiagScratch();
    ctx->idiag = s;
    s->ncell = (size_t)ctx->g.nx * ctx->g.ny * ctx->g.nz;
    PF_CUDA_TRY(cudaMalloc(&s->phi, s->ncell * sizeof(double)));
    PF_CUDA_TRY(cudaMalloc(&s->part, kDiagBlocks * sizeof(DiagPartial)));
    PF_CUDA_TRY(cudaMalloc(&s->total, sizeof(DiagPartial)));
    PF_CUDA_TRY(cudaMallocHost(&s->h_total, sizeof(DiagPartial)));
    PF_CUDA_TRY(cudaEventCreateWithFlags(&s->copied, cudaEventDisableTiming));
  }
  *out = s;
  return PF_OK;
}

}  // namespace

// With wait == false the totals are copied back behind an event and turned
// into statistics by interface_diagnostics_finish, so that the caller's
// stream keeps going.
int interface_diagnostics(pf_ctx* ctx, const pf_phase* ph, pf_interface_stats* st, bool wait) {
  StageScope stage(ctx, PF_STAGE_DIAG);
  DiagScratch* s = nullptr;
  int rc = scratch(ctx, &s);
  if (rc) return rc;
  // etaPhi and the denominator in the reference's order (src/physics/phasefield.h:10-14)
  PhiK P;
  P.rmin = std::log(ph->rho_l / ph->rho_g) * ph->rho_g * ph->rho_tilde_0;
  P.den = ph->alpha_phi * ph->rho_tilde_0 * ph->rho_l;
  const DevGrid G = dev_grid(ctx);
  const int nb = kDiagBlocks;
  (++ctx->launches), k_cell_phi<<<nb, kDiagNT, 0, ctx->stream>>>(G, P, s->phi);
  const Lattice L{s->phi, ctx->g.nx, ctx->g.ny, ctx->g.nz, ctx->g.dx};
  (++ctx->launches), k_diag_cells<<<nb, kDiagNT, 0, ctx->stream>>>(G, L, s->part);
  (++ctx->launches), k_diag_total<<<1, kDiagNT, 0, ctx->stream>>>(s->part, nb, s->total);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_total, s->total, sizeof(DiagPartial), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaEventRecord(s->copied, ctx->stream));
  s->pending = true;
  if (!wait) return PF_OK;
  rc = interface_diagnostics_finish(ctx);
  if (!rc && st) *st = ctx->diag_last;
  return rc;
}

int interface_diagnostics_finish(pf_ctx* ctx) {
  DiagScratch* s = static_cast<DiagScratch*>(ctx->idiag);
  if (!s || !s->pending) return PF_OK;
  PF_CUDA_TRY(cudaEventSynchronize(s->copied));
  s->pending = false;
  const DiagPartial& t = *s->h_total;
  // finishStats (:55-66)
  pf_interface_stats out{};
  out.sample_cells = t.samples;
  out.interface_cells = t.interface;
  out.finite = t.finite;
  out.phi_min = t.samples ? t.phi_min : 0.0;
  out.phi_max = t.samples ? t.phi_max : 0.0;
  out.phi_mean = t.samples ? t.phi_sum / (double)t.samples : 0.0;
  out.grad_mean = t.interface ? t.grad_sum / (double)t.interface : 0.0;
  out.grad_max = t.grad_max;
  out.curvature_abs_mean = t.interface ? t.curv_sum / (double)t.interface : 0.0;
  out.curvature_abs_max = t.curv_max;
  out.surface_tension_candidate = (t.finite && t.interface > 0 && t.grad_max > 1e-5) ? 1 : 0;
  ctx->diag_last = out;
  return PF_OK;
}

// applySparseSurfaceTension3D (src/driver/interface_diagnostics3d.cpp:405-447)
int surface_tension(pf_ctx* ctx, const pf_phase* ph, double dt, double strength, double max_dv, int radius,
                    pf_surface_stats* st) {
  StageScope stage(ctx, PF_STAGE_DIAG);
  pf_surface_stats out{};
  out.finite = 1;
  out.enabled = strength > 0.0 && dt > 0.0;
  out.strength = strength;
  out.max_delta_speed_limit = max_dv;
  out.curvature_smoothing_radius = std::min(3, std::max(0, radius));
  {  // capillaryDtLimit (:78-83), initSurfaceStats (:85-99)
    const double rho_min = std::min(ph->rho_l, ph->rho_g);
    const double kpi = 3.14159265358979323846;
    out.capillary_dt_limit = (ctx->g.dx <= 0.0 || strength <= 0.0 || rho_min <= 0.0 || !std::isfinite(rho_min))
                                 ? 0.0
                                 : std::sqrt((rho_min * ctx->g.dx * ctx->g.dx * ctx->g.dx) / (2.0 * kpi * strength));
    out.capillary_stable = !out.enabled || out.capillary_dt_limit <= 0.0 || dt <= out.capillary_dt_limit + 1e-12;
  }
  if (out.enabled) {
    DiagScratch* s = nullptr;
    int rc = scratch(ctx, &s);
    if (rc) return rc;
    if (!s->h) {
      PF_CUDA_TRY(cudaMalloc(&s->h, 3 * s->ncell * sizeof(float)));
      PF_CUDA_TRY(cudaMalloc(&s->ok, s->ncell));
      PF_CUDA_TRY(cudaMalloc(&s->spart, (kDiagBlocks + 1) * sizeof(SurfPartial)));
      PF_CUDA_TRY(cudaMalloc(&s->bad, sizeof(int)));
    }
    PhiK P;
    P.rmin = std::log(ph->rho_l / ph->rho_g) * ph->rho_g * ph->rho_tilde_0;
    P.den = ph->alpha_phi * ph->rho_tilde_0 * ph->rho_l;
    const DevGrid G = dev_grid(ctx);
    const int nb = kDiagBlocks;
    const int big = 0x7fffffff;
    PF_CUDA_TRY(cudaMemcpyAsync(s->bad, &big, sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
    (++ctx->launches), k_cell_phi<<<nb, kDiagNT, 0, ctx->stream>>>(G, P, s->phi);
    const Lattice L{s->phi, ctx->g.nx, ctx->g.ny, ctx->g.nz, ctx->g.dx};
    (++ctx->launches), k_surface_cells<<<nb, kDiagNT, 0, ctx->stream>>>(G, L, strength, dt, max_dv,
                                                                         out.curvature_smoothing_radius, s->h, s->ok,
                                                                         s->bad, s->spart);
    (++ctx->launches), k_surface_total<<<1, kDiagNT, 0, ctx->stream>>>(s->spart, nb, s->spart + nb);
    rc = pool_sync(ctx);
    if (rc) return rc;
    if (ctx->nslots > 0)
      (++ctx->launches), k_surface_faces<<<std::min(ctx->nslots, 64 * ctx->num_sms), PF_TV, 0, ctx->stream>>>(
          G, ctx->nslots, s->h, s->ok, s->bad);
    PF_CUDA_TRY(cudaGetLastError());
    SurfPartial t;
    PF_CUDA_TRY(cudaMemcpyAsync(&t, s->spart + nb, sizeof(t), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    out.applied_cells = t.applied;
    out.finite = t.finite;
    out.max_delta_speed = t.dv_max;
    out.raw_curvature_abs_max = t.raw_max;
    out.smoothed_curvature_abs_max = t.sm_max;
    if (t.applied > 0) {  // finishSurfaceStats (:128-135)
      out.mean_delta_speed = t.dv_sum / (double)t.applied;
      out.raw_curvature_abs_mean = t.raw_sum / (double)t.applied;
      out.smoothed_curvature_abs_mean = t.sm_sum / (double)t.applied;
    }
  }
  ctx->surface_last = out;
  if (st) *st = out;
  return PF_OK;
}

void diag_free(pf_ctx* ctx) {
  DiagScratch* s = static_cast<DiagScratch*>(ctx->idiag);
  if (!s) return;
  cudaFree(s->phi);
  cudaFree(s->h);
  cudaFree(s->ok);
  cudaFree(s->spart);
  cudaFree(s->bad);
  cudaFree(s->part);
  cudaFree(s->total);
  cudaFreeHost(s->h_total);
  if (s->copied) cudaEventDestroy(s->copied);
  delete s;
  ctx->idiag = nullptr;
}

}  // namespace pf
