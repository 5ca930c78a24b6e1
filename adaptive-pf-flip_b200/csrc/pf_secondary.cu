// pf_secondary.cu -- the secondary particles of SparseSim3DTP::step()
// (src/driver/sparse_sim3d_tp.cpp:185-337; src/driver/secondary_particles3d.h:
// 9-467): escaped particles branched into droplet and bubble sets, their
// lifecycle (gravity or buoyancy, damping, drag, expiry, reabsorption into the
// primary set) and the spray seeds emitted from the liquid particles.
//
// The two sets live on the device in FP64 SoA (positions, velocities,
// volumes) with an age per particle, as the reference keeps them in FP64.
// Every per-particle expression rounds as the reference's does (_rn
// intrinsics, so no FMA contraction; the drag factor's exp is evaluated on the
// host), statistics are summed by one thread in particle order, and removals
// and appends keep particle order (order-preserving selects), so the sets and
// statistics equal the reference's arithmetic on the same inputs.  Spray
// candidates are ranked by a stable descending radix sort of their scores:
// equal scores keep particle order, where the reference's std::sort leaves
// them unspecified.
//
// Host round trips per step: one for the lifecycle, one for the escapes, one
// (two when the fallback ranking runs) for the spray candidates and one for
// the ranked window the seeds are made from.
#include <cub/cub.cuh>
#include <thrust/iterator/counting_iterator.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "pf_ctx.h"

namespace pf {
namespace {

constexpr int kSecNT = 256;

struct SecSet {
  double *x = nullptr, *y = nullptr, *z = nullptr, *vx = nullptr, *vy = nullptr, *vz = nullptr, *vol = nullptr;
  int* age = nullptr;
  size_t n = 0, cap = 0;
};

struct Primary {
  float *px, *py, *pz, *vx, *vy, *vz, *vol;
  uint8_t* type;
};

// device result slots, read back in one copy each
enum : int {
  I_TALLY = 0,  // 8 per type: advected, reabsorbed, expired, dragged, to primary, finite
  I_REAB = 16,  // + type: reabsorbed particles selected for the primary set
  I_KEEP = 18,  // + type: survivors
  I_ESC = 20,   // + type: escaped particles of the type
  I_NIMPACT = 24,
  I_FINITE = 25,
  I_NCAND = 26,
  I_COUNT = 32
};
enum : int {
  D_TALLY = 0,    // 4 per type: reabsorbed, expired, to primary and surviving volume
  D_ESCVOL = 8,   // + type: volume of the escaped particles appended
  D_SETVOL = 12,  // + type: volume of each set before the spray seeds
  D_BOUNDS = 16,  // min xyz, max xyz, any liquid particle
  D_GEOM = 24,    // surface y, impact y, centre x, centre z
  D_COUNT = 32
};

struct SecState {
  SecSet set[2];  // droplets (type 0), bubbles (type 1)
  SecSet tmp[2];  // compaction targets, swapped with set
  pf_secondary_cfg cfg{};
  pf_secondary_stats last{};
  int spray_index = 0;
  // lifecycle scratch, per type
  int* outcome[2] = {};  // 0 kept, 1 not finite, 2 reabsorbed, 3 expired
  int* keep_idx[2] = {};
  int* reab_idx[2] = {};
  size_t lcap[2] = {};
  // primary-sized scratch
  int* esc_idx[2] = {};
  int* cflag = nullptr;
  double* score = nullptr;
  double* key = nullptr;
  double* key_sorted = nullptr;
  int* cand = nullptr;
  int* cand_sorted = nullptr;
  uint8_t* impact = nullptr;
  double* part = nullptr;  // per-block liquid bounds
  size_t pcap = 0;
  void* cub_tmp = nullptr;
  size_t cub_bytes = 0;
  double* window = nullptr;  // pinned: the ranked candidates, 7 doubles each
  size_t window_cap = 0;
  int* d_ints = nullptr;
  double* d_sums = nullptr;
  int* h_ints = nullptr;  // pinned
  double* h_sums = nullptr;
};

__device__ __forceinline__ bool finite_particle(double x, double y, double z, double vx, double vy, double vz,
                                                double v) {
  return isfinite(x) && isfinite(y) && isfinite(z) && isfinite(vx) && isfinite(vy) && isfinite(vz) && isfinite(v);
}

// std::max / std::min as the reference applies them
__host__ __device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__host__ __device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

struct Advance {
  double dt, accel, damping, lo[3], hi[3], b0[3], b1[3];
  int band, lifetime;
};

// advanceSecondarySet3D's per-particle update (secondary_particles3d.h:345-427)
__global__ void k_sec_advance(SecSet s, Advance a, int* outcome) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= s.n) return;
  double x = s.x[p], y = s.y[p], z = s.z[p], vx = s.vx[p], vy = s.vy[p], vz = s.vz[p];
  if (!finite_particle(x, y, z, vx, vy, vz, s.vol[p])) {
    outcome[p] = 1;
    return;
  }
  const int age = s.age[p] + 1;
  s.age[p] = age;
  vy = __dadd_rn(vy, __dmul_rn(a.accel, a.dt));
  vx = __dmul_rn(vx, a.damping);
  vy = __dmul_rn(vy, a.damping);
  vz = __dmul_rn(vz, a.damping);
  x = __dadd_rn(x, __dmul_rn(vx, a.dt));
  y = __dadd_rn(y, __dmul_rn(vy, a.dt));
  z = __dadd_rn(z, __dmul_rn(vz, a.dt));
  x = dmax(a.lo[0], dmin(a.hi[0], x));
  y = dmax(a.lo[1], dmin(a.hi[1], y));
  z = dmax(a.lo[2], dmin(a.hi[2], z));
  s.x[p] = x;
  s.y[p] = y;
  s.z[p] = z;
  s.vx[p] = vx;
  s.vy[p] = vy;
  s.vz[p] = vz;
  const bool inside = a.band && x > a.b0[0] && x < a.b1[0] && y > a.b0[1] && y < a.b1[1] && z > a.b0[2] &&
                      z < a.b1[2];
  outcome[p] = inside ? 2 : (a.lifetime >= 0 && age >= a.lifetime) ? 3 : 0;
}

// The statistics of one set in particle order (one thread), and the volume of
// the survivors (secondaryVolumeSum3D after the compaction: the same order).
__global__ void k_sec_tally(SecSet s, const int* outcome, double scale, int dragged, int to_primary, int* ints,
                            double* sums) {
  int adv = 0, reab = 0, expd = 0, drag = 0, toprim = 0, finite = 1;
  double vreab = 0.0, vexp = 0.0, vprim = 0.0, vcur = 0.0;
  for (size_t p = 0; p < s.n; ++p) {
    const int o = outcome[p];
    const double v = __dmul_rn(s.vol[p], scale);
    if (o == 1) {
      finite = 0;
      ++expd;
      vexp = __dadd_rn(vexp, v);
      continue;
    }
    ++adv;
    if (dragged) ++drag;
    if (o == 2) {
      ++reab;
      vreab = __dadd_rn(vreab, v);
      if (to_primary) {
        ++toprim;
        vprim = __dadd_rn(vprim, v);
      }
    } else if (o == 3) {
      ++expd;
      vexp = __dadd_rn(vexp, v);
    } else {
      vcur = __dadd_rn(vcur, v);
    }
  }
  ints[0] = adv;
  ints[1] = reab;
  ints[2] = expd;
  ints[3] = drag;
  ints[4] = toprim;
  ints[5] = finite;
  sums[0] = vreab;
  sums[1] = vexp;
  sums[2] = vprim;
  sums[3] = vcur;
}

// secondaryVolumeSum3D over [from, n) in particle order (one thread)
__global__ void k_sec_volume(SecSet s, size_t from, double scale, double* out) {
  double v = 0.0;
  for (size_t p = from; p < s.n; ++p) v = __dadd_rn(v, __dmul_rn(s.vol[p], scale));
  *out = v;
}

// the survivors, gathered in order into d
__global__ void k_sec_gather(SecSet s, SecSet d, const int* idx, int count) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int p = idx[q];
  d.x[q] = s.x[p];
  d.y[q] = s.y[p];
  d.z[q] = s.z[p];
  d.vx[q] = s.vx[p];
  d.vy[q] = s.vy[p];
  d.vz[q] = s.vz[p];
  d.vol[q] = s.vol[p];
  d.age[q] = s.age[p];
}

// reabsorbed particles appended to the primary set in order (Particles3DTP::add)
__global__ void k_sec_to_primary(SecSet s, const int* idx, int count, Primary P, size_t base, uint8_t type) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int p = idx[q];
  const size_t o = base + (size_t)q;
  P.px[o] = (float)s.x[p];
  P.py[o] = (float)s.y[p];
  P.pz[o] = (float)s.z[p];
  P.vx[o] = (float)s.vx[p];
  P.vy[o] = (float)s.vy[p];
  P.vz[o] = (float)s.vz[p];
  P.vol[o] = (float)s.vol[p];
  P.type[o] = type;
}

// storeEscapedParticles (sparse_sim3d_tp.cpp:192-218): the escaped particles
// appended with age 0
__global__ void k_sec_escape_append(Primary P, const int* idx, int count, SecSet s, size_t base) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= count) return;
  const int p = idx[q];
  const size_t o = base + (size_t)q;
  s.x[o] = P.px[p];
  s.y[o] = P.py[p];
  s.z[o] = P.pz[p];
  s.vx[o] = P.vx[p];
  s.vy[o] = P.vy[p];
  s.vz[o] = P.vz[p];
  s.vol[o] = P.vol[p];
  s.age[o] = 0;
}

struct OutcomeIs {
  const int* o;
  int want;
  __device__ bool operator()(int p) const { return o[p] == want; }
};

struct EscapedOfType {
  const int* esc;
  const uint8_t* type;
  uint8_t want;
  __device__ bool operator()(int p) const { return esc[p] != 0 && type[p] == want; }
};

// liquidParticleBounds3D (secondary_particles3d.h:128-134): per-block extrema
__global__ void k_sec_bounds(Primary P, size_t n, double* part) {
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  double any = 0.0;
  for (size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x; p < n; p += (size_t)gridDim.x * blockDim.x) {
    if (P.type[p] != 0) continue;
    const double q[3] = {P.px[p], P.py[p], P.pz[p]};
    any = 1.0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      mn[a] = fmin(mn[a], q[a]);
      mx[a] = fmax(mx[a], q[a]);
    }
  }
  __shared__ double sh[7][kSecNT];
  for (int a = 0; a < 3; ++a) {
    sh[a][threadIdx.x] = mn[a];
    sh[3 + a][threadIdx.x] = mx[a];
  }
  sh[6][threadIdx.x] = any;
  __syncthreads();
  for (int w = kSecNT / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) {
      for (int a = 0; a < 3; ++a) {
        sh[a][threadIdx.x] = fmin(sh[a][threadIdx.x], sh[a][threadIdx.x + w]);
        sh[3 + a][threadIdx.x] = fmax(sh[3 + a][threadIdx.x], sh[3 + a][threadIdx.x + w]);
      }
      sh[6][threadIdx.x] = fmax(sh[6][threadIdx.x], sh[6][threadIdx.x + w]);
    }
    __syncthreads();
  }
  if (threadIdx.x < 7) part[7 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// the bounds over all blocks and the spray geometry derived from them
// (emitSecondarySpraySeeds3D, secondary_particles3d.h:160-166)
__global__ void k_sec_geometry(const double* part, int nb, double impact_fraction, double* out) {
  double r[7] = {INFINITY, INFINITY, INFINITY, -INFINITY, -INFINITY, -INFINITY, 0.0};
  for (int b = 0; b < nb; ++b)
    for (int a = 0; a < 7; ++a) r[a] = a < 3 ? fmin(r[a], part[7 * b + a]) : fmax(r[a], part[7 * b + a]);
  for (int a = 0; a < 7; ++a) out[D_BOUNDS + a] = r[a];
  const double h = __dsub_rn(r[4], r[1]);
  out[D_GEOM + 0] = __dadd_rn(r[1], __dmul_rn(0.68, h));
  out[D_GEOM + 1] = __dadd_rn(r[1], __dmul_rn(dmax(0.0, dmin(1.0, impact_fraction)), h));
  out[D_GEOM + 2] = __dmul_rn(0.5, __dadd_rn(r[0], r[3]));
  out[D_GEOM + 3] = __dmul_rn(0.5, __dadd_rn(r[2], r[5]));
}

// the spray candidates' flags and scores (secondary_particles3d.h:168-199);
// the fallback ranks every finite liquid particle by its height
__global__ void k_sec_score(Primary P, size_t n, const double* geom, int impact_on, double downward_min, int fallback,
                            int* flag, double* score, uint8_t* impact, int* ints) {
  const size_t p = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  int nimp = 0, bad = 0;
  if (p < n) {
    int f = 0;
    double sc = 0.0;
    uint8_t im = 0;
    if (P.type[p] == 0) {
      const double x = P.px[p], y = P.py[p], z = P.pz[p], vx = P.vx[p], vy = P.vy[p], vz = P.vz[p];
      if (!finite_particle(x, y, z, vx, vy, vz, P.vol[p])) {
        bad = 1;
      } else if (fallback) {
        f = 1;
        sc = y;
      } else {
        const double surface_y = geom[0], impact_y = geom[1], cx = geom[2], cz = geom[3];
        const double hspeed = __dsqrt_rn(__dadd_rn(__dmul_rn(vx, vx), __dmul_rn(vz, vz)));
        const double upward = dmax(0.0, vy);
        const double downward = dmax(0.0, -vy);
        const double near = dmax(0.0, __dsub_rn(y, surface_y));
        const bool imp = impact_on && y <= impact_y && downward >= downward_min;
        const double ex = __dsub_rn(x, cx), ez = __dsub_rn(z, cz);
        const double lateral = __dsqrt_rn(__dadd_rn(__dmul_rn(ex, ex), __dmul_rn(ez, ez)));
        const double depth = dmax(0.0, __dsub_rn(impact_y, y));
        double s = __dadd_rn(__dmul_rn(near, 4.0), __dmul_rn(upward, 2.0));
        s = __dadd_rn(s, __dmul_rn(hspeed, 0.25));
        s = __dadd_rn(s, __dmul_rn(lateral, 0.03));
        s = __dadd_rn(s, imp ? __dadd_rn(__dmul_rn(downward, 2.5), __dmul_rn(depth, 0.8)) : 0.0);
        if (y >= surface_y || upward > 0.02 || hspeed > 0.25 || imp) {
          f = 1;
          sc = s;
          im = imp ? 1 : 0;
          nimp = imp ? 1 : 0;
        }
      }
    }
    flag[p] = f;
    score[p] = sc;
    impact[p] = im;
  }
  const unsigned m = __ballot_sync(0xffffffffu, nimp), b = __ballot_sync(0xffffffffu, bad);
  if ((threadIdx.x & 31) == 0) {
    if (m) atomicAdd(&ints[I_NIMPACT], __popc(m));
    if (b) atomicAnd(&ints[I_FINITE], 0);
  }
}

__global__ void k_sec_keys(const int* cand, const int* count, const double* score, double* key) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r < *count) key[r] = score[cand[r]];
}

__global__ void k_sec_reset_ints(int* ints) {
  ints[I_NIMPACT] = 0;
  ints[I_FINITE] = 1;
}

// the ranked candidates' positions, velocities and impact flags (7 doubles)
__global__ void k_sec_take(Primary P, const uint8_t* impact, const int* idx, int m, double* out) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= m) return;
  const int p = idx[r];
  double* o = out + 7 * (size_t)r;
  o[0] = P.px[p];
  o[1] = P.py[p];
  o[2] = P.pz[p];
  o[3] = P.vx[p];
  o[4] = P.vy[p];
  o[5] = P.vz[p];
  o[6] = impact[p];
}

// ---- host helpers -----------------------------------------------------------

template <class T>
void free_dev(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

int grow_set(pf_ctx* ctx, SecSet& s, size_t need) {
  if (need <= s.cap) return PF_OK;
  size_t cap = std::max<size_t>(need, 2 * s.cap);
  cap = std::max<size_t>(cap, 256);
  SecSet t;
  t.cap = cap;
  t.n = s.n;
  double** d[7] = {&t.x, &t.y, &t.z, &t.vx, &t.vy, &t.vz, &t.vol};
  double* o[7] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.vol};
  for (int a = 0; a < 7; ++a) {
    PF_CUDA_TRY(cudaMalloc(d[a], cap * sizeof(double)));
    if (s.n) PF_CUDA_TRY(cudaMemcpyAsync(*d[a], o[a], s.n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
  }
  PF_CUDA_TRY(cudaMalloc(&t.age, cap * sizeof(int)));
  if (s.n) PF_CUDA_TRY(cudaMemcpyAsync(t.age, s.age, s.n * sizeof(int), cudaMemcpyDeviceToDevice, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  for (int a = 0; a < 7; ++a)
    if (o[a]) cudaFree(o[a]);
  if (s.age) cudaFree(s.age);
  s = t;
  return PF_OK;
}

void free_set(SecSet& s) {
  double* o[7] = {s.x, s.y, s.z, s.vx, s.vy, s.vz, s.vol};
  for (double* q : o)
    if (q) cudaFree(q);
  if (s.age) cudaFree(s.age);
  s = SecSet{};
}

// SparseSim3DTP's defaults (src/driver/sparse_sim3d_tp.h:82-137)
void default_cfg(pf_secondary_cfg* c) {
  *c = pf_secondary_cfg{};
  c->droplet_lifetime_steps = c->bubble_lifetime_steps = 48;
  c->velocity_damping = 0.98;
  c->reabsorb_margin_cells = 1.0;
  c->droplet_gravity_scale = 1.0;
  c->bubble_buoyancy_scale = 0.25;
  c->spray_droplet_fraction = 0.9;
  c->spray_droplet_volume = 0.55;
  c->spray_bubble_volume = 0.45;
  c->spray_min_interface_cells = 1;
  c->spray_min_interface_grad_max = 1e-5;
  c->spray_impact_region_fraction = 0.55;
  c->spray_impact_downward_speed_min = 1.0;
  c->spray_impact_foam_fraction = 0.3;
}

int sec_state(pf_ctx* ctx, SecState** out) {
  SecState* s = static_cast<SecState*>(ctx->secondary);
  if (!s) {
    s = new SecState();
    ctx->secondary = s;
    default_cfg(&s->cfg);
    PF_CUDA_TRY(cudaMalloc(&s->d_ints, I_COUNT * sizeof(int)));
    PF_CUDA_TRY(cudaMalloc(&s->d_sums, D_COUNT * sizeof(double)));
    PF_CUDA_TRY(cudaMallocHost(&s->h_ints, I_COUNT * sizeof(int)));
    PF_CUDA_TRY(cudaMallocHost(&s->h_sums, D_COUNT * sizeof(double)));
    PF_CUDA_TRY(cudaMemsetAsync(s->d_ints, 0, I_COUNT * sizeof(int), ctx->stream));
    PF_CUDA_TRY(cudaMemsetAsync(s->d_sums, 0, D_COUNT * sizeof(double), ctx->stream));
  }
  *out = s;
  return PF_OK;
}

int life_scratch(pf_ctx* ctx, SecState* s, int t, size_t n) {
  if (n <= s->lcap[t]) return PF_OK;
  free_dev(s->outcome[t]);
  free_dev(s->keep_idx[t]);
  free_dev(s->reab_idx[t]);
  s->lcap[t] = 0;
  const size_t cap = std::max<size_t>(2 * n, 1024);
  PF_CUDA_TRY(cudaMalloc(&s->outcome[t], cap * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->keep_idx[t], cap * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->reab_idx[t], cap * sizeof(int)));
  s->lcap[t] = cap;
  return PF_OK;
}

int primary_scratch(pf_ctx* ctx, SecState* s) {
  const size_t n = ctx->cap + 1;
  if (s->pcap >= n) return PF_OK;
  for (int t = 0; t < 2; ++t) free_dev(s->esc_idx[t]);
  free_dev(s->cflag);
  free_dev(s->score);
  free_dev(s->key);
  free_dev(s->key_sorted);
  free_dev(s->cand);
  free_dev(s->cand_sorted);
  free_dev(s->impact);
  free_dev(s->part);
  s->pcap = 0;
  for (int t = 0; t < 2; ++t) PF_CUDA_TRY(cudaMalloc(&s->esc_idx[t], n * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->cflag, n * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->score, n * sizeof(double)));
  PF_CUDA_TRY(cudaMalloc(&s->key, n * sizeof(double)));
  PF_CUDA_TRY(cudaMalloc(&s->key_sorted, n * sizeof(double)));
  PF_CUDA_TRY(cudaMalloc(&s->cand, n * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->cand_sorted, n * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->impact, n));
  PF_CUDA_TRY(cudaMalloc(&s->part, (size_t)7 * 8 * ctx->num_sms * sizeof(double)));
  s->pcap = n;
  return PF_OK;
}

// CUB temporary storage of at least `bytes`
int cub_storage(pf_ctx* ctx, SecState* s, size_t bytes) {
  if (bytes <= s->cub_bytes) return PF_OK;
  free_dev(s->cub_tmp);
  s->cub_bytes = 0;
  PF_CUDA_TRY(cudaMalloc(&s->cub_tmp, bytes));
  s->cub_bytes = bytes;
  return PF_OK;
}

// order-preserving selection of the indices in [0, n) that satisfy pred
template <class Pred>
int select_if(pf_ctx* ctx, SecState* s, int n, Pred pred, int* out, int* count) {
  if (n <= 0) {
    PF_CUDA_TRY(cudaMemsetAsync(count, 0, sizeof(int), ctx->stream));
    return PF_OK;
  }
  thrust::counting_iterator<int> first(0);
  size_t bytes = 0;
  PF_CUDA_TRY(cub::DeviceSelect::If(nullptr, bytes, first, out, count, n, pred, ctx->stream));
  int rc = cub_storage(ctx, s, bytes);
  if (rc) return rc;
  bytes = s->cub_bytes;
  PF_CUDA_TRY(cub::DeviceSelect::If(s->cub_tmp, bytes, first, out, count, n, pred, ctx->stream));
  return PF_OK;
}

int select_flagged(pf_ctx* ctx, SecState* s, int n, const int* flags, int* out, int* count) {
  thrust::counting_iterator<int> first(0);
  size_t bytes = 0;
  PF_CUDA_TRY(cub::DeviceSelect::Flagged(nullptr, bytes, first, flags, out, count, n, ctx->stream));
  int rc = cub_storage(ctx, s, bytes);
  if (rc) return rc;
  bytes = s->cub_bytes;
  PF_CUDA_TRY(cub::DeviceSelect::Flagged(s->cub_tmp, bytes, first, flags, out, count, n, ctx->stream));
  return PF_OK;
}

int read_back(pf_ctx* ctx, SecState* s) {
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_ints, s->d_ints, I_COUNT * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_sums, s->d_sums, D_COUNT * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

Primary primary_of(pf_ctx* ctx) {
  return Primary{ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy, ctx->vz, ctx->vol, ctx->type};
}

// advanceSecondaryParticles3D (secondary_particles3d.h:429-467) as
// advanceSecondaryLifecycle applies it (sparse_sim3d_tp.cpp:226-274)
int lifecycle(pf_ctx* ctx, SecState* s, double dt, double gravity, double Vp) {
  pf_secondary_stats& st = s->last;
  const pf_secondary_cfg& c = s->cfg;
  st.lifecycle_enabled = c.lifecycle ? 1 : 0;
  st.lifecycle_finite = 1;
  if (s->set[0].n == 0 && s->set[1].n == 0) return PF_OK;
  if (!(c.lifecycle && dt > 0.0)) {
    // nothing moves: the current volumes of the sets as they are
    for (int t = 0; t < 2; ++t)
      (++ctx->launches), k_sec_volume<<<1, 1, 0, ctx->stream>>>(s->set[t], 0, Vp, s->d_sums + D_TALLY + 4 * t + 3);
    PF_CUDA_TRY(cudaGetLastError());
    int rc = read_back(ctx, s);
    if (rc) return rc;
    st.lifecycle_droplet_volume = s->h_sums[D_TALLY + 3];
    st.lifecycle_bubble_volume = s->h_sums[D_TALLY + 7];
    return PF_OK;
  }
  const Geom& g = ctx->g;
  const double o[3] = {g.ox, g.oy, g.oz};
  const int nn[3] = {g.nx, g.ny, g.nz};
  const double margin = dmax(0.0, c.reabsorb_margin_cells) * g.dx;
  bool ran[2] = {false, false};
  for (int t = 0; t < 2; ++t) {
    SecSet& set = s->set[t];
    if (set.n == 0) continue;
    ran[t] = true;
    int rc = life_scratch(ctx, s, t, set.n);
    if (rc) return rc;
    Advance a{};
    a.dt = dt;
    a.accel = t == 0 ? gravity * c.droplet_gravity_scale : -gravity * c.bubble_buoyancy_scale;
    const double drag = t == 0 ? c.droplet_drag : c.bubble_drag;
    a.damping = dmax(0.0, c.velocity_damping);
    if (drag > 0.0) a.damping *= std::exp(-drag * dt);
    for (int d = 0; d < 3; ++d) {
      a.lo[d] = o[d] + 0.5 * g.dx;
      a.hi[d] = o[d] + ((double)nn[d] - 0.5) * g.dx;
      a.b0[d] = o[d] + (0.5 * g.dx) + margin;
      a.b1[d] = o[d] + ((double)nn[d] - 0.5) * g.dx - margin;
    }
    a.band = !(a.b0[0] >= a.b1[0] || a.b0[1] >= a.b1[1] || a.b0[2] >= a.b1[2]);
    a.lifetime = t == 0 ? c.droplet_lifetime_steps : c.bubble_lifetime_steps;
    (++ctx->launches), k_sec_advance<<<nblocks(set.n, kSecNT), kSecNT, 0, ctx->stream>>>(set, a, s->outcome[t]);
    (++ctx->launches), k_sec_tally<<<1, 1, 0, ctx->stream>>>(set, s->outcome[t], Vp, drag > 0.0 ? 1 : 0,
                                                             c.reabsorb_to_primary ? 1 : 0, s->d_ints + I_TALLY + 8 * t,
                                                             s->d_sums + D_TALLY + 4 * t);
    PF_CUDA_TRY(cudaGetLastError());
    rc = select_if(ctx, s, (int)set.n, OutcomeIs{s->outcome[t], 0}, s->keep_idx[t], s->d_ints + I_KEEP + t);
    if (rc) return rc;
    if (c.reabsorb_to_primary) {
      rc = select_if(ctx, s, (int)set.n, OutcomeIs{s->outcome[t], 2}, s->reab_idx[t], s->d_ints + I_REAB + t);
      if (rc) return rc;
    }
  }
  int rc = read_back(ctx, s);
  if (rc) return rc;
  int iv[2][6] = {{0, 0, 0, 0, 0, 1}, {0, 0, 0, 0, 0, 1}};
  double dv[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
  int reab[2] = {0, 0}, kept[2] = {0, 0};
  for (int t = 0; t < 2; ++t) {
    if (!ran[t]) continue;
    for (int q = 0; q < 6; ++q) iv[t][q] = s->h_ints[I_TALLY + 8 * t + q];
    for (int q = 0; q < 4; ++q) dv[t][q] = s->h_sums[D_TALLY + 4 * t + q];
    reab[t] = c.reabsorb_to_primary ? s->h_ints[I_REAB + t] : 0;
    kept[t] = s->h_ints[I_KEEP + t];
  }
  // reabsorbed droplets, then bubbles, appended to the primary set
  if (ctx->np + (size_t)reab[0] + (size_t)reab[1] > ctx->cap)
    return set_error(ctx, PF_ERR_CAPACITY, "secondary reabsorption exceeds max_particles");
  for (int t = 0; t < 2; ++t) {
    if (reab[t] <= 0) continue;
    (++ctx->launches), k_sec_to_primary<<<nblocks(reab[t], kSecNT), kSecNT, 0, ctx->stream>>>(
        s->set[t], s->reab_idx[t], reab[t], primary_of(ctx), ctx->np, (uint8_t)t);
    PF_CUDA_TRY(cudaGetLastError());
    ctx->np += (size_t)reab[t];
    ctx->bins_valid = false;
  }
  // the survivors, in order
  for (int t = 0; t < 2; ++t) {
    if (!ran[t]) continue;
    rc = grow_set(ctx, s->tmp[t], s->set[t].cap);
    if (rc) return rc;
    if (kept[t] > 0)
      (++ctx->launches), k_sec_gather<<<nblocks(kept[t], kSecNT), kSecNT, 0, ctx->stream>>>(s->set[t], s->tmp[t],
                                                                                            s->keep_idx[t], kept[t]);
    PF_CUDA_TRY(cudaGetLastError());
    std::swap(s->set[t], s->tmp[t]);
    s->set[t].n = (size_t)kept[t];
    s->tmp[t].n = 0;
  }
  st.advected_droplets = iv[0][0];
  st.advected_bubbles = iv[1][0];
  st.reabsorbed_droplets = iv[0][1];
  st.reabsorbed_bubbles = iv[1][1];
  st.expired_droplets = iv[0][2];
  st.expired_bubbles = iv[1][2];
  st.dragged_droplets = iv[0][3];
  st.dragged_bubbles = iv[1][3];
  st.reabsorbed_droplets_to_primary = iv[0][4];
  st.reabsorbed_bubbles_to_primary = iv[1][4];
  st.lifecycle_finite = iv[0][5] && iv[1][5] ? 1 : 0;
  st.reabsorbed_droplet_volume = dv[0][0];
  st.reabsorbed_bubble_volume = dv[1][0];
  st.expired_droplet_volume = dv[0][1];
  st.expired_bubble_volume = dv[1][1];
  st.reabsorbed_droplet_volume_to_primary = dv[0][2];
  st.reabsorbed_bubble_volume_to_primary = dv[1][2];
  st.lifecycle_droplet_volume = dv[0][3];
  st.lifecycle_bubble_volume = dv[1][3];
  return PF_OK;
}

// storeEscapedParticles (sparse_sim3d_tp.cpp:192-218)
int store_escaped(pf_ctx* ctx, SecState* s, const int* esc_flags, double Vp) {
  const int n = (int)ctx->np;
  int rc = primary_scratch(ctx, s);
  if (rc) return rc;
  for (int t = 0; t < 2; ++t) {
    rc = select_if(ctx, s, n, EscapedOfType{esc_flags, ctx->type, (uint8_t)t}, s->esc_idx[t], s->d_ints + I_ESC + t);
    if (rc) return rc;
  }
  rc = read_back(ctx, s);
  if (rc) return rc;
  pf_secondary_stats& st = s->last;
  for (int t = 0; t < 2; ++t) {
    const int k = s->h_ints[I_ESC + t];
    SecSet& set = s->set[t];
    const size_t base = set.n;
    if (k > 0) {
      rc = grow_set(ctx, set, set.n + (size_t)k);
      if (rc) return rc;
      (++ctx->launches), k_sec_escape_append<<<nblocks(k, kSecNT), kSecNT, 0, ctx->stream>>>(primary_of(ctx),
                                                                                             s->esc_idx[t], k, set, base);
      set.n += (size_t)k;
    }
    // the appended records' volume, read back with the spray's candidates
    (++ctx->launches), k_sec_volume<<<1, 1, 0, ctx->stream>>>(set, base, Vp, s->d_sums + D_ESCVOL + t);
    PF_CUDA_TRY(cudaGetLastError());
    if (t == 0) st.escaped_droplets_added = k;
    else st.escaped_bubbles_added = k;
  }
  return PF_OK;
}

// emitSecondarySpraySeeds3D (secondary_particles3d.h:136-278) on the context's
// particles.  On return h_sums holds D_ESCVOL and D_SETVOL, and the seeds are
// appended to the sets.
int spray(pf_ctx* ctx, SecState* s, double Vp, const pf_interface_stats& iface) {
  pf_secondary_stats& st = s->last;
  const pf_secondary_cfg& c = s->cfg;
  st.spray_enabled = c.spray_emission ? 1 : 0;
  st.spray_finite = 1;
  st.spray_requested_particles = std::max(0, c.spray_particles_per_step);
  st.spray_interface_gate_enabled = c.spray_interface_gate ? 1 : 0;
  st.spray_interface_gate_passed = 1;
  st.spray_interface_cells = iface.interface_cells;
  st.spray_interface_grad_max = iface.grad_max;
  st.spray_interface_curvature_abs_max = iface.curvature_abs_max;
  for (int t = 0; t < 2; ++t)
    (++ctx->launches), k_sec_volume<<<1, 1, 0, ctx->stream>>>(s->set[t], 0, Vp, s->d_sums + D_SETVOL + t);
  PF_CUDA_TRY(cudaGetLastError());
  bool emit = c.spray_emission && c.spray_particles_per_step > 0;
  if (emit && c.spray_interface_gate) {
    const bool fin = std::isfinite(iface.grad_max) && std::isfinite(iface.curvature_abs_max);
    const bool pass = fin && iface.interface_cells >= std::max(0, c.spray_min_interface_cells) &&
                      iface.grad_max >= c.spray_min_interface_grad_max &&
                      iface.curvature_abs_max >= c.spray_min_interface_curvature_abs_max;
    st.spray_interface_gate_passed = pass ? 1 : 0;
    if (!fin) st.spray_finite = 0;
    emit = pass;
  }
  const size_t n = ctx->np;
  if (!emit || n == 0) return read_back(ctx, s);
  int rc = primary_scratch(ctx, s);
  if (rc) return rc;
  const Primary P = primary_of(ctx);
  const int nbb = std::min(nblocks(n, kSecNT), 8 * ctx->num_sms);
  (++ctx->launches), k_sec_bounds<<<nbb, kSecNT, 0, ctx->stream>>>(P, n, s->part);
  (++ctx->launches), k_sec_geometry<<<1, 1, 0, ctx->stream>>>(s->part, nbb, c.spray_impact_region_fraction,
                                                              s->d_sums);
  PF_CUDA_TRY(cudaGetLastError());
  const int nb = nblocks(n, kSecNT);
  int ncand = 0;
  for (int fallback = 0; fallback < 2; ++fallback) {
    (++ctx->launches), k_sec_reset_ints<<<1, 1, 0, ctx->stream>>>(s->d_ints);
    (++ctx->launches), k_sec_score<<<nb, kSecNT, 0, ctx->stream>>>(
        P, n, s->d_sums + D_GEOM, c.spray_impact_candidates ? 1 : 0, c.spray_impact_downward_speed_min, fallback,
        s->cflag, s->score, s->impact, s->d_ints);
    PF_CUDA_TRY(cudaGetLastError());
    rc = select_flagged(ctx, s, (int)n, s->cflag, s->cand, s->d_ints + I_NCAND);
    if (rc) return rc;
    (++ctx->launches), k_sec_keys<<<nb, kSecNT, 0, ctx->stream>>>(s->cand, s->d_ints + I_NCAND, s->score, s->key);
    PF_CUDA_TRY(cudaGetLastError());
    rc = read_back(ctx, s);
    if (rc) return rc;
    if (!(s->h_sums[D_BOUNDS + 6] > 0.0)) return PF_OK;  // no liquid particle
    if (fallback == 0) {
      st.spray_impact_candidate_liquid_particles = s->h_ints[I_NIMPACT];
      if (!s->h_ints[I_FINITE]) st.spray_finite = 0;
    }
    ncand = s->h_ints[I_NCAND];
    if (ncand > 0) break;
  }
  st.spray_candidate_liquid_particles = ncand;
  if (ncand == 0) return PF_OK;
  // stable descending order of the scores: equal scores keep particle order
  size_t bytes = 0;
  PF_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(nullptr, bytes, s->key, s->key_sorted, s->cand,
                                                        s->cand_sorted, ncand, 0, 64, ctx->stream));
  rc = cub_storage(ctx, s, bytes);
  if (rc) return rc;
  bytes = s->cub_bytes;
  PF_CUDA_TRY(cub::DeviceRadixSort::SortPairsDescending(s->cub_tmp, bytes, s->key, s->key_sorted, s->cand,
                                                        s->cand_sorted, ncand, 0, 64, ctx->stream));
  const int requested = std::max(0, c.spray_particles_per_step);
  st.spray_effective_requested_particles = requested;
  const int window = (int)std::min<size_t>((size_t)ncand, (size_t)std::max(1, requested * 3));
  if ((size_t)window > s->window_cap) {
    if (s->window) cudaFreeHost(s->window);
    s->window = nullptr;
    s->window_cap = 0;
    PF_CUDA_TRY(cudaMallocHost(&s->window, (size_t)7 * window * sizeof(double)));
    s->window_cap = (size_t)window;
  }
  // the unsorted keys are spent: the window goes there when it fits
  double* dwin = s->key;
  double* dtmp = nullptr;
  if ((size_t)7 * window > s->pcap) {
    PF_CUDA_TRY(cudaMalloc(&dtmp, (size_t)7 * window * sizeof(double)));
    dwin = dtmp;
  }
  (++ctx->launches), k_sec_take<<<nblocks(window, kSecNT), kSecNT, 0, ctx->stream>>>(P, s->impact, s->cand_sorted,
                                                                                     window, dwin);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->window, dwin, (size_t)7 * window * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (dtmp) cudaFree(dtmp);
  if (e != cudaSuccess) return set_cuda_error(ctx, e, "spray candidates", __FILE__, __LINE__);
  // the seeds (secondary_particles3d.h:216-276), in the reference's arithmetic
  const double* h = s->window;
  const double mn_y = s->h_sums[D_BOUNDS + 1];
  const double cx = s->h_sums[D_GEOM + 2], cz = s->h_sums[D_GEOM + 3];
  const int frame = s->spray_index;
  const double dfrac = dmax(0.0, dmin(1.0, c.spray_droplet_fraction));
  int ndrop = (int)std::floor((double)requested * dfrac + 0.5);
  ndrop = std::max(0, std::min(requested, ndrop));
  const int nbub = std::max(0, requested - ndrop);
  const double foam_fraction = dmax(0.0, dmin(1.0, c.spray_impact_foam_fraction));
  int foam_stride = requested + 1;
  if (foam_fraction > 0.0) foam_stride = std::max(1, (int)std::floor((1.0 / foam_fraction) + 0.5));
  std::vector<double> seed[2][7];
  std::vector<int> seed_age[2];
  for (int k = 0; k < ndrop; ++k) {
    const size_t r = ((size_t)k * 37u + (size_t)frame * 11u) % (size_t)window;
    const double* q = h + 7 * r;
    const double dx = q[0] - cx, dz = q[2] - cz;
    const double len = std::sqrt(dx * dx + dz * dz);
    const double ox = len > 1e-8 ? dx / len : 0.0, oz = len > 1e-8 ? dz / len : 0.0;
    const double lift = 0.18 + 0.035 * (double)((k + frame) % 5);
    const bool foam = q[6] != 0.0 && ((k + frame) % foam_stride == 0);
    const double p[3] = {q[0] + 0.035 * ox, q[1] + (foam ? 0.025 : 0.04 + 0.01 * (double)(k % 3)), q[2] + 0.035 * oz};
    double v[3];
    if (foam) {
      v[0] = 0.08 * ox;
      v[1] = 0.08;
      v[2] = 0.08 * oz;
    } else {
      v[0] = q[3] + 0.16 * ox;
      v[1] = q[4] + lift;
      v[2] = q[5] + 0.16 * oz;
    }
    const double speed = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    seed_age[0].push_back(foam ? 6 : (speed > 1.0 ? 0 : (k % 4 == 0 ? 5 : 2)));
    for (int a = 0; a < 3; ++a) {
      seed[0][a].push_back(p[a]);
      seed[0][3 + a].push_back(v[a]);
    }
    seed[0][6].push_back(c.spray_droplet_volume);
    if (foam) ++st.spray_foam_ready_droplets;
    ++st.spray_emitted_droplets;
    st.spray_emitted_droplet_volume += c.spray_droplet_volume * Vp;
  }
  for (int k = 0; k < nbub; ++k) {
    const size_t r = ((size_t)k * 53u + (size_t)frame * 7u) % (size_t)window;
    const double* q = h + 7 * r;
    seed_age[1].push_back(0);
    seed[1][0].push_back(q[0]);
    seed[1][1].push_back(dmax(mn_y + 0.25, q[1] - 0.12));
    seed[1][2].push_back(q[2]);
    seed[1][3].push_back(0.0);
    seed[1][4].push_back(0.16);
    seed[1][5].push_back(0.0);
    seed[1][6].push_back(c.spray_bubble_volume);
    ++st.spray_emitted_bubbles;
    st.spray_emitted_bubble_volume += c.spray_bubble_volume * Vp;
  }
  for (int t = 0; t < 2; ++t) {
    const size_t k = seed_age[t].size();
    if (!k) continue;
    SecSet& set = s->set[t];
    rc = grow_set(ctx, set, set.n + k);
    if (rc) return rc;
    double* dst[7] = {set.x, set.y, set.z, set.vx, set.vy, set.vz, set.vol};
    for (int a = 0; a < 7; ++a)
      PF_CUDA_TRY(cudaMemcpyAsync(dst[a] + set.n, seed[t][a].data(), k * sizeof(double), cudaMemcpyHostToDevice,
                                  ctx->stream));
    PF_CUDA_TRY(cudaMemcpyAsync(set.age + set.n, seed_age[t].data(), k * sizeof(int), cudaMemcpyHostToDevice,
                                ctx->stream));
    set.n += k;
  }
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));  // the seeds' host vectors go out of scope
  return PF_OK;
}

// emitSecondarySpray's bookkeeping (sparse_sim3d_tp.cpp:276-337) around the
// seeds; each set's current volume continues the device's sum over the
// particles before the seeds with the seeds, in order
int spray_step(pf_ctx* ctx, SecState* s, double Vp, const pf_interface_stats& iface) {
  pf_secondary_stats& st = s->last;
  const size_t before[2] = {s->set[0].n, s->set[1].n};
  int rc = spray(ctx, s, Vp, iface);
  if (rc) return rc;
  ++s->spray_index;
  st.spray_step_index = s->spray_index;
  st.escaped_droplet_volume_added = st.escaped_droplets_added ? s->h_sums[D_ESCVOL] : 0.0;
  st.escaped_bubble_volume_added = st.escaped_bubbles_added ? s->h_sums[D_ESCVOL + 1] : 0.0;
  st.escape_droplet_volume = st.escaped_droplet_volume_added;
  st.escape_bubble_volume = st.escaped_bubble_volume_added;
  st.escaped_droplets_added += st.spray_emitted_droplets;
  st.escaped_bubbles_added += st.spray_emitted_bubbles;
  st.escaped_droplet_volume_added += st.spray_emitted_droplet_volume;
  st.escaped_bubble_volume_added += st.spray_emitted_bubble_volume;
  for (int t = 0; t < 2; ++t) {
    double v = s->h_sums[D_SETVOL + t];
    const double seed_vol = t == 0 ? s->cfg.spray_droplet_volume : s->cfg.spray_bubble_volume;
    for (size_t p = before[t]; p < s->set[t].n; ++p) v += seed_vol * Vp;
    if (t == 0) st.droplet_volume_current = v;
    else st.bubble_volume_current = v;
  }
  return PF_OK;
}

}  // namespace

// the escape flags the step's advection writes, or none
int* secondary_escape_flags(pf_ctx* ctx) {
  const SecState* s = static_cast<const SecState*>(ctx->secondary);
  if (!s || !s->cfg.escaped_particle_branching) return nullptr;
  return ctx->d_flags;
}

bool secondary_active(const pf_ctx* ctx) {
  const SecState* s = static_cast<const SecState*>(ctx->secondary);
  if (!s) return false;
  const pf_secondary_cfg& c = s->cfg;
  return c.escaped_particle_branching || c.lifecycle || c.spray_emission || s->set[0].n || s->set[1].n;
}

// whether the lifecycle may move particles into the primary set
bool secondary_reabsorbs(const pf_ctx* ctx) {
  const SecState* s = static_cast<const SecState*>(ctx->secondary);
  return s && s->cfg.lifecycle && s->cfg.reabsorb_to_primary && (s->set[0].n || s->set[1].n);
}

// advanceSecondaryLifecycle (sparse_sim3d_tp.cpp:226-274)
int secondary_lifecycle(pf_ctx* ctx, double dt, double gravity, double Vp) {
  SecState* s = nullptr;
  int rc = sec_state(ctx, &s);
  if (rc) return rc;
  s->last = pf_secondary_stats{};
  return lifecycle(ctx, s, dt, gravity, Vp);
}

// storeEscapedParticles and emitSecondarySpray (sparse_sim3d_tp.cpp:192-218, 276-337)
int secondary_after_advect(pf_ctx* ctx, const int* esc_flags, double Vp, const pf_interface_stats& iface) {
  SecState* s = nullptr;
  int rc = sec_state(ctx, &s);
  if (rc) return rc;
  s->last.escaped_droplets_added = s->last.escaped_bubbles_added = 0;
  if (esc_flags && ctx->np > 0) {
    rc = store_escaped(ctx, s, esc_flags, Vp);
    if (rc) return rc;
  }
  return spray_step(ctx, s, Vp, iface);
}

void secondary_free(pf_ctx* ctx) {
  SecState* s = static_cast<SecState*>(ctx->secondary);
  if (!s) return;
  for (int t = 0; t < 2; ++t) {
    free_set(s->set[t]);
    free_set(s->tmp[t]);
    free_dev(s->outcome[t]);
    free_dev(s->keep_idx[t]);
    free_dev(s->reab_idx[t]);
    free_dev(s->esc_idx[t]);
  }
  free_dev(s->cflag);
  free_dev(s->score);
  free_dev(s->key);
  free_dev(s->key_sorted);
  free_dev(s->cand);
  free_dev(s->cand_sorted);
  free_dev(s->impact);
  free_dev(s->part);
  free_dev(s->cub_tmp);
  free_dev(s->d_ints);
  free_dev(s->d_sums);
  if (s->window) cudaFreeHost(s->window);
  if (s->h_ints) cudaFreeHost(s->h_ints);
  if (s->h_sums) cudaFreeHost(s->h_sums);
  delete s;
  ctx->secondary = nullptr;
}

int take_upload_for(pf_ctx* ctx);

}  // namespace pf

using namespace pf;

extern "C" {

int pf_secondary_default_cfg(pf_secondary_cfg* out) {
  if (!out) return PF_ERR_INVALID;
  default_cfg(out);
  return PF_OK;
}

int pf_set_secondary(pf_ctx* ctx, const pf_secondary_cfg* cfg) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  SecState* s = nullptr;
  const int rc = sec_state(ctx, &s);
  if (rc) return rc;
  if (cfg) {
    s->cfg = *cfg;
  } else {
    s->cfg.escaped_particle_branching = s->cfg.lifecycle = s->cfg.spray_emission = 0;
  }
  return PF_OK;
}

int pf_get_secondary_stats(const pf_ctx* ctx, pf_secondary_stats* out) {
  if (!ctx || !out) return PF_ERR_INVALID;
  const SecState* s = static_cast<const SecState*>(ctx->secondary);
  *out = s ? s->last : pf_secondary_stats{};
  return PF_OK;
}

int pf_secondary_count(const pf_ctx* ctx, int which, size_t* n) {
  if (!ctx || !n || which < 0 || which > 1) return PF_ERR_INVALID;
  const SecState* s = static_cast<const SecState*>(ctx->secondary);
  *n = s ? s->set[which].n : 0;
  return PF_OK;
}

int pf_get_secondary(pf_ctx* ctx, int which, double* pos, double* vel, double* vol, int* age) {
  if (!ctx || which < 0 || which > 1) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  SecState* s = static_cast<SecState*>(ctx->secondary);
  if (!s || s->set[which].n == 0) return PF_OK;
  const SecSet& set = s->set[which];
  const size_t n = set.n;
  std::vector<double> tmp(n);
  const double* src[6] = {set.x, set.y, set.z, set.vx, set.vy, set.vz};
  for (int a = 0; a < 6; ++a) {
    double* out = a < 3 ? pos : vel;
    if (!out) continue;
    PF_CUDA_TRY(cudaMemcpyAsync(tmp.data(), src[a], n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (size_t p = 0; p < n; ++p) out[3 * p + a % 3] = tmp[p];
  }
  if (vol) PF_CUDA_TRY(cudaMemcpyAsync(vol, set.vol, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
  if (age) PF_CUDA_TRY(cudaMemcpyAsync(age, set.age, n * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

int pf_set_secondary_particles(pf_ctx* ctx, int which, size_t n, const double* pos, const double* vel,
                               const double* vol, const int* age) {
  if (!ctx || which < 0 || which > 1 || (n && (!pos || !vel || !vol || !age))) return PF_ERR_INVALID;
  if (n > (size_t)0x7fffffff) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  SecState* s = nullptr;
  int rc = sec_state(ctx, &s);
  if (rc) return rc;
  SecSet& set = s->set[which];
  set.n = 0;
  rc = grow_set(ctx, set, n);
  if (rc) return rc;
  std::vector<double> tmp(n);
  double* dst[6] = {set.x, set.y, set.z, set.vx, set.vy, set.vz};
  for (int a = 0; a < 6 && n; ++a) {
    const double* in = a < 3 ? pos : vel;
    for (size_t p = 0; p < n; ++p) tmp[p] = in[3 * p + a % 3];
    PF_CUDA_TRY(cudaMemcpyAsync(dst[a], tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  }
  if (n) {
    PF_CUDA_TRY(cudaMemcpyAsync(set.vol, vol, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    PF_CUDA_TRY(cudaMemcpyAsync(set.age, age, n * sizeof(int), cudaMemcpyHostToDevice, ctx->stream));
  }
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  set.n = n;
  return PF_OK;
}

int pf_secondary_advance(pf_ctx* ctx, double dt, double gravity, double Vp) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int rc = take_upload_for(ctx);
  if (rc) return rc;
  return secondary_lifecycle(ctx, dt, gravity, Vp);
}

int pf_secondary_spray(pf_ctx* ctx, double Vp, const pf_interface_stats* iface) {
  if (!ctx || !iface) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  int rc = take_upload_for(ctx);
  if (rc) return rc;
  SecState* s = nullptr;
  rc = sec_state(ctx, &s);
  if (rc) return rc;
  s->last = pf_secondary_stats{};
  return spray_step(ctx, s, Vp, *iface);
}

}  // extern "C"
