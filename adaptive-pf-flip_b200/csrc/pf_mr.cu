// pf_mr.cu -- the reference's 2-level multires step (MRSim3DTP::step,
// src/driver/multires_sim3d_tp.cpp:671-733) on the GPU: dynamic refinement,
// markCells, P2G over leaf-cell face patches, gravity and walls, the
// finite-volume pressure system on the leaf cells with its Jacobi PCG
// (adaptive restart, optional flexible beta), the velocity update, G2P and
// RK2/RK3 advection.
//
// Layout.  The reference's MRLayout3D<4> (src/grid/multires_layout3d.h:25-162)
// holds level-1 blocks of 8^3 fine cells, each either a leaf (4^3 coarse cells
// of 2 dx) or split into eight level-0 blocks (4^3 fine cells).  Here that is
// one byte per level-1 block ("refined").  A fine cell (i, j, k) belongs to the
// fine leaf (i, j, k) in a refined block and to the coarse leaf
// (i & ~1, j & ~1, k & ~1) otherwise.
//
// Faces.  MRMacGrid3D (src/grid/multires_mac_grid3d.h:35-189) keeps one value
// per fine face patch on a leaf cell's boundary.  Here every face field is a
// dense FP32 array over the fine face lattice; a patch at position `pos` along
// its axis is on a leaf boundary iff pos is even, pos is the domain's far side,
// or a fine cell beside it lies in a refined block.  Other patches are never
// written and read 0, as the reference's maps return 0 for absent keys.
//
// Markers and pressure are per fine cell (the leaf's value replicated), so a
// marker lookup at a fine cell is one load.
//
// Pressure.  The unknowns are the fluid leaf cells in the reference's
// leafCells order (level, block (bx, by, bz), cell (lz, ly, lx)); the order
// only decides the pinned cell.  Rows are CSR in FP64 with the off-diagonal
// terms in the reference's face-visit order (visitCellFaces,
// src/pressure/multires_pressure3d.cpp:102-137), so each row's products sum in
// the reference's order; the PCG's inner products are fixed-order block
// reductions (another order than the reference's sequential sums).
#include <algorithm>
#include <climits>
#include <cmath>
#include <vector>

#include "pf_solver.cuh"

namespace pf {
namespace {

constexpr int kMrNT = 256;
constexpr int kMrPoll = 16;        // PCG iterations launched between polls

struct MrGeom {
  int nx, ny, nz;
  double dx;
  double inv_dx;  // 1/dx
  int dx_pow2;    // dx is a power of two: x / dx == x * inv_dx exactly
  int MX, MY, MZ;      // level-1 blocks, ceil(n / 8)
  int BX0, BY0, BZ0;   // level-0 blocks, ceil(n / 4)
  const uint8_t* refined;
};

// PCG control block in device memory; done: 0 running, 1 converged,
// 2 breakdown, 3 iteration cap, 4 not run (non-finite initial residual)
struct MrCtl {
  double rz, alpha, beta, res, res0, prev, tol, growth;
  int it, max_iter, done, restarts, beta_resets, pin, adaptive, flexible, jacobi;
  unsigned counter;
};
enum { kMrInit = 0, kMrPAp = 1, kMrUpdate = 2 };

struct MrState {
  MrGeom g{};
  size_t nface[3] = {};
  size_t ncell = 0;
  size_t nkey0 = 0, nkey1 = 0;
  uint8_t* refined = nullptr;
  std::vector<uint8_t> h_refined;
  float* f[9] = {};      // u v w mu mv mw, the saved u v w
  float2* acc[3] = {};   // P2G scratch: (momentum, raw mass) per face
  uint8_t* mk = nullptr; // per fine cell
  float* pcell = nullptr;
  int* cell_idx = nullptr;
  int *flag0 = nullptr, *pos0 = nullptr, *flag1 = nullptr, *pos1 = nullptr;
  int4* cells = nullptr;  // fluid leaf cells: fine origin and level
  int* row_len = nullptr;    // off-diagonal terms per row
  int* slice_len = nullptr;  // entries per 32-row slice (32 x its longest row)
  int* slice_ptr = nullptr;  // exclusive scan of slice_len
  int* col = nullptr;
  double* coef = nullptr;
  size_t nnz_cap = 0;
  int* minmax = nullptr;   // 12 ints
  int* counters = nullptr; // 8 clamp counters + pin probe
  MrCtl* ctl = nullptr;
  MrCtl* h_ctl = nullptr;
  int* h_ints = nullptr;   // pinned read-backs
  double* partials = nullptr;
  pf_mr_dynamic dyn{1, 1, 2, 1, 0};
  int retained_valid = 0, rbox[6] = {};
  int last_fine_leaves = 0, budget_limited = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
};

// ---- lattice helpers ----------------------------------------------------

// x / dx, as a product where that is exact
__device__ __forceinline__ double mr_grid(const MrGeom& g, double x) { return g.dx_pow2 ? x * g.inv_dx : x / g.dx; }

__device__ __forceinline__ bool mr_in(const MrGeom& g, int i, int j, int k) {
  return i >= 0 && i < g.nx && j >= 0 && j < g.ny && k >= 0 && k < g.nz;
}
__device__ __forceinline__ size_t mr_cell(const MrGeom& g, int i, int j, int k) {
  return (size_t)i + (size_t)g.nx * ((size_t)j + (size_t)g.ny * (size_t)k);
}
__device__ __forceinline__ size_t mr_face(const MrGeom& g, int axis, int i, int j, int k) {
  const size_t X = (size_t)g.nx + (axis == 0), Y = (size_t)g.ny + (axis == 1);
  return (size_t)i + X * ((size_t)j + Y * (size_t)k);
}
__device__ __forceinline__ bool mr_refined(const MrGeom& g, int i, int j, int k) {
  return g.refined[(i >> 3) + g.MX * ((j >> 3) + g.MY * (k >> 3))] != 0;
}
// level (0 or 1) of the leaf holding fine cell (i, j, k) and its origin
__device__ __forceinline__ int mr_leaf(const MrGeom& g, int i, int j, int k, int* o) {
  if (mr_refined(g, i, j, k)) {
    o[0] = i;
    o[1] = j;
    o[2] = k;
    return 0;
  }
  o[0] = i & ~1;
  o[1] = j & ~1;
  o[2] = k & ~1;
  return 1;
}
__device__ __forceinline__ int mr_marker(const MrGeom& g, const uint8_t* mk, int i, int j, int k) {
  return mr_in(g, i, j, k) ? (int)mk[mr_cell(g, i, j, k)] : 2;
}
// the patch (axis; c) in range is on a leaf cell's boundary (enumerateFaces,
// src/grid/multires_mac_grid3d.h:123-163): its position along the axis is
// even (a coarse leaf's side), the domain's far side, or beside a fine leaf
__device__ __forceinline__ bool mr_face_valid(const MrGeom& g, int axis, int i, int j, int k) {
  const int c[3] = {i, j, k};
  const int n = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
  const int pos = c[axis];
  if ((pos & 1) == 0 || pos == n) return true;
  int l[3] = {i, j, k};
  l[axis] = pos - 1;
  if (mr_refined(g, l[0], l[1], l[2])) return true;
  return pos < n && mr_refined(g, i, j, k);
}

// betaFromRawMass (src/pressure/multires_pressure3d.cpp:94-99)
struct MrPhase {
  double rho_l, rho_g, rmin, invden;
};
__device__ __forceinline__ double mr_beta(double raw, const MrPhase& P) {
  double phi;
  if (raw < P.rmin) {
    phi = 0.0;
  } else {
    const double s = sqrt((raw - P.rmin) * P.invden);
    phi = 1.0 < s ? 1.0 : s;
  }
  return 1.0 / (phi * P.rho_l + (1.0 - phi) * P.rho_g);
}

// ---- fixed-order reductions finished by the last CTA --------------------

__device__ __forceinline__ void block_sum3_max(double& a, double& b, double& c, double& m) {
  double z = 0.0;
  block_sum_max(a, m);
  __syncthreads();
  block_sum_max(b, z);
  __syncthreads();
  z = 0.0;
  block_sum_max(c, z);
}

__device__ void mr_finalize(MrCtl* ctl, int stage, double s0, double s1, double s2, double m) {
  switch (stage) {
    case kMrInit: {  // s0 = r.z, m = max|r0|
      ctl->res0 = m;
      ctl->res = m;
      ctl->prev = m;
      double tol = ctl->tol;  // holds max(abs, 0) on entry
      const double rel = ctl->beta;  // holds the relative tolerance on entry
      if (rel * m > tol) tol = rel * m;
      ctl->tol = tol;
      ctl->beta = 0.0;
      ctl->rz = s0;
      ctl->it = 0;
      if (!isfinite(m)) ctl->done = 4;  // no solve, neither converged nor broken down
      else if (!(m >= tol)) ctl->done = 1;
      else if (!isfinite(s0)) ctl->done = 2;
      else ctl->done = 0;
      break;
    }
    case kMrPAp: {  // s0 = p.Ap
      if (!isfinite(s0) || fabs(s0) < 1e-30) {
        ctl->done = 2;
        break;
      }
      const double alpha = ctl->rz / s0;
      if (!isfinite(alpha)) ctl->done = 2;
      else ctl->alpha = alpha;
      break;
    }
    case kMrUpdate: {  // s0 = r.z (new), s1 = r.(z - z_prev), s2 = non-finite count, m = max|r|
      ctl->it += 1;
      ctl->res = m;
      if (s2 > 0.0 || !isfinite(m)) {
        ctl->done = 2;
        break;
      }
      if (m < ctl->tol) {
        ctl->done = 1;
        break;
      }
      const bool restart = ctl->adaptive && ctl->growth > 0.0 && m > ctl->prev * ctl->growth &&
                           m > ctl->res0 * ctl->growth && ctl->it < ctl->max_iter;
      if (!isfinite(s0)) {
        ctl->done = 2;
        break;
      }
      double beta = 0.0;
      if (restart) {
        ctl->restarts += 1;
      } else if (ctl->rz != 0.0) {
        beta = ctl->flexible ? s1 / ctl->rz : s0 / ctl->rz;
        if (!isfinite(beta)) {
          beta = 0.0;
          ctl->beta_resets += 1;
        }
        if (beta < 0.0) {
          beta = 0.0;
          ctl->beta_resets += 1;
        }
      }
      ctl->beta = beta;
      ctl->rz = s0;
      ctl->prev = m;
      if (ctl->it >= ctl->max_iter) ctl->done = 3;
      break;
    }
  }
}

__device__ void mr_reduce(double s0, double s1, double s2, double m, double* partials, MrCtl* ctl, int stage) {
  __shared__ bool am_last;
  block_sum3_max(s0, s1, s2, m);
  if (threadIdx.x == 0) {
    partials[4 * blockIdx.x + 0] = s0;
    partials[4 * blockIdx.x + 1] = s1;
    partials[4 * blockIdx.x + 2] = s2;
    partials[4 * blockIdx.x + 3] = m;
    __threadfence();
    const unsigned t = atomicAdd(&ctl->counter, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  double a = 0.0, b = 0.0, c = 0.0, mm = 0.0;
  for (int q = threadIdx.x; q < (int)gridDim.x; q += blockDim.x) {
    a += __ldcg(&partials[4 * q + 0]);
    b += __ldcg(&partials[4 * q + 1]);
    c += __ldcg(&partials[4 * q + 2]);
    mm = fmax(mm, __ldcg(&partials[4 * q + 3]));
  }
  block_sum3_max(a, b, c, mm);
  if (threadIdx.x == 0) {
    mr_finalize(ctl, stage, a, b, c, mm);
    ctl->counter = 0;
  }
}

// ---- dynamic refinement: particle cell bounds ---------------------------

__global__ void k_mr_minmax_init(int* mm, int nx, int ny, int nz) {
  const int t = threadIdx.x;
  if (t < 12) {
    const int n[3] = {nx, ny, nz};
    mm[t] = (t % 6) < 3 ? n[t % 3] : -1;
  }
}

// min/max fine cell of all particles and of the gas particles
// (updateDynamicRefinement, src/driver/multires_sim3d_tp.cpp:577-623)
__global__ void __launch_bounds__(kMrNT) k_mr_bounds(MrGeom g, const float* px, const float* py, const float* pz,
                                                   const uint8_t* type, size_t n, int* mm) {
  __shared__ int s[12];
  if (threadIdx.x < 12) s[threadIdx.x] = (threadIdx.x % 6) < 3 ? INT_MAX : -1;
  __syncthreads();
  int lo[6] = {INT_MAX, INT_MAX, INT_MAX, INT_MAX, INT_MAX, INT_MAX}, hi[6] = {-1, -1, -1, -1, -1, -1};
  for (size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const double x = px[q], y = py[q], z = pz[q];
    if (!isfinite(x) || !isfinite(y) || !isfinite(z)) continue;
    const int c[3] = {(int)mr_grid(g, x), (int)mr_grid(g, y), (int)mr_grid(g, z)};
    if (!mr_in(g, c[0], c[1], c[2])) continue;
    const bool gas = type[q] == 1;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      lo[d] = min(lo[d], c[d]);
      hi[d] = max(hi[d], c[d]);
      if (gas) {
        lo[3 + d] = min(lo[3 + d], c[d]);
        hi[3 + d] = max(hi[3 + d], c[d]);
      }
    }
  }
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    atomicMin(&s[(d / 3) * 6 + d % 3], lo[d]);
    atomicMax(&s[(d / 3) * 6 + 3 + d % 3], hi[d]);
  }
  __syncthreads();
  if (threadIdx.x < 12) {
    if ((threadIdx.x % 6) < 3) atomicMin(&mm[threadIdx.x], s[threadIdx.x]);
    else atomicMax(&mm[threadIdx.x], s[threadIdx.x]);
  }
}

// ---- markCells (src/driver/multires_sim3d_tp.cpp:40-73) ------------------

// walls: a leaf holding a domain-boundary fine cell is solid, all else empty
__global__ void k_mr_mark_walls(MrGeom g, uint8_t* mk) {
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % g.nx), j = (int)((e / g.nx) % g.ny), k = (int)(e / ((size_t)g.nx * g.ny));
    int o[3];
    const int s = 1 << mr_leaf(g, i, j, k, o);
    const bool wall = o[0] == 0 || o[0] + s >= g.nx || o[1] == 0 || o[1] + s >= g.ny || o[2] == 0 ||
                      o[2] + s >= g.nz;
    mk[e] = wall ? 2 : 0;
  }
}

// particles: the leaf of each particle's fine cell becomes fluid unless solid
__global__ void k_mr_mark_particles(MrGeom g, const float* px, const float* py, const float* pz, size_t n,
                                    uint8_t* mk) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const int i = (int)mr_grid(g, (double)px[q]), j = (int)mr_grid(g, (double)py[q]), k = (int)mr_grid(g, (double)pz[q]);
  if (!mr_in(g, i, j, k) || mk[mr_cell(g, i, j, k)] == 2) return;
  int o[3];
  const int s = 1 << mr_leaf(g, i, j, k, o);
  for (int z = o[2]; z < o[2] + s && z < g.nz; ++z)
    for (int y = o[1]; y < o[1] + s && y < g.ny; ++y)
      for (int x = o[0]; x < o[0] + s && x < g.nx; ++x) mk[mr_cell(g, x, y, z)] = 1;
}

// ---- P2G (src/driver/multires_ops3d_tp.cpp:20-130, 209-274) --------------


struct MrFaces {
  float* f[9];
};

// P2G: one thread per particle (memory order), the momentum and raw mass of
// a patch added together by one vector atomic into an interleaved scratch
// lattice; k_mr_split then writes u = momentum / mass (where mass > 0) and
// the mass.  Accumulation order is the atomics' (not the reference's
// particle order).
// One particle's splat onto the leaf-boundary patches of face axis AX within
// the kernel radius (collectWeightedFaces: every lattice patch with |d| < 1.5
// per axis, at most 3 per axis, in (k, j, i) order over clamped ranges),
// normalised by their sum.  The squared distance splits per axis, so each of
// the 27 weights costs two adds and the cubic in FP32 (the reference's FP64
// weights to within FP32 rounding); they are held in registers between the
// sum and the splat.  Patch validity is tested per patch only where the
// candidates' cells straddle both levels.  Momentum and raw mass of a patch
// go out in one vector atomic.
template <int AX>
__device__ __forceinline__ void mr_p2g_axis(const MrGeom& g, double px, double py, double pz, float mp, float v,
                                            float2* acc) {
  const double c[3] = {px, py, pz};
  const int n[3] = {g.nx, g.ny, g.nz};
  int p0[3], cnt[3];
  float e[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double s = d == AX ? c[d] : c[d] - 0.5;
    const int top = d == AX ? n[d] : n[d] - 1;
    const int first = (int)floor(s - 1.5) + 1;
    const int lo = max(first, 0), hi = min(first + 2, top);
    p0[d] = lo;
    cnt[d] = max(0, hi - lo + 1);
    e[d] = (float)(s - (double)lo);
  }
  if (cnt[0] == 0 || cnt[1] == 0 || cnt[2] == 0) return;
  int mode;  // 0 all refined, 1 all coarse, 2 mixed
  {
    int cl[3], ch[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      cl[d] = max(0, p0[d] - (d == AX ? 1 : 0));
      ch[d] = min(n[d] - 1, p0[d] + cnt[d] - 1);
    }
    int nref = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) nref += mr_refined(g, q & 1 ? ch[0] : cl[0], q & 2 ? ch[1] : cl[1], q & 4 ? ch[2] : cl[2]);
    mode = nref == 8 ? 0 : nref == 0 ? 1 : 2;
  }
  const int na = n[AX];
  float w[27];
  float wsum = 0.0f;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float dz = e[2] - (float)k;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const float dy = e[1] - (float)j;
      const float dyz = dy * dy + dz * dz;
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        float ww = 0.0f;
        if (i < cnt[0] && j < cnt[1] && k < cnt[2]) {
          const float dx = e[0] - (float)i;
          const float t = 1.0f - (dx * dx + dyz) * (1.0f / 2.25f);
          if (t > 0.0f) {
            bool ok = true;
            if (mode != 0) {
              const int pos = AX == 0 ? p0[0] + i : AX == 1 ? p0[1] + j : p0[2] + k;
              const bool edge = (pos & 1) == 0 || pos == na;
              ok = edge || (mode == 2 && mr_face_valid(g, AX, p0[0] + i, p0[1] + j, p0[2] + k));
            }
            if (ok) {
              ww = t * t * t;
              wsum += ww;
            }
          }
        }
        w[i + 3 * j + 9 * k] = ww;
      }
    }
  }
  if (!(wsum > 0.0f)) return;
  const float inv = 1.0f / wsum;
  const size_t X = (size_t)g.nx + (AX == 0), Y = (size_t)g.ny + (AX == 1);
  float2* base = acc + mr_face(g, AX, p0[0], p0[1], p0[2]);
#pragma unroll
  for (int k = 0; k < 3; ++k)
#pragma unroll
    for (int j = 0; j < 3; ++j)
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const float ww = w[i + 3 * j + 9 * k];
        if (ww > 0.0f) {
          const float wn = ww * inv;
          atomicAdd(base + (i + X * (j + Y * k)), make_float2(wn * mp * v, wn * mp));
        }
      }
}

__global__ void __launch_bounds__(kMrNT) k_mr_p2g(MrGeom g, const float* px, const float* py, const float* pz,
                                                const float* vx, const float* vy, const float* vz, const float* vol,
                                                const uint8_t* type, size_t n, double mpl, double mpg, float2* acc0,
                                                float2* acc1, float2* acc2) {
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= n) return;
  const float mp = (float)((type[q] == 0 ? mpl : mpg) * (double)vol[q]);
  const double x = mr_grid(g, (double)px[q]), y = mr_grid(g, (double)py[q]), z = mr_grid(g, (double)pz[q]);
  mr_p2g_axis<0>(g, x, y, z, mp, vx[q], acc0);
  mr_p2g_axis<1>(g, x, y, z, mp, vy[q], acc1);
  mr_p2g_axis<2>(g, x, y, z, mp, vz[q], acc2);
}

// u = momentum / mass where the mass is positive (else the momentum, 0), mass
__global__ void k_mr_split(const float2* __restrict__ acc, float* u, float* mass, size_t n) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    const float2 a = acc[e];
    mass[e] = a.y;
    u[e] = a.y > 0.0f ? a.x / a.y : a.x;
  }
}

// applyGravity and applyWallBoundary (src/driver/multires_sim3d_tp.cpp:75-99)
// on one axis's lattice.  Patches off the face list hold 0 and no mass, so
// neither pass changes them.
__global__ void k_mr_forces(MrGeom g, int axis, float* u, const float* mass, float dv) {
  const int X = g.nx + (axis == 0), Y = g.ny + (axis == 1), Z = g.nz + (axis == 2);
  const int n = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
  const size_t tot = (size_t)X * Y * Z;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % X), j = (int)((e / X) % Y), k = (int)(e / ((size_t)X * Y));
    const int c = axis == 0 ? i : axis == 1 ? j : k;
    float v = u[e];
    if (axis == 1 && mass[e] > 0.0f) v = v + dv;
    if (c == 0 || c == 1 || c == n - 1 || c == n) v = 0.0f;
    u[e] = v;
  }
}

// ---- projection (src/pressure/multires_pressure3d.cpp:749-1527) ----------

// fluid flags over the leafCells key spaces: level-0 keys
// ((bx BY0 + by) BZ0 + bz) 64 + (lz 16 + ly 4 + lx), level-1 keys
// ((bx MY + by) MZ + bz) 64 + (lz 16 + ly 4 + lx)
__device__ __forceinline__ void mr_key0(const MrGeom& g, size_t key, int* c) {
  const int l = (int)(key & 63);
  size_t b = key >> 6;
  const int bz = (int)(b % g.BZ0);
  b /= g.BZ0;
  const int by = (int)(b % g.BY0), bx = (int)(b / g.BY0);
  c[0] = 4 * bx + (l & 3);
  c[1] = 4 * by + ((l >> 2) & 3);
  c[2] = 4 * bz + (l >> 4);
}
__device__ __forceinline__ void mr_key1(const MrGeom& g, size_t key, int* c) {
  const int l = (int)(key & 63);
  size_t b = key >> 6;
  const int bz = (int)(b % g.MZ);
  b /= g.MZ;
  const int by = (int)(b % g.MY), bx = (int)(b / g.MY);
  c[0] = 8 * bx + 2 * (l & 3);
  c[1] = 8 * by + 2 * ((l >> 2) & 3);
  c[2] = 8 * bz + 2 * (l >> 4);
}

__global__ void k_mr_flags(MrGeom g, const uint8_t* mk, int level, size_t nkey, int* flag) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nkey; e += (size_t)gridDim.x * blockDim.x) {
    int c[3];
    if (level == 0) mr_key0(g, e, c);
    else mr_key1(g, e, c);
    int ok = 0;
    if (mr_in(g, c[0], c[1], c[2]) && mr_refined(g, c[0], c[1], c[2]) == (level == 0))
      ok = mk[mr_cell(g, c[0], c[1], c[2])] == 1;
    flag[e] = ok;
  }
}

// the fluid cells' origins and levels; their fine cells' row index
__global__ void k_mr_cells(MrGeom g, int level, size_t nkey, const int* flag, const int* pos, const int* base,
                           int4* cells, int* cell_idx) {
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < nkey; e += (size_t)gridDim.x * blockDim.x) {
    if (!flag[e]) continue;
    int c[3];
    if (level == 0) mr_key0(g, e, c);
    else mr_key1(g, e, c);
    const int row = pos[e] + (base ? *base : 0);
    cells[row] = make_int4(c[0], c[1], c[2], level);
    const int s = 1 << level;
    for (int z = c[2]; z < c[2] + s && z < g.nz; ++z)
      for (int y = c[1]; y < c[1] + s && y < g.ny; ++y)
        for (int x = c[0]; x < c[0] + s && x < g.nx; ++x) cell_idx[mr_cell(g, x, y, z)] = row;
  }
}

// visitCellFaces (:102-137): the fine patches on a leaf's boundary in the
// reference's order, each with the fine neighbour across it and the outward
// sign.  fn(axis, face, neighbour, sign).
template <class Fn>
__device__ __forceinline__ void mr_visit(const MrGeom& g, int4 c, Fn&& fn) {
  const int s = 1 << c.w;
  const int x0 = c.x, y0 = c.y, z0 = c.z, x1 = x0 + s, y1 = y0 + s, z1 = z0 + s;
  const int cx1 = min(g.nx, x1), cy1 = min(g.ny, y1), cz1 = min(g.nz, z1);
  for (int z = z0; z < cz1; ++z)
    for (int y = y0; y < cy1; ++y) {
      fn(0, x0, y, z, x0 - 1, y, z, -1.0);
      fn(0, min(x1, g.nx), y, z, x1, y, z, 1.0);
    }
  for (int z = z0; z < cz1; ++z)
    for (int x = x0; x < cx1; ++x) {
      fn(1, x, y0, z, x, y0 - 1, z, -1.0);
      fn(1, x, min(y1, g.ny), z, x, y1, z, 1.0);
    }
  for (int y = y0; y < cy1; ++y)
    for (int x = x0; x < cx1; ++x) {
      fn(2, x, y, z0, x, y, z0 - 1, -1.0);
      fn(2, x, y, min(z1, g.nz), x, y, z1, 1.0);
    }
}

// findPinCell (:190-200): does any fluid cell see an empty (Dirichlet) cell?
__global__ void k_mr_pin_probe(MrGeom g, const uint8_t* mk, const int4* cells, int N, int* air) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    bool found = false;
    mr_visit(g, cells[r], [&](int, int, int, int, int ni, int nj, int nk, double) {
      if (mr_marker(g, mk, ni, nj, nk) == 0) found = true;
    });
    if (found) atomicOr(air, 1);
  }
}

__device__ __forceinline__ int mr_pin(const int* air, int N) { return (*air || N == 0) ? -1 : 0; }

// the most face patches a leaf visits: 6 faces of a 2x2-patch coarse leaf
constexpr int kMrMaxPatches = 24;

// The row builders keep a row's distinct columns in a local array and search
// it below its running count, which the front end cannot tell apart from a
// read of unset entries (diagnostic 549).
#pragma nv_diag_suppress 549

// off-diagonal terms of each row: one per distinct neighbour leaf
__global__ void k_mr_row_count(MrGeom g, const uint8_t* mk, const int4* cells, const int* cell_idx, int N,
                               const int* air, int* row_len) {
  const int pin = mr_pin(air, N);
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    int cols[kMrMaxPatches];
    int n = 0;
    if (r != pin)
      mr_visit(g, cells[r], [&](int, int, int, int, int ni, int nj, int nk, double) {
        if (mr_marker(g, mk, ni, nj, nk) == 2) return;
        const int o = cell_idx[mr_cell(g, ni, nj, nk)];  // marker < 2: in the domain
        if (o < 0 || o == pin) return;
        int q = 0;
        while (q < n && cols[q] != o) ++q;
        if (q == n && n < kMrMaxPatches) cols[n++] = o;
      });
    row_len[r] = n;
  }
}

// The rows are stored as 32-row slices (sliced ELLPACK): term t of row r is
// entry slice_ptr[r / 32] + 32 t + r % 32, so a warp's 32 rows load each term
// position together; a slice is as wide as its longest row and shorter rows
// end in (col = r, coef = 0) terms, which add an exact zero.  A row holds one
// term per neighbour leaf, in the order the reference's visit first meets it;
// the patches a coarse face shares with one coarse neighbour (up to 4) are
// summed into that term in visit order.  The reference keeps one term per
// patch; merging them regroups the row's sum (the operator is the same up to
// rounding, and stays symmetric: both rows of a pair visit their shared
// patches in the same order) and cuts a coarse row from 24 stored terms to 6.
__global__ void k_mr_slices(int N, const int* row_len, int* slice_len) {
  const int nslice = (N + 31) / 32;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s <= nslice; s += gridDim.x * blockDim.x) {
    int w = 0;
    if (s < nslice)
      for (int r = 32 * s; r < min(N, 32 * s + 32); ++r) w = max(w, row_len[r]);
    slice_len[s] = 32 * w;
  }
}

struct MrVecs {
  double *x, *r, *z, *p, *Ap, *diag;
};

// rows (:788-822): diagonal, off-diagonal terms and right-hand side; then
// x = 0, r = b, z = M^-1 r, p = 0 (the first direction is z), and r.z,
// max|r| -> tolerance
__global__ void __launch_bounds__(kMrNT) k_mr_rows(MrGeom g, const uint8_t* mk, const int4* cells,
                                                 const int* cell_idx, int N, const int* air, MrFaces F, MrPhase P,
                                                 double dt, double c_div, const int* slice_ptr, int* col,
                                                 double* coef, MrVecs V, MrCtl* ctl, double* partials) {
  const int pin = mr_pin(air, N);
  const double area = g.dx * g.dx * 1.0 * 1.0;
  const int jacobi = ctl->jacobi;
  double rz = 0.0, rmax = 0.0;
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    const int4 c = cells[r];
    const double h = g.dx * (double)(1 << c.w);
    const double vol = h * h * h;
    double diag = 0.0, div = 0.0;
    const int base = slice_ptr[r >> 5] + (r & 31);
    const int width = (slice_ptr[(r >> 5) + 1] - slice_ptr[r >> 5]) >> 5;
    int t = 0;
    int cols[kMrMaxPatches];
    double cfs[kMrMaxPatches];
    if (r == pin) {
      diag = 1.0;
    } else {
      mr_visit(g, c, [&](int axis, int fi, int fj, int fk, int ni, int nj, int nk, double sign) {
        const int m = mr_marker(g, mk, ni, nj, nk);
        if (m == 2) return;
        // neighborDistance (:214-225) and projectionCoefficient (:233-244)
        double other = h;
        if (mr_in(g, ni, nj, nk)) {
          int o[3];
          other = g.dx * (double)(1 << mr_leaf(g, ni, nj, nk, o));
        }
        const double dist = 0.5 * h + 0.5 * other;
        const size_t f = mr_face(g, axis, fi, fj, fk);
        double coeff = 0.0;
        if (!(dist <= 0.0 || vol <= 0.0)) coeff = dt * mr_beta((double)F.f[3 + axis][f], P) * area / dist / vol;
        diag += coeff;
        const int o = mr_in(g, ni, nj, nk) ? cell_idx[mr_cell(g, ni, nj, nk)] : -1;
        if (o >= 0 && o != pin) {
          int q = 0;
          while (q < t && cols[q] != o) ++q;
          if (q < t) {
            cfs[q] += coeff;
          } else if (t < kMrMaxPatches) {
            cols[t] = o;
            cfs[t] = coeff;
            ++t;
          }
        }
        div += sign * (double)F.f[axis][f] * area / vol;
      });
      for (int q = 0; q < t; ++q) {
        col[base + 32 * q] = cols[q];
        coef[base + 32 * q] = cfs[q];
      }
    }
    for (; t < width; ++t) {
      col[base + 32 * t] = r;
      coef[base + 32 * t] = 0.0;
    }
    const double b = r == pin ? 0.0 : -div + c_div;
    V.diag[r] = diag;
    V.x[r] = 0.0;
    V.r[r] = b;
    const double z = (jacobi && diag > 0.0) ? b / diag : b;
    V.z[r] = z;
    V.p[r] = 0.0;
    rz += b * z;
    rmax = fmax(rmax, fabs(b));
  }
  mr_reduce(rz, 0.0, 0.0, rmax, partials, ctl, kMrInit);
}

// The direction p = z + beta p_prev (the previous iteration's update, or a
// restart's beta = 0) formed where it is used, Ap (applyA, :824-838) and
// p.Ap -> alpha.  p_prev and p are separate buffers, alternated by the host.
#pragma nv_diag_default 549

// Two rows per thread and pass (rows r and r + stride, in that order, so the
// p.Ap partial keeps the one-row order): the slice offsets, the column and
// coefficient loads and the neighbour gathers of both rows go out together,
// so a row's three dependent rounds of memory latency overlap the other's.
constexpr int kMrSpmvRows = 2;
__global__ void __launch_bounds__(kMrNT) k_mr_spmv(int N, const int* __restrict__ slice_ptr,
                                                 const int* __restrict__ col, const double* __restrict__ coef,
                                                 const double* __restrict__ z, const double* __restrict__ p_prev,
                                                 double* p, double* Ap, const double* __restrict__ diag, MrCtl* ctl,
                                                 double* partials, const int* air) {
  pdl_wait();
  pdl_launch_dependents();
  if (ctl->done) return;
  const int pin = mr_pin(air, N);
  const double beta = ctl->beta;
  const int stride = gridDim.x * blockDim.x;
  double pap = 0.0;
  for (int r0 = blockIdx.x * blockDim.x + threadIdx.x; r0 < N; r0 += kMrSpmvRows * stride) {
    int rr[kMrSpmvRows], b0[kMrSpmvRows], w[kMrSpmvRows];
    double zr[kMrSpmvRows], pq[kMrSpmvRows], dg[kMrSpmvRows], off[kMrSpmvRows];
#pragma unroll
    for (int k = 0; k < kMrSpmvRows; ++k) {
      const int r = r0 + k * stride;
      rr[k] = r;
      w[k] = 0;
      b0[k] = 0;
      off[k] = 0.0;
      if (r < N) {
        zr[k] = z[r];
        pq[k] = p_prev[r];
        dg[k] = diag[r];
        const int s = r >> 5;
        const int a = slice_ptr[s];
        b0[k] = a + (r & 31);
        w[k] = r == pin ? 0 : (slice_ptr[s + 1] - a) >> 5;
      }
    }
    int wmax = 0;
#pragma unroll
    for (int k = 0; k < kMrSpmvRows; ++k) wmax = max(wmax, w[k]);
    // the loads of four terms per row go out together; each row's sum keeps its term order
    for (int t = 0; t < wmax; t += 4) {
      int cc[kMrSpmvRows][4];
      double cf[kMrSpmvRows][4], pv[kMrSpmvRows][4];
#pragma unroll
      for (int k = 0; k < kMrSpmvRows; ++k)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const bool in = t + u < w[k];
          cc[k][u] = in ? col[b0[k] + 32 * (t + u)] : -1;
          cf[k][u] = in ? coef[b0[k] + 32 * (t + u)] : 0.0;
        }
#pragma unroll
      for (int k = 0; k < kMrSpmvRows; ++k)
#pragma unroll
        for (int u = 0; u < 4; ++u) pv[k][u] = cc[k][u] >= 0 ? z[cc[k][u]] + beta * p_prev[cc[k][u]] : 0.0;
#pragma unroll
      for (int k = 0; k < kMrSpmvRows; ++k)
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (t + u < w[k]) off[k] += cf[k][u] * pv[k][u];
    }
#pragma unroll
    for (int k = 0; k < kMrSpmvRows; ++k) {
      const int r = rr[k];
      if (r >= N) continue;
      const double pr = zr[k] + beta * pq[k];
      const double ap = r == pin ? pr : dg[k] * pr - off[k];
      p[r] = pr;
      Ap[r] = ap;
      pap += pr * ap;
    }
  }
  mr_reduce(pap, 0.0, 0.0, 0.0, partials, ctl, kMrPAp);
}

// x += alpha p, r -= alpha Ap, z = M^-1 r; r.z, r.(z - z_prev), max|r|.
// A thread takes kMrRows rows per pass and issues all their loads before its
// first store, so their memory latencies overlap (the vectors may alias as
// far as the compiler knows, which would otherwise order every load of a row
// after the previous row's stores).
constexpr int kMrRows = 4;
__global__ void __launch_bounds__(kMrNT) k_mr_update(int N, MrVecs V, MrCtl* ctl, double* partials) {
  pdl_wait();
  pdl_launch_dependents();
  if (ctl->done) return;
  const double alpha = ctl->alpha;
  const int jacobi = ctl->jacobi, flexible = ctl->flexible;
  const int stride = gridDim.x * blockDim.x;
  double rz = 0.0, num = 0.0, bad = 0.0, rmax = 0.0;
  for (int r0 = blockIdx.x * blockDim.x + threadIdx.x; r0 < N; r0 += kMrRows * stride) {
    double x[kMrRows], p[kMrRows], rr[kMrRows], ap[kMrRows], d[kMrRows], zp[kMrRows];
#pragma unroll
    for (int k = 0; k < kMrRows; ++k) {
      const int r = r0 + k * stride;
      if (r < N) {
        x[k] = V.x[r];
        p[k] = V.p[r];
        rr[k] = V.r[r];
        ap[k] = V.Ap[r];
        d[k] = V.diag[r];
        zp[k] = V.z[r];
      }
    }
#pragma unroll
    for (int k = 0; k < kMrRows; ++k) {
      const int r = r0 + k * stride;
      if (r >= N) continue;
      const double xn = x[k] + alpha * p[k];
      const double rn = rr[k] - alpha * ap[k];
      V.x[r] = xn;
      V.r[r] = rn;
      if (!isfinite(xn) || !isfinite(rn)) bad += 1.0;
      if (isfinite(rn)) rmax = fmax(rmax, fabs(rn));
      const double z = (jacobi && d[k] > 0.0) ? rn / d[k] : rn;
      V.z[r] = z;
      rz += rn * z;
      if (flexible) num += rn * (z - zp[k]);
    }
  }
  mr_reduce(rz, num, bad, rmax, partials, ctl, kMrUpdate);
}

__global__ void k_mr_ctl_init(MrCtl* ctl, int max_iter, double abs_tol, double rel_tol, int jacobi, int flexible,
                              int adaptive, double growth) {
  *ctl = MrCtl{};
  ctl->max_iter = max_iter;
  ctl->tol = abs_tol > 0.0 ? abs_tol : 0.0;
  ctl->beta = rel_tol > 0.0 ? rel_tol : 0.0;  // read by the kMrInit stage
  ctl->jacobi = jacobi;
  ctl->flexible = flexible;
  ctl->adaptive = adaptive;
  ctl->growth = growth;
}

// g.p per leaf cell
__global__ void k_mr_pressure(MrGeom g, const int4* cells, int N, const double* x, float* pcell) {
  for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < N; r += gridDim.x * blockDim.x) {
    const int4 c = cells[r];
    const int s = 1 << c.w;
    const float v = (float)x[r];
    for (int z = c.z; z < c.z + s && z < g.nz; ++z)
      for (int y = c.y; y < c.y + s && y < g.ny; ++y)
        for (int xx = c.x; xx < c.x + s && xx < g.nx; ++xx) pcell[mr_cell(g, xx, y, z)] = v;
  }
}

// the velocity update (:1454-1524) on one axis's lattice
__global__ void k_mr_velocity(MrGeom g, int axis, const uint8_t* mk, const int* cell_idx, const int4* cells,
                              const double* x, float* u, const float* mass, MrPhase P, double dt) {
  const int X = g.nx + (axis == 0), Y = g.ny + (axis == 1), Z = g.nz + (axis == 2);
  const size_t tot = (size_t)X * Y * Z;
  for (size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (size_t)gridDim.x * blockDim.x) {
    const int i = (int)(e % X), j = (int)((e / X) % Y), k = (int)(e / ((size_t)X * Y));
    const int li = i - (axis == 0), lj = j - (axis == 1), lk = k - (axis == 2);
    const int lm = mr_marker(g, mk, li, lj, lk), rm = mr_marker(g, mk, i, j, k);
    const bool lf = lm == 1, rf = rm == 1;
    if (!lf && !rf) continue;
    if (!mr_face_valid(g, axis, i, j, k)) continue;
    if (lm == 2 || rm == 2) {
      u[e] = 0.0f;
      continue;
    }
    // neighborDistance from the fluid cell on the reference side
    const int ri = lf ? li : i, rj = lf ? lj : j, rk = lf ? lk : k;
    const int oi = lf ? i : li, oj = lf ? j : lj, ok = lf ? k : lk;
    const int ref = cell_idx[mr_cell(g, ri, rj, rk)];
    double dist = g.dx;
    if (ref >= 0) {
      const double h = g.dx * (double)(1 << cells[ref].w);
      double other = h;
      if (mr_in(g, oi, oj, ok)) {
        int o[3];
        other = g.dx * (double)(1 << mr_leaf(g, oi, oj, ok, o));
      }
      dist = 0.5 * h + 0.5 * other;
    }
    double pl = 0.0, pr = 0.0;
    if (lf) {
      const int a = cell_idx[mr_cell(g, li, lj, lk)];
      pl = a >= 0 ? x[a] : 0.0;
    }
    if (rf) {
      const int b = cell_idx[mr_cell(g, i, j, k)];
      pr = b >= 0 ? x[b] : 0.0;
    }
    const double beta = mr_beta((double)mass[e], P);
    u[e] = (float)((double)u[e] - dt * beta * (pr - pl) / dist);
  }
}

// ---- G2P and advection (src/driver/multires_ops3d_tp.cpp:132-207, 276-355)

// sampleU / sampleV / sampleW: clamped trilinear over the fine face lattice
__device__ __forceinline__ double mr_sample(const MrGeom& g, const float* __restrict__ f, int axis, double x, double y,
                                            double z) {
  const double p[3] = {mr_grid(g, x), mr_grid(g, y), mr_grid(g, z)};
  int b[3];
  double fr[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double s = d == axis ? p[d] : p[d] - 0.5;
    b[d] = (int)floor(s);
    fr[d] = s - b[d];
  }
  const int top[3] = {g.nx - (axis != 0), g.ny - (axis != 1), g.nz - (axis != 2)};
  double s = 0.0;
#pragma unroll
  for (int dz = 0; dz < 2; ++dz) {
    const double wz = dz == 0 ? 1.0 - fr[2] : fr[2];
    const int k = max(0, min(top[2], b[2] + dz));
#pragma unroll
    for (int dy = 0; dy < 2; ++dy) {
      const double wy = dy == 0 ? 1.0 - fr[1] : fr[1];
      const int j = max(0, min(top[1], b[1] + dy));
#pragma unroll
      for (int dx = 0; dx < 2; ++dx) {
        const double wx = dx == 0 ? 1.0 - fr[0] : fr[0];
        const int i = max(0, min(top[0], b[0] + dx));
        s += wx * wy * wz * (double)__ldg(f + mr_face(g, axis, i, j, k));
      }
    }
  }
  return s;
}

__global__ void __launch_bounds__(kMrNT) k_mr_g2p_advect(MrGeom g, MrFaces F, float* px, float* py, float* pz,
                                                       float* vx, float* vy, float* vz, const uint8_t* type, size_t n,
                                                       double aL, double aG, double dt, int order, int* counters) {
  __shared__ int tally[8];
  if (threadIdx.x < 8) tally[threadIdx.x] = 0;
  __syncthreads();
  const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned cnt[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (q < n) {
    const double x0[3] = {(double)px[q], (double)py[q], (double)pz[q]};
    const double a = type[q] == 0 ? aL : aG;
    double k1[3];
    float* vp[3] = {vx, vy, vz};
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) k1[ax] = mr_sample(g, F.f[ax], ax, x0[0], x0[1], x0[2]);
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
      const double d = k1[ax] - mr_sample(g, F.f[6 + ax], ax, x0[0], x0[1], x0[2]);
      const double flip = (double)vp[ax][q] + d;
      vp[ax][q] = (float)(a * flip + (1.0 - a) * k1[ax]);
    }
    double k2[3], nx[3];
    if (order == 3) {
      double m1[3], m2[3], k3[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) m1[c] = x0[c] + k1[c] * (0.5 * dt);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) k2[ax] = mr_sample(g, F.f[ax], ax, m1[0], m1[1], m1[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) m2[c] = x0[c] - k1[c] * dt + k2[c] * (2.0 * dt);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) k3[ax] = mr_sample(g, F.f[ax], ax, m2[0], m2[1], m2[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) nx[c] = x0[c] + (k1[c] + k2[c] * 4.0 + k3[c]) * (dt / 6.0);
    } else {
      double mid[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) mid[c] = x0[c] + k1[c] * (0.5 * dt);
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) k2[ax] = mr_sample(g, F.f[ax], ax, mid[0], mid[1], mid[2]);
#pragma unroll
      for (int c = 0; c < 3; ++c) nx[c] = x0[c] + k2[c] * dt;
    }
    const int nn[3] = {g.nx, g.ny, g.nz};
    float* pp[3] = {px, py, pz};
    bool any = false;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const double lo = 0.5 * g.dx, hi = ((double)nn[c] - 0.5) * g.dx;
      const bool l = nx[c] < lo, h = nx[c] > hi;
      cnt[2 + 2 * c] += l;
      cnt[3 + 2 * c] += h;
      any = any || l || h;
      pp[c][q] = (float)fmax(lo, fmin(hi, nx[c]));
    }
    // ParticleEscapeStats3D::recordClamp: only the two phases are counted
    if (type[q] == 0) cnt[0] += any;
    else if (type[q] == 1) cnt[1] += any;
  }
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const unsigned w = __reduce_add_sync(0xffffffffu, cnt[c]);
    if ((threadIdx.x & 31) == 0 && w) atomicAdd(&tally[c], (int)w);
  }
  __syncthreads();
  if (threadIdx.x < 8 && tally[threadIdx.x]) atomicAdd(&counters[threadIdx.x], tally[threadIdx.x]);
}

// ---- host side ------------------------------------------------------------

int grid_for(size_t n, int cap) {
  const size_t b = (n + kMrNT - 1) / kMrNT;
  return (int)std::max<size_t>(1, std::min<size_t>(b, (size_t)cap));
}

int mr_state(pf_ctx* ctx, MrState** out) {
  MrState* s = static_cast<MrState*>(ctx->mr);
  if (s) {
    *out = s;
    return PF_OK;
  }
  s = new MrState();
  ctx->mr = s;
  const Geom& G = ctx->g;
  if (G.ox != 0.0 || G.oy != 0.0 || G.oz != 0.0)
    return set_error(ctx, PF_ERR_INVALID, "multires: the grid origin must be 0 (MRLayout3D has none)");
  MrGeom& g = s->g;
  g.nx = G.nx;
  g.ny = G.ny;
  g.nz = G.nz;
  g.dx = G.dx;
  g.inv_dx = G.inv_dx;
  g.dx_pow2 = G.dx_pow2;
  g.MX = (g.nx + 7) / 8;
  g.MY = (g.ny + 7) / 8;
  g.MZ = (g.nz + 7) / 8;
  g.BX0 = (g.nx + 3) / 4;
  g.BY0 = (g.ny + 3) / 4;
  g.BZ0 = (g.nz + 3) / 4;
  const size_t nblk = (size_t)g.MX * g.MY * g.MZ;
  s->ncell = (size_t)g.nx * g.ny * g.nz;
  s->nkey0 = (size_t)g.BX0 * g.BY0 * g.BZ0 * 64;
  s->nkey1 = nblk * 64;
  if (s->ncell > (size_t)INT_MAX / 2 || s->nkey0 > ctx->cells_cap + 1)
    return set_error(ctx, PF_ERR_INVALID, "multires: grid too large for this context");
  for (int a = 0; a < 3; ++a)
    s->nface[a] = (size_t)(g.nx + (a == 0)) * (size_t)(g.ny + (a == 1)) * (size_t)(g.nz + (a == 2));
  s->h_refined.assign(nblk, 0);
  PF_CUDA_TRY(cudaMalloc(&s->refined, nblk));
  PF_CUDA_TRY(cudaMemset(s->refined, 0, nblk));
  g.refined = s->refined;
  for (int q = 0; q < 9; ++q) {
    PF_CUDA_TRY(cudaMalloc(&s->f[q], s->nface[q % 3] * sizeof(float)));
    PF_CUDA_TRY(cudaMemset(s->f[q], 0, s->nface[q % 3] * sizeof(float)));
  }
  for (int a = 0; a < 3; ++a) PF_CUDA_TRY(cudaMalloc(&s->acc[a], s->nface[a] * sizeof(float2)));
  PF_CUDA_TRY(cudaMalloc(&s->mk, s->ncell));
  PF_CUDA_TRY(cudaMemset(s->mk, 0, s->ncell));
  PF_CUDA_TRY(cudaMalloc(&s->pcell, s->ncell * sizeof(float)));
  PF_CUDA_TRY(cudaMemset(s->pcell, 0, s->ncell * sizeof(float)));
  PF_CUDA_TRY(cudaMalloc(&s->cell_idx, s->ncell * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->flag0, (s->nkey0 + 1) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->pos0, (s->nkey0 + 1) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->flag1, (s->nkey1 + 1) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->pos1, (s->nkey1 + 1) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->cells, s->ncell * sizeof(int4)));
  PF_CUDA_TRY(cudaMalloc(&s->row_len, (s->ncell + 1) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->slice_len, (s->ncell / 32 + 3) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->slice_ptr, (s->ncell / 32 + 3) * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->minmax, 16 * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->counters, 16 * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->ctl, sizeof(MrCtl)));
  PF_CUDA_TRY(cudaMallocHost(&s->h_ctl, sizeof(MrCtl)));
  PF_CUDA_TRY(cudaMallocHost(&s->h_ints, 32 * sizeof(int)));
  PF_CUDA_TRY(cudaMalloc(&s->partials, 4 * (s->ncell / kMrNT + 2) * sizeof(double)));
  PF_CUDA_TRY(cudaEventCreate(&s->e0));
  PF_CUDA_TRY(cudaEventCreate(&s->e1));
  *out = s;
  return PF_OK;
}

int upload_levels(pf_ctx* ctx, MrState* s) {
  PF_CUDA_TRY(cudaMemcpyAsync(s->refined, s->h_refined.data(), s->h_refined.size(), cudaMemcpyHostToDevice,
                              ctx->stream));
  // the copy reads pageable memory: wait, so that the host vector may change
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

// ---- layout and dynamic refinement, host side -----------------------------
// (src/grid/multires_layout3d.h:53-94, src/driver/multires_sim3d_tp.cpp:119-227)

struct Box {
  int x0 = 0, y0 = 0, z0 = 0, x1 = 0, y1 = 0, z1 = 0;
  bool valid = false;
};

void refine_box(const MrGeom& g, std::vector<uint8_t>& ref, int x0, int y0, int z0, int x1, int y1, int z1) {
  auto cl = [](int v, int n) { return std::max(0, std::min(n, v)); };
  x0 = cl(x0, g.nx);
  y0 = cl(y0, g.ny);
  z0 = cl(z0, g.nz);
  x1 = cl(x1, g.nx);
  y1 = cl(y1, g.ny);
  z1 = cl(z1, g.nz);
  if (!(x0 < x1 && y0 < y1 && z0 < z1)) return;
  for (int bz = 0; bz < g.MZ; ++bz)
    for (int by = 0; by < g.MY; ++by)
      for (int bx = 0; bx < g.MX; ++bx) {
        const int bx0 = 8 * bx, by0 = 8 * by, bz0 = 8 * bz;
        const int bx1 = std::min(g.nx, bx0 + 8), by1 = std::min(g.ny, by0 + 8), bz1 = std::min(g.nz, bz0 + 8);
        if (bx0 < x1 && bx1 > x0 && by0 < y1 && by1 > y0 && bz0 < z1 && bz1 > z0)
          ref[bx + g.MX * (by + g.MY * bz)] = 1;
      }
}

int count_fine_leaves(const MrGeom& g, const std::vector<uint8_t>& ref) {
  int n = 0;
  for (int bz = 0; bz < g.MZ; ++bz)
    for (int by = 0; by < g.MY; ++by)
      for (int bx = 0; bx < g.MX; ++bx) {
        if (!ref[bx + g.MX * (by + g.MY * bz)]) continue;
        for (int c = 0; c < 8; ++c)
          if ((2 * bx + (c & 1)) * 4 < g.nx && (2 * by + ((c >> 1) & 1)) * 4 < g.ny &&
              (2 * bz + (c >> 2)) * 4 < g.nz)
            ++n;
      }
  return n;
}

Box clamp_box(const MrGeom& g, Box b) {
  if (!b.valid) return b;
  auto cl = [](int v, int n) { return std::max(0, std::min(n, v)); };
  b.x0 = cl(b.x0, g.nx);
  b.y0 = cl(b.y0, g.ny);
  b.z0 = cl(b.z0, g.nz);
  b.x1 = cl(b.x1, g.nx);
  b.y1 = cl(b.y1, g.ny);
  b.z1 = cl(b.z1, g.nz);
  b.valid = b.x0 < b.x1 && b.y0 < b.y1 && b.z0 < b.z1;
  return b;
}

int fine_leaves_for(const MrGeom& g, const Box& b) {
  std::vector<uint8_t> ref((size_t)g.MX * g.MY * g.MZ, 0);
  if (b.valid) refine_box(g, ref, b.x0, b.y0, b.z0, b.x1, b.y1, b.z1);
  return count_fine_leaves(g, ref);
}

int update_refinement(pf_ctx* ctx, MrState* s) {
  StageScope stage(ctx, PF_STAGE_ADAPT);
  const MrGeom& g = s->g;
  const size_t n = ctx->np;
  (++ctx->launches), k_mr_minmax_init<<<1, 32, 0, ctx->stream>>>(s->minmax, g.nx, g.ny, g.nz);
  if (n > 0)
    (++ctx->launches), k_mr_bounds<<<grid_for(n, 4 * ctx->num_sms), kMrNT, 0, ctx->stream>>>(
        g, ctx->px, ctx->py, ctx->pz, ctx->type, n, s->minmax);
  PF_CUDA_TRY(cudaGetLastError());
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_ints, s->minmax, 12 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int* m = s->h_ints;  // min xyz, max xyz, gas min xyz, gas max xyz
  Box desired;
  auto include = [&](int x0, int y0, int z0, int x1, int y1, int z1) {
    if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;
    if (!desired.valid) {
      desired = Box{x0, y0, z0, x1, y1, z1, true};
      return;
    }
    desired.x0 = std::min(desired.x0, x0);
    desired.y0 = std::min(desired.y0, y0);
    desired.z0 = std::min(desired.z0, z0);
    desired.x1 = std::max(desired.x1, x1);
    desired.y1 = std::max(desired.y1, y1);
    desired.z1 = std::max(desired.z1, z1);
  };
  const pf_mr_dynamic& d = s->dyn;
  if (m[3] >= 0) {
    const int pad = std::max(0, d.particle_padding);
    include(m[0] - pad, m[1] - pad, m[2] - pad, m[3] + pad + 1, m[4] + pad + 1, m[5] + pad + 1);
  }
  if (m[9] >= 0) {
    const int pad = std::max(0, d.gas_padding);
    include(m[6] - pad, m[7] - pad, m[8] - pad, m[9] + pad + 1, m[10] + pad + 1, m[11] + pad + 1);
  }
  desired = clamp_box(g, desired);
  Box target;
  s->budget_limited = 0;
  if (desired.valid) {
    const Box retained{s->rbox[0], s->rbox[1], s->rbox[2], s->rbox[3], s->rbox[4], s->rbox[5], s->retained_valid != 0};
    const bool contains = retained.valid && retained.x0 <= desired.x0 && retained.y0 <= desired.y0 &&
                          retained.z0 <= desired.z0 && retained.x1 >= desired.x1 && retained.y1 >= desired.y1 &&
                          retained.z1 >= desired.z1;
    if (contains) {
      target = retained;
    } else {
      const int pad = std::max(0, d.hysteresis_cells);
      target = clamp_box(g, Box{desired.x0 - pad, desired.y0 - pad, desired.z0 - pad, desired.x1 + pad,
                                desired.y1 + pad, desired.z1 + pad, true});
    }
    // fitBoxToFineLeafBudget (:212-227)
    if (target.valid && d.max_fine_leaves > 0 && fine_leaves_for(g, target) > d.max_fine_leaves) {
      s->budget_limited = 1;
      const double cx = 0.5 * (double)(target.x0 + target.x1), cy = 0.5 * (double)(target.y0 + target.y1);
      const double cz = 0.5 * (double)(target.z0 + target.z1);
      while (fine_leaves_for(g, target) > d.max_fine_leaves) {
        const int ext[3] = {target.x1 - target.x0, target.y1 - target.y0, target.z1 - target.z0};
        int axis = 0;
        if (ext[1] > ext[axis]) axis = 1;
        if (ext[2] > ext[axis]) axis = 2;
        if (ext[axis] <= 1) break;
        if (axis == 0) {
          if ((target.x1 - cx) >= (cx - target.x0)) --target.x1;
          else ++target.x0;
        } else if (axis == 1) {
          if ((target.y1 - cy) >= (cy - target.y0)) --target.y1;
          else ++target.y0;
        } else {
          if ((target.z1 - cz) >= (cz - target.z0)) --target.z1;
          else ++target.z0;
        }
        target.valid = target.x0 < target.x1 && target.y0 < target.y1 && target.z0 < target.z1;
        if (!target.valid) break;
      }
    }
  }
  s->retained_valid = target.valid ? 1 : 0;
  if (target.valid) {
    s->rbox[0] = target.x0;
    s->rbox[1] = target.y0;
    s->rbox[2] = target.z0;
    s->rbox[3] = target.x1;
    s->rbox[4] = target.y1;
    s->rbox[5] = target.z1;
  }
  std::fill(s->h_refined.begin(), s->h_refined.end(), 0);
  if (target.valid) refine_box(g, s->h_refined, target.x0, target.y0, target.z0, target.x1, target.y1, target.z1);
  s->last_fine_leaves = count_fine_leaves(g, s->h_refined);
  return upload_levels(ctx, s);
}

MrPhase phase_of(const pf_phase* ph) {
  MrPhase P;
  P.rho_l = ph->rho_l;
  P.rho_g = ph->rho_g;
  P.rmin = std::log(ph->rho_l / ph->rho_g) * ph->rho_g * ph->rho_tilde_0;
  P.invden = 1.0 / (ph->alpha_phi * ph->rho_tilde_0 * ph->rho_l);
  return P;
}

MrFaces faces_of(MrState* s) {
  MrFaces F;
  for (int q = 0; q < 9; ++q) F.f[q] = s->f[q];
  return F;
}

int mark_cells_mr(pf_ctx* ctx, MrState* s) {
  StageScope stage(ctx, PF_STAGE_MARK);
  const size_t n = ctx->np;
  (++ctx->launches), k_mr_mark_walls<<<grid_for(s->ncell, 8 * ctx->num_sms), kMrNT, 0, ctx->stream>>>(s->g, s->mk);
  if (n > 0)
    (++ctx->launches), k_mr_mark_particles<<<grid_for(n, INT_MAX), kMrNT, 0, ctx->stream>>>(s->g, ctx->px, ctx->py,
                                                                                           ctx->pz, n, s->mk);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int p2g_mr(pf_ctx* ctx, MrState* s, const pf_phase* ph, double Vp) {
  StageScope stage(ctx, PF_STAGE_SPLAT);
  for (int a = 0; a < 3; ++a)
    PF_CUDA_TRY(cudaMemsetAsync(s->acc[a], 0, s->nface[a] * sizeof(float2), ctx->stream));
  const size_t n = ctx->np;
  if (n > 0)
    (++ctx->launches), k_mr_p2g<<<grid_for(n, INT_MAX), kMrNT, 0, ctx->stream>>>(
        s->g, ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy, ctx->vz, ctx->vol, ctx->type, n, ph->rho_l * Vp,
        ph->rho_g * Vp, s->acc[0], s->acc[1], s->acc[2]);
  for (int a = 0; a < 3; ++a)
    (++ctx->launches), k_mr_split<<<grid_for(s->nface[a], 8 * ctx->num_sms), kMrNT, 0, ctx->stream>>>(
        s->acc[a], s->f[a], s->f[3 + a], s->nface[a]);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

int project_mr(pf_ctx* ctx, MrState* s, const pf_mr_step_cfg* cfg, pf_mr_step_stats* st) {
  StageScope stage(ctx, PF_STAGE_PROJECT);
  const MrGeom& g = s->g;
  const int big = 8 * ctx->num_sms;
  PF_CUDA_TRY(cudaMemsetAsync(s->pcell, 0, s->ncell * sizeof(float), ctx->stream));
  PF_CUDA_TRY(cudaMemsetAsync(s->cell_idx, 0xff, s->ncell * sizeof(int), ctx->stream));
  (++ctx->launches), k_mr_flags<<<grid_for(s->nkey0, big), kMrNT, 0, ctx->stream>>>(g, s->mk, 0, s->nkey0, s->flag0);
  (++ctx->launches), k_mr_flags<<<grid_for(s->nkey1, big), kMrNT, 0, ctx->stream>>>(g, s->mk, 1, s->nkey1, s->flag1);
  PF_CUDA_TRY(cudaGetLastError());
  int* tot = ctx->d_scalar;  // [0] level-0 fluid cells, [1] level-1, [2] nonzeros, [3] air
  int rc = scan_exclusive(ctx, s->flag0, s->pos0, (int)s->nkey0, tot + 0);
  if (!rc) rc = scan_exclusive(ctx, s->flag1, s->pos1, (int)s->nkey1, tot + 1);
  if (rc) return rc;
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_ints, tot, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int N = s->h_ints[0] + s->h_ints[1];
  st->active_cells = N;
  st->pinned_cell = -1;
  if (N == 0) {
    st->converged = 1;
    return PF_OK;
  }
  (++ctx->launches), k_mr_cells<<<grid_for(s->nkey0, big), kMrNT, 0, ctx->stream>>>(g, 0, s->nkey0, s->flag0, s->pos0,
                                                                                    nullptr, s->cells, s->cell_idx);
  (++ctx->launches), k_mr_cells<<<grid_for(s->nkey1, big), kMrNT, 0, ctx->stream>>>(g, 1, s->nkey1, s->flag1, s->pos1,
                                                                                    tot + 0, s->cells, s->cell_idx);
  PF_CUDA_TRY(cudaMemsetAsync(tot + 3, 0, sizeof(int), ctx->stream));
  (++ctx->launches), k_mr_pin_probe<<<grid_for(N, big), kMrNT, 0, ctx->stream>>>(g, s->mk, s->cells, N, tot + 3);
  (++ctx->launches), k_mr_row_count<<<grid_for(N, big), kMrNT, 0, ctx->stream>>>(g, s->mk, s->cells, s->cell_idx, N,
                                                                                 tot + 3, s->row_len);
  PF_CUDA_TRY(cudaGetLastError());
  const int nslice = (N + 31) / 32;
  (++ctx->launches), k_mr_slices<<<grid_for(nslice + 1, big), kMrNT, 0, ctx->stream>>>(N, s->row_len, s->slice_len);
  PF_CUDA_TRY(cudaGetLastError());
  rc = scan_exclusive(ctx, s->slice_len, s->slice_ptr, nslice + 1, tot + 2);  // total = stored entries
  if (rc) return rc;
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_ints + 2, tot + 2, 2 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const size_t nnz = (size_t)std::max(s->h_ints[2], 0);
  st->pinned_cell = s->h_ints[3] ? -1 : 0;
  if (nnz > s->nnz_cap) {
    if (s->col) PF_CUDA_TRY(cudaFree(s->col));
    if (s->coef) PF_CUDA_TRY(cudaFree(s->coef));
    s->col = nullptr;
    s->coef = nullptr;
    s->nnz_cap = 0;
    const size_t cap = nnz + nnz / 2 + 1024;
    PF_CUDA_TRY(cudaMalloc(&s->col, cap * sizeof(int)));
    PF_CUDA_TRY(cudaMalloc(&s->coef, cap * sizeof(double)));
    s->nnz_cap = cap;
  }
  // the context's FP64 solver vectors (sized for every tile of the pool) hold
  // the multires unknowns: N <= nx ny nz <= their length
  // the direction alternates between ctx->p and ctx->cy
  MrVecs V{ctx->x, ctx->r, ctx->cx, ctx->p, ctx->Ap, ctx->diag};
  double* pbuf[2] = {ctx->p, ctx->cy};
  // 4 CTAs per SM: more CTAs spend more on the last-CTA reductions' atomics
  // than they gain in load parallelism
  const int nred = grid_for(N, 4 * ctx->num_sms);
  // the update keeps kMrRows rows of loads in flight per thread (94
  // registers): one wave of 2 CTAs per SM
  const int nupd = grid_for(N, 2 * ctx->num_sms);
  // the SpMV keeps two rows in flight per thread (80 registers): one wave of
  // 3 CTAs per SM
  const int nspmv = grid_for(N, 3 * ctx->num_sms);
  (++ctx->launches), k_mr_ctl_init<<<1, 1, 0, ctx->stream>>>(s->ctl, cfg->cg_iters, cfg->cg_tol, cfg->cg_rel_tol,
                                                             cfg->jacobi, cfg->flexible_beta, cfg->adaptive_restart,
                                                             cfg->restart_growth);
  PF_CUDA_TRY(cudaEventRecord(s->e0, ctx->stream));
  (++ctx->launches), k_mr_rows<<<nred, kMrNT, 0, ctx->stream>>>(g, s->mk, s->cells, s->cell_idx, N, tot + 3,
                                                                faces_of(s), phase_of(&cfg->phase), cfg->dt,
                                                                cfg->c_div, s->slice_ptr, s->col, s->coef, V, s->ctl,
                                                                s->partials);
  PF_CUDA_TRY(cudaGetLastError());
  MrCtl c{};
  int launched = 0;
  stage_begin(ctx, PF_STAGE_PCG);
  while (true) {
    PF_CUDA_TRY(cudaMemcpyAsync(s->h_ctl, s->ctl, sizeof(MrCtl), cudaMemcpyDeviceToHost, ctx->stream));
    PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    c = *s->h_ctl;
    if (c.done || launched >= cfg->cg_iters) break;
    const int batch = std::min(kMrPoll, cfg->cg_iters - launched);
    for (int b = 0; b < batch; ++b) {
      const int q = (launched + b) & 1;
      double* p_prev = pbuf[q];
      double* p = pbuf[q ^ 1];
      // programmatic dependent launches: each kernel's CTAs are scheduled
      // while its predecessor drains and wait for it before reading anything
      ++ctx->launches;
      PF_CUDA_TRY(launch_pdl(k_mr_spmv, dim3(nspmv), dim3(kMrNT), ctx->stream, N, (const int*)s->slice_ptr,
                             (const int*)s->col, (const double*)s->coef, (const double*)V.z, (const double*)p_prev,
                             p, V.Ap, (const double*)V.diag, s->ctl, s->partials, (const int*)(tot + 3)));
      MrVecs Vi = V;
      Vi.p = p;
      ++ctx->launches;
      PF_CUDA_TRY(launch_pdl(k_mr_update, dim3(nupd), dim3(kMrNT), ctx->stream, N, Vi, s->ctl, s->partials));
    }
    PF_CUDA_TRY(cudaGetLastError());
    launched += batch;
  }
  PF_CUDA_TRY(cudaEventRecord(s->e1, ctx->stream));
  stage_end(ctx, PF_STAGE_PCG);
  st->iterations = c.it;
  st->restarts = c.restarts;
  st->beta_resets = c.beta_resets;
  st->converged = c.done == 1 ? 1 : 0;
  st->breakdown = c.done == 2 ? 1 : 0;
  st->initial_residual = c.res0;
  st->final_residual = c.res;
  st->effective_tolerance = c.tol;
  (++ctx->launches), k_mr_pressure<<<grid_for(N, big), kMrNT, 0, ctx->stream>>>(g, s->cells, N, V.x, s->pcell);
  const MrPhase P = phase_of(&cfg->phase);
  for (int a = 0; a < 3; ++a)
    (++ctx->launches), k_mr_velocity<<<grid_for(s->nface[a], big), kMrNT, 0, ctx->stream>>>(
        g, a, s->mk, s->cell_idx, s->cells, V.x, s->f[a], s->f[3 + a], P, cfg->dt);
  PF_CUDA_TRY(cudaGetLastError());
  return PF_OK;
}

}  // namespace

void mr_free(pf_ctx* ctx) {
  MrState* s = static_cast<MrState*>(ctx->mr);
  if (!s) return;
  auto F = [](void* p) { if (p) cudaFree(p); };
  F(s->refined);
  for (int q = 0; q < 9; ++q) F(s->f[q]);
  for (int a = 0; a < 3; ++a) F(s->acc[a]);
  F(s->mk); F(s->pcell); F(s->cell_idx); F(s->flag0); F(s->pos0); F(s->flag1); F(s->pos1); F(s->cells);
  F(s->row_len); F(s->slice_len); F(s->slice_ptr); F(s->col); F(s->coef); F(s->minmax); F(s->counters); F(s->ctl); F(s->partials);
  if (s->h_ctl) cudaFreeHost(s->h_ctl);
  if (s->h_ints) cudaFreeHost(s->h_ints);
  if (s->e0) cudaEventDestroy(s->e0);
  if (s->e1) cudaEventDestroy(s->e1);
  delete s;
  ctx->mr = nullptr;
}

int take_upload_for(pf_ctx* ctx);

}  // namespace pf

using namespace pf;

extern "C" {

int pf_mr_set_layout(pf_ctx* ctx, const pf_mr_box* boxes, int n) {
  if (!ctx || n < 0 || (n > 0 && !boxes)) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  std::fill(s->h_refined.begin(), s->h_refined.end(), 0);
  for (int b = 0; b < n; ++b)
    refine_box(s->g, s->h_refined, boxes[b].x0, boxes[b].y0, boxes[b].z0, boxes[b].x1, boxes[b].y1, boxes[b].z1);
  s->last_fine_leaves = count_fine_leaves(s->g, s->h_refined);
  return upload_levels(ctx, s);
}

int pf_mr_set_levels(pf_ctx* ctx, const uint8_t* refined) {
  if (!ctx || !refined) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  for (size_t t = 0; t < s->h_refined.size(); ++t) s->h_refined[t] = refined[t] ? 1 : 0;
  s->last_fine_leaves = count_fine_leaves(s->g, s->h_refined);
  return upload_levels(ctx, s);
}

int pf_mr_get_levels(pf_ctx* ctx, uint8_t* refined, int* blocks3) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  if (blocks3) {
    blocks3[0] = s->g.MX;
    blocks3[1] = s->g.MY;
    blocks3[2] = s->g.MZ;
  }
  if (refined) std::copy(s->h_refined.begin(), s->h_refined.end(), refined);
  return PF_OK;
}

int pf_mr_set_dynamic(pf_ctx* ctx, const pf_mr_dynamic* dyn) {
  if (!ctx || !dyn) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  s->dyn = *dyn;
  return PF_OK;
}

int pf_mr_reset_refinement(pf_ctx* ctx) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  s->retained_valid = 0;
  s->budget_limited = 0;
  return PF_OK;
}

int pf_mr_update_refinement(pf_ctx* ctx, int* state8) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (!rc) rc = take_upload_for(ctx);
  if (!rc && s->dyn.enabled) rc = update_refinement(ctx, s);
  if (rc) return rc;
  if (state8) {
    state8[0] = s->retained_valid;
    for (int d = 0; d < 6; ++d) state8[1 + d] = s->rbox[d];
    state8[7] = s->budget_limited;
  }
  return PF_OK;
}

int pf_mr_p2g(pf_ctx* ctx, const pf_phase* phase, double Vp) {
  if (!ctx || !phase) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (!rc) rc = take_upload_for(ctx);
  if (!rc) rc = p2g_mr(ctx, s, phase, Vp);
  if (!rc) PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return rc;
}

int pf_mr_step(pf_ctx* ctx, const pf_mr_step_cfg* cfg, pf_mr_step_stats* stats) {
  if (!ctx || !cfg || (cfg->advect_order != 2 && cfg->advect_order != 3) || cfg->cg_iters < 0)
    return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (!rc) rc = take_upload_for(ctx);
  if (rc) return rc;
  pf_mr_step_stats st{};
  // updateDynamicRefinement, markCells, P2G, saved copy, gravity, walls,
  // projection, G2P, advection
  if (s->dyn.enabled) {
    rc = update_refinement(ctx, s);
    if (rc) return rc;
  }
  rc = mark_cells_mr(ctx, s);
  if (!rc) rc = p2g_mr(ctx, s, &cfg->phase, cfg->Vp);
  if (rc) return rc;
  {
    StageScope stage(ctx, PF_STAGE_BOUNDARY);
    for (int a = 0; a < 3; ++a)
      PF_CUDA_TRY(cudaMemcpyAsync(s->f[6 + a], s->f[a], s->nface[a] * sizeof(float), cudaMemcpyDeviceToDevice,
                                  ctx->stream));
    const int big = 8 * ctx->num_sms;
    const float dv = (float)(cfg->dt * cfg->gravity);
    for (int a = 0; a < 3; ++a)
      (++ctx->launches), k_mr_forces<<<grid_for(s->nface[a], big), kMrNT, 0, ctx->stream>>>(s->g, a, s->f[a],
                                                                                            s->f[3 + a], dv);
    PF_CUDA_TRY(cudaGetLastError());
  }
  rc = project_mr(ctx, s, cfg, &st);
  if (rc) return rc;
  const size_t n = ctx->np;
  stage_begin(ctx, PF_STAGE_G2P);
  PF_CUDA_TRY(cudaMemsetAsync(s->counters, 0, 8 * sizeof(int), ctx->stream));
  if (n > 0)
    (++ctx->launches), k_mr_g2p_advect<<<grid_for(n, INT_MAX), kMrNT, 0, ctx->stream>>>(
        s->g, faces_of(s), ctx->px, ctx->py, ctx->pz, ctx->vx, ctx->vy, ctx->vz, ctx->type, n, cfg->alpha_l,
        cfg->alpha_g, cfg->dt, cfg->advect_order, s->counters);
  PF_CUDA_TRY(cudaGetLastError());
  stage_end(ctx, PF_STAGE_G2P);
  ctx->bins_valid = false;
  PF_CUDA_TRY(cudaMemcpyAsync(s->h_ints + 8, s->counters, 8 * sizeof(int), cudaMemcpyDeviceToHost, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  const int* c = s->h_ints + 8;
  st.clamp.clamped_liquid = c[0];
  st.clamp.clamped_gas = c[1];
  st.clamp.x_lo = c[2];
  st.clamp.x_hi = c[3];
  st.clamp.y_lo = c[4];
  st.clamp.y_hi = c[5];
  st.clamp.z_lo = c[6];
  st.clamp.z_hi = c[7];
  st.fine_leaves = s->last_fine_leaves;
  float ms = 0.0f;
  if (st.active_cells > 0 && cudaEventElapsedTime(&ms, s->e0, s->e1) == cudaSuccess) st.solve_ms = ms;
  if (stats) *stats = st;
  return PF_OK;
}

int pf_mr_get_face(pf_ctx* ctx, int field, float* dense) {
  if (!ctx || !dense || field < 0 || field > 8) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  PF_CUDA_TRY(cudaMemcpyAsync(dense, s->f[field], s->nface[field % 3] * sizeof(float), cudaMemcpyDefault,
                              ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

int pf_mr_get_cells(pf_ctx* ctx, uint8_t* marker, float* pressure) {
  if (!ctx) return PF_ERR_INVALID;
  cudaSetDevice(ctx->device);
  MrState* s = nullptr;
  int rc = mr_state(ctx, &s);
  if (rc) return rc;
  if (marker) PF_CUDA_TRY(cudaMemcpyAsync(marker, s->mk, s->ncell, cudaMemcpyDefault, ctx->stream));
  if (pressure)
    PF_CUDA_TRY(cudaMemcpyAsync(pressure, s->pcell, s->ncell * sizeof(float), cudaMemcpyDefault, ctx->stream));
  PF_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
  return PF_OK;
}

}  // extern "C"
