/*
 * pf_oracle.c -- CPU restatement of the adaptive-pf-flip sparse 3D two-phase
 * step.  TEST INFRASTRUCTURE ONLY (the checker, never the product): see
 * pf_oracle.h for the representation and the rules this file follows.
 *
 * Build: plain C99, no FMA contraction (-ffp-contract=off) so that every
 * double expression rounds exactly as the reference's C++ does on x86-64.
 */
#include "pf_oracle.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

struct pfo_grid {
  int nx, ny, nz;
  double dx, ox, oy, oz;
  int dim[PFO_NFIELDS][3];  /* node lattice per field */
  int bdim[PFO_NFIELDS][3]; /* 4^3 block lattice per field */
  float* val[PFO_NFIELDS];
  unsigned char* act[PFO_NFIELDS];
};

/* ------------------------------------------------------------------ */
/* storage helpers: SparseBlockGrid3D<4> semantics                     */
/* (src/grid/sparse_block_grid3d.h:10-68)                              */
/* ------------------------------------------------------------------ */

static size_t nodes_of(const pfo_grid* g, int f) {
  return (size_t)g->dim[f][0] * g->dim[f][1] * g->dim[f][2];
}
static size_t blocks_of(const pfo_grid* g, int f) {
  return (size_t)g->bdim[f][0] * g->bdim[f][1] * g->bdim[f][2];
}
static size_t nidx(const pfo_grid* g, int f, int i, int j, int k) {
  return (size_t)i + (size_t)g->dim[f][0] * ((size_t)j + (size_t)g->dim[f][1] * (size_t)k);
}
static int in_field(const pfo_grid* g, int f, int i, int j, int k) {
  return i >= 0 && j >= 0 && k >= 0 && i < g->dim[f][0] && j < g->dim[f][1] && k < g->dim[f][2];
}
/* activateBlock (:34-44): mark the 4^3 block holding node (i,j,k) active. */
static void activate(pfo_grid* g, int f, int i, int j, int k) {
  size_t b = (size_t)(i / 4) + (size_t)g->bdim[f][0] * ((size_t)(j / 4) + (size_t)g->bdim[f][1] * (size_t)(k / 4));
  g->act[f][b] = 1;
}
/* ref (:46-49): activate, then hand out the node. */
static float* ref(pfo_grid* g, int f, int i, int j, int k) {
  activate(g, f, i, j, k);
  return &g->val[f][nidx(g, f, i, j, k)];
}
/* get (:50-55): zero outside the lattice; zero in inactive blocks (kept zero here). */
static float get(const pfo_grid* g, int f, int i, int j, int k) {
  if (!in_field(g, f, i, j, k)) return 0.0f;
  return g->val[f][nidx(g, f, i, j, k)];
}

pfo_grid* pfo_grid_create(int nx, int ny, int nz, double dx, double ox, double oy, double oz) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0.0)) return NULL;
  pfo_grid* g = (pfo_grid*)calloc(1, sizeof(pfo_grid));
  if (!g) return NULL;
  g->nx = nx; g->ny = ny; g->nz = nz;
  g->dx = dx; g->ox = ox; g->oy = oy; g->oz = oz;
  /* SparseMacGrid3D constructor, src/grid/sparse_mac_grid3d.h:16-20 */
  const int d[PFO_NFIELDS][3] = {
    {nx + 1, ny, nz}, {nx, ny + 1, nz}, {nx, ny, nz + 1},
    {nx + 1, ny, nz}, {nx, ny + 1, nz}, {nx, ny, nz + 1},
    {nx, ny, nz}, {nx, ny, nz}};
  for (int f = 0; f < PFO_NFIELDS; ++f) {
    for (int a = 0; a < 3; ++a) {
      g->dim[f][a] = d[f][a];
      g->bdim[f][a] = (d[f][a] + 3) / 4;
    }
    g->val[f] = (float*)calloc(nodes_of(g, f), sizeof(float));
    g->act[f] = (unsigned char*)calloc(blocks_of(g, f), 1);
    if (!g->val[f] || !g->act[f]) { pfo_grid_destroy(g); return NULL; }
  }
  return g;
}

void pfo_grid_destroy(pfo_grid* g) {
  if (!g) return;
  for (int f = 0; f < PFO_NFIELDS; ++f) { free(g->val[f]); free(g->act[f]); }
  free(g);
}

int pfo_grid_copy(pfo_grid* dst, const pfo_grid* src) {
  if (!dst || !src || dst->nx != src->nx || dst->ny != src->ny || dst->nz != src->nz) return -1;
  dst->dx = src->dx; dst->ox = src->ox; dst->oy = src->oy; dst->oz = src->oz;
  for (int f = 0; f < PFO_NFIELDS; ++f) {
    memcpy(dst->val[f], src->val[f], nodes_of(src, f) * sizeof(float));
    memcpy(dst->act[f], src->act[f], blocks_of(src, f));
  }
  return 0;
}

int pfo_field_dims(const pfo_grid* g, int f, int* dims3, int* bdims3) {
  if (!g || f < 0 || f >= PFO_NFIELDS) return -1;
  for (int a = 0; a < 3; ++a) {
    if (dims3) dims3[a] = g->dim[f][a];
    if (bdims3) bdims3[a] = g->bdim[f][a];
  }
  return 0;
}

int pfo_get_field(const pfo_grid* g, int f, float* dense, unsigned char* act) {
  if (!g || f < 0 || f >= PFO_NFIELDS) return -1;
  if (dense) memcpy(dense, g->val[f], nodes_of(g, f) * sizeof(float));
  if (act) memcpy(act, g->act[f], blocks_of(g, f));
  return 0;
}

/* Import a field: nodes outside the given active blocks are forced to zero so
 * the "inactive => zero" invariant holds. */
int pfo_set_field(pfo_grid* g, int f, const float* dense, const unsigned char* act) {
  if (!g || f < 0 || f >= PFO_NFIELDS || !dense || !act) return -1;
  memcpy(g->act[f], act, blocks_of(g, f));
  const int X = g->dim[f][0], Y = g->dim[f][1], Z = g->dim[f][2];
  for (int k = 0; k < Z; ++k)
    for (int j = 0; j < Y; ++j)
      for (int i = 0; i < X; ++i) {
        size_t b = (size_t)(i / 4) + (size_t)g->bdim[f][0] * ((size_t)(j / 4) + (size_t)g->bdim[f][1] * (size_t)(k / 4));
        size_t n = nidx(g, f, i, j, k);
        g->val[f][n] = act[b] ? dense[n] : 0.0f;
      }
  return 0;
}

/* clear (:64-67) plus the zero-fill that activateBlock performs on reuse. */
int pfo_clear_field(pfo_grid* g, int f) {
  if (!g || f < 0 || f >= PFO_NFIELDS) return -1;
  memset(g->val[f], 0, nodes_of(g, f) * sizeof(float));
  memset(g->act[f], 0, blocks_of(g, f));
  return 0;
}

int pfo_clear_all(pfo_grid* g) {
  for (int f = 0; f < PFO_NFIELDS; ++f)
    if (pfo_clear_field(g, f)) return -1;
  return 0;
}

/* ------------------------------------------------------------------ */
/* Eq. 7 phase field (src/physics/phasefield.h:10-18)                  */
/* ------------------------------------------------------------------ */

double pfo_phi_from_raw(double raw, const pfo_phase* pp) {
  const double eta = log(pp->rho_l / pp->rho_g);
  const double rmin = eta * pp->rho_g * pp->rho_tilde_0;
  if (raw < rmin) return 0.0;
  double excess = raw - rmin;
  if (excess < 0.0) excess = 0.0;
  const double v = sqrt(excess / (pp->alpha_phi * pp->rho_tilde_0 * pp->rho_l));
  return 1.0 < v ? 1.0 : v; /* std::min(v, 1.0), NaN included */
}

double pfo_beta_from_raw(double raw, const pfo_phase* pp) {
  const double phi = pfo_phi_from_raw(raw, pp);
  const double rho = phi * pp->rho_l + (1.0 - phi) * pp->rho_g;
  return 1.0 / rho;
}

/* ------------------------------------------------------------------ */
/* Eq. 6 normalized cubic kernel (src/driver/sparse_ops3d_tp.cpp:15-21) */
/* ------------------------------------------------------------------ */

static const double KERNEL_RADIUS = 1.5;

static double cubic_weight(double d2) {
  const double q = d2 / (KERNEL_RADIUS * KERNEL_RADIUS);
  const double t = 1.0 - q;
  return t > 0.0 ? t * t * t : 0.0;
}

/* calibrateRhoTilde0 (src/transfer/transfer3d_tp.cpp:29-36): splat a full
 * 8^3 unit lattice at 8 particles per cell into a dense FP64 u-face mass
 * field and read the raw density at face (4,4,4). */
double pfo_calibrate_rho_tilde0(const pfo_phase* pp, double Vp) {
  enum { N = 8 };
  const int X = N + 1, Y = N, Z = N;
  double* mass = (double*)calloc((size_t)X * Y * Z, sizeof(double));
  if (!mass) return 1.0;
  const double mp = pp->rho_l * Vp;
  for (int k = 0; k < N; ++k)
    for (int j = 0; j < N; ++j)
      for (int i = 0; i < N; ++i)
        for (int s = 0; s < 8; ++s) {
          const double x = i + 0.25 + 0.5 * (s & 1);
          const double y = j + 0.25 + 0.5 * ((s >> 1) & 1);
          const double z = k + 0.25 + 0.5 * ((s >> 2) & 1);
          const double gx = x, gy = y - 0.5, gz = z - 0.5;
          const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
          double wsum = 0.0;
          for (int dk = -2; dk <= 3; ++dk)
            for (int dj = -2; dj <= 3; ++dj)
              for (int di = -2; di <= 3; ++di) {
                const int a = i0 + di, b = j0 + dj, c = k0 + dk;
                if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
                const double ex = gx - a, ey = gy - b, ez = gz - c;
                wsum += cubic_weight(ex * ex + ey * ey + ez * ez);
              }
          if (wsum <= 0.0) continue;
          for (int dk = -2; dk <= 3; ++dk)
            for (int dj = -2; dj <= 3; ++dj)
              for (int di = -2; di <= 3; ++di) {
                const int a = i0 + di, b = j0 + dj, c = k0 + dk;
                if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
                const double ex = gx - a, ey = gy - b, ez = gz - c;
                const double w = cubic_weight(ex * ex + ey * ey + ez * ez) / wsum;
                if (w <= 0.0) continue;
                mass[(size_t)a + (size_t)X * ((size_t)b + (size_t)Y * c)] += w * mp;
              }
        }
  const double raw = mass[4 + X * (4 + Y * 4)];
  free(mass);
  return raw > 0.0 ? raw / pp->rho_l : 1.0;
}

/* ------------------------------------------------------------------ */
/* P2G (src/driver/sparse_ops3d_tp.cpp:23-75, 95-153)                  */
/* ------------------------------------------------------------------ */

/* preactivateKernel (:23-40): activate the block of every window node with
 * nonzero weight.  Only nodes with k in [klo, khi) are visited (the slab of
 * the thread that owns those blocks; see pfo_p2g). */
static void preactivate(pfo_grid* g, int f, double gx, double gy, double gz, int klo, int khi) {
  const int X = g->dim[f][0], Y = g->dim[f][1], Z = g->dim[f][2];
  const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
  for (int dk = -2; dk <= 3; ++dk)
    for (int dj = -2; dj <= 3; ++dj)
      for (int di = -2; di <= 3; ++di) {
        const int a = i0 + di, b = j0 + dj, c = k0 + dk;
        if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
        if (c < klo || c >= khi) continue;
        const double ex = gx - a, ey = gy - b, ez = gz - c;
        if (cubic_weight(ex * ex + ey * ey + ez * ez) <= 0.0) continue;
        activate(g, f, a, b, c);
      }
}

/* splatKernelColor (:42-75) without the colour filter: each node still
 * receives its contributions in particle-index order, which is the order the
 * reference's owning colour thread adds them in.  The weight sum runs over the
 * whole window; only nodes with k in [klo, khi) are written. */
static void splat(pfo_grid* g, int fmom, int fmass, double gx, double gy, double gz,
                  double mom, double mass, int klo, int khi) {
  const int X = g->dim[fmom][0], Y = g->dim[fmom][1], Z = g->dim[fmom][2];
  const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
  if (k0 + 3 < klo || k0 - 2 >= khi) return;
  double wsum = 0.0;
  for (int dk = -2; dk <= 3; ++dk)
    for (int dj = -2; dj <= 3; ++dj)
      for (int di = -2; di <= 3; ++di) {
        const int a = i0 + di, b = j0 + dj, c = k0 + dk;
        if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
        const double ex = gx - a, ey = gy - b, ez = gz - c;
        wsum += cubic_weight(ex * ex + ey * ey + ez * ez);
      }
  if (wsum <= 0.0) return;
  for (int dk = -2; dk <= 3; ++dk)
    for (int dj = -2; dj <= 3; ++dj)
      for (int di = -2; di <= 3; ++di) {
        const int a = i0 + di, b = j0 + dj, c = k0 + dk;
        if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
        if (c < klo || c >= khi) continue;
        const double ex = gx - a, ey = gy - b, ez = gz - c;
        const double w = cubic_weight(ex * ex + ey * ey + ez * ez) / wsum;
        if (w <= 0.0) continue;
        float* pm = ref(g, fmom, a, b, c);
        *pm += (float)(w * mom);
        float* pw = ref(g, fmass, a, b, c);
        *pw += (float)(w * mass);
      }
}

/* One thread's share of P2G: every node with k in [klo, khi), i.e. whole
 * 4^3 block layers, so no block byte or node is written by two threads.  The
 * thread visits all particles in index order, so each node receives its
 * contributions in the sequential order and the result does not depend on
 * the number of threads. */
typedef struct {
  pfo_grid* g;
  size_t n;
  const double *pos, *vel, *vol;
  const unsigned char* type;
  const pfo_phase* pp;
  double Vp;
  int klo, khi;
} p2g_slab;

static void* p2g_slab_run(void* arg) {
  const p2g_slab* s = (const p2g_slab*)arg;
  pfo_grid* g = s->g;
  const double* pos = s->pos;
  for (size_t p = 0; p < s->n; ++p) {
    const double px = (pos[3 * p + 0] - g->ox) / g->dx;
    const double py = (pos[3 * p + 1] - g->oy) / g->dx;
    const double pz = (pos[3 * p + 2] - g->oz) / g->dx;
    preactivate(g, PFO_U, px, py - 0.5, pz - 0.5, s->klo, s->khi);
    preactivate(g, PFO_MU, px, py - 0.5, pz - 0.5, s->klo, s->khi);
    preactivate(g, PFO_V, px - 0.5, py, pz - 0.5, s->klo, s->khi);
    preactivate(g, PFO_MV, px - 0.5, py, pz - 0.5, s->klo, s->khi);
    preactivate(g, PFO_W, px - 0.5, py - 0.5, pz, s->klo, s->khi);
    preactivate(g, PFO_MW, px - 0.5, py - 0.5, pz, s->klo, s->khi);
  }
  for (size_t p = 0; p < s->n; ++p) {
    const double rho = s->type[p] == 0 ? s->pp->rho_l : s->pp->rho_g;
    const double mp = rho * s->Vp * s->vol[p];
    const double px = (pos[3 * p + 0] - g->ox) / g->dx;
    const double py = (pos[3 * p + 1] - g->oy) / g->dx;
    const double pz = (pos[3 * p + 2] - g->oz) / g->dx;
    splat(g, PFO_U, PFO_MU, px, py - 0.5, pz - 0.5, mp * s->vel[3 * p + 0], mp, s->klo, s->khi);
    splat(g, PFO_V, PFO_MV, px - 0.5, py, pz - 0.5, mp * s->vel[3 * p + 1], mp, s->klo, s->khi);
    splat(g, PFO_W, PFO_MW, px - 0.5, py - 0.5, pz, mp * s->vel[3 * p + 2], mp, s->klo, s->khi);
  }
  return NULL;
}

/* Threads for P2G: PFO_THREADS if set, else the online CPUs, at most 64. */
static int p2g_threads(void) {
  const char* e = getenv("PFO_THREADS");
  long t = e ? strtol(e, NULL, 10) : sysconf(_SC_NPROCESSORS_ONLN);
  if (t < 1) t = 1;
  if (t > 64) t = 64;
  return (int)t;
}

int pfo_p2g(pfo_grid* g, size_t n, const double* pos, const double* vel,
            const unsigned char* type, const double* vol, const pfo_phase* pp, double Vp) {
  if (!g || !pp || (n && (!pos || !vel || !type || !vol))) return -1;
  for (int f = PFO_U; f <= PFO_MW; ++f) pfo_clear_field(g, f);
  /* block layers along z (the w lattice has the most) shared out in order */
  const int layers = g->bdim[PFO_W][2];
  int nt = p2g_threads();
  if (nt > layers) nt = layers;
  p2g_slab slabs[64];
  pthread_t tid[64];
  for (int t = 0; t < nt; ++t) {
    p2g_slab* s = &slabs[t];
    s->g = g; s->n = n; s->pos = pos; s->vel = vel; s->vol = vol; s->type = type; s->pp = pp; s->Vp = Vp;
    s->klo = 4 * (int)((long)layers * t / nt);
    s->khi = 4 * (int)((long)layers * (t + 1) / nt);
  }
  int started = 0;
  for (int t = 1; t < nt; ++t) {
    if (pthread_create(&tid[t], NULL, p2g_slab_run, &slabs[t]) != 0) break;
    started = t;
  }
  /* slabs whose thread did not start run here, after slab 0 */
  p2g_slab_run(&slabs[0]);
  for (int t = started + 1; t < nt; ++t) p2g_slab_run(&slabs[t]);
  for (int t = 1; t <= started; ++t) pthread_join(tid[t], NULL);
  /* normalisation (:126-152): u = momentum / raw mass where the mass is > 0 */
  for (int a = 0; a < 3; ++a) {
    const int fv = PFO_U + a, fm = PFO_MU + a;
    const size_t nn = nodes_of(g, fv);
    for (size_t q = 0; q < nn; ++q) {
      const float m = g->val[fm][q];
      if (m > 0.0f) g->val[fv][q] = g->val[fv][q] / m;
    }
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* markCells / applyGravity / applyWallBoundary                        */
/* (src/driver/sparse_sim3d_tp.cpp:22-97)                              */
/* ------------------------------------------------------------------ */

static int cell_of(const pfo_grid* g, int i, int j, int k) {
  return (int)(get(g, PFO_MK, i, j, k) + 0.5f); /* sparse_mac_grid3d.h:39 */
}
static void set_cell(pfo_grid* g, int i, int j, int k, int c) {
  *ref(g, PFO_MK, i, j, k) = (float)c;
}

int pfo_mark_cells(pfo_grid* g, size_t n, const double* pos) {
  if (!g || (n && !pos)) return -1;
  pfo_clear_field(g, PFO_MK);
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j) { set_cell(g, 0, j, k, 2); set_cell(g, g->nx - 1, j, k, 2); }
  for (int k = 0; k < g->nz; ++k)
    for (int i = 0; i < g->nx; ++i) { set_cell(g, i, 0, k, 2); set_cell(g, i, g->ny - 1, k, 2); }
  for (int j = 0; j < g->ny; ++j)
    for (int i = 0; i < g->nx; ++i) { set_cell(g, i, j, 0, 2); set_cell(g, i, j, g->nz - 1, 2); }
  for (size_t p = 0; p < n; ++p) {
    /* truncation toward zero, as the reference's (int) cast */
    const int i = (int)((pos[3 * p + 0] - g->ox) / g->dx);
    const int j = (int)((pos[3 * p + 1] - g->oy) / g->dx);
    const int k = (int)((pos[3 * p + 2] - g->oz) / g->dx);
    if (i >= 0 && i < g->nx && j >= 0 && j < g->ny && k >= 0 && k < g->nz &&
        cell_of(g, i, j, k) != 2)
      set_cell(g, i, j, k, 1);
  }
  return 0;
}

int pfo_apply_gravity(pfo_grid* g, double dt, double gravity) {
  if (!g) return -1;
  const float dv = (float)(dt * gravity);
  const int X = g->dim[PFO_V][0], Y = g->dim[PFO_V][1], Z = g->dim[PFO_V][2];
  for (int k = 0; k < Z; ++k)
    for (int j = 0; j < Y; ++j)
      for (int i = 0; i < X; ++i) {
        if (get(g, PFO_MV, i, j, k) > 0.0f) {
          const float cur = get(g, PFO_V, i, j, k);
          *ref(g, PFO_V, i, j, k) = cur + dv;
        }
      }
  return 0;
}

int pfo_apply_wall_boundary(pfo_grid* g) {
  if (!g) return -1;
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j) {
      *ref(g, PFO_U, 0, j, k) = 0.0f; *ref(g, PFO_U, 1, j, k) = 0.0f;
      *ref(g, PFO_U, nx - 1, j, k) = 0.0f; *ref(g, PFO_U, nx, j, k) = 0.0f;
    }
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) {
      *ref(g, PFO_V, i, 0, k) = 0.0f; *ref(g, PFO_V, i, 1, k) = 0.0f;
      *ref(g, PFO_V, i, ny - 1, k) = 0.0f; *ref(g, PFO_V, i, ny, k) = 0.0f;
    }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      *ref(g, PFO_W, i, j, 0) = 0.0f; *ref(g, PFO_W, i, j, 1) = 0.0f;
      *ref(g, PFO_W, i, j, nz - 1) = 0.0f; *ref(g, PFO_W, i, j, nz) = 0.0f;
    }
  return 0;
}

/* ------------------------------------------------------------------ */
/* Projection (src/driver/sparse_ops3d_tp.cpp:234-423)                 */
/* ------------------------------------------------------------------ */

static int in_cells(const pfo_grid* g, int i, int j, int k) {
  return i >= 0 && i < g->nx && j >= 0 && j < g->ny && k >= 0 && k < g->nz;
}
static int is_fluid(const pfo_grid* g, int i, int j, int k) {
  return in_cells(g, i, j, k) && cell_of(g, i, j, k) == 1;
}
static int is_solid(const pfo_grid* g, int i, int j, int k) {
  return !in_cells(g, i, j, k) || cell_of(g, i, j, k) == 2;
}
static int is_air(const pfo_grid* g, int i, int j, int k) {
  return in_cells(g, i, j, k) && cell_of(g, i, j, k) == 0;
}

/* collectCellsWithMarker (src/driver/sparse_ops3d_common.h:65-85): the cells
 * with the marker, ascending in c = i + nx*(j + ny*k).  A dense scan in
 * linear order yields exactly the sorted list. */
int pfo_collect_cells(const pfo_grid* g, int marker, int* out, size_t* n) {
  if (!g || !n) return -1;
  size_t cnt = 0;
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i)
        if (cell_of(g, i, j, k) == marker) {
          if (out) out[cnt] = i + g->nx * (j + g->ny * k);
          ++cnt;
        }
  *n = cnt;
  return 0;
}

static int lower_index(const int* sorted, int n, int key) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = lo + (hi - lo) / 2;
    if (sorted[mid] < key) lo = mid + 1; else hi = mid;
  }
  return (lo < n && sorted[lo] == key) ? lo : -1;
}

static double dot_seq(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int t = 0; t < n; ++t) s += a[t] * b[t];
  return s;
}

int pfo_project(pfo_grid* g, const pfo_phase* pp, double dt, const pfo_solve_cfg* cfg,
                pfo_solve_stats* st) {
  if (!g || !pp || !cfg) return -1;
  pfo_solve_stats local;
  memset(&local, 0, sizeof(local));
  local.pin_cell = -1;
  pfo_clear_field(g, PFO_P);

  size_t ncell = 0;
  pfo_collect_cells(g, 1, NULL, &ncell);
  const int N = (int)ncell;
  local.n_cells = N;
  if (N == 0) { if (st) *st = local; return 0; }
  int* cells = (int*)malloc(sizeof(int) * (size_t)N);
  pfo_collect_cells(g, 1, cells, &ncell);

  static const int OI[6] = {1, -1, 0, 0, 0, 0};
  static const int OJ[6] = {0, 0, 1, -1, 0, 0};
  static const int OK[6] = {0, 0, 0, 0, 1, -1};
  const double scale = dt / (g->dx * g->dx);
  const int nx = g->nx, ny = g->ny;

  /* pin the first cell iff no fluid cell has an air neighbour (:250-264) */
  int pin = -1, touches_air = 0;
  for (int t = 0; t < N && !touches_air; ++t) {
    const int i = cells[t] % nx, q = cells[t] / nx, j = q % ny, k = q / ny;
    for (int d = 0; d < 6; ++d)
      if (is_air(g, i + OI[d], j + OJ[d], k + OK[d])) { touches_air = 1; break; }
  }
  if (!touches_air) pin = cells[0];
  local.pin_cell = pin;

  const size_t NN = ncell;
  double* x = (double*)calloc(NN, sizeof(double));
  double* r = (double*)calloc((size_t)N, sizeof(double));
  double* z = (double*)calloc((size_t)N, sizeof(double));
  double* pd = (double*)calloc((size_t)N, sizeof(double));
  double* Ap = (double*)calloc((size_t)N, sizeof(double));
  double* diag = (double*)calloc((size_t)N, sizeof(double));
  int* nbr = (int*)malloc(sizeof(int) * 6 * (size_t)N);
  double* coef = (double*)calloc(6 * (size_t)N, sizeof(double));

  /* right-hand side: -div(u)/dx + c_div, solid-side faces read as zero (:266-283) */
  for (int t = 0; t < N; ++t) {
    if (cells[t] == pin) { r[t] = 0.0; continue; }
    const int i = cells[t] % nx, q = cells[t] / nx, j = q % ny, k = q / ny;
    const double uR = is_solid(g, i + 1, j, k) ? 0.0 : (double)get(g, PFO_U, i + 1, j, k);
    const double uL = is_solid(g, i - 1, j, k) ? 0.0 : (double)get(g, PFO_U, i, j, k);
    const double vT = is_solid(g, i, j + 1, k) ? 0.0 : (double)get(g, PFO_V, i, j + 1, k);
    const double vB = is_solid(g, i, j - 1, k) ? 0.0 : (double)get(g, PFO_V, i, j, k);
    const double wU = is_solid(g, i, j, k + 1) ? 0.0 : (double)get(g, PFO_W, i, j, k + 1);
    const double wD = is_solid(g, i, j, k - 1) ? 0.0 : (double)get(g, PFO_W, i, j, k);
    r[t] = -((uR - uL) + (vT - vB) + (wU - wD)) / g->dx + cfg->c_div;
  }

  /* assembly: beta of each face from its raw mass (:285-313) */
  for (int t = 0; t < N; ++t) {
    const int i = cells[t] % nx, q = cells[t] / nx, j = q % ny, k = q / ny;
    const double fb[6] = {
      pfo_beta_from_raw(get(g, PFO_MU, i + 1, j, k), pp),
      pfo_beta_from_raw(get(g, PFO_MU, i, j, k), pp),
      pfo_beta_from_raw(get(g, PFO_MV, i, j + 1, k), pp),
      pfo_beta_from_raw(get(g, PFO_MV, i, j, k), pp),
      pfo_beta_from_raw(get(g, PFO_MW, i, j, k + 1), pp),
      pfo_beta_from_raw(get(g, PFO_MW, i, j, k), pp)};
    for (int d = 0; d < 6; ++d) {
      nbr[6 * t + d] = -1;
      const int a = i + OI[d], b = j + OJ[d], c = k + OK[d];
      if (is_solid(g, a, b, c)) continue;
      diag[t] += fb[d];
      coef[6 * t + d] = fb[d];
      const int nc = a + nx * (b + ny * c);
      if (is_fluid(g, a, b, c) && nc != pin) nbr[6 * t + d] = lower_index(cells, N, nc);
    }
  }

  /* Jacobi PCG in FP64 (:315-364), optional relative tolerance */
  double res0 = 0.0;
  for (int t = 0; t < N; ++t) res0 = fmax(res0, fabs(r[t]));
  double tol = cfg->abs_tol;
  if (cfg->rel_tol > 0.0 && cfg->rel_tol * res0 > tol) tol = cfg->rel_tol * res0;
  local.res0 = res0;
  local.res_final = res0;
  local.tol_effective = tol;
  if (res0 >= tol) {
    for (int t = 0; t < N; ++t) {
      const double dd = cells[t] == pin ? 1.0 : scale * diag[t];
      z[t] = dd > 0.0 ? r[t] / dd : 0.0;
    }
    memcpy(pd, z, sizeof(double) * NN);
    double rz = dot_seq(r, z, N);
    for (int it = 0; it < cfg->max_iter; ++it) {
      for (int t = 0; t < N; ++t) {
        if (cells[t] == pin) { Ap[t] = pd[t]; continue; }
        double off = 0.0;
        for (int d = 0; d < 6; ++d)
          if (nbr[6 * t + d] >= 0) off += coef[6 * t + d] * pd[nbr[6 * t + d]];
        Ap[t] = scale * (diag[t] * pd[t] - off);
      }
      const double pAp = dot_seq(pd, Ap, N);
      if (fabs(pAp) < 1e-30) { local.breakdown = 1; break; }
      const double alpha = rz / pAp;
      for (int t = 0; t < N; ++t) {
        x[t] += alpha * pd[t];
        r[t] -= alpha * Ap[t];
      }
      double res = 0.0;
      for (int t = 0; t < N; ++t) res = fmax(res, fabs(r[t]));
      local.iterations = it + 1;
      local.res_final = res;
      if (res < tol) { local.converged = 1; break; }
      for (int t = 0; t < N; ++t) {
        const double dd = cells[t] == pin ? 1.0 : scale * diag[t];
        z[t] = dd > 0.0 ? r[t] / dd : 0.0;
      }
      const double rzn = dot_seq(r, z, N);
      const double beta = rzn / rz;
      rz = rzn;
      for (int t = 0; t < N; ++t) pd[t] = z[t] + beta * pd[t];
    }
  } else {
    local.converged = 1;
  }

  /* pressure write-back (:366-372) */
  for (int t = 0; t < N; ++t) {
    const int i = cells[t] % nx, q = cells[t] / nx, j = q % ny, k = q / ny;
    *ref(g, PFO_P, i, j, k) = (float)x[t];
  }

  /* velocity update on faces next to fluid cells (:374-422); faces are
   * independent, so a lattice sweep visits the same set as the sorted lists */
  const double s = dt / g->dx;
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 1; i < g->nx; ++i) {
        const int lf = is_fluid(g, i - 1, j, k), rf = is_fluid(g, i, j, k);
        if (!lf && !rf) continue;
        if (is_solid(g, i - 1, j, k) || is_solid(g, i, j, k)) { *ref(g, PFO_U, i, j, k) = 0.0f; continue; }
        const double pl = lf ? (double)get(g, PFO_P, i - 1, j, k) : 0.0;
        const double pr = rf ? (double)get(g, PFO_P, i, j, k) : 0.0;
        const float cur = get(g, PFO_U, i, j, k);
        *ref(g, PFO_U, i, j, k) = cur - (float)(s * pfo_beta_from_raw(get(g, PFO_MU, i, j, k), pp) * (pr - pl));
      }
  for (int k = 0; k < g->nz; ++k)
    for (int j = 1; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const int bf = is_fluid(g, i, j - 1, k), tf = is_fluid(g, i, j, k);
        if (!bf && !tf) continue;
        if (is_solid(g, i, j - 1, k) || is_solid(g, i, j, k)) { *ref(g, PFO_V, i, j, k) = 0.0f; continue; }
        const double pb = bf ? (double)get(g, PFO_P, i, j - 1, k) : 0.0;
        const double pt = tf ? (double)get(g, PFO_P, i, j, k) : 0.0;
        const float cur = get(g, PFO_V, i, j, k);
        *ref(g, PFO_V, i, j, k) = cur - (float)(s * pfo_beta_from_raw(get(g, PFO_MV, i, j, k), pp) * (pt - pb));
      }
  for (int k = 1; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const int df = is_fluid(g, i, j, k - 1), uf = is_fluid(g, i, j, k);
        if (!df && !uf) continue;
        if (is_solid(g, i, j, k - 1) || is_solid(g, i, j, k)) { *ref(g, PFO_W, i, j, k) = 0.0f; continue; }
        const double pdn = df ? (double)get(g, PFO_P, i, j, k - 1) : 0.0;
        const double pup = uf ? (double)get(g, PFO_P, i, j, k) : 0.0;
        const float cur = get(g, PFO_W, i, j, k);
        *ref(g, PFO_W, i, j, k) = cur - (float)(s * pfo_beta_from_raw(get(g, PFO_MW, i, j, k), pp) * (pup - pdn));
      }

  free(cells); free(x); free(r); free(z); free(pd); free(Ap); free(diag); free(nbr); free(coef);
  if (st) *st = local;
  return 0;
}

/* ------------------------------------------------------------------ */
/* G2P and advection (src/driver/sparse_ops3d_tp.cpp:155-232,          */
/* src/driver/sparse_ops3d_common.h:30-63)                             */
/* ------------------------------------------------------------------ */

/* sampleField: clamped trilinear interpolation, FP64 weights, float result. */
static float sample(const pfo_grid* g, int f, double gx, double gy, double gz) {
  const int X = g->dim[f][0], Y = g->dim[f][1], Z = g->dim[f][2];
  const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
  const double fx = gx - i0, fy = gy - j0, fz = gz - k0;
  const double wx[2] = {1.0 - fx, fx}, wy[2] = {1.0 - fy, fy}, wz[2] = {1.0 - fz, fz};
  double s = 0.0;
  for (int dk = 0; dk < 2; ++dk)
    for (int dj = 0; dj < 2; ++dj)
      for (int di = 0; di < 2; ++di) {
        int a = i0 + di, b = j0 + dj, c = k0 + dk;
        a = a < 0 ? 0 : (a > X - 1 ? X - 1 : a);
        b = b < 0 ? 0 : (b > Y - 1 ? Y - 1 : b);
        c = c < 0 ? 0 : (c > Z - 1 ? Z - 1 : c);
        s += wx[di] * wy[dj] * wz[dk] * get(g, f, a, b, c);
      }
  return (float)s;
}

static void sample_velocity(const pfo_grid* g, double px, double py, double pz, double out[3]) {
  out[0] = sample(g, PFO_U, px, py - 0.5, pz - 0.5);
  out[1] = sample(g, PFO_V, px - 0.5, py, pz - 0.5);
  out[2] = sample(g, PFO_W, px - 0.5, py - 0.5, pz);
}

int pfo_g2p(const pfo_grid* g, const pfo_grid* saved, size_t n, const double* pos, double* vel,
            const unsigned char* type, double aL, double aG) {
  if (!g || !saved || (n && (!pos || !vel || !type))) return -1;
  for (size_t p = 0; p < n; ++p) {
    const double a = type[p] == 0 ? aL : aG;
    const double px = (pos[3 * p + 0] - g->ox) / g->dx;
    const double py = (pos[3 * p + 1] - g->oy) / g->dx;
    const double pz = (pos[3 * p + 2] - g->oz) / g->dx;
    double cur[3], old[3];
    sample_velocity(g, px, py, pz, cur);
    sample_velocity(saved, px, py, pz, old);
    for (int c = 0; c < 3; ++c) {
      const double flip = vel[3 * p + c] + (cur[c] - old[c]);
      vel[3 * p + c] = flip * a + cur[c] * (1.0 - a);
    }
  }
  return 0;
}

static void velocity_at(const pfo_grid* g, const double q[3], double out[3]) {
  sample_velocity(g, (q[0] - g->ox) / g->dx, (q[1] - g->oy) / g->dx, (q[2] - g->oz) / g->dx, out);
}

int pfo_advect(const pfo_grid* g, size_t n, double* pos, const unsigned char* type,
               const double* vel, const double* vol, double dt, int order,
               pfo_clamp_stats* st, double* escape_out, size_t* n_escape) {
  if (!g || (n && (!pos || !type))) return -1;
  const double lo[3] = {g->ox + 0.5 * g->dx, g->oy + 0.5 * g->dx, g->oz + 0.5 * g->dx};
  const double hi[3] = {g->ox + (g->nx - 0.5) * g->dx, g->oy + (g->ny - 0.5) * g->dx,
                        g->oz + (g->nz - 0.5) * g->dx};
  pfo_clamp_stats cs;
  memset(&cs, 0, sizeof(cs));
  size_t nesc = 0;
  for (size_t p = 0; p < n; ++p) {
    const double x0[3] = {pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]};
    double nxt[3], k1[3], k2[3];
    velocity_at(g, x0, k1);
    if (order == 3) {
      /* advectRK3 (:192-197) */
      double m1[3], m2[3], k3[3];
      for (int c = 0; c < 3; ++c) m1[c] = x0[c] + k1[c] * (0.5 * dt);
      velocity_at(g, m1, k2);
      for (int c = 0; c < 3; ++c) m2[c] = (x0[c] - k1[c] * dt) + k2[c] * (2.0 * dt);
      velocity_at(g, m2, k3);
      for (int c = 0; c < 3; ++c) nxt[c] = x0[c] + ((k1[c] + k2[c] * 4.0) + k3[c]) * (dt / 6.0);
    } else {
      /* advectMidpoint (:185-190) */
      double mid[3];
      for (int c = 0; c < 3; ++c) mid[c] = x0[c] + k1[c] * (0.5 * dt);
      velocity_at(g, mid, k2);
      for (int c = 0; c < 3; ++c) nxt[c] = x0[c] + k2[c] * dt;
    }
    /* boundary clamp and escape statistics (:204-231, particle_escape3d.h:59-79) */
    int low[3], high[3];
    for (int c = 0; c < 3; ++c) {
      low[c] = nxt[c] < lo[c];
      high[c] = nxt[c] > hi[c];
      nxt[c] = fmax(lo[c], fmin(hi[c], nxt[c]));
    }
    const int clamped = low[0] || high[0] || low[1] || high[1] || low[2] || high[2];
    if (clamped) {
      if (type[p] == 0) ++cs.clamped_liquid; else if (type[p] == 1) ++cs.clamped_gas;
      cs.x_lo += low[0]; cs.x_hi += high[0];
      cs.y_lo += low[1]; cs.y_hi += high[1];
      cs.z_lo += low[2]; cs.z_hi += high[2];
      if (escape_out && vel && vol) {
        double* rec = escape_out + 8 * nesc;
        rec[0] = type[p];
        rec[1] = nxt[0]; rec[2] = nxt[1]; rec[3] = nxt[2];
        rec[4] = vel[3 * p]; rec[5] = vel[3 * p + 1]; rec[6] = vel[3 * p + 2];
        rec[7] = vol[p];
      }
      ++nesc;
    }
    pos[3 * p] = nxt[0]; pos[3 * p + 1] = nxt[1]; pos[3 * p + 2] = nxt[2];
  }
  if (st) *st = cs;
  if (n_escape) *n_escape = nesc;
  return 0;
}

/* ------------------------------------------------------------------ */
/* One solver step in SparseSim3DTP::step() order                      */
/* (src/driver/sparse_sim3d_tp.cpp:854-884) with particle adaptivity,  */
/* diagnostics, surface tension and secondary particles off (their     */
/* defaults, src/driver/sparse_sim3d_tp.h:29-160).                     */
/* ------------------------------------------------------------------ */

int pfo_step(pfo_grid* g, pfo_grid* saved, size_t n, double* pos, double* vel,
             const unsigned char* type, const double* vol, const pfo_phase* pp,
             const pfo_step_cfg* cfg, pfo_solve_stats* sst, pfo_clamp_stats* cst) {
  if (!g || !saved || !pp || !cfg) return -1;
  if (pfo_mark_cells(g, n, pos)) return -1;
  if (pfo_p2g(g, n, pos, vel, type, vol, pp, cfg->Vp)) return -1;
  pfo_grid_copy(saved, g);
  pfo_apply_gravity(g, cfg->dt, cfg->gravity);
  pfo_apply_wall_boundary(g);
  pfo_solve_cfg sc = {cfg->cg_iters, cfg->cg_tol, cfg->cg_rel_tol, cfg->c_div};
  pfo_project(g, pp, cfg->dt, &sc, sst);
  pfo_g2p(g, saved, n, pos, vel, type, cfg->alpha_l, cfg->alpha_g);
  return pfo_advect(g, n, pos, type, vel, vol, cfg->dt, cfg->advect_order, cst, NULL, NULL);
}

/* ------------------------------------------------------------------ */
/* Particle adaptivity (src/driver/particle_adaptivity3d.h)            */
/* ------------------------------------------------------------------ */

/* ParticleCellDomain3D::particleCell (particle_adaptivity3d.h:36-47): finite
 * position, truncating (int) casts of (x - o) / dx, inside the grid. */
static int adapt_cell(const pfo_grid* g, const double* x, int* i, int* j, int* k) {
  if (!isfinite(x[0]) || !isfinite(x[1]) || !isfinite(x[2])) return 0;
  *i = (int)((x[0] - g->ox) / g->dx);
  *j = (int)((x[1] - g->oy) / g->dx);
  *k = (int)((x[2] - g->oz) / g->dx);
  return in_cells(g, *i, *j, *k);
}

static size_t lin_cell(const pfo_grid* g, int i, int j, int k) {
  return (size_t)i + (size_t)g->nx * ((size_t)j + (size_t)g->ny * (size_t)k);
}

/* mix32 (particle_adaptivity3d.h:75-82): the 32-bit integer finaliser */
static unsigned mix32(unsigned x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

/* particleScore (particle_adaptivity3d.h:84-102): cell and 1/1024-cell
 * quantised in-cell position hashed with the seed */
unsigned pfo_particle_score(const pfo_grid* g, const double* x, int i, int j, int k, unsigned seed) {
  const int qx = (int)((x[0] - (g->ox + i * g->dx)) / g->dx * 1024.0);
  const int qy = (int)((x[1] - (g->oy + j * g->dx)) / g->dx * 1024.0);
  const int qz = (int)((x[2] - (g->oz + k * g->dx)) / g->dx * 1024.0);
  unsigned h = seed;
  h ^= mix32((unsigned)i + 0x9e3779b9u);
  h ^= mix32((unsigned)j + 0x85ebca6bu);
  h ^= mix32((unsigned)k + 0xc2b2ae35u);
  h ^= mix32((unsigned)(qx & 2047) + 0x27d4eb2fu);
  h ^= mix32((unsigned)(qy & 2047) + 0x165667b1u);
  h ^= mix32((unsigned)(qz & 2047) + 0xd3a2646cu);
  return mix32(h);
}

/* slotScore (particle_adaptivity3d.h:104-109) */
unsigned pfo_slot_score(size_t cell, int slot, unsigned seed) {
  unsigned h = seed;
  h ^= mix32((unsigned)cell + 0x68bc21ebu);
  h ^= mix32((unsigned)slot + 0x02e5be93u);
  return mix32(h);
}

/* Particles3DTP::eraseIf (src/particles/particles3d_tp.h:13-35): survivors
 * keep their order */
static size_t keep_only(size_t n, double* pos, double* vel, unsigned char* type, double* vol,
                        const unsigned char* keep) {
  size_t w = 0;
  for (size_t r = 0; r < n; ++r) {
    if (!keep[r]) continue;
    if (w != r) {
      memcpy(pos + 3 * w, pos + 3 * r, 3 * sizeof(double));
      memcpy(vel + 3 * w, vel + 3 * r, 3 * sizeof(double));
      type[w] = type[r];
      vol[w] = vol[r];
    }
    ++w;
  }
  return w;
}

/* any flag set in the (2r+1)^3 box around (i, j, k), clipped to the grid */
static int any_in_box(const pfo_grid* g, const unsigned char* flag, int i, int j, int k, int r) {
  for (int kk = k - r; kk <= k + r; ++kk) {
    if (kk < 0 || kk >= g->nz) continue;
    for (int jj = j - r; jj <= j + r; ++jj) {
      if (jj < 0 || jj >= g->ny) continue;
      for (int ii = i - r; ii <= i + r; ++ii) {
        if (ii < 0 || ii >= g->nx) continue;
        if (flag[lin_cell(g, ii, jj, kk)]) return 1;
      }
    }
  }
  return 0;
}

/* applyNarrowBandAir (particle_adaptivity3d.h:111-166): gas particles (type 1)
 * survive only in a valid cell within `radius` cells (Chebyshev) of a cell
 * holding a liquid particle; nothing happens when no cell holds liquid. */
int pfo_narrow_band_air(const pfo_grid* g, size_t* n, double* pos, double* vel, unsigned char* type, double* vol,
                        int radius, pfo_band_stats* st) {
  memset(st, 0, sizeof(*st));
  const size_t nc = (size_t)g->nx * g->ny * g->nz;
  unsigned char* liquid = (unsigned char*)calloc(nc ? nc : 1, 1);
  unsigned char* keep = (unsigned char*)malloc(*n ? *n : 1);
  if (!liquid || !keep) { free(liquid); free(keep); return -1; }
  for (size_t p = 0; p < *n; ++p) {
    int i, j, k;
    if (type[p] != 0 || !adapt_cell(g, pos + 3 * p, &i, &j, &k)) continue;
    unsigned char* f = &liquid[lin_cell(g, i, j, k)];
    if (!*f) { *f = 1; ++st->liquid_cells; }
  }
  if (st->liquid_cells > 0) {
    const int r = radius > 0 ? radius : 0;
    for (size_t p = 0; p < *n; ++p) {
      keep[p] = 1;
      if (type[p] != 1) continue;
      ++st->gas_before;
      int i, j, k;
      keep[p] = adapt_cell(g, pos + 3 * p, &i, &j, &k) && any_in_box(g, liquid, i, j, k, r);
      if (keep[p]) ++st->gas_after;
    }
    const size_t m = keep_only(*n, pos, vel, type, vol, keep);
    st->removed = (int)(*n - m);
    *n = m;
  }
  free(liquid);
  free(keep);
  return 0;
}

typedef struct { size_t index, cell; unsigned score; double volume; } coarse_entry;

static int coarse_less(const void* a, const void* b) {
  const coarse_entry* x = (const coarse_entry*)a;
  const coarse_entry* y = (const coarse_entry*)b;
  if (x->cell != y->cell) return x->cell < y->cell ? -1 : 1;
  if (x->score != y->score) return x->score < y->score ? -1 : 1;
  return x->index < y->index ? -1 : (x->index > y->index);
}

/* applyTypedParticleCoarsening (particle_adaptivity3d.h:168-248): per cell
 * the `target` particles of type ptype with the lowest (score, index) stay
 * and share the cell's summed volume (summed in that order); the others of
 * that type, and those of that type outside the grid, are erased. */
int pfo_coarsen_particles(const pfo_grid* g, size_t* n, double* pos, double* vel, unsigned char* type, double* vol,
                          int ptype, int target, unsigned seed, pfo_coarsen_stats* st) {
  memset(st, 0, sizeof(*st));
  const size_t tgt = (size_t)(target > 1 ? target : 1);
  coarse_entry* e = (coarse_entry*)malloc((*n ? *n : 1) * sizeof(coarse_entry));
  unsigned char* keep = (unsigned char*)calloc(*n ? *n : 1, 1);
  if (!e || !keep) { free(e); free(keep); return -1; }
  size_t ne = 0;
  for (size_t p = 0; p < *n; ++p) {
    if (type[p] != (unsigned char)ptype) continue;
    ++st->before;
    int i, j, k;
    if (!adapt_cell(g, pos + 3 * p, &i, &j, &k)) continue;
    e[ne].index = p;
    e[ne].cell = lin_cell(g, i, j, k);
    e[ne].score = pfo_particle_score(g, pos + 3 * p, i, j, k, seed);
    e[ne].volume = vol[p];
    ++ne;
  }
  qsort(e, ne, sizeof(coarse_entry), coarse_less);
  for (size_t a = 0; a < ne;) {
    size_t b = a + 1;
    while (b < ne && e[b].cell == e[a].cell) ++b;
    ++st->cells;
    const size_t count = b - a;
    if (count > tgt) ++st->overfull_cells;
    const size_t keep_count = count < tgt ? count : tgt;
    double sum = 0.0;
    for (size_t t = a; t < b; ++t) sum += e[t].volume;
    const double kept = keep_count > 0 ? sum / (double)keep_count : 0.0;
    for (size_t t = 0; t < keep_count; ++t) {
      keep[e[a + t].index] = 1;
      vol[e[a + t].index] = kept;
      ++st->after;
    }
    a = b;
  }
  for (size_t p = 0; p < *n; ++p)
    if (type[p] != (unsigned char)ptype) keep[p] = 1;
  const size_t m = keep_only(*n, pos, vel, type, vol, keep);
  st->removed = (int)(*n - m);
  *n = m;
  free(e);
  free(keep);
  return 0;
}

/* applyLiquidParticleRefill (particle_adaptivity3d.h:250-374): every cell
 * holding fewer than `target` liquid particles (near gas within
 * interface_radius, when interface_only) gets target - count new liquid
 * particles at sub-cell centres taken in slotScore order, with the cell's mean
 * liquid velocity; the cell's liquid volume is split evenly over old and new.
 * Cells are visited in linear order against an optional budget. */
int pfo_refill_liquid(const pfo_grid* g, size_t* n, size_t cap, double* pos, double* vel, unsigned char* type,
                      double* vol, int target, unsigned seed, int interface_only, int interface_radius, int max_added,
                      pfo_refill_stats* st) {
  memset(st, 0, sizeof(*st));
  const int tgt = target > 1 ? target : 1;
  const size_t nc = (size_t)g->nx * g->ny * g->nz;
  const size_t n0 = *n;
  int* count = (int*)calloc(nc + 1, sizeof(int));
  size_t* start = (size_t*)calloc(nc + 1, sizeof(size_t));
  size_t* list = (size_t*)malloc((n0 ? n0 : 1) * sizeof(size_t));
  unsigned char* gas = (unsigned char*)calloc(nc ? nc : 1, 1);
  long long* cell_of_p = (long long*)malloc((n0 ? n0 : 1) * sizeof(long long));
  if (!count || !start || !list || !gas || !cell_of_p) {
    free(count); free(start); free(list); free(gas); free(cell_of_p);
    return -1;
  }
  /* liquid particles per cell, in particle order */
  for (size_t p = 0; p < n0; ++p) {
    int i, j, k;
    cell_of_p[p] = -1;
    if (!adapt_cell(g, pos + 3 * p, &i, &j, &k)) continue;
    const size_t c = lin_cell(g, i, j, k);
    if (type[p] == 0) {
      cell_of_p[p] = (long long)c;
      ++count[c];
    } else if (type[p] == 1) {
      gas[c] = 1;
    }
  }
  for (size_t c = 0; c < nc; ++c) start[c + 1] = start[c] + (size_t)count[c];
  {
    size_t* fill = (size_t*)malloc((nc ? nc : 1) * sizeof(size_t));
    if (!fill) { free(count); free(start); free(list); free(gas); free(cell_of_p); return -1; }
    memcpy(fill, start, nc * sizeof(size_t));
    for (size_t p = 0; p < n0; ++p)
      if (cell_of_p[p] >= 0) list[fill[cell_of_p[p]]++] = p;
    free(fill);
  }
  /* the total to add, for the capacity check before anything changes */
  const int r = interface_radius > 0 ? interface_radius : 0;
  long long budget = max_added > 0 ? max_added : 2147483647LL;
  size_t to_add_total = 0;
  {
    long long b = budget;
    for (size_t c = 0; c < nc; ++c) {
      const int cnt = count[c];
      if (cnt <= 0 || cnt >= tgt) continue;
      const int i = (int)(c % (size_t)g->nx), j = (int)((c / (size_t)g->nx) % (size_t)g->ny),
                k = (int)(c / ((size_t)g->nx * (size_t)g->ny));
      if (interface_only && !any_in_box(g, gas, i, j, k, r)) continue;
      if (b <= 0) continue;
      const long long want = tgt - cnt, add = want < b ? want : b;
      to_add_total += (size_t)add;
      b -= add;
    }
  }
  if (n0 + to_add_total > cap) {
    free(count); free(start); free(list); free(gas); free(cell_of_p);
    return -1;
  }
  for (size_t c = 0; c < nc; ++c) {
    const int cnt = count[c];
    if (cnt <= 0) continue;
    ++st->cells;
    st->before += cnt;
    st->after += cnt;
    const int i = (int)(c % (size_t)g->nx), j = (int)((c / (size_t)g->nx) % (size_t)g->ny),
              k = (int)(c / ((size_t)g->nx * (size_t)g->ny));
    const int near = any_in_box(g, gas, i, j, k, r);
    if (near) ++st->interface_cells;
    if (interface_only && !near) continue;
    if (cnt >= tgt) continue;
    ++st->underfull_cells;
    if (budget <= 0) { st->budget_limited = 1; continue; }
    double vsum = 0.0, u[3] = {0.0, 0.0, 0.0};
    for (size_t t = start[c]; t < start[c + 1]; ++t) {
      const size_t p = list[t];
      vsum += vol[p];
      for (int a = 0; a < 3; ++a) u[a] += vel[3 * p + a];
    }
    const double inv = 1.0 / (double)cnt;
    const double avg[3] = {u[0] * inv, u[1] * inv, u[2] * inv};
    int slots[8] = {0, 1, 2, 3, 4, 5, 6, 7};
    for (int a = 1; a < 8; ++a) { /* insertion sort by (slotScore, slot) */
      const int s = slots[a];
      const unsigned ss = pfo_slot_score(c, s, seed);
      int b = a - 1;
      while (b >= 0) {
        const unsigned sb = pfo_slot_score(c, slots[b], seed);
        if (sb < ss || (sb == ss && slots[b] < s)) break;
        slots[b + 1] = slots[b];
        --b;
      }
      slots[b + 1] = s;
    }
    const int want = tgt - cnt;
    const int add = (long long)want < budget ? want : (int)budget;
    if (add < want) st->budget_limited = 1;
    const double split = vsum / (double)(cnt + add);
    for (size_t t = start[c]; t < start[c + 1]; ++t) vol[list[t]] = split;
    for (int a = 0; a < add; ++a) {
      const int s = slots[a & 7];
      const double sx = 0.25 + 0.5 * (double)(s & 1);
      const double sy = 0.25 + 0.5 * (double)((s >> 1) & 1);
      const double sz = 0.25 + 0.5 * (double)((s >> 2) & 1);
      const size_t q = (*n)++;
      pos[3 * q + 0] = g->ox + ((double)i + sx) * g->dx;
      pos[3 * q + 1] = g->oy + ((double)j + sy) * g->dx;
      pos[3 * q + 2] = g->oz + ((double)k + sz) * g->dx;
      for (int d = 0; d < 3; ++d) vel[3 * q + d] = avg[d];
      type[q] = 0;
      vol[q] = split;
      ++st->added;
      ++st->after;
    }
    budget -= add;
  }
  free(count); free(start); free(list); free(gas); free(cell_of_p);
  return 0;
}

/* ------------------------------------------------------------------ */
/* Interface diagnostics (src/driver/interface_diagnostics3d.cpp)      */
/* ------------------------------------------------------------------ */

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* sparseCellPhi (interface_diagnostics3d.cpp:138-148): the mean phase field of
 * the cell's six face raw masses; 0 outside the grid */
static double cell_phi(const pfo_grid* g, const pfo_phase* pp, int i, int j, int k) {
  if (!in_cells(g, i, j, k)) return 0.0;
  double sum = 0.0;
  sum += pfo_phi_from_raw(get(g, PFO_MU, i, j, k), pp);
  sum += pfo_phi_from_raw(get(g, PFO_MU, i + 1, j, k), pp);
  sum += pfo_phi_from_raw(get(g, PFO_MV, i, j, k), pp);
  sum += pfo_phi_from_raw(get(g, PFO_MV, i, j + 1, k), pp);
  sum += pfo_phi_from_raw(get(g, PFO_MW, i, j, k), pp);
  sum += pfo_phi_from_raw(get(g, PFO_MW, i, j, k + 1), pp);
  return sum / 6.0;
}

/* sparsePhiClamped (:150-156) */
static double phi_clamped(const pfo_grid* g, const pfo_phase* pp, int i, int j, int k) {
  return cell_phi(g, pp, clampi(i, 0, g->nx - 1), clampi(j, 0, g->ny - 1), clampi(k, 0, g->nz - 1));
}

/* sparseGradient (:158-175): central differences of the clamped phi, one-sided
 * at the walls */
static void phi_gradient(const pfo_grid* g, const pfo_phase* pp, int i, int j, int k, double out[3]) {
  const int im = clampi(i - 1, 0, g->nx - 1), ip = clampi(i + 1, 0, g->nx - 1);
  const int jm = clampi(j - 1, 0, g->ny - 1), jp = clampi(j + 1, 0, g->ny - 1);
  const int km = clampi(k - 1, 0, g->nz - 1), kp = clampi(k + 1, 0, g->nz - 1);
  const double dx = g->dx;
  out[0] = (phi_clamped(g, pp, ip, j, k) - phi_clamped(g, pp, im, j, k)) / ((ip - im > 1 ? ip - im : 1) * dx);
  out[1] = (phi_clamped(g, pp, i, jp, k) - phi_clamped(g, pp, i, jm, k)) / ((jp - jm > 1 ? jp - jm : 1) * dx);
  out[2] = (phi_clamped(g, pp, i, j, kp) - phi_clamped(g, pp, i, j, km)) / ((kp - km > 1 ? kp - km : 1) * dx);
}

static double vlen(const double v[3]) { return sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]); }

/* sparseNormal / normalizeGradient (:177-186): zero below |grad| = 1e-12 */
static void phi_normal(const pfo_grid* g, const pfo_phase* pp, int i, int j, int k, double out[3]) {
  double gr[3];
  phi_gradient(g, pp, i, j, k, gr);
  const double mag = vlen(gr);
  if (mag <= 1e-12 || !isfinite(mag)) {
    out[0] = out[1] = out[2] = 0.0;
    return;
  }
  const double s = 1.0 / mag;
  out[0] = gr[0] * s;
  out[1] = gr[1] * s;
  out[2] = gr[2] * s;
}

/* sparseCurvature (:188-208): divergence of the normal */
static double phi_curvature(const pfo_grid* g, const pfo_phase* pp, int i, int j, int k) {
  const int im = clampi(i - 1, 0, g->nx - 1), ip = clampi(i + 1, 0, g->nx - 1);
  const int jm = clampi(j - 1, 0, g->ny - 1), jp = clampi(j + 1, 0, g->ny - 1);
  const int km = clampi(k - 1, 0, g->nz - 1), kp = clampi(k + 1, 0, g->nz - 1);
  const double dx = g->dx;
  double nxm[3], nxp[3], nym[3], nyp[3], nzm[3], nzp[3];
  phi_normal(g, pp, im, j, k, nxm);
  phi_normal(g, pp, ip, j, k, nxp);
  phi_normal(g, pp, i, jm, k, nym);
  phi_normal(g, pp, i, jp, k, nyp);
  phi_normal(g, pp, i, j, km, nzm);
  phi_normal(g, pp, i, j, kp, nzp);
  return (nxp[0] - nxm[0]) / ((ip - im > 1 ? ip - im : 1) * dx) +
         (nyp[1] - nym[1]) / ((jp - jm > 1 ? jp - jm : 1) * dx) +
         (nzp[2] - nzm[2]) / ((kp - km > 1 ? kp - km : 1) * dx);
}

/* diagnoseSparseInterface3D (:363-379) with accumulate / finishStats
 * (:26-66): over the fluid cells in ascending linear order */
int pfo_interface_diagnostics(const pfo_grid* g, const pfo_phase* pp, pfo_interface_stats* st) {
  memset(st, 0, sizeof(*st));
  st->finite = 1;
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        if (cell_of(g, i, j, k) != 1) continue;
        const double phi = cell_phi(g, pp, i, j, k);
        double gr[3];
        phi_gradient(g, pp, i, j, k, gr);
        const double gm = vlen(gr);
        const double curv = phi_curvature(g, pp, i, j, k);
        if (!isfinite(phi) || !isfinite(gm) || !isfinite(curv)) {
          st->finite = 0;
          continue;
        }
        if (st->sample_cells == 0) {
          st->phi_min = phi;
          st->phi_max = phi;
        } else {
          st->phi_min = phi < st->phi_min ? phi : st->phi_min;
          st->phi_max = phi > st->phi_max ? phi : st->phi_max;
        }
        ++st->sample_cells;
        st->phi_mean += phi;
        if (!(phi > 0.05 && phi < 0.95)) continue;
        ++st->interface_cells;
        st->grad_mean += gm;
        st->grad_max = gm > st->grad_max ? gm : st->grad_max;
        const double ac = fabs(curv);
        st->curvature_abs_mean += ac;
        st->curvature_abs_max = ac > st->curvature_abs_max ? ac : st->curvature_abs_max;
      }
  if (st->sample_cells > 0) st->phi_mean /= (double)st->sample_cells;
  if (st->interface_cells > 0) {
    st->grad_mean /= (double)st->interface_cells;
    st->curvature_abs_mean /= (double)st->interface_cells;
  }
  st->surface_tension_candidate = st->finite && st->interface_cells > 0 && st->grad_max > 1e-5;
  return 0;
}

/* ------------------------------------------------------------------ */
/* Surface tension (src/driver/interface_diagnostics3d.cpp:405-447)    */
/* ------------------------------------------------------------------ */

static int interface_phi(double phi) { return phi > 0.05 && phi < 0.95; }

/* sparseSmoothedCurvature (:209-233): mean raw curvature of the interface
 * cells in the (2r+1)^3 clamped neighbourhood */
static double smoothed_curvature(const pfo_grid* g, const pfo_phase* pp, int i, int j, int k, double raw, int r) {
  if (r <= 0 || !isfinite(raw)) return raw;
  double sum = 0.0;
  int count = 0;
  for (int dz = -r; dz <= r; ++dz)
    for (int dy = -r; dy <= r; ++dy)
      for (int dx = -r; dx <= r; ++dx) {
        const int ni = clampi(i + dx, 0, g->nx - 1), nj = clampi(j + dy, 0, g->ny - 1),
                  nk = clampi(k + dz, 0, g->nz - 1);
        if (!interface_phi(cell_phi(g, pp, ni, nj, nk))) continue;
        const double c = phi_curvature(g, pp, ni, nj, nk);
        if (!isfinite(c)) continue;
        sum += c;
        ++count;
      }
  return count > 0 ? sum / (double)count : raw;
}

/* applySparseSurfaceTension3D (:405-447) with initSurfaceStats,
 * limitedDelta, accumulateSurfaceStats, finishSurfaceStats (:68-135): cells
 * in ascending order, each adding half its capillary velocity change to its
 * six faces where the face holds mass; the finite flag, once cleared, stops
 * every later update. */
int pfo_surface_tension(pfo_grid* g, const pfo_phase* pp, double dt, double strength, double max_delta_speed,
                        int smoothing_radius, pfo_surface_stats* st) {
  memset(st, 0, sizeof(*st));
  st->finite = 1;
  st->enabled = strength > 0.0 && dt > 0.0;
  st->strength = strength;
  st->max_delta_speed_limit = max_delta_speed;
  st->curvature_smoothing_radius = clampi(smoothing_radius, 0, 3);
  {
    const double rho_min = pp->rho_l < pp->rho_g ? pp->rho_l : pp->rho_g;
    const double kpi = 3.14159265358979323846;
    st->capillary_dt_limit = (g->dx <= 0.0 || strength <= 0.0 || rho_min <= 0.0 || !isfinite(rho_min))
                                 ? 0.0
                                 : sqrt((rho_min * g->dx * g->dx * g->dx) / (2.0 * kpi * strength));
  }
  st->capillary_stable = !st->enabled || st->capillary_dt_limit <= 0.0 || dt <= st->capillary_dt_limit + 1e-12;
  if (!st->enabled) return 0;
  const int r = st->curvature_smoothing_radius;
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        if (cell_of(g, i, j, k) != 1) continue;
        const double phi = cell_phi(g, pp, i, j, k);
        if (!interface_phi(phi)) continue;
        double gr[3];
        phi_gradient(g, pp, i, j, k, gr);
        if (vlen(gr) <= 1e-5) continue;
        const double raw = phi_curvature(g, pp, i, j, k);
        const double sm = smoothed_curvature(g, pp, i, j, k, raw, r);
        const double s = -strength * sm * dt;
        double d[3] = {gr[0] * s, gr[1] * s, gr[2] * s};
        const double mag0 = vlen(d);
        if (!isfinite(mag0)) {
          d[0] = d[1] = d[2] = 0.0;
        } else if (max_delta_speed > 0.0 && mag0 > max_delta_speed) {
          const double f = max_delta_speed / mag0;
          d[0] *= f;
          d[1] *= f;
          d[2] *= f;
        }
        const double mag = vlen(d);
        if (!isfinite(mag) || !isfinite(raw) || !isfinite(sm)) {
          st->finite = 0;
          continue;
        }
        ++st->applied_cells;
        st->mean_delta_speed += mag;
        st->max_delta_speed = mag > st->max_delta_speed ? mag : st->max_delta_speed;
        st->raw_curvature_abs_mean += fabs(raw);
        st->raw_curvature_abs_max = fabs(raw) > st->raw_curvature_abs_max ? fabs(raw) : st->raw_curvature_abs_max;
        st->smoothed_curvature_abs_mean += fabs(sm);
        st->smoothed_curvature_abs_max =
            fabs(sm) > st->smoothed_curvature_abs_max ? fabs(sm) : st->smoothed_curvature_abs_max;
        if (!st->finite) continue;
        if (get(g, PFO_MU, i, j, k) > 0.0f) *ref(g, PFO_U, i, j, k) += (float)(0.5 * d[0]);
        if (get(g, PFO_MU, i + 1, j, k) > 0.0f) *ref(g, PFO_U, i + 1, j, k) += (float)(0.5 * d[0]);
        if (get(g, PFO_MV, i, j, k) > 0.0f) *ref(g, PFO_V, i, j, k) += (float)(0.5 * d[1]);
        if (get(g, PFO_MV, i, j + 1, k) > 0.0f) *ref(g, PFO_V, i, j + 1, k) += (float)(0.5 * d[1]);
        if (get(g, PFO_MW, i, j, k) > 0.0f) *ref(g, PFO_W, i, j, k) += (float)(0.5 * d[2]);
        if (get(g, PFO_MW, i, j, k + 1) > 0.0f) *ref(g, PFO_W, i, j, k + 1) += (float)(0.5 * d[2]);
      }
  if (st->applied_cells > 0) {
    const double den = (double)st->applied_cells;
    st->mean_delta_speed /= den;
    st->raw_curvature_abs_mean /= den;
    st->smoothed_curvature_abs_mean /= den;
  }
  return 0;
}
