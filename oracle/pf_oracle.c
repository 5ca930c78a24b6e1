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
#include <stdlib.h>
#include <string.h>

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
  return v < 1.0 ? v : 1.0;
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
 * nonzero weight. */
static void preactivate(pfo_grid* g, int f, double gx, double gy, double gz) {
  const int X = g->dim[f][0], Y = g->dim[f][1], Z = g->dim[f][2];
  const int i0 = (int)floor(gx), j0 = (int)floor(gy), k0 = (int)floor(gz);
  for (int dk = -2; dk <= 3; ++dk)
    for (int dj = -2; dj <= 3; ++dj)
      for (int di = -2; di <= 3; ++di) {
        const int a = i0 + di, b = j0 + dj, c = k0 + dk;
        if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
        const double ex = gx - a, ey = gy - b, ez = gz - c;
        if (cubic_weight(ex * ex + ey * ey + ez * ez) <= 0.0) continue;
        activate(g, f, a, b, c);
      }
}

/* splatKernelColor (:42-75) without the colour filter: each node still
 * receives its contributions in particle-index order, which is the order the
 * reference's owning colour thread adds them in. */
static void splat(pfo_grid* g, int fmom, int fmass, double gx, double gy, double gz,
                  double mom, double mass) {
  const int X = g->dim[fmom][0], Y = g->dim[fmom][1], Z = g->dim[fmom][2];
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
  if (wsum <= 0.0) return;
  for (int dk = -2; dk <= 3; ++dk)
    for (int dj = -2; dj <= 3; ++dj)
      for (int di = -2; di <= 3; ++di) {
        const int a = i0 + di, b = j0 + dj, c = k0 + dk;
        if (a < 0 || a >= X || b < 0 || b >= Y || c < 0 || c >= Z) continue;
        const double ex = gx - a, ey = gy - b, ez = gz - c;
        const double w = cubic_weight(ex * ex + ey * ey + ez * ez) / wsum;
        if (w <= 0.0) continue;
        float* pm = ref(g, fmom, a, b, c);
        *pm += (float)(w * mom);
        float* pw = ref(g, fmass, a, b, c);
        *pw += (float)(w * mass);
      }
}

int pfo_p2g(pfo_grid* g, size_t n, const double* pos, const double* vel,
            const unsigned char* type, const double* vol, const pfo_phase* pp, double Vp) {
  if (!g || !pp || (n && (!pos || !vel || !type || !vol))) return -1;
  for (int f = PFO_U; f <= PFO_MW; ++f) pfo_clear_field(g, f);
  for (size_t p = 0; p < n; ++p) {
    const double px = (pos[3 * p + 0] - g->ox) / g->dx;
    const double py = (pos[3 * p + 1] - g->oy) / g->dx;
    const double pz = (pos[3 * p + 2] - g->oz) / g->dx;
    preactivate(g, PFO_U, px, py - 0.5, pz - 0.5);
    preactivate(g, PFO_MU, px, py - 0.5, pz - 0.5);
    preactivate(g, PFO_V, px - 0.5, py, pz - 0.5);
    preactivate(g, PFO_MV, px - 0.5, py, pz - 0.5);
    preactivate(g, PFO_W, px - 0.5, py - 0.5, pz);
    preactivate(g, PFO_MW, px - 0.5, py - 0.5, pz);
  }
  for (size_t p = 0; p < n; ++p) {
    const double rho = type[p] == 0 ? pp->rho_l : pp->rho_g;
    const double mp = rho * Vp * vol[p];
    const double px = (pos[3 * p + 0] - g->ox) / g->dx;
    const double py = (pos[3 * p + 1] - g->oy) / g->dx;
    const double pz = (pos[3 * p + 2] - g->oz) / g->dx;
    splat(g, PFO_U, PFO_MU, px, py - 0.5, pz - 0.5, mp * vel[3 * p + 0], mp);
    splat(g, PFO_V, PFO_MV, px - 0.5, py, pz - 0.5, mp * vel[3 * p + 1], mp);
    splat(g, PFO_W, PFO_MW, px - 0.5, py - 0.5, pz, mp * vel[3 * p + 2], mp);
  }
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
