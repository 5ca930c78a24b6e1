/*
 * pf_oracle_mr.c -- CPU restatement of the reference's 2-level multires 3D
 * two-phase step (MRSim3DTP::step without its off-by-default options).
 *
 * TEST INFRASTRUCTURE ONLY: the checker the GPU multires path is compared
 * against; never linked into or called by the product library.
 *
 * Restated (paths relative to the adaptive-pf-flip source tree):
 *   layout                src/grid/multires_layout3d.h:25-162
 *   leaf cells / faces    src/grid/multires_scalar_grid3d.h:19-144,
 *                         src/grid/multires_mac_grid3d.h:35-189
 *   markCells, gravity,   src/driver/multires_sim3d_tp.cpp:23-99
 *   walls
 *   dynamic refinement    src/driver/multires_sim3d_tp.cpp:119-227, 577-669
 *   P2G, G2P, advection   src/driver/multires_ops3d_tp.cpp:13-355
 *   projection            src/pressure/multires_pressure3d.cpp:90-245 (cells,
 *                         coefficients), 749-1527 (rows, PCG with Jacobi,
 *                         adaptive restart and optional flexible beta,
 *                         velocity update)
 *   step order            src/driver/multires_sim3d_tp.cpp:671-733
 *
 * Representation: the layout is one flag per level-1 block (8^3 fine cells),
 * set when the block is split into its level-0 children.  Face fields are
 * dense float arrays over the fine face lattice (u: (nx+1, ny, nz), ...);
 * a fine face patch that is not on a leaf cell's boundary is never written and
 * reads 0, as MRMacGrid3D's maps return 0 for absent keys.  Markers and
 * pressure are stored per fine cell, each fine cell holding the value of the
 * leaf cell that contains it.  Every floating-point expression keeps the
 * reference's operation order, so the results equal the compiled reference's.
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "pf_oracle.h"

struct pfo_mr {
  int nx, ny, nz;
  double dx;
  int MX, MY, MZ;         /* level-1 block counts, ceil(n / 8) */
  unsigned char* refined; /* [MX*MY*MZ] */
  float* f[PFO_MR_NFACE]; /* u v w mu mv mw, then the saved u v w */
  float* mk;              /* per fine cell: marker of its leaf cell */
  float* p;               /* per fine cell: pressure of its leaf cell */
  /* updateDynamicRefinement state */
  int retained_valid, rx0, ry0, rz0, rx1, ry1, rz1;
  int last_fine_leaves, budget_limited;
};

/* ---- lattice helpers ---------------------------------------------------- */

static size_t face_count(const pfo_mr* m, int axis) {
  return (size_t)(m->nx + (axis == 0)) * (size_t)(m->ny + (axis == 1)) * (size_t)(m->nz + (axis == 2));
}
static size_t face_index(const pfo_mr* m, int axis, int i, int j, int k) {
  const size_t X = (size_t)(m->nx + (axis == 0)), Y = (size_t)(m->ny + (axis == 1));
  return (size_t)i + X * ((size_t)j + Y * (size_t)k);
}
static size_t cell_index(const pfo_mr* m, int i, int j, int k) {
  return (size_t)i + (size_t)m->nx * ((size_t)j + (size_t)m->ny * (size_t)k);
}
static int in_domain(const pfo_mr* m, int i, int j, int k) {
  return i >= 0 && i < m->nx && j >= 0 && j < m->ny && k >= 0 && k < m->nz;
}

/* the leaf cell holding fine cell (i, j, k) (in the domain): its level and
 * fine-cell origin; MRScalarGrid3D::cellAtFineCell via leafAtFineCell */
typedef struct {
  int level, x0, y0, z0;
} leaf_t;
static leaf_t leaf_of(const pfo_mr* m, int i, int j, int k) {
  leaf_t c;
  const int t = (i >> 3) + m->MX * ((j >> 3) + m->MY * (k >> 3));
  if (m->refined[t]) {
    c.level = 0;
    c.x0 = i;
    c.y0 = j;
    c.z0 = k;
  } else {
    c.level = 1;
    c.x0 = i & ~1;
    c.y0 = j & ~1;
    c.z0 = k & ~1;
  }
  return c;
}
static double leaf_h(const pfo_mr* m, int level) { return m->dx * (double)(1 << level); }

/* cell(g, i, j, k) / markerAtFineCell: 2 outside the domain */
static int marker_at(const pfo_mr* m, int i, int j, int k) {
  if (!in_domain(m, i, j, k)) return 2;
  return (int)(m->mk[cell_index(m, i, j, k)] + 0.5f);
}

/* write v into every fine cell of the leaf cell holding (i, j, k) */
static void set_leaf(const pfo_mr* m, float* a, int i, int j, int k, float v) {
  const leaf_t c = leaf_of(m, i, j, k);
  const int s = 1 << c.level;
  for (int z = c.z0; z < c.z0 + s && z < m->nz; ++z)
    for (int y = c.y0; y < c.y0 + s && y < m->ny; ++y)
      for (int x = c.x0; x < c.x0 + s && x < m->nx; ++x) a[cell_index(m, x, y, z)] = v;
}

/* Is the fine face patch (axis; i, j, k) on the boundary of a leaf cell
 * (MRMacGrid3D::enumerateFaces)?  Its neighbours along the axis are fine
 * cells c-1 and c; the patch is a face of the leaf holding c-1 if it lies at
 * that leaf's far side (clipped to the domain), and of the leaf holding c if
 * it lies at that leaf's near side. */
static int face_valid(const pfo_mr* m, int axis, int i, int j, int k) {
  const int n[3] = {m->nx, m->ny, m->nz};
  int c[3] = {i, j, k};
  const int pos = c[axis];
  if (pos < 0 || pos > n[axis]) return 0;
  for (int d = 0; d < 3; ++d)
    if (d != axis && (c[d] < 0 || c[d] >= n[d])) return 0;
  if (pos >= 1) {
    c[axis] = pos - 1;
    const leaf_t L = leaf_of(m, c[0], c[1], c[2]);
    const int o[3] = {L.x0, L.y0, L.z0};
    int far = o[axis] + (1 << L.level);
    if (far > n[axis]) far = n[axis];
    if (far == pos) return 1;
  }
  if (pos < n[axis]) {
    c[axis] = pos;
    const leaf_t R = leaf_of(m, c[0], c[1], c[2]);
    const int o[3] = {R.x0, R.y0, R.z0};
    if (o[axis] == pos) return 1;
  }
  return 0;
}

/* ---- creation ----------------------------------------------------------- */

pfo_mr* pfo_mr_create(int nx, int ny, int nz, double dx) {
  if (nx <= 0 || ny <= 0 || nz <= 0 || !(dx > 0.0)) return NULL;
  pfo_mr* m = (pfo_mr*)calloc(1, sizeof(pfo_mr));
  if (!m) return NULL;
  m->nx = nx;
  m->ny = ny;
  m->nz = nz;
  m->dx = dx;
  m->MX = (nx + 7) / 8;
  m->MY = (ny + 7) / 8;
  m->MZ = (nz + 7) / 8;
  m->refined = (unsigned char*)calloc((size_t)m->MX * m->MY * m->MZ, 1);
  int ok = m->refined != NULL;
  for (int q = 0; q < PFO_MR_NFACE; ++q) {
    m->f[q] = (float*)calloc(face_count(m, q % 3), sizeof(float));
    ok = ok && m->f[q];
  }
  m->mk = (float*)calloc((size_t)nx * ny * nz, sizeof(float));
  m->p = (float*)calloc((size_t)nx * ny * nz, sizeof(float));
  if (!ok || !m->mk || !m->p) {
    pfo_mr_destroy(m);
    return NULL;
  }
  return m;
}

void pfo_mr_destroy(pfo_mr* m) {
  if (!m) return;
  free(m->refined);
  for (int q = 0; q < PFO_MR_NFACE; ++q) free(m->f[q]);
  free(m->mk);
  free(m->p);
  free(m);
}

void pfo_mr_dims(const pfo_mr* m, int* blocks3) {
  blocks3[0] = m->MX;
  blocks3[1] = m->MY;
  blocks3[2] = m->MZ;
}

int pfo_mr_get_levels(const pfo_mr* m, unsigned char* refined) {
  memcpy(refined, m->refined, (size_t)m->MX * m->MY * m->MZ);
  return 0;
}

int pfo_mr_set_levels(pfo_mr* m, const unsigned char* refined) {
  const size_t n = (size_t)m->MX * m->MY * m->MZ;
  for (size_t t = 0; t < n; ++t) m->refined[t] = refined[t] ? 1 : 0;
  return 0;
}

int pfo_mr_get_face(const pfo_mr* m, int field, float* out) {
  if (field < 0 || field >= PFO_MR_NFACE) return -1;
  memcpy(out, m->f[field], face_count(m, field % 3) * sizeof(float));
  return 0;
}

int pfo_mr_set_face(pfo_mr* m, int field, const float* in) {
  if (field < 0 || field >= PFO_MR_NFACE) return -1;
  memcpy(m->f[field], in, face_count(m, field % 3) * sizeof(float));
  return 0;
}

int pfo_mr_get_cells(const pfo_mr* m, float* marker, float* pressure) {
  const size_t n = (size_t)m->nx * m->ny * m->nz;
  if (marker) memcpy(marker, m->mk, n * sizeof(float));
  if (pressure) memcpy(pressure, m->p, n * sizeof(float));
  return 0;
}

int pfo_mr_face_valid(const pfo_mr* m, int axis, unsigned char* out) {
  const int X = m->nx + (axis == 0), Y = m->ny + (axis == 1), Z = m->nz + (axis == 2);
  for (int k = 0; k < Z; ++k)
    for (int j = 0; j < Y; ++j)
      for (int i = 0; i < X; ++i) out[face_index(m, axis, i, j, k)] = (unsigned char)face_valid(m, axis, i, j, k);
  return 0;
}

/* ---- layout (src/grid/multires_layout3d.h:53-94; multires_sim3d_tp.cpp:158-180) */

/* number of level-0 children intersecting the domain of level-1 block t */
static int children_in_domain(const pfo_mr* m, int bx, int by, int bz) {
  int n = 0;
  for (int cz = 0; cz < 2; ++cz)
    for (int cy = 0; cy < 2; ++cy)
      for (int cx = 0; cx < 2; ++cx) {
        const int x0 = (2 * bx + cx) * 4, y0 = (2 * by + cy) * 4, z0 = (2 * bz + cz) * 4;
        if (x0 < m->nx && y0 < m->ny && z0 < m->nz) ++n;
      }
  return n;
}

/* refineFineCellBox on the current flags: level-1 blocks overlapping the
 * (clamped) box are split; level-0 blocks stay */
static void refine_box(pfo_mr* m, int x0, int y0, int z0, int x1, int y1, int z1) {
#define CLAMP(v, n) ((v) < 0 ? 0 : (v) > (n) ? (n) : (v))
  x0 = CLAMP(x0, m->nx);
  y0 = CLAMP(y0, m->ny);
  z0 = CLAMP(z0, m->nz);
  x1 = CLAMP(x1, m->nx);
  y1 = CLAMP(y1, m->ny);
  z1 = CLAMP(z1, m->nz);
#undef CLAMP
  if (!(x0 < x1 && y0 < y1 && z0 < z1)) return;
  for (int bz = 0; bz < m->MZ; ++bz)
    for (int by = 0; by < m->MY; ++by)
      for (int bx = 0; bx < m->MX; ++bx) {
        const int s = 8;
        const int bx0 = bx * s, by0 = by * s, bz0 = bz * s;
        const int bx1 = m->nx < bx0 + s ? m->nx : bx0 + s;
        const int by1 = m->ny < by0 + s ? m->ny : by0 + s;
        const int bz1 = m->nz < bz0 + s ? m->nz : bz0 + s;
        if (bx0 < x1 && bx1 > x0 && by0 < y1 && by1 > y0 && bz0 < z1 && bz1 > z0)
          m->refined[bx + m->MX * (by + m->MY * bz)] = 1;
      }
}

int pfo_mr_set_layout(pfo_mr* m, const int* boxes, int nbox) {
  memset(m->refined, 0, (size_t)m->MX * m->MY * m->MZ);
  for (int b = 0; b < nbox; ++b)
    refine_box(m, boxes[6 * b + 0], boxes[6 * b + 1], boxes[6 * b + 2], boxes[6 * b + 3], boxes[6 * b + 4],
               boxes[6 * b + 5]);
  return 0;
}

int pfo_mr_count_fine_leaves(const pfo_mr* m) {
  int n = 0;
  for (int bz = 0; bz < m->MZ; ++bz)
    for (int by = 0; by < m->MY; ++by)
      for (int bx = 0; bx < m->MX; ++bx)
        if (m->refined[bx + m->MX * (by + m->MY * bz)]) n += children_in_domain(m, bx, by, bz);
  return n;
}

/* ---- dynamic refinement (src/driver/multires_sim3d_tp.cpp:119-227, 577-669) */

typedef struct {
  int x0, y0, z0, x1, y1, z1, valid;
} box3;

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }

static void include_box(box3* b, int x0, int y0, int z0, int x1, int y1, int z1) {
  if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;
  if (!b->valid) {
    box3 n = {x0, y0, z0, x1, y1, z1, 1};
    *b = n;
    return;
  }
  b->x0 = imin(b->x0, x0);
  b->y0 = imin(b->y0, y0);
  b->z0 = imin(b->z0, z0);
  b->x1 = imax(b->x1, x1);
  b->y1 = imax(b->y1, y1);
  b->z1 = imax(b->z1, z1);
}

static box3 clamp_box(const pfo_mr* m, box3 b) {
  if (!b.valid) return b;
  b.x0 = imax(0, imin(m->nx, b.x0));
  b.y0 = imax(0, imin(m->ny, b.y0));
  b.z0 = imax(0, imin(m->nz, b.z0));
  b.x1 = imax(0, imin(m->nx, b.x1));
  b.y1 = imax(0, imin(m->ny, b.y1));
  b.z1 = imax(0, imin(m->nz, b.z1));
  b.valid = b.x0 < b.x1 && b.y0 < b.y1 && b.z0 < b.z1;
  return b;
}

static box3 expand_box(const pfo_mr* m, box3 b, int pad) {
  if (!b.valid) return b;
  pad = imax(0, pad);
  box3 e = {b.x0 - pad, b.y0 - pad, b.z0 - pad, b.x1 + pad, b.y1 + pad, b.z1 + pad, 1};
  return clamp_box(m, e);
}

static int contains_box(box3 o, box3 in) {
  return o.valid && in.valid && o.x0 <= in.x0 && o.y0 <= in.y0 && o.z0 <= in.z0 && o.x1 >= in.x1 &&
         o.y1 >= in.y1 && o.z1 >= in.z1;
}

/* countLevel(0) of layoutWithFineBox(base, b) */
static int fine_leaves_for_box(pfo_mr* m, box3 b) {
  unsigned char* save = (unsigned char*)malloc((size_t)m->MX * m->MY * m->MZ);
  memcpy(save, m->refined, (size_t)m->MX * m->MY * m->MZ);
  memset(m->refined, 0, (size_t)m->MX * m->MY * m->MZ);
  if (b.valid) refine_box(m, b.x0, b.y0, b.z0, b.x1, b.y1, b.z1);
  const int n = pfo_mr_count_fine_leaves(m);
  memcpy(m->refined, save, (size_t)m->MX * m->MY * m->MZ);
  free(save);
  return n;
}

static int box_extent(box3 b, int axis) { return axis == 0 ? b.x1 - b.x0 : axis == 1 ? b.y1 - b.y0 : b.z1 - b.z0; }

static int shrink_largest_axis(box3* b, double cx, double cy, double cz) {
  int axis = 0;
  if (box_extent(*b, 1) > box_extent(*b, axis)) axis = 1;
  if (box_extent(*b, 2) > box_extent(*b, axis)) axis = 2;
  if (box_extent(*b, axis) <= 1) return 0;
  if (axis == 0) {
    if ((b->x1 - cx) >= (cx - b->x0)) --b->x1;
    else ++b->x0;
  } else if (axis == 1) {
    if ((b->y1 - cy) >= (cy - b->y0)) --b->y1;
    else ++b->y0;
  } else {
    if ((b->z1 - cz) >= (cz - b->z0)) --b->z1;
    else ++b->z0;
  }
  b->valid = b->x0 < b->x1 && b->y0 < b->y1 && b->z0 < b->z1;
  return b->valid;
}

static box3 fit_budget(pfo_mr* m, box3 b, int max_fine, int* limited) {
  *limited = 0;
  if (!b.valid || max_fine <= 0) return b;
  if (fine_leaves_for_box(m, b) <= max_fine) return b;
  *limited = 1;
  const double cx = 0.5 * (double)(b.x0 + b.x1), cy = 0.5 * (double)(b.y0 + b.y1), cz = 0.5 * (double)(b.z0 + b.z1);
  while (fine_leaves_for_box(m, b) > max_fine)
    if (!shrink_largest_axis(&b, cx, cy, cz)) break;
  return b;
}

int pfo_mr_update_refinement(pfo_mr* m, const pfo_mr_dynamic* dyn, size_t n, const double* pos,
                             const unsigned char* type) {
  if (!dyn->enabled) return 0;
  int mn[3] = {m->nx, m->ny, m->nz}, mx[3] = {-1, -1, -1};
  int gmn[3] = {m->nx, m->ny, m->nz}, gmx[3] = {-1, -1, -1};
  for (size_t q = 0; q < n; ++q) {
    const double* x = pos + 3 * q;
    if (!isfinite(x[0]) || !isfinite(x[1]) || !isfinite(x[2])) continue;
    const int c[3] = {(int)(x[0] / m->dx), (int)(x[1] / m->dx), (int)(x[2] / m->dx)};
    if (!in_domain(m, c[0], c[1], c[2])) continue;
    for (int d = 0; d < 3; ++d) {
      mn[d] = imin(mn[d], c[d]);
      mx[d] = imax(mx[d], c[d]);
      if (type[q] == 1) {
        gmn[d] = imin(gmn[d], c[d]);
        gmx[d] = imax(gmx[d], c[d]);
      }
    }
  }
  box3 desired = {0, 0, 0, 0, 0, 0, 0};
  if (mx[0] >= 0) {
    const int pad = imax(0, dyn->particle_padding);
    include_box(&desired, mn[0] - pad, mn[1] - pad, mn[2] - pad, mx[0] + pad + 1, mx[1] + pad + 1, mx[2] + pad + 1);
  }
  if (gmx[0] >= 0) {
    const int pad = imax(0, dyn->gas_padding);
    include_box(&desired, gmn[0] - pad, gmn[1] - pad, gmn[2] - pad, gmx[0] + pad + 1, gmx[1] + pad + 1,
                gmx[2] + pad + 1);
  }
  desired = clamp_box(m, desired);
  box3 target = {0, 0, 0, 0, 0, 0, 0};
  m->budget_limited = 0;
  if (desired.valid) {
    const box3 retained = {m->rx0, m->ry0, m->rz0, m->rx1, m->ry1, m->rz1, m->retained_valid};
    target = contains_box(retained, desired) ? retained : expand_box(m, desired, dyn->hysteresis_cells);
    target = fit_budget(m, target, dyn->max_fine_leaves, &m->budget_limited);
  }
  m->retained_valid = target.valid;
  if (target.valid) {
    m->rx0 = target.x0;
    m->ry0 = target.y0;
    m->rz0 = target.z0;
    m->rx1 = target.x1;
    m->ry1 = target.y1;
    m->rz1 = target.z1;
  }
  memset(m->refined, 0, (size_t)m->MX * m->MY * m->MZ);
  if (target.valid) refine_box(m, target.x0, target.y0, target.z0, target.x1, target.y1, target.z1);
  m->last_fine_leaves = pfo_mr_count_fine_leaves(m);
  return 0;
}

void pfo_mr_refinement_state(const pfo_mr* m, int* out8) {
  out8[0] = m->retained_valid;
  out8[1] = m->rx0;
  out8[2] = m->ry0;
  out8[3] = m->rz0;
  out8[4] = m->rx1;
  out8[5] = m->ry1;
  out8[6] = m->rz1;
  out8[7] = m->budget_limited;
}

/* ---- markCells (src/driver/multires_sim3d_tp.cpp:40-73) ---------------- */

int pfo_mr_mark_cells(pfo_mr* m, size_t n, const double* pos) {
  const int nx = m->nx, ny = m->ny, nz = m->nz;
  memset(m->mk, 0, (size_t)nx * ny * nz * sizeof(float));
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j) {
      set_leaf(m, m->mk, 0, j, k, 2.0f);
      set_leaf(m, m->mk, nx - 1, j, k, 2.0f);
    }
  for (int k = 0; k < nz; ++k)
    for (int i = 0; i < nx; ++i) {
      set_leaf(m, m->mk, i, 0, k, 2.0f);
      set_leaf(m, m->mk, i, ny - 1, k, 2.0f);
    }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      set_leaf(m, m->mk, i, j, 0, 2.0f);
      set_leaf(m, m->mk, i, j, nz - 1, 2.0f);
    }
  for (size_t q = 0; q < n; ++q) {
    const int i = (int)(pos[3 * q] / m->dx), j = (int)(pos[3 * q + 1] / m->dx), k = (int)(pos[3 * q + 2] / m->dx);
    if (in_domain(m, i, j, k) && marker_at(m, i, j, k) != 2) set_leaf(m, m->mk, i, j, k, 1.0f);
  }
  return 0;
}

/* ---- P2G (src/driver/multires_ops3d_tp.cpp:20-130, 209-274) ------------- */

static double mr_kernel(double d2) {
  const double r = 1.5;
  const double q = d2 / (r * r);
  const double t = 1.0 - q;
  return t > 0.0 ? t * t * t : 0.0;
}
static int lo_range(double c, int lo, int hi) { return imax(lo, imin(hi, (int)floor(c - 1.5))); }
static int hi_range(double c, int lo, int hi) { return imax(lo, imin(hi, (int)ceil(c + 1.5))); }

typedef struct {
  size_t at;
  double w;
} wface;

/* collectWeightedFaces: the faces of one axis within the kernel radius that
 * are leaf-cell boundary patches, in (k, j, i) order, and their weight sum */
static double collect(const pfo_mr* m, int axis, double px, double py, double pz, wface* out, int* nout) {
  const double c[3] = {px, py, pz};
  int lo[3], hi[3];
  const int n[3] = {m->nx, m->ny, m->nz};
  for (int d = 0; d < 3; ++d) {
    const double s = d == axis ? c[d] : c[d] - 0.5;
    const int top = d == axis ? n[d] : n[d] - 1;
    lo[d] = lo_range(s, 0, top);
    hi[d] = hi_range(s, 0, top);
  }
  double sum = 0.0;
  int cnt = 0;
  for (int k = lo[2]; k <= hi[2]; ++k)
    for (int j = lo[1]; j <= hi[1]; ++j)
      for (int i = lo[0]; i <= hi[0]; ++i) {
        const double fx = axis == 0 ? (double)i : (double)i + 0.5;
        const double fy = axis == 1 ? (double)j : (double)j + 0.5;
        const double fz = axis == 2 ? (double)k : (double)k + 0.5;
        const double dx = px - fx, dy = py - fy, dz = pz - fz;
        const double w = mr_kernel(dx * dx + dy * dy + dz * dz);
        if (w <= 0.0) continue;
        if (!face_valid(m, axis, i, j, k)) continue;
        out[cnt].at = face_index(m, axis, i, j, k);
        out[cnt].w = w;
        ++cnt;
        sum += w;
      }
  *nout = cnt;
  return sum;
}

int pfo_mr_p2g(pfo_mr* m, size_t n, const double* pos, const double* vel, const unsigned char* type,
               const double* vol, const pfo_phase* pp, double Vp) {
  for (int q = 0; q < 6; ++q) memset(m->f[q], 0, face_count(m, q % 3) * sizeof(float));
  wface buf[125];
  for (size_t q = 0; q < n; ++q) {
    const double rho = type[q] == 0 ? pp->rho_l : pp->rho_g;
    const double mp = rho * Vp * vol[q];
    const double px = pos[3 * q] / m->dx, py = pos[3 * q + 1] / m->dx, pz = pos[3 * q + 2] / m->dx;
    for (int axis = 0; axis < 3; ++axis) {
      int cnt = 0;
      const double wsum = collect(m, axis, px, py, pz, buf, &cnt);
      if (!(wsum > 0.0)) continue;
      float* mom = m->f[axis];
      float* mass = m->f[3 + axis];
      for (int e = 0; e < cnt; ++e) {
        const double w = buf[e].w / wsum;
        if (w <= 0.0) continue;
        mom[buf[e].at] += (float)(w * mp * vel[3 * q + axis]);
        mass[buf[e].at] += (float)(w * mp);
      }
    }
  }
  for (int axis = 0; axis < 3; ++axis) {
    float* u = m->f[axis];
    const float* mu = m->f[3 + axis];
    const size_t nf = face_count(m, axis);
    for (size_t e = 0; e < nf; ++e)
      if (mu[e] > 0.0f) u[e] /= mu[e];
  }
  return 0;
}

/* ---- gravity and walls (src/driver/multires_sim3d_tp.cpp:75-99) -------- */

int pfo_mr_apply_gravity(pfo_mr* m, double dt, double gravity) {
  float* v = m->f[1];
  const float* mv = m->f[4];
  for (int k = 0; k < m->nz; ++k)
    for (int j = 0; j <= m->ny; ++j)
      for (int i = 0; i < m->nx; ++i) {
        if (!face_valid(m, 1, i, j, k)) continue;
        const size_t e = face_index(m, 1, i, j, k);
        if (mv[e] > 0.0f) v[e] = v[e] + (float)(dt * gravity);
      }
  return 0;
}

int pfo_mr_apply_walls(pfo_mr* m) {
  const int n[3] = {m->nx, m->ny, m->nz};
  for (int axis = 0; axis < 3; ++axis) {
    const int X = m->nx + (axis == 0), Y = m->ny + (axis == 1), Z = m->nz + (axis == 2);
    for (int k = 0; k < Z; ++k)
      for (int j = 0; j < Y; ++j)
        for (int i = 0; i < X; ++i) {
          const int c = axis == 0 ? i : axis == 1 ? j : k;
          if (c == 0 || c == 1 || c == n[axis] - 1 || c == n[axis])
            if (face_valid(m, axis, i, j, k)) m->f[axis][face_index(m, axis, i, j, k)] = 0.0f;
        }
  }
  return 0;
}

/* ---- projection (src/pressure/multires_pressure3d.cpp) ----------------- */

typedef struct {
  leaf_t key;
  double h, volume;
} pcell;

/* betaFromRawMass (:94-99) */
static double beta_from_raw_mass(double raw, const pfo_phase* pp) {
  const double rmin = log(pp->rho_l / pp->rho_g) * pp->rho_g * pp->rho_tilde_0;
  const double invden = 1.0 / (pp->alpha_phi * pp->rho_tilde_0 * pp->rho_l);
  double phi;
  if (raw < rmin) {
    phi = 0.0;
  } else {
    const double s = sqrt((raw - rmin) * invden);
    phi = 1.0 < s ? 1.0 : s;
  }
  return 1.0 / (phi * pp->rho_l + (1.0 - phi) * pp->rho_g);
}

/* the fluid leaf cells in leafCells order (levels ascending, then blocks by
 * (bx, by, bz), then cells by (lz, ly, lx)); index map per fine cell */
static int fluid_cells(const pfo_mr* m, pcell** out, int* idx) {
  const size_t nc = (size_t)m->nx * m->ny * m->nz;
  for (size_t e = 0; e < nc; ++e) idx[e] = -1;
  pcell* cells = (pcell*)malloc(nc * sizeof(pcell) + 1);
  int N = 0;
  /* level 0: blocks of 4^3 fine cells inside refined level-1 blocks */
  const int BX = (m->nx + 3) / 4, BY = (m->ny + 3) / 4, BZ = (m->nz + 3) / 4;
  for (int bx = 0; bx < BX; ++bx)
    for (int by = 0; by < BY; ++by)
      for (int bz = 0; bz < BZ; ++bz) {
        if (!m->refined[(bx >> 1) + m->MX * ((by >> 1) + m->MY * (bz >> 1))]) continue;
        for (int lz = 0; lz < 4; ++lz)
          for (int ly = 0; ly < 4; ++ly)
            for (int lx = 0; lx < 4; ++lx) {
              const int x = 4 * bx + lx, y = 4 * by + ly, z = 4 * bz + lz;
              if (!in_domain(m, x, y, z)) continue;
              if (marker_at(m, x, y, z) != 1) continue;
              leaf_t c = {0, x, y, z};
              cells[N].key = c;
              cells[N].h = leaf_h(m, 0);
              cells[N].volume = cells[N].h * cells[N].h * cells[N].h;
              idx[cell_index(m, x, y, z)] = N;
              ++N;
            }
      }
  /* level 1: the unsplit blocks, 4^3 cells of 2^3 fine cells */
  for (int bx = 0; bx < m->MX; ++bx)
    for (int by = 0; by < m->MY; ++by)
      for (int bz = 0; bz < m->MZ; ++bz) {
        if (m->refined[bx + m->MX * (by + m->MY * bz)]) continue;
        for (int lz = 0; lz < 4; ++lz)
          for (int ly = 0; ly < 4; ++ly)
            for (int lx = 0; lx < 4; ++lx) {
              const int x = 8 * bx + 2 * lx, y = 8 * by + 2 * ly, z = 8 * bz + 2 * lz;
              if (!in_domain(m, x, y, z)) continue;
              if (marker_at(m, x, y, z) != 1) continue;
              leaf_t c = {1, x, y, z};
              cells[N].key = c;
              cells[N].h = leaf_h(m, 1);
              cells[N].volume = cells[N].h * cells[N].h * cells[N].h;
              for (int dz = 0; dz < 2; ++dz)
                for (int dy = 0; dy < 2; ++dy)
                  for (int dx = 0; dx < 2; ++dx)
                    if (in_domain(m, x + dx, y + dy, z + dz)) idx[cell_index(m, x + dx, y + dy, z + dz)] = N;
              ++N;
            }
      }
  *out = cells;
  return N;
}

/* visitCellFaces (:102-137): fine patches on the cell's boundary, with the
 * fine neighbour cell across each and the outward sign */
typedef struct {
  int axis, fi, fj, fk;  /* face patch */
  int ni, nj, nk;        /* neighbour fine cell */
  double sign;
} visit_t;

static int visit_faces(const pfo_mr* m, const leaf_t* c, visit_t* v) {
  const int s = 1 << c->level;
  const int x0 = c->x0, y0 = c->y0, z0 = c->z0, x1 = x0 + s, y1 = y0 + s, z1 = z0 + s;
  const int cx0 = imax(0, x0), cx1 = imin(m->nx, x1), cy0 = imax(0, y0), cy1 = imin(m->ny, y1);
  const int cz0 = imax(0, z0), cz1 = imin(m->nz, z1);
  int n = 0;
  for (int z = cz0; z < cz1; ++z)
    for (int y = cy0; y < cy1; ++y) {
      visit_t a = {0, x0, y, z, x0 - 1, y, z, -1.0};
      visit_t b = {0, imin(x1, m->nx), y, z, x1, y, z, 1.0};
      v[n++] = a;
      v[n++] = b;
    }
  for (int z = cz0; z < cz1; ++z)
    for (int x = cx0; x < cx1; ++x) {
      visit_t a = {1, x, y0, z, x, y0 - 1, z, -1.0};
      visit_t b = {1, x, imin(y1, m->ny), z, x, y1, z, 1.0};
      v[n++] = a;
      v[n++] = b;
    }
  for (int y = cy0; y < cy1; ++y)
    for (int x = cx0; x < cx1; ++x) {
      visit_t a = {2, x, y, z0, x, y, z0 - 1, -1.0};
      visit_t b = {2, x, y, imin(z1, m->nz), x, y, z1, 1.0};
      v[n++] = a;
      v[n++] = b;
    }
  return n;
}

/* neighborDistance (:214-225) */
static double neighbor_distance(const pfo_mr* m, const pcell* c, int i, int j, int k) {
  double other = c->h;
  if (in_domain(m, i, j, k)) other = leaf_h(m, leaf_of(m, i, j, k).level);
  return 0.5 * c->h + 0.5 * other;
}

static double face_value(const pfo_mr* m, int axis, int i, int j, int k) {
  return (double)m->f[axis][face_index(m, axis, i, j, k)];
}
static double face_mass(const pfo_mr* m, int axis, int i, int j, int k) {
  return (double)m->f[3 + axis][face_index(m, axis, i, j, k)];
}

typedef struct {
  int n, cap;
  int* col;
  double* coeff;
} offrow;

static double dotv(const double* a, const double* b, int n) {
  double s = 0.0;
  for (int i = 0; i < n; ++i) s += a[i] * b[i];
  return s;
}
static double max_abs(const double* v, int n) {
  double m = 0.0;
  for (int i = 0; i < n; ++i)
    if (isfinite(v[i])) m = m > fabs(v[i]) ? m : fabs(v[i]);
  return m;
}

int pfo_mr_project(pfo_mr* m, const pfo_phase* pp, double dt, const pfo_mr_solve_cfg* cfg, pfo_mr_solve_stats* st) {
  pfo_mr_solve_stats S;
  memset(&S, 0, sizeof(S));
  S.pinned_cell = -1;
  S.max_iterations = cfg->max_iter;
  const size_t nc = (size_t)m->nx * m->ny * m->nz;
  int* idx = (int*)malloc(nc * sizeof(int));
  pcell* cells = NULL;
  const int N = fluid_cells(m, &cells, idx);
  S.active_cells = N;
  memset(m->p, 0, nc * sizeof(float));
  if (N == 0) {
    S.converged = 1;
    *st = S;
    free(idx);
    free(cells);
    return 0;
  }
  visit_t* vis = (visit_t*)malloc(sizeof(visit_t) * 6 * 4);
  /* findPinCell (:190-200) */
  int air = 0;
  for (int c = 0; c < N && !air; ++c) {
    const int nv = visit_faces(m, &cells[c].key, vis);
    for (int e = 0; e < nv; ++e)
      if (marker_at(m, vis[e].ni, vis[e].nj, vis[e].nk) == 0) air = 1;
  }
  const int pin = air ? -1 : 0;
  S.pinned_cell = pin;
  /* rows (:792-822) */
  double* diag = (double*)calloc((size_t)N, sizeof(double));
  double* divg = (double*)calloc((size_t)N, sizeof(double));
  offrow* off = (offrow*)calloc((size_t)N, sizeof(offrow));
  const double area = m->dx * m->dx * 1.0 * 1.0;
  for (int c = 0; c < N; ++c) {
    off[c].col = (int*)malloc(24 * sizeof(int));
    off[c].coeff = (double*)malloc(24 * sizeof(double));
    if (c == pin) {
      diag[c] = 1.0;
      continue;
    }
    const int nv = visit_faces(m, &cells[c].key, vis);
    for (int e = 0; e < nv; ++e) {
      const visit_t* f = &vis[e];
      if (marker_at(m, f->ni, f->nj, f->nk) == 2) continue;
      double coeff = 0.0;
      const double dist = neighbor_distance(m, &cells[c], f->ni, f->nj, f->nk);
      if (!(dist <= 0.0 || cells[c].volume <= 0.0)) {
        const double beta = beta_from_raw_mass(face_mass(m, f->axis, f->fi, f->fj, f->fk), pp);
        coeff = dt * beta * area / dist / cells[c].volume;
      }
      diag[c] += coeff;
      const int nidx = in_domain(m, f->ni, f->nj, f->nk) ? idx[cell_index(m, f->ni, f->nj, f->nk)] : -1;
      if (nidx >= 0 && nidx != pin) {
        off[c].col[off[c].n] = nidx;
        off[c].coeff[off[c].n] = coeff;
        off[c].n++;
      }
      const double v = face_value(m, f->axis, f->fi, f->fj, f->fk);
      divg[c] += f->sign * v * area / cells[c].volume;
    }
  }
  for (int c = 0; c < N; ++c)
    if (diag[c] > 0.0) {
      S.min_positive_diag = S.min_positive_diag == 0.0 ? diag[c] : fmin(S.min_positive_diag, diag[c]);
      S.max_diag = fmax(S.max_diag, diag[c]);
    }
  double* x = (double*)calloc((size_t)N, sizeof(double));
  double* rhs = (double*)calloc((size_t)N, sizeof(double));
  double* r = (double*)calloc((size_t)N, sizeof(double));
  double* z = (double*)calloc((size_t)N, sizeof(double));
  double* zp = (double*)calloc((size_t)N, sizeof(double));
  double* p = (double*)calloc((size_t)N, sizeof(double));
  double* Ap = (double*)calloc((size_t)N, sizeof(double));
  double res0 = 0.0;
  for (int c = 0; c < N; ++c) {
    rhs[c] = c == pin ? 0.0 : -divg[c] + cfg->c_div;
    r[c] = rhs[c];
    res0 = fmax(res0, fabs(r[c]));
  }
  S.initial_residual = S.final_residual = res0;
  const double abs_tol = fmax(0.0, cfg->abs_tol), rel_tol = fmax(0.0, cfg->rel_tol);
  const double eff = fmax(abs_tol, rel_tol * res0);
  S.effective_tolerance = eff;
  S.converged = res0 < eff;
#define APPLY_A(in, out)                                                       \
  for (int c = 0; c < N; ++c) {                                                \
    if (c == pin) {                                                            \
      (out)[c] = (in)[c];                                                      \
      continue;                                                                \
    }                                                                          \
    double o_ = 0.0;                                                           \
    for (int t = 0; t < off[c].n; ++t) o_ += off[c].coeff[t] * (in)[off[c].col[t]]; \
    (out)[c] = diag[c] * (in)[c] - o_;                                         \
  }
#define PRECOND()                                                              \
  for (int c = 0; c < N; ++c) z[c] = (cfg->jacobi && diag[c] > 0.0) ? r[c] / diag[c] : r[c];
  if (res0 >= eff) {
    PRECOND();
    for (int c = 0; c < N; ++c) p[c] = z[c];
    double rz = dotv(r, z, N);
    if (!isfinite(rz)) {
      S.breakdown = 1;
      S.final_residual = max_abs(r, N);
    }
    double prev = S.final_residual;
    for (int it = 0; !S.breakdown && it < cfg->max_iter; ++it) {
      APPLY_A(p, Ap);
      const double pAp = dotv(p, Ap, N);
      if (!isfinite(pAp) || fabs(pAp) < 1e-30) {
        S.breakdown = 1;
        S.final_residual = max_abs(r, N);
        break;
      }
      const double alpha = rz / pAp;
      if (!isfinite(alpha)) {
        S.breakdown = 1;
        S.final_residual = max_abs(r, N);
        break;
      }
      double res = 0.0;
      int finite_state = 1;
      for (int c = 0; c < N; ++c) {
        x[c] += alpha * p[c];
        r[c] -= alpha * Ap[c];
        finite_state = finite_state && isfinite(x[c]) && isfinite(r[c]);
        if (isfinite(r[c])) res = fmax(res, fabs(r[c]));
      }
      S.iterations = it + 1;
      S.final_residual = res;
      if (!finite_state || !isfinite(res)) {
        S.breakdown = 1;
        S.final_residual = max_abs(r, N);
        break;
      }
      if (res < eff) {
        S.converged = 1;
        break;
      }
      if (cfg->adaptive_restart && cfg->restart_growth > 0.0 && res > prev * cfg->restart_growth &&
          res > res0 * cfg->restart_growth && it + 1 < cfg->max_iter) {
        PRECOND();
        rz = dotv(r, z, N);
        if (!isfinite(rz)) {
          S.breakdown = 1;
          S.final_residual = max_abs(r, N);
          break;
        }
        for (int c = 0; c < N; ++c) p[c] = z[c];
        S.restarts++;
        prev = res;
        continue;
      }
      prev = res;
      memcpy(zp, z, (size_t)N * sizeof(double));
      PRECOND();
      const double rz_next = dotv(r, z, N);
      if (!isfinite(rz_next)) {
        S.breakdown = 1;
        S.final_residual = max_abs(r, N);
        break;
      }
      double beta = 0.0;
      if (rz != 0.0) {
        if (cfg->flexible_beta) {
          double num = 0.0;
          for (int c = 0; c < N; ++c) num += r[c] * (z[c] - zp[c]);
          beta = num / rz;
        } else {
          beta = rz_next / rz;
        }
      }
      if (!isfinite(beta)) {
        beta = 0.0;
        S.beta_resets++;
      }
      if (beta < 0.0) {
        beta = 0.0;
        S.beta_resets++;
      }
      rz = rz_next;
      for (int c = 0; c < N; ++c) p[c] = z[c] + beta * p[c];
    }
  }
#undef APPLY_A
#undef PRECOND
  /* g.p per leaf cell */
  for (int c = 0; c < N; ++c) set_leaf(m, m->p, cells[c].key.x0, cells[c].key.y0, cells[c].key.z0, (float)x[c]);
  /* velocity update (:1454-1524) */
  for (int axis = 0; axis < 3; ++axis) {
    const int X = m->nx + (axis == 0), Y = m->ny + (axis == 1), Z = m->nz + (axis == 2);
    for (int k = 0; k < Z; ++k)
      for (int j = 0; j < Y; ++j)
        for (int i = 0; i < X; ++i) {
          if (!face_valid(m, axis, i, j, k)) continue;
          const int li = i - (axis == 0), lj = j - (axis == 1), lk = k - (axis == 2);
          const int lm = marker_at(m, li, lj, lk), rm = marker_at(m, i, j, k);
          const int lf = lm == 1, rf = rm == 1;
          if (!lf && !rf) continue;
          float* u = &m->f[axis][face_index(m, axis, i, j, k)];
          if (lm == 2 || rm == 2) {
            *u = 0.0f;
            continue;
          }
          double dist = m->dx;
          const int ri = lf ? li : i, rj = lf ? lj : j, rk = lf ? lk : k;
          const int ref = in_domain(m, ri, rj, rk) ? idx[cell_index(m, ri, rj, rk)] : -1;
          if (ref >= 0) {
            const int oi = lf ? i : li, oj = lf ? j : lj, ok = lf ? k : lk;
            dist = neighbor_distance(m, &cells[ref], oi, oj, ok);
          }
          double pl = 0.0, pr = 0.0;
          if (lf) {
            const int a = in_domain(m, li, lj, lk) ? idx[cell_index(m, li, lj, lk)] : -1;
            pl = a >= 0 ? x[a] : 0.0;
          }
          if (rf) {
            const int b = in_domain(m, i, j, k) ? idx[cell_index(m, i, j, k)] : -1;
            pr = b >= 0 ? x[b] : 0.0;
          }
          const double beta = beta_from_raw_mass(face_mass(m, axis, i, j, k), pp);
          *u = (float)((double)*u - dt * beta * (pr - pl) / dist);
        }
  }
  for (int c = 0; c < N; ++c) {
    free(off[c].col);
    free(off[c].coeff);
  }
  free(off);
  free(diag);
  free(divg);
  free(x);
  free(rhs);
  free(r);
  free(z);
  free(zp);
  free(p);
  free(Ap);
  free(vis);
  free(cells);
  free(idx);
  *st = S;
  return 0;
}

/* ---- G2P and advection (src/driver/multires_ops3d_tp.cpp:132-207, 276-355) */

static double trilerp(double fx, double fy, double fz, const double v[2][2][2]) {
  double s = 0.0;
  for (int dz = 0; dz < 2; ++dz) {
    const double wz = dz == 0 ? 1.0 - fz : fz;
    for (int dy = 0; dy < 2; ++dy) {
      const double wy = dy == 0 ? 1.0 - fy : fy;
      for (int dx = 0; dx < 2; ++dx) {
        const double wx = dx == 0 ? 1.0 - fx : fx;
        s += wx * wy * wz * v[dx][dy][dz];
      }
    }
  }
  return s;
}

/* sampleU / sampleV / sampleW of face field `fld` (axis a) */
static double sample_axis(const pfo_mr* m, const float* fld, int axis, double x, double y, double z) {
  const double p[3] = {x / m->dx, y / m->dx, z / m->dx};
  int b[3];
  double fr[3];
  for (int d = 0; d < 3; ++d) {
    const double s = d == axis ? p[d] : p[d] - 0.5;
    b[d] = (int)floor(s);
    fr[d] = s - b[d];
  }
  const int top[3] = {m->nx - (axis != 0), m->ny - (axis != 1), m->nz - (axis != 2)};
  double v[2][2][2];
  for (int dz = 0; dz < 2; ++dz)
    for (int dy = 0; dy < 2; ++dy)
      for (int dx = 0; dx < 2; ++dx) {
        const int i = imax(0, imin(top[0], b[0] + dx));
        const int j = imax(0, imin(top[1], b[1] + dy));
        const int k = imax(0, imin(top[2], b[2] + dz));
        v[dx][dy][dz] = (double)fld[face_index(m, axis, i, j, k)];
      }
  return trilerp(fr[0], fr[1], fr[2], v);
}

int pfo_mr_g2p(const pfo_mr* m, size_t n, const double* pos, double* vel, const unsigned char* type, double aL,
               double aG) {
  for (size_t q = 0; q < n; ++q) {
    const double a = type[q] == 0 ? aL : aG;
    const double* x = pos + 3 * q;
    double cur[3], d[3];
    for (int ax = 0; ax < 3; ++ax) cur[ax] = sample_axis(m, m->f[ax], ax, x[0], x[1], x[2]);
    for (int ax = 0; ax < 3; ++ax) d[ax] = cur[ax] - sample_axis(m, m->f[6 + ax], ax, x[0], x[1], x[2]);
    for (int ax = 0; ax < 3; ++ax) {
      const double flip = vel[3 * q + ax] + d[ax];
      vel[3 * q + ax] = a * flip + (1.0 - a) * cur[ax];
    }
  }
  return 0;
}

static void sample_velocity(const pfo_mr* m, const double* x, double* out) {
  for (int ax = 0; ax < 3; ++ax) out[ax] = sample_axis(m, m->f[ax], ax, x[0], x[1], x[2]);
}

int pfo_mr_advect(const pfo_mr* m, size_t n, double* pos, const unsigned char* type, double dt, int order,
                  pfo_clamp_stats* st) {
  const double lo[3] = {0.5 * m->dx, 0.5 * m->dx, 0.5 * m->dx};
  const double hi[3] = {((double)m->nx - 0.5) * m->dx, ((double)m->ny - 0.5) * m->dx, ((double)m->nz - 0.5) * m->dx};
  pfo_clamp_stats s;
  memset(&s, 0, sizeof(s));
  for (size_t q = 0; q < n; ++q) {
    double* x = pos + 3 * q;
    double k1[3], k2[3], nx[3];
    sample_velocity(m, x, k1);
    if (order == 3) {
      double a[3], b[3], k3[3];
      for (int c = 0; c < 3; ++c) a[c] = x[c] + k1[c] * (0.5 * dt);
      sample_velocity(m, a, k2);
      for (int c = 0; c < 3; ++c) b[c] = x[c] - k1[c] * dt + k2[c] * (2.0 * dt);
      sample_velocity(m, b, k3);
      for (int c = 0; c < 3; ++c) nx[c] = x[c] + (k1[c] + k2[c] * 4.0 + k3[c]) * (dt / 6.0);
    } else {
      double mid[3];
      for (int c = 0; c < 3; ++c) mid[c] = x[c] + k1[c] * (0.5 * dt);
      sample_velocity(m, mid, k2);
      for (int c = 0; c < 3; ++c) nx[c] = x[c] + k2[c] * dt;
    }
    int l[3], h[3], any = 0;
    for (int c = 0; c < 3; ++c) {
      l[c] = nx[c] < lo[c];
      h[c] = nx[c] > hi[c];
      any = any || l[c] || h[c];
      x[c] = fmax(lo[c], fmin(hi[c], nx[c]));
    }
    /* ParticleEscapeStats3D::recordClamp */
    if (any) {
      if (type[q] == 0) s.clamped_liquid++;
      else if (type[q] == 1) s.clamped_gas++;
    }
    s.x_lo += l[0];
    s.x_hi += h[0];
    s.y_lo += l[1];
    s.y_hi += h[1];
    s.z_lo += l[2];
    s.z_hi += h[2];
  }
  if (st) *st = s;
  return 0;
}

/* ---- the step (src/driver/multires_sim3d_tp.cpp:671-733) --------------- */

int pfo_mr_step(pfo_mr* m, const pfo_mr_dynamic* dyn, size_t n, double* pos, double* vel,
                const unsigned char* type, const double* vol, const pfo_phase* pp, const pfo_mr_step_cfg* cfg,
                pfo_mr_solve_stats* sst, pfo_clamp_stats* cst) {
  if (dyn && dyn->enabled) pfo_mr_update_refinement(m, dyn, n, pos, type);
  pfo_mr_mark_cells(m, n, pos);
  pfo_mr_p2g(m, n, pos, vel, type, vol, pp, cfg->Vp);
  for (int a = 0; a < 3; ++a) memcpy(m->f[6 + a], m->f[a], face_count(m, a) * sizeof(float));
  pfo_mr_apply_gravity(m, cfg->dt, cfg->gravity);
  pfo_mr_apply_walls(m);
  pfo_mr_project(m, pp, cfg->dt, &cfg->solve, sst);
  pfo_mr_g2p(m, n, pos, vel, type, cfg->alpha_l, cfg->alpha_g);
  pfo_mr_advect(m, n, pos, type, cfg->dt, cfg->advect_order, cst);
  return 0;
}
