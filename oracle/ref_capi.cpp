// ref_capi.cpp -- TEST INFRASTRUCTURE ONLY.
//
// A thin extern "C" wrapper that drives the UNMODIFIED adaptive-pf-flip
// reference (its sparse 3D two-phase sources compiled where they lie, see
// oracle/Makefile) so Python tests can feed it the same seeded inputs as the
// GPU path and the C restatement.  Nothing here reimplements reference
// arithmetic: every operation calls the reference's own public API
//   spP2G3D_tp / spProjectStepVC3D / spG2P3D_tp / spAdvect3D_tp
//     (src/driver/sparse_ops3d_tp.h:8-15)
//   SparseSim3DTP::step()   (src/driver/sparse_sim3d_tp.cpp:854-884)
//   calibrateRhoTilde0      (src/transfer/transfer3d_tp.cpp:29-36)
//   phiFromRawDensity / betaFromPhi (src/physics/phasefield.h:10-18)
//   pa3d::applyNarrowBandAir / applyTypedParticleCoarsening /
//   applyLiquidParticleRefill (src/driver/particle_adaptivity3d.h:111-374)
//   diagnoseSparseInterface3D (src/driver/interface_diagnostics3d.cpp:363-379)
//   applySparseSurfaceTension3D (src/driver/interface_diagnostics3d.cpp:405-447)
//   sparse3d::collectCellsWithMarker (src/driver/sparse_ops3d_common.h:65-85)
//   writeSparseRenderCache3D (src/driver/render_cache3d.h:617-663)
// and converts between its SparseMacGrid3D<4> block pool and dense arrays
// plus one activity byte per 4^3 block.
#include "driver/interface_diagnostics3d.h"
#include "driver/particle_adaptivity3d.h"
#include "driver/render_cache3d.h"
#include "driver/sparse_ops3d_common.h"
#include "driver/sparse_ops3d_tp.h"
#include "driver/sparse_sim3d_tp.h"
#include "grid/sparse_mac_grid3d.h"
#include "particles/particles3d_tp.h"
#include "physics/phasefield.h"
#include "transfer/transfer3d_tp.h"

#include <cstddef>
#include <cstring>
#include <new>

namespace {

struct Handle {
  SparseSim3DTP sim;
  Handle(int nx, int ny, int nz, double dx) : sim(nx, ny, nz, dx) {}
};

SparseBlockGrid3D<4>* fieldOf(SparseMacGrid3D<4>& g, int f) {
  switch (f) {
    case 0: return &g.uf;
    case 1: return &g.vf;
    case 2: return &g.wf;
    case 3: return &g.muf;
    case 4: return &g.mvf;
    case 5: return &g.mwf;
    case 6: return &g.pf;
    case 7: return &g.mkf;
    default: return nullptr;
  }
}

PhaseParams phaseOf(const double* ph) {
  PhaseParams pp;
  pp.rho_l = ph[0];
  pp.rho_g = ph[1];
  pp.alpha_phi = ph[2];
  pp.rho_tilde_0 = ph[3];
  return pp;
}

}  // namespace

extern "C" {

void* pfr_create(int nx, int ny, int nz, double dx, double ox, double oy, double oz) {
  Handle* h = new (std::nothrow) Handle(nx, ny, nz, dx);
  if (!h) return nullptr;
  h->sim.grid.ox = ox;
  h->sim.grid.oy = oy;
  h->sim.grid.oz = oz;
  return h;
}

void pfr_destroy(void* hp) { delete static_cast<Handle*>(hp); }

int pfr_copy_grid(void* dst, const void* src) {
  static_cast<Handle*>(dst)->sim.grid = static_cast<const Handle*>(src)->sim.grid;
  return 0;
}

int pfr_get_field(void* hp, int f, float* dense, unsigned char* act) {
  SparseBlockGrid3D<4>* fld = fieldOf(static_cast<Handle*>(hp)->sim.grid, f);
  if (!fld) return -1;
  const size_t nb = fld->totalBlocks();
  for (size_t b = 0; b < nb; ++b) act[b] = fld->blockmap[b] >= 0 ? 1 : 0;
  for (int k = 0; k < fld->nz; ++k)
    for (int j = 0; j < fld->ny; ++j)
      for (int i = 0; i < fld->nx; ++i)
        dense[(size_t)i + (size_t)fld->nx * ((size_t)j + (size_t)fld->ny * k)] = fld->get(i, j, k);
  return 0;
}

int pfr_set_field(void* hp, int f, const float* dense, const unsigned char* act) {
  SparseBlockGrid3D<4>* fld = fieldOf(static_cast<Handle*>(hp)->sim.grid, f);
  if (!fld) return -1;
  fld->clear();
  for (int bz = 0; bz < fld->nbz; ++bz)
    for (int by = 0; by < fld->nby; ++by)
      for (int bx = 0; bx < fld->nbx; ++bx)
        if (act[fld->bid(bx, by, bz)]) fld->activateBlock(bx, by, bz);
  for (int k = 0; k < fld->nz; ++k)
    for (int j = 0; j < fld->ny; ++j)
      for (int i = 0; i < fld->nx; ++i)
        if (fld->blockActive(i / 4, j / 4, k / 4))
          fld->ref(i, j, k) = dense[(size_t)i + (size_t)fld->nx * ((size_t)j + (size_t)fld->ny * k)];
  return 0;
}

// Active block ids in the reference's allocation order.
int pfr_active_block_ids(void* hp, int f, int* out, size_t* n) {
  SparseBlockGrid3D<4>* fld = fieldOf(static_cast<Handle*>(hp)->sim.grid, f);
  if (!fld) return -1;
  const auto& ids = fld->activeBlockIds();
  if (out) std::memcpy(out, ids.data(), ids.size() * sizeof(int));
  *n = ids.size();
  return 0;
}

// Cells with the given marker, ascending linear index, as the projection
// enumerates them.
int pfr_collect_cells(void* hp, int marker, int* out, size_t* n) {
  const std::vector<int> cells = sparse3d::collectCellsWithMarker(static_cast<Handle*>(hp)->sim.grid, marker);
  if (out) {
    if (cells.size() > *n) return -1;
    std::memcpy(out, cells.data(), cells.size() * sizeof(int));
  }
  *n = cells.size();
  return 0;
}

// writeSparseRenderCache3D on this handle's simulation state, with phase, Vp
// and the last effective dt as given.  cam: position, target, up (3 doubles
// each), fov_degrees, near_clip, far_clip, focal_length_mm.  Returns -1 if
// the writer throws (an invalid path or metadata), 0 otherwise.
int pfr_write_render_cache(void* hp, const char* path, int frame, double time, double dt, const double* phase,
                           double Vp, const double* cam) {
  SparseSim3DTP& s = static_cast<Handle*>(hp)->sim;
  s.phase = phaseOf(phase);
  s.Vp = Vp;
  s.effective_dt_last = dt;
  RenderCacheCamera3D c;
  c.position = Vec3{cam[0], cam[1], cam[2]};
  c.target = Vec3{cam[3], cam[4], cam[5]};
  c.up = Vec3{cam[6], cam[7], cam[8]};
  c.fov_degrees = cam[9];
  c.near_clip = cam[10];
  c.far_clip = cam[11];
  c.focal_length_mm = cam[12];
  try {
    writeSparseRenderCache3D(s, path, frame, time, c);
  } catch (...) {
    return -1;
  }
  return 0;
}

int pfr_set_particles(void* hp, size_t n, const double* pos, const double* vel,
                      const unsigned char* type, const double* vol) {
  Particles3DTP& ps = static_cast<Handle*>(hp)->sim.particles;
  ps = Particles3DTP();
  for (size_t p = 0; p < n; ++p)
    ps.add({pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]},
           {vel[3 * p], vel[3 * p + 1], vel[3 * p + 2]}, type[p], vol[p]);
  return 0;
}

size_t pfr_num_particles(void* hp) { return static_cast<Handle*>(hp)->sim.particles.size(); }

int pfr_get_particles(void* hp, double* pos, double* vel, unsigned char* type, double* vol) {
  const Particles3DTP& ps = static_cast<Handle*>(hp)->sim.particles;
  for (size_t p = 0; p < ps.size(); ++p) {
    if (pos) { pos[3 * p] = ps.pos[p].x; pos[3 * p + 1] = ps.pos[p].y; pos[3 * p + 2] = ps.pos[p].z; }
    if (vel) { vel[3 * p] = ps.vel[p].x; vel[3 * p + 1] = ps.vel[p].y; vel[3 * p + 2] = ps.vel[p].z; }
    if (type) type[p] = ps.type[p];
    if (vol) vol[p] = ps.volume[p];
  }
  return 0;
}

int pfr_p2g(void* hp, const double* phase, double Vp) {
  Handle* h = static_cast<Handle*>(hp);
  spP2G3D_tp(h->sim.grid, h->sim.particles, phaseOf(phase), Vp);
  return 0;
}

int pfr_project(void* hp, const double* phase, double dt, int iters, double tol, double cdiv) {
  Handle* h = static_cast<Handle*>(hp);
  spProjectStepVC3D(h->sim.grid, phaseOf(phase), dt, iters, tol, cdiv);
  return 0;
}

int pfr_g2p(void* hp, const void* savedp, double aL, double aG) {
  Handle* h = static_cast<Handle*>(hp);
  const Handle* s = static_cast<const Handle*>(savedp);
  spG2P3D_tp(h->sim.grid, h->sim.particles, s->sim.grid, aL, aG);
  return 0;
}

// stats8: clamped_liquid, clamped_gas, x_lo, x_hi, y_lo, y_hi, z_lo, z_hi
int pfr_advect(void* hp, double dt, int order, int* stats8, double* escape_out, size_t* n_escape) {
  Handle* h = static_cast<Handle*>(hp);
  ParticleEscapeStats3D st;
  ParticleEscapeBuffer3D buf;
  spAdvect3D_tp(h->sim.particles, h->sim.grid, dt, &st, order, escape_out ? &buf : nullptr);
  if (stats8) {
    stats8[0] = st.clamped_liquid; stats8[1] = st.clamped_gas;
    stats8[2] = st.clamped_x_lo; stats8[3] = st.clamped_x_hi;
    stats8[4] = st.clamped_y_lo; stats8[5] = st.clamped_y_hi;
    stats8[6] = st.clamped_z_lo; stats8[7] = st.clamped_z_hi;
  }
  if (escape_out) {
    for (size_t r = 0; r < buf.records.size(); ++r) {
      const EscapedParticleRecord3D& e = buf.records[r];
      double* o = escape_out + 8 * r;
      o[0] = e.type; o[1] = e.pos.x; o[2] = e.pos.y; o[3] = e.pos.z;
      o[4] = e.vel.x; o[5] = e.vel.y; o[6] = e.vel.z; o[7] = e.volume;
    }
    if (n_escape) *n_escape = buf.records.size();
  }
  return 0;
}

// cfg: dt, gravity, Vp, alpha_l, alpha_g, cg_iters, cg_tol, advect_order
int pfr_step(void* hp, const double* phase, const double* cfg) {
  Handle* h = static_cast<Handle*>(hp);
  SparseSim3DTP& s = h->sim;
  s.phase = phaseOf(phase);
  s.dt = cfg[0];
  s.gravity = cfg[1];
  s.Vp = cfg[2];
  s.alpha_liquid = cfg[3];
  s.alpha_gas = cfg[4];
  s.cg_iters = (int)cfg[5];
  s.cg_tol = cfg[6];
  s.advection_order = (int)cfg[7];
  s.step();
  return 0;
}

double pfr_calibrate_rho_tilde0(const double* phase, double Vp) {
  return calibrateRhoTilde0(phaseOf(phase), Vp);
}

double pfr_phi_from_raw(double raw, const double* phase) {
  return phiFromRawDensity(raw, phaseOf(phase));
}

double pfr_beta_from_raw(double raw, const double* phase) {
  PhaseParams pp = phaseOf(phase);
  return betaFromPhi(phiFromRawDensity(raw, pp), pp);
}

// ---- particle adaptivity on the handle's particles and grid domain ----
static pa3d::ParticleCellDomain3D domainOf(const Handle* h) {
  const auto& g = h->sim.grid;
  return pa3d::ParticleCellDomain3D{g.nx, g.ny, g.nz, g.dx, g.ox, g.oy, g.oz};
}

// out4: removed, liquidCells, gasBefore, gasAfter
int pfr_narrow_band_air(void* hp, int radius, int* out4) {
  Handle* h = static_cast<Handle*>(hp);
  const auto r = pa3d::applyNarrowBandAir(h->sim.particles, domainOf(h), true, radius);
  const int v[4] = {r.removed, r.liquidCells, r.gasBefore, r.gasAfter};
  std::memcpy(out4, v, sizeof(v));
  return 0;
}

// out5: removed, cells, overfullCells, particlesBefore, particlesAfter
int pfr_coarsen_particles(void* hp, int ptype, int target, unsigned seed, int* out5) {
  Handle* h = static_cast<Handle*>(hp);
  const auto r = pa3d::applyTypedParticleCoarsening(h->sim.particles, domainOf(h), true,
                                                    static_cast<unsigned char>(ptype), target, seed);
  const int v[5] = {r.removed, r.cells, r.overfullCells, r.particlesBefore, r.particlesAfter};
  std::memcpy(out5, v, sizeof(v));
  return 0;
}

// out7: added, cells, interfaceCells, underfullCells, budgetLimited, particlesBefore, particlesAfter
int pfr_refill_liquid(void* hp, int target, unsigned seed, int interface_only, int interface_radius,
                      int max_added, int* out7) {
  Handle* h = static_cast<Handle*>(hp);
  const auto r = pa3d::applyLiquidParticleRefill(h->sim.particles, domainOf(h), true, target, seed,
                                                 interface_only != 0, interface_radius, max_added);
  const int v[7] = {r.added, r.cells, r.interfaceCells, r.underfullCells, r.budgetLimited, r.particlesBefore,
                    r.particlesAfter};
  std::memcpy(out7, v, sizeof(v));
  return 0;
}

// ints4: sample_cells, interface_cells, finite, surface_tension_candidate;
// dbl7: phi_min, phi_max, phi_mean, grad_mean, grad_max, curvature_abs_mean, curvature_abs_max
int pfr_interface_diagnostics(void* hp, const double* phase, int* ints4, double* dbl7) {
  Handle* h = static_cast<Handle*>(hp);
  const InterfaceDiagnostics3D d = diagnoseSparseInterface3D(h->sim.grid, phaseOf(phase));
  const int iv[4] = {d.sample_cells, d.interface_cells, d.finite, d.surface_tension_candidate};
  const double dv[7] = {d.phi_min, d.phi_max, d.phi_mean, d.grad_mean, d.grad_max, d.curvature_abs_mean,
                        d.curvature_abs_max};
  std::memcpy(ints4, iv, sizeof(iv));
  std::memcpy(dbl7, dv, sizeof(dv));
  return 0;
}

// ints5: enabled, applied_cells, finite, curvature_smoothing_radius, capillary_stable;
// dbl9: strength, max_delta_speed_limit, mean_delta_speed, max_delta_speed, raw_curvature_abs_mean,
//       raw_curvature_abs_max, smoothed_curvature_abs_mean, smoothed_curvature_abs_max, capillary_dt_limit
int pfr_surface_tension(void* hp, const double* phase, double dt, double strength, double max_dv, int radius,
                        int* ints5, double* dbl9) {
  Handle* h = static_cast<Handle*>(hp);
  const SurfaceTensionStats3D s =
      applySparseSurfaceTension3D(h->sim.grid, phaseOf(phase), dt, strength, max_dv, radius);
  const int iv[5] = {s.enabled, s.applied_cells, s.finite, s.curvature_smoothing_radius, s.capillary_stable};
  const double dv[9] = {s.strength, s.max_delta_speed_limit, s.mean_delta_speed, s.max_delta_speed,
                        s.raw_curvature_abs_mean, s.raw_curvature_abs_max, s.smoothed_curvature_abs_mean,
                        s.smoothed_curvature_abs_max, s.capillary_dt_limit};
  std::memcpy(ints5, iv, sizeof(iv));
  std::memcpy(dbl9, dv, sizeof(dv));
  return 0;
}

}  // extern "C"
