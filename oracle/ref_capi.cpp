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
//   writeRenderCacheManifest3D (src/driver/render_cache3d.h:711-755)
//   MRSim3DTP (src/driver/multires_sim3d_tp.h:10-191): step(),
//     initBubbleTankInterfaceBand(), updateDynamicRefinement(), and
//     mrP2G3D_tp (src/driver/multires_ops3d_tp.cpp:209-274)
// and converts between its SparseMacGrid3D<4> block pool and dense arrays
// plus one activity byte per 4^3 block, and between MRMacGrid3D<4>'s maps and
// dense fine lattices (absent face keys and cells read 0).
#include "driver/interface_diagnostics3d.h"
#include "driver/multires_ops3d_tp.h"
#include "driver/multires_sim3d_tp.h"
#include "driver/particle_adaptivity3d.h"
#include "driver/render_cache3d.h"
#include "driver/sparse_ops3d_common.h"
#include "driver/sparse_ops3d_tp.h"
#include "driver/sparse_sim3d_tp.h"
#include "grid/sparse_mac_grid3d.h"
#include "particles/particles3d_tp.h"
#include "physics/phasefield.h"
#include "transfer/transfer3d_tp.h"

#include <algorithm>
#include <cstddef>
#include <cstring>
#include <map>
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


// ---- secondary particles (src/driver/secondary_particles3d.h, the escape
// branching, lifecycle and spray emission of SparseSim3DTP::step,
// src/driver/sparse_sim3d_tp.cpp:192-337) ------------------------------------

// iv: escaped_particle_branching, secondary_particle_lifecycle,
//     secondary_droplet_lifetime_steps, secondary_bubble_lifetime_steps,
//     secondary_reabsorb_to_primary, secondary_spray_emission,
//     secondary_spray_particles_per_step, secondary_spray_interface_gate,
//     secondary_spray_min_interface_cells, secondary_spray_impact_candidates
// dv: secondary_velocity_damping, secondary_reabsorb_margin_cells,
//     secondary_droplet_gravity_scale, secondary_bubble_buoyancy_scale,
//     secondary_droplet_drag, secondary_bubble_drag,
//     secondary_spray_droplet_fraction, secondary_spray_droplet_volume,
//     secondary_spray_bubble_volume, secondary_spray_min_interface_grad_max,
//     secondary_spray_min_interface_curvature_abs_max,
//     secondary_spray_impact_region_fraction,
//     secondary_spray_impact_downward_speed_min, secondary_spray_impact_foam_fraction
int pfr_set_secondary(void* hp, const int* iv, const double* dv) {
  SparseSim3DTP& s = static_cast<Handle*>(hp)->sim;
  s.escaped_particle_branching = iv[0] != 0;
  s.secondary_particle_lifecycle = iv[1] != 0;
  s.secondary_droplet_lifetime_steps = iv[2];
  s.secondary_bubble_lifetime_steps = iv[3];
  s.secondary_reabsorb_to_primary = iv[4] != 0;
  s.secondary_spray_emission = iv[5] != 0;
  s.secondary_spray_particles_per_step = iv[6];
  s.secondary_spray_interface_gate = iv[7] != 0;
  s.secondary_spray_min_interface_cells = iv[8];
  s.secondary_spray_impact_candidates = iv[9] != 0;
  s.secondary_velocity_damping = dv[0];
  s.secondary_reabsorb_margin_cells = dv[1];
  s.secondary_droplet_gravity_scale = dv[2];
  s.secondary_bubble_buoyancy_scale = dv[3];
  s.secondary_droplet_drag = dv[4];
  s.secondary_bubble_drag = dv[5];
  s.secondary_spray_droplet_fraction = dv[6];
  s.secondary_spray_droplet_volume = dv[7];
  s.secondary_spray_bubble_volume = dv[8];
  s.secondary_spray_min_interface_grad_max = dv[9];
  s.secondary_spray_min_interface_curvature_abs_max = dv[10];
  s.secondary_spray_impact_region_fraction = dv[11];
  s.secondary_spray_impact_downward_speed_min = dv[12];
  s.secondary_spray_impact_foam_fraction = dv[13];
  return 0;
}

static Particles3DTP& secondarySet(SparseSim3DTP& s, int which) {
  return which == 0 ? s.escaped_droplets : s.escaped_bubbles;
}
static std::vector<int>& secondaryAges(SparseSim3DTP& s, int which) {
  return which == 0 ? s.escaped_droplet_ages : s.escaped_bubble_ages;
}

size_t pfr_secondary_count(void* hp, int which) {
  return secondarySet(static_cast<Handle*>(hp)->sim, which).size();
}

int pfr_get_secondary(void* hp, int which, double* pos, double* vel, double* vol, int* ages) {
  SparseSim3DTP& s = static_cast<Handle*>(hp)->sim;
  const Particles3DTP& ps = secondarySet(s, which);
  const std::vector<int>& ag = secondaryAges(s, which);
  for (size_t p = 0; p < ps.size(); ++p) {
    pos[3 * p] = ps.pos[p].x; pos[3 * p + 1] = ps.pos[p].y; pos[3 * p + 2] = ps.pos[p].z;
    vel[3 * p] = ps.vel[p].x; vel[3 * p + 1] = ps.vel[p].y; vel[3 * p + 2] = ps.vel[p].z;
    vol[p] = ps.volume[p];
    ages[p] = p < ag.size() ? ag[p] : 0;
  }
  return 0;
}

int pfr_set_secondary_set(void* hp, int which, size_t n, const double* pos, const double* vel, const double* vol,
                          const int* ages) {
  SparseSim3DTP& s = static_cast<Handle*>(hp)->sim;
  Particles3DTP& ps = secondarySet(s, which);
  std::vector<int>& ag = secondaryAges(s, which);
  ps = Particles3DTP();
  ag.clear();
  for (size_t p = 0; p < n; ++p) {
    ps.add({pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]}, {vel[3 * p], vel[3 * p + 1], vel[3 * p + 2]},
           (unsigned char)which, vol[p]);
    ag.push_back(ages[p]);
  }
  return 0;
}

// the last step's statistics: iv (30 ints) and dv (20 doubles), in the
// field order of SecondaryParticleLifecycleStats3D,
// SecondarySprayEmissionStats3D and the added counts
int pfr_secondary_stats(void* hp, int* iv, double* dv) {
  SparseSim3DTP& s = static_cast<Handle*>(hp)->sim;
  const SecondaryParticleLifecycleStats3D& l = s.secondary_lifecycle_stats_last;
  const SecondarySprayEmissionStats3D& e = s.secondary_spray_emission_stats_last;
  const int I[30] = {l.enabled, l.finite, l.advected_droplets, l.advected_bubbles, l.reabsorbed_droplets,
                     l.reabsorbed_bubbles, l.expired_droplets, l.expired_bubbles, l.dragged_droplets,
                     l.dragged_bubbles, l.reabsorbed_droplets_to_primary, l.reabsorbed_bubbles_to_primary,
                     e.enabled, e.finite, e.requested_particles, e.effective_requested_particles,
                     e.interface_gate_enabled, e.interface_gate_passed, e.interface_cells,
                     e.candidate_liquid_particles, e.impact_candidate_liquid_particles, e.foam_ready_droplets,
                     e.emitted_droplets, e.emitted_bubbles, s.escaped_droplets_added_last,
                     s.escaped_bubbles_added_last, s.secondary_spray_emission_step_index, 0, 0, 0};
  const double D[20] = {l.current_droplet_volume, l.current_bubble_volume, l.reabsorbed_droplet_volume,
                        l.reabsorbed_bubble_volume, l.expired_droplet_volume, l.expired_bubble_volume,
                        l.reabsorbed_droplet_volume_to_primary, l.reabsorbed_bubble_volume_to_primary,
                        e.interface_grad_max, e.interface_curvature_abs_max, e.emitted_droplet_volume,
                        e.emitted_bubble_volume, s.escaped_droplet_volume_added_last,
                        s.escaped_bubble_volume_added_last, s.secondary_droplet_volume_current_last,
                        s.secondary_bubble_volume_current_last, 0, 0, 0, 0};
  std::memcpy(iv, I, sizeof(I));
  std::memcpy(dv, D, sizeof(D));
  return 0;
}

// writeRenderCacheManifest3D (src/driver/render_cache3d.h:711-755) for frames
// given as parallel arrays; -1 if the writer throws.
int pfr_write_render_manifest(const char* path, const char* sim_kind, int nx, int ny, int nz, double dx, int n,
                              const int* frame, const int* step, const double* time, const char* const* paths,
                              const long long* bytes) {
  std::vector<RenderCacheManifestFrame3D> frames;
  for (int i = 0; i < n; ++i) frames.push_back(RenderCacheManifestFrame3D{frame[i], step[i], time[i], paths[i], bytes[i]});
  try {
    writeRenderCacheManifest3D(path, sim_kind, nx, ny, nz, dx, frames);
  } catch (...) {
    return -1;
  }
  return 0;
}

// ---- multires (MRSim3DTP) -------------------------------------------------

struct MRHandle {
  MRSim3DTP sim;
  MRHandle(int nx, int ny, int nz, double dx) : sim(nx, ny, nz, dx) {}
};

void* pfr_mr_create(int nx, int ny, int nz, double dx) { return new (std::nothrow) MRHandle(nx, ny, nz, dx); }

void pfr_mr_destroy(void* hp) { delete static_cast<MRHandle*>(hp); }

// d: dt, gravity, Vp, alpha_liquid, alpha_gas, cg_tol, cg_rel_tol, cg_restart_growth
// i: advection_order, cg_iters, cg_jacobi_preconditioner, cg_flexible_beta,
//    cg_adaptive_restart, dynamic_refinement, dynamic_particle_padding,
//    dynamic_gas_padding, dynamic_hysteresis_cells, dynamic_max_fine_leaves
int pfr_mr_configure(void* hp, const double* phase, const double* d, const int* i) {
  MRSim3DTP& s = static_cast<MRHandle*>(hp)->sim;
  s.phase = phaseOf(phase);
  s.dt = d[0];
  s.gravity = d[1];
  s.Vp = d[2];
  s.alpha_liquid = d[3];
  s.alpha_gas = d[4];
  s.cg_tol = d[5];
  s.cg_rel_tol = d[6];
  s.cg_restart_growth = d[7];
  s.advection_order = i[0];
  s.cg_iters = i[1];
  s.cg_jacobi_preconditioner = i[2] != 0;
  s.cg_flexible_beta = i[3] != 0;
  s.cg_adaptive_restart = i[4] != 0;
  s.dynamic_refinement = i[5] != 0;
  s.dynamic_particle_padding = i[6];
  s.dynamic_gas_padding = i[7];
  s.dynamic_hysteresis_cells = i[8];
  s.dynamic_max_fine_leaves = i[9];
  return 0;
}

// The layout setCoarseEverywhere(1) + refineFineCellBox of each clamped box
// (as the static layouts of multires_sim3d_tp.cpp:158-170 are made), and a
// fresh grid on it.
int pfr_mr_set_layout(void* hp, const int* boxes, int nbox) {
  MRSim3DTP& s = static_cast<MRHandle*>(hp)->sim;
  s.layout.setCoarseEverywhere(1);
  for (int b = 0; b < nbox; ++b) {
    const int* q = boxes + 6 * b;
    const int x0 = std::max(0, std::min(s.layout.nx, q[0])), y0 = std::max(0, std::min(s.layout.ny, q[1]));
    const int z0 = std::max(0, std::min(s.layout.nz, q[2])), x1 = std::max(0, std::min(s.layout.nx, q[3]));
    const int y1 = std::max(0, std::min(s.layout.ny, q[4])), z1 = std::max(0, std::min(s.layout.nz, q[5]));
    if (x0 < x1 && y0 < y1 && z0 < z1) s.layout.refineFineCellBox(x0, y0, z0, x1, y1, z1);
  }
  s.layout.enforceTwoToOneBalance();
  s.grid = MRMacGrid3D<4>(s.layout);
  return 0;
}

// One byte per level-1 block (x fastest): 1 where the layout holds its
// level-0 children.
int pfr_mr_get_levels(void* hp, unsigned char* refined) {
  const MRLayout3D<4>& L = static_cast<MRHandle*>(hp)->sim.layout;
  const int MX = L.levelBlockCountX(1), MY = L.levelBlockCountY(1), MZ = L.levelBlockCountZ(1);
  std::memset(refined, 0, (size_t)MX * MY * MZ);
  for (const MRBlockKey3D& b : L.leaves())
    if (b.level == 0) refined[(b.bx >> 1) + MX * ((b.by >> 1) + MY * (b.bz >> 1))] = 1;
  return 0;
}

int pfr_mr_count_level(void* hp, int level) {
  return (int)static_cast<MRHandle*>(hp)->sim.layout.countLevel(level);
}

int pfr_mr_set_particles(void* hp, size_t n, const double* pos, const double* vel, const unsigned char* type,
                         const double* vol) {
  Particles3DTP& ps = static_cast<MRHandle*>(hp)->sim.particles;
  ps = Particles3DTP();
  for (size_t p = 0; p < n; ++p)
    ps.add({pos[3 * p], pos[3 * p + 1], pos[3 * p + 2]}, {vel[3 * p], vel[3 * p + 1], vel[3 * p + 2]}, type[p],
           vol[p]);
  return 0;
}

size_t pfr_mr_num_particles(void* hp) { return static_cast<MRHandle*>(hp)->sim.particles.size(); }

int pfr_mr_get_particles(void* hp, double* pos, double* vel, unsigned char* type, double* vol) {
  const Particles3DTP& ps = static_cast<MRHandle*>(hp)->sim.particles;
  for (size_t p = 0; p < ps.size(); ++p) {
    if (pos) { pos[3 * p] = ps.pos[p].x; pos[3 * p + 1] = ps.pos[p].y; pos[3 * p + 2] = ps.pos[p].z; }
    if (vel) { vel[3 * p] = ps.vel[p].x; vel[3 * p + 1] = ps.vel[p].y; vel[3 * p + 2] = ps.vel[p].z; }
    if (type) type[p] = ps.type[p];
    if (vol) vol[p] = ps.volume[p];
  }
  return 0;
}

int pfr_mr_init_bubble_tank(void* hp) {
  static_cast<MRHandle*>(hp)->sim.initBubbleTankInterfaceBand();
  return 0;
}

// updateDynamicRefinement; out7: retained box (valid, x0, y0, z0, x1, y1, z1)
int pfr_mr_update_refinement(void* hp, int* out8) {
  MRSim3DTP& s = static_cast<MRHandle*>(hp)->sim;
  s.updateDynamicRefinement();
  const int v[8] = {s.dynamic_retained_box_valid, s.dynamic_retained_x0, s.dynamic_retained_y0,
                    s.dynamic_retained_z0, s.dynamic_retained_x1, s.dynamic_retained_y1, s.dynamic_retained_z1,
                    s.dynamic_budget_limited};
  std::memcpy(out8, v, sizeof(v));
  return 0;
}

int pfr_mr_p2g(void* hp) {
  MRSim3DTP& s = static_cast<MRHandle*>(hp)->sim;
  mrP2G3D_tp(s.grid, s.particles, s.phase, s.Vp);
  return 0;
}

// step(); ints10: active cells, pinned cell, iterations, restarts, beta resets,
// converged, breakdown, fine leaves, clamped liquid, clamped gas;
// dbl3: initial, final residual, effective tolerance
int pfr_mr_step(void* hp, int* ints10, double* dbl3) {
  MRSim3DTP& s = static_cast<MRHandle*>(hp)->sim;
  s.step();
  const MRPressureSolveStats3D& st = s.last_pressure_stats;
  const int iv[10] = {st.active_cells, st.pinned_cell, st.iterations, st.restarts, st.beta_resets,
                      st.converged ? 1 : 0, st.breakdown ? 1 : 0, (int)s.layout.countLevel(0),
                      s.particle_boundary_clamped_liquid_last, s.particle_boundary_clamped_gas_last};
  const double dv[3] = {st.initial_residual, st.final_residual, st.effective_tolerance};
  std::memcpy(ints10, iv, sizeof(iv));
  std::memcpy(dbl3, dv, sizeof(dv));
  return 0;
}

// a face field on the dense fine face lattice: 0..5 = u v w mu mv mw
int pfr_mr_get_face(void* hp, int field, float* dense) {
  const MRMacGrid3D<4>& g = static_cast<MRHandle*>(hp)->sim.grid;
  const std::map<MRFaceKey3D, float>* maps[6] = {&g.ufield, &g.vfield, &g.wfield, &g.mu, &g.mv, &g.mw};
  if (field < 0 || field > 5) return -1;
  const int axis = field % 3;
  const size_t X = (size_t)g.layout.nx + (axis == 0), Y = (size_t)g.layout.ny + (axis == 1);
  const size_t Z = (size_t)g.layout.nz + (axis == 2);
  std::memset(dense, 0, X * Y * Z * sizeof(float));
  for (const auto& kv : *maps[field]) {
    const MRFaceKey3D& f = kv.first;
    if (f.fineX < 0 || f.fineY < 0 || f.fineZ < 0 || (size_t)f.fineX >= X || (size_t)f.fineY >= Y ||
        (size_t)f.fineZ >= Z)
      return -2;
    dense[(size_t)f.fineX + X * ((size_t)f.fineY + Y * (size_t)f.fineZ)] = kv.second;
  }
  return 0;
}

// the valid faces of one axis (the face list of the current layout)
int pfr_mr_face_valid(void* hp, int axis, unsigned char* dense) {
  const MRMacGrid3D<4>& g = static_cast<MRHandle*>(hp)->sim.grid;
  const std::vector<MRFaceKey3D>& faces = axis == 0 ? g.uFaceRefs() : axis == 1 ? g.vFaceRefs() : g.wFaceRefs();
  const size_t X = (size_t)g.layout.nx + (axis == 0), Y = (size_t)g.layout.ny + (axis == 1);
  const size_t Z = (size_t)g.layout.nz + (axis == 2);
  std::memset(dense, 0, X * Y * Z);
  for (const MRFaceKey3D& f : faces) dense[(size_t)f.fineX + X * ((size_t)f.fineY + Y * (size_t)f.fineZ)] = 1;
  return 0;
}

// marker and pressure per fine cell (the value of its leaf cell)
int pfr_mr_get_cells(void* hp, float* marker, float* pressure) {
  const MRMacGrid3D<4>& g = static_cast<MRHandle*>(hp)->sim.grid;
  const int nx = g.layout.nx, ny = g.layout.ny, nz = g.layout.nz;
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const size_t o = (size_t)i + (size_t)nx * ((size_t)j + (size_t)ny * k);
        if (marker) marker[o] = g.marker.get(g.marker.cellAtFineCell(i, j, k));
        if (pressure) pressure[o] = g.p.get(g.p.cellAtFineCell(i, j, k));
      }
  return 0;
}

}  // extern "C"
