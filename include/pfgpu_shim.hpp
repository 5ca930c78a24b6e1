// pfgpu_shim.hpp -- C++ adapters from the reference's own grid and particle
// types to the libpfgpu C ABI (pfgpu.h).
//
// The templates below work on any type with the member names of
// SparseMacGrid3D<4> (src/grid/sparse_mac_grid3d.h:6-47: nx, ny, nz, dx,
// ox, oy, oz and the fields uf, vf, wf, muf, mvf, mwf, pf, mkf, each a
// SparseBlockGrid3D<4> with nx/ny/nz, nbx/nby/nbz, blockmap, pool,
// active_block_ids, activateBlock, clear) and of Particles3DTP
// (src/particles/particles3d_tp.h:4-35: pos, vel as std::vector<Vec3> of three
// doubles, type, volume).  They need no reference header themselves; a
// translation unit that includes the reference's headers instantiates them
// behind functions with the reference's exact signatures (see
// adaptive-pf-flip_b200/shim/sparse_ops3d_tp_gpu.cpp).
//
// Each call moves the fields it reads to the device and the fields it writes
// back into the caller's block pool, so the caller's objects hold exactly what
// the reference's in-place functions would leave in them (values and the
// active 4^3 block set; blocks are reallocated in ascending id order, which
// only changes the order of active_block_ids).  Errors throw
// std::runtime_error carrying pf_last_error().
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "pfgpu.h"

namespace pfgpu {

inline void check(int rc, pf_ctx* ctx, const char* what) {
  if (rc != PF_OK) {
    std::string msg = std::string(what) + " failed (" + std::to_string(rc) + ")";
    if (ctx) msg += std::string(": ") + pf_last_error(ctx);
    throw std::runtime_error(msg);
  }
}

// A small cache of device contexts keyed by the host grid's address and shape.
class ContextCache {
 public:
  ~ContextCache() {
    for (Entry& e : entries_) pf_destroy(e.ctx);
  }
  template <class Grid>
  pf_ctx* get(const Grid& g, size_t particles) {
    ++clock_;
    for (Entry& e : entries_) {
      if (e.key == (const void*)&g && e.nx == g.nx && e.ny == g.ny && e.nz == g.nz && e.dx == g.dx &&
          e.ox == g.ox && e.oy == g.oy && e.oz == g.oz && e.cap >= particles) {
        e.used = clock_;
        return e.ctx;
      }
    }
    return create((const void*)&g, g.nx, g.ny, g.nz, g.dx, g.ox, g.oy, g.oz, particles);
  }

  // A context for a particle cell domain (nx, ny, nz, dx, ox, oy, oz), which
  // has no lasting address: matched by shape and origin.
  template <class Domain>
  pf_ctx* get_domain(const Domain& d, size_t particles) {
    ++clock_;
    for (Entry& e : entries_) {
      if (!e.key && e.nx == d.nx && e.ny == d.ny && e.nz == d.nz && e.dx == d.dx && e.ox == d.ox &&
          e.oy == d.oy && e.oz == d.oz && e.cap >= particles) {
        e.used = clock_;
        return e.ctx;
      }
    }
    return create(nullptr, d.nx, d.ny, d.nz, d.dx, d.ox, d.oy, d.oz, particles);
  }

 private:
  struct Entry {
    const void* key;
    int nx, ny, nz;
    double dx, ox, oy, oz;
    size_t cap;
    pf_ctx* ctx;
    unsigned long long used;
  };
  pf_ctx* create(const void* key, int nx, int ny, int nz, double dx, double ox, double oy, double oz,
                 size_t particles) {
    if (entries_.size() >= kMax) {
      size_t lru = 0;
      for (size_t i = 1; i < entries_.size(); ++i)
        if (entries_[i].used < entries_[lru].used) lru = i;
      pf_destroy(entries_[lru].ctx);
      entries_.erase(entries_.begin() + (long)lru);
    }
    pf_grid_desc d{nx, ny, nz, dx, ox, oy, oz, particles > 0 ? particles : 1, 0};
    pf_ctx* ctx = nullptr;
    check(pf_create(&d, &ctx), nullptr, "pf_create");
    entries_.push_back(Entry{key, nx, ny, nz, dx, ox, oy, oz, d.max_particles, ctx, clock_});
    return ctx;
  }
  static constexpr size_t kMax = 4;
  std::vector<Entry> entries_;
  unsigned long long clock_ = 0;
};

inline ContextCache& cache() {
  static ContextCache c;
  return c;
}

template <class Grid>
auto field_of(Grid& g, int f) -> decltype((g.uf)) {
  switch (f) {
    case PF_U: return g.uf;
    case PF_V: return g.vf;
    case PF_W: return g.wf;
    case PF_MU: return g.muf;
    case PF_MV: return g.mvf;
    case PF_MW: return g.mwf;
    case PF_P: return g.pf;
    default: return g.mkf;
  }
}

// SparseBlockGrid3D<4> block pool -> dense lattice + activity bytes -> device
template <class Grid>
void upload_field(pf_ctx* ctx, Grid& g, int f) {
  auto& F = field_of(g, f);
  const size_t X = (size_t)F.nx, Y = (size_t)F.ny, Z = (size_t)F.nz;
  std::vector<float> dense(X * Y * Z, 0.0f);
  std::vector<uint8_t> act(F.blockmap.size(), 0);
  for (int b : F.active_block_ids) {
    act[(size_t)b] = 1;
    const int bx = b % F.nbx, q = b / F.nbx, by = q % F.nby, bz = q / F.nby;
    const auto& blk = F.pool[(size_t)F.blockmap[(size_t)b]];
    for (int lz = 0; lz < 4; ++lz)
      for (int ly = 0; ly < 4; ++ly)
        for (int lx = 0; lx < 4; ++lx) {
          const int i = bx * 4 + lx, j = by * 4 + ly, k = bz * 4 + lz;
          if (i >= F.nx || j >= F.ny || k >= F.nz) continue;
          dense[(size_t)i + X * ((size_t)j + Y * (size_t)k)] = blk[(size_t)(lx + 4 * (ly + 4 * lz))];
        }
  }
  check(pf_grid_set_field(ctx, f, dense.data(), act.data()), ctx, "pf_grid_set_field");
}

// device -> dense + activity -> the caller's block pool (clear, reactivate, fill)
template <class Grid>
void download_field(pf_ctx* ctx, Grid& g, int f) {
  auto& F = field_of(g, f);
  const size_t X = (size_t)F.nx, Y = (size_t)F.ny, Z = (size_t)F.nz;
  std::vector<float> dense(X * Y * Z);
  std::vector<uint8_t> act(F.blockmap.size());
  check(pf_grid_get_field(ctx, f, dense.data(), act.data()), ctx, "pf_grid_get_field");
  F.clear();
  for (int bz = 0; bz < F.nbz; ++bz)
    for (int by = 0; by < F.nby; ++by)
      for (int bx = 0; bx < F.nbx; ++bx) {
        const int b = bx + F.nbx * (by + F.nby * bz);
        if (!act[(size_t)b]) continue;
        const int pi = F.activateBlock(bx, by, bz);
        auto& blk = F.pool[(size_t)pi];
        for (int lz = 0; lz < 4; ++lz)
          for (int ly = 0; ly < 4; ++ly)
            for (int lx = 0; lx < 4; ++lx) {
              const int i = bx * 4 + lx, j = by * 4 + ly, k = bz * 4 + lz;
              if (i >= F.nx || j >= F.ny || k >= F.nz) continue;
              blk[(size_t)(lx + 4 * (ly + 4 * lz))] = dense[(size_t)i + X * ((size_t)j + Y * (size_t)k)];
            }
      }
}

template <class Particles>
void upload_particles(pf_ctx* ctx, const Particles& ps) {
  const size_t n = ps.size();
  static const double zero3[3] = {0.0, 0.0, 0.0};
  static const uint8_t zero_t = 0;
  static const double one = 1.0;
  check(pf_upload_particles_f64(ctx, n, n ? &ps.pos[0].x : zero3, n ? &ps.vel[0].x : zero3,
                                n ? (const uint8_t*)ps.type.data() : &zero_t, n ? ps.volume.data() : &one),
        ctx, "pf_upload_particles_f64");
}

template <class Phase>
pf_phase phase_of(const Phase& pp) {
  return pf_phase{pp.rho_l, pp.rho_g, pp.alpha_phi, pp.rho_tilde_0};
}

// spP2G3D_tp (src/driver/sparse_ops3d_tp.cpp:95-153)
template <class Grid, class Particles, class Phase>
void p2g(Grid& g, const Particles& ps, const Phase& pp, double Vp) {
  pf_ctx* ctx = cache().get(g, ps.size());
  upload_particles(ctx, ps);
  const pf_phase ph = phase_of(pp);
  check(pf_p2g(ctx, &ph, Vp), ctx, "pf_p2g");
  for (int f = PF_U; f <= PF_MW; ++f) download_field(ctx, g, f);
}

// spProjectStepVC3D (src/driver/sparse_ops3d_tp.cpp:234-423): the plain FP64
// Jacobi-PCG with the reference's absolute max-norm stop.
template <class Grid, class Phase>
pf_solve_stats project(Grid& g, const Phase& pp, double dt, int cg_iters, double cg_tol, double c_div,
                       int mode = PF_SOLVER_PLAIN, double rel_tol = 0.0) {
  pf_ctx* ctx = cache().get(g, 0);
  for (int f = 0; f < PF_NFIELDS; ++f) upload_field(ctx, g, f);
  const pf_phase ph = phase_of(pp);
  pf_solve_cfg cfg{mode, cg_iters, cg_tol, rel_tol, c_div, 0, 0, 0, 0.0};
  pf_solve_stats st{};
  check(pf_project(ctx, &ph, dt, &cfg, &st), ctx, "pf_project");
  download_field(ctx, g, PF_P);
  for (int f = PF_U; f <= PF_W; ++f) download_field(ctx, g, f);
  return st;
}

// spG2P3D_tp (src/driver/sparse_ops3d_tp.cpp:155-172)
template <class Grid, class Particles>
void g2p(const Grid& g, Particles& ps, const Grid& saved, double aL, double aG) {
  pf_ctx* ctx = cache().get(g, ps.size());
  pf_ctx* sctx = cache().get(saved, 0);
  Grid& gm = const_cast<Grid&>(g);
  Grid& sm = const_cast<Grid&>(saved);
  for (int f = PF_U; f <= PF_W; ++f) {
    upload_field(ctx, gm, f);
    upload_field(sctx, sm, f);
  }
  upload_particles(ctx, ps);
  check(pf_g2p(ctx, sctx, aL, aG), ctx, "pf_g2p");
  if (ps.size()) check(pf_download_particles_f64(ctx, nullptr, &ps.vel[0].x, nullptr, nullptr), ctx, "download");
}

// spAdvect3D_tp (src/driver/sparse_ops3d_tp.cpp:201-232); Stats/Buffer are
// ParticleEscapeStats3D / ParticleEscapeBuffer3D (src/driver/particle_escape3d.h)
template <class Grid, class Particles, class Stats, class Buffer>
void advect(Particles& ps, const Grid& g, double dt, Stats* stats, int order, Buffer* buffer) {
  pf_ctx* ctx = cache().get(g, ps.size());
  Grid& gm = const_cast<Grid&>(g);
  for (int f = PF_U; f <= PF_W; ++f) upload_field(ctx, gm, f);
  upload_particles(ctx, ps);
  pf_clamp_stats cs{};
  std::vector<double> esc(buffer ? 8 * (ps.size() ? ps.size() : 1) : 0);
  size_t nesc = 0;
  check(pf_advect(ctx, dt, order == 3 ? 3 : 2, &cs, buffer ? esc.data() : nullptr, &nesc), ctx, "pf_advect");
  if (ps.size()) check(pf_download_particles_f64(ctx, &ps.pos[0].x, nullptr, nullptr, nullptr), ctx, "download");
  if (stats) {
    stats->clamped_liquid += cs.clamped_liquid;
    stats->clamped_gas += cs.clamped_gas;
    stats->clamped_x_lo += cs.x_lo;
    stats->clamped_x_hi += cs.x_hi;
    stats->clamped_y_lo += cs.y_lo;
    stats->clamped_y_hi += cs.y_hi;
    stats->clamped_z_lo += cs.z_lo;
    stats->clamped_z_hi += cs.z_hi;
  }
  if (buffer) {
    for (size_t r = 0; r < nesc; ++r) {
      const double* e = &esc[8 * r];
      using V = typename std::decay<decltype(ps.pos[0])>::type;
      buffer->record((unsigned char)e[0], V{e[1], e[2], e[3]}, V{e[4], e[5], e[6]}, e[7]);
    }
  }
}

// ---- particle adaptivity (src/driver/particle_adaptivity3d.h:111-374) ----
// Domain has the members of pa3d::ParticleCellDomain3D (nx, ny, nz, dx, ox,
// oy, oz).  The particle set is rewritten: erasures keep the survivors' order,
// refill appends.

// the device particle set -> the caller's, resized to the device count
template <class Particles>
void download_all_particles(pf_ctx* ctx, Particles& ps) {
  const size_t n = pf_num_particles(ctx);
  ps.pos.resize(n);
  ps.vel.resize(n);
  ps.type.resize(n);
  ps.volume.resize(n);
  if (n)
    check(pf_download_particles_f64(ctx, &ps.pos[0].x, &ps.vel[0].x, (uint8_t*)ps.type.data(), ps.volume.data()),
          ctx, "pf_download_particles_f64");
}

template <class Particles, class Domain>
pf_band_stats narrow_band_air(Particles& ps, const Domain& d, int radius) {
  pf_ctx* ctx = cache().get_domain(d, ps.size());
  upload_particles(ctx, ps);
  pf_band_stats st{};
  check(pf_narrow_band_air(ctx, radius, &st), ctx, "pf_narrow_band_air");
  download_all_particles(ctx, ps);
  return st;
}

template <class Particles, class Domain>
pf_coarsen_stats coarsen_particles(Particles& ps, const Domain& d, int type, int target, unsigned seed) {
  pf_ctx* ctx = cache().get_domain(d, ps.size());
  upload_particles(ctx, ps);
  pf_coarsen_stats st{};
  check(pf_coarsen_particles(ctx, type, target, seed, &st), ctx, "pf_coarsen_particles");
  download_all_particles(ctx, ps);
  return st;
}

// A context too small for the result is replaced by one that holds it: the
// failed call reports in `added` how many particles it would add.
template <class Particles, class Domain>
pf_refill_stats refill_liquid(Particles& ps, const Domain& d, int target, unsigned seed, bool interface_only,
                              int interface_radius, int max_added) {
  size_t cap = ps.size();
  for (int attempt = 0; attempt < 2; ++attempt) {
    pf_ctx* ctx = cache().get_domain(d, cap);
    upload_particles(ctx, ps);
    pf_refill_stats st{};
    const int rc = pf_refill_liquid(ctx, target, seed, interface_only ? 1 : 0, interface_radius, max_added, &st);
    if (rc == PF_ERR_CAPACITY && attempt == 0) {
      cap = ps.size() + (size_t)st.added;
      continue;
    }
    check(rc, ctx, "pf_refill_liquid");
    download_all_particles(ctx, ps);
    return st;
  }
  return pf_refill_stats{};
}

}  // namespace pfgpu
