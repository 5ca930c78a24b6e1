// driver/particle_adaptivity3d.h -- drop-in for the reference's header of the
// same path (src/driver/particle_adaptivity3d.h): the same pa3d types and
// functions, run on the B200 through libpfgpu (include/pfgpu.h).
//
// A build that puts adaptive-pf-flip_b200/shim ahead of the reference's src/
// on the include path compiles SparseSim3DTP (src/driver/sparse_sim3d_tp.cpp)
// and MRSim3DTP unchanged against it: their applyNarrowBandAir,
// applyGasParticleCoarsening, applyLiquidParticleCoarsening and
// applyLiquidParticleRefill then run on the GPU.  Results equal the
// reference's, with positions, velocities and volumes rounded to the device's
// FP32 particle storage.
#pragma once

#include <cstdint>

#include "particles/particles3d_tp.h"
#include "pfgpu_shim.hpp"

namespace pa3d {

// ParticleCellDomain3D (src/driver/particle_adaptivity3d.h:13-47): the cell
// lattice particles are binned on
struct ParticleCellDomain3D {
  int nx = 0;
  int ny = 0;
  int nz = 0;
  double dx = 1.0;
  double ox = 0.0;
  double oy = 0.0;
  double oz = 0.0;
};

// result records (src/driver/particle_adaptivity3d.h:49-72)
struct NarrowBandAirResult3D {
  int removed = 0;
  int liquidCells = 0;
  int gasBefore = 0;
  int gasAfter = 0;
};

struct GasParticleCoarseningResult3D {
  int removed = 0;
  int cells = 0;
  int overfullCells = 0;
  int particlesBefore = 0;
  int particlesAfter = 0;
};

struct LiquidParticleRefillResult3D {
  int added = 0;
  int cells = 0;
  int interfaceCells = 0;
  int underfullCells = 0;
  int budgetLimited = 0;
  int particlesBefore = 0;
  int particlesAfter = 0;
};

inline NarrowBandAirResult3D applyNarrowBandAir(Particles3DTP& particles, const ParticleCellDomain3D& domain,
                                                bool enabled, int radius) {
  NarrowBandAirResult3D r;
  if (!enabled) return r;
  const pf_band_stats s = pfgpu::narrow_band_air(particles, domain, radius);
  r.removed = s.removed;
  r.liquidCells = s.liquid_cells;
  r.gasBefore = s.gas_before;
  r.gasAfter = s.gas_after;
  return r;
}

inline GasParticleCoarseningResult3D applyTypedParticleCoarsening(Particles3DTP& particles,
                                                                  const ParticleCellDomain3D& domain, bool enabled,
                                                                  unsigned char particleType,
                                                                  int particlesPerCellTarget, uint32_t seed) {
  GasParticleCoarseningResult3D r;
  if (!enabled) return r;
  const pf_coarsen_stats s = pfgpu::coarsen_particles(particles, domain, particleType, particlesPerCellTarget, seed);
  r.removed = s.removed;
  r.cells = s.cells;
  r.overfullCells = s.overfull_cells;
  r.particlesBefore = s.before;
  r.particlesAfter = s.after;
  return r;
}

inline GasParticleCoarseningResult3D applyGasParticleCoarsening(Particles3DTP& particles,
                                                                const ParticleCellDomain3D& domain, bool enabled,
                                                                int particlesPerCellTarget, uint32_t seed) {
  return applyTypedParticleCoarsening(particles, domain, enabled, 1, particlesPerCellTarget, seed);
}

inline LiquidParticleRefillResult3D applyLiquidParticleRefill(Particles3DTP& particles,
                                                              const ParticleCellDomain3D& domain, bool enabled,
                                                              int particlesPerCellTarget, uint32_t seed,
                                                              bool interfaceOnly = false, int interfaceRadius = 1,
                                                              int maxAddedPerStep = 0) {
  LiquidParticleRefillResult3D r;
  if (!enabled) return r;
  const pf_refill_stats s = pfgpu::refill_liquid(particles, domain, particlesPerCellTarget, seed, interfaceOnly,
                                                 interfaceRadius, maxAddedPerStep);
  r.added = s.added;
  r.cells = s.cells;
  r.interfaceCells = s.interface_cells;
  r.underfullCells = s.underfull_cells;
  r.budgetLimited = s.budget_limited;
  r.particlesBefore = s.before;
  r.particlesAfter = s.after;
  return r;
}

}  // namespace pa3d
