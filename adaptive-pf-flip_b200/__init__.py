"""B200 (sm_100a) solver-step backend for the sparse 3D two-phase Phase-Field-FLIP
step of adaptive-pf-flip.

The Python side mirrors the reference's C++ interface for this path, with the
same names, argument meanings and order:

    spP2G3D_tp(grid, particles, phase, Vp)                  src/driver/sparse_ops3d_tp.h:9
    spProjectStepVC3D(grid, phase, dt, cg_iters, cg_tol, divergenceCorrection=0.0)
                                                            src/driver/sparse_ops3d_tp.h:10
    spG2P3D_tp(grid, particles, saved, aL, aG)              src/driver/sparse_ops3d_tp.h:12
    spAdvect3D_tp(particles, grid, dt, stats=None, advectionOrder=2, escapeBuffer=None)
                                                            src/driver/sparse_ops3d_tp.h:13
    SparseSim3DTP(nx, ny, nz, dx).step()                    src/driver/sparse_sim3d_tp.cpp:854-884
    applyNarrowBandAir(particles, grid, enabled, radius)    src/driver/particle_adaptivity3d.h:111
    applyTypedParticleCoarsening(particles, grid, enabled, particleType, target, seed)
                                                            src/driver/particle_adaptivity3d.h:168
    applyLiquidParticleRefill(particles, grid, enabled, target, seed, interfaceOnly,
                              interfaceRadius, maxAddedPerStep)
                                                            src/driver/particle_adaptivity3d.h:264
    diagnoseSparseInterface3D(grid, phase)                  src/driver/interface_diagnostics3d.cpp:363
    MRSim3DTP (2-level multires step)                       src/driver/multires_sim3d_tp.cpp:671-733
    SparseMacGrid3D, Particles3DTP, PhaseParams             src/grid/sparse_mac_grid3d.h,
                                                            src/particles/particles3d_tp.h,
                                                            src/physics/phasefield.h

Every compute call goes through libpfgpu.so (include/pfgpu.h); nothing here
computes on the CPU except scalar phase-field helpers used on results.
"""
from ._lib import (PF_MK, PF_MU, PF_MV, PF_MW, PF_P, PF_PRECOND_EXACT_COARSE, PF_PRECOND_JACOBI,
                   PF_PRECOND_NETWORK, PF_SCENE_BUBBLE_TANK, PF_SCENE_RAYLEIGH_TAYLOR, PF_SOLVER_LEARNED, PF_SOLVER_MIXED, PF_SOLVER_PLAIN, PF_U, PF_V, PF_W, PfError,
                   load)
from .learned import LearnedCoarseSolver
from .multires import MRSim3DTP
from .sparse import (ParticleEscapeBuffer3D, ParticleEscapeStats3D, Particles3DTP, PhaseParams, SolverConfig,
                     SparseMacGrid3D, SparseSim3DTP, applyGasParticleCoarsening, applyLiquidParticleRefill,
                     applyNarrowBandAir, applySparseSurfaceTension3D, applyTypedParticleCoarsening, betaFromPhi, calibrateRhoTilde0,
                     defaultRenderCacheCamera3D, densityFromPhi, diagnoseSparseInterface3D, etaPhi, phiFromRawDensity, spAdvect3D_tp, spG2P3D_tp, spP2G3D_tp, writeSparseRenderCache3D,
                     RenderCacheManifestFrame3D, writeRenderCacheManifest3D,
                     spProjectStepVC3D)
from . import scenes

__all__ = [
    "PF_U", "PF_V", "PF_W", "PF_MU", "PF_MV", "PF_MW", "PF_P", "PF_MK",
    "PF_SOLVER_PLAIN", "PF_SOLVER_MIXED", "PF_SOLVER_LEARNED", "PfError", "load",
    "PF_PRECOND_NETWORK", "PF_PRECOND_EXACT_COARSE", "PF_PRECOND_JACOBI", "PF_SCENE_RAYLEIGH_TAYLOR",
    "PF_SCENE_BUBBLE_TANK", "LearnedCoarseSolver", "MRSim3DTP",
    "PhaseParams", "Particles3DTP", "SparseMacGrid3D", "SparseSim3DTP", "SolverConfig",
    "ParticleEscapeStats3D", "ParticleEscapeBuffer3D",
    "spP2G3D_tp", "spProjectStepVC3D", "spG2P3D_tp", "spAdvect3D_tp", "calibrateRhoTilde0",
    "etaPhi", "phiFromRawDensity", "densityFromPhi", "betaFromPhi", "scenes",
    "applyNarrowBandAir", "applyTypedParticleCoarsening", "applyGasParticleCoarsening", "applyLiquidParticleRefill",
    "diagnoseSparseInterface3D", "applySparseSurfaceTension3D",
    "writeSparseRenderCache3D", "defaultRenderCacheCamera3D", "writeRenderCacheManifest3D",
    "RenderCacheManifestFrame3D",
]
