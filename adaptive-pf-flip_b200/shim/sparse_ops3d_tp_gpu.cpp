// sparse_ops3d_tp_gpu.cpp -- drop-in replacement for the reference's
// src/driver/sparse_ops3d_tp.cpp.
//
// Build it in place of that file, with the reference's src/ and this
// repository's include/ on the include path, and link libpfgpu.so:
// spP2G3D_tp, spProjectStepVC3D, spG2P3D_tp and spAdvect3D_tp keep their
// declarations in src/driver/sparse_ops3d_tp.h:8-15 and run on the B200
// through the C ABI (include/pfgpu.h).  Callers such as
// SparseSim3DTP::step() (src/driver/sparse_sim3d_tp.cpp:854-884) need no
// change.
#include <type_traits>

#include "driver/sparse_ops3d_tp.h"
#include "grid/sparse_mac_grid3d.h"
#include "particles/particles3d_tp.h"
#include "physics/phasefield.h"
#include "pfgpu_shim.hpp"

void spP2G3D_tp(SparseMacGrid3D<4>& g, const Particles3DTP& ps, const PhaseParams& pp, double Vp) {
  pfgpu::p2g(g, ps, pp, Vp);
}

void spProjectStepVC3D(SparseMacGrid3D<4>& g, const PhaseParams& pp, double dt, int cg_iters, double cg_tol,
                       double divergenceCorrection) {
  pfgpu::project(g, pp, dt, cg_iters, cg_tol, divergenceCorrection);
}

void spG2P3D_tp(const SparseMacGrid3D<4>& g, Particles3DTP& ps, const SparseMacGrid3D<4>& saved, double aL,
                double aG) {
  pfgpu::g2p(g, ps, saved, aL, aG);
}

void spAdvect3D_tp(Particles3DTP& ps, const SparseMacGrid3D<4>& g, double dt, ParticleEscapeStats3D* stats,
                   int advectionOrder, ParticleEscapeBuffer3D* escapeBuffer) {
  pfgpu::advect(ps, g, dt, stats, advectionOrder, escapeBuffer);
}
