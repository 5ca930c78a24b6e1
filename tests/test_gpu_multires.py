"""The 2-level multires step on the GPU (pf_mr_step, MRSim3DTP) against the
oracle's restatement (oracle/pf_oracle_mr.c), which the CPU suite pins bit for
bit to the reference's own MRSim3DTP::step.

The GPU keeps particles in FP32 and splats with FP32 atomics (another
accumulation order than the reference's particle order); its PCG sums inner
products in another order.  Layouts, face lists, markers, the unknown count
and the pinned cell are therefore exact, and values are compared on the
field's scale: P2G within 1e-5, a whole step within 1e-5 when both solves
converge tightly (relative tolerance 1e-10), and a few default steps of the
bubble tank within 1e-4 against the oracle run with its particle state
rounded to FP32 after every step.
"""
import numpy as np
import pytest

import oracle as O
from gpu_helpers import rel_err
from oracle.multires import MRSettings, OracleMR, face_shape

pytestmark = pytest.mark.gpu


def _phase(Vp=1.0):
    pp = O.PhaseParams(1.0, 0.01)
    pp.rho_tilde_0 = O.Oracle().calibrate_rho_tilde0(pp, Vp)
    return pp


def _scene(nx, ny, nz, dx, seed, speed=0.3):
    """Water in the lower 70% with a gas sphere, eight jittered particles per
    cell, random velocities: FP32 positions and velocities."""
    rng = np.random.default_rng(seed)
    k, j, i = np.meshgrid(np.arange(1, nz - 1), np.arange(1, int(0.7 * ny)), np.arange(1, nx - 1), indexing="ij")
    cells = np.stack([i.ravel(), j.ravel(), k.ravel()], 1).astype(np.float64)
    s = np.arange(8)
    sub = np.stack([0.25 + 0.5 * (s & 1), 0.25 + 0.5 * ((s >> 1) & 1), 0.25 + 0.5 * ((s >> 2) & 1)], 1)
    pos = (cells[:, None, :] + sub[None] + rng.uniform(-0.2, 0.2, (len(cells), 8, 3))).reshape(-1, 3) * dx
    c = cells + 0.5 - np.array([nx / 2, 0.3 * ny, nz / 2])
    gas = np.repeat(((c * c).sum(1) < (0.2 * nx) ** 2).astype(np.uint8), 8)
    vel = rng.normal(0.0, speed, pos.shape)
    return pos.astype(np.float32), vel.astype(np.float32), gas


def _pair(pf, n, dx, settings, pos, vel, typ, boxes=None):
    sim = pf.MRSim3DTP(*n, dx, max_particles=len(pos))
    for name in ("dt", "gravity", "Vp", "alpha_liquid", "alpha_gas", "advection_order", "cg_iters", "cg_tol",
                 "cg_rel_tol", "cg_jacobi_preconditioner", "cg_flexible_beta", "cg_adaptive_restart",
                 "cg_restart_growth", "dynamic_refinement", "dynamic_particle_padding", "dynamic_gas_padding",
                 "dynamic_hysteresis_cells", "dynamic_max_fine_leaves"):
        setattr(sim, name, getattr(settings, name))
    ph = settings.phase
    sim.phase = pf.PhaseParams(ph.rho_l, ph.rho_g, ph.alpha_phi, ph.rho_tilde_0)
    o = OracleMR(*n, dx, settings)
    if boxes is not None:
        sim.set_layout(boxes)
        o.set_layout(boxes)
    sim.set_particles(pos, vel, typ)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), typ)
    return sim, o


def test_mr_p2g_matches_oracle(pf):
    n, dx = (24, 20, 18), 1.0 / 16
    s = MRSettings(phase=_phase())
    pos, vel, typ = _scene(*n, dx, 1)
    sim, o = _pair(pf, n, dx, s, pos, vel, typ, boxes=[(4, 3, 2, 13, 9, 10)])
    assert np.array_equal(sim.levels(), o.levels())
    sim.p2g()
    o.p2g()
    for f in range(6):
        g, c = sim.face(f), o.face(f)
        # FP32 weights: a patch at the kernel's edge may get a weight of order
        # 1e-21 on one side only
        tiny = 1e-9 * float(np.abs(c).max())
        assert np.array_equal(np.abs(g) > tiny, np.abs(c) > tiny), f"face field {f}: touched patches differ"
        assert rel_err(g, c) < 1e-5, f"face field {f}: {rel_err(g, c)}"
    for ax in range(3):
        valid = o.face_valid(ax).astype(bool)
        assert not np.any(sim.face(3 + ax)[~valid]), "mass off the face list"
        assert np.array_equal(valid, pf.multires.valid_faces(sim.levels(), *n, ax))
    sim.close()


@pytest.mark.parametrize("order,flexible", [(2, False), (3, True)])
def test_mr_step_matches_oracle(pf, order, flexible):
    """One step on a static layout with coarse fluid cells beside fine ones
    and a domain that is not a multiple of the 8-cell block."""
    n, dx = (20, 13, 18), 1.0 / 16
    s = MRSettings(dt=1 / 60, phase=_phase(), dynamic_refinement=False, advection_order=order,
                   cg_flexible_beta=flexible, cg_iters=4000, cg_rel_tol=1e-10, cg_tol=0.0)
    pos, vel, typ = _scene(*n, dx, 3)
    sim, o = _pair(pf, n, dx, s, pos, vel, typ, boxes=[(3, 2, 5, 11, 7, 12)])
    st = sim.step()
    so, co = o.step()
    assert (st.active_cells, st.pinned_cell) == (so.active_cells, so.pinned_cell)
    assert st.converged and so.converged
    assert abs(st.iterations - so.iterations) <= max(3, so.iterations // 20), (st.iterations, so.iterations)
    mk, p = sim.cells()
    mo, po = o.cells()
    assert np.array_equal(mk, mo.astype(np.uint8)), "markers differ"
    assert rel_err(p, po) < 1e-5, f"pressure {rel_err(p, po)}"
    for f in range(9):
        err = rel_err(sim.face(f), o.face(f))
        assert err < 1e-5, f"face field {f}: {err}"
    gp, gv, _, _ = sim.get_particles()
    assert np.max(np.abs(gp - o.pos)) < 1e-5 * dx
    assert rel_err(gv, o.vel) < 1e-5
    assert (st.clamp.clamped_liquid, st.clamp.clamped_gas) == (co.clamped_liquid, co.clamped_gas)
    sim.close()


def test_mr_bubble_tank_dynamic_steps_track_oracle(pf):
    """The reference's bubble tank with dynamic refinement (MRSim3DTP
    defaults): the layout follows the particles exactly each step; fields and
    particles stay within 1e-4 of the oracle with FP32 particle state."""
    n, dx = (32, 40, 32), 1.0 / 32
    s = MRSettings(dt=1 / 120, phase=_phase(), cg_iters=2000, cg_rel_tol=1e-9, cg_tol=0.0)
    sim = pf.MRSim3DTP(*n, dx, max_particles=1 << 18)
    sim.dt, sim.cg_iters, sim.cg_rel_tol, sim.cg_tol = s.dt, s.cg_iters, s.cg_rel_tol, s.cg_tol
    sim.initBubbleTankInterfaceBand()
    ph = sim.phase
    assert ph.rho_tilde_0 == s.phase.rho_tilde_0
    pos, vel, typ, _ = sim.get_particles()
    o = OracleMR(*n, dx, s)
    o.set_particles(pos.astype(np.float64), vel.astype(np.float64), typ)
    o.update_refinement()
    assert np.array_equal(sim.levels(), o.levels())
    assert 0 < sim.levels().sum() < sim.levels().size
    for step in range(4):
        st = sim.step()
        so, _ = o.step()
        o.pos = o.pos.astype(np.float32).astype(np.float64)
        o.vel = o.vel.astype(np.float32).astype(np.float64)
        assert np.array_equal(sim.levels(), o.levels()), f"step {step}: layouts differ"
        assert st.active_cells == so.active_cells and st.converged
        mk, p = sim.cells()
        mo, po = o.cells()
        assert np.array_equal(mk, mo.astype(np.uint8)), f"step {step}: markers differ"
        assert rel_err(p, po) < 1e-4, f"step {step}: pressure {rel_err(p, po)}"
        gp, gv, _, _ = sim.get_particles()
        assert rel_err(gv, o.vel) < 1e-4, f"step {step}: velocities {rel_err(gv, o.vel)}"
        assert np.max(np.abs(gp - o.pos)) < 1e-4 * dx
    assert sim.activePressureCellCount() < n[0] * n[1] * n[2]
    assert sim.uFaceCount() == int(o.face_valid(0).sum())
    sim.close()


def test_mr_dynamic_refinement_matches_oracle(pf):
    n = (24, 16, 20)
    s = MRSettings(phase=_phase(), dynamic_particle_padding=1, dynamic_gas_padding=2, dynamic_hysteresis_cells=2,
                   dynamic_max_fine_leaves=40)
    sim = pf.MRSim3DTP(*n, 1.0, max_particles=256)
    sim.dynamic_particle_padding, sim.dynamic_gas_padding = 1, 2
    sim.dynamic_hysteresis_cells, sim.dynamic_max_fine_leaves = 2, 40
    o = OracleMR(*n, 1.0, s)
    rng = np.random.default_rng(4)
    centre = np.array([6.0, 5.0, 7.0])
    for move in range(6):
        pos = (centre + rng.uniform(-2.5, 2.5, (200, 3))).astype(np.float32)
        typ = (rng.uniform(size=200) < 0.2).astype(np.uint8)
        sim.set_particles(pos, np.zeros((200, 3)), typ)
        o.set_particles(pos.astype(np.float64), np.zeros((200, 3)), typ)
        assert np.array_equal(np.array(sim.updateDynamicRefinement()), o.update_refinement()), move
        assert np.array_equal(sim.levels(), o.levels())
        centre = centre + np.array([1.5, 0.5, 1.0]) * (move % 2 * 2 - 1) + np.array([0.7, 0.4, 0.6])
    sim.close()


def test_mr_face_shapes(pf):
    assert face_shape(5, 6, 7, 0) == (7, 6, 6)
