"""The 2-level multires restatement (oracle/pf_oracle_mr.c) against the
reference's own MRSim3DTP (src/driver/multires_sim3d_tp.cpp:671-733), compiled
from its sources into oracle/_ref.  Both run in FP64 in the same operation
order, so layouts, face lists, fields, markers, pressure, particles and the
solver's statistics must agree bit for bit, step after step.

Cases:
* the reference's bubble tank (initBubbleTankInterfaceBand) with dynamic
  refinement, the MRSim3DTP defaults;
* a static layout with coarse fluid cells beside fine ones (dynamic
  refinement off) on a domain that is not a multiple of the 8-cell level-1
  block, RK3 advection, flexible beta;
* the dynamic refinement box logic alone: padding, hysteresis and the
  fine-leaf budget.
"""
import numpy as np
import pytest

import oracle as O
from oracle.multires import MRSettings, OracleMR, ReferenceMR

pytestmark = pytest.mark.skipif(not O.reference_available(), reason="compiled reference (oracle/_ref) not built")


def _phase(Vp=1.0):
    pp = O.PhaseParams(1.0, 0.01)
    pp.rho_tilde_0 = O.Oracle().calibrate_rho_tilde0(pp, Vp)
    return pp


def _same(a, b):
    return np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))


def _compare(o, r, label):
    assert np.array_equal(o.levels(), r.levels()), f"{label}: layouts differ"
    for ax in range(3):
        assert np.array_equal(o.face_valid(ax), r.face_valid(ax)), f"{label}: face lists differ (axis {ax})"
    for f in range(6):
        assert _same(o.face(f), r.face(f)), f"{label}: face field {f} differs"
    mo, po = o.cells()
    mr, pr = r.cells()
    assert _same(mo, mr), f"{label}: markers differ"
    assert _same(po, pr), f"{label}: pressure differs"
    assert _same(o.pos, r.pos) and _same(o.vel, r.vel), f"{label}: particles differ"


def _stats_equal(a, b):
    for name in ("active_cells", "pinned_cell", "iterations", "restarts", "beta_resets", "converged", "breakdown"):
        assert getattr(a, name) == getattr(b, name), (name, getattr(a, name), getattr(b, name))
    for name in ("initial_residual", "final_residual", "effective_tolerance"):
        assert getattr(a, name) == getattr(b, name), (name, getattr(a, name), getattr(b, name))


def test_bubble_tank_dynamic_refinement_steps_equal_reference():
    n = (16, 24, 16)
    s = MRSettings(dt=1 / 120, phase=_phase())
    r = ReferenceMR(*n, 1.0 / 16, s)
    r.init_bubble_tank()
    o = OracleMR(*n, 1.0 / 16, s)
    o.set_particles(r.pos, r.vel, r.type, r.volume)
    o.set_levels(r.levels())
    o.update_refinement()  # the retained box the reference's init left behind
    assert np.array_equal(o.levels(), r.levels())
    for step in range(3):
        so, co = o.step()
        sr, cr = r.step()
        _stats_equal(so, sr)
        assert (co.clamped_liquid, co.clamped_gas) == (cr.clamped_liquid, cr.clamped_gas)
        _compare(o, r, f"step {step}")
    assert 0 < o.fine_leaves() == r.fine_leaves()
    assert so.active_cells > 0 and so.iterations > 0


def _coarse_fluid_scene(nx, ny, nz, dx, seed):
    rng = np.random.default_rng(seed)
    pos, vel, typ = [], [], []
    for k in range(1, nz - 1):
        for j in range(1, int(0.7 * ny)):
            for i in range(1, nx - 1):
                for s in range(8):
                    p = np.array([i + 0.25 + 0.5 * (s & 1), j + 0.25 + 0.5 * ((s >> 1) & 1),
                                  k + 0.25 + 0.5 * ((s >> 2) & 1)]) + rng.uniform(-0.2, 0.2, 3)
                    pos.append(p * dx)
                    c = np.array([i + 0.5 - nx / 2, j + 0.5 - 0.3 * ny, k + 0.5 - nz / 2])
                    typ.append(1 if (c * c).sum() < (0.2 * nx) ** 2 else 0)
                    vel.append(rng.normal(0.0, 0.3, 3))
    return np.array(pos), np.array(vel), np.array(typ, np.uint8)


def test_static_layout_with_coarse_fluid_equals_reference():
    n = (20, 13, 18)
    dx = 1.0 / 16
    s = MRSettings(dt=1 / 60, phase=_phase(), dynamic_refinement=False, advection_order=3, cg_flexible_beta=True,
                   cg_iters=400)
    pos, vel, typ = _coarse_fluid_scene(*n, dx, 3)
    boxes = [(3, 2, 5, 11, 7, 12)]
    r = ReferenceMR(*n, dx, s)
    r.set_layout(boxes)
    r.set_particles(pos, vel, typ)
    o = OracleMR(*n, dx, s)
    o.set_layout(boxes)
    o.set_particles(pos, vel, typ)
    assert np.array_equal(o.levels(), r.levels())
    assert 0 < int(o.levels().sum()) < o.levels().size  # both levels present
    for step in range(2):
        so, co = o.step()
        sr, cr = r.step()
        _stats_equal(so, sr)
        assert co.as_tuple()[:2] == (cr.clamped_liquid, cr.clamped_gas)
        _compare(o, r, f"step {step}")
    mk, _ = o.cells()
    lv = np.repeat(np.repeat(np.repeat(o.levels(), 8, 0), 8, 1), 8, 2)[: n[2], : n[1], : n[0]]
    assert np.any((mk == 1) & (lv == 0)), "no coarse fluid cell in the scene"
    assert np.any((mk == 1) & (lv == 1)), "no fine fluid cell in the scene"


@pytest.mark.parametrize("budget", [0, 40])
def test_dynamic_refinement_box_equals_reference(budget):
    n = (24, 16, 20)
    s = MRSettings(phase=_phase(), dynamic_particle_padding=1, dynamic_gas_padding=2, dynamic_hysteresis_cells=2,
                   dynamic_max_fine_leaves=budget)
    r = ReferenceMR(*n, 1.0, s)
    o = OracleMR(*n, 1.0, s)
    rng = np.random.default_rng(budget + 1)
    centre = np.array([6.0, 5.0, 7.0])
    for move in range(6):
        pos = centre + rng.uniform(-2.5, 2.5, (200, 3))
        typ = (rng.uniform(size=200) < 0.2).astype(np.uint8)
        vel = np.zeros((200, 3))
        r.set_particles(pos, vel, typ)
        o.set_particles(pos, vel, typ)
        sr = r.update_refinement()
        so = o.update_refinement()
        assert np.array_equal(sr, so), (move, sr, so)
        assert np.array_equal(o.levels(), r.levels())
        assert o.fine_leaves() == r.fine_leaves()
        centre = centre + np.array([1.5, 0.5, 1.0]) * (move % 2 * 2 - 1) + np.array([0.7, 0.4, 0.6])


@pytest.mark.parametrize("n,boxes", [((20, 13, 18), [(3, 2, 5, 11, 7, 12)]), ((16, 24, 16), [(0, 0, 0, 16, 14, 16)]),
                                     ((9, 17, 7), [(8, 0, 0, 9, 9, 7), (0, 16, 0, 2, 17, 2)])])
def test_closed_form_face_list_equals_oracle(pf, n, boxes):
    """The GPU's face-patch rule (even position, far side, or beside a refined
    block) written in numpy in the package, against the restated face list."""
    o = OracleMR(*n, 1.0)
    o.set_layout(boxes)
    for ax in range(3):
        assert np.array_equal(pf.multires.valid_faces(o.levels(), *n, ax), o.face_valid(ax).astype(bool))
