"""The step's own controls on the GPU: the adaptive timestep
(computeAdaptiveParticleTimestep3D, src/driver/timestep3d.h:16-50) and the
volume-correcting divergence target (updateVolumeCorrectionStats,
src/driver/sparse_sim3d_tp.cpp:368-379), applied by pf_step after the
particle adaptivity as SparseSim3DTP::step() does."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sim(pf, n=16, seed=4, speed=0.0, **kw):
    sc = pf.scenes.rayleigh_taylor(n, seed=seed)
    vel = sc["vel"].copy()
    if speed:
        rng = np.random.default_rng(seed)
        vel = rng.normal(0, speed, vel.shape).astype(np.float32)
    sim = pf.SparseSim3DTP(n, n, n, 1.0 / n, max_particles=len(sc["pos"]))
    sim.phase = pf.PhaseParams(sc["rho_l"], sc["rho_g"])
    sim.phase.rho_tilde_0 = pf.calibrateRhoTilde0(sim.phase, 1.0)
    sim.dt = 1 / 120
    sim.solver = pf.SolverConfig(rel_tol=1e-8)
    sim.cg_iters, sim.cg_tol = 4000, 0.0
    for k, v in kw.items():
        setattr(sim, k, v)
    sim.set_particles(sc["pos"], vel, sc["type"], sc["volume"])
    return sim, sc, vel


def _stepped(pf, speed=3.0, **kw):
    sim, _, _ = _sim(pf, speed=speed, **kw)
    sim.step()
    return sim


def _distance(a, b):
    """max |velocity difference| after the step, over the velocity scale"""
    va, vb = a.get_particles()[1].astype(np.float64), b.get_particles()[1].astype(np.float64)
    return float(np.max(np.abs(va - vb)) / np.max(np.abs(vb)))


def test_adaptive_timestep_limits_dt_and_the_step_uses_it(pf):
    sim, sc, vel = _sim(pf, speed=3.0, adaptive_timestep=True, adaptive_cfl=0.5, adaptive_min_dt=1e-5)
    sim.step()
    v = vel.astype(np.float64)
    vmax = float(np.max(np.sqrt(v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])))
    assert sim.max_particle_speed_last == vmax
    cfl_dt = 0.5 * (1.0 / 16) / vmax
    assert sim.cfl_limit_dt_last == cfl_dt
    expected = min(1 / 120, max(1e-5, min(1 / 120, cfl_dt)))
    assert sim.effective_dt_last == expected and sim.adaptive_timestep_limited_last == 1
    # the step ran with the effective dt: it matches a step with the controls off
    # and dt = effective dt (to P2G's atomic-order rounding), not one with dt
    assert _distance(sim, _stepped(pf, dt=expected)) < 1e-2 * _distance(sim, _stepped(pf, dt=1 / 120))


def test_adaptive_timestep_off_reports_speed_and_keeps_dt(pf):
    sim, _, vel = _sim(pf, speed=3.0)
    sim.step()
    assert sim.effective_dt_last == 1 / 120 and sim.adaptive_timestep_limited_last == 0
    assert sim.max_particle_speed_last > 0.0


def test_volume_correction_sets_the_divergence_target(pf):
    sc = pf.scenes.rayleigh_taylor(16, seed=4)
    liquid = sc["type"] == 0
    vol = float(np.sum(sc["volume"][liquid].astype(np.float64)))  # Vp = 1
    target = 1.02 * vol
    sim, _, _ = _sim(pf, c_div_volume_correction=True, c_div_strength=0.7, liquid_volume_target=target)
    sim.step()
    assert sim.liquid_volume_current_last == pytest.approx(vol, rel=1e-12)
    err = target - sim.liquid_volume_current_last
    assert sim.liquid_volume_error_last == err
    assert sim.c_div_last == 0.7 * err / ((1 / 120) * target) and sim.c_div_last > 0.0
    # the projection used that c_div: the step matches one without the correction
    # but with c_div given (to P2G's atomic-order rounding), not one with c_div 0
    same = _distance(sim, _stepped(pf, speed=0.0, c_div_last=sim.c_div_last))
    assert same < 1e-2 * _distance(sim, _stepped(pf, speed=0.0, c_div_last=0.0))
