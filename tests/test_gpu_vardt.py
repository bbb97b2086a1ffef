"""CFL / corrector-controlled timestep (d_timestep < 0): non_maxtstep + tim_new_tstep
before each predictor, operators rebuilt on a change (main.F90:126-134).

i_time_step_control = 2 (below) and i_time_step_control = 1, the controller of every
reference test case and of the Christensen benchmarks (tests/parameters-case1_symmetry.F90:
237-243: d_timestep = -5e-5, d_corr_upper = 0.02, d_corr_lower = 0.002): tim_corr_dt is
the corrector norm itself, dt halves above d_corr_upper, grows by 1.273974 below
d_corr_lower (kept within 3 %), the first step takes min(dt/1e3, 1e-8), and the corrector
repeats while its norm exceeds 1 (timestep.F90:744-777, 843-853).

CPU: the oracle's first step uses dt = min(dt/1e3, 1e-10) * courant (tim_step == 0,
timestep.F90:862) and later steps grow dt by at most 2/courant * courant = 2.
GPU: the device against the oracle step by step over 40 steps (Boussinesq) and 20 steps
(anelastic with composition): tim_dt and tim_cfl_dt to 1e-9 at every step (so every
3 % keep-or-change decision of tim_new_tstep agrees), tim_corr_dt to 1e-6 once dt has
grown past 1e-7 (step 12 on), the coefficients after the last step to 1e-9.  While dt is
tiny (8e-11 at step 0, doubling per step) the corrector norm behind
tim_corr_dt = dt sqrt(d_dterr / dterr) is close to the rounding level of the state
(dterr ~ 1e-13 at step 1), so its value there carries rounding noise in any
implementation; dt is then bound by the 2x growth limit, not by it.
"""
import importlib

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def test_oracle_first_step_dt():
    cfg = syn.config_parity(L=16, M=16, N=13, timestep=-1e-5)
    o = ol.Oracle(cfg)
    for f, (re, im) in syn.boussinesq_state(cfg).items():
        o.set_coll(f, re, im)
    o.set_time(0.0, 1e-5)
    o.step(1)
    dt, corr_dt, cfl_dt = o.dt_control()
    assert dt == min(min(cfl_dt, 1e-5) / 1e3, 1e-10) * cfg.courant
    prev = dt
    for _ in range(5):
        o.step(1)
        dt = o.dt_control()[0]
        assert dt <= 2.0 * prev * (1 + 1e-15)
        prev = dt
    o.close()


def run_pair(cfg, nsteps, prof=None, composition=False):
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    if prof is not None:
        g.set_reference_state(prof)
        o.set_reference_state(prof)
    for f, (re, im) in syn.boussinesq_state(cfg, seed=17, composition=composition).items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)
    g.set_time(0.0, 1e-5)
    o.set_time(0.0, 1e-5)
    for k in range(nsteps):
        sg, so = g.step(1), o.step(1)
        assert sg.correctors == so.correctors, k
        a, b = g.dt_control(), o.dt_control()
        for j, tol in ((0, 1e-9), (1, 1e-6 if k >= 12 else 1.0), (2, 1e-9)):
            assert abs(a[j] - b[j]) <= tol * abs(b[j]), (k, j, a, b)
    print("dt after %d steps: %.3e (oracle %.3e)" % (nsteps, a[0], b[0]))
    for f in range(6 if composition else 5):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-9, f
        assert relerr(a[1], b[1]) < 1e-9, f
    t_dev, t_orc = g.get_time()[0], o.energies()["time"]
    assert abs(t_dev - t_orc) <= 1e-12 * t_orc
    g.close()
    o.close()


@pytest.mark.gpu
def test_variable_dt_boussinesq():
    run_pair(syn.config_parity(N=17, timestep=-1e-5), 40)


@pytest.mark.gpu
def test_variable_dt_anelastic():
    cfg = syn.config_anelastic(L=16, N=17, timestep=-5e-5)
    run_pair(cfg, 20, prof=syn.polytrope_reference_state(cfg.N, cfg.rratio), composition=True)


def control1_cfg(**kw):
    base = dict(N=17, timestep=-5e-5, time_step_control=1, corr_upper=0.02, corr_lower=0.002)
    base.update(kw)
    return syn.config_parity(**base)


def test_oracle_control1_dt_rules():
    """The oracle's tim_new_tstep under i_time_step_control = 1: the first dt is
    min(dt/1e3, 1e-8); afterwards each dt is the previous one, halved, or grown by
    1.273974, as tim_corr_dt (the last corrector norm) lies above d_corr_upper, below
    d_corr_lower or between (timestep.F90:843-853)."""
    cfg = control1_cfg(L=16, M=16, N=13)
    o = ol.Oracle(cfg)
    for f, (re, im) in syn.boussinesq_state(cfg, seed=3).items():
        o.set_coll(f, re, im)
    o.set_time(0.0, 5e-5)
    o.step(1)
    dt = o.dt_control()[0]
    assert dt == min(5e-5 / 1e3, 1e-8)
    grew = False
    for _ in range(12):
        corr = o.dt_control()[1]
        o.step(1)
        new = o.dt_control()[0]
        want = dt * (0.5 if corr > cfg.corr_upper else 1.273974 if corr < cfg.corr_lower else 1.0)
        if not (want < dt * 0.97 or want > dt * 1.03):
            want = dt
        assert new == want, (dt, corr, new)
        grew |= new > dt
        dt = new
    assert grew
    o.close()


@pytest.mark.gpu
def test_variable_dt_control1():
    """Device against the oracle step by step under i_time_step_control = 1: the dt
    sequence and the corrector count at every step, tim_corr_dt (the corrector norm) to
    1e-6 (while dt is tiny the norm is close to the rounding level of the state: 2e-10 at
    dt = 1.6e-8, where the two differ by 3e-9 of it; the decisions it drives compare it
    with d_corr_lower = 0.002), the state at the end."""
    cfg = control1_cfg()
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    for f, (re, im) in syn.boussinesq_state(cfg, seed=23).items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)
    g.set_time(0.0, 5e-5)
    o.set_time(0.0, 5e-5)
    for k in range(30):
        sg, so = g.step(1), o.step(1)
        assert sg.correctors == so.correctors, k
        a, b = g.dt_control(), o.dt_control()
        assert a[0] == b[0] or abs(a[0] - b[0]) <= 1e-12 * b[0], (k, a, b)
        assert abs(a[1] - b[1]) <= 1e-6 * abs(b[1]), (k, a, b)
    for f in range(5):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-10, f
        assert relerr(a[1], b[1]) < 1e-10, f
    g.close()
    o.close()
