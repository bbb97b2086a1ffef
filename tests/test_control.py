"""The main loop's predictor/corrector control (timestep.F90 tim_check_cgce :744-830 and
tim_new_tstep :837-870) as the library runs it -- the same functions execute on the device
inside the one-graph step -- against the oracle's restatement, on host-side inputs only
(no device work): every exit of both controllers, including the ones a healthy run never
reaches (a growing corrector norm, more than 10 iterations, dt -> 0)."""
import importlib
import itertools

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
lsd = pkg.lsd

FIELDS = ("t", "dt", "dterr", "corr_dt", "lasterr", "cfl_dt", "it", "step", "pcn")


def state(**kw):
    s = capi.LsdPcState()
    base = dict(t=0.25, dt=1e-5, dterr=0.0, corr_dt=0.0, lasterr=1e99, cfl_dt=0.0, it=1, step=40, pcn=-1)
    base.update(kw)
    for k, v in base.items():
        setattr(s, k, v)
    return s


def copy(s):
    c = capi.LsdPcState()
    ctypes_fields = [f for f, _ in capi.LsdPcState._fields_]
    for f in ctypes_fields:
        setattr(c, f, getattr(s, f))
    return c


def cfg_for(control, **kw):
    base = dict(time_step_control=control, timestep=-5e-5, dterr=0.025, corr_upper=0.02, corr_lower=0.002)
    base.update(kw)
    return capi.template_config(**base)


def compare_check(cfg, s):
    a, b = copy(s), copy(s)
    ra = lsd.tim_check_cgce(cfg, a)
    rb = ol.tim_check_cgce(cfg, b)
    assert ra == rb, (ra, rb)
    for f in FIELDS:
        if f == "step" and rb != 0:
            continue  # the reference also ends the run (tim_step = i_maxtstep - 1)
        assert getattr(a, f) == getattr(b, f), (f, getattr(a, f), getattr(b, f))
    return ra, a


@pytest.mark.parametrize("control", [1, 2])
def test_check_cgce_matches_oracle_on_a_grid(control):
    cfg = cfg_for(control)
    dterrs = (1e-9, 1e-3, 0.02, 0.025, 0.03, 0.049, 0.06, 0.9, 1.0, 1.5, 3.0)
    lasts = (1e99, 0.5, 0.03, 2.0)
    n = 0
    for it, d, last, dt, step, pcn in itertools.product((1, 2, 5, 10, 11, 12), dterrs, lasts, (1e-5, 1e-13),
                                                        (0, 31), (-1, 2)):
        compare_check(cfg, state(it=it, dterr=d, lasterr=last, dt=dt, step=step, pcn=pcn))
        n += 1
    assert n > 1000


def test_check_cgce_exits_control1():
    cfg = cfg_for(1)
    rc, s = compare_check(cfg, state(it=1, dterr=0.01))  # converged at the first corrector
    assert rc == capi.LSD_OK and s.it == 0 and s.corr_dt == 0.01 and s.dterr == 0.0
    rc, s = compare_check(cfg, state(it=1, dterr=1.5))  # norm above 1: one more corrector
    assert rc == capi.LSD_OK and s.it == 2 and s.lasterr == 1.5
    rc, s = compare_check(cfg, state(it=3, dterr=2.0, lasterr=1.5))  # growing above 1: give up
    assert rc == capi.LSD_ENOTCONVERGED and s.it == 0
    rc, s = compare_check(cfg, state(it=3, dterr=0.8, lasterr=0.5))  # growing below 1: accept
    assert rc == capi.LSD_OK and s.it == 0
    rc, s = compare_check(cfg, state(it=11, dterr=1.2, lasterr=1.3))  # more than 10 iterations
    assert rc == capi.LSD_ENOTCONVERGED and s.it == 0
    rc, s = compare_check(cfg, state(it=2, dterr=1e-3, dt=1e-13, step=31))  # dt -> 0
    assert rc == capi.LSD_ENOTCONVERGED


def test_check_cgce_exits_control2():
    cfg = cfg_for(2)
    rc, s = compare_check(cfg, state(it=1, dterr=0.01, dt=1e-5))
    assert rc == capi.LSD_OK and s.it == 0 and s.corr_dt == 1e-5 * np.sqrt(0.025 / 0.01)
    rc, s = compare_check(cfg, state(it=1, dterr=0.03))  # above d_dterr: iterate
    assert rc == capi.LSD_OK and s.it == 2
    rc, s = compare_check(cfg, state(it=2, dterr=0.04, lasterr=0.03))  # growing, < 2 d_dterr
    assert rc == capi.LSD_OK and s.it == 0 and s.corr_dt == s.dt / (10 * cfg.courant)
    rc, s = compare_check(cfg, state(it=2, dterr=0.06, lasterr=0.03))  # growing, > 2 d_dterr
    assert rc == capi.LSD_ENOTCONVERGED
    rc, s = compare_check(cfg, state(it=11, dterr=0.03, lasterr=0.04))
    assert rc == capi.LSD_ENOTCONVERGED
    rc, s = compare_check(cfg, state(it=2, dterr=0.03, lasterr=0.04, pcn=2))  # tim_pcn correctors
    assert rc == capi.LSD_OK and s.it == 0


@pytest.mark.parametrize("control", [1, 2])
def test_new_tstep_matches_oracle(control):
    cfg = cfg_for(control)
    for dt, corr, cfl, step in itertools.product((1e-5, 3e-7), (0.0, 1e-4, 0.001, 0.01, 0.05, 1e-6),
                                                 (0.0, 1e-6, 1e-4), (0, 7)):
        a, b = state(dt=dt, corr_dt=corr, cfl_dt=cfl, step=step), state(dt=dt, corr_dt=corr, cfl_dt=cfl, step=step)
        na, nb = lsd.tim_new_tstep(cfg, a), ol.tim_new_tstep(cfg, b)
        assert na == nb and a.dt == b.dt, (dt, corr, cfl, step, a.dt, b.dt)
