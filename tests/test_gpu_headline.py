"""The device path pinned to the reference's own output, and the headline resolution
(lmax 127, Nr 129) against the oracle.

* The Christensen case 1 state of the reference (tests/state.cdf.in, read through
  state.load_state) advanced by the reference's first step (dt = 4.59265755232e-6): the
  device agrees with the oracle to 1e-12 per coefficient, and both reproduce the
  increments of the reference's second output row within the bands of
  tests/case1_fixture.py.
* L = M = 128, N = 129 (Th = 192, Ph = 384), the seeded l^-2 state, dt = 2e-6: three
  steps of the plain FP64 device path against the oracle, coefficients to 1e-12 of each
  field's largest magnitude and energies to 1e-12; the tensor-core path at five int8
  slices (the benchmark's setting) to the tolerances stated below.
"""
import importlib
import os

import numpy as np
import pytest

import case1_fixture as case1
import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic
ENERGY_KEYS = ("KE", "ME", "KE_ax", "ME_ax", "KE_dis", "ME_dis", "topflx", "botflx")


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def coeff_err(g, o, fields=range(5)):
    worst = 0.0
    for f in fields:
        a, b = g.get_coll(f), o.get_coll(f)
        worst = max(worst, relerr(a[0], b[0]), relerr(a[1], b[1]))
    return worst


@pytest.mark.gpu
def test_golden_first_step_on_device(parity_report):
    r0, r1 = case1.golden_rows()
    cfg = case1.config(timestep=r1["time"], time_step_control=1)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    fields, _ = case1.load(cfg)
    for f, (re, im) in fields.items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)
    before = case1.dat_columns(g.energies(), cfg.Pm)
    sg, so = g.step(1), o.step(1)
    assert sg.steps_done == so.steps_done == 1 and sg.correctors == so.correctors == 1
    err = coeff_err(g, o)
    parity_report("case1 first step, device vs oracle coefficients", err, 1e-12)
    assert err <= 1e-12, err
    after = case1.dat_columns(g.energies(), cfg.Pm)
    ratios = case1.check_first_step(before, after)
    for k, v in ratios.items():
        parity_report("case1 first step, increment of %s / reference's" % k, v)
    g.close()
    o.close()


@pytest.fixture(scope="module")
def dynamo128_oracle():
    """The oracle's state and energies after 3 steps at L = M = 128, N = 129."""
    ol.set_threads(os.cpu_count() or 1)
    cfg = syn.config_dynamo128()
    o = ol.Oracle(cfg)
    init = syn.boussinesq_state(cfg)
    for f, (re, im) in init.items():
        o.set_coll(f, re, im)
    st = o.step(3)
    out = {f: o.get_coll(f) for f in range(5)}
    e = o.energies()
    o.close()
    return init, out, e, st


# (precision, slices, coefficient tolerance, energy tolerance)
DYNAMO128_CASES = [
    (capi.PREC_FP64, 0, 1e-12, 1e-12),
    (capi.PREC_OZAKI, 5, 1e-9, 1e-11),
]


@pytest.mark.gpu
@pytest.mark.parametrize("prec,S,tol_c,tol_e", DYNAMO128_CASES)
def test_dynamo128_steps_vs_oracle(dynamo128_oracle, parity_report, prec, S, tol_c, tol_e):
    init, ref, eo, so = dynamo128_oracle
    g = pkg.Context(syn.config_dynamo128(precision=prec, ozaki_slices=S))
    for f, (re, im) in init.items():
        g.set_coll(f, re, im)
    sg = g.step(3)
    assert sg.steps_done == so.steps_done == 3 and sg.correctors == so.correctors
    worst = 0.0
    for f in range(5):
        a, b = g.get_coll(f), ref[f]
        worst = max(worst, relerr(a[0], b[0]), relerr(a[1], b[1]))
    eg = g.energies()
    werr = max(abs(eg[k] - eo[k]) / abs(eo[k]) for k in ENERGY_KEYS)
    tag = "FP64" if prec == capi.PREC_FP64 else "tensor cores S=%d" % S
    parity_report("lmax127 Nr129 3 steps %s: coefficients" % tag, worst, tol_c)
    parity_report("lmax127 Nr129 3 steps %s: energies" % tag, werr, tol_e)
    assert worst <= tol_c, worst
    assert werr <= tol_e, werr
    g.close()
