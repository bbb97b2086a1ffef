"""Composition (two-component convection, composition.F90, nonlinear.F90:294-357) on the
device against the oracle.

Size-independent property (CPU, oracle only): with Sc = Pr, comp_bc = cod_bc, the same
boundary values and sources and Ra_comp = 0, composition obeys the codensity's equation
with the codensity's initial value, so Comp(t) == C(t) and comp_NC == cod_NC exactly
(the velocity does not feel the composition when Ra_comp = 0).

Parity (GPU, through the C ABI), relative to the largest magnitude of the compared array:
  one nonlinear evaluation, predictor, corrector  1e-11 (FP64), 5e-11 (tensor cores, S = 7)
  100 steps: energies 1e-9, coefficients 1e-10
"""
import importlib

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def comp_cfg(**kw):
    base = dict(N=17, comp_tstep=1, Ra_comp=150.0, Sc=3.0, comp_bc=1, source_comp=0.25)
    base.update(kw)
    return syn.config_parity(**base)


def test_oracle_composition_tracks_codensity():
    cfg = comp_cfg(L=16, M=16, N=13, Ra_comp=0.0, Sc=1.0, source_comp=0.0)
    o = ol.Oracle(cfg)
    st = syn.boussinesq_state(cfg)
    for f, (re, im) in st.items():
        o.set_coll(f, re, im)
    o.set_coll(capi.COMP_C, *st[capi.COD_C])
    o.nonlinear()
    a, b = o.get_nonlinear(capi.N_COMP), o.get_nonlinear(capi.N_COD)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    o.step(5)
    a, b = o.get_coll(capi.COMP_C), o.get_coll(capi.COD_C)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    o.close()


def load_both(g, o, fields):
    for f, (re, im) in fields.items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)


@pytest.mark.gpu
@pytest.mark.parametrize("prec,S,tol", [(capi.PREC_FP64, 0, 1e-11), (capi.PREC_OZAKI, 7, 5e-11)])
def test_composition_evaluation_and_step(prec, S, tol):
    cfg = comp_cfg()
    g = pkg.Context(comp_cfg(precision=prec, ozaki_slices=S))
    o = ol.Oracle(cfg)
    load_both(g, o, syn.boussinesq_state(cfg, seed=7, composition=True))
    g.nonlinear()
    o.nonlinear()
    for w in range(6):
        a, b = g.get_nonlinear(w), o.get_nonlinear(w)
        assert relerr(a[0], b[0]) < tol, ("nl", w)
        assert relerr(a[1], b[1]) < tol, ("nl", w)
    g.predictor(); o.predictor()
    g.nonlinear(); o.nonlinear()
    d1, d2 = g.corrector(), o.corrector()
    assert abs(d1 - d2) <= 1e-9 * abs(d2)
    for f in range(6):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < tol, ("corr", f)
        assert relerr(a[1], b[1]) < tol, ("corr", f)
    g.close()
    o.close()


@pytest.mark.gpu
def test_composition_hundred_steps():
    """L = M = 32, N = 33, dt = 1e-5, Ra_comp = 150, Sc = 3, 100 steps (FP64)."""
    cfg = comp_cfg(N=33)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    load_both(g, o, syn.boussinesq_state(cfg, composition=True))
    sg, so = g.step(100), o.step(100)
    assert sg.steps_done == so.steps_done == 100
    assert sg.correctors == so.correctors
    eg, eo = g.energies(), o.energies()
    for k in ("KE", "ME", "KE_dis", "ME_dis", "topflx", "botflx"):
        assert abs(eg[k] - eo[k]) <= 1e-9 * abs(eo[k]), (k, eg[k], eo[k])
    for f in range(6):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-10, f
        assert relerr(a[1], b[1]) < 1e-10, f
    g.close()
    o.close()
