"""Streamed inputs (lsd_stage_coll / lsd_commit_staged) against lsd_set_coll.

* Staging and committing the five fields (and the inner core's two) gives the same state
  as lsd_set_coll, bit for bit.
* A run that stages the next step's fields while each step runs (the pattern of the
  end-to-end measurement) produces, step by step, the same energies and coefficients as
  a run that uploads with lsd_set_coll before each step.
* A commit with nothing staged is refused (LSD_ESTATE) and leaves the context usable.
"""
import importlib

import numpy as np
import pytest

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def pinned_fields(cfg, seed):
    import torch
    out = {}
    for f, (re, im) in syn.boussinesq_state(cfg, seed=seed).items():
        pr = torch.empty(re.shape, dtype=torch.float64, pin_memory=True).numpy()
        pi = torch.empty(im.shape, dtype=torch.float64, pin_memory=True).numpy()
        pr[...] = re
        pi[...] = im
        out[f] = (pr, pi)
    return out


@pytest.mark.gpu
def test_stage_commit_equals_set_coll():
    cfg = syn.config_inner_core(L=16, N=17, Nic=9)
    a, b = pkg.Context(cfg), pkg.Context(cfg)
    fields = pinned_fields(cfg, 3)
    # the inner core's field: the outer core's value at r_i continued inwards as (r / r_i)^2
    ric = syn.inner_core_grid(cfg.Nic, cfg.rratio)
    w = (ric / ric[-1]) ** 2
    for f, fo in ((capi.MAG_IC_TOR, capi.MAG_TOR), (capi.MAG_IC_POL, capi.MAG_POL)):
        fields[f] = tuple(np.ascontiguousarray(x[:, :1] * w[None, :]) for x in fields[fo])
    a.load_fields(fields)
    b.stage_fields(fields)
    b.commit_staged()
    for f in fields:
        x, y = a.get_coll(f), b.get_coll(f)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), f
    with pytest.raises(pkg.LsdError):
        b.commit_staged()
    a.step(2)
    b.step(2)
    for f in fields:
        x, y = a.get_coll(f), b.get_coll(f)
        assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), f
    a.close()
    b.close()


@pytest.mark.gpu
def test_streamed_steps_equal_serial_steps():
    cfg = syn.config_parity(L=32, M=32, N=17)
    a, b = pkg.Context(cfg), pkg.Context(cfg)
    inputs = [pinned_fields(cfg, 10 + k) for k in range(4)]
    b.stage_fields(inputs[0])
    for k in range(4):
        a.load_fields(inputs[k])
        a.step(1)
        b.commit_staged()
        if k + 1 < 4:
            b.stage_fields(inputs[k + 1])  # crosses PCIe while this step runs
        b.step(1)
        ea, eb = a.energies(), b.energies()
        for key in ("KE", "ME", "KE_dis", "ME_dis"):
            assert ea[key] == eb[key], (k, key)
        for f in range(5):
            x, y = a.get_coll(f), b.get_coll(f)
            assert np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1]), (k, f)
    a.close()
    b.close()
