"""Ensembles: independent runs at their own resolutions stepped together (lsd_ensemble_*).

* A small mixed ensemble (anelastic L = 16 and 24 with composition, Boussinesq L = 32)
  against one oracle per member after 10 steps: energies 1e-9, coefficients 1e-10.
* The anelastic ensemble workload at full size: 8 members, two each at L = M = 64, 96,
  128, 192 with N = L + 1, the n = 2 polytrope (N_rho = 3) on each member's grid,
  codensity + composition, l^-2 seeded perturbations (a different seed per member).
  Checked by (a) the L = 64 member against the oracle after 5 steps (energies 1e-9) and
  (b) lock-step ensemble stepping against stand-alone stepping of the same member
  (identical coefficients: every sum that feeds the state, dterr included, is formed in
  a fixed order), then 200 ensemble steps.
"""
import importlib
import time

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def ensemble_configs():
    return [syn.config_anelastic(L=L) for L in (64, 64, 96, 96, 128, 128, 192, 192)]


def setup_member(ctx, cfg, seed):
    if not cfg.boussinesq:
        ctx.set_reference_state(syn.polytrope_reference_state(cfg.N, cfg.rratio))
    st = syn.boussinesq_state(cfg, seed=seed, composition=bool(cfg.comp_tstep))
    for f, (re, im) in st.items():
        ctx.set_coll(f, re, im)
    return st


@pytest.mark.gpu
def test_small_ensemble_against_oracle():
    cfgs = [syn.config_anelastic(L=16, N=17), syn.config_anelastic(L=24, N=25),
            syn.config_parity(L=32, M=32, N=17)]
    ens = pkg.Ensemble(cfgs)
    oracles = []
    for i, (m, cfg) in enumerate(zip(ens.members, cfgs)):
        st = setup_member(m, cfg, seed=100 + i)
        o = ol.Oracle(cfg)
        if not cfg.boussinesq:
            o.set_reference_state(syn.polytrope_reference_state(cfg.N, cfg.rratio))
        for f, (re, im) in st.items():
            o.set_coll(f, re, im)
        oracles.append(o)
    stats = ens.step(10)
    for i, (m, o) in enumerate(zip(ens.members, oracles)):
        so = o.step(10)
        assert stats[i].steps_done == so.steps_done == 10
        assert stats[i].correctors == so.correctors, i
        eg, eo = m.energies(), o.energies()
        for k in ("KE", "ME", "KE_dis", "ME_dis", "topflx", "botflx"):
            assert abs(eg[k] - eo[k]) <= 1e-9 * abs(eo[k]), (i, k, eg[k], eo[k])
        for f in range(6 if cfgs[i].comp_tstep else 5):
            a, b = m.get_coll(f), o.get_coll(f)
            assert relerr(a[0], b[0]) < 1e-10, (i, f)
            assert relerr(a[1], b[1]) < 1e-10, (i, f)
        o.close()
    ens.close()


@pytest.mark.gpu
def test_anelastic_ensemble_full_size():
    cfgs = ensemble_configs()
    ens = pkg.Ensemble(cfgs)
    for i, (m, cfg) in enumerate(zip(ens.members, cfgs)):
        setup_member(m, cfg, seed=syn.SEED + i)
    # (a) the L = 64 member against the oracle, 5 steps
    o = ol.Oracle(cfgs[0])
    o.set_reference_state(syn.polytrope_reference_state(cfgs[0].N, cfgs[0].rratio))
    for f, (re, im) in syn.boussinesq_state(cfgs[0], seed=syn.SEED, composition=True).items():
        o.set_coll(f, re, im)
    # (b) stand-alone contexts of one member of each resolution
    solo = {}
    for i in (0, 2, 4, 6):
        c = pkg.Context(cfgs[i])
        setup_member(c, cfgs[i], seed=syn.SEED + i)
        solo[i] = c
    stats = ens.step(5)
    so = o.step(5)
    assert stats[0].correctors == so.correctors
    eg, eo = ens.members[0].energies(), o.energies()
    for k in ("KE", "ME", "KE_dis", "ME_dis", "topflx", "botflx"):
        assert abs(eg[k] - eo[k]) <= 1e-9 * abs(eo[k]), (k, eg[k], eo[k])
    o.close()
    for i, c in solo.items():
        s = c.step(5)
        assert s.correctors == stats[i].correctors, i
        for f in range(6):
            a, b = c.get_coll(f), ens.members[i].get_coll(f)
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), (i, f)
        c.close()
    # 200 steps of the whole ensemble
    t0 = time.perf_counter()
    stats = ens.step(200)
    dt = time.perf_counter() - t0
    for i, s in enumerate(stats):
        assert s.steps_done == 200
        e = ens.members[i].energies()
        assert all(np.isfinite(v) for v in e.values()), i
    print("ensemble of 8 anelastic runs (L = 64..192): 200 steps in %.2f s (%.1f ensemble steps/s)"
          % (dt, 200 / dt))
    ens.close()
