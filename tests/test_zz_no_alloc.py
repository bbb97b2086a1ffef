"""lsd_energies_static (no allocation, static device scratch) against lsd_energies.

Collected last (file name), so it runs both alone in a fresh process and after every
other test of the suite.  Two calls in a row check that nothing of the previous call's
scratch contents leaks into the next: every slot is overwritten by a fixed-order tree sum
(no atomics), so the two entry points give the same bits.
"""
import importlib

import numpy as np
import pytest

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def test_static_energies_exported():
    lib = pkg.load_library()
    assert hasattr(lib, "lsd_energies_static")


@pytest.mark.gpu
def test_static_energies_match_twice_in_a_row():
    cfg = syn.config_parity(N=17)
    g = pkg.Context(cfg)
    for f, (re, im) in syn.boussinesq_state(cfg).items():
        g.set_coll(f, re, im)
    for _ in range(2):
        a = g.energies_static()
        b = g.energies()
        for k in capi.ENERGY_NAMES:
            assert a[k] == b[k], (k, a[k], b[k])
    g.step(3)
    a, b = g.energies_static(), g.energies()
    for k in capi.ENERGY_NAMES:
        assert a[k] == b[k], (k, a[k], b[k])
    g.close()


@pytest.mark.gpu
def test_static_energies_few_harmonics():
    """A run with very few harmonics (L = M = 4, Mp = 1: H = 10) still has pinned staging
    room for the energies (the context sizes it at creation)."""
    cfg = capi.template_config(L=4, M=4, Mp=1, N=33, timestep=1e-6)
    g = pkg.Context(cfg)
    for f, (re, im) in syn.boussinesq_state(cfg).items():
        g.set_coll(f, re, im)
    a, b = g.energies_static(), g.energies()
    for k in capi.ENERGY_NAMES:
        assert a[k] == b[k], (k, a[k], b[k])
    g.close()


@pytest.mark.gpu
def test_static_energies_reject_more_shells_than_the_scratch():
    cfg = capi.template_config(L=4, M=4, Mp=1, N=1030, timestep=1e-6)
    g = pkg.Context(cfg)
    with pytest.raises(pkg.LsdError) as e:
        g.energies_static()
    assert e.value.status == capi.LSD_EARG
    assert "1024" in str(e.value)
    g.close()
