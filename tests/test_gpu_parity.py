"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Tolerances (relative to the largest magnitude of the compared array):
  integer layouts                  bit-exact
  tables, grid, weights            1e-13
  single transforms                1e-12
  one nonlinear evaluation / step  1e-11
  energies after 100 steps         1e-9
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
state = pkg.state
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    s = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / s)


def small_cfg(**kw):
    base = dict(N=17)
    base.update(kw)
    return syn.config_parity(**base)


@pytest.fixture(scope="module")
def pair():
    cfg = small_cfg()
    return pkg.Context(cfg), ol.Oracle(cfg), cfg


def test_library_exports_every_header_symbol():
    lib = pkg.load_library()
    for name in pkg.lsd.exported_symbols():
        assert hasattr(lib, name), name


@pytest.mark.gpu
def test_layout_tables_grid(pair):
    g, o, cfg = pair
    for a, b in zip(g.harmonics(), o.harmonics()):
        assert (a == b).all()
    assert (g.theta_map() == o.theta_map()).all()
    assert relerr(g.radial_grid(), o.radial_grid()) < 1e-15
    assert relerr(g.radial_weights(), o.radial_weights()) < 1e-12
    gp, gw = g.gauss()
    gp2, gw2 = o.gauss()
    assert np.abs(gp - gp2).max() < 1e-15
    assert relerr(gw, gw2) < 1e-13
    for t in range(8):
        assert relerr(g.legendre_table(t), o.legendre_table(t)) < 1e-13, capi.LEG_NAMES[t]


@pytest.mark.gpu
@pytest.mark.parametrize("LMMp", [(32, 32, 1), (64, 16, 4), (24, 8, 2), (64, 64, 1)])
def test_transforms(LMMp):
    L, M, Mp = LMMp
    cfg = capi.template_config(L=L, M=M, Mp=Mp, N=9, timestep=1e-5)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    rng = np.random.default_rng(L + M)
    l, m, s = o.harmonics()
    H, N = o.H, o.N

    def spec():
        re = rng.standard_normal((N, H))
        im = rng.standard_normal((N, H))
        im[:, m == 0] = 0
        return re, im

    sre, sim = spec()
    assert relerr(g.tra_spec2phys(sre, sim), o.spec2phys(sre, sim)) < 1e-12
    p = rng.standard_normal((N, o.Ph, o.Th))
    a, b = g.tra_phys2spec(p), o.phys2spec(p)
    assert relerr(a[0], b[0]) < 1e-12 and relerr(a[1], b[1]) < 1e-12
    q, sv, tv = spec(), spec(), spec()
    for x, y in zip(g.tra_qst2rtp(q, sv, tv), o.qst2rtp(q, sv, tv)):
        assert relerr(x, y) < 1e-12
    r, th, ph = (rng.standard_normal((N, o.Ph, o.Th)) for _ in range(3))
    for x, y in zip(g.tra_rtp2qst(r, th, ph), o.rtp2qst(r, th, ph)):
        assert relerr(x[0], y[0]) < 1e-12 and relerr(x[1], y[1]) < 1e-12
    for x, y in zip(g.tra_grad(sre, sim), o.grad(sre, sim)):
        assert relerr(x, y) < 1e-12
    g.close()


def load_both(g, o, fields):
    for f, (re, im) in fields.items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)


@pytest.mark.gpu
def test_nonlinear_terms(pair):
    g, o, cfg = pair
    load_both(g, o, syn.boussinesq_state(cfg))
    g.nonlinear()
    o.nonlinear()
    for w in range(5):
        a, b = g.get_nonlinear(w), o.get_nonlinear(w)
        assert relerr(a[0], b[0]) < 1e-11, w
        assert relerr(a[1], b[1]) < 1e-11, w


@pytest.mark.gpu
def test_predictor_corrector(pair):
    g, o, cfg = pair
    load_both(g, o, syn.boussinesq_state(cfg, seed=5))
    g.nonlinear(); o.nonlinear()
    g.predictor(); o.predictor()
    for f in range(5):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-11, ("pred", f)
        assert relerr(a[1], b[1]) < 1e-11, ("pred", f)
    g.nonlinear(); o.nonlinear()
    d1 = g.corrector()
    d2 = o.corrector()
    assert abs(d1 - d2) <= 1e-10 * abs(d2)
    for f in range(5):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-11, ("corr", f)
        assert relerr(a[1], b[1]) < 1e-11, ("corr", f)


@pytest.mark.gpu
def test_hundred_steps_energies():
    """The plain FP64 Boussinesq shell at L=M=32, N=33, dt=1e-5, 100 steps."""
    cfg = syn.config_parity()
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    load_both(g, o, syn.boussinesq_state(cfg))
    sg = g.step(100)
    so = o.step(100)
    assert sg.steps_done == so.steps_done == 100
    assert sg.correctors == so.correctors
    eg, eo = g.energies(), o.energies()
    for k in ("KE", "ME", "KE_ax", "ME_ax", "KE_dis", "ME_dis", "topflx", "botflx"):
        assert abs(eg[k] - eo[k]) <= 1e-9 * abs(eo[k]), (k, eg[k], eo[k])
    for f in range(5):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-10, f
    g.close()


@pytest.mark.gpu
def test_golden_t0_energies_on_device(parity_report):
    """Device energies of the reference's tests/state.cdf.in (read by state.load_state)
    equal its own t=0 output row."""
    cfg = case1.config()
    g = pkg.Context(cfg)
    fields, r = case1.load(cfg)
    assert np.abs(g.radial_grid() - r).max() < 1e-14
    for f, (re, im) in fields.items():
        g.set_coll(f, re, im)
    e = case1.dat_columns(g.energies(), cfg.Pm)
    want = case1.golden_rows()[0]
    worst = 0.0
    for k in ("KE", "KE_ax", "topflx", "botflx", "Edis", "ME", "ME_ax", "Mdis", "dipole"):
        err = abs(e[k] - want[k]) / abs(want[k])
        worst = max(worst, err)
        assert err <= 1e-11, (k, e[k], want[k])
    parity_report("t=0 energies vs reference row, max rel", worst, 1e-11)
    g.close()


@pytest.mark.gpu
def test_batched_banded_solve():
    """One launch factorises every operator, one launch solves every right-hand side;
    compared with LAPACK (scipy) and by the residual."""
    import scipy.linalg.lapack as lapack
    import torch
    n, kl, nmat, nrhs = 65, 4, 12, 300
    rng = np.random.default_rng(11)
    ab = np.zeros((nmat, n, 3 * kl + 1))
    ab[:, :, kl:] = rng.standard_normal((nmat, n, 2 * kl + 1))
    ab[:, :, 2 * kl] += 4.0
    cfg = small_cfg()
    g = pkg.Context(cfg)
    d_ab = torch.tensor(ab, device="cuda", dtype=torch.float64)
    d_ip = torch.zeros((nmat, n), device="cuda", dtype=torch.int32)
    d_info = torch.zeros(nmat, device="cuda", dtype=torch.int32)
    g.banded_factor_device(n, kl, nmat, d_ab.data_ptr(), d_ip.data_ptr(), d_info.data_ptr())
    g.synchronize()
    assert (d_info.cpu().numpy() == 0).all()
    lu_g = d_ab.cpu().numpy()
    for k in range(nmat):
        lu_l, ip_l, info = lapack.dgbtrf(ab[k].T.copy(), kl, kl)
        assert relerr(lu_g[k].T, lu_l) < 1e-13
        assert (d_ip.cpu().numpy()[k] == ip_l + 1).all()
    rmap = rng.integers(0, nmat, nrhs).astype(np.int32)
    b = rng.standard_normal((n, nrhs))
    d_b = torch.tensor(b, device="cuda", dtype=torch.float64)
    d_map = torch.tensor(rmap, device="cuda")
    g.banded_solve_device(n, kl, nmat, d_ab.data_ptr(), d_ip.data_ptr(), nrhs, d_map.data_ptr(), d_b.data_ptr())
    g.synchronize()
    x = d_b.cpu().numpy()
    for r in range(0, nrhs, 7):
        k = rmap[r]
        A = np.zeros((n, n))
        for j in range(n):
            for i in range(max(0, j - kl), min(n, j + kl + 1)):
                A[i, j] = ab[k, j, 2 * kl + i - j]
        res = np.abs(A @ x[:, r] - b[:, r]).max() / np.abs(b[:, r]).max()
        assert res < 1e-13
    g.close()


@pytest.mark.gpu
def test_tensor_core_int8_selftest():
    """One tcgen05 int8 product (128x32x64) through the library's descriptors and TMEM
    read-out equals the exact integer product."""
    g = pkg.Context(small_cfg())
    assert g.selftest(0) == 0.0
    g.close()
