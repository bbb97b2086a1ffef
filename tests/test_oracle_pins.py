"""Pins of the CPU oracle against the reference's own outputs and against independent
implementations of the third-party algorithms the reference calls (LAPACK via scipy,
FFTW's DFT via numpy, Gauss-Legendre and associated Legendre functions via numpy/scipy)."""
import importlib
import json
import math
import os

import numpy as np
import pytest
import scipy.linalg.lapack as lapack
import scipy.special as sps

import case1_fixture as case1
import oracle_lib as ol

capi = importlib.import_module("leeds-code_b200.capi")
state = importlib.import_module("leeds-code_b200.state")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def case1_oracle(**over):
    cfg = case1.config(**over)
    o = ol.Oracle(cfg)
    fields, r = case1.load(cfg)
    for f, (re, im) in fields.items():
        o.set_coll(f, re, im)
    return o, cfg, r


def test_golden_t0_energies():
    """Energies of the reference's tests/state.cdf.in, read by state.load_state, equal the
    reference's own t=0 output row (12 digits).  The field is loaded in the current
    normalisation (B / sqrt 2, tests/case1_fixture.py); the shipped .dat files predate
    that and the viscous-dissipation prefactor change in io_write2files (io.F90:238-247)."""
    o, cfg, r = case1_oracle()
    np.testing.assert_allclose(o.radial_grid(), r, rtol=0, atol=1e-15)
    e = case1.dat_columns(o.energies(), cfg.Pm)
    want = case1.golden_rows()[0]
    for k in ("KE", "KE_ax", "topflx", "botflx", "Edis", "ME", "ME_ax", "Mdis", "dipole"):
        assert abs(e[k] - want[k]) <= 1e-11 * abs(want[k]), (k, e[k], want[k])
    assert abs(e["quadrupole"] - want["quadrupole"]) <= 1e-11 * abs(want["dipole"])


def test_golden_first_step():
    """One timestep of the oracle from the reference's state (dt = 4.59265755232e-6, the
    reference's first step; one predictor and one corrector, implicit 0.5) against the
    reference's second output row: every energy increment within the band measured for
    the restated equations (tests/case1_fixture.py, main.F90:100-164)."""
    r0, r1 = case1.golden_rows()
    o, cfg, _ = case1_oracle(timestep=r1["time"], time_step_control=1)
    before = case1.dat_columns(o.energies(), cfg.Pm)
    st = o.step(1)
    assert st.steps_done == 1 and st.correctors == 1 and abs(st.t - r1["time"]) < 1e-20
    after = case1.dat_columns(o.energies(), cfg.Pm)
    case1.check_first_step(before, after)


@pytest.mark.parametrize("L,M,Mp", [(48, 12, 4), (80, 20, 4), (64, 32, 2)])
def test_load_state_truncation(L, M, Mp):
    """io_load_state re-truncation (io.F90:1299-1354): a run with other L, M, Mp takes the
    file's (l, m) where both have it; modes the file lacks start at zero (the reference
    fills them with unseeded noise of amplitude d_init_pert)."""
    from scipy.io import netcdf_file
    f = netcdf_file(case1.state_file(), "r", mmap=False)
    raw = np.array(f.variables["uP"].data, dtype=np.float64)
    f.close()
    fields, _, _, _ = state.load_state(case1.state_file(), L, M, Mp, 64)
    re, im = fields[capi.VEL_POL]
    l, m_, _ = state.folded_harmonics(L, M, Mp)
    idx = state.state_nh(l, m_, 64, 16, 4)
    assert re.shape == (len(l), 64)
    for nh in range(len(l)):
        if idx[nh] >= 0:
            assert np.array_equal(re[nh], raw[0, idx[nh]]) and np.array_equal(im[nh], raw[1, idx[nh]])
        else:
            assert not re[nh].any() and not im[nh].any()
    if L <= 64 and M * Mp <= 64 and Mp % 4 == 0:
        assert (idx >= 0).all() and len(l) < raw.shape[1]  # truncated: every run mode from the file
    else:
        assert (idx >= 0).any() and (idx < 0).any()  # padded: some modes start at zero


def test_layout_folded_order():
    """Harmonic tables equal _loop_setlm (parallel.h_template:54-80); the file order map
    is a bijection onto io_state_nh (io.F90:1258-1272)."""
    for (L, M, Mp) in [(32, 32, 1), (64, 16, 4), (128, 128, 1), (48, 12, 2)]:
        cfg = capi.template_config(L=L, M=M, Mp=Mp, N=9, timestep=1e-5)
        o = ol.Oracle(cfg)
        l, m, s = o.harmonics()
        l2, m2, s2 = state.folded_harmonics(L, M, Mp)
        assert (l == l2).all() and (m == m2).all() and (s == s2).all()
        idx = state.state_nh(l, m, L, M, Mp)
        assert sorted(idx.tolist()) == list(range(len(l)))
        thm = o.theta_map()
        assert sorted(thm.tolist()) == list(range(M))
        # first appearance order: 0, M-1, 1, M-2, ...
        exp = [v for j in range(M // 2) for v in (j, M - 1 - j)]
        assert thm.tolist() == exp


def test_dgbtrf_dgbtrs_vs_lapack():
    """Banded LU restatement equals LAPACK dgbtrf/dgbtrs (scipy's build)."""
    rng = np.random.default_rng(7)
    for n, kl in [(33, 3), (129, 3), (257, 4), (20, 2)]:
        ab = np.zeros((3 * kl + 1, n))
        ab[kl:, :] = rng.standard_normal((2 * kl + 1, n))
        ab[2 * kl, :] += 0.3  # mild diagonal, pivoting still happens
        lu_o, ip_o, info_o = ol.dgbtrf(ab, kl)
        lu_l, ip_l, info_l = lapack.dgbtrf(ab.copy(), kl, kl)
        assert info_o == info_l == 0
        assert (ip_o == ip_l + 1).all()
        np.testing.assert_allclose(lu_o, lu_l, rtol=1e-13, atol=1e-13 * np.abs(lu_l).max())
        b = rng.standard_normal(n)
        x_o = ol.dgbtrs(lu_o, kl, ip_o, b)
        x_l, info = lapack.dgbtrs(lu_l, kl, kl, b, ip_l)
        np.testing.assert_allclose(x_o, x_l, rtol=1e-12, atol=1e-13 * np.abs(x_l).max())


def test_mat_invert_vs_numpy():
    rng = np.random.default_rng(3)
    for n in (2, 5, 7):
        a = rng.standard_normal((n, n)) + n * np.eye(n)
        x, info = ol.mat_invert(a)
        assert info == 0
        np.testing.assert_allclose(x, np.linalg.inv(a), rtol=1e-12, atol=1e-13)


@pytest.mark.parametrize("n", [48, 96, 192, 384, 768])
def test_fft_vs_numpy(n):
    """FFTW contract: c2r unnormalised, DC/Nyquist imaginary parts ignored; r2c exact
    zero imaginary DC."""
    rng = np.random.default_rng(n)
    M = n // 3
    y = rng.standard_normal(n // 2 + 1) + 1j * rng.standard_normal(n // 2 + 1)
    y[M:] = 0
    x = ol.fft_c2r(n, y)
    yy = y.copy()
    yy[0] = yy[0].real
    np.testing.assert_allclose(x, np.fft.irfft(yy, n) * n, rtol=0, atol=1e-13 * np.abs(x).max())
    xr = rng.standard_normal(n)
    Y = ol.fft_r2c(xr)
    assert Y[0].imag == 0.0
    np.testing.assert_allclose(Y, np.fft.rfft(xr), rtol=0, atol=1e-13 * np.abs(Y).max())


def test_gauss_legendre_vs_numpy():
    for L in (32, 64, 128, 256):
        cfg = capi.template_config(L=L, M=2, Mp=1, N=9, timestep=1e-5)
        o = ol.Oracle(cfg)
        gp, gw = o.gauss()
        x, w = np.polynomial.legendre.leggauss(3 * L // 2)
        # the reference stops Newton at |dz| <= 1e-13 (gauwts.f:22,66), so weights agree
        # with a fully converged quadrature to a few 1e-12 only
        np.testing.assert_allclose(gp, x, rtol=0, atol=2e-15)
        np.testing.assert_allclose(gw, w, rtol=1e-9, atol=5e-13)
        assert abs(gw.sum() - 2.0) < 1e-12


def test_schmidt_legendre_vs_scipy():
    """P tables are Schmidt semi-normalised without the Condon-Shortley phase
    (legendre.F90:29-31)."""
    L, M = 32, 32
    cfg = capi.template_config(L=L, M=M, Mp=1, N=9, timestep=1e-5)
    o = ol.Oracle(cfg)
    gp, gw = o.gauss()
    l, m, s = o.harmonics()
    P = o.legendre_table(capi.LEG_P)
    x = gp[: o.Th2]
    for nh in range(o.H):
        ll, mm = int(l[nh]), int(m[nh])
        ref = sps.lpmv(mm, ll, x) * (-1) ** mm
        if mm > 0:
            ref = ref * math.sqrt(2.0 * math.factorial(ll - mm) / math.factorial(ll + mm))
        np.testing.assert_allclose(P[:, nh], ref, rtol=1e-11, atol=1e-13)
    # normalisation: int P^2 sin dth = 2(2-d_m0)/(2l+1) using the full Gauss grid
    for nh in range(0, o.H, 7):
        ll, mm = int(l[nh]), int(m[nh])
        half = P[:, nh]
        full = np.concatenate([half, half[::-1] * (-1) ** (ll + mm)])
        integ = np.sum(full ** 2 * gw)
        np.testing.assert_allclose(integ, 2 * (2 - (mm == 0)) / (2 * ll + 1), rtol=1e-12)


def test_sht_round_trip_exact():
    """Band-limited spec -> phys -> spec is the identity (Gauss quadrature exact)."""
    cfg = capi.template_config(L=32, M=32, Mp=1, N=9, timestep=1e-5)
    o = ol.Oracle(cfg)
    l, m, s = o.harmonics()
    rng = np.random.default_rng(1)
    sre = rng.standard_normal((o.N, o.H))
    sim = rng.standard_normal((o.N, o.H))
    sim[:, m == 0] = 0
    p = o.spec2phys(sre, sim)
    b_re, b_im = o.phys2spec(p)
    # exact up to the reference's Gauss-weight convergence (|dz| <= 1e-13)
    np.testing.assert_allclose(b_re, sre, rtol=0, atol=1e-11)
    np.testing.assert_allclose(b_im, sim, rtol=0, atol=1e-11)
    # vector round trip: qst -> rtp -> qst for l >= 1 coefficients
    q = (rng.standard_normal((o.N, o.H)), rng.standard_normal((o.N, o.H)))
    sv = (rng.standard_normal((o.N, o.H)), rng.standard_normal((o.N, o.H)))
    tv = (rng.standard_normal((o.N, o.H)), rng.standard_normal((o.N, o.H)))
    for a in (q, sv, tv):
        a[1][:, m == 0] = 0
    for a in (sv, tv):
        a[0][:, l == 0] = 0
        a[1][:, l == 0] = 0
    r, th, ph = o.qst2rtp(q, sv, tv)
    q2, s2, t2 = o.rtp2qst(r, th, ph)
    for a, b in ((q, q2), (sv, s2), (tv, t2)):
        np.testing.assert_allclose(b[0], a[0], rtol=0, atol=1e-10)
        np.testing.assert_allclose(b[1], a[1], rtol=0, atol=1e-10)


def test_operator_solve_residual_small():
    """The oracle's operator solves (tim_zerobc + tim_invX; the poloidal velocity's
    composite) at L = M = 16, N = 33, KL = 4: the second-order families' residuals from
    their LAPACK factors (as the device test forms them), and the composite's x = 0,
    dx/dr = 0 at both walls (vel_gre_adjust)."""
    from test_gpu_configs import lu_apply, LU_INDEX
    cfg = capi.template_config(L=16, M=16, Mp=1, N=33, KL=4, timestep=2e-6, E=3e-4, Pm=3.0, Ra=200.0)
    o = ol.Oracle(cfg)
    l, m, _ = o.harmonics()
    rng = np.random.default_rng(4)
    N, H = o.N, o.H
    for f, idx in LU_INDEX.items():
        re, im = rng.standard_normal((H, N)), rng.standard_normal((H, N))
        xr, xi = o.operator_solve(f, re, im)
        for deg in range(0 if f == capi.COD_C else 1, 16):
            cols = np.nonzero(l == deg)[0]
            ab, ipiv = o.operator_lu(idx, deg)
            b = re[cols].T.copy()
            b[0], b[-1] = 0.0, 0.0
            res = lu_apply(ab, ipiv, 4, xr[cols].T) - b
            assert np.abs(res).max() <= 1e-13 * np.abs(b).max(), (f, deg)
    re, im = rng.standard_normal((H, N)), rng.standard_normal((H, N))
    xr, xi = o.operator_solve(capi.VEL_POL, re, im)
    band = o.dr(1)  # first radial derivative, Fortran band: D(i, j) at [KL + i - j, j]
    kl = 4
    D = np.zeros((N, N))
    for j in range(N):
        for i in range(max(0, j - kl), min(N, j + kl + 1)):
            D[i, j] = band[kl + i - j, j]
    ok = l > 0
    for x in (xr, xi):
        assert np.abs(x[ok][:, [0, -1]]).max() <= 1e-13 * np.abs(x).max()
        dx = x[ok] @ D.T
        assert np.abs(dx[:, [0, -1]]).max() <= 1e-10 * np.abs(dx).max()
    o.close()
