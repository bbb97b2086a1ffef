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

import oracle_lib as ol

capi = importlib.import_module("leeds-code_b200.capi")
state = importlib.import_module("leeds-code_b200.state")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def case1_oracle():
    z = np.load(os.path.join(GOLDEN, "state_case1.npz"))
    cfg = capi.template_config(L=int(z["L"]), M=int(z["M"]), Mp=int(z["Mp"]), N=len(z["r"]),
                               timestep=float(z["dt"]), Ra=float(z["Ra"]), Pr=float(z["Pr"]),
                               Pm=float(z["Pm"]), E=float(z["E"]), rratio=float(z["riro"]),
                               implicit=0.5)
    o = ol.Oracle(cfg)
    l, m_, _ = state.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    idx = state.state_nh(l, m_, cfg.L, cfg.M, cfg.Mp)
    for name, f in (("uT", 0), ("uP", 1), ("C", 2), ("BT", 3), ("BP", 4)):
        d = z[name]
        o.set_coll(f, d[0, idx, :], d[1, idx, :])
    return o, z


def test_golden_t0_energies():
    """Energies of tests/state.cdf.in equal the reference's own t=0 output row (12 digits).
    The shipped .dat files predate two prefactor changes in io_write2files
    (io.F90:238-247): magnetic energy and ohmic dissipation were half of today's
    Pm/E and 2Pm/E, viscous dissipation used 1/2 instead of Pm."""
    o, z = case1_oracle()
    np.testing.assert_allclose(o.radial_grid(), z["r"], rtol=0, atol=1e-15)
    e = o.energies()
    g = json.load(open(os.path.join(GOLDEN, "golden_t0.json")))
    v, m = g["vel_energy_t0"], g["mag_energy_t0"]
    Pm = float(z["Pm"])
    checks = [
        (e["KE"], v["KE"]), (e["KE_ax"], v["KE_ax"]), (e["topflx"], v["topflx"]),
        (e["botflx"], v["botflx"]), (e["KE_dis"] * 0.5 / Pm, v["Edis"]),
        (e["ME"] / 2, m["ME"]), (e["ME_ax"] / 2, m["ME_ax"]), (e["ME_dis"] / 2, m["Mdis"]),
        (e["dipole"], m["dipole"]),
    ]
    for got, want in checks:
        assert abs(got - want) <= 1e-11 * abs(want), (got, want)
    assert abs(e["quadrupole"] - m["quadrupole"]) <= 1e-11 * abs(m["dipole"])


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
