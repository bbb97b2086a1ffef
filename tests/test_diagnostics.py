"""The other diagnostics of io_write2files (io.F90:290-340): lsd_diagnostics against the
oracle's restatement (orc_diagnostics).

CPU (oracle only):
* the spectra sum to the energies: sum over l (and over m) of the velocity spectrum is
  KE of io_write_vel_energy, of the field spectrum ME (io_save_spectrum,
  io_save_spectrum_anelastic with the density weights);
* the partitions add up: Et + Ep = KE, and the toroidal part is KE_tor;
* io_write_cmb of a pure axial dipole: theta = 0 (g10 > 0) or pi, fdip = 1, all of the
  surface energy in l = 1 and in m = 0;
* io_write_nussel of the conductive l = 0 profile (ri ro / r - ri) / (ro - ri): Nu = 1 to
  the finite-difference error of dr(1); io_save_profile returns the same column.
GPU: lsd_diagnostics against orc_diagnostics after 3 steps (Boussinesq with an l = 0
codensity profile; anelastic with composition): scalars, spectra and profiles to 1e-9
of their scale, lpol exactly; at the full lmax 127 / Nr 129 size the spectrum sums
against lsd_energies.
"""
import importlib

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def conductive(cfg):
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    ri = cfg.rratio / (1.0 - cfg.rratio)
    ro = 1.0 / (1.0 - cfg.rratio)
    return (ri * ro / r - ri) / (ro - ri)


def state_with_profiles(cfg, seed=syn.SEED, composition=False):
    st = syn.boussinesq_state(cfg, seed=seed, composition=composition)
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    k0 = int(np.flatnonzero((l == 0) & (m_ == 0))[0])
    for f in ((capi.COD_C, capi.COMP_C) if composition else (capi.COD_C,)):
        re, im = st[f]
        re = re.copy()
        re[k0, :] = conductive(cfg)
        st[f] = (re, im)
    return st


def load(obj, cfg, st, prof=None):
    if prof is not None:
        obj.set_reference_state(prof)
    for f, (re, im) in st.items():
        obj.set_coll(f, re, im)


def test_oracle_spectra_and_partitions_sum_to_energies():
    for cfg, prof, comp in ((syn.config_parity(L=16, M=16, N=13), None, False),
                            (syn.config_anelastic(L=16, N=17), "poly", True)):
        o = ol.Oracle(cfg)
        load(o, cfg, state_with_profiles(cfg, composition=comp),
             syn.polytrope_reference_state(cfg.N, cfg.rratio) if prof else None)
        sc, sp, pr = o.diagnostics()
        e = o.energies()
        for f, E in (("vel", e["KE"]), ("mag", e["ME"])):
            assert abs(sp[f + "_l"][:, 0].sum() - E) <= 1e-12 * E, f
            assert abs(sp[f + "_m"][:, 0].sum() - E) <= 1e-12 * E, f
        for f in ("vel", "mag"):
            np.testing.assert_allclose(sp[f + "_l"][:, 1] + sp[f + "_l"][:, 2], sp[f + "_l"][:, 0], rtol=1e-13)
        assert abs(sc["vel_Et"] + sc["vel_Ep"] - e["KE"]) <= 1e-12 * e["KE"]
        assert abs(sc["vel_Et"] - e["KE_tor"]) <= 1e-12 * e["KE_tor"]
        assert abs(sc["mag_Et"] + sc["mag_Ep"] - e["ME"]) <= 1e-12 * e["ME"]
        assert sc["vel_lpol"] == 1 + int(np.argmax(sp["vel_l"][:, 1]))
        # the Rm / Elsasser relations of io_write_dyn_outputs
        ri, ro = cfg.rratio / (1 - cfg.rratio), 1 / (1 - cfg.rratio)
        vol = 4.0 / 3.0 * np.pi * (ro ** 3 - ri ** 3)
        assert abs(sc["Rm"] - np.sqrt(2 * e["KE"] / vol)) <= 1e-14 * sc["Rm"]
        assert abs(sc["M_ratio"] - e["ME"] / e["KE"]) <= 1e-14 * sc["M_ratio"]
        assert sc["time"] == e["time"]
        assert pr["r"][0] < pr["r"][-1]
        o.close()


def test_oracle_cmb_axial_dipole():
    cfg = syn.config_parity(L=16, M=16, N=13)
    o = ol.Oracle(cfg)
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    H = len(l)
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    for sign, theta in ((1.0, 0.0), (-1.0, np.pi)):
        re = np.zeros((H, cfg.N))
        re[int(np.flatnonzero((l == 1) & (m_ == 0))[0]), :] = sign * r ** 2
        o.set_coll(capi.MAG_POL, re, np.zeros((H, cfg.N)))
        sc, sp, _ = o.diagnostics()
        assert sc["cmb_theta"] == theta
        assert abs(sc["fdip"] - 1.0) <= 1e-15
        assert sc["cmb_El1"] == sc["cmb_EPol"] == sc["cmb_El12"] == sc["cmb_Epas"]
        assert sp["mag_l"][1, 0] == sp["mag_l"][:, 0].sum()
    o.close()


def test_oracle_nusselt_conductive():
    cfg = syn.config_parity(L=16, M=16, N=33)
    o = ol.Oracle(cfg)
    st = state_with_profiles(cfg)
    o.set_coll(capi.COD_C, *st[capi.COD_C])
    sc, _, pr = o.diagnostics()
    assert abs(sc["nus_Nu"] - 1.0) < 1e-4, sc["nus_Nu"]
    assert abs(sc["nus_Nu_bot"] - 1.0) < 1e-4, sc["nus_Nu_bot"]
    assert sc["nus_T_ri"] == 1.0 and sc["nus_T_ro"] == 0.0
    np.testing.assert_array_equal(pr["temp_C"], conductive(cfg))
    o.close()


def compare(dg, do, label):
    sg, spg, pg = dg
    so, spo, po = do
    for k, b in so.items():
        a = sg[k]
        tol = 1e-3 if k == "tim_corr_dt" else 1e-9
        if k == "vel_lpol":
            assert a == b, (label, k, a, b)
        else:
            assert abs(a - b) <= tol * abs(b) + 1e-14, (label, k, a, b)
    for k, b in spo.items():
        np.testing.assert_allclose(spg[k], b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-300), err_msg=label + k)
    for k, b in po.items():
        np.testing.assert_allclose(pg[k], b, rtol=0, atol=1e-9 * max(np.abs(b).max(), 1e-300), err_msg=label + k)


@pytest.mark.gpu
def test_gpu_diagnostics_boussinesq():
    cfg = syn.config_parity(L=32, M=32, N=17)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    st = state_with_profiles(cfg, seed=23)
    load(g, cfg, st)
    load(o, cfg, st)
    compare(g.diagnostics(), o.diagnostics(), "t0 ")
    g.step(3)
    o.step(3)
    dg, do = g.diagnostics(), o.diagnostics()
    compare(dg, do, "t3 ")
    assert abs(dg[0]["nus_Nu"] - 1.0) < 0.05
    g.close()
    o.close()


@pytest.mark.gpu
def test_gpu_diagnostics_anelastic_composition():
    cfg = syn.config_anelastic(L=16, N=17)
    prof = syn.polytrope_reference_state(cfg.N, cfg.rratio)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    st = state_with_profiles(cfg, seed=29, composition=True)
    load(g, cfg, st, prof)
    load(o, cfg, st, prof)
    g.step(3)
    o.step(3)
    compare(g.diagnostics(), o.diagnostics(), "anelastic ")
    g.close()
    o.close()


@pytest.mark.gpu
def test_gpu_diagnostics_full_size():
    """lmax 127, Nr 129: the spectrum sums against lsd_energies (no oracle at this size)."""
    cfg = syn.config_dynamo128()
    g = pkg.Context(cfg)
    load(g, cfg, state_with_profiles(cfg))
    g.step(2)
    sc, sp, pr = g.diagnostics()
    e = g.energies()
    for f, E in (("vel", e["KE"]), ("mag", e["ME"])):
        assert abs(sp[f + "_l"][:, 0].sum() - E) <= 1e-12 * E, f
        assert abs(sp[f + "_m"][:, 0].sum() - E) <= 1e-12 * E, f
    assert abs(sc["vel_Et"] + sc["vel_Ep"] - e["KE"]) <= 1e-12 * e["KE"]
    w = g.radial_weights()
    assert abs(np.dot(pr["vel_E"], w) - e["KE"]) <= 1e-12 * e["KE"]
    assert 1 <= sc["vel_lpol"] <= cfg.L
    assert all(np.isfinite(v) for v in sc.values())
    g.close()
