"""The conducting, rotating inner core on the device against the oracle (Christensen case 2
parameters: E = 1e-3, Ra = 7.15e4, Pm = 5, Nic > 1, b_rot_tstep).

The starting state: the seeded l^-2 state with its field continued into the inner core by
io_ic_extend (a r^3 + b r^2) and rot_omega = 1.5.
* L = M = 16, N = 17, Nic = 9, fixed dt 1e-5, FP64, 10 steps: the corrector counts equal
  the oracle's; every coefficient of the outer and inner core to 1e-10 of its field's scale;
  rot_omega, the viscous and the magnetic torque to 1e-9; the diagnostics (with the inner
  core's mag_ic.dat record and rot_torque.dat) to 1e-9.
* The same with the CFL / corrector-controlled dt (d_timestep = -5e-5), 20 steps: the dt
  sequence (1e-9) and rot_omega.
* The case 2 resolution of the reference's INFO file (L = 64, M = 16, Mp = 4, N = 64,
  Nic = 16), tensor-core Legendre transforms, 3 steps against the FP64 oracle: fields and
  rotation to 1e-9.
* Free decay of the whole conducting sphere on the device (Ra = 0, field 1e-7): the decay
  rates of the l = 1 poloidal and toroidal modes equal the oracle's to 1e-9 and 2 k^2
  (poloidal) to 1e-6.
"""
import importlib

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def relerr(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300))


def start(cfg, o, seed=31, omega=1.5):
    """the state of both sides: seeded outer core, io_ic_extend for the inner core"""
    st = syn.boussinesq_state(cfg, seed=seed)
    band = o.dr(1)
    KL = cfg.KL
    first = [band[KL + 1 - j, j - 1] for j in range(1, KL + 2)]  # dr(1) at point 1
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    ric = syn.inner_core_grid(cfg.Nic, cfg.rratio)
    st[capi.MAG_IC_TOR] = syn.ic_extend(*st[capi.MAG_TOR], r, first, ric)
    st[capi.MAG_IC_POL] = syn.ic_extend(*st[capi.MAG_POL], r, first, ric)
    return st, omega


def load(objs, st, omega):
    for x in objs:
        for f, (re, im) in st.items():
            x.set_coll(f, re, im)
        x.set_rotation(omega)


def compare_all(g, o, tol, label):
    for f in (capi.VEL_TOR, capi.VEL_POL, capi.COD_C, capi.MAG_TOR, capi.MAG_POL, capi.MAG_IC_TOR, capi.MAG_IC_POL):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < tol, (label, f, relerr(a[0], b[0]))
        assert relerr(a[1], b[1]) < tol, (label, f, relerr(a[1], b[1]))
    ra, rb = g.rotation(), o.rotation()
    for k in range(3):
        assert abs(ra[k] - rb[k]) <= tol * 10 * abs(rb[k]) + 1e-300, (label, k, ra, rb)


@pytest.mark.gpu
def test_inner_core_fixed_dt():
    cfg = syn.config_inner_core(L=16, N=17, Nic=9)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    st, om = start(cfg, o)
    load((g, o), st, om)
    sg, so = g.step(10), o.step(10)
    assert sg.correctors == so.correctors
    compare_all(g, o, 1e-10, "fixed dt")
    rot = g.rotation()
    assert rot[0] != om and rot[1] != 0.0 and rot[2] != 0.0
    from test_diagnostics import compare
    compare(g.diagnostics(), o.diagnostics(), "inner core ")
    d = g.diagnostics()[0]
    assert d["ic_E"] > 0 and d["rot_omega"] == rot[0]
    g.close()
    o.close()


@pytest.mark.gpu
def test_inner_core_variable_dt():
    cfg = syn.config_inner_core(L=16, N=17, Nic=9, timestep=-5e-5)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    st, om = start(cfg, o, seed=37, omega=-2.0)
    load((g, o), st, om)
    g.set_time(0.0, 5e-5)
    o.set_time(0.0, 5e-5)
    for k in range(20):
        sg, so = g.step(1), o.step(1)
        assert sg.correctors == so.correctors, k
        a, b = g.dt_control(), o.dt_control()
        assert abs(a[0] - b[0]) <= 1e-9 * b[0], (k, a, b)
    compare_all(g, o, 1e-9, "variable dt")
    g.close()
    o.close()


@pytest.mark.gpu
def test_inner_core_case2_resolution_tensor_cores():
    cfg = syn.config_inner_core(L=64, M=16, Mp=4, N=64, Nic=16, KL=4, precision=capi.PREC_OZAKI, timestep=2e-5)
    ocfg = syn.config_inner_core(L=64, M=16, Mp=4, N=64, Nic=16, KL=4, timestep=2e-5)
    g, o = pkg.Context(cfg), ol.Oracle(ocfg)
    st, om = start(cfg, o, seed=41, omega=-13.3)
    load((g, o), st, om)
    sg, so = g.step(3), o.step(3)
    assert sg.correctors == so.correctors
    compare_all(g, o, 1e-9, "case 2 resolution")
    g.close()
    o.close()


def decay(obj, cfg, steps, dt):
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    H = len(l)
    for f in range(5):
        obj.set_coll(f, np.zeros((H, cfg.N)), np.zeros((H, cfg.N)))
    k10 = int(np.flatnonzero((l == 1) & (m_ == 0))[0])
    from scipy.special import spherical_jn
    from scipy.optimize import brentq
    ro = 1.0 / (1.0 - cfg.rratio)
    kp = np.pi / ro
    kt = brentq(lambda x: spherical_jn(1, x), 4.0, 4.7) / ro
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    ric = syn.inner_core_grid(cfg.Nic, cfg.rratio)
    for f, fi, k in ((capi.MAG_POL, capi.MAG_IC_POL, kp), (capi.MAG_TOR, capi.MAG_IC_TOR, kt)):
        for ff, rr in ((f, r), (fi, ric)):
            re = np.zeros((H, len(rr)))
            re[k10] = 1e-7 * spherical_jn(1, k * rr)
            obj.set_coll(ff, re, np.zeros_like(re))
    obj.step(steps // 2)
    e1 = obj.energies()
    obj.step(steps // 2)
    e2 = obj.energies()
    T = dt * (steps // 2)
    pol = lambda e: e["ME"] - e["ME_tor"]
    return np.log(pol(e1) / pol(e2)) / T, np.log(e1["ME_tor"] / e2["ME_tor"]) / T, 2 * kp * kp


@pytest.mark.gpu
def test_inner_core_free_decay():
    cfg = syn.config_inner_core(L=8, N=25, Nic=13, KL=4, E=0.1, Ra=0.0, rot_tstep=0, timestep=2e-4)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    rg, tg, ep = decay(g, cfg, 300, 2e-4)
    ro_, to, _ = decay(o, cfg, 300, 2e-4)
    assert abs(rg - ro_) <= 1e-9 * ro_ and abs(tg - to) <= 1e-9 * to, (rg, ro_, tg, to)
    assert abs(rg / ep - 1) < 1e-6, (rg, ep)
    g.close()
    o.close()
