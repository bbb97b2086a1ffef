"""The conducting, rotating inner core in the oracle (Nic > 1; magnetic.F90:62-461,
timestep.F90:218-344, 594-634; rotation.F90; nonlinear.F90:451-538).

* Free decay of a whole conducting sphere: with no flow (Ra = 0, a field of 1e-7 so that
  the Lorentz force is ~1e-14) the l = 1 poloidal mode j_1(k r) with j_0(k r_o) = 0 and the
  toroidal mode j_1(k r) with j_1(k r_o) = 0 decay as exp(-k^2 t) through inner and outer
  core alike: the coupled operator, the regularity row at the innermost point and the
  continuity rows at r_i.  The energy decay rates match 2 k^2 (poloidal to 1e-6, toroidal
  to 1e-3); with an insulating inner core (Nic = 1) the same start decays at rates more
  than 5e-3 (poloidal) and 1e-1 (toroidal) away.
* The field at r_i is one unknown of the coupled solve: the inner core's outer value
  equals the outer core's inner value after every step.
* Rigid rotation of the fluid (vel_Tor(l=1, m=0) = Omega r) carries no viscous stress:
  the viscous torque vanishes to rounding (non_rotation); a rotating inner core under a
  fluid at rest is braked (torque of the opposite sign) and its rate changes by
  dt / I * torque over a predictor.
"""
import importlib

import numpy as np
from scipy.special import spherical_jn
from scipy.optimize import brentq

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def zero_state(o, cfg):
    H = o.H
    for f in range(5):
        o.set_coll(f, np.zeros((H, cfg.N)), np.zeros((H, cfg.N)))
    if cfg.Nic > 1:
        for f in (capi.MAG_IC_TOR, capi.MAG_IC_POL):
            o.set_coll(f, np.zeros((H, cfg.Nic)), np.zeros((H, cfg.Nic)))


def decay_rates(Nic, steps=300, dt=2e-4):
    cfg = syn.config_inner_core(L=8, N=25, Nic=Nic, KL=4, E=0.1, Ra=0.0, rot_tstep=0, timestep=dt)
    o = ol.Oracle(cfg)
    zero_state(o, cfg)
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    k10 = int(np.flatnonzero((l == 1) & (m_ == 0))[0])
    ro = 1.0 / (1.0 - cfg.rratio)
    kp = np.pi / ro                                               # j_0(k ro) = 0
    kt = brentq(lambda x: spherical_jn(1, x), 4.0, 4.7) / ro      # j_1(k ro) = 0
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    amp = 1e-7
    for f, k in ((capi.MAG_POL, kp), (capi.MAG_TOR, kt)):
        re = np.zeros((o.H, cfg.N))
        re[k10] = amp * spherical_jn(1, k * r)
        o.set_coll(f, re, np.zeros_like(re))
    if Nic > 1:
        ric = syn.inner_core_grid(Nic, cfg.rratio)
        for f, k in ((capi.MAG_IC_POL, kp), (capi.MAG_IC_TOR, kt)):
            re = np.zeros((o.H, Nic))
            re[k10] = amp * spherical_jn(1, k * ric)
            o.set_coll(f, re, np.zeros_like(re))
    o.step(steps // 2)
    e1 = o.energies()
    o.step(steps // 2)
    e2 = o.energies()
    T = dt * (steps // 2)
    pol = lambda e: e["ME"] - e["ME_tor"]
    rp = np.log(pol(e1) / pol(e2)) / T
    rt = np.log(e1["ME_tor"] / e2["ME_tor"]) / T
    o.close()
    return rp, rt, 2 * kp * kp, 2 * kt * kt


def test_free_decay_whole_sphere():
    rp, rt, ep, et = decay_rates(Nic=13)
    assert abs(rp / ep - 1) < 1e-6, (rp, ep)
    # the toroidal condition BTor = 0 sits at the innermost point r_1 = r_i sin(pi / (4 Nic - 2))
    # > 0, not at the centre: a hole of k r_1 ~ 0.1 that shifts this eigenvalue by ~2e-4
    assert abs(rt / et - 1) < 1e-3, (rt, et)
    rp1, rt1, _, _ = decay_rates(Nic=1)
    assert abs(rp1 / ep - 1) > 5e-3 and abs(rt1 / et - 1) > 1e-1, (rp1, rt1)


def test_field_continuous_across_inner_boundary():
    cfg = syn.config_inner_core(L=12, N=17, Nic=9, KL=3, timestep=2e-5)
    o = ol.Oracle(cfg)
    st = syn.boussinesq_state(cfg, seed=5)
    for f, (re, im) in st.items():
        o.set_coll(f, re, im)
    o.set_rotation(2.0)
    o.step(3)
    for f, fi in ((capi.MAG_TOR, capi.MAG_IC_TOR), (capi.MAG_POL, capi.MAG_IC_POL)):
        a, b = o.get_coll(f), o.get_coll(fi)
        assert np.abs(a[0]).max() > 0
        assert np.array_equal(a[0][:, 0], b[0][:, -1]) and np.array_equal(a[1][:, 0], b[1][:, -1])
    o.close()


def test_viscous_torque_rigid_rotation_and_braking():
    cfg = syn.config_inner_core(L=12, N=17, Nic=9, KL=3, Ra=0.0, timestep=1e-5)
    o = ol.Oracle(cfg)
    zero_state(o, cfg)
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    k10 = int(np.flatnonzero((l == 1) & (m_ == 0))[0])
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    re = np.zeros((o.H, cfg.N))
    re[k10] = 3.0 * r
    o.set_coll(capi.VEL_TOR, re, np.zeros_like(re))
    o.nonlinear()
    rigid = o.rotation()
    # fluid at rest, inner core rotating: the viscous torque brakes it
    zero_state(o, cfg)
    re[k10] = 0.0
    re[k10, 0] = 3.0 * r[0]   # the no-slip value at r_i, zero elsewhere
    o.set_coll(capi.VEL_TOR, re, np.zeros_like(re))
    o.set_rotation(3.0)
    o.nonlinear()
    w0, tv, tm = o.rotation()
    o.predictor()
    w1 = o.rotation()[0]
    ri = r[0]
    inertia = 8 * np.pi / 15 * ri ** 5
    o.close()
    assert abs(rigid[1]) < 1e-9 * abs(tv), (rigid, tv)
    assert tv < 0 and tm == 0.0
    assert abs(w1 - (w0 + cfg.timestep / inertia * tv)) <= 1e-12 * abs(w1)


def test_state_file_round_trip_inner_core(tmp_path):
    """save_state / load_state / load_rotation with the inner core's field (icBT, icBP on
    the r dimension, Nic entries written) and icOmega."""
    cfg = syn.config_inner_core(L=12, N=17, Nic=9)
    st = syn.boussinesq_state(cfg, seed=3)
    rng = np.random.default_rng(4)
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    for f in (capi.MAG_IC_TOR, capi.MAG_IC_POL):
        re = rng.standard_normal((len(l), cfg.Nic))
        im = rng.standard_normal((len(l), cfg.Nic))
        im[m_ == 0] = 0.0
        st[f] = (re, im)
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    ric = syn.inner_core_grid(cfg.Nic, cfg.rratio)
    p = str(tmp_path / "state.cdf")
    pkg.state.save_state(p, st, cfg.L, cfg.M, cfg.Mp, r, ric, 0.25, 1e-5, {}, omega=-13.3)
    out, t, dt, r2 = pkg.state.load_state(p, cfg.L, cfg.M, cfg.Mp, cfg.N, r_expected=r, Nic=cfg.Nic)
    assert t == 0.25 and dt == 1e-5 and pkg.state.load_rotation(p) == -13.3
    for f, (re, im) in st.items():
        assert np.array_equal(out[f][0], re) and np.array_equal(out[f][1], im), f


def test_state_file_radial_interpolation(tmp_path):
    """load_state onto a run with other N and Nic (io_interp_wts / io_interp): smooth radial
    profiles come back to 1e-6 at the points of the [0, 1] mapping, a file on the run's own
    grid exactly."""
    cfg = syn.config_inner_core(L=8, N=33, Nic=17)
    l, m_, _ = syn.folded_harmonics(cfg.L, cfg.M, cfg.Mp)
    r = syn.chebyshev_grid(cfg.N, cfg.rratio, cfg.alpha)
    ric = syn.inner_core_grid(cfg.Nic, cfg.rratio)
    amp = np.arange(1, len(l) + 1, dtype=np.float64)[:, None]
    f_oc = lambda x: np.sin(2.0 * x) * np.exp(-x)
    f_ic = lambda x: x ** 2 * np.cos(x)
    st = {capi.VEL_TOR: (amp * f_oc(r)[None, :], -amp * f_oc(r)[None, :]),
          capi.MAG_IC_TOR: (amp * f_ic(ric)[None, :], amp * f_ic(ric)[None, :])}
    p = str(tmp_path / "state.cdf")
    pkg.state.save_state(p, st, cfg.L, cfg.M, cfg.Mp, r, ric, 0.0, 1e-5, {})
    r2 = syn.chebyshev_grid(25, cfg.rratio, cfg.alpha)
    ric2 = syn.inner_core_grid(11, cfg.rratio)
    out, _, _, _ = pkg.state.load_state(p, cfg.L, cfg.M, cfg.Mp, 25, r_expected=r2, Nic=11, ric_expected=ric2)
    err_oc = np.abs(out[capi.VEL_TOR][0] - amp * f_oc(r2)[None, :]).max() / amp.max()
    # both grids are mapped onto [0, 1] (io.F90:1377-1378): the inner core's first point
    # depends on Nic, so the run's point t lands on the file's radius ric[0] + t (ric[-1] - ric[0])
    t = (ric2 - ric2[0]) / (ric2[-1] - ric2[0])
    err_ic = np.abs(out[capi.MAG_IC_TOR][0] - amp * f_ic(ric[0] + t * (ric[-1] - ric[0]))[None, :]).max() / amp.max()
    assert err_oc < 1e-6 and err_ic < 1e-6, (err_oc, err_ic)
    same, _, _, _ = pkg.state.load_state(p, cfg.L, cfg.M, cfg.Mp, cfg.N, r_expected=r, Nic=cfg.Nic,
                                         ric_expected=ric)
    assert np.array_equal(same[capi.VEL_TOR][0], st[capi.VEL_TOR][0])
