"""The anelastic equations (b_boussinesq = .false.) and the stress-free angular-momentum
correction, on the device against the oracle.

Oracle pins (CPU):
  * the n = 2 polytrope generated here equals the reference's own anelastic-benchmark
    planet_model.txt.in (tests/golden, 128 shells) to the file's printed digits;
  * tra_qst2rtp_vel's qv1, qv2 (Legendre sums with the qva, qvb tables) equal
    (cot u_th + d_phi u_ph / sin) / r and (d_phi u_th / sin - cot u_ph) / r formed from
    its own u_th, u_ph with an FFT phi-derivative, to 1e-12 (this identity is how the
    device forms them);
  * with the neutral reference state rho = T = eta = 1, xi = dxi/dr = deta/dr = 0 the
    anelastic operators (tim_lumesh_vel_X, tim_lumesh_Gre_X, tim_iclumesh_*_X) factorise
    to the Boussinesq ones bit for bit.
Parity (GPU, relative to the largest magnitude of the compared array):
  unit transforms 1e-12; one evaluation, predictor and corrector 1e-11 (FP64), 5e-11
  (tensor cores, S = 7); 100 steps: energies 1e-9, coefficients 1e-10.
"""
import importlib
import os

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def anel_cfg(**kw):
    base = dict(L=16, N=17)
    base.update(kw)
    return syn.config_anelastic(**base)


def test_polytrope_matches_reference_planet_model():
    ref = np.loadtxt(os.path.join(GOLDEN, "planet_model_anelastic_benchmark.txt"))
    assert ref.shape == (128, 7)
    prof = syn.polytrope_reference_state(128)
    assert np.array_equal(prof.T, ref)


def test_oracle_qv_identity():
    cfg = anel_cfg(L=24, M=24, N=9)
    o = ol.Oracle(cfg)
    l, m, _ = o.harmonics()
    rng = np.random.default_rng(3)

    def spec():
        re = rng.standard_normal((o.N, o.H))
        im = rng.standard_normal((o.N, o.H))
        im[:, m == 0] = 0.0
        return re, im

    r, th, ph, dur, qv1, dutr, dupr, qv2 = o.qst2rtp_vel(*(spec() for _ in range(6)))
    gp, _ = o.gauss()
    sn = np.sqrt((1.0 + gp) * (1.0 - gp))
    cot, s1 = gp / sn, 1.0 / sn
    rr = o.radial_grid()[:, None, None]

    def dphi(f):  # Mp = 1: bin b <-> m = b
        F = np.fft.rfft(f, axis=1)
        F = F * (1j * np.arange(F.shape[1]))[None, :, None]
        return np.fft.irfft(F, n=f.shape[1], axis=1)

    q1 = (cot * th + s1 * dphi(ph)) / rr
    q2 = (s1 * dphi(th) - cot * ph) / rr
    assert relerr(q1, qv1) < 1e-12
    assert relerr(q2, qv2) < 1e-12
    o.close()


def test_oracle_neutral_reference_state_operators():
    ca = anel_cfg(L=12, M=12, N=13, comp_tstep=0)
    cb = type(ca).from_buffer_copy(ca)
    cb.boussinesq = 1
    b = ol.Oracle(cb)
    a = ol.Oracle(ca)
    N = a.N
    neutral = np.zeros((7, N))
    neutral[[0, 3, 5]] = 1.0
    a.set_reference_state(neutral)
    for which in range(6):
        for l in (1, 5, 11):
            la, pa = a.operator_lu(which, l)
            lb, pb = b.operator_lu(which, l)
            assert np.array_equal(la, lb) and np.array_equal(pa, pb), (which, l)
    a.close()
    b.close()


def load_both(g, o, fields):
    for f, (re, im) in fields.items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)


@pytest.mark.gpu
def test_anelastic_unit_transforms():
    cfg = anel_cfg(L=32, M=32, N=9)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    l, m, _ = o.harmonics()
    rng = np.random.default_rng(7)

    def spec():
        re = rng.standard_normal((o.N, o.H))
        im = rng.standard_normal((o.N, o.H))
        im[:, m == 0] = 0.0
        return re, im

    ins = [spec() for _ in range(6)]
    names = ("r", "th", "ph", "dur", "qv1", "dutr", "dupr", "qv2")
    for nm, x, y in zip(names, g.tra_qst2rtp_vel(*ins), o.qst2rtp_vel(*ins)):
        assert relerr(x, y) < 1e-12, nm
    assert relerr(g.tra_dth(*ins[0]), o.dth(*ins[0])) < 1e-12
    g.close()
    o.close()


@pytest.mark.gpu
@pytest.mark.parametrize("prec,S,tol", [(capi.PREC_FP64, 0, 1e-11), (capi.PREC_OZAKI, 7, 5e-11)])
def test_anelastic_evaluation_and_step(prec, S, tol):
    cfg = anel_cfg()
    g = pkg.Context(anel_cfg(precision=prec, ozaki_slices=S))
    o = ol.Oracle(cfg)
    prof = syn.polytrope_reference_state(cfg.N, cfg.rratio)
    g.set_reference_state(prof)
    o.set_reference_state(prof)
    load_both(g, o, syn.boussinesq_state(cfg, seed=11, composition=True))
    g.nonlinear()
    o.nonlinear()
    for w in range(6):
        a, b = g.get_nonlinear(w), o.get_nonlinear(w)
        assert relerr(a[0], b[0]) < tol, ("nl", w, relerr(a[0], b[0]))
        assert relerr(a[1], b[1]) < tol, ("nl", w, relerr(a[1], b[1]))
    g.predictor(); o.predictor()
    for f in range(6):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < tol, ("pred", f)
        assert relerr(a[1], b[1]) < tol, ("pred", f)
    g.nonlinear(); o.nonlinear()
    d1, d2 = g.corrector(), o.corrector()
    assert abs(d1 - d2) <= 1e-9 * abs(d2)
    for f in range(6):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < tol, ("corr", f)
        assert relerr(a[1], b[1]) < tol, ("corr", f)
    ea, eb = g.energies(), o.energies()
    for k in ("KE", "ME", "KE_dis", "ME_dis", "topflx", "botflx", "KE_ax", "ME_ax"):
        assert abs(ea[k] - eb[k]) <= 1e-10 * abs(eb[k]), (k, ea[k], eb[k])
    g.close()
    o.close()


@pytest.mark.gpu
def test_anelastic_hundred_steps():
    """L = M = 32, N = 33, the polytrope, composition on, stress-free, 100 steps (FP64)."""
    cfg = anel_cfg(L=32, N=33)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    prof = syn.polytrope_reference_state(cfg.N, cfg.rratio)
    g.set_reference_state(prof)
    o.set_reference_state(prof)
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


@pytest.mark.gpu
def test_boussinesq_stress_free_angular_momentum():
    """vel_bc = 4 (stress-free) Boussinesq: vel_angmomclr before every evaluation."""
    cfg = syn.config_parity(N=17, vel_bc=4)
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    load_both(g, o, syn.boussinesq_state(cfg, seed=13))
    sg, so = g.step(20), o.step(20)
    assert sg.correctors == so.correctors
    for f in range(5):
        a, b = g.get_coll(f), o.get_coll(f)
        assert relerr(a[0], b[0]) < 1e-10, f
        assert relerr(a[1], b[1]) < 1e-10, f
    g.close()
    o.close()
