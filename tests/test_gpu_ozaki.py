"""The tensor-core (Ozaki int8-slice) Legendre path against the CPU oracle.

Each operand is scaled by a power of two per row (spectral coefficients of one shell and
order m) or per column (one theta row, or one harmonic), rounded to an integer of 8S - 2
bits and split into S balanced base-256 int8 digits; the products of digit pairs whose
index sum is below S are accumulated exactly in int32 on the tcgen05 tensor cores and
recombined exactly (in int64 where the sum's bound allows, else in FP64).  Rounding costs 2^(1-8S) and the dropped tail about (S + 1) 2^(2-8S)
of (row max) x (column max) per product, so a single transform agrees with the FP64
oracle to about 1e-14 of the largest output for S >= 7 (FP64 rounding), 1e-11 for S = 6
and 3e-9 for S = 5.  Tolerances (relative to the largest magnitude of the compared array):
  single transforms, S = 3, 4    5e-3, 2e-5 (the S = 5 bar times 256 per slice, 4x margin)
  single transforms, S = 5       2e-8
  single transforms, S = 6       1e-10
  single transforms, S = 7, 8    5e-13
  one nonlinear evaluation       2e-12 (default S = 7)
  energies after 100 steps       1e-9 (the mixed-precision acceptance bar)
"""
import importlib

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic


def relerr(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    s = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / s)


def test_ozaki_slices_are_validated():
    """lsd_create rejects slice counts outside 2..8 before touching a device."""
    cfg = syn.config_parity(precision=capi.PREC_OZAKI, ozaki_slices=9)
    with pytest.raises(pkg.LsdError) as e:
        pkg.Context(cfg)
    assert e.value.status == capi.LSD_EARG


@pytest.mark.gpu
@pytest.mark.parametrize("LMMp,S,tol", [((32, 32, 1), 7, 5e-13), ((64, 16, 4), 7, 5e-13),
                                         ((24, 8, 2), 7, 5e-13), ((32, 32, 1), 8, 5e-13),
                                         ((64, 16, 4), 6, 1e-10), ((64, 16, 4), 5, 2e-8),
                                         # 48-column synthesis chunks with 18 theta rows (masked)
                                         ((24, 8, 2), 5, 2e-8),
                                         # fewer slices: 256 times per slice, 4x margin
                                         ((64, 16, 4), 4, 2e-5), ((32, 32, 1), 3, 5e-3)])
def test_ozaki_transforms(LMMp, S, tol):
    L, M, Mp = LMMp
    cfg = capi.template_config(L=L, M=M, Mp=Mp, N=9, timestep=1e-5, precision=capi.PREC_OZAKI,
                               ozaki_slices=S)
    ref = capi.template_config(L=L, M=M, Mp=Mp, N=9, timestep=1e-5)
    g, o = pkg.Context(cfg), ol.Oracle(ref)
    rng = np.random.default_rng(L + M + S)
    l, m, s = o.harmonics()
    H, N = o.H, o.N

    def spec():
        re = rng.standard_normal((N, H)) / (1.0 + l) ** 2
        im = rng.standard_normal((N, H)) / (1.0 + l) ** 2
        im[:, m == 0] = 0
        return re, im

    errs = {}
    sre, sim = spec()
    errs["spec2phys"] = relerr(g.tra_spec2phys(sre, sim), o.spec2phys(sre, sim))
    p = rng.standard_normal((N, o.Ph, o.Th))
    a, b = g.tra_phys2spec(p), o.phys2spec(p)
    errs["phys2spec"] = max(relerr(a[0], b[0]), relerr(a[1], b[1]))
    q, sv, tv = spec(), spec(), spec()
    errs["qst2rtp"] = max(relerr(x, y) for x, y in zip(g.tra_qst2rtp(q, sv, tv), o.qst2rtp(q, sv, tv)))
    r, th, ph = (rng.standard_normal((N, o.Ph, o.Th)) for _ in range(3))
    errs["rtp2qst"] = max(max(relerr(x[0], y[0]), relerr(x[1], y[1]))
                          for x, y in zip(g.tra_rtp2qst(r, th, ph), o.rtp2qst(r, th, ph)))
    errs["grad"] = max(relerr(x, y) for x, y in zip(g.tra_grad(sre, sim), o.grad(sre, sim)))
    print(LMMp, S, errs)
    for k, v in errs.items():
        assert v < tol, (k, v)
    g.close()


@pytest.mark.gpu
def test_ozaki_nonlinear_terms():
    cfg = syn.config_parity(N=17, precision=capi.PREC_OZAKI)
    g, o = pkg.Context(cfg), ol.Oracle(syn.config_parity(N=17))
    for f, (re, im) in syn.boussinesq_state(cfg).items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)
    g.nonlinear()
    o.nonlinear()
    for w in range(5):
        a, b = g.get_nonlinear(w), o.get_nonlinear(w)
        e = max(relerr(a[0], b[0]), relerr(a[1], b[1]))
        print("nonlinear", w, e)
        assert e < 2e-12, w
    g.close()


@pytest.mark.gpu
def test_ozaki_hundred_steps_energies():
    """Mixed-precision run of the L=M=32, N=33 shell: energies after 100 steps within 1e-9
    of the FP64 oracle, and the same corrector iteration count."""
    ref = syn.config_parity()
    cfg = syn.config_parity(precision=capi.PREC_OZAKI)
    g, o = pkg.Context(cfg), ol.Oracle(ref)
    for f, (re, im) in syn.boussinesq_state(ref).items():
        g.set_coll(f, re, im)
        o.set_coll(f, re, im)
    sg = g.step(100)
    so = o.step(100)
    assert sg.steps_done == so.steps_done == 100
    assert sg.correctors == so.correctors
    eg, eo = g.energies(), o.energies()
    for k in ("KE", "ME", "KE_ax", "ME_ax", "KE_dis", "ME_dis", "topflx", "botflx"):
        err = abs(eg[k] - eo[k]) / abs(eo[k])
        print(k, err)
        assert err <= 1e-9, (k, eg[k], eo[k])
    g.close()
