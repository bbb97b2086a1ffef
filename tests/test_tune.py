"""The autotuner (lsd_tune_candidates / lsd_tune_choose / lsd_get_tuning / lsd_set_tuning).

CPU: the candidate lists of several configurations (every phi-FFT plan multiplies out to
P2 = 3M/2 and is compiled, the default plan comes first, the tensor-core GEMM's tiles
respect the shared-memory limit of their CTAs per SM) and the selection rule on made-up
timings.
GPU: a tuned context reports parameters from its candidate lists; the solve mapping (CTA
size) leaves every bit of a run unchanged; another FFT plan changes coefficients only at
the rounding level (1e-12); a tuned context steps like an untuned one.
"""
import importlib

import numpy as np
import pytest

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi
syn = pkg.synthetic
lsd = pkg.lsd


@pytest.mark.parametrize("L,M,Mp,prec,S", [(32, 32, 1, 0, 0), (64, 16, 4, 0, 0), (128, 128, 1, 1, 5),
                                           (128, 128, 1, 1, 7), (192, 192, 1, 1, 8), (256, 256, 1, 0, 0)])
def test_candidates(L, M, Mp, prec, S):
    cfg = capi.template_config(L=L, M=M, Mp=Mp, N=33, precision=prec, ozaki_slices=S)
    sp = lsd.tune_candidates(cfg)
    P2 = 3 * M // 2
    assert sp["fft"], sp
    G0 = 1
    while G0 < 16 and P2 % (2 * G0) == 0:
        G0 *= 2
    assert sp["fft"][0] == (P2 // G0, G0)  # the default plan first
    for E, G in sp["fft"]:
        assert E * G == P2 and G in (4, 8, 16)
    assert sp["solve_threads"] == [128, 64, 32]
    if prec == capi.PREC_OZAKI:
        Sx = S or 7

        nc = 48 if Sx <= 5 else 32  # the synthesis chunk's columns

        def fits(nst, ctas):  # ring stages + 4 KB static, 1 KB reserved per CTA, 228 KB per SM
            return (nst * Sx * (4096 + nc * 32) + 4096) * ctas <= 228 * 1024 - 1024 * ctas
        default_stages = 3 if fits(3, 2) else 2
        assert sp["gemm"][0] == (default_stages, 2 if fits(default_stages, 2) else 1)
        for nst, ctas in sp["gemm"]:
            assert 2 <= nst <= 4 and ctas in (1, 2) and fits(nst, ctas)
        assert len(set(sp["gemm"])) == len(sp["gemm"])
    else:
        assert sp["gemm"] == []


def test_choose_rule():
    assert lsd.tune_choose([1.0, 0.99]) == 0        # within 2 %: keep the default
    assert lsd.tune_choose([1.0, 0.97]) == 1
    assert lsd.tune_choose([1.0, 1.2, 0.5], dflt=1) == 2
    assert lsd.tune_choose([1.0, 1.2, 1.19], dflt=1) == 0
    assert lsd.tune_choose([2.0, 1.0, 1.0]) == 1     # ties: the first fastest
    assert lsd.tune_choose([]) == -1


def test_config_field():
    cfg = capi.template_config(autotune=1)
    assert cfg.autotune == 1 and list(cfg.reserved) == [0] * 5


def run(cfg, steps=5, tuning=None):
    g = pkg.Context(cfg)
    if tuning:
        g.set_tuning(**tuning)
    for f, (re, im) in syn.boussinesq_state(cfg).items():
        g.set_coll(f, re, im)
    g.step(steps)
    out = [g.get_coll(f) for f in range(5)], g.energies(), g.tuning()
    g.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("prec,S", [(capi.PREC_FP64, 0), (capi.PREC_OZAKI, 5)])
def test_tuned_context(prec, S, parity_report):
    cfg = syn.config_parity(precision=prec, ozaki_slices=S)
    base, e0, t0 = run(cfg)
    assert t0["tuned"] == 0
    cfg_t = syn.config_parity(precision=prec, ozaki_slices=S, autotune=1)
    tuned, e1, t1 = run(cfg_t)
    sp = lsd.tune_candidates(cfg_t)
    assert t1["tuned"] == 1 and t1["ms_fft"] > 0 and t1["ms_solve"] > 0
    assert (t1["fft_E"], t1["fft_G"]) in sp["fft"] and t1["solve_threads"] in sp["solve_threads"]
    if prec == capi.PREC_OZAKI:
        assert (t1["gemm_stages"], t1["gemm_ctas_per_sm"]) in sp["gemm"] and t1["ms_gemm"] > 0
    for k in ("KE", "ME", "KE_dis", "ME_dis"):
        err = abs(e1[k] - e0[k]) / abs(e0[k])
        parity_report("tuned vs default context, %s" % k, err, 1e-12)
        assert err <= 1e-12, (k, err)
    print("tuning", t1)


@pytest.mark.gpu
def test_solve_mapping_is_bit_exact():
    cfg = syn.config_parity()
    base, _, _ = run(cfg, steps=3)
    for th in (64, 32):
        other, _, t = run(cfg, steps=3, tuning={"solve_threads": th})
        assert t["solve_threads"] == th
        for (a, b) in zip(base, other):
            assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]), th


@pytest.mark.gpu
def test_other_fft_plan(parity_report):
    cfg = syn.config_parity()
    sp = lsd.tune_candidates(cfg)
    base, _, _ = run(cfg, steps=3)
    for E, G in sp["fft"][1:]:
        other, _, t = run(cfg, steps=3, tuning={"fft_E": E, "fft_G": G})
        assert (t["fft_E"], t["fft_G"]) == (E, G)
        worst = 0.0
        for (a, b) in zip(base, other):
            d = np.hypot(a[0] - b[0], a[1] - b[1]).max() / max(np.hypot(a[0], a[1]).max(), 1e-300)
            worst = max(worst, d)
        parity_report("FFT plan (%d, %d) vs default, coefficients after 3 steps" % (E, G), worst, 1e-12)
        assert worst <= 1e-12, (E, G, worst)
