"""Parity at the sizes of the other scope configurations.

config[1]: the SHT round trip at lmax = mmax = 255 (L = M = 256, Th = 384, Ph = 768),
64 shells x 8 scalar fields, coefficients N(0,1) l^-1 from the seed (l = 0: 1), through
the device-resident batched entry points.  Per field: the synthesis against the oracle
(field 0, all 64 shells), the analysis of the oracle's grid values against the oracle's
analysis, and the round trip synthesis -> analysis of every field against the input.
The round trip is exact only up to the reference's Gauss nodes (Newton stopped at
1e-13, auxiliary/gauwts.f), about 3e-11 at this size for any arithmetic, so it is
checked against the oracle's own round trip of field 0 and bounded by 5e-11 per field.
Variants: the plain FP64 contraction and the tensor-core contraction at several slice
counts (S balanced base-256 int8 digits, 8S - 2 bits of the FP64 mantissa, rounded).
Tolerances, relative to the largest magnitude of the compared field:
  FP64            synthesis, analysis, round trip vs the oracle's: 1e-12
  tensor, S = 8   1e-13
  tensor, S = 7   5e-12
  tensor, S = 5   2e-8    (38 bits)
  tensor, S = 4   1e-6    (30 bits, about FP32)
config[2]: batched banded solves at N = 257, KL = 4.
  * On the context's own Crank-Nicolson operators at L = M = 256 (dt = 2e-6, E = 3e-4,
    Pm = 3, implicit 0.6; lsd_operator_solve_device): every (l, m) right-hand side of the
    codensity, the toroidal velocity, the field's toroidal and poloidal scalars and the
    poloidal velocity's fourth-order composite (5 x 32896 complex columns) in one launch,
    against the oracle's tim_invX / composite on the same right-hand sides, and the
    backward error of the second-order families from the LAPACK factors (tolerances in
    test_operator_solves_n257).
  * On random band matrices (lsd_banded_*_device): one operator per degree l < 256 for
    4 fields, every (l, m) right-hand side (Re and Im columns, 4 x 32896 x 2), residual
    |A x - b| / |b| <= 1e-13 on a sample checked on the host.
"""
import importlib
import time

import numpy as np
import pytest

import oracle_lib as ol

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi


def sht256_cfg(**kw):
    return capi.template_config(L=256, M=256, Mp=1, N=64, timestep=1e-5, **kw)


def seeded_spectra(nf, N, l, m, seed=1):
    rng = np.random.default_rng(seed)
    amp = np.where(l == 0, 1.0, 1.0 / np.maximum(l, 1))
    re = rng.standard_normal((nf, N, l.size)) * amp
    im = rng.standard_normal((nf, N, l.size)) * amp
    im[:, :, m == 0] = 0.0
    return re, im


@pytest.fixture(scope="module")
def sht256_reference():
    o = ol.Oracle(sht256_cfg())
    l, m, _ = o.harmonics()
    re, im = seeded_spectra(8, o.N, l, m)
    p0 = o.spec2phys(re[0], im[0])
    a0 = o.phys2spec(p0)
    return re, im, p0, a0


def relerr(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("prec,S,tol", [(capi.PREC_FP64, 0, 1e-12), (capi.PREC_OZAKI, 8, 1e-13),
                                        (capi.PREC_OZAKI, 7, 5e-12), (capi.PREC_OZAKI, 5, 2e-8),
                                        (capi.PREC_OZAKI, 4, 1e-6)])
def test_sht_round_trip_lmax255(sht256_reference, prec, S, tol):
    import torch
    re, im, p0, a0 = sht256_reference
    nf = re.shape[0]
    g = pkg.Context(sht256_cfg(precision=prec, ozaki_slices=S))
    N, H, Ph, Th = g.N, g.H, g.Ph, g.Th
    spec = np.stack([re, im], axis=-1)  # [f][n][nh][2]
    d_spec = torch.tensor(spec, device="cuda", dtype=torch.float64).contiguous()
    d_phys = torch.empty((nf, N, Ph, Th), device="cuda", dtype=torch.float64)
    d_back = torch.empty_like(d_spec)
    g.sht_synth_device(nf, d_spec.data_ptr(), d_phys.data_ptr())
    g.sht_analys_device(nf, d_phys.data_ptr(), d_back.data_ptr())
    g.synchronize()
    # wall time of round trips with the inputs resident in HBM (host-synchronised)
    t0 = time.perf_counter()
    for _ in range(3):
        g.sht_synth_device(nf, d_spec.data_ptr(), d_phys.data_ptr())
        g.sht_analys_device(nf, d_phys.data_ptr(), d_back.data_ptr())
    g.synchronize()
    ms = (time.perf_counter() - t0) * 1e3 / 3
    phys = d_phys.cpu().numpy()
    back = d_back.cpu().numpy()
    # analysis of the oracle's grid values (field 0)
    d_p0 = torch.tensor(p0, device="cuda", dtype=torch.float64).contiguous()
    d_a0 = torch.empty((N, H, 2), device="cuda", dtype=torch.float64)
    g.sht_analys_device(1, d_p0.data_ptr(), d_a0.data_ptr())
    g.synchronize()
    a0g = d_a0.cpu().numpy()
    e_syn = relerr(phys[0], p0)
    e_ana = max(relerr(a0g[..., 0], a0[0]), relerr(a0g[..., 1], a0[1]))
    e_rt = [relerr(back[f], spec[f]) for f in range(nf)]
    rt_oracle = np.stack([a0[0], a0[1]], axis=-1)
    e_rt_vs = relerr(back[0], rt_oracle)
    flops = 2 * 2 * 4 * H * (Th // 2) * N * nf  # complex x real MACs of synthesis + analysis
    print("prec %d S %d: synthesis %.2e analysis %.2e, round trip vs oracle's %.2e (vs input max %.2e), "
          "%.2f ms per round trip of %d fields (%.2f TF/s Legendre-equivalent, host-timed)"
          % (prec, S, e_syn, e_ana, e_rt_vs, max(e_rt), ms, nf, flops / (ms * 1e-3) / 1e12))
    assert e_syn <= tol, e_syn
    assert e_ana <= tol, e_ana
    assert e_rt_vs <= max(tol, 1e-12), e_rt_vs
    assert max(e_rt) <= max(tol, 5e-11), e_rt
    g.close()


@pytest.mark.gpu
def test_batched_banded_solves_n257():
    import torch
    import scipy.linalg.lapack as lapack
    n, kl, L, nfield = 257, 4, 256, 4
    H = L * L - (L - 1) * L // 2  # (l, m) pairs, m <= l < L
    nmat = nfield * L
    rng = np.random.default_rng(257)
    ab = np.zeros((nmat, n, 3 * kl + 1))
    ab[:, :, kl:] = rng.standard_normal((nmat, n, 2 * kl + 1))
    ab[:, :, 2 * kl] += 6.0
    # every (field, l, m) right-hand side, Re and Im columns; column r uses matrix map[r]
    degs = np.concatenate([np.full(l + 1, l) for l in range(L)])
    assert degs.size == H
    rmap = np.concatenate([f * L + np.repeat(degs, 2) for f in range(nfield)]).astype(np.int32)
    nrhs = rmap.size
    g = pkg.Context(capi.template_config(L=16, M=16, Mp=1, N=9, timestep=1e-5))
    d_ab = torch.tensor(ab, device="cuda", dtype=torch.float64)
    d_ip = torch.zeros((nmat, n), device="cuda", dtype=torch.int32)
    d_info = torch.zeros(nmat, device="cuda", dtype=torch.int32)
    d_b = torch.randn((n, nrhs), device="cuda", dtype=torch.float64,
                      generator=torch.Generator(device="cuda").manual_seed(5))
    b = d_b.cpu().numpy()
    d_map = torch.tensor(rmap, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.banded_factor_device(n, kl, nmat, d_ab.data_ptr(), d_ip.data_ptr(), d_info.data_ptr())
    g.banded_solve_device(n, kl, nmat, d_ab.data_ptr(), d_ip.data_ptr(), nrhs, d_map.data_ptr(), d_b.data_ptr())
    g.synchronize()
    dt = time.perf_counter() - t0
    assert (d_info.cpu().numpy() == 0).all()
    x = d_b.cpu().numpy()
    print("factor %d operators + %d right-hand sides (n=%d, kl=%d): %.2f ms" % (nmat, nrhs, n, kl, dt * 1e3))
    sample = rng.choice(nrhs, 300, replace=False)
    worst = 0.0
    for r in sample:
        k = rmap[r]
        A = np.zeros((n, n))
        for j in range(n):
            for i in range(max(0, j - kl), min(n, j + kl + 1)):
                A[i, j] = ab[k, j, 2 * kl + i - j]
        res = np.abs(A @ x[:, r] - b[:, r]).max() / np.abs(b[:, r]).max()
        worst = max(worst, res)
    assert worst <= 1e-13, worst
    # and the factors equal LAPACK's for a few operators
    lu_g = d_ab.cpu().numpy()
    for k in (0, 255, 511, 1023):
        lu_l, ip_l, info = lapack.dgbtrf(ab[k].T.copy(), kl, kl)
        assert np.abs(lu_g[k].T - lu_l).max() <= 1e-13 * np.abs(lu_l).max()
    g.close()


def lu_apply(ab, ipiv, kl, x):
    """A x from LAPACK band LU factors: ab (3 kl + 1, n) band storage (0-based rows, U in
    rows 0..2 kl, the multipliers below), ipiv 1-based; x (n, ncols).  Undoes dgbtrs's
    forward elimination (b[j+1..] -= l_j b[j] after swapping j and ipiv[j]) on U x."""
    n = ab.shape[1]
    y = np.zeros_like(x)
    for j in range(n):
        i0 = max(0, j - 2 * kl)
        y[i0:j + 1] += ab[2 * kl + np.arange(i0, j + 1) - j, j][:, None] * x[j]
    for j in range(n - 2, -1, -1):
        km = min(kl, n - 1 - j)
        y[j + 1:j + 1 + km] += ab[2 * kl + 1:2 * kl + 1 + km, j][:, None] * y[j]
        p = ipiv[j] - 1
        if p != j:
            y[[j, p]] = y[[p, j]]
    return y


SOLVE257_FIELDS = (capi.COD_C, capi.VEL_TOR, capi.MAG_TOR, capi.MAG_POL, capi.VEL_POL)
# oracle operator_lu index of each second-order family
LU_INDEX = {capi.VEL_TOR: 0, capi.COD_C: 3, capi.MAG_TOR: 4, capi.MAG_POL: 5}


def masked_err(a, b, keep):
    """max |a - b| over the complex coefficients of the harmonics `keep` ((H, N) arrays),
    relative to the largest |b| there"""
    d = np.hypot(a[0] - b[0], a[1] - b[1])[keep]
    return float(d.max() / max(np.hypot(b[0], b[1])[keep].max(), 1e-300))


@pytest.mark.gpu
def test_operator_solves_n257(parity_report):
    """The five operator families at N = 257, KL = 4 on every (l, m) column.
    Forward error against the oracle's tim_invX / composite over the solved columns
    (l = 0 only for the codensity), bounded by max(1e-12, 4 x the oracle's own change when
    the right-hand sides are perturbed in the last bit; the operators and Green's functions
    are built on each side in their own order, the composite differs by 2.5e-13): the
    Chebyshev grid's wall rows
    (1/dr^2 ~ 7e8 against the O(1) boundary rows) make the operators badly scaled for
    right-hand sides that are random in every row, and the codensity's wall values move by
    6e-11 of its largest solution value under such a perturbation.  Backward error of the
    second-order families from the oracle's LAPACK factors, |A x - b| / (|A| |x| + |b|)
    (infinity norms, per column, a sample of degrees): <= 1e-15.  The unsolved l = 0
    columns (tim_invX skips them) equal the right-hand side with zeroed boundary rows."""
    import torch
    syn = pkg.synthetic
    cfg = syn.config_solve257()
    g, o = pkg.Context(cfg), ol.Oracle(cfg)
    l, m, _ = o.harmonics()
    nf, N, H = len(SOLVE257_FIELDS), o.N, o.H
    re, im = syn.seeded_rhs(nf, N, H, m)
    d = torch.tensor(np.stack([re, im], axis=-1), device="cuda", dtype=torch.float64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.operator_solve_device(SOLVE257_FIELDS, d.data_ptr())
    g.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    x = d.cpu().numpy()
    del d
    print("operator solves: %d fields x %d (l, m) columns, N = %d, KL = 4: %.2f ms (host-timed)" % (nf, H, N, ms))
    rng = np.random.default_rng(3)
    for k, f in enumerate(SOLVE257_FIELDS):
        zero = f in (capi.COD_C, capi.COMP_C)
        keep = np.ones(H, bool) if zero else l > 0
        xo = o.operator_solve(f, re[k].T, im[k].T)  # (H, N)
        xg = (x[k, :, :, 0].T, x[k, :, :, 1].T)
        sens = 0.0
        for _ in range(2):
            pr = re[k] * (1.0 + 1e-16 * rng.standard_normal(re[k].shape))
            pi = im[k] * (1.0 + 1e-16 * rng.standard_normal(im[k].shape))
            sens = max(sens, masked_err(o.operator_solve(f, pr.T, pi.T), xo, keep))
        err = masked_err(xg, xo, keep)
        tol = max(1e-12, 4.0 * sens)
        parity_report("solve257 field %d: device vs oracle (solved columns)" % f, err, tol)
        parity_report("solve257 field %d: oracle vs last-bit perturbed right-hand sides" % f, sens)
        assert err <= tol, (f, err, sens)
        if not zero:  # l = 0: not solved, the right-hand side with zero boundary rows
            c0 = np.nonzero(l == 0)[0]
            for part, b in ((0, re[k]), (1, im[k])):
                want = b[:, c0].T.copy()
                want[:, [0, -1]] = 0.0
                assert np.array_equal(xg[part][c0], want), f
        if f not in LU_INDEX:
            continue
        worst = 0.0
        for deg in (1, 2, 17, 128, 255) + ((0,) if zero else ()):
            cols = np.nonzero(l == deg)[0]
            ab, ipiv = o.operator_lu(LU_INDEX[f], deg)
            Anorm = np.abs(lu_apply(ab, ipiv, 4, np.eye(N))).sum(axis=1).max()
            for part in (0, 1):
                xs = xg[part][cols].T  # (N, ncols)
                bs = (re if part == 0 else im)[k][:, cols].copy()
                bs[0], bs[-1] = 0.0, 0.0  # tim_zerobc
                res = np.abs(lu_apply(ab, ipiv, 4, xs) - bs).max(axis=0)
                den = Anorm * np.abs(xs).max(axis=0) + np.abs(bs).max(axis=0)
                ok = den > 0
                if ok.any():
                    worst = max(worst, float((res[ok] / den[ok]).max()))
        parity_report("solve257 field %d: backward error |A x - b| / (|A| |x| + |b|)" % f, worst, 1e-15)
        assert worst <= 1e-15, (f, worst)
    g.close()
    o.close()
