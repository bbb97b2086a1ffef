"""Seeded synthetic initial states and workload configurations.

No public dataset or checkpoint exists for these workloads; the states are drawn from a
fixed seed with the shapes and amplitude spectra of the named configurations:
complex FP64 coefficients ~ N(0,1) for every (l, m), scaled by 1e-3 * l^-2 and by the
radial profile sin(pi (r - ri)) on the reference's Chebyshev grid (meshs.F90:135-143);
l = 0 coefficients are zero (the l = 0 velocity and magnetic modes are not stepped,
timestep.F90:579, and the codensity's l = 0 profile comes from its boundary condition,
codensity.F90:165-181); m = 0 imaginary parts are zero.
"""
import numpy as np

from . import capi
from .state import folded_harmonics, state_nh

SEED = 20261203


def chebyshev_grid(N, rratio, alpha=-1.0):
    """mes_oc%r(:,1) of meshs.F90:135-143."""
    n = np.arange(1, N + 1)
    if alpha > 0:
        r = 0.5 * (1.0 + np.arcsin(alpha * np.cos(np.pi * (N - n) / (N - 1))) / np.arcsin(alpha))
    else:
        r = 0.5 * (1.0 + np.cos(np.pi * (N - n) / (N - 1)))
    return r + rratio / (1.0 - rratio)


def boussinesq_state(cfg, seed=SEED, amplitude=1e-3, fields=(capi.VEL_TOR, capi.VEL_POL, capi.COD_C,
                                                             capi.MAG_TOR, capi.MAG_POL),
                     composition=False):
    """dict field -> (re, im), each (H, N) == Fortran coll (N, H).

    Draw order: for each field in (uT, uP, C, BT, BP) and then, with composition=True,
    Comp, one (H_file, 2) standard-normal block in the state-file (m-major) harmonic order
    of io_state_nh (so the first five fields do not depend on composition)."""
    L, M, Mp, N = cfg.L, cfg.M, cfg.Mp, cfg.N
    l, m_, _ = folded_harmonics(L, M, Mp)
    H = len(l)
    idx = state_nh(l, m_, L, M, Mp)
    r = chebyshev_grid(N, cfg.rratio, cfg.alpha)
    ri = cfg.rratio / (1.0 - cfg.rratio)
    prof = np.sin(np.pi * (r - ri))
    rng = np.random.Generator(np.random.PCG64(seed))
    amp = np.zeros(H)
    amp[l > 0] = amplitude / l[l > 0].astype(np.float64) ** 2
    out = {}
    order = [capi.VEL_TOR, capi.VEL_POL, capi.COD_C, capi.MAG_TOR, capi.MAG_POL]
    if composition:
        order.append(capi.COMP_C)
        fields = tuple(fields) + (capi.COMP_C,)
    for f in order:
        z = rng.standard_normal((H, 2))[idx]  # file order -> folded order
        re = (z[:, 0] * amp)[:, None] * prof[None, :]
        im = (z[:, 1] * amp)[:, None] * prof[None, :]
        im[m_ == 0, :] = 0.0
        if f in fields:
            out[f] = (np.ascontiguousarray(re), np.ascontiguousarray(im))
    return out


def polytrope_reference_state(N, rratio=0.35, alpha=-1.0, n=2.0, c0=-0.459754, c1=1.515898, file_precision=True):
    """The seven columns of planet_model.txt.in (io.F90:559-608) for a polytrope of index n
    (Jones et al. 2011, Icarus 216, 120-135): zeta = c0 + c1/r, rho = zeta^n,
    xi = rho'/rho = -n c1 / (r^2 zeta), dxi/dr = 2 n c1/(r^3 zeta) - n c1^2/(r^4 zeta^2),
    T = zeta/c1, dT/dr = -1/r^2, eta = 1, deta/dr = 0, on the Chebyshev grid.  The default
    constants give rho_i/rho_o = e^3 at rratio 0.35 (N_rho = 3).  With file_precision the
    values are rounded as the text file stores them (%12.8f for the first five columns,
    %12.8e for the diffusivity).  Returns (7, N)."""
    r = chebyshev_grid(N, rratio, alpha)
    zeta = c0 + c1 / r
    cols = [zeta ** n, -n * c1 / (r ** 2 * zeta),
            2 * n * c1 / (r ** 3 * zeta) - n * c1 * c1 / (r ** 4 * zeta * zeta),
            zeta / c1, -1.0 / (r * r), np.ones(N), np.zeros(N)]
    prof = np.array(cols, dtype=np.float64)
    if file_precision:
        for k in range(5):
            prof[k] = [float("%12.8f" % v) for v in prof[k]]
        for k in (5, 6):
            prof[k] = [float("%12.8e" % v) for v in prof[k]]
    return prof


def random_spectral(L, M, Mp, nshell, nfield, seed=SEED, power=1.0):
    """Random complex coefficients ~ N(0,1) * l^-power (l = 0 -> 1), m = 0 imaginary zero.
    Returns interleaved complex array [field][shell][H] (harmonic fastest)."""
    l, m_, _ = folded_harmonics(L, M, Mp)
    H = len(l)
    rng = np.random.Generator(np.random.PCG64(seed))
    a = np.ones(H)
    a[l > 0] = 1.0 / l[l > 0].astype(np.float64) ** power
    z = rng.standard_normal((nfield, nshell, H, 2)) * a[None, None, :, None]
    z[:, :, m_ == 0, 1] = 0.0
    return z  # (..., 2) = (re, im)


# ---- named workloads ------------------------------------------------------------------
def config_parity(**kw):
    """Plain FP64 Boussinesq MHD shell at L = M = 32 (lmax = mmax = 31; Th = 48, Ph = 96),
    N = 33, E = 3e-4, Ra = 200, Pr = 1, Pm = 3, dt = 1e-5, no-slip, fixed T, insulating."""
    base = dict(L=32, M=32, Mp=1, N=33, Nic=1, KL=3, rratio=0.35, E=3e-4, Ra=200.0, Pr=1.0,
                Pm=3.0, vel_bc=1, cod_bc=1, timestep=1e-5, implicit=0.6, time_step_control=2)
    base.update(kw)
    return capi.template_config(**base)


def config_anelastic(L=64, **kw):
    """Anelastic dynamo shell (n = 2 polytrope, N_rho = 3, the reference's anelastic
    benchmark parameters Ra = 8e4, Pr = 1, Pm = 50, E = 2e-3, rratio 0.35, stress-free
    walls, fixed entropy) at L = M, N = L + 1, with composition (Sc = 3, Ra_comp = 4e4,
    fixed composition), fixed dt = 1e-6, implicit 0.5."""
    base = dict(L=L, M=L, Mp=1, N=L + 1, Nic=1, KL=3, rratio=0.35, E=2e-3, Ra=8.0e4, Pr=1.0,
                Pm=50.0, vel_bc=4, cod_bc=1, comp_bc=1, comp_tstep=1, Sc=3.0, Ra_comp=4.0e4,
                boussinesq=0, timestep=1e-6, implicit=0.5, time_step_control=2)
    base.update(kw)
    return capi.template_config(**base)


def config_inner_core(L=32, **kw):
    """Christensen case 2 parameters (conducting, rotating inner core; E = 1e-3,
    Ra = 7.15e4, Pr = 1, Pm = 5, rratio 0.35, no-slip walls, fixed T; the reference's
    tests/parameters-case2.F90) at L = M, N = L + 1, Nic = L / 2 + 1, KL = 3, fixed
    dt = 1e-5, implicit 0.5."""
    base = dict(L=L, M=L, Mp=1, N=L + 1, Nic=L // 2 + 1, KL=3, rratio=0.35, E=1e-3, Ra=7.15e4, Pr=1.0,
                Pm=5.0, vel_bc=1, cod_bc=1, timestep=1e-5, implicit=0.5, time_step_control=2, rot_tstep=1)
    base.update(kw)
    return capi.template_config(**base)


def inner_core_grid(Nic, rratio):
    """mes_ic%r(:,1) (meshs.F90:165-169): ri cos(pi (Nic - n) / (2 Nic - 1)), n = 1..Nic."""
    ri = rratio / (1.0 - rratio)
    N_ = 2 * Nic
    n = np.arange(Nic + 1, N_ + 1)
    return ri * np.cos(np.pi * (N_ - n) / float(N_ - 1))


def ic_extend(re, im, r_oc, dr1_first, r_ic):
    """io_ic_extend (io.F90:1438-1477): continue an outer-core field (H, N) into the inner
    core as a r^3 + b r^2, matching its value and dr(1) derivative at r_i.  dr1_first: the
    weights of dr(1) at the first point on points 1..KL+1."""
    ri = r_oc[0]
    out = []
    for x in (re, im):
        f = x[:, 0]
        f1 = np.zeros_like(f)
        for j, w in enumerate(dr1_first):
            f1 = f1 + w * x[:, j]
        a = (f1 * ri - 2.0 * f) / ri ** 3
        b = (f - a * ri ** 3) / ri ** 2
        out.append(a[:, None] * r_ic[None, :] ** 3 + b[:, None] * r_ic[None, :] ** 2)
    return out[0], out[1]


def config_dynamo128(**kw):
    """Full Boussinesq dynamo step at lmax = mmax = 127 (L = M = 128; Th = 192, Ph = 384),
    N = 129, parameters of config_parity, dt = 2e-6."""
    base = dict(L=128, M=128, Mp=1, N=129, Nic=1, KL=3, rratio=0.35, E=3e-4, Ra=200.0, Pr=1.0,
                Pm=3.0, vel_bc=1, cod_bc=1, timestep=2e-6, implicit=0.6, time_step_control=2)
    base.update(kw)
    return capi.template_config(**base)


def config_solve257(**kw):
    """Batched banded solves: L = M = 256, Mp = 1, N = 257, KL = 4 (the 9-point stencil),
    with the operator parameters of config_dynamo128 (E = 3e-4, Ra = 200, Pr = 1, Pm = 3,
    dt = 2e-6, implicit 0.6)."""
    base = dict(L=256, M=256, Mp=1, N=257, KL=4, E=3e-4, Ra=200.0, Pr=1.0, Pm=3.0, vel_bc=1, cod_bc=1,
                timestep=2e-6, implicit=0.6, time_step_control=2)
    base.update(kw)
    return capi.template_config(**base)


def seeded_rhs(nfield, N, H, hm, seed=SEED):
    """complex N(0, 1) right-hand sides [field][N][H] (re, im), Im = 0 where m = 0"""
    rng = np.random.default_rng(seed)
    re = rng.standard_normal((nfield, N, H))
    im = rng.standard_normal((nfield, N, H))
    im[:, :, np.asarray(hm) == 0] = 0.0
    return re, im


ENSEMBLE_L = (64, 64, 96, 96, 128, 128, 192, 192)


def config_ensemble(**kw):
    """The anelastic ensemble: eight runs of config_anelastic, two each at L = M = 64, 96,
    128, 192 with N = L + 1 (Th = 3L/2, Ph = 2 Th), N_rho = 3 polytrope, codensity +
    composition; kw apply to every member (e.g. precision, ozaki_slices)."""
    return [config_anelastic(L=L, **kw) for L in ENSEMBLE_L]


def setup_ensemble_member(ctx, cfg, seed):
    """reference state (polytrope on the member's grid) and the seeded l^-2 state"""
    if not cfg.boussinesq:
        ctx.set_reference_state(polytrope_reference_state(cfg.N, cfg.rratio))
    st = boussinesq_state(cfg, seed=seed, composition=bool(cfg.comp_tstep))
    for f, (re, im) in st.items():
        ctx.set_coll(f, re, im)
    return st
