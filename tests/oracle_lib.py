"""ctypes wrapper of the CPU FP64 oracle (oracle/liblsd_oracle.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
use this.  Arrays follow the reference's Fortran layouts (see include/lsd_b200.h).
"""
import ctypes
import importlib
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
capi = importlib.import_module("leeds-code_b200.capi")

_LIB = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


def load():
    global _LIB
    if _LIB is not None:
        return _LIB
    path = os.path.join(ROOT, "oracle", "liblsd_oracle.so")
    if not os.path.exists(path):
        subprocess.check_call(["sh", os.path.join(ROOT, "oracle", "build_oracle.sh")])
    lib = ctypes.CDLL(path)
    lib.orc_create.restype = ctypes.c_void_p
    lib.orc_create.argtypes = [ctypes.POINTER(capi.LsdConfig), _I]
    vp = ctypes.c_void_p
    sigs = {
        "orc_destroy": (None, [vp]),
        "orc_sizes": (None, [vp, ctypes.POINTER(capi.LsdSizes)]),
        "orc_harmonics": (None, [vp, _I, _I, _I]),
        "orc_theta_map": (None, [vp, _I]),
        "orc_radial_grid": (None, [vp, _D]),
        "orc_radial_weights": (None, [vp, _D]),
        "orc_dr": (None, [vp, ctypes.c_int, _D]),
        "orc_gauss": (None, [vp, _D, _D]),
        "orc_legendre_table": (ctypes.c_int, [vp, ctypes.c_int, _D]),
        "orc_operator_lu": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, _D, _I]),
        "orc_dgbtrf": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _D, _I]),
        "orc_dgbtrs": (None, [ctypes.c_int, ctypes.c_int, _D, _I, _D]),
        "orc_mat_invert": (ctypes.c_int, [ctypes.c_int, _D]),
        "orc_fft_c2r": (None, [ctypes.c_int, _D, _D, ctypes.c_int, _D]),
        "orc_fft_r2c": (None, [ctypes.c_int, _D, _D, _D]),
        "orc_set_coll": (ctypes.c_int, [vp, ctypes.c_int, _D, _D]),
        "orc_get_coll": (ctypes.c_int, [vp, ctypes.c_int, _D, _D]),
        "orc_get_nonlinear": (ctypes.c_int, [vp, ctypes.c_int, _D, _D]),
        "orc_set_time": (None, [vp, ctypes.c_double]),
        "orc_spec2phys": (ctypes.c_int, [vp, _D, _D, _D]),
        "orc_phys2spec": (ctypes.c_int, [vp, _D, _D, _D]),
        "orc_qst2rtp": (ctypes.c_int, [vp] + [_D] * 9),
        "orc_rtp2qst": (ctypes.c_int, [vp] + [_D] * 9),
        "orc_grad": (ctypes.c_int, [vp, _D, _D, _D, _D]),
        "orc_nonlinear": (ctypes.c_int, [vp]),
        "orc_predictor": (ctypes.c_int, [vp]),
        "orc_corrector": (ctypes.c_int, [vp, _D]),
        "orc_step": (ctypes.c_int, [vp, ctypes.c_int, ctypes.POINTER(capi.LsdStats)]),
        "orc_energies": (ctypes.c_int, [vp, _D]),
        "orc_diagnostics": (ctypes.c_int, [vp, _D, _D, _D]),
        "orc_set_rotation": (ctypes.c_int, [vp, ctypes.c_double]),
        "orc_get_rotation": (None, [vp, _D]),
        "orc_set_threads": (ctypes.c_int, [ctypes.c_int]),
        "orc_set_reference_state": (ctypes.c_int, [vp, _D]),
        "orc_dth": (ctypes.c_int, [vp, _D, _D, _D]),
        "orc_set_dt": (ctypes.c_int, [vp, ctypes.c_double]),
        "orc_dt_control": (None, [vp, _D]),
        "orc_qst2rtp_vel": (ctypes.c_int, [vp, ctypes.POINTER(_D), ctypes.POINTER(_D)]),
        "orc_operator_solve": (ctypes.c_int, [vp, ctypes.c_int, _D, _D]),
        "orc_tim_check_cgce": (ctypes.c_int, [ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(capi.LsdPcState)]),
        "orc_tim_new_tstep": (ctypes.c_int, [ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(capi.LsdPcState), _I]),
    }
    for name, (res, args) in sigs.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _LIB = lib
    return lib


def tim_check_cgce(cfg, state):
    """The oracle's tim_check_cgce on a capi.LsdPcState (in place); returns the status."""
    return load().orc_tim_check_cgce(ctypes.byref(cfg), ctypes.byref(state))


def tim_new_tstep(cfg, state):
    nd = ctypes.c_int(0)
    load().orc_tim_new_tstep(ctypes.byref(cfg), ctypes.byref(state), ctypes.byref(nd))
    return bool(nd.value)


def set_threads(n):
    return load().orc_set_threads(int(n))


class Oracle:
    """One oracle instance (the whole reference state of one run)."""

    def __init__(self, cfg):
        self.lib = load()
        st = ctypes.c_int(0)
        self.h = self.lib.orc_create(ctypes.byref(cfg), ctypes.byref(st))
        if not self.h:
            raise RuntimeError("oracle create failed: status %d" % st.value)
        s = capi.LsdSizes()
        self.lib.orc_sizes(self.h, ctypes.byref(s))
        self.sz = {k: getattr(s, k) for k, _ in capi.LsdSizes._fields_}
        self.H, self.N, self.Th, self.Th2, self.Ph = (self.sz[k] for k in ("H", "N", "Th", "Th2", "Ph"))
        self.cfg_Nic = cfg.Nic

    def close(self):
        if self.h:
            self.lib.orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- layout and tables
    def harmonics(self):
        l, m, s = (np.zeros(self.H, np.int32) for _ in range(3))
        self.lib.orc_harmonics(self.h, _ip(l), _ip(m), _ip(s))
        return l, m, s

    def theta_map(self):
        t = np.zeros(2 * self.sz["Hc"], np.int32)
        self.lib.orc_theta_map(self.h, _ip(t))
        return t

    def radial_grid(self):
        r = np.zeros(self.N)
        self.lib.orc_radial_grid(self.h, _dp(r))
        return r

    def radial_weights(self):
        r = np.zeros(self.N)
        self.lib.orc_radial_weights(self.h, _dp(r))
        return r

    def dr(self, order):
        kl = self.sz["KL"]
        b = np.zeros((self.N, 2 * kl + 1))
        self.lib.orc_dr(self.h, order, _dp(b))
        return b.T.copy()  # (2KL+1, N) Fortran band

    def gauss(self):
        gp, gw = np.zeros(self.Th), np.zeros(self.Th)
        self.lib.orc_gauss(self.h, _dp(gp), _dp(gw))
        return gp, gw

    def legendre_table(self, which):
        t = np.zeros((self.H, self.Th2))
        assert self.lib.orc_legendre_table(self.h, which, _dp(t)) == 0
        return t.T.copy()  # (Th2, H)

    def operator_solve(self, f, re, im):
        """tim_zerobc + tim_invX of field f's operator (the poloidal velocity's composite)
        on (H, N) arrays; returns the solution"""
        re = np.array(re, dtype=np.float64, order="C")
        im = np.array(im, dtype=np.float64, order="C")
        assert self.lib.orc_operator_solve(self.h, f, _dp(re), _dp(im)) == 0
        return re, im

    def operator_lu(self, which, l):
        kl = self.sz["KL"]
        ab = np.zeros((self.N, 3 * kl + 1))
        ipiv = np.zeros(self.N, np.int32)
        assert self.lib.orc_operator_lu(self.h, which, l, _dp(ab), _ip(ipiv)) == 0
        return ab.T.copy(), ipiv

    # ---- state (coll arrays returned as (H, N) C-order == Fortran (N, H))
    def rows(self, f):
        """radial points of a field: Nic for the inner core's, N otherwise"""
        return self.cfg_Nic if f in (capi.MAG_IC_TOR, capi.MAG_IC_POL) else self.N

    def set_coll(self, f, re, im):
        re = np.ascontiguousarray(re, dtype=np.float64)
        im = np.ascontiguousarray(im, dtype=np.float64)
        assert re.size == self.rows(f) * self.H
        assert self.lib.orc_set_coll(self.h, f, _dp(re), _dp(im)) == 0

    def get_coll(self, f):
        n = self.rows(f)
        re, im = np.zeros((self.H, n)), np.zeros((self.H, n))
        assert self.lib.orc_get_coll(self.h, f, _dp(re), _dp(im)) == 0
        return re, im

    def get_nonlinear(self, f):
        re, im = np.zeros((self.H, self.N)), np.zeros((self.H, self.N))
        assert self.lib.orc_get_nonlinear(self.h, f, _dp(re), _dp(im)) == 0
        return re, im

    def set_time(self, t, dt=None):
        self.lib.orc_set_time(self.h, t)
        if dt is not None:
            assert self.lib.orc_set_dt(self.h, dt) == 0

    def dt_control(self):
        """tim_dt, tim_corr_dt, tim_cfl_dt (io.F90:2346)."""
        out = np.zeros(3)
        self.lib.orc_dt_control(self.h, _dp(out))
        return out

    # ---- transforms: spec as (N, H) C-order == Fortran (H, N); phys (N, Ph, Th)
    def spec2phys(self, sre, sim):
        p = np.zeros((self.N, self.Ph, self.Th))
        self.lib.orc_spec2phys(self.h, _dp(np.ascontiguousarray(sre)), _dp(np.ascontiguousarray(sim)), _dp(p))
        return p

    def phys2spec(self, p):
        sre, sim = np.zeros((self.N, self.H)), np.zeros((self.N, self.H))
        self.lib.orc_phys2spec(self.h, _dp(np.ascontiguousarray(p)), _dp(sre), _dp(sim))
        return sre, sim

    def qst2rtp(self, q, s, t):
        outs = [np.zeros((self.N, self.Ph, self.Th)) for _ in range(3)]
        args = [np.ascontiguousarray(x) for x in (q[0], q[1], s[0], s[1], t[0], t[1])]
        self.lib.orc_qst2rtp(self.h, *[_dp(a) for a in args], *[_dp(o) for o in outs])
        return outs

    def rtp2qst(self, r, th, ph):
        outs = [np.zeros((self.N, self.H)) for _ in range(6)]
        ins = [np.ascontiguousarray(x) for x in (r, th, ph)]
        self.lib.orc_rtp2qst(self.h, *[_dp(a) for a in ins], *[_dp(o) for o in outs])
        return (outs[0], outs[1]), (outs[2], outs[3]), (outs[4], outs[5])

    def qst2rtp_vel(self, q, s, t, qr, sr, tr):
        """tra_qst2rtp_vel: -> r, th, ph, dur, qv1, dutr, dupr, qv2."""
        ins = [np.ascontiguousarray(x) for pair in (q, s, t, qr, sr, tr) for x in pair]
        outs = [np.zeros((self.N, self.Ph, self.Th)) for _ in range(8)]
        pin = (_D * 12)(*[_dp(a) for a in ins])
        pout = (_D * 8)(*[_dp(a) for a in outs])
        assert self.lib.orc_qst2rtp_vel(self.h, pin, pout) == 0
        return outs

    def dth(self, sre, sim):
        p = np.zeros((self.N, self.Ph, self.Th))
        self.lib.orc_dth(self.h, _dp(np.ascontiguousarray(sre)), _dp(np.ascontiguousarray(sim)), _dp(p))
        return p

    def set_reference_state(self, prof):
        """prof: (7, N) rho, xi, dxi/dr, T, dT/dr, eta, deta/dr (planet_model.txt.in)."""
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        assert prof.shape == (7, self.N)
        rc = self.lib.orc_set_reference_state(self.h, _dp(prof))
        if rc != 0:
            raise RuntimeError("oracle reference state failed: %d" % rc)

    def grad(self, sre, sim):
        t, p = np.zeros((self.N, self.Ph, self.Th)), np.zeros((self.N, self.Ph, self.Th))
        self.lib.orc_grad(self.h, _dp(np.ascontiguousarray(sre)), _dp(np.ascontiguousarray(sim)), _dp(t), _dp(p))
        return t, p

    # ---- stepping
    def nonlinear(self):
        assert self.lib.orc_nonlinear(self.h) == 0

    def predictor(self):
        assert self.lib.orc_predictor(self.h) == 0

    def corrector(self):
        d = ctypes.c_double(0)
        assert self.lib.orc_corrector(self.h, ctypes.byref(d)) == 0
        return d.value

    def step(self, n):
        st = capi.LsdStats()
        rc = self.lib.orc_step(self.h, int(n), ctypes.byref(st))
        if rc != 0:
            raise RuntimeError("oracle step failed: %d" % rc)
        return st

    def energies(self):
        e = np.zeros(capi.NENERGY)
        self.lib.orc_energies(self.h, _dp(e))
        return dict(zip(capi.ENERGY_NAMES, e))

    def set_rotation(self, omega):
        assert self.lib.orc_set_rotation(self.h, float(omega)) == 0

    def rotation(self):
        """rot_omega, rot_velTorq, rot_magTorq"""
        out = np.zeros(3)
        self.lib.orc_get_rotation(self.h, _dp(out))
        return out

    def diagnostics(self):
        """orc_diagnostics, unpacked like Context.diagnostics."""
        L, M, N = (self.sz[k] for k in ("L", "M", "N"))
        sc = np.zeros(capi.NDIAG)
        sp = np.zeros(capi.spectra_size(L, M))
        pr = np.zeros((len(capi.PROFILE_NAMES), N))
        self.lib.orc_diagnostics(self.h, _dp(sc), _dp(sp), _dp(pr))
        return (dict(zip(capi.DIAG_NAMES, sc)), capi.split_spectra(sp, L, M),
                dict(zip(capi.PROFILE_NAMES, pr)))


def dgbtrf(ab, kl):
    """oracle dgbtrf on a (3kl+1, n) Fortran band array; returns (lu, ipiv 1-based, info)."""
    lib = load()
    n = ab.shape[1]
    a = np.asfortranarray(ab, dtype=np.float64).copy(order="F")
    ipiv = np.zeros(n, np.int32)
    info = lib.orc_dgbtrf(n, kl, a.ctypes.data_as(_D), _ip(ipiv))
    return a, ipiv, info


def dgbtrs(lu, kl, ipiv, b):
    lib = load()
    n = lu.shape[1]
    a = np.asfortranarray(lu, dtype=np.float64)
    x = np.array(b, dtype=np.float64, copy=True)
    lib.orc_dgbtrs(n, kl, a.ctypes.data_as(_D), _ip(np.ascontiguousarray(ipiv, np.int32)), _dp(x))
    return x


def mat_invert(a):
    lib = load()
    x = np.asfortranarray(a, dtype=np.float64).copy(order="F")
    info = lib.orc_mat_invert(x.shape[0], x.ctypes.data_as(_D))
    return x, info


def fft_c2r(n, y):
    lib = load()
    yre = np.ascontiguousarray(y.real, np.float64)
    yim = np.ascontiguousarray(y.imag, np.float64)
    x = np.zeros(n)
    lib.orc_fft_c2r(n, _dp(yre), _dp(yim), len(y), _dp(x))
    return x


def fft_r2c(x):
    lib = load()
    n = len(x)
    yre, yim = np.zeros(n // 2 + 1), np.zeros(n // 2 + 1)
    lib.orc_fft_r2c(n, _dp(np.ascontiguousarray(x, np.float64)), _dp(yre), _dp(yim))
    return yre + 1j * yim
