"""Python host interface of the B200 dynamo-step library (ctypes over liblsd_b200.so).

Method names follow the reference's Fortran module procedures that the library
replaces (transform.fftw3.F90 tra_*, nonlinear.F90 non_*, the *_predictor/_corrector
sequence of main.F90, io.F90 energy writers).  A non-zero status from the C ABI raises
LsdError, the counterpart of the reference's `stop 'message'`.

Array conventions (numpy, C order) equal the reference's Fortran layouts:
  coll  (H, N)       == Fortran Re(i_N, 0:i_H1)
  spec  (N, H)       == Fortran Re(0:i_H1, i_N)
  phys  (N, Ph, Th)  == Fortran Re(i_Th, 0:i_Ph-1, i_N)
"""
import ctypes
import os

import numpy as np

from . import capi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "liblsd_b200.so")
_LIB = None
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_V = ctypes.c_void_p


class LsdError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("lsd status %d (%s): %s" % (status, capi.STATUS_NAMES.get(status, "?"), message))
        self.status = status


def load_library(path=None):
    """Load liblsd_b200.so (fails loudly when it is missing: there is no fallback)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError("liblsd_b200.so not built (%s); run the package build first" % p)
    lib = ctypes.CDLL(p)
    sigs = {
        "lsd_config_default": [ctypes.POINTER(capi.LsdConfig)],
        "lsd_create": [ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(_V)],
        "lsd_destroy": [_V],
        "lsd_get_sizes": [_V, ctypes.POINTER(capi.LsdSizes)],
        "lsd_harmonics": [_V, _I, _I, _I],
        "lsd_theta_map": [_V, _I],
        "lsd_radial_grid": [_V, _D],
        "lsd_radial_weights": [_V, _D],
        "lsd_gauss": [_V, _D, _D],
        "lsd_legendre_table": [_V, ctypes.c_int, _D],
        "lsd_set_coll": [_V, ctypes.c_int, _D, _D],
        "lsd_get_coll": [_V, ctypes.c_int, _D, _D],
        "lsd_get_nonlinear": [_V, ctypes.c_int, _D, _D],
        "lsd_set_time": [_V, ctypes.c_double, ctypes.c_double],
        "lsd_get_time": [_V, _D, _D, _I],
        "lsd_tra_spec2phys": [_V, _D, _D, _D],
        "lsd_tra_phys2spec": [_V, _D, _D, _D],
        "lsd_tra_qst2rtp": [_V] + [_D] * 9,
        "lsd_tra_rtp2qst": [_V] + [_D] * 9,
        "lsd_tra_grad": [_V, _D, _D, _D, _D],
        "lsd_tra_dth": [_V, _D, _D, _D],
        "lsd_tra_qst2rtp_vel": [_V] + [_D] * 20,
        "lsd_set_reference_state": [_V, _D],
        "lsd_get_dt_control": [_V, _D],
        "lsd_ensemble_create": [ctypes.c_int, ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(_V)],
        "lsd_ensemble_destroy": [_V],
        "lsd_ensemble_size": [_V],
        "lsd_ensemble_member": [_V, ctypes.c_int, ctypes.POINTER(_V)],
        "lsd_ensemble_step": [_V, ctypes.c_int, ctypes.POINTER(capi.LsdStats)],
        "lsd_sht_synth_device": [_V, ctypes.c_int, _V, _V],
        "lsd_sht_analys_device": [_V, ctypes.c_int, _V, _V],
        "lsd_matrices": [_V],
        "lsd_nonlinear": [_V],
        "lsd_predictor": [_V],
        "lsd_corrector": [_V, _D],
        "lsd_step": [_V, ctypes.c_int, ctypes.POINTER(capi.LsdStats)],
        "lsd_energies": [_V, _D],
        "lsd_energies_static": [_V, _D],
        "lsd_diagnostics": [_V, _D, _D, _D],
        "lsd_stage_coll": [_V, ctypes.c_int, _D, _D],
        "lsd_commit_staged": [_V],
        "lsd_set_rotation": [_V, ctypes.c_double],
        "lsd_get_rotation": [_V, _D],
        "lsd_banded_factor_device": [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int, _V, _V, _V],
        "lsd_banded_solve_device": [_V, ctypes.c_int, ctypes.c_int, ctypes.c_int, _V, _V, ctypes.c_int, _V, _V],
        "lsd_profile_phases": [_V, _D, _I],
        "lsd_selftest": [_V, ctypes.c_int, _D],
        "lsd_synchronize": [_V],
        "lsd_last_elapsed_ms": [_V, _D],
        "lsd_kernel_launches": [_V, ctypes.POINTER(ctypes.c_longlong)],
        "lsd_operator_solve_device": [_V, ctypes.c_int, _I, _V],
        "lsd_get_stream": [_V, ctypes.POINTER(_V)],
        "lsd_ensemble_last_elapsed_ms": [_V, _D],
        "lsd_tune_candidates": [ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(capi.LsdTuneSpace)],
        "lsd_tune_choose": [ctypes.c_int, _D, ctypes.c_int],
        "lsd_get_tuning": [_V, ctypes.POINTER(capi.LsdTuning)],
        "lsd_set_tuning": [_V, ctypes.POINTER(capi.LsdTuning)],
        "lsd_tim_check_cgce": [ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(capi.LsdPcState)],
        "lsd_tim_new_tstep": [ctypes.POINTER(capi.LsdConfig), ctypes.POINTER(capi.LsdPcState), _I],
    }
    for name, args in sigs.items():
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = args
    lib.lsd_last_error.restype = ctypes.c_char_p
    lib.lsd_last_error.argtypes = [_V]
    lib.lsd_ensemble_last_error.restype = ctypes.c_char_p
    lib.lsd_ensemble_last_error.argtypes = [_V]
    _LIB = lib
    return lib


def tune_candidates(cfg):
    """lsd_tune_candidates: the autotuner's candidate lists for cfg (no device work)"""
    sp = capi.LsdTuneSpace()
    rc = load_library().lsd_tune_candidates(ctypes.byref(cfg), ctypes.byref(sp))
    if rc:
        raise LsdError(rc, "lsd_tune_candidates")
    return {"fft": [(sp.fft_E[i], sp.fft_G[i]) for i in range(sp.nfft)],
            "gemm": [(sp.gemm_stages[i], sp.gemm_ctas[i]) for i in range(sp.ngemm)],
            "solve_threads": [sp.solve_threads[i] for i in range(sp.nsolve)]}


def tune_choose(ms, dflt=0):
    """lsd_tune_choose: the selection rule on candidate timings ms"""
    a = (ctypes.c_double * len(ms))(*ms)
    return load_library().lsd_tune_choose(len(ms), a, int(dflt))


def tim_check_cgce(cfg, state):
    """tim_check_cgce (timestep.F90:744-830) through the C ABI on a capi.LsdPcState (updated
    in place); returns the status (LSD_OK or LSD_ENOTCONVERGED).  Host only."""
    return load_library().lsd_tim_check_cgce(ctypes.byref(cfg), ctypes.byref(state))


def tim_new_tstep(cfg, state):
    """tim_new_tstep (timestep.F90:837-870) through the C ABI; returns tim_new_dt."""
    nd = ctypes.c_int(0)
    rc = load_library().lsd_tim_new_tstep(ctypes.byref(cfg), ctypes.byref(state), ctypes.byref(nd))
    if rc:
        raise LsdError(rc, "lsd_tim_new_tstep")
    return bool(nd.value)


def exported_symbols():
    """Names of the C entry points declared in include/lsd_b200.h."""
    hdr = os.path.join(os.path.dirname(_HERE), "include", "lsd_b200.h")
    names = []
    import re
    for line in open(hdr):
        m = re.match(r"\s*(?:int|const char\*)\s+(lsd_\w+)\s*\(", line)
        if m:
            names.append(m.group(1))
    return names


def _dp(a):
    return a.ctypes.data_as(_D)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class Context:
    """One simulation context on one GPU (the reference's module state of one run)."""

    def __init__(self, cfg, _handle=None):
        self.lib = load_library()
        self.owned = _handle is None
        if _handle is None:
            h = _V()
            rc = self.lib.lsd_create(ctypes.byref(cfg), ctypes.byref(h))
            if rc != 0:
                msg = self.lib.lsd_last_error(None)
                raise LsdError(rc, "lsd_create: " + (msg.decode() if msg else ""))
        else:
            h = _handle
        self.h = h
        self.cfg = cfg
        s = capi.LsdSizes()
        self._ok(self.lib.lsd_get_sizes(self.h, ctypes.byref(s)))
        self.sizes = {k: getattr(s, k) for k, _ in capi.LsdSizes._fields_}
        self.H, self.N, self.Th, self.Th2, self.Ph = (self.sizes[k] for k in ("H", "N", "Th", "Th2", "Ph"))

    def _ok(self, rc):
        if rc != 0:
            msg = self.lib.lsd_last_error(self.h)
            raise LsdError(rc, msg.decode() if msg else "")
        return rc

    def close(self):
        if getattr(self, "h", None):
            if self.owned:
                self.lib.lsd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- layout / tables
    def harmonics(self):
        l, m, s = (np.zeros(self.H, np.int32) for _ in range(3))
        I = ctypes.POINTER(ctypes.c_int)
        self._ok(self.lib.lsd_harmonics(self.h, l.ctypes.data_as(I), m.ctypes.data_as(I), s.ctypes.data_as(I)))
        return l, m, s

    def theta_map(self):
        t = np.zeros(2 * self.sizes["Hc"], np.int32)
        self._ok(self.lib.lsd_theta_map(self.h, t.ctypes.data_as(ctypes.POINTER(ctypes.c_int))))
        return t

    def radial_grid(self):
        r = np.zeros(self.N)
        self._ok(self.lib.lsd_radial_grid(self.h, _dp(r)))
        return r

    def radial_weights(self):
        r = np.zeros(self.N)
        self._ok(self.lib.lsd_radial_weights(self.h, _dp(r)))
        return r

    def gauss(self):
        gp, gw = np.zeros(self.Th), np.zeros(self.Th)
        self._ok(self.lib.lsd_gauss(self.h, _dp(gp), _dp(gw)))
        return gp, gw

    def legendre_table(self, which):
        t = np.zeros((self.H, self.Th2))
        self._ok(self.lib.lsd_legendre_table(self.h, which, _dp(t)))
        return t.T.copy()

    # ---- state (coll (H, N))
    def rows(self, field):
        """radial points of a field: Nic for the inner core's (MAG_IC_*), N otherwise"""
        return self.cfg.Nic if field in (capi.MAG_IC_TOR, capi.MAG_IC_POL) else self.N

    def set_coll(self, field, re, im):
        re, im = _c(re), _c(im)
        n = self.rows(field)
        assert re.size == self.H * n and im.size == self.H * n
        self._ok(self.lib.lsd_set_coll(self.h, field, _dp(re), _dp(im)))

    def stage_coll(self, field, re, im):
        """lsd_stage_coll: enqueue the upload of one field (keep re, im alive and unchanged
        until a later waiting call -- step, energies, get_coll -- has returned after the commit)."""
        n = self.rows(field)
        assert re.size == self.H * n and im.size == self.H * n
        assert re.flags["C_CONTIGUOUS"] and im.flags["C_CONTIGUOUS"]
        self._ok(self.lib.lsd_stage_coll(self.h, field, _dp(re), _dp(im)))

    def stage_fields(self, fields):
        for f, (re, im) in fields.items():
            self.stage_coll(f, re, im)

    def commit_staged(self):
        """lsd_commit_staged: the staged fields become the state."""
        self._ok(self.lib.lsd_commit_staged(self.h))

    def get_coll(self, field):
        n = self.rows(field)
        re, im = np.zeros((self.H, n)), np.zeros((self.H, n))
        self._ok(self.lib.lsd_get_coll(self.h, field, _dp(re), _dp(im)))
        return re, im

    def get_nonlinear(self, which):
        re, im = np.zeros((self.H, self.N)), np.zeros((self.H, self.N))
        self._ok(self.lib.lsd_get_nonlinear(self.h, which, _dp(re), _dp(im)))
        return re, im

    def set_time(self, t, dt):
        self._ok(self.lib.lsd_set_time(self.h, float(t), float(dt)))

    def get_time(self):
        t, dt, st = ctypes.c_double(), ctypes.c_double(), ctypes.c_int()
        self._ok(self.lib.lsd_get_time(self.h, ctypes.byref(t), ctypes.byref(dt), ctypes.byref(st)))
        return t.value, dt.value, st.value

    # ---- transforms (transform.fftw3.F90)
    def tra_spec2phys(self, sre, sim):
        p = np.zeros((self.N, self.Ph, self.Th))
        self._ok(self.lib.lsd_tra_spec2phys(self.h, _dp(_c(sre)), _dp(_c(sim)), _dp(p)))
        return p

    def tra_phys2spec(self, p):
        sre, sim = np.zeros((self.N, self.H)), np.zeros((self.N, self.H))
        self._ok(self.lib.lsd_tra_phys2spec(self.h, _dp(_c(p)), _dp(sre), _dp(sim)))
        return sre, sim

    def tra_qst2rtp(self, q, s, t):
        outs = [np.zeros((self.N, self.Ph, self.Th)) for _ in range(3)]
        ins = [_c(x) for x in (q[0], q[1], s[0], s[1], t[0], t[1])]
        self._ok(self.lib.lsd_tra_qst2rtp(self.h, *[_dp(a) for a in ins], *[_dp(o) for o in outs]))
        return outs

    def tra_rtp2qst(self, r, th, ph):
        outs = [np.zeros((self.N, self.H)) for _ in range(6)]
        ins = [_c(x) for x in (r, th, ph)]
        self._ok(self.lib.lsd_tra_rtp2qst(self.h, *[_dp(a) for a in ins], *[_dp(o) for o in outs]))
        return (outs[0], outs[1]), (outs[2], outs[3]), (outs[4], outs[5])

    def tra_grad(self, sre, sim):
        t, p = np.zeros((self.N, self.Ph, self.Th)), np.zeros((self.N, self.Ph, self.Th))
        self._ok(self.lib.lsd_tra_grad(self.h, _dp(_c(sre)), _dp(_c(sim)), _dp(t), _dp(p)))
        return t, p

    def tra_dth(self, sre, sim):
        p = np.zeros((self.N, self.Ph, self.Th))
        self._ok(self.lib.lsd_tra_dth(self.h, _dp(_c(sre)), _dp(_c(sim)), _dp(p)))
        return p

    def tra_qst2rtp_vel(self, q, s, t, qr, sr, tr):
        """tra_qst2rtp_vel: -> r, th, ph, dur, qv1, dutr, dupr, qv2."""
        outs = [np.zeros((self.N, self.Ph, self.Th)) for _ in range(8)]
        ins = [_c(x) for pair in (q, s, t, qr, sr, tr) for x in pair]
        self._ok(self.lib.lsd_tra_qst2rtp_vel(self.h, *[_dp(a) for a in ins], *[_dp(o) for o in outs]))
        return outs

    def set_rotation(self, omega):
        """lsd_set_rotation: the inner core's rotation rate rot_omega."""
        self._ok(self.lib.lsd_set_rotation(self.h, float(omega)))

    def rotation(self):
        """lsd_get_rotation: rot_omega, rot_velTorq, rot_magTorq."""
        out = np.zeros(3)
        self._ok(self.lib.lsd_get_rotation(self.h, _dp(out)))
        return out

    def dt_control(self):
        """tim_dt, tim_corr_dt, tim_cfl_dt (io.F90:2346)."""
        out = np.zeros(3)
        self._ok(self.lib.lsd_get_dt_control(self.h, _dp(out)))
        return out

    # ---- anelastic reference state (io.F90:559-608)
    def set_reference_state(self, prof):
        """prof: (7, N) rho, xi, dxi/dr, T, dT/dr, eta, deta/dr (planet_model.txt.in)."""
        prof = np.ascontiguousarray(prof, dtype=np.float64)
        if prof.shape != (7, self.N):
            raise ValueError("reference state must be (7, N)")
        self._ok(self.lib.lsd_set_reference_state(self.h, _dp(prof)))

    # ---- time stepping (main.F90:100-164)
    def matrices(self):
        self._ok(self.lib.lsd_matrices(self.h))

    def nonlinear(self):
        self._ok(self.lib.lsd_nonlinear(self.h))

    def predictor(self):
        self._ok(self.lib.lsd_predictor(self.h))

    def corrector(self):
        d = ctypes.c_double()
        self._ok(self.lib.lsd_corrector(self.h, ctypes.byref(d)))
        return d.value

    def step(self, nsteps=1):
        st = capi.LsdStats()
        self._ok(self.lib.lsd_step(self.h, int(nsteps), ctypes.byref(st)))
        return st

    def energies(self):
        e = np.zeros(capi.NENERGY)
        self._ok(self.lib.lsd_energies(self.h, _dp(e)))
        return dict(zip(capi.ENERGY_NAMES, e))

    def diagnostics(self):
        """lsd_diagnostics: (scalars {name: value}, spectra {name: array}, profiles {name: array})."""
        L, M, N = (self.sizes[k] for k in ("L", "M", "N"))
        sc = np.zeros(capi.NDIAG)
        sp = np.zeros(capi.spectra_size(L, M))
        pr = np.zeros((len(capi.PROFILE_NAMES), N))
        self._ok(self.lib.lsd_diagnostics(self.h, _dp(sc), _dp(sp), _dp(pr)))
        return (dict(zip(capi.DIAG_NAMES, sc)), capi.split_spectra(sp, L, M),
                dict(zip(capi.PROFILE_NAMES, pr)))

    def energies_static(self):
        """lsd_energies_static: the same diagnostics with a static device scratch (no allocation)."""
        e = np.zeros(capi.NENERGY)
        self._ok(self.lib.lsd_energies_static(self.h, _dp(e)))
        return dict(zip(capi.ENERGY_NAMES, e))

    # ---- device-resident work (pointers from torch / cuda-python allocations)
    def sht_synth_device(self, nbatch, d_spec, d_phys):
        self._ok(self.lib.lsd_sht_synth_device(self.h, int(nbatch), _V(d_spec), _V(d_phys)))

    def sht_analys_device(self, nbatch, d_phys, d_spec):
        self._ok(self.lib.lsd_sht_analys_device(self.h, int(nbatch), _V(d_phys), _V(d_spec)))

    def banded_factor_device(self, n, kl, nmat, d_ab, d_ipiv, d_info):
        self._ok(self.lib.lsd_banded_factor_device(self.h, n, kl, nmat, _V(d_ab), _V(d_ipiv), _V(d_info)))

    def banded_solve_device(self, n, kl, nmat, d_ab, d_ipiv, nrhs, d_map, d_b):
        self._ok(self.lib.lsd_banded_solve_device(self.h, n, kl, nmat, _V(d_ab), _V(d_ipiv), nrhs, _V(d_map), _V(d_b)))

    def tuning(self):
        """the context's launch parameters (lsd_get_tuning) as a dict"""
        t = capi.LsdTuning()
        self._ok(self.lib.lsd_get_tuning(self.h, ctypes.byref(t)))
        return {k: getattr(t, k) for k, _ in capi.LsdTuning._fields_ if k != "reserved"}

    def set_tuning(self, **kw):
        """change launch parameters (lsd_set_tuning); unspecified ones keep their values"""
        t = capi.LsdTuning()
        self._ok(self.lib.lsd_get_tuning(self.h, ctypes.byref(t)))
        for k, v in kw.items():
            setattr(t, k, v)
        self._ok(self.lib.lsd_set_tuning(self.h, ctypes.byref(t)))

    def stream(self):
        """the context's CUDA stream handle (int), e.g. for torch.cuda.ExternalStream"""
        v = _V()
        self._ok(self.lib.lsd_get_stream(self.h, ctypes.byref(v)))
        return v.value or 0

    def operator_solve_device(self, fields, d_data):
        """lsd_operator_solve_device: the context's operators applied in place to
        len(fields) consecutive device fields [N][H] complex at d_data (one launch)."""
        f = (ctypes.c_int * len(fields))(*fields)
        self._ok(self.lib.lsd_operator_solve_device(self.h, len(fields), f, _V(d_data)))

    PHASES = ["spectral_prep", "synthesis", "fft_products", "analysis", "spectral_tail",
              "predictor_solve", "corrector_solve"]

    def profile_phases(self):
        """Device milliseconds of the phases of one full step (it advances the state)."""
        ms = np.zeros(7)
        n = ctypes.c_int(7)
        self._ok(self.lib.lsd_profile_phases(self.h, _dp(ms), ctypes.byref(n)))
        return dict(zip(self.PHASES, ms))

    def selftest(self, which=0):
        r = ctypes.c_double(-1.0)
        self._ok(self.lib.lsd_selftest(self.h, int(which), ctypes.byref(r)))
        return r.value

    def synchronize(self):
        self._ok(self.lib.lsd_synchronize(self.h))

    def last_elapsed_ms(self):
        d = ctypes.c_double()
        self._ok(self.lib.lsd_last_elapsed_ms(self.h, ctypes.byref(d)))
        return d.value

    def kernel_launches(self):
        n = ctypes.c_longlong()
        self._ok(self.lib.lsd_kernel_launches(self.h, ctypes.byref(n)))
        return n.value

    # ---- convenience
    def load_fields(self, fields):
        for f, (re, im) in fields.items():
            self.set_coll(f, re, im)


class Ensemble:
    """n independent runs (their own configurations and resolutions) on one GPU, stepped
    together by one graph launch whose branches are the members' step loops
    (lsd_ensemble_*).  members[i] is a Context view of run i (set_coll,
    set_reference_state, energies, ...)."""

    def __init__(self, cfgs):
        self.lib = load_library()
        arr = (capi.LsdConfig * len(cfgs))(*cfgs)
        h = _V()
        rc = self.lib.lsd_ensemble_create(len(cfgs), arr, ctypes.byref(h))
        if rc != 0:
            raise LsdError(rc, "lsd_ensemble_create failed")
        self.h = h
        self.members = []
        for i, cfg in enumerate(cfgs):
            m = _V()
            self._ok(self.lib.lsd_ensemble_member(self.h, i, ctypes.byref(m)))
            self.members.append(Context(cfg, _handle=m))

    def _ok(self, rc):
        if rc != 0:
            msg = self.lib.lsd_ensemble_last_error(self.h)
            raise LsdError(rc, msg.decode() if msg else "")
        return rc

    def last_elapsed_ms(self):
        """device time of the last step() call's graph launch"""
        d = ctypes.c_double()
        self._ok(self.lib.lsd_ensemble_last_elapsed_ms(self.h, ctypes.byref(d)))
        return d.value

    def step(self, nsteps=1):
        st = (capi.LsdStats * len(self.members))()
        self._ok(self.lib.lsd_ensemble_step(self.h, int(nsteps), st))
        return list(st)

    def close(self):
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None
            self.lib.lsd_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
