"""Argument and configuration checks of the C ABI, on any machine (no device is touched).

* lsd_create refuses each configuration outside the reference's own parameter rules
  (par_precompute: L > (M-1) Mp, M even) or this library's scope with LSD_EARG and the
  reason, before it looks for a device; a valid configuration gets past these checks
  (LSD_ECUDA when the machine has no GPU).
* The entry points given a null context return LSD_EARG.
"""
import ctypes
import importlib

import pytest

pkg = importlib.import_module("leeds-code_b200")
capi = pkg.capi

BAD = [
    (dict(L=1), "bad resolution"),
    (dict(M=1), "bad resolution"),
    (dict(Mp=0), "bad resolution"),
    (dict(KL=1), "bad resolution"),
    (dict(KL=9), "bad resolution"),
    (dict(KL=7), "KL = 2..6"),
    (dict(N=7, KL=3), "bad resolution"),
    (dict(L=60, M=16, Mp=4), "set L > (M-1)*Mp"),
    (dict(L=64, M=15, Mp=4), "M even"),
    (dict(Nic=0), "Nic must be >= 1"),
    (dict(Nic=5, KL=3), "2 KL + 1 <= Nic <= N"),
    (dict(Nic=65, N=64), "2 KL + 1 <= Nic <= N"),
    (dict(Nic=17, boussinesq=0), "Boussinesq"),
    (dict(Nic=17, vel_bc=3), "no-slip inner wall"),
    (dict(rot_tstep=1, boussinesq=0), "Boussinesq"),
    (dict(timestep=0.0), "d_timestep"),
    (dict(mag_tstep=0), "must all be stepped"),
    (dict(precision=7), "unknown precision"),
    (dict(precision=capi.PREC_OZAKI, ozaki_slices=1), "ozaki_slices"),
]


def create(cfg):
    lib = pkg.load_library()
    h = ctypes.c_void_p()
    rc = lib.lsd_create(ctypes.byref(cfg), ctypes.byref(h))
    return lib, rc, h


@pytest.mark.parametrize("over,why", BAD, ids=[str(o) for o, _ in BAD])
def test_create_rejects(over, why):
    cfg = capi.template_config(**over)
    with pytest.raises(pkg.LsdError) as e:
        pkg.Context(cfg)
    assert e.value.status == capi.LSD_EARG
    assert why in str(e.value), str(e.value)


def test_create_accepts_valid_configuration():
    import torch
    cfg = capi.template_config()
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: creation would proceed")
    lib, rc, h = create(cfg)
    assert rc == capi.LSD_ECUDA and not h.value


def test_null_arguments():
    lib = pkg.load_library()
    assert lib.lsd_create(None, None) == capi.LSD_EARG
    cfg = capi.template_config()
    assert lib.lsd_create(ctypes.byref(cfg), None) == capi.LSD_EARG
    z = ctypes.c_void_p()
    d = ctypes.c_double()
    assert lib.lsd_set_coll(z, 0, None, None) == capi.LSD_EARG
    assert lib.lsd_get_coll(z, 0, None, None) == capi.LSD_EARG
    assert lib.lsd_stage_coll(z, 0, None, None) == capi.LSD_EARG
    assert lib.lsd_commit_staged(z) == capi.LSD_EARG
    assert lib.lsd_step(z, 1, None) == capi.LSD_EARG
    assert lib.lsd_energies(z, ctypes.byref(d)) == capi.LSD_EARG
    assert lib.lsd_energies_static(z, ctypes.byref(d)) == capi.LSD_EARG
    assert lib.lsd_diagnostics(z, ctypes.byref(d), None, None) == capi.LSD_EARG
    assert lib.lsd_set_time(z, ctypes.c_double(0.0), ctypes.c_double(1e-5)) == capi.LSD_EARG
    assert lib.lsd_set_rotation(z, ctypes.c_double(1.0)) == capi.LSD_EARG
    assert lib.lsd_synchronize(z) == capi.LSD_EARG
