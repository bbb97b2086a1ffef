"""Host-side state-file I/O in the reference's classic netCDF layout.

Reads and writes the `state.cdf` files of program/io.F90 (io_load_state :349-483,
io_save_state :1502-1621) with scipy.io.netcdf_file.  Coefficients are stored in the
file in plain m-major harmonic order (io_state_nh, io.F90:1258-1272) and in memory in
the reference's folded order (parallel.h_template:54-80); this module maps between the
two.  A file on another radial grid (a different N, or points more than 1e-8 apart,
io.F90:407-418) is interpolated onto the run's grid as io_interp_wts / io_interp do
(io.F90:1360-1431): both grids mapped onto [0, 1], a local polynomial through the 2 KL + 1
nearest file points.
"""
import numpy as np

from . import capi

STATE_VARS = ("uT", "uP", "C", "BT", "BP")
FIELD_OF_VAR = {"uT": capi.VEL_TOR, "uP": capi.VEL_POL, "C": capi.COD_C,
                "BT": capi.MAG_TOR, "BP": capi.MAG_POL, "Comp": capi.COMP_C}
# the inner core's field: declared on the outer core's r dimension, its first Nic radial
# entries written (io.F90:1594-1595, 1613-1614; read back with Nic rows, io.F90:445-446)
IC_FIELD_OF_VAR = {"icBT": capi.MAG_IC_TOR, "icBP": capi.MAG_IC_POL}


def folded_harmonics(L, M, Mp):
    """(l, m_, s) of every nh in the folded order of _loop_setlm (parallel.h_template:54-80)."""
    sz = capi.derived_sizes(L, M, Mp)
    Hc, Hr, H = sz["Hc"], sz["Hr"], sz["H"]
    l_ = np.zeros(H, np.int64)
    m_ = np.zeros(H, np.int64)
    nh = 0
    for j in range(1, Hc + 1):
        for i in range(1, Hr + 1):
            m = j - 1
            l = m * Mp + i - 1
            if l >= L:
                m = 2 * Hc - j
                l = L - Hr + i - 1
            l_[nh], m_[nh] = l, m * Mp
            nh += 1
    return l_, m_, (l_ + m_) % 2


def state_nh(l, m_, L, M, Mp):
    """io_state_nh (io.F90:1258-1272): file index of (l, m_), -1 when absent."""
    l = np.asarray(l)
    m_ = np.asarray(m_)
    ok = (m_ % Mp == 0) & (l < L) & (m_ < M * Mp)
    m = m_ // Mp
    nh = L * m - Mp * (m - 1) * m // 2 + l - m_
    return np.where(ok, nh, -1)


def interp_weights(xi, xo, KL):
    """io_interp_wts (io.F90:1360-1396): for every output point the file points l..r and
    the first row of the inverse Taylor matrix (the value's weights)."""
    xi = np.asarray(xi, dtype=np.float64)
    xo = np.asarray(xo, dtype=np.float64)
    xi1 = (xi - xi[0]) / (xi[-1] - xi[0])
    xo1 = (xo - xo[0]) / (xo[-1] - xo[0])
    out = []
    for x in xo1:
        j = 0
        while xi1[j] < x - 1e-8:
            j += 1
        lo, hi = max(0, j - KL), min(j + KL, len(xi) - 1)
        nn = hi - lo + 1
        A = np.ones((nn, nn))
        for c in range(1, nn):
            A[:, c] = A[:, c - 1] * (xi1[lo:hi + 1] - x) / c
        out.append((lo, hi, np.linalg.inv(A)[0]))
    return out


def interp_columns(a, w):
    """io_interp (io.F90:1402-1431) of every row of a (H, ni) onto the output points of w"""
    out = np.zeros((a.shape[0], len(w)))
    for n, (lo, hi, wt) in enumerate(w):
        out[:, n] = a[:, lo:hi + 1] @ wt
    return out


def load_state(path, L, M, Mp, N, r_expected=None, Nic=1, ric_expected=None, KL=3):
    """Return dict(field -> (re, im) arrays of shape (H, N)), t, dt, r.

    Modes of the run that are not in the file are zero (the reference fills them with
    uniform noise of amplitude d_init_pert from an unseeded generator, io.F90:1316-1324,
    which no run can reproduce).  With Nic > 1 the inner core's field (icBT, icBP) is
    returned too, arrays (H, Nic), when the file holds it (interpolated onto ric_expected
    when its grid differs); otherwise the run continues the outer core's field inward
    (synthetic.ic_extend, io.F90:440-443).  r is the file's grid."""
    from scipy.io import netcdf_file
    f = netcdf_file(path, "r", mmap=False)
    r = np.array(f.variables["r"].data, dtype=np.float64)
    ric = np.array(f.variables["icr"].data, dtype=np.float64) if "icr" in f.variables else np.zeros(1)
    # io.F90:407-418: interpolate when the sizes differ or the points are more than 1e-8 apart
    w_oc = w_ic = None
    if len(r) != N or (r_expected is not None and np.max(np.abs(r - r_expected)) > 1e-8):
        if r_expected is None:
            raise ValueError("state has %d radial points, run has %d: pass the run's grid" % (len(r), N))
        w_oc = interp_weights(r, r_expected, KL)
    nic_file = len(ric)
    ic_ok = Nic > 1 and nic_file > 1
    if ic_ok and (nic_file != Nic or (ric_expected is not None and np.max(np.abs(ric - ric_expected)) > 1e-8)):
        if ric_expected is None:
            raise ValueError("state has %d inner-core points, run has %d: pass the run's grid" % (nic_file, Nic))
        w_ic = interp_weights(ric, ric_expected, KL)
    l, m_, _ = folded_harmonics(L, M, Mp)
    out = {}
    for name, var in f.variables.items():
        if name in FIELD_OF_VAR:
            field, rows, nfile, w = FIELD_OF_VAR[name], N, len(r), w_oc
        elif name in IC_FIELD_OF_VAR and ic_ok:
            field, rows, nfile, w = IC_FIELD_OF_VAR[name], Nic, nic_file, w_ic
        else:
            continue
        a = var._attributes
        Lf, Mf, Mpf = int(a["L"]), int(a["M"]), int(a["Mp"])
        data = np.array(var.data, dtype=np.float64)  # (2, Hfile, N)
        idx = state_nh(l, m_, Lf, Mf, Mpf)
        re = np.zeros((len(l), nfile))
        im = np.zeros((len(l), nfile))
        ok = idx >= 0
        re[ok] = data[0, idx[ok], :nfile]
        im[ok] = data[1, idx[ok], :nfile]
        if w is not None:
            re, im = interp_columns(re, w), interp_columns(im, w)
        out[field] = (re, im)
    t = float(f._attributes.get("t", 0.0))
    dt = float(f.variables["dt"].data) if "dt" in f.variables else 0.0
    f.close()
    return out, t, dt, r


def load_rotation(path):
    """The inner core's rotation rate rot_omega of a state file ('icOmega', io.F90:431-432)."""
    from scipy.io import netcdf_file
    f = netcdf_file(path, "r", mmap=False)
    w = float(f.variables["icOmega"].data) if "icOmega" in f.variables else 0.0
    f.close()
    return w


def save_state(path, fields, L, M, Mp, r, ric, t, dt, attrs, omega=0.0):
    """Write a state file in the current layout of io_save_state (dims r, icr, H, ReIm).
    fields may hold the inner core's (MAG_IC_TOR / MAG_IC_POL, (H, Nic)); omega: rot_omega."""
    from scipy.io import netcdf_file
    l, m_, _ = folded_harmonics(L, M, Mp)
    H = len(l)
    idx = state_nh(l, m_, L, M, Mp)
    f = netcdf_file(path, "w", version=1)
    f.t = t
    for k, v in attrs.items():
        setattr(f, k, v)
    N = len(r)
    f.createDimension("r", N)
    f.createDimension("icr", len(ric))
    f.createDimension("H", H)
    f.createDimension("ReIm", 2)
    vr = f.createVariable("r", "d", ("r",))
    vr[:] = r
    vic = f.createVariable("icr", "d", ("icr",))
    vic[:] = ric
    vdt = f.createVariable("dt", "d", ())
    vdt[...] = dt  # a 0-d variable (assignValue fails on numpy 2 for these)
    vom = f.createVariable("icOmega", "d", ())
    vom[...] = omega
    inv = {v: k for k, v in FIELD_OF_VAR.items()}
    inv.update({v: k for k, v in IC_FIELD_OF_VAR.items()})
    for fld, (re, im) in fields.items():
        v = f.createVariable(inv[fld], "d", ("ReIm", "H", "r"))
        data = np.zeros((2, H, N))
        rows = re.shape[1]
        data[0, idx, :rows] = re
        data[1, idx, :rows] = im
        v[:] = data
        v.L, v.M, v.Mp = np.int32(L), np.int32(M), np.int32(Mp)
    f.close()
