"""ctypes mirror of include/lsd_b200.h (the C ABI of liblsd_b200.so).

The structures and constants here are the Python view of the C header; the header is
the source of truth.  Nothing in this module computes: it only describes the ABI.
"""
import ctypes

LSD_OK = 0
LSD_EARG = 1
LSD_ECUDA = 2
LSD_ESINGULAR = 3
LSD_ENOTCONVERGED = 4
LSD_ENONFINITE = 5
LSD_ESTATE = 6
LSD_ENOMEM = 7

STATUS_NAMES = {
    0: "ok", 1: "bad argument", 2: "CUDA error", 3: "singular banded operator",
    4: "corrector did not converge", 5: "non-finite state", 6: "call out of order",
    7: "device allocation failed",
}

VEL_TOR, VEL_POL, COD_C, MAG_TOR, MAG_POL, COMP_C = range(6)
MAG_IC_TOR, MAG_IC_POL = 6, 7  # the conducting inner core's field, (H, Nic) arrays
FIELD_NAMES = ["vel_Tor", "vel_Pol", "cod_C", "mag_Tor", "mag_Pol", "comp_C"]
N_VEL_TOR, N_VEL_POL, N_COD, N_MAG_TOR, N_MAG_POL, N_COMP = range(6)

(LEG_P, LEG_P_, LEG_SIN1MP, LEG_LLP_, LEG_LLSIN1MP, LEG_GWP, LEG_GWLLP_,
 LEG_GWLLSIN1MP) = range(8)
LEG_NAMES = ["P", "P_", "sin1mP", "llP_", "llsin1mP", "gwP", "gwllP_", "gwllsin1mP"]

PREC_FP64 = 0
PREC_OZAKI = 1

ENERGY_NAMES = [
    "time", "KE", "KE_tor", "KE_sym", "KE_l1", "KE_tm0", "KE_dis", "KE_ax",
    "ME", "ME_tor", "ME_sym", "ME_l1", "ME_tm0", "ME_dis", "dipole", "quadrupole",
    "ME_ax", "topflx", "botflx",
]
NENERGY = len(ENERGY_NAMES)

# lsd_diagnostics scalars (LSD_D_* order of the header)
DIAG_NAMES = (
    ["time"]
    + ["vel_" + k for k in ("Et", "Ep", "Etas", "Epas", "Etes", "Epes", "Etesas", "Epesas", "l_Eofl", "lpol")]
    + ["mag_" + k for k in ("Et", "Ep", "Etas", "Epas", "Etes", "Epes", "Etesas", "Epesas")]
    + ["cmb_" + k for k in ("EPol", "ESym", "El1", "theta", "phi", "Epas", "El12")]
    + ["nus_" + k for k in ("Nu", "T_ro", "T_ri", "dCdr_ri", "dCdr_ro", "Nu_top", "Nu_bot", "Nu_flux")]
    + ["nuscomp_" + k for k in ("Nu", "T_ro", "T_ri", "dCdr_ri", "dCdr_ro", "Nu_top", "Nu_bot", "Nu_flux")]
    + ["Rm", "Re", "Pe", "Pe_comp", "Rossby", "M_ratio", "Elsasser", "Lehnert", "fdip", "fohm", "theta_dip",
       "Nusselt", "Sherwood"]
    + ["tim_dt", "tim_corr_dt", "tim_cfl_dt"]
    + ["rot_omega", "rot_velTorq", "rot_magTorq"]
    + ["ic_" + k for k in ("E", "Et", "Esym", "El1", "ETm0", "EDis", "Dip", "Quad", "Eaxtot")]
    + ["icpart_" + k for k in ("Et", "Ep", "Etas", "Epas", "Etes", "Epes", "Etesas", "Epesas")]
)
NDIAG = len(DIAG_NAMES)
PROFILE_NAMES = ["r", "vel_E", "vel_Epol", "vel_Etor", "mag_E", "mag_Epol", "mag_Etor",
                 "temp_C", "temp_dCdr", "comp_C", "comp_dCdr"]


def spectra_size(L, M):
    """doubles of the lsd_diagnostics spectra buffer"""
    return 8 * (L + M)


def split_spectra(buf, L, M):
    """lsd_diagnostics spectra -> {name: array}: vel_l / vel_m / mag_l / mag_m are
    (L or M, 3) arrays of E, Epol, Etor; cod_l / cod_m / comp_l / comp_m are E."""
    out, o = {}, 0
    for f in ("vel", "mag"):
        out[f + "_l"] = buf[o:o + 3 * L].reshape(L, 3); o += 3 * L
        out[f + "_m"] = buf[o:o + 3 * M].reshape(M, 3); o += 3 * M
    for f in ("cod", "comp"):
        out[f + "_l"] = buf[o:o + L]; o += L
        out[f + "_m"] = buf[o:o + M]; o += M
    return out


class LsdConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "L", "M", "Mp", "N", "Nic", "KL",
        "vel_bc", "cod_bc", "comp_bc", "time_step_control",
        "boussinesq", "vel_tstep", "cod_tstep", "comp_tstep", "mag_tstep",
        "precision", "device", "ozaki_slices")] + \
        [(n, ctypes.c_double) for n in (
            "rratio", "alpha", "Ra", "Ra_comp", "Pr", "Sc", "Pm", "E", "Hyp",
            "implicit", "timestep", "dterr", "courant", "corr_upper", "corr_lower",
            "source", "source_comp", "qi", "qo", "qi_comp", "qo_comp")] + \
        [("rot_tstep", ctypes.c_int), ("rot_force_0", ctypes.c_int), ("autotune", ctypes.c_int),
         ("reserved", ctypes.c_int * 5)]


class LsdSizes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in
                ("H", "Th", "Th2", "Ph", "Ma", "Hc", "Hr", "N", "L", "M", "Mp", "KL")]


class LsdStats(ctypes.Structure):
    _fields_ = [("steps_done", ctypes.c_int), ("correctors", ctypes.c_int),
                ("evaluations", ctypes.c_int), ("kernel_launches", ctypes.c_int),
                ("last_dterr", ctypes.c_double), ("t", ctypes.c_double),
                ("dt", ctypes.c_double)]


class LsdTuning(ctypes.Structure):
    """lsd_tuning: the tunable launch parameters of a context"""
    _fields_ = [(n, ctypes.c_int) for n in ("tuned", "fft_E", "fft_G", "gemm_stages", "gemm_ctas_per_sm",
                                            "solve_threads")] + [("reserved", ctypes.c_int * 2)] + \
        [(n, ctypes.c_double) for n in ("ms_fft", "ms_gemm", "ms_solve")]


TUNE_MAX = 8


class LsdTuneSpace(ctypes.Structure):
    _fields_ = [("nfft", ctypes.c_int), ("fft_E", ctypes.c_int * TUNE_MAX), ("fft_G", ctypes.c_int * TUNE_MAX),
                ("ngemm", ctypes.c_int), ("gemm_stages", ctypes.c_int * TUNE_MAX),
                ("gemm_ctas", ctypes.c_int * TUNE_MAX), ("nsolve", ctypes.c_int),
                ("solve_threads", ctypes.c_int * TUNE_MAX)]


class LsdPcState(ctypes.Structure):
    """lsd_pc_state: tim_t, tim_dt, tim_dterr, tim_corr_dt, lasterr, tim_cfl_dt, tim_it,
    tim_step, tim_pcn of timestep.F90."""
    _fields_ = [(n, ctypes.c_double) for n in ("t", "dt", "dterr", "corr_dt", "lasterr", "cfl_dt")] + \
        [(n, ctypes.c_int) for n in ("it", "step", "pcn", "reserved")]


def template_config(**overrides):
    """The parameter values of Scripts/parameters.F90_template, then `overrides`."""
    c = LsdConfig()
    vals = dict(
        L=64, M=16, Mp=4, N=64, Nic=1, KL=3,
        vel_bc=1, cod_bc=1, comp_bc=1, time_step_control=2,
        boussinesq=1, vel_tstep=1, cod_tstep=1, comp_tstep=0, mag_tstep=1,
        precision=PREC_FP64, device=0, ozaki_slices=0,
        rratio=0.35, alpha=-1.0, Ra=6.5e4, Ra_comp=1.0, Pr=1.0, Sc=1.0, Pm=5.0,
        E=1.0e-3, Hyp=0.0, implicit=0.6, timestep=-5e-5, dterr=0.025,
        courant=float(ctypes.c_float(0.8).value), corr_upper=0.020, corr_lower=0.00200,
        source=0.0, source_comp=0.0, qi=0.0, qo=-1.0, qi_comp=0.0, qo_comp=-1.0,
    )
    vals.update(overrides)
    for k, v in vals.items():
        setattr(c, k, v)
    return c


def derived_sizes(L, M, Mp):
    """Sizes from parameters.F90_template:251-262 and parallel.h_template:54-62."""
    Ma = M * 3 // 2
    H = L * M - Mp * (M - 1) * M // 2
    Th = L * 3 // 2
    Th2 = (Th + 1) // 2
    Ph = Ma * 2
    Hc = (M + 1) // 2
    Hr = H // Hc
    return dict(H=H, Th=Th, Th2=Th2, Ph=Ph, Ma=Ma, Hc=Hc, Hr=Hr)
