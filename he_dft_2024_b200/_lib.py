"""ctypes binding of libhedft.so (include/he_dft.h).

The library is required: importing the binding without it, or calling into it without a CUDA
device, raises.  There is no fallback implementation of any routine.
"""
import ctypes
import os
import re

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
LIB_PATH = os.path.join(PKG, "libhedft.so")
HEADER = os.path.join(ROOT, "include", "he_dft.h")

HE_OK, HE_ERR_ARG, HE_ERR_CUDA, HE_ERR_STATE, HE_ERR_NOMEM = 0, 1, 2, 3, 4
HE_MODE_DYNAMICS, HE_MODE_STATICS, HE_MODE_QUANTUM = 0, 1, 2
HE_MAX_QIMP = 4
HE_PREC_F64, HE_PREC_MIXED = 0, 1

FIELDS = dict(
    psi=0, den=1, pot4=2, dencg=3, delj4=4, uimp=5, fden=6, pc=7, q=8, psiold1=9, psiold2=10,
    psiold3=11, hpsiold1=12, hpsiold2=13, dxden=14, dyden=15, dzden=16, hpsi=17, fvlj4=18,
    wcgk=19, rimp=20, vimp=21, aimp=22, F=23, rimpold=24, vimpold=25, aimpold=26, pcr=27, pcv=28,
    qr=29, qv=30, ring=31, psix=32, upotx=33, potx4=34, denx=35, pcx=36, qx=37, psixold=38,
    hpsixold=39, uimpk=40, uimpkk=41, denalf=42, falfs=43, intxalf=44, intyalf=45, intzalf=46,
    ualphas=47, kalfs=48)


class HeGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("xmax", ctypes.c_double), ("ymax", ctypes.c_double), ("zmax", ctypes.c_double),
                ("npd", ctypes.c_int), ("icon", ctypes.c_int)]


class HeFunctional(ctypes.Structure):
    _fields_ = [("core4", ctypes.c_char * 4),
                ("h4", ctypes.c_double), ("eps4", ctypes.c_double), ("sigma4", ctypes.c_double),
                ("cp4", ctypes.c_double), ("cpp4", ctypes.c_double), ("den4c", ctypes.c_double),
                ("alphas", ctypes.c_double), ("l", ctypes.c_double), ("den0s", ctypes.c_double),
                ("h2o2m4", ctypes.c_double), ("lsolid", ctypes.c_int),
                ("C", ctypes.c_double), ("beta", ctypes.c_double), ("den_m", ctypes.c_double)]


class HeAbsorber(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("lambdah", "txmean", "txsurf", "tymean", "tysurf", "tzmean", "tzsurf")]


class HeImpurities(ctypes.Structure):
    _fields_ = [("n_imp", ctypes.c_int),
                ("m_imp_u", ctypes.POINTER(ctypes.c_double)),
                ("potion", ctypes.POINTER(ctypes.c_double)),
                ("npot", ctypes.c_int),
                ("delinter", ctypes.c_double), ("rmaxinterpol", ctypes.c_double),
                ("ii_kind", ctypes.c_int),
                ("ii_D", ctypes.c_double), ("ii_re", ctypes.c_double), ("ii_a", ctypes.c_double),
                ("ii_rcut", ctypes.c_double), ("ii_umax", ctypes.c_double)]


class HePairPot(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("D", ctypes.c_double), ("re", ctypes.c_double),
                ("a", ctypes.c_double), ("rcut", ctypes.c_double), ("umax", ctypes.c_double)]


class HeQImpurities(ctypes.Structure):
    _fields_ = [("n_imp", ctypes.c_int),
                ("m_imp_u", ctypes.POINTER(ctypes.c_double)),
                ("mu4", ctypes.c_double),
                ("he_x", HePairPot * HE_MAX_QIMP),
                ("x_x", HePairPot * (HE_MAX_QIMP * HE_MAX_QIMP)),
                ("uimp_k", ctypes.POINTER(ctypes.c_double)),
                ("uimp_k_k", ctypes.POINTER(ctypes.c_double)),
                ("n_spline", ctypes.c_int), ("nq", ctypes.c_int), ("parabolic", ctypes.c_int)]


class HeEnergies(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in
                ("etot4", "ekin4", "elj4", "ecor4", "esolid", "ealphas", "ekinx", "eHeX",
                 "eimpu_impu", "eimpu", "etot")]


class HeKernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 40), ("launches", ctypes.c_longlong),
                ("ms", ctypes.c_double)]


class HeError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"he_dft status {status}: {msg}")
        self.status = status


def header_functions():
    """Names of the functions declared in include/he_dft.h."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(he_[a-z0-9_]+)\s*\(", src)))


_lib = None


def load():
    """Load libhedft.so (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: run `python -m he_dft_2024_b200.build` "
                          "(or __graft_entry__.build()) first")
    L = ctypes.CDLL(LIB_PATH)
    vp, ip, dp = ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_double)
    d = ctypes.c_double
    sig = {
        "he_ctx_create": (ip, [ctypes.POINTER(HeGrid), ctypes.POINTER(HeFunctional), ip, ip,
                               ctypes.POINTER(vp)]),
        "he_ctx_destroy": (None, [vp]),
        "he_last_error": (ctypes.c_char_p, [vp]),
        "he_launch_count": (ctypes.c_longlong, [vp]),
        "he_device_bytes": (ctypes.c_size_t, [vp]),
        "he_set_stream": (ip, [vp, vp]),
        "he_synchronize": (ip, [vp]),
        "he_set_kernels": (ip, [vp, dp, dp, dp]),
        "he_compute_kernels": (ip, [vp]),
        "he_set_absorber": (ip, [vp, ctypes.POINTER(HeAbsorber)]),
        "he_set_impurities": (ip, [vp, ctypes.POINTER(HeImpurities)]),
        "he_upload": (ip, [vp, ip, vp, ctypes.c_size_t]),
        "he_download": (ip, [vp, ip, vp, ctypes.c_size_t]),
        "he_poten": (ip, [vp]),
        "he_potenimp": (ip, [vp]),
        "he_lstopimp": (ip, [vp, ctypes.POINTER(ip)]),
        "he_forceimp": (ip, [vp, dp]),
        "he_set_accel": (ip, [vp]),
        "he_steprk": (ip, [vp, d]),
        "he_steppc": (ip, [vp, d, dp, dp, dp]),
        "he_energy": (ip, [vp, ctypes.POINTER(HeEnergies)]),
        "he_derden": (ip, [vp]),
        "he_refresh_density": (ip, [vp]),
        "he_evolo0": (ip, [vp, dp, dp, ip]),
        "he_steprkr": (ip, [vp, d, dp, dp, ip]),
        "he_steppcr": (ip, [vp, d, dp, dp, ip, dp]),
        "he_statics_iterations": (ip, [vp, ip, d, dp, dp, ip, dp]),
        "he_varmu": (ip, [vp, ip, d, dp]),
        "he_timing": (ip, [vp, ip]),
        "he_tuned_tiles": (ip, [vp, ctypes.POINTER(ip), ctypes.POINTER(ip), ctypes.POINTER(ip)]),
        "he_autotune_report": (ip, [vp, ctypes.c_char_p, ctypes.c_size_t]),
        "he_set_fft_variant": (ip, [vp, ip, ip, ip]),
        "he_state_fingerprint": (ip, [vp, ctypes.POINTER(ctypes.c_ulonglong)]),
        "he_join": (ip, [vp]),
        "he_timing_report": (ip, [vp, ctypes.POINTER(HeKernelTime), ip, ctypes.POINTER(ip)]),
        "he_set_quantum_impurities": (ip, [vp, ctypes.POINTER(HeQImpurities)]),
        "he_qimp_moments": (ip, [vp, dp]),
        "he_observables": (ip, [vp, ip, dp]),
        "he_ft_v_spline_table": (ip, [ctypes.POINTER(HePairPot), d, d, ip, ip, dp, ip,
                                      ctypes.c_char_p, ctypes.c_size_t]),
        "he_ctx_group": (ip, [ctypes.POINTER(vp), ip]),
        "he_group_size": (ip, [vp]),
        "he_upload_member": (ip, [vp, ip, ip, vp, ctypes.c_size_t]),
        "he_download_member": (ip, [vp, ip, ip, vp, ctypes.c_size_t]),
        "he_member_mu": (ip, [vp, ip, ip, dp]),
        "he_statics_iterations_members": (ip, [vp, ip, d, ip, dp, dp, dp]),
        "he_energy_members": (ip, [vp, ctypes.POINTER(HeEnergies)]),
        "he_qimp_moments_members": (ip, [vp, dp]),
        "he_energy_noalloc": (ip, [ctypes.POINTER(HeGrid), ctypes.POINTER(HeFunctional), ip, vp,
                                   vp, vp, vp, vp, vp, ctypes.POINTER(HeEnergies),
                                   ctypes.c_char_p, ctypes.c_size_t]),
    }
    for name, (res, args) in sig.items():
        f = getattr(L, name)
        f.restype = res
        f.argtypes = args
    _lib = L
    return L


def dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
