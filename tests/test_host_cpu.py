"""Host-side checks that need no GPU: the C-ABI library loads and exports the header's symbols,
argument validation mirrors the reference's STOP conditions, and workload set-up logic."""
import ctypes
import json
import os

import numpy as np
import pytest

from he_dft_2024_b200 import _lib, config as C

HERE = os.path.dirname(os.path.abspath(__file__))
CONST = json.load(open(os.path.join(HERE, "golden", "constants.json")))


def test_library_exports_every_header_symbol():
    L = _lib.load()
    names = _lib.header_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_library_defines_every_kernel_it_launches():
    # the heavy kernels are compiled in their own translation units from the host objects'
    # undefined symbols; the linked library must leave none of the package's symbols undefined
    import shutil
    import subprocess
    if not shutil.which("nm"):
        pytest.skip("nm not available")
    lib = _lib.load()._name
    und = subprocess.run(["nm", "-u", "-C", lib], capture_output=True, text=True, check=True).stdout
    missing = [ln.strip() for ln in und.splitlines() if "he::" in ln]
    assert not missing, missing[:5]


def _create(nx=32, ny=32, nz=32, npd=13, icon=13, core=b"OT ", mode=0, den0s=0.04):
    L = _lib.load()
    g = _lib.HeGrid(nx, ny, nz, 10.0, 10.0, 10.0, npd, icon)
    f = _lib.HeFunctional(core, 2.190323, 10.22, 2.556, -2.41186e4, 1.8585e6, 0.062, 54.31, 1.0,
                          den0s, 6.05969638298, 1, 3.1577504e4, 40.0, 0.37)
    h = ctypes.c_void_p()
    st = L.he_ctx_create(ctypes.byref(g), ctypes.byref(f), mode, 0, ctypes.byref(h))
    msg = L.he_last_error(h.value).decode() if h.value else ""
    L.he_ctx_destroy(h.value)
    return st, msg


def test_tstgrid_sizes_enforced():
    # tstgrid.f90:9-13: the reference STOPs on 'NX is not correct'
    for n in (7, 11, 14, 22, 100 + 28):
        if n in CONST["tstgrid"]:
            continue
        st, msg = _create(nx=n)
        assert st == _lib.HE_ERR_ARG and "tstgrid" in msg


@pytest.mark.parametrize("kw,text", [
    (dict(npd=11), "npd"),
    (dict(icon=25), "icon"),
    (dict(core=b"XX "), "core4"),
    (dict(core=b"OTC", den0s=0.0), "den0s"),
    (dict(core=b"OTE"), "core4"),
    (dict(mode=7), "mode"),
    (dict(ny=1), "ny must be at least 2"),
])
def test_bad_arguments_rejected(kw, text):
    st, msg = _create(**kw)
    assert st == _lib.HE_ERR_ARG and text in msg


@pytest.mark.parametrize("shape", [(45, 32, 32), (27, 27, 27), (75, 45, 25)])
def test_odd_tstgrid_sizes_pass_validation(shape):
    # odd nx and odd ny*nz are admissible (tstgrid.f90:9-13); without a GPU the create then fails
    # at the device, not at the argument checks
    st, msg = _create(*shape)
    assert st != _lib.HE_ERR_ARG, msg


def test_no_cpu_fallback_without_device():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    st, msg = _create()
    assert st == _lib.HE_ERR_CUDA, msg


def test_potion_table_follows_potenimpini():
    w = C.tddft_1000()
    potion, npot, delinter, rmax = C.potion_table(w)
    assert npot == 100 * 128 + 1 and rmax == 160.0
    assert delinter == rmax / (npot - 1)
    r = np.arange(npot) * delinter
    e = 1 - np.exp(-0.8 * (r - 6.5))
    morse = 2.0 * (e * e - 1)
    # Select_Pot contract: r < r_cutoff gives umax (the capped Morse core, umax = V(r_cutoff))
    expect = np.where(r < C.MORSE_RCUT, C.MORSE_UMAX, morse)
    np.testing.assert_allclose(potion[0], expect, rtol=1e-15)
    assert C.MORSE_UMAX == pytest.approx(2.0 * ((1 - np.exp(-0.8 * (2.0 - 6.5))) ** 2 - 1))
    assert potion.shape == (1, npot)


def test_woods_saxon_normalised_and_seeded():
    w = C.statics_500()
    a, b = C.woods_saxon(w), C.woods_saxon(w)
    assert np.array_equal(a, b)
    assert abs(a.sum() * w.dxyz - 500) < 1e-9
    w2 = C.replace(w, seed=7)
    assert not np.array_equal(a, C.woods_saxon(w2))


def test_time_steps():
    w = C.tddft_1000()
    assert w.deltat == pytest.approx(1e-4 / 7.63822291, rel=1e-15)
    s = C.statics_500()
    assert s.deltat_statics == pytest.approx(0.1 * 0.7 ** 2 / (4 * 6.05969638298), rel=1e-15)
