"""he_energy_noalloc: the energy sums on device arrays owned by the caller, with no device
allocation inside the library.

Callers whose device memory all belongs to them -- a Fortran driver whose arrays live in OpenACC
or CUDA Fortran data regions sized at start-up, or a job that reserves the GPU's memory in its own
pool -- cannot let a library call cudaMalloc.  This entry point serves them: its only scratch is a
fixed device array inside the library (grids up to 256^3).  The GPU test checks it against the
context API's he_energy on the same state, on two calls in a row (the scratch keeps the previous
call's contents, so the second call checks that the counter is cleared).  This file is collected
last on purpose and must also pass when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from he_dft_2024_b200 import _lib, config as C, driver as D

RTOL = 1e-12
HE_KEYS = ("ekin4", "elj4", "ecor4", "esolid", "etot4")


def _grid_fun(w, core=b"OT "):
    g = _lib.HeGrid(w.nx, w.ny, w.nz, w.xmax, w.ymax, w.zmax, w.npd, w.icon)
    f = _lib.HeFunctional(core, w.h4, w.eps4, w.sigma4, w.cp4, w.cpp4, w.den4c, w.alphas, w.l,
                          w.den0s, w.h2o2m4, w.lsolid, w.C, w.beta, w.den_m)
    return g, f


def _noalloc(w, mode, ptrs, stream):
    L = _lib.load()
    g, f = _grid_fun(w)
    out = _lib.HeEnergies()
    err = ctypes.create_string_buffer(256)
    st = L.he_energy_noalloc(ctypes.byref(g), ctypes.byref(f), mode, *ptrs, stream,
                             ctypes.byref(out), err, 256)
    assert st == 0, err.value.decode()
    return {k: getattr(out, k) for k, _ in _lib.HeEnergies._fields_}


def test_noalloc_rejects_grids_beyond_its_scratch():
    """Sizes beyond the fixed scratch are refused before any device work (no GPU needed)."""
    L = _lib.load()
    w = C.replace(C.tddft_1000(), nx=512, ny=512, nz=512)
    g, f = _grid_fun(w)
    out = _lib.HeEnergies()
    err = ctypes.create_string_buffer(256)
    dummy = ctypes.c_void_p(16)
    st = L.he_energy_noalloc(ctypes.byref(g), ctypes.byref(f), _lib.HE_MODE_DYNAMICS, dummy, dummy,
                             dummy, dummy, None, None, ctypes.byref(out), err, 256)
    assert st == _lib.HE_ERR_ARG
    assert b"256^3" in err.value


@pytest.mark.parametrize("core", [b"OTC", b"XX "])
def test_noalloc_refuses_cores_it_cannot_total(core):
    """core4='OTC' adds the alpha_s energy to etot4, which this entry point does not compute; it
    and unknown cores are refused on the host, before any device work (no GPU needed)."""
    L = _lib.load()
    w = C.tddft_1000(n=32)
    g, f = _grid_fun(w, core)
    out = _lib.HeEnergies()
    err = ctypes.create_string_buffer(256)
    dummy = ctypes.c_void_p(16)
    st = L.he_energy_noalloc(ctypes.byref(g), ctypes.byref(f), _lib.HE_MODE_DYNAMICS, dummy, dummy,
                             dummy, dummy, None, None, ctypes.byref(out), err, 256)
    assert st == _lib.HE_ERR_ARG
    assert b"core4" in err.value


@pytest.mark.gpu
@pytest.mark.parametrize("mode,icon", [("dynamics", 13), ("dynamics", 18), ("statics", 13)])
def test_energy_noalloc_matches_he_energy_twice(mode, icon):
    import torch
    from he_dft_2024_b200.context import Context

    if mode == "dynamics":
        w = C.replace(C.tddft_1000(n=32), xmax=20.0, ymax=20.0, zmax=20.0, n4=300,
                      rimp0=((0.5, -0.3, 8.0),), deltatps=5e-4, icon=icon)
    else:
        w = C.replace(C.statics_500(), nx=32, ny=32, nz=32, xmax=11.2, ymax=11.2, zmax=11.2)
    with Context(w, mode=mode) as ctx:
        if mode == "dynamics":
            D.dynamics_setup(ctx, D.initial_wavefunction(w, C.woods_saxon(w)), w.n_imp)
            for it in range(1, 5):
                D.dynamics_iteration(ctx, it, w.deltat, w.n_imp)
            names = ("psi", "den", "dencg", "delj4", "uimp")
        else:
            mu = D.statics_setup(ctx, C.woods_saxon(w), w.n4)
            for it in range(1, 4):
                mu, _ = D.statics_iteration(ctx, it, w.deltat_statics, mu, w.n4)
            names = ("psi", "den", "dencg", "delj4")
        ref = ctx.energy()
        host = {n: np.ascontiguousarray(ctx.download(n).ravel(order="F")) for n in names}

    dev = {n: torch.from_numpy(v).cuda() for n, v in host.items()}
    ptrs = [ctypes.c_void_p(dev[n].data_ptr()) for n in ("psi", "den", "dencg", "delj4")]
    ptrs.append(ctypes.c_void_p(dev["uimp"].data_ptr()) if "uimp" in dev else None)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    m = _lib.HE_MODE_DYNAMICS if mode == "dynamics" else _lib.HE_MODE_STATICS
    first = _noalloc(w, m, ptrs, stream)
    second = _noalloc(w, m, ptrs, stream)
    keys = HE_KEYS + (("eHeX",) if mode == "dynamics" else ())
    for got in (first, second):
        for k in keys:
            assert abs(got[k] - ref[k]) <= RTOL * max(abs(ref[k]), 1e-12), (k, got[k], ref[k])
