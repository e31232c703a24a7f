"""Pins the CPU oracle to the reference's own known answers (no GPU).

* 13-point Bickley weights: bit-exact against the BLOCK DATA table text
  (Dynamics_TDDFT/mates.f:786-879 == blockds.f:615-708), fixture tests/golden/bickley13.json.
* icon=13 boundary rows: applying the Redef recipe (redef.f:151-170 then :133-150) to the table
  gives the centred row shifted with zero fill, i.e. zero padding, which is what the oracle and
  the device stencils implement.
* b = bforce(OT, 10.22, 2.556, 2.190323) ~ b4 = -718.99 (modules.f90:233, fforma.f90:256-280).
* bulk equation of state mu(rho0) = b rho + 3/2 cp4 rho^2 + 4/3 cpp4 rho^3
  (He_statics/rhoasin0.f90:53-63) ~ Chempo = -7.15 K (He_statics/modules.f90:130), reproduced by
  the oracle's poten on a uniform density.
"""
import json
import os

import numpy as np
import pytest
from scipy.special import sici

from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "bickley13.json")))
CONST = json.load(open(os.path.join(HERE, "golden", "constants.json")))


def golden_matrix(k):
    return np.array([float.fromhex(e["hex"]) for e in GOLD[f"K{k}"]]).reshape(13, 13)


def cfg(n=(16, 16, 16), xmax=(8.0, 8.0, 8.0), **kw):
    d = dict(nx=n[0], ny=n[1], nz=n[2], xmax=xmax[0], ymax=xmax[1], zmax=xmax[2], npd=13, icon=13,
             core="OT", h4=CONST["h4ot"], eps4=CONST["eps4"], sigma4=CONST["sigma4"],
             cp4=CONST["cp4"], cpp4=CONST["cpp4"], den4c=0.062, alphas=54.31, l=1.0, den0s=0.04,
             h2o2m4=CONST["h2o2m4"], lsolid=0, C=CONST["C"], beta=CONST["beta"],
             den_m=CONST["den_m"], lambdah=2.0, txmean=1000.0, txsurf=2.0, tymean=1000.0,
             tysurf=2.0, tzmean=1000.0, tzsurf=2.0, n_imp=0, dtmin=1e-10, sdmu=0.1, dmumax=100.0)
    d.update(kw)
    return d


def test_centred_rows_bit_exact():
    w1, w2 = O.bickley13()
    g1, g2 = golden_matrix(1), golden_matrix(2)
    assert [v.hex() for v in w1] == [v.hex() for v in g1[6]]
    assert [v.hex() for v in w2] == [v.hex() for v in g2[6]]


def redef_icon13(cd):
    """redef.f:151-170 (ICON=13: rows KO2..1 from the row below, shifted left, zero fill) followed
    by :133-150 (ICON=12: rows KO2+2..K from the row above, shifted right, zero fill)."""
    c = cd.copy()
    k, ko2 = 13, 6
    for i in range(ko2, 0, -1):        # I = KO2..1 (1-based)
        c[i - 1, : k - 1] = c[i, 1:k]
        c[i - 1, k - 1] = 0.0
    for i in range(ko2 + 2, k + 1):    # I = KO2+2..K
        c[i - 1, 1:k] = c[i - 2, 0:k - 1]
        c[i - 1, 0] = 0.0
    return c


@pytest.mark.parametrize("k", [1, 2])
def test_icon13_boundary_rows_are_zero_padding(k):
    c = redef_icon13(golden_matrix(k))
    centred = golden_matrix(k)[6]
    n = 20
    f = np.random.default_rng(1).normal(size=n)
    fp = np.concatenate([np.zeros(6), f, np.zeros(6)])
    padded = np.array([centred @ fp[i:i + 13] for i in range(n)])
    # Deriv1D_p row use (init_deriv_parallel.f90:140-158 pattern): first rows use f(1:k),
    # last rows f(n-k+1:n)
    ref = np.empty(n)
    for i in range(n):
        if i < 6:
            ref[i] = c[i] @ f[:13]
        elif i >= n - 6:
            ref[i] = c[i - n + 13] @ f[n - 13:]
        else:
            ref[i] = centred @ f[i - 6:i + 7]
    np.testing.assert_allclose(ref, padded, rtol=0, atol=1e-13)


def redef_icon24(cd):
    """redef.f:245-279 (ICON=24: rows K..KO2+2 from the centred row, folded at the last point)
    then, with TORNA, :18-56 (ICON=4, IP=+1: rows 1..KO2 folded at the first point), written out
    loop by loop on the row-major K x K block (CD(j + (i-1)K) = c[i-1, j-1])."""
    c = cd.copy()
    k, ko2, ko2p1 = 13, 6, 7
    i0 = ko2p1
    C = lambda i, j: c[i - 1, j - 1]
    for i in range(k, ko2 + 1, -1):            # I = K..KO2+2
        j0 = ko2p1 - i + k
        j1 = j0
        c[i - 1, k - 1] = C(i0, j0)
        for j in range(k - 1, 0, -1):
            j0 -= 1
            j1 += 1
            if j0 >= 1:
                c[i - 1, j - 1] = C(i0, j0) + C(i0, j1) if j1 <= k else C(i0, j0)
            else:
                c[i - 1, j - 1] = 0.0
    for i in range(1, ko2 + 1):                # ICON=4, I = 1..KO2
        j0 = ko2p1 - i + 1
        j1 = j0
        c[i - 1, 0] = C(i0, j0)
        for j in range(2, k + 1):
            j0 += 1
            j1 -= 1
            if j0 <= k:
                c[i - 1, j - 1] = C(i0, j0) + C(i0, j1) if j1 >= 1 else C(i0, j0)
            else:
                c[i - 1, j - 1] = 0.0
    return c


@pytest.mark.parametrize("k", [1, 2])
def test_icon24_boundary_rows_are_even_reflection(k):
    """icon=24's Redef rows equal the centred stencil on a field reflected evenly about its first
    and last points (numpy's 'reflect' padding), which the oracle and device stencils use."""
    c = redef_icon24(golden_matrix(k))
    centred = golden_matrix(k)[6]
    n = 20
    f = np.random.default_rng(2).normal(size=n)
    fp = np.pad(f, 6, mode="reflect")
    mirrored = np.array([centred @ fp[i:i + 13] for i in range(n)])
    ref = np.empty(n)
    for i in range(n):
        if i < 6:
            ref[i] = c[i] @ f[:13]
        elif i >= n - 6:
            ref[i] = c[i - n + 13] @ f[n - 13:]
        else:
            ref[i] = centred @ f[i - 6:i + 7]
    np.testing.assert_allclose(ref, mirrored, rtol=0, atol=1e-12)


def test_bforce_matches_b4():
    b_ot = O.lib().ho_bforce(0, CONST["eps4"], CONST["sigma4"], CONST["h4ot"])
    b_op = O.lib().ho_bforce(1, CONST["eps4"], CONST["sigma4"], CONST["h4op"])
    assert abs(b_ot - CONST["b4"]) < 0.01
    assert abs(b_op - CONST["b4"]) < 0.01
    # the literal hc=2.359665 with the OT core is a different functional (|b| ~ 1677)
    assert abs(O.lib().ho_bforce(0, CONST["eps4"], CONST["sigma4"], CONST["h4op"]) + 1677.4) < 0.2


def test_bulk_chemical_potential():
    c = cfg(icon=8)
    d = O.Dynamics(c)
    rho0 = CONST["densat4"]
    d.set("den", np.full(16 ** 3, rho0))
    d.poten()
    pot = d.get("pot4")
    b = O.lib().ho_bforce(0, CONST["eps4"], CONST["sigma4"], CONST["h4ot"])
    mu = b * rho0 + 1.5 * CONST["cp4"] * rho0 ** 2 + 4.0 / 3.0 * CONST["cpp4"] * rho0 ** 3
    np.testing.assert_allclose(pot, mu, rtol=1e-12)
    mu_b4 = CONST["b4"] * rho0 + 1.5 * CONST["cp4"] * rho0 ** 2 + 4.0 / 3.0 * CONST["cpp4"] * rho0 ** 3
    assert abs(mu_b4 - (-7.1448)) < 5e-4
    assert abs(mu_b4 - CONST["chempo"]) < 0.01


def test_sine_integral():
    xs = np.concatenate([np.linspace(1e-6, 4.0, 200), np.linspace(4.0, 60.0, 400)])
    ours = np.array([O.lib().ho_sine_integral(x) for x in xs])
    np.testing.assert_allclose(ours, sici(xs)[0], rtol=2e-15, atol=2e-16)


@pytest.mark.parametrize("n", [(16, 16, 16), (24, 20, 18), (30, 16, 12), (32, 48, 40)])
def test_fft_matches_pocketfft(n):
    c = cfg(n=n)
    a = np.random.default_rng(2).normal(size=n)
    spec = O.r2c(c, a)
    ref = np.fft.rfftn(a, axes=(2, 1, 0))
    np.testing.assert_allclose(spec, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    back = O.c2r(c, spec)
    np.testing.assert_allclose(back, a, rtol=0, atol=1e-13 * np.abs(a).max())


def np_deriv(f, w, h, axis, icon=13):
    n = f.shape[axis]
    if n < 13:
        return np.zeros_like(f)
    pad = [(0, 0)] * 3
    pad[axis] = (6, 6)
    fp = np.pad(f, pad, mode={8: "wrap", 24: "reflect"}.get(icon, "constant"))
    out = np.zeros_like(f)
    for m in range(13):
        sl = [slice(None)] * 3
        sl[axis] = slice(m, m + n)
        out = out + w[m] * fp[tuple(sl)]
    return out / h


@pytest.mark.parametrize("icon", [13, 8, 24])
@pytest.mark.parametrize("id_", [1, 2])
def test_derivatives(icon, id_):
    n = (20, 16, 14)
    c = cfg(n=n, xmax=(5.0, 4.0, 3.5), icon=icon)
    rng = np.random.default_rng(3)
    f = rng.normal(size=n) + 1j * rng.normal(size=n)
    w1, w2 = O.bickley13()
    w = w1 if id_ == 1 else w2
    hs = [2 * 5.0 / 20, 2 * 4.0 / 16, 2 * 3.5 / 14]
    for ax in range(3):
        got = O.deriv(c, f, id_, ax)
        ref = np_deriv(f, w, hs[ax] ** id_, ax, icon)
        np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-11)


def test_short_axis_derivative_is_zero():
    c = cfg(n=(16, 16, 12))
    f = np.random.default_rng(4).normal(size=(16, 16, 12))
    assert np.all(O.deriv(c, f, 2, 2) == 0.0)
