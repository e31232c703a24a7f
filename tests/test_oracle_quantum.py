"""The oracle's quantum-impurity restatement checked against independent computations (CPU).

The reference ships no test vectors for this path (Dynamics_quantum_impurities), so the pieces are
pinned to independent mathematics: the spline of mates.f against scipy's clamped cubic spline,
findi against a bisection by numpy, FT_V_spline against direct quadrature of
4 pi/q int r sin(qr) V(r) dr, and the quantum time step against conservation laws of the exact
dynamics it discretises (norm of psix, energy drift small over a few steps).
"""
import numpy as np
import pytest
from scipy.integrate import quad
from scipy.interpolate import CubicSpline

from oracle import oracle as O
from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D


def test_spline_matches_scipy_clamped_second_derivative():
    rng = np.random.default_rng(3)
    x = np.sort(rng.uniform(0.0, 10.0, 40))
    y = np.sin(x) + 0.1 * x
    s1, sn = -np.sin(x[0]), -np.sin(x[-1])
    a, b, c, d = O.spline(x, y, s1, sn)
    cs = CubicSpline(x, y, bc_type=((2, s1), (2, sn)))
    xt = np.linspace(x[0], x[-1], 777)
    k = np.array([O.findi(x, v) for v in xt]) - 1
    got = a[k] + xt * (b[k] + xt * (c[k] + xt * d[k]))
    assert np.max(np.abs(got - cs(xt))) < 1e-11


def test_findi_bisection():
    x = np.linspace(0.0, 1.0, 101)
    for xc in (-1.0, 0.0, 1e-9, 0.5, 0.505, 0.99, 1.0, 2.0):
        i = O.findi(x, xc)
        if xc > x[-1]:
            assert i == 100
        elif xc <= x[0]:
            assert i == 1
        else:
            assert x[i - 1] < xc <= x[i]


MORSE = [1, 2.0, 6.5, 0.8, C.MORSE_RCUT, C.MORSE_UMAX]


def _v(r):
    if r < MORSE[4]:
        return MORSE[5]
    e = 1.0 - np.exp(-MORSE[3] * (r - MORSE[2]))
    return MORSE[1] * (e * e - 1.0)


@pytest.mark.parametrize("p", [0.0, 0.05, 0.3, 1.0, 3.0])
def test_ft_v_spline_matches_quadrature(p):
    got = O.ft_vpp_point(MORSE, p)
    q = 2 * np.pi * p
    f = (lambda r: 4 * np.pi * r * r * _v(r)) if p == 0 else (lambda r: 4 * np.pi * r * np.sin(q * r) / q * _v(r))
    ref = quad(f, 0, MORSE[4], limit=400)[0] + quad(f, MORSE[4], 60.0, limit=4000)[0]
    # the reference's spline has h = 0.05 A; its quadrature error is O(1e-6) relative
    assert abs(got - ref) <= 2e-5 * max(abs(ref), 50.0)


def test_ft_v_spline_small_q_redefinition():
    """Momenta p <= small_q = 0.01 are replaced by the natural cubic spline through p = 0 and the
    first three momenta above small_q (FT_V_spline.f90:229-258)."""
    hp = 0.01
    v = O.ft_vpp_table(MORSE, 100.0, hp, nspline=4001)
    raw = [O.ft_vpp_point(MORSE, i * hp, 4001) for i in (0, 2, 3, 4)]
    assert v[0] == raw[0] and v[2] == raw[1] and v[4] == raw[3]
    nat = CubicSpline([0.0, 0.02, 0.03, 0.04], raw, bc_type="natural")
    assert abs(v[1] - nat(0.01)) < 1e-9 * abs(raw[0])


def test_quantum_step_conserves_norm_and_energy_approximately():
    w = C.replace(C.quantum_2000(n=32), xmax=12.0, ymax=12.0, zmax=12.0, n4=300, n_spline=4001,
                  deltatps=2e-4)
    o = O.QDynamics(w.as_dict())
    den = C.woods_saxon(w)
    D.quantum_setup(o, D.initial_wavefunction(w, den), [C.psix_initial(w)])
    e0 = o.energy()["etot"]
    m0 = o.moments()[0]
    for it in range(1, 7):
        D.quantum_iteration(o, it, w.deltat)
    m = o.moments()[0]
    assert abs(m0[0] - 1.0) < 1e-12
    assert abs(m[0] - 1.0) < 1e-3
    assert abs(o.energy()["etot"] - e0) < 1e-2 * abs(e0)
