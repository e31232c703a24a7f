"""The C++ oracle against a second restatement written independently from the Fortran in numpy
(oracle/numpy_ref.py), on identical seeded inputs, no GPU: set-up, the RK-Gill start and
predictor-corrector steps of the classical-impurity dynamics (Dynamics_TDDFT/DFT4He3d.f90:
562-697).  A misreading of poten, potenimp/forceimp, steprk, steppc or energy in one of the two
would show here.  Bar: 1e-13 relative in E/N, the rho L2 norm and each energy term per step;
psi to 1e-13 of its max; the impurity position to 1e-13 A."""
import numpy as np
import pytest

from oracle import oracle as O
from oracle.numpy_ref import NumpyDynamics
from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D

TOL = 1e-13


def small(n, **kw):
    w = C.tddft_1000(n=n)
    return C.replace(w, xmax=0.625 * n, ymax=0.625 * n, zmax=0.625 * n, n4=300,
                     rimp0=((0.5, -0.3, 0.2 * n),), vimp0_aps=((0.0, 0.0, -3.0),),
                     deltatps=5e-4, **kw)


@pytest.mark.parametrize("n,n_imp,lsolid", [(16, 1, 1), (24, 1, 1), (20, 0, 0), (32, 1, 1)])
def test_oracle_matches_numpy_restatement(n, n_imp, lsolid):
    w = small(n, lsolid=lsolid)
    if n_imp == 0:
        w = C.replace(w, n_imp=0, m_imp_u=(), rimp0=(), vimp0_aps=())
    o = O.Dynamics(w.as_dict(), m_imp_u=w.m_imp_u)
    p = NumpyDynamics(w, o.get("fvlj4"), o.get("wcgk"))
    psi0 = D.initial_wavefunction(w, C.woods_saxon(w), kick=(0.0, 0.0, 0.05))
    for s in (o, p):
        D.dynamics_setup(s, psi0, w.n_imp)
    for it in range(1, 13):
        errs = [D.dynamics_iteration(s, it, w.deltat, w.n_imp) for s in (o, p)]
        if it > 3:
            # errHe, errimp, errvimp are sums of |pc|, the predictor-corrector difference: a few
            # ulps of psi, rimp and vimp, so they agree to rounding on the scale of those fields
            scale = (np.max(np.abs(o.get("psi"))),) + ((np.max(np.abs(o.get("rimp"))),
                                                        np.max(np.abs(o.get("vimp")))) if w.n_imp else (1.0, 1.0))
            for a, b, sc in zip(errs[1], errs[0], scale):
                assert abs(a - b) <= TOL * sc, (it, a, b)
        eo, ep = o.energy(), p.energy()
        for k in ("etot", "ekin4", "elj4", "ecor4", "esolid", "eHeX", "ekinx"):
            assert abs(ep[k] - eo[k]) <= TOL * max(abs(eo[k]), 1e-10), (it, k, ep[k], eo[k])
        lo, lp = np.linalg.norm(o.get("den")), np.linalg.norm(p.get("den"))
        assert abs(lp - lo) <= TOL * lo, it
        po, pp = o.get("psi"), p.get("psi")
        assert np.max(np.abs(pp - po)) <= TOL * np.max(np.abs(po)), it
        for name in ("pot4", "dencg", "delj4", "uimp"):
            a, b = p.get(name), o.get(name)
            assert np.max(np.abs(a - b)) <= TOL * max(np.max(np.abs(b)), 1e-300), (it, name)
        if w.n_imp:
            np.testing.assert_allclose(p.get("rimp"), o.get("rimp"), rtol=0, atol=TOL)
            np.testing.assert_allclose(p.get("vimp"), o.get("vimp"), rtol=TOL, atol=1e-12)
