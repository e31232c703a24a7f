"""Driver sequences of the reference main loops, written against the call surface only.

These functions mirror what the unchanged Fortran drivers do around the replaced routines
(Dynamics_TDDFT/DFT4He3d.f90:540-576 set-up and :671-697 loop; He_statics/BCN4HeDFT.f90:815-875
set-up and :1086-1160 loop).  They take any object exposing the routines (the device Context,
or the CPU oracle in the tests), so both sides run the identical sequence.
"""
import numpy as np

from .config import Workload, grid_axes


def initial_wavefunction(w: Workload, den, kick=(0.0, 0.0, 0.0)):
    """psi = sqrt(den) * exp(i (x*lx + y*ly + z*lz)) (DFT4He3d.f90:540-557)."""
    x, y, z = grid_axes(w)
    lx, ly, lz = kick
    ph = x[:, None, None] * lx + y[None, :, None] * ly + z[None, None, :] * lz
    return np.asfortranarray(np.sqrt(den) * (np.cos(ph) + 1j * np.sin(ph)))


def dynamics_setup(s, psi, n_imp):
    """den = conjg(psi)*psi; potenimp; poten; forceimp; aimp = F/m (DFT4He3d.f90:562-573)."""
    s.set("psi", psi) if hasattr(s, "set") else s.upload("psi", psi)
    den = (np.conj(psi) * psi).real
    s.set("den", den) if hasattr(s, "set") else s.upload("den", den)
    if n_imp > 0:
        s.potenimp()
    s.poten()
    if n_imp > 0:
        s.forceimp()
        s.set_accel()


def dynamics_iteration(s, iteraux, deltat, n_imp, lrk=False, errors=False):
    """One pass of the time loop body (DFT4He3d.f90:677-697): steprk for the first three
    iterations (or always when lrk), steppc after; then potenimp, poten, forceimp, aimp=F/m."""
    err = None
    if iteraux <= 3 or lrk:
        s.steprk(deltat)
    else:
        err = s.steppc(deltat) if errors or not hasattr(s, "upload") else s.steppc(deltat, errors=False)
    if n_imp > 0:
        s.potenimp()
    s.poten()
    if n_imp > 0:
        s.forceimp()
        s.set_accel()
    return err


def statics_setup(s, den, n4):
    """psi = sqrt(den); derden; fden; dencg; poten; evolo(0) (BCN4HeDFT.f90:815-875, :1050)."""
    psi = np.sqrt(den)
    put = s.set if hasattr(s, "set") else s.upload
    put("den", den)
    put("psi", psi)
    s.refresh() if hasattr(s, "refresh") else s.refresh_density()
    s.poten()
    mu, _ = s.evolo0(0.0, n4)
    return mu


def statics_iteration(s, iterrk, deltat, mu4, n4):
    """One pass of the statics loop (BCN4HeDFT.f90:1113-1160) with Lrkpc: steprkr for the first
    four iterations, steppcr after; then derden, fden, dencg and poten (ppot = 1)."""
    if iterrk <= 4:
        mu4, err = s.steprkr(deltat, mu4, n4)
    else:
        mu4, err = s.steppcr(deltat, mu4, n4)
    s.refresh() if hasattr(s, "refresh") else s.refresh_density()
    s.poten()
    return mu4, err


def quantum_setup(s, psi, psix):
    """Quantum-impurity start (Dynamics_quantum_impurities/DFT4He3d.f90:538-541): psi and the
    impurity wave functions psix (list, one (nx,ny,nz) array per impurity) in place,
    den = conjg(psi)*psi, then potenimp and poten."""
    den = (np.conj(psi) * psi).real
    if hasattr(s, "set"):
        s.set("psi", psi)
        s.set("den", den)
        for i, f in enumerate(psix):
            s.set(f"psix:{i}", f)
    else:
        s.upload("psi", psi)
        s.upload("den", den)
        s.upload("psix", np.stack([np.asarray(f) for f in psix], axis=-1))
    s.potenimp()
    s.poten()


def quantum_iteration(s, iteraux, deltat, lrk=False, errors=False):
    """One pass of the quantum time loop (Dynamics_quantum_impurities/DFT4He3d.f90:666-677):
    steprk for the first three iterations (or always when lrk), steppc(deltat,errHe,errpsix)
    after; then potenimp and poten."""
    err = None
    if iteraux <= 3 or lrk:
        s.steprk(deltat)
    elif hasattr(s, "upload"):
        err = s.steppc(deltat, errors=errors)
        err = err[:2] if err else None
    else:
        err = s.steppc(deltat)
    s.potenimp()
    s.poten()
    return err


def statics_relax(s, den, n4, deltat, iterations, chunk=50):
    """The statics recipe as a start state for real time: psi = sqrt(den), then `iterations`
    imaginary-time passes (four steprkr, then steppcr; BCN4HeDFT.f90:1086-1160), after which the
    driver writes den (printout.f90:52-69) and the dynamics reads it back (readenc.f90:90-110,
    psi = sqrt(den)).  A device context runs the steppcr passes through he_statics_iterations,
    `chunk` at a time.  Returns (den, mu4, mu4err)."""
    mu = statics_setup(s, den, n4)
    err = 0.0
    it = 1
    while it <= min(4, iterations):
        mu, err = statics_iteration(s, it, deltat, mu, n4)
        it += 1
    while it <= iterations:
        k = min(chunk, iterations - it + 1)
        if hasattr(s, "statics_iterations"):
            mu, err = s.statics_iterations(k, deltat, mu, n4)
        else:
            for j in range(k):
                mu, err = statics_iteration(s, it + j, deltat, mu, n4)
        it += k
    out = s.download("den") if hasattr(s, "download") else s.get("den")
    return np.asfortranarray(np.asarray(out).reshape(np.shape(den), order="F")), mu, err


def statics_setup_group(leader, dens, n4):
    """statics_setup for every member of a group (he_ctx_group): member m starts from dens[m];
    one launch per kernel covers all members.  Returns the members' mu4."""
    for m, den in enumerate(dens):
        leader.upload_member(m, "den", den)
        leader.upload_member(m, "psi", np.sqrt(den))
    leader.refresh_density()
    leader.poten()
    leader.evolo0(0.0, n4)
    return leader.member_mu(n4)


def statics_iteration_group(leader, iterrk, deltat, n4):
    """statics_iteration for every member of a group; returns the members' mu4."""
    if iterrk <= 4:
        leader.steprkr(deltat, 0.0, n4)
    else:
        leader.steppcr(deltat, 0.0, n4)
    mu = leader.member_mu(n4, after_rk=iterrk <= 4)
    leader.refresh_density()
    leader.poten()
    return mu
