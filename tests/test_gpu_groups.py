"""Groups of statics droplets (he_ctx_group): one launch per kernel advances every member, and
each member must come out exactly as the same droplet run alone on the same kernel variants.

Three 4He_500 droplets with different seeded noise on 32^3 and 64^3 grids run the statics loop
(BCN4HeDFT.f90:1113-1160: four steprkr iterations, then steppcr with derden, fden, dencg and
poten) as a group and one by one; mu per iteration, the energies and the final densities must be
bit-identical.  Groups outside their scope are refused."""
import numpy as np
import pytest

from he_dft_2024_b200 import config as C
from he_dft_2024_b200 import driver as D
from he_dft_2024_b200._lib import HeError
from he_dft_2024_b200.context import Context

pytestmark = pytest.mark.gpu


def pin(ctx, n):
    ctx.set_fft_variant("x", 0, 8)
    ctx.set_fft_variant("y", 1, 8)
    ctx.set_fft_variant("z", 0, 8)
    if n == 64:
        ctx.set_fft_variant("yz", 1, 8)


@pytest.mark.parametrize("n", [32, 64])
def test_group_members_equal_droplets_run_alone(n):
    base = C.replace(C.statics_500(), nx=n, ny=n, nz=n, xmax=0.35 * n, ymax=0.35 * n, zmax=0.35 * n)
    ws = [C.replace(base, seed=1234 + 7 * k) for k in range(3)]
    dens = [C.woods_saxon(w) for w in ws]
    dt, n4 = base.deltat_statics, base.n4
    iters, chunk = 10, 6
    # alone
    ref = []
    for w, den in zip(ws, dens):
        with Context(w, mode="statics") as c:
            pin(c, n)
            mus = [D.statics_setup(c, den, n4)]
            mu = mus[0]
            for it in range(1, iters + 1):
                mu, _ = D.statics_iteration(c, it, dt, mu, n4)
                mus.append(mu)
            mu, _ = c.statics_iterations(chunk, dt, mu, n4)
            mus.append(mu)
            ref.append(dict(mu=np.array(mus), e=c.energy(), den=c.download("den")))
    # as a group
    ctxs = [Context(w, mode="statics") for w in ws]
    for c in ctxs:
        pin(c, n)
    lead = ctxs[0]
    try:
        lead.group(ctxs[1:])
        assert lead.members == 3
        mus = [D.statics_setup_group(lead, dens, n4)]
        for it in range(1, iters + 1):
            mus.append(D.statics_iteration_group(lead, it, dt, n4))
        mu, _, _ = lead.statics_iterations_members(chunk, dt, mus[-1], n4)
        mus.append(mu)
        es = lead.energy_members()
        got_den = [lead.download_member(m, "den") for m in range(3)]
    finally:
        lead.close()
    mus = np.array(mus)
    for m in range(3):
        assert np.array_equal(mus[:, m], ref[m]["mu"]), (m, mus[:, m] - ref[m]["mu"])
        for k in ("etot", "ekin4", "elj4", "ecor4", "esolid"):
            assert es[m][k] == ref[m]["e"][k], (m, k)
        assert np.array_equal(got_den[m], ref[m]["den"]), m


def test_groups_outside_their_scope_are_refused():
    w = C.replace(C.statics_500(), nx=32, ny=32, nz=32, xmax=11.2, ymax=11.2, zmax=11.2)
    a, b = Context(w, mode="statics"), Context(C.replace(w, nx=40, xmax=14.0), mode="statics")
    d = Context(C.replace(C.tddft_1000(n=32), n_imp=0, m_imp_u=(), rimp0=(), vimp0_aps=()))
    try:
        with pytest.raises(HeError):
            a.group([b])          # different grid
        with pytest.raises(HeError):
            d.group([d])          # dynamics mode, and a repeated member
        assert a.members == 1
    finally:
        for c in (a, b, d):
            c.close()


@pytest.mark.parametrize("precision", ["f64", "mixed"])
def test_quantum_group_members_equal_trajectories_run_alone(precision):
    """Three quantum-impurity trajectories with different kicks on 32^3 (one 23 u impurity each):
    set up on their own, then grouped; RK-Gill start and predictor-corrector steps with one launch
    per kernel must leave every member exactly as the trajectory run alone (psi, psix, energies,
    impurity moments)."""
    ws = [C.replace(C.quantum_2000(n=32, speed_ms=s, direction=d), n4=300, xmax=12.0, ymax=12.0,
                    zmax=12.0, deltatps=5e-4)
          for s, d in ((100.0, (0, 0, 1)), (250.0, (1, 0, 0)), (400.0, (0, 1, 1)))]
    steps = 6

    def make(w):
        c = Context(w, mode="quantum", precision=precision)
        c.set_fft_variant("x", 0, 8)
        c.set_fft_variant("y", 1, 8)
        c.set_fft_variant("z", 0, 8)
        den = C.woods_saxon(w)
        D.quantum_setup(c, D.initial_wavefunction(w, den), [C.psix_initial(w, 0)])
        return c

    ref = []
    for w in ws:
        with make(w) as c:
            for it in range(1, steps + 1):
                D.quantum_iteration(c, it, w.deltat)
            ref.append(dict(psi=c.download("psi"), psix=c.download("psix"), e=c.energy(),
                            mom=c.qimp_moments()))
    ctxs = [make(w) for w in ws]
    lead = ctxs[0]
    try:
        lead.group(ctxs[1:])
        for it in range(1, steps + 1):
            D.quantum_iteration(lead, it, ws[0].deltat)
        es = lead.energy_members()
        mom = lead.qimp_moments_members()
        got = [dict(psi=lead.download_member(m, "psi")) for m in range(3)]
    finally:
        lead.close()
    for m in range(3):
        assert np.array_equal(got[m]["psi"], ref[m]["psi"]), m
        for k in ("etot", "ekin4", "ekinx", "eHeX"):
            assert es[m][k] == ref[m]["e"][k], (m, k, es[m][k], ref[m]["e"][k])
        assert np.array_equal(mom[m], ref[m]["mom"]), m
