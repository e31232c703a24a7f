"""The table index of updatepoten (Dynamics_TDDFT/potenimp.f90:102, ir = int(r/DelInter)+1) as the
impurity field kernel computes it: from q = r * (1/DelInter), falling back to the IEEE division
only when q lies within 1e-9 of an integer.  On every grid point of the benchmark grids, for
impurity positions along the trajectory, that index equals int() of the IEEE quotient (no GPU:
numpy's division, product and square root are the IEEE operations the kernel uses)."""
import numpy as np
import pytest

from he_dft_2024_b200 import config as C


def kernel_index(r, inv, d):
    q = r * inv
    i0 = q.astype(np.int64)
    fr = q - i0
    near = (fr < 1e-9) | (fr > 1.0 - 1e-9) | (q >= 131072.0)
    i0[near] = (r[near] / d).astype(np.int64)
    return i0, int(near.sum())


@pytest.mark.parametrize("wname", ["tddft_1000", "tddft_5000_256"])
def test_reciprocal_index_equals_ieee_index_on_every_grid_point(wname):
    w = getattr(C, wname)()
    _, npot, d, rmax = C.potion_table(w)
    inv = 1.0 / d
    x, y, z = C.grid_axes(w)
    total = fallback = 0
    zs = (30.0, 17.3, 0.0, -11.8) if w.nx <= 128 else (30.0, 0.0)
    for rz in zs:                                # along the inward trajectory and past the centre
        rx, ry = 0.0, 0.0
        zt = (z - rz) ** 2
        yt = (y - ry)[:, None] ** 2 + zt[None, :]
        r = np.sqrt((x - rx)[:, None, None] ** 2 + yt[None, :, :])
        assert r.max() <= rmax
        ref = (r / d).astype(np.int64)
        got, nf = kernel_index(r.ravel(), inv, d)
        assert np.array_equal(got, ref.ravel())
        total += r.size
        fallback += nf
    # the division runs on few points: those whose radius is (nearly) a multiple of DelInter,
    # e.g. on the axes through the impurity when h is a multiple of DelInter
    assert fallback < 0.02 * total
