"""Restart files (he_dft_2024_b200/checkpoint.py): round trips and reading Fortran list-directed
output as the reference's compilers write it (repeat counts, D exponents, spaced complex
constants, logicals, several values per line)."""
import numpy as np

from he_dft_2024_b200 import checkpoint as K
from he_dft_2024_b200 import config as C


def small():
    return C.replace(C.tddft_1000(n=32), nx=8, ny=6, nz=4, xmax=4.0, ymax=3.0, zmax=2.0)


def test_density_round_trip_is_exact(tmp_path):
    w = small()
    den = np.random.default_rng(1).random((8, 6, 4)) * 0.02
    p = tmp_path / "den.dat"
    K.write_density(p, w, den, iteration=17, limp=True, rimp=(0.5, -1.0, 2.0))
    hdr, got = K.read_density(p)
    assert hdr["nx"] == 8 and hdr["ny"] == 6 and hdr["nz"] == 4 and hdr["limp"] is True
    assert hdr["rimp"] == (0.5, -1.0, 2.0)
    assert np.array_equal(got, den)


def test_wavefunction_round_trip_is_exact(tmp_path):
    w = small()
    rng = np.random.default_rng(2)
    psi = rng.normal(size=(8, 6, 4)) + 1j * rng.normal(size=(8, 6, 4))
    rimp = np.array([[0.1, 0.2, 30.0]])
    vimp = np.array([[0.0, 0.0, -22.9]])
    p = tmp_path / "psi.dat"
    K.write_wavefunction(p, w, psi, rimp, vimp, iteration=5, time_ps=5e-4,
                         energies={"etot": -1.5}, observables={"n": 300.0})
    hdr, r, v, got = K.read_wavefunction(p, 1)
    assert np.array_equal(got, psi) and np.array_equal(r, rimp) and np.array_equal(v, vimp)
    try:
        K.read_wavefunction(p, 2)
        raise AssertionError("impurity count mismatch accepted")
    except ValueError as e:
        assert "inconsistent" in str(e)


def test_reads_fortran_list_directed_output(tmp_path):
    # what ifort / gfortran write for `write(10,*)` of a header, N_imp, rimp, vimp and psi
    text = """#  
#  Density after               5 iterations
#  
   4.0000000000000000        3.0000000000000000        2.0000000000000000     
   1.0000000000000000        1.0D0        1.0000000000000000     ,  2  2  1
           1
   0.0000000000000000        0.0000000000000000        30.000000000000000     
   2*0.0000000000000000       -22.900000000000002     
 (  1.0000000000000000     , -0.50000000000000000     ) 2*(  0.0000000000000000     ,  0.0000000000000000     )
 (-2.5D-01,3.0E+00)
"""
    p = tmp_path / "f.dat"
    p.write_text(text)
    hdr, r, v, psi = K.read_wavefunction(p, 1)
    assert (hdr["nx"], hdr["ny"], hdr["nz"]) == (2, 2, 1)
    assert np.array_equal(r, [[0.0, 0.0, 30.0]])
    assert np.array_equal(v, [[0.0, 0.0, -22.900000000000002]])
    assert np.array_equal(psi.ravel(order="F"), [1 - 0.5j, 0, 0, -0.25 + 3j])
