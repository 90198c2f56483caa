"""Generate tests/golden/fixture_22x22x10.npz from the reference's test data.

Reads python_tests/data/geometry.txt and dielectrics.txt of Topo-DDA (the
22x22x10 structure of python_tests/test_DDAModel.py:29-35 and
test_DDAModelWrapper.py:151) and stores them compactly:
  geometry  int8[3N]    (checked equal to the x-fastest generator)
  header    int32[4]    (Nx, Ny, Nz, N)
  rho_bits  uint8       packbits of the per-dipole density (values 0/1,
                        the three per-dipole copies checked equal)
  expected_objective    11.005338768207627 and its rel. tolerance 1e-4
                        (python_tests/test_DDAModelWrapper.py:40)
  oracle_objective / oracle_iterations  this repository's oracle on the same
                        inputs (tol 1e-5), for regression.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT  (a Topo-DDA checkout)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def main(ref_root):
    from oracle import dda_oracle as O

    data = os.path.join(ref_root, "python_tests", "data")
    gc = np.loadtxt(os.path.join(data, "geometry.txt"), dtype=np.int64)
    header = gc[:4].astype(np.int32)
    geo = gc[4:]
    nx, ny, nz, n = (int(v) for v in header)
    assert np.array_equal(geo, O.generate_geometry(nx, ny, nz)), "geometry is not x-fastest"
    diel = np.loadtxt(os.path.join(data, "dielectrics.txt"))
    assert diel.size == 3 * n
    trip = diel.reshape(-1, 3)
    assert np.all(trip == trip[:, :1]), "per-dipole triplets differ"
    rho = trip[:, 0]
    assert set(np.unique(rho)) <= {0.0, 1.0}
    args = O.reference_fixture(data)
    m = O.OracleModel(**args)
    info = m.solveElectricField(np.zeros(3 * n, complex), 100000, 1e-5)
    J = m.calculateObjective()
    out = os.path.join(HERE, "fixture_22x22x10.npz")
    np.savez_compressed(out, header=header, geometry=geo.astype(np.int8),
                        rho_bits=np.packbits(rho.astype(np.uint8)),
                        expected_objective=np.float64(11.005338768207627),
                        expected_rel_tol=np.float64(1e-4),
                        oracle_objective=np.float64(J), oracle_iterations=np.int64(info.iterations))
    print(out, "oracle J =", J, "iterations", info.iterations)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <Topo-DDA checkout root>")
    main(sys.argv[1])
