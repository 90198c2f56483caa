"""The oracle pinned against the reference's own known-answer tests
(python_tests/test_DDAModelWrapper.py:32-48)."""
import numpy as np
import pytest

from cases import fixture22_args


def test_geometry_generator_matches_reference_fixture(fixture22):
    from oracle.dda_oracle import generate_geometry

    nx, ny, nz, n = (int(v) for v in fixture22["header"])
    assert (nx, ny, nz, n) == (22, 22, 10, 4840)
    assert np.array_equal(generate_geometry(nx, ny, nz), fixture22["geometry"])


def test_product_geometry_generator_matches_reference_fixture(fixture22):
    # pure numpy: importing the package does not load the CUDA library
    from dda_model import _generate_geometry

    nx, ny, nz, _ = (int(v) for v in fixture22["header"])
    assert np.array_equal(_generate_geometry(nx, ny, nz), fixture22["geometry"])


def test_oracle_objective_matches_reference_known_answer(fixture22, sici):
    """Objective 11.005338768207627 at rel 1e-4 (test_DDAModelWrapper.py:40)."""
    from oracle.dda_oracle import OracleModel

    m = OracleModel(**fixture22_args(fixture22, sici))
    info = m.solveElectricField(np.zeros(3 * m.N, complex), 100000, 1e-5)
    assert info.converged
    J = m.calculateObjective()
    assert J == pytest.approx(float(fixture22["expected_objective"]), rel=float(fixture22["expected_rel_tol"]))
    assert J == pytest.approx(float(fixture22["oracle_objective"]), rel=1e-12)
    assert info.iterations == int(fixture22["oracle_iterations"])
