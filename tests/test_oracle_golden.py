"""The C oracle against the reference's own kernels (golden fixtures).

The fixtures in tests/golden/ were produced by the reference's unmodified
Taichi kernels executed serially (tests/golden/make_golden.py); this pins the
oracle before it is used to check the CUDA path.
"""
import pytest

import cases


@pytest.fixture(scope="module")
def oracle_backend():
    return cases.OracleBackend()


@pytest.mark.parametrize("name", cases.CASES)
def test_oracle_matches_reference_kernel(oracle_backend, name):
    cases.check_case(oracle_backend, name)
