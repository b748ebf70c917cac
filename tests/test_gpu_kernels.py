"""CUDA kernels (through the C ABI) against the reference's own kernels and
against the oracle.

* every golden case: the CUDA result vs the reference output (tolerance of
  cases.RTOL);
* every golden case: the CUDA result vs the C oracle on the same inputs --
  the two share the float32 expression order and the exponential, so all
  fields must agree to cases.RTOL and flags / integer fields bit-exactly;
* larger seeded states (up to 48x40x36) for the stencil kernels, vs the oracle.
"""
import copy

import numpy as np
import pytest

import cases
import state_gen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cuda_backend():
    from cuda_backend import CudaBackend
    return CudaBackend()


@pytest.fixture(scope="module")
def oracle_backend():
    return cases.OracleBackend()


@pytest.mark.parametrize("name", cases.CASES)
def test_cuda_matches_reference_kernel(cuda_backend, name):
    cases.check_case(cuda_backend, name)


@pytest.mark.parametrize("name", cases.CASES)
def test_cuda_matches_oracle(cuda_backend, oracle_backend, name):
    a, st, _ = cases.full_inputs(name)
    st_o = copy.deepcopy(st)
    ex_c = cases.run_case(cuda_backend, name, st, a)
    ex_o = cases.run_case(oracle_backend, name, st_o, a)
    for f, v in st.items():
        if isinstance(v, np.ndarray):
            cases.compare(name, v, st_o[f], f)
            if v.dtype.kind in "iu":
                assert np.array_equal(v, st_o[f])
    if name == "lorentz":   # grid sums in double, block order vs serial order
        np.testing.assert_allclose(ex_c, ex_o, rtol=cases.RTOL)
    else:
        assert ex_c == ex_o or name in ("deposit",)


BIG = ["inject_gauss", "inject_goldak", "thermal", "vof", "vof_wet", "contact", "contact_s5",
       "forces", "forces_wet", "csf_wet", "collide_mrt", "collide_srt", "stream", "tail",
       "heat_loss", "deposit", "lorentz"]


@pytest.mark.parametrize("shape", [(48, 40, 36), (33, 17, 70)])
@pytest.mark.parametrize("name", BIG)
def test_cuda_matches_oracle_on_larger_states(cuda_backend, oracle_backend, name, shape):
    a, _, _ = cases.full_inputs(name)
    nx, ny, nz = shape
    st = state_gen.seeded_state(nx, ny, nz, seed=100 + BIG.index(name))
    st = {k: (np.ascontiguousarray(v) if isinstance(v, np.ndarray) else v) for k, v in st.items()}
    st["phi_tmp"] = np.zeros_like(st["phi"])
    a = dict(a)
    a["nz_solid"] = st["nz_solid"]
    a.setdefault("arc_k", float(st["nz_solid"] + 1))
    for key in ("arc_i", "arc_j"):
        if key in a:
            a[key] = a[key] * (nx if key == "arc_i" else ny) / (13.0 if key == "arc_i" else 11.0)
    st_o = copy.deepcopy(st)
    cases.run_case(cuda_backend, name, st, a)
    cases.run_case(oracle_backend, name, st_o, a)
    for f, v in st.items():
        if isinstance(v, np.ndarray):
            cases.compare("%s %s" % (name, shape), v, st_o[f], f)
