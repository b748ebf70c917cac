"""Material data on the host: YAML loading, surfactant models and the knot
arrays the table kernels receive, pinned to values the reference produced
(the ``refresh`` kernel fixture and the table step fixtures)."""
import json
import os

import numpy as np
import pytest

import cases
from waam_solver_b200 import materials as M
from waam_solver_b200.gpu_tables import MaterialGPUTables


def _fixture_args(name):
    z = np.load(os.path.join(cases.GOLDEN, name))
    return json.loads(str(z["args"]))


def _step_material():
    z = np.load(os.path.join(cases.GOLDEN, "step_t1_plate.npz"))
    sc = json.loads(str(z["scalars"]))
    rec = sc["material"]
    mat = M.from_constants("ER70S-6", rec["constants"])
    mat.tables = M.MaterialTables(**{k: [tuple(r) for r in v] for k, v in rec["tables"].items()})
    return mat, sc


def test_sahoo_table_matches_reference_upload():
    """The validated ER70S-6 file (28 ppm S, Sahoo model): the 8-knot dgamma/dT
    table from T_liquidus to 2600 K and the scalar at T_liquidus + 50 K."""
    a = _fixture_args("k_refresh.npz")
    table = M.build_sahoo_dgamma_table(28.0, 1793.0, max(1793.0 + 800.0, 2600.0), n=8)
    assert np.array_equal(np.array([t for t, _ in table], np.float32),
                          np.array(a["dgamma_T"], np.float32))
    assert np.array_equal(np.array([v for _, v in table], np.float32),
                          np.array(a["dgamma_V"], np.float32))
    assert M.dgamma_dT_sahoo(1793.0 + 50.0, 28.0) == pytest.approx(a["dgamma_fallback"],
                                                                   rel=1e-14)


def test_gpu_tables_match_reference_upload():
    mat, sc = _step_material()
    t = MaterialGPUTables(mat)
    a = _fixture_args("k_refresh.npz")
    assert t.enabled
    for short in ("cp", "k", "mu", "dgamma"):
        assert np.array_equal(getattr(t, short + "_T"), np.array(a[short + "_T"], np.float32))
        assert np.array_equal(getattr(t, short + "_V"), np.array(a[short + "_V"], np.float32))
        assert getattr(t, "n_" + short) == a["n_" + short]
    assert t.dgamma_fallback == pytest.approx(a["dgamma_fallback"], rel=1e-14)
    # twin.py:271-273: H_sol from cp(T_solidus)
    H_sol = mat.rho * mat.cp_at(mat.T_solidus) * mat.T_solidus
    assert H_sol == pytest.approx(sc["H_sol"], rel=1e-14)
    assert H_sol + mat.rho * mat.L_fusion == pytest.approx(sc["H_liq"], rel=1e-14)
    # the ctypes struct carries the same knots
    st = t.struct
    assert st.n_cp == t.n_cp and list(st.cp_V)[: t.n_cp] == list(t.cp_V[: t.n_cp])


def test_property_without_table_gets_one_knot_at_300K():
    mat = M.from_constants("m", M.LEGACY_LIBRARY["SS316L"])
    mat.tables = M.MaterialTables(cp=[(300.0, 500.0), (1000.0, 650.0)])
    t = MaterialGPUTables(mat)
    assert t.n_cp == 2 and t.n_k == 1 and t.k_T[0] == 300.0 and t.k_V[0] == np.float32(16.3)
    many = M.MaterialTables(mu=[(300.0 + 100 * q, 0.006 - 1e-4 * q) for q in range(11)])
    mat.tables = many
    assert MaterialGPUTables(mat).n_mu == 8        # knots past the eighth are dropped
    assert not MaterialGPUTables(M.from_constants("c", M.LEGACY_LIBRARY["SS316L"])).enabled


def test_interp_linear_edges():
    knots = [(300.0, 1.0), (1000.0, 3.0), (1000.0, 5.0), (2000.0, 7.0)]
    assert M.interp_linear(100.0, knots, -1.0) == 1.0
    assert M.interp_linear(3000.0, knots, -1.0) == 7.0
    assert M.interp_linear(650.0, knots, -1.0) == pytest.approx(2.0)
    assert M.interp_linear(1000.0, knots, -1.0) == 3.0     # first matching segment
    assert M.interp_linear(500.0, [], -1.0) == -1.0


YAML = """
name: TestSteel
status: placeholder
constants:
  k: 20.0
  rho: 7500.0
  cp: 600.0
  T_solidus: 1700.0
  T_liquidus: 1780.0
  L_fusion: 260000.0
  gamma_0: 1.7
  dgamma_dT: -4.0e-4
  mu: 0.006
tables:
  cp:
    - [1000, 650]
    - [300, 550]
    - [1, 2, 3]
  dgamma_dT:
    - [1780, -4.0e-4]
    - [2200, -3.0e-4]
surface:
  contact_angle_deg: 60.0
surfactant:
  model: %s
  sulphur_ppm: %s
electrical:
  rho_e_ohm_m: 2.0e-7
"""


def test_yaml_loading_heiple_scale(tmp_path):
    p = tmp_path / "TestSteel.yaml"
    p.write_text(YAML % ("heiple", "45.0"))
    m = M.load_material(str(p))
    assert m.contact_angle_deg == 60.0 and m.rho_e_ohm_m == 2.0e-7 and m.sulphur_ppm == 45.0
    assert m.tables.cp == [(300.0, 550.0), (1000.0, 650.0)]     # sorted, bad row dropped
    scale = 1.0 - 1.35 * 0.5
    assert m.dgamma_dT == pytest.approx(-4.0e-4 * scale)
    assert m.tables.dgamma_dT[1][1] == pytest.approx(-3.0e-4 * scale)
    assert m.alpha == pytest.approx(20.0 / (7500.0 * 600.0))
    p.write_text(YAML % ("heiple", "80.0"))                      # sign flip above 60 ppm
    assert M.load_material(str(p)).dgamma_dT == pytest.approx(4.0e-4 * 0.35)


def test_yaml_loading_sahoo_and_name_resolution(tmp_path, monkeypatch):
    d = tmp_path / "placeholders"
    d.mkdir()
    (d / "TestSteel.yaml").write_text(YAML % ("sahoo", "28.0"))
    monkeypatch.setenv("WAAM_MATERIALS_DIR", str(tmp_path))
    m = M.load_material("TestSteel")
    assert len(m.tables.dgamma_dT) == 8 and m.tables.dgamma_dT[0][0] == 1780.0
    assert m.tables.dgamma_dT[-1][0] == 2600.0
    assert m.T_ref_gamma == 1780.0
    assert m.dgamma_dT == pytest.approx(M.dgamma_dT_sahoo(1830.0, 28.0))
    # a name with no file falls back to the built-in library
    legacy = M.load_material("ER70S-6")
    assert legacy.rho == 7000.0 and legacy.T_solidus == 1748.0 and not legacy.has_tables
    with pytest.raises(KeyError):
        M.load_material("Unobtainium")
    hs = M.load_material("ER70S-6", high_sulphur=True)
    assert hs.sulphur_ppm == 150.0 and hs.dgamma_dT == pytest.approx(4.3e-4)
