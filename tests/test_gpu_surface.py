"""The phi = 0.5 surface and the liquid crop of the export (export/vtk_io.py:
170-224), built on the device.

* cell -> corner averaging equals the float32 mean of the sharing cells;
* the marching-tetrahedra surface of a sphere is closed (every edge in two
  triangles), faces outwards and encloses the sphere's volume; its vertices
  lie where the corner field interpolates to 0.5;
* ``export_surface`` on a twin state writes PolyData with the reference's
  point arrays; ``export_volume(crop_liquid=True)`` keeps exactly the cells
  with f_l >= 0.05, with the full export's values.
"""
import math

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


class _G:
    def __init__(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.device = torch.device("cuda", 0)


def _corner_mean(a):
    nx, ny, nz = a.shape
    out = np.zeros((nx + 1, ny + 1, nz + 1), np.float32)
    for I in range(nx + 1):
        for J in range(ny + 1):
            for K in range(nz + 1):
                acc, cnt = np.float32(0.0), 0
                for i in (I - 1, I):
                    for j in (J - 1, J):
                        for k in (K - 1, K):
                            if 0 <= i < nx and 0 <= j < ny and 0 <= k < nz:
                                acc = np.float32(acc + a[i, j, k])
                                cnt += 1
                out[I, J, K] = np.float32(acc / np.float32(cnt))
    return out


def test_cell_to_point_is_the_mean_of_the_sharing_cells():
    from waam_solver_b200 import _native
    rng = np.random.default_rng(2)
    a = rng.normal(0.0, 1.0, (6, 5, 7)).astype(np.float32)
    t = torch.from_numpy(a).cuda()
    out = torch.empty((7 * 6 * 8,), device="cuda")
    _native.call("waam_cell_to_point", t.data_ptr(), None, None, None, out.data_ptr(), None,
                 None, None, 6, 5, 7, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy().reshape(7, 6, 8), _corner_mean(a))


def test_sphere_surface_is_closed_outward_and_encloses_the_ball():
    from waam_solver_b200.export import isosurface
    n, R, w = 40, 12.3, 1.5
    c = (n - 1) / 2.0
    i, j, k = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    r = np.sqrt((i - c) ** 2 + (j - c) ** 2 + (k - c) ** 2)
    phi = (0.5 + 0.5 * np.tanh((R - r) / w)).astype(np.float32)
    T = (300.0 + r).astype(np.float32)
    g = _G(n, n, n)
    verts, tris, attrs = isosurface(g, torch.from_numpy(phi).cuda(),
                                    [torch.from_numpy(T).cuda()], 0.5, 1.0, (0.0, 0.0, 0.0))
    # closed: every undirected edge in exactly two triangles, once in each direction
    e = np.concatenate([tris[:, [0, 1]], tris[:, [1, 2]], tris[:, [2, 0]]])
    und = np.sort(e, axis=1)
    _, cnt = np.unique(und, axis=0, return_counts=True)
    assert np.all(cnt == 2)
    _, cnt_dir = np.unique(e, axis=0, return_counts=True)
    assert np.all(cnt_dir == 1)
    a, b, cc = verts[tris[:, 0]], verts[tris[:, 1]], verts[tris[:, 2]]
    cross = np.cross(b - a, cc - a).astype(np.float64)
    area = 0.5 * np.linalg.norm(cross, axis=1).sum()
    vol = np.einsum("ij,ij->i", a.astype(np.float64), cross).sum() / 6.0
    # the corner averaging shifts the 0.5 level by a fraction of a cell
    center = np.array([c + 0.5] * 3)
    rad = np.linalg.norm(verts - center, axis=1)
    R_eff = float(np.median(rad))
    assert abs(R_eff - R) < 0.5
    assert abs(area - 4 * math.pi * R_eff ** 2) < 0.02 * 4 * math.pi * R_eff ** 2
    assert abs(vol - 4.0 / 3.0 * math.pi * R_eff ** 3) < 0.02 * 4.0 / 3.0 * math.pi * R_eff ** 3
    assert vol > 0.0                     # faces point outwards
    # the temperature attribute follows the radius it was built from
    assert np.allclose(attrs[:, 0], 300.0 + np.clip(rad - 0.0, 0, None), atol=1.5)


def test_export_surface_and_crop_liquid(tmp_path):
    import state_gen
    from waam_solver_b200 import export as E
    from test_gpu_step import _config_twins
    shape = (24, 16, 20)
    tw, ot, dx = _config_twins("c2", *shape)
    st = state_gen.seeded_state(*shape, seed=17, nz_solid=tw.nz_solid)
    tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
    p = E.export_surface(tw, str(tmp_path / "surf.vtp"))
    assert p is not None
    got = E.read_vtk_xml(p)
    for name in ("phi", "Liquid_Fraction", "Temperature_K", "Curvature_kappa"):
        assert got[name].shape[0] == got["Points"].shape[0]
    assert np.all(got["phi"] == np.float32(0.5))
    assert got["connectivity"].shape[0] == 3 * int(got["_attrs"].get("NumberOfPolys", 0) or
                                                   got["offsets"].shape[0])
    full = E.read_vtk_xml(tw.export_vtk_full(str(tmp_path / "full.vti")))
    crop = E.export_volume(tw, str(tmp_path / "crop.vti"), tiers=(0, 3), crop_liquid=True)
    assert crop.endswith(".vtu")
    c = E.read_vtk_xml(crop)
    keep = np.nonzero(full["Liquid_Fraction"] >= np.float32(0.05))[0]
    assert c["types"].shape[0] == keep.size > 0
    for name in ("Temperature_K", "Liquid_Fraction", "Curvature_kappa"):
        assert np.array_equal(c[name], full[name][keep]), name
