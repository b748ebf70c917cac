"""Headless research export (reference export/vtk_io.py, bundle.py, meta.py).

Volume snapshots are VTK XML ImageData (``.vti``) files with the reference's
array names, units and tiers; tracers are VTK XML PolyData (``.vtp``); a
bundle adds the telemetry and metadata JSON and the probe CSV; a sequence adds
a ParaView ``.pvd`` collection.  The files are written by this module
directly (raw appended binary, UInt64 headers), so neither PyVista nor a
graphics stack is needed.

Every volume array is computed on the device in its physical units and in
VTK cell order (x fastest) by one ``waam_export_pack`` launch into a staging
buffer, and reaches the host in a single copy.  ``read_vtk_xml`` reads the
files back (tests, post-processing without VTK).

The phi = 0.5 surface (``export_surface``) is contoured on the device: cell
values averaged to the cell corners (as VTK's cell_data_to_point_data) and
cut by marching tetrahedra (the reference calls PyVista's contour filter, a
different triangulation of the same isosurface); triangle vertices are merged
by lattice edge on the host and written as PolyData.  ``crop_liquid`` keeps
the cells with a liquid fraction of at least 0.05 (the reference's threshold)
as an UnstructuredGrid of voxels (``.vtu``).  ``export_npz`` writes the raw
state for Python post-processing.
"""
from __future__ import annotations

import json
import pathlib
import xml.etree.ElementTree as ET

import numpy as np
import torch

from . import _native, kernels

TIER_CORE = 0
TIER_MATERIAL = 1
TIER_FORCES = 2
TIER_DERIVED = 3
TIER_MAP = {0: TIER_CORE, 1: TIER_MATERIAL, 2: TIER_FORCES, 3: TIER_DERIVED}
WAAM_TWIN_VERSION = "2.0.0"

N = _native
_F32, _I32 = "Float32", "Int32"


def vtk_imagedata_path(path):
    p = pathlib.Path(path)
    if p.suffix.lower() in (".vts", ""):
        return str(p.with_suffix(".vti"))
    return str(path)


def _prepare_derived(twin, tiers):
    """vtk_io.py:66-79: curvature and vorticity into the export buffers."""
    if TIER_DERIVED not in tiers:
        return
    g = twin.grid
    g.ensure_export_buffers()
    kernels.compute_curvature_field(g.phi, g.flags, g.kappa_field, g.FLAG_GAS, g.nx, g.ny, g.nz)
    kernels.compute_vorticity_magnitude(g.ux, g.uy, g.uz, g.flags, g.vorticity_mag, g.dx, g.dt,
                                        g.FLAG_GAS, g.nx, g.ny, g.nz)


def volume_channels(twin, tiers):
    """(name, VTK type, channel) of every volume array, vtk_io.py:82-166 order.

    The scalars follow numpy's float32 evaluation of the reference: Python
    floats enter as float32 and operations run left to right."""
    g = twin.grid
    f32 = lambda v: float(np.float32(v))  # noqa: E731
    dx, dt = f32(g.dx), f32(g.dt)
    ch = []

    def add(name, op, srcs, a=0.0, b=0.0, c=0.0, typ=_F32):
        ch.append((name, typ, (op, a, b, c, srcs)))

    if TIER_CORE in tiers:
        add("Temperature_K", N.EXPORT_COPY, [g.T])
        add("Temperature_C", N.EXPORT_ADD, [g.T], a=f32(-273.15))
        add("Liquid_Fraction", N.EXPORT_COPY, [g.f_l])
        add("VOF_phi", N.EXPORT_COPY, [g.phi])
        add("Cell_Flags", N.EXPORT_COPY_I32, [g.flags], typ=_I32)
        add("T_max_K", N.EXPORT_COPY, [g.T_max])
        add("T_prev_K", N.EXPORT_COPY, [g.T_prev])
        add("dTdt_Ks", N.EXPORT_COPY, [g.dT_dt])
        add("Cooling_Rate_Ks", N.EXPORT_NEG, [g.dT_dt])
        add("Enthalpy_Jm3", N.EXPORT_COPY, [g.H])
        add("Time_above_800C_s", N.EXPORT_COPY, [g.time_above_800_s])
        add("Time_above_1100C_s", N.EXPORT_COPY, [g.time_above_1100_s])
        add("Time_above_solidus_s", N.EXPORT_COPY, [g.time_above_solidus_s])
        add("Velocity_X_ms", N.EXPORT_LU_VEL, [g.ux], a=dx, b=dt)
        add("Velocity_Y_ms", N.EXPORT_LU_VEL, [g.uy], a=dx, b=dt)
        add("Velocity_Z_ms", N.EXPORT_LU_VEL, [g.uz], a=dx, b=dt)
        add("Speed_ms", N.EXPORT_SPEED, [g.ux, g.uy, g.uz], a=dx, b=dt)
        add("Density_lu", N.EXPORT_COPY, [g.rho])
        add("Pressure_Pa_gauge", N.EXPORT_PRESSURE, [g.rho], a=f32(1.0 / 3.0), b=f32(g.mat.rho),
            c=f32((g.dx / g.dt) ** 2))
    if TIER_MATERIAL in tiers and twin.use_material_tables:
        add("RhoCp_Jm3K", N.EXPORT_COPY, [g.cp_rho_field])
        add("Alpha_lu", N.EXPORT_COPY, [g.alpha_lu_field])
        add("DgammaDT_lu", N.EXPORT_COPY, [g.dgamma_lu_field])
        add("Tau_SRT", N.EXPORT_COPY, [g.tau_field])
    if TIER_FORCES in tiers:
        add("BodyForce_X_ms2", N.EXPORT_LU_ACC, [g.Fx_snap], a=dx, b=dt)
        add("BodyForce_Y_ms2", N.EXPORT_LU_ACC, [g.Fy_snap], a=dx, b=dt)
        add("BodyForce_Z_ms2", N.EXPORT_LU_ACC, [g.Fz_snap], a=dx, b=dt)
        add("BodyForce_mag_ms2", N.EXPORT_ACC_MAG, [g.Fx_snap, g.Fy_snap, g.Fz_snap], a=dx, b=dt)
        if twin.enable_lorentz:
            g.ensure_lorentz_fields()
            for name, t in (("CurrentDensity_X_Am2", g.Jx), ("CurrentDensity_Y_Am2", g.Jy),
                            ("CurrentDensity_Z_Am2", g.Jz), ("MagneticField_X_T", g.Bx),
                            ("MagneticField_Y_T", g.By), ("MagneticField_Z_T", g.Bz)):
                add(name, N.EXPORT_COPY, [t])
    if TIER_DERIVED in tiers:
        add("Curvature_kappa", N.EXPORT_COPY, [g.kappa_field])
        add("Vorticity_mag_1s", N.EXPORT_COPY, [g.vorticity_mag])
        add("Mushy_Zone", N.EXPORT_MUSHY, [g.f_l])
    return ch


def gather_volume(twin, tiers=(TIER_CORE, TIER_DERIVED)):
    """{name: numpy array in VTK cell order (x fastest)} for the volume tiers:
    one pack launch and one device-to-host copy."""
    g = twin.grid
    tiers = tuple(TIER_MAP.get(t, t) for t in tiers)
    _prepare_derived(twin, tiers)
    ch = volume_channels(twin, tiers)
    n = g.n_cells
    stage = torch.empty(len(ch) * n, dtype=torch.int32, device=g.device)
    for lo in range(0, len(ch), N.MAX_EXPORT_CHANNELS):
        part = ch[lo:lo + N.MAX_EXPORT_CHANNELS]
        kernels.export_pack([c for _, _, c in part], g.nx, g.ny, g.nz, stage[lo * n:])
    host = stage.cpu().numpy()
    out = {}
    for q, (name, typ, _) in enumerate(ch):
        raw = host[q * n:(q + 1) * n]
        out[name] = raw if typ == _I32 else raw.view(np.float32)
    return out


# ---- VTK XML (raw appended, UInt64 headers) -------------------------------
_VTK_TYPES = {np.dtype(np.float32): "Float32", np.dtype(np.int32): "Int32",
              np.dtype(np.int64): "Int64", np.dtype(np.uint8): "UInt8",
              np.dtype(np.float64): "Float64"}
_NP_TYPES = {v: k for k, v in _VTK_TYPES.items()}


class _Appended:
    def __init__(self):
        self.blocks, self.offset = [], 0

    def add(self, arr):
        data = np.ascontiguousarray(arr).tobytes()
        off = self.offset
        self.blocks.append(np.array([len(data)], dtype="<u8").tobytes() + data)
        self.offset += 8 + len(data)
        return off


def _array_tag(name, arr, app, ncomp=1):
    return ('<DataArray type="%s" Name="%s" NumberOfComponents="%d" format="appended" '
            'offset="%d"/>' % (_VTK_TYPES[np.asarray(arr).dtype], name, ncomp, app.add(arr)))


def _write_vtk(path, head_lines, app):
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "wb") as fh:
        fh.write("\n".join(head_lines).encode())
        fh.write(b'\n  <AppendedData encoding="raw">\n   _')
        for b in app.blocks:
            fh.write(b)
        fh.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return str(path)


def write_vti(path, nx, ny, nz, spacing, origin, cell_arrays):
    """ImageData with nx*ny*nz cells; arrays in VTK cell order."""
    app = _Appended()
    ext = "0 %d 0 %d 0 %d" % (nx, ny, nz)
    lines = ['<?xml version="1.0"?>',
             '<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" '
             'header_type="UInt64">',
             '  <ImageData WholeExtent="%s" Origin="%.9g %.9g %.9g" Spacing="%.9g %.9g %.9g">'
             % ((ext,) + tuple(origin) + tuple(spacing)),
             '    <Piece Extent="%s">' % ext, "      <CellData>"]
    for name, arr in cell_arrays.items():
        lines.append("        " + _array_tag(name, arr, app))
    lines += ["      </CellData>", "    </Piece>", "  </ImageData>"]
    return _write_vtk(path, lines, app)


def write_vtp_points(path, points, point_arrays):
    """PolyData of points, one vertex cell per point."""
    pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    npt = pts.shape[0]
    app = _Appended()
    lines = ['<?xml version="1.0"?>',
             '<VTKFile type="PolyData" version="1.0" byte_order="LittleEndian" '
             'header_type="UInt64">',
             "  <PolyData>",
             '    <Piece NumberOfPoints="%d" NumberOfVerts="%d" NumberOfLines="0" '
             'NumberOfStrips="0" NumberOfPolys="0">' % (npt, npt), "      <PointData>"]
    for name, arr in point_arrays.items():
        lines.append("        " + _array_tag(name, arr, app))
    lines += ["      </PointData>", "      <Points>",
              "        " + _array_tag("Points", pts, app, ncomp=3), "      </Points>",
              "      <Verts>",
              "        " + _array_tag("connectivity", np.arange(npt, dtype=np.int64), app),
              "        " + _array_tag("offsets", np.arange(1, npt + 1, dtype=np.int64), app),
              "      </Verts>", "    </Piece>", "  </PolyData>"]
    return _write_vtk(path, lines, app)


def write_vtp_triangles(path, points, tris, point_arrays):
    """PolyData of triangles (tris: (T, 3) vertex indices)."""
    pts = np.ascontiguousarray(points, dtype=np.float32).reshape(-1, 3)
    tris = np.ascontiguousarray(tris, dtype=np.int64).reshape(-1, 3)
    app = _Appended()
    lines = ['<?xml version="1.0"?>',
             '<VTKFile type="PolyData" version="1.0" byte_order="LittleEndian" '
             'header_type="UInt64">',
             "  <PolyData>",
             '    <Piece NumberOfPoints="%d" NumberOfVerts="0" NumberOfLines="0" '
             'NumberOfStrips="0" NumberOfPolys="%d">' % (pts.shape[0], tris.shape[0]),
             "      <PointData>"]
    for name, arr in point_arrays.items():
        lines.append("        " + _array_tag(name, arr, app))
    lines += ["      </PointData>", "      <Points>",
              "        " + _array_tag("Points", pts, app, ncomp=3), "      </Points>",
              "      <Polys>",
              "        " + _array_tag("connectivity", tris.reshape(-1), app),
              "        " + _array_tag("offsets", 3 * np.arange(1, tris.shape[0] + 1,
                                                           dtype=np.int64), app),
              "      </Polys>", "    </Piece>", "  </PolyData>"]
    return _write_vtk(path, lines, app)


VTK_VOXEL = 11


def write_vtu_voxels(path, nx, ny, nz, spacing, origin, cell_ids, cell_arrays):
    """UnstructuredGrid of the voxels cell_ids (VTK cell order of an nx*ny*nz
    ImageData), points shared, arrays given per kept cell."""
    cell_ids = np.asarray(cell_ids, dtype=np.int64)
    i = cell_ids % nx
    j = (cell_ids // nx) % ny
    k = cell_ids // (nx * ny)
    # voxel corner order: x fastest, then y, then z
    di = np.array([0, 1, 0, 1, 0, 1, 0, 1])
    dj = np.array([0, 0, 1, 1, 0, 0, 1, 1])
    dk = np.array([0, 0, 0, 0, 1, 1, 1, 1])
    corner = ((i[:, None] + di) + (nx + 1) * ((j[:, None] + dj) + (ny + 1) * (k[:, None] + dk)))
    uniq, inv = np.unique(corner.reshape(-1), return_inverse=True)
    I = uniq % (nx + 1)
    J = (uniq // (nx + 1)) % (ny + 1)
    K = uniq // ((nx + 1) * (ny + 1))
    pts = np.stack([origin[0] + spacing[0] * I, origin[1] + spacing[1] * J,
                    origin[2] + spacing[2] * K], axis=1).astype(np.float32)
    nc = cell_ids.shape[0]
    app = _Appended()
    lines = ['<?xml version="1.0"?>',
             '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian" '
             'header_type="UInt64">',
             "  <UnstructuredGrid>",
             '    <Piece NumberOfPoints="%d" NumberOfCells="%d">' % (pts.shape[0], nc),
             "      <CellData>"]
    for name, arr in cell_arrays.items():
        lines.append("        " + _array_tag(name, arr, app))
    lines += ["      </CellData>", "      <Points>",
              "        " + _array_tag("Points", pts, app, ncomp=3), "      </Points>",
              "      <Cells>",
              "        " + _array_tag("connectivity", inv.astype(np.int64), app),
              "        " + _array_tag("offsets", 8 * np.arange(1, nc + 1, dtype=np.int64), app),
              "        " + _array_tag("types", np.full(nc, VTK_VOXEL, dtype=np.uint8), app),
              "      </Cells>", "    </Piece>", "  </UnstructuredGrid>"]
    return _write_vtk(path, lines, app)


def read_vtk_xml(path):
    """Arrays of a raw-appended VTK XML file written here: {name: array}, plus
    "_attrs" with the dataset element's attributes."""
    raw = pathlib.Path(path).read_bytes()
    start = raw.index(b'<AppendedData encoding="raw">')
    body = raw.index(b"_", start) + 1
    root = ET.fromstring(raw[:start].decode() + "</VTKFile>")
    out = {"_attrs": dict(root[0].attrib)}
    for da in root.iter("DataArray"):
        off = body + int(da.get("offset"))
        nbytes = int(np.frombuffer(raw[off:off + 8], dtype="<u8")[0])
        arr = np.frombuffer(raw[off + 8:off + 8 + nbytes], dtype=_NP_TYPES[da.get("type")])
        ncomp = int(da.get("NumberOfComponents", "1"))
        out[da.get("Name")] = arr.reshape(-1, ncomp) if ncomp > 1 else arr
    return out


# ---- reference export entry points -----------------------------------------
def export_volume(twin, path, tiers=(TIER_CORE, TIER_DERIVED), crop_liquid=False):
    """vtk_io.py:82-166.  crop_liquid: only the cells with Liquid_Fraction >= 0.05
    (vtk_io.py:170-171), written as an UnstructuredGrid (``.vtu``; the
    reference's threshold output is unstructured too, which its ``.vti`` name
    does not fit).  Returns None when no cell qualifies."""
    g = twin.grid
    arrays = gather_volume(twin, tiers)
    spacing = (g.dx * 1000.0,) * 3
    origin = (twin._window_offset_x_m * 1000.0, 0.0, 0.0)
    if crop_liquid and "Liquid_Fraction" in arrays:
        keep = np.nonzero(arrays["Liquid_Fraction"] >= np.float32(0.05))[0]
        if keep.size == 0:
            return None
        out = str(pathlib.Path(vtk_imagedata_path(path)).with_suffix(".vtu"))
        return write_vtu_voxels(out, g.nx, g.ny, g.nz, spacing, origin, keep,
                                {k: np.ascontiguousarray(v[keep]) for k, v in arrays.items()})
    out = vtk_imagedata_path(path)
    write_vti(out, g.nx, g.ny, g.nz, spacing, origin, arrays)
    return out


def isosurface(g, iso_cells, attr_cells, iso=0.5, spacing=1.0, origin=(0.0, 0.0, 0.0)):
    """Marching-tetrahedra isosurface of a cell field at ``iso`` after the
    cell-to-corner averaging: (points (V, 3), triangles (T, 3), interpolated
    attributes (V, len(attr_cells))), vertices merged by lattice edge, order
    fixed.  None when the surface is empty."""
    nx, ny, nz = g.nx, g.ny, g.nz
    npts = (nx + 1) * (ny + 1) * (nz + 1)
    fields = [iso_cells] + list(attr_cells)
    if len(fields) > 4:
        raise ValueError("isosurface: at most three attributes")
    pts = torch.empty((len(fields), npts), dtype=torch.float32, device=g.device)
    cptr = [t.data_ptr() for t in fields] + [None] * (4 - len(fields))
    pptr = [pts[m].data_ptr() for m in range(len(fields))] + [None] * (4 - len(fields))
    st = torch.cuda.current_stream().cuda_stream
    N.call("waam_cell_to_point", *cptr, *pptr, nx, ny, nz, st)
    count = torch.zeros(1, dtype=torch.int64, device=g.device)
    cap = max(1 << 16, 4 * (nx * ny + ny * nz + nx * nz))
    na = len(attr_cells)
    aptr = [pts[1 + m].data_ptr() for m in range(na)] + [None] * (3 - na)
    while True:
        keys = torch.empty(3 * cap, dtype=torch.int64, device=g.device)
        vals = torch.empty((3 * cap, 6), dtype=torch.float32, device=g.device)
        order = torch.empty(cap, dtype=torch.int64, device=g.device)
        N.call("waam_isosurface", pts[0].data_ptr(), *aptr, nx, ny, nz, float(iso),
               float(spacing), float(origin[0]), float(origin[1]), float(origin[2]),
               keys.data_ptr(), vals.data_ptr(), order.data_ptr(), count.data_ptr(), cap, st)
        n_tri = int(count.item())
        if n_tri <= cap:
            break
        cap = n_tri
    if n_tri == 0:
        return None
    order_h = order[:n_tri].cpu().numpy()
    perm = np.argsort(order_h, kind="stable")
    keys_h = keys[:3 * n_tri].cpu().numpy().reshape(n_tri, 3)[perm].reshape(-1)
    vals_h = vals[:3 * n_tri].cpu().numpy().reshape(n_tri, 3, 6)[perm].reshape(-1, 6)
    uniq, first, inv = np.unique(keys_h, return_index=True, return_inverse=True)
    verts = vals_h[first]
    return verts[:, :3], inv.reshape(n_tri, 3), verts[:, 3:3 + na]


def export_surface(twin, path, include_kappa=True):
    """vtk_io.py:180-224: the phi = 0.5 surface (the bead's free surface), or the
    f_l = 0.5 surface when phi has none, as PolyData with the corner-averaged
    phi, Liquid_Fraction, Temperature_K (and Curvature_kappa) interpolated to
    its vertices.  Returns None when neither surface exists."""
    g = twin.grid
    if include_kappa:
        g.ensure_export_buffers()
        kernels.compute_curvature_field(g.phi, g.flags, g.kappa_field, g.FLAG_GAS, g.nx, g.ny,
                                        g.nz)
    names = {"phi": g.phi, "Liquid_Fraction": g.f_l, "Temperature_K": g.T}
    if include_kappa:
        names["Curvature_kappa"] = g.kappa_field
    h = g.dx * 1000.0
    origin = (twin._window_offset_x_m * 1000.0, 0.0, 0.0)
    for scalar in ("phi", "Liquid_Fraction"):
        others = [k for k in names if k != scalar]
        surf = isosurface(g, names[scalar], [names[k] for k in others], 0.5, h, origin)
        if surf is None:
            continue
        verts, tris, attrs = surf
        point_arrays = {}
        for k in names:
            if k == scalar:
                point_arrays[k] = np.full(verts.shape[0], 0.5, dtype=np.float32)
            else:
                point_arrays[k] = np.ascontiguousarray(attrs[:, others.index(k)])
        return write_vtp_triangles(path, verts, tris, point_arrays)
    return None


def export_tracers(twin, path):
    """vtk_io.py:227-255: active tracers in mm (world x), state and trapped."""
    g = twin.grid
    pos = g.porosity_pos.cpu().numpy()
    active = g.porosity_active.cpu().numpy()
    mask = active > 0
    if not mask.any():
        return None
    pts = pos[mask].copy()
    pts[:, 0] += twin._window_offset_x_m
    pts *= 1000.0
    return write_vtp_points(path, pts, {"state": active[mask].astype(np.int32),
                                        "trapped": (active[mask] == 2).astype(np.int32)})


def export_npz(twin, path):
    """The raw state (grid.state_dict) plus the time and window offset, for
    Python post-processing."""
    st = twin.grid.state_dict()
    st["step"] = np.array(twin._step_n)
    st["dx"] = np.array(twin.grid.dx)
    st["dt"] = np.array(twin.grid.dt)
    st["window_offset_x_m"] = np.array(twin._window_offset_x_m)
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    np.savez_compressed(path, **st)
    return str(path)


def build_meta_dict(twin, job_path=None):
    """meta.py:15-95."""
    g = twin.grid
    mat = twin.mat
    telem = twin.get_telemetry()
    job = getattr(twin, "_job_config", None)
    r3 = lambda v: round(float(v), 3)  # noqa: E731
    meta = {
        "waam_twin_version": WAAM_TWIN_VERSION,
        "step": twin._step_n,
        "sim_time_ms": telem["sim_time_ms"],
        "grid": {"nx": g.nx, "ny": g.ny, "nz": g.nz, "dx_mm": round(g.dx * 1000.0, 6),
                 "dt_us": round(g.dt * 1e6, 4)},
        "origin_mm": [round(twin._window_offset_x_m * 1000.0, 4), 0.0, 0.0],
        "window_offset_x_mm": telem["window_offset_x_mm"],
        "preset": getattr(twin, "preset_name", None),
        "plate_thickness_mm": (None if getattr(twin, "plate_thickness_mm", None) is None
                               else r3(twin.plate_thickness_mm)),
        "plate_size_mm": (None if not getattr(twin, "plate_size_mm", None)
                          else [r3(twin.plate_size_mm[0]), r3(twin.plate_size_mm[1])]),
        "plate_origin_mm": (None if not getattr(twin, "plate_origin_mm", None)
                            else [r3(twin.plate_origin_mm[0]), r3(twin.plate_origin_mm[1])]),
        "plate_ij": list(twin.resolve_plate_ij()),
        "nz_solid": int(twin.nz_solid),
        "substrate_thickness_mm": round(float(twin.nz_solid) * g.dx * 1000.0, 3),
        "material": {"name": mat.name, "status": mat.status, "T_solidus_K": mat.T_solidus,
                     "T_liquidus_K": mat.T_liquidus, "rho_kgm3": mat.rho},
        "physics_flags": {
            "enable_vof": twin.enable_vof, "enable_csf_tension": twin.enable_csf_tension,
            "enable_recoil": twin.enable_recoil,
            "use_recoil_clausius_clapeyron": twin.use_recoil_clausius_clapeyron,
            "enable_lorentz": twin.enable_lorentz, "enable_gas_shear": twin.enable_gas_shear,
            "enable_droplet_impact_pressure": twin.enable_droplet_impact_pressure,
            "enable_substrate_growth": twin.enable_substrate_growth,
            "enable_moving_window": twin.enable_moving_window,
            "enable_wetting": twin.enable_wetting,
            "enable_hydrostatic_gravity": twin.enable_hydrostatic_gravity,
            "enable_bead_freeze": twin.enable_bead_freeze, "enable_ctwd": twin.enable_ctwd,
            "contact_angle_deg": twin.contact_angle_deg,
            "enable_heat_loss": twin.enable_heat_loss, "C_darcy": twin.C_darcy,
            "heat_source": twin.heat_source_name, "welding_current_A": twin.welding_current_A},
        "unit_conversions": {
            "velocity_lu_to_ms": "u_ms = u_lu * dx / dt",
            "force_lu_to_ms2": "a_ms2 = F_lu * dx / dt^2",
            "pressure_pa_gauge": "P = (rho_lu - 1) * cs^2 * rho_phys * (dx/dt)^2"},
        "telemetry": telem,
    }
    if job_path:
        meta["job_path"] = job_path
    if job:
        meta["process"] = job.get("process", {})
        meta["reference"] = job.get("reference", {})
    return meta


def write_meta_json(twin, path, job_path=None):
    path = pathlib.Path(path)
    path.parent.mkdir(parents=True, exist_ok=True)
    with open(path, "w") as f:
        json.dump(build_meta_dict(twin, job_path), f, indent=2)


def export_research_bundle(twin, out_dir, tag=None, tiers=(0, 1, 3), include_surface=True,
                           include_tracers=True, include_sidecar=True, crop_liquid=False,
                           job_path=None):
    """bundle.py:36-98: volume, tracers, telemetry, metadata, probes."""
    out_dir = pathlib.Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    tier_tuple = tuple(TIER_MAP.get(t, t) for t in tiers)
    step_tag = tag or "step_%06d" % twin._step_n
    paths = {}
    p = export_volume(twin, str(out_dir / ("volume_%s.vti" % step_tag)), tiers=tier_tuple,
                      crop_liquid=crop_liquid)
    if p:
        paths["volume"] = p
    if include_surface and twin.enable_vof:
        p = export_surface(twin, str(out_dir / ("surface_%s.vtp" % step_tag)))
        if p:
            paths["surface"] = p
    if include_tracers:
        p = export_tracers(twin, str(out_dir / ("tracers_%s.vtp" % step_tag)))
        if p:
            paths["tracers"] = p
    telem_path = out_dir / ("telemetry_%s.json" % step_tag)
    with open(telem_path, "w") as f:
        json.dump(twin.get_telemetry(), f, indent=2)
    paths["telemetry"] = str(telem_path)
    if include_sidecar:
        meta_path = out_dir / ("meta_%s.json" % step_tag)
        write_meta_json(twin, meta_path, job_path=job_path)
        paths["meta"] = str(meta_path)
    rec = getattr(twin, "probe_recorder", None)
    if rec is not None and rec.probes:
        probe_path = out_dir / "probes.csv"
        rec.write_csv(probe_path)
        paths["probes"] = str(probe_path)
    return paths


def write_pvd(collection_path, vti_paths, times_s=None):
    """bundle.py:101-131: ParaView collection, paths relative to the .pvd."""
    collection_path = pathlib.Path(collection_path).resolve()
    pvd_dir = collection_path.parent
    lines = ['<?xml version="1.0"?>', '<VTKFile type="Collection" version="0.1">',
             "  <Collection>"]
    for i, vti in enumerate(vti_paths):
        p = pathlib.Path(vti)
        p = (pathlib.Path.cwd() / p).resolve() if not p.is_absolute() else p.resolve()
        try:
            rel = p.relative_to(pvd_dir)
        except ValueError:
            rel = pathlib.Path(p.name)
        t = times_s[i] if times_s is not None and i < len(times_s) else float(i)
        lines.append('    <DataSet timestep="%.9g" file="%s"/>' % (t, rel.as_posix()))
    lines += ["  </Collection>", "</VTKFile>"]
    collection_path.write_text("\n".join(lines))


def export_research_sequence(twin, out_dir, n_steps, every_n=100, torch_x_m=0.01,
                             torch_y_m=None, is_welding=True, max_frames=200, tiers=(0, 3),
                             job_path=None, after_frame=None):
    """bundle.py:134-170: step, export a bundle every ``every_n`` steps, write the
    .pvd of the volumes."""
    out_dir = pathlib.Path(out_dir)
    out_dir.mkdir(parents=True, exist_ok=True)
    g = twin.grid
    if torch_y_m is None:
        torch_y_m = (g.ny // 2) * g.dx
    vti_paths, times = [], []
    frame = 0
    for step_i in range(n_steps):
        twin.step(torch_x_m, torch_y_m, is_welding=is_welding)
        if step_i % every_n != 0 and step_i != n_steps - 1:
            continue
        if frame >= max_frames:
            break
        sub = out_dir / ("frame_%04d" % frame)
        paths = export_research_bundle(twin, sub, tag="step_%06d" % twin._step_n, tiers=tiers,
                                       include_surface=True,
                                       include_tracers=(frame == 0 or frame % 5 == 0),
                                       job_path=job_path)
        if after_frame is not None:
            after_frame(frame, sub, paths)
        if "volume" in paths:
            vti_paths.append(paths["volume"])
            times.append(twin._step_n * g.dt)
        frame += 1
    if vti_paths:
        write_pvd(out_dir / "sequence.pvd", vti_paths, times_s=times)
    return vti_paths
