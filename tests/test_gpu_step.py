"""Full coupled steps on the GPU: the fused pipeline and the operator-by-
operator driver against the reference's own steps (golden fixtures), against
the CPU oracle on larger configurations, and run-to-run determinism."""
import numpy as np
import pytest
import torch

import cases
import steps
from gpu_twins import set_host_state, twin_for_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mode", ["fused", "operators"])
@pytest.mark.parametrize("name", steps.STEP_CASES)
def test_single_steps_match_reference(name, mode):
    tw, sc, extra, states, positions = twin_for_case(name, mode)
    for s in range(len(states) - 1):
        tw.grid.load_state(states[s])
        set_host_state(tw, name, s, extra, positions)
        x, y = positions[s]
        tw.step(float(x), float(y), True)
        torch.cuda.synchronize()
        got = tw.grid.state_dict()
        assert got["read_is_a"] == states[s + 1]["read_is_a"]
        steps.compare_state("%s/%s step %d" % (name, mode, s), got, states[s + 1],
                            fields=steps.fields_for(name), reference=True)


@pytest.mark.parametrize("name", steps.STEP_CASES)
def test_fused_matches_oracle_over_trajectory(name):
    from test_oracle_steps import make_oracle
    tw, sc, extra, states, positions = twin_for_case(name, "fused")
    ot = make_oracle(name)[0]
    tw.grid.load_state(states[0])
    set_host_state(tw, name, 0, extra, positions)
    ot.load(states[0])
    ot.last_drop = extra.get("last_drop", 0.0)
    for x, y in positions[: len(states) - 1]:
        tw.step(float(x), float(y), True)
        ot.step(float(x), float(y), True)
    torch.cuda.synchronize()
    steps.compare_state("%s fused vs oracle" % name, tw.grid.state_dict(), ot.s,
                        fields=steps.fields_for(name))


def _config_twins(kind, nx, ny, nz, material=None, **more):
    """A c1-like (Gaussian, no wire) or c2-like (Goldak, 100 Hz droplets, wetting,
    CSF, hydrostatic) run from reset, on the GPU and on the oracle.  ``material``:
    (MaterialProps, oracle constants, oracle tables) of steps.material_for."""
    from oracle.oracle_step import OracleTwin
    from waam_solver_b200 import WAAMTwin
    from waam_solver_b200.materials import from_constants
    from waam_solver_b200.physics.arc import Goldak3D
    dx = 2.5e-4 if kind == "c1" else 2e-4
    common = dict(use_srt=False, enable_vof=True, travel_speed_m_s=0.008)
    if kind == "c1":
        kw = dict(heat_source="gaussian2d", arc_power_W=3000.0, arc_efficiency=0.75,
                  arc_sigma_mm=1.0, droplet_freq_hz=0.0, **common)
        host = {}
        goldak = None
    else:
        kw = dict(heat_source="goldak", arc_power_W=4000.0, arc_efficiency=0.78,
                  arc_sigma_mm=1.0, droplet_freq_hz=100.0, enable_wetting=True,
                  enable_csf_tension=True, enable_hydrostatic_gravity=True, **common)
        host = dict(wire_feed_m_s=0.1, droplet_transfer_mode="pulsed", pulse_frequency_hz=100.0,
                    droplet_size_jitter=0.0)
        goldak = dict(ff=0.6, fr=1.4, a_front=5.0, a_rear=12.0, b=5.0, c=4.0)
    kw.update(more)
    mat = from_constants("m", steps.MATERIAL, contact_angle_deg=30.0)
    omat, otables = steps.MATERIAL, None
    if material is not None:
        import dataclasses
        mat, omat, otables = material
        mat = dataclasses.replace(mat, contact_angle_deg=30.0)
        omat = {k: v for k, v in omat.items() if k != "contact_angle_deg"}
    tw = WAAMTwin(material=mat, nx=nx, ny=ny, nz=nz, dx=dx, max_tracers=64, **kw)
    for k, v in host.items():
        setattr(tw, k, v)
    if goldak:
        tw.arc_source = Goldak3D(**goldak)
    tw.reset()
    okw = {k: v for k, v in kw.items() if k not in ("step_mode", "population_dtype")}
    ot = OracleTwin(nx, ny, nz, dx, omat, goldak=goldak, tables=otables, contact_angle_deg=30.0,
                    **okw, **host)
    ot.reset()
    return tw, ot, dx


@pytest.mark.parametrize("kind,shape,n_steps", [("c1", (48, 24, 24), 30),
                                                 ("c2", (56, 32, 28), 30)])
def test_fused_matches_oracle_from_reset(kind, shape, n_steps):
    tw, ot, dx = _config_twins(kind, *shape)
    # seed a molten state so every operator is active from the first step
    import state_gen
    st = state_gen.seeded_state(*shape, seed=7, nz_solid=tw.nz_solid)
    st["read_is_a"] = True
    tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
    ot.load({k: v for k, v in st.items() if k != "nz_solid"})
    if kind == "c2":
        tw._last_droplet_time = -1.0
        ot.last_drop = -1.0
    y = (shape[1] // 2) * dx
    for s in range(n_steps):
        x = 0.3 * shape[0] * dx + s * 0.008 * dx * 0.1
        tw.step(x, y, True)
        ot.step(x, y, True)
        torch.cuda.synchronize()
        steps.compare_state("%s step %d" % (kind, s), tw.grid.state_dict(), ot.s)
    if kind == "c2":
        assert tw._n_droplets_fired == ot.n_drops >= 1
        assert abs(tw._deposited_volume_m3 - ot.deposited) <= 1e-6 * max(ot.deposited, 1e-30)
        # porosity tracers spawned by the droplets and advected every step
        g = tw.grid
        assert int(g.tracer_head.item()) == int(ot.s["tracer_head"][0]) >= 50
        assert np.array_equal(g.porosity_active.cpu().numpy(), ot.s["porosity_active"])
        steps.compare("tracers", g.porosity_pos.cpu().numpy(), ot.s["porosity_pos"],
                      "porosity_pos")


def test_fused_is_deterministic():
    runs = []
    for _ in range(2):
        tw, ot, dx = _config_twins("c2", 40, 24, 24)
        tw._last_droplet_time = -1.0
        for s in range(12):
            tw.step(0.3 * 40 * dx + s * 1e-6, 12 * dx, True)
        torch.cuda.synchronize()
        runs.append(tw.grid.state_dict())
    for k, v in runs[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, runs[1][k]), k


def test_graph_replay_matches_eager_launches():
    """Steps replayed from captured CUDA graphs equal eagerly launched steps bitwise."""
    states = []
    for graphs in (False, True):
        tw, ot, dx = _config_twins("c2", 40, 24, 24)
        tw.use_cuda_graphs = graphs
        tw._last_droplet_time = -1.0
        for s in range(16):
            tw.step(0.3 * 40 * dx + s * 1e-6, 12 * dx, True)
        torch.cuda.synchronize()
        if graphs:
            assert any(e["graph"] is not None for e in tw._graphs.values())
        states.append(tw.grid.state_dict())
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, states[1][k]), k


@pytest.mark.parametrize("step_mode", ["fused", "operators"])
@pytest.mark.parametrize("cc", [True, False])
def test_recoil_and_gas_shear_steps_match_oracle(step_mode, cc):
    """Vapour recoil (Clausius-Clapeyron or T-ratio form) and shielding-gas shear
    on: steps from a seeded hot pool against the oracle, in the fused step (both
    terms inside the collision's force assembly) and through the operators."""
    import state_gen
    shape = (40, 24, 24)
    tw, ot, dx = _config_twins("c2", *shape, enable_recoil=True, enable_gas_shear=True,
                               use_recoil_clausius_clapeyron=cc, step_mode=step_mode)
    st = state_gen.seeded_state(*shape, seed=9, nz_solid=tw.nz_solid)
    T = st["T"]
    hot = (st["flags"] == 4) | (st["flags"] == 0)
    st["T"] = np.where(hot, np.maximum(T, 3150.0), T).astype(np.float32)
    st["read_is_a"] = True
    tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
    ot.load({k: v for k, v in st.items() if k != "nz_solid"})
    y = (shape[1] // 2) * dx
    for s in range(4):
        x = 0.3 * shape[0] * dx + s * 0.008 * dx * 0.1
        tw.step(x, y, True)
        ot.step(x, y, True)
        torch.cuda.synchronize()
        steps.compare_state("recoil step %d" % s, tw.grid.state_dict(), ot.s)


@pytest.mark.parametrize("dtype", ["float32", "float16"])
@pytest.mark.parametrize("lorentz", [False, True])
def test_pipelined_stream_matches_in_order_stream(lorentz, dtype):
    """Each step's stream left to run beside the next step's arc, thermal and VOF
    stages (joined before the column pass) gives the same states, bit for bit,
    as the stream run in order -- and so does the collision left pending as
    well, and the stream held back one more step to run beside the next
    collision on the cells it does not write (lagged) -- over droplet steps,
    graph replays and the Lorentz split step, in float32 and 16-bit population
    storage; the state read-out runs the pending work."""
    states = []
    more = dict(enable_lorentz=True, welding_current_A=180.0) if lorentz else {}
    more["population_dtype"] = dtype
    for mode in ("in_order", "stream", "stream_collide", "lagged"):
        tw, ot, dx = _config_twins("c2", 40, 24, 24, **more)
        tw.pipeline_stream = mode != "in_order"
        tw.pipeline_collide = mode in ("stream_collide", "lagged")
        tw.pipeline_lag_stream = mode == "lagged"
        tw._last_droplet_time = -1.0
        for s in range(24):
            # a non-welding stretch switches the arc off and on
            tw.step(0.3 * 40 * dx + s * 1e-6, 12 * dx, not 10 <= s < 13)
        g = tw.grid
        if mode != "in_order":
            assert g._stream_pending
        if mode in ("stream_collide", "lagged") and not lorentz:
            assert g._collide_pending
            assert g.__dict__.get("_lag_pending", False) == (mode == "lagged")
            u = g.ux.clone()              # reading a collision output runs the pending work
            assert not g._collide_pending and not g._stream_pending
            assert not g._lag_pending
        torch.cuda.synchronize()
        states.append(g.state_dict())
        assert tw._n_droplets_fired >= 1
    for other in states[1:]:
        for k, v in states[0].items():
            if isinstance(v, np.ndarray):
                assert np.array_equal(v, other[k]), k


LORENTZ_FIELDS = ("phi_elec", "Jx", "Jy", "Jz", "Bx", "By", "Bz", "elec_rad_bins")


@pytest.mark.parametrize("step_mode", ["fused", "operators"])
def test_lorentz_steps_match_oracle(step_mode):
    """Welding current on: the potential solve (cold start, then warm), J, B and
    J x B, step by step against the oracle -- in the fused step (J x B added
    inside the collision, before the force clamp) and through the operators."""
    shape = (40, 24, 24)
    tw, ot, dx = _config_twins("c2", *shape, enable_lorentz=True, welding_current_A=180.0,
                               lorentz_jacobi_iters=40, step_mode=step_mode)
    import state_gen
    st = state_gen.seeded_state(*shape, seed=9, nz_solid=tw.nz_solid)
    st["read_is_a"] = True
    tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
    ot.load({k: v for k, v in st.items() if k != "nz_solid"})
    y = (shape[1] // 2) * dx
    for s in range(5):
        x = 0.3 * shape[0] * dx + s * 0.008 * dx * 0.1
        tw.step(x, y, True)
        ot.step(x, y, True)
        torch.cuda.synchronize()
        assert tw._lorentz_last_iters == ot.lorentz_iters[-1], (s, tw._lorentz_last_iters,
                                                                ot.lorentz_iters)
        g = tw.grid
        got = {f: getattr(g, f).cpu().numpy() for f in LORENTZ_FIELDS}
        steps.compare_state("lorentz step %d" % s, dict(tw.grid.state_dict(), **got),
                            ot.s, fields=steps.FIELDS + list(LORENTZ_FIELDS))
    assert ot.lorentz_iters[0] > ot.lorentz_iters[-1]    # cold start, then warm starts


def test_overlapped_step_matches_serial_stage_timing_path():
    """The fused step with its second-stream overlap equals the serial path
    that records stage events, bit for bit."""
    states = []
    for timed in (False, True):
        tw, ot, dx = _config_twins("c2", 40, 24, 24)
        tw.use_cuda_graphs = False
        tw._last_droplet_time = -1.0
        for s in range(8):
            if timed:
                evs = [torch.cuda.Event(enable_timing=True) for _ in range(7)]
                for e in evs:
                    e.record()      # torch creates the CUDA event on its first record
                tw._stage_events = evs
            tw.step(0.3 * 40 * dx + s * 1e-6, 12 * dx, True)
        tw._stage_events = None
        torch.cuda.synchronize()
        states.append(tw.grid.state_dict())
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, states[1][k]), k


def _table_material():
    """The validated ER70S-6 file as the reference loads it (tables + Sahoo)."""
    sc, kw, states, positions = steps.load_step_case("t1_plate")
    opt, extra = steps.driver_options("t1_plate", sc, kw)
    return steps.material_for("t1_plate", extra)


@pytest.mark.parametrize("variable_tau", [True, False])
def test_table_path_matches_oracle_from_seeded_pool(variable_tau):
    """Material tables on a c2-like run (droplets, wetting, CSF, heat losses,
    substrate growth and trailing freeze): every step of the fused pipeline
    against the oracle, property fields included; the variable-tau SRT or,
    with use_variable_tau off, the MRT collision."""
    shape = (40, 24, 24)
    tw, ot, dx = _config_twins("c2", *shape, material=_table_material(),
                               use_variable_tau=variable_tau, enable_heat_loss=True,
                               enable_substrate_growth=True, enable_bead_freeze=True)
    assert tw.use_material_tables and ot.use_tables
    assert tw.H_sol == pytest.approx(ot.H_sol, rel=1e-14)
    import state_gen
    st = state_gen.seeded_state(*shape, seed=11, nz_solid=tw.nz_solid)
    st["read_is_a"] = True
    tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
    ot.load({k: v for k, v in st.items() if k != "nz_solid"})
    tw._last_droplet_time = -1.0
    ot.last_drop = -1.0
    y = (shape[1] // 2) * dx
    fields = steps.FIELDS + steps.PROP_FIELDS
    for s in range(16):
        x = 0.3 * shape[0] * dx + s * 0.008 * dx * 0.1
        tw.step(x, y, True)
        ot.step(x, y, True)
        torch.cuda.synchronize()
        steps.compare_state("tables step %d" % s, tw.grid.state_dict(), ot.s, fields=fields)
    assert tw._n_droplets_fired == ot.n_drops >= 1


def test_table_path_operators_equal_fused():
    """The operator-by-operator table path and the fused pipeline agree."""
    shape = (40, 24, 24)
    out = []
    for mode in ("operators", "fused"):
        tw, ot, dx = _config_twins("c1", *shape, material=_table_material(),
                                   enable_heat_loss=True, step_mode=mode)
        import state_gen
        st = state_gen.seeded_state(*shape, seed=12, nz_solid=tw.nz_solid)
        st["read_is_a"] = True
        tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
        for s in range(6):
            tw.step(0.3 * shape[0] * dx + s * 1e-6, (shape[1] // 2) * dx, True)
        torch.cuda.synchronize()
        out.append(tw.grid.state_dict())
    steps.compare_state("operators vs fused (tables)", out[0], out[1],
                        fields=steps.FIELDS + steps.PROP_FIELDS)


@pytest.mark.parametrize("kind,tables", [("c1", False), ("c2", True)])
def test_moving_window_matches_oracle(kind, tables):
    """enable_moving_window (twin.py:599-631): the torch crosses the trigger, all
    fields (and the tracers) move back in one launch, the run continues in the
    window's coordinates; every step against the oracle."""
    shape = (40, 24, 24)
    more = dict(enable_moving_window=True)
    if tables:
        more.update(material=_table_material(), enable_heat_loss=True)
    tw, ot, dx = _config_twins(kind, *shape, **more)
    import state_gen
    st = state_gen.seeded_state(*shape, seed=13, nz_solid=tw.nz_solid)
    st["read_is_a"] = True
    tw.grid.load_state({k: v for k, v in st.items() if k != "nz_solid"})
    ot.load({k: v for k, v in st.items() if k != "nz_solid"})
    if kind == "c2":
        tw._last_droplet_time = -1.0
        ot.last_drop = -1.0
    y = (shape[1] // 2) * dx
    fields = steps.FIELDS + (steps.PROP_FIELDS if tables else [])
    for s in range(10):
        x = 19.0 * dx + s * 0.25 * dx
        tw.step(x, y, True)
        ot.step(x, y, True)
        torch.cuda.synchronize()
        assert tw._window_offset_x_m == pytest.approx(ot.window_offset, abs=1e-15)
        steps.compare_state("window step %d" % s, tw.grid.state_dict(), ot.s, fields=fields)
    assert tw._window_offset_x_m > 0.0
    if kind == "c2":
        g = tw.grid
        assert np.array_equal(g.porosity_active.cpu().numpy(), ot.s["porosity_active"])
        steps.compare("tracers", g.porosity_pos.cpu().numpy(), ot.s["porosity_pos"],
                      "porosity_pos")


def test_operator_calls_after_pipelined_steps_see_streamed_populations():
    """After fused steps that leave their stream (and collision) pending, the
    kept operator API reads g.f_src / g.f_dst through the grid, which runs the
    pending work first: an operator-API collide + stream + swap after the
    steps gives, bit for bit, the state of the same calls after in-order
    steps."""
    from waam_solver_b200.physics import lbm
    states = []
    for pipelined in (False, True):
        tw, ot, dx = _config_twins("c2", 40, 24, 24)
        tw.pipeline_stream = tw.pipeline_collide = pipelined
        tw._last_droplet_time = -1.0
        for s in range(9):
            tw.step(0.3 * 40 * dx + s * 1e-6, 12 * dx, True)
        g = tw.grid
        if pipelined:
            assert g._stream_pending and g._collide_pending
        lbm.collide_mrt(g.f_src, g.f_dst, g.rho, g.ux, g.uy, g.uz, g.Fx, g.Fy, g.Fz, g.f_l,
                        g.flags, g.ex, g.ey, g.ez, g.w, g.opp, tw.omega, tw.omega_bulk,
                        tw.C_darcy, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
        assert not g._stream_pending and not g._collide_pending
        lbm.stream(g.f_dst, g.f_src, g.flags, g.FLAG_SOLID, g.FLAG_GAS, g.nx, g.ny, g.nz)
        g.swap_buffers()
        torch.cuda.synchronize()
        states.append(g.state_dict())
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, states[1][k]), k


@pytest.mark.parametrize("lorentz", [False, True])
def test_quiet_tile_skipping_matches_working_every_tile(lorentz):
    """Quiet-tile skipping with the lagged stream (the defaults) against every
    tile worked and the stream run one step earlier, bit for bit, on a grid
    tall enough for quiet tiles (nz = 96: three 32-cell k tiles over a
    19-cell plate), through droplet steps (the tile history restarts), graph
    replays and the pipelined stream and collision -- the lagged stream
    reads flag copies that quiet tiles must still write; the skipping really
    skips (the work list is shorter than the tile count).  With the welding
    current's Lorentz force (and VOF, so J x B stays on the active cells) the
    tiles are skipped on the split steps as well."""
    states, counts = [], []
    more = dict(enable_lorentz=True, welding_current_A=180.0) if lorentz else {}
    for skip in (False, True):
        tw, ot, dx = _config_twins("c2", 40, 32, 96, **more)
        tw.skip_quiet_tiles = skip
        tw.pipeline_lag_stream = skip
        tw._last_droplet_time = -1.0
        g = tw.grid
        n_tiles = g.tile_list.numel() - 1
        for s in range(40):
            tw.step(0.3 * 40 * dx + s * 1e-6, 16 * dx, not 25 <= s < 28)
            if s == 35:
                worked, total = g.worked_tiles()
                assert total == n_tiles
                counts.append(worked)
        torch.cuda.synchronize()
        states.append(g.state_dict())
    assert counts[0] == n_tiles and 0 < counts[1] < n_tiles, (counts, n_tiles)
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, states[1][k]), k


def test_quiet_tile_history_restarts_after_operator_calls():
    """An operator-API call that writes flags / phi / f_l / H / T between fused
    steps (here update_flags_from_phi) restarts the quiet-tile history: the
    next step works every tile; so do load_state and invalidate()."""
    from waam_solver_b200 import kernels
    tw, ot, dx = _config_twins("c2", 40, 32, 96)
    g = tw.grid
    for s in range(4):
        tw.step(0.3 * 40 * dx + s * 1e-6, 16 * dx, True)
    assert tw._fused_params.tile_skip == 1
    kernels.update_flags_from_phi(g.phi, g.f_l, g.flags, tw.nz_solid, 0, 1, 2, 4)
    tw.step(0.3 * 40 * dx + 5e-6, 16 * dx, True)
    assert tw._fused_params.tile_skip == 0
    tw.step(0.3 * 40 * dx + 6e-6, 16 * dx, True)
    assert tw._fused_params.tile_skip == 1
    g.load_state(g.state_dict())
    tw.step(0.3 * 40 * dx + 7e-6, 16 * dx, True)
    assert tw._fused_params.tile_skip == 0
    tw.step(0.3 * 40 * dx + 8e-6, 16 * dx, True)
    tw.invalidate()
    tw.step(0.3 * 40 * dx + 9e-6, 16 * dx, True)
    assert tw._fused_params.tile_skip == 0


def _cache_slots(g):
    """(cell index, stamp, stored populations as integers) of every slot of the
    compact copy that goes with the buffer the next collision reads."""
    from waam_solver_b200.grid import raw_field
    a_first = g._read_buf is raw_field(g, "f_a")
    cache = g.pop_caches[0 if a_first else 1]
    if g.population_storage == 0:
        w = cache.view(torch.int32).view(-1, 24)
        return w[:, 19], w[:, 20], w[:, :19]
    w = cache.view(torch.int32).view(-1, 12)
    pops = cache.view(torch.int16).view(-1, 24)[:, :19].to(torch.int32)
    return w[:, 10], w[:, 11], pops


@pytest.mark.parametrize("dtype,lorentz", [("float32", False), ("float16", False),
                                           ("bfloat16", False), ("float32", True)])
def test_population_cache_matches_plane_reads(dtype, lorentz):
    """The collision's compact copy of its output, read back by the next
    collision for the cells active in both steps, against the 19 population
    planes read every step (no copy), bit for bit, through droplet steps, graph
    replays, the pipelined and lagged stream and (with the welding current)
    the Lorentz split step, in float32 and 16-bit population storage.  The
    copy really is read (cache_read on the regular steps) and every slot the
    last collision wrote holds its cell's stored populations."""
    states = []
    more = dict(enable_lorentz=True, welding_current_A=180.0) if lorentz else {}
    more["population_dtype"] = dtype
    for cached in (False, True):
        tw, ot, dx = _config_twins("c2", 40, 32, 96, **more)
        tw.population_cache = cached
        tw._last_droplet_time = -1.0
        g = tw.grid
        reads = 0
        for s in range(40):
            tw.step(0.3 * 40 * dx + s * 1e-6, 16 * dx, not 25 <= s < 28)
            reads += tw._fused_params.cache_read
        torch.cuda.synchronize()
        states.append(g.state_dict())
        assert tw._n_droplets_fired >= 1
        if not cached:
            assert getattr(g, "pop_caches", None) is None and reads == 0
            continue
        assert reads >= 30
        tag, stamp, pops = _cache_slots(g)
        live = (stamp == int(g.pop_cache_stamp.item())) & (tag >= 0)
        cells = tag[live].long()
        assert cells.numel() >= 40 * 32      # two plate-top cells per column, at least
        f = g._read_buf.reshape(19, -1)
        stored = f.view(torch.int32) if g.population_storage == 0 else f.view(torch.int16)
        assert torch.equal(stored[:, cells].T.to(torch.int32), pops[live])
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, states[1][k]), k


def test_population_cache_read_stops_after_other_population_writes():
    """The next collision reads the compact copy only when nothing but the
    fused step wrote the populations since the previous collision: not on a
    droplet step (the deposition writes them before its collision), nor
    after an operator-API stream call, a state load or invalidate()."""
    from waam_solver_b200 import kernels
    tw, ot, dx = _config_twins("c2", 40, 32, 96)
    g = tw.grid
    x = lambda s: 0.3 * 40 * dx + s * 1e-6   # noqa: E731
    for s in range(4):
        tw.step(x(s), 16 * dx, True)
    assert tw._fused_params.cache_read == 1
    kernels.stream(g.f_src, g.f_dst, g.flags, 1, 2, g.nx, g.ny, g.nz)
    tw.step(x(4), 16 * dx, True)
    assert tw._fused_params.cache_read == 0
    tw.step(x(5), 16 * dx, True)
    assert tw._fused_params.cache_read == 1
    g.load_state(g.state_dict())
    tw.step(x(6), 16 * dx, True)
    assert tw._fused_params.cache_read == 0
    tw.step(x(7), 16 * dx, True)
    tw.invalidate()
    tw.step(x(8), 16 * dx, True)
    assert tw._fused_params.cache_read == 0
    tw._last_droplet_time = -1.0
    n0 = tw._n_droplets_fired
    tw.step(x(9), 16 * dx, True)
    assert tw._n_droplets_fired == n0 + 1 and tw._fused_params.cache_read == 0
    tw.step(x(10), 16 * dx, True)
    assert tw._fused_params.cache_read == 1


def test_population_cache_after_reloading_an_older_state():
    """Back to an older state (as the adjoint's checkpoints and FD probes do):
    the first collision after the reload, left pending by its step, must not
    read the copy the newer state's last collision wrote -- the pending
    collision reads as its own step decided (collide_prev_cache_read), not as
    the step that runs it.  Against the same sequence without the copy."""
    states = []
    for cached in (False, True):
        tw, ot, dx = _config_twins("c2", 40, 32, 96)
        tw.population_cache = cached
        g = tw.grid
        x = lambda s: 0.3 * 40 * dx + s * 1e-6   # noqa: E731
        for s in range(6):
            tw.step(x(s), 16 * dx, True)
        older = g.state_dict()
        for s in range(6, 16):
            tw.step(x(s), 16 * dx, True)
        g.load_state(older)
        reads = []
        for s in range(6, 14):
            tw.step(x(s), 16 * dx, True)
            reads.append(tw._fused_params.cache_read)
        assert reads[0] == 0 and (sum(reads[1:]) > 0) == cached
        torch.cuda.synchronize()
        states.append(g.state_dict())
    for k, v in states[0].items():
        if isinstance(v, np.ndarray):
            assert np.array_equal(v, states[1][k]), k
