"""The CUDA backend against the oracle and the reference's golden outputs, on a GPU.

The claim tested is the strong one: in float64 and in float32 the sweeps perform the same
roundings as the NumPy reference, so fields, recordings and energies agree bit for bit
(the reference's own backend parity tests ask for rtol 1e-11, ``tests/test_c_backend.py:51-65``).
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from ac_fdtd_b200 import AIR, CudaAcousticFDTD, WallAdmittances, gaussian_pulse
from oracle.leapfrog import OracleFDTD
from tests.cases import CONFIGURATIONS, GRID, RECEIVER, SOURCE, full_room, plain_room, prepare

pytestmark = pytest.mark.gpu


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


SCHEMES = ["two_sweeps", "fused", "staged"]


def paired(dtype=np.float64, steps_per_graph=64, scheme="two_sweeps", **configuration):
    oracle = prepare(OracleFDTD(GRID, AIR, dtype=dtype, **configuration))
    cuda = prepare(CudaAcousticFDTD(GRID, dtype=dtype, steps_per_graph=steps_per_graph,
                                    scheme=scheme, **configuration))
    return oracle, cuda


def assert_same_state(cuda, oracle):
    np.testing.assert_array_equal(cuda.p, oracle.p)
    for axis in range(3):
        np.testing.assert_array_equal(cuda.velocity[axis], oracle.velocity[axis])
    np.testing.assert_array_equal(cuda.recorded_pressure, oracle.recorded_pressure)


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("name", list(CONFIGURATIONS))
def test_matches_the_oracle_bitwise(name, dtype, scheme, golden_meta, golden_trajectories):
    oracle, cuda = paired(dtype=dtype, scheme=scheme, **CONFIGURATIONS[name])
    oracle.run(150)
    cuda.run(150)
    assert_same_state(cuda, oracle)
    # ... and therefore the reference's own run, pinned in the golden fixtures.
    key = f"{np.dtype(dtype).name}/{name}/"
    assert digest(cuda.p) == golden_meta["trajectories"][key]["p"]
    np.testing.assert_array_equal(cuda.recorded_pressure, golden_trajectories[key + "recording"])
    if dtype == np.float64:
        assert cuda.energy() == pytest.approx(oracle.energy(), rel=1e-12)
    else:
        assert cuda.energy() == pytest.approx(oracle.energy(), rel=1e-5)


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_relaxation_states_match(dtype):
    configuration = CONFIGURATIONS["everything at once"]
    oracle, cuda = paired(dtype=dtype, **configuration)
    oracle.run(77)
    cuda.run(77)
    states = cuda.relaxation_states
    assert len(states) == len(oracle.relax) == 3
    for got, (want, *_rest) in zip(states, oracle.relax, strict=True):
        np.testing.assert_array_equal(got, want)


def test_graphs_and_step_by_step_launches_agree_bitwise():
    configuration = CONFIGURATIONS["everything at once"]
    _, graphed = paired(steps_per_graph=16, **configuration)
    _, direct = paired(steps_per_graph=0, **configuration)
    graphed.run(150)
    direct.run(150)
    np.testing.assert_array_equal(graphed.p, direct.p)
    np.testing.assert_array_equal(graphed.recorded_pressure, direct.recorded_pressure)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_running_in_pieces_is_the_same_as_running_at_once(scheme):
    _, whole = paired(walls=WallAdmittances.uniform(0.2), steps_per_graph=16, scheme=scheme)
    _, pieces = paired(walls=WallAdmittances.uniform(0.2), steps_per_graph=16, scheme=scheme)
    whole.run(120)
    for n in (30, 1, 16, 40, 33):
        pieces.run(n)
    np.testing.assert_array_equal(pieces.p, whole.p)
    np.testing.assert_array_equal(pieces.recorded_pressure, whole.recorded_pressure)


@pytest.mark.parametrize("scheme", SCHEMES)
def test_state_written_between_runs_is_used(scheme):
    oracle, cuda = paired(walls=WallAdmittances.uniform(0.3), scheme=scheme)
    oracle.run(20)
    cuda.run(20)
    rng = np.random.default_rng(9)
    new_p = rng.standard_normal(GRID.shape)
    new_vy = rng.standard_normal(GRID.velocity_shape(1)) * 1e-3
    for solver in (oracle, cuda):
        solver.p[:] = new_p
        solver.velocity[1][:] = new_vy
    oracle.run(25)
    cuda.run(25)
    assert_same_state(cuda, oracle)


def test_sources_receivers_edge_cases():
    """Two sources in one cell, a source longer than the run, a receiver added mid-run."""
    oracle, cuda = paired(walls=WallAdmittances.uniform(0.1))
    for solver in (oracle, cuda):
        solver.add_volume_source(SOURCE, np.linspace(0.0, 1.0, 7))
        solver.add_volume_source((0.05, 0.45, 0.4), np.ones(500))
    oracle.run(30)
    cuda.run(30)
    late = [s.add_pressure_receiver((0.59, 0.01, 0.44)) for s in (oracle, cuda)]
    assert late[0] == late[1] == 1
    oracle.run(40)
    cuda.run(40)
    np.testing.assert_array_equal(cuda.p, oracle.p)
    np.testing.assert_array_equal(cuda.recording(0), np.array(oracle.receivers[0][1]))
    np.testing.assert_array_equal(cuda.recording(1), np.array(oracle.receivers[1][1]))
    assert cuda.recording(1).size == 40
    with pytest.raises(ValueError):
        cuda.recorded_pressure  # noqa: B018 -- ragged recordings are refused, as NumPy does


def test_receivers_record_the_same_samples_as_probing_by_hand():
    solver = CudaAcousticFDTD(GRID, dtype=np.float64)
    solver.add_volume_source(SOURCE, np.ones(50))
    solver.add_pressure_receiver(RECEIVER)
    solver.run(20)
    solver.run(20)
    recorded = solver.recorded_pressure
    assert recorded.shape == (1, 40)
    assert recorded[0, -1] == solver.p[GRID.cell_index(RECEIVER)]


def test_rigid_walls_are_never_written_to():
    solver = CudaAcousticFDTD(GRID)
    solver.p[:] = np.random.default_rng(0).standard_normal(GRID.shape)
    solver.run(20)
    for axis in range(3):
        wall = solver.velocity[axis]
        lower = tuple(0 if a == axis else slice(None) for a in range(3))
        upper = tuple(-1 if a == axis else slice(None) for a in range(3))
        assert np.all(wall[lower] == 0.0)
        assert np.all(wall[upper] == 0.0)


def test_plain_room_matches_the_reference(golden_meta, golden_rooms):
    meta = golden_meta["rooms"]["plain"]
    grid, objects = plain_room(meta)
    solver = CudaAcousticFDTD(grid, **objects)
    solver.add_volume_source(meta["source"], golden_rooms["plain/signal"])
    solver.add_pressure_receiver(meta["receiver"])
    solver.run(meta["steps"])
    np.testing.assert_array_equal(solver.recorded_pressure, golden_rooms["plain/numpy/recording"])
    assert digest(solver.p) == golden_meta["rooms"]["plain/numpy/p"]


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_walls_sponge_air_room_matches_the_reference(dtype, scheme, golden_meta, golden_rooms):
    meta = golden_meta["rooms"]["full"]
    grid, objects = full_room(meta)
    solver = CudaAcousticFDTD(grid, dtype=dtype, scheme=scheme, **objects)
    solver.add_volume_source(meta["points"][0], gaussian_pulse(meta["steps"], solver.dt, 4000.0))
    for point in meta["points"][1:]:
        solver.add_pressure_receiver(point)
    solver.run(meta["steps"])
    name = np.dtype(dtype).name
    np.testing.assert_array_equal(solver.recorded_pressure,
                                  golden_rooms[f"full/{name}/numpy/recording"])
    assert digest(solver.p) == golden_meta["rooms"][f"full/{name}/numpy/p"]
    # The reference C backend differs from NumPy by rounding order only.
    c = golden_rooms[f"full/{name}/c/recording"]
    scale = np.max(np.abs(c))
    tol = 1e-13 if dtype == np.float64 else 1e-5
    assert np.max(np.abs(solver.recorded_pressure - c)) <= tol * scale


@pytest.mark.parametrize("scheme", SCHEMES)
def test_odd_and_degenerate_grids(scheme):
    """Sizes that are not multiples of the 4-element vector, and 1-cell-wide ducts."""
    from ac_fdtd_b200 import AbsorbingLayer, AirAbsorption, Grid

    for shape in ((1, 1, 9), (5, 1, 1), (3, 2, 7), (2, 3, 1), (7, 5, 13), (4, 4, 4), (3, 5, 8)):
        grid = Grid(dx=0.02, nx=shape[0], ny=shape[1], nz=shape[2])
        configuration = dict(walls=WallAdmittances(0.4, 0.1, 0.0, 0.7, 0.2, 0.0),
                             absorbing_layer=AbsorbingLayer(thickness=2),
                             air_absorption=AirAbsorption())
        oracle = OracleFDTD(grid, AIR, **configuration)
        cuda = CudaAcousticFDTD(grid, scheme=scheme, **configuration)
        prefetching = CudaAcousticFDTD(grid, scheme=scheme, **configuration)
        prefetching.set_prefetch(True)
        rng = np.random.default_rng(sum(shape))
        initial = rng.standard_normal(shape)
        point = tuple((n - 0.5) * 0.02 for n in shape)
        for solver in (oracle, cuda, prefetching):
            solver.p[:] = initial
            solver.add_volume_source((0.0, 0.0, 0.0), np.hanning(12))
            solver.add_pressure_receiver(point)
        oracle.run(40)
        cuda.run(40)
        prefetching.run(40)
        assert_same_state(cuda, oracle)
        assert_same_state(prefetching, oracle)


def test_switching_schemes_mid_run_and_odd_step_counts():
    """The fused scheme alternates between two copies of p and v; switching schemes, odd runs,
    energy, state access and graph replays from either copy must all see the current state."""
    configuration = CONFIGURATIONS["everything at once"]
    oracle, cuda = paired(steps_per_graph=8, scheme="fused", **configuration)
    plan = [("fused", 9), ("fused", 17), ("two_sweeps", 5), ("fused", 3), ("staged", 16),
            ("two_sweeps", 8), ("fused", 1), ("staged", 7), ("fused", 2), ("staged", 1)]
    total = 0
    for scheme, n in plan:
        cuda.set_scheme(scheme)
        cuda.run(n)
        oracle.run(n)
        total += n
        assert cuda.energy() == pytest.approx(oracle.energy(), rel=1e-12)
        np.testing.assert_array_equal(cuda.p, oracle.p)
    assert_same_state(cuda, oracle)
    assert cuda.step_index == total


@pytest.mark.parametrize("scheme", SCHEMES)
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_l2_prefetch_forced_on_matches_the_oracle(dtype, scheme):
    """Rooms this small stay in L2, so the plane prefetch is off by default; forced on (and
    toggled mid-run, with graphs captured either way) the results stay bit-identical."""
    configuration = CONFIGURATIONS["everything at once"]
    oracle, cuda = paired(dtype=dtype, steps_per_graph=8, scheme=scheme, **configuration)
    assert not cuda.prefetch
    cuda.set_prefetch(True)
    assert cuda.prefetch
    for enabled, n in ((True, 37), (False, 9), (True, 16), (None, 5)):
        cuda.set_prefetch(enabled)
        cuda.run(n)
        oracle.run(n)
    assert not cuda.prefetch
    assert_same_state(cuda, oracle)


def test_l2_prefetch_follows_the_size_of_the_fields():
    """On by default once the fields a step streams exceed L2 (126 MB on a B200): a 200^3
    fp32 room's seven fields take 235 MB; a 96^3 room's 27 MB, or 43 MB with the fused
    scheme's second copy of p and v."""
    from ac_fdtd_b200 import AirAbsorption, Grid

    big = CudaAcousticFDTD(Grid(dx=0.02, nx=200, ny=200, nz=200), dtype=np.float32,
                           air_absorption=AirAbsorption())
    small = CudaAcousticFDTD(Grid(dx=0.02, nx=96, ny=96, nz=96), dtype=np.float32,
                             air_absorption=AirAbsorption(), scheme="fused")
    assert big.prefetch and not small.prefetch
    big.set_prefetch(False)
    small.set_prefetch(True)
    assert small.prefetch and not big.prefetch
    big.close()
    small.close()


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_staged_geometries_match_the_oracle(dtype):
    """Rows per CTA, ring depth and planes per CTA change only which CTA computes a cell and
    when its inputs arrive; every geometry must give the oracle's bits, on grids whose rows and
    planes do not divide evenly, and no wait may run out."""
    from ac_fdtd_b200 import AbsorbingLayer, AirAbsorption, Grid

    configuration = dict(walls=WallAdmittances(0.4, 0.1, 0.0, 0.7, 0.2, 0.05),
                         absorbing_layer=AbsorbingLayer(thickness=3),
                         air_absorption=AirAbsorption())
    for shape in ((13, 11, 23), (6, 1, 5), (1, 7, 3), (9, 10, 40)):
        grid = Grid(dx=0.02, nx=shape[0], ny=shape[1], nz=shape[2])
        initial = np.random.default_rng(sum(shape)).standard_normal(shape)
        receiver = tuple((n - 0.5) * 0.02 for n in shape)
        oracle = OracleFDTD(grid, AIR, dtype=dtype, **configuration)
        oracle.p[:] = initial
        oracle.add_volume_source((0.01, 0.01, 0.01), np.hanning(9))
        oracle.add_pressure_receiver(receiver)
        oracle.run(21)
        for rows, stages, planes, vector in ((1, 2, 1, 2), (2, 0, 3, 4), (3, 3, 4, 2),
                                             (4, 4, 64, 4), (2, 8, 5, 2), (1, 0, 7, 4)):
            cuda = CudaAcousticFDTD(grid, dtype=dtype, steps_per_graph=6, **configuration)
            cuda.set_staging(rows, stages, planes, vector)
            cuda.set_scheme("staged")
            cuda.p[:] = initial
            cuda.add_volume_source((0.01, 0.01, 0.01), np.hanning(9))
            cuda.add_pressure_receiver(receiver)
            cuda.run(21)
            cuda.check_device()
            assert_same_state(cuda, oracle)


@pytest.mark.parametrize("vector", [2, 4])
def test_staged_points_in_one_tile(vector):
    """The staged sweep gathers the sources and receivers of each CTA's tile once per launch:
    several sources in one cell must still add up in the order they were added, receivers must
    read the finished pressure, and a tile holding more points than the gathered list takes
    (here 41 in one y row) must fall back to scanning every point -- all bit for bit."""
    configuration = dict(walls=WallAdmittances.uniform(0.2))
    oracle = OracleFDTD(GRID, AIR, **configuration)
    cuda = CudaAcousticFDTD(GRID, steps_per_graph=8, **configuration)
    cuda.set_staging(1, 0, 5, vector)
    cuda.set_scheme("staged")
    rng = np.random.default_rng(3)
    initial = rng.standard_normal(GRID.shape)
    signals = [rng.standard_normal(40) for _ in range(3)]
    row = [(0.315, 0.255, (k + 0.5) * 0.03) for k in range(GRID.shape[2])]
    for solver in (oracle, cuda):
        solver.p[:] = initial
        for signal in signals:                       # three sources, one cell
            solver.add_volume_source((0.2, 0.2, 0.2), signal)
        solver.add_volume_source((0.2, 0.2, 0.23), signals[0][::-1])
        solver.add_pressure_receiver((0.2, 0.2, 0.2))
        for point in row + row + row[:11]:           # 41 receivers in one row of one tile
            solver.add_pressure_receiver(point)
    oracle.run(30)
    cuda.run(30)
    cuda.check_device()
    assert_same_state(cuda, oracle)


def test_an_explicit_device_gives_the_same_results():
    """device= selects the GPU in the library's own runtime; on device 0 the results equal the
    default construction bit for bit, for a single room and a batch."""
    from ac_fdtd_b200 import RoomBatch

    oracle, default = paired(walls=WallAdmittances.uniform(0.2))
    explicit = prepare(CudaAcousticFDTD(GRID, device=0, walls=WallAdmittances.uniform(0.2)))
    for solver in (oracle, default, explicit):
        solver.run(40)
    assert_same_state(explicit, oracle)
    batch = RoomBatch([dict(grid=GRID)], dtype=np.float64, device=0)
    batch.set_field(0, 0, np.random.default_rng(0).standard_normal(GRID.shape))
    batch.run(5)
    assert np.all(np.isfinite(batch.p(0)))


@pytest.mark.parametrize("faces", [None, ((0, 0), (0, 1)), ((1, 1), (2, 0))])
def test_lean_single_precision_fused_column_matches_the_oracle(faces):
    """Single precision runs the fused step through the lean column (packed arithmetic, damping
    skipped where the profile is exactly 1; rows of a multiple of 4 cells without padding
    lanes, others with fix-ups in their last chunk). Grids with one chunk,
    one row, one plane, sponges on every face or on some only (so rows, chunks and planes
    with and without damping meet in one warp), walls, air, points on the edges: the
    oracle's float32 bits, with the L2 prefetch off and on."""
    from ac_fdtd_b200 import AbsorbingLayer, AirAbsorption, Grid

    layer = AbsorbingLayer(thickness=3) if faces is None else AbsorbingLayer(thickness=3, faces=faces)
    configuration = dict(walls=WallAdmittances(0.4, 0.1, 0.0, 0.7, 0.2, 0.05),
                         absorbing_layer=layer, air_absorption=AirAbsorption())
    for shape in ((13, 11, 24), (1, 1, 4), (6, 1, 8), (2, 9, 4), (9, 10, 40), (5, 3, 12),
                  (4, 37, 132), (13, 11, 23), (6, 1, 5), (2, 9, 1), (1, 1, 2), (5, 3, 7),
                  (4, 37, 133), (7, 6, 6)):
        grid = Grid(dx=0.02, nx=shape[0], ny=shape[1], nz=shape[2])
        initial = np.random.default_rng(sum(shape)).standard_normal(shape).astype(np.float32)
        corner = tuple((n - 0.5) * 0.02 for n in shape)
        oracle = OracleFDTD(grid, AIR, dtype=np.float32, **configuration)
        solvers = [oracle]
        for prefetch in (False, True):
            cuda = CudaAcousticFDTD(grid, dtype=np.float32, scheme="fused", steps_per_graph=6,
                                    **configuration)
            cuda.set_prefetch(prefetch)
            solvers.append(cuda)
        for solver in solvers:
            solver.p[:] = initial
            solver.add_volume_source((0.0, 0.0, 0.0), np.hanning(12))
            solver.add_volume_source(corner, np.hanning(7))
            solver.add_pressure_receiver(corner)
            solver.add_pressure_receiver((0.0, corner[1], 0.0))
        for solver in solvers:
            solver.run(33)
        for cuda in solvers[1:]:
            assert_same_state(cuda, oracle)
            for got, (want, *_rest) in zip(cuda.relaxation_states, oracle.relax, strict=True):
                np.testing.assert_array_equal(got, want)
            cuda.close()


@pytest.mark.parametrize("planes", [1, 3, 16])
def test_lean_column_plane_groups_and_graphs(planes):
    """Blocks marching 1, 3 or 16 planes (a group ending inside the sponge, the last group
    short), in graph replays and run in pieces, on a 48^2 x 64 room with the bench's sponge on
    both x faces: the two-sweep scheme's bits."""
    from ac_fdtd_b200 import AbsorbingLayer, AirAbsorption, Grid

    grid = Grid(dx=0.01, nx=50, ny=48, nz=64)
    configuration = dict(walls=WallAdmittances(0.3, 0.2, 0.1, 0.05, 0.25, 0.15),
                         absorbing_layer=AbsorbingLayer(thickness=8, faces=((0, 0), (0, 1))),
                         air_absorption=AirAbsorption())
    initial = np.random.default_rng(5).standard_normal(grid.shape).astype(np.float32)
    out = []
    for scheme in ("two_sweeps", "fused"):
        cuda = CudaAcousticFDTD(grid, dtype=np.float32, scheme=scheme, steps_per_graph=8,
                                **configuration)
        if scheme == "fused":
            cuda.set_launch(64, planes)
        cuda.p[:] = initial
        cuda.add_volume_source((0.2, 0.2, 0.3), np.hanning(20))
        cuda.add_pressure_receiver((0.45, 0.3, 0.1))
        for n in (17, 1, 24):
            cuda.run(n)
        out.append((cuda.p.copy(), cuda.recorded_pressure, [v.copy() for v in cuda.velocity]))
        cuda.close()
    np.testing.assert_array_equal(out[0][0], out[1][0])
    np.testing.assert_array_equal(out[0][1], out[1][1])
    for a, b in zip(out[0][2], out[1][2], strict=True):
        np.testing.assert_array_equal(a, b)
