"""The oracle is pinned to the reference before anything is checked against it.

Every number here was produced by running ac-fdtd itself (``tests/golden/make_golden.py``);
the NumPy restatement in ``oracle/`` must reproduce it bit for bit.
"""

from __future__ import annotations

import hashlib

import numpy as np
import pytest

from ac_fdtd_b200 import AIR, AbsorbingLayer, AirAbsorption, Grid, WallAdmittances
from oracle.leapfrog import OracleFDTD, oracle_layer_factors, oracle_processes, oracle_wall_list
from tests.cases import CONFIGURATIONS, GRID, full_room, plain_room, prepare


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def realise(spec):
    out = {}
    if "walls" in spec:
        kind, value = spec["walls"]
        out["walls"] = WallAdmittances.uniform(value) if kind == "uniform" else WallAdmittances(**value)
    if "absorbing_layer" in spec:
        layer = dict(spec["absorbing_layer"])
        if "faces" in layer:
            layer["faces"] = tuple(tuple(f) for f in layer["faces"])
        out["absorbing_layer"] = AbsorbingLayer(**layer)
    if "air_absorption" in spec:
        out["air_absorption"] = AirAbsorption(**spec["air_absorption"])
    return out


def test_oracle_setup_is_the_reference_setup(golden_meta, golden_setup):
    for name, case in golden_meta["setup"].items():
        grid = Grid(dx=case["dx"], nx=case["shape"][0], ny=case["shape"][1], nz=case["shape"][2])
        objects = realise(case["spec"])
        oracle = OracleFDTD(grid, AIR, dtype=np.dtype(case["dtype"]), **objects)
        scalars = golden_setup[name + "/scalars"]
        got = [oracle.dt, oracle.cv, oracle.cp, oracle.cs, oracle.relax_scale]
        assert np.array_equal(np.array(got, dtype=np.float64), scalars), name
        relax = np.array([[float(d), float(m), float(g)] for _, d, m, g in oracle.relax]).reshape(-1, 3)
        assert np.array_equal(relax, golden_setup[name + "/relax"]), name
        xi = objects["walls"].values if "walls" in objects else (0.0,) * 6
        index, a = oracle_wall_list(case["shape"], AIR.sound_speed, oracle.dt, case["dx"], xi)
        assert np.array_equal(index, golden_setup[name + "/wall_index"]), name
        assert np.array_equal(a, golden_setup[name + "/wall_a"]), name
        if "air_absorption" in objects:
            processes = np.array(oracle_processes(objects["air_absorption"], AIR.sound_speed, oracle.dt))
            assert np.array_equal(processes.reshape(-1, 2), golden_setup[name + "/processes"]), name
        if "absorbing_layer" in objects:
            cells, faces = oracle_layer_factors(case["shape"], case["dx"], AIR.sound_speed,
                                                oracle.dt, objects["absorbing_layer"])
            for axis in range(3):
                assert np.array_equal(cells[axis], golden_setup[name + f"/cell{axis}"]), name
                assert np.array_equal(faces[axis], golden_setup[name + f"/face{axis}"]), name


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("name", list(CONFIGURATIONS))
def test_oracle_trajectories_match_the_reference_bitwise(name, dtype, golden_meta,
                                                          golden_trajectories):
    oracle = prepare(OracleFDTD(GRID, AIR, dtype=np.dtype(dtype), **CONFIGURATIONS[name]))
    oracle.run(150)
    key = f"{dtype}/{name}/"
    np.testing.assert_array_equal(oracle.recorded_pressure, golden_trajectories[key + "recording"])
    assert digest(oracle.p) == golden_meta["trajectories"][key]["p"]
    for axis in range(3):
        assert digest(oracle.velocity[axis]) == golden_meta["trajectories"][key]["v"][axis]
    assert oracle.energy() == golden_trajectories[key + "energy"][0]


def test_oracle_plain_room_matches_the_reference(golden_meta, golden_rooms):
    meta = golden_meta["rooms"]["plain"]
    grid, objects = plain_room(meta)
    oracle = OracleFDTD(grid, AIR, **objects)
    oracle.add_volume_source(meta["source"], golden_rooms["plain/signal"])
    oracle.add_pressure_receiver(meta["receiver"])
    oracle.run(meta["steps"])
    np.testing.assert_array_equal(oracle.recorded_pressure, golden_rooms["plain/numpy/recording"])
    assert digest(oracle.p) == golden_meta["rooms"]["plain/numpy/p"]


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_oracle_full_room_matches_the_reference(dtype, golden_meta, golden_rooms):
    from ac_fdtd_b200 import gaussian_pulse

    meta = golden_meta["rooms"]["full"]
    grid, objects = full_room(meta)
    oracle = OracleFDTD(grid, AIR, dtype=np.dtype(dtype), **objects)
    oracle.add_volume_source(meta["points"][0], gaussian_pulse(meta["steps"], oracle.dt, 4000.0))
    for point in meta["points"][1:]:
        oracle.add_pressure_receiver(point)
    oracle.run(meta["steps"])
    np.testing.assert_array_equal(oracle.recorded_pressure,
                                  golden_rooms[f"full/{dtype}/numpy/recording"])
    assert digest(oracle.p) == golden_meta["rooms"][f"full/{dtype}/numpy/p"]


def test_reference_c_driver_reproduces_the_reference_c_backend(golden_meta, golden_rooms):
    """The ctypes driver of the compiled reference C (the timed CPU baseline) is pinned too."""
    from oracle import ref_c

    if not ref_c.available() and not ref_c.build():
        pytest.skip("reference C sources not present and oracle/_ref not built")
    from ac_fdtd_b200 import gaussian_pulse

    meta = golden_meta["rooms"]["plain"]
    grid, objects = plain_room(meta)
    solver = ref_c.RefCSolver(grid, AIR, **objects)
    solver.add_volume_source(meta["source"], golden_rooms["plain/signal"])
    solver.add_pressure_receiver(meta["receiver"])
    solver.run(meta["steps"])
    np.testing.assert_array_equal(solver.recorded_pressure, golden_rooms["plain/c/recording"])

    meta = golden_meta["rooms"]["full"]
    grid, objects = full_room(meta)
    for dtype in ("float64", "float32"):
        solver = ref_c.RefCSolver(grid, AIR, dtype=np.dtype(dtype), **objects)
        solver.add_volume_source(meta["points"][0], gaussian_pulse(meta["steps"], solver.dt, 4000.0))
        for point in meta["points"][1:]:
            solver.add_pressure_receiver(point)
        solver.run(meta["steps"])
        np.testing.assert_array_equal(solver.recorded_pressure,
                                      golden_rooms[f"full/{dtype}/c/recording"])
        assert digest(solver.p) == golden_meta["rooms"][f"full/{dtype}/c/p"]
