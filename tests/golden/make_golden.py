"""Generate the golden fixtures in this folder by running the ac-fdtd reference itself.

Run in the build container, where the reference is mounted (it is not on the GPU machines):

    python tests/golden/make_golden.py [/root/reference]

The reference is copied to a scratch directory first, because its C backend compiles its
shared library next to its own source. Outputs (all committed, all small):

* ``setup.npz`` -- the reference's FP64 host setup for a set of rooms: scheme constants after
  the dtype cast, the sparse wall list, the layer factors and the relaxation processes.
* ``trajectories.npz`` -- the five parity configurations of the reference's own backend tests
  (``tests/test_c_backend.py:15-42``) run for 150 steps in float64 and float32 by the NumPy
  reference: receiver recordings, energies, and SHA-256 digests plus norms of the final fields.
* ``impulse.npz`` -- ``simulate_impulse_response`` on a small room (recordings, deconvolved
  signals, excitation) with the statistical formulae and decay metrics of that run.
* ``rooms.npz`` -- two small rooms in the shape of the benchmark configurations (64^3-like
  plain walls with a Gaussian-derivative source; a walls + sponge + ISO air room with four
  receivers), recordings from the NumPy reference and from the reference C backend.
"""

from __future__ import annotations

import hashlib
import json
import shutil
import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent


def digest(array: np.ndarray) -> str:
    return hashlib.sha256(np.ascontiguousarray(array).tobytes()).hexdigest()


def norms(array: np.ndarray) -> np.ndarray:
    a = np.asarray(array, dtype=np.float64)
    return np.array([a.sum(), (a * a).sum(), np.abs(a).max()])


# The parity configurations of the reference's backend tests, as plain data.
CONFIGURATIONS = {
    "rigid": {},
    "absorbing walls": {"walls": ("uniform", 0.3)},
    "absorbing layer": {"absorbing_layer": {"thickness": 4}},
    "air absorption": {"air_absorption": {}},
    "everything at once": {
        "walls": ("faces", {"x_min": 0.2, "z_max": 0.7}),
        "absorbing_layer": {"thickness": 3},
        "air_absorption": {"temperature": 15.0, "relative_humidity": 70.0},
    },
}
GRID_LENGTHS, GRID_DX = (0.6, 0.5, 0.45), 0.03
SOURCE, RECEIVER = (0.2, 0.2, 0.2), (0.4, 0.3, 0.3)
STEPS = 150


def realise(ref, spec: dict) -> dict:
    """Turn a plain-data configuration into reference objects."""
    out = {}
    if "walls" in spec:
        kind, value = spec["walls"]
        out["walls"] = (ref.WallAdmittances.uniform(value) if kind == "uniform"
                        else ref.WallAdmittances(**value))
    if "absorbing_layer" in spec:
        out["absorbing_layer"] = ref.AbsorbingLayer(**spec["absorbing_layer"])
    if "air_absorption" in spec:
        out["air_absorption"] = ref.AirAbsorption(**spec["air_absorption"])
    return out


SETUP_CASES = {
    "walls_layer_air_f64": dict(shape=(20, 17, 15), dx=0.03, dtype="float64",
                                spec=CONFIGURATIONS["everything at once"]),
    "walls_layer_air_f32": dict(shape=(20, 17, 15), dx=0.03, dtype="float32",
                                spec=CONFIGURATIONS["everything at once"]),
    "uniform_walls_f32": dict(shape=(9, 7, 5), dx=0.05, dtype="float32",
                              spec={"walls": ("uniform", 0.3)}),
    "duct_f64": dict(shape=(30, 1, 1), dx=0.01, dtype="float64",
                     spec={"walls": ("faces", {"x_min": 1.0, "x_max": 0.25}),
                           "air_absorption": {}}),
    "bench_like_f32": dict(shape=(24, 20, 18), dx=343.2 / 40000.0, dtype="float32",
                           spec={"walls": ("faces", {"x_min": 0.11, "x_max": 0.05, "y_min": 0.2,
                                                     "y_max": 0.31, "z_min": 0.07, "z_max": 0.4}),
                                 "absorbing_layer": {"thickness": 6, "faces": ((0, 0), (0, 1))},
                                 "air_absorption": {"temperature": 20.0,
                                                    "relative_humidity": 50.0}}),
    "dry_no_classical_f64": dict(shape=(6, 5, 4), dx=0.02, dtype="float64",
                                 spec={"air_absorption": {"temperature": 25.0,
                                                          "relative_humidity": 30.0,
                                                          "classical": False}}),
}


def make_setup(ref_pkg) -> dict:
    from ac_fdtd.boundaries import layer_factors, wall_update_coefficients

    data = {}
    meta = {}
    for name, case in SETUP_CASES.items():
        grid = ref_pkg.Grid(dx=case["dx"], nx=case["shape"][0], ny=case["shape"][1],
                            nz=case["shape"][2])
        objects = realise(ref_pkg, case["spec"])
        solver = ref_pkg.AcousticFDTD(grid, dtype=np.dtype(case["dtype"]), **objects)
        prefix = name + "/"
        data[prefix + "scalars"] = np.array(
            [solver.dt, solver._velocity_coefficient, solver._pressure_coefficient,
             solver._source_coefficient, solver._relaxation_target_scale], dtype=np.float64)
        data[prefix + "relax"] = np.array(
            [[float(d), float(m), float(g)] for _, d, m, g in solver._relaxation]).reshape(-1, 3)
        index, coefficient = wall_update_coefficients(grid, ref_pkg.AIR, solver.dt, solver.walls)
        data[prefix + "wall_index"] = index
        data[prefix + "wall_a"] = coefficient
        if "air_absorption" in objects:
            processes = objects["air_absorption"].processes(ref_pkg.AIR.sound_speed, solver.dt)
            data[prefix + "processes"] = np.array(
                [[p.strength, p.relaxation_time] for p in processes]).reshape(-1, 2)
        if "absorbing_layer" in objects:
            pf, vf = layer_factors(grid, ref_pkg.AIR, solver.dt, objects["absorbing_layer"])
            for a in range(3):
                data[prefix + f"cell{a}"] = pf[a]
                data[prefix + f"face{a}"] = vf[a][a]
                for comp in range(3):
                    if comp != a:
                        assert np.array_equal(vf[comp][a], pf[a])
        meta[name] = {"shape": case["shape"], "dx": case["dx"], "dtype": case["dtype"],
                      "spec": case["spec"]}
    return data, meta


def make_trajectories(ref_pkg) -> tuple[dict, dict]:
    grid = ref_pkg.Grid.from_lengths(GRID_LENGTHS, GRID_DX)
    data, meta = {}, {}
    for dtype in ("float64", "float32"):
        for name, spec in CONFIGURATIONS.items():
            solver = ref_pkg.AcousticFDTD(grid, dtype=np.dtype(dtype), **realise(ref_pkg, spec))
            solver.p[:] = np.random.default_rng(0).standard_normal(grid.shape)
            signal = np.exp(-(((np.arange(200) - 30) / 8.0) ** 2))
            solver.add_volume_source(SOURCE, signal)
            solver.add_pressure_receiver(RECEIVER)
            solver.run(STEPS)
            key = f"{dtype}/{name}/"
            data[key + "recording"] = solver.recorded_pressure
            data[key + "energy"] = np.array([solver.energy()])
            data[key + "p_norms"] = norms(solver.p)
            for a in range(3):
                data[key + f"v{a}_norms"] = norms(solver.velocity[a])
            meta[key] = {"p": digest(solver.p),
                         "v": [digest(solver.velocity[a]) for a in range(3)]}
    meta["grid"] = {"lengths": GRID_LENGTHS, "dx": GRID_DX, "shape": list(grid.shape)}
    return data, meta


def make_rooms(ref_pkg, c_backend) -> tuple[dict, dict]:
    data, meta = {}, {}
    # Plain walls, Gaussian-derivative source (a 32^3 stand-in for the 64^3 plain-method room).
    dx = 343.2 / (10 * 1000.0)
    grid = ref_pkg.Grid(dx=dx, nx=32, ny=32, nz=32)
    walls = ref_pkg.WallAdmittances.from_absorption(0.15)
    probe = ref_pkg.AcousticFDTD(grid, walls=walls)
    n_steps = 400
    t = (np.arange(n_steps) + 0.5) * probe.dt
    width = np.sqrt(np.log(10.0 ** 2)) / (np.pi * 1000.0)
    centre = 4.0 * width
    signal = -2.0 * (t - centre) / width**2 * np.exp(-(((t - centre) / width) ** 2))
    src = tuple((i + 0.5) * dx for i in (8, 8, 10))
    rec = tuple((i + 0.5) * dx for i in (22, 20, 12))
    for backend, make in (("numpy", ref_pkg.AcousticFDTD), ("c", c_backend.CAcousticFDTD)):
        solver = make(grid, walls=walls)
        solver.add_volume_source(src, signal)
        solver.add_pressure_receiver(rec)
        solver.run(n_steps)
        data[f"plain/{backend}/recording"] = solver.recorded_pressure
        meta[f"plain/{backend}/p"] = digest(solver.p)
    data["plain/signal"] = signal
    meta["plain"] = {"shape": [32, 32, 32], "dx": dx, "absorption": 0.15, "source": src,
                     "receiver": rec, "steps": n_steps}

    # Walls + sponge on two opposite faces + ISO air, four receivers, both precisions.
    rng = np.random.default_rng(2024)
    dx = 343.2 / (10 * 4000.0)
    shape = (28, 24, 22)
    grid = ref_pkg.Grid(dx=dx, nx=shape[0], ny=shape[1], nz=shape[2])
    alphas = rng.uniform(0.05, 0.5, 6)
    walls = ref_pkg.WallAdmittances(*[ref_pkg.admittance_from_absorption(a) for a in alphas])
    layer = ref_pkg.AbsorbingLayer(thickness=6, faces=((0, 0), (0, 1)))
    air = ref_pkg.AirAbsorption(temperature=20.0, relative_humidity=50.0)
    n_steps = 250
    cells = [tuple(int(v) for v in rng.integers(7, np.array(shape) - 7)) for _ in range(5)]
    points = [tuple((i + 0.5) * dx for i in c) for c in cells]
    for dtype in ("float64", "float32"):
        for backend, make in (("numpy", ref_pkg.AcousticFDTD), ("c", c_backend.CAcousticFDTD)):
            solver = make(grid, dtype=np.dtype(dtype), walls=walls, absorbing_layer=layer,
                          air_absorption=air)
            signal = ref_pkg.gaussian_pulse(n_steps, solver.dt, 4000.0)
            solver.add_volume_source(points[0], signal)
            for point in points[1:]:
                solver.add_pressure_receiver(point)
            solver.run(n_steps)
            data[f"full/{dtype}/{backend}/recording"] = solver.recorded_pressure
            meta[f"full/{dtype}/{backend}/p"] = digest(solver.p)
    meta["full"] = {"shape": list(shape), "dx": dx, "alphas": alphas.tolist(),
                    "layer": {"thickness": 6, "faces": [[0, 0], [0, 1]]},
                    "air": {"temperature": 20.0, "relative_humidity": 50.0},
                    "points": points, "steps": n_steps}
    return data, meta


def make_impulse(ref_pkg) -> tuple[dict, dict]:
    """The reference's room workflow end to end on a small room, plus its statistical formulae."""
    from ac_fdtd import metrics

    room = ref_pkg.Room((0.62, 0.5, 0.41), absorption=0.3)
    source, receivers = (0.2, 0.17, 0.15), [(0.45, 0.33, 0.28), (0.1, 0.4, 0.3)]
    ir = ref_pkg.simulate_impulse_response(room, source, receivers, max_frequency=1500.0)
    data = {"signals": ir.signals, "recorded": ir.recorded, "excitation": ir.excitation}
    formulae = {
        "sabine": room.sabine_reverberation_time(), "eyring": room.eyring_reverberation_time(),
        "diffuse_absorption": room.diffuse_absorption, "air_coefficient": room.air_coefficient(1000.0),
        "t20": metrics.reverberation_time(ir.signals[0], ir.sample_rate, 20.0),
        "edt": metrics.early_decay_time(ir.signals[0], ir.sample_rate),
        "c2ms": metrics.clarity(ir.signals[0], ir.sample_rate, split=0.002),
    }
    meta = {"dimensions": room.dimensions, "absorption": room.absorption, "source": source,
            "receivers": receivers, "max_frequency": 1500.0, "sample_rate": ir.sample_rate,
            "shape": list(ir.grid.shape), "formulae": formulae}
    return data, meta


def make_io(ref_pkg, scratch: Path) -> tuple[dict, dict]:
    """The reference's export path: rational-ratio resampling from grid rates to audio rates,
    and a WAV file written and read back."""
    from scipy.io import wavfile

    from ac_fdtd import io as ref_io

    rng = np.random.default_rng(11)
    signal = rng.standard_normal((3, 1200)) * np.exp(-np.arange(1200) / 300.0)
    data = {"signal": signal}
    cases = [(29716.4, 48000.0), (59432.7, 44100.0), (17150.0, 48000.0), (48000.0, 48000.0)]
    for n, (source_rate, target_rate) in enumerate(cases):
        data[f"resampled_{n}"] = ref_io.resample(signal, source_rate, target_rate)
    path = ref_io.write_wav(scratch / "ir.wav", signal, 29716.4)
    rate, written = wavfile.read(path)
    data["wav"] = written
    path = ref_io.write_wav(scratch / "raw.wav", signal[0], 29716.4, target_rate=None, normalise=False)
    rate_raw, written_raw = wavfile.read(path)
    data["wav_raw"] = written_raw
    meta = {"cases": cases, "wav_rate": int(rate), "wav_raw_rate": int(rate_raw)}
    return data, meta


def main(reference: str = "/root/reference", *parts: str) -> None:
    """Regenerate every fixture, or only the named parts (setup, trajectories, rooms, impulse,
    io); golden.json keeps the entries of the parts not regenerated."""
    scratch = Path(tempfile.mkdtemp(prefix="acfdtd_ref_"))
    shutil.copytree(Path(reference) / "src", scratch / "src")
    sys.path.insert(0, str(scratch / "src"))
    import ac_fdtd as ref_pkg
    from ac_fdtd import c_backend

    if parts:
        meta = json.loads((HERE / "golden.json").read_text())
        if "io" in parts:
            io_data, meta["io"] = make_io(ref_pkg, scratch)
            np.savez_compressed(HERE / "io.npz", **io_data)
        unknown = set(parts) - {"io"}
        if unknown:
            raise SystemExit(f"only 'io' can be regenerated on its own, not {sorted(unknown)}")
        (HERE / "golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
        shutil.rmtree(scratch)
        return

    setup, setup_meta = make_setup(ref_pkg)
    np.savez_compressed(HERE / "setup.npz", **setup)
    traj, traj_meta = make_trajectories(ref_pkg)
    np.savez_compressed(HERE / "trajectories.npz", **traj)
    rooms, rooms_meta = make_rooms(ref_pkg, c_backend)
    np.savez_compressed(HERE / "rooms.npz", **rooms)
    impulse, impulse_meta = make_impulse(ref_pkg)
    np.savez_compressed(HERE / "impulse.npz", **impulse)
    io_data, io_meta = make_io(ref_pkg, scratch)
    np.savez_compressed(HERE / "io.npz", **io_data)
    meta = {"setup": setup_meta, "trajectories": traj_meta, "rooms": rooms_meta,
            "impulse": impulse_meta, "io": io_meta,
            "generator": "tests/golden/make_golden.py", "numpy": np.__version__}
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    shutil.rmtree(scratch)
    print("wrote", sorted(p.name for p in HERE.glob("*.np*")), "golden.json")


if __name__ == "__main__":
    main(*sys.argv[1:])
