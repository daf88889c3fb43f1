"""Generate the golden fixtures in this folder by running the ac-fdtd reference itself.

Run in the build container, where the reference is mounted (it is not on the GPU machines):

    python tests/golden/make_golden.py <path of the ac-fdtd checkout> [part ...]

(or set AC_FDTD_REFERENCE to that path and pass only the parts).

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
import os
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


def make_autograd(ref_pkg) -> tuple[dict, dict]:
    """Gradients of a linear receiver loss by PyTorch autograd through the reference's Torch
    backend (CPU, float64): with respect to the source signal, the initial pressure, the six wall
    admittances and the air's relaxation strengths and times. Autograd needs every coefficient as
    a tensor of those parameters, so the wall coefficient and the relaxation coefficients are
    rebuilt here with the reference's formulas (boundaries.py wall_update_coefficients,
    torch_backend.py __init__), and the backend's two updates that write through out= (which
    autograd cannot follow) are replaced by the same operations in the same order without it."""
    import math

    import torch

    from ac_fdtd import AbsorbingLayer, AirAbsorption, Grid, WallAdmittances
    from ac_fdtd.boundaries import FACES
    from ac_fdtd.sources import gaussian_pulse
    from ac_fdtd.torch_backend import TorchAcousticFDTD

    torch.set_default_dtype(torch.float64)
    grid = Grid(dx=0.05, nx=14, ny=12, nz=10)
    xi = np.array([0.31, 0.12, 0.45, 0.2, 0.08, 0.27])
    air = AirAbsorption(temperature=20.0, relative_humidity=50.0)
    source, receivers = (0.22, 0.31, 0.19), [(0.55, 0.4, 0.35), (0.1, 0.5, 0.42), (0.63, 0.12, 0.08)]
    steps = 90
    solver = TorchAcousticFDTD(grid, dtype=torch.float64, walls=WallAdmittances(*xi),
                               absorbing_layer=AbsorbingLayer(thickness=3), air_absorption=air)
    rng = np.random.default_rng(21)
    p0 = rng.standard_normal(grid.shape)
    w = rng.standard_normal((len(receivers), steps))
    signal = gaussian_pulse(steps, solver.dt, 2500.0)

    p0_t = torch.tensor(p0, requires_grad=True)
    signal_t = torch.tensor(signal, requires_grad=True)
    xi_t = torch.tensor(xi, requires_grad=True)
    processes = air.processes(solver.medium.sound_speed, solver.dt)
    strength_t = torch.tensor([q.strength for q in processes], requires_grad=True)
    tau_t = torch.tensor([q.relaxation_time for q in processes], requires_grad=True)

    # walls: a = sum over the faces touching a cell of c dt xi_f / (2 dx), at the reference's cells
    scale = solver.medium.sound_speed * solver.dt / (2.0 * grid.dx)
    a_field = torch.zeros(grid.shape)
    for f, (axis, side) in enumerate(FACES):
        mask = torch.zeros(grid.shape)
        index = [slice(None)] * 3
        index[axis] = 0 if side == 0 else grid.shape[axis] - 1
        mask[tuple(index)] = 1.0
        a_field = a_field + mask * (scale * xi_t[f])
    a = a_field.reshape(-1)[solver._wall_indices]
    solver._wall_from_updated = 1.0 / (1.0 + a)
    solver._wall_from_previous = a / (1.0 + a)

    # air: the backend's relaxation coefficients as functions of the strengths and times
    c, rho, dt, dx = solver.medium.sound_speed, solver.medium.density, solver.dt, grid.dx
    relaxed = c**2 / (1.0 + strength_t.sum())
    relaxation = []
    for r in range(len(processes)):
        decay = torch.exp(-dt / tau_t[r])
        mean_weight = (tau_t[r] / dt) * (1.0 - decay)
        relaxation.append((torch.zeros(grid.shape), decay, dt * mean_weight,
                           rho * relaxed * strength_t[r] / dx))
    target_scale = dt * sum(gain for _, _, _, gain in relaxation)

    from ac_fdtd.torch_backend import _lower, _upper

    def update_pressure():
        flat = solver.p.view(-1)
        previous = flat[solver._wall_indices].clone()
        divergence = solver.velocity[0][_upper(0)] - solver.velocity[0][_lower(0)]
        for axis in (1, 2):
            divergence = divergence + (solver.velocity[axis][_upper(axis)] - solver.velocity[axis][_lower(axis)])
        for k, (state, decay, mean_weight, gain) in enumerate(relaxation):
            target = divergence * gain
            offset = state - target
            relaxation[k] = (offset * decay + target, decay, mean_weight, gain)
            solver.p = solver.p + offset * mean_weight
        solver.p = solver.p + divergence * target_scale
        solver.p = solver.p - divergence * solver._pressure_coefficient
        flat = solver.p.reshape(-1)
        updated = flat[solver._wall_indices] * solver._wall_from_updated - previous * solver._wall_from_previous
        solver.p = flat.index_put((solver._wall_indices,), updated).reshape(grid.shape)

    solver._update_pressure = update_pressure
    solver._relaxation = []
    solver.p = p0_t * 1.0
    solver.velocity = [v.clone() for v in solver.velocity]
    solver._sources = [(int(np.ravel_multi_index(grid.cell_index(source), grid.shape)), signal_t)]
    for point in receivers:
        solver.add_pressure_receiver(point)
    solver.run(steps)
    loss = (torch.tensor(w) * solver._recording).sum()
    loss.backward()
    data = {"p0": p0, "w": w, "signal": signal, "recording": solver._recording.detach().numpy(),
            "grad_signal": signal_t.grad.numpy(), "grad_p0": p0_t.grad.numpy(),
            "grad_xi": xi_t.grad.numpy(), "grad_strength": strength_t.grad.numpy(),
            "grad_relaxation_time": tau_t.grad.numpy()}
    meta = {"shape": list(grid.shape), "dx": grid.dx, "xi": xi.tolist(), "layer_thickness": 3,
            "air": {"temperature": 20.0, "relative_humidity": 50.0}, "source": source,
            "receivers": receivers, "steps": steps, "max_frequency": 2500.0,
            "torch": torch.__version__, "loss": float(loss.detach())}
    return data, meta


def main(reference: str, *parts: str) -> None:
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
        if "autograd" in parts:
            ag_data, meta["autograd"] = make_autograd(ref_pkg)
            np.savez_compressed(HERE / "autograd.npz", **ag_data)
        unknown = set(parts) - {"io", "autograd"}
        if unknown:
            raise SystemExit(f"only 'io' and 'autograd' can be regenerated on their own, not {sorted(unknown)}")
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
    ag_data, ag_meta = make_autograd(ref_pkg)
    np.savez_compressed(HERE / "autograd.npz", **ag_data)
    meta = {"setup": setup_meta, "trajectories": traj_meta, "rooms": rooms_meta,
            "impulse": impulse_meta, "io": io_meta, "autograd": ag_meta,
            "generator": "tests/golden/make_golden.py", "numpy": np.__version__}
    (HERE / "golden.json").write_text(json.dumps(meta, indent=1, sort_keys=True) + "\n")
    shutil.rmtree(scratch)
    print("wrote", sorted(p.name for p in HERE.glob("*.np*")), "golden.json")


if __name__ == "__main__":
    arguments = sys.argv[1:]
    if arguments and Path(arguments[0], "src", "ac_fdtd").is_dir():
        main(*arguments)
    elif os.environ.get("AC_FDTD_REFERENCE"):
        main(os.environ["AC_FDTD_REFERENCE"], *arguments)
    else:
        sys.exit("usage: make_golden.py <ac-fdtd checkout> [part ...] "
                 "(or set AC_FDTD_REFERENCE)")
