"""The adjoint kernels give the exact gradient of the discrete leapfrog.

* Dot-product identity: recordings are linear in the initial pressure, so for any weights y,
  <rec(p0), y> = <p0, lambda_p0(y)> to rounding -- a test of the transposed sweeps alone.
* Central finite differences in float64 (relative step 1e-6) for the six wall admittances,
  per-patch admittances, source samples and ISO relaxation strengths; agreement within 1e-6
  relative to the largest gradient of the group. A wall behind a sponge has a gradient 1e4
  times smaller than the others; its finite difference at step 1e-6 is then limited by the
  rounding of the loss (it converges to the adjoint's value only for steps of 1e-4 and up), so
  each group is held to 1e-6 of its own scale rather than of each entry. The ISO strengths are
  themselves 1e-5 to 1e-3, so a relative step of 1e-6 moves the loss by less than its rounding;
  their differences use a relative step of 1e-4, where the central difference has converged
  (checked against steps from 1e-5 to 1e-3 on the oracle).
"""

from __future__ import annotations

import numpy as np
import pytest

from ac_fdtd_b200 import AbsorbingLayer, AirAbsorption, Grid, WallAdmittances, gaussian_pulse
from ac_fdtd_b200.adjoint import DifferentiableRoom, FixedProcesses
from ac_fdtd_b200.boundaries import WallPatches

pytestmark = pytest.mark.gpu

GRID = Grid(dx=0.05, nx=14, ny=12, nz=10)
XI = (0.31, 0.12, 0.45, 0.2, 0.08, 0.27)
SOURCE = (0.22, 0.31, 0.19)
RECEIVERS = [(0.55, 0.4, 0.35), (0.1, 0.5, 0.42), (0.63, 0.12, 0.08)]
STEPS = 90


def make_room(walls=None, air=None, layer=None, wrt=("signal", "walls"), dtype=np.float64,
              every=None, steps=STEPS):
    room = DifferentiableRoom(GRID, dtype=dtype, walls=walls or WallAdmittances(*XI),
                              absorbing_layer=layer, air_absorption=air, max_steps=steps,
                              wrt=wrt, checkpoint_every=every)
    room.solver.add_volume_source(SOURCE, gaussian_pulse(steps, room.dt, 2500.0))
    for point in RECEIVERS:
        room.solver.add_pressure_receiver(point)
    return room


def weights(seed=0, steps=STEPS):
    return np.random.default_rng(seed).standard_normal((len(RECEIVERS), steps))


def loss(rec, w):
    return 0.5 * float(np.sum(w * rec.astype(np.float64) ** 2))


def test_dot_product_identity_of_the_transposed_sweeps():
    air = AirAbsorption(temperature=18.0, relative_humidity=40.0)
    room = make_room(air=air, layer=AbsorbingLayer(thickness=3))
    room.solver.clear_sources()
    p0 = np.random.default_rng(1).standard_normal(GRID.shape)
    y = weights(2)
    rec = room.forward(STEPS, p0=p0)
    grads = room.backward(y)
    lhs = float(np.sum(rec * y))
    rhs = float(np.sum(p0 * grads.initial_p))
    assert lhs == pytest.approx(rhs, rel=1e-12)


@pytest.mark.parametrize("with_layer", [False, True])
def test_wall_and_source_gradients_match_central_differences(with_layer):
    layer = AbsorbingLayer(thickness=3, faces=((0, 1), (2, 0))) if with_layer else None
    air = AirAbsorption()
    w = weights(3)
    room = make_room(air=air, layer=layer)
    base = room.forward(STEPS)
    grads = room.backward(w * base)

    def value(xi=XI, signal=None):
        room.set_parameters(walls=WallAdmittances(*xi))
        if signal is not None:
            room.solver.clear_sources()
            room.solver.add_volume_source(SOURCE, signal)
        return loss(room.forward(STEPS), w)

    fds = []
    for f in range(6):
        h = 1e-6 * XI[f]
        plus = list(XI)
        minus = list(XI)
        plus[f] += h
        minus[f] -= h
        fds.append((value(plus) - value(minus)) / (2 * h))
    fds = np.array(fds)
    assert np.max(np.abs(grads.walls - fds)) <= 1e-6 * np.max(np.abs(fds)), (grads.walls, fds)
    value(XI)
    signal = gaussian_pulse(STEPS, room.dt, 2500.0)
    samples = (3, 10, 25, 60)
    fds = []
    for n in samples:
        h = 1e-6 * max(abs(signal[n]), 1e-3)
        plus, minus = signal.copy(), signal.copy()
        plus[n] += h
        minus[n] -= h
        fds.append((value(signal=plus) - value(signal=minus)) / (2 * h))
    fds = np.array(fds)
    got = grads.signal[0, list(samples)]
    assert np.max(np.abs(got - fds)) <= 1e-6 * np.max(np.abs(grads.signal)), (got, fds)


def test_patch_gradients_match_central_differences():
    P = 2
    values = np.random.default_rng(4).uniform(0.05, 0.6, (6, P, P))
    w = weights(5)
    room = make_room(walls=WallPatches(values))
    grads = room.backward(w * room.forward(STEPS))
    assert grads.walls.shape == (6, P, P)
    checked = ((0, 0, 1), (3, 1, 1), (5, 1, 0), (2, 0, 0))
    fds = []
    for f, a, b in checked:
        h = 1e-6 * values[f, a, b]
        plus, minus = values.copy(), values.copy()
        plus[f, a, b] += h
        minus[f, a, b] -= h
        room.set_parameters(walls=WallPatches(plus))
        lp = loss(room.forward(STEPS), w)
        room.set_parameters(walls=WallPatches(minus))
        lm = loss(room.forward(STEPS), w)
        fds.append((lp - lm) / (2 * h))
    got = np.array([grads.walls[c] for c in checked])
    assert np.max(np.abs(got - np.array(fds))) <= 1e-6 * np.max(np.abs(grads.walls)), (got, fds)


@pytest.mark.parametrize("every", [7, 90, None])
def test_air_strength_gradients_match_central_differences(every):
    air = AirAbsorption(temperature=22.0, relative_humidity=35.0)
    room = make_room(air=air, wrt=("signal", "walls", "air"), every=every)
    c, dt = 343.2, room.dt
    processes = air.processes(room.solver.medium.sound_speed, dt)
    strengths = np.array([p.strength for p in processes])
    taus = np.array([p.relaxation_time for p in processes])
    w = weights(6)
    room.set_parameters(air_absorption=FixedProcesses(strengths, taus))
    grads = room.backward(w * room.forward(STEPS))
    fds = []
    for r in range(len(processes)):
        h = 1e-4 * strengths[r]
        plus, minus = strengths.copy(), strengths.copy()
        plus[r] += h
        minus[r] -= h
        room.set_parameters(air_absorption=FixedProcesses(plus, taus))
        lp = loss(room.forward(STEPS), w)
        room.set_parameters(air_absorption=FixedProcesses(minus, taus))
        lm = loss(room.forward(STEPS), w)
        fds.append((lp - lm) / (2 * h))
    fds = np.array(fds)
    assert np.max(np.abs(grads.strength - fds)) <= 1e-6 * np.max(np.abs(fds)), (grads.strength, fds)
    r = 1
    h = 1e-4 * taus[r]
    plus, minus = taus.copy(), taus.copy()
    plus[r] += h
    minus[r] -= h
    room.set_parameters(air_absorption=FixedProcesses(strengths, plus))
    lp = loss(room.forward(STEPS), w)
    room.set_parameters(air_absorption=FixedProcesses(strengths, minus))
    lm = loss(room.forward(STEPS), w)
    fd_tau = (lp - lm) / (2 * h)
    assert abs(grads.relaxation_time[r] - fd_tau) <= 1e-6 * np.max(np.abs(grads.relaxation_time))


def test_single_precision_adjoint_tracks_double():
    w = weights(7)
    g64 = make_room(air=AirAbsorption()).backward
    r64 = make_room(air=AirAbsorption())
    grads64 = r64.backward(w * r64.forward(STEPS))
    r32 = make_room(air=AirAbsorption(), dtype=np.float32)
    grads32 = r32.backward(w * r32.forward(STEPS))
    del g64
    np.testing.assert_allclose(grads32.walls, grads64.walls, rtol=2e-3)
    scale = np.max(np.abs(grads64.signal))
    assert np.max(np.abs(grads32.signal - grads64.signal)) < 1e-3 * scale


def test_torch_autograd_function_backpropagates():
    torch = pytest.importorskip("torch")
    from ac_fdtd_b200.adjoint import room_response

    room = make_room()
    xi = torch.tensor(XI, dtype=torch.float64, requires_grad=True)
    signal = torch.tensor(gaussian_pulse(STEPS, room.dt, 2500.0), requires_grad=True)
    rec = room_response(room, SOURCE, xi, signal, STEPS)
    target = torch.zeros_like(rec)
    loss_t = 0.5 * ((rec - target) ** 2).sum()
    loss_t.backward()
    direct = room.backward(rec.detach().numpy())
    np.testing.assert_allclose(xi.grad.numpy(), direct.walls, rtol=1e-12)
    np.testing.assert_allclose(signal.grad.numpy(), direct.signal[0], rtol=1e-12, atol=1e-300)


def test_differentiable_room_full_size_matches_central_differences():
    """The differentiable configuration at its full size in float64: 128^3, 3000 steps, L2
    misfit to the signals of the true admittances from a start perturbed by up to 30 %: the six
    wall admittances and four of the 3000 source samples against central differences."""
    from ac_fdtd_b200.workloads import differentiable_room

    grid, true_xi, start_xi, source, receivers = differentiable_room()
    steps = 3000
    room = DifferentiableRoom(grid, dtype=np.float64, walls=WallAdmittances(*true_xi),
                              max_steps=steps, wrt=("signal", "walls"))
    signal = gaussian_pulse(steps, room.dt, 2000.0)
    room.solver.add_volume_source(source, signal)
    for point in receivers:
        room.solver.add_pressure_receiver(point)
    target = room.forward(steps).copy()

    def misfit(xi):
        room.set_parameters(walls=WallAdmittances(*xi))
        rec = room.forward(steps)
        return 0.5 * float(np.sum((rec - target) ** 2)), rec

    value, rec = misfit(start_xi)
    grads = room.backward(rec - target)
    fds = []
    for f in range(6):
        h = 1e-6 * start_xi[f]
        plus, minus = start_xi.copy(), start_xi.copy()
        plus[f] += h
        minus[f] -= h
        fds.append((misfit(plus)[0] - misfit(minus)[0]) / (2 * h))
    fds = np.array(fds)
    assert value > 0
    assert np.max(np.abs(grads.walls - fds)) <= 1e-6 * np.max(np.abs(fds)), (grads.walls, fds)

    # source samples at the start walls: before, at and after the pulse's peak, and late in the
    # run (recordings are linear in the signal, so the central difference is exact to rounding)
    room.set_parameters(walls=WallAdmittances(*start_xi))
    samples = (5, int(np.argmax(signal)), 400, 2500)

    def misfit_signal(sig):
        room.solver.clear_sources()
        room.solver.add_volume_source(source, sig)
        rec = room.forward(steps)
        return 0.5 * float(np.sum((rec - target) ** 2))

    fds = []
    for n in samples:
        h = 1e-6 * max(abs(signal[n]), 1e-3)
        plus, minus = signal.copy(), signal.copy()
        plus[n] += h
        minus[n] -= h
        fds.append((misfit_signal(plus) - misfit_signal(minus)) / (2 * h))
    fds = np.array(fds)
    got = grads.signal[0, list(samples)]
    assert np.max(np.abs(got - fds)) <= 1e-6 * np.max(np.abs(grads.signal)), (got, fds)


def test_air_gradients_agree_with_and_without_recompute():
    """Whole-run history (the recorded run keeps D and psi) and checkpoint recompute give the
    same gradients bit for bit, also for a run shorter than the prepared capacity."""
    air = AirAbsorption(temperature=19.0, relative_humidity=55.0)
    results = []
    for every in (STEPS, 9):
        room = make_room(air=air, wrt=("signal", "walls", "air"), every=every)
        assert room.checkpoint_every == every
        w = weights(8, steps=STEPS - 13)
        g = room.backward(w * room.forward(STEPS - 13))
        results.append((g.strength, g.relaxation_time, g.walls, g.signal))
        room.solver.close()
    for a, b in zip(*results, strict=True):
        np.testing.assert_array_equal(a, b)
    auto = make_room(air=air, wrt=("signal", "walls", "air"))
    assert auto.checkpoint_every == STEPS          # a small room's history always fits


def test_single_precision_packed_air_adjoint_tracks_double():
    """Single precision with nz a multiple of 4 reverses its steps with the packed adjoint step,
    air sums included; against the double-precision generic adjoint: walls and source to
    2e-3 / 1e-3 as the unpacked single-precision adjoint, the ISO strengths and times to 2e-3 of
    their largest gradient. With whole-run history and with checkpoint recompute the single-
    precision gradients agree bit for bit."""
    grid = Grid(dx=0.05, nx=14, ny=12, nz=12)
    air = AirAbsorption(temperature=19.0, relative_humidity=55.0)
    steps = 77

    def gradients(dtype, every):
        room = DifferentiableRoom(grid, dtype=dtype, walls=WallAdmittances(*XI), air_absorption=air,
                                  max_steps=steps, wrt=("signal", "walls", "air"), checkpoint_every=every)
        room.solver.add_volume_source(SOURCE, gaussian_pulse(steps, room.dt, 2500.0))
        for point in RECEIVERS:
            room.solver.add_pressure_receiver(point)
        rec = room.forward(steps).astype(np.float64)
        w = np.random.default_rng(12).standard_normal(rec.shape)
        g = room.backward(w * rec)
        room.solver.close()
        return g

    g64 = gradients(np.float64, steps)
    g32 = gradients(np.float32, steps)
    g32_recompute = gradients(np.float32, 9)
    for name in ("walls", "signal", "strength", "relaxation_time"):
        np.testing.assert_array_equal(getattr(g32, name), getattr(g32_recompute, name))
    np.testing.assert_allclose(g32.walls, g64.walls, rtol=2e-3)
    assert np.max(np.abs(g32.signal - g64.signal)) < 1e-3 * np.max(np.abs(g64.signal))
    for name in ("strength", "relaxation_time"):
        a, b = getattr(g32, name), getattr(g64, name)
        assert np.max(np.abs(a - b)) <= 2e-3 * np.max(np.abs(b)), (name, a, b)


@pytest.mark.parametrize("every", [STEPS, 9])
def test_l2_prefetch_leaves_gradients_unchanged(every):
    """The plane prefetch (off by default at this size, forced on here) touches no arithmetic:
    forward recordings and every gradient are bit-identical, with and without recompute."""
    air = AirAbsorption(temperature=21.0, relative_humidity=45.0)
    results = []
    for prefetch in (False, True):
        room = make_room(air=air, layer=AbsorbingLayer(thickness=3),
                         wrt=("signal", "walls", "air"), every=every)
        room.solver.set_prefetch(prefetch)
        assert room.solver.prefetch == prefetch
        w = weights(3)
        rec = room.forward(STEPS)
        g = room.backward(w * rec)
        results.append((rec, g.strength, g.relaxation_time, g.walls, g.signal, g.initial_p))
        room.solver.close()
    for a, b in zip(*results, strict=True):
        np.testing.assert_array_equal(a, b)
