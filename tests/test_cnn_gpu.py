"""The learned short-range network on the GPU against its CPU restatement.

Forward pass, gradients and Adam are compared with the float64 oracle on the
same inputs, with the convolution weights and the input rounded to BF16 as the
tensor cores see them (intermediate activations are BF16 on the device, so
the tolerances are relative norms of a few 1e-3 per layer).  Then the network
is trained on boxes the solver generates and must beat the method without it
on a held-out box.
"""
import numpy as np
import pytest

import cnn_oracle as co

pytestmark = pytest.mark.gpu


def _quantised(params, c_in):
    """Convolution weights rounded to BF16 (biases and head stay FP32)."""
    parts = co.unflatten(params.astype(np.float64), c_in)
    for k in (0, 2, 4):
        parts[k] = co.to_bf16(parts[k])
    return co.flatten(parts)


def _rel(a, b):
    return float(np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-30))


def _batch(seed, B=2, D=14, n=400, c_in=2):
    rng = np.random.default_rng(seed)
    x0 = rng.normal(size=(B, D, D, D, c_in)).astype(np.float32)
    pb = rng.integers(0, B, n).astype(np.int32)
    ps = rng.uniform(0.0, D - 7 - 1e-3, (n, 3)).astype(np.float32)
    tg = rng.normal(size=(n, 3)).astype(np.float32)
    w = rng.uniform(0.5, 1.5, n).astype(np.float32)
    return x0, pb, ps, tg, w


def _net(seed=0):
    from treepm import learned
    return learned.Network(2, params=learned.init_params(2, seed))


@pytest.mark.parametrize("D,c_in", [(7, 2), (12, 2), (21, 2), (12, 10)])
def test_forward_matches_oracle(D, c_in):
    from treepm import learned
    net = learned.Network(c_in, params=learned.init_params(c_in, 1))
    p = net.params()
    rng = np.random.default_rng(D)
    x0 = rng.normal(size=(3, D, D, D, c_in)).astype(np.float32)
    got = net.forward(x0)
    ref = co.forward(_quantised(p, c_in), co.to_bf16(x0))["out"]
    assert got.shape == ref.shape
    assert _rel(got, ref) < 2e-2, _rel(got, ref)
    # with the activations rounded to BF16 between layers, as the device stores them
    ref16 = co.forward(_quantised(p, c_in), co.to_bf16(x0), bf16_activations=True)["out"]
    assert _rel(got, ref16) < 5e-3, _rel(got, ref16)


def test_trained_network_forward_matches_oracle():
    """The committed network (trained weights amplify rounding more than a
    random initialisation) against the BF16-activation restatement."""
    import os
    from treepm import learned
    path = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gadget-ng_b200", "treepm",
                        "weights", "learned_sr.npz")
    net = learned.Network.load(path)
    x0 = np.random.default_rng(3).normal(size=(2, 10, 10, 10, net.c_in)).astype(np.float32)
    got = net.forward(x0)
    ref = co.forward(_quantised(net.params(), net.c_in), co.to_bf16(x0), bf16_activations=True)["out"]
    # one-ulp BF16 rounding flips of intermediate activations (FP32 against
    # float64 accumulation) are amplified by the trained weights
    assert _rel(got, ref) < 3e-2, _rel(got, ref)


def test_gradients_match_oracle():
    net = _net(2)
    p = net.params()
    x0, pb, ps, tg, w = _batch(3)
    loss, grad = net.loss_grad(x0, pb, ps, tg, w)
    ref_loss, ref_grad = co.loss_and_grads(_quantised(p, 2), co.to_bf16(x0), pb, ps.astype(np.float64), tg, w)
    assert abs(loss - ref_loss) < 1e-2 * ref_loss
    parts, refs = co.unflatten(grad, 2), co.unflatten(ref_grad, 2)
    for k, (g, r) in enumerate(zip(parts, refs)):
        cos = float(np.dot(g.ravel(), r.ravel()) / (np.linalg.norm(g) * np.linalg.norm(r) + 1e-30))
        assert _rel(g, r) < 5e-2 and cos > 0.998, (k, _rel(g, r), cos)


def test_adam_matches_oracle():
    net = _net(4)
    p = net.params().astype(np.float64)
    m = np.zeros_like(p)
    v = np.zeros_like(p)
    rng = np.random.default_rng(5)
    for step in range(1, 4):
        g = rng.normal(size=p.shape).astype(np.float32)
        net.adam_step(g, lr=1e-3)
        p, m, v = co.adam(p, g.astype(np.float64), m, v, step, lr=1e-3)
    assert np.max(np.abs(net.params() - p)) < 1e-6


def test_invalid_particle_coordinates_are_rejected():
    from treepm import TreePmError
    net = _net(0)
    x0, pb, ps, tg, w = _batch(6, n=10)
    ps[0, 0] = 7.5  # beyond the last interpolation cell of an 8^3 output
    with pytest.raises(TreePmError):
        net.loss_grad(x0, pb, ps, tg, w)


@pytest.fixture(scope="module")
def trained():
    """A network trained on solver-generated 64^3 clustered boxes (the
    benchmark's cell size), with one held-out box."""
    from treepm import learned
    net = learned.Network(learned.C_IN, params=learned.init_params(learned.C_IN, 7))
    boxes = [learned.training_box(300 + k) for k in range(5)]
    for k, b in enumerate(boxes):
        learned.capture(net, b, 64, held_out=(k == 4))
    p0 = net.params()
    net.set_params(np.zeros_like(p0))
    zero = net.evaluate(held_out=True)  # the loss of predicting no short range
    net.set_params(p0)
    hist = net.train(2000, batch=64, lr=1e-3, seed=11)
    after = net.evaluate(held_out=True)
    return net, boxes[4], zero, after, hist


def test_training_reduces_held_out_loss(trained):
    """The held-out loss falls well below that of predicting zero."""
    net, _, zero, after, hist = trained
    assert np.all(np.isfinite(hist))
    assert after < 0.3 * zero, (zero, after)


def test_learned_solver_beats_the_method_without_it(trained):
    """PM + network (+ walk in dense cells) against the accurate TreePM on the
    held-out box, next to the same solver whose network predicts zero (PM
    alone outside dense cells).  On a B200 the network brings the rms error
    from 9 % to 4 % after 4000 steps on 8 boxes."""
    from treepm import learned, ics
    net, box, _, _, _ = trained
    phys = ics.physics(box, 64, 1.0)
    ref_s = learned.solver_for(box, 64)
    ref_s.set_particles(box.positions(), box.mass)
    ref_s.compute_forces(phys["eps2"], phys["g"])
    _, _, ref = ref_s.get_state(box.n, pos=False, vel=False)

    def run(network):
        s = learned.solver_for(box, 64)
        s.set_learned(network)
        s.set_particles(box.positions(), box.mass)
        s.compute_forces(phys["eps2"], phys["g"])
        _, _, a = s.get_state(box.n, pos=False, vel=False)
        st = s.stats()
        return a, st

    zero = learned.Network(learned.C_IN, params=np.zeros(net.n_params, np.float32))
    zero.set_scales(*net.scales())
    a_net, st = run(net)
    a_zero, st0 = run(zero)
    assert 0 < st["learned_particles"] < box.n and st["learned_particles"] == st0["learned_particles"]
    err = lambda a: float(np.sqrt(np.mean(np.sum((a - ref) ** 2, 1) / np.sum(ref ** 2, 1))))
    assert err(a_net) < 0.6 * err(a_zero), (err(a_net), err(a_zero))


def test_near_field_sum_matches_direct_pairs():
    """The exact near-field option: with a zero network and near_cells = 1, the
    short range of every network particle is the sum over pairs closer than
    one cell (complete split kernel, softened, minimum image) — checked
    against a direct float64 sum."""
    import math
    from scipy.special import erfc
    from treepm import learned, ics
    box = ics.lattice_box(16, 12.5, 1.0, seed=21)
    mesh = 16
    phys = ics.physics(box, mesh, 1.0)
    net = learned.Network(learned.C_IN, params=np.zeros(learned.Network(learned.C_IN).n_params, np.float32))
    net.set_near(1.0)
    net.set_scales(np.zeros(learned.C_IN), np.ones(learned.C_IN), 1.0, 1e6)
    s = learned.solver_for(box, mesh)
    s.set_learned(net)
    pos = box.positions()
    s.set_particles(pos, box.mass)
    s.compute_forces(phys["eps2"], phys["g"])
    assert s.stats()["learned_particles"] == box.n
    _, sr = s.force_parts(box.n)
    L = box.box_size
    rn = L / mesh
    t = np.arange(0, box.n, 37)
    ref = np.zeros((len(t), 3))
    for k, i in enumerate(t):
        d = pos - pos[i]
        d -= L * np.round(d / L)
        r2b = np.sum(d * d, 1)
        m = (r2b < rn * rn) & (np.arange(box.n) != i)
        r2 = r2b[m] + phys["eps2"]
        r = np.sqrt(r2)
        x = r / (math.sqrt(2.0) * phys["r_split"])
        w = erfc(x) + 2.0 / math.sqrt(math.pi) * x * np.exp(-x * x)
        ref[k] = phys["g"] * np.sum((box.mass[m] * w / (r2 * r))[:, None] * d[m], 0)
    err = np.linalg.norm(sr[t] - ref, axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-30)
    assert np.sqrt(np.mean(err ** 2)) < 1e-4, float(np.sqrt(np.mean(err ** 2)))


@pytest.mark.gpu
def test_tensor_core_wait_times_out_and_reports():
    """Failure detection without a fault: a conv tile whose MMAs are never
    issued waits on an mbarrier nothing completes; the wait must give up at
    its 2 s limit, flag the timeout and free its TMEM, and a normal tile must
    then run on the same context (checked inside the self-test).  A network
    forward afterwards still matches the oracle."""
    import ctypes as C
    from treepm import load
    t = C.c_double(0.0)
    assert load().tpm_selftest_bounded_wait(0, C.byref(t)) == 0
    assert 1.9 < t.value < 10.0
    net = _net(0)
    x0, pb, ps, tg, w = _batch(7, n=10)
    loss, grads = net.loss_grad(x0, pb, ps, tg, w)
    assert np.isfinite(loss)
