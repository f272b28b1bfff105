"""The learned planner's MLP on the GPU: forward and gradients against the
CPU oracle (the same BF16-rounded weights, FP64 reference), training, and
plans chosen with the model giving the unfused state (1e-5, complex64)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_forward_and_gradients_match_oracle(oracle):
    from ket_b200.planner import CostModel
    m = CostModel(seed=3)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((37, 48)).astype(np.float32)
    y = rng.standard_normal(37).astype(np.float32)
    w = m.weights()  # BF16-rounded values the kernels use
    out = m.forward(x)
    ref = oracle.mlp_forward(w, x)
    assert np.abs(out - ref).max() < 1e-4 * (1 + np.abs(ref).max())
    loss, g = m.gradients(x, y)
    ref_loss, ref_g = oracle.mlp_backward(w, x, y)
    assert abs(loss - ref_loss) < 1e-4 * (1 + abs(ref_loss))
    for a, b in zip(g, ref_g):
        assert np.abs(a - b).max() < 1e-4 * (1 + np.abs(b).max())
    m.close()


def test_training_reduces_loss():
    from ket_b200.planner import CostModel
    rng = np.random.default_rng(1)
    x = rng.standard_normal((4096, 48)).astype(np.float32)
    wt = rng.standard_normal(48).astype(np.float32)
    y = (np.tanh(x @ wt / 7.0) * 3 + 0.1 * rng.standard_normal(4096)).astype(np.float32)
    m = CostModel(seed=5)
    before = float(np.mean((m.forward(x) - y) ** 2))
    m.train(x, y, steps=1500, minibatch=256, lr=2e-3)
    after = float(np.mean((m.forward(x) - y) ** 2))
    assert after < 0.2 * before
    m.close()


def test_learned_plans_are_correct(oracle):
    import ket_b200 as ket
    from ket_b200.planner import CostModel, measure_passes
    from ket_b200.workloads import random_mixed
    m = CostModel(seed=9)
    xs, ys = [], []
    for s in range(6):
        x, y = measure_passes(random_mixed(14, 6, seed=100 + s))
        xs.append(x)
        ys.append(y)
    m.train(np.concatenate(xs), np.concatenate(ys), steps=800, minibatch=128, lr=2e-3)
    m.attach()
    try:
        for s in range(4):
            c = random_mixed(13, 12, seed=200 + s)
            want = oracle.run(13, c.to_ops(), fuse=0)
            d = ket.run_device(c, options=ket.make_options("c64", "learned", 5, True))
            assert np.abs(d.to_numpy() - want).max() < 1e-5
            st = ket.plan_stats(c, ket.make_options("c64", "learned", 5, True))
            assert st["predicted_us"] > 0
            d.close()
    finally:
        CostModel.detach()
        m.close()
