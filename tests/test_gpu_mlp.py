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


def test_trained_network_predicts_pass_times_better_than_the_static_model():
    """What the trained cost model adds over the planner without it: on
    held-out corpus circuits, the network's pass-time predictions beat the
    static model (time proportional to the bytes a pass moves, its one scale
    fitted to these very passes), and on the held-out circuits where the
    learned plan differs from greedy it is no slower."""
    import ket_b200 as ket
    from ket_b200 import planner as pl
    from ket_b200.workloads import random_mixed
    model = pl.CostModel.load()
    rows_x, rows_y, rows_b = [], [], []
    for n, d, s in [(22, 30, 11), (23, 40, 12), (24, 25, 13), (25, 35, 14)]:
        c = random_mixed(n, d, seed=s)
        for fusion, k in (("none", 5), ("greedy", 3), ("greedy", 5)):
            plan = ket.Plan(n, c.to_ops(), ket.make_options("c64", fusion, k, True))
            ms = pl.timed_execute(plan, pl._state(n))
            for rep in range(2):  # best of three per pass
                ms = np.minimum(ms, pl.timed_execute(plan, pl._state(n)))
            for i in range(len(ms)):
                rows_x.append(pl.pass_features(plan, i))
                rows_y.append(np.log(max(float(ms[i]) * 1e3, 1e-3)))
                rows_b.append(plan.pass_bytes(i))
            plan.close()
    x = np.array(rows_x, dtype=np.float32)
    y = np.array(rows_y)
    b = np.array(rows_b)
    net = model.forward(x).astype(np.float64)
    # static model: log t = log(bytes) + log(scale), the scale fitted here
    static = np.log(b) + np.mean(y - np.log(b))
    rmse_net = float(np.sqrt(np.mean((net - y) ** 2)))
    rmse_static = float(np.sqrt(np.mean((static - y) ** 2)))
    print(f"pass-time log-RMSE: network {rmse_net:.3f}, static {rmse_static:.3f} over {len(y)} passes")
    assert rmse_net < rmse_static
    # held-out circuits whose learned plan differs from greedy (planner_eval.json)
    import json
    import os
    rows = json.load(open(os.path.join(os.path.dirname(pl.__file__), "data", "planner_eval.json")))["rows"]
    diff = [r for r in rows if not r["same_plan"] and r["n"] <= 26]
    tg = tl = 0.0
    for r in diff:
        c = random_mixed(r["n"], r["depth"], seed=r["seed"])
        pl.CostModel.detach()
        pg = ket.Plan(r["n"], c.to_ops(), ket.make_options("c64", "greedy", 0, True))
        model.attach()
        plr = ket.Plan(r["n"], c.to_ops(), ket.make_options("c64", "learned", 0, True))
        pl.CostModel.detach()
        st = pl._state(r["n"])
        g = min(float(pl.timed_execute(pg, st).sum()) for _ in range(3))
        l_ = min(float(pl.timed_execute(plr, st).sum()) for _ in range(3))
        tg, tl = tg + g, tl + l_
        pg.close()
        plr.close()
    if diff:
        print(f"learned / greedy on {len(diff)} differing held-out circuits: {tl / tg:.4f}")
        assert tl <= 1.02 * tg
