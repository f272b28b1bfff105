"""The learned fusion planner: cost-model training and evaluation.

* ``CostModel`` wraps the on-GPU MLP (ketgpu_mlp_*: 48 -> 128 -> 128 -> 1,
  BF16 weights, FP32 accumulation, hand-written forward/backward/Adam
  kernels).  It regresses log(pass time in microseconds).
* ``measure_passes`` produces training rows: every candidate plan of a
  circuit (unfused, and greedy blocks at k = 3..6) is executed with per-pass
  CUDA-event timing (ketgpu_plan_execute_timed) and each pass contributes its
  48 features (ketgpu_plan_pass_features) and its measured time.
* With a model attached (``CostModel.attach``) the planner's FUSE_LEARNED
  mode scores every candidate block both fused and as separate gates and
  keeps the partition with the least predicted time; without one it falls
  back to greedy fusion.

``python -m ket_b200.planner`` runs the corpus experiment: 2000 seeded random
circuits (22-32 qubits, depth 20-60, gate mix H/S/T/Rx/Ry/Rz/U/CX/CZ/CP/CRz/
SWAP/CCX/CSWAP), trains on timings measured on 1500 of them, and on the 500
held out compares learned plans with greedy and unfused ones (time, and the
state against the unfused one).
"""
from __future__ import annotations

import argparse
import ctypes as ct
import json
import os
import time
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from . import _lib
from ._lib import check, lib
from .api import DeviceState, Plan, make_options
from .circuit import Circuit

NF = 48
HID = 128
DATA_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
DEFAULT_MODEL = os.path.join(DATA_DIR, "cost_model.npz")


class CostModel:
    """The MLP cost model on the current CUDA device."""

    def __init__(self, seed: int = 1):
        h = ct.c_void_p()
        check(lib.ketgpu_mlp_create(seed, ct.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            lib.ketgpu_mlp_destroy(self._h)
            self._h = ct.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def weights(self) -> List[np.ndarray]:
        w = [np.zeros((HID, NF), np.float32), np.zeros(HID, np.float32), np.zeros((HID, HID), np.float32),
             np.zeros(HID, np.float32), np.zeros(HID, np.float32), np.zeros(1, np.float32)]
        check(lib.ketgpu_mlp_get_weights(self._h, *[a.ctypes.data for a in w]))
        return w

    def set_weights(self, w: Sequence[np.ndarray]) -> None:
        ws = [np.ascontiguousarray(a, dtype=np.float32) for a in w]
        check(lib.ketgpu_mlp_set_weights(self._h, *[a.ctypes.data for a in ws]))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros(len(x), dtype=np.float32)
        check(lib.ketgpu_mlp_forward(self._h, x.ctypes.data, len(x), out.ctypes.data))
        return out

    def gradients(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        g = [np.zeros((HID, NF), np.float32), np.zeros(HID, np.float32), np.zeros((HID, HID), np.float32),
             np.zeros(HID, np.float32), np.zeros(HID, np.float32), np.zeros(1, np.float32)]
        loss = ct.c_float()
        check(lib.ketgpu_mlp_gradients(self._h, x.ctypes.data, y.ctypes.data, len(x), ct.byref(loss),
                                       *[a.ctypes.data for a in g]))
        return loss.value, g

    def train(self, x: np.ndarray, y: np.ndarray, steps: int = 2000, minibatch: int = 256,
              lr: float = 1e-3) -> float:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.ascontiguousarray(y, dtype=np.float32)
        loss = ct.c_float()
        check(lib.ketgpu_mlp_train(self._h, x.ctypes.data, y.ctypes.data, len(x), steps, minibatch, lr,
                                   ct.byref(loss)))
        return loss.value

    def predict_us(self, x: np.ndarray) -> np.ndarray:
        return np.exp(self.forward(x).astype(np.float64))

    def attach(self) -> None:
        check(lib.ketgpu_planner_set_model(self._h))

    @staticmethod
    def detach() -> None:
        check(lib.ketgpu_planner_set_model(None))

    def save(self, path: str) -> None:
        w = self.weights()
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, w1=w[0], b1=w[1], w2=w[2], b2=w[3], w3=w[4], b3=w[5])

    @classmethod
    def load(cls, path: str = DEFAULT_MODEL) -> "CostModel":
        d = np.load(path)
        m = cls()
        m.set_weights([d["w1"], d["b1"], d["w2"], d["b2"], d["w3"], d["b3"]])
        return m


def pass_features(plan: Plan, index: int) -> np.ndarray:
    out = np.zeros(NF, dtype=np.float32)
    check(lib.ketgpu_plan_pass_features(plan._h, index, out.ctypes.data))
    return out


_states: Dict[int, DeviceState] = {}


def _state(n: int) -> DeviceState:
    if n not in _states:
        _states[n] = DeviceState(n, "c64")
    return _states[n]


def timed_execute(plan: Plan, state: DeviceState) -> np.ndarray:
    npass = int(plan.stats()["n_passes"])
    ms = np.zeros(max(1, npass), dtype=np.float32)
    check(lib.ketgpu_plan_execute_timed(plan._h, state.handle, ms.ctypes.data))
    return ms[:npass]


def measure_passes(circuit: Circuit, variants=(("none", 5), ("greedy", 3), ("greedy", 4), ("greedy", 5),
                                               ("greedy", 6))) -> Tuple[np.ndarray, np.ndarray]:
    """Training rows (features, log us) from every pass of each candidate plan."""
    n = circuit.n_qubits
    st = _state(n)
    ops = circuit.to_ops()
    xs, ys = [], []
    for fusion, k in variants:
        plan = Plan(n, ops, make_options("c64", fusion, k, True))
        ms = timed_execute(plan, st)  # matrices are uploaded before the first event
        for i in range(len(ms)):
            xs.append(pass_features(plan, i))
            ys.append(np.log(max(float(ms[i]) * 1e3, 1e-3)))
        plan.close()
    return np.array(xs, dtype=np.float32), np.array(ys, dtype=np.float32)


def corpus(count: int = 2000, seed: int = 2024, nmin: int = 22, nmax: int = 32, dmin: int = 20,
           dmax: int = 60) -> List[Tuple[int, int, int]]:
    """(n, depth, circuit seed) for each circuit of the corpus."""
    g = np.random.default_rng(seed)
    return [(int(g.integers(nmin, nmax + 1)), int(g.integers(dmin, dmax + 1)), int(g.integers(0, 2**31)))
            for _ in range(count)]


def plan_signature(plan: Plan) -> bytes:
    """Pass kinds, sizes, bytes and cost-model features of every pass: equal
    for two plans that apply the same passes."""
    import ctypes as ct
    parts = []
    for i in range(int(plan.stats()["n_passes"])):
        kind, k, tc, b = ct.c_int32(), ct.c_int32(), ct.c_int32(), ct.c_double()
        check(lib.ketgpu_plan_pass_info(plan._h, i, ct.byref(kind), ct.byref(k), ct.byref(tc), ct.byref(b)))
        parts.append(np.array([kind.value, k.value, tc.value, b.value], dtype=np.float64).tobytes())
        parts.append(pass_features(plan, i).tobytes())
    return b"".join(parts)


def plan_time_ms(circuit: Circuit, fusion: str, k: int = 5, reps: int = 1) -> Tuple[float, Plan]:
    plan = Plan(circuit.n_qubits, circuit.to_ops(), make_options("c64", fusion, k, True))
    st = _state(circuit.n_qubits)
    best = min(float(timed_execute(plan, st).sum()) for _ in range(reps))
    return best, plan


def main(argv: Optional[Sequence[str]] = None) -> None:
    from .workloads import random_mixed
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", type=int, default=1500)
    ap.add_argument("--eval", type=int, default=500)
    ap.add_argument("--train-gates", type=int, default=0,
                    help="gates of each training circuit that are timed (0: the whole circuit)")
    ap.add_argument("--check", type=int, default=60, help="held-out circuits whose states are compared")
    ap.add_argument("--unfused", type=int, default=60, help="held-out circuits also timed unfused")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--out", required=True, help="JSON file for the training and evaluation record")
    ap.add_argument("--save", default=DEFAULT_MODEL)
    ap.add_argument("--nmax", type=int, default=32)
    ap.add_argument("--load", default=None, help="evaluate this trained model (skips measuring and training)")
    ap.add_argument("--measure-budget-s", type=float, default=0.0,
                    help="stop timing training circuits after this many seconds (0: no limit); the record "
                         "states how many circuits were timed")
    args = ap.parse_args(argv)

    circs = corpus(args.train + args.eval, nmax=args.nmax)
    train_spec, eval_spec = circs[:args.train], circs[args.train:]
    # one-time warm-up: module load and first launches outside any timing
    w = random_mixed(12, 4, seed=1)
    measure_passes(w)
    t0 = time.time()
    X, Y = [], []
    if args.load:
        train_spec = []
    timed_circuits = 0
    for j, (n, d, s) in enumerate(train_spec):
        if args.measure_budget_s > 0 and time.time() - t0 > args.measure_budget_s:
            break
        timed_circuits += 1
        c = random_mixed(n, d, seed=s)
        sub = c
        if args.train_gates > 0:
            sub = Circuit(n)
            sub._gates = c.gates[:args.train_gates]
        x, y = measure_passes(sub)
        X.append(x)
        Y.append(y)
        if j % 100 == 0:
            print(f"measured {j}/{len(train_spec)} circuits, {sum(len(a) for a in X)} rows, "
                  f"{time.time() - t0:.0f} s", flush=True)
    t_measure = time.time() - t0
    curve = []
    if args.load:
        model = CostModel.load(args.load)
        X = np.zeros((0, NF), dtype=np.float32)
        loss0 = loss = train_rmse = None
        t_train = 0.0
    else:
        X = np.concatenate(X)
        Y = np.concatenate(Y)
        os.makedirs(os.path.dirname(args.out) or ".", exist_ok=True)
        np.savez_compressed(os.path.splitext(args.out)[0] + "_rows.npz", X=X, Y=Y)
        model = CostModel(seed=7)
        loss0 = float(np.mean((model.forward(X) - Y) ** 2))
        t1 = time.time()
        # Adam in the library's kernels, in 30 legs; the full-batch mean
        # squared error after each leg is the loss curve
        curve = []
        legs = [(args.steps // 20, 2e-3)] * 20 + [(args.steps // 20, 5e-4)] * 10
        for steps, lr in legs:
            model.train(X, Y, steps=max(1, steps), minibatch=512, lr=lr)
            curve.append(float(np.mean((model.forward(X) - Y) ** 2)))
        loss = curve[-1]
        t_train = time.time() - t1
        pred = model.forward(X)
        train_rmse = float(np.sqrt(np.mean((pred - Y) ** 2)))
        model.save(args.save)

    # held-out evaluation
    rng = np.random.default_rng(99)
    check_set = set(rng.choice(len(eval_spec), min(args.check, len(eval_spec)), replace=False).tolist())
    unfused_set = set(rng.choice(len(eval_spec), min(args.unfused, len(eval_spec)), replace=False).tolist())
    rows = []
    Xe, Ye = [], []
    for i, (n, d, s) in enumerate(eval_spec):
        c = random_mixed(n, d, seed=s)
        # plans are built first, then timed in an order that alternates from
        # circuit to circuit (the plan timed second runs on a warmer GPU)
        CostModel.detach()
        p_greedy = Plan(n, c.to_ops(), make_options("c64", "greedy", 0, True))  # library default k
        model.attach()
        p_learned = Plan(n, c.to_ops(), make_options("c64", "learned", 0, True))
        CostModel.detach()
        st_ = _state(n)
        if i % 2 == 0:
            t_greedy = float(timed_execute(p_greedy, st_).sum())
            t_learned = float(timed_execute(p_learned, st_).sum())
        else:
            t_learned = float(timed_execute(p_learned, st_).sum())
            t_greedy = float(timed_execute(p_greedy, st_).sum())
        # the fixed alternative: greedy growth with 5-qubit blocks
        p_greedy5 = Plan(n, c.to_ops(), make_options("c64", "greedy", 5, True))
        t_greedy5 = float(timed_execute(p_greedy5, st_).sum())
        p_greedy5.close()
        same = plan_signature(p_greedy) == plan_signature(p_learned)
        if not same:  # two more alternating timings of each plan, best of three
            st = _state(n)
            for _ in range(2):
                t_greedy = min(t_greedy, float(timed_execute(p_greedy, st).sum()))
                t_learned = min(t_learned, float(timed_execute(p_learned, st).sum()))
        pred_learned = float(p_learned.stats()["predicted_us"]) / 1e3
        row = {"n": n, "depth": d, "seed": s, "gates": int(p_greedy.stats()["n_gates"]),
               "greedy_ms": t_greedy, "learned_ms": t_learned, "greedy5_ms": t_greedy5, "learned_pred_ms": pred_learned,
               "greedy_passes": int(p_greedy.stats()["n_passes"]), "learned_passes": int(p_learned.stats()["n_passes"]),
               "same_plan": bool(same)}
        if i in unfused_set or i in check_set:
            CostModel.detach()
            t_un, p_un = plan_time_ms(c, "none")
            if i in unfused_set:
                row["unfused_ms"] = t_un
            if i in check_set:
                ref = _state(n)
                ref.reset()
                p_un.execute(ref)
                for name, p in (("greedy", p_greedy), ("learned", p_learned)):
                    other = DeviceState(n, "c64")
                    p.execute(other)
                    cmp = other.compare(ref)
                    row[name + "_max_abs_vs_unfused"] = cmp["max_abs"]
                    other.close()
            p_un.close()
        p_greedy.close()
        p_learned.close()
        rows.append(row)
        if i % 50 == 0:
            print(f"evaluated {i}/{len(eval_spec)}", flush=True)
    CostModel.detach()
    gt = np.array([r["greedy_ms"] for r in rows])
    lt = np.array([r["learned_ms"] for r in rows])
    un = [(r["unfused_ms"], r["greedy_ms"], r["learned_ms"]) for r in rows if "unfused_ms" in r]
    errs = [max(r["greedy_max_abs_vs_unfused"], r["learned_max_abs_vs_unfused"]) for r in rows
            if "greedy_max_abs_vs_unfused" in r]
    import hashlib
    model_path = args.load or args.save
    summary = {
        "model": model_path,
        "model_sha256": hashlib.sha256(open(model_path, "rb").read()).hexdigest(),
        "train_circuits": len(train_spec), "train_circuits_timed": timed_circuits if not args.load else 0,
        "train_gates_per_circuit": args.train_gates or "all",
        "eval_circuits": len(eval_spec), "train_rows": int(len(X)),
        "measure_s": t_measure, "train_s": t_train, "loss_initial": loss0, "loss_final": loss,
        "loss_curve": curve, "train_rmse_log_us": train_rmse,
        "eval_total_greedy_ms": float(gt.sum()), "eval_total_learned_ms": float(lt.sum()),
        "eval_learned_over_greedy": float(lt.sum() / gt.sum()),
        "eval_learned_over_greedy_k5": float(lt.sum() / sum(r["greedy5_ms"] for r in rows)),
        "eval_greedy_k5_over_greedy": float(sum(r["greedy5_ms"] for r in rows) / gt.sum()),
        "eval_learned_over_greedy_geomean": float(np.exp(np.mean(np.log(lt / gt)))),
        "eval_same_plan_count": int(sum(r["same_plan"] for r in rows)),
        "eval_differing_plans": int(sum(not r["same_plan"] for r in rows)),
        "eval_differing_learned_over_greedy": (float(sum(r["learned_ms"] for r in rows if not r["same_plan"]) /
                                                     sum(r["greedy_ms"] for r in rows if not r["same_plan"]))
                                               if any(not r["same_plan"] for r in rows) else None),
        "eval_same_plan_measured_ratio": (float(sum(r["learned_ms"] for r in rows if r["same_plan"]) /
                                                sum(r["greedy_ms"] for r in rows if r["same_plan"]))
                                          if any(r["same_plan"] for r in rows) else None),
        "eval_learned_faster_count": int((lt < gt * 0.995).sum()), "eval_learned_slower_count": int((lt > gt * 1.005).sum()),
        "unfused_subset": len(un), "unfused_total_ms": float(sum(u for u, _, _ in un)),
        "greedy_total_on_unfused_subset_ms": float(sum(g for _, g, _ in un)),
        "learned_total_on_unfused_subset_ms": float(sum(l for _, _, l in un)),
        "checked_states": len(errs), "max_abs_vs_unfused": float(max(errs)) if errs else None,
    }
    os.makedirs(os.path.dirname(args.out) or ".", exist_ok=True)
    with open(args.out, "w") as f:
        json.dump({"summary": summary, "rows": rows}, f)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
