"""Learned fusion planning: an MLP cost model over the engine's passes.

The engine records each pass's device time (``record_passes``). A small FP32
MLP (``aleph_b200_mlp_*``: 3 hidden layers of 128 ReLU units, trained with
MSE + Adam by this library's CUDA kernels) learns log(time per algorithmic
GB) from pass features. ``LearnedPlanner`` scores candidate planner
configurations (register qubits per tile, kernel occupancy variant, tensor-core
blocks or CUDA-core tiles, block window search) by summing the predicted
times of the passes each one would launch (``describe_plan``, host only), in
place of the fixed greedy configuration. ``autotune`` keeps a learned choice
only when it is measured faster than the greedy plan and its final state
matches the greedy plan's within the precision's tolerance: the greedy plan
stays the fallback and the yardstick.

The reference has no counterpart: its fusion is the greedy FuseKq heuristic
(crates/aleph-ir/src/passes/fuse_kq.rs:268-400).
"""
from __future__ import annotations

import ctypes as ct
import math
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

from . import abi
from .backend import B200SvBackend, BackendError, describe_plan
from .circuit import Flat, flatten

KINDS = ("tile", "block", "kq", "smem", "measure", "renorm")
N_FEATURES = 20


def default_occupancy(precision: str) -> int:
    """The tile kernel variant a plan gets with tile_occupancy = 0."""
    return 2 if precision == "f64" else 4


def pass_features(rec: dict, precision: str) -> np.ndarray:
    """Feature vector of one pass record (``pass_records`` / ``describe_plan``)."""
    f = np.zeros(N_FEATURES, dtype=np.float32)
    k = rec["kind"]
    if k in KINDS:
        f[KINDS.index(k)] = 1.0
    n = max(1, rec["n"])
    f[6] = 1.0 if precision == "f64" else 0.0
    f[7] = n / 34.0
    f[8] = math.log2(max(rec["bytes"], 1.0)) / 40.0
    f[9] = rec["gates"] / 64.0
    f[10] = rec.get("lane_ops", 0) / 32.0
    f[11] = rec.get("dense_ops", 0) / 64.0
    f[12] = rec.get("diag_ops", 0) / 64.0
    f[13] = rec.get("post_ops", 0) / 48.0
    occ = rec.get("variant", 0) or (default_occupancy(precision) if k == "tile" else 0)
    f[14] = occ / 4.0
    qs = rec.get("qubits", [])
    if qs:
        f[15] = min(qs) / n
        f[16] = max(qs) / n
        f[17] = sum(1 for q in qs if q < 7) / 6.0
        f[18] = len(qs) / 8.0
        f[19] = float(np.mean(qs)) / n
    return f


def target(rec: dict) -> float:
    """Regression target: log(ms per algorithmic GB)."""
    return math.log(max(rec["ms"], 1e-6) / (rec["bytes"] / 1e9))


def predicted_ms(y: np.ndarray, recs) -> np.ndarray:
    return np.exp(y) * np.array([r["bytes"] for r in recs]) / 1e9


# ---- the cost model on the device ---------------------------------------------------------
class CostModel:
    """The MLP behind ``aleph_b200_mlp_*`` (training and inference run on the GPU)."""

    def __init__(self, backend: B200SvBackend, hidden: int = 128, seed: int = 0, n_features: int = N_FEATURES):
        self.backend, self.hidden, self.n_features = backend, hidden, n_features
        p = ct.c_void_p()
        backend._check(backend.lib.aleph_b200_mlp_create(backend.handle, n_features, hidden, seed, ct.byref(p)))
        self.ptr = p
        self.x_mean = np.zeros(n_features, np.float32)
        self.x_std = np.ones(n_features, np.float32)

    def _norm(self, X):
        return np.ascontiguousarray(((np.asarray(X, np.float32) - self.x_mean) / self.x_std).astype(np.float32))

    def fit(self, X, y, epochs: int = 200, batch: int = 256, lr: float = 1e-3, seed: int = 0) -> float:
        X = np.asarray(X, np.float32)
        self.x_mean = X.mean(axis=0)
        self.x_std = np.where(X.std(axis=0) > 1e-6, X.std(axis=0), 1.0).astype(np.float32)
        Xn, yv = self._norm(X), np.ascontiguousarray(np.asarray(y, np.float32))
        loss = ct.c_float()
        b = self.backend
        b._check(b.lib.aleph_b200_mlp_train(b.handle, self.ptr, Xn.ctypes.data_as(ct.POINTER(ct.c_float)),
                                            yv.ctypes.data_as(ct.POINTER(ct.c_float)), len(yv), epochs,
                                            min(batch, len(yv)), lr, seed, ct.byref(loss)))
        return loss.value

    def predict(self, X) -> np.ndarray:
        Xn = self._norm(np.atleast_2d(X))
        out = np.zeros(len(Xn), np.float32)
        b = self.backend
        b._check(b.lib.aleph_b200_mlp_predict(b.handle, self.ptr, Xn.ctypes.data_as(ct.POINTER(ct.c_float)), len(Xn),
                                              out.ctypes.data_as(ct.POINTER(ct.c_float))))
        return out

    def gradients(self, X, y):
        """(loss, flat parameter gradients) of one batch, X already normalised."""
        X = np.ascontiguousarray(np.asarray(X, np.float32))
        y = np.ascontiguousarray(np.asarray(y, np.float32))
        g = np.zeros(self.param_count(), np.float32)
        loss = ct.c_float()
        b = self.backend
        b._check(b.lib.aleph_b200_mlp_gradients(b.handle, self.ptr, X.ctypes.data_as(ct.POINTER(ct.c_float)),
                                                y.ctypes.data_as(ct.POINTER(ct.c_float)), len(y),
                                                g.ctypes.data_as(ct.POINTER(ct.c_float)), ct.byref(loss)))
        return loss.value, g

    def param_count(self) -> int:
        n = ct.c_uint64()
        self.backend._check(self.backend.lib.aleph_b200_mlp_params(self.backend.handle, self.ptr, None, None,
                                                                   ct.byref(n)))
        return n.value

    def get_params(self) -> np.ndarray:
        out = np.zeros(self.param_count(), np.float32)
        self.backend._check(self.backend.lib.aleph_b200_mlp_params(
            self.backend.handle, self.ptr, out.ctypes.data_as(ct.POINTER(ct.c_float)), None, None))
        return out

    def set_params(self, params) -> None:
        p = np.ascontiguousarray(np.asarray(params, np.float32))
        if p.size != self.param_count():
            raise ValueError("parameter count mismatch")
        self.backend._check(self.backend.lib.aleph_b200_mlp_params(
            self.backend.handle, self.ptr, None, p.ctypes.data_as(ct.POINTER(ct.c_float)), None))

    def save(self, path) -> None:
        np.savez_compressed(path, params=self.get_params(), x_mean=self.x_mean, x_std=self.x_std,
                            hidden=self.hidden, n_features=self.n_features)

    @classmethod
    def load(cls, backend: B200SvBackend, path) -> "CostModel":
        d = np.load(path)
        m = cls(backend, hidden=int(d["hidden"]), n_features=int(d["n_features"]))
        m.set_params(d["params"])
        m.x_mean, m.x_std = d["x_mean"].astype(np.float32), d["x_std"].astype(np.float32)
        return m

    def free(self) -> None:
        if self.ptr:
            self.backend.lib.aleph_b200_mlp_free(self.backend.handle, self.ptr)
            self.ptr = None


# ---- candidate planner configurations --------------------------------------------------
@dataclass(frozen=True)
class PlanChoice:
    tile_r: int = 5
    tile_occupancy: int = 0
    block_window_search: bool = True
    tensor_blocks: bool = True  # TC32 handles only

    def apply(self, backend: B200SvBackend) -> None:
        backend.set_tuning("tile_r", self.tile_r)
        backend.set_tuning("tile_occupancy", self.tile_occupancy)
        backend.set_tuning("block_window_search", int(self.block_window_search))
        if backend.precision == "tc32":
            backend.set_tuning("tensor_blocks", int(self.tensor_blocks))

    def describe_precision(self, precision: str) -> str:
        return "f32" if precision == "tc32" and not self.tensor_blocks else precision


GREEDY = PlanChoice()


def candidates(precision: str) -> list[PlanChoice]:
    """The configurations the learned planner chooses among (greedy first)."""
    tile_prec = "f32" if precision == "tc32" else precision
    occs = [0] + [o for o in (2, 3, 4) if o != default_occupancy(tile_prec)]  # 0 is the default variant
    tiles = [PlanChoice(tile_r=r, tile_occupancy=o) for r in (3, 4, 5) for o in occs]
    if precision == "tc32":
        blocks = [PlanChoice(block_window_search=w) for w in (True, False)]
        return blocks + [PlanChoice(tile_r=c.tile_r, tile_occupancy=c.tile_occupancy, tensor_blocks=False)
                         for c in tiles]
    return [GREEDY] + [c for c in tiles if c != GREEDY]


@dataclass
class Scored:
    choice: PlanChoice
    predicted_ms: float
    passes: int


class LearnedPlanner:
    """Scores candidate configurations with the cost model."""

    def __init__(self, model: CostModel):
        self.model = model

    def score(self, n: int, instructions, precision: str) -> list[Scored]:
        flat = instructions if isinstance(instructions, Flat) else flatten(instructions)
        out = []
        for c in candidates(precision):
            dp = c.describe_precision(precision)
            recs = describe_plan(n, flat, dp, tile_r=c.tile_r, block_window_search=c.block_window_search,
                                 tile_occupancy=c.tile_occupancy)
            X = np.stack([pass_features(r, dp) for r in recs]) if recs else np.zeros((0, N_FEATURES), np.float32)
            ms = float(predicted_ms(self.model.predict(X), recs).sum()) if recs else 0.0
            out.append(Scored(c, ms, len(recs)))
        return sorted(out, key=lambda s: s.predicted_ms)


# ---- measurement, data collection and the autotuner -----------------------------------
def state_signature(backend: B200SvBackend, st, n: int) -> np.ndarray:
    """What the autotuner compares between plans: the amplitudes up to n = 26;
    above that, eight windows of 4096 amplitudes spread over the state (at
    fixed seeded offsets) plus the marginal distributions of the lowest and
    the highest 10 qubits."""
    if n <= 26:
        return backend.statevector(st)
    rng = np.random.default_rng(n)
    starts = [0, (1 << n) - 4096] + [int(x) * 4096 for x in rng.integers(0, (1 << n) // 4096, 6)]
    amps = np.concatenate([backend.amplitude_range(st, a, 4096) for a in starts])
    k = min(10, n)
    lo = backend.probabilities(st, list(range(k)))
    hi = backend.probabilities(st, list(range(n - k, n)))
    return np.concatenate([amps, lo, hi])


def measure(backend: B200SvBackend, n: int, flat: Flat, choice: PlanChoice, repeats: int = 2):
    """(device ms of the plan's passes, pass records, state signature)."""
    choice.apply(backend)
    plan = backend.compile(n, flat)
    st = backend.allocate(n)
    backend.set_tuning("record_passes", 0)
    backend.reset_state(st)
    plan.execute(st)  # warm-up
    backend.set_tuning("record_passes", 1)
    best, recs = None, None
    for _ in range(repeats):
        backend.reset_state(st)
        plan.execute(st)
        r = backend.pass_records()
        t = sum(x["ms"] for x in r)
        if best is None or t < best:
            best, recs = t, r
    backend.set_tuning("record_passes", 0)
    sig = state_signature(backend, st, n)
    st.free()
    plan.free()
    return best, recs, sig


def collect(backend: B200SvBackend, circuits, choices=None, repeats: int = 1):
    """Training data: (features, targets) of every pass of every (circuit, choice) run."""
    X, y = [], []
    prec = backend.precision
    for n, instr in circuits:
        flat = instr if isinstance(instr, Flat) else flatten(instr)
        for c in choices or candidates(prec):
            _, recs, _ = measure(backend, n, flat, c, repeats)
            dp = c.describe_precision(prec)
            for r in recs:
                if r["kind"] == "renorm":
                    continue
                X.append(pass_features(r, dp))
                y.append(target(r))
    return np.array(X, np.float32), np.array(y, np.float32)


def circuit_work(n: int, instr) -> float:
    """Relative collection cost of a circuit: amplitudes x instructions."""
    return float(1 << n) * max(1, len(instr) if not isinstance(instr, Flat) else instr.n)


def shard_circuits(circuits, rank: int = 0, world: int = 1):
    """This rank's share of the training circuits, for collection on several
    GPUs. The circuits are independent units with no exchange between GPUs:
    largest first, each goes to the rank with the least work so far
    (amplitudes x instructions). Every rank computes the same assignment."""
    w = [circuit_work(n, instr) for n, instr in circuits]
    load = [0.0] * world
    mine = []
    for i in sorted(range(len(circuits)), key=lambda i: (-w[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        load[r] += w[i]
        if r == rank:
            mine.append(i)
    return [circuits[i] for i in sorted(mine)]


def gather_samples(X: np.ndarray, y: np.ndarray, world: int = 1):
    """Every rank's (features, targets), concatenated in rank order on every
    rank (an all-gather of Python objects over the default process group)."""
    if world == 1:
        return X, y
    import torch.distributed as dist

    parts = [None] * world
    dist.all_gather_object(parts, (X, y))
    return (np.concatenate([p[0] for p in parts if len(p[1])]).astype(np.float32),
            np.concatenate([p[1] for p in parts if len(p[1])]).astype(np.float32))


TOLERANCE = {"f64": 1e-12, "f32": 1e-5, "tc32": 1e-5}


@dataclass
class AutotuneResult:
    choice: PlanChoice
    greedy_ms: float
    chosen_ms: float
    measured: dict = field(default_factory=dict)
    rejected: list = field(default_factory=list)


def autotune(backend: B200SvBackend, n: int, instructions, planner: LearnedPlanner | None = None, top_k: int = 2):
    """Measure the greedy plan and the planner's top-k; keep the fastest whose
    state matches the greedy plan's within tolerance (the greedy plan otherwise)."""
    flat = instructions if isinstance(instructions, Flat) else flatten(instructions)
    g_ms, _, g_psi = measure(backend, n, flat, GREEDY)
    res = AutotuneResult(GREEDY, g_ms, g_ms, {GREEDY: g_ms})
    if planner is None:
        GREEDY.apply(backend)
        return res
    tol = TOLERANCE[backend.precision]
    for s in [s for s in planner.score(n, flat, backend.precision) if s.choice != GREEDY][:top_k]:
        try:
            ms, _, psi = measure(backend, n, flat, s.choice)
        except BackendError as e:
            res.rejected.append((s.choice, str(e)))
            continue
        res.measured[s.choice] = ms
        if psi.shape != g_psi.shape or np.abs(psi - g_psi).max() > tol:
            res.rejected.append((s.choice, "state differs from the greedy plan's"))
            continue
        if ms < res.chosen_ms:
            res.choice, res.chosen_ms = s.choice, ms
    res.choice.apply(backend)
    return res


MODEL_PATH = Path(__file__).resolve().parent / "cost_model.npz"


# ---- training set and held-out evaluation ------------------------------------------------
def training_circuits(sizes=(22, 26, 30), seed: int = 0):
    """Generated training circuits at each size n: random brickwall (depth
    10, 25, 60), the textbook QFT on a product state, QAOA p = 1, 3, 6 on
    random 3-regular graphs, and Grover (multi-controlled Z in CX + T) with
    n/2 + 1 data qubits and 2 iterations."""
    from . import workloads as W

    rng = np.random.default_rng(seed)
    out = []
    for n in sizes:
        for d in (10, 25, 60):
            out.append((n, W.brickwall(n, d, seed=int(rng.integers(1 << 30))).instructions))
        out.append((n, W.qft_product(n, seed=int(rng.integers(1 << 30))).instructions))
        m = n - (n % 2)
        for p in (1, 3, 6):
            edges = W.random_3_regular(m, rng)
            out.append((m, W.qaoa_maxcut(m, edges, rng.uniform(0, np.pi, p), rng.uniform(0, np.pi, p)).instructions))
        nd = n // 2 + 1
        out.append((2 * nd - 2, W.grover(nd, int(rng.integers(1 << nd)), 2).instructions))
    return out


def large_training_circuits(precision: str, seed: int = 7):
    """Pass samples at the top of the engine's range (FP64 to n = 33, FP32 and
    TC32 to n = 32): the depth-10 brickwall and the QFT. These states are 64
    to 128 GiB, so they run under the few candidates of ``large_choices``."""
    from . import workloads as W

    rng = np.random.default_rng(seed)
    sizes = (32, 33) if precision == "f64" else (31, 32)
    out = []
    for n in sizes:
        out.append((n, W.brickwall(n, 10, seed=int(rng.integers(1 << 30))).instructions))
        out.append((n, W.qft_product(n, seed=int(rng.integers(1 << 30))).instructions))
    return out


def large_choices(precision: str) -> list[PlanChoice]:
    """The candidates sampled at the largest sizes: the greedy configuration
    and its nearest neighbours (4 and 3 register qubits, the other occupancy
    variants at 4)."""
    c = candidates(precision)
    if precision == "tc32":
        return c[:2] + [x for x in c[2:] if x.tile_r == 5][:2]
    default = default_occupancy(precision)
    # FP64 tiles at 5 register qubits spill above two blocks per SM: left out here
    return [x for x in c if x.tile_r == 4 or (x.tile_r == 5 and (precision != "f64" or x.tile_occupancy in (0, default)))]


def heldout_circuits(precision: str, n_brick: int | None = None, n_grover_data: int = 16, n_qft: int = 30,
                     seed: int = 1):
    """Held-out evaluation circuits at the configured sizes (none of them in
    the training set): a depth-40 random brickwall (n = 33 for FP64, 32 for
    FP32 / TC32), Grover with 16 data qubits (30 qubits with the ancillas) and
    20 iterations, and the textbook QFT on a product state at n = 30."""
    from . import workloads as W

    rng = np.random.default_rng(seed)
    nb = n_brick or (33 if precision == "f64" else 32)
    return [("brickwall", nb, W.brickwall(nb, 40, seed=seed).instructions),
            ("grover", 2 * n_grover_data - 2,
             W.grover(n_grover_data, int(rng.integers(1 << n_grover_data)), 20).instructions),
            ("qft", n_qft, W.qft_product(n_qft, seed=seed).instructions)]


def evaluate(model_path, precisions=("f64", "tc32"), **heldout_kw) -> list:
    """The learned planner (autotuned: kept only if measured faster and
    state-equal) against the greedy plan on the held-out circuits."""
    evals = []
    for prec in precisions:
        bq = B200SvBackend(seed=0, precision=prec)
        mq = CostModel.load(bq, model_path)
        planner = LearnedPlanner(mq)
        for name, n, instr in heldout_circuits(prec, **heldout_kw):
            flat = flatten(instr)
            scored = planner.score(n, flat, prec)
            res = autotune(bq, n, flat, planner, top_k=2)
            evals.append({"precision": prec, "circuit": name, "n": n, "gates": int(flat.n),
                          "greedy_ms": round(res.greedy_ms, 3), "learned_ms": round(res.chosen_ms, 3),
                          "gain": round(res.greedy_ms / res.chosen_ms, 4), "choice": res.choice.__dict__,
                          "top_predicted": [(s.choice.__dict__, round(s.predicted_ms, 2)) for s in scored[:3]],
                          "greedy_predicted_ms": round(next(s.predicted_ms for s in scored if s.choice == GREEDY), 2),
                          "measured": {str(k.__dict__): round(v, 3) for k, v in res.measured.items()},
                          "rejected": [str(r[1]) for r in res.rejected]})
        mq.free()
        bq.close()
    return evals


def main(argv=None) -> int:
    """python -m aleph_b200.learned [--out PATH] [--epochs E]: collect pass
    timings on the GPU (f64, f32 and tc32 handles; n = 22..30 under every
    candidate configuration, n = 31..33 under the few of ``large_choices``),
    train the cost model, evaluate the learned planner against the greedy
    plan on the held-out circuits, print one JSON summary and save the model.
    With --eval-only: the held-out evaluation of the model at --out, without
    collecting or training."""
    import argparse
    import json
    import time

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(MODEL_PATH))
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--sizes", default="22,26,30")
    ap.add_argument("--no-large", action="store_true", help="skip the n = 31..33 samples")
    ap.add_argument("--heldout-brick", type=int, default=0, help="brickwall qubits (0: 33 FP64 / 32 TC32)")
    ap.add_argument("--heldout-grover", type=int, default=16)
    ap.add_argument("--heldout-qft", type=int, default=30)
    ap.add_argument("--eval-only", action="store_true")
    args = ap.parse_args(argv)
    hk = {"n_brick": args.heldout_brick or None, "n_grover_data": args.heldout_grover, "n_qft": args.heldout_qft}
    if args.eval_only:
        print(json.dumps({"model": str(args.out), "heldout": evaluate(args.out, **hk)}))
        return 0
    # under torchrun every rank (one per GPU) collects its share of the
    # circuits; rank 0 trains and evaluates on the gathered samples
    import os

    world, rank = int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=3600))
    t0 = time.perf_counter()
    Xs, ys = [], []
    circuits = training_circuits(tuple(int(x) for x in args.sizes.split(",")))
    n_large = 0
    for prec in ("f64", "f32", "tc32"):
        be = B200SvBackend(seed=0, precision=prec)
        X, y = collect(be, shard_circuits(circuits, rank, world))
        Xs.append(X)
        ys.append(y)
        if not args.no_large:
            big = large_training_circuits(prec)
            X, y = collect(be, shard_circuits(big, rank, world), large_choices(prec))
            Xs.append(X)
            ys.append(y)
            n_large += len(y)
        be.close()
    X, y = gather_samples(np.concatenate(Xs), np.concatenate(ys), world)
    t_collect = time.perf_counter() - t0
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()
        if rank != 0:
            return 0
    be = B200SvBackend(seed=0, precision="f64")
    model = CostModel(be, seed=0)
    # hold out every 10th sample to report the fit
    val = np.arange(len(y)) % 10 == 0
    t1 = time.perf_counter()
    loss = model.fit(X[~val], y[~val], epochs=args.epochs, batch=256, lr=1e-3)
    t_train = time.perf_counter() - t1
    pred = model.predict(X[val])
    val_rmse = float(np.sqrt(np.mean((pred - y[val]) ** 2)))
    base_rmse = float(np.sqrt(np.mean((y[val] - y[~val].mean()) ** 2)))
    model.save(args.out)
    t2 = time.perf_counter()
    evals = evaluate(args.out, **hk)
    print(json.dumps({"samples": int(len(y)), "large_samples": int(n_large), "circuits": len(circuits),
                      "collect_s": round(t_collect, 1), "train_s": round(t_train, 2),
                      "train_samples_per_s": round(args.epochs * (~val).sum() / t_train),
                      "final_batch_loss": loss, "val_rmse_log": val_rmse, "val_rmse_mean_predictor": base_rmse,
                      "eval_s": round(time.perf_counter() - t2, 1), "heldout": evals}))
    model.free()
    be.close()
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
