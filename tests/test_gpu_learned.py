"""The learned planner's cost model on the GPU: forward/backward against a
numpy FP32 restatement (gradient check), training, and the autotuner's
keep-only-if-faster-and-equal rule."""
import numpy as np
import pytest

from aleph_b200 import learned, workloads
from aleph_b200.backend import B200SvBackend

pytestmark = pytest.mark.gpu


def numpy_forward_backward(params, X, y, F, H):
    """FP32 numpy restatement of kernels_mlp.cu: layers F->H->H->H->1, ReLU, MSE."""
    shapes = [(F, H), (H, H), (H, H), (H, 1)]
    Ws, bs, off = [], [], 0
    for i, o in shapes:
        Ws.append(params[off:off + i * o].reshape(o, i))
        off += i * o
        bs.append(params[off:off + o])
        off += o
    acts, a = [], X
    for layer, (W, b) in enumerate(zip(Ws, bs)):
        z = a @ W.T + b
        a = np.maximum(z, 0) if layer < 3 else z
        acts.append(a)
    yhat = acts[-1][:, 0]
    loss = np.mean((yhat - y) ** 2)
    grads = []
    d = (2 * (yhat - y) / len(y))[:, None]
    for layer in range(3, -1, -1):
        if layer < 3:
            d = d * (acts[layer] > 0)
        xin = X if layer == 0 else acts[layer - 1]
        grads.append((d.T @ xin, d.sum(axis=0)))
        d = d @ Ws[layer]
    flat = []
    for gw, gb in reversed(grads):
        flat += [gw.reshape(-1), gb]
    return loss, np.concatenate(flat).astype(np.float32)


def test_mlp_gradients_match_numpy():
    be = B200SvBackend(seed=0, precision="f32")
    m = learned.CostModel(be, hidden=128, seed=3)
    rng = np.random.default_rng(0)
    X = rng.standard_normal((96, learned.N_FEATURES)).astype(np.float32)
    y = rng.standard_normal(96).astype(np.float32)
    loss, g = m.gradients(X, y)
    want_loss, want_g = numpy_forward_backward(m.get_params().astype(np.float64), X.astype(np.float64),
                                               y.astype(np.float64), learned.N_FEATURES, 128)
    assert abs(loss - want_loss) <= 1e-4 * max(1.0, abs(want_loss))
    assert np.abs(g - want_g).max() <= 1e-4 * max(1.0, np.abs(want_g).max())
    m.free()


def test_mlp_trains_and_round_trips(tmp_path):
    be = B200SvBackend(seed=0, precision="f32")
    m = learned.CostModel(be, hidden=128, seed=1)
    rng = np.random.default_rng(1)
    X = rng.uniform(-1, 1, (4096, learned.N_FEATURES)).astype(np.float32)
    y = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * X[:, 3] ** 2).astype(np.float32)
    before = float(np.mean((m.predict(X) - y) ** 2))
    m.fit(X, y, epochs=60, batch=256, lr=2e-3)
    after = float(np.mean((m.predict(X) - y) ** 2))
    assert after < 0.05 * before and after < 0.02
    path = tmp_path / "m.npz"
    m.save(path)
    m2 = learned.CostModel.load(be, path)
    assert np.allclose(m2.predict(X[:64]), m.predict(X[:64]), atol=1e-6)
    m.free()
    m2.free()


@pytest.mark.parametrize("precision", ["f64", "tc32"])
def test_autotune_keeps_only_faster_equal_plans(precision):
    be = B200SvBackend(seed=0, precision=precision)
    n = 20
    c = workloads.brickwall(n, 16, seed=9)
    # a model fitted on this circuit's own pass timings
    X, y = learned.collect(be, [(n, c.instructions)], learned.candidates(precision)[:4])
    m = learned.CostModel(be, seed=2)
    m.fit(X, y, epochs=50, batch=64)
    planner = learned.LearnedPlanner(m)
    scored = planner.score(n, c.instructions, precision)
    assert all(np.isfinite(s.predicted_ms) and s.predicted_ms > 0 for s in scored)
    res = learned.autotune(be, n, c.instructions, planner, top_k=2)
    assert res.chosen_ms <= res.greedy_ms
    # the kept plan reproduces the greedy plan's state
    st = be.allocate(n)
    be.apply_stream(st, c.instructions)
    learned.GREEDY.apply(be)
    ref = be.allocate(n)
    be.apply_stream(ref, c.instructions)
    tol = learned.TOLERANCE[precision]
    assert np.abs(be.statevector(st) - be.statevector(ref)).max() <= tol
    m.free()


def test_committed_cost_model_scores_candidates():
    if not learned.MODEL_PATH.exists():
        pytest.skip("no trained cost model in the tree")
    be = B200SvBackend(seed=0, precision="f64")
    m = learned.CostModel.load(be, learned.MODEL_PATH)
    scored = learned.LearnedPlanner(m).score(24, workloads.brickwall(24, 20, seed=4).instructions, "f64")
    assert len(scored) == len(learned.candidates("f64"))
    assert all(np.isfinite(s.predicted_ms) and s.predicted_ms > 0 for s in scored)
    m.free()


def test_trained_model_gains_on_a_heldout_circuit():
    """The committed cost model on a circuit outside its training set: the
    textbook QFT on a product state at n = 30, FP64 (learned.heldout_circuits).
    The model ranks a non-greedy configuration first, and the autotuner
    measures the greedy plan and the top two. It keeps the model's choice only
    because that choice is faster and its state matches the greedy plan's
    (amplitude windows and marginals at 1e-12). The measured gain clears 3%
    (1.066x when the model was trained). The kept configuration is also held
    to the oracle on the n = 24 copy of the circuit."""
    if not learned.MODEL_PATH.exists():
        pytest.skip("no trained cost model in the tree")
    from oracle import oracle

    be = B200SvBackend(seed=0, precision="f64")
    m = learned.CostModel.load(be, learned.MODEL_PATH)
    name, n, instr = learned.heldout_circuits("f64")[2]
    assert name == "qft" and n == 30
    planner = learned.LearnedPlanner(m)
    top = planner.score(n, instr, "f64")[0].choice
    assert top != learned.GREEDY
    res = learned.autotune(be, n, instr, planner, top_k=2)
    assert res.choice == top and not res.rejected
    assert res.greedy_ms / res.chosen_ms >= 1.03
    small = workloads.qft_product(24, seed=1)
    st = be.allocate(24)  # autotune left the kept configuration applied
    be.apply_stream(st, small.instructions)
    want, _ = oracle.run(24, small.instructions)
    assert np.abs(be.statevector(st) - want).max() <= 1e-12
    st.free()
    m.free()
