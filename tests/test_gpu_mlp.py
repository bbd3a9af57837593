"""The lambda-placement network's tensor-core kernels against the CPU oracle
(oracle/mlp_oracle.py): forward pass, loss and every parameter gradient, and
Adam training.  The oracle rounds to BF16 where the kernels do, so the
remaining difference is FP32 accumulation and the exponential of SiLU."""
import numpy as np
import pytest

from oracle import mlp_oracle as M

pytestmark = pytest.mark.gpu

Y_TOL = 2e-3        # forward, relative to max |y|, against the BF16-rounding oracle
G_TOL = 1e-2        # gradient blocks, relative norm error, against the BF16-rounding oracle


def _data(n, seed):
    rng = np.random.default_rng(seed)
    x = rng.normal(size=(n, M.IN)).astype(np.float32)
    teacher = M.init(seed + 100)
    t, _ = M.forward(teacher, x)
    return x, t.astype(np.float32)


def _blocks(g):
    d = M.unpack(g)
    return {k: d[k] for k, _ in M.SHAPES}


@pytest.mark.parametrize("n", [1, 128, 200, 1000])
def test_forward_matches_oracle(n):
    from q_b200 import mlp
    p = mlp.init(3)
    x, _ = _data(n, 5)
    y = mlp.forward(p, x)
    yb, _ = M.forward(p, x, bf=True)
    y64, _ = M.forward(p, x)
    scale = np.abs(yb).max()
    assert np.abs(y - yb).max() <= Y_TOL * scale
    assert np.abs(y - y64).max() <= 3e-2 * scale


@pytest.mark.parametrize("n", [77, 256, 300])
def test_gradient_matches_oracle(n):
    from q_b200 import mlp
    p = mlp.init(7)
    x, t = _data(n, 11)
    t = t + np.random.default_rng(1).normal(0, 0.3, t.shape).astype(np.float32)
    L, g = mlp.loss_grad(p, x, t)
    Lb, gb = M.loss_grad(p, x, t, bf=True)
    L64, g64 = M.loss_grad(p, x, t)
    assert abs(L - Lb) <= 1e-3 * Lb and abs(L - L64) <= 2e-2 * L64
    for (k, a), b, c in zip(_blocks(g).items(), _blocks(gb).values(), _blocks(g64).values()):
        assert np.linalg.norm(a - b) <= G_TOL * np.linalg.norm(b), k
        assert np.linalg.norm(a - c) <= 5e-2 * np.linalg.norm(c), k


def test_training_follows_the_oracle():
    """300 full-batch Adam steps inside one launch: the loss falls as the
    oracle's BF16-rounded Adam run does, step for step within 5%."""
    from q_b200 import mlp
    x, t = _data(400, 21)
    p0 = mlp.init(9)
    p, hist = mlp.train(p0, x, t, 300, lr=2e-3)
    pb, hb = M.train(p0, x, t, 300, lr=2e-3, bf=True)
    assert np.all(np.isfinite(hist)) and hist[-1] < 0.2 * hist[0]
    assert np.all(np.abs(hist - hb) <= 0.05 * hb)
    Lend, _ = mlp.loss_grad(p, x, t)
    assert abs(Lend - M.loss_grad(pb, x, t, bf=True)[0]) <= 0.05 * Lend


def test_weight_decay_follows_the_oracle():
    from q_b200 import mlp
    x, t = _data(300, 23)
    p0 = mlp.init(4)
    p, hist = mlp.train(p0, x, t, 200, lr=2e-3, weight_decay=0.05)
    pb, hb = M.train(p0, x, t, 200, lr=2e-3, weight_decay=0.05, bf=True)
    assert np.all(np.abs(hist - hb) <= 0.05 * hb)
    w = M.weight_mask() > 0
    # decay shrinks the weights against the run without it
    pn, _ = mlp.train(p0, x, t, 200, lr=2e-3)
    assert np.linalg.norm(p[w]) < np.linalg.norm(pn[w])


def test_invalid_arguments():
    from q_b200 import QBError, mlp
    p = mlp.init(0)
    with pytest.raises(QBError) as e:
        mlp.forward(p, np.zeros((0, mlp.IN), np.float32))
    assert e.value.code == 1
    with pytest.raises(QBError):
        mlp.forward(p, np.zeros((mlp.MAX_SAMPLES + 1, mlp.IN), np.float32))
    with pytest.raises(ValueError):
        mlp.forward(p[:-1], np.zeros((3, mlp.IN), np.float32))


def test_tensor_core_wait_times_out_and_recovers():
    """Every tensor-core completion wait of the network kernel is bounded.  A
    wait limit of 0 polls makes the first wait give up: the call returns
    QB_ERR_TIMEOUT (after the kernel has drained its in-flight MMAs and
    released its tensor memory), and the next call with the default limit
    runs normally on the same context."""
    from q_b200 import mlp
    from q_b200._lib import QBError, lib
    p = mlp.init(4)
    x, t = _data(130, 7)
    assert lib.qb_mlp_set_wait_limit(0) == 0
    try:
        for call in (lambda: mlp.forward(p, x), lambda: mlp.train(p, x, t, 5)):
            with pytest.raises(QBError) as err:
                call()
            assert err.value.code == 8          # QB_ERR_TIMEOUT
    finally:
        assert lib.qb_mlp_set_wait_limit(67108864) == 0
    y = mlp.forward(p, x)
    yb, _ = M.forward(p, x, bf=True)
    assert np.abs(y - yb).max() <= Y_TOL * np.abs(yb).max()
