"""CPU checks of the learned surrogate: the oracle's backward pass against
central finite differences (the pin of the gradient oracle), the parameter
layout shared by the oracle, the Python API and the library, and the flume
batch the training data comes from."""
import numpy as np
import pytest

from oracle import surrogate_oracle as SO
from uph_b200 import _lib
from uph_b200 import surrogate as SG


def small_graph(seed=0, n_side=7, jitter=0.15):
    """A jittered lattice patch: fluid rows on top of two wall rows."""
    rng = np.random.default_rng(seed)
    dx = 1.0
    xs, ys = np.meshgrid(np.arange(n_side) * dx, np.arange(n_side) * dx)
    x = xs.ravel() + rng.uniform(-jitter, jitter, xs.size)
    y = ys.ravel() + rng.uniform(-jitter, jitter, xs.size)
    n = x.size
    n_wall = 2 * n_side
    order = np.argsort(-y, kind="stable")  # fluid (upper rows) first, walls last
    x, y = x[order], y[order]
    itype = np.ones(n, np.int32)
    itype[n - n_wall:] = 2
    itype[n - n_side:] = 3
    u = rng.normal(0, 0.05, n)
    v = rng.normal(0, 0.05, n)
    rho = 1000.0 * (1 + rng.normal(0, 0.003, n))
    g = SO.Graph(x, y, 2.6 * dx, rho, 3.0)
    F = SO.node_features(u, v, rho, itype, 0.1, 1000.0, 0.01)
    return g, F, n - n_wall


def test_layouts_agree():
    off, total = SO.offsets(3)
    assert total == int(_lib.lib().uph_sur_param_count(3))
    assert total == SG.init_params(0, 3).size
    assert [k for k, _ in SO.layout(3)] == [k for k, _ in SG.param_layout(3)]
    assert int(_lib.lib().uph_sur_param_count(0)) == -1
    p = SO.unpack(SG.init_params(1, 3).astype(np.float64), 3)
    assert np.all(p["enc1.w"][:, SO.NFEAT_USED:] == 0)
    assert np.all(p["dec2.w"][SO.NOUT:] == 0)


@pytest.mark.parametrize("rounds", [1, 3])
def test_oracle_gradient_matches_finite_differences(rounds):
    """The float64 oracle's analytic gradient against central differences
    (step 1e-6, relative error <= 1e-5 on entries with |g| > 1e-6 of the
    largest): pins the backward restatement every GPU gradient is checked
    against."""
    g, F, nf = small_graph()
    rng = np.random.default_rng(5)
    flat = SG.init_params(3, rounds).astype(np.float64)
    # larger output and residual layers so every block carries gradient
    W = SO.unpack(flat, rounds)
    W["dec2.w"][:SO.NOUT] *= 10.0
    for r in range(rounds):
        W[f"r{r}.n2.w"] *= 10.0
        W[f"r{r}.pq.b"][:] = rng.normal(0, 0.1, W[f"r{r}.pq.b"].shape)
    target = rng.normal(0, 1, (nf, SO.NOUT))
    out, cache = SO.forward(flat, F, g, rounds, emulate=False)
    loss, dout = SO.loss_and_grad(out, target, nf)
    grad = SO.backward(cache, dout)
    off, _ = SO.offsets(rounds)
    checked = 0
    for name, (o, shape) in off.items():
        size = int(np.prod(shape))
        blk = np.abs(grad[o:o + size])
        if blk.max() == 0:
            continue
        cand = np.flatnonzero(blk > 1e-3 * blk.max())
        for k in rng.choice(cand, size=min(3, cand.size), replace=False):
            i = o + int(k)
            e = 1e-6
            fp = flat.copy()
            fp[i] += e
            fm = flat.copy()
            fm[i] -= e
            fd = (SO.loss_of(fp, F, g, target, nf, rounds) - SO.loss_of(fm, F, g, target, nf, rounds)) / (2 * e)
            assert abs(fd - grad[i]) <= 1e-5 * max(abs(grad[i]), 1e-3 * np.abs(grad).max()), (name, k, fd, grad[i])
            checked += 1
    assert checked >= 3 * (4 + 6 * rounds)


def test_emulated_forward_close_to_float64():
    """BF16 rounding at the GPU's rounding points moves the outputs by well
    under 5% of their scale (the emulation is the GPU's comparison form)."""
    g, F, nf = small_graph(1)
    flat = SG.init_params(4, 3)
    o64, _ = SO.forward(flat, F, g, 3, emulate=False)
    o16, _ = SO.forward(flat, F, g, 3, emulate=True)
    err = np.linalg.norm(o16[:, :5] - o64[:, :5]) / np.linalg.norm(o64[:, :5])
    assert 0 < err < 0.05


def test_flume_batch_geometry():
    b = SG.flume_batch([(0.02, 1.0), (0.06, 1.6)], length=1.0, depth=0.2, dx=0.02, layers=2)
    d = b.deck
    st = b.state
    nf = d.n_fluid
    assert nf == 2 * 50 * 10
    pos = st["Position"]
    lo, hi = np.array(b.box[:2]), np.array(b.box[2:])
    assert np.all(pos >= lo) and np.all(pos <= hi)
    # flumes do not interact: the vertical gap exceeds the interaction radius plus strokes
    f0 = pos[:nf // 2]
    f1 = pos[nf // 2:nf]
    assert f1[:, 1].min() - f0[:, 1].max() > 4 * 1.3 * 0.02
    # per-flume piston amplitude and frequency, one entry per moving particle
    x0, hs, om = b.wall_table
    assert x0.size == d.moving.shape[0]
    assert set(np.round(hs, 6)) == {0.02, 0.06}
    assert np.allclose(sorted(set(np.round(om, 6))), sorted({round(2 * np.pi / 1.0, 6), round(2 * np.pi / 1.6, 6)}))
    sponge = st["spongeFactor"]
    assert np.all(sponge[pos[:nf, 0] >= 0.7] > 0) and np.all(sponge[pos[:nf, 0] < 0.7] == 0)


def test_state_errors_and_surface_heights():
    pos = np.array([[0.05, 0.4], [0.06, 0.5], [0.55, 0.3], [1.5, 9.0]])
    h = SG.surface_heights(pos, 0.0, 1.0, 2)
    assert h.tolist() == [0.5, 0.3]
    a = {"density": np.array([1000.0, 1010.0, 1000.0, 1000.0]), "Position": pos}
    b = {"density": np.array([1000.0, 1000.0, 1000.0, 1000.0]), "Position": pos + [0.0, 0.01]}
    e = SG.state_errors(a, b, 3, 0.5, 0.0, 1.0, 2)
    assert e["rho_max"] == pytest.approx(0.01)
    assert e["rho_rms"] == pytest.approx(0.01 / np.sqrt(3))
    assert e["surface"] == pytest.approx(0.02)
