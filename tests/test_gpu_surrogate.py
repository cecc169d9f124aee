"""The learned surrogate on the GPU against its CPU oracle
(oracle/surrogate_oracle.py, BF16 rounding emulated at the GPU's rounding
points), and its judged coupling to the plain solver.

Tolerances: the GPU and the oracle differ by FP32 vs float64 accumulation
(~1e-6 relative) plus the rare value that lands on the other side of a BF16
rounding boundary or of a ReLU kink; outputs agree to 1e-2 and every
gradient block to 3e-2 of its norm."""
import numpy as np
import pytest

from oracle import surrogate_oracle as SO
from uph_b200 import surrogate as SG
from uph_b200._capi import PREC_FP64, PROFILE_WCSPH

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _batch():
    return SG.flume_batch([(0.04, 1.2)], length=1.0, depth=0.2, dx=0.02, layers=2)


def _frame(seed=0):
    b = _batch()
    st = {k: v.copy() for k, v in b.state.items()}
    rng = np.random.default_rng(seed)
    nf = b.deck.n_fluid
    st["Velocity"][:nf] += rng.normal(0, 0.05, (nf, 2))
    st["density"][:nf] *= 1 + rng.normal(0, 2e-5, nf)
    st["Position"][:nf] += rng.uniform(-0.002, 0.002, (nf, 2))
    return b, st


def _cfg(b, K=5):
    p = b.deck.uph_params(PROFILE_WCSPH, PREC_FP64)
    return SG.NetConfig.for_params(p, K, vel_scale=0.1, rho_scale=0.01)


def _params(seed=3):
    flat = SG.init_params(seed, 3).astype(np.float64)
    W = SO.unpack(flat, 3)
    W["dec2.w"][:SO.NOUT] *= 10.0
    for r in range(3):
        W[f"r{r}.n2.w"] *= 10.0
    return flat.astype(np.float32)


def _oracle(b, st, cfg, flat):
    nf = b.deck.n_fluid
    pos = st["Position"]
    g = SO.Graph(pos[:, 0], pos[:, 1], cfg.radius, st["density"], cfg.rho0 * cfg.edge_rho_scale)
    F = SO.node_features(st["Velocity"][:, 0], st["Velocity"][:, 1], st["density"], st["itype"], cfg.vel_scale,
                         cfg.rho0, cfg.rho_scale)
    return g, F, nf


def _target(nf, seed=1):
    return np.random.default_rng(seed).normal(0, 1, (nf, SO.NOUT))


def test_forward_matches_oracle():
    b, st = _frame()
    cfg = _cfg(b)
    flat = _params()
    sur = SG.Surrogate(cfg, b.deck.n_all, flat)
    nodes = SG.Nodes.from_state(st, b.deck.n_fluid, b.box)
    out = sur.forward(nodes).cpu().numpy().astype(np.float64)
    g, F, nf = _oracle(b, st, cfg, flat)
    ref, _ = SO.forward(flat, F, g, 3, emulate=True)
    ref = ref[:, :SO.NOUT]
    err = np.linalg.norm(out - ref) / np.linalg.norm(ref)
    assert err <= 1e-2, err
    assert np.abs(out - ref).max() <= 2e-2 * np.abs(ref).max()


def test_gradients_match_oracle():
    b, st = _frame(1)
    cfg = _cfg(b)
    flat = _params(4)
    sur = SG.Surrogate(cfg, b.deck.n_all, flat)
    nodes = SG.Nodes.from_state(st, b.deck.n_fluid, b.box)
    g, F, nf = _oracle(b, st, cfg, flat)
    tgt = _target(nf)
    loss, grad = sur.gradients(nodes, torch.as_tensor(tgt, dtype=torch.float32, device="cuda").contiguous())
    grad = grad.cpu().numpy().astype(np.float64)
    out, cache = SO.forward(flat, F, g, 3, emulate=True)
    ref_loss, dout = SO.loss_and_grad(out, tgt, nf)
    ref = SO.backward(cache, dout)
    assert loss == pytest.approx(ref_loss, rel=1e-3)
    off, _ = SO.offsets(3)
    worst = 0.0
    for name, (o, shape) in off.items():
        sz = int(np.prod(shape))
        rn = np.linalg.norm(ref[o:o + sz])
        if rn == 0:
            assert np.all(grad[o:o + sz] == 0), name
            continue
        e = np.linalg.norm(grad[o:o + sz] - ref[o:o + sz]) / rn
        worst = max(worst, e)
        assert e <= 3e-2, (name, e)
    print("largest block-relative gradient error", worst)


def test_forward_backward_bitwise_reproducible():
    b, st = _frame(2)
    cfg = _cfg(b)
    sur = SG.Surrogate(cfg, b.deck.n_all, _params(5))
    nodes = SG.Nodes.from_state(st, b.deck.n_fluid, b.box)
    tgt = torch.as_tensor(_target(b.deck.n_fluid, 2), dtype=torch.float32, device="cuda").contiguous()
    l1, g1 = sur.gradients(nodes, tgt)
    l2, g2 = sur.gradients(nodes, tgt)
    assert l1 == l2
    assert torch.equal(g1, g2)
    assert torch.equal(sur.forward(nodes), sur.forward(nodes))


def test_training_reduces_loss():
    """300 Adam steps on one frame fit a smooth function of the node state
    (the loss falls by more than 10x): the training kernels learn."""
    b, st = _frame(3)
    cfg = _cfg(b)
    sur = SG.Surrogate(cfg, b.deck.n_all, seed=6)
    nodes = SG.Nodes.from_state(st, b.deck.n_fluid, b.box)
    nf = b.deck.n_fluid
    u, v = st["Velocity"][:nf, 0] / 0.1, st["Velocity"][:nf, 1] / 0.1
    r = (st["density"][:nf] / 1000.0 - 1) / 0.01
    tgt = np.stack([u, v, u * v, np.tanh(r), 0.5 * u - v], 1)
    tgt = torch.as_tensor(tgt, dtype=torch.float32, device="cuda").contiguous()
    first, _ = sur.gradients(nodes, tgt, want_grad=False)
    for it in range(300):
        sur.gradients(nodes, tgt, want_grad=False, want_loss=False)
        sur.adam(1e-3)
    last, _ = sur.gradients(nodes, tgt, want_grad=False)
    assert last < first / 10, (first, last)


def _sim(b):
    from uph_b200.sim import Simulation
    sim = Simulation(b.deck.uph_params(PROFILE_WCSPH, PREC_FP64))
    sim.upload(b.state, 0)
    sim.set_wall_motion(*b.wall_table)
    return sim


def _judge(**kw):
    return SG.Judge(depth=0.2, surface_x0=0.0, surface_x1=1.0, surface_bins=20, **kw)


def _plain_equal(sur, judge, n_macro):
    b = _batch()
    a, p = _sim(b), _sim(b)
    a.step(3)
    p.step(3)
    rep = sur.advance(a, n_macro, judge)
    for _ in range(n_macro):
        p.step(sur.cfg.macro_steps)
    sa, sp = a.download(), p.download()
    for k in ("Position", "Velocity", "density"):
        assert np.array_equal(sa[k], sp[k]), k
    return rep


def test_failing_judge_on_every_step_reproduces_the_plain_solver():
    """Every macro step judged and every check failed (threshold 1e-12, no
    extra fallback): the state is bitwise the plain solver's trajectory."""
    b = _batch()
    sur = SG.Surrogate(_cfg(b, K=5), b.deck.n_all, _params(7))
    rep = _plain_equal(sur, _judge(judge_every=1, fallback_macro=0, max_rho_err=1e-12), 4)
    assert (rep.judged_steps, rep.failed_checks, rep.network_steps, rep.plain_steps) == (4, 4, 0, 20)
    assert rep.max_rho_err > 0


def test_sanity_guard_rejects_implausible_predictions():
    """A network whose density output is far off (+1000 kg/m^3 per macro
    step) never touches the state: every prediction is rejected and the
    plain solver takes each macro step."""
    b = _batch()
    flat = _params(9)
    off, _ = SO.offsets(3)
    flat[off["dec2.b"][0] + 4] = 1000.0
    sur = SG.Surrogate(_cfg(b, K=5), b.deck.n_all, flat)
    rep = _plain_equal(sur, _judge(judge_every=3, fallback_macro=0), 4)
    assert (rep.rejected_steps, rep.network_steps, rep.plain_steps) == (4, 0, 20)


def test_failed_check_hands_over_to_the_plain_solver():
    """A check over threshold starts `fallback_macro` plain macro steps; the
    counts follow the schedule net, judged(fail), plain, plain, net, ..."""
    b = _batch()
    cfg = _cfg(b, K=5)
    # freshly initialised weights: small predictions the guard never rejects
    sur = SG.Surrogate(cfg, b.deck.n_all, SG.init_params(8))
    sim = _sim(b)
    sim.step(2)
    rep = sur.advance(sim, 7, _judge(judge_every=2, fallback_macro=2, max_rho_err=1e-12))
    assert (rep.macro_steps, rep.network_steps, rep.judged_steps, rep.failed_checks) == (7, 2, 2, 2)
    assert rep.plain_steps == 5 * 5
    # generous thresholds: nothing fails, every second macro step is judged
    # and its prediction kept
    sim2 = _sim(b)
    sim2.step(2)
    rep2 = sur.advance(sim2, 7, _judge(judge_every=2, max_rho_err=1e9, max_surface_err=1e9))
    assert (rep2.network_steps, rep2.judged_steps, rep2.failed_checks, rep2.plain_steps) == (7, 3, 0, 15)
    st = sim2.download()
    assert np.all(np.isfinite(st["Position"])) and np.all(np.isfinite(st["density"]))
    sim2.step(10)  # the plain solver carries on from a network-made state


def test_fused_node_chain_matches_per_layer_gemms():
    """The fused per-round kernels (every layer of a round on chip) against
    one GEMM per layer, on 40k nodes so that every persistent CTA runs
    several tiles: the same network, to FP32-accumulation-order accuracy."""
    rng = np.random.default_rng(11)
    nx, ny = 400, 100
    dx = 0.005
    xs, ys = np.meshgrid(np.arange(nx) * dx, np.arange(ny) * dx)
    x = (xs.ravel() + rng.uniform(-0.1, 0.1, xs.size) * dx)
    y = (ys.ravel() + rng.uniform(-0.1, 0.1, xs.size) * dx)
    n = x.size
    itype = np.ones(n, np.int32)
    itype[-2 * nx:] = 2
    nf = n - 2 * nx
    st = {"Position": np.stack([x, y], 1), "Velocity": rng.normal(0, 0.05, (n, 2)),
          "density": 1000.0 * (1 + rng.normal(0, 0.003, n)), "itype": itype}
    box = (-0.02, -0.02, nx * dx + 0.02, ny * dx + 0.02)
    cfg = SG.NetConfig(rounds=3, macro_steps=40, radius=2.6 * dx, dt=5e-5)
    sur = SG.Surrogate(cfg, n, _params(12))
    nodes = SG.Nodes.from_state(st, nf, box)
    fused = sur.forward(nodes).cpu().numpy()
    sur.set_fused(False)
    plain = sur.forward(nodes).cpu().numpy()
    scale = np.abs(plain).max()
    assert scale > 0
    err = np.abs(fused - plain).max() / scale
    print("fused vs per-layer max |diff| / max |out|:", err)
    assert err <= 1e-5
