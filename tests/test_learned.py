"""Learned warm start: the CPU restatement (oracle/learned_oracle.py) checked
by finite differences, and the CUDA features, tensor-core inference and GPU
trainer checked against it.

Tolerances: features 1e-5 (float32 of FP64 geometry); network outputs
2e-2 of the output scale (BF16 activations may round differently after
FP32 sums in another order); gradients 2e-2 relative in norm.
"""
import numpy as np
import pytest

from oracle import learned_oracle as LO


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 1.0 + 2 ** -9], dtype=np.float32)
    r = LO.bf16(x)
    assert r.tolist() == [1.0, 1.0, 1.0 + 2 ** -6, -2.5, 1.0]


def test_oracle_backward_matches_finite_differences():
    rng = np.random.default_rng(0)
    p = LO.init_params(1)
    x = rng.normal(size=(6, LO.IN)).astype(np.float32)
    y = rng.normal(size=(6, LO.OUT)).astype(np.float32)
    loss, g = LO.loss_grad(p, x, y, rounding=False)
    assert np.isfinite(loss) and g.shape == (LO.NPARAM,)
    idx = rng.choice(LO.NPARAM, size=24, replace=False)
    # include biases and the last layer, where gradients are largest
    idx = np.concatenate([idx, [LO.H * LO.IN + 3, LO.NPARAM - 1, LO.NPARAM - 13 - 5]])
    for i in idx:
        h = 1e-2 * max(1.0, abs(float(p[i])))
        pp, pm = p.copy(), p.copy()
        pp[i] += h; pm[i] -= h
        fd = (LO.loss_grad(pp, x, y, rounding=False)[0] - LO.loss_grad(pm, x, y, rounding=False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 2e-2 * max(abs(fd), 1e-3), (i, fd, g[i])


def _norm(rng):
    return np.concatenate([rng.normal(scale=0.1, size=48), rng.uniform(0.5, 2.0, 48),
                           rng.normal(scale=0.1, size=12), rng.uniform(0.5, 2.0, 12)]).astype(np.float32)


@pytest.mark.gpu
def test_mlp_tensor_core_forward_matches_oracle(chain_scene):
    from colb_b200 import params as P
    from colb_b200.engine import Engine
    rng = np.random.default_rng(3)
    e = Engine(P.reference_params(), chain_scene)
    p = LO.init_params(2)
    p[-LO.OUT:] = rng.normal(size=LO.OUT)          # nonzero output bias
    norm = _norm(rng)
    e.set_mlp(p, norm)
    for n in (1, 128, 300):
        x = rng.normal(size=(n, 48)).astype(np.float32)
        y = e.mlp_forward(x)
        ref = LO.forward(p, norm, x)
        assert np.all(np.isfinite(y))
        assert np.abs(y - ref).max() <= 2e-2 * np.abs(ref).max(), n
    # twice in a row gives the same answer (no state kept between calls)
    assert np.array_equal(e.mlp_forward(x), y)


@pytest.mark.gpu
def test_trainer_gradient_matches_oracle():
    from colb_b200.engine import Trainer
    rng = np.random.default_rng(4)
    p = LO.init_params(5)
    x = rng.normal(size=(96, 48)).astype(np.float32)
    y = rng.normal(size=(96, 12)).astype(np.float32)
    t = Trainer(p)
    loss, g = t.grad(x, y)
    lref, gref = LO.loss_grad(p, x, y)
    assert loss == pytest.approx(lref, rel=1e-3)
    assert np.linalg.norm(g - gref) <= 2e-2 * np.linalg.norm(gref)


@pytest.mark.gpu
def test_trainer_reduces_loss_and_returns_parameters():
    from colb_b200.engine import Trainer
    rng = np.random.default_rng(6)
    x = rng.normal(size=(2048, 48)).astype(np.float32)
    w = rng.normal(size=(48, 12)).astype(np.float32) / 7
    y = np.tanh(x @ w).astype(np.float32)
    t = Trainer(LO.init_params(7))
    t.set_data(x, y)
    losses = [t.epoch(rng.permutation(len(x)), 128, 1e-3) for _ in range(8)]
    assert losses[-1] < 0.3 * losses[0]
    p = t.params()
    l_after, _ = LO.loss_grad(p, x[:256], y[:256])
    assert l_after == pytest.approx(losses[-1], rel=0.5)


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["net", "cubes"])
def test_features_match_oracle(which):
    from colb_b200 import params as P, scene as S
    from colb_b200.engine import Engine
    from oracle import oracle as O
    if which == "net":
        sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    else:
        sc = S.config1_cubes(seed=1)
        st = sc["state"].copy()
        st[:, 25] -= st[:, 25].min() - 0.5 * np.sqrt(3) - 0.02     # lower layer close to the ground
        st[:, 1] = st[:, 25]
        sc = dict(sc, state=st)
    p = P.config_params()
    e = Engine(p, sc)
    f = e.features()
    radius = LO.FEAT_RADIUS_DHAT * p.dhat
    o = O.OracleWorld(P.config_params(cand_dist=radius), sc)
    quads, kinds = o.pairs()
    assert len(quads) > 0
    pl = sc["planes"]
    ref = LO.features(sc["state"], o.vertices(), sc["vert_body"], sc["mass"], quads, kinds, pl, p.dt, list(p.gravity), p.dhat)
    assert np.allclose(f[:, :16], ref[:, :16], atol=1e-5, rtol=1e-5)
    # nearest-pair slots: distances agree; directions agree where distances are not tied
    d_gpu, d_ref = f[:, 16::4], ref[:, 16::4]
    assert np.allclose(d_gpu, d_ref, atol=1e-6)
    for b in range(len(f)):
        for k in range(8):
            tied = np.sum(np.abs(d_ref[b] - d_ref[b, k]) < 1e-6) > 1
            if not tied:
                assert np.allclose(f[b, 17 + 4 * k:20 + 4 * k], ref[b, 17 + 4 * k:20 + 4 * k], atol=1e-5), (b, k)


@pytest.mark.gpu
def test_trained_network_gain_over_plain(capsys):
    """What the shipped network changes on an unseen 8 x 8 net over 40 steps:
    Newton iterations per step of warm_start 3 against the plain start.  Both
    must converge every step with no intersection, and the measured ratio
    must reproduce the one recorded when the network was trained
    (colb_b200/learned.py writes it into the model file, meta["probe"]),
    within 0.1: the test asserts the gain (or loss) that the shipped model
    claims, whichever it is."""
    from colb_b200 import learned as Lr, params as P, scene as S
    from colb_b200.engine import Engine
    params, norm, meta = Lr.load()
    probe = meta.get("probe", dict(n=8, seed=Lr.PROBE_SEED, steps=Lr.PROBE_STEPS, iter_ratio=None))
    sc = S.config2_chain_net(n=probe["n"], seed=probe["seed"])
    iters = {}
    for ws in (0, 3):
        e = Engine(P.config_params(dt=1.0 / 240.0, warm_start=ws), sc)
        if ws == 3:
            e.set_mlp(params, norm)
        tot = unconv = 0
        for _ in range(probe["steps"]):
            rc, st = e.step(1, allow=(-6, -7))
            tot += st.newton_iters
            unconv += st.unconverged
        assert unconv == 0
        assert e.count_intersections() == 0
        iters[ws] = tot / probe["steps"]
    ratio = iters[3] / iters[0]
    with capsys.disabled():
        print(f"\nlearned warm start: {iters[3]:.2f} Newton iterations/step vs {iters[0]:.2f} plain "
              f"(ratio {ratio:.2f}; recorded at training {probe['iter_ratio']})")
    if probe["iter_ratio"] is not None:
        assert abs(ratio - probe["iter_ratio"]) <= 0.1
