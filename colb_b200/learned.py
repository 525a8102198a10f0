"""Learned warm start (no counterpart in the reference).

The plain solver generates its own training data: at the start of every
step the per-body features (abd_get_features) are recorded, and after the
step the converged increment.  The network (48 -> 256 -> 256 -> 256 -> 12,
include/abd_b200.h) learns the body-frame correction to the inertial
increment, per unit time; it is trained on the GPU by the library's own
kernels (abd_trainer_*) and used through warm_start 3, where the Newton +
CCD loop always runs from the guess to the same residual, so the network
only changes where Newton starts.

    python -m colb_b200.learned --out colb_b200/data/warmstart_net16.npz

trains the network shipped with the package on at least 2e5 (features,
converged increment) pairs from 16 x 16 chain nets (seeds TRAIN_SEEDS, 200
steps each from t = 0: fall, impact and rest), then evaluates it against the
plain start on held-out seeds (EVAL_SEEDS) and stores that evaluation in the
model file's metadata.
"""
import argparse
import json
import os
import time

import numpy as np

from . import params as P, scene as S
from .engine import Engine, Trainer, MLP_IN, MLP_OUT, MLP_NPARAM

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_MODEL = os.path.join(HERE, "data", "warmstart_net16.npz")


def body_targets(s0, s1, dt, gravity):
    """Body-frame correction to the inertial increment, per unit time, of
    every body between states s0 (start of the step) and s1 (after it):
    y[0:3] = q (dc - dt v - dt^2 g) / dt, y[3:12] = q (dq - dt qdot)^T / dt."""
    g = np.asarray(gravity, np.float64)
    q = s0[:, 3:12].reshape(-1, 3, 3)
    dc = s1[:, 0:3] - s0[:, 0:3] - dt * s0[:, 12:15] - dt * dt * g
    dq = (s1[:, 3:12] - s0[:, 3:12] - dt * s0[:, 15:24]).reshape(-1, 3, 3)
    yc = np.einsum("bij,bj->bi", q, dc) / dt
    yM = np.einsum("bik,bjk->bij", q, dq) / dt
    return np.concatenate([yc, yM.reshape(-1, 9)], axis=1).astype(np.float32)


def collect(engine, steps, mass):
    """Runs `steps` plain steps and returns (features, targets) of the dynamic
    bodies at every step."""
    prm = engine.params
    dyn = np.asarray(mass) > 0
    X, Y = [], []
    for _ in range(steps):
        f = engine.features()
        s0 = engine.get_state()
        engine.step(1, allow=(-6, -7))
        s1 = engine.get_state()
        X.append(f[dyn])
        Y.append(body_targets(s0, s1, prm.dt, list(prm.gravity))[dyn])
    return np.concatenate(X), np.concatenate(Y)


def c2_scenes(seeds, vary=True):
    """16 x 16 chain nets of the chain-net configuration (R = 1, r = 0.25,
    corners pinned) with the given seeds; `vary` also draws the pitch in
    [1.48, 1.49], the lift in [0.85, 0.9] and the velocity noise in
    [1e-3, 5e-2] from the seed."""
    out = []
    for sd in seeds:
        rng = np.random.default_rng(10_000 + sd)
        kw = dict(pitch=float(rng.uniform(1.48, 1.49)), lift=float(rng.uniform(0.85, 0.9)),
                  vel_noise=float(rng.uniform(1e-3, 5e-2))) if vary else {}
        out.append(S.config2_chain_net(n=16, seed=int(sd), **kw))
    return out


def evaluate(params, norm, scenes, steps, rest_from=120, dt=1.0 / 240.0, device=0, log=None):
    """Plain start against the learned warm start on each scene from t = 0:
    Newton iterations and device milliseconds per step, over all steps and
    over the steps from `rest_from` on (the resting net), with the
    unconverged steps and intersections of both."""
    rows = []
    for k, sc in enumerate(scenes):
        row = {}
        for name, ws in (("plain", 0), ("learned", 3)):
            e = Engine(P.config_params(dt=dt, warm_start=ws), sc, device=device)
            if ws == 3:
                e.set_mlp(params, norm)
            it, ms, unconv = [], [], 0
            for _ in range(steps):
                rc, st = e.step(1, allow=(-6, -7))
                it.append(st.newton_iters); ms.append(st.gpu_ms); unconv += st.unconverged
            it, ms = np.array(it, float), np.array(ms, float)
            row[name] = dict(iters=float(it.mean()), ms=float(ms.mean()), iters_rest=float(it[rest_from:].mean()),
                             ms_rest=float(ms[rest_from:].mean()), unconverged=int(unconv),
                             intersections=int(e.count_intersections()))
            e.close()
        row["iter_ratio"] = row["learned"]["iters"] / row["plain"]["iters"]
        row["iter_ratio_rest"] = row["learned"]["iters_rest"] / row["plain"]["iters_rest"]
        row["time_ratio"] = row["learned"]["ms"] / row["plain"]["ms"]
        rows.append(row)
        if log:
            log(f"eval scene {k}: {json.dumps(row)}")
    mean = lambda key: float(np.mean([r[key] for r in rows]))
    return dict(scenes=rows, iter_ratio=mean("iter_ratio"), iter_ratio_rest=mean("iter_ratio_rest"),
                time_ratio=mean("time_ratio"), steps=steps, rest_from=rest_from)


def training_scenes(count, seed=0, n_range=(8, 16)):
    """Chain nets of varied size, pitch, lift and initial velocity noise
    (pitch in [1.48, 1.495] and lift in [0.82, 0.9] keep the links apart at
    t = 0)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(count):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        out.append(S.config2_chain_net(n=n, seed=1000 + 97 * seed + k, pitch=float(rng.uniform(1.48, 1.495)),
                                       lift=float(rng.uniform(0.82, 0.9)), vel_noise=float(rng.uniform(1e-3, 0.2))))
    return out


def fit_norm(X, Y):
    xm, xs = X.mean(0), X.std(0)
    ym, ys = Y.mean(0), Y.std(0)
    xs = np.where(xs > 1e-6, xs, 1.0)
    ys = np.where(ys > 1e-6, ys, 1.0)
    return np.concatenate([xm, xs, ym, ys]).astype(np.float32)


def init_params(seed=0):
    """He-normal hidden layers, a small output layer, zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for (n_out, n_in, scale) in [(256, MLP_IN, 1.0), (256, 256, 1.0), (256, 256, 1.0), (MLP_OUT, 256, 0.1)]:
        parts.append((rng.normal(size=(n_out, n_in)) * np.sqrt(2.0 / n_in) * scale).ravel())
        parts.append(np.zeros(n_out))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == MLP_NPARAM
    return p


def train(X, Y, epochs=40, batch=512, lr=1e-3, seed=0, device=0, log=None):
    """Trains on the GPU; returns (params, norm, per-epoch losses)."""
    norm = fit_norm(X, Y)
    Xn = ((X - norm[:MLP_IN]) / norm[MLP_IN:2 * MLP_IN]).astype(np.float32)
    Yn = ((Y - norm[2 * MLP_IN:2 * MLP_IN + MLP_OUT]) / norm[2 * MLP_IN + MLP_OUT:]).astype(np.float32)
    t = Trainer(init_params(seed), device=device)
    t.set_data(Xn, Yn)
    rng = np.random.default_rng(seed)
    losses = []
    for ep in range(epochs):
        lr_ep = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs))
        losses.append(t.epoch(rng.permutation(len(Xn)), batch, lr_ep))
        if log:
            log(f"epoch {ep} loss {losses[-1]:.5f}")
    params = t.params()
    t.close()
    return params, norm, losses


def save(path, params, norm, meta=None):
    os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
    np.savez(path, params=params.astype(np.float32), norm=norm.astype(np.float32),
             meta=json.dumps(meta or {}))


def load(path=DEFAULT_MODEL):
    z = np.load(path)
    return z["params"], z["norm"], json.loads(str(z["meta"]))


def run_steps(engine, steps):
    """Steps one at a time; returns (Newton iterations per step, device ms per step)."""
    iters, ms = [], []
    for _ in range(steps):
        rc, st = engine.step(1, allow=(-6, -7))
        iters.append(st.newton_iters / max(1, engine.ns))
        ms.append(st.gpu_ms)
    return np.array(iters), np.array(ms)


TRAIN_SEEDS = tuple(range(1000, 1004))    # chain-net seeds the network is trained on
EVAL_SEEDS = (500, 501)                    # held out: never seen in training (the benchmark net is seed 0)
PROBE_SEED, PROBE_STEPS = 123, 40          # the unseen 8 x 8 net of the short check


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=DEFAULT_MODEL)
    ap.add_argument("--pairs", type=int, default=200_000, help="training pairs to collect (at least)")
    ap.add_argument("--steps", type=int, default=200, help="steps per training scene")
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--eval-steps", type=int, default=160)
    ap.add_argument("--seed", type=int, default=0)
    args = ap.parse_args()
    t0 = time.time()
    Xs, Ys = [], []
    seeds = []
    for sd in TRAIN_SEEDS + tuple(range(2000, 2100)):
        if sum(len(x) for x in Xs) >= args.pairs:
            break
        sc = c2_scenes([sd])[0]
        e = Engine(P.config_params(dt=1.0 / 240.0), sc)
        X, Y = collect(e, args.steps, sc["mass"])
        Xs.append(X); Ys.append(Y); seeds.append(sd)
        e.close()
        print(f"scene seed {sd}: {len(X)} pairs ({time.time() - t0:.1f} s)", flush=True)
    X, Y = np.concatenate(Xs), np.concatenate(Ys)
    print(f"collected {len(X)} pairs in {time.time() - t0:.1f} s", flush=True)
    t1 = time.time()
    params, norm, losses = train(X, Y, epochs=args.epochs, seed=args.seed, log=print)
    train_s = time.time() - t1
    ev = evaluate(params, norm, c2_scenes(EVAL_SEEDS), args.eval_steps, log=print)
    # the short check tests/test_learned.py repeats: an unseen 8 x 8 net, 40 steps
    probe = evaluate(params, norm, [S.config2_chain_net(n=8, seed=PROBE_SEED)], PROBE_STEPS, rest_from=0)
    meta = dict(pairs=int(len(X)), epochs=args.epochs, final_loss=float(losses[-1]), train_seconds=train_s,
                train_seeds=seeds, steps=args.steps, seed=args.seed, eval_seeds=list(EVAL_SEEDS), eval=ev,
                probe=dict(seed=PROBE_SEED, n=8, steps=PROBE_STEPS, iter_ratio=probe["iter_ratio"],
                           plain_iters=probe["scenes"][0]["plain"]["iters"],
                           learned_iters=probe["scenes"][0]["learned"]["iters"]))
    save(args.out, params, norm, meta)
    print(json.dumps({k: v for k, v in meta.items() if k != "eval"}))
    print(f"eval: iterations learned/plain {ev['iter_ratio']:.3f} (resting {ev['iter_ratio_rest']:.3f}), "
          f"device time learned/plain {ev['time_ratio']:.3f}")
    print(f"saved {args.out} ({time.time() - t0:.1f} s)")


if __name__ == "__main__":
    main()
