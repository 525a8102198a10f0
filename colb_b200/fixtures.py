"""Pre-rolled benchmark states.

The chain-net workload is timed in the middle of its 500-step trajectory,
where the links rest on one another, rather than in the first steps where
the net still falls freely.  The state after `steps` plain FP64 steps of
config2_chain_net(n=16, seed=0) is stored once so that every arm (the GPU
library, the CPU restatement) starts from the same bytes:

    python -m colb_b200.fixtures          # writes colb_b200/data/net16_t120.npz

The pile workload (4096 icospheres dropped into a 12 x 12 x 40 open box) is
timed while the spheres land on one another; its state after 100 FP64
steps of config5_pile(seed=0), stepped with one step length per contact
group (the plain line search does not reach the 1e-5 residual within 64
iterations there), is stored the same way:

    python -m colb_b200.fixtures --which pile   # writes colb_b200/data/pile_t100.npz
"""
import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NET16_T120 = os.path.join(HERE, "data", "net16_t120.npz")
PILE_T100 = os.path.join(HERE, "data", "pile_t100.npz")


def make_net16(steps=120, path=NET16_T120, seed=0):
    from . import params as P, scene as S
    from .engine import Engine
    sc = S.config2_chain_net(n=16, seed=seed)
    e = Engine(P.config_params(dt=1.0 / 240.0), sc)
    iters = []
    for _ in range(steps):
        rc, st = e.step(1)
        iters.append(st.newton_iters)
    state = e.get_state()
    assert e.count_intersections() == 0
    np.savez(path, state=state, steps=steps, seed=seed, iters=np.array(iters, np.int32))
    return state


def load_net16(path=NET16_T120):
    z = np.load(path)
    return z["state"], int(z["steps"]), int(z["seed"])


def make_pile(steps=100, path=PILE_T100, seed=0):
    from . import params as P, scene as S
    from .engine import Engine
    sc = S.config5_pile(seed=seed)
    e = Engine(P.config_params(ls_groups=1), sc)
    iters, unconv = [], 0
    for _ in range(steps):
        rc, st = e.step(1, allow=(-6,))
        iters.append(st.newton_iters)
        unconv += st.unconverged
    state = e.get_state()
    assert e.count_intersections() == 0
    np.savez_compressed(path, state=state, steps=steps, seed=seed, iters=np.array(iters, np.int32), unconverged=unconv)
    return state


def load_pile(path=PILE_T100):
    z = np.load(path)
    return z["state"], int(z["steps"]), int(z["seed"])


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--which", choices=["net16", "pile"], default="net16")
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    if a.which == "pile":
        out = a.out or PILE_T100
        make_pile(a.steps or 100, out)
    else:
        out = a.out or NET16_T120
        make_net16(a.steps or 120, out)
    print("wrote", out)


if __name__ == "__main__":
    main()
