"""Pre-rolled benchmark states.

The chain-net workload is timed in the middle of its 500-step trajectory,
where the links rest on one another, rather than in the first steps where
the net still falls freely.  The state after `steps` plain FP64 steps of
config2_chain_net(n=16, seed=0) is stored once so that every arm (the GPU
library, the CPU restatement) starts from the same bytes:

    python -m colb_b200.fixtures          # writes colb_b200/data/net16_t120.npz
"""
import argparse
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NET16_T120 = os.path.join(HERE, "data", "net16_t120.npz")


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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=120)
    ap.add_argument("--out", default=NET16_T120)
    a = ap.parse_args()
    make_net16(a.steps, a.out)
    print("wrote", a.out)


if __name__ == "__main__":
    main()
