"""The benchmarked workloads against the CPU oracle (needs a GPU).

bench.py times the 16 x 16 chain mail (256 torus links, 73,728 vertices)
from its stored resting state, the falling cubes and the batch of uneven
scenes.  These tests run the CUDA path on exactly those inputs and
parameters and compare with oracle/abd_oracle.c step by step:
  * FP64: positions within 1e-6 of the scene extent and the same number of
    Newton iterations in every step;
  * mixed FP32/FP64: positions within 1e-4 of the FP64 oracle, the error of
    every step printed;
  * no intersection at any compared step.
The oracle steps the 256-link net in about 20-50 s per step on 8-16 host
threads, so the net is compared over 3 steps.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import fixtures, params as P, scene as S
from colb_b200.engine import Engine

pytestmark = pytest.mark.gpu

NET16_STEPS = 3


def _rel(x, ref):
    return float(np.abs(x - ref).max() / np.abs(ref).max())


@pytest.fixture(scope="module")
def net16_oracle():
    """Oracle trajectory of the net16 workload (bench.py --workload net16):
    config2_chain_net(n=16) from its state after 120 FP64 steps, dt = 1/240."""
    state, _, seed = fixtures.load_net16()
    sc = dict(S.config2_chain_net(n=16, seed=seed), state=state)
    O.set_threads(os.cpu_count() or 1)
    o = O.OracleWorld(P.config_params(dt=1.0 / 240.0), [sc])
    xs, iters = [], []
    for _ in range(NET16_STEPS):
        rc, st = o.step(1)
        xs.append(o.vertices())
        iters.append(st.newton_iters)
    return sc, xs, iters


def test_net16_fp64_matches_oracle_with_equal_newton_counts(net16_oracle):
    sc, xs, iters = net16_oracle
    e = Engine(P.config_params(dt=1.0 / 240.0), sc)
    got = []
    for k in range(NET16_STEPS):
        rc, st = e.step(1)
        got.append(st.newton_iters)
        err = _rel(e.vertices(), xs[k])
        print(f"net16 fp64 step {k}: rel err {err:.2e}, Newton {st.newton_iters} (oracle {iters[k]})")
        assert err <= 1e-6
        assert st.unconverged == 0
    assert got == iters
    assert e.count_intersections() == 0


def test_net16_mixed_within_1e4_of_fp64_oracle(net16_oracle):
    sc, xs, iters = net16_oracle
    e = Engine(P.config_params(dt=1.0 / 240.0, precision=1), sc)
    errs = []
    for k in range(NET16_STEPS):
        rc, st = e.step(1)
        errs.append(_rel(e.vertices(), xs[k]))
    print("net16 mixed: per-step rel position error vs the FP64 oracle", ["%.2e" % v for v in errs])
    assert max(errs) <= 1e-4
    assert e.count_intersections() == 0


def test_config1_cubes_full_200_steps():
    """The falling-cubes configuration for all of its 200 steps (dt = 1/120).
    Positions stay within 1e-6 of the oracle at every tenth step.  Newton
    iteration counts may differ by one in a step whose last residual lands
    within rounding of the 1e-5 tolerance (the two sum gradients and
    energies in different orders), so the totals must agree to 2 %."""
    sc = S.config1_cubes(seed=0)
    p = P.config_params()
    e, o = Engine(p, sc), O.OracleWorld(p, sc)
    tot_e = tot_o = 0
    for _ in range(20):
        rc, st = e.step(10)
        rco, sto = o.step(10)
        assert _rel(e.vertices(), o.vertices()) <= 1e-6
        tot_e += st.newton_iters
        tot_o += sto.newton_iters
        assert e.count_intersections() == 0
    assert abs(tot_e - tot_o) <= 0.02 * tot_o, (tot_e, tot_o)


def test_config3_batch_of_32_scenes():
    """32 uneven scenes (4..64 cubes / tori each) in one handle for 5 steps,
    every scene stepping with its own Newton loop, against the oracle
    stepping the same batch."""
    scenes = S.config3_batch(n_scenes=32, seed=0)
    p = P.config_params()
    e, o = Engine(p, scenes), O.OracleWorld(p, scenes)
    O.set_threads(os.cpu_count() or 1)
    for _ in range(5):
        rc, st = e.step(1)
        rco, sto = o.step(1)
        assert _rel(e.vertices(), o.vertices()) <= 1e-6
        assert st.newton_iters == sto.newton_iters and st.unconverged == sto.unconverged == 0
    assert e.count_intersections() == 0
