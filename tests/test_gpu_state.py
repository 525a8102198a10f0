"""abd_set_state / abd_get_state round trips (needs a GPU).

A host loop that reads the state after every step and hands it back before
the next keeps the swept candidate list (the positions are bit-identical);
a state with moved bodies drops it.  Either way the steps are those of an
untouched handle: states agree to 1e-9 of the scene extent (energies are
summed with atomics, so runs agree to rounding, not bit for bit)."""
import numpy as np
import pytest

from colb_b200 import params as P, scene as S
from colb_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _net():
    return S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2), P.config_params(dt=1.0 / 240.0, linear_solver=2)


def test_round_trip_each_step_equals_plain_stepping():
    sc, p = _net()
    a, b = Engine(p, sc), Engine(p, sc)
    buf = np.zeros((b.nb, 48))
    for _ in range(6):
        ra, sa = a.step(1)
        b.get_state(out=buf)
        b.set_state(buf)
        rb, sb = b.step(1)
        assert sa.newton_iters == sb.newton_iters
    xa, xb = a.vertices(), b.vertices()
    assert np.abs(xa - xb).max() <= 1e-9 * np.abs(xa).max()


def test_moved_state_steps_like_a_fresh_handle():
    sc, p = _net()
    a = Engine(p, sc)
    a.step(2)
    s2 = a.get_state()
    a.step(3)
    a.set_state(s2)                   # bodies move back: the swept list is dropped
    a.step(3)
    fresh = Engine(p, dict(sc, state=s2))
    fresh.step(3)
    xa, xf = a.vertices(), fresh.vertices()
    assert np.abs(xa - xf).max() <= 1e-9 * np.abs(xf).max()
    assert a.count_intersections() == 0
