"""Line search as one CUDA graph per Newton iteration (AbdParams.ls_graph):
the while-node repeats apply / energies / decide on the device, so the
decisions, step lengths and trajectories are those of the host loop (needs a
GPU).  Energies are summed with atomics in either mode, so states are
compared at 1e-9 of the scene extent; iteration and trial counts must match."""
import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import params as P, scene as S
from colb_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _both(sc, steps, chunks=3, **over):
    a = Engine(P.config_params(ls_graph=0, **over), sc)
    b = Engine(P.config_params(ls_graph=1, **over), sc)
    graphs = 0
    for _ in range(chunks):
        ra, sa = a.step(steps)
        rb, sb = b.step(steps)
        assert sa.newton_iters == sb.newton_iters
        assert sa.ls_trials == sb.ls_trials
        assert sa.ls_graph_launches == 0
        graphs += sb.ls_graph_launches
        xa, xb = a.vertices(), b.vertices()
        assert np.abs(xa - xb).max() <= 1e-9 * np.abs(xa).max()
    return graphs, b


@pytest.mark.parametrize("autotune", [0, 1])
def test_graph_line_search_equals_host_loop_net(autotune):
    """3x3 chain mail in contact from the first step; with the autotuner on
    the graph starts once the energy kernels' launch shapes are chosen."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    graphs, b = _both(sc, 2, dt=1.0 / 240.0, linear_solver=2, autotune=autotune)
    assert graphs > 0
    assert b.count_intersections() == 0


def test_graph_line_search_with_contact_groups_matches_oracle():
    """27 icospheres landing in a small box, one step length per contact
    group, the search run as a graph: same as the host loop and as the
    oracle."""
    sc = S.config5_pile(n=27, seed=0, box=(3.3, 3.3, 40.0))
    graphs, b = _both(sc, 8, chunks=3, lin_tol=1e-10, ls_groups=1, autotune=0)
    assert graphs > 0
    o = O.OracleWorld(P.config_params(lin_tol=1e-10, ls_groups=1), sc)
    o.step(24)
    xb, xo = b.vertices(), o.vertices()
    assert np.abs(xb - xo).max() <= 1e-6 * np.abs(xo).max()


def test_graph_rebuilt_when_swept_list_grows():
    """A minimal contact capacity makes the swept list grow during the
    run; the graph is captured again around the new list."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    graphs, _ = _both(sc, 2, dt=1.0 / 240.0, linear_solver=2, autotune=0, contact_capacity=1)
    assert graphs > 0


def test_graph_parameter_is_validated():
    from colb_b200.engine import AbdError
    sc = S.config1_cubes(seed=0)
    with pytest.raises(AbdError):
        Engine(P.config_params(ls_graph=2), sc)
