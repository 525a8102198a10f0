"""Line search per contact group (AbdParams.ls_groups): CUDA path vs the
CPU oracle in the same mode, and the mode against the scene line search
(needs a GPU).  Trajectory tolerance 1e-6 of the scene extent, as for the
scene line search."""
import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import params as P, scene as S
from colb_b200.engine import Engine, AbdError

pytestmark = pytest.mark.gpu


def _compare(sc, p, chunks, n):
    e, o = Engine(p, sc), O.OracleWorld(p, sc)
    ie = io = 0
    for _ in range(chunks):
        rc, se = e.step(n)
        _, so = o.step(n)
        ie += se.newton_iters; io += so.newton_iters
        xe, xo = e.vertices(), o.vertices()
        assert np.abs(xe - xo).max() <= 1e-6 * np.abs(xo).max()
        assert e.count_intersections() == 0
    return ie, io


def test_groups_cubes_trajectory_matches_oracle():
    """8 cubes landing on the ground plane (contacts from step 18)."""
    sc = S.config1_cubes(seed=0)
    ie, io = _compare(sc, P.config_params(lin_tol=1e-10, ls_groups=1), 4, 10)
    assert abs(ie - io) <= 2


def test_groups_pile_trajectory_matches_oracle():
    """27 icospheres dropped into a 3.3 x 3.3 open box: walls, ground and
    sphere-sphere contacts from step 18 on."""
    sc = S.config5_pile(n=27, seed=0, box=(3.3, 3.3, 40.0))
    _compare(sc, P.config_params(lin_tol=1e-10, ls_groups=1), 5, 5)


def test_groups_one_group_equals_scene_line_search():
    """A 3x3 chain mail in contact from the first step forms one group, so
    the group line search takes the scene's step lengths."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    base = dict(dt=1.0 / 240.0, linear_solver=2)
    a, b = Engine(P.config_params(ls_groups=0, **base), sc), Engine(P.config_params(ls_groups=1, **base), sc)
    for _ in range(3):
        ra, sa = a.step(2); rb, sb = b.step(2)
        assert sa.newton_iters == sb.newton_iters
        xa, xb = a.vertices(), b.vertices()
        assert np.abs(xa - xb).max() <= 1e-9 * np.abs(xa).max()


def test_groups_batch_equals_single_scenes():
    """Groups never span scenes: a batch of three scenes steps like the
    three scenes on their own."""
    scs = S.config3_batch(n_scenes=3, seed=5, nmin=4, nmax=8)
    p = P.config_params(lin_tol=1e-10, ls_groups=1)
    eb = Engine(p, scs)
    eb.step(25)
    xb = eb.vertices()
    off = 0
    for sc in scs:
        es = Engine(p, sc)
        es.step(25)
        xs = es.vertices()
        assert np.abs(xb[off:off + len(xs)] - xs).max() <= 1e-6 * np.abs(xs).max()
        off += len(xs)


def test_groups_parameter_is_validated():
    sc = S.config1_cubes(seed=0)
    with pytest.raises(AbdError):
        Engine(P.config_params(ls_groups=2), sc)
