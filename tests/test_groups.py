"""Line search per contact group (AbdParams.ls_groups) on the CPU oracle.

Bodies whose swept, padded boxes over a Newton step do not overlap
(transitively) cannot touch anywhere along that step, so the incremental
potential is a sum of independent group energies and each group may take
its own CCD bound and back-off.  The step's solution is the same minimiser:
a converged step in either mode lands on the same state up to the Newton
tolerance.
"""
import numpy as np

from oracle import oracle as O
from colb_b200 import params as P, scene as S


def _run(sc, steps, **over):
    w = O.OracleWorld(P.config_params(lin_tol=1e-10, **over), [sc])
    iters, unconv = 0, 0
    for _ in range(steps):
        rc, st = w.step(1)
        iters += st.newton_iters
        unconv += st.unconverged
    return w.vertices(), iters, unconv


def test_groups_reach_the_same_states_as_one_step_length():
    """8 cubes falling onto the ground plane, 40 steps (they land at step
    18): with one step length per cube group the trajectory is the same to
    the Newton tolerance and needs no more iterations."""
    sc = S.config1_cubes(seed=0)
    x0, it0, u0 = _run(sc, 40, ls_groups=0)
    x1, it1, u1 = _run(sc, 40, ls_groups=1)
    assert u0 == 0 and u1 == 0
    assert np.abs(x1 - x0).max() <= 1e-6 * np.abs(x0).max()
    assert it1 <= it0


def test_groups_without_contact_equal_the_scene_line_search():
    """Before the first contact every group takes the full step, as the
    scene does: the two modes agree to rounding."""
    sc = S.config1_cubes(seed=3)
    x0, it0, _ = _run(sc, 10, ls_groups=0)
    x1, it1, _ = _run(sc, 10, ls_groups=1)
    assert it0 == it1
    assert np.abs(x1 - x0).max() <= 1e-12 * np.abs(x0).max()
