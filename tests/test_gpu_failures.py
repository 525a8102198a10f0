"""Failure reporting and the quadratic barrier on the GPU (needs a GPU).

Every failure here is made on the host: a non-finite state handed to
abd_set_state, a Krylov iteration cap of 1, a CCD iteration cap of 1, and a
non-finite Newton increment written over the solver's output by the
library's test hook (AbdParams.test_inject).  None of them faults, traps or
hangs the GPU: the library turns each into a status code (the reference
has none of these; its contact buffer wraps silently, contact.py:137, and
its loop stops at the cap without a report, abd.py:699).
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import params as P, scene as S
from colb_b200._abi import (ABD_ERR_CCD_CAP, ABD_ERR_NAN, ABD_ERR_SOLVER_CAP, ABD_INJECT_DU_NONFINITE,
                             ABD_INJECT_SWEPT_FULL,
                            BARRIER_QUADRATIC, SOLVER_PCG)
from colb_b200.engine import AbdError, Engine

pytestmark = pytest.mark.gpu


def test_non_finite_state_is_rejected(chain_scene):
    e = Engine(P.reference_params(), chain_scene)
    before = e.get_state()
    bad = before.copy()
    bad[7, 25] = np.nan
    rc = e.L.abd_set_state(e.h, bad.ctypes.data_as(C.POINTER(C.c_double)), e.nb)
    assert rc == ABD_ERR_NAN
    assert b"body 7" in e.L.abd_last_error(e.h)
    bad[7, 25] = np.inf
    with pytest.raises(AbdError) as ei:
        e.set_state(bad)
    assert ei.value.code == ABD_ERR_NAN
    assert np.array_equal(e.get_state(), before)       # the state is left unchanged
    rc, st = e.step(1)
    assert rc == 0 and st.unconverged == 0


def test_krylov_cap_is_reported(chain_scene, chain_pairs):
    """lin_max_iter = 1: every Krylov solve stops above tolerance; the step
    still runs (with that increment) and returns ABD_ERR_SOLVER_CAP."""
    e = Engine(P.reference_params(linear_solver=SOLVER_PCG, hess_mode=1, lin_max_iter=1), chain_scene)
    e.set_state(chain_pairs["states"][2])
    rc, st = e.step(1, allow=(ABD_ERR_SOLVER_CAP, -6))
    assert rc == ABD_ERR_SOLVER_CAP
    assert st.solver_capped > 0 and st.newton_iters > 0
    assert np.all(np.isfinite(e.get_state()))
    with pytest.raises(AbdError) as ei:
        e.solve()
    assert ei.value.code == ABD_ERR_SOLVER_CAP
    # with the default cap the same solve reaches its tolerance
    ok = Engine(P.reference_params(linear_solver=SOLVER_PCG, hess_mode=1), chain_scene)
    ok.set_state(chain_pairs["states"][2])
    rc, st = ok.step(1)
    assert rc == 0 and st.solver_capped == 0


def _head_on_cubes():
    """Two unit cubes 0.05 apart closing at 12 m/s (no gravity): at
    dt = 1/120 the first Newton direction moves them 0.1 towards each other,
    more than the gap, so additive CCD needs several iterations."""
    V, F = S.cube_mesh(1.0)
    bodies = [S._body(V, F, 1000.0, [0.0, 0.0, 0.0], v=np.array([6.0, 0.0, 0.0])),
              S._body(V, F, 1000.0, [1.05, 0.0, 0.0], v=np.array([-6.0, 0.0, 0.0]))]
    return S.assemble_bodies(bodies)


def test_ccd_cap_is_reported_and_conservative():
    """ccd_max_iter = 1: queries that need more additive-CCD iterations stop
    at the time reached (a conservative bound), the step reports
    ABD_ERR_CCD_CAP, and no intersection appears."""
    sc = _head_on_cubes()
    e = Engine(P.config_params(gravity=[0.0, 0.0, 0.0], ccd_max_iter=1), sc)
    rc, st = e.step(2, allow=(ABD_ERR_CCD_CAP,))
    assert rc == ABD_ERR_CCD_CAP
    assert e.count_intersections() == 0
    assert np.all(np.isfinite(e.get_state()))
    ref = Engine(P.config_params(gravity=[0.0, 0.0, 0.0]), sc)
    rc, st = ref.step(2)
    assert rc == 0 and ref.count_intersections() == 0


def test_mixed_precision_guard_replaces_a_non_finite_increment():
    """The first Newton increment of every step of scene 0 is overwritten
    with NaN after the FP32 solve (test hook); the guard must replace it by
    the block-Jacobi direction, and the step must still converge to the
    FP64 solution within the mixed-precision tolerance."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    e = Engine(P.config_params(dt=1.0 / 240.0, precision=1, test_inject=ABD_INJECT_DU_NONFINITE), sc)
    ref = Engine(P.config_params(dt=1.0 / 240.0, lin_tol=1e-10), sc)
    for _ in range(3):
        rc, st = e.step(1)
        ref.step(1)
        assert rc == 0 and st.du_guard_hits == 1 and st.unconverged == 0
        x, xr = e.vertices(), ref.vertices()
        assert np.all(np.isfinite(x))
        assert np.abs(x - xr).max() <= 1e-4 * np.abs(xr).max()
    assert e.count_intersections() == 0
    plain = Engine(P.config_params(dt=1.0 / 240.0, precision=1), sc)
    rc, st = plain.step(1)
    assert st.du_guard_hits == 0


def test_swept_list_that_does_not_fit_caps_the_step_length():
    """A swept candidate list that does not fit even after growing (an
    increment that sweeps most primitives into reach) is built for a quarter
    of the increment, then a sixteenth, ..., and the line search caps its step
    length at that fraction, so the list still covers every position it
    visits.  The test hook makes the first list of every step "not fit": the
    steps must still converge, without intersections, to the positions of a
    run without the hook."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    a = Engine(P.config_params(dt=1.0 / 240.0, test_inject=ABD_INJECT_SWEPT_FULL), sc)
    b = Engine(P.config_params(dt=1.0 / 240.0), sc)
    for _ in range(3):
        ra, sa = a.step(1)
        rb, sb = b.step(1)
        assert ra == 0 and rb == 0 and sa.unconverged == 0 and sb.unconverged == 0
        assert sa.newton_iters >= sb.newton_iters
        xa, xb = a.vertices(), b.vertices()
        assert np.abs(xa - xb).max() <= 1e-6 * np.abs(xb).max()
    assert a.count_intersections() == 0


def test_quadratic_barrier_assembly_and_trajectory(chain_scene, chain_pairs):
    """barrier.py:23-44, b = (x - xh)^2 in x = d^2: gradient and Hessian at
    a contact state (1e-9), then a short trajectory (1e-6 of the extent)."""
    p = P.reference_params(barrier=BARRIER_QUADRATIC, lin_tol=1e-10)
    e, o = Engine(p, chain_scene), O.OracleWorld(p, chain_scene)
    st = chain_pairs["states"][2]
    e.set_state(st); o.set_state(st)
    assert e.energy()[0] == pytest.approx(o.energy()[0], rel=1e-11)
    ge, He = e.assemble(); go, Ho = o.assemble()
    assert np.abs(ge - go).max() <= 1e-9 * np.abs(go).max()
    assert np.abs(He - Ho).max() <= 1e-9 * np.abs(Ho).max()
    e2, o2 = Engine(p, chain_scene), O.OracleWorld(p, chain_scene)
    for _ in range(3):
        e2.step(4); o2.step(4)
        xe, xo = e2.vertices(), o2.vertices()
        assert np.abs(xe - xo).max() <= 1e-6 * np.abs(xo).max()
