"""CUDA path vs the CPU oracle on the same seeded inputs (needs a GPU).

Bit-exact: vertex transform, candidate pair sets (float32 EE predicate and
float64 PT / half-space filters).  FP64 tolerances: energy 1e-11 rel,
gradient / Hessian 1e-9 rel, trajectories 1e-6 rel of the scene extent
(the FP64 trajectory tolerance).  Mixed precision: 1e-4.
"""
import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import params as P, scene as S
from colb_b200.engine import Engine

pytestmark = pytest.mark.gpu


def _edge_pairs(sc, quads):
    key = {(a, b): i for i, (a, b) in enumerate(sc["edges"])}
    return np.array([(key[(q[0], q[1])], key[(q[2], q[3])]) for q in quads], dtype=np.int32).reshape(-1, 2)


def _pair(params, sc):
    return Engine(params, sc), O.OracleWorld(params, sc)


def test_transform_bitexact(chain_scene, chain_pairs):
    e, o = _pair(P.reference_params(), chain_scene)
    for k in range(3):
        e.set_state(chain_pairs["states"][k]); o.set_state(chain_pairs["states"][k])
        assert np.array_equal(e.vertices(), o.vertices())


@pytest.mark.parametrize("broadphase", [1, 2])
def test_chain_pairs_bitexact_vs_golden(chain_scene, chain_pairs, broadphase):
    e = Engine(P.reference_params(broadphase=broadphase), chain_scene)
    for k in range(3):
        e.set_state(chain_pairs["states"][k])
        quads, kinds = e.pairs()
        assert np.all(kinds == 0)
        assert np.array_equal(_edge_pairs(chain_scene, quads), chain_pairs[f"pairs{k}"])


@pytest.mark.parametrize("broadphase", [1, 2])
@pytest.mark.parametrize("which", ["cubes", "net"])
def test_config_pairs_match_oracle(which, broadphase):
    sc = S.config1_cubes(seed=3) if which == "cubes" else S.config2_chain_net(n=3, seed=1)
    p = P.config_params(cand_dist=0.05, broadphase=broadphase)
    e, o = _pair(p, sc)
    st = sc["state"].copy()
    rng = np.random.default_rng(5)
    st[:, 24:27] += rng.normal(scale=0.05, size=(len(st), 3))
    e.set_state(st); o.set_state(st)
    qe, ke = e.pairs(); qo, ko = o.pairs()
    assert np.array_equal(ke, ko) and np.array_equal(qe, qo)


def test_energy_matches_oracle(chain_scene, chain_pairs):
    e, o = _pair(P.reference_params(), chain_scene)
    for k in range(3):
        e.set_state(chain_pairs["states"][k]); o.set_state(chain_pairs["states"][k])
        assert e.energy()[0] == pytest.approx(o.energy()[0], rel=1e-11)


@pytest.mark.parametrize("hess_mode", [0, 1])
def test_assembly_matches_oracle(chain_scene, chain_pairs, hess_mode):
    p = P.reference_params(hess_mode=hess_mode)
    e, o = _pair(p, chain_scene)
    st = chain_pairs["states"][2]
    e.set_state(st); o.set_state(st)
    ge, He = e.assemble(); go, Ho = o.assemble()
    assert np.abs(ge - go).max() <= 1e-9 * np.abs(go).max()
    assert np.abs(He - Ho).max() <= 1e-9 * np.abs(Ho).max()


def test_assembly_config_contacts():
    sc = S.config1_cubes(seed=2)
    st = sc["state"].copy()
    st[:4, 25] -= st[:4, 25] - 0.5 * np.sqrt(3) + 0.0  # drop the lower layer near the ground
    p = P.config_params(dhat=0.3, cand_dist=0.3)
    e, o = _pair(p, sc)
    e.set_state(st); o.set_state(st)
    ge, He = e.assemble(); go, Ho = o.assemble()
    assert np.abs(go).max() > 0
    assert np.abs(ge - go).max() <= 1e-9 * np.abs(go).max()
    assert np.abs(He - Ho).max() <= 1e-9 * np.abs(Ho).max()


@pytest.mark.parametrize("solver", [0, 1])
def test_solve_matches_dense(chain_scene, chain_pairs, solver):
    p = P.reference_params(linear_solver=solver, lin_tol=1e-12, hess_mode=1)
    e, o = _pair(p, chain_scene)
    st = chain_pairs["states"][1]
    e.set_state(st); o.set_state(st)
    du, it = e.solve()
    g, H = o.assemble()
    ref = np.linalg.solve(H, g)
    assert np.abs(du - ref).max() <= 1e-8 * np.abs(ref).max()
    assert it > 0


@pytest.mark.parametrize("hess_mode", [0, 1])
@pytest.mark.parametrize("precision", [0, 1])
def test_direct_solve_by_components(chain_scene, chain_pairs, hess_mode, precision):
    """The direct solver factors each connected component of the contact
    graph on its own (block inverse, shared-memory factorization for up to
    12 bodies, cuSOLVER above); the result must equal one dense solve."""
    eps = 2.2e-16 if precision == 0 else 1.2e-7
    cases = [(chain_scene, chain_pairs["states"][k]) for k in (1, 2)]
    # chain mail in contact: 25, 49 and 64 links in one component (the band
    # solver's window wraps once the component is wider than its band)
    for n in (5, 7, 8):
        cases.append((S.config2_chain_net(n=n, pitch=1.5 - 5e-4, seed=3), None))
    for sc, st in cases:
        if st is None:
            p = P.config_params(linear_solver=2, hess_mode=hess_mode, precision=precision)
        else:
            p = P.reference_params(linear_solver=2, hess_mode=hess_mode, precision=precision)
        e, o = _pair(p, sc)
        if st is not None:
            e.set_state(st); o.set_state(st)
        du, it = e.solve()
        g, H = o.assemble()
        ref = np.linalg.solve(H, g)
        assert it == 1
        # backward error of a stable factorization, and the forward error it implies
        n = len(g)
        back = np.abs(H @ du - g).max() / (np.abs(H).max() * np.abs(du).max() + np.abs(g).max())
        assert back <= 10 * n * eps
        ev = np.abs(np.linalg.eigvalsh(H))
        cond = ev.max() / ev.min()
        assert np.abs(du - ref).max() <= max(1e-8, 10 * n * cond * eps) * np.abs(ref).max()


@pytest.mark.parametrize("broadphase", [1, 2])
def test_reference_chain_trajectory(chain_scene, broadphase):
    p = P.reference_params(lin_tol=1e-10, broadphase=broadphase)
    e, o = _pair(p, chain_scene)
    for _ in range(4):
        rc, se = e.step(5)
        o.step(5)
        xe, xo = e.vertices(), o.vertices()
        scale = np.abs(xo).max()
        assert np.abs(xe - xo).max() <= 1e-6 * scale
    assert se.unconverged == 0


@pytest.mark.parametrize("broadphase", [1, 2])
def test_config_cubes_trajectory_and_no_intersection(broadphase):
    sc = S.config1_cubes(seed=0)
    p = P.config_params(lin_tol=1e-10, broadphase=broadphase)
    e, o = _pair(p, sc)
    for _ in range(3):
        e.step(10); o.step(10)
        xe, xo = e.vertices(), o.vertices()
        assert np.abs(xe - xo).max() <= 1e-6 * np.abs(xo).max()
        assert e.count_intersections() == 0


@pytest.mark.parametrize("warm_start", [1, 2])
def test_warm_start_trajectory_matches_oracle(warm_start):
    """Inertial (2) and user (1) warm starts: CCD-clipped, halved until the
    energy drops below that of now, then the same Newton loop."""
    sc = S.config1_cubes(seed=4)
    p = P.config_params(lin_tol=1e-10, warm_start=warm_start)
    e, o = _pair(p, sc)
    rng = np.random.default_rng(1)
    for _ in range(6):
        if warm_start == 1:
            dq = rng.normal(scale=1e-3, size=(e.nb, 12)).astype(np.float32)
            e.set_warm_start(dq); o.set_warm_start(dq)
        e.step(2 if warm_start == 2 else 1); o.step(2 if warm_start == 2 else 1)
        xe, xo = e.vertices(), o.vertices()
        assert np.abs(xe - xo).max() <= 1e-6 * np.abs(xo).max()
        assert e.count_intersections() == 0


def test_autotuner_picks_listed_launch_shapes():
    """The autotuner times every candidate launch shape during the first
    iterations, keeps the fastest, and the trajectory still matches the oracle."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    p = P.config_params(dt=1.0 / 240.0, autotune=1)
    e, o = _pair(p, sc)
    e.step(3); o.step(3)
    tuned = e.autotune()
    assert (tuned["contact_threads"], tuned["contacts_per_block"]) in [(64, 2), (128, 4), (256, 8), (64, 1), (128, 1)]
    assert tuned["list_energy_threads"] in (64, 128, 256, 512)
    assert tuned["body_energy_threads"] in (64, 128, 256, 512)
    assert np.abs(e.vertices() - o.vertices()).max() <= 1e-6 * np.abs(o.vertices()).max()
    off = Engine(P.config_params(dt=1.0 / 240.0, autotune=0), sc)
    off.step(1)
    assert set(off.autotune().values()) == {-1}


def test_batch_equals_single_scenes():
    scenes = S.config3_batch(n_scenes=4, seed=7, nmin=4, nmax=8)
    p = P.config_params(lin_tol=1e-10)
    eb = Engine(p, scenes)
    eb.step(3)
    sb = eb.get_state()
    off = 0
    for sc in scenes:
        e = Engine(p, sc)
        e.step(3)
        n = len(sc["mass"])
        assert np.abs(e.get_state() - sb[off:off + n]).max() <= 1e-9 * max(1.0, np.abs(sb).max())
        off += n


def test_mixed_precision_close_to_fp64(chain_scene):
    e64 = Engine(P.reference_params(lin_tol=1e-9), chain_scene)
    e32 = Engine(P.reference_params(lin_tol=1e-6, precision=1), chain_scene)
    e64.step(10); e32.step(10)
    x64, x32 = e64.vertices(), e32.vertices()
    assert np.abs(x64 - x32).max() <= 1e-4 * np.abs(x64).max()


@pytest.mark.parametrize("broadphase", [1, 2])
def test_contact_capacity_grows(chain_scene, chain_pairs, broadphase):
    e = Engine(P.reference_params(contact_capacity=64, broadphase=broadphase), chain_scene)
    e.set_state(chain_pairs["states"][2])
    quads, _ = e.pairs()
    assert np.array_equal(_edge_pairs(chain_scene, quads), chain_pairs["pairs2"])


def test_invalid_arguments_return_errors(chain_scene):
    import ctypes
    from colb_b200.engine import AbdError
    with pytest.raises(AbdError):
        Engine(P.reference_params(dhat=-1.0), chain_scene)
    e = Engine(P.reference_params(), chain_scene)
    st = np.zeros((e.nb + 1, 48))
    rc = e.L.abd_set_state(e.h, st.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), e.nb + 1)
    assert rc == -1 and b"mismatch" in e.L.abd_last_error(e.h)
    # a warm start whose body count differs from the handle's
    ws = np.zeros((e.nb + 1, 12), dtype=np.float32)
    rc = e.L.abd_set_warm_start(e.h, ws.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), e.nb + 1)
    assert rc == -1 and b"mismatch" in e.L.abd_last_error(e.h)
    rc = e.L.abd_set_warm_start(e.h, None, e.nb)
    assert rc == -1
    e.set_warm_start(np.zeros((e.nb, 12)))   # the right size is accepted


def test_net_trajectory_matches_oracle():
    """3x3 chain mail with contacts from the first step (pitch just under
    the touching distance): PT + EE contacts, log barrier, direct solve,
    CCD, monotone line search."""
    sc = S.config2_chain_net(n=3, pitch=1.5 - 5e-4, seed=2)
    p = P.config_params(dt=1.0 / 240.0, linear_solver=2)
    e, o = _pair(p, sc)
    for _ in range(3):
        rc, se = e.step(2)
        o.step(2)
        xe, xo = e.vertices(), o.vertices()
        assert np.abs(xe - xo).max() <= 1e-6 * np.abs(xo).max()
    assert se.n_active > 0
    assert e.count_intersections() == 0
