"""The CPU oracle against finite differences, analytic values, the
committed golden fixtures and its own invariants (no GPU)."""
import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import params as P, scene as S

rng = np.random.default_rng(1)


def fd(fun, x, h=1e-6):
    n = x.size
    g = np.zeros(n)
    for i in range(n):
        e = np.zeros(n); e[i] = h
        g[i] = (fun(x + e) - fun(x - e)) / (2 * h)
    return g


@pytest.mark.parametrize("kind,n", [("pp", 6), ("pe", 9), ("ee", 12), ("pt", 12)])
def test_squared_distance_derivatives(kind, n):
    for _ in range(5):
        x = rng.normal(size=n)
        f, g, H = O.d2(kind, x)
        gf = fd(lambda y: O.d2(kind, y)[0], x)
        Hf = np.stack([fd(lambda y: O.d2(kind, y)[1][i], x) for i in range(n)])
        assert np.allclose(g, gf, rtol=1e-6, atol=1e-6 * np.abs(g).max())
        assert np.allclose(H, Hf, rtol=1e-5, atol=1e-5 * np.abs(H).max())
        assert np.allclose(H, H.T, atol=1e-12 * np.abs(H).max())


def test_squared_distance_values():
    p, a, b = np.array([0., 1, 0]), np.array([-1., 0, 0]), np.array([1., 0, 0])
    assert O.d2("pe", np.concatenate([p, a, b]))[0] == pytest.approx(1.0)
    # skew lines at distance 2
    x = np.array([-1., 0, 0, 1, 0, 0, 0, -1, 2, 0, 1, 2])
    assert O.d2("ee", x)[0] == pytest.approx(4.0)
    # point above a triangle plane
    x = np.array([0.2, 0.2, 3.0, 0, 0, 0, 1, 0, 0, 0, 1, 0])
    assert O.d2("pt", x)[0] == pytest.approx(9.0)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_barrier_derivatives(kind):
    xh = 0.095 ** 2
    for x in [0.1 * xh, 0.5 * xh, 0.9 * xh]:
        b = O.barrier(kind, x, xh)
        h = 1e-9 * xh
        bp, bm = O.barrier(kind, x + h, xh), O.barrier(kind, x - h, xh)
        assert (bp[0] - bm[0]) / (2 * h) == pytest.approx(b[1], rel=1e-5)
        assert (bp[1] - bm[1]) / (2 * h) == pytest.approx(b[2], rel=1e-5)
    assert np.all(O.barrier(kind, xh, xh) == 0) and np.all(O.barrier(kind, 2 * xh, xh) == 0)


def test_cubic_barrier_values():
    # barrier.py:47-65: b = -(x-xh)^3, b' = -3(x-xh)^2, b'' = -6(x-xh)
    xh, x = 0.009025, 0.004
    t = x - xh
    assert np.allclose(O.barrier(0, x, xh), [-t ** 3, -3 * t * t, -6 * t], rtol=1e-14)


def test_ortho_derivatives_and_identity():
    q = np.eye(3) + 0.1 * rng.normal(size=(3, 3))
    e, g, H = O.ortho(q.ravel(), 1e5)
    assert g == pytest.approx(fd(lambda y: O.ortho(y, 1e5)[0], q.ravel(), 1e-7), rel=1e-5)
    Hf = np.stack([fd(lambda y: O.ortho(y, 1e5)[1][i], q.ravel(), 1e-7) for i in range(9)])
    assert np.allclose(H, Hf, rtol=1e-5, atol=1e-4)
    e0, g0, _ = O.ortho(np.eye(3).ravel(), 1e5)
    assert e0 == 0 and np.all(g0 == 0)


def test_psd_projection():
    for n in (6, 9, 12):
        A = rng.normal(size=(n, n)); A = A + A.T
        w, V = np.linalg.eigh(A)
        assert np.allclose(O.psd_project(A), V @ np.diag(np.maximum(w, 0)) @ V.T, atol=1e-12)


def test_segment_predicate_matches_golden():
    c = np.load("tests/golden/segseg_cases.npz")
    for i in range(0, len(c["pts"]), 7):
        o = O.seg_seg_f32(*c["pts"][i])
        assert o[0] == c["s"][i] and o[1] == c["t"][i] and o[2] == c["d"][i]


def _edge_pairs(sc, quads):
    key = {(a, b): i for i, (a, b) in enumerate(sc["edges"])}
    return np.array([(key[(q[0], q[1])], key[(q[2], q[3])]) for q in quads], dtype=np.int32).reshape(-1, 2)


def test_chain_pair_sets_match_golden(chain_scene, chain_pairs):
    w = O.OracleWorld(P.reference_params(), chain_scene)
    for k in range(3):
        w.set_state(chain_pairs["states"][k])
        quads, kinds = w.pairs()
        assert np.all(kinds == 0)
        assert np.array_equal(_edge_pairs(chain_scene, quads), chain_pairs[f"pairs{k}"])


def test_pair_list_sorted_and_unique(chain_scene, chain_pairs):
    w = O.OracleWorld(P.reference_params(), chain_scene)
    w.set_state(chain_pairs["states"][2])
    ij = _edge_pairs(chain_scene, w.pairs()[0])
    assert np.all(ij[:, 0] < ij[:, 1])
    keys = ij[:, 0].astype(np.int64) * 10 ** 6 + ij[:, 1]
    assert np.all(np.diff(keys) > 0)


def test_accd_conservative():
    # point falling onto a triangle: hit before the plane, after s-fraction of the gap
    x = np.array([0.2, 0.2, 1.0, 0, 0, 0, 1, 0, 0, 0, 1, 0])
    p = np.zeros(12); p[2] = -2.0
    hit, t = O.accd(1, x, p, s=0.1)
    assert hit and 0.4 < t < 0.5
    p[2] = -0.5
    assert not O.accd(1, x, p, s=0.1)[0]


@pytest.mark.parametrize("hess_mode", [0, 1])
def test_gradient_matches_energy_fd(chain_scene, chain_pairs, hess_mode):
    """The assembled gradient is the derivative of the oracle energy (with
    contacts active at the perturbed state).  FP64 closest points: the
    reference's float32 distance is quantised far above a 1e-7 FD step."""
    sc = dict(chain_scene)
    st = chain_pairs["states"][2].copy()
    w = O.OracleWorld(P.reference_params(ee_f32=0, hess_mode=hess_mode), sc)
    w.set_state(st)
    g, _ = w.assemble(dense=False)
    e0 = w.energy()[0]
    idx = rng.choice(np.nonzero(sc["mass"] > 0)[0], 4, replace=False)
    for b in idx:
        for k in (0, 4, 11):
            h = 1e-7
            s1, s2 = st.copy(), st.copy()
            s1[b, 24 + k] += h; s2[b, 24 + k] -= h
            w.set_state(s1); ep = w.energy()[0]
            w.set_state(s2); em = w.energy()[0]
            assert (ep - em) / (2 * h) == pytest.approx(g[12 * b + k], rel=2e-4, abs=1e-6)
    assert np.isfinite(e0)


def test_gradient_matches_energy_fd_point_triangle_and_ground():
    """Two icospheres 0.5 dhat apart (one rotated, so no two edges are
    parallel), the lower one 0.4 dhat above the ground: point-triangle,
    edge-edge and half-space contacts with the log barrier; the assembled
    gradient is the central difference of the oracle energy."""
    V, F = S.icosphere_mesh(1, 1.0)
    r, dh = 0.3, 1e-3
    Va = V * r
    Vb = Va @ S._rand_rotation(np.random.default_rng(3)).T
    cA = np.array([0.0, -Va[:, 1].min() + 0.4 * dh, 0.0])
    cB = cA + Va[np.argmax(Va[:, 1])] - Vb[np.argmin(Vb[:, 1])] + np.array([0.0, 0.5 * dh, 0.0])
    sc = S.assemble_bodies([S._body(Va, F, 1000.0, cA), S._body(Vb, F, 1000.0, cB)], planes=[S.GROUND])
    w = O.OracleWorld(P.config_params(), sc)
    st = w.get_state()
    _, kinds = w.pairs()
    assert set(np.unique(kinds)) == {0, 1, 2}
    g, _ = w.assemble(dense=False)
    for b in range(2):
        for k in range(12):
            h = 1e-7
            s1, s2 = st.copy(), st.copy()
            s1[b, 24 + k] += h; s2[b, 24 + k] -= h
            w.set_state(s1); ep = w.energy()[0]
            w.set_state(s2); em = w.energy()[0]
            assert (ep - em) / (2 * h) == pytest.approx(g[12 * b + k], rel=1e-5, abs=1e-6 * np.abs(g).max())


def test_reference_chain_steps_converge(chain_scene):
    w = O.OracleWorld(P.reference_params(), chain_scene)
    rc, st = w.step(3)
    assert rc == 0 and st.unconverged == 0 and st.steps == 3
    x = w.vertices()
    assert np.isfinite(x).all()


def test_batch_equals_independent_scenes():
    scenes = S.config3_batch(n_scenes=3, seed=4, nmin=4, nmax=6)
    p = P.config_params()
    wb = O.OracleWorld(p, scenes)
    wb.step(2)
    sb = wb.get_state()
    off = 0
    for sc in scenes:
        w = O.OracleWorld(p, sc)
        w.step(2)
        n = len(sc["mass"])
        assert np.array_equal(w.get_state(), sb[off:off + n])
        off += n


def test_config_cubes_fall_without_intersection():
    sc = S.config1_cubes(seed=0)
    w = O.OracleWorld(P.config_params(), sc)
    assert w.count_intersections() == 0
    rc, st = w.step(5)
    assert rc == 0
    assert w.count_intersections() == 0
    assert st.newton_iters >= 5
