"""Scene construction (host logic, no GPU)."""
import numpy as np
import pytest

from colb_b200 import scene as S


def test_euler_matches_composition():
    R = S.euler_xyz_deg([90.0, 0.0, 90.0])
    assert np.allclose(R @ R.T, np.eye(3))
    # extrinsic x then z: e_x -> e_x (Rx) -> e_y (Rz)
    assert np.allclose(R @ [1, 0, 0], [0, 1, 0], atol=1e-12)


def test_chain_scene_fixture(chain_scene):
    sc = chain_scene
    assert len(sc["mass"]) == 144 and len(sc["xbar"]) == 3168 and len(sc["edges"]) == 3168
    assert (sc["mass"] <= 0).sum() == 24
    assert np.allclose(sc["inertia_J"][sc["mass"] > 0], 0.4 * 1.0 * 0.16)
    qd = sc["state"][0, 15:24].reshape(3, 3)
    assert np.allclose(qd, S.skew([3.0, 3.0, 0.0]))


def test_mass_properties():
    V, F = S.cube_mesh(1.0)
    m, c, Sm = S.mass_properties(V, F, 1000.0)
    assert m == pytest.approx(1000.0) and np.allclose(c, 0)
    assert np.allclose(Sm, np.eye(3) * 1000.0 / 12.0)
    V, F = S.torus_mesh(1.0, 0.25, 96, 48)
    m, c, _ = S.mass_properties(V, F, 1.0)
    assert m == pytest.approx(2 * np.pi ** 2 * 1.0 * 0.25 ** 2, rel=5e-3)


def test_meshes_closed_and_oriented():
    for V, F in (S.cube_mesh(), S.torus_mesh(), S.icosphere_mesh(1), S.icosphere_mesh(2)):
        E = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
        # every directed edge appears once and its reverse once
        fw = set(map(tuple, E)); bw = set(map(tuple, E[:, ::-1]))
        assert fw == bw and len(fw) == len(E)
        assert S.mass_properties(V, F, 1.0)[0] > 0


def test_config_sizes():
    c1 = S.config1_cubes()
    assert len(c1["mass"]) == 8 and len(c1["xbar"]) == 64 and len(c1["tris"]) == 96
    c2 = S.config2_chain_net(n=4)
    assert len(c2["mass"]) == 16 and len(c2["xbar"]) == 16 * 288 and len(c2["tris"]) == 16 * 576
    assert (c2["mass"] <= 0).sum() == 4
    b = S.config3_batch(n_scenes=20)
    nbs = [len(s["mass"]) for s in b]
    assert min(nbs) >= 4 and max(nbs) <= 64


def test_pile_config_and_fixture():
    """4096 icospheres (42 or 162 vertices, radius 0.2..0.5) inside the
    12 x 12 open box with ground and four walls, no two overlapping at t = 0;
    the stored benchmark state has the scene's shape and stays in the box."""
    from colb_b200 import fixtures
    sc = S.config5_pile()
    nb = len(sc["mass"])
    assert nb == 4096 and len(sc["planes"]) == 5
    counts = np.bincount(sc["vert_body"], minlength=nb)
    assert set(np.unique(counts)) <= {42, 162}
    c = sc["state"][:, :3]
    r = np.array([np.linalg.norm(sc["xbar"][sc["vert_body"] == b], axis=1).max() for b in range(0, nb, 97)])
    assert r.min() >= 0.2 - 1e-9 and r.max() <= 0.5 + 1e-9
    assert c[:, 0].min() > 0.0 and c[:, 0].max() < 12.0 and c[:, 2].min() > 0.0 and c[:, 2].max() < 12.0
    # neighbours on the 1.05 grid: centre distance exceeds the sum of the radii
    d = np.linalg.norm(c[1] - c[0])
    assert d > 1.0
    state, t0, seed = fixtures.load_pile()
    assert state.shape == (nb, 48) and np.isfinite(state).all() and t0 == 100 and seed == 0
    cn = state[:, 24:27]
    assert cn[:, 1].min() > 0.0 and cn[:, 0].min() > 0.0 and cn[:, 0].max() < 12.0


def test_load_ma_roundtrip(tmp_path):
    p = tmp_path / "t.ma"
    p.write_text("3 2 1\nv 0 0 0 0.1\nv 1 0 0 0.1\nv 0 1 0 0.1\ne 0 1\ne 1 2\nf 0 1 2\n")
    V, E, F, R = S.load_ma(str(p))
    assert V.shape == (3, 3) and F.shape == (1, 3)
    assert sorted(map(tuple, E)) == [(0, 1), (0, 2), (1, 2)]
