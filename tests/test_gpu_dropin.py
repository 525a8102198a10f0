"""The Python drop-in class `colb_b200.abd.NewtonAbd` (needs a GPU).

It mirrors the attributes the reference's driver uses (viewer.py:44-47 with
abd.py:583-599, :674-702, :748-757 and utils/data_collector.py:4-55):
construct with a time step and a scene, `step()`, `history` (a BDFAffine
structured array), `compute_V()`, `get_contact_points()`, `reset()`,
`frame` and the `profiler` npz.  Trajectories are compared with the CPU
oracle at the FP64 tolerance, 1e-6 of the scene extent.
"""
import os

import numpy as np
import pytest

from oracle import oracle as O
from colb_b200 import params as P
from colb_b200.abd import BDF_AFFINE, NewtonAbd, Profiller

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CHAIN = os.path.join(GOLDEN, "chains_scene.npz")


def test_newton_abd_steps_like_the_oracle(chain_scene):
    h = 8e-3
    sim = NewtonAbd(h, CHAIN, params=P.reference_params(lin_tol=1e-10))
    o = O.OracleWorld(P.reference_params(lin_tol=1e-10, dt=h), chain_scene)
    assert sim.n_bodies == len(chain_scene["mass"]) and sim.frame == 0
    hist0 = sim.history
    assert hist0.dtype == BDF_AFFINE and hist0.shape == (sim.n_bodies,)
    assert np.array_equal(hist0.view(np.float64).reshape(sim.n_bodies, 48), chain_scene["state"])
    for f in range(3):
        st = sim.step()
        o.step(1)
        assert sim.frame == f + 1
        V = sim.compute_V()
        assert V.shape == (len(chain_scene["xbar"]), 3)
        xo = o.vertices()
        assert np.abs(V - xo).max() <= 1e-6 * np.abs(xo).max()
        # the profiler row of this frame: one residual per Newton iteration,
        # the last below the tolerance (abd.py:695-699)
        row = sim.profiler.convergence[f]
        n = st.newton_iters
        assert n >= 1 and np.all(row[:n] > 0) and np.all(row[n:] == 0)
        assert row[n - 1] < 1e-5
        assert np.all(sim.profiler.alphas[f, :n] > 0)
    # history.nxt after forward_states equals now (abd.py:574-581)
    hist = sim.history
    assert np.array_equal(hist["now"]["c"], hist["nxt"]["c"])
    assert np.abs(hist["nxt"]["c"] - o.get_state()[:, 24:27]).max() <= 1e-6 * np.abs(xo).max()


def test_newton_abd_contact_points_reset_and_profiler_file(chain_scene, chain_pairs, tmp_path):
    sim = NewtonAbd(8e-3, dict(chain_scene))
    st = np.asarray(chain_pairs["states"][2], dtype=np.float64)
    sim.history = st.view(BDF_AFFINE).reshape(sim.n_bodies)
    assert np.array_equal(sim.history.view(np.float64).reshape(-1, 48), st)
    pts, mag = sim.get_contact_points()
    # abd.py:748-757: EE closest-point midpoints of the pairs closer than
    # 2 * thickness, with magnitude |d - 2 thickness|
    assert pts.ndim == 2 and pts.shape[1] == 3 and len(pts) == len(mag) > 0
    assert np.all(mag >= 0) and np.all(mag <= P.REFERENCE["dhat"])
    pairs = sim.detect_collision()
    assert sim.n_contacts == len(pairs) == len(chain_pairs["pairs2"])
    sim.step()
    path = os.path.join(tmp_path, "profiler.npz")
    sim.profiler.save(path)
    d = np.load(path)
    assert set(d.files) == {"convergence", "alphas"}
    assert d["convergence"].shape == (50, 16)      # Profiller(max_iters=16, frames=50), abd.py:599
    back = Profiller(16, 50)
    back.load(path)
    assert np.array_equal(back.convergence, sim.profiler.convergence)
    sim.reset()
    assert sim.frame == 0
    assert np.array_equal(sim.history.view(np.float64).reshape(-1, 48), chain_scene["state"])
    assert sim.compute_g() > 0
