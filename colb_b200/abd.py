"""`NewtonAbd` — drop-in for the reference's solver class.

Mirrors the Python surface of `NewtonAbd` in abd.py:583-757 of
Luke-Skycrawler/colb (driven by viewer.py:44-47): construct with a time step
and a scene, call `step()` once per frame, read `history`, `compute_V()`,
`get_contact_points()`, `frame`, `profiler`.  The work runs in
libabd_b200.so on the GPU; there is no CPU path.

Differences from the reference, all deliberate:
  * the Hessian is assembled without the contact/inertia triplet overlap
    of abd.py:111 vs abd.py:311-334 (contacts at list index i overwrote the
    inertia blocks of bodies 4i..4i+3);
  * the contact list is sorted and grows on demand instead of wrapping at
    10000 entries (contact.py:8, :137);
  * the linear solve (ABD_SOLVER_AUTO) is a direct solve per connected
    component of the contact graph (banded block Cholesky, shared-memory
    dense factorization, or block-Jacobi preconditioned BiCGSTAB / PCG when
    the components are too large), not Warp's unpreconditioned bicgstab;
    the reference's own solver_config="cg" choice maps to
    ABD_SOLVER_BICGSTAB, which stops at the same relative tolerance.
"""
import json
import os
import numpy as np

from . import scene as _scene
from .engine import Engine
from ._abi import ABD_ERR_CCD_CAP, ABD_ERR_NEWTON_CAP, ABD_ERR_SOLVER_CAP
from .params import reference_params

# numpy view of the BDFAffine struct (BDF1.py:11-14, quat_util.py:40-47)
AFFINE_STATE = np.dtype([("c", "<f8", (3,)), ("q", "<f8", (3, 3)), ("v", "<f8", (3,)), ("qdot", "<f8", (3, 3))])
BDF_AFFINE = np.dtype([("now", AFFINE_STATE), ("nxt", AFFINE_STATE)])


class Profiller:
    """Per-(frame, iteration) residual and step length, like
    utils/data_collector.py:4-55 (same attribute names and npz keys)."""

    def __init__(self, max_iters, frames=4000):
        self.convergence = np.zeros((frames, max_iters))
        self.alphas = np.zeros_like(self.convergence)

    def recorded_attributes(self):
        return {"convergence": float, "alphas": float}

    def save(self, filename):
        np.savez(filename, **{k: getattr(self, k) for k in self.recorded_attributes()})

    def load(self, filename):
        d = np.load(filename)
        for k in self.recorded_attributes():
            if k in d:
                setattr(self, k, d[k])


class Soup:
    """Host view of the concatenated geometry (geometry.py:22-28)."""

    def __init__(self, sc):
        self.xcs = sc["xbar"]
        self.triangles = sc["tris"].reshape(-1)
        self.edges = sc["edges"].reshape(-1)
        self.body = sc["vert_body"]


class NewtonAbd:
    """NewtonAbd(h, config_file) as in abd.py:584.  `config_file` may be a
    reference JSON scene (e.g. assets/chains.json), an .npz scene written by
    colb_b200.scene.save_npz_scene, or a scene dict.  The profiler records
    `frames` frames of at most newton_max_iter iterations, like the
    reference's Profiller(max_iters=16, frames=50) (abd.py:599)."""

    def __init__(self, h, config_file, params=None, device=0, frames=50):
        if isinstance(config_file, dict):
            sc = config_file
        elif str(config_file).endswith(".npz"):
            sc = _scene.load_npz_scene(config_file)
        else:
            sc = _scene.load_json_scene(config_file)
        self.scene = sc
        p = params if params is not None else reference_params()
        p.dt = h
        self.params = p
        self.dt = h
        self.n_bodies = len(sc["mass"])
        self.n_nodes = len(sc["xbar"])
        self.soup = Soup(sc)
        self.E = sc["edges"]
        self.F = sc["tris"]
        self.V0 = sc["xbar"]
        self.engine = Engine(p, sc, device=device)
        self._initial_state = sc["state"].copy()
        self.frame = 0
        self.profiler = Profiller(max_iters=p.newton_max_iter, frames=frames)
        self.last_stats = None
        self.last_rc = 0
        self.V = self.compute_V()

    # abd_simple.py:64-69
    def reset(self):
        self.engine.set_state(self._initial_state)
        self.frame = 0
        self.compute_V()

    @property
    def history(self):
        """BDFAffine array (numpy structured copy of the device state)."""
        return self.engine.get_state().view(BDF_AFFINE).reshape(self.n_bodies)

    @history.setter
    def history(self, value):
        arr = np.ascontiguousarray(value)
        if arr.dtype == BDF_AFFINE:
            arr = arr.view(np.float64)
        self.engine.set_state(np.asarray(arr, dtype=np.float64).reshape(self.n_bodies, 48))

    # abd.py:674-702
    def step(self):
        # a Krylov, Newton or CCD iteration cap ends the step with the iterate
        # reached, as the reference's loop does (abd.py:699); the status is
        # kept in last_rc
        rc, st = self.engine.step(1, allow=(ABD_ERR_SOLVER_CAP, ABD_ERR_NEWTON_CAP, ABD_ERR_CCD_CAP))
        self.last_rc = rc
        self.last_stats = st
        res, alpha, ips = self.engine.profile(0)
        n = min(len(res), self.profiler.convergence.shape[1])
        if self.frame < self.profiler.convergence.shape[0]:
            self.profiler.convergence[self.frame, :n] = res[:n]
            self.profiler.alphas[self.frame, :n] = alpha[:n]
        self.frame += 1
        return st

    # abd_simple.py:71-78
    def compute_V(self, ret=True):
        V = self.engine.vertices()
        self.V = V
        return V if ret else None

    # abd.py:748-757
    def get_contact_points(self):
        pts, d = self.engine.contact_points()
        l0 = self.params.dhat
        valid = d < l0
        return pts[valid], np.abs(d[valid] - l0)

    def detect_collision(self):
        pairs, kinds = self.engine.pairs()
        self.n_contacts = len(pairs)
        return pairs

    def compute_g(self):
        return float(self.engine.energy()[0])
