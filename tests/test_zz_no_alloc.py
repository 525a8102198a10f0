"""abd_ee_pairs_static: edge-edge candidate pairs without any device
allocation, for callers that cannot call cudaMalloc when they need the
pairs (their host owns device memory through its own pool, or forbids
allocation after start-up).  The caller passes device buffers; all scratch
lives in static device arrays of the library.

Checked against the handle-based entry point (abd_get_pairs) on the
reference chain scene at several states, on two calls in a row, so the
second call also proves that the shared static scratch is cleared between
calls.  Pair sets are integer data: they must match exactly.  This file is
collected last so that a stop-at-first-failure run has already run every
other test."""
import ctypes as C

import numpy as np
import pytest

from colb_b200 import params as P
from colb_b200.engine import Engine, load_library

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_static_pairs_match_handle_pairs(chain_scene, chain_pairs):
    import torch
    L = load_library()
    e = Engine(P.reference_params(), chain_scene)
    edges = torch.from_numpy(np.ascontiguousarray(chain_scene["edges"], dtype=np.int32)).cuda()
    nv, ne = len(chain_scene["xbar"]), len(chain_scene["edges"])
    cap = 8192
    out = torch.full((cap, 4), -7, dtype=torch.int32, device="cuda")
    n_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
    cand = P.REFERENCE["cand_dist"]
    for k in (2, 0, 1):          # the largest set first, so the smaller ones follow stale contents
        e.set_state(chain_pairs["states"][k])
        want, _ = e.pairs()
        x = torch.from_numpy(e.vertices()).cuda()
        for call in range(2):
            rc = L.abd_ee_pairs_static(_ptr(x), _ptr(edges), nv, ne, cand, _ptr(out), cap, _ptr(n_dev), None)
            assert rc == 0, L.abd_last_error(None)
            n = int(n_dev.item())
            got = out[:n].cpu().numpy()
            assert n == len(want), (k, call, n, len(want))
            assert np.array_equal(got, want), (k, call)


def test_static_pairs_reject_oversize_and_bad_edges():
    import torch
    L = load_library()
    x = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    edges = torch.tensor([[0, 1], [2, 9]], dtype=torch.int32, device="cuda")
    out = torch.zeros((4, 4), dtype=torch.int32, device="cuda")
    n_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
    too_many = (1 << 16) + 1
    assert L.abd_ee_pairs_static(_ptr(x), _ptr(edges), 4, too_many, 0.1, _ptr(out), 4, _ptr(n_dev), None) == -1
    assert b"n_edges" in L.abd_last_error(None)
    assert L.abd_ee_pairs_static(_ptr(x), _ptr(edges), 4, 2, 0.1, _ptr(out), 4, _ptr(n_dev), None) == -1
    assert b"edge index" in L.abd_last_error(None)


def test_static_pairs_overflow_reports_full_count(chain_scene, chain_pairs):
    """A cap below the pair count: ABD_ERR_CONTACT_OVERFLOW, the complete
    count in *n_pairs_dev, and nothing written at or beyond row cap."""
    import torch
    L = load_library()
    e = Engine(P.reference_params(), chain_scene)
    e.set_state(chain_pairs["states"][2])
    want, _ = e.pairs()
    x = torch.from_numpy(e.vertices()).cuda()
    edges = torch.from_numpy(np.ascontiguousarray(chain_scene["edges"], dtype=np.int32)).cuda()
    nv, ne = len(chain_scene["xbar"]), len(chain_scene["edges"])
    cap = 3
    out = torch.full((64, 4), -7, dtype=torch.int32, device="cuda")
    n_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.abd_ee_pairs_static(_ptr(x), _ptr(edges), nv, ne, P.REFERENCE["cand_dist"], _ptr(out), cap, _ptr(n_dev), None)
    assert rc == -3, L.abd_last_error(None)
    assert int(n_dev.item()) == len(want) > cap
    rows = out.cpu().numpy()
    assert np.all(rows[cap:] == -7)
    # the rows below cap are valid candidate quadruples of the full set
    assert {tuple(r) for r in rows[:cap]} <= {tuple(r) for r in want}


def test_static_pairs_accept_the_maximum_size():
    """ABD_STATIC_MAX_EDGES edges fit the static scratch (sort and scan
    included): 65,536 disjoint unit segments on a line, 0.5 apart, give
    exactly the pairs of neighbours closer than the candidate distance."""
    import torch
    L = load_library()
    ne = 1 << 16
    xs = np.zeros((2 * ne, 3))
    xs[0::2, 0] = np.arange(ne) * 1.5
    xs[1::2, 0] = np.arange(ne) * 1.5 + 1.0
    edges = np.arange(2 * ne, dtype=np.int32).reshape(ne, 2)
    x = torch.from_numpy(xs).cuda()
    ed = torch.from_numpy(edges).cuda()
    cap = 2 * ne
    out = torch.full((cap, 4), -7, dtype=torch.int32, device="cuda")
    n_dev = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.abd_ee_pairs_static(_ptr(x), _ptr(ed), 2 * ne, ne, 0.6, _ptr(out), cap, _ptr(n_dev), None)
    assert rc == 0, L.abd_last_error(None)
    n = int(n_dev.item())
    assert n == ne - 1
    got = out[:n].cpu().numpy()
    want = np.stack([edges[:-1, 0], edges[:-1, 1], edges[1:, 0], edges[1:, 1]], axis=1)
    assert np.array_equal(got, want)
