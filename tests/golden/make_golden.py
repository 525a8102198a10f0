"""Generates the committed fixtures in tests/golden from the reference's own
assets.  Run in a checkout where the reference (Luke-Skycrawler/colb) is
mounted; the GPU-side tests only read the .npz files written here.

Usage: COLB_REFERENCE=<reference checkout> python tests/golden/make_golden.py

  chains_scene.npz   assets/chains.json + assets/link.ma of the reference,
                     loaded the way utils/scene.py:55-85 and medial.py:17-51
                     do (rest vertices rotated by the xyz Euler angles and
                     scaled by 2, mass/1000, J = 0.4 m 0.4^2,
                     qdot = skew(3,3,0)): 144 bodies, 3168 vertices / edges.
  chains_pairs.npz   the candidate edge-edge pair set of that scene at t = 0
                     and at two perturbed states, computed here by a
                     vectorised float32 numpy restatement of the reference's
                     predicate (contact.py:158-168: i < j, no shared vertex,
                     float32 segment distance < (0.0475+0.0475)*2), which is
                     independent of the C oracle it pins.
  segseg_cases.npz   random and degenerate float32 segment pairs (parallel,
                     touching, zero-length, endpoint-closest) with the numpy
                     restatement's (s, t, d).

The reference's Warp runtime is not installable here, so these fixtures
pin the restatement, not Warp's compiled closest_point_edge_edge.
"""
import os
import sys
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", ".."))
# the checkout of the reference whose assets/ the fixtures are built from;
# there is no default, so the script never reads a path it was not given
REF = os.environ.get("COLB_REFERENCE")


def seg_seg_f32(p1, q1, p2, q2, eps=np.float32(1e-6)):
    """Ericson §5.1.9 closest points, vectorised, every operation in
    float32 with one rounding (numpy float32 arithmetic)."""
    f = np.float32
    p1, q1, p2, q2 = [np.asarray(a, dtype=f) for a in (p1, q1, p2, q2)]

    def dot(a, b):
        return (a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1]) + a[..., 2] * b[..., 2]

    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, ff = dot(d1, d1), dot(d2, d2), dot(d2, r)
    c = dot(d1, r)
    b = dot(d1, d2)
    n = a.shape
    s = np.zeros(n, dtype=f)
    t = np.zeros(n, dtype=f)
    with np.errstate(divide="ignore", invalid="ignore"):
        both = (a <= eps) & (e <= eps)
        a_small = (a <= eps) & ~both
        e_small = (e <= eps) & ~(a <= eps)
        gen = ~(a <= eps) & ~(e <= eps)
        t = np.where(a_small, np.clip(ff / e, f(0), f(1)), t)
        s = np.where(e_small, np.clip(-c / a, f(0), f(1)), s)
        denom = a * e - b * b
        sg = np.where(denom != 0, np.clip((b * ff - c * e) / denom, f(0), f(1)), f(0)).astype(f)
        tg = ((b * sg + ff) / e).astype(f)
        lo, hi = tg < 0, tg > 1
        sg = np.where(lo, np.clip(-c / a, f(0), f(1)), np.where(hi, np.clip((b - c) / a, f(0), f(1)), sg)).astype(f)
        tg = np.where(lo, f(0), np.where(hi, f(1), tg)).astype(f)
        s = np.where(gen, sg, s).astype(f)
        t = np.where(gen, tg, t).astype(f)
    dv = (p1 + d1 * s[..., None]) - (p2 + d2 * t[..., None])
    return s, t, np.sqrt(dot(dv, dv)).astype(f)


def pair_set(x, edges, cand=(0.0475 + 0.0475) * 2.0):
    xf = x.astype(np.float32)
    ne = len(edges)
    out = []
    thr = np.float32(cand)
    for i in range(ne - 1):
        j = np.arange(i + 1, ne)
        a, b = edges[i], edges[j]
        conn = (a[0] == b[:, 0]) | (a[0] == b[:, 1]) | (a[1] == b[:, 0]) | (a[1] == b[:, 1])
        j, b = j[~conn], b[~conn]
        if len(j) == 0:
            continue
        p1 = np.broadcast_to(xf[a[0]], (len(j), 3))
        q1 = np.broadcast_to(xf[a[1]], (len(j), 3))
        _, _, d = seg_seg_f32(p1, q1, xf[b[:, 0]], xf[b[:, 1]])
        keep = d < thr
        out += [(i, jj) for jj in j[keep]]
    return np.array(out, dtype=np.int32).reshape(-1, 2)


def main():
    from colb_b200 import scene as S
    sc = S.load_json_scene(os.path.join(REF, "assets", "chains.json"), root=REF)
    S.save_npz_scene(os.path.join(HERE, "chains_scene.npz"), sc)
    rng = np.random.default_rng(0)
    states, sets = [], []
    for k in range(3):
        st = sc["state"].copy()
        if k > 0:
            # rigid-ish perturbation of the nxt state: small translations and
            # affine noise so that new pairs come within the filter distance
            nb = len(st)
            st[:, 24:27] += rng.normal(scale=0.08 * k, size=(nb, 3))
            st[:, 27:36] += rng.normal(scale=0.02 * k, size=(nb, 9))
        x = S.transform(sc, st)
        states.append(st)
        sets.append(pair_set(x, sc["edges"]))
    np.savez_compressed(os.path.join(HERE, "chains_pairs.npz"), states=np.array(states),
                        **{f"pairs{k}": p for k, p in enumerate(sets)})
    # segment cases
    n = 4000
    P = rng.normal(size=(n, 4, 3)).astype(np.float32)
    # degenerate families
    P[:500, 1] = P[:500, 0]                                      # zero-length first segment
    P[500:1000, 3] = P[500:1000, 2]                              # zero-length second
    P[1000:1500, 3] = P[1000:1500, 2] + (P[1000:1500, 1] - P[1000:1500, 0])   # parallel
    P[1500:2000, 2] = P[1500:2000, 1]                            # touching at an endpoint
    P[2000:2500, 2:] = P[2000:2500, :2] + np.float32(1e-3)       # nearly coincident
    P[2500:3000] *= np.float32(1e-3)                             # tiny scale
    s, t, d = seg_seg_f32(P[:, 0], P[:, 1], P[:, 2], P[:, 3])
    np.savez_compressed(os.path.join(HERE, "segseg_cases.npz"), pts=P, s=s, t=t, d=d)
    print("pairs:", [len(p) for p in sets])


if __name__ == "__main__":
    if not REF:
        sys.exit("set COLB_REFERENCE to the reference checkout (the directory holding assets/chains.json)")
    main()
