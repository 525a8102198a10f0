"""CPU restatement of the learned warm start (test infrastructure only).

The learned warm start has no counterpart in the reference (it is one of
this library's additions), so this module restates the library's own
definitions for the tests to check the CUDA path against:

- `features(...)`: the 48 per-body features (include/abd_b200.h, "Learned
  warm start"), from the candidate pairs within ABD_FEAT_RADIUS_DHAT * dhat
  and closest points by Ericson, Real-Time Collision Detection, 5.1.9
  (segment-segment) and 5.1.5 (point-triangle);
- `forward(...)`, `loss_grad(...)`: the network 48 -> 256 -> 256 -> 256 ->
  12 with GELU, BF16 rounding of weights and activations (round to nearest
  even) and FP32 accumulation, and the gradient of the mean-squared error
  with straight-through rounding, the same definitions the trainer uses.

Nothing in the product imports this module.
"""
import numpy as np
from scipy.special import erf

IN, H, OUT = 48, 256, 12
NPARAM = H * IN + H + 2 * (H * H + H) + OUT * H + OUT
FEAT_RADIUS_DHAT = 50.0


def bf16(x):
    """Round float32 to the nearest bfloat16 (ties to even), as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return r.view(np.float32).reshape(x.shape)


def unpack(p):
    p = np.asarray(p, dtype=np.float32)
    o = 0
    out = []
    for (n_out, n_in) in [(H, IN), (H, H), (H, H), (OUT, H)]:
        W = p[o:o + n_out * n_in].reshape(n_out, n_in); o += n_out * n_in
        b = p[o:o + n_out]; o += n_out
        out.append((W, b))
    assert o == NPARAM
    return out


def pack(layers):
    return np.concatenate([np.concatenate([W.ravel(), b.ravel()]) for W, b in layers]).astype(np.float32)


def init_params(seed=0):
    rng = np.random.default_rng(seed)
    layers = []
    for (n_out, n_in) in [(H, IN), (H, H), (H, H), (OUT, H)]:
        W = rng.normal(scale=np.sqrt(2.0 / n_in), size=(n_out, n_in)).astype(np.float32)
        layers.append((W, np.zeros(n_out, np.float32)))
    W4, b4 = layers[-1]
    layers[-1] = (W4 * 0.1, b4)
    return pack(layers)


def gelu(z):
    z64 = z.astype(np.float64)
    return (0.5 * z64 * (1.0 + erf(z64 / np.sqrt(2.0)))).astype(np.float32)


def gelu_grad(z):
    z64 = z.astype(np.float64)
    return (0.5 * (1.0 + erf(z64 / np.sqrt(2.0))) + z64 * np.exp(-0.5 * z64 * z64) / np.sqrt(2 * np.pi)).astype(np.float32)


def forward_normalised(p, xn, rounding=True):
    """Network on normalised inputs -> normalised outputs; returns (y, cache)."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))
    h = rnd(xn)
    cache = [h]
    for i, (W, b) in enumerate(unpack(p)):
        z = (h @ rnd(W).T + b).astype(np.float32)
        if i < 3:
            cache.append(z)
            h = rnd(gelu(z))
            cache.append(h)
        else:
            return z, cache


def forward(p, norm, x):
    """Raw features -> de-normalised outputs, as abd_mlp_forward."""
    norm = np.asarray(norm, dtype=np.float32)
    xn = ((np.asarray(x, np.float32) - norm[:IN]) / norm[IN:2 * IN]).astype(np.float32)
    y, _ = forward_normalised(p, xn)
    return y * norm[2 * IN + OUT:] + norm[2 * IN:2 * IN + OUT]


def loss_grad(p, xn, yn, rounding=True):
    """Mean-squared error over all outputs and its gradient (parameter blob)."""
    rnd = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float32))
    y, cache = forward_normalised(p, xn, rounding)
    n = len(xn)
    e = y - yn
    loss = float(np.sum(e.astype(np.float64) ** 2) / (n * OUT))
    dz = (2.0 * e / (n * OUT)).astype(np.float32)
    layers = unpack(p)
    hs = [cache[0], cache[2], cache[4], cache[6]]
    zs = [cache[1], cache[3], cache[5]]
    grads = [None] * 4
    for l in range(3, -1, -1):
        W, _ = layers[l]
        # the GPU trainer's backward GEMMs run on the tensor cores with BF16
        # operands and FP32 sums: dW = bf16(dZ)^T H, dH = bf16(dZ) bf16(W);
        # the bias gradient sums the FP32 dZ
        dzr = rnd(dz)
        grads[l] = (dzr.T @ hs[l], dz.sum(axis=0))
        if l > 0:
            dh = dzr @ rnd(W)
            dz = (dh * gelu_grad(zs[l - 1])).astype(np.float32)
    return loss, pack(grads)


# ------------------------------------------------------------------ features
def _closest_seg_seg(p1, q1, p2, q2):
    d1, d2, r = q1 - p1, q2 - p2, p1 - p2
    a, e, f = d1 @ d1, d2 @ d2, d2 @ r
    if a <= 0 and e <= 0:
        s = t = 0.0
    elif a <= 0:
        s, t = 0.0, np.clip(f / e, 0, 1)
    else:
        c = d1 @ r
        if e <= 0:
            t, s = 0.0, np.clip(-c / a, 0, 1)
        else:
            b = d1 @ d2
            den = a * e - b * b
            s = np.clip((b * f - c * e) / den, 0, 1) if den != 0 else 0.0
            t = (b * s + f) / e
            if t < 0:
                t, s = 0.0, np.clip(-c / a, 0, 1)
            elif t > 1:
                t, s = 1.0, np.clip((b - c) / a, 0, 1)
    return p1 + s * d1, p2 + t * d2


def _pt_region(p, a, b, c):
    ab, ac, ap = b - a, c - a, p - a
    d1, d2 = ab @ ap, ac @ ap
    if d1 <= 0 and d2 <= 0:
        return 0
    bp = p - b
    d3, d4 = ab @ bp, ac @ bp
    if d3 >= 0 and d4 <= d3:
        return 1
    vc = d1 * d4 - d3 * d2
    if vc <= 0 and d1 >= 0 and d3 <= 0:
        return 3
    cp = p - c
    d5, d6 = ab @ cp, ac @ cp
    if d6 >= 0 and d5 <= d6:
        return 2
    vb = d5 * d2 - d1 * d6
    if vb <= 0 and d2 >= 0 and d6 <= 0:
        return 5
    va = d3 * d6 - d5 * d4
    if va <= 0 and (d4 - d3) >= 0 and (d5 - d6) >= 0:
        return 4
    return 6


def _tri_closest(p, a, b, c):
    r = _pt_region(p, a, b, c)
    T = [a, b, c]
    if r <= 2:
        return T[r]
    if r <= 5:
        e0, e1 = T[r - 3], T[(r - 3 + 1) % 3]
        e = e1 - e0
        t = np.clip((p - e0) @ e / (e @ e), 0, 1) if e @ e > 0 else 0.0
        return e0 + t * e
    n = np.cross(b - a, c - a)
    return p - ((p - a) @ n / (n @ n)) * n


def features(state, x, vbody, mass, quads, kinds, planes, dt, gravity, dhat):
    """48 features per body.  `quads`/`kinds` are the candidate pairs within
    the feature radius as abd_get_pairs returns them (global vertex ids; PG
    entries carry (vertex, plane)), `x` the vertex positions."""
    nb = len(state)
    radius = FEAT_RADIUS_DHAT * dhat
    g = np.asarray(gravity, np.float64)
    recs = [[] for _ in range(nb)]
    for q, k in zip(quads, kinds):
        if k == 0:
            pa, pb = _closest_seg_seg(x[q[0]], x[q[1]], x[q[2]], x[q[3]])
            ba, bb = vbody[q[0]], vbody[q[2]]
        elif k == 1:
            pa = x[q[0]]
            pb = _tri_closest(pa, x[q[1]], x[q[2]], x[q[3]])
            ba, bb = vbody[q[0]], vbody[q[1]]
        else:
            pl = planes[q[1]]
            pa = x[q[0]]
            d = pl[:3] @ pa - pl[3]
            pb = pa - d * pl[:3]
            ba, bb = vbody[q[0]], -1
        dv = pa - pb
        d = float(np.sqrt(dv @ dv))
        n = dv / d if d > 0 else np.zeros(3)
        if k == 2:
            n = np.asarray(planes[q[1]][:3], np.float64)
        df = np.float32(d)
        if mass[ba] > 0:
            recs[ba].append((df, n))
        if bb >= 0 and mass[bb] > 0:
            recs[bb].append((df, -n))
    F = np.zeros((nb, 48), np.float32)
    gn = np.linalg.norm(g)
    gd = g / gn if gn > 0 else np.zeros(3)
    for b in range(nb):
        if not mass[b] > 0:
            continue
        s = state[b]
        qm = s[3:12].reshape(3, 3)
        v, qd = s[12:15], s[15:24].reshape(3, 3)
        F[b, 0:3] = qm @ (v + dt * g)
        F[b, 3:12] = (qm @ qd.T).ravel()
        F[b, 12:15] = qm @ gd
        F[b, 15] = np.log1p(np.float32(len(recs[b])))
        order = sorted(range(len(recs[b])), key=lambda i: (recs[b][i][0], i))
        for k in range(8):
            if k < len(order):
                d, n = recs[b][order[k]]
                F[b, 16 + 4 * k] = d / radius
                F[b, 17 + 4 * k:20 + 4 * k] = qm @ n
            else:
                F[b, 16 + 4 * k] = 1.0
    return F
