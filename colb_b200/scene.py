"""Scene construction.

Two sources of scenes:

* The reference's own scene format (utils/scene.py:8-85, medial.py:17-51 of
  Luke-Skycrawler/colb): a JSON list of objects {obj, p, euler, mass, ...}
  whose meshes are `.ma` medial meshes.  Rest vertices are
  V_file @ R_euler('xyz', degrees).T * 2 (utils/scene.py:75-85), masses are
  json_mass / 1000 with J = 0.4 m 0.4^2 (abd_simple.py:18-22,
  rbd_simple.py:42-48), and every body starts at c = p, q = I, v = 0,
  qdot = skew(3, 3, 0) (abd_simple.py:37-49).

* Seeded synthetic scenes of closed triangle meshes (cubes, tori,
  icospheres) for the benchmark workloads.  Their mass is density x volume
  and J is one third of the trace of the second-moment matrix about the
  centroid (the reference's scalar-J mass model M = diag(m, J, J, J)).

A scene is a dict of numpy arrays: xbar (nv,3), vert_body (nv,), edges
(ne,2), tris (nt,3), mass (nb,), inertia_J (nb,), state (nb,48), planes
(np,4).
"""
import json
import os
import numpy as np

ST_NOW, ST_NXT, ST_C, ST_Q, ST_V, ST_QD = 0, 24, 0, 3, 12, 15


# --------------------------------------------------------------------------
# state helpers (BDFAffine layout, BDF1.py:11-14 / quat_util.py:40-47)
# --------------------------------------------------------------------------
def skew(v):
    """wp.skew: [a]x with [a]x b = a x b."""
    return np.array([[0.0, -v[2], v[1]], [v[2], 0.0, -v[0]], [-v[1], v[0], 0.0]])


def make_state(c, q=None, v=None, qdot=None):
    """(nb,48) BDFAffine array with now == nxt."""
    c = np.asarray(c, dtype=np.float64).reshape(-1, 3)
    nb = len(c)
    st = np.zeros((nb, 48))
    qq = np.tile(np.eye(3), (nb, 1, 1)) if q is None else np.asarray(q, dtype=np.float64).reshape(nb, 3, 3)
    vv = np.zeros((nb, 3)) if v is None else np.asarray(v, dtype=np.float64).reshape(nb, 3)
    qd = np.zeros((nb, 3, 3)) if qdot is None else np.asarray(qdot, dtype=np.float64).reshape(nb, 3, 3)
    for base in (ST_NOW, ST_NXT):
        st[:, base + ST_C:base + ST_C + 3] = c
        st[:, base + ST_Q:base + ST_Q + 9] = qq.reshape(nb, 9)
        st[:, base + ST_V:base + ST_V + 3] = vv
        st[:, base + ST_QD:base + ST_QD + 9] = qd.reshape(nb, 9)
    return st


def transform(scene, state=None):
    """x = q^T xbar + c of the nxt state (abd_simple.py:26-35)."""
    st = scene["state"] if state is None else state
    b = scene["vert_body"]
    q = st[b, ST_NXT + ST_Q:ST_NXT + ST_Q + 9].reshape(-1, 3, 3)
    c = st[b, ST_NXT + ST_C:ST_NXT + ST_C + 3]
    return np.einsum("vrk,vr->vk", q, scene["xbar"]) + c


# --------------------------------------------------------------------------
# reference scene format
# --------------------------------------------------------------------------
def euler_xyz_deg(angles):
    """scipy Rotation.from_euler('xyz', angles, degrees=True).as_matrix():
    extrinsic rotations about x, then y, then z."""
    ax, ay, az = np.radians(np.asarray(angles, dtype=np.float64))
    cx, sx, cy, sy, cz, sz = np.cos(ax), np.sin(ax), np.cos(ay), np.sin(ay), np.cos(az), np.sin(az)
    Rx = np.array([[1, 0, 0], [0, cx, -sx], [0, sx, cx]])
    Ry = np.array([[cy, 0, sy], [0, 1, 0], [-sy, 0, cy]])
    Rz = np.array([[cz, -sz, 0], [sz, cz, 0], [0, 0, 1]])
    return Rz @ Ry @ Rx


def triangle_edges(F):
    """Unique undirected edges of a triangle list, each row sorted."""
    F = np.asarray(F, dtype=np.int64).reshape(-1, 3)
    if len(F) == 0:
        return np.zeros((0, 2), dtype=np.int64)
    E = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    return np.unique(np.sort(E, axis=1), axis=0)


def load_ma(path):
    """`.ma` medial mesh (medial.py:17-51): 'v x y z r', 'e i j', 'f i j k'
    lines; the edge set is the union of the listed edges and the triangle
    edges, each sorted, unique."""
    V, E0, F = [], [], []
    with open(path) as f:
        for line in f:
            p = line.split()
            if not p:
                continue
            if p[0] == "v":
                V.append([float(t) for t in p[1:]])
            elif p[0] == "e":
                E0.append([int(t) for t in p[1:]])
            elif p[0] == "f":
                F.append([int(t) for t in p[1:]])
    V = np.array(V, dtype=np.float64)
    F = np.array(F, dtype=np.int64).reshape(-1, 3)
    E = np.concatenate([np.array(E0, dtype=np.int64).reshape(-1, 2), triangle_edges(F)])
    E = np.unique(np.sort(E, axis=1), axis=0)
    return V[:, :3], E, F, V[:, 3] if V.shape[1] > 3 else None


def scene_from_objects(objects, mesh_loader):
    """Concatenate reference-format objects (geometry.py:31-73)."""
    xs, bs, es, fs, ps, ms = [], [], [], [], [], []
    nv = 0
    for bi, obj in enumerate(objects):
        V, E, F = mesh_loader(obj["obj"])
        R = euler_xyz_deg(obj.get("euler", [0.0, 0.0, 0.0]))
        v = V @ R.T * 2  # utils/scene.py:83
        xs.append(v)
        bs.append(np.full(len(v), bi))
        es.append(E + nv)
        fs.append(F + nv)
        ps.append(obj.get("p", [0.0, 0.0, 0.0]))
        ms.append(obj.get("mass", 1.0))
        nv += len(v)
    m = np.array(ms, dtype=np.float64) / 1000.0          # abd_simple.py:18-22
    J = 0.4 * m * 0.4 * 0.4                             # rbd_simple.py:42-48
    st = make_state(np.array(ps, dtype=np.float64),
                    qdot=np.tile(skew([3.0, 3.0, 0.0]), (len(objects), 1, 1)))  # abd_simple.py:37-49
    return dict(xbar=np.concatenate(xs), vert_body=np.concatenate(bs).astype(np.int32),
                edges=np.concatenate(es).astype(np.int32), tris=np.concatenate(fs).astype(np.int32).reshape(-1, 3),
                mass=m, inertia_J=J, state=st, planes=np.zeros((0, 4)))


def load_json_scene(path, root=None):
    """A reference scene file such as assets/chains.json; mesh paths in it
    are resolved against `root` (default: the directory above the JSON)."""
    root = root or os.path.dirname(os.path.dirname(os.path.abspath(path)))
    with open(path) as f:
        objects = json.load(f)
    cache = {}

    def loader(rel):
        if rel not in cache:
            full = rel if os.path.isabs(rel) else os.path.join(root, rel)
            if not full.endswith(".ma"):
                raise ValueError(f"only .ma meshes are read here: {rel}")
            V, E, F, _ = load_ma(full)
            cache[rel] = (V, E, F)
        return cache[rel]

    return scene_from_objects(objects, loader)


def load_npz_scene(path):
    d = np.load(path)
    return {k: d[k] for k in d.files}


def save_npz_scene(path, scene):
    np.savez_compressed(path, **scene)


# --------------------------------------------------------------------------
# synthetic meshes
# --------------------------------------------------------------------------
def cube_mesh(size=1.0):
    h = 0.5 * size
    V = np.array([[x, y, z] for x in (-h, h) for y in (-h, h) for z in (-h, h)], dtype=np.float64)
    # outward-oriented triangles
    F = np.array([
        [0, 1, 3], [0, 3, 2],   # x = -h
        [4, 6, 7], [4, 7, 5],   # x = +h
        [0, 4, 5], [0, 5, 1],   # y = -h
        [2, 3, 7], [2, 7, 6],   # y = +h
        [0, 2, 6], [0, 6, 4],   # z = -h
        [1, 5, 7], [1, 7, 3],   # z = +h
    ], dtype=np.int64)
    return V, F


def torus_mesh(R=1.0, r=0.25, nu=24, nv=12):
    """Torus around the z axis (ring in the xy plane)."""
    u = 2 * np.pi * np.arange(nu) / nu
    v = 2 * np.pi * np.arange(nv) / nv
    U, W = np.meshgrid(u, v, indexing="ij")
    X = (R + r * np.cos(W)) * np.cos(U)
    Y = (R + r * np.cos(W)) * np.sin(U)
    Z = r * np.sin(W)
    V = np.stack([X, Y, Z], -1).reshape(-1, 3)
    F = []
    for i in range(nu):
        for j in range(nv):
            a = i * nv + j
            b = ((i + 1) % nu) * nv + j
            c = ((i + 1) % nu) * nv + (j + 1) % nv
            d = i * nv + (j + 1) % nv
            F += [[a, b, c], [a, c, d]]
    return V, np.array(F, dtype=np.int64)


def icosphere_mesh(subdiv=1, radius=1.0):
    t = (1.0 + 5 ** 0.5) / 2.0
    V = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    F = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5],
         [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    V = [np.array(v, dtype=np.float64) / np.linalg.norm(v) for v in V]
    for _ in range(subdiv):
        mid = {}
        nF = []

        def m(a, b):
            key = (min(a, b), max(a, b))
            if key not in mid:
                p = V[a] + V[b]
                V.append(p / np.linalg.norm(p))
                mid[key] = len(V) - 1
            return mid[key]

        for a, b, c in F:
            ab, bc, ca = m(a, b), m(b, c), m(c, a)
            nF += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        F = nF
    return np.array(V) * radius, np.array(F, dtype=np.int64)


def mass_properties(V, F, density):
    """Volume, centroid and second moments of a closed, outward-oriented
    triangle mesh by the divergence theorem (signed tetrahedra from the
    origin)."""
    a, b, c = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    det = np.einsum("ij,ij->i", a, np.cross(b, c))
    vol = det.sum() / 6.0
    cen = ((a + b + c) * det[:, None]).sum(0) / (24.0 * vol)
    # second moment of each tet (0, a, b, c): det/120 * (sum_i x_i x_i^T + (sum x)(sum x)^T)
    s = a + b + c
    S = (np.einsum("t,ti,tj->ij", det, a, a) + np.einsum("t,ti,tj->ij", det, b, b)
         + np.einsum("t,ti,tj->ij", det, c, c) + np.einsum("t,ti,tj->ij", det, s, s)) / 120.0
    S = S - vol * np.outer(cen, cen)
    m = density * vol
    return m, cen, density * S


def _rand_rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def assemble_bodies(bodies, planes=None):
    """bodies: list of dict(V (body frame, centroid at 0), F, c, v, mass, J, pinned)."""
    xs, bs, es, fs = [], [], [], []
    nv = 0
    ms, Js, cs, vs = [], [], [], []
    for bi, b in enumerate(bodies):
        V, F = b["V"], b["F"]
        xs.append(V)
        bs.append(np.full(len(V), bi))
        es.append(triangle_edges(F) + nv)
        fs.append(F + nv)
        nv += len(V)
        ms.append(-abs(b["mass"]) if b.get("pinned") else b["mass"])
        Js.append(b["J"])
        cs.append(b["c"])
        vs.append(b.get("v", np.zeros(3)))
    st = make_state(np.array(cs), v=np.array(vs))
    return dict(xbar=np.concatenate(xs), vert_body=np.concatenate(bs).astype(np.int32),
                edges=np.concatenate(es).astype(np.int32), tris=np.concatenate(fs).astype(np.int32),
                mass=np.array(ms, dtype=np.float64), inertia_J=np.array(Js, dtype=np.float64),
                state=st, planes=np.zeros((0, 4)) if planes is None else np.asarray(planes, dtype=np.float64))


def _body(V, F, density, c, R=None, v=None, pinned=False):
    m, cen, S = mass_properties(V, F, density)
    Vb = V - cen
    if R is not None:
        Vb = Vb @ R.T
    return dict(V=Vb, F=F, c=np.asarray(c, dtype=np.float64), v=np.zeros(3) if v is None else v,
                mass=m, J=np.trace(S) / 3.0, pinned=pinned)


GROUND = [0.0, 1.0, 0.0, 0.0]


def config1_cubes(seed=0, spacing=1.05):
    """8 unit cubes in a 2x2x2 grid with seeded rotations and +-0.01 jitter,
    at rest above the ground plane y = 0.  The grid pitch is `spacing`
    times the cube's circumscribed diameter so that no two rotated cubes
    overlap at t = 0."""
    rng = np.random.default_rng(seed)
    V, F = cube_mesh(1.0)
    pitch = spacing * np.sqrt(3.0)
    bodies = []
    for i in range(2):
        for j in range(2):
            for k in range(2):
                R = _rand_rotation(rng)
                c = np.array([i * pitch, 0.5 * np.sqrt(3.0) + 0.05 + j * pitch, k * pitch])
                c += rng.uniform(-0.01, 0.01, 3)
                bodies.append(_body(V, F, 1000.0, c, R))
    return assemble_bodies(bodies, planes=[GROUND])


def config2_chain_net(n=16, seed=0, pitch=1.48, R=1.0, r=0.25, nu=24, nv=12, vel_noise=1e-3, lift=0.9):
    """n x n net of torus links in the xz plane, `pitch` apart, built as
    square chain mail:
      * (even, even) sites: flat links (axis y);
      * (odd, even) sites: standing links in the xy plane, each threading
        its two flat neighbours along x;
      * (even, odd) sites: standing links in the yz plane, threading along z;
      * (odd, odd) sites: flat links raised by `lift`, resting on the mail.
    Standing links are the 90-degree rotations of the flat ones about the
    grid axes.  Two interlocked links whose centres are 2(R - r) = 1.5 apart
    touch with zero gap, so the default pitch of 1.48 leaves a 0.02 gap.
    The four corner links are pinned; every other link gets a seeded
    +-vel_noise initial velocity."""
    rng = np.random.default_rng(seed)
    V, F = torus_mesh(R, r, nu, nv)           # ring in the xy plane (axis z)
    flat = np.array([[1, 0, 0], [0, 0, -1], [0, 1, 0]], dtype=np.float64)    # axis z -> y
    stand_x = np.eye(3)                                                       # xy plane
    stand_z = np.array([[0, 0, 1], [0, 1, 0], [-1, 0, 0]], dtype=np.float64)  # yz plane
    bodies = []
    corners = {(0, 0), (0, n - 1), (n - 1, 0), (n - 1, n - 1)}
    for i in range(n):
        for j in range(n):
            y = 0.0
            if i % 2 == 0 and j % 2 == 0:
                Rm = flat
            elif i % 2 == 1 and j % 2 == 0:
                Rm = stand_x
            elif i % 2 == 0 and j % 2 == 1:
                Rm = stand_z
            else:
                Rm, y = flat, lift
            pinned = (i, j) in corners
            v = np.zeros(3) if pinned else rng.uniform(-vel_noise, vel_noise, 3)
            bodies.append(_body(V, F, 1000.0, [i * pitch, y, j * pitch], Rm, v=v, pinned=pinned))
    return assemble_bodies(bodies)


def config3_batch(n_scenes=512, seed=0, nmin=4, nmax=64):
    """n_scenes independent scenes; each has round(exp(U(ln nmin, ln nmax)))
    bodies, cubes or tori 50/50, seeded poses in a 10x10x10 box above the
    ground and velocities U(-1,1)^3.  Bodies are placed on a jittered
    lattice so that none overlap at t = 0."""
    rng = np.random.default_rng(seed)
    cube = cube_mesh(1.0)
    tor = torus_mesh(0.5, 0.125, 24, 12)
    scenes = []
    for s in range(n_scenes):
        nb = int(round(np.exp(rng.uniform(np.log(nmin), np.log(nmax)))))
        slots = rng.permutation(125)[:nb]
        bodies = []
        for k in range(nb):
            sx, sy, sz = slots[k] % 5, (slots[k] // 5) % 5, slots[k] // 25
            c = np.array([sx * 2.0 + 1.0, 1.0 + sy * 2.0, sz * 2.0 + 1.0]) + rng.uniform(-0.1, 0.1, 3)
            V, F = cube if rng.uniform() < 0.5 else tor
            bodies.append(_body(V, F, 1000.0, c, _rand_rotation(rng), v=rng.uniform(-1, 1, 3)))
        scenes.append(assemble_bodies(bodies, planes=[GROUND]))
    return scenes


def config5_pile(n=4096, seed=0, box=(12.0, 12.0, 40.0)):
    """n icospheres (subdivision 1 or 2, radius U(0.2,0.5)) dropped into an
    open box [0,bx] x [0,height) x [0,bz] with walls as half-spaces; the
    box's 40 is its height (y)."""
    rng = np.random.default_rng(seed)
    meshes = {1: icosphere_mesh(1, 1.0), 2: icosphere_mesh(2, 1.0)}
    bx, bz, h = box[0], box[1], box[2]
    per = int(np.floor(bx / 1.05))
    bodies = []
    for k in range(n):
        sd = 1 if rng.uniform() < 0.5 else 2
        rad = rng.uniform(0.2, 0.5)
        V, F = meshes[sd]
        ix, iz, iy = k % per, (k // per) % per, k // (per * per)
        c = np.array([0.55 + ix * 1.05, 0.6 + iy * 1.05, 0.55 + iz * 1.05]) + rng.uniform(-0.02, 0.02, 3)
        bodies.append(_body(V * rad, F, 1000.0, c, _rand_rotation(rng)))
    planes = [GROUND, [1, 0, 0, 0.0], [-1, 0, 0, -bx], [0, 0, 1, 0.0], [0, 0, -1, -bz]]
    return assemble_bodies(bodies, planes=planes)


def concat_scenes(scenes):
    """Merge scenes into one (used by the oracle-side of batch tests)."""
    out = {k: [] for k in ("xbar", "vert_body", "edges", "tris", "mass", "inertia_J", "state", "planes")}
    nv = nb = 0
    for s in scenes:
        out["xbar"].append(s["xbar"])
        out["vert_body"].append(s["vert_body"] + nb)
        out["edges"].append(s["edges"] + nv)
        out["tris"].append(s["tris"] + nv)
        out["mass"].append(s["mass"])
        out["inertia_J"].append(s["inertia_J"])
        out["state"].append(s["state"])
        out["planes"].append(s["planes"])
        nv += len(s["xbar"])
        nb += len(s["mass"])
    return {k: np.concatenate(v) for k, v in out.items()}
