"""ctypes binding of the CPU oracle (oracle/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline leg, never by the colb_b200 package.  The oracle is
an FP64 C restatement of the reference's ABD Newton step (see
abd_oracle.c for the file:line map).  Parity is unpinned against the
reference itself (no Warp here, no reference tests or fixtures); see
tests/golden for the restatement-level fixtures that pin it.
"""
import ctypes as C
import os
import subprocess
import numpy as np

from colb_b200._abi import AbdStepStats, scene_descs

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build():
    subprocess.check_call(["make", "-s", "-C", _HERE])


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            build()
        L = C.CDLL(_LIB)
        dp, fp, ip = C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int32)
        L.oracle_create.restype = C.c_void_p
        L.oracle_create.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        L.oracle_destroy.argtypes = [C.c_void_p]
        for n in ("oracle_set_state", "oracle_get_state", "oracle_get_vertices"):
            getattr(L, n).argtypes = [C.c_void_p, dp]
        L.oracle_get_pairs.argtypes = [C.c_void_p, ip, ip, C.c_int, C.POINTER(C.c_int)]
        L.oracle_energy.argtypes = [C.c_void_p, dp]
        L.oracle_assemble.argtypes = [C.c_void_p, dp, dp]
        L.oracle_solve.argtypes = [C.c_void_p, dp, C.POINTER(C.c_int)]
        L.oracle_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(AbdStepStats)]
        L.oracle_get_profile.argtypes = [C.c_void_p, C.c_int, dp, dp, C.POINTER(C.c_int), C.c_int, C.POINTER(C.c_int)]
        L.oracle_set_warm_start.argtypes = [C.c_void_p, fp, C.c_int]
        L.oracle_count_intersections.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        L.oracle_set_threads.argtypes = [C.c_int]
        L.oracle_barrier.argtypes = [C.c_int, C.c_double, C.c_double, dp]
        L.oracle_ortho.argtypes = [dp, C.c_double, dp, dp, dp]
        L.oracle_seg_seg_f32.argtypes = [fp, fp, fp, fp, C.c_float, fp]
        L.oracle_seg_seg_f64.argtypes = [dp, dp, dp, dp, C.c_double, dp]
        for n in ("oracle_d2_pp", "oracle_d2_pe", "oracle_d2_ee_line", "oracle_d2_pt_plane"):
            getattr(L, n).argtypes = [dp, dp, dp, dp]
        L.oracle_pt_region.argtypes = [dp, dp, dp, dp]
        L.oracle_pt_dist2.argtypes = [dp, dp, dp, dp]
        L.oracle_pt_dist2.restype = C.c_double
        L.oracle_psd_project.argtypes = [C.c_int, dp]
        L.oracle_accd.argtypes = [C.c_int, dp, dp, C.c_double, C.c_double, dp]
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


# ---- primitive functions -------------------------------------------------
def barrier(kind, x, xhat):
    o = np.zeros(3)
    lib().oracle_barrier(kind, x, xhat, _dp(o))
    return o


def ortho(q9, k):
    q9 = np.ascontiguousarray(q9, dtype=np.float64)
    e = np.zeros(1); g = np.zeros(9); H = np.zeros(81)
    lib().oracle_ortho(_dp(q9), k, _dp(e), _dp(g), _dp(H))
    return e[0], g, H.reshape(9, 9)


def seg_seg_f32(p1, q1, p2, q2, eps=1e-6):
    a = [np.ascontiguousarray(v, dtype=np.float32) for v in (p1, q1, p2, q2)]
    o = np.zeros(3, dtype=np.float32)
    lib().oracle_seg_seg_f32(*[_fp(v) for v in a], C.c_float(eps), _fp(o))
    return o


def seg_seg_f64(p1, q1, p2, q2, eps=1e-12):
    a = [np.ascontiguousarray(v, dtype=np.float64) for v in (p1, q1, p2, q2)]
    o = np.zeros(3)
    lib().oracle_seg_seg_f64(*[_dp(v) for v in a], eps, _dp(o))
    return o


def d2(kind, x):
    """kind in pp, pe, ee, pt; x stacked stencil points."""
    x = np.ascontiguousarray(x, dtype=np.float64).ravel()
    n = x.size
    f = np.zeros(1); g = np.zeros(n); H = np.zeros(n * n)
    fn = {"pp": "oracle_d2_pp", "pe": "oracle_d2_pe", "ee": "oracle_d2_ee_line", "pt": "oracle_d2_pt_plane"}[kind]
    getattr(lib(), fn)(_dp(x), _dp(f), _dp(g), _dp(H))
    return f[0], g, H.reshape(n, n)


def pt_region(p, a, b, c):
    v = [np.ascontiguousarray(t, dtype=np.float64) for t in (p, a, b, c)]
    return lib().oracle_pt_region(*[_dp(t) for t in v])


def pt_dist2(p, a, b, c):
    v = [np.ascontiguousarray(t, dtype=np.float64) for t in (p, a, b, c)]
    return lib().oracle_pt_dist2(*[_dp(t) for t in v])


def psd_project(H):
    H = np.ascontiguousarray(H, dtype=np.float64).copy()
    lib().oracle_psd_project(H.shape[0], _dp(H))
    return H


def accd(kind, x12, p12, s=0.1, tmax=1.0):
    x = np.ascontiguousarray(x12, dtype=np.float64).ravel()
    p = np.ascontiguousarray(p12, dtype=np.float64).ravel()
    t = np.zeros(1)
    hit = lib().oracle_accd(kind, _dp(x), _dp(p), s, tmax, _dp(t))
    return bool(hit), t[0]


def set_threads(n):
    lib().oracle_set_threads(int(n))


# ---- whole world ----------------------------------------------------------
class OracleWorld:
    """Same calls as the CUDA handle (colb_b200.engine.Engine), on the CPU."""

    def __init__(self, params, scenes):
        if isinstance(scenes, dict):
            scenes = [scenes]
        self.params = params
        self._descs, self._keep = scene_descs(scenes)
        self.nb = sum(len(s["mass"]) for s in scenes)
        self.nv = sum(len(s["xbar"]) for s in scenes)
        self.ns = len(scenes)
        self._p = params
        self.h = lib().oracle_create(C.byref(self._p), C.cast(self._descs, C.c_void_p), len(scenes))

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_destroy(self.h)
            self.h = None

    def get_state(self):
        st = np.zeros((self.nb, 48))
        lib().oracle_get_state(self.h, _dp(st))
        return st

    def set_state(self, st):
        st = np.ascontiguousarray(st, dtype=np.float64)
        lib().oracle_set_state(self.h, _dp(st))

    def vertices(self):
        x = np.zeros((self.nv, 3))
        lib().oracle_get_vertices(self.h, _dp(x))
        return x

    def pairs(self, cap=1 << 22):
        out = np.zeros((cap, 4), dtype=np.int32)
        kinds = np.zeros(cap, dtype=np.int32)
        n = C.c_int()
        lib().oracle_get_pairs(self.h, _ip(out), _ip(kinds), cap, C.byref(n))
        return out[:n.value].copy(), kinds[:n.value].copy()

    def energy(self):
        e = np.zeros(self.ns)
        lib().oracle_energy(self.h, _dp(e))
        return e

    def assemble(self, dense=True):
        g = np.zeros(self.nb * 12)
        H = np.zeros((self.nb * 12, self.nb * 12)) if dense else None
        lib().oracle_assemble(self.h, _dp(g), _dp(H) if dense else None)
        return g, H

    def solve(self):
        du = np.zeros(self.nb * 12)
        it = C.c_int()
        lib().oracle_solve(self.h, _dp(du), C.byref(it))
        return du, it.value

    def step(self, n=1):
        st = AbdStepStats()
        rc = lib().oracle_step(self.h, n, C.byref(st))
        return rc, st

    def profile(self, scene=0, cap=1 << 16):
        r = np.zeros(cap); a = np.zeros(cap); ips = np.zeros(cap, dtype=np.int32)
        n = C.c_int()
        lib().oracle_get_profile(self.h, scene, _dp(r), _dp(a), _ip(ips), cap, C.byref(n))
        return r[:n.value].copy(), a[:n.value].copy(), ips

    def set_warm_start(self, dq):
        dq = np.ascontiguousarray(dq, dtype=np.float32)
        return lib().oracle_set_warm_start(self.h, _fp(dq), self.nb)

    def count_intersections(self):
        n = C.c_int()
        lib().oracle_count_intersections(self.h, C.byref(n))
        return n.value
