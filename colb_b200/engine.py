"""ctypes binding of libabd_b200.so (the C ABI in include/abd_b200.h).

`Engine` owns one library handle.  The library is built in-tree by
colb_b200/build_lib.py; importing this module never falls back to any other
implementation: if the library or a CUDA device is missing, constructing an
Engine raises.
"""
import ctypes as C
import os
import numpy as np

from ._abi import AbdParams, AbdStepStats, scene_descs, ABD_OK

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libabd_b200.so")
_lib = None

# every symbol include/abd_b200.h declares
EXPORTS = [
    "abd_default_params", "abd_create", "abd_destroy", "abd_get_sizes", "abd_set_state", "abd_get_state",
    "abd_step", "abd_get_profile", "abd_get_vertices", "abd_get_pairs", "abd_get_contact_points",
    "abd_energy", "abd_assemble", "abd_solve", "abd_set_warm_start", "abd_get_features",
    "abd_count_intersections", "abd_last_error", "abd_abi_version", "abd_set_timing", "abd_get_timing",
    "abd_ee_pairs_static", "abd_set_mlp", "abd_mlp_forward", "abd_trainer_create", "abd_trainer_destroy",
    "abd_trainer_last_error", "abd_trainer_set_data", "abd_trainer_epoch", "abd_trainer_grad", "abd_trainer_params",
    "abd_get_autotune",
]
MLP_IN, MLP_OUT, MLP_NPARAM, MLP_NNORM = 48, 12, 147212, 120
PHASES = ["detect", "assemble", "solve", "energy", "ccd", "other", "energy_query", "spmv", "asm_keys", "asm_body",
          "asm_contact", "asm_inverse", "dense", "swept", "energy_list", "ls_trials", "band"]


class AbdError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libabd_b200 error {code}: {msg}")
        self.code = code


def load_library(path=LIB_PATH):
    """Load libabd_b200.so and declare argument types; raises if absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run colb_b200/build_lib.py (or __graft_entry__.build())")
    L = C.CDLL(path)
    vp, dp, fp, ip = C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_float), C.POINTER(C.c_int32)
    L.abd_default_params.argtypes = [C.POINTER(AbdParams)]
    L.abd_default_params.restype = None
    L.abd_create.argtypes = [C.POINTER(AbdParams), vp, C.c_int32, C.c_int32, C.POINTER(vp)]
    L.abd_destroy.argtypes = [vp]
    L.abd_get_sizes.argtypes = [vp, ip, ip, ip, ip, ip]
    L.abd_set_state.argtypes = [vp, dp, C.c_int32]
    L.abd_get_state.argtypes = [vp, dp]
    L.abd_step.argtypes = [vp, C.c_int32, C.POINTER(AbdStepStats)]
    L.abd_get_profile.argtypes = [vp, C.c_int32, dp, dp, ip, C.c_int32, ip]
    L.abd_get_vertices.argtypes = [vp, dp]
    L.abd_get_pairs.argtypes = [vp, ip, ip, C.c_int32, ip]
    L.abd_get_contact_points.argtypes = [vp, dp, dp, C.c_int32, ip]
    L.abd_energy.argtypes = [vp, dp]
    L.abd_assemble.argtypes = [vp, dp, dp]
    L.abd_solve.argtypes = [vp, dp, ip]
    L.abd_set_warm_start.argtypes = [vp, fp, C.c_int32]
    L.abd_get_features.argtypes = [vp, fp, C.c_int32]
    L.abd_count_intersections.argtypes = [vp, ip]
    L.abd_last_error.argtypes = [vp]
    L.abd_last_error.restype = C.c_char_p
    L.abd_abi_version.argtypes = []
    L.abd_set_timing.argtypes = [vp, C.c_int32, C.c_int32]
    L.abd_get_timing.argtypes = [vp, dp, C.POINTER(C.c_int64), dp]
    L.abd_ee_pairs_static.argtypes = [vp, vp, C.c_int32, C.c_int32, C.c_double, vp, C.c_int32, vp, vp]
    L.abd_set_mlp.argtypes = [vp, fp, fp]
    L.abd_get_autotune.argtypes = [vp, ip, C.c_int32, ip]
    L.abd_mlp_forward.argtypes = [vp, fp, C.c_int32, fp]
    L.abd_trainer_create.argtypes = [C.c_int32, fp, C.POINTER(vp)]
    L.abd_trainer_destroy.argtypes = [vp]
    L.abd_trainer_last_error.argtypes = [vp]
    L.abd_trainer_last_error.restype = C.c_char_p
    L.abd_trainer_set_data.argtypes = [vp, fp, fp, C.c_int32]
    L.abd_trainer_epoch.argtypes = [vp, ip, C.c_int32, C.c_int32, C.c_float, fp]
    L.abd_trainer_grad.argtypes = [vp, fp, fp, C.c_int32, fp, fp]
    L.abd_trainer_params.argtypes = [vp, fp]
    _lib = L
    return L


def default_params():
    p = AbdParams()
    load_library().abd_default_params(C.byref(p))
    return p


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ip(a):
    return a.ctypes.data_as(C.POINTER(C.c_int32))


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a if shape is None else a.reshape(shape)


class Engine:
    """One device handle over one scene or a batch of independent scenes."""

    def __init__(self, params, scenes, device=0):
        if isinstance(scenes, dict):
            scenes = [scenes]
        self.L = load_library()
        self.params = params
        descs, self._keep = scene_descs(scenes)
        h = C.c_void_p()
        rc = self.L.abd_create(C.byref(params), C.cast(descs, C.c_void_p), len(scenes), device, C.byref(h))
        if rc != ABD_OK:
            raise AbdError(rc, self.L.abd_last_error(None).decode())
        self.h = h
        sz = [C.c_int32() for _ in range(5)]
        self.L.abd_get_sizes(self.h, *[C.byref(s) for s in sz])
        self.nb, self.nv, self.ne, self.nt, self.ns = [s.value for s in sz]

    def _check(self, rc, allow=()):
        if rc != ABD_OK and rc not in allow:
            raise AbdError(rc, self.L.abd_last_error(self.h).decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.abd_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_state(self, out=None):
        """(nb, 48) float64 BDFAffine rows; `out` (C-contiguous float64 of that
        shape, e.g. pinned memory) receives the copy instead of a new array."""
        if out is None:
            out = np.zeros((self.nb, 48))
        elif out.dtype != np.float64 or out.shape != (self.nb, 48) or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("get_state: out must be a C-contiguous float64 array of shape (nb, 48)")
        self._check(self.L.abd_get_state(self.h, _dp(out)))
        return out

    def set_state(self, st):
        st = np.ascontiguousarray(st, dtype=np.float64).reshape(self.nb, 48)
        self._check(self.L.abd_set_state(self.h, _dp(st), self.nb))

    def step(self, n=1, allow=()):
        st = AbdStepStats()
        rc = self._check(self.L.abd_step(self.h, n, C.byref(st)), allow)
        return rc, st

    def profile(self, scene=0, cap=1 << 18):
        r = np.zeros(cap); a = np.zeros(cap); ips = np.zeros(cap, dtype=np.int32)
        n = C.c_int32()
        self._check(self.L.abd_get_profile(self.h, scene, _dp(r), _dp(a), _ip(ips), cap, C.byref(n)))
        return r[:n.value].copy(), a[:n.value].copy(), ips

    def vertices(self):
        x = np.zeros((self.nv, 3))
        self._check(self.L.abd_get_vertices(self.h, _dp(x)))
        return x

    def pairs(self, cap=1 << 22):
        out = np.zeros((cap, 4), dtype=np.int32)
        kinds = np.zeros(cap, dtype=np.int32)
        n = C.c_int32()
        self._check(self.L.abd_get_pairs(self.h, _ip(out), _ip(kinds), cap, C.byref(n)))
        return out[:n.value].copy(), kinds[:n.value].copy()

    def contact_points(self, cap=1 << 20):
        p = np.zeros((cap, 3)); d = np.zeros(cap)
        n = C.c_int32()
        self._check(self.L.abd_get_contact_points(self.h, _dp(p), _dp(d), cap, C.byref(n)))
        m = min(n.value, cap)
        return p[:m].copy(), d[:m].copy()

    def energy(self):
        e = np.zeros(self.ns)
        self._check(self.L.abd_energy(self.h, _dp(e)))
        return e

    def assemble(self, dense=True):
        g = np.zeros(self.nb * 12)
        H = np.zeros((self.nb * 12, self.nb * 12)) if dense else None
        self._check(self.L.abd_assemble(self.h, _dp(g), _dp(H) if dense else None))
        return g, H

    def solve(self):
        du = np.zeros(self.nb * 12)
        it = C.c_int32()
        self._check(self.L.abd_solve(self.h, _dp(du), C.byref(it)))
        return du, it.value

    def set_warm_start(self, dq):
        dq = np.ascontiguousarray(dq, dtype=np.float32).reshape(self.nb, 12)
        self._check(self.L.abd_set_warm_start(self.h, dq.ctypes.data_as(C.POINTER(C.c_float)), self.nb))

    def set_mlp(self, params, norm):
        """Network of the learned warm start (warm_start 3): ABD_MLP_NPARAM
        parameters and ABD_MLP_NNORM normalisation floats."""
        params = _f32(params, (MLP_NPARAM,)); norm = _f32(norm, (MLP_NNORM,))
        self._check(self.L.abd_set_mlp(self.h, _fp(params), _fp(norm)))

    def mlp_forward(self, x):
        x = _f32(x).reshape(-1, MLP_IN)
        y = np.zeros((len(x), MLP_OUT), dtype=np.float32)
        self._check(self.L.abd_mlp_forward(self.h, _fp(x), len(x), _fp(y)))
        return y

    def features(self):
        f = np.zeros((self.nb, 48), dtype=np.float32)
        self._check(self.L.abd_get_features(self.h, f.ctypes.data_as(C.POINTER(C.c_float)), self.nb))
        return f

    def autotune(self):
        """Launch shapes the autotuner chose (-1 while still timing): contact
        assembly threads and contacts per block, list-energy and body-energy
        threads per block."""
        v = np.zeros(8, dtype=np.int32)
        n = C.c_int32()
        self._check(self.L.abd_get_autotune(self.h, _ip(v), 8, C.byref(n)))
        return dict(zip(["contact_threads", "contacts_per_block", "list_energy_threads", "body_energy_threads"],
                        v[:n.value].tolist()))

    def set_timing(self, on=True, reset=True):
        self._check(self.L.abd_set_timing(self.h, int(on), int(reset)))

    def timing(self):
        ms = np.zeros(len(PHASES)); n = np.zeros(len(PHASES), dtype=np.int64); by = np.zeros(len(PHASES))
        self._check(self.L.abd_get_timing(self.h, _dp(ms), n.ctypes.data_as(C.POINTER(C.c_int64)), _dp(by)))
        return {PHASES[i]: dict(ms=float(ms[i]), launches=int(n[i]), bytes=float(by[i])) for i in range(len(PHASES))}

    def count_intersections(self):
        n = C.c_int32()
        self._check(self.L.abd_count_intersections(self.h, C.byref(n)))
        return n.value


class Trainer:
    """GPU trainer of the warm-start network (abd_trainer_*)."""

    def __init__(self, params, device=0):
        self.L = load_library()
        h = C.c_void_p()
        params = _f32(params, (MLP_NPARAM,))
        rc = self.L.abd_trainer_create(device, _fp(params), C.byref(h))
        self.h = h
        if rc != ABD_OK:
            msg = self.L.abd_trainer_last_error(h).decode() if h.value else "no device"
            self.close()
            raise AbdError(rc, msg)

    def _check(self, rc):
        if rc != ABD_OK:
            raise AbdError(rc, self.L.abd_trainer_last_error(self.h).decode())

    def set_data(self, x, y):
        x = _f32(x).reshape(-1, MLP_IN); y = _f32(y).reshape(-1, MLP_OUT)
        self._check(self.L.abd_trainer_set_data(self.h, _fp(x), _fp(y), len(x)))

    def epoch(self, order, batch, lr):
        order = np.ascontiguousarray(order, dtype=np.int32)
        loss = C.c_float()
        self._check(self.L.abd_trainer_epoch(self.h, _ip(order), len(order), batch, lr, C.byref(loss)))
        return loss.value

    def grad(self, x, y):
        x = _f32(x).reshape(-1, MLP_IN); y = _f32(y).reshape(-1, MLP_OUT)
        g = np.zeros(MLP_NPARAM, dtype=np.float32)
        loss = C.c_float()
        self._check(self.L.abd_trainer_grad(self.h, _fp(x), _fp(y), len(x), _fp(g), C.byref(loss)))
        return loss.value, g

    def params(self):
        p = np.zeros(MLP_NPARAM, dtype=np.float32)
        self._check(self.L.abd_trainer_params(self.h, _fp(p)))
        return p

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.L.abd_trainer_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
