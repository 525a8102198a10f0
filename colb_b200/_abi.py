"""ctypes mirror of include/abd_b200.h (the C ABI of libabd_b200.so).

The structs are laid out field for field like the header; the status codes
and enums carry the same values.  Both the CUDA library and the test-side
CPU oracle take these structs.
"""
import ctypes as C

ABD_OK = 0
ABD_ERR_INVALID_ARG = -1
ABD_ERR_CUDA = -2
ABD_ERR_CONTACT_OVERFLOW = -3
ABD_ERR_NAN = -4
ABD_ERR_SOLVER_CAP = -5
ABD_ERR_NEWTON_CAP = -6
ABD_ERR_CCD_CAP = -7
ABD_ERR_NO_DEVICE = -8
ABD_ERR_NOT_BUILT = -9
ABD_INJECT_DU_NONFINITE = 1
ABD_INJECT_SWEPT_FULL = 2
ABD_CCD_MAX_ITER = 100000

BARRIER_CUBIC, BARRIER_QUADRATIC, BARRIER_LOG = 0, 1, 2
HESS_REFERENCE, HESS_PROJECTED = 0, 1
SOLVER_BICGSTAB, SOLVER_PCG, SOLVER_DIRECT, SOLVER_AUTO = 0, 1, 2, 3
PREC_FP64, PREC_MIXED = 0, 1
CONTACT_EE, CONTACT_PT, CONTACT_PG = 0, 1, 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class AbdParams(C.Structure):
    _fields_ = [
        ("dt", C.c_double),
        ("gravity", C.c_double * 3),
        ("kappa", C.c_double),
        ("k_ortho", C.c_double),
        ("dhat", C.c_double),
        ("cand_dist", C.c_double),
        ("barrier", C.c_int32),
        ("hess_mode", C.c_int32),
        ("contact_ee", C.c_int32),
        ("contact_pt", C.c_int32),
        ("self_contact", C.c_int32),
        ("ee_f32", C.c_int32),
        ("linear_solver", C.c_int32),
        ("lin_max_iter", C.c_int32),
        ("lin_tol", C.c_double),
        ("newton_tol", C.c_double),
        ("newton_max_iter", C.c_int32),
        ("ccd", C.c_int32),
        ("ccd_scale", C.c_double),
        ("ls_min_alpha", C.c_double),
        ("precision", C.c_int32),
        ("contact_capacity", C.c_int32),
        ("pinned_diag", C.c_double),
        ("warm_start", C.c_int32),
        ("broadphase", C.c_int32),
        ("autotune", C.c_int32),
        ("ls_groups", C.c_int32),
        ("ls_graph", C.c_int32),
        ("ccd_max_iter", C.c_int32),
        ("test_inject", C.c_int32),
        ("reserved", C.c_int32 * 1),
    ]


class AbdSceneDesc(C.Structure):
    _fields_ = [
        ("n_bodies", C.c_int32),
        ("n_verts", C.c_int32),
        ("n_edges", C.c_int32),
        ("n_tris", C.c_int32),
        ("xbar", _dp),
        ("vert_body", _ip),
        ("edges", _ip),
        ("tris", _ip),
        ("mass", _dp),
        ("inertia_J", _dp),
        ("state", _dp),
        ("n_planes", C.c_int32),
        ("planes", _dp),
    ]


class AbdStepStats(C.Structure):
    _fields_ = [
        ("steps", C.c_int32),
        ("newton_iters", C.c_int32),
        ("max_newton_iters", C.c_int32),
        ("lin_iters", C.c_int32),
        ("n_pairs", C.c_int32),
        ("n_active", C.c_int32),
        ("unconverged", C.c_int32),
        ("ls_trials", C.c_int32),
        ("last_residual", C.c_double),
        ("min_toi", C.c_double),
        ("gpu_ms", C.c_double),
        ("kernel_launches", C.c_int32),
        ("comp_band", C.c_int32),
        ("comp_small", C.c_int32),
        ("comp_large", C.c_int32),
        ("krylov_fallbacks", C.c_int32),
        ("ls_graph_launches", C.c_int32),
        ("solver_capped", C.c_int32),
        ("du_guard_hits", C.c_int32),
        ("host_syncs", C.c_int32),
        ("reserved_stats", C.c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved_stats"}


def params_from_dict(d):
    """Build an AbdParams from a plain dict (keys = field names)."""
    p = AbdParams()
    for k, v in d.items():
        if k == "gravity":
            p.gravity = (C.c_double * 3)(*v)
        else:
            setattr(p, k, v)
    return p


def params_to_dict(p):
    out = {}
    for k, _ in AbdParams._fields_:
        if k == "reserved":
            continue
        v = getattr(p, k)
        out[k] = list(v) if k == "gravity" else v
    return out


class SceneArrays:
    """Keeps the numpy arrays behind one AbdSceneDesc alive."""

    def __init__(self, scene):
        import numpy as np
        self.xbar = np.ascontiguousarray(scene["xbar"], dtype=np.float64)
        self.vert_body = np.ascontiguousarray(scene["vert_body"], dtype=np.int32)
        self.edges = np.ascontiguousarray(scene["edges"], dtype=np.int32).reshape(-1, 2)
        self.tris = np.ascontiguousarray(scene["tris"], dtype=np.int32).reshape(-1, 3)
        self.mass = np.ascontiguousarray(scene["mass"], dtype=np.float64)
        self.J = np.ascontiguousarray(scene["inertia_J"], dtype=np.float64)
        self.state = np.ascontiguousarray(scene["state"], dtype=np.float64).reshape(-1, 48)
        self.planes = np.ascontiguousarray(scene.get("planes", np.zeros((0, 4))), dtype=np.float64).reshape(-1, 4)
        d = AbdSceneDesc()
        d.n_bodies = len(self.mass)
        d.n_verts = len(self.vert_body)
        d.n_edges = len(self.edges)
        d.n_tris = len(self.tris)
        d.xbar = self.xbar.ctypes.data_as(_dp)
        d.vert_body = self.vert_body.ctypes.data_as(_ip)
        d.edges = self.edges.ctypes.data_as(_ip)
        d.tris = self.tris.ctypes.data_as(_ip)
        d.mass = self.mass.ctypes.data_as(_dp)
        d.inertia_J = self.J.ctypes.data_as(_dp)
        d.state = self.state.ctypes.data_as(_dp)
        d.n_planes = len(self.planes)
        d.planes = self.planes.ctypes.data_as(_dp)
        self.desc = d


def scene_descs(scenes):
    """Array of AbdSceneDesc for a list of scene dicts, plus the keep-alive list."""
    keep = [SceneArrays(s) for s in scenes]
    arr = (AbdSceneDesc * len(keep))(*[k.desc for k in keep])
    return arr, keep
