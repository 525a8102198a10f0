"""Solver parameter sets.

`reference_params()` carries the constants of the reference hot path
(Luke-Skycrawler/colb): dt = 8e-3 (links.py:16), gravity (0,-10,0)
(abd.py:28), kappa = 4e8 (abd.py:30), k_ortho = 1e5 (ortho.py:5),
dhat = 2 * 0.0475 (barrier.py:4-5), candidate filter
(thickness + buffer) * 2 = 0.19 (contact.py:7-9, :168), Newton tolerance
1e-5 and 16 iterations (abd.py:679, :699), Krylov tolerance 1e-5
(abd.py:636), line-search floor 1e-2 (gauss_newton.py:110), pinned diagonal
100 (abd.py:146) and EE-only contact with float32 closest points
(contact.py:143-169, abd.py:190).

`config_params()` carries the synthetic-scene physics: triangle meshes
with point-triangle + edge-edge + half-space contact, dhat = 1e-3,
kappa = 1e7, k_ortho = 1e7, gravity (0,-9.8,0), CCD-bounded line search.
Two choices differ from the reference constants because the stiff log
barrier at dhat = 1e-3 needs them: the back-off line search keeps halving
until the energy decreases (floor 1e-12 instead of accepting 1/64
unconditionally, gauss_newton.py:110), and impacts take up to ~25 Newton
iterations, so the cap is 64 (the residual target stays 1e-5).
"""
from ._abi import (AbdParams, params_from_dict, params_to_dict, BARRIER_CUBIC, BARRIER_LOG,
                   HESS_REFERENCE, HESS_PROJECTED, SOLVER_BICGSTAB, SOLVER_PCG, SOLVER_AUTO, PREC_FP64)

REFERENCE = dict(
    dt=8e-3,
    gravity=[0.0, -10.0, 0.0],
    kappa=4e8,
    k_ortho=1e5,
    dhat=0.0475 * 2,
    cand_dist=(0.0475 + 0.0475) * 2.0,
    barrier=BARRIER_CUBIC,
    hess_mode=HESS_REFERENCE,
    contact_ee=1,
    contact_pt=0,
    self_contact=1,
    ee_f32=1,
    linear_solver=SOLVER_BICGSTAB,
    lin_max_iter=1000,
    lin_tol=1e-5,
    newton_tol=1e-5,
    newton_max_iter=16,
    ccd=0,
    ccd_scale=0.1,
    ls_min_alpha=1e-2,
    precision=PREC_FP64,
    contact_capacity=1 << 16,
    pinned_diag=100.0,
    warm_start=0,
    autotune=1,
    ls_groups=0,
    ls_graph=0,
)

CONFIG = dict(
    dt=1.0 / 120.0,
    gravity=[0.0, -9.8, 0.0],
    kappa=1e7,
    k_ortho=1e7,
    dhat=1e-3,
    cand_dist=1e-3,
    barrier=BARRIER_LOG,
    hess_mode=HESS_PROJECTED,
    contact_ee=1,
    contact_pt=1,
    self_contact=0,
    ee_f32=0,
    linear_solver=SOLVER_AUTO,
    lin_max_iter=2000,
    lin_tol=1e-6,
    newton_tol=1e-5,
    newton_max_iter=64,
    ccd=1,
    ccd_scale=0.1,
    ls_min_alpha=1e-12,
    precision=PREC_FP64,
    contact_capacity=1 << 20,
    pinned_diag=100.0,
    warm_start=0,
    autotune=1,
    ls_groups=0,
    ls_graph=1,
)


def reference_params(**over) -> AbdParams:
    d = dict(REFERENCE)
    d.update(over)
    return params_from_dict(d)


def config_params(**over) -> AbdParams:
    d = dict(CONFIG)
    d.update(over)
    return params_from_dict(d)


__all__ = ["REFERENCE", "CONFIG", "reference_params", "config_params", "params_from_dict",
           "params_to_dict", "AbdParams"]
