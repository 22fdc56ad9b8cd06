"""Python host binding of the asd2g C ABI (include/asd2g.h) via ctypes.

This mirrors what the reference's drivers do with LevelSetSolver2D /
MACSolver2D / PoissonSolver2D (tests/LargeTests/*.cpp) on top of the B200
library: fields are numpy float64 arrays of shape (nx+6, ny+6) in the
reference layout idx(i,j) = j + (ny+6)*i.  There is no CPU fallback: loading
fails with an error when libasd2g.so is missing, and every call raises
``Asd2gError`` on a negative status.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libasd2g.so")

BC_NAMES = ["periodic", "neumann", "dirichlet", "axisym", "wall", "inlet", "outlet", "pressure", "lsfree", "custom"]
BC = {n: i for i, n in enumerate(BC_NAMES)}

# fields (enum asd2g_field)
LS, U, V, PS, P, KAPPA, H, HS, DIV, UHAT, VHAT, LSB, LS0, W0, W1, W2, W3 = range(17)
FIELDS = dict(ls=LS, u=U, v=V, ps=PS, p=P, kappa=KAPPA, H=H, HS=HS, div=DIV, uhat=UHAT, vhat=VHAT, lsB=LSB,
              ls0=LS0, w0=W0, w1=W1, w2=W2, w3=W3)
# reinit modes
REINIT_ORIGINAL, REINIT_SUSSMAN, REINIT_MINRK2, REINIT_FIRSTTIME, REINIT_MINRK2_SUSSMAN = range(5)
# solvers
PCG, PCG_REFERENCE, BICGSTAB, BICGSTAB_REFERENCE, MGPCG, UNET = range(6)
NOT_CONVERGED = 1
CURVATURE_REFERENCE, CURVATURE_DIVERGENCE = 0, 1
FLAG_NO_CLUSTER_PCG = 1
FLAG_NO_PERSIST_MG = 2
PRECISION_FP64, PRECISION_MIXED = 0, 1
ERRORS = {-1: "invalid argument", -2: "CUDA error", -3: "out of device memory", -4: "unsupported",
          -5: "non-finite value", -6: "Krylov breakdown", -7: "checkpoint I/O", -8: "internal error"}


class Asd2gError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"asd2g error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class _Params(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("nbc", C.c_int32), ("precision", C.c_int32),
                ("base_x", C.c_double), ("base_y", C.c_double), ("dx", C.c_double), ("dy", C.c_double),
                ("bc_u", C.c_int32 * 4), ("bc_v", C.c_int32 * 4), ("bc_p", C.c_int32 * 4),
                ("bcc_u", C.c_double * 4), ("bcc_v", C.c_double * 4), ("bcc_p", C.c_double * 4),
                ("rho_h", C.c_double), ("rho_l", C.c_double), ("mu_h", C.c_double), ("mu_l", C.c_double),
                ("sigma", C.c_double), ("gravity", C.c_double), ("g_axis", C.c_int32), ("fix_gravity", C.c_int32),
                ("time_order", C.c_int32), ("solver_flags", C.c_int32), ("cfl", C.c_double),
                ("ls_max_atime", C.c_double), ("numbers_given", C.c_int32), ("curvature", C.c_int32),
                ("re", C.c_double), ("we", C.c_double), ("fr", C.c_double)]


EXPORTS = [
    "asd2g_version", "asd2g_last_error", "asd2g_create", "asd2g_destroy", "asd2g_sync", "asd2g_field_ptr",
    "asd2g_upload", "asd2g_upload_async", "asd2g_upload_staged", "asd2g_download_staged", "asd2g_join_copies",
    "asd2g_sync_copies", "asd2g_download", "asd2g_copy_field", "asd2g_fill_field", "asd2g_apply_bc",
    "asd2g_ls_advect", "asd2g_ls_weno_rhs", "asd2g_reinit", "asd2g_subcell_eno", "asd2g_eno",
    "asd2g_sussman_constraint", "asd2g_heaviside_deriv", "asd2g_smoothed_sign", "asd2g_ls_step",
    "asd2g_kappa", "asd2g_heaviside", "asd2g_convection", "asd2g_viscosity", "asd2g_momentum_rhs",
    "asd2g_intermediate_vel", "asd2g_divergence", "asd2g_update_vel", "asd2g_update_dt",
    "asd2g_assemble_gfm", "asd2g_get_system", "asd2g_solve_pressure", "asd2g_true_residual",
    "asd2g_droplet_step", "asd2g_run_steps", "asd2g_checkpoint_save", "asd2g_checkpoint_load",
    "asd2g_checkpoint_info", "asd2g_pcg_solve_static", "asd2g_weno5_line", "asd2g_weno_absgrad",
    "asd2g_apply_bc_side", "asd2g_update_ntk", "asd2g_csr_solve", "asd2g_volume", "asd2g_last_volume",
    "asd2g_batch_create", "asd2g_batch_destroy", "asd2g_batch_upload", "asd2g_batch_download",
    "asd2g_batch_field_ptr", "asd2g_batch_offset", "asd2g_batch_assemble", "asd2g_batch_solve", "asd2g_batch_sync",
    "asd2g_batch_step", "asd2g_batch_volume", "asd2g_batch_tile_shape",
    "asd2g_batch_set_preconditioner_net", "asd2g_batch_solve_with", "asd2g_batch_last_fallback",
    "asd2g_conv_wpack_bytes", "asd2g_conv_pack_weights", "asd2g_conv3x3_bf16",
    "asd2g_unet_create", "asd2g_unet_destroy", "asd2g_unet_nparams", "asd2g_unet_init", "asd2g_unet_set_params",
    "asd2g_unet_get_params", "asd2g_unet_get_grads", "asd2g_unet_forward", "asd2g_unet_train_step",
    "asd2g_unet_train_step_residual", "asd2g_unet_train_step_energy",
    "asd2g_unet_error_flag", "asd2g_unet_set_stream", "asd2g_set_preconditioner_net", "asd2g_last_fallback",
    "asd2g_last_solve_one_launch",
    "asd2g_axi_kappa", "asd2g_axi_rhs_u", "asd2g_axi_rhs_v", "asd2g_axi_viscosity", "asd2g_axi_hat",
    "asd2g_axi_divergence",
    "asd2g_axi_assemble", "asd2g_axi_update_dt", "asd2g_axi_step",
    "asd2g_pc_training_pair", "asd2g_pc_training_pair_at",
]

_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load libasd2g.so (no fallback: raises if it is absent)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python -m asd2_b200.build`")
    L = C.CDLL(path)
    S = C.c_void_p
    dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
    ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
    fp = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
    I, D = C.c_int, C.c_double
    sig = {
        "asd2g_version": ([], I), "asd2g_last_error": ([], C.c_char_p),
        "asd2g_create": ([C.POINTER(_Params), C.c_void_p, C.POINTER(S)], I),
        "asd2g_destroy": ([S], I), "asd2g_sync": ([S], I),
        "asd2g_field_ptr": ([S, I, C.POINTER(C.c_void_p)], I),
        "asd2g_upload": ([S, I, dp], I), "asd2g_download": ([S, I, dp], I),
        "asd2g_upload_async": ([S, I, dp], I),
        "asd2g_upload_staged": ([S, I, dp], I), "asd2g_download_staged": ([S, I, dp], I),
        "asd2g_join_copies": ([S, I], I), "asd2g_sync_copies": ([S], I),
        "asd2g_copy_field": ([S, I, I], I), "asd2g_fill_field": ([S, I, D], I),
        "asd2g_apply_bc": ([S, I, C.c_char], I),
        "asd2g_ls_advect": ([S, D], I), "asd2g_ls_weno_rhs": ([S, I, I, I, I], I), "asd2g_reinit": ([S, I], I),
        "asd2g_subcell_eno": ([S, I, I, I], I), "asd2g_eno": ([S, I, I, I], I),
        "asd2g_sussman_constraint": ([S, I, I, I, I], I), "asd2g_heaviside_deriv": ([S, I, I], I),
        "asd2g_smoothed_sign": ([S, I, I], I), "asd2g_ls_step": ([S, D, I], I),
        "asd2g_kappa": ([S], I), "asd2g_heaviside": ([S], I), "asd2g_convection": ([S, I, I, I, I], I),
        "asd2g_viscosity": ([S, I, I, I, I, I, I], I), "asd2g_momentum_rhs": ([S, I, I, I, I, I, I], I),
        "asd2g_intermediate_vel": ([S, D, I], I), "asd2g_divergence": ([S, I, I, I], I),
        "asd2g_update_vel": ([S, D], I), "asd2g_update_dt": ([S, C.POINTER(D)], I),
        "asd2g_assemble_gfm": ([S, D, I], I),
        "asd2g_get_system": ([S, dp, dp, dp, dp, dp, dp, C.POINTER(I)], I),
        "asd2g_solve_pressure": ([S, I, D, I, D, C.POINTER(I), C.POINTER(D)], I),
        "asd2g_true_residual": ([S, C.POINTER(D)], I),
        "asd2g_droplet_step": ([S, C.POINTER(D), I, I, D, I, C.POINTER(I), C.POINTER(D)], I),
        "asd2g_checkpoint_save": ([S, C.c_char_p, D, C.c_longlong, D], I),
        "asd2g_checkpoint_load": ([S, C.c_char_p, C.POINTER(D), C.POINTER(C.c_longlong), C.POINTER(D)], I),
        "asd2g_checkpoint_info": ([C.c_char_p, C.POINTER(I), C.POINTER(I), C.POINTER(D), C.POINTER(C.c_longlong),
                                   C.POINTER(D)], I),
        "asd2g_run_steps": ([S, I, C.POINTER(D), I, I, D, I, C.POINTER(I), C.POINTER(C.c_longlong), C.POINTER(D)],
                            I),
        "asd2g_pcg_solve_static": ([I, I, I, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, D, I,
                                    C.c_void_p, C.POINTER(I), C.POINTER(D)], I),
        "asd2g_weno5_line": ([S, dp, dp, dp, D, I], I), "asd2g_weno_absgrad": ([S, I, I, I], I),
        "asd2g_apply_bc_side": ([S, I, C.c_char, I, I], I), "asd2g_update_ntk": ([S, I, I, I], I),
        "asd2g_axi_kappa": ([S], I), "asd2g_axi_rhs_u": ([S, D, I, I, I, I, I], I),
        "asd2g_axi_rhs_v": ([S, D, I, I, I, I, I, I], I), "asd2g_axi_hat": ([S, I, D, I, I, I, I], I),
        "asd2g_axi_viscosity": ([S, I, I, I, I, I, I, I], I),
        "asd2g_axi_divergence": ([S, I, I, I, I], I), "asd2g_axi_assemble": ([S, D, I], I),
        "asd2g_axi_update_dt": ([S, C.POINTER(D)], I),
        "asd2g_axi_step": ([S, C.POINTER(D), I, C.c_void_p, C.c_void_p, I, D, I, C.POINTER(I), C.POINTER(D)], I),
        "asd2g_csr_solve": ([S, I, I, ip, ip, dp, dp, dp, dp, D, I, C.POINTER(I), C.POINTER(D)], I),
        "asd2g_volume": ([S, C.POINTER(D), C.POINTER(D)], I),
        "asd2g_last_volume": ([S, C.POINTER(D), C.POINTER(D)], I),
        "asd2g_batch_create": ([C.POINTER(_Params), I, C.c_void_p, C.POINTER(S)], I),
        "asd2g_batch_destroy": ([S], I), "asd2g_batch_sync": ([S], I),
        "asd2g_batch_upload": ([S, I, I, dp], I), "asd2g_batch_download": ([S, I, I, dp], I),
        "asd2g_batch_field_ptr": ([S, I, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t)], I),
        "asd2g_batch_offset": ([S, I, C.POINTER(C.c_size_t)], I),
        "asd2g_batch_assemble": ([S, dp], I),
        "asd2g_batch_solve": ([S, D, I, ip, dp], I),
        "asd2g_batch_step": ([S, dp, I, D, I, ip, dp], I),
        "asd2g_batch_volume": ([S, dp, dp], I),
        "asd2g_batch_tile_shape": ([S, C.POINTER(I), C.POINTER(I), C.POINTER(C.c_float)], I),
        "asd2g_batch_set_preconditioner_net": ([S, S], I),
        "asd2g_batch_solve_with": ([S, I, C.c_double, I, ip, dp], I),
        "asd2g_batch_last_fallback": ([S, C.POINTER(I)], I),
        "asd2g_conv_wpack_bytes": ([I, I], C.c_size_t),
        "asd2g_conv_pack_weights": ([C.c_void_p, I, I, I, I, C.c_void_p, C.c_void_p], I),
        "asd2g_conv3x3_bf16": ([C.c_void_p, I, I, I, I, C.c_void_p, C.c_void_p, I, C.c_void_p, C.c_void_p, I,
                                C.c_void_p, C.c_void_p], I),
        "asd2g_unet_create": ([I, I, I, C.c_void_p, C.POINTER(S)], I), "asd2g_unet_destroy": ([S], I),
        "asd2g_unet_nparams": ([S], C.c_size_t), "asd2g_unet_init": ([S, C.c_ulonglong], I),
        "asd2g_unet_set_params": ([S, fp], I), "asd2g_unet_get_params": ([S, fp], I),
        "asd2g_unet_get_grads": ([S, fp], I),
        "asd2g_unet_forward": ([S, I, I, I, C.c_void_p, C.c_void_p], I),
        "asd2g_unet_train_step": ([S, I, I, I, C.c_void_p, C.c_void_p, C.c_float, C.POINTER(C.c_float)], I),
        "asd2g_unet_train_step_residual": ([S, I, I, I, C.c_void_p, C.c_float, C.POINTER(C.c_float)], I),
        "asd2g_unet_train_step_energy": ([S, I, I, I, C.c_void_p, C.c_void_p, C.c_float, C.POINTER(C.c_float)],
                                         I),
        "asd2g_unet_error_flag": ([S, C.POINTER(I)], I), "asd2g_unet_set_stream": ([S, C.c_void_p], I),
        "asd2g_set_preconditioner_net": ([S, S], I), "asd2g_last_fallback": ([S, C.POINTER(I)], I),
        "asd2g_last_solve_one_launch": ([S, C.POINTER(I)], I),
        "asd2g_pc_training_pair": ([S, C.c_void_p, C.c_void_p], I),
        "asd2g_pc_training_pair_at": ([S, I, C.c_void_p, C.c_void_p], I),
    }
    for name, (args, res) in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def _bcs(names):
    return [BC[n.lower()] for n in names]


@dataclass
class Params:
    nx: int
    ny: int
    dx: float
    dy: float
    bc_u: tuple = ("dirichlet",) * 4
    bc_v: tuple = ("dirichlet",) * 4
    bc_p: tuple = ("neumann",) * 4
    bcc_u: tuple = (0.0,) * 4
    bcc_v: tuple = (0.0,) * 4
    bcc_p: tuple = (0.0,) * 4
    rho_h: float = 1000.0
    rho_l: float = 1.0
    mu_h: float = 1.0e-3
    mu_l: float = 1.0e-5
    sigma: float = 0.0728
    g: float = 9.8
    g_axis: int = 1
    fix_gravity: int = 0
    time_order: int = 2
    cfl: float = 0.5
    ls_max_atime: float = 0.0
    base_x: float = 0.0
    base_y: float = 0.0
    precision: int = 0
    solver_flags: int = 0
    curvature: int = 0  # CURVATURE_REFERENCE or CURVATURE_DIVERGENCE

    def c(self) -> _Params:
        p = _Params()
        p.nx, p.ny, p.nbc, p.precision = self.nx, self.ny, 3, self.precision
        p.base_x, p.base_y, p.dx, p.dy = self.base_x, self.base_y, self.dx, self.dy
        for k, (a, b, c) in enumerate(zip(_bcs(self.bc_u), _bcs(self.bc_v), _bcs(self.bc_p))):
            p.bc_u[k], p.bc_v[k], p.bc_p[k] = a, b, c
            p.bcc_u[k], p.bcc_v[k], p.bcc_p[k] = self.bcc_u[k], self.bcc_v[k], self.bcc_p[k]
        p.rho_h, p.rho_l, p.mu_h, p.mu_l = self.rho_h, self.rho_l, self.mu_h, self.mu_l
        p.sigma, p.gravity, p.g_axis, p.fix_gravity = self.sigma, self.g, self.g_axis, self.fix_gravity
        p.time_order, p.cfl, p.ls_max_atime = self.time_order, self.cfl, self.ls_max_atime
        p.solver_flags = self.solver_flags
        p.curvature = self.curvature
        return p

    @classmethod
    def from_case(cls, case, **kw):
        fl = dict(case.fluid)
        fl.pop("g", None)
        g = case.fluid.get("g", 9.8)
        return cls(case.nx, case.ny, case.dx, case.dy, bc_u=case.bc_u, bc_v=case.bc_v, bc_p=case.bc_p, g=g,
                   **{k: v for k, v in fl.items() if k in cls.__dataclass_fields__}, **kw)


class Session:
    """One grid's device state on the B200 (an asd2g session)."""

    def __init__(self, params: Params, stream: int | None = None):
        self.L = load()
        self.params = params
        self.shape = (params.nx + 6, params.ny + 6)
        h = C.c_void_p()
        self._check(self.L.asd2g_create(C.byref(params.c()), C.c_void_p(stream) if stream else None, C.byref(h)))
        self.h = h

    # ---- plumbing ----
    def _check(self, rc):
        if rc < 0:
            raise Asd2gError(rc, self.L.asd2g_last_error().decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.asd2g_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def sync(self):
        self._check(self.L.asd2g_sync(self.h))

    @staticmethod
    def _f(f):
        return FIELDS[f] if isinstance(f, str) else int(f)

    def upload(self, f, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        assert a.shape == self.shape, (a.shape, self.shape)
        self._check(self.L.asd2g_upload(self.h, self._f(f), a))

    def upload_async(self, f, arr):
        """Queue the upload without waiting: arr must be a C-contiguous
        float64 array of the field's shape (ideally pinned) that stays
        unchanged until the session next synchronises."""
        if not (isinstance(arr, np.ndarray) and arr.dtype == np.float64 and arr.flags.c_contiguous
                and arr.shape == self.shape):
            raise ValueError("upload_async needs a C-contiguous float64 array of the field's shape")
        self._check(self.L.asd2g_upload_async(self.h, self._f(f), arr))


    def _check_host(self, arr, what):
        if not (isinstance(arr, np.ndarray) and arr.dtype == np.float64 and arr.flags.c_contiguous
                and arr.shape == self.shape):
            raise ValueError(f"{what} needs a C-contiguous float64 array of the field's shape")

    def upload_staged(self, f, arr):
        """Upload on the session's copy stream after the compute work queued
        so far (asd2g_upload_staged); join_copies(1) before its first reader."""
        self._check_host(arr, "upload_staged")
        self._check(self.L.asd2g_upload_staged(self.h, self._f(f), arr))

    def download_staged(self, f, out):
        """Download into out (pinned, float64, the field's shape) on the copy
        stream after the compute work queued so far (asd2g_download_staged)."""
        self._check_host(out, "download_staged")
        self._check(self.L.asd2g_download_staged(self.h, self._f(f), out))

    def join_copies(self, which=3):
        """Later compute work waits for the staged uploads (1), downloads (2) or both (3)."""
        self._check(self.L.asd2g_join_copies(self.h, which))

    def sync_copies(self):
        self._check(self.L.asd2g_sync_copies(self.h))
    def download(self, f):
        out = np.empty(self.shape)
        self._check(self.L.asd2g_download(self.h, self._f(f), out))
        return out

    def ptr(self, f) -> int:
        p = C.c_void_p()
        self._check(self.L.asd2g_field_ptr(self.h, self._f(f), C.byref(p)))
        return p.value

    def copy(self, dst, src):
        self._check(self.L.asd2g_copy_field(self.h, self._f(dst), self._f(src)))

    def fill(self, f, value):
        self._check(self.L.asd2g_fill_field(self.h, self._f(f), float(value)))

    def apply_bc(self, f, kind):
        self._check(self.L.asd2g_apply_bc(self.h, self._f(f), kind.upper().encode()))

    # ---- level set ----
    def ls_advect(self, dt):
        self._check(self.L.asd2g_ls_advect(self.h, dt))

    def ls_weno_rhs(self, ls="ls", uc="w0", vc="w1", out="w2"):
        self._check(self.L.asd2g_ls_weno_rhs(self.h, self._f(ls), self._f(uc), self._f(vc), self._f(out)))

    def reinit(self, mode):
        self._check(self.L.asd2g_reinit(self.h, mode))

    def ls_step(self, dt, mode):
        self._check(self.L.asd2g_ls_step(self.h, dt, mode))

    def weno5_line(self, F, d, n):
        FP, FM = np.zeros(n + 6), np.zeros(n + 6)
        self._check(self.L.asd2g_weno5_line(self.h, np.ascontiguousarray(F, dtype=np.float64), FP, FM, d, n))
        return FP, FM

    def weno_absgrad(self, ls, ls0, out):
        self._check(self.L.asd2g_weno_absgrad(self.h, self._f(ls), self._f(ls0), self._f(out)))

    def apply_bc_side(self, f, kind, side, fill=-1):
        self._check(self.L.asd2g_apply_bc_side(self.h, self._f(f), kind.upper().encode(), side, fill))

    def update_ntk(self, ls, nxf, nyf):
        self._check(self.L.asd2g_update_ntk(self.h, self._f(ls), self._f(nxf), self._f(nyf)))

    def csr_solve(self, solver, a, ia, ja, diag, b, tol=1e-6, maxit=100000):
        x = np.zeros(len(ia) - 1)
        it, res = C.c_int(), C.c_double()
        rc = self._check(self.L.asd2g_csr_solve(self.h, solver, len(ia) - 1, np.ascontiguousarray(ia, np.int32),
                                                np.ascontiguousarray(ja, np.int32), np.ascontiguousarray(a, float),
                                                np.ascontiguousarray(diag, float), np.ascontiguousarray(b, float), x,
                                                tol, maxit, C.byref(it), C.byref(res)))
        return x, dict(status=rc, iters=it.value, resid=res.value)

    def subcell_eno(self, ls, ls0, out):
        self._check(self.L.asd2g_subcell_eno(self.h, self._f(ls), self._f(ls0), self._f(out)))

    def eno(self, ls, ls0, out):
        self._check(self.L.asd2g_eno(self.h, self._f(ls), self._f(ls0), self._f(out)))

    def sussman_constraint(self, ls, ls0, hd, out):
        self._check(self.L.asd2g_sussman_constraint(self.h, self._f(ls), self._f(ls0), self._f(hd), self._f(out)))

    def heaviside_deriv(self, ls, out):
        self._check(self.L.asd2g_heaviside_deriv(self.h, self._f(ls), self._f(out)))

    def smoothed_sign(self, ls, out):
        self._check(self.L.asd2g_smoothed_sign(self.h, self._f(ls), self._f(out)))

    # ---- momentum ----
    def kappa(self):
        self._check(self.L.asd2g_kappa(self.h))

    def heaviside(self):
        self._check(self.L.asd2g_heaviside(self.h))

    def convection(self, u, v, cu, cv):
        self._check(self.L.asd2g_convection(self.h, *(self._f(x) for x in (u, v, cu, cv))))

    def viscosity(self, u, v, ls, h, du, dv):
        self._check(self.L.asd2g_viscosity(self.h, *(self._f(x) for x in (u, v, ls, h, du, dv))))

    def momentum_rhs(self, ls, u, v, h, fu, fv):
        self._check(self.L.asd2g_momentum_rhs(self.h, *(self._f(x) for x in (ls, u, v, h, fu, fv))))

    def intermediate_vel(self, dt, h="HS"):
        self._check(self.L.asd2g_intermediate_vel(self.h, dt, self._f(h)))

    def divergence(self, u="uhat", v="vhat", div="div"):
        self._check(self.L.asd2g_divergence(self.h, self._f(u), self._f(v), self._f(div)))

    def update_vel(self, dt):
        self._check(self.L.asd2g_update_vel(self.h, dt))

    def update_dt(self) -> float:
        d = C.c_double()
        self._check(self.L.asd2g_update_dt(self.h, C.byref(d)))
        return d.value

    # ---- pressure ----
    def assemble_gfm(self, dt, recompute_kappa=True):
        self._check(self.L.asd2g_assemble_gfm(self.h, dt, 1 if recompute_kappa else 0))

    def get_system(self):
        n = self.params.nx * self.params.ny
        arrs = [np.zeros(n) for _ in range(6)]
        pin = C.c_int()
        self._check(self.L.asd2g_get_system(self.h, *arrs, C.byref(pin)))
        return dict(diag=arrs[0], cw=arrs[1], ce=arrs[2], cs=arrs[3], cn=arrs[4], rhs=arrs[5], pinned=pin.value)

    def solve_pressure(self, solver=PCG, tol=1e-10, maxit=100000, dt=1.0):
        it, res = C.c_int(), C.c_double()
        rc = self._check(self.L.asd2g_solve_pressure(self.h, solver, tol, maxit, dt, C.byref(it), C.byref(res)))
        return dict(status=rc, iters=it.value, resid=res.value)

    def true_residual(self) -> float:
        d = C.c_double()
        self._check(self.L.asd2g_true_residual(self.h, C.byref(d)))
        return d.value

    def droplet_step(self, dt, reinit_mode=REINIT_MINRK2, solver=PCG, tol=1e-10, maxit=200000):
        d, it, res = C.c_double(dt), C.c_int(), C.c_double()
        rc = self._check(self.L.asd2g_droplet_step(self.h, C.byref(d), reinit_mode, solver, tol, maxit,
                                                   C.byref(it), C.byref(res)))
        return dict(status=rc, dt_next=d.value, iters=it.value, resid=res.value)

    # ---- axisymmetric MAC solver (x is r, y is z; base_x is kBaseR) ----
    def axi_kappa(self):
        self._check(self.L.asd2g_axi_kappa(self.h))

    def axi_rhs_u(self, dt, ls="ls", u="u", v="v", h="HS", out="w0"):
        self._check(self.L.asd2g_axi_rhs_u(self.h, dt, *(self._f(x) for x in (ls, u, v, h, out))))

    def axi_rhs_v(self, dt, ls="ls", u="u", uhat="uhat", v="v", h="HS", out="w0"):
        self._check(self.L.asd2g_axi_rhs_v(self.h, dt, *(self._f(x) for x in (ls, u, uhat, v, h, out))))

    def axi_viscosity(self, ls="ls", u="u", uhat="uhat", v="v", h="HS", du="w0", dv="w1"):
        self._check(self.L.asd2g_axi_viscosity(self.h, *(self._f(x) for x in (ls, u, uhat, v, h, du, dv))))

    def axi_hat(self, comp, dt, ls="ls", rhs="w0", h="HS", out=None):
        """GetUHat (comp 0) / GetVHat (comp 1) into out (default uhat / vhat)."""
        out = ("uhat" if comp == 0 else "vhat") if out is None else out
        self._check(self.L.asd2g_axi_hat(self.h, comp, dt, *(self._f(x) for x in (ls, rhs, h, out))))

    def axi_divergence(self, u="uhat", v="vhat", div="div", for_poisson=True):
        self._check(self.L.asd2g_axi_divergence(self.h, self._f(u), self._f(v), self._f(div),
                                                1 if for_poisson else 0))

    def axi_assemble(self, dt, recompute_kappa=True):
        self._check(self.L.asd2g_axi_assemble(self.h, dt, 1 if recompute_kappa else 0))

    def axi_update_dt(self) -> float:
        d = C.c_double()
        self._check(self.L.asd2g_axi_update_dt(self.h, C.byref(d)))
        return d.value

    def axi_step(self, dt, reinit_mode=REINIT_MINRK2, ls_bc=None, ls_bcc=None, solver=PCG, tol=1e-10,
                 maxit=200000):
        """One step of the reference's axisymmetric driver; ls_bc: the level-set
        solver's four P-grid kinds (names or asd2g_bc values; None: the
        session's pressure kinds) with constants ls_bcc."""
        kinds = consts = None
        if ls_bc is not None:
            kinds = (C.c_int32 * 4)(*[BC[k] if isinstance(k, str) else int(k) for k in ls_bc])
            consts = (C.c_double * 4)(*(ls_bcc if ls_bcc is not None else (0.0,) * 4))
        d, it, res = C.c_double(dt), C.c_int(), C.c_double()
        rc = self._check(self.L.asd2g_axi_step(self.h, C.byref(d), reinit_mode,
                                               C.cast(kinds, C.c_void_p) if kinds is not None else None,
                                               C.cast(consts, C.c_void_p) if consts is not None else None,
                                               solver, tol, maxit, C.byref(it), C.byref(res)))
        return dict(status=rc, dt_next=d.value, iters=it.value, resid=res.value)

    def run_steps(self, nsteps, dt, reinit_mode=REINIT_MINRK2, solver=MGPCG, tol=1e-10, maxit=10000):
        """nsteps droplet steps on the device (one step graph per step, the
        solver loop a device-side WHILE node, one synchronisation)."""
        d, n, it, res = C.c_double(dt), C.c_int(), C.c_longlong(), C.c_double()
        rc = self._check(self.L.asd2g_run_steps(self.h, int(nsteps), C.byref(d), reinit_mode, solver, tol, maxit,
                                                C.byref(n), C.byref(it), C.byref(res)))
        return dict(status=rc, dt_next=d.value, steps=n.value, iters=it.value, max_resid=res.value)

    def checkpoint_save(self, path, t=0.0, step=0, dt=0.0):
        """Write LS, U, V, PS, P (padded FP64) with t, step and dt to a checkpoint file."""
        self._check(self.L.asd2g_checkpoint_save(self.h, os.fsencode(path), t, step, dt))

    def checkpoint_load(self, path):
        """Replace the fields from a checkpoint; returns dict(t, step, dt)."""
        t, n, d = C.c_double(), C.c_longlong(), C.c_double()
        self._check(self.L.asd2g_checkpoint_load(self.h, os.fsencode(path), C.byref(t), C.byref(n), C.byref(d)))
        return dict(t=t.value, step=n.value, dt=d.value)

    def set_preconditioner_net(self, net):
        self._check(self.L.asd2g_set_preconditioner_net(self.h, net.h if net is not None else None))
        self._pc_net = net  # the session refers to it: keep it alive while attached

    def last_solve_one_launch(self) -> bool:
        """True when the last pressure solve ran as one kernel launch."""
        f = C.c_int()
        self._check(self.L.asd2g_last_solve_one_launch(self.h, C.byref(f)))
        return bool(f.value)

    def last_fallback(self) -> int:
        f = C.c_int()
        self._check(self.L.asd2g_last_fallback(self.h, C.byref(f)))
        return f.value

    def training_pair(self, feats, target, iters=0):
        """Learned-preconditioner training pair of the last solved system into
        device tensors: features of the residual the V-cycle leaves at the
        MG-FCG iterate after `iters` iterations, and the unit-RMS error it leaves."""
        self._check(self.L.asd2g_pc_training_pair_at(self.h, int(iters), C.c_void_p(feats.data_ptr()),
                                                     C.c_void_p(target.data_ptr())))

    def volume(self):
        """FP64 (sum H dx dy, sum HS dx dy) of the current level set."""
        a, b = C.c_double(), C.c_double()
        self._check(self.L.asd2g_volume(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def last_volume(self):
        a, b = C.c_double(), C.c_double()
        self._check(self.L.asd2g_last_volume(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value


class Batch:
    """Many GFM pressure systems of uneven sizes solved together
    (asd2g_batch_*): one kernel launch per phase for the whole batch."""

    def __init__(self, params: list, stream: int | None = None):
        self.L = load()
        self.params = list(params)
        arr = (_Params * len(self.params))(*[p.c() for p in self.params])
        h = C.c_void_p()
        self._check(self.L.asd2g_batch_create(arr, len(self.params), C.c_void_p(stream) if stream else None,
                                              C.byref(h)))
        self.h = h

    def _check(self, rc):
        if rc < 0:
            raise Asd2gError(rc, self.L.asd2g_last_error().decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.asd2g_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, inst, field, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        p = self.params[inst]
        assert a.size == (p.nx + 6) * (p.ny + 6)
        self._check(self.L.asd2g_batch_upload(self.h, inst, Session._f(field), a.ravel()))

    def download(self, inst, field):
        p = self.params[inst]
        out = np.zeros((p.nx + 6, p.ny + 6))
        self._check(self.L.asd2g_batch_download(self.h, inst, Session._f(field), out.ravel()))
        return out

    def assemble(self, dts):
        self._check(self.L.asd2g_batch_assemble(self.h, np.ascontiguousarray(dts, dtype=np.float64)))

    def solve(self, tol=1e-8, maxit=10000, solver=None):
        """Solve every assembled system; solver MGPCG (default) or UNET (the
        learned preconditioner, after set_preconditioner_net).  Returns
        dict(status, iters[count], resid[count]) and, for UNET, fallback."""
        n = len(self.params)
        it, res = np.zeros(n, np.int32), np.zeros(n)
        if solver is None or solver == MGPCG:
            rc = self._check(self.L.asd2g_batch_solve(self.h, tol, maxit, it, res))
            return dict(status=rc, iters=it, resid=res)
        rc = self._check(self.L.asd2g_batch_solve_with(self.h, solver, tol, maxit, it, res))
        fb = C.c_int()
        self._check(self.L.asd2g_batch_last_fallback(self.h, C.byref(fb)))
        return dict(status=rc, iters=it, resid=res, fallback=bool(fb.value))

    def set_preconditioner_net(self, net):
        """Copy the network's weights into the batch for solver=UNET (None detaches)."""
        self._check(self.L.asd2g_batch_set_preconditioner_net(self.h, net.h if net is not None else None))

    def step(self, dts, reinit_mode=REINIT_MINRK2, tol=1e-10, maxit=10000):
        """One full droplet step of every instance (MG-FCG pressure solve);
        returns dict(status, dt_next[count], iters[count], resid[count])."""
        n = len(self.params)
        d = np.array(dts, dtype=np.float64).copy()
        it, res = np.zeros(n, np.int32), np.zeros(n)
        rc = self._check(self.L.asd2g_batch_step(self.h, d, reinit_mode, tol, maxit, it, res))
        return dict(status=rc, dt_next=d, iters=it, resid=res)

    def volume(self):
        """(sharp, smooth) FP64 volume of every instance after the last step."""
        n = len(self.params)
        a, b = np.zeros(n), np.zeros(n)
        self._check(self.L.asd2g_batch_volume(self.h, a, b))
        return a, b

    def tile_shape(self):
        """(rows, cols) of the multigrid tiles in use and the tuning trial times (ms) per candidate."""
        r, c, ms = C.c_int(), C.c_int(), (C.c_float * 3)()
        self._check(self.L.asd2g_batch_tile_shape(self.h, C.byref(r), C.byref(c), ms))
        return (r.value, c.value), list(ms)

    def sync(self):
        self._check(self.L.asd2g_batch_sync(self.h))


UNET_LAYERS = [(4, 16, 1), (16, 16, 1), (16, 32, 1), (32, 32, 1), (32, 64, 1), (64, 64, 1), (64, 128, 1),
               (128, 128, 1), (192, 64, 1), (64, 64, 1), (96, 32, 1), (32, 32, 1), (48, 16, 1), (16, 16, 1),
               (16, 1, 0)]


def checkpoint_info(path):
    """Header of a checkpoint file after verifying its checksum (no GPU needed):
    dict(nx, ny, t, step, dt); raises Asd2gError(-7) for an invalid file."""
    L = load()
    nx, ny, t, n, d = C.c_int(), C.c_int(), C.c_double(), C.c_longlong(), C.c_double()
    rc = L.asd2g_checkpoint_info(os.fsencode(path), C.byref(nx), C.byref(ny), C.byref(t), C.byref(n), C.byref(d))
    if rc < 0:
        raise Asd2gError(rc, L.asd2g_last_error().decode())
    return dict(nx=nx.value, ny=ny.value, t=t.value, step=n.value, dt=d.value)


class UNet:
    """The learned preconditioner network (asd2g_unet_*).  Inputs and outputs
    are device tensors (torch CUDA tensors or raw device pointers)."""

    def __init__(self, max_batch, max_h, max_w, stream: int | None = None):
        self.L = load()
        h = C.c_void_p()
        rc = self.L.asd2g_unet_create(max_batch, max_h, max_w, C.c_void_p(stream) if stream else None, C.byref(h))
        self._check(rc)
        self.h = h
        self.n = int(self.L.asd2g_unet_nparams(self.h))

    def _check(self, rc):
        if rc < 0:
            raise Asd2gError(rc, self.L.asd2g_last_error().decode())
        return rc

    def close(self):
        if getattr(self, "h", None):
            self.L.asd2g_unet_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _ptr(t):
        return C.c_void_p(t if isinstance(t, int) else t.data_ptr())

    def init(self, seed=0):
        self._check(self.L.asd2g_unet_init(self.h, seed))

    def params(self):
        a = np.zeros(self.n, np.float32)
        self._check(self.L.asd2g_unet_get_params(self.h, a))
        return a

    def set_params(self, a):
        self._check(self.L.asd2g_unet_set_params(self.h, np.ascontiguousarray(a, dtype=np.float32)))

    def grads(self):
        a = np.zeros(self.n, np.float32)
        self._check(self.L.asd2g_unet_get_grads(self.h, a))
        return a

    def forward(self, feats, out, B, H, W):
        self._check(self.L.asd2g_unet_forward(self.h, B, H, W, self._ptr(feats), self._ptr(out)))

    def train_step(self, feats, target, B, H, W, lr):
        loss = C.c_float()
        self._check(self.L.asd2g_unet_train_step(self.h, B, H, W, self._ptr(feats), self._ptr(target), lr,
                                                 C.byref(loss)))
        return loss.value

    def train_step_residual(self, feats, B, H, W, lr):
        """Adam step on the residual loss 1 - cos^2(A out, r) (r = feats[..., 0],
        A the 5-point operator of feats[..., 1:4]); returns the mean loss."""
        loss = C.c_float()
        self._check(self.L.asd2g_unet_train_step_residual(self.h, B, H, W, self._ptr(feats), lr, C.byref(loss)))
        return loss.value

    def train_step_energy(self, feats, target, B, H, W, lr):
        """Adam step on the energy loss 1 - (u'At)^2 / ((u'Au)(t'At)) (A the
        5-point operator of feats[..., 1:4]); returns the mean loss."""
        loss = C.c_float()
        self._check(self.L.asd2g_unet_train_step_energy(self.h, B, H, W, self._ptr(feats), self._ptr(target), lr,
                                                        C.byref(loss)))
        return loss.value

    def error_flag(self):
        f = C.c_int()
        self._check(self.L.asd2g_unet_error_flag(self.h, C.byref(f)))
        return f.value

    @staticmethod
    def layout():
        """(w_offset, b_offset, cin, cout, relu) of each layer in the flat parameter vector."""
        out, off = [], 0
        for cin, cout, relu in UNET_LAYERS:
            wo = off
            off += cout * cin * 9
            bo = off
            off += (cout + 15) // 16 * 16
            out.append((wo, bo, cin, cout, relu))
        return out, off

