"""ctypes bindings for the two CPU checkers.

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() and
by bench.py's CPU-baseline leg.  The product package never imports this.

* ``Oracle`` wraps liboracle.so, the plain-C restatement in asd2_oracle.c.
* ``Reference`` wraps _ref/libasd2ref.so, the reference's own sources compiled
  unmodified against the shims in ref_shim/ (present only where the reference
  tree was available at build time).

All field arrays are float64 numpy arrays of shape (nx+6, ny+6) in C order,
which is exactly the reference layout idx(i,j) = j + (ny+6)*i.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libasd2ref.so")

# BC2D order (include/common.h:4)
BC_NAMES = ["periodic", "neumann", "dirichlet", "axisym", "wall", "inlet", "outlet",
            "pressure", "lsfree", "custom"]
BC = {n: i for i, n in enumerate(BC_NAMES)}

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_u8 = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


class _Grid(C.Structure):
    _fields_ = [("nx", C.c_int32), ("ny", C.c_int32), ("dx", C.c_double), ("dy", C.c_double),
                ("bc_u", C.c_int32 * 4), ("bc_v", C.c_int32 * 4), ("bc_p", C.c_int32 * 4),
                ("cu", C.c_double * 4), ("cv", C.c_double * 4), ("cp", C.c_double * 4)]


class _Fluid(C.Structure):
    _fields_ = [("rho_h", C.c_double), ("rho_l", C.c_double), ("mu_h", C.c_double), ("mu_l", C.c_double),
                ("sigma", C.c_double), ("g", C.c_double), ("g_axis", C.c_int32), ("fix_gravity", C.c_int32),
                ("time_order", C.c_int32), ("cfl", C.c_double)]


@dataclass
class GridSpec:
    """Grid, spacing and the W/E/S/N boundary names of the U, V and P grids."""
    nx: int
    ny: int
    dx: float
    dy: float
    bc_u: tuple = ("dirichlet",) * 4
    bc_v: tuple = ("dirichlet",) * 4
    bc_p: tuple = ("neumann",) * 4
    cu: tuple = (0.0,) * 4
    cv: tuple = (0.0,) * 4
    cp: tuple = (0.0,) * 4

    @property
    def shape(self):
        return (self.nx + 6, self.ny + 6)

    def zeros(self):
        return np.zeros(self.shape)

    def c(self) -> _Grid:
        g = _Grid()
        g.nx, g.ny, g.dx, g.dy = self.nx, self.ny, self.dx, self.dy
        for k in range(4):
            g.bc_u[k] = BC[self.bc_u[k]]
            g.bc_v[k] = BC[self.bc_v[k]]
            g.bc_p[k] = BC[self.bc_p[k]]
            g.cu[k], g.cv[k], g.cp[k] = self.cu[k], self.cv[k], self.cp[k]
        return g


@dataclass
class FluidSpec:
    rho_h: float = 1000.0
    rho_l: float = 1.0
    mu_h: float = 1.0e-3
    mu_l: float = 1.0e-5
    sigma: float = 0.0728
    g: float = 9.8
    g_axis: int = 1           # GAXISENUM2D::Y
    fix_gravity: int = 0      # 0 reproduces the reference (no gravity on V for axis Y)
    time_order: int = 2       # RK3
    cfl: float = 0.5

    def c(self) -> _Fluid:
        f = _Fluid()
        for k, _ in _Fluid._fields_:
            setattr(f, k, getattr(self, k))
        return f


def _load(path):
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    return C.CDLL(path)


class Oracle:
    """The C restatement (asd2_oracle.c)."""

    def __init__(self, path: str = ORACLE_SO):
        L = self.L = _load(path)
        G, F = C.POINTER(_Grid), C.POINTER(_Fluid)
        sig = {
            "ora_bc_u": [G, _dp], "ora_bc_v": [G, _dp], "ora_bc_p": [G, _dp],
            "ora_unit_weno5": [_dp, _dp, _dp, C.c_double, C.c_int],
            "ora_ls_weno_rhs": [G, _dp, _dp, _dp, _dp],
            "ora_ls_advect": [G, _dp, _dp, _dp, C.c_double],
            "ora_smoothed_sign": [G, _dp, _dp], "ora_heaviside_deriv": [G, _dp, _dp],
            "ora_eno_absgrad": [G, _dp, _dp, _dp], "ora_subcell_eno_absgrad": [G, _dp, _dp, _dp],
            "ora_sussman_constraint": [G, _dp, _dp, _dp, _dp],
            "ora_reinit": [G, C.c_int, C.c_double, _dp],
            "ora_kappa": [G, _dp, _dp], "ora_ntk": [G, _dp, _dp, _dp], "ora_heaviside": [G, _dp, _dp], "ora_smooth_heaviside": [G, _dp, _dp],
            "ora_conv_u": [G, _dp, _dp, _dp], "ora_conv_v": [G, _dp, _dp, _dp],
            "ora_visc_u": [G, F, _dp, _dp, _dp, _dp, _dp], "ora_visc_v": [G, F, _dp, _dp, _dp, _dp, _dp],
            "ora_rhs_u": [G, F, _dp, _dp, _dp, _dp, _dp], "ora_rhs_v": [G, F, _dp, _dp, _dp, _dp, _dp],
            "ora_intermediate_vel": [G, F, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp],
            "ora_divergence": [G, _dp, _dp, _dp],
            "ora_update_vel": [G, F, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp, _dp, _dp],
            "ora_gfm_assemble": [G, F, C.c_double, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp],
            "ora_gfm_to_csr": [G, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _ip, _ip, _dp],
            "ora_gfm_apply": [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp],
            "ora_pcg": [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, C.c_double, C.c_int,
                        C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)],
            "ora_bicgstab": [C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, C.c_double, C.c_int,
                             C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)],
            "ora_gather": [G, _dp, _dp], "ora_scatter": [G, _dp, _dp],
            "ora_interface_mask": [G, _dp, _u8], "ora_ghost_face_mask": [G, _dp, _u8],
            "ora_axi_kappa": [G, C.c_double, _dp, _dp],
            "ora_axi_visc_u": [G, F, _dp, _dp, _dp, _dp, _dp],
            "ora_axi_visc_v": [G, F, _dp, _dp, _dp, _dp, _dp, _dp],
            "ora_axi_rhs_u": [G, F, C.c_double, _dp, _dp, _dp, _dp, _dp],
            "ora_axi_rhs_v": [G, F, C.c_double, _dp, _dp, _dp, _dp, _dp, _dp],
            "ora_axi_uhat": [G, F, C.c_double, _dp, _dp, _dp, _dp],
            "ora_axi_vhat": [G, F, C.c_double, _dp, _dp, _dp, _dp],
            "ora_axi_div4p": [G, C.c_double, _dp, _dp, _dp],
            "ora_axi_divergence": [G, C.c_double, _dp, _dp, _dp],
            "ora_axi_assemble": [G, F, C.c_double, C.c_double, _dp, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp, _dp,
                                 _dp, _dp],
        }
        for name, args in sig.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = None
        L.ora_update_dt.argtypes = [G, F, _dp, _dp]
        L.ora_update_dt.restype = C.c_double
        L.ora_reinit_steps.argtypes = [G, C.c_double]
        L.ora_reinit_steps.restype = C.c_int
        L.ora_gfm_assemble.restype = C.c_int
        L.ora_gfm_to_csr.restype = C.c_int
        L.ora_pcg.restype = C.c_int
        L.ora_bicgstab.restype = C.c_int
        L.ora_axi_assemble.restype = C.c_int
        L.ora_axi_update_dt.argtypes = [G, F, _dp, _dp, _dp]
        L.ora_axi_update_dt.restype = C.c_double

    # ---- boundary ----
    def bc(self, g: GridSpec, kind: str, a: np.ndarray) -> np.ndarray:
        getattr(self.L, "ora_bc_" + kind.lower())(C.byref(g.c()), a)
        return a

    # ---- level set ----
    def unit_weno5(self, F, d, n):
        FP, FM = np.zeros(n + 6), np.zeros(n + 6)
        self.L.ora_unit_weno5(np.ascontiguousarray(F, dtype=np.float64), FP, FM, d, n)
        return FP, FM

    def ls_weno_rhs(self, g, ls, u, v):
        out = g.zeros()
        self.L.ora_ls_weno_rhs(C.byref(g.c()), ls, u, v, out)
        return out

    def ls_advect(self, g, ls, u, v, dt):
        self.L.ora_ls_advect(C.byref(g.c()), ls, u, v, dt)
        return ls

    def reinit(self, g, mode: int, ls, max_atime: float = 0.0):
        self.L.ora_reinit(C.byref(g.c()), mode, max_atime, ls)
        return ls

    def reinit_steps(self, g, max_atime: float = 0.0) -> int:
        return self.L.ora_reinit_steps(C.byref(g.c()), max_atime)

    def _unary(self, name, g, *arrs):
        out = g.zeros()
        getattr(self.L, name)(C.byref(g.c()), *arrs, out)
        return out

    def smoothed_sign(self, g, ls): return self._unary("ora_smoothed_sign", g, ls)
    def heaviside_deriv(self, g, ls): return self._unary("ora_heaviside_deriv", g, ls)
    def eno_absgrad(self, g, ls, ls0): return self._unary("ora_eno_absgrad", g, ls, ls0)
    def subcell_eno_absgrad(self, g, ls, ls0): return self._unary("ora_subcell_eno_absgrad", g, ls, ls0)
    def sussman_constraint(self, g, ls, ls0, hd): return self._unary("ora_sussman_constraint", g, ls, ls0, hd)
    def heaviside(self, g, ls): return self._unary("ora_heaviside", g, ls)

    def ntk(self, g, ls, nxo, nyo):
        """UpdateNTK's unit normal into nxo / nyo (cells it skips keep their values)."""
        self.L.ora_ntk(C.byref(g.c()), ls, nxo, nyo)
        return nxo, nyo
    def smooth_heaviside(self, g, ls): return self._unary("ora_smooth_heaviside", g, ls)
    def conv_u(self, g, u, v): return self._unary("ora_conv_u", g, u, v)
    def conv_v(self, g, u, v): return self._unary("ora_conv_v", g, u, v)
    def divergence(self, g, u, v): return self._unary("ora_divergence", g, u, v)

    def kappa(self, g, ls, kappa=None):
        k = g.zeros() if kappa is None else kappa
        self.L.ora_kappa(C.byref(g.c()), ls, k)
        return k

    def visc_u(self, g, f, u, v, ls, H):
        out = g.zeros()
        self.L.ora_visc_u(C.byref(g.c()), C.byref(f.c()), u, v, ls, H, out)
        return out

    def visc_v(self, g, f, u, v, ls, H):
        out = g.zeros()
        self.L.ora_visc_v(C.byref(g.c()), C.byref(f.c()), u, v, ls, H, out)
        return out

    def rhs_u(self, g, f, ls, u, v, H):
        out = g.zeros()
        self.L.ora_rhs_u(C.byref(g.c()), C.byref(f.c()), ls, u, v, H, out)
        return out

    def rhs_v(self, g, f, ls, u, v, H):
        out = g.zeros()
        self.L.ora_rhs_v(C.byref(g.c()), C.byref(f.c()), ls, u, v, H, out)
        return out

    def intermediate_vel(self, g, f, dt, ls, u, v, H):
        uh, vh = g.zeros(), g.zeros()
        self.L.ora_intermediate_vel(C.byref(g.c()), C.byref(f.c()), dt, ls, u, v, uh, vh, H)
        return uh, vh

    def update_vel(self, g, f, dt, u, v, us, vs, ps, ls, H, kappa):
        self.L.ora_update_vel(C.byref(g.c()), C.byref(f.c()), dt, u, v, us, vs, ps, ls, H, kappa)
        return u, v

    def update_dt(self, g, f, u, v) -> float:
        return self.L.ora_update_dt(C.byref(g.c()), C.byref(f.c()), u, v)

    # ---- GFM pressure ----
    def gfm_assemble(self, g, f, dt, ls, kappa, H, div, recompute_kappa=True):
        n = g.nx * g.ny
        d, cw, ce, cs, cn, rhs = (np.zeros(n) for _ in range(6))
        pinned = self.L.ora_gfm_assemble(C.byref(g.c()), C.byref(f.c()), dt, ls, kappa, H, div,
                                         1 if recompute_kappa else 0, d, cw, ce, cs, cn, rhs)
        return dict(diag=d, cw=cw, ce=ce, cs=cs, cn=cn, rhs=rhs, pinned=pinned)

    def gfm_to_csr(self, g, sysd):
        n = g.nx * g.ny
        a, ia, ja, b = np.zeros(5 * n), np.zeros(n + 1, np.int32), np.zeros(5 * n, np.int32), np.zeros(n)
        rows = self.L.ora_gfm_to_csr(C.byref(g.c()), sysd["diag"], sysd["cw"], sysd["ce"], sysd["cs"],
                                     sysd["cn"], sysd["rhs"], sysd["pinned"], a, ia, ja, b)
        nnz = int(ia[rows])
        return a[:nnz].copy(), ia[:rows + 1].copy(), ja[:nnz].copy(), b[:rows].copy()

    def gfm_apply(self, g, sysd, x):
        y = np.zeros(g.nx * g.ny)
        self.L.ora_gfm_apply(g.nx, g.ny, sysd["diag"], sysd["cw"], sysd["ce"], sysd["cs"], sysd["cn"],
                             sysd["pinned"], np.ascontiguousarray(x, dtype=np.float64), y)
        return y

    def pcg(self, g, sysd, tol=1e-10, maxit=100000, mode=0, b=None):
        x = np.zeros(g.nx * g.ny)
        r, tr = C.c_double(), C.c_double()
        bb = sysd["rhs"] if b is None else np.ascontiguousarray(b, dtype=np.float64)
        it = self.L.ora_pcg(g.nx, g.ny, sysd["diag"], sysd["cw"], sysd["ce"], sysd["cs"], sysd["cn"],
                            sysd["pinned"], bb, x, tol, maxit, mode, C.byref(r), C.byref(tr))
        return x, it, r.value, tr.value

    def bicgstab(self, g, sysd, tol=1e-10, maxit=100000, mode=0):
        x = np.zeros(g.nx * g.ny)
        r, tr = C.c_double(), C.c_double()
        it = self.L.ora_bicgstab(g.nx, g.ny, sysd["diag"], sysd["cw"], sysd["ce"], sysd["cs"], sysd["cn"],
                                 sysd["pinned"], sysd["rhs"], x, tol, maxit, mode, C.byref(r), C.byref(tr))
        return x, it, r.value, tr.value

    def gather(self, g, padded):
        out = np.zeros(g.nx * g.ny)
        self.L.ora_gather(C.byref(g.c()), padded, out)
        return out

    def scatter(self, g, nat, padded=None):
        p = g.zeros() if padded is None else padded
        self.L.ora_scatter(C.byref(g.c()), np.ascontiguousarray(nat, dtype=np.float64), p)
        return p

    def interface_mask(self, g, ls0):
        m = np.zeros(g.nx * g.ny, np.uint8)
        self.L.ora_interface_mask(C.byref(g.c()), ls0, m)
        return m

    def ghost_face_mask(self, g, ls):
        m = np.zeros(g.nx * g.ny, np.uint8)
        self.L.ora_ghost_face_mask(C.byref(g.c()), ls, m)
        return m

    # ---- composed droplet step (tests/LargeTests/test_mac2d_large.cpp:496-552) ----
    def droplet_step(self, g, f, st, tol=1e-10, maxit=200000, reinit_mode=2, pcg_mode=0, bicgstab_mode=None):
        """One full two-phase step in the driver's order, with the pressure
        system solved by the fixed-order FP64 PCG to ``tol`` (``pcg_mode`` 1:
        the reference's own CG iteration; ``bicgstab_mode`` not None: BiCGStab
        in that mode instead of CG).  ``st`` is a dict
        with ls, u, v, ps, p, kappa (padded) and dt; it is updated in place and
        the Poisson statistics are returned."""
        ls, u, v = st["ls"], st["u"], st["v"]
        dt = st["dt"]
        lsB = ls.copy()
        self.ls_advect(g, ls, u, v, dt)
        self.bc(g, "p", ls)
        self.reinit(g, reinit_mode, ls)
        self.bc(g, "p", ls)
        self.kappa(g, ls, st["kappa"])
        H = self.heaviside(g, ls)
        HS = self.smooth_heaviside(g, ls)
        uh, vh = self.intermediate_vel(g, f, dt, ls, u, v, HS)
        self.bc(g, "u", uh)
        self.bc(g, "v", vh)
        div = self.divergence(g, uh, vh)
        sysd = self.gfm_assemble(g, f, dt, ls, st["kappa"], H, div, recompute_kappa=f.sigma != 0.0)
        if bicgstab_mode is None:
            x, it, res, tres = self.pcg(g, sysd, tol=tol, maxit=maxit, mode=pcg_mode)
        else:
            x, it, res, tres = self.bicgstab(g, sysd, tol=tol, maxit=maxit, mode=bicgstab_mode)
        ps = g.zeros()
        self.scatter(g, x, ps)
        self.bc(g, "p", ps)
        st["ps"] = ps
        p = g.zeros()
        p[3:-3, 3:-3] = ps[3:-3, 3:-3] / dt
        st["p"] = p
        self.update_vel(g, f, dt, u, v, uh, vh, ps, ls, H, st["kappa"])
        st["dt_used"] = dt
        st["dt"] = self.update_dt(g, f, u, v)
        st["lsB"] = lsB
        return dict(iters=it, resid=res, true_resid=tres, sys=sysd, div=div, H=H, HS=HS, uhat=uh, vhat=vh)


    # ---- axisymmetric MAC solver (mac2dAxisym.cpp); x is r, y is z ----
    def axi_kappa(self, g, base_r, ls, kappa=None):
        k = g.zeros() if kappa is None else kappa
        self.L.ora_axi_kappa(C.byref(g.c()), base_r, ls, k)
        return k

    def axi_visc(self, g, f, u, uhat, v, ls, H):
        a, b = g.zeros(), g.zeros()
        self.L.ora_axi_visc_u(C.byref(g.c()), C.byref(f.c()), u, v, ls, H, a)
        self.L.ora_axi_visc_v(C.byref(g.c()), C.byref(f.c()), u, uhat, v, ls, H, b)
        return a, b

    def axi_rhs_u(self, g, f, dt, ls, u, v, H):
        out = g.zeros()
        self.L.ora_axi_rhs_u(C.byref(g.c()), C.byref(f.c()), dt, ls, u, v, H, out)
        return out

    def axi_rhs_v(self, g, f, dt, ls, u, uhat, v, H):
        out = g.zeros()
        self.L.ora_axi_rhs_v(C.byref(g.c()), C.byref(f.c()), dt, ls, u, uhat, v, H, out)
        return out

    def axi_uhat(self, g, f, dt, ls, rhs, H):
        out = g.zeros()
        self.L.ora_axi_uhat(C.byref(g.c()), C.byref(f.c()), dt, ls, rhs, H, out)
        return out

    def axi_vhat(self, g, f, dt, ls, rhs, H):
        out = g.zeros()
        self.L.ora_axi_vhat(C.byref(g.c()), C.byref(f.c()), dt, ls, rhs, H, out)
        return out

    def axi_div4p(self, g, base_r, u, v):
        out = g.zeros()
        self.L.ora_axi_div4p(C.byref(g.c()), base_r, u, v, out)
        return out

    def axi_divergence(self, g, base_r, u, v):
        out = g.zeros()
        self.L.ora_axi_divergence(C.byref(g.c()), base_r, u, v, out)
        return out

    def axi_assemble(self, g, f, base_r, dt, ls, kappa, H, div, recompute_kappa=True):
        n = g.nx * g.ny
        d, cw, ce, cs, cn, rhs = (np.zeros(n) for _ in range(6))
        pinned = self.L.ora_axi_assemble(C.byref(g.c()), C.byref(f.c()), base_r, dt, ls, kappa, H, div,
                                         1 if recompute_kappa else 0, d, cw, ce, cs, cn, rhs)
        return dict(diag=d, cw=cw, ce=ce, cs=cs, cn=cn, rhs=rhs, pinned=pinned)

    def axi_update_dt(self, g, f, u, v, kappa) -> float:
        return self.L.ora_axi_update_dt(C.byref(g.c()), C.byref(f.c()), u, v, kappa)

    def axi_step(self, g, f, st, base_r=0.0, ls_grid=None, tol=1e-10, maxit=200000, reinit_mode=2, pcg_mode=0):
        """One step of the reference's axisymmetric driver
        (tests/LargeTests/test_mac2d_large.cpp:1264-1303): level set advected
        and reinitialised on ``ls_grid`` (the level-set solver's boundary
        kinds; default g), curvature, Heaviside, the implicit viscous uhat and
        vhat, the r-weighted divergence, the assembly solved by the
        fixed-order FP64 PCG to ``tol`` (``pcg_mode`` 1: the reference's own CG
        iteration), the projection and the next dt.
        ``st`` holds ls, u, v, kappa (padded) and dt; updated in place."""
        lg = g if ls_grid is None else ls_grid
        ls, u, v = st["ls"], st["u"], st["v"]
        dt = st["dt"]
        lsB = ls.copy()
        self.ls_advect(lg, ls, u, v, dt)
        self.bc(lg, "p", ls)
        self.reinit(lg, reinit_mode, ls)
        self.bc(lg, "p", ls)
        self.axi_kappa(g, base_r, ls, st["kappa"])
        H = self.heaviside(g, ls)
        HS = self.smooth_heaviside(g, ls)
        rhs_u = self.axi_rhs_u(g, f, dt, ls, u, v, HS)
        uh = self.axi_uhat(g, f, dt, ls, rhs_u, HS)
        self.bc(g, "u", uh)
        rhs_v = self.axi_rhs_v(g, f, dt, ls, u, uh, v, HS)
        vh = self.axi_vhat(g, f, dt, ls, rhs_v, HS)
        self.bc(g, "v", vh)
        div = self.axi_div4p(g, base_r, uh, vh)
        self.bc(lg, "p", ls)  # the driver fills the level set again here (:1294)
        sysd = self.axi_assemble(g, f, base_r, dt, ls, st["kappa"], H, div, recompute_kappa=f.sigma != 0.0)
        x, it, res, tres = self.pcg(g, sysd, tol=tol, maxit=maxit, mode=pcg_mode)
        ps = g.zeros()
        self.scatter(g, x, ps)
        self.bc(g, "p", ps)  # SolvePoisson's own fill
        self.bc(g, "p", ps)  # and the driver's (:1299); with mixed kinds the corners differ after the second
        st["ps"] = ps
        self.update_vel(g, f, dt, u, v, uh, vh, ps, ls, H, st["kappa"])
        self.bc(g, "u", u)  # the driver's fills after UpdateVel's own (:1304-1305)
        self.bc(g, "v", v)
        st["dt_used"] = dt
        st["dt"] = self.axi_update_dt(g, f, u, v, st["kappa"])
        return dict(iters=it, resid=res, true_resid=tres, sys=sysd, div=div, H=H, HS=HS, uhat=uh, vhat=vh,
                    rhs_u=rhs_u, rhs_v=rhs_v)


class Reference:
    """The reference's own classes, compiled unmodified (oracle/_ref)."""

    def __init__(self, g: GridSpec, f: FluidSpec | None = None, len_x=None, len_y=None,
                 base_x=0.0, base_y=0.0, ls_max_atime=0.0, path: str = REF_SO):
        L = self.L = _load(path)
        f = f or FluidSpec()
        self.g = g
        L.ref_create.restype = C.c_void_p
        L.ref_create.argtypes = [C.c_int, C.c_int] + [C.c_double] * 9 + [C.c_int, C.c_double, C.c_int,
                                                                          C.c_double, C.c_double]
        lx = g.dx * g.nx if len_x is None else len_x
        ly = g.dy * g.ny if len_y is None else len_y
        self.h = C.c_void_p(L.ref_create(g.nx, g.ny, base_x, base_y, lx, ly, f.rho_h, f.rho_l, f.mu_h, f.mu_l,
                                         f.g, f.g_axis, f.sigma, f.time_order, f.cfl, ls_max_atime))
        V = C.c_void_p
        for name, args, res in [
            ("ref_set_bc", [V, C.c_int, C.c_char, C.c_char_p], None),
            ("ref_set_bc_const", [V, C.c_int, C.c_char, _dp], None),
            ("ref_apply_bc", [V, C.c_int, C.c_char, _dp], None),
            ("ref_ls_advect", [V, _dp, _dp, _dp, C.c_double], None),
            ("ref_ls_weno_rhs", [V, _dp, _dp, _dp, _dp], None),
            ("ref_unit_weno5", [V, _dp, _dp, _dp, C.c_double, C.c_int], None),
            ("ref_reinit", [V, C.c_int, _dp], None),
            ("ref_subcell_eno", [V, _dp, _dp, _dp], None), ("ref_eno", [V, _dp, _dp, _dp], None),
            ("ref_weno_absgrad", [V, _dp, _dp, _dp], None),
            ("ref_sussman_constraint", [V, _dp, _dp, _dp, _dp], None),
            ("ref_heaviside_deriv", [V, _dp, _dp], None), ("ref_smoothed_sign", [V, _dp, _dp], None),
            ("ref_mac_set_state", [V, _dp, _dp, _dp, C.c_double], None),
            ("ref_mac_get_state", [V, _dp, _dp, _dp, _dp, _dp], C.c_double),
            ("ref_mac_set_kappa", [V, _dp], None),
            ("ref_mac_kappa", [V, _dp, _dp], None), ("ref_mac_ntk", [V, _dp, _dp, _dp], None), ("ref_mac_heaviside", [V, _dp, _dp, _dp], None),
            ("ref_mac_conv", [V, _dp, _dp, _dp, _dp], None),
            ("ref_mac_visc", [V, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_mac_rhs", [V, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_mac_intermediate", [V, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_mac_div", [V, _dp, _dp, _dp], None),
            ("ref_mac_outres", [V, C.c_int, C.c_int, C.c_double, C.c_char_p, C.c_char_p, _dp, _dp, _dp, _dp],
             C.c_int),
            ("ref_mac_poisson", [V, _dp, _dp, _dp, _dp, _dp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)], C.c_int),
            ("ref_capture_copy", [_dp, _ip, _ip, _dp], C.c_int),
            ("ref_mac_cg", [V, _dp, _dp, _dp, _ip, _ip, C.c_int, _dp, C.c_int], None),
            ("ref_mac_bicgstab", [V, _dp, _dp, _dp, _ip, _ip, C.c_int, _dp, C.c_int], None),
            ("ref_mac_update_vel", [V, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_mac_update_dt", [V, _dp, _dp], C.c_double),
            ("ref_destroy", [V], None),
        ]:
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        for which in (0, 1):
            for kind, names, consts in (("U", g.bc_u, g.cu), ("V", g.bc_v, g.cv), ("P", g.bc_p, g.cp)):
                L.ref_set_bc(self.h, which, kind.encode(), " ".join(names).encode())
                L.ref_set_bc_const(self.h, which, kind.encode(), np.array(consts, dtype=np.float64))

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def z(self):
        return self.g.zeros()

    def bc(self, kind, a, which=0):
        self.L.ref_apply_bc(self.h, which, kind.upper().encode(), a)
        return a

    def ls_advect(self, ls, u, v, dt):
        self.L.ref_ls_advect(self.h, ls, u, v, dt)
        return ls

    def ls_weno_rhs(self, ls, u, v):
        out = self.z()
        self.L.ref_ls_weno_rhs(self.h, ls, u, v, out)
        return out

    def unit_weno5(self, F, d, n):
        FP, FM = np.zeros(n + 6), np.zeros(n + 6)
        self.L.ref_unit_weno5(self.h, np.ascontiguousarray(F, dtype=np.float64), FP, FM, d, n)
        return FP, FM

    def reinit(self, mode, ls):
        self.L.ref_reinit(self.h, mode, ls)
        return ls

    def outres(self, m_iter, it, t, vel_base, div_base, u, v, ps, ls):
        """MACSolver2D::OutRes (Tecplot ASCII) into <base>_ASCII.plt."""
        return self.L.ref_mac_outres(self.h, m_iter, it, t, os.fsencode(vel_base), os.fsencode(div_base), u, v, ps,
                                     ls)

    def _u(self, name, *arrs):
        out = self.z()
        getattr(self.L, name)(self.h, *arrs, out)
        return out

    def subcell_eno_absgrad(self, ls, ls0): return self._u("ref_subcell_eno", ls, ls0)
    def eno_absgrad(self, ls, ls0): return self._u("ref_eno", ls, ls0)
    def sussman_constraint(self, ls, ls0, hd): return self._u("ref_sussman_constraint", ls, ls0, hd)
    def heaviside_deriv(self, ls): return self._u("ref_heaviside_deriv", ls)
    def smoothed_sign(self, ls): return self._u("ref_smoothed_sign", ls)

    def set_state(self, u, v, ps, dt):
        self.L.ref_mac_set_state(self.h, u, v, ps, dt)

    def get_state(self):
        u, v, ps, p, k = (self.z() for _ in range(5))
        dt = self.L.ref_mac_get_state(self.h, u, v, ps, p, k)
        return dict(u=u, v=v, ps=ps, p=p, kappa=k, dt=dt)

    def set_kappa(self, k):
        self.L.ref_mac_set_kappa(self.h, k)

    def kappa(self, ls): return self._u("ref_mac_kappa", ls)

    def ntk(self, ls, nxo, nyo):
        self.L.ref_mac_ntk(self.h, ls, nxo, nyo)
        return nxo, nyo

    def heaviside(self, ls):
        H, HS = self.z(), self.z()
        self.L.ref_mac_heaviside(self.h, ls, H, HS)
        return H, HS

    def conv(self, u, v):
        a, b = self.z(), self.z()
        self.L.ref_mac_conv(self.h, u, v, a, b)
        return a, b

    def visc(self, u, v, ls, H):
        a, b = self.z(), self.z()
        self.L.ref_mac_visc(self.h, u, v, ls, H, a, b)
        return a, b

    def rhs(self, ls, u, v, H):
        a, b = self.z(), self.z()
        self.L.ref_mac_rhs(self.h, ls, u, v, H, a, b)
        return a, b

    def intermediate_vel(self, ls, u, v, H):
        uh, vh = self.z(), self.z()
        self.L.ref_mac_intermediate(self.h, ls, u, v, uh, vh, H)
        return uh, vh

    def divergence(self, u, v): return self._u("ref_mac_div", u, v)

    def poisson_capture(self, div, ls, lsB, H, maxiter=0):
        """SolvePoisson with maxiter CG iterations; returns ps and the
        reference-assembled CSR system (a, ia, ja, b)."""
        ps = self.z()
        m, nnz, nb = C.c_int(), C.c_int(), C.c_int()
        rc = self.L.ref_mac_poisson(self.h, ps, div, ls, lsB, H, maxiter, C.byref(m), C.byref(nnz), C.byref(nb))
        if rc != 0:
            raise RuntimeError("no system captured")
        a, ia, ja, b = np.zeros(nnz.value), np.zeros(m.value + 1, np.int32), np.zeros(nnz.value, np.int32), \
            np.zeros(nb.value)
        self.L.ref_capture_copy(a, ia, ja, b)
        return ps, (a, ia, ja, b)

    def cg(self, rhs_padded, csr, mdiag, maxiter):
        a, ia, ja = csr
        ps = self.z()
        self.L.ref_mac_cg(self.h, ps, rhs_padded, a, ia, ja, len(ia) - 1, mdiag, maxiter)
        return ps

    def bicgstab(self, rhs_padded, csr, mdiag, maxiter):
        a, ia, ja = csr
        ps = self.z()
        self.L.ref_mac_bicgstab(self.h, ps, rhs_padded, a, ia, ja, len(ia) - 1, mdiag, maxiter)
        return ps

    def update_vel(self, uhat, vhat, ps, ls, lsB, H):
        self.L.ref_mac_update_vel(self.h, uhat, vhat, ps, ls, lsB, H)

    def update_dt(self, u, v) -> float:
        return self.L.ref_mac_update_dt(self.h, u, v)


class AxiReference:
    """The reference's MACSolver2DAxisym, compiled unmodified (oracle/_ref).
    Grid x is r, y is z; gravity axis 0 = R, 1 = Z."""

    def __init__(self, g: GridSpec, f: FluidSpec | None = None, base_r=0.0, base_z=0.0, len_r=None, len_z=None,
                 path: str = REF_SO):
        """len_r / len_z: the domain lengths the reference divides by nr / nz
        for its spacings (default dr * nr, dz * nz)."""
        L = self.L = _load(path)
        f = f or FluidSpec()
        self.g = g
        V = C.c_void_p
        L.ref_axi_create.restype = V
        L.ref_axi_create.argtypes = [C.c_int, C.c_int] + [C.c_double] * 9 + [C.c_int, C.c_double, C.c_double]
        lr = g.dx * g.nx if len_r is None else len_r
        lz = g.dy * g.ny if len_z is None else len_z
        self.h = V(L.ref_axi_create(g.nx, g.ny, base_r, base_z, lr, lz, f.rho_h, f.rho_l, f.mu_h,
                                    f.mu_l, f.g, f.g_axis, f.sigma, f.cfl))
        for name, args, res in [
            ("ref_axi_set_bc", [V, C.c_char, C.c_char_p, _dp], None),
            ("ref_axi_tdma", [V, _dp, _dp, _dp, _dp, C.c_int], C.c_int),
            ("ref_axi_apply_bc", [V, C.c_char, _dp], None),
            ("ref_axi_set_state", [V, _dp, _dp, _dp, C.c_double], None),
            ("ref_axi_get_state", [V, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_kappa", [V, _dp, _dp], None),
            ("ref_axi_visc", [V, _dp, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_rhs_u", [V, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_rhs_v", [V, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_uhat", [V, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_vhat", [V, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_div", [V, _dp, _dp, _dp, _dp], None),
            ("ref_axi_poisson", [V, _dp, _dp, _dp, _dp, _dp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                 C.POINTER(C.c_int)], C.c_int),
            ("ref_capture_copy", [_dp, _ip, _ip, _dp], C.c_int),
            ("ref_axi_update_vel", [V, _dp, _dp, _dp, _dp, _dp, _dp], None),
            ("ref_axi_update_dt", [V, _dp, _dp], C.c_double),
            ("ref_axi_destroy", [V], None),
        ]:
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        for kind, names, consts in (("U", g.bc_u, g.cu), ("V", g.bc_v, g.cv), ("P", g.bc_p, g.cp)):
            L.ref_axi_set_bc(self.h, kind.encode(), " ".join(names).encode(), np.array(consts, dtype=np.float64))

    def close(self):
        if self.h:
            self.L.ref_axi_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def z(self):
        return self.g.zeros()

    def bc(self, kind, a):
        self.L.ref_axi_apply_bc(self.h, kind.upper().encode(), a)
        return a

    def set_state(self, u, v, kappa, dt):
        self.L.ref_axi_set_state(self.h, u, v, kappa, dt)

    def get_state(self):
        u, v, ps, p, k = (self.z() for _ in range(5))
        self.L.ref_axi_get_state(self.h, u, v, ps, p, k)
        return dict(u=u, v=v, ps=ps, p=p, kappa=k)

    def tdma(self, a, b, c, d):
        """SolveTDMA on copies; returns (c, d) as the reference leaves them."""
        f = lambda x: np.array(x, dtype=np.float64)
        a, b, c, d = f(a), f(b), f(c), f(d)
        rc = self.L.ref_axi_tdma(self.h, a, b, c, d, len(d))
        return rc, c, d

    def kappa(self, ls):
        out = self.z()
        self.L.ref_axi_kappa(self.h, ls, out)
        return out

    def visc(self, u, uhat, v, ls, H):
        a, b = self.z(), self.z()
        self.L.ref_axi_visc(self.h, u, uhat, v, ls, H, a, b)
        return a, b

    def rhs_u(self, ls, u, v, H):
        out = self.z()
        self.L.ref_axi_rhs_u(self.h, ls, u, v, H, out)
        return out

    def rhs_v(self, ls, u, uhat, v, H):
        out = self.z()
        self.L.ref_axi_rhs_v(self.h, ls, u, uhat, v, H, out)
        return out

    def uhat(self, ls, u, rhs, H):
        out = self.z()
        self.L.ref_axi_uhat(self.h, ls, u, rhs, H, out)
        return out

    def vhat(self, ls, v, rhs, H):
        out = self.z()
        self.L.ref_axi_vhat(self.h, ls, v, rhs, H, out)
        return out

    def divergences(self, u, v):
        a, b = self.z(), self.z()
        self.L.ref_axi_div(self.h, u, v, a, b)
        return a, b

    def poisson_capture(self, div, ls, lsB, H, maxiter=0):
        ps = self.z()
        m, nnz, nb = C.c_int(), C.c_int(), C.c_int()
        rc = self.L.ref_axi_poisson(self.h, ps, div, ls, lsB, H, maxiter, C.byref(m), C.byref(nnz), C.byref(nb))
        if rc != 0:
            raise RuntimeError("no system captured")
        a, ia, ja, b = np.zeros(nnz.value), np.zeros(m.value + 1, np.int32), np.zeros(nnz.value, np.int32), \
            np.zeros(nb.value)
        self.L.ref_capture_copy(a, ia, ja, b)
        return ps, (a, ia, ja, b)

    def update_vel(self, uhat, vhat, ps, ls, lsB, H):
        self.L.ref_axi_update_vel(self.h, uhat, vhat, ps, ls, lsB, H)

    def update_dt(self, u, v) -> float:
        return self.L.ref_axi_update_dt(self.h, u, v)


def have_reference() -> bool:
    return os.path.exists(REF_SO)
