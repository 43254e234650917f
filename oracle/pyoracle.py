"""ctypes wrapper of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
CPU-baseline leg of bench.py, where it is the checker (or the timed CPU
restatement of the reference).  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_up = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")


def build() -> str:
    """Compile the oracle with its Makefile (a few seconds with g++)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        build()
    L = C.CDLL(_LIB_PATH)
    V = C.c_void_p
    L.orc_create.restype = V
    L.orc_create.argtypes = [C.c_int, C.c_int, _dp, _dp, _dp, _dp, C.c_double, _dp, _dp, C.c_int]
    L.orc_destroy.argtypes = [V]
    L.orc_grid_info.argtypes = [V, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_pgrid_velocity.argtypes = [V, _dp]
    L.orc_iface_z.argtypes = [V, C.c_int, _dp]
    L.orc_iface_vel.argtypes = [V, C.c_int, _dp, _dp]
    L.orc_region_nnode.restype = C.c_int
    L.orc_region_nnode.argtypes = [V, C.c_int, C.POINTER(C.c_int)]
    L.orc_region_tables.argtypes = [V, C.c_int, _ip, _ip, _ip, _dp, _dp, _dp, _ip]
    L.orc_fully_regular.argtypes = [V, _up]
    L.orc_cut_cells.argtypes = [V, C.c_int, C.POINTER(C.c_int), _ip, _ip]
    L.orc_inv_idx.restype = C.c_int
    L.orc_inv_idx.argtypes = [V, _ip, C.POINTER(C.c_int)]
    L.orc_forward.restype = C.c_int
    L.orc_forward.argtypes = [V, C.c_int, C.c_double, C.c_int]
    L.orc_source_z.restype = C.c_double
    L.orc_source_z.argtypes = [V, C.c_int]
    L.orc_field.restype = C.c_int
    L.orc_field.argtypes = [V, C.c_int, C.c_int, _dp, _dp, _dp]
    L.orc_set_field.restype = C.c_int
    L.orc_set_field.argtypes = [V, C.c_int, C.c_int, _dp, _dp, _dp]
    L.orc_propagate.restype = C.c_int
    L.orc_propagate.argtypes = [V, C.c_int, _ip, _dp, _dp, _dp]
    L.orc_trace.restype = C.c_int
    L.orc_trace.argtypes = [V, C.c_int, C.c_int, C.c_double, C.c_double,
                            C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_int),
                            _ip, _dp, C.c_int, C.POINTER(C.c_int), _dp, C.c_int,
                            C.POINTER(C.c_int)]
    L.orc_lsqr.restype = C.c_int
    L.orc_lsqr.argtypes = [V, C.c_int, C.c_int, _ip, _dp, _ip, _dp, _dp, _dp, C.c_double,
                           C.c_double, C.c_double, C.c_double, C.c_double, C.c_int, _dp,
                           C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_spmv.argtypes = [C.c_int, C.c_int, _ip, _dp, _ip, C.c_int, _dp, _dp]
    L.orc_laplacian.argtypes = [V, C.c_int, _dp, _dp]
    L.orc_lsqr_smooth.argtypes = [V, C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                  C.c_double, C.c_double, C.c_double, C.c_int, C.c_void_p,
                                  C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
    L.orc_lsqr_geom.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                C.c_int] + [C.c_void_p] * 6 + [C.c_double] * 5 + \
        [C.c_int, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.orc_gauss_smooth.restype = C.c_int
    L.orc_gauss_smooth.argtypes = [V, C.c_double, C.c_double, C.c_double, _dp, C.c_int,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
    _lib = L
    return L


TF_REGION = {1: 5, 2: 2, 3: 2, 4: 6, 5: 6, 6: 1, 7: 1, 8: 1, 9: 1, 10: 1, 11: 5, 12: 1}


class Oracle:
    """One oracle model (geometry + per-source time fields)."""

    def __init__(self, model, iface_inv: int = 4):
        L = lib()
        self.model = model
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        vel = f(model.vel)  # (nzs, nx): ix fastest in memory
        self.h = L.orc_create(model.nx, model.zrel.size, f(model.xpos), f(model.topo),
                              f(model.zrel), vel, float(model.vwater), f(model.sed_z),
                              f(model.moho_z), iface_inv)
        nx, nz, dx, x0 = C.c_int(), C.c_int(), C.c_double(), C.c_double()
        L.orc_grid_info(self.h, C.byref(nx), C.byref(nz), C.byref(dx), C.byref(x0))
        self.nx, self.nz, self.dx, self.x0 = nx.value, nz.value, dx.value, x0.value

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.orc_destroy(self.h)
            self.h = None

    def pgrid_velocity(self):
        out = np.zeros(self.nx * self.nz)
        lib().orc_pgrid_velocity(self.h, out)
        return out.reshape(self.nz, self.nx)

    def iface_z(self, k):
        out = np.zeros(self.nx)
        lib().orc_iface_z(self.h, k, out)
        return out

    def iface_vel(self, k):
        a, b = np.zeros(self.nx), np.zeros(self.nx)
        lib().orc_iface_vel(self.h, k, a, b)
        return a, b

    def region(self, r):
        ng = C.c_int()
        n = lib().orc_region_nnode(self.h, r, C.byref(ng))
        i1, i2, i3 = (np.zeros(n, np.int32) for _ in range(3))
        x, z, v = np.zeros(n), np.zeros(n), np.zeros(n)
        rid = np.zeros(self.nx * self.nz, np.int32)
        lib().orc_region_tables(self.h, r, i1, i2, i3, x, z, v, rid)
        return dict(nnode=n, ngnode=ng.value, i1=i1, i2=i2, i3=i3, x=x, z=z, vel=v,
                    rid=rid.reshape(self.nz, self.nx))

    def fully_regular(self):
        out = np.zeros(self.nx * self.nz, np.uint8)
        lib().orc_fully_regular(self.h, out)
        return out.reshape(self.nz, self.nx)

    def cut_cells(self, k):
        n = C.c_int()
        cx = np.zeros(self.nx, np.int32)
        cz = np.zeros(self.nx, np.int32)
        lib().orc_cut_cells(self.h, k, C.byref(n), cx, cz)
        return cx[: n.value], cz[: n.value]

    def inv_idx(self):
        out = np.zeros(self.nx * self.nz, np.int32)
        nvp = C.c_int()
        npar = lib().orc_inv_idx(self.h, out, C.byref(nvp))
        return out.reshape(self.nz, self.nx), nvp.value, npar

    def forward(self, slot, sx, phase_mask=0b11111):
        return lib().orc_forward(self.h, slot, float(sx), int(phase_mask))

    def source_z(self, slot):
        return lib().orc_source_z(self.h, slot)

    def field(self, slot, tf):
        n = lib().orc_region_nnode(self.h, TF_REGION[tf], None)
        T, gx, gz = np.zeros(n), np.zeros(n), np.zeros(n)
        ok = lib().orc_field(self.h, slot, tf, T, gx, gz)
        return (T, gx, gz) if ok >= 0 else None

    def set_field(self, slot, tf, T, gx, gz):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        return lib().orc_set_field(self.h, slot, tf, f(T), f(gx), f(gz))

    def propagate(self, reg, status, T, gx, gz):
        st = np.ascontiguousarray(status, dtype=np.int32).copy()
        T, gx, gz = (np.ascontiguousarray(a, dtype=np.float64).copy() for a in (T, gx, gz))
        lib().orc_propagate(self.h, reg, st, T, gx, gz)
        return st, T, gx, gz

    def trace(self, slot, phase, rx, rz, cap=200000, pts_cap=50000):
        t, valid, nnz, npts, nsec = C.c_double(), C.c_int(), C.c_int(), C.c_int(), C.c_int()
        idx = np.zeros(cap, np.int32)
        val = np.zeros(cap)
        pts = np.zeros(2 * pts_cap)
        lib().orc_trace(self.h, slot, phase, float(rx), float(rz), C.byref(t), C.byref(valid),
                        C.byref(nnz), idx, val, cap, C.byref(npts), pts, pts_cap, C.byref(nsec))
        k, p = nnz.value, npts.value
        return dict(t=t.value, valid=bool(valid.value), idx=idx[:k].copy(), val=val[:k].copy(),
                    pts=pts[: 2 * p].reshape(-1, 2).copy(), nsec=nsec.value)

    def lsqr(self, ndata, nparm, gindx, gval, row_ptr, residual, gtg, dm_sum, eps_min, wdv,
             wdv_iface, w_smooth, w_smooth_iface, max_iter):
        dm = np.zeros(nparm)
        it, rn, t2 = C.c_int(), C.c_double(), C.c_double()
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        lib().orc_lsqr(self.h, ndata, nparm, i32(gindx), f64(gval), i32(row_ptr), f64(residual),
                       f64(gtg), f64(dm_sum), eps_min, wdv, wdv_iface, w_smooth, w_smooth_iface,
                       max_iter, dm, C.byref(it), C.byref(rn), C.byref(t2))
        return dm, it.value, rn.value, t2.value

    def gauss_smooth(self, which, mvscale, corr_x=0.0, corr_z=0.0, corr_x_iface=0.0):
        """1-based CSR (rp, col, val) of R_h (which 0), R_v (1) or the
        interface R_h (2) of build_gauss_smooth_matrix /
        build_iface_gauss_smooth_matrix."""
        mv = np.ascontiguousarray(mvscale, dtype=np.float64)
        rp = np.zeros(mv.size + 1, np.int32)
        n = lib().orc_gauss_smooth(self.h, corr_x, corr_z, corr_x_iface, mv, which, None, None,
                                   None, 0)
        col, val = np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1))
        lib().orc_gauss_smooth(self.h, corr_x, corr_z, corr_x_iface, mv, which,
                               rp.ctypes.data_as(C.c_void_p), col.ctypes.data_as(C.c_void_p),
                               val.ctypes.data_as(C.c_void_p), n)
        return rp, col[:n], val[:n]

    def lsqr_smooth(self, smooth_type, ndata, nparm, gindx, gval, row_ptr, residual, gtg, dm_sum,
                    mvscale, corr_x, corr_z, corr_x_iface, eps_min, wdv, wdv_iface, w_smooth,
                    w_smooth_iface, max_iter):
        """run_lsqr for smooth_type 1, 2 or 3; returns (dm, iters, rnorm, test2)."""
        keep = []

        def p(a, t):
            a = np.ascontiguousarray(a, dtype=t)
            keep.append(a)
            return a.ctypes.data_as(C.c_void_p)
        dm = np.zeros(nparm)
        it, rn, t2 = C.c_int(), C.c_double(), C.c_double()
        lib().orc_lsqr_smooth(self.h, smooth_type, ndata, nparm, p(gindx, np.int32),
                              p(gval, np.float64), p(row_ptr, np.int32), p(residual, np.float64),
                              p(gtg, np.float64), p(dm_sum, np.float64), p(mvscale, np.float64),
                              corr_x, corr_z, corr_x_iface, eps_min, wdv, wdv_iface, w_smooth,
                              w_smooth_iface, max_iter, dm.ctypes.data_as(C.c_void_p),
                              C.byref(it), C.byref(rn), C.byref(t2))
        return dm, it.value, rn.value, t2.value

    def laplacian(self, nparm, v):
        out = np.zeros(nparm)
        lib().orc_laplacian(self.h, nparm, np.ascontiguousarray(v, dtype=np.float64), out)
        return out


def lsqr_geom(inv_idx, n_vel_parms, iface_nx, ndata, nparm, gindx, gval, row_ptr, residual, gtg,
              dm_sum, eps_min, wdv, wdv_iface, w_smooth, w_smooth_iface, max_iter):
    """run_lsqr (smooth_type 1) with the Laplacian on the parameter grid
    inv_idx (nz, nx); returns (dm, iters, rnorm, test2)."""
    keep = []

    def p(a, t):
        a = np.ascontiguousarray(a, dtype=t)
        keep.append(a)
        return a.ctypes.data_as(C.c_void_p)
    inv = np.ascontiguousarray(inv_idx, dtype=np.int32)
    dm = np.zeros(nparm)
    it, rn, t2 = C.c_int(), C.c_double(), C.c_double()
    lib().orc_lsqr_geom(inv.shape[1], inv.shape[0], p(inv, np.int32), n_vel_parms, iface_nx,
                        ndata, nparm, p(gindx, np.int32), p(gval, np.float64),
                        p(row_ptr, np.int32), p(residual, np.float64), p(gtg, np.float64),
                        p(dm_sum, np.float64), eps_min, wdv, wdv_iface, w_smooth, w_smooth_iface,
                        max_iter, dm.ctypes.data_as(C.c_void_p), C.byref(it), C.byref(rn),
                        C.byref(t2))
    return dm, it.value, rn.value, t2.value


def spmv(ndata, nparm, gindx, gval, row_ptr, x, transpose=False):
    out = np.zeros(nparm if transpose else ndata)
    lib().orc_spmv(ndata, nparm, np.ascontiguousarray(gindx, dtype=np.int32),
                   np.ascontiguousarray(gval, dtype=np.float64),
                   np.ascontiguousarray(row_ptr, dtype=np.int32), int(transpose),
                   np.ascontiguousarray(x, dtype=np.float64), out)
    return out
