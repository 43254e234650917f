"""Python host interface of the B200 forward-and-sensitivity path.

Mirrors the reference's operator interface for the path: a model built from
read_smesh-level arrays, `forward` solving the time fields of the enabled
phases for every OBS source (run_forward2d's stage loop,
src/inversion2d.f90:4184-4476), and field access in the reference's region
node order.  All work goes through the C ABI of include/fmt2d_gpu.h.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .synth import SmeshModel

PHASES = {"Pg": 1, "PsedP": 2, "PmP": 3, "Pg_ss": 4, "Pg_ss2": 5}
TF_REGION = {1: 5, 2: 2, 3: 2, 4: 6, 5: 6, 6: 1, 7: 1, 8: 1, 9: 1, 10: 1, 11: 5, 12: 1}
PHASE_FIELDS = {1: (1,), 2: (2, 3), 3: (4, 5), 4: (1, 6, 7, 8), 5: (9, 10, 11, 12)}


def phase_mask(phases) -> int:
    m = 0
    for p in phases:
        m |= 1 << ((PHASES[p] if isinstance(p, str) else int(p)) - 1)
    return m


def fields_of(mask: int) -> list[int]:
    out = set()
    for p in range(1, 6):
        if mask & (1 << (p - 1)):
            out.update(PHASE_FIELDS[p])
    return sorted(out)


def select_data(phase, obs, t_calc, valid, row_ptr, gindx, gval, mvscale, *, crit_chi,
                wt_psed=1.0, wt_pmp=1.0, wt_pgss=1.0):
    """read_frechet_data2d's selection with lsqr_inversion2d's weighting
    (fmt2d_select_data) over a batch of traced picks and their 1-based CSR
    rows.  Returns (row_ptr, gindx, gval, residual, data_wt, pick_of_row) of
    the kept picks, ready for Fmt2d.set_frechet / Fmt2d.lsqr."""
    L = N.lib()
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    phase, valid, row_ptr, gindx = i32(phase), i32(valid), i32(row_ptr), i32(gindx)
    obs, t_calc, gval, mvscale = f64(obs), f64(t_calc), f64(gval), f64(mvscale)
    n = phase.size
    nnz = max(gindx.size, 1)
    rp, gi, gv = np.zeros(n + 1, np.int32), np.zeros(nnz, np.int32), np.zeros(nnz)
    res, wt, pk = np.zeros(max(n, 1)), np.zeros(max(n, 1)), np.zeros(max(n, 1), np.int32)
    nd = C.c_int()
    rc = L.fmt2d_select_data(n, N.ptr(phase), N.ptr(obs), N.ptr(t_calc), N.ptr(valid),
                             N.ptr(row_ptr), N.ptr(gindx), N.ptr(gval), mvscale.size,
                             N.ptr(mvscale), float(crit_chi), float(wt_psed), float(wt_pmp),
                             float(wt_pgss), C.byref(nd), N.ptr(rp), N.ptr(gi), N.ptr(gv),
                             N.ptr(res), N.ptr(wt), N.ptr(pk))
    if rc != 0:
        raise N.Fmt2dError(f"fmt2d_select_data failed ({rc}): bad arguments")
    k, kk = nd.value, int(rp[nd.value]) - 1
    return rp[:k + 1], gi[:kk], gv[:kk], res[:k], wt[:k], pk[:k]


def forward_batch(contexts, sources, phases=(1, 2, 3, 4, 5)):
    """fmt2d_forward of several contexts (one model each) at once: contexts
    is a list of Fmt2d, sources a list of OBS x arrays (one per context);
    phases applies to all.  Raises on the first failing context."""
    n = len(contexts)
    if n == 0 or len(sources) != n:
        raise ValueError("one source array per context")
    xs = [np.ascontiguousarray(x, dtype=np.float64) for x in sources]
    hs = (C.c_void_p * n)(*[g.h.value for g in contexts])
    ps = (C.c_void_p * n)(*[x.ctypes.data for x in xs])
    ns = np.array([x.size for x in xs], dtype=np.int32)
    mask = phase_mask(phases)
    ms = np.full(n, mask, dtype=np.int32)
    st = np.zeros(n, dtype=np.int32)
    rc = N.lib().fmt2d_forward_batch(hs, n, ps, N.ptr(ns), N.ptr(ms), N.ptr(st))
    for g, x in zip(contexts, xs):
        g.mask, g.nsrc = mask, x.size
    if rc != 0:
        i = int(np.flatnonzero(st != 0)[0])
        contexts[i]._check(int(st[i]), f"fmt2d_forward_batch (context {i})")
    return contexts


def project_rows(row_ptr, gindx, gval, nfine, p_row_ptr, p_col, p_val):
    """Rows of G P (fmt2d_project_rows): 1-based CSR (row_ptr, gindx, gval)
    over the fine parameters mapped onto a coarse grid's parameters."""
    L = N.lib()
    i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
    f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
    rp, gi, gv = i32(row_ptr), i32(gindx), f64(gval)
    prp, pc, pv = i32(p_row_ptr), i32(p_col), f64(p_val)
    nd = rp.size - 1
    nnz = C.c_longlong()
    args = (nd, N.ptr(rp), N.ptr(gi), N.ptr(gv), int(nfine), N.ptr(prp), N.ptr(pc), N.ptr(pv))
    if L.fmt2d_project_rows(*args, None, None, None, C.byref(nnz)) != 0:
        raise N.Fmt2dError("fmt2d_project_rows: bad arguments")
    orp = np.zeros(nd + 1, np.int32)
    ogi, ogv = np.zeros(max(nnz.value, 1), np.int32), np.zeros(max(nnz.value, 1))
    L.fmt2d_project_rows(*args, N.ptr(orp), N.ptr(ogi), N.ptr(ogv), C.byref(nnz))
    return orp, ogi[:nnz.value], ogv[:nnz.value]


class Fmt2d:
    """One context (device buffers + stream).  device=-1 gives a host-only
    context for the model tables."""

    def __init__(self, device: int = 0):
        self.L = N.lib()
        h = C.c_void_p()
        rc = self.L.fmt2d_ctx_create(C.byref(h), int(device))
        if rc != 0:
            raise N.Fmt2dError(f"fmt2d_ctx_create(device={device}) failed with code {rc}")
        self.h = h
        self.device = device
        self._keep = None
        self.npick, self.frechet_nnz = 0, None

    def close(self):
        if getattr(self, "h", None):
            self.L.fmt2d_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc: int, what: str):
        if rc != 0:
            buf = C.create_string_buffer(512)
            self.L.fmt2d_last_error(self.h, buf, 512)
            cls = N.Fmt2dNotConverged if rc == N.ERR_CONVERGE else N.Fmt2dError
            raise cls(f"{what} failed ({rc}): {buf.value.decode()}", rc)

    def upload(self, m: SmeshModel, iface_inv: int = 4):
        f = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        keep = [f(m.xpos), f(m.topo), f(m.zrel), f(m.vel), f(m.sed_z), f(m.moho_z)]
        d = N.ModelDesc(m.nx, m.zrel.size, N.ptr(keep[0]), N.ptr(keep[1]), N.ptr(keep[2]),
                        N.ptr(keep[3]), float(m.vwater), N.ptr(keep[4]), N.ptr(keep[5]),
                        int(iface_inv))
        self._check(self.L.fmt2d_upload_model(self.h, C.byref(d)), "fmt2d_upload_model")
        nx, nz, dx, x0 = C.c_int(), C.c_int(), C.c_double(), C.c_double()
        self._check(self.L.fmt2d_model_info(self.h, C.byref(nx), C.byref(nz), C.byref(dx),
                                            C.byref(x0)), "fmt2d_model_info")
        self.nx, self.nz, self.dx, self.x0 = nx.value, nz.value, dx.value, x0.value
        self.model = m
        self.iface_inv = int(iface_inv)
        return self

    def velocity(self) -> np.ndarray:
        """Propagation-grid velocity (nz, nx) of the current model."""
        v = np.zeros(self.nx * self.nz)
        self._check(self.L.fmt2d_model_velocity(self.h, N.ptr(v)), "fmt2d_model_velocity")
        return v.reshape(self.nz, self.nx)

    def interface(self, k: int) -> np.ndarray:
        """Node depths of interface k (1..5)."""
        z = np.zeros(self.nx)
        self._check(self.L.fmt2d_model_interface(self.h, int(k), N.ptr(z)),
                    "fmt2d_model_interface")
        return z

    def update_model(self, vel=None, iface_z=None):
        """A model step (fmt2d_update_model): new propagation-grid velocity
        (nz, nx) and / or new depths of the inverted interface."""
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).ravel()
        z = None if iface_z is None else np.ascontiguousarray(iface_z, dtype=np.float64)
        if v is not None and v.size != self.nx * self.nz:
            raise ValueError("vel must have nz * nx entries")
        if z is not None and z.size != self.nx:
            raise ValueError("iface_z must have nx entries")
        self._check(self.L.fmt2d_update_model(self.h, N.ptr(v), N.ptr(z)), "fmt2d_update_model")
        return self

    def region_nodes(self, r: int):
        n = C.c_int()
        self._check(self.L.fmt2d_region_nodes(self.h, r, C.byref(n), None, None, None),
                    "fmt2d_region_nodes")
        i1, i2, i3 = (np.zeros(n.value, np.int32) for _ in range(3))
        self._check(self.L.fmt2d_region_nodes(self.h, r, C.byref(n), N.ptr(i1), N.ptr(i2),
                                              N.ptr(i3)), "fmt2d_region_nodes")
        return i1, i2, i3

    def region_geometry(self, r: int):
        """Node x, z and FP64 velocity of region r in the reference's order."""
        n = self.region_nnode(r)
        x, z, v = np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(self.L.fmt2d_region_geometry(self.h, r, N.ptr(x), N.ptr(z), N.ptr(v)),
                    "fmt2d_region_geometry")
        return x, z, v

    def region_nnode(self, r: int) -> int:
        n = C.c_int()
        self._check(self.L.fmt2d_region_nodes(self.h, r, C.byref(n), None, None, None),
                    "fmt2d_region_nodes")
        return n.value

    def inv_index(self):
        out = np.zeros(self.nx * self.nz, np.int32)
        nvp, npar = C.c_int(), C.c_int()
        self._check(self.L.fmt2d_inv_index(self.h, N.ptr(out), C.byref(nvp), C.byref(npar)),
                    "fmt2d_inv_index")
        return out.reshape(self.nz, self.nx), nvp.value, npar.value

    def projection(self, kx: int, kz: int, ki: int) -> dict:
        """Coarse inversion grid every kx columns / kz rows (interface every
        ki nodes) and its projection P onto the model's parameters
        (fmt2d_projection).  Returns dict(P=(row_ptr, col, val), nvp, npar,
        coarse_idx (nzc, nxc))."""
        nxc, nzc, nvp, npar, nnz = C.c_int(), C.c_int(), C.c_int(), C.c_int(), C.c_longlong()
        sizes = (C.byref(nxc), C.byref(nzc), C.byref(nvp), C.byref(npar))
        self._check(self.L.fmt2d_projection(self.h, kx, kz, ki, *sizes, None, None, None, None,
                                            C.byref(nnz)), "fmt2d_projection")
        nfine = self.inv_index()[2]
        cidx = np.zeros(nxc.value * nzc.value, np.int32)
        rp = np.zeros(nfine + 1, np.int32)
        col, val = np.zeros(max(nnz.value, 1), np.int32), np.zeros(max(nnz.value, 1))
        self._check(self.L.fmt2d_projection(self.h, kx, kz, ki, *sizes, N.ptr(cidx), N.ptr(rp),
                                            N.ptr(col), N.ptr(val), C.byref(nnz)),
                    "fmt2d_projection")
        return dict(P=(rp, col[:nnz.value], val[:nnz.value]), nvp=nvp.value, npar=npar.value,
                    coarse_idx=cidx.reshape(nzc.value, nxc.value))

    def gauss_smooth(self, which: int, mvscale, corr_x=0.0, corr_z=0.0, corr_x_iface=0.0):
        """1-based CSR (row_ptr, col, val) of the Gaussian smoothing matrix R_h
        (which 0), R_v (1) or the interface R_h (2) (fmt2d_gauss_smooth)."""
        mv = np.ascontiguousarray(mvscale, dtype=np.float64)
        npar = self.inv_index()[2]
        if mv.size != npar:
            raise ValueError(f"mvscale has {mv.size} entries, the model has {npar} parameters")
        nnz = C.c_longlong()
        self._check(self.L.fmt2d_gauss_smooth(self.h, int(which), float(corr_x), float(corr_z),
                                              float(corr_x_iface), N.ptr(mv), None, None, None,
                                              C.byref(nnz)), "fmt2d_gauss_smooth")
        rp = np.zeros(mv.size + 1, np.int32)
        col, val = np.zeros(max(nnz.value, 1), np.int32), np.zeros(max(nnz.value, 1))
        self._check(self.L.fmt2d_gauss_smooth(self.h, int(which), float(corr_x), float(corr_z),
                                              float(corr_x_iface), N.ptr(mv), N.ptr(rp),
                                              N.ptr(col), N.ptr(val), C.byref(nnz)),
                    "fmt2d_gauss_smooth")
        return rp, col[:nnz.value], val[:nnz.value]

    def forward(self, src_x, phases=(1, 2, 3, 4, 5)):
        src_x = np.ascontiguousarray(src_x, dtype=np.float64)
        self.mask = phase_mask(phases)
        self._check(self.L.fmt2d_forward(self.h, src_x, src_x.size, self.mask), "fmt2d_forward")
        self.nsrc = src_x.size
        return self

    def field(self, src: int, tf: int):
        n = self.region_nnode(TF_REGION[tf])
        T, gx, gz = np.zeros(n), np.zeros(n), np.zeros(n)
        self._check(self.L.fmt2d_get_field(self.h, src, tf, N.ptr(T), N.ptr(gx), N.ptr(gz)),
                    "fmt2d_get_field")
        return T, gx, gz

    STATS = ("steps", "batches", "passes", "passed", "solve_ms", "launches", "nodes",
             "evals", "steps_all", "capped", "writes", "unsettled", "cyc_eval", "cyc_arb",
             "cyc_eval_cut", "cyc_spread", "cyc_release", "cut_evals", "cut_steps")

    def stats(self) -> dict:
        """Counters of the last forward (fmt2d_stats)."""
        v = np.zeros(len(self.STATS))
        self._check(self.L.fmt2d_stats(self.h, N.ptr(v), v.size), "fmt2d_stats")
        return {k: (round(float(x), 3) if k == "solve_ms" else int(x))
                for k, x in zip(self.STATS, v)}

    # ------------------------------------------------------------ rays and Frechet rows
    def trace(self, src, phase, rx, rz):
        """Ray backtrace and Frechet rows of picks on the last forward's fields
        (fmt2d_trace).  Returns (t_calc, valid, nnz)."""
        src = np.ascontiguousarray(src, dtype=np.int32)
        phase = np.ascontiguousarray(phase, dtype=np.int32)
        rx = np.ascontiguousarray(rx, dtype=np.float64)
        rz = np.ascontiguousarray(rz, dtype=np.float64)
        n = src.size
        t = np.zeros(n)
        v = np.zeros(n, np.int32)
        nnz = C.c_longlong()
        self._check(self.L.fmt2d_trace(self.h, N.ptr(src), N.ptr(phase), N.ptr(rx), N.ptr(rz), n,
                                       N.ptr(t), N.ptr(v), C.byref(nnz)), "fmt2d_trace")
        self.npick, self.frechet_nnz = n, nnz.value
        return t, v.astype(bool), nnz.value

    def trace_times(self, src, phase, rx, rz):
        """Receiver times and valid flags of picks on the last forward's fields,
        without Frechet rows (fmt2d_trace_times).  Returns (t_calc, valid)."""
        src = np.ascontiguousarray(src, dtype=np.int32)
        phase = np.ascontiguousarray(phase, dtype=np.int32)
        rx = np.ascontiguousarray(rx, dtype=np.float64)
        rz = np.ascontiguousarray(rz, dtype=np.float64)
        n = src.size
        t = np.zeros(n)
        v = np.zeros(n, np.int32)
        self._check(self.L.fmt2d_trace_times(self.h, N.ptr(src), N.ptr(phase), N.ptr(rx),
                                             N.ptr(rz), n, N.ptr(t), N.ptr(v)),
                    "fmt2d_trace_times")
        self.npick, self.frechet_nnz = n, None
        return t, v.astype(bool)

    def misfit_gradient(self, src, phase, rx, rz, t_obs, sigma, want=("slow",)):
        """Misfit 0.5*sum(((t_calc - t_obs)/sigma)^2) over the valid picks
        (phases 1-5; t_obs < 0: no pick) on the last forward's fields and its
        gradient by the discrete adjoint of the fields
        (fmt2d_misfit_gradient).  Returns a dict: misfit, t_calc, valid,
        grad_slow and / or grad_vel ((nz, nx)) and / or grad_iface ((5, nx):
        node depths of interfaces 1..5), as `want` asks, and info (the
        adjoint's counters, see the header)."""
        src = np.ascontiguousarray(src, dtype=np.int32)
        phase = np.ascontiguousarray(phase, dtype=np.int32)
        rx = np.ascontiguousarray(rx, dtype=np.float64)
        rz = np.ascontiguousarray(rz, dtype=np.float64)
        t_obs = np.ascontiguousarray(t_obs, dtype=np.float64)
        sigma = np.broadcast_to(np.asarray(sigma, dtype=np.float64), src.shape).copy()
        n = src.size
        t = np.zeros(n)
        v = np.zeros(n, np.int32)
        J = C.c_double()
        gs = np.zeros(self.nx * self.nz) if "slow" in want else None
        gvel = np.zeros(self.nx * self.nz) if "vel" in want else None
        gif = np.zeros(5 * self.nx) if "iface" in want else None
        info = np.zeros(8)
        self._check(self.L.fmt2d_misfit_gradient(
            self.h, N.ptr(src), N.ptr(phase), N.ptr(rx), N.ptr(rz), N.ptr(t_obs), N.ptr(sigma), n,
            C.byref(J), N.ptr(t), N.ptr(v), N.ptr(gs), N.ptr(gvel), N.ptr(gif), N.ptr(info)),
            "fmt2d_misfit_gradient")
        self.npick, self.frechet_nnz = n, None
        out = {"misfit": J.value, "t_calc": t, "valid": v.astype(bool), "info": info}
        if gs is not None:
            out["grad_slow"] = gs.reshape(self.nz, self.nx)
        if gvel is not None:
            out["grad_vel"] = gvel.reshape(self.nz, self.nx)
        if gif is not None:
            out["grad_iface"] = gif.reshape(5, self.nx)
        return out

    def gradient_on_params(self, grad: dict, proj: dict | None = None) -> np.ndarray:
        """A misfit_gradient result on the inversion parameters
        (fmt2d_inv_index numbering: the velocity parameters, then the inverted
        interface's nodes): d misfit / d slowness at each parameter's node and
        d misfit / d depth at each interface node.  With proj (a projection()
        dict), P^T times that vector: the gradient on the coarse grid's
        parameters."""
        inv, nvp, npar = self.inv_index()
        g = np.zeros(npar)
        act = inv > 0
        g[inv[act] - 1] = grad["grad_slow"][act]
        if npar > nvp:
            if "grad_iface" not in grad:
                raise ValueError("the gradient lacks grad_iface (want 'iface')")
            g[nvp:] = grad["grad_iface"][self.iface_inv - 1][: npar - nvp]
        if proj is None:
            return g
        rp, col, val = proj["P"]
        rows = np.repeat(np.arange(npar), np.diff(rp))
        out = np.zeros(proj["npar"])
        np.add.at(out, col - 1, val * g[rows])
        return out

    def trace_entries(self):
        """Per pick of the last trace (fmt2d_trace_entries): water time, entry
        x, entry z (the seafloor entry point of an in-water pick of phases
        1-3, else the receiver)."""
        wt, ex, ez = np.zeros(self.npick), np.zeros(self.npick), np.zeros(self.npick)
        self._check(self.L.fmt2d_trace_entries(self.h, N.ptr(wt), N.ptr(ex), N.ptr(ez)),
                    "fmt2d_trace_entries")
        return wt, ex, ez

    def frechet_rows(self, index_base: int = 1):
        """CSR (row_ptr, gindx, gval) of the last trace (fmt2d_frechet_rows)."""
        if self.frechet_nnz is None:
            raise RuntimeError("Frechet rows: call trace() first (trace_times and "
                               "misfit_gradient compute no rows)")
        rp = np.zeros(self.npick + 1, np.int32)
        gi = np.zeros(max(self.frechet_nnz, 1), np.int32)
        gv = np.zeros(max(self.frechet_nnz, 1))
        self._check(self.L.fmt2d_frechet_rows(self.h, N.ptr(rp), N.ptr(gi), N.ptr(gv),
                                              int(index_base)), "fmt2d_frechet_rows")
        return rp, gi[: self.frechet_nnz], gv[: self.frechet_nnz]

    # ------------------------------------------------------------ G and LSQR
    def set_frechet(self, ndata: int, nparm: int, row_ptr, gindx, gval, index_base: int = 1):
        """Sensitivity matrix as CSR (read_frechet_data2d's gindx / gval /
        row_ptr, 1-based by default)."""
        rp = np.ascontiguousarray(row_ptr, dtype=np.int32)
        gi = np.ascontiguousarray(gindx, dtype=np.int32)
        gv = np.ascontiguousarray(gval, dtype=np.float64)
        if rp.size != ndata + 1:
            raise ValueError("row_ptr needs ndata + 1 entries")
        self._check(self.L.fmt2d_set_frechet(self.h, int(ndata), int(nparm), N.ptr(rp), N.ptr(gi),
                                             N.ptr(gv), int(index_base)), "fmt2d_set_frechet")
        self.ndata, self.nparm = int(ndata), int(nparm)
        return self

    def spmv(self, x, transpose: bool = False):
        x = np.ascontiguousarray(x, dtype=np.float64)
        if x.size != (self.ndata if transpose else self.nparm):
            raise ValueError("x has the wrong length")
        y = np.zeros(self.nparm if transpose else self.ndata)
        self._check(self.L.fmt2d_spmv(self.h, int(bool(transpose)), N.ptr(x), N.ptr(y)),
                    "fmt2d_spmv")
        return y

    def gtg_diag(self):
        out = np.zeros(self.nparm)
        self._check(self.L.fmt2d_gtg_diag(self.h, N.ptr(out)), "fmt2d_gtg_diag")
        return out

    def set_param_grid(self, coarse_idx=None, n_vel_parms=0, iface_nodes=0):
        """The LSQR's parameter grid (fmt2d_set_param_grid): coarse_idx (nzc,
        nxc) of fmt2d_projection with its velocity and interface parameter
        counts, or None for the model's own numbering."""
        if coarse_idx is None:
            rc = self.L.fmt2d_set_param_grid(self.h, 0, 0, None, 0, 0)
        else:
            ci = np.ascontiguousarray(coarse_idx, dtype=np.int32)
            rc = self.L.fmt2d_set_param_grid(self.h, ci.shape[1], ci.shape[0], N.ptr(ci),
                                             int(n_vel_parms), int(iface_nodes))
        self._check(rc, "fmt2d_set_param_grid")
        return self

    def set_smoothing(self, mvscale, corr_x=0.0, corr_z=0.0, corr_x_iface=0.0):
        """Gaussian smoothing operators of the smooth_type 2/3 LSQR layouts
        (fmt2d_set_smoothing): R_h (corr_x > 0), R_v (corr_z > 0) and the
        interface R_h (corr_x_iface > 0), mvscale folded in."""
        mv = np.ascontiguousarray(mvscale, dtype=np.float64)
        npar = self.inv_index()[2]
        if mv.size != npar:
            raise ValueError(f"mvscale has {mv.size} entries, the model has {npar} parameters")
        self._check(self.L.fmt2d_set_smoothing(self.h, float(corr_x), float(corr_z),
                                               float(corr_x_iface), N.ptr(mv)),
                    "fmt2d_set_smoothing")
        return self

    def lsqr(self, residual, dm_sum=None, gtg_diag=None, *, wdv=0.0, wdv_iface=0.0,
             w_smooth=0.0, w_smooth_iface=0.0, eps_min=0.0, max_iter=2000, smooth_type=1):
        """run_lsqr on the current G; returns (dm, iters, rnorm, bnorm, test2)."""
        f = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        r, s, g = f(residual), f(dm_sum), f(gtg_diag)
        p = N.LsqrParams(int(smooth_type), int(max_iter), float(wdv), float(wdv_iface),
                         float(w_smooth), float(w_smooth_iface), float(eps_min))
        dm = np.zeros(self.nparm)
        it, rn, bn, t2 = C.c_int(), C.c_double(), C.c_double(), C.c_double()
        self._check(self.L.fmt2d_lsqr(self.h, C.byref(p), N.ptr(r), N.ptr(g), N.ptr(s), N.ptr(dm),
                                      C.byref(it), C.byref(rn), C.byref(bn), C.byref(t2)),
                    "fmt2d_lsqr")
        return dm, it.value, rn.value, bn.value, t2.value

    def lsqr_damped(self, residual, dm_sum=None, gtg_diag=None, mvscale=None, *,
                    lam_damp=0.0, lam_damp_iface=0.0, target_dv=0.0, target_dd=0.0,
                    w_smooth=0.0, w_smooth_iface=0.0, eps_min=0.0, max_iter=2000,
                    smooth_type=1):
        """lsqr_inversion2d's damping choice (src/inversion2d.f90:533-739):
        a fixed damping weight (lam_damp > 0) or tomo2d's auto damping towards
        the RMS velocity change target_dv and depth change target_dd, each
        solve an fmt2d_lsqr on the current G.  mvscale (column scaling, for
        the depth change of interface parameters) defaults to ones and gtg_diag
        to this G's column norms.  Returns a damping.DampingResult."""
        from .damping import damping_search
        if gtg_diag is None:
            gtg_diag = self.gtg_diag()
        gtg_diag = np.ascontiguousarray(gtg_diag, dtype=np.float64)
        if mvscale is None:
            mvscale = np.ones(self.nparm)
        _, nvp, _ = self.inv_index()

        def solve(wdv, wdi):
            return self.lsqr(residual, dm_sum, gtg_diag, wdv=wdv, wdv_iface=wdi,
                             w_smooth=w_smooth, w_smooth_iface=w_smooth_iface,
                             eps_min=eps_min, max_iter=max_iter, smooth_type=smooth_type)[0]

        return damping_search(solve, dm_sum, gtg_diag, mvscale, eps_min, nvp,
                              lam_damp=lam_damp, lam_damp_iface=lam_damp_iface,
                              target_dv=target_dv, target_dd=target_dd)

    def lsqr_stats(self):
        ms, n = C.c_double(), C.c_int()
        self._check(self.L.fmt2d_lsqr_stats(self.h, C.byref(ms), C.byref(n)), "fmt2d_lsqr_stats")
        return {"ms": ms.value, "launches": n.value}

    def set_iface_window(self, cells: float):
        """Window of the stages seeded along an interface when set_schedule's
        window_cells is 0 (fmt2d_set_iface_window; 0: none)."""
        self._check(self.L.fmt2d_set_iface_window(self.h, float(cells)), "fmt2d_set_iface_window")
        return self

    def set_schedule(self, window_cells: float = 0.0, max_passes: int = 6, max_steps: int = 0):
        """Eikonal solve schedule (fmt2d_set_schedule).  window_cells > 0 holds
        new times beyond a window of that many cells (at the region's largest
        velocity) until the times below it settle; 0 (the default) sets none
        for stages that start from the point source and 32 cells for stages
        seeded along an interface.  max_passes bounds the solve passes (each ends in a fixed-point
        check of every node), max_steps the steps of one field's solve (0: the
        library default)."""
        self._check(self.L.fmt2d_set_schedule(self.h, float(window_cells), int(max_passes),
                                              int(max_steps)), "fmt2d_set_schedule")
        return self

    def set_solve_threads(self, threads: int = 0):
        """Threads of each field's solve block (fmt2d_set_solve_threads): 256,
        384 or 512, 0 for the default; results are identical for every size."""
        self._check(self.L.fmt2d_set_solve_threads(self.h, int(threads)),
                    "fmt2d_set_solve_threads")
        return self

    def autotune(self, src_x, phases=(1, 2, 3, 4, 5)) -> dict:
        """Pick the fastest solve block size for this workload (fmt2d_autotune);
        the context keeps it.  Returns {"threads": chosen, "ms": {size: ms}}."""
        src_x = np.ascontiguousarray(src_x, dtype=np.float64)
        t = C.c_int()
        ms = np.zeros(3)
        self._check(self.L.fmt2d_autotune(self.h, src_x, src_x.size, phase_mask(phases),
                                          C.byref(t), N.ptr(ms)), "fmt2d_autotune")
        self.mask, self.nsrc = phase_mask(phases), src_x.size
        return {"threads": t.value, "ms": dict(zip((256, 384, 512), ms.round(3).tolist()))}

    def stream(self) -> int:
        """cudaStream_t (as an integer) that the context's work runs on."""
        s = C.c_void_p()
        self._check(self.L.fmt2d_stream(self.h, C.byref(s)), "fmt2d_stream")
        return int(s.value or 0)
