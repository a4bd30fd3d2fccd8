"""ctypes front end of the CPU checker (oracle/liboracle.so + the reference SuperLU in oracle/_ref).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU-baseline and reference
arms load it as the checker. The product (the CUDA library) never uses it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SLU = os.path.join(HERE, "_ref", "libslu_ref.so")

_L = None


def available() -> bool:
    return os.path.exists(LIB) and os.path.exists(SLU)


def load():
    global _L
    if _L is not None:
        return _L
    if not available():
        raise RuntimeError("oracle not built (make -C oracle oracle ref)")
    L = C.CDLL(LIB)
    vp, i32, d = C.c_void_p, C.c_int32, C.c_double
    L.oracle_load_superlu.argtypes = [C.c_char_p]
    if L.oracle_load_superlu(SLU.encode()) != 0:
        raise RuntimeError("cannot load the reference SuperLU from " + SLU)
    L.oracle_net_create.restype = vp
    L.oracle_net_create.argtypes = [vp, vp]
    L.oracle_net_destroy.argtypes = [vp]
    L.oracle_nnz.argtypes = [vp]
    L.oracle_jac_pattern.argtypes = [vp, vp, vp, vp]
    L.oracle_eval_rates.argtypes = [vp, d, d, d, vp, vp]
    L.oracle_dxdt.argtypes = [vp, vp, vp, vp]
    L.oracle_jacobian.argtypes = [vp, vp, vp, d, vp, vp, vp]
    L.oracle_solve_reduced.argtypes = [vp, vp, vp, vp, d, vp, vp]
    L.oracle_integrate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, i32]
    L.oracle_calculate_ye.argtypes = [vp, vp]
    L.oracle_calculate_ye.restype = d
    L.oracle_sortedsum.argtypes = [vp, i32]
    L.oracle_sortedsum.restype = d
    L.oracle_set_rhs_noise.argtypes = [vp, i32]
    L.oracle_set_lu_permute.argtypes = [vp, i32]
    L.oracle_mix_d_lagrangian.argtypes = [i32, vp, vp, vp, vp]
    L.oracle_vital_reference.argtypes = [i32, d, d, d]
    L.oracle_vital_reference.restype = d
    L.oracle_mix_diffusion.argtypes = [i32, i32, vp, i32, vp, vp, vp, d, d, i32, vp]
    L.oracle_mix_diffusion.restype = i32
    L.oracle_nse.argtypes = [vp, i32, vp, vp, vp, vp, i32, vp, vp, vp, vp]
    L.oracle_integrate_trajectories.argtypes = [vp, i32, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp, i32]
    _L = L
    return L


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


class Oracle:
    def __init__(self, net, knobs):
        from importlib import import_module
        abi = import_module("nuppn_modular2-ininet3_b200.abi")
        self.L = load()
        self.net = net
        self.knobs = knobs
        self._desc = abi.make_desc(net)
        self._abi = abi
        self.h = self.L.oracle_net_create(C.byref(self._desc), C.byref(knobs))

    def __del__(self):
        try:
            self.L.oracle_net_destroy(self.h)
        except Exception:
            pass

    def nnz(self):
        return self.L.oracle_nnz(self.h)

    def jac_pattern(self):
        n = self.nnz()
        row = np.zeros(n, np.int32); col = np.zeros(n, np.int32)
        dmap = np.zeros(self.net.nre * 8, np.int32)
        self.L.oracle_jac_pattern(self.h, _p(row), _p(col), _p(dmap))
        return row, col, dmap.reshape(-1, 8)

    def evaluate_all_rates(self, t9, rho, ye, X):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        out = np.zeros((X.shape[0], self.net.nre))
        t9, rho, ye = (np.broadcast_to(np.asarray(a, float), (X.shape[0],)) for a in (t9, rho, ye))
        for z in range(X.shape[0]):
            row = np.ascontiguousarray(X[z]); o = np.zeros(self.net.nre)
            self.L.oracle_eval_rates(self.h, float(t9[z]), float(rho[z]), float(ye[z]), _p(row), _p(o))
            out[z] = o
        return out

    def calculate_dxdt(self, v, X):
        X = np.atleast_2d(X); v = np.atleast_2d(v)
        out = np.zeros((X.shape[0], self.net.nsp))
        for z in range(X.shape[0]):
            vr = np.ascontiguousarray(v[z], dtype=np.float64); xr = np.ascontiguousarray(X[z], dtype=np.float64)
            o = np.zeros(self.net.nsp)
            self.L.oracle_dxdt(self.h, _p(vr), _p(xr), _p(o))
            out[z] = o
        return out

    def calculate_jacobian(self, v, X, dt):
        X = np.atleast_2d(X); v = np.atleast_2d(v)
        nz, n = X.shape[0], self.nnz()
        dt = np.broadcast_to(np.asarray(dt, float), (nz,))
        jac = np.zeros((nz, n)); es = np.zeros((nz, n), np.uint8); mk = np.zeros((nz, self.net.nsp), np.uint8)
        for z in range(nz):
            vr = np.ascontiguousarray(v[z], dtype=np.float64); xr = np.ascontiguousarray(X[z], dtype=np.float64)
            j = np.zeros(n); e = np.zeros(n, np.uint8); m = np.zeros(self.net.nsp, np.uint8)
            self.L.oracle_jacobian(self.h, _p(vr), _p(xr), float(dt[z]), _p(j), _p(e), _p(m))
            jac[z], es[z], mk[z] = j, e, m
        return jac, es, mk

    def solve_reduced(self, jac, es, mask, dt, b):
        jac = np.atleast_2d(jac); nz = jac.shape[0]
        dt = np.broadcast_to(np.asarray(dt, float), (nz,))
        x = np.zeros((nz, self.net.nsp)); ierr = np.zeros(nz, np.int32)
        for z in range(nz):
            xo = np.zeros(self.net.nsp)
            ierr[z] = self.L.oracle_solve_reduced(
                self.h, _p(np.ascontiguousarray(jac[z])), _p(np.ascontiguousarray(np.atleast_2d(es)[z])),
                _p(np.ascontiguousarray(np.atleast_2d(mask)[z])), float(dt[z]),
                _p(np.ascontiguousarray(np.atleast_2d(b)[z], dtype=np.float64)), _p(xo))
            x[z] = xo
        return x, ierr

    def set_rhs_noise(self, seed):
        """seed >= 0: from now on every dX/dt entry is scaled by 1 - 2^-52, 1 or 1 + 2^-52 at random
        (a rounding-sized change, per zone and seed deterministic); None or < 0: off."""
        self.L.oracle_set_rhs_noise(self.h, -1 if seed is None else int(seed))

    def set_lu_permute(self, seed):
        """seed >= 0: from now on SuperLU factors every Bader-Deuflhard system under a seeded symmetric
        permutation (same system, another elimination order and rounding); None or < 0: off."""
        self.L.oracle_set_lu_permute(self.h, -1 if seed is None else int(seed))

    def integrate_network(self, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, bd_state=None, nthreads=1):
        X = np.array(np.atleast_2d(X), dtype=np.float64, order="C", copy=True)
        nz = X.shape[0]
        f = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, float), (nz,)))
        t9_0, t9_1, rho_0, rho_1, dtwant = f(t9_0), f(t9_1), f(rho_0), f(rho_1), f(dtwant)
        ye = np.array(f(ye), copy=True)
        ierr = np.zeros(nz, np.int32)
        stats = (self._abi.ZoneStats * nz)()
        bd = np.zeros(nz, np.int32) if bd_state is None else np.array(bd_state, dtype=np.int32, copy=True)
        self.L.oracle_integrate(self.h, nz, _p(X), X.shape[1], _p(t9_0), _p(t9_1), _p(rho_0), _p(rho_1), _p(ye),
                                _p(dtwant), _p(ierr), stats, _p(bd), int(nthreads))
        return X, ye, ierr, stats, bd

    def integrate_trajectories(self, X, time, t9, rho, nthreads=1):
        """tppnp's trajectory loop per zone: X[nz, nsp], per-zone time/t9/rho [nz, npts]."""
        X = np.array(np.atleast_2d(X), dtype=np.float64, order="C", copy=True)
        nz = X.shape[0]
        f = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, float), (nz, np.shape(a)[-1])))
        time, t9, rho = f(time), f(t9), f(rho)
        ye, ierr, fail = np.zeros(nz), np.zeros(nz, np.int32), np.zeros(nz, np.int32)
        stats = (self._abi.ZoneStats * nz)()
        self.L.oracle_integrate_trajectories(self.h, nz, time.shape[1], _p(X), X.shape[1], _p(time), _p(t9), _p(rho),
                                             _p(ye), _p(ierr), _p(fail), stats, int(nthreads))
        return X, ye, ierr, fail, stats

    def compute_nse(self, t9, rho, ye):
        """compute_nse (nse_swj.F90:272-384) per zone from a fresh state: X, mu_p, mu_n, iterations, ierr."""
        t9 = np.ascontiguousarray(np.atleast_1d(t9), dtype=np.float64)
        nz = len(t9)
        f = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, float), (nz,)))
        rho, ye = f(rho), f(ye)
        X = np.zeros((nz, self.net.nsp))
        mu_p, mu_n = np.zeros(nz), np.zeros(nz)
        it, ierr = np.zeros(nz, np.int32), np.zeros(nz, np.int32)
        if self.L.oracle_nse(self.h, nz, _p(t9), _p(rho), _p(ye), _p(X), self.net.nsp, _p(mu_p), _p(mu_n),
                             _p(it), _p(ierr)) != 0:
            raise ValueError("network has no protons or no Ni56 for NSE")
        return X, mu_p, mu_n, it, ierr

    def calculate_ye(self, X):
        x = np.ascontiguousarray(X, dtype=np.float64)
        return self.L.oracle_calculate_ye(self.h, _p(x))


def vital_reference(slot, t9, rho, xprot=0.0) -> float:
    """The reference's own VITAL formula for one slot (vital.F90:339-571; slots 1-9, 14-17, 73)."""
    return load().oracle_vital_reference(int(slot), float(t9), float(rho), float(xprot))


def mix_d_lagrangian(d_eul, rho, rad):
    """mix_calculate_D_Lagrangian (mixing.F90:60-98) on the CPU."""
    L = load()
    d_eul, rho, rad = (np.ascontiguousarray(v, np.float64) for v in (d_eul, rho, rad))
    out = np.zeros(d_eul.size)
    L.oracle_mix_d_lagrangian(d_eul.size, _p(d_eul), _p(rho), _p(rad), _p(out))
    return out


def mix_diffusion(X, d_lagr, dzeit, sig_term_limit, xm=None, dq=None, consider=None):
    """mixdiff08 (mixing.F90:104-146) on the CPU: one diffusion step of X[m, nsp] (shells x species)
    by matrixdiffus on xm, or matrixdiffus_mesa on dq when dq is given. Returns (X after the step,
    d_lagr as the matrix routine limited it, status: 0, or < 0 for a zero width or pivot)."""
    L = load()
    X = np.array(X, dtype=np.float64, order="C", copy=True)
    d = np.array(d_lagr, dtype=np.float64, copy=True)
    mesa = dq is not None
    xm_ = None if mesa else np.ascontiguousarray(xm, np.float64)
    dq_ = np.ascontiguousarray(dq, np.float64) if mesa else None
    cons = None if consider is None else np.ascontiguousarray(consider, np.uint8)
    st = L.oracle_mix_diffusion(X.shape[0], X.shape[1], _p(X), X.shape[1], _p(xm_), _p(dq_), _p(d), float(dzeit),
                                float(sig_term_limit), int(mesa), _p(cons))
    return X, d, st


def sortedsum(a) -> float:
    a = np.ascontiguousarray(a, dtype=np.float64)
    return load().oracle_sortedsum(_p(a), len(a))
