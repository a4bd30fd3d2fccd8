"""Host-side mirror of the reference's solver interface, over the C ABI (include/nuppn.h).

``Network`` arrays go in once (``NetworkSolver(net)``); afterwards the calls mirror the reference's
entry points, batched over zones:

* ``evaluate_all_rates(t9, rho, ye, X)``          physics/source/evaluate_rates.F90:14
* ``integrate_network(X, t9_0, t9_1, rho_0, rho_1, ye, dtwant)``   solver/source/solver.F90:53
* ``calculate_dxdt`` / ``calculate_jacobian``       solver/source/jac_rhs.F90:217, 282

Per-zone outcomes use the reference's error codes (``abi.ERROR_CODE``); library failures raise
``NuppnError``. The CUDA library is required: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import abi
from . import synthnet as sn

_LIB = None
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libnuppn_b200.so")


class NuppnError(RuntimeError):
    pass


def load_library():
    """Load libnuppn_b200.so (built in-tree); raise if it is missing."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise NuppnError(f"CUDA library not built: {LIB_PATH} (run __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    vp, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
    L.nuppn_abi_version.restype = i32
    L.nuppn_status_string.restype = C.c_char_p
    L.nuppn_status_string.argtypes = [i32]
    L.nuppn_last_error.restype = C.c_char_p
    L.nuppn_default_knobs.argtypes = [vp]
    L.nuppn_net_create.argtypes = [vp, vp, i32, C.POINTER(vp)]
    L.nuppn_net_destroy.argtypes = [vp]
    L.nuppn_net_info_get.argtypes = [vp, vp]
    L.nuppn_set_knobs.argtypes = [vp, vp]
    L.nuppn_jac_pattern.argtypes = [vp, vp, vp, vp]
    L.nuppn_eval_rates.argtypes = [vp, i32, vp, vp, vp, vp, i32, vp]
    L.nuppn_dxdt.argtypes = [vp, i32, vp, vp, i32, vp]
    L.nuppn_jacobian.argtypes = [vp, i32, vp, vp, i32, vp, vp, vp, vp]
    L.nuppn_solve_reduced.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp]
    L.nuppn_integrate.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_integrate_device.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_autotune.argtypes = [vp, i32, vp, i32, vp, vp, vp, vp, vp, vp, i32, vp, i32, vp]
    L.nuppn_integrate_multi.argtypes = [vp, i32, i32, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_integrate_multi_device.argtypes = [vp, i32, i32, vp, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_networksetup_write.argtypes = [C.c_char_p, vp]
    L.nuppn_networksetup_read.argtypes = [C.c_char_p, vp]
    L.nuppn_isotopedatabase_read.argtypes = [C.c_char_p, i32, vp, vp, vp, C.c_char_p]
    d = C.c_double
    L.nuppn_write_iso_massf.argtypes = [C.c_char_p, i32, d, d, d, d, d, d, d, d, i32, vp, vp, vp, vp, vp, vp]
    L.nuppn_write_flux.argtypes = [C.c_char_p, i32, vp, vp, vp, vp, vp, vp]
    L.nuppn_tppnp_header.argtypes = [C.c_char_p, vp, vp, vp]
    L.nuppn_mix_d_lagrangian.argtypes = [i32, vp, vp, vp, vp]
    L.nuppn_mix_diffusion.argtypes = [i32, i32, vp, C.c_int64, C.c_int64, vp, vp, vp, d, d, i32, vp]
    L.nuppn_mix_diffusion_device.argtypes = [i32, i32, vp, C.c_int64, C.c_int64, vp, vp, vp, d, d, i32, vp, vp]
    L.nuppn_tppnp_next.argtypes = [C.c_char_p, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_launch_count.argtypes = [vp]
    L.nuppn_launch_count.restype = i64
    L.nuppn_nse.argtypes = [vp, i32, vp, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_integrate_trajectories.argtypes = [vp, i32, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp]
    L.nuppn_integrate_trajectories_device.argtypes = [vp, i32, i32, vp, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    f64, i64 = C.c_double, C.c_int64
    L.nuppn_serve_open.argtypes = [vp, i32, i32, C.POINTER(vp)]
    L.nuppn_serve_submit.argtypes = [vp, vp, f64, f64, f64, f64, f64, f64, i32, C.POINTER(i64)]
    L.nuppn_serve_submit_trajectory.argtypes = [vp, vp, i32, vp, vp, vp, C.POINTER(i64)]
    L.nuppn_serve_poll.argtypes = [vp, i64, C.POINTER(i32), vp, vp, vp, vp, vp, vp]
    L.nuppn_serve_info.argtypes = [vp, vp]
    L.nuppn_serve_close.argtypes = [vp]
    for name in ("nuppn_net_create", "nuppn_net_destroy", "nuppn_net_info_get", "nuppn_set_knobs",
                 "nuppn_jac_pattern", "nuppn_eval_rates", "nuppn_dxdt", "nuppn_jacobian",
                 "nuppn_solve_reduced", "nuppn_integrate", "nuppn_integrate_device", "nuppn_nse",
                 "nuppn_integrate_trajectories", "nuppn_integrate_trajectories_device",
                 "nuppn_serve_open", "nuppn_serve_submit", "nuppn_serve_submit_trajectory", "nuppn_serve_poll",
                 "nuppn_serve_info", "nuppn_serve_close", "nuppn_autotune", "nuppn_integrate_multi",
                 "nuppn_integrate_multi_device", "nuppn_networksetup_write", "nuppn_networksetup_read",
                 "nuppn_isotopedatabase_read", "nuppn_write_iso_massf", "nuppn_write_flux", "nuppn_tppnp_header", "nuppn_tppnp_next", "nuppn_mix_d_lagrangian", "nuppn_mix_diffusion",
                 "nuppn_mix_diffusion_device"):
        getattr(L, name).restype = i32
    _LIB = L
    return L


def _p(a):
    return None if a is None else C.c_void_p(a.ctypes.data)


def _f64(a, n=None):
    """Per-zone float64 array; a scalar (or a length-1 array) is broadcast to n zones."""
    a = np.asarray(a, dtype=np.float64)
    if n is not None:
        if a.size == 1:
            a = np.full(n, float(a.reshape(-1)[0]))
        elif a.shape != (n,):
            raise ValueError(f"expected {n} per-zone values, got shape {a.shape}")
    return np.ascontiguousarray(a)


class NetworkSolver:
    """One network on one device (the module state of the reference, as a handle)."""

    def __init__(self, net: sn.Network, knobs: abi.Knobs | None = None, device: int = 0):
        self.L = load_library()
        self.net = net
        self.knobs = knobs or abi.default_knobs()
        self._desc = abi.make_desc(net)
        h = C.c_void_p()
        self._check(self.L.nuppn_net_create(C.byref(self._desc), C.byref(self.knobs), device, C.byref(h)))
        self.h = h
        info = abi.NetInfo()
        self._check(self.L.nuppn_net_info_get(self.h, C.byref(info)))
        self.info = info
        # right after creation the handle holds only the zone-shared network arena (and a 256-byte
        # zone counter): the workspace and staging buffers are allocated by the first call
        self.arena_bytes = int(info.device_bytes)

    def _check(self, st):
        if st != 0:
            msg = self.L.nuppn_last_error().decode()
            raise NuppnError(f"{self.L.nuppn_status_string(st).decode()}: {msg}")

    def close(self):
        if getattr(self, "h", None):
            self.L.nuppn_net_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_knobs(self, knobs: abi.Knobs):
        self.knobs = knobs
        self._check(self.L.nuppn_set_knobs(self.h, C.byref(knobs)))

    @property
    def nsp(self):
        return self.net.nsp

    @property
    def nre(self):
        return self.net.nre

    def launches(self) -> int:
        return int(self.L.nuppn_launch_count(self.h))

    def jac_pattern(self):
        nnz = self.info.nnz_jac
        row = np.zeros(nnz, np.int32); col = np.zeros(nnz, np.int32)
        dmap = np.zeros(self.nre * 8, np.int32)
        self._check(self.L.nuppn_jac_pattern(self.h, _p(row), _p(col), _p(dmap)))
        return row, col, dmap.reshape(self.nre, 8)

    def evaluate_all_rates(self, t9, rho, ye, X):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        nz = X.shape[0]
        t9, rho, ye = _f64(t9, nz), _f64(rho, nz), _f64(ye, nz)
        v = np.zeros((nz, self.nre))
        self._check(self.L.nuppn_eval_rates(self.h, nz, _p(t9), _p(rho), _p(ye), _p(X), X.shape[1], _p(v)))
        return v

    def calculate_dxdt(self, v, X):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        v = np.ascontiguousarray(np.atleast_2d(v), dtype=np.float64)
        out = np.zeros((X.shape[0], self.nsp))
        self._check(self.L.nuppn_dxdt(self.h, X.shape[0], _p(v), _p(X), X.shape[1], _p(out)))
        return out

    def calculate_jacobian(self, v, X, dt):
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        v = np.ascontiguousarray(np.atleast_2d(v), dtype=np.float64)
        nz = X.shape[0]
        dt = _f64(dt, nz)
        nnz = self.info.nnz_jac
        jac = np.zeros((nz, nnz)); es = np.zeros((nz, nnz), np.uint8); mask = np.zeros((nz, self.nsp), np.uint8)
        self._check(self.L.nuppn_jacobian(self.h, nz, _p(v), _p(X), X.shape[1], _p(dt), _p(jac), _p(es), _p(mask)))
        return jac, es, mask

    def solve_reduced(self, jac, entry_set, mask, dt, b):
        jac = np.ascontiguousarray(np.atleast_2d(jac), dtype=np.float64)
        nz = jac.shape[0]
        es = np.ascontiguousarray(np.atleast_2d(entry_set), dtype=np.uint8)
        mk = np.ascontiguousarray(np.atleast_2d(mask), dtype=np.uint8)
        b = np.ascontiguousarray(np.atleast_2d(b), dtype=np.float64)
        dt = _f64(dt, nz)
        x = np.zeros((nz, self.nsp))
        self._check(self.L.nuppn_solve_reduced(self.h, nz, _p(jac), _p(es), _p(mk), _p(dt), _p(b), _p(x)))
        return x

    def integrate_trajectories(self, X, time, t9, rho):
        """tppnp's trajectory loop for every zone in one launch (nuppn_integrate_trajectories):
        X[nz, nsp] starting compositions, per-zone time/t9/rho [nz, npts]. Returns (X, ye, ierr, fail,
        stats)."""
        X = np.array(np.atleast_2d(X), dtype=np.float64, order="C", copy=True)
        nz = X.shape[0]
        f = lambda a: np.ascontiguousarray(np.broadcast_to(np.asarray(a, np.float64), (nz, np.shape(a)[-1])))
        time, t9, rho = f(time), f(t9), f(rho)
        ye, ierr, fail = np.zeros(nz), np.zeros(nz, np.int32), np.zeros(nz, np.int32)
        stats = (abi.ZoneStats * nz)()
        p = lambda a: C.c_void_p(a.ctypes.data)
        self._check(self.L.nuppn_integrate_trajectories(self.h, nz, time.shape[1], p(X), X.shape[1], p(time), p(t9),
                                                        p(rho), p(ye), p(ierr), p(fail), stats))
        return X, ye, ierr, fail, stats

    def integrate_trajectories_device(self, X, time, t9, rho, ye, ierr, fail=None, stats=None, bd_state=None,
                                      stream=0):
        """Device-resident form (torch CUDA tensors); time/t9/rho are [nz, npts]."""
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        self._check(self.L.nuppn_integrate_trajectories_device(
            self.h, X.shape[0], time.shape[1], ptr(X), X.shape[1], ptr(time), ptr(t9), ptr(rho), ptr(ye), ptr(ierr),
            ptr(fail), ptr(stats), ptr(bd_state), C.c_void_p(stream)))

    def compute_nse(self, t9, rho, ye):
        """compute_nse per zone (nuppn_nse): X[nz, nsp], mu_p, mu_n, iterations, ierr."""
        t9 = np.ascontiguousarray(np.atleast_1d(t9), dtype=np.float64)
        nz = len(t9)
        rho, ye = _f64(rho, nz), _f64(ye, nz)
        X = np.zeros((nz, self.nsp))
        mu_p, mu_n = np.zeros(nz), np.zeros(nz)
        it, ierr = np.zeros(nz, np.int32), np.zeros(nz, np.int32)
        p = lambda a: C.c_void_p(a.ctypes.data)
        self._check(self.L.nuppn_nse(self.h, nz, p(t9), p(rho), p(ye), p(X), p(mu_p), p(mu_n), p(it), p(ierr)))
        return X, mu_p, mu_n, it, ierr

    def integrate_network(self, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, bd_state=None):
        """Advance every zone; returns (X, ye, ierr, stats, bd_state). X is not modified."""
        X = np.array(np.atleast_2d(X), dtype=np.float64, order="C", copy=True)
        nz = X.shape[0]
        t9_0, t9_1, rho_0, rho_1 = _f64(t9_0, nz), _f64(t9_1, nz), _f64(rho_0, nz), _f64(rho_1, nz)
        ye = np.array(_f64(ye, nz), copy=True)
        dtwant = _f64(dtwant, nz)
        ierr = np.zeros(nz, np.int32)
        stats = (abi.ZoneStats * nz)()
        bd = np.zeros(nz, np.int32) if bd_state is None else np.array(bd_state, dtype=np.int32, copy=True)
        self._check(self.L.nuppn_integrate(self.h, nz, _p(X), X.shape[1], _p(t9_0), _p(t9_1), _p(rho_0),
                                           _p(rho_1), _p(ye), _p(dtwant), _p(ierr), stats, _p(bd)))
        return X, ye, ierr, stats, bd

    def autotune(self, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, sample=0):
        """nuppn_autotune: time each kernel shape on this batch (host arrays), keep the fastest.
        Returns one dict per candidate (shape knobs, zones per SM, ms per call, zone-steps/s, chosen)."""
        X = np.ascontiguousarray(np.atleast_2d(X), dtype=np.float64)
        nz = X.shape[0]
        f = lambda a: _f64(a, nz)
        args = [f(a) for a in (t9_0, t9_1, rho_0, rho_1, ye, dtwant)]
        rep = (abi.TuneResult * 16)()
        n = C.c_int32(0)
        self._check(self.L.nuppn_autotune(self.h, nz, _p(X), X.shape[1], *[_p(a) for a in args], int(sample), rep, 16,
                                          C.byref(n)))
        return [{k: getattr(rep[i], k) for k, _ in abi.TuneResult._fields_ if k != "reserved"}
                for i in range(n.value)]

    def integrate_device(self, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, ierr, stats=None, bd_state=None,
                         stream=0):
        """Device-resident form: arguments are torch CUDA tensors (or objects with data_ptr())."""
        ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
        self._check(self.L.nuppn_integrate_device(
            self.h, X.shape[0], ptr(X), X.shape[1], ptr(t9_0), ptr(t9_1), ptr(rho_0), ptr(rho_1), ptr(ye),
            ptr(dtwant), ptr(ierr), ptr(stats), ptr(bd_state), C.c_void_p(stream)))


# rate-source labels written to networksetup.txt's lab column, by descriptor source (NUPPN_SRC_*)
_SRC_LABEL = {0: "OOOOO", 1: "VITAL", 2: "JINAC", 3: "NETB1", 4: "FFW85", 5: "KADON", 6: "ALPHA"}


def _str5(items):
    return b"".join(s.encode()[:5].ljust(5) for s in items)


def networksetup_write(path, net, t9=0.0, rho=0.0, v=None):
    """write_networksetup (networksetup.F90:55-115) for a network description: its species, their
    switches, A and Z, and every reaction slot with k1..k8, the reaction type label and the rate
    factor; v (the rates at t9, rho) is written as 0 if not given. Host only."""
    L = load_library()
    nsp, nre = net.nsp, net.nre
    zis = C.create_string_buffer(_str5(net.zis), 5 * nsp)
    labb = C.create_string_buffer(_str5([sn.RLABELS.get(int(t), "     ") for t in net.ilabb]), 5 * nre)
    lab = C.create_string_buffer(_str5([_SRC_LABEL.get(int(x), "     ") for x in net.src]), 5 * nre)
    arr = {"considerisotope": np.ascontiguousarray(net.considerisotope, np.uint8),
           "anetw": np.ascontiguousarray(net.anetw, np.float64), "znetw": np.ascontiguousarray(net.znetw, np.float64),
           "isomeric_state": np.ones(nsp, np.int32),
           "considerreaction": np.ascontiguousarray(net.considerreaction, np.uint8),
           "k": np.ascontiguousarray(net.k, np.int32),
           "v": np.zeros(nre) if v is None else np.ascontiguousarray(v, np.float64),
           "ilabb": np.ascontiguousarray(net.ilabb, np.int32), "rfac": np.ascontiguousarray(net.rfac, np.float64),
           "bind_energy_diff": np.zeros(nre)}
    ns = abi.NetSetup(nsp=nsp, nre=nre, nisomers=0, nreac_isomers=0, t9=float(t9), rho=float(rho),
                      zis=C.cast(zis, C.c_void_p), lab=C.cast(lab, C.c_void_p), labb=C.cast(labb, C.c_void_p),
                      **{k: a.ctypes.data for k, a in arr.items()})
    if L.nuppn_networksetup_write(str(path).encode(), C.byref(ns)) != 0:
        raise NuppnError(L.nuppn_last_error().decode())


def networksetup_read(path):
    """read_networksetup (networksetup.F90:140-260): a dict of the file's arrays (zis, lab, labb as
    lists of 5-character strings; k as [nre, 8] with 0-based species indices) and its header."""
    L = load_library()
    ns = abi.NetSetup()
    if L.nuppn_networksetup_read(str(path).encode(), C.byref(ns)) != 0:
        raise NuppnError(L.nuppn_last_error().decode())
    nsp, nre = ns.nsp, ns.nre
    zis, lab, labb = (C.create_string_buffer(5 * max(n, 1)) for n in (nsp, nre, nre))
    arr = {"considerisotope": np.zeros(nsp, np.uint8), "anetw": np.zeros(nsp), "znetw": np.zeros(nsp),
           "isomeric_state": np.zeros(nsp, np.int32), "considerreaction": np.zeros(nre, np.uint8),
           "k": np.zeros((nre, 8), np.int32), "v": np.zeros(nre), "ilabb": np.zeros(nre, np.int32),
           "rfac": np.zeros(nre), "bind_energy_diff": np.zeros(nre)}
    for k, a in arr.items():
        setattr(ns, k, a.ctypes.data)
    ns.zis, ns.lab, ns.labb = (C.cast(b, C.c_void_p) for b in (zis, lab, labb))
    if L.nuppn_networksetup_read(str(path).encode(), C.byref(ns)) != 0:
        raise NuppnError(L.nuppn_last_error().decode())
    split = lambda b, n: [b.raw[5 * i:5 * i + 5].decode() for i in range(n)]
    arr.update(zis=split(zis, nsp), lab=split(lab, nre), labb=split(labb, nre), t9=ns.t9, rho=ns.rho,
               nisomers=ns.nisomers, nreac_isomers=ns.nreac_isomers)
    return arr


AVOGADRO = 6.022140857e23  # constants.F90:29, the value the reference's number densities use


def write_iso_massf(path, net, X, model, dzeit, agej, t9, rho, total_energy_flux=0.0, isomeric_state=None):
    """ppn's iso_massf<mmmmm>.DAT (printonecycle, ppn.F90:519-536) for one zone's abundances X of a
    network description, byte for byte: the header with the neutron, proton and alpha number
    densities as the reference computes them (X(n) rho N_A, X(p) rho N_A, X(He4)/4 rho N_A) and one
    line per considered species. Host only."""
    L = load_library()
    X = np.ascontiguousarray(X, np.float64)
    nsp = net.nsp
    if X.shape != (nsp,):
        raise NuppnError(f"X must have {nsp} entries")
    yn = X[net.species_index("NEUT ")]
    yp = X[net.species_index("PROT ")]
    ya = X[net.species_index("HE  4")] * 0.25
    z = np.ascontiguousarray(net.znetw, np.float64)
    a = np.ascontiguousarray(net.anetw, np.float64)
    iso = np.ones(nsp, np.int32) if isomeric_state is None else np.ascontiguousarray(isomeric_state, np.int32)
    cons = np.ascontiguousarray(net.considerisotope, np.uint8)
    names = C.create_string_buffer(_str5(net.zis), 5 * nsp)
    st = L.nuppn_write_iso_massf(str(path).encode(), int(model), float(dzeit), float(agej), float(t9), float(rho),
                                 yn * rho * AVOGADRO, yp * rho * AVOGADRO, ya * rho * AVOGADRO,
                                 float(total_energy_flux), nsp, _p(z), _p(a), _p(iso), _p(X),
                                 C.cast(names, C.c_void_p), _p(cons))
    if st != 0:
        raise NuppnError(L.nuppn_last_error().decode())


def write_flux(path, net, flux, bind_energy_diff, timescale, nreac=None):
    """ppn's flux_<mmmmm>.DAT (printonecycle, ppn.F90:496-510), byte for byte: per network reaction
    (the first nreac slots, all by default) Z and A of k1, k3, k5 and k7, the flux dY/dt, the energy
    flux * bind_energy_diff and the reaction's time scale, clamped as the reference prints them. Host
    only."""
    L = load_library()
    n = net.nre if nreac is None else int(nreac)
    flux = np.ascontiguousarray(flux, np.float64)[:n]
    energy = np.ascontiguousarray(flux * np.asarray(bind_energy_diff, np.float64)[:n])
    ts = np.ascontiguousarray(timescale, np.float64)[:n]
    k = np.ascontiguousarray(np.asarray(net.k)[:n], np.int32)
    z = np.ascontiguousarray(net.znetw, np.float64)
    a = np.ascontiguousarray(net.anetw, np.float64)
    st = L.nuppn_write_flux(str(path).encode(), n, _p(k), _p(z), _p(a), _p(flux), _p(energy), _p(ts))
    if st != 0:
        raise NuppnError(L.nuppn_last_error().decode())


def mix_d_lagrangian(d_eul, rho, rad):
    """mppnp's mix_calculate_D_Lagrangian (mixing.F90:60-98): the Lagrangian diffusion coefficient
    of each shell from the Eulerian one, the density and the radius (solar units). Host only."""
    L = load_library()
    d_eul, rho, rad = (np.ascontiguousarray(v, np.float64) for v in (d_eul, rho, rad))
    out = np.zeros(d_eul.size)
    if L.nuppn_mix_d_lagrangian(d_eul.size, _p(d_eul), _p(rho), _p(rad), _p(out)) != 0:
        raise NuppnError(L.nuppn_last_error().decode())
    return out


def _mix_strides(shape, strides):
    """(shell_stride, species_stride) in elements of a float64 array X[shells, species]."""
    sh, sp = (st // 8 for st in strides)
    return (sh, 1) if shape[1] == 1 and sp != 1 else ((1, sp) if shape[0] == 1 and sh != 1 else (sh, sp))


def mix_diffusion(X, d_lagr, dzeit, sig_term_limit, xm=None, dq=None, consider=None):
    """mppnp's diffusive mixing step (mixdiff08, mixing.F90:104-146) on the GPU: X[m, nsp] (shells x
    species) after one fully implicit step of dzeit, by matrixdiffus on the mass coordinates xm, or
    matrixdiffus_mesa on the shell masses dq when dq is given. X may be C-ordered (rows of species) or
    Fortran-ordered (columns of shells, mppnp's yps layout); the result keeps its order. Returns (X,
    d_lagr as limited by sig_term_limit); X is not modified."""
    L = load_library()
    X = np.array(X, dtype=np.float64, order="F" if np.isfortran(X) else "C", copy=True)
    d = np.array(d_lagr, dtype=np.float64, copy=True)
    mesa = dq is not None
    xm_ = None if mesa else np.ascontiguousarray(xm, np.float64)
    dq_ = np.ascontiguousarray(dq, np.float64) if mesa else None
    cons = None if consider is None else np.ascontiguousarray(consider, np.uint8)
    sh, sp = _mix_strides(X.shape, X.strides)
    if L.nuppn_mix_diffusion(X.shape[0], X.shape[1], _p(X), sh, sp, _p(xm_), _p(dq_), _p(d), float(dzeit),
                             float(sig_term_limit), int(mesa), _p(cons)) != 0:
        raise NuppnError(L.nuppn_last_error().decode())
    return X, d


def mix_diffusion_device(X, d_lagr, dzeit, sig_term_limit, xm=None, dq=None, consider=None, stream=None):
    """mix_diffusion on a device-resident float64 tensor X[m, nsp] (shells x species), in place, on
    `stream` (a torch.cuda.Stream or None): rows of species (X.stride(1) == 1, e.g. a column slice of
    a wider array) or columns of shells (X.stride(0) == 1, e.g. the transpose of a [nsp, msl] array).
    Returns d_lagr as limited by sig_term_limit."""
    import torch

    L = load_library()
    if not X.is_cuda or X.dtype != torch.float64 or X.dim() != 2:
        raise NuppnError("mix_diffusion_device: X must be a 2-D float64 CUDA tensor")
    d = np.array(d_lagr, dtype=np.float64, copy=True)
    mesa = dq is not None
    xm_ = None if mesa else np.ascontiguousarray(xm, np.float64)
    dq_ = np.ascontiguousarray(dq, np.float64) if mesa else None
    cons = None if consider is None else np.ascontiguousarray(consider, np.uint8)
    sp_ = None if stream is None else C.c_void_p(stream.cuda_stream)
    sh, sp = _mix_strides(tuple(X.shape), tuple(8 * st for st in X.stride()))
    if L.nuppn_mix_diffusion_device(X.shape[0], X.shape[1], C.c_void_p(X.data_ptr()), sh, sp, _p(xm_), _p(dq_),
                                    _p(d), float(dzeit), float(sig_term_limit), int(mesa), _p(cons), sp_) != 0:
        raise NuppnError(L.nuppn_last_error().decode())
    return d


def tppnp_read(path, limit=None):
    """tppnp's binary trajectory file (traj_data.F90:73-168): a list of dicts, one per tracer (the
    first `limit`), with pnum, mass, posini, posfin, time (s), t9 (the file's temperature / 1e9),
    rho (g/cm^3) and the initial composition a, z, zis (5-character names) and x. Host only."""
    L = load_library()
    hdr = [C.c_int32() for _ in range(3)]
    if L.nuppn_tppnp_header(str(path).encode(), *[C.byref(h) for h in hdr]) != 0:
        raise NuppnError(L.nuppn_last_error().decode())
    n = hdr[0].value if limit is None else min(int(limit), hdr[0].value)
    pos = C.c_int64(0)
    out = []
    for _ in range(n):
        pn, nt, ni = C.c_int32(), C.c_int32(), C.c_int32()
        mass = C.c_double()
        pi, pf = np.zeros(3), np.zeros(3)
        args = [C.byref(pos), C.byref(pn), C.byref(nt), C.byref(ni), C.byref(mass), _p(pi), _p(pf)]
        if L.nuppn_tppnp_next(str(path).encode(), *args, None, None, None, None, None, None, None) != 0:
            raise NuppnError(L.nuppn_last_error().decode())
        t, t9, rho = np.zeros(nt.value), np.zeros(nt.value), np.zeros(nt.value)
        a, z, x = np.zeros(ni.value, np.int32), np.zeros(ni.value, np.int32), np.zeros(ni.value)
        zis = C.create_string_buffer(5 * max(ni.value, 1))
        if L.nuppn_tppnp_next(str(path).encode(), *args, _p(t), _p(t9), _p(rho), _p(a), _p(z),
                              C.cast(zis, C.c_void_p), _p(x)) != 0:
            raise NuppnError(L.nuppn_last_error().decode())
        names = [zis.raw[5 * i:5 * i + 5].decode() for i in range(ni.value)]
        out.append({"pnum": pn.value, "mass": mass.value, "posini": pi, "posfin": pf, "time": t, "t9": t9,
                    "rho": rho, "a": a, "z": z, "zis": names, "x": x})
    return out, {"num_tracers": hdr[0].value, "nsteps_min": hdr[1].value, "nsteps_max": hdr[2].value}


def tppnp_initial_abundances(net, traj):
    """A tracer's initial composition on a network's species, matched by (Z, A), as tppnp's
    abundance initialisation sets x_in = max(x, 1e-99) by species (traj_data.F90:160-163); species
    the tracer does not list, and listed isotopes the network lacks, are left at 1e-99 / dropped.
    Returns (X[nsp], the tracer's mass fraction that found no species)."""
    X = np.full(net.nsp, 1e-99)
    where = {(int(zz), int(aa)): i for i, (zz, aa) in enumerate(zip(net.znetw, net.anetw))
             if net.zis[i] != "OOOOO"}
    lost = 0.0
    for zz, aa, xx in zip(traj["z"], traj["a"], traj["x"]):
        i = where.get((int(zz), int(aa)))
        if i is None:
            lost += max(float(xx), 0.0)
        else:
            X[i] = max(float(xx), 1e-99)
    return X, lost


def _handles(solvers):
    arr = (C.c_void_p * len(solvers))(*[s.h.value for s in solvers])
    return arr


def integrate_multi(solvers, net_of, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, bd_state=None):
    """nuppn_integrate_multi: zones of several networks (solvers[net_of[z]]) in one launch. X rows have
    the largest network's nsp entries (zone z uses the first nsp of its own). Returns (X, ye, ierr,
    stats, bd_state); X is not modified."""
    X = np.array(np.atleast_2d(X), dtype=np.float64, order="C", copy=True)
    nz = X.shape[0]
    net_of = np.ascontiguousarray(net_of, dtype=np.int32)
    t9_0, t9_1, rho_0, rho_1 = _f64(t9_0, nz), _f64(t9_1, nz), _f64(rho_0, nz), _f64(rho_1, nz)
    ye = np.array(_f64(ye, nz), copy=True)
    dtwant = _f64(dtwant, nz)
    ierr = np.zeros(nz, np.int32)
    stats = (abi.ZoneStats * nz)()
    bd = np.zeros(nz, np.int32) if bd_state is None else np.array(bd_state, dtype=np.int32, copy=True)
    s0 = solvers[0]
    s0._check(s0.L.nuppn_integrate_multi(_handles(solvers), len(solvers), nz, _p(net_of), _p(X), X.shape[1],
                                         _p(t9_0), _p(t9_1), _p(rho_0), _p(rho_1), _p(ye), _p(dtwant), _p(ierr),
                                         stats, _p(bd)))
    return X, ye, ierr, stats, bd


def integrate_multi_device(solvers, net_of, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, ierr, stats=None,
                           bd_state=None, stream=0):
    """Device-resident form of integrate_multi: torch CUDA tensors (or objects with data_ptr())."""
    ptr = lambda t: None if t is None else C.c_void_p(t.data_ptr())
    s0 = solvers[0]
    s0._check(s0.L.nuppn_integrate_multi_device(
        _handles(solvers), len(solvers), int(X.shape[0]), ptr(net_of), ptr(X), int(X.shape[1]), ptr(t9_0),
        ptr(t9_1), ptr(rho_0), ptr(rho_1), ptr(ye), ptr(dtwant), ptr(ierr), ptr(stats), ptr(bd_state),
        C.c_void_p(stream)))


class Server:
    """A device-resident request loop (nuppn_serve_*): each request is one zone (integrate_network's
    arguments) or one trajectory; a persistent launch takes requests from a device queue as they are
    submitted, one per zone group, and returns each result as soon as it is done. `slots` = zones
    integrated at once (0: all the GPU holds), `queue` = requests on the device at once (0: 4 x slots).
    Submit, poll and close from one thread; do not change the solver's knobs while the server is open."""

    def __init__(self, solver: NetworkSolver, slots: int = 0, queue: int = 0):
        self.solver, self.L = solver, solver.L
        h = C.c_void_p()
        solver._check(self.L.nuppn_serve_open(solver.h, int(slots), int(queue), C.byref(h)))
        self.h = h

    def submit(self, X, t9_0, t9_1, rho_0, rho_1, ye, dtwant, bd_state=0) -> int:
        x = np.ascontiguousarray(X, dtype=np.float64)
        rid = C.c_int64()
        self.solver._check(self.L.nuppn_serve_submit(self.h, _p(x), float(t9_0), float(t9_1), float(rho_0),
                                                     float(rho_1), float(ye), float(dtwant), int(bd_state),
                                                     C.byref(rid)))
        return rid.value

    def submit_trajectory(self, X, time, t9, rho) -> int:
        x = np.ascontiguousarray(X, dtype=np.float64)
        tt, tp, tr = (np.ascontiguousarray(a, dtype=np.float64) for a in (time, t9, rho))
        rid = C.c_int64()
        self.solver._check(self.L.nuppn_serve_submit_trajectory(self.h, _p(x), tt.size, _p(tt), _p(tp), _p(tr),
                                                                C.byref(rid)))
        return rid.value

    def poll(self, rid: int):
        """None while the request runs, else (X, ye, ierr, stats, bd_state, fail)."""
        if getattr(self, "_xbuf", None) is None:
            self._xbuf = np.zeros(self.solver.nsp)
        done = C.c_int32()
        ye, ierr, bd, fail = C.c_double(), C.c_int32(), C.c_int32(), C.c_int32()
        st = abi.ZoneStats()
        self.solver._check(self.L.nuppn_serve_poll(self.h, rid, C.byref(done), _p(self._xbuf), C.byref(ye),
                                                   C.byref(ierr), C.byref(st), C.byref(bd), C.byref(fail)))
        if not done.value:
            return None
        return self._xbuf.copy(), ye.value, ierr.value, st, bd.value, fail.value

    def wait(self, rid: int, timeout: float = 300.0):
        import time as _time
        t_end = _time.monotonic() + timeout
        while True:
            r = self.poll(rid)
            if r is not None:
                return r
            if _time.monotonic() > t_end:
                raise TimeoutError(f"request {rid} not finished after {timeout} s")
            _time.sleep(2e-4)

    def info(self) -> abi.ServeStats:
        s = abi.ServeStats()
        self.solver._check(self.L.nuppn_serve_info(self.h, C.byref(s)))
        return s

    def close(self):
        if self.h:
            self.L.nuppn_serve_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
