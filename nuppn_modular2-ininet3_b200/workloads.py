"""Seeded zone batches for the benchmark and parity cases (numpy default_rng, PCG64).

* ``hburn_zone``    ppn-style single H-burning zone, ~300-species network, backward Euler,
                    T9 = 0.020, rho = 100, X(H1) = 0.70, X(He4) = 0.28, Z = 0.02 over stable species,
                    200 frame steps with dt log-spaced 1e3 .. 1e13 s.
* ``heshell_batch`` He-burning shell zones on the ~1100-species network, Bader-Deuflhard:
                    T9 ~ U[0.10, 0.30], rho log-U[1e2, 1e4], X(He4) = 0.97, X(C12) = 0.01,
                    X(Ne22) = 0.02, trace Fe56 = 1e-3 (renormalised), each species x lognormal(0.05),
                    one integrate_network call of 1e10 s per zone.
"""
from __future__ import annotations

import dataclasses

import numpy as np

from . import synthnet as sn


@dataclasses.dataclass
class ZoneBatch:
    X: np.ndarray
    t9_0: np.ndarray
    t9_1: np.ndarray
    rho_0: np.ndarray
    rho_1: np.ndarray
    ye: np.ndarray
    dtwant: np.ndarray

    @property
    def nz(self):
        return self.X.shape[0]

    def take(self, idx):
        return ZoneBatch(*(getattr(self, f.name)[idx] for f in dataclasses.fields(self)))


def _ye_of(net: sn.Network, X: np.ndarray) -> np.ndarray:
    """calculate_ye (utils.F90:537-553) on a batch, for the initial Ye of a composition."""
    a = net.anetw.copy()
    a[a == 0] = 1.0
    eta = np.where(net.considerisotope.astype(bool), (net.anetw - 2.0 * net.znetw) * X / a, 0.0)
    return (1.0 - eta.sum(axis=1)) * 0.5


_NETS: dict = {}


def network(nnn: int, seed: int = 20240611, database: str | None = None) -> sn.Network:
    key = (nnn, seed, database)
    if key not in _NETS:
        _NETS[key] = sn.build_network(nnn, seed, database=database)
    return _NETS[key]


def heshell_batch(nz: int, net: sn.Network | None = None, seed: int = 2, dtwant: float = 1.0e10) -> ZoneBatch:
    net = net or network(1107)
    rng = np.random.default_rng(seed)
    X = np.full((nz, net.nsp), 1.0e-99)
    base = {"HE  4": 0.97, "C  12": 0.01, "NE 22": 0.02, "FE 56": 1.0e-3}
    for name, x in base.items():
        if name in net.zis:  # small networks may stop below Fe
            X[:, net.species_index(name)] = x
    X /= X.sum(axis=1, keepdims=True)
    nonz = X > 1e-90
    X = np.where(nonz, X * np.exp(rng.normal(0.0, 0.05, size=X.shape)), X)
    X /= np.where(nonz, X, 0.0).sum(axis=1, keepdims=True) + np.where(~nonz, X, 0.0).sum(axis=1, keepdims=True)
    t9 = rng.uniform(0.10, 0.30, nz)
    rho = 10.0 ** rng.uniform(2.0, 4.0, nz)
    return ZoneBatch(X=X, t9_0=t9.copy(), t9_1=t9.copy(), rho_0=rho.copy(), rho_1=rho.copy(),
                     ye=_ye_of(net, X), dtwant=np.full(nz, dtwant))


def nse_batch(nz: int, net: sn.Network | None = None, seed: int = 5, dtwant: float = 1.0e-2) -> ZoneBatch:
    """Hot zones in nuclear statistical equilibrium: T9 ~ U[6, 10], rho log-U[1e6, 1e8],
    Ye ~ U[0.46, 0.50]; the starting composition is a Si28 seed (replaced by the NSE distribution
    on the first step). One integrate_network call of dtwant seconds each."""
    net = net or network(1107)
    rng = np.random.default_rng(seed)
    X = np.full((nz, net.nsp), 1.0e-99)
    X[:, net.species_index("SI 28")] = 1.0
    t9 = rng.uniform(6.0, 10.0, nz)
    rho = 10.0 ** rng.uniform(6.0, 8.0, nz)
    ye = rng.uniform(0.46, 0.50, nz)
    return ZoneBatch(X=X, t9_0=t9.copy(), t9_1=t9.copy(), rho_0=rho.copy(), rho_1=rho.copy(), ye=ye,
                     dtwant=np.full(nz, dtwant))


@dataclasses.dataclass
class Trajectories:
    """Explosive-burning trajectories T9(t) = T9_0 exp(-t / (3 tau)), rho(t) = rho_0 exp(-t / tau) on a
    common time grid; X0 and Ye0 are the starting composition and electron fraction."""
    t9_0: np.ndarray
    rho_0: np.ndarray
    tau: np.ndarray
    X0: np.ndarray
    ye0: np.ndarray
    times: np.ndarray

    @property
    def nz(self):
        return len(self.t9_0)

    def t9(self, t):
        return self.t9_0 * np.exp(-t / (3.0 * self.tau))

    def rho(self, t):
        return self.rho_0 * np.exp(-t / self.tau)

    def grids(self):
        """Per-zone time, T9 and rho at every grid point, [nz, npts] each."""
        tt = np.broadcast_to(self.times, (self.nz, len(self.times))).copy()
        return tt, self.t9(tt.T).T.copy(), self.rho(tt.T).T.copy()

    def interval(self, k, X, ye):
        """ZoneBatch for grid interval k (times[k] .. times[k+1]) from the state X, ye."""
        t0, t1 = self.times[k], self.times[k + 1]
        return ZoneBatch(X=X, t9_0=self.t9(t0), t9_1=self.t9(t1), rho_0=self.rho(t0), rho_1=self.rho(t1), ye=ye,
                         dtwant=np.full(self.nz, t1 - t0))


def trajectory_batch(nz: int, net: sn.Network | None = None, seed: int = 7, t9_range=(2.0, 5.0),
                     npts: int = 201, t_end: float = 10.0) -> Trajectories:
    """tppnp-style trajectories: T9_0 ~ U[t9_range], rho_0 log-U[1e6, 1e8] g/cm^3, tau ~ U[0.1, 1] s,
    Ye ~ U[0.48, 0.50], on npts points: t = 0 and npts-1 log-spaced times from 1e-6 s to t_end. The
    seed is Si28 with the Fe56 admixture that gives the drawn Ye (Ye from the composition as
    calculate_ye, utils.F90:537-553)."""
    net = net or network(1107)
    rng = np.random.default_rng(seed)
    t9_0 = rng.uniform(t9_range[0], t9_range[1], nz)
    rho_0 = 10.0 ** rng.uniform(6.0, 8.0, nz)
    tau = rng.uniform(0.1, 1.0, nz)
    ye = rng.uniform(0.48, 0.50, nz)
    isi, ife = net.species_index("SI 28"), net.species_index("FE 56")
    ye_fe = net.znetw[ife] / net.anetw[ife]
    f = (ye - ye_fe) / (0.5 - ye_fe)
    X = np.full((nz, net.nsp), 1.0e-99)
    X[:, isi] = f
    X[:, ife] = 1.0 - f
    times = np.concatenate([[0.0], 10.0 ** np.linspace(-6.0, np.log10(t_end), npts - 1)])
    return Trajectories(t9_0=t9_0, rho_0=rho_0, tau=tau, X0=X, ye0=_ye_of(net, X), times=times)


def hburn_zone(net: sn.Network | None = None) -> tuple[ZoneBatch, np.ndarray]:
    """One H-burning zone and its 200 frame time steps (dt log-spaced 1e3 .. 1e13 s)."""
    net = net or network(300)
    X = np.full((1, net.nsp), 1.0e-99)
    X[0, net.species_index("PROT ")] = 0.70
    X[0, net.species_index("HE  4")] = 0.28
    # metals: stable (near-valley) species, abundance falling with A (solar-scaled shape)
    stable = [i for i in range(net.nsp) if net.considerisotope[i] and net.anetw[i] > 4
              and abs((net.anetw[i] - net.znetw[i]) - sn.n_center(int(net.znetw[i]))) <= 1.0]
    w = np.array([10.0 ** (-0.045 * net.anetw[i]) for i in stable])
    X[0, stable] = 0.02 * w / w.sum()
    X /= X.sum()
    dts = 10.0 ** np.linspace(3.0, 13.0, 200)
    zb = ZoneBatch(X=X, t9_0=np.array([0.020]), t9_1=np.array([0.020]), rho_0=np.array([100.0]),
                   rho_1=np.array([100.0]), ye=_ye_of(net, X), dtwant=np.array([dts[0]]))
    return zb, dts


def mixed_networks():
    """The three networks of the uneven-size batch: ~200 species (the Z <= 30 part of the reference's
    isotopedatabase.txt, its first 201 lines), the ~1100-species network of the He-shell batch, and
    ~2500 species (the first 2500 lines of isotopedatabase_all.txt)."""
    return network(201, database="isotopedatabase"), network(1107), network(2500, database="isotopedatabase_all")


def mixed_batch(nz: int, seed: int = 4, dtwant: float = 1.0e10):
    """Uneven-size batch: 40 % H-burning zones on the ~200-species network (T9 U[0.015, 0.08], rho
    log-U[1, 1e3], X(H1) = 0.70, X(He4) = 0.28, Z = 0.02 over the stable species), 50 % He-shell
    zones on the ~1100-species network (as heshell_batch), 10 % zones on the ~2500-species network
    (T9 U[0.3, 1.0], rho log-U[1e4, 1e6], the He-shell composition), each one integrate_network call
    of dtwant. Returns (networks, [(network index, ZoneBatch)]), the zones of each network together,
    and the network index of every zone in batch order."""
    nets = mixed_networks()
    rng = np.random.default_rng(seed)
    counts = [int(round(0.4 * nz)), 0, int(round(0.1 * nz))]
    counts[1] = nz - counts[0] - counts[2]
    hb, _ = hburn_zone(nets[0])
    X0 = np.repeat(hb.X, counts[0], axis=0)
    t9 = rng.uniform(0.015, 0.08, counts[0])
    rho = 10.0 ** rng.uniform(0.0, 3.0, counts[0])
    small = ZoneBatch(X=X0, t9_0=t9.copy(), t9_1=t9.copy(), rho_0=rho.copy(), rho_1=rho.copy(),
                      ye=_ye_of(nets[0], X0), dtwant=np.full(counts[0], dtwant))
    mid = heshell_batch(counts[1], net=nets[1], seed=seed + 1, dtwant=dtwant)
    big = heshell_batch(counts[2], net=nets[2], seed=seed + 2, dtwant=dtwant)
    t9b = rng.uniform(0.3, 1.0, counts[2])
    rhob = 10.0 ** rng.uniform(4.0, 6.0, counts[2])
    big.t9_0[:], big.t9_1[:], big.rho_0[:], big.rho_1[:] = t9b, t9b, rhob, rhob
    net_of = np.concatenate([np.full(c, i, np.int32) for i, c in enumerate(counts)])
    return nets, [(0, small), (1, mid), (2, big)], net_of
