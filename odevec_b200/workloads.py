"""Seeded synthetic inputs for the benchmark configurations.

No public data set is involved: every workload is generated from a seed
with the shapes, sizes and value distributions of the configurations below.

* ROBER      - y1 ~ U(0.9, 1), y2 = 0, y3 = 1 - y1; t 0 -> 1e5; rtol 1e-4,
               atol 1e-10; dt_in = 1e-10 (tests/rober.f90:58); lockstep
               groups of 32 (nvector = 32).
* OREGO      - y0 = (1, 2, 3), each scaled by 10^U(log10 0.9, log10 1.1);
               t_end ~ U(30, 360) per cell; rtol 1e-6, atol 1e-10;
               dt_in = 1e-10 (tests/orego.f90:129); per-cell control.
* PRIMORDIAL - log-uniform n_H 1e-2..1e6 cm^-3, T 10..1e4 K (state
               entry 14), ionisation fraction 1e-6..1e-2, H2 fraction
               1e-8..1e-2, other species 1e-20..1e-6 of n_H; hydrogen,
               helium (He/H = 0.08) and deuterium (D/H = 2.6e-5) nuclei
               and charge conserved by construction; t_end log-uniform
               1e8..1e13 s; rtol 1e-6, atol 1e-20; dt_in as the reference
               driver (tests/primordial.f90:73).
* SYN64      - abundances log-uniform 1e-20..1; t_end 1e10 s; rtol 1e-5,
               atol 1e-25.
* HCTOY      - the heating/cooling test network: n_H 1..1e4, Tgas
               100..1e4 K, t_end 1e8..1e11 s; rtol 1e-6, atol 1e-20.
"""
from __future__ import annotations

import dataclasses
from typing import Optional

import numpy as np


@dataclasses.dataclass
class Workload:
    name: str
    network: str          # variant tag
    y: np.ndarray         # (neq, ncells) float64
    t0: np.ndarray        # (ncells,)
    dt0: np.ndarray       # (ncells,)
    t_stop: np.ndarray    # (ncells,)
    rtol: float
    atol: float
    dt_min: float
    group: int
    seed: int

    @property
    def ncells(self) -> int:
        return self.y.shape[1]


def rober(ncells: int = 4096, seed: int = 1, network: str = "ROBER_DENSE_NONE") -> Workload:
    rng = np.random.default_rng(seed)
    y = np.zeros((3, ncells))
    y[0] = rng.uniform(0.9, 1.0, ncells)
    y[2] = 1.0 - y[0]
    return Workload("ROBER", network, y, np.zeros(ncells), np.full(ncells, 1e-10),
                    np.full(ncells, 1e5), 1e-4, 1e-10, 1e-20, 32, seed)


def orego(ncells: int = 65536, seed: int = 2, network: str = "OREGO_CSC_CMK") -> Workload:
    rng = np.random.default_rng(seed)
    base = np.array([1.0, 2.0, 3.0])[:, None]
    y = base * 10.0 ** rng.uniform(np.log10(0.9), np.log10(1.1), (3, ncells))
    t_stop = rng.uniform(30.0, 360.0, ncells)
    return Workload("OREGO", network, y, np.zeros(ncells), np.full(ncells, 1e-10), t_stop,
                    1e-6, 1e-10, 1e-10, 1, seed)


# species order of the primordial network
E, HM, H, HE, H2, D, HD, HP, HEP, H2P, DP, HEPP, CR, G, TGAS, DUMMY = range(16)


def primordial_state(rng, ncells: int, tgas: Optional[np.ndarray] = None) -> np.ndarray:
    lu = lambda lo, hi, n=ncells: 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), n)
    nH = lu(1e-2, 1e6)
    T = lu(10.0, 1e4) if tgas is None else np.broadcast_to(tgas, (ncells,)).astype(float)
    xe = lu(1e-6, 1e-2)
    xh2 = lu(1e-8, 1e-2)
    y = np.zeros((16, ncells))
    y[HP] = xe * nH
    y[H2] = xh2 * nH
    for s in (HM, HD, HEP, H2P, DP, HEPP):
        y[s] = lu(1e-20, 1e-6) * nH
    y[HE] = 0.08 * nH - y[HEP] - y[HEPP]
    y[D] = 2.6e-5 * nH - y[DP] - y[HD]
    y[H] = nH - y[HP] - y[HM] - 2.0 * y[H2] - 2.0 * y[H2P] - y[HD]
    y[E] = y[HP] + y[HEP] + 2.0 * y[HEPP] + y[H2P] + y[DP] - y[HM]
    y[TGAS] = T
    assert np.all(y[:12] > 0.0)
    return y


def primordial_invariants(y: np.ndarray):
    """(hydrogen nuclei, helium nuclei, deuterium nuclei, net charge) per cell."""
    hn = y[H] + y[HP] + y[HM] + 2 * y[H2] + 2 * y[H2P] + y[HD]
    he = y[HE] + y[HEP] + y[HEPP]
    dn = y[D] + y[DP] + y[HD]
    q = y[HP] + y[HEP] + 2 * y[HEPP] + y[H2P] + y[DP] - y[HM] - y[E]
    return hn, he, dn, q


def primordial(ncells: int = 1048576, seed: int = 3, network: str = "PRIMORDIAL_CSC_FF",
               rtol: float = 1e-6, atol: float = 1e-20) -> Workload:
    rng = np.random.default_rng(seed)
    y = primordial_state(rng, ncells)
    t_stop = 10.0 ** rng.uniform(8.0, 13.0, ncells)
    return Workload("PRIMORDIAL", network, y, np.zeros(ncells),
                    np.full(ncells, 2.2954626201190183e-26), t_stop, rtol, atol, 1e-20, 1, seed)


def syn64(ncells: int = 262144, seed: int = 4, network: str = "SYN64_CSC_CMK") -> Workload:
    rng = np.random.default_rng(seed)
    y = 10.0 ** rng.uniform(-20.0, 0.0, (64, ncells))
    return Workload("SYN64", network, y, np.zeros(ncells), np.full(ncells, 1e-10),
                    np.full(ncells, 1e10), 1e-5, 1e-25, 1e-20, 1, seed)


def hctoy(ncells: int = 65536, seed: int = 6, network: str = "HCTOY_DENSE_NONE") -> Workload:
    """The heating/cooling test network (E, H+, H, H2, HE, CR, g, Tgas,
    dummy): log-uniform n_H 1..1e4 cm^-3, ionisation fraction 1e-4..1e-1, H2
    fraction 1e-6..1e-1, He/H 0.08, Tgas 100..1e4 K, t_end log-uniform
    1e8..1e11 s; rtol 1e-6, atol 1e-20."""
    rng = np.random.default_rng(seed)
    lu = lambda lo, hi: 10.0 ** rng.uniform(np.log10(lo), np.log10(hi), ncells)
    nH = lu(1.0, 1e4)
    y = np.zeros((9, ncells))
    y[1] = lu(1e-4, 1e-1) * nH
    y[0] = y[1]
    y[3] = lu(1e-6, 1e-1) * nH
    y[2] = nH - y[1] - 2.0 * y[3]
    y[4] = 0.08 * nH
    y[7] = lu(100.0, 1e4)
    t_stop = lu(1e8, 1e11)
    return Workload("HCTOY", network, y, np.zeros(ncells), np.full(ncells, 1e-10), t_stop,
                    1e-6, 1e-20, 1e-20, 1, seed)


BUILDERS = {"ROBER": rober, "OREGO": orego, "PRIMORDIAL": primordial, "SYN64": syn64, "HCTOY": hctoy}
