"""Chemical networks that the preprocessor turns into device code.

Each loader returns a :class:`Network`: the SymPy right-hand side ``rhs`` as a
column matrix in the state symbols ``y``, plus the rate-coefficient symbols
``k`` when the rates are computed at run time (PRIMORDIAL) rather than baked
into the expressions as constants (ROBER, OREGO, KROME dumps).

Symbol names follow the reference preprocessor: state symbols are named
``y(:,1) .. y(:,neq)`` and rate symbols ``k(:,1) .. k(:,nrea)``
(``pre_odevec/example_systems.py:10,27,65-66``).  SymPy orders the factors of
a product and the terms of a sum by symbol name, and that order fixes the
floating-point evaluation order of every emitted expression; keeping the same
names makes the emitted arithmetic identical to the reference's generated code.

Networks:

* ROBER - Robertson's three-species problem
  (``pre_odevec/example_systems.py:3-17``).
* OREGO - the Oregonator (``pre_odevec/example_systems.py:20-37``).
* PRIMORDIAL - the 16-species / 38-reaction primordial-gas network
  (``pre_odevec/example_systems.py:40-191``).  It is written here as a
  reaction list (the reaction names are those of the rate-coefficient
  function, ``src/odevec_commons.F90:143-371``); the mass-action right-hand
  side built from the list equals the reference's hand-expanded one term by
  term (checked in the tests against the reference's generated code).
* KROME - a Python dump defining ``y``, ``rhs``, ``neq``, ``nrea``
  (``pre_odevec.py:97-105``).
"""
from __future__ import annotations

import dataclasses
from typing import List, Optional, Sequence, Tuple

import sympy as sp


@dataclasses.dataclass
class Network:
    name: str
    neq: int
    nrea: int
    y: List[sp.Symbol]
    rhs: sp.Matrix
    k: List[sp.Symbol] = dataclasses.field(default_factory=list)
    # rate model used by the device code when ``k`` is non-empty
    rates: Optional[str] = None
    # index of the gas temperature in the state vector (PRIMORDIAL only)
    idx_tgas: Optional[int] = None
    species: Optional[List[str]] = None
    # species masses (g) and their inverses (1/g) for the mass-fraction <->
    # number-density format of the operator-split caller; 0 marks an entry
    # that is not a species abundance (temperature, counters)
    masses: Optional[List[float]] = None
    imasses: Optional[List[float]] = None
    # --heatcool=1: the gas-temperature row (index neq-2, KROME's layout:
    # chemical species, CR, g, Tgas, dummy) is the heating/cooling term of
    # this header (ov_hc_heating, ov_hc_cooling, ov_hc_gamma, OV_HC_BOLTZMANN,
    # OV_HC_NMOLS) instead of the dump's expression
    heatcool_header: Optional[str] = None

    @property
    def heatcool(self) -> bool:
        return self.heatcool_header is not None

    @property
    def nmols(self) -> int:
        """chemical species (KROME's nmols): all but CR, g, Tgas and dummy"""
        return self.neq - 4


def state_symbols(neq: int) -> List[sp.Symbol]:
    return [sp.Symbol("y(:,%d)" % (i + 1)) for i in range(neq)]


def rate_symbols(nrea: int) -> List[sp.Symbol]:
    return [sp.Symbol("k(:,%d)" % (i + 1)) for i in range(nrea)]


def load_rober() -> Network:
    """Robertson: k1=0.04, k2=3e7, k3=1e4 (``pre_odevec/example_systems.py:12-15``)."""
    y = state_symbols(3)
    rhs = sp.Matrix([
        -0.04 * y[0] + 1e4 * y[1] * y[2],
        0.04 * y[0] - 3e7 * y[1] * y[1] - 1e4 * y[1] * y[2],
        3e7 * y[1] * y[1],
    ])
    return Network("ROBER", 3, 0, y, rhs, species=["A", "B", "C"])


def load_orego() -> Network:
    """Oregonator: s=77.27, q=8.375e-6, w=0.161, f=1
    (``pre_odevec/example_systems.py:29-35``)."""
    y = state_symbols(3)
    s, q, w = 77.27, 8.375e-6, 0.161
    rhs = sp.Matrix([
        s * y[0] + s * y[1] - s * q * y[0] ** 2 - s * y[0] * y[1],
        1.0 / s * y[2] - 1.0 / s * y[1] - 1.0 / s * y[0] * y[1],
        w * y[0] - w * y[2],
    ])
    return Network("OREGO", 3, 0, y, rhs, species=["X", "Y", "Z"])


PRIMORDIAL_SPECIES = ["E", "H-", "H", "HE", "H2", "D", "HD", "H+", "HE+",
                      "H2+", "D+", "HE++", "CR", "g", "Tgas", "dummy"]

# KROME's species masses (g) and inverse masses (1/g) for the 12 chemical
# species, as the reference's PRIMORDIAL driver converts with them
# (tests/primordial.f90:145-210); the inverses are KROME's own rounded
# values, not 1/mass.  CR, g, Tgas and dummy carry no mass.
PRIMORDIAL_MASSES = [9.10938188e-28, 1.67444345638e-24, 1.67353251819e-24, 6.69206503638e-24,
                     3.34706503638e-24, 3.34603251819e-24, 5.01956503638e-24, 1.67262158e-24,
                     6.69115409819e-24, 3.34615409819e-24, 3.34512158e-24, 6.69024316e-24,
                     0.0, 0.0, 0.0, 0.0]
PRIMORDIAL_IMASSES = [1.09776932527e+27, 5.9721335838e+23, 5.97538433901e+23, 1.49430705554e+23,
                      2.9876921695e+23, 2.98861411108e+23, 1.99220448934e+23, 5.97863863505e+23,
                      1.4945104915e+23, 2.98850552203e+23, 2.98942796572e+23, 1.49471398286e+23,
                      0.0, 0.0, 0.0, 0.0]

# (reactants, products) for rate coefficient k(:,i), i = 1..38.  A species
# listed twice takes part twice (mass action: the flux is k * prod(y_r)).
PRIMORDIAL_REACTIONS: List[Tuple[Tuple[str, ...], Tuple[str, ...]]] = [
    (("H", "E"), ("H+", "E", "E")),            # 1
    (("H+", "E"), ("H",)),                     # 2   T <= 5500 K
    (("H+", "E"), ("H",)),                     # 3   T >  5500 K
    (("HE", "E"), ("HE+", "E", "E")),          # 4
    (("HE+", "E"), ("HE",)),                   # 5   T <= 9280 K
    (("HE+", "E"), ("HE",)),                   # 6   T >  9280 K
    (("HE+", "E"), ("HE++", "E", "E")),        # 7
    (("HE++", "E"), ("HE+",)),                 # 8
    (("H", "E"), ("H-",)),                     # 9
    (("H-", "H"), ("H2", "E")),                # 10  T <  1160 K
    (("H-", "H"), ("H2", "E")),                # 11  T >  1160 K
    (("H", "H+"), ("H2+",)),                   # 12  T <= 6700 K
    (("H", "H+"), ("H2+",)),                   # 13  T >  6700 K
    (("H2+", "H"), ("H2", "H+")),              # 14
    (("H2", "H+"), ("H2+", "H")),              # 15  T >  3480 K
    (("H2", "E"), ("H", "H", "E")),            # 16
    (("H2", "H"), ("H", "H", "H")),            # 17
    (("H-", "E"), ("H", "E", "E")),            # 18
    (("H-", "H"), ("H", "H", "E")),            # 19  T <= 1160 K
    (("H-", "H"), ("H", "H", "E")),            # 20  T >  1160 K
    (("H-", "H+"), ("H", "H")),                # 21
    (("H-", "H+"), ("H2+", "E")),              # 22
    (("H2+", "E"), ("H", "H")),                # 23  T <= 617 K
    (("H2+", "E"), ("H", "H")),                # 24  T >  617 K
    (("H2+", "H-"), ("H", "H2")),              # 25
    (("H", "H", "H"), ("H2", "H")),            # 26  T <= 300 K
    (("H", "H", "H"), ("H2", "H")),            # 27  T >  300 K
    (("H2", "H", "H"), ("H2", "H2")),          # 28  T <= 300 K
    (("H2", "H", "H"), ("H2", "H2")),          # 29  T >  300 K
    (("H+", "D"), ("H", "D+")),                # 30
    (("H", "D+"), ("H+", "D")),                # 31
    (("H2", "D+"), ("HD", "H+")),              # 32
    (("HD", "H+"), ("H2", "D+")),              # 33
    (("H2", "D"), ("HD", "H")),                # 34  T <= 2000 K
    (("H2", "D"), ("HD", "H")),                # 35  T >  2000 K
    (("HD", "H"), ("H2", "D")),                # 36
    (("D", "H-"), ("HD", "E")),                # 37
    (("D+", "E"), ("D",)),                     # 38
]


def mass_action_rhs(y: Sequence[sp.Symbol], k: Sequence[sp.Symbol],
                    species: Sequence[str],
                    reactions: Sequence[Tuple[Sequence[str], Sequence[str]]]) -> sp.Matrix:
    """Net mass-action production rate of every species."""
    index = {s: i for i, s in enumerate(species)}
    rows = [sp.Integer(0)] * len(species)
    for r, (reac, prod) in enumerate(reactions):
        flux = k[r]
        for s in reac:
            flux = flux * y[index[s]]
        net = {}
        for s in reac:
            net[s] = net.get(s, 0) - 1
        for s in prod:
            net[s] = net.get(s, 0) + 1
        for s, c in net.items():
            if c:
                rows[index[s]] = rows[index[s]] + c * flux
    return sp.Matrix(rows)


def load_primordial() -> Network:
    neq, nrea = 16, 38
    y = state_symbols(neq)
    k = rate_symbols(nrea)
    rhs = mass_action_rhs(y, k, PRIMORDIAL_SPECIES, PRIMORDIAL_REACTIONS)
    return Network("PRIMORDIAL", neq, nrea, y, rhs, k=k, rates="primordial",
                   masses=list(PRIMORDIAL_MASSES), imasses=list(PRIMORDIAL_IMASSES),
                   idx_tgas=14, species=list(PRIMORDIAL_SPECIES))


def load_krome_dump(path: str, name: str = "KROME") -> Network:
    """Reads a network dumped as Python source defining ``y`` (list of state
    symbols), ``rhs`` (SymPy column), ``neq`` and ``nrea``; mirrors the
    reference's loader (``pre_odevec.py:97-105``), which executes the dump."""
    ns: dict = {}
    exec("from sympy import *", ns)
    with open(path) as fh:
        exec(compile(fh.read(), path, "exec"), ns)
    y = list(ns["y"])
    rhs = sp.Matrix(ns["rhs"])
    neq = int(ns["neq"])
    nrea = int(ns.get("nrea", 0))
    if rhs.shape != (neq, 1) or len(y) != neq:
        raise ValueError("KROME dump %s: rhs/y do not have neq=%d rows" % (path, neq))
    free = set().union(*[e.free_symbols for e in rhs]) - set(y)
    if free:
        raise ValueError("KROME dump %s: rhs has symbols other than y: %s"
                         % (path, sorted(map(str, free))))
    return Network(name, neq, nrea, y, rhs)


def enable_heatcool(net: Network, header: str) -> Network:
    """Makes the gas temperature (state entry neq-2) follow the heating and
    cooling functions of `header` (pre_odevec.py:148-190, 556-561).  The rate
    coefficients of a network with a temperature-dependent rate model are
    computed once per solve from the initial temperature, so such a network
    cannot take a temperature equation."""
    if net.neq < 5:
        raise SystemExit("# Error: --heatcool=1 needs the KROME species layout (chemical species, CR, g, "
                         "Tgas, dummy): at least 5 species")
    if net.rates:
        raise SystemExit("# Error: --heatcool=1 needs rate coefficients that do not depend on the "
                         "temperature (a KROME dump); %s computes its rates from Tgas once per solve"
                         % net.name)
    if sp.sympify(net.rhs[net.neq - 2]) != 0:
        raise SystemExit("# Error: --heatcool=1 replaces the Tgas row (species %d), which must be 0 in the "
                         "network" % (net.neq - 1))
    net.heatcool_header = header
    net.idx_tgas = net.neq - 2
    return net


def load(example: str, kromefile: Optional[str] = None) -> Network:
    """Network by name, as ``get_system_to_solve`` selects it (``pre_odevec.py:45-107``)."""
    ex = example.upper()
    if ex == "ROBER":
        return load_rober()
    if ex == "OREGO":
        return load_orego()
    if ex == "PRIMORDIAL":
        return load_primordial()
    if ex == "KROME":
        if not kromefile:
            raise ValueError("--example=KROME needs --krome_setupfile")
        return load_krome_dump(kromefile)
    raise ValueError("unknown example %r" % example)
