"""Band occupations: fixed filling and broadened (smeared) filling.

Host-side FP64 arithmetic on a few thousand eigenvalues per SCF iteration.
The broadened step functions and the Fermi-level search follow the
reference's ``qepy_pw/occupations.py`` (``smearing_order`` :42-51,
``wgauss`` :610-647, ``w1gauss`` :714-752, ``smeared_occupations``
:755-908), which in turn restates Quantum ESPRESSO's ``wgauss``,
``w1gauss`` and ``efermig``.  Energies are in Hartree; ``degauss`` is given
in Hartree as well (the caller halves the input's Rydberg value, as
``qepy_pw/pw/scf.py:3686-3694`` does).

Orders (QE's ``ngauss``): 0 Gaussian, n > 0 Methfessel-Paxton of order n,
-1 Marzari-Vanderbilt cold smearing, -99 Fermi-Dirac.
"""

from __future__ import annotations

import math

import numpy as np
from scipy.special import erfc

SMEARING_ORDERS = {
    "gaussian": 0, "gauss": 0,
    "methfessel-paxton": 1, "m-p": 1, "mp": 1,
    "marzari-vanderbilt": -1, "cold": -1, "m-v": -1, "mv": -1,
    "fermi-dirac": -99, "f-d": -99, "fd": -99,
}


def smearing_order(name: str) -> int:
    key = str(name).strip().lower().replace("_", "-")
    if key not in SMEARING_ORDERS:
        raise ValueError(f"unknown smearing {name!r}")
    return SMEARING_ORDERS[key]


def _hermite_terms(x: np.ndarray, order: int):
    """Yield (n, H_{2n-1}(x) e^{-x^2}, H_{2n}(x) e^{-x^2}, H_{2n-2} e^{-x^2},
    A_n) for n = 1..order, A_n = (-1)^n / (n! 4^n sqrt(pi))."""
    gauss = np.exp(-np.minimum(200.0, x * x))
    h_even = gauss            # H_0 e^{-x^2}
    h_odd = np.zeros_like(x)  # H_{-1} placeholder
    degree = 0
    coefficient = 1.0 / math.sqrt(math.pi)
    for n in range(1, order + 1):
        # H_{k+1} = 2x H_k - 2k H_{k-1}
        h_odd = 2.0 * x * h_even - 2.0 * degree * h_odd
        degree += 1
        previous_even = h_even
        h_even = 2.0 * x * h_odd - 2.0 * degree * h_even
        degree += 1
        coefficient = -coefficient / (4.0 * n)
        yield degree, h_odd, h_even, previous_even, coefficient


def wgauss(x, order: int) -> np.ndarray:
    """Broadened step function theta(x) for the given order."""
    x = np.asarray(x, dtype=float)
    if order == -99:
        out = np.where(x > 0.0, 1.0, 0.0)
        mid = np.abs(x) <= 200.0
        out[mid] = 1.0 / (1.0 + np.exp(-x[mid]))
        return out
    if order == -1:
        s = x - 1.0 / math.sqrt(2.0)
        return 0.5 * _erf(s) + np.exp(-np.minimum(200.0, s * s)) / math.sqrt(2.0 * math.pi) + 0.5
    if order < 0:
        raise ValueError(f"invalid smearing order {order}")
    out = 0.5 * erfc(-x)
    for _deg, h_odd, _h_even, _prev, a_n in _hermite_terms(x, order):
        out = out - a_n * h_odd
    return out


def w1gauss(x, order: int) -> np.ndarray:
    """Per-state contribution to the smearing (-TS) energy, in units of
    the broadening."""
    x = np.asarray(x, dtype=float)
    if order == -99:
        out = np.zeros_like(x)
        mid = np.abs(x) <= 36.0
        f = 1.0 / (1.0 + np.exp(-x[mid]))
        out[mid] = f * np.log(f) + (1.0 - f) * np.log(1.0 - f)
        return out
    if order == -1:
        s = x - 1.0 / math.sqrt(2.0)
        return s * np.exp(-np.minimum(200.0, s * s)) / math.sqrt(2.0 * math.pi)
    if order < 0:
        raise ValueError(f"invalid smearing order {order}")
    out = -0.5 * np.exp(-np.minimum(200.0, x * x)) / math.sqrt(math.pi)
    for degree, _h_odd, h_even, previous_even, a_n in _hermite_terms(x, order):
        out = out - a_n * (0.5 * h_even + degree * previous_even)
    return out


def _erf(x: np.ndarray) -> np.ndarray:
    return 1.0 - erfc(x)


def _delta(x: np.ndarray, order: int) -> np.ndarray:
    """d wgauss / dx for the orders the Newton refinement needs."""
    if order == -99:
        out = np.zeros_like(x)
        mid = np.abs(x) <= 36.0
        out[mid] = 1.0 / (2.0 + np.exp(-x[mid]) + np.exp(x[mid]))
        return out
    if order == -1:
        s = x - 1.0 / math.sqrt(2.0)
        return np.exp(-np.minimum(200.0, s * s)) / math.sqrt(math.pi) * (1.0 - math.sqrt(2.0) * s)
    g = np.exp(-np.minimum(200.0, x * x)) / math.sqrt(math.pi)
    if order == 0:
        return g
    if order == 1:
        return g * (1.5 - x * x)
    raise ValueError("Newton refinement supports orders 0, 1, -1, -99")


def _delta_prime(x: np.ndarray, order: int) -> np.ndarray:
    if order == -99:
        out = np.zeros_like(x)
        mid = np.abs(x) <= 36.0
        e = np.exp(x[mid])
        out[mid] = -(e - 1.0 / e) / (2.0 + e + 1.0 / e) ** 2
        return out
    if order == -1:
        s = x - 1.0 / math.sqrt(2.0)
        g = np.exp(-np.minimum(200.0, s * s)) / math.sqrt(math.pi)
        return g * (2.0 * math.sqrt(2.0) * x * x - 6.0 * x + math.sqrt(2.0))
    g = np.exp(-np.minimum(200.0, x * x)) / math.sqrt(math.pi)
    if order == 0:
        return -2.0 * x * g
    if order == 1:
        return x * (2.0 * x * x - 5.0) * g
    raise ValueError("Newton refinement supports orders 0, 1, -1, -99")


def fixed_occupations(nbnd: int, occupied: int, nk: int) -> list[np.ndarray]:
    """Two electrons in each of the lowest ``occupied`` bands at every k."""
    out = []
    for _ in range(nk):
        f = np.zeros(nbnd)
        f[:occupied] = 2.0
        out.append(f)
    return out


def smeared_occupations(eigenvalues, weights, nelec: float, degauss: float, order: int,
                        spin_degeneracy: float = 2.0):
    """Fermi level, occupations (0..2 per band) and the smearing energy
    (-TS, Hartree) for broadened filling of ``nelec`` electrons."""
    if degauss <= 0.0:
        raise ValueError("degauss must be positive")
    w = np.asarray(weights, dtype=float)
    w = w * (2.0 / spin_degeneracy) / w.sum()
    eps = np.concatenate([np.asarray(e, dtype=float) for e in eigenvalues])
    wt = np.concatenate([np.full(len(e), wk) for wk, e in zip(w, eigenvalues)])
    capacity = spin_degeneracy * float(np.sum(wt))
    if not 0.0 < nelec < capacity - 1.0e-12:
        raise ValueError(f"{capacity:.6g} smeared states cannot hold {nelec:.6g} electrons; "
                         "add empty bands")

    def count(ef: float, n: int = order) -> float:
        return spin_degeneracy * float(np.dot(wt, wgauss((ef - eps) / degauss, n)))

    lo = min(float(e[0]) for e in eigenvalues) - 10.0 * degauss
    hi = max(float(e[-1]) for e in eigenvalues) + 10.0 * degauss
    while count(lo) > nelec:
        lo -= 10.0 * degauss
    while count(hi) < nelec:
        hi += 10.0 * degauss

    def bisect(n: int) -> float:
        a, b = lo, hi
        if count(a, n) - nelec > 1.0e-12 or count(b, n) - nelec < -1.0e-12:
            raise ValueError("cannot bracket the Fermi energy")
        for _ in range(300):
            mid = 0.5 * (a + b)
            r = count(mid, n) - nelec
            if abs(r) < 1.0e-12:
                return mid
            if r < 0.0:
                a = mid
            else:
                b = mid
        raise ValueError("Fermi-energy bisection did not converge")

    ef = bisect(-99 if order == -99 else 0)
    if order not in (0, -99):
        # Newton minimisation of (N(ef) - nelec)^2 from the Gaussian estimate
        for _ in range(300):
            x = (ef - eps) / degauss
            r = count(ef) - nelec
            d1 = spin_degeneracy * float(np.dot(wt, _delta(x, order))) / degauss
            d2 = spin_degeneracy * float(np.dot(wt, _delta_prime(x, order))) / degauss ** 2
            den = abs(2.0 * (d1 * d1 + r * d2))
            if den <= 1.0e-10:
                break
            nxt = ef - 2.0 * r * d1 / den
            if abs(nxt - ef) < 1.0e-10 or abs(count(nxt) - nelec) < 1.0e-10:
                ef = nxt
                break
            ef = nxt
        if abs(count(ef) - nelec) >= 1.0e-2:
            ef = bisect(order)
    x = (ef - eps) / degauss
    flat = spin_degeneracy * wgauss(x, order)
    bounds = np.cumsum([len(e) for e in eigenvalues[:-1]])
    occupations = [part.copy() for part in np.split(flat, bounds)]
    demet = spin_degeneracy * degauss * float(np.dot(wt, w1gauss(x, order)))
    return float(ef), occupations, demet
