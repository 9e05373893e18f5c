"""Lattice descriptors D3Q19 / D3Q27 on the host.

Direction order, opposites and weights are OpenLB's
(``src/descriptor/definition/common.h:120-168`` and ``:313-366``): the kernels
and the ABI's population layout depend on this exact order.
"""
from __future__ import annotations

from dataclasses import dataclass
from fractions import Fraction

import numpy as np

_C19 = [
    (0, 0, 0),
    (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 1, 0), (-1, 0, -1),
    (-1, 0, 1), (0, -1, -1), (0, -1, 1),
    (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1),
    (1, 0, -1), (0, 1, 1), (0, 1, -1),
]
_W19 = [Fraction(1, 3)] + [Fraction(1, 18)] * 3 + [Fraction(1, 36)] * 6 + \
       [Fraction(1, 18)] * 3 + [Fraction(1, 36)] * 6

_C27 = [
    (0, 0, 0),
    (-1, 0, 0), (0, -1, 0), (0, 0, -1), (-1, -1, 0), (-1, 1, 0), (-1, 0, -1),
    (-1, 0, 1), (0, -1, -1), (0, -1, 1), (-1, -1, -1), (-1, -1, 1), (-1, 1, -1), (-1, 1, 1),
    (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, -1, 0), (1, 0, 1),
    (1, 0, -1), (0, 1, 1), (0, 1, -1), (1, 1, 1), (1, 1, -1), (1, -1, 1), (1, -1, -1),
]
_W27 = [Fraction(8, 27)] + [Fraction(2, 27)] * 3 + [Fraction(1, 54)] * 6 + [Fraction(1, 216)] * 4 + \
       [Fraction(2, 27)] * 3 + [Fraction(1, 54)] * 6 + [Fraction(1, 216)] * 4


@dataclass(frozen=True)
class Descriptor:
    name: str
    q: int
    c: np.ndarray          # (q, 3) int
    opposite: np.ndarray   # (q,) int
    weights: tuple         # Fractions

    def w(self, dtype=np.float64) -> np.ndarray:
        """Weights rounded in `dtype` as Fraction::as<T>() does (T(num)/T(den))."""
        dt = np.dtype(dtype).type
        return np.array([dt(f.numerator) / dt(f.denominator) for f in self.weights], dtype=dtype)

    def equilibrium(self, rho, u, dtype=np.float32) -> np.ndarray:
        """Shifted second-order equilibrium (src/dynamics/lbm.h:50-64), evaluated
        in `dtype` with the reference's operation order; shape (q, n)."""
        dt = np.dtype(dtype).type
        rho = np.asarray(rho, dtype=dtype).reshape(-1)
        u = np.asarray(u, dtype=dtype).reshape(3, -1)
        usqr = u[0] * u[0]
        usqr = usqr + u[1] * u[1]
        usqr = usqr + u[2] * u[2]
        w = self.w(dtype)
        out = np.empty((self.q, rho.size), dtype=dtype)
        three = dt(3)
        for i in range(self.q):
            cu = np.zeros_like(rho)
            first = True
            for d in range(3):
                c = int(self.c[i, d])
                if c == 0:
                    continue
                term = u[d] if c == 1 else -u[d]
                cu = term.copy() if first else cu + term
                first = False
            bracket = dt(1) + three * cu
            bracket = bracket + dt(4.5) * cu * cu
            bracket = bracket - dt(1.5) * usqr
            out[i] = rho * w[i] * bracket - w[i]
        return out


D3Q19 = Descriptor("D3Q19", 19, np.array(_C19, dtype=np.int32),
                   np.array([0] + list(range(10, 19)) + list(range(1, 10)), dtype=np.int32), tuple(_W19))
D3Q27 = Descriptor("D3Q27", 27, np.array(_C27, dtype=np.int32),
                   np.array([0] + list(range(14, 27)) + list(range(1, 14)), dtype=np.int32), tuple(_W27))


def descriptor(name) -> Descriptor:
    if name in (19, "D3Q19", "d3q19"):
        return D3Q19
    if name in (27, "D3Q27", "d3q27"):
        return D3Q27
    raise ValueError(f"unknown lattice {name!r}")
