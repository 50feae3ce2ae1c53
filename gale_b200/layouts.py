"""Initial material-point layouts of the reference, restated (host side; run once per model).

`SpaceFillerParticleLayout` (StgDomain/Swarm/src/SpaceFillerParticleLayout.cxx:204-241) fills
the domain with `averageInitialParticlesPerCell × global cell count` points
(GlobalParticleLayout.cxx:182) whose coordinates come from one Sobol generator per axis
(StgDomain/Utils/src/SobolGenerator.cxx).  Points are created in sequence order and each is
added to the cell that contains it (GlobalParticleLayout.cxx:263-297), so the point order
returned here is the swarm's initial order.

The Sobol generator follows the published construction: direction numbers from a primitive
polynomial and its initial numbers m_1..m_s (the table of Joe and Kuo, ACM TOMS 29(1), 2003,
which the reference carries as SobolGenerator_PolynomialDegree / _PolynomialCoefficient /
_InitialDirectionNumbers), the recurrence
    m_i = 2 a_1 m_{i-1} ⊕ 4 a_2 m_{i-2} ⊕ … ⊕ 2^s m_{i-s} ⊕ m_{i-s},
and the Gray-code update x_{n+1} = x_n ⊕ (m_c << (30 − c − 1)) with c the position of the
rightmost zero bit of n, on a 30-bit word (SobolGenerator.cxx:198-298).  The reference hands
out table rows in creation order (`SobolGenerator_NewFromTable`, :467-492), so a layout's x,
y (and z) generators use rows 0, 1 (and 2) when it is the first layout of the run.
"""
from __future__ import annotations

from typing import List, Sequence

import numpy as np

WORD_BITS = 30

# The first rows of the Joe–Kuo table (degree s, coefficient bits a_1..a_{s-1} packed with
# a_1 as the most significant of the s−1 bits, initial direction numbers m_1..m_s).  These
# are published constants of the Sobol construction; a layout needs one row per axis.
SOBOL_TABLE = [
    (1, 0, (1,)),
    (2, 1, (1, 1)),
    (3, 1, (1, 3, 7)),
    (3, 2, (1, 1, 5)),
    (4, 1, (1, 3, 1, 1)),
    (4, 4, (1, 1, 3, 7)),
]


class SobolGenerator:
    """One axis of the reference's Sobol sequence (`SobolGenerator_GetNextNumber`)."""

    def __init__(self, degree: int, coefficient: int, initial: Sequence[int]):
        self.s = int(degree)
        self.a = int(coefficient)
        self.m: List[int] = [int(v) for v in initial[:degree]]
        self.index = 0   # lastCalculated_I
        self.value = 0   # lastCalculatedNumber (0.5 truncated to an unsigned int)

    @classmethod
    def from_table(cls, row: int) -> "SobolGenerator":
        s, a, m = SOBOL_TABLE[row]
        return cls(s, a, m)

    def direction(self, i: int) -> int:
        """m_i by the recurrence over the polynomial's coefficients (GetDirectionalNumber)."""
        while len(self.m) <= i:
            k = len(self.m)
            s = self.s
            r = 0
            last = 0
            for c in range(s):
                # coefficient c < s−1 is a_{c+1} (bit s−2−c of the packed word); c = s−1 is
                # the leading term, always present
                if c == s - 1 or (self.a >> (s - 2 - c)) & 1:
                    last = self.m[k - 1 - c]
                    r ^= (1 << (c + 1)) * last
            r ^= last
            self.m.append(r & 0xFFFFFFFF)
        return self.m[i]

    def next(self) -> float:
        n = self.index
        c = 0
        while n & 1:
            n >>= 1
            c += 1
        self.index += 1
        v = (self.direction(c) << (WORD_BITS - c - 1)) & 0xFFFFFFFF
        self.value ^= v
        return self.value / float(1 << WORD_BITS)


def space_filler(mesh, average_per_cell: float, first_row: int = 0) -> np.ndarray:
    """Point coordinates [n, dim] of SpaceFillerParticleLayout on a regular mesh description
    (`abi.MeshDesc`), in creation order.  `first_row` is the Sobol table row of the x axis
    (0 for the first layout of a run)."""
    dim = mesh.dim
    ncell = int(np.prod([mesh.elements[d] for d in range(dim)]))
    total = int(ncell * float(average_per_cell))
    gens = [SobolGenerator.from_table(first_row + d) for d in range(dim)]
    lo = [float(mesh.min[d]) for d in range(dim)]
    hi = [float(mesh.max[d]) for d in range(dim)]
    out = np.empty((total, dim))
    for p in range(total):
        for d in range(dim):
            # SobolGenerator_GetNextNumber_WithMinMax: (max − min)·x + min
            out[p, d] = (hi[d] - lo[d]) * gens[d].next() + lo[d]
    return out
