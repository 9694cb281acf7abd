"""Numpy restatement of ProtoMol's tabulated Lennard-Jones potential.
TEST INFRASTRUCTURE ONLY: imported by tests/ to check the GPU path, never by
the product.

It follows

* LookupTable<LennardJonesLookupValues, 7, double>
  (protomol/src/protomol/force/table/LookupTable.h:71-158 build, 196-214
  index / interpolate): 128 intervals per octave of r^2 from
  lowerboundExp2(0.1) = 1/16 up to the octave holding cutoff^2, each grid
  point holding (value, d/dr^2, c, d) of the switched r^-12 part (A) and of
  the switched -r^-6 part (B); c and d are the cubic Hermite coefficients of
  the interval that starts at the point, refined twice;
* LennardJonesLookupValues::assign (LennardJonesTableForce.h:24-34) for the
  grid values; and
* LennardJonesTableForce::operator() (LennardJonesTableForce.h:68-89) for the
  per-pair lookup, inside OneAtomPair<BC, UniversalSwitchingFunction, ...>
  (OneAtomPair.h:56-111): pairs beyond the table switch's cutoff are skipped
  (LennardJonesTableForce::CUTOFF = 1), and no further switch is applied.

The switching functions are restated in the reference's own power form
(C2SwitchingFunction.h:42-53, CnSwitchingFunction.cpp:149-172,
CmpCnCnSwitchingFunction.h:44-84).

Parity status: pinned against the reference's own LennardJonesTableForce
registrations compiled from its sources (tests/golden/ljtable_ref.npz, made
by tests/golden/make_golden.py --ljtable-only).
"""
from __future__ import annotations

import struct

import numpy as np

PRE = 7
N = 1 << PRE          # intervals per octave
SHIFT = 52 - PRE      # low mantissa bits below the table's hash
STEP = 8              # doubles per grid point: A (v, g, c, d), B (v, g, c, d)

# the smoothstep polynomials of orders 2, 3, 4, (5: an all-zero row in the
# reference), 6 in powers of (r - cutoff) / (switchon - cutoff), and their
# derivatives
_CN_V = [[10., -15., 6.], [35., -84., 70., -20.], [126., -420., 540., -315., 70.], [],
         [1716., -9009., 20020., -24024., 16380., -6006., 924.]]
_CN_D = [[30., -60., 30.], [140., -420., 420., -140.],
         [630., -2520., 3780., -2520., 630.], [],
         [12012., -72072., 180180., -240240., 180180., -72072., 12012.]]


def _bits(x: float) -> int:
    return struct.unpack("<q", struct.pack("<d", x))[0]


def _from_bits(b: int) -> float:
    return struct.unpack("<d", struct.pack("<q", b))[0]


def lowerbound_exp2(r: float) -> float:
    """MathUtilities.cpp:52-61: the largest power of two <= r."""
    res = 1.0
    while res < r:
        res *= 2.0
    while res > r:
        res /= 2.0
    return res


def switch(kind, p, r2):
    """(value, deriv) of a switching function at r^2 (deriv = dS/dr / r);
    kind "C2", "Cn" or "ComplimentCnCn"; p = (switchon, cutoff, order,
    switchoff)."""
    ron, rc, order, roff = (float(x) for x in p)
    if kind == "C2":
        if r2 > rc * rc:
            return 0.0, 0.0
        if r2 < ron * ron:
            return 1.0, 0.0
        t = rc * rc - ron * ron
        s1, s2, s3 = 1.0 / (t * t * t), rc * rc - 3.0 * ron * ron, 4.0 / (t * t * t)
        c2 = rc * rc - r2
        c4 = c2 * (s2 + 2.0 * r2)
        return s1 * (c2 * c4), s3 * (c2 * c2 - c4)
    if kind == "Cn":
        cut = roff if roff else rc
        n = int(order)
        idx = n - 2
        if n == 5:
            n = 2
        if r2 > cut * cut:
            return 0.0, 0.0
        if r2 < ron * ron:
            return 1.0, 0.0
        irange = [(ron - rc) ** -(n + 1)]
        for _ in range(n):
            irange.append(irange[-1] / (ron - rc))
        sq = np.sqrt(r2)
        sd = sq - cut
        c = [sd ** n]
        for _ in range(n + 1):
            c.append(c[-1] * sd)
        v = d = 0.0
        for i in range(n + 1):
            v += _CN_V[idx][i] * c[i + 1] * irange[i]
            d += _CN_D[idx][i] * c[i] * irange[i]
        return v, d / sq
    if kind == "ComplimentCnCn":
        n = 2 if order == 5.0 else int(order)
        idx = n - 2
        ir = [1.0 / (ron - roff) ** (n + 1)]
        it = [1.0 / (roff - rc) ** (n + 1)]
        for _ in range(n):
            ir.append(ir[-1] / (ron - roff))
            it.append(it[-1] / (roff - rc))
        if r2 > rc * rc:
            return 0.0, 0.0
        if r2 > roff * roff:
            sq = np.sqrt(r2)
            sd = sq - rc
            c = [sd ** n]
            for _ in range(n + 1):
                c.append(c[-1] * sd)
            v = d = 0.0
            for i in range(n + 1):
                v += _CN_V[idx][i] * c[i + 1] * it[i]
                d += _CN_D[idx][i] * c[i] * it[i]
            return v, d / sq
        if r2 >= ron * ron:
            sq = np.sqrt(r2)
            sd = sq - roff
            c = [sd ** n]
            for _ in range(n + 1):
                c.append(c[-1] * sd)
            v = d = 0.0
            for i in range(n + 1):
                v += _CN_V[idx][i] * c[i + 1] * ir[i]
                d -= _CN_D[idx][i] * c[i] * ir[i]
            return 1.0 - v, d / sq
        return 0.0, 0.0
    raise ValueError(kind)


def switch_cutoff(kind, p):
    ron, rc, order, roff = (float(x) for x in p)
    if kind == "Cn" and roff:
        return roff
    return rc


class LJTable:
    """The grid of one LennardJonesTableForce<S, 7, double>(swf)."""

    def __init__(self, kind, p):
        self.kind = kind
        self.p = tuple(float(x) for x in p)
        rc = switch_cutoff(kind, p)
        self.cut2 = rc * rc
        lo = lowerbound_exp2(0.1)
        expn = lambda a: _bits(lowerbound_exp2(a)) >> 52  # noqa: E731
        octaves = expn(self.cut2) + 1 - expn(0.1)
        self.first = _bits(lo) >> SHIFT      # grid-point units (the reference: x STEP)
        self.last = octaves * N
        npt = octaves * N + 1
        t = np.zeros((npt, STEP))
        for i in range(npt):
            base = lo * (1 << (i // N))
            dl = base / N
            r = base + dl * (i % N)
            r1 = np.sqrt(r)
            v, d = switch(kind, self.p, r)
            # powers of 1/r1 by squaring, as MathUtilities.h:79-90 forms them
            ip = 1.0 / r1
            p3 = (ip * ip) * ip
            p6 = p3 * p3
            p4 = (ip * ip) * (ip * ip)
            p7 = p6 * ip
            e = p6 * p6
            f = 12.0 * (p7 * p7)
            t[i, 0] = e * v
            t[i, 1] = -0.5 * (f * v - e * d)
            e = -p6
            f = -6.0 * (p4 * p4)
            t[i, 4] = e * v
            t[i, 5] = -0.5 * (f * v - e * d)
            if i > 0:
                x = lo * (1 << ((i - 1) // N)) / N
                for j in (0, 4):
                    v1, g1 = t[i - 1, j], t[i - 1, j + 1]
                    v2, g2 = t[i, j], t[i, j + 1]
                    c = (3.0 * (v2 - v1) - x * (2.0 * g1 + g2)) / (x * x)
                    dd = (-2.0 * (v2 - v1) + x * (g1 + g2)) / (x * x * x)
                    for _ in range(2):
                        dv = (v1 - v2) + ((dd * x + c) * x + g1) * x
                        dg = (g1 - g2) + (3.0 * dd * x + 2.0 * c) * x
                        c -= (3.0 * dv - x * dg) / (x * x)
                        dd -= (-2.0 * dv + x * dg) / (x * x * x)
                    t[i - 1, j + 2] = c
                    t[i - 1, j + 3] = dd
        self.t = t

    def index(self, r2):
        """(grid point, dt) of r^2 (LookupTable::index)."""
        r2 = np.asarray(r2, dtype=np.float64)
        b = r2.view(np.int64)
        i = (b >> SHIFT) - self.first
        low = r2 - (b & ~np.int64((1 << SHIFT) - 1)).view(np.float64)
        dt = np.where((i < 0) | (i > self.last), 0.0, low)
        return np.clip(i, 0, self.last), dt

    def eval(self, r2, A, B):
        """(energy, force / r) per pair (LennardJonesTableForce::operator()
        with LookupTable::interpolate)."""
        i, dt = self.index(r2)
        t = self.t[i]
        a = t[:, 0] * A + t[:, 4] * B
        b = t[:, 1] * A + t[:, 5] * B
        c = t[:, 2] * A + t[:, 6] * B
        d = t[:, 3] * A + t[:, 7] * B
        e = ((dt * d + c) * dt + b) * dt + a
        f = -2.0 * ((3.0 * dt * d + 2.0 * c) * dt + b)
        return e, f


def all_pairs(sysd, pos, table: LJTable, periodic=True):
    """Forces and LJ energy of OneAtomPair<BC, Universal,
    LennardJonesTableForce<...>> over all pairs (minimum image on the
    orthogonal box when periodic); the cell walk of the reference visits the
    same pairs within the cutoff.  Returns (forces, energy)."""
    pos = np.asarray(pos, dtype=np.float64)
    n = len(pos)
    typ = np.asarray(sysd["type"])
    lj = np.asarray(sysd["lj"], dtype=np.float64).reshape(-1, 4)
    nt = int(round(np.sqrt(lj.shape[0])))
    mol = np.asarray(sysd["mol"])
    box = np.diag(np.asarray(sysd["box"], float)) if np.ndim(sysd["box"]) == 2 else \
        np.asarray(sysd["box"], float)
    kinds = {}
    for a, b, k in np.asarray(sysd["excl"]).reshape(-1, 3):
        if a != b:
            kinds[(min(a, b), max(a, b))] = int(k)
    F = np.zeros_like(pos)
    E = 0.0
    for i in range(n - 1):
        d = pos[i + 1:] - pos[i]
        if periodic:
            d -= box * np.rint(d / box)
        r2 = (d * d).sum(1)
        js = np.arange(i + 1, n)
        m = r2 <= table.cut2
        kind = np.zeros(n - i - 1, np.int64)
        for k, j in enumerate(js):
            if m[k] and mol[j] == mol[i]:
                kind[k] = kinds.get((i, j), 0)
        m &= kind != 2
        p = lj[typ[i] * nt + typ[js[m]]]
        mod = kind[m] == 1
        A = np.where(mod, p[:, 2], p[:, 0])
        B = np.where(mod, p[:, 3], p[:, 1])
        e, f = table.eval(r2[m], A, B)
        E += e.sum()
        fij = d[m] * f[:, None]
        F[i] -= fij.sum(0)
        np.add.at(F, js[m], fij)
    return F, E
