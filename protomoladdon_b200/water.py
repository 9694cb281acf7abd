"""Seeded synthetic periodic water boxes (TIP3P-style rigid geometry).

The benchmark and test workloads are generated here, not read from files:

* oxygens on a k x k x k cubic lattice (spacing 3.104 A), each jittered by
  U(-0.1, 0.1) A per axis; box edge = k * spacing;
* each molecule rotated by a uniformly random orientation (unit quaternion
  from three uniforms, Shoemake's method);
* O-H 0.9572 A, H-O-H 104.52 deg; charges O -0.834 e, H +0.417 e, scaled by
  ProtoMol's SQRTCOULOMBCONSTANT 18.2226123264
  (protomol/src/protomol/base/PMConstants.cpp:64,
  protomol/src/protomol/topology/BuildTopology.cpp:92) so Coulomb needs no
  prefactor;
* Lennard-Jones only on O-O (sigma 3.1507 A, epsilon 0.1521 kcal/mol,
  A = 4 eps sigma^12, B = 4 eps sigma^6), A14/B14 = A/B;
* the three intramolecular pairs of each water are fully excluded;
* optional Na+/Cl- ions replacing a fraction of the waters (one ion per
  replaced water, at its oxygen site; sigma 2.43/4.04 A, epsilon
  0.047/0.15 kcal/mol, Lorentz-Berthelot mixing);
* Maxwell-Boltzmann velocities (kT/m in ProtoMol's AKMA units, the units of
  protomol/src/protomol/topology/TopologyUtilities.cpp:20-48).

Random numbers come from numpy's PCG64 stream seeded with ``seed``.
"""
from __future__ import annotations

import math

import numpy as np

SQRT_COULOMB = 18.2226123264
BOLTZMANN = 0.001987191  # kcal/mol/K
LATTICE = 3.104
R_OH = 0.9572
THETA_HOH = math.radians(104.52)
MASS_O, MASS_H, MASS_NA, MASS_CL = 15.9994, 1.008, 22.98977, 35.453
Q_O, Q_H = -0.834, 0.417
SIG_O, EPS_O = 3.1507, 0.1521
SIG_NA, EPS_NA = 2.43, 0.047
SIG_CL, EPS_CL = 4.04, 0.15

T_O, T_H, T_NA, T_CL = 0, 1, 2, 3


def _lj_table(with_ions: bool) -> np.ndarray:
    sig = [SIG_O, 0.0] + ([SIG_NA, SIG_CL] if with_ions else [])
    eps = [EPS_O, 0.0] + ([EPS_NA, EPS_CL] if with_ions else [])
    nt = len(sig)
    t = np.zeros((nt, nt, 4))
    for a in range(nt):
        for b in range(nt):
            if eps[a] == 0.0 or eps[b] == 0.0:
                continue
            s = 0.5 * (sig[a] + sig[b]) if a != b else sig[a]
            e = math.sqrt(eps[a] * eps[b]) if a != b else eps[a]
            A = 4.0 * e * s ** 12
            B = 4.0 * e * s ** 6
            t[a, b] = (A, B, A, B)
    return t


def _random_rotations(rng, m):
    u1, u2, u3 = rng.random(m), rng.random(m), rng.random(m)
    a = np.sqrt(1.0 - u1)
    b = np.sqrt(u1)
    qw = a * np.sin(2 * np.pi * u2)
    qx = a * np.cos(2 * np.pi * u2)
    qy = b * np.sin(2 * np.pi * u3)
    qz = b * np.cos(2 * np.pi * u3)
    R = np.empty((m, 3, 3))
    R[:, 0, 0] = 1 - 2 * (qy * qy + qz * qz)
    R[:, 0, 1] = 2 * (qx * qy - qz * qw)
    R[:, 0, 2] = 2 * (qx * qz + qy * qw)
    R[:, 1, 0] = 2 * (qx * qy + qz * qw)
    R[:, 1, 1] = 1 - 2 * (qx * qx + qz * qz)
    R[:, 1, 2] = 2 * (qy * qz - qx * qw)
    R[:, 2, 0] = 2 * (qx * qz - qy * qw)
    R[:, 2, 1] = 2 * (qy * qz + qx * qw)
    R[:, 2, 2] = 1 - 2 * (qx * qx + qy * qy)
    return R


def water_box(k: int, *, rc: float, ron: float, seed: int = 1234,
              spacing: float = LATTICE, ion_fraction: float = 0.0,
              nmol: int | None = None, box: float | None = None,
              temperature: float = 300.0, cellsize: float | None = None) -> dict:
    """Builds one periodic water box as a dict of flat arrays.

    ``k`` lattice sites per axis; ``nmol`` (default k**3) molecules occupy the
    first ``nmol`` sites of a seeded permutation.  ``box`` overrides the edge
    (default k * spacing; the lattice spacing is then box / k).
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    nsite = k ** 3
    if nmol is None:
        nmol = nsite
    if box is None:
        box = k * spacing
    else:
        spacing = box / k
    sites = np.stack(np.meshgrid(np.arange(k), np.arange(k), np.arange(k), indexing="ij"),
                     -1).reshape(-1, 3).astype(np.float64)
    if nmol < nsite:
        sites = sites[rng.permutation(nsite)[:nmol]]
    o = (sites + 0.5) * spacing + rng.uniform(-0.1, 0.1, size=(nmol, 3))
    R = _random_rotations(rng, nmol)
    half = 0.5 * THETA_HOH
    h_local = np.array([[R_OH * math.sin(half), 0.0, R_OH * math.cos(half)],
                        [-R_OH * math.sin(half), 0.0, R_OH * math.cos(half)]])
    h = o[:, None, :] + np.einsum("mij,hj->mhi", R, h_local)
    n_ion_pairs = int(round(ion_fraction * nmol / 2.0))
    is_ion = np.zeros(nmol, dtype=np.int8)  # 0 water, 1 Na, 2 Cl
    if n_ion_pairs:
        pick = rng.permutation(nmol)[:2 * n_ion_pairs]
        is_ion[pick[:n_ion_pairs]] = 1
        is_ion[pick[n_ion_pairs:]] = 2
    pos, typ, q, mol, mass, excl = [], [], [], [], [], []
    a = 0
    for m in range(nmol):
        if is_ion[m]:
            pos.append(o[m])
            na = is_ion[m] == 1
            typ.append(T_NA if na else T_CL)
            q.append(1.0 if na else -1.0)
            mass.append(MASS_NA if na else MASS_CL)
            mol.append(m)
            a += 1
            continue
        pos.extend([o[m], h[m, 0], h[m, 1]])
        typ.extend([T_O, T_H, T_H])
        q.extend([Q_O, Q_H, Q_H])
        mass.extend([MASS_O, MASS_H, MASS_H])
        mol.extend([m, m, m])
        excl.extend([(a, a + 1, 2), (a, a + 2, 2), (a + 1, a + 2, 2)])
        a += 3
    n = a
    pos = np.asarray(pos, dtype=np.float64)
    mass = np.asarray(mass, dtype=np.float64)
    vel = rng.standard_normal((n, 3)) * np.sqrt(BOLTZMANN * temperature / mass)[:, None]
    if cellsize is None:
        cellsize = 0.5 * rc
    return dict(
        pos=pos, vel=vel,
        type=np.asarray(typ, dtype=np.int32),
        qscaled=np.asarray(q, dtype=np.float64) * SQRT_COULOMB,
        mol=np.asarray(mol, dtype=np.int32),
        mass=mass,
        lj=_lj_table(ion_fraction > 0.0),
        excl=np.asarray(excl, dtype=np.int32).reshape(-1, 3),
        coulomb_scaling=1.0,
        box=np.array([box, box, box], dtype=np.float64),
        origin=np.array([0.5 * box] * 3, dtype=np.float64),
        cellsize=float(cellsize), ron=float(ron), rc_lj=float(rc), rc_coul=float(rc),
        rc_alg=float(rc), n=n,
    )


D_OH = R_OH
D_HH = 2.0 * R_OH * math.sin(0.5 * THETA_HOH)


def rigid_waters(sysd) -> np.ndarray:
    """(O, H1, H2) atom triples of every 3-atom O-H-H molecule, for the
    rigid-water (SETTLE) integrator; constraint lengths D_OH and D_HH."""
    mol = np.asarray(sysd["mol"])
    typ = np.asarray(sysd["type"])
    order = np.argsort(mol, kind="stable")
    bounds = np.flatnonzero(np.diff(np.r_[-1, mol[order], mol.max() + 1 if mol.size else 0]))
    out = []
    for a, b in zip(bounds[:-1], bounds[1:]):
        atoms = order[a:b]
        if len(atoms) == 3 and typ[atoms[0]] == T_O and (typ[atoms[1:]] == T_H).all():
            out.append(atoms)
    return np.asarray(out, dtype=np.int32).reshape(-1, 3)


def many_types(sysd, n_o_types=14, n_h_types=10, n_unused=6, seed=7):
    """The same atoms spread over many Lennard-Jones types, as a force-field
    topology has them: each oxygen gets one of ``n_o_types`` O-like types
    (sigma 3.0-3.3 A, epsilon 0.12-0.18 kcal/mol), each hydrogen one of
    ``n_h_types`` H-like types with a small LJ term (sigma 0.9-1.5 A,
    epsilon 0.02-0.05), and ``n_unused`` more types appear only in the table
    (like the unused types of a parameter file); Lorentz-Berthelot mixing,
    A14/B14 at half strength.  Charges, geometry and exclusions unchanged."""
    rng = np.random.Generator(np.random.PCG64(seed))
    d = dict(sysd)
    typ = np.asarray(sysd["type"]).copy()
    o = typ == T_O
    h = typ == T_H
    typ[o] = rng.integers(0, n_o_types, size=int(o.sum()))
    typ[h] = n_o_types + rng.integers(0, n_h_types, size=int(h.sum()))
    nt = n_o_types + n_h_types + n_unused
    sig = np.concatenate([rng.uniform(3.0, 3.3, n_o_types), rng.uniform(0.9, 1.5, n_h_types),
                          rng.uniform(1.0, 4.0, n_unused)])
    eps = np.concatenate([rng.uniform(0.12, 0.18, n_o_types),
                          rng.uniform(0.02, 0.05, n_h_types), rng.uniform(0.01, 0.2, n_unused)])
    t = np.zeros((nt, nt, 4))
    for a in range(nt):
        for b in range(nt):
            sg = 0.5 * (sig[a] + sig[b])
            ep = math.sqrt(eps[a] * eps[b])
            A = 4.0 * ep * sg ** 12
            B = 4.0 * ep * sg ** 6
            t[a, b] = (A, B, 0.5 * A, 0.5 * B)
    d["type"] = typ.astype(np.int32)
    d["lj"] = t
    return d


def sheared(sysd, sxy=0.3, sxz=0.0, syz=0.0):
    """The box made a general periodic cell by shear: basis e1 = (L, 0, 0),
    e2 = (sxy L, L, 0), e3 = (sxz L, syz L, L) (rows of the 3x3 "box"); each
    molecule moves rigidly with the shear of its first atom, so the geometry
    and the density stay the water box's.  The origin is the cell's centre."""
    d = dict(sysd)
    L = float(np.asarray(sysd["box"])[0])
    mol = np.asarray(sysd["mol"])
    pos = np.array(sysd["pos"], dtype=np.float64)
    first = np.full(mol.max() + 1, -1)
    for i in range(len(mol) - 1, -1, -1):
        first[mol[i]] = i
    a = pos[first[mol]]
    pos[:, 0] += sxy * a[:, 1] + sxz * a[:, 2]
    pos[:, 1] += syz * a[:, 2]
    e = np.array([[L, 0.0, 0.0], [sxy * L, L, 0.0], [sxz * L, syz * L, L]])
    d["pos"] = pos
    d["box"] = e
    d["origin"] = 0.5 * e.sum(0)
    return d


# Named workloads (sizes from the reference-facing benchmark definitions).
def small_648(seed=1234):
    """216 waters, 6^3 lattice, box 18.624 A, rc 8, C2 from 7."""
    return water_box(6, rc=8.0, ron=7.0, seed=seed)


def medium_41k(seed=1234):
    """13,824 waters (41,472 atoms), 24^3 lattice, box 74.496 A, rc 10, C2 from 9."""
    return water_box(24, rc=10.0, ron=9.0, seed=seed)


def large_331k(seed=1234):
    """110,592 sites (331,776 atoms before ions), 48^3 lattice, box 148.992 A,
    rc 12, 2% of waters replaced by Na+/Cl- pairs."""
    return water_box(48, rc=12.0, ron=11.0, seed=seed, ion_fraction=0.02)


def batch_boxes(count=512, seed=1234, rc=9.0, ron=8.0, density=0.0334,
                nmin=300, nmax=6000):
    """Uneven periodic boxes: atom counts log-uniform in [nmin, nmax] rounded to
    whole waters, at ``density`` molecules/A^3.  Boxes below 2 rc are grown to
    2 rc (density then falls below the target for the smallest systems)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for b in range(count):
        natoms = math.exp(rng.uniform(math.log(nmin), math.log(nmax)))
        nmol = max(1, int(round(natoms / 3.0)))
        edge = max((nmol / density) ** (1.0 / 3.0), 2.0 * rc)
        k = int(math.ceil(nmol ** (1.0 / 3.0)))
        out.append(water_box(k, rc=rc, ron=ron, seed=seed * 7919 + b, nmol=nmol, box=edge))
    return out
