"""Generates the committed golden fixtures from the reference itself.

Run in a tree where the reference sources are available and
``make -C oracle ref`` has built oracle/_ref/libpmref.so:

    python tests/golden/make_golden.py <reference tree>

(or with the tree in the PROTOMOL_REFERENCE environment variable).

Fixtures (all inputs and outputs FP64):

* water423.npz -- the reference's periodic water test system
  (test/tests/data/water_423.{psf,pdb} + par_all27_prot_lipid.inp), read by
  the reference's own PSF/PAR/PDB readers and topology builder, with the t=0
  LENNARDJONES and COULOMB energies of its golden
  test/tests/expected/water_CHARMM_PERIODIC_L.energy (columns 10-11), and the
  reference's combined LJ(C2, switchon 0.1, cutoff 6.5) + Coulomb(C1, 6.5)
  forces, energies, atomic and molecular virial on those positions.
* water648_ref.npz -- the seeded 216-water box (protomoladdon_b200.water.
  small_648, seed 1234): reference forces, energies, virials, plus 20 FP64
  leapfrog steps at 1 fs through the reference force.
* modified_ref.npz -- the same box with every intramolecular O-H pair made
  EXCLUSION_MODIFIED (1-4 style) and coulombScalingFactor 0.5, exercising
  A14/B14 and the Coulomb scaling branch.
* ewald_{water,modified,ions}_ref.npz -- the reference's real-space Ewald
  force (NonbondedFullEwaldSystemForce<PBC, CubicCellManager, real only,
  Cutoff>) on the 648-atom box (alpha 0.30, rc 8), on the modified box
  (default alpha, accuracy 1e-5) and on a box with 10% of the waters
  replaced by Na+/Cl- (alpha 0.30, rc 9): forces, Coulomb energy, atomic and
  molecular virial from the reference as shipped (``poly5_*``, erfc by the
  Abramowitz & Stegun polynomial) and built with -DUSE_EWALD_EXACT_ERF
  (``exact_*``).  ``--ewald-only`` writes just these.
* pairs_ref.npz -- the reference's other periodic cutoff registrations
  (OneAtomPair / OneAtomPairTwo with C1, C2, Cn switches) on the 648-atom
  box: per case ``<case>_{forces,energies,virial,molvirial}`` and the switch
  specs ``<case>_lj`` / ``<case>_coul`` ({kind code, switchon, cutoff,
  order, switchoff}, kind 0 = absent).  ``--pairs-only`` writes just this.
* vacuum_ref.npz -- the reference's vacuum cutoff force (OneAtomPairTwo<
  VacuumBoundaryConditions, C2, LJ, C1, Coulomb>) on a water droplet (the
  whole molecules of the 648-atom box within 8.5 A of its centre, unwrapped
  around it), rc 8 / C2 from 7: forces, energies, virials.
  ``--vacuum-only`` writes just this.
* ljtable_{water,modified,vacuum}_ref.npz -- the reference's tabulated LJ
  registrations (OneAtomPair<BC, UniversalSwitchingFunction,
  LennardJonesTableForce<S, 7, Real>>, S = C2, Cn, ComplimentCnCn) on the
  648-atom box, on the modified box (A14/B14 through the table) and, with
  vacuum boundaries, on the droplet: per case
  ``<case>_{forces,energies,virial,molvirial}`` and ``<case>_lj`` (the
  switch spec as in pairs_ref.npz).  ``--ljtable-only`` writes just these.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as O  # noqa: E402
from protomoladdon_b200 import water  # noqa: E402


def golden_energy_row(path):
    with open(path) as fh:
        cols = fh.readline().split()
    return float(cols[9]), float(cols[10])  # E_VdW (LJ), E_coulomb


def sysd_arrays(s):
    keys = ("pos", "type", "qscaled", "mol", "mass", "lj", "excl", "box", "origin")
    out = {k: np.asarray(s[k]) for k in keys}
    for k in ("coulomb_scaling", "cellsize", "ron", "rc_lj", "rc_coul", "rc_alg"):
        out[k] = np.float64(s[k])
    return out


def main(ref_root):
    data = os.path.join(ref_root, "test", "tests", "data")
    exp = os.path.join(ref_root, "test", "tests", "expected", "water_CHARMM_PERIODIC_L.energy")
    s = O.ref_load_psf(os.path.join(data, "water_423.psf"),
                       os.path.join(data, "par_all27_prot_lipid.inp"),
                       os.path.join(data, "water_423.pos.pdb"), exclude="scaled1-4")
    # conf: cellBasisVector 28 A cube at origin 0, cellsize 6.5, LJ C2
    # (switchon 0.1, cutoff 6.5), Coulomb C1 (cutoff 6.5)
    s.update(box=np.array([28.0, 28.0, 28.0]), origin=np.zeros(3), cellsize=6.5, ron=0.1,
             rc_lj=6.5, rc_coul=6.5, rc_alg=6.5, coulomb_scaling=1.0)
    R = O.RefForce(s)
    f, e, v, mv = R.evaluate(s["pos"], 2)
    elj, ecoul = golden_energy_row(exp)
    np.savez_compressed(os.path.join(HERE, "water423.npz"), **sysd_arrays(s),
                        golden_elj=elj, golden_ecoul=ecoul, ref_forces=f, ref_energies=e,
                        ref_virial=v, ref_molvirial=mv)
    R.close()

    w = water.small_648()
    R = O.RefForce(w)
    f, e, v, mv = R.evaluate(w["pos"], 2)
    p20, v20, e20 = R.leapfrog(w["pos"], w["vel"], 1.0, 20)
    np.savez_compressed(os.path.join(HERE, "water648_ref.npz"), **sysd_arrays(w),
                        vel=w["vel"], ref_forces=f, ref_energies=e, ref_virial=v,
                        ref_molvirial=mv, lf20_pos=p20, lf20_vel=v20, lf20_energies=e20)
    R.close()

    m = dict(w)
    ex = m["excl"].copy()
    oh = m["type"][ex[:, 0]] == water.T_O  # the two O-H pairs of each water; H-H stays full
    ex[oh, 2] = 1
    m["excl"] = ex
    m["coulomb_scaling"] = 0.5
    R = O.RefForce(m)
    f, e, v, mv = R.evaluate(m["pos"], 2)
    np.savez_compressed(os.path.join(HERE, "modified_ref.npz"), **sysd_arrays(m),
                        ref_forces=f, ref_energies=e, ref_virial=v, ref_molvirial=mv)
    R.close()
    many_types_fixture()
    print("wrote fixtures to", HERE)


def triclinic_fixture():
    """A sheared 9^3 water box (2,187 atoms; e2 = (0.3 L, L, 0), e3 =
    (0.1 L, -0.2 L, L)), rc 6, C2 from 5, with the reference's pair function
    over all pairs at its minimal image (NonbondedSimpleFullSystemForce).  Its
    cell-list force is not used: on general cells it misses pairs across the
    sheared faces, and on this box it stops on an array-bounds assertion."""
    t = water.sheared(water.water_box(9, rc=6.0, ron=5.0, seed=17), 0.3, 0.1, -0.2)
    R = O.RefForce(t)
    f, e, v, mv = R.evaluate_allpairs(t["pos"], 2)
    np.savez_compressed(os.path.join(HERE, "triclinic_ref.npz"), **sysd_arrays(t),
                        ref_forces=f, ref_energies=e, ref_virial=v, ref_molvirial=mv)
    R.close()


def many_types_fixture():
    """The 648-atom box over 30 LJ types (24 used) with the H-H pair of each
    water modified (A14/B14, Coulomb scaling 0.5) and O-H fully excluded."""
    t = water.many_types(water.small_648())
    ex = t["excl"].copy()
    ex[t["type"][ex[:, 0]] >= 14, 2] = 1  # H-H modified, O-H full
    t["excl"] = ex
    t["coulomb_scaling"] = 0.5
    R = O.RefForce(t)
    f, e, v, mv = R.evaluate(t["pos"], 2)
    np.savez_compressed(os.path.join(HERE, "manytypes_ref.npz"), **sysd_arrays(t),
                        ref_forces=f, ref_energies=e, ref_virial=v, ref_molvirial=mv)
    R.close()


def ewald_fixtures():
    w = water.small_648()
    m = dict(w)
    ex = m["excl"].copy()
    ex[m["type"][ex[:, 0]] == water.T_O, 2] = 1
    m["excl"] = ex
    m["coulomb_scaling"] = 0.5
    ions = water.water_box(6, rc=9.0, ron=8.0, seed=77, ion_fraction=0.1)
    cases = [("ewald_water_ref.npz", w, 0.30, float(np.exp(-(0.30 * 8.0) ** 2))),
             ("ewald_modified_ref.npz", m, -1.0, 1e-5),
             ("ewald_ions_ref.npz", ions, 0.30, float(np.exp(-(0.30 * 9.0) ** 2)))]
    for name, sysd, alpha, acc in cases:
        out = dict(sysd_arrays(sysd), alpha=np.float64(alpha), accuracy=np.float64(acc))
        for tag, exact in (("poly5", False), ("exact", True)):
            R = O.RefForce(sysd, exact_erfc=exact)
            f, e, v, mv = R.ewald_real(sysd["pos"], alpha, acc, 2)
            R.close()
            out.update({f"{tag}_forces": f, f"{tag}_energy": np.float64(e),
                        f"{tag}_virial": v, f"{tag}_molvirial": mv})
        np.savez_compressed(os.path.join(HERE, name), **out)
    print("wrote Ewald fixtures to", HERE)


PAIR_CASES = {
    # name: (LJ switch, Coulomb switch), each (kind, switchon, cutoff, order, switchoff)
    "c2_c2": (("C2", 6.5, 8.0, 0, 0), ("C2", 0.0, 8.0, 0, 0)),
    "c2_cn": (("C2", 6.5, 8.0, 0, 0), ("Cn", 5.0, 8.0, 4, 0)),
    "cn_cn": (("Cn", 6.0, 8.0, 3, 8.0), ("Cn", 4.0, 8.0, 6, 0)),
    "lj_c1": (("C1", 0.0, 8.0, 0, 0), None),
    "lj_cn": (("Cn", 6.5, 8.0, 2, 0), None),
    "coul_c2": (None, ("C2", 3.0, 8.0, 0, 0)),
    "coul_cn": (None, ("Cn", 5.0, 8.0, 4, 0)),
    # ComplimentCnCn: switchon, cutoff, order, switchoff (the periodic LJ+Coulomb
    # registration; single potentials; order 5 read as 2; switchoff == cutoff).
    # (A window that keeps only the LJ tail beyond the first shell leaves net
    # forces ~1e-3 of the pair forces, where a relative force bound measures
    # FP32 cancellation, not the switch: the LJ case starts at switchon 0.)
    "cm_cm": (("ComplimentCnCn", 3.0, 8.0, 4, 6.0), ("ComplimentCnCn", 2.0, 8.0, 2, 5.0)),
    "lj_cm": (("ComplimentCnCn", 0.0, 8.0, 6, 5.0), None),
    "coul_cm": (None, ("ComplimentCnCn", 1.0, 8.0, 3, 8.0)),
    "cm5_c1": (("ComplimentCnCn", 3.0, 8.0, 5, 6.5), ("C1", 0.0, 8.0, 0, 0)),
}


def pair_fixtures():
    w = water.small_648()
    out = dict(sysd_arrays(w))
    codes = {"C1": 1, "C2": 2, "Cn": 3, "ComplimentCnCn": 4}
    R = O.RefForce(w)
    for name, (lj, co) in PAIR_CASES.items():
        f, e, v, mv = R.pair_eval(w["pos"], lj, co, 8.0, 2)
        out.update({f"{name}_forces": f, f"{name}_energies": e, f"{name}_virial": v,
                    f"{name}_molvirial": mv})
        for tag, sw in (("lj", lj), ("coul", co)):
            out[f"{name}_{tag}"] = (np.zeros(5) if sw is None else
                                    np.array([codes[sw[0]], *sw[1:]], dtype=np.float64))
    R.close()
    np.savez_compressed(os.path.join(HERE, "pairs_ref.npz"), **out)
    print("wrote switch-policy fixtures to", HERE)


def droplet():
    """Whole waters of the 648-atom box within 8.5 A of its centre, as a
    non-periodic cluster (positions unwrapped around the centre)."""
    w = water.small_648()
    box = np.asarray(w["box"], float)
    c = np.zeros(3)
    pos = w["pos"] - c
    pos -= box * np.rint(pos / box)
    mol = w["mol"]
    nmol = mol.max() + 1
    keep_mol = np.zeros(nmol, bool)
    for m in range(nmol):
        at = np.nonzero(mol == m)[0]
        com = pos[at[0]]  # the oxygen
        # whole molecule on the same side as its oxygen
        pos[at] = com + (pos[at] - com) - box * np.rint((pos[at] - com) / box)
        keep_mol[m] = np.linalg.norm(com) <= 8.5
    keep = keep_mol[mol]
    idx = np.nonzero(keep)[0]
    remap = -np.ones(len(mol), int)
    remap[idx] = np.arange(len(idx))
    mol_new = np.unique(mol[idx], return_inverse=True)[1]
    ex = np.asarray(w["excl"]).reshape(-1, 3)
    ex = ex[keep[ex[:, 0]] & keep[ex[:, 1]]].copy()
    ex[:, 0] = remap[ex[:, 0]]
    ex[:, 1] = remap[ex[:, 1]]
    d = dict(w)
    d.update(pos=pos[idx], type=w["type"][idx], qscaled=w["qscaled"][idx], mol=mol_new,
             mass=w["mass"][idx], excl=ex, n=len(idx), ron=7.0, rc_lj=8.0, rc_coul=8.0,
             rc_alg=8.0, cellsize=4.0)
    return d


def vacuum_fixture():
    d = droplet()
    f, e, v, mv = O.ref_vacuum_eval(d, d["pos"], 2)
    np.savez_compressed(os.path.join(HERE, "vacuum_ref.npz"), **sysd_arrays(d),
                        ref_forces=f, ref_energies=e, ref_virial=v, ref_molvirial=mv)
    print("wrote the vacuum fixture to", HERE)


LJTABLE_CASES = {
    # file: {case: (switch kind, switchon, cutoff, order, switchoff)}
    "water": {"t_c2": ("C2", 6.5, 8.0, 0, 0), "t_cn": ("Cn", 6.0, 8.0, 3, 8.0),
              "t_cm": ("ComplimentCnCn", 0.0, 8.0, 6, 5.0)},
    "modified": {"t_c2": ("C2", 7.0, 8.0, 0, 0)},
    "vacuum": {"t_c2": ("C2", 7.0, 8.0, 0, 0), "t_cn": ("Cn", 6.0, 8.0, 4, 0),
               "t_cm": ("ComplimentCnCn", 0.0, 8.0, 4, 6.0)},
}


def ljtable_fixtures():
    codes = {"C2": 2, "Cn": 3, "ComplimentCnCn": 4}
    w = water.small_648()
    m = dict(w)
    ex = np.asarray(m["excl"]).copy()
    ex[m["type"][ex[:, 0]] == water.T_O, 2] = 1  # the O-H pairs modified (A14/B14)
    m["excl"] = ex
    m["coulomb_scaling"] = 0.5
    systems = {"water": w, "modified": m, "vacuum": droplet()}
    for name, cases in LJTABLE_CASES.items():
        d = systems[name]
        out = dict(sysd_arrays(d))
        R = None if name == "vacuum" else O.RefForce(d)
        for case, sw in cases.items():
            if R is None:
                f, e, v, mv = O.ref_vacuum_table_eval(d, d["pos"], sw, 8.0, 2)
            else:
                f, e, v, mv = R.pair_eval(d["pos"], sw, None, 8.0, 2, lj_table=True)
            out.update({f"{case}_forces": f, f"{case}_energies": e, f"{case}_virial": v,
                        f"{case}_molvirial": mv,
                        f"{case}_lj": np.array([codes[sw[0]], *sw[1:]], dtype=np.float64)})
        if R is not None:
            R.close()
        np.savez_compressed(os.path.join(HERE, f"ljtable_{name}_ref.npz"), **out)
    print("wrote the tabulated-LJ fixtures to", HERE)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    only = [a for a in sys.argv[1:] if a.endswith("-only")]
    if not only:
        ref = args[0] if args else os.environ.get("PROTOMOL_REFERENCE")
        if not ref:
            sys.exit("usage: make_golden.py <reference tree> (or set PROTOMOL_REFERENCE)")
        main(ref)
    if not only or "--ewald-only" in only:
        ewald_fixtures()
    if not only or "--pairs-only" in only:
        pair_fixtures()
    if not only or "--vacuum-only" in only:
        vacuum_fixture()
    if "--manytypes-only" in only:
        many_types_fixture()
    if not only or "--triclinic-only" in only:
        triclinic_fixture()
    if not only or "--ljtable-only" in only:
        ljtable_fixtures()
