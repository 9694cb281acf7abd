"""ctypes front end for the CPU checkers.  TEST INFRASTRUCTURE ONLY.

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline leg of bench.py
import this module.  It wraps

* ``oracle/_build/libpmoracle.so`` -- pm_oracle.c, the C restatement of
  ProtoMol's NonbondedCutoffSystemForce<CubicCellManager, OneAtomPairTwo<
  PeriodicBoundaryConditions, C2, LennardJones, C1, Coulomb>>; and
* ``oracle/_ref/libpmref.so`` -- the reference's own sources compiled by
  oracle/Makefile, driven through ref_driver.cpp and ref_ewald.cpp (present
  only where the reference tree was available at build time; the file
  travels with the repo copy); ``libpmref_exacterf.so`` is the same with the
  Ewald force built with -DUSE_EWALD_EXACT_ERF.

The real-space Ewald term (NonbondedFullEwaldSystemForce<PBC, CubicCellManager,
real only, CutoffSwitchingFunction>) is restated in pm_oracle.c as well and
pinned against both reference builds.

Parity status: the restatement is pinned bit for bit against the compiled
reference on seeded water boxes and against the reference's periodic water
golden (tests/golden/water423.npz, t = 0 energies of
test/tests/expected/water_CHARMM_PERIODIC_L.energy).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATE_SO = os.path.join(HERE, "_build", "libpmoracle.so")
REF_SO = os.path.join(HERE, "_ref", "libpmref.so")
REF_EXACT_SO = os.path.join(HERE, "_ref", "libpmref_exacterf.so")

_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int


class _PmoSystem(ctypes.Structure):
    _fields_ = [
        ("n", _I), ("ntypes", _I),
        ("type", _P), ("qscaled", _P), ("mol", _P), ("mass", _P), ("lj", _P),
        ("nexcl", _I), ("excl", _P),
        ("coulomb_scaling", _D),
        ("box", _D * 3), ("origin", _D * 3),
        ("cellsize", _D), ("ron", _D), ("rc_lj", _D), ("rc_coul", _D),
        ("rc_alg", _D),
    ]


def _ptr(a):
    return a.ctypes.data_as(_P) if a is not None else None


_restate = None
_ref = None


def restate_lib():
    global _restate
    if _restate is None:
        if not os.path.exists(RESTATE_SO):
            raise RuntimeError(f"oracle restatement not built: {RESTATE_SO} (run make -C oracle restate)")
        lib = ctypes.CDLL(RESTATE_SO)
        lib.pmo_eval.argtypes = [ctypes.POINTER(_PmoSystem), _P, _P, _P, _P, _P, _I, _I]
        lib.pmo_eval.restype = _I
        lib.pmo_count_pairs.argtypes = [ctypes.POINTER(_PmoSystem), _P]
        lib.pmo_count_pairs.restype = ctypes.c_longlong
        lib.pmo_leapfrog.argtypes = [ctypes.POINTER(_PmoSystem), _P, _P, _P, _D, _I, _P]
        lib.pmo_leapfrog.restype = _I
        lib.pmo_settle.argtypes = [_I, _P, _P, _D, _D, _P, _P]
        lib.pmo_settle.restype = None
        lib.pmo_leapfrog_rigid.argtypes = [ctypes.POINTER(_PmoSystem), _P, _P, _P, _D, _I, _I,
                                           _P, _D, _D, _P]
        lib.pmo_leapfrog_rigid.restype = _I
        lib.pmo_eval_ewald_real.argtypes = [ctypes.POINTER(_PmoSystem), _D, _D, _I, _P, _P, _P,
                                            _P, _P, _I, _I]
        lib.pmo_eval_ewald_real.restype = _I
        lib.pmo_ewald_constants.argtypes = [ctypes.POINTER(_PmoSystem), _D, _D, _P]
        lib.pmo_ewald_constants.restype = _I
        lib.pmo_count_pairs_ewald.argtypes = [ctypes.POINTER(_PmoSystem), _D, _D, _P]
        lib.pmo_count_pairs_ewald.restype = ctypes.c_longlong
        _restate = lib
    return _restate


_ref_exact = None


def ref_available(exact_erfc: bool = False) -> bool:
    return os.path.exists(REF_EXACT_SO if exact_erfc else REF_SO)


def ref_lib(exact_erfc: bool = False):
    """The compiled reference; exact_erfc selects the build whose Ewald force
    uses libm erfc."""
    global _ref, _ref_exact
    lib = _ref_exact if exact_erfc else _ref
    if lib is None:
        path = REF_EXACT_SO if exact_erfc else REF_SO
        if not os.path.exists(path):
            raise RuntimeError(f"reference oracle not built: {path} (run make -C oracle ref)")
        lib = ctypes.CDLL(path)
        lib.pmref_create.restype = _P
        lib.pmref_create.argtypes = [_I, _P, _P, _P, _P, _I, _P, _I, _P, _D, _P, _P,
                                     _D, _D, _D, _D, _D]
        lib.pmref_destroy.argtypes = [_P]
        lib.pmref_eval.argtypes = [_P, _P, _P, _P, _P, _P, _I]
        lib.pmref_eval.restype = _I
        lib.pmref_leapfrog.argtypes = [_P, _P, _P, _P, _D, _I, _P]
        lib.pmref_leapfrog.restype = _I
        lib.pmref_load_psf.restype = _I
        lib.pmref_ewald_eval.argtypes = [_P, _D, _D, _P, _P, _P, _P, _P, _I]
        lib.pmref_ewald_eval.restype = _I
        lib.pmref_ewald_exact_erfc.restype = _I
        lib.pmref_hessian.argtypes = [_P, _P, _P, _D, _D, _D, _D]
        lib.pmref_hessian.restype = _I
        lib.pmref_pair_eval.argtypes = [_P, _I, _P, _I, _P, _D, _P, _P, _P, _P, _P, _I]
        lib.pmref_pair_eval.restype = _I
        lib.pmref_set_box.argtypes = [_P, _P, _P, _P, _P]
        lib.pmref_set_box.restype = _I
        lib.pmref_eval_allpairs.argtypes = [_P, _P, _P, _P, _P, _P, _I]
        lib.pmref_eval_allpairs.restype = _I
        if exact_erfc:
            _ref_exact = lib
        else:
            _ref = lib
    return lib


class _Arrays:
    """Keeps contiguous copies of a system's arrays alive for a C call."""

    def __init__(self, sysd):
        self.type = np.ascontiguousarray(sysd["type"], dtype=np.int32)
        self.q = np.ascontiguousarray(sysd["qscaled"], dtype=np.float64)
        self.mol = np.ascontiguousarray(sysd["mol"], dtype=np.int32)
        self.mass = np.ascontiguousarray(sysd["mass"], dtype=np.float64)
        self.lj = np.ascontiguousarray(sysd["lj"], dtype=np.float64).reshape(-1)
        ex = np.asarray(sysd["excl"], dtype=np.int32).reshape(-1, 3)
        self.nexcl = ex.shape[0]
        self.excl = np.ascontiguousarray(ex.reshape(-1)) if self.nexcl else np.zeros(3, np.int32)
        self.ntypes = int(round(np.sqrt(self.lj.size // 4)))
        self.n = self.type.size


def _pmo_struct(sysd, ar: _Arrays):
    s = _PmoSystem()
    s.n = ar.n
    s.ntypes = ar.ntypes
    s.type, s.qscaled, s.mol, s.mass, s.lj = (_ptr(ar.type), _ptr(ar.q), _ptr(ar.mol),
                                              _ptr(ar.mass), _ptr(ar.lj))
    s.nexcl = ar.nexcl
    s.excl = _ptr(ar.excl)
    s.coulomb_scaling = float(sysd.get("coulomb_scaling", 1.0))
    for k in range(3):
        s.box[k] = float(sysd["box"][k])
        s.origin[k] = float(sysd.get("origin", (0.0, 0.0, 0.0))[k])
    s.cellsize = float(sysd["cellsize"])
    s.ron, s.rc_lj, s.rc_coul, s.rc_alg = (float(sysd["ron"]), float(sysd["rc_lj"]),
                                           float(sysd["rc_coul"]), float(sysd["rc_alg"]))
    return s


def restate_eval(sysd, pos, virial_mode=2, brute=False):
    """Returns (forces[n,3], energies[2] = (coulomb, lj), virial[9], molvirial[9])."""
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    f = np.zeros(p.size)
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    rc = lib.pmo_eval(ctypes.byref(st), _ptr(p), _ptr(f), _ptr(e), _ptr(v), _ptr(mv),
                      int(virial_mode), int(bool(brute)))
    if rc:
        raise RuntimeError(f"pmo_eval failed: {rc}")
    return f.reshape(-1, 3), e, v, mv


def restate_ewald_real(sysd, pos, alpha, accuracy, exact_erfc=False, virial_mode=2,
                       brute=False):
    """The real-space Ewald term; returns (forces[n,3], coulomb energy,
    virial[9], molvirial[9])."""
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    f = np.zeros(p.size)
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    rc = lib.pmo_eval_ewald_real(ctypes.byref(st), float(alpha), float(accuracy),
                                 int(bool(exact_erfc)), _ptr(p), _ptr(f), _ptr(e), _ptr(v),
                                 _ptr(mv), int(virial_mode), int(bool(brute)))
    if rc:
        raise RuntimeError(f"pmo_eval_ewald_real failed: {rc}")
    return f.reshape(-1, 3), float(e[0]), v, mv


def ewald_constants(sysd, alpha, accuracy):
    """(alpha, rc, 2 alpha / sqrt(pi), alpha^2) as the reference derives them."""
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    out = np.zeros(4)
    if lib.pmo_ewald_constants(ctypes.byref(st), float(alpha), float(accuracy), _ptr(out)):
        raise RuntimeError("bad Ewald parameters")
    return tuple(float(x) for x in out)


def restate_count_pairs_ewald(sysd, pos, alpha, accuracy) -> int:
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    return int(lib.pmo_count_pairs_ewald(ctypes.byref(st), float(alpha), float(accuracy),
                                         _ptr(p)))


def restate_count_pairs(sysd, pos) -> int:
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    return int(lib.pmo_count_pairs(ctypes.byref(st), _ptr(p)))


def restate_leapfrog(sysd, pos, vel, dt_fs, nsteps):
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1).copy()
    v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1).copy()
    e = np.zeros(2)
    rc = lib.pmo_leapfrog(ctypes.byref(st), _ptr(p), _ptr(v), _ptr(ar.mass), float(dt_fs),
                          int(nsteps), _ptr(e))
    if rc:
        raise RuntimeError(f"pmo_leapfrog failed: {rc}")
    return p.reshape(-1, 3), v.reshape(-1, 3), e


def restate_settle(widx, mass, doh, dhh, old_pos, new_pos):
    """SETTLE of the listed waters; returns the constrained positions."""
    lib = restate_lib()
    w = np.ascontiguousarray(widx, dtype=np.int32).reshape(-1)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    o = np.ascontiguousarray(old_pos, dtype=np.float64).reshape(-1)
    out = np.ascontiguousarray(new_pos, dtype=np.float64).reshape(-1).copy()
    lib.pmo_settle(w.size // 3, _ptr(w), _ptr(m), float(doh), float(dhh), _ptr(o), _ptr(out))
    return out.reshape(-1, 3)


def restate_leapfrog_rigid(sysd, pos, vel, dt_fs, nsteps, widx, doh, dhh):
    lib = restate_lib()
    ar = _Arrays(sysd)
    st = _pmo_struct(sysd, ar)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1).copy()
    v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1).copy()
    w = np.ascontiguousarray(widx, dtype=np.int32).reshape(-1)
    e = np.zeros(2)
    rc = lib.pmo_leapfrog_rigid(ctypes.byref(st), _ptr(p), _ptr(v), _ptr(ar.mass), float(dt_fs),
                                int(nsteps), w.size // 3, _ptr(w), float(doh), float(dhh),
                                _ptr(e))
    if rc:
        raise RuntimeError(f"pmo_leapfrog_rigid failed: {rc}")
    return p.reshape(-1, 3), v.reshape(-1, 3), e


class RefForce:
    """The reference's own NonbondedCutoffSystemForce (compiled from its
    sources) on one system; evaluate() calls SystemForce::evaluate."""

    def __init__(self, sysd, exact_erfc=False):
        self.lib = ref_lib(exact_erfc)
        self._sys = {k: sysd[k] for k in ("ron", "rc_lj", "rc_coul", "rc_alg")}
        self.ar = _Arrays(sysd)
        ar = self.ar
        basis = np.asarray(sysd["box"], dtype=np.float64)
        # a 3x3 box holds the basis vectors as rows (a general periodic cell)
        box = np.ascontiguousarray(np.diag(basis) if basis.shape == (3, 3) else basis)
        org = np.ascontiguousarray(sysd.get("origin", (0.0, 0.0, 0.0)), dtype=np.float64)
        self._keep = (box, org)
        self.n = ar.n
        self.h = self.lib.pmref_create(
            ar.n, _ptr(ar.type), _ptr(ar.q), _ptr(ar.mol), _ptr(ar.mass), ar.ntypes,
            _ptr(ar.lj), ar.nexcl, _ptr(ar.excl), float(sysd.get("coulomb_scaling", 1.0)),
            _ptr(box), _ptr(org), float(sysd["cellsize"]), float(sysd["ron"]),
            float(sysd["rc_lj"]), float(sysd["rc_coul"]), float(sysd["rc_alg"]))
        if basis.shape == (3, 3):
            self.set_box(basis[0], basis[1], basis[2], org)

    def evaluate(self, pos, virial_mode=2):
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        f = np.zeros(p.size)
        e = np.zeros(2)
        v = np.zeros(9)
        mv = np.zeros(9)
        self.lib.pmref_eval(self.h, _ptr(p), _ptr(f), _ptr(e), _ptr(v), _ptr(mv), int(virial_mode))
        return f.reshape(-1, 3), e, v, mv

    def set_box(self, e1, e2, e3, origin):
        """PeriodicBoundaryConditions::set with a general basis (the
        reference's non-orthogonal minimal image)."""
        vec = [np.ascontiguousarray(x, dtype=np.float64) for x in (e1, e2, e3, origin)]
        self._keep_box = vec
        self.lib.pmref_set_box(self.h, *[_ptr(x) for x in vec])

    def evaluate_allpairs(self, pos, virial_mode=2):
        """The same pair function over every pair i < j at the minimal image
        (NonbondedSimpleFullSystemForce): no cell list."""
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        f = np.zeros(p.size)
        e = np.zeros(2)
        v = np.zeros(9)
        mv = np.zeros(9)
        self.lib.pmref_eval_allpairs(self.h, _ptr(p), _ptr(f), _ptr(e), _ptr(v), _ptr(mv),
                                     int(virial_mode))
        return f.reshape(-1, 3), e, v, mv

    def ewald_real(self, pos, alpha, accuracy, virial_mode=2):
        """The reference's real-space Ewald force on this topology: (forces,
        coulomb energy, virial, molvirial)."""
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        f = np.zeros(p.size)
        e = np.zeros(2)
        v = np.zeros(9)
        mv = np.zeros(9)
        self.lib.pmref_ewald_eval(self.h, float(alpha), float(accuracy), _ptr(p), _ptr(f),
                                  _ptr(e), _ptr(v), _ptr(mv), int(virial_mode))
        return f.reshape(-1, 3), float(e[0]), v, mv

    SWITCH_KINDS = {None: 0, "C1": 1, "C2": 2, "Cn": 3, "ComplimentCnCn": 4}

    def pair_eval(self, pos, lj, coulomb, rc_alg, virial_mode=2, lj_table=False):
        """The reference's NonbondedCutoffSystemForce with OneAtomPair /
        OneAtomPairTwo and the given switches: lj / coulomb are None or
        (kind, switchon, cutoff, order, switchoff) with kind C1, C2, Cn or
        ComplimentCnCn.  lj_table: OneAtomPair<PBC, Universal,
        LennardJonesTableForce<S, 7, Real>> with S = lj's switch (C2, Cn or
        ComplimentCnCn; no Coulomb term).
        Returns (forces, energies (coulomb, lj), virial, molvirial)."""
        def spec(x):
            if x is None:
                return 0, np.zeros(4)
            return self.SWITCH_KINDS[x[0]], np.asarray(x[1:5], dtype=np.float64)
        kl, pl = spec(lj)
        kc, pc = spec(coulomb)
        if lj_table:
            kl |= 16
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        f = np.zeros(p.size)
        e = np.zeros(2)
        v = np.zeros(9)
        mv = np.zeros(9)
        rc = self.lib.pmref_pair_eval(self.h, kl, _ptr(pl), kc, _ptr(pc), float(rc_alg), _ptr(p),
                                      _ptr(f), _ptr(e), _ptr(v), _ptr(mv), int(virial_mode))
        if rc:
            raise RuntimeError("pmref_pair_eval failed")
        return f.reshape(-1, 3), e, v, mv

    def hessian(self, pos):
        """The reference's analytic Hessian of the LJ(C2) + Coulomb(C1) energy
        (Hessian::evaluate, not mass-weighted) as a dense (3n, 3n) array."""
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
        n3 = p.size
        h = np.zeros(n3 * n3)
        s = self._sys
        self.lib.pmref_hessian(self.h, _ptr(p), _ptr(h), float(s["ron"]), float(s["rc_lj"]),
                               float(s["rc_coul"]), float(s["rc_alg"]))
        return h.reshape(n3, n3).T  # column-major -> [row, col]

    def leapfrog(self, pos, vel, dt_fs, nsteps):
        p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1).copy()
        v = np.ascontiguousarray(vel, dtype=np.float64).reshape(-1).copy()
        e = np.zeros(2)
        self.lib.pmref_leapfrog(self.h, _ptr(p), _ptr(v), _ptr(self.ar.mass), float(dt_fs),
                                int(nsteps), _ptr(e))
        return p.reshape(-1, 3), v.reshape(-1, 3), e

    def close(self):
        if self.h:
            self.lib.pmref_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ref_vacuum_eval(sysd, pos, virial_mode=2):
    """The reference's vacuum cutoff force (OneAtomPairTwo<VacuumBoundary
    Conditions, C2, LJ, C1, Coulomb>) on the system's arrays and cutoffs:
    (forces, energies (coulomb, lj), virial, molvirial)."""
    lib = ref_lib()
    lib.pmref_vacuum_eval.argtypes = [_I, _P, _P, _P, _P, _I, _P, _I, _P, _D, _D, _D, _D, _D,
                                      _D, _P, _P, _P, _P, _P, _I]
    lib.pmref_vacuum_eval.restype = _I
    ar = _Arrays(sysd)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    f = np.zeros(p.size)
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    lib.pmref_vacuum_eval(ar.n, _ptr(ar.type), _ptr(ar.q), _ptr(ar.mol), _ptr(ar.mass), ar.ntypes,
                          _ptr(ar.lj), ar.nexcl, _ptr(ar.excl),
                          float(sysd.get("coulomb_scaling", 1.0)), float(sysd["cellsize"]),
                          float(sysd["ron"]), float(sysd["rc_lj"]), float(sysd["rc_coul"]),
                          float(sysd["rc_alg"]), _ptr(p), _ptr(f), _ptr(e), _ptr(v), _ptr(mv),
                          int(virial_mode))
    return f.reshape(-1, 3), e, v, mv


def ref_vacuum_table_eval(sysd, pos, lj, rc_alg, virial_mode=2):
    """The reference's vacuum tabulated LJ (OneAtomPair<VacuumBoundary
    Conditions, Universal, LennardJonesTableForce<S, 7, Real>>), lj = (kind,
    switchon, cutoff, order, switchoff) with kind C2, Cn or ComplimentCnCn:
    (forces, energies (coulomb, lj), virial, molvirial)."""
    lib = ref_lib()
    lib.pmref_vacuum_table_eval.argtypes = [_I, _P, _P, _P, _P, _I, _P, _I, _P, _D, _D, _I, _P,
                                            _D, _P, _P, _P, _P, _P, _I]
    lib.pmref_vacuum_table_eval.restype = _I
    ar = _Arrays(sysd)
    p = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1)
    sp = np.asarray(lj[1:5], dtype=np.float64)
    f = np.zeros(p.size)
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    rc = lib.pmref_vacuum_table_eval(ar.n, _ptr(ar.type), _ptr(ar.q), _ptr(ar.mol), _ptr(ar.mass),
                                     ar.ntypes, _ptr(ar.lj), ar.nexcl, _ptr(ar.excl),
                                     float(sysd.get("coulomb_scaling", 1.0)),
                                     float(sysd["cellsize"]), RefForce.SWITCH_KINDS[lj[0]],
                                     _ptr(sp), float(rc_alg), _ptr(p), _ptr(f), _ptr(e), _ptr(v),
                                     _ptr(mv), int(virial_mode))
    if rc:
        raise RuntimeError("pmref_vacuum_table_eval failed")
    return f.reshape(-1, 3), e, v, mv


def ref_load_psf(psf, par, pdb, exclude="scaled1-4"):
    """Reads a PSF/PAR/PDB triple with the reference's readers and topology
    builder; returns a dict of the arrays the nonbonded force consumes."""
    lib = ref_lib()
    n, nt, ne = _I(), _I(), _I()
    args = [psf.encode(), par.encode(), pdb.encode(), exclude.encode()]
    rc = lib.pmref_load_psf(*args, ctypes.byref(n), ctypes.byref(nt), ctypes.byref(ne),
                            None, None, None, None, None, None, None)
    if rc:
        raise RuntimeError(f"pmref_load_psf failed: {rc}")
    N, NT, NE = n.value, nt.value, ne.value
    pos = np.zeros(3 * N)
    typ = np.zeros(N, np.int32)
    q = np.zeros(N)
    mol = np.zeros(N, np.int32)
    mass = np.zeros(N)
    lj = np.zeros(4 * NT * NT)
    ex = np.zeros(3 * max(NE, 1), np.int32)
    rc = lib.pmref_load_psf(*args, ctypes.byref(n), ctypes.byref(nt), ctypes.byref(ne),
                            _ptr(pos), _ptr(typ), _ptr(q), _ptr(mol), _ptr(mass), _ptr(lj),
                            _ptr(ex))
    if rc:
        raise RuntimeError(f"pmref_load_psf failed: {rc}")
    return dict(pos=pos.reshape(N, 3), type=typ, qscaled=q, mol=mol, mass=mass,
                lj=lj.reshape(NT, NT, 4), excl=ex[:3 * NE].reshape(NE, 3))
