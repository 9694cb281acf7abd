"""Host-side mirror of ProtoMol's SystemForce interface for the B200 force.

``NonbondedCutoffB200SystemForce`` stands where the reference registers
``NonbondedCutoffSystemForce<CubicCellManager, OneAtomPairTwo<
PeriodicBoundaryConditions, C2SwitchingFunction, LennardJonesForce,
C1SwitchingFunction, CoulombForce>>``
(protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:75-76):

* keyword ``NonbondedCutoffB200`` (the reference's ``NonbondedCutoff`` id is
  taken by the CPU prototype and duplicate ids throw,
  protomol/src/protomol/base/Factory.h:50-58);
* ``make(values)`` takes the reference's parameter list in its order
  (OneAtomPairTwo::getParameters then NonbondedCutoffForce::getParameters):
  ``[-switchon, C2 -cutoff, C1 -cutoff, algorithm -cutoff]`` and applies
  C2SwitchingFunction::make's check 0 <= switchon < cutoff
  (protomol/src/protomol/switch/C2SwitchingFunction.cpp:30-41);
* ``evaluate(topo, positions, forces, energies)`` is
  SystemForce::evaluate (protomol/src/protomol/force/system/SystemForce.h:
  35-38): forces and energies are accumulated into, the virial is added when
  ``energies.virial`` is on and the molecular virial when
  ``energies.molecular_virial`` is on.

Every call goes through libpmb200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import re

import numpy as np

from . import _lib
from ._lib import PmbError

_P = ctypes.c_void_p


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class ScalarStructure:
    """Energies and virials with the reference's index layout
    (protomol/src/protomol/type/ScalarStructure.h:26-67)."""
    COULOMB, LENNARDJONES = 0, 1
    VIRIALXX = 7
    MOLVIRIALXX = 16
    LAST = 36

    def __init__(self, virial=False, molecular_virial=False):
        self.table = np.zeros(self.LAST)
        self.virial = virial
        self.molecular_virial = molecular_virial

    def clear(self):
        self.table[:] = 0.0

    def __getitem__(self, k):
        return self.table[k]

    def __setitem__(self, k, v):
        self.table[k] = v

    def virial_matrix(self):
        return self.table[self.VIRIALXX:self.VIRIALXX + 9].reshape(3, 3)

    def molvirial_matrix(self):
        return self.table[self.MOLVIRIALXX:self.MOLVIRIALXX + 9].reshape(3, 3)


class PeriodicTopology:
    """The parts of Topology<PeriodicBoundaryConditions, CubicCellManager> the
    force reads, as flat arrays (see pmb200_set_topology / pmb200_set_box)."""

    def __init__(self, type, qscaled, mol, lj, excl, box, origin=(0.0, 0.0, 0.0),
                 mass=None, coulomb_scaling=1.0, cellsize=0.0):
        self.type = np.ascontiguousarray(type, dtype=np.int32)
        self.qscaled = np.ascontiguousarray(qscaled, dtype=np.float64)
        self.mol = np.ascontiguousarray(mol, dtype=np.int32)
        self.mass = None if mass is None else np.ascontiguousarray(mass, dtype=np.float64)
        lj = np.asarray(lj, dtype=np.float64)
        self.ntypes = int(round((lj.size // 4) ** 0.5))
        self.lj = np.ascontiguousarray(lj.reshape(-1))
        self.excl = np.ascontiguousarray(np.asarray(excl, dtype=np.int32).reshape(-1, 3))
        box = np.asarray(box, dtype=np.float64)
        if box.shape == (3,):
            box = np.diag(box)
        self.e = np.ascontiguousarray(box.reshape(3, 3))
        self.origin = np.ascontiguousarray(origin, dtype=np.float64)
        self.coulomb_scaling = float(coulomb_scaling)
        self.cellsize = float(cellsize)
        self.version = 0
        # vacuum boundaries: (lo[3], hi[3]) of the cell domain; None = periodic
        self.domain = None

    @property
    def n(self):
        return self.type.size

    @classmethod
    def from_dict(cls, d):
        return cls(d["type"], d["qscaled"], d["mol"], d["lj"], d["excl"], d["box"],
                   d.get("origin", (0.0, 0.0, 0.0)), d.get("mass"),
                   d.get("coulomb_scaling", 1.0), d.get("cellsize_gpu", 0.0))


_ID_RE = re.compile(r"-(\w+)\s+([^\s-][^\s]*)")


class NonbondedCutoffB200SystemForce:
    keyword = "NonbondedCutoffB200"

    def __init__(self, switchon, cutoff_lj, cutoff_coul, cutoff_alg, precision="mixed",
                 device=0, cellsize=0.0):
        if not (switchon >= 0.0 and cutoff_lj > 0.0 and switchon < cutoff_lj):
            raise ValueError(
                f"C2 switching function: 0 <= switchon (={switchon}) < cutoff (={cutoff_lj}).")
        self.switchon = float(switchon)
        self.cutoff_lj = float(cutoff_lj)
        self.cutoff_coul = float(cutoff_coul)
        self.cutoff_alg = float(cutoff_alg)
        self.precision = precision
        self.device = int(device)
        self.cellsize = float(cellsize)
        self._ctx = None
        self._topo_key = None
        self._box_key = None

    # ---- Makeable -------------------------------------------------------
    @classmethod
    def make(cls, values, **kw):
        """values in the reference's order: switchon, C2 cutoff, C1 cutoff,
        algorithm cutoff."""
        if len(values) != 4:
            raise ValueError(f"{cls.keyword} takes 4 parameters, got {len(values)}")
        return cls(*[float(v) for v in values], **kw)

    @classmethod
    def from_id(cls, force_id, **kw):
        """Parses a config force line such as
        ``LennardJones Coulomb -algorithm NonbondedCutoffB200
        -switchingFunction C2 -switchingFunction C1 -switchon 9 -cutoff 10
        -cutoff 10 -cutoff 10``."""
        toks = force_id.split()
        if toks[:2] != ["LennardJones", "Coulomb"]:
            raise ValueError("expected 'LennardJones Coulomb' potentials")
        opts = list(zip(toks[2::2], toks[3::2])) if len(toks) % 2 == 0 else None
        if opts is None:
            raise ValueError(f"cannot parse force id {force_id!r}")
        alg = [v for k, v in opts if k == "-algorithm"]
        if alg != [cls.keyword]:
            raise ValueError(f"algorithm must be {cls.keyword}")
        sw = [v for k, v in opts if k == "-switchingFunction"]
        if sw != ["C2", "C1"]:
            raise ValueError("switching functions must be C2 (LennardJones) then C1 (Coulomb)")
        ron = [float(v) for k, v in opts if k == "-switchon"]
        cut = [float(v) for k, v in opts if k == "-cutoff"]
        if len(ron) != 1 or len(cut) != 3:
            raise ValueError("need -switchon and three -cutoff values")
        return cls(ron[0], cut[0], cut[1], cut[2], **kw)

    def get_id(self):
        return (f"LennardJones Coulomb -algorithm {self.keyword} -switchingFunction C2 "
                f"-switchingFunction C1 -switchon {self.switchon:g} -cutoff {self.cutoff_lj:g} "
                f"-cutoff {self.cutoff_coul:g} -cutoff {self.cutoff_alg:g}")

    # ---- context --------------------------------------------------------
    def _check(self, rc):
        if rc != _lib.PMB200_OK:
            msg = _lib.lib().pmb200_last_error(self._ctx) if self._ctx else b""
            raise PmbError(rc, (msg or b"").decode())

    def _ensure(self, topo: PeriodicTopology):
        L = _lib.lib()
        if self._ctx is None:
            self._ctx = self._create(topo)
            if getattr(self, "_pair_kernel", _lib.PMB200_KERNEL_SEARCH):
                self._check(L.pmb200_set_pair_kernel(self._ctx, self._pair_kernel))
        # the cached topology is held by reference with its version: an id()
        # alone can be handed to a new topology once the old one is freed
        key = self._topo_key
        if key is None or key[0] is not topo or key[1] != topo.version:
            ex = topo.excl.reshape(-1)
            self._check(L.pmb200_set_topology(
                self._ctx, topo.n, _ptr(topo.type), _ptr(topo.qscaled), _ptr(topo.mol),
                _ptr(topo.mass), topo.ntypes, _ptr(topo.lj), topo.excl.shape[0],
                _ptr(ex) if ex.size else None, topo.coulomb_scaling))
            self._topo_key = (topo, topo.version)
            self._box_key = None
        dom = None if topo.domain is None else tuple(
            np.ascontiguousarray(x, dtype=np.float64) for x in topo.domain)
        bkey = (topo.e.tobytes(), topo.origin.tobytes(),
                None if dom is None else (dom[0].tobytes(), dom[1].tobytes()))
        if self._box_key != bkey:
            if dom is not None:
                self._check(L.pmb200_set_vacuum_domain(self._ctx, _ptr(dom[0]), _ptr(dom[1])))
            else:
                e1, e2, e3 = (np.ascontiguousarray(topo.e[k]) for k in range(3))
                self._check(L.pmb200_set_box(self._ctx, _ptr(e1), _ptr(e2), _ptr(e3),
                                             _ptr(topo.origin)))
            self._box_key = bkey

    def _create(self, topo):
        p = _lib.Params(_lib.PMB200_MIXED if self.precision == "mixed" else _lib.PMB200_FP64,
                        self.device, self.switchon, self.cutoff_lj, self.cutoff_coul,
                        self.cutoff_alg, self.cellsize or topo.cellsize)
        h = _P()
        rc = _lib.lib().pmb200_create(ctypes.byref(p), ctypes.byref(h))
        if rc != _lib.PMB200_OK:
            raise PmbError(rc, "pmb200_create rejected the parameters")
        return h

    def uncache(self):
        self._topo_key = None
        self._box_key = None

    # ---- SystemForce ----------------------------------------------------
    def evaluate(self, topo: PeriodicTopology, positions, forces, energies: ScalarStructure):
        """Accumulates forces (n,3 float64, C-contiguous, modified in place)
        and energies like SystemForce::evaluate."""
        self._host_eval(topo, positions, forces, energies, None)

    def number_of_blocks(self, topo):
        """Force::numberOfBlocks: the cells of the device grid (one process,
        Parallel::getNumberOfPackages(n) == n)."""
        self._ensure(topo)
        d, _ = self.grid()
        return int(d[0] * d[1] * d[2])

    def parallel_evaluate(self, topo, positions, forces, energies, rank, nranks):
        """SystemForce::parallelEvaluate of one rank in the reference's static
        mode (Parallel::next() grants block i to rank i mod nranks): block i
        of numberOfBlocks covers the cells [n i / count, n (i + 1) / count).
        Summed over the ranks (Parallel::reduce) it is evaluate()."""
        count = self.number_of_blocks(topo)
        n = count
        for i in range(rank, count, nranks):
            lo, hi = n * i // count, n * (i + 1) // count
            self.evaluate_cells(topo, positions, forces, energies, lo, hi)

    def evaluate_cells(self, topo, positions, forces, energies, cell_lo, cell_hi):
        """The pairs whose i-cell lies in [cell_lo, cell_hi) (see
        pmb200_eval_cells), accumulated like evaluate()."""
        self._host_eval(topo, positions, forces, energies, (int(cell_lo), int(cell_hi)))

    def _host_eval(self, topo, positions, forces, energies, cells):
        self._ensure(topo)
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        if not (isinstance(forces, np.ndarray) and forces.dtype == np.float64
                and forces.flags.c_contiguous):
            raise TypeError("forces must be a C-contiguous float64 numpy array")
        flags = _lib.PMB200_ENERGY
        vir = np.zeros(9)
        mvir = np.zeros(9)
        if energies.virial:
            flags |= _lib.PMB200_VIRIAL
        if energies.molecular_virial:
            flags |= _lib.PMB200_MOLVIRIAL
        e = np.zeros(2)
        if cells is None:
            self._check(_lib.lib().pmb200_eval(self._ctx, _ptr(pos), _ptr(forces), _ptr(e),
                                               _ptr(vir), _ptr(mvir), flags))
        else:
            self._check(_lib.lib().pmb200_eval_cells(self._ctx, _ptr(pos), _ptr(forces), _ptr(e),
                                                     _ptr(vir), _ptr(mvir), flags, cells[0],
                                                     cells[1]))
        energies[ScalarStructure.COULOMB] += e[0]
        energies[ScalarStructure.LENNARDJONES] += e[1]
        if energies.virial:
            energies.table[ScalarStructure.VIRIALXX:ScalarStructure.VIRIALXX + 9] += vir
        if energies.molecular_virial:
            energies.table[ScalarStructure.MOLVIRIALXX:ScalarStructure.MOLVIRIALXX + 9] += mvir

    def evaluate_device(self, topo, pos_ptr, force_ptr, out_ptr=None, flags=0, stream=None):
        """Device-resident evaluation on raw device pointers (ints), e.g.
        ``tensor.data_ptr()``; forces are accumulated, out (20 doubles) is
        overwritten.  Asynchronous: call sync()."""
        self._ensure(topo)
        self._check(_lib.lib().pmb200_eval_device(
            self._ctx, _P(pos_ptr), _P(force_ptr), _P(out_ptr) if out_ptr else None,
            int(flags), _P(stream) if stream else None))

    def autotune(self, topo, pos_ptr, reps=10, stream=None):
        """pmb200_autotune on device positions (a raw pointer): times the
        evaluation over cell sizes and, for mixed precision, warps per i-cell,
        applies the fastest and returns the choice as a dict."""
        self._ensure(topo)
        r = (ctypes.c_double * 8)()
        self._check(_lib.lib().pmb200_autotune(self._ctx, _P(pos_ptr),
                                               _P(stream) if stream else None, int(reps), r))
        names = {_lib.PMB200_KERNEL_SEARCH: "search", _lib.PMB200_KERNEL_TILES: "tiles",
                 _lib.PMB200_KERNEL_CLUSTERS: "clusters"}
        return {"cellsize_hint": r[0], "warps_per_cell_energy": int(r[1]),
                "warps_per_cell_forces": int(r[2]), "ms_energy": r[3], "ms_forces": r[4],
                "configurations_timed": int(r[5]), "kernel_energy": names[int(r[6])],
                "kernel_forces": names[int(r[7])]}

    def set_pair_kernel(self, kernel):
        """The mixed pair kernel: "search" (default), "tiles" (cluster pairs of a
        cell) or "clusters" (supercluster lists; pmb200_set_pair_kernel)."""
        k = {"search": _lib.PMB200_KERNEL_SEARCH, "tiles": _lib.PMB200_KERNEL_TILES,
             "clusters": _lib.PMB200_KERNEL_CLUSTERS}[kernel]
        self._pair_kernel = k
        if self._ctx is not None:
            self._check(_lib.lib().pmb200_set_pair_kernel(self._ctx, k))

    def shard_eval_device(self, topo, pos_ptr, shard, nshards, facc_ptr, out_ptr=None, flags=0,
                          stream=None):
        """Shard ``shard`` of ``nshards`` of one evaluation (its run of i-cells)
        into the int64 fixed-point accumulator ``facc`` (3n, overwritten) and,
        when flags ask, its share of the energies / virials into out (20);
        sum both over the shards, then shard_finalize."""
        self._ensure(topo)
        self._check(_lib.lib().pmb200_shard_eval_device(
            self._ctx, _P(pos_ptr), int(shard), int(nshards), _P(facc_ptr),
            _P(out_ptr) if out_ptr else None, int(flags), _P(stream) if stream else None))

    def shard_finalize(self, facc_ptr, force_ptr, stream=None):
        """Adds the forces of a summed shard accumulator to ``force`` (3n)."""
        self._check(_lib.lib().pmb200_shard_finalize(
            self._ctx, _P(facc_ptr), _P(force_ptr), _P(stream) if stream else None))

    def leapfrog_device(self, topo, pos_ptr, vel_ptr, force_ptr, dt_fs, nsteps, out_ptr=None,
                        flags=0, stream=None):
        self._ensure(topo)
        self._check(_lib.lib().pmb200_leapfrog_device(
            self._ctx, _P(pos_ptr), _P(vel_ptr), _P(force_ptr), _P(out_ptr) if out_ptr else None,
            float(dt_fs), int(nsteps), int(flags), _P(stream) if stream else None))

    def step_device(self, topo, pos_ptr, vel_ptr, force_ptr, dt_fs, stream, out_ptr=None,
                    flags=0):
        """One leapfrog iteration (kick + drift, new forces) as a graph replay."""
        self._ensure(topo)
        self._check(_lib.lib().pmb200_step_device(
            self._ctx, _P(pos_ptr), _P(vel_ptr), _P(force_ptr), _P(out_ptr) if out_ptr else None,
            float(dt_fs), int(flags), _P(stream)))

    def param_grad_device(self, topo, pos_ptr, dq_ptr, dlj_ptr, stream=None):
        """dE/dq_scaled per atom and dE/d{A, B, A14, B14} per table entry
        (FP64 kernel; see pmb200_param_grad_device)."""
        self._ensure(topo)
        self._check(_lib.lib().pmb200_param_grad_device(
            self._ctx, _P(pos_ptr), _P(dq_ptr), _P(dlj_ptr), _P(stream) if stream else None))

    def hvp_device(self, topo, pos_ptr, w_ptr, hv_ptr, dq_ptr=None, dlj_ptr=None, stream=None):
        """hv = H w and the derivatives of w . grad E with respect to the
        charges and the table (FP64 kernel; see pmb200_hvp_device)."""
        self._ensure(topo)
        self._check(_lib.lib().pmb200_hvp_device(
            self._ctx, _P(pos_ptr), _P(w_ptr), _P(hv_ptr), _P(dq_ptr) if dq_ptr else None,
            _P(dlj_ptr) if dlj_ptr else None, _P(stream) if stream else None))

    def update_params(self, topo, q_scaled=None, lj=None):
        """New charges and/or LJ table (host arrays) for the same topology;
        the topology object's arrays are updated too."""
        self._ensure(topo)
        q = None if q_scaled is None else np.ascontiguousarray(q_scaled, dtype=np.float64)
        t = None if lj is None else np.ascontiguousarray(lj, dtype=np.float64).reshape(-1)
        self._check(_lib.lib().pmb200_update_params(self._ctx, _ptr(q), _ptr(t)))
        if q is not None:
            topo.qscaled = q.copy()
        if t is not None:
            topo.lj = t.copy()

    def update_params_device(self, topo, q_ptr=None, lj_ptr=None, stream=None):
        """New charges (n doubles) and/or LJ table (ntypes^2 * 4 doubles)
        from device pointers, queued on ``stream`` (see
        pmb200_update_params_device); the topology's host arrays are left as
        they are."""
        self._ensure(topo)
        self._check(_lib.lib().pmb200_update_params_device(
            self._ctx, _P(q_ptr) if q_ptr else None, _P(lj_ptr) if lj_ptr else None,
            _P(stream) if stream else None))

    def set_rigid_waters(self, topo, widx, d_oh, d_hh):
        """SETTLE constraints for the device integrator (see pmb200.h)."""
        self._ensure(topo)
        w = np.ascontiguousarray(widx, dtype=np.int32).reshape(-1)
        self._check(_lib.lib().pmb200_set_rigid_waters(self._ctx, w.size // 3,
                                                       _ptr(w) if w.size else None,
                                                       float(d_oh), float(d_hh)))

    def set_kernel_timing(self, on):
        self._check(_lib.lib().pmb200_set_kernel_timing(self._ctx, 1 if on else 0))

    def last_kernel_ms(self):
        v = ctypes.c_float()
        self._check(_lib.lib().pmb200_last_kernel_ms(self._ctx, ctypes.byref(v)))
        return float(v.value)

    def sync(self):
        self._check(_lib.lib().pmb200_sync(self._ctx))

    def last_pair_count(self):
        v = ctypes.c_longlong()
        self._check(_lib.lib().pmb200_last_pair_count(self._ctx, ctypes.byref(v)))
        return v.value

    def grid(self):
        d = (ctypes.c_int * 3)()
        e = (ctypes.c_double * 3)()
        self._check(_lib.lib().pmb200_grid(self._ctx, d, e))
        return tuple(d), tuple(e)

    def close(self):
        if self._ctx is not None:
            _lib.lib().pmb200_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class EwaldRealB200SystemForce(NonbondedCutoffB200SystemForce):
    """The real-space term of ProtoMol's Ewald sum on the B200: stands where
    the reference registers ``NonbondedFullEwaldSystemForce<
    PeriodicBoundaryConditions, CubicCellManager, true, false, false,
    CutoffSwitchingFunction>``
    (protomol/src/protomol/module/NonbondedFullElectrostaticForceModule.cpp:34,
    id ``Coulomb -algorithm FullEwald -real``), under its own algorithm
    keyword ``FullEwaldB200``.  Parameters in the reference's order
    (NonbondedFullEwaldSystemForce::getParameters): ``-alpha`` (<= 0: the
    reference's default from N and the volume) and ``-accuracy`` (> 0);
    rc = sqrt(-log(accuracy)) / alpha.  ``erfc`` picks the Abramowitz & Stegun
    polynomial of the reference's default build ("poly5") or erfc itself
    ("exact", the reference built with -DUSE_EWALD_EXACT_ERF).  The energy
    goes to COULOMB; everything else is inherited."""

    keyword = "FullEwaldB200"

    def __init__(self, alpha=-1.0, accuracy=1e-5, precision="mixed", device=0, cellsize=0.0,
                 erfc="poly5"):
        if not accuracy > 0.0:
            raise ValueError(f"accuracy (={accuracy}) must be positive")
        if erfc not in ("poly5", "exact"):
            raise ValueError("erfc must be 'poly5' or 'exact'")
        self.alpha = float(alpha)
        self.accuracy = float(accuracy)
        self.erfc = erfc
        self.precision = precision
        self.device = int(device)
        self.cellsize = float(cellsize)
        self._ctx = None
        self._topo_key = None
        self._box_key = None

    @classmethod
    def make(cls, values, **kw):
        """values in the reference's order: alpha, accuracy."""
        if len(values) != 2:
            raise ValueError(f"{cls.keyword} takes 2 parameters, got {len(values)}")
        return cls(float(values[0]), float(values[1]), **kw)

    @classmethod
    def from_id(cls, force_id, **kw):
        """Parses ``Coulomb -algorithm FullEwaldB200 -real -alpha 0.3
        -accuracy 1e-6`` (-alpha and -accuracy may be left out: -1 and 1e-5,
        the reference's defaults)."""
        toks = force_id.split()
        if not toks or toks[0] != "Coulomb":
            raise ValueError("expected the 'Coulomb' potential")
        if "-real" not in toks or "-reciprocal" in toks or "-correction" in toks:
            raise ValueError("only the real-space term (-real) is offered")
        rest = [t for t in toks[1:] if t != "-real"]
        opts = dict(zip(rest[0::2], rest[1::2]))
        if len(rest) % 2 or opts.get("-algorithm") != cls.keyword:
            raise ValueError(f"cannot parse force id {force_id!r}")
        return cls(float(opts.get("-alpha", -1.0)), float(opts.get("-accuracy", 1e-5)), **kw)

    def get_id(self):
        return (f"Coulomb -algorithm {self.keyword} -real -alpha {self.alpha:g} "
                f"-accuracy {self.accuracy:g}")

    def _create(self, topo):
        p = _lib.EwaldParams(
            _lib.PMB200_MIXED if self.precision == "mixed" else _lib.PMB200_FP64, self.device,
            _lib.PMB200_ERFC_EXACT if self.erfc == "exact" else _lib.PMB200_ERFC_POLY5,
            self.alpha, self.accuracy, self.cellsize or topo.cellsize)
        h = _P()
        rc = _lib.lib().pmb200_create_ewald_real(ctypes.byref(p), ctypes.byref(h))
        if rc != _lib.PMB200_OK:
            raise PmbError(rc, "pmb200_create_ewald_real rejected the parameters")
        return h

    def ewald_info(self):
        """(alpha, rc) in use, once the topology and box are set."""
        a, r = ctypes.c_double(), ctypes.c_double()
        self._check(_lib.lib().pmb200_ewald_info(self._ctx, ctypes.byref(a), ctypes.byref(r)))
        return a.value, r.value


class NonbondedCutoffB200PairForce(NonbondedCutoffB200SystemForce):
    """The other periodic cutoff registrations of NonbondedCutoffForceModule
    (protomol/src/protomol/module/NonbondedCutoffForceModule.cpp:53-82):
    OneAtomPair<PBC, S, LennardJonesForce>, OneAtomPair<PBC, S, CoulombForce>
    and OneAtomPairTwo<PBC, S1, LennardJonesForce, S2, CoulombForce> with S
    among C1, C2, Cn, ComplimentCnCn.  ``lj`` / ``coulomb``: None (term
    absent) or a tuple (kind, switchon, cutoff, order, switchoff); C1 reads
    the cutoff, C2 switchon and cutoff, Cn and ComplimentCnCn all four (see
    pmb200_create_pair).  ``lj_table``: the tabulated registrations
    OneAtomPair<PBC, UniversalSwitchingFunction, LennardJonesTableForce<S, 7,
    Real>> (NonbondedCutoffForceModule.cpp:67-72; id ``LennardJonesTable``),
    S = ``lj``'s switch among C2, Cn, ComplimentCnCn, with no Coulomb term."""

    keyword = "NonbondedCutoffB200"
    _KIND = {None: _lib.PMB200_SW_NONE, "C1": _lib.PMB200_SW_C1, "C2": _lib.PMB200_SW_C2,
             "Cn": _lib.PMB200_SW_CN, "ComplimentCnCn": _lib.PMB200_SW_CMPCNCN}
    # switch parameters as the reference lists them (getParameters;
    # CmpCnCnSwitchingFunction.cpp:35-50 for ComplimentCnCn)
    _PARAMS = {"C1": ["-cutoff"], "C2": ["-switchon", "-cutoff"],
               "Cn": ["-n", "-switchon", "-switchoff", "-cutoff"],
               "ComplimentCnCn": ["-switchon", "-switchoff", "-cutoff", "-n"]}

    def __init__(self, lj=None, coulomb=None, cutoff_alg=None, precision="mixed", device=0,
                 cellsize=0.0, lj_table=False):
        def norm(sw):
            if sw is None:
                return None
            sw = tuple(sw) + (0.0,) * (5 - len(sw))
            if sw[0] not in self._PARAMS:
                raise ValueError(f"switching function {sw[0]!r}: C1, C2, Cn or ComplimentCnCn")
            return (sw[0],) + tuple(float(x) for x in sw[1:5])
        self.lj = norm(lj)
        self.coulomb = norm(coulomb)
        if self.lj is None and self.coulomb is None:
            raise ValueError("need a Lennard-Jones or a Coulomb term")
        self.lj_table = bool(lj_table)
        if self.lj_table and (self.lj is None or self.coulomb is not None
                              or self.lj[0] not in ("C2", "Cn", "ComplimentCnCn")):
            raise ValueError("LennardJonesTable: a C2, Cn or ComplimentCnCn switch and no "
                             "Coulomb term")
        rcs = [s[2] for s in (self.lj, self.coulomb) if s is not None]
        self.cutoff_alg = float(cutoff_alg if cutoff_alg is not None else max(rcs))
        self.precision = precision
        self.device = int(device)
        self.cellsize = float(cellsize)
        self._ctx = None
        self._topo_key = None
        self._box_key = None

    def _create(self, topo):
        def arr(sw):
            return (ctypes.c_double * 4)(*(sw[1:5] if sw else (0.0,) * 4))
        p = _lib.PairParams(
            _lib.PMB200_MIXED if self.precision == "mixed" else _lib.PMB200_FP64, self.device,
            self._KIND[self.lj[0] if self.lj else None]
            | (_lib.PMB200_SW_TABLE if self.lj_table else 0), arr(self.lj),
            self._KIND[self.coulomb[0] if self.coulomb else None], arr(self.coulomb),
            self.cutoff_alg, self.cellsize or topo.cellsize)
        h = _P()
        rc = _lib.lib().pmb200_create_pair(ctypes.byref(p), ctypes.byref(h))
        if rc != _lib.PMB200_OK:
            raise PmbError(rc, "pmb200_create_pair rejected the parameters")
        return h

    @classmethod
    def _switch_args(cls, sw):
        kind, ron, rc, order, roff = sw
        vals = {"-cutoff": rc, "-switchon": ron, "-n": order, "-switchoff": roff}
        return " ".join(f"{k} {vals[k]:g}" for k in cls._PARAMS[kind])

    def get_id(self):
        pots = [n for n, s in (("LennardJonesTable" if self.lj_table else "LennardJones",
                               self.lj), ("Coulomb", self.coulomb)) if s]
        sws = [s for s in (self.lj, self.coulomb) if s]
        head = " ".join(pots) + f" -algorithm {self.keyword} " + " ".join(
            f"-switchingFunction {s[0]}" for s in sws)
        return head + " " + " ".join(self._switch_args(s) for s in sws) + \
            f" -cutoff {self.cutoff_alg:g}"

    @classmethod
    def from_id(cls, force_id, **kw):
        toks = force_id.split()
        pots = []
        while toks and not toks[0].startswith("-"):
            pots.append(toks.pop(0))
        table = pots == ["LennardJonesTable"]
        if table:
            pots = ["LennardJones"]
            kw = dict(kw, lj_table=True)
        if pots not in (["LennardJones"], ["Coulomb"], ["LennardJones", "Coulomb"]):
            raise ValueError(f"potentials {pots}: LennardJones and/or Coulomb, or "
                             "LennardJonesTable")
        pairs = list(zip(toks[0::2], toks[1::2]))
        if len(toks) % 2:
            raise ValueError(f"cannot parse force id {force_id!r}")
        if [v for k, v in pairs if k == "-algorithm"] != [cls.keyword]:
            raise ValueError(f"algorithm must be {cls.keyword}")
        sws = [v for k, v in pairs if k == "-switchingFunction"]
        if len(sws) != len(pots):
            raise ValueError("one switching function per potential")
        params = [(k, float(v)) for k, v in pairs if k not in ("-algorithm", "-switchingFunction")]
        specs = []
        for sw in sws:
            if sw not in cls._PARAMS:
                raise ValueError(f"switching function {sw!r}: C1, C2, Cn or ComplimentCnCn")
            vals = {}
            for key in cls._PARAMS[sw]:
                if not params or params[0][0] != key:
                    raise ValueError(f"{sw}: expected {key}")
                vals[key] = params.pop(0)[1]
            specs.append((sw, vals.get("-switchon", 0.0), vals["-cutoff"], vals.get("-n", 0.0),
                          vals.get("-switchoff", 0.0)))
        if len(params) != 1 or params[0][0] != "-cutoff":
            raise ValueError("expected the algorithm -cutoff last")
        lj = specs[0] if pots[0] == "LennardJones" else None
        co = specs[-1] if pots[-1] == "Coulomb" else None
        return cls(lj, co, params[0][1], **kw)
