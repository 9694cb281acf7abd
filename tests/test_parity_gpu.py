"""GPU parity: libpmb200 (through its C ABI) against the reference's own
outputs (committed fixtures) and the CPU oracle on the same inputs.

Tolerances (written here, checked below):
* FP64 kernel: forces RMS relative <= 1e-12, energies/virial relative
  <= 1e-11 -- only the summation order differs from the reference.
* mixed kernel: forces RMS relative <= 1e-5;
  energies: relative <= 1e-6 on the 41,472-atom box; on the small boxes,
  whose lattice-start Coulomb energy cancels to ~1e-4 of the summed pair
  magnitudes, |dE| <= 1e-6 * sum over pairs |E_pair| (bounded here by
  2e-3 kcal/mol); virial relative <= 1e-5.
"""
import numpy as np
import pytest

from oracle import oracle as O
from protomoladdon_b200 import _lib, water
from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)
from protomoladdon_b200._lib import PmbError

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def run(d, precision, virial=True, molvir=True, pos=None, F0=None):
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    F = np.zeros_like(d["pos"]) if F0 is None else F0.copy()
    E = ScalarStructure(virial=virial, molecular_virial=molvir)
    f.evaluate(topo, d["pos"] if pos is None else pos, F, E)
    pairs = f.last_pair_count()
    f.close()
    return F, E, pairs


@pytest.mark.parametrize("fx", ["water423", "water648", "modified648"])
def test_fp64_matches_reference(fx, request):
    d = request.getfixturevalue(fx)
    F, E, _ = run(d, "fp64")
    assert rms_rel(F, d["ref_forces"]) <= 1e-12
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-11 * abs(e[0])
    assert abs(E[1] - e[1]) <= 1e-11 * abs(e[1])
    assert np.allclose(E.virial_matrix().ravel(), d["ref_virial"], rtol=1e-11, atol=1e-9)
    assert np.allclose(E.molvirial_matrix().ravel(), d["ref_molvirial"], rtol=1e-11, atol=1e-9)


@pytest.mark.parametrize("fx", ["water423", "water648", "modified648"])
def test_mixed_matches_reference(fx, request):
    d = request.getfixturevalue(fx)
    F, E, _ = run(d, "mixed")
    assert rms_rel(F, d["ref_forces"]) <= 1e-5
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 2e-3
    assert abs(E[1] - e[1]) <= 2e-3
    v = d["ref_virial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-5 * np.abs(v).max()
    mv = d["ref_molvirial"]
    assert np.abs(E.molvirial_matrix().ravel() - mv).max() <= 1e-5 * np.abs(v).max()


def test_golden_energies_through_gpu(water423):
    """The reference's t = 0 golden energies (8 significant digits)."""
    for prec in ("fp64", "mixed"):
        _, E, _ = run(water423, prec, virial=False, molvir=False)
        assert abs(E[1] - water423["golden_elj"]) <= 5e-4
        assert abs(E[0] - water423["golden_ecoul"]) <= 5e-4


@pytest.fixture(scope="module")
def medium():
    s = water.medium_41k()
    f, e, v, mv = O.restate_eval(s, s["pos"], virial_mode=1)
    s.update(ref_forces=f, ref_energies=e, ref_virial=v)
    s["ref_pairs"] = O.restate_count_pairs(s, s["pos"])
    return s


def test_medium_41k_mixed(medium):
    F, E, pairs = run(medium, "mixed", molvir=False)
    assert rms_rel(F, medium["ref_forces"]) <= 1e-5
    e = medium["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-6 * abs(e[0])
    assert abs(E[1] - e[1]) <= 1e-6 * abs(e[1])
    v = medium["ref_virial"]
    assert np.abs(E.virial_matrix().ravel() - v).max() <= 1e-5 * np.abs(v).max()
    assert abs(pairs - medium["ref_pairs"]) <= 1e-6 * medium["ref_pairs"]


def test_medium_41k_fp64(medium):
    F, E, pairs = run(medium, "fp64", molvir=False)
    assert rms_rel(F, medium["ref_forces"]) <= 1e-12
    e = medium["ref_energies"]
    assert np.allclose([E[0], E[1]], e, rtol=1e-11)
    assert pairs == medium["ref_pairs"]


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_deterministic_and_accumulates(water648, precision):
    F1, E1, _ = run(water648, precision)
    F2, E2, _ = run(water648, precision)
    assert np.array_equal(F1, F2) and np.array_equal(E1.table, E2.table)
    F3, _, _ = run(water648, precision, F0=F1)
    assert np.allclose(F3, 2 * F1, rtol=1e-15, atol=1e-12)


@pytest.mark.parametrize("box,virial", [("water648", True), ("water648", False),
                                        ("medium", False)])
def test_fused_reduction_equals_separate_kernels(box, virial, request):
    """Mixed energy evaluations finalize the forces and reduce the partial
    rows in one launch (k_finalize_reduce); the kernel-timing mode runs
    k_finalize, k_reduce1 and k_reduce2 instead.  Same sums in the same order:
    forces, energies, virials and pair counts equal bit for bit, on a box of
    fewer atoms than reduction blocks and on one of more, twice in a row (the
    arrival counter starts from zero again)."""
    d = request.getfixturevalue(box)
    topo = PeriodicTopology.from_dict(d)
    res = []
    for timing in (False, True, False):
        f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                           precision="mixed")
        f.set_pair_kernel("search")
        f._ensure(topo)
        f.set_kernel_timing(timing)
        for _ in range(2):
            F = np.zeros_like(d["pos"])
            E = ScalarStructure(virial=virial, molecular_virial=virial)
            f.evaluate(topo, d["pos"], F, E)
            res.append((F, E.table.copy(), f.last_pair_count()))
        f.close()
    for F, T, p in res[1:]:
        assert np.array_equal(F, res[0][0])
        assert np.array_equal(T, res[0][1])
        assert p == res[0][2]


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_unwrapped_and_translated_positions(water648, precision):
    L = water648["box"]
    shift = np.array([5 * L[0], -3 * L[1], 2 * L[2]])
    F0, E0, _ = run(water648, precision)
    F1, E1, _ = run(water648, precision, pos=water648["pos"] + shift)
    tol = 1e-10 if precision == "fp64" else 1e-5
    assert rms_rel(F1, F0) <= tol


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_ions_four_types(precision):
    s = water.water_box(12, rc=12.0, ron=11.0, ion_fraction=0.04, seed=5)
    f, e, v, _ = O.restate_eval(s, s["pos"], virial_mode=1)
    F, E, _ = run(s, precision, molvir=False)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rms_rel(F, f) <= tol
    assert abs(E[1] - e[1]) <= (1e-11 if precision == "fp64" else 1e-5) * abs(e[1])


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_non_cubic_box(precision):
    s = water.water_box(8, rc=9.0, ron=8.0, seed=3)
    s["box"] = s["box"] * np.array([1.0, 1.13, 0.97])
    s["pos"] = s["pos"] * np.array([1.0, 1.13, 0.97])
    s["origin"] = 0.5 * s["box"]
    f, e, v, _ = O.restate_eval(s, s["pos"], virial_mode=1)
    F, E, _ = run(s, precision, molvir=False)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rms_rel(F, f) <= tol


def test_errors_are_reported(water648):
    d = dict(water648)
    pos = d["pos"].copy()
    pos[5, 1] = np.nan
    with pytest.raises(PmbError) as ei:
        run(d, "mixed", pos=pos)
    assert ei.value.code == _lib.PMB200_EDEVICE
    small = dict(water648)
    small["box"] = np.array([15.0, 15.0, 15.0])  # < 2 * cutoff 8
    with pytest.raises(PmbError) as ei:
        run(small, "fp64")
    assert ei.value.code == _lib.PMB200_EUNSUPPORTED


def test_coincident_atoms_are_reported(water648):
    """Two atoms of different molecules at one position: the reference
    divides by zero; the mixed kernel's pair force leaves the fixed-point
    range and the evaluation reports a device error."""
    d = dict(water648)
    pos = d["pos"].copy()
    pos[9] = pos[0]  # atom 9 belongs to another water than atom 0
    assert d["mol"][9] != d["mol"][0]
    with pytest.raises(PmbError) as ei:
        run(d, "mixed", pos=pos)
    assert ei.value.code == _lib.PMB200_EDEVICE


def test_empty_system(water648):
    d = dict(water648)
    for k in ("type", "qscaled", "mol", "mass"):
        d[k] = water648[k][:0]
    d["pos"] = water648["pos"][:0]
    d["excl"] = np.zeros((0, 3), np.int32)
    F, E, pairs = run(d, "mixed")
    assert F.shape == (0, 3) and E[0] == 0.0 and E[1] == 0.0 and pairs == 0


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 2e-5)])
def test_leapfrog_device_vs_reference(water648, precision, tol):
    import torch
    d = water648
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    dev = torch.device("cuda:0")
    pos = torch.tensor(d["pos"], dtype=torch.float64, device=dev).contiguous()
    vel = torch.tensor(d["vel"], dtype=torch.float64, device=dev).contiguous()
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device=dev)
    f.leapfrog_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), 1.0, 20,
                      out.data_ptr(), _lib.PMB200_ENERGY)
    f.sync()
    p = pos.cpu().numpy()
    v = vel.cpu().numpy()
    f.close()
    assert np.abs(p - d["lf20_pos"]).max() <= tol * 10
    assert rms_rel(v, d["lf20_vel"]) <= tol * 10
    e = out.cpu().numpy()[:2]
    # unconstrained hydrogens collapse onto neighbouring oxygens in 20 fs, so
    # the final Coulomb energy is ~1e4; mixed: 2e-6 relative, FP64: 5e-3 abs
    rtol = 2e-6 if precision == "mixed" else 0.0
    assert np.allclose(e, d["lf20_energies"], rtol=rtol, atol=5e-3)


def test_device_path_equals_host_path(water648):
    """The host-buffer call of a mixed context is the device evaluation with
    its forces read back in FP32: bit for bit; energies and virial unchanged."""
    import torch
    d = water648
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"])
    F, E, _ = run(d, "mixed", molvir=False)
    pos = torch.tensor(d["pos"], dtype=torch.float64, device="cuda:0")
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device="cuda:0")
    f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(),
                      _lib.PMB200_ENERGY | _lib.PMB200_VIRIAL)
    f.sync()
    f.close()
    Fd = frc.cpu().numpy()
    assert np.array_equal(Fd.astype(np.float32).astype(np.float64), F)
    assert rms_rel(F, Fd) <= 1e-7
    o = out.cpu().numpy()
    assert o[0] == E[0] and o[1] == E[1]
    assert np.array_equal(o[2:11], E.virial_matrix().ravel())


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-9), ("mixed", 1e-5)])
def test_rigid_leapfrog_device_vs_oracle(water648, precision, tol):
    """SETTLE-constrained leapfrog on the device against the oracle's."""
    import torch
    d = water648
    w = water.rigid_waters(d)
    p_ref, v_ref, e_ref = O.restate_leapfrog_rigid(d, d["pos"], d["vel"], 1.0, 20, w,
                                                   water.D_OH, water.D_HH)
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision=precision)
    f.set_rigid_waters(topo, w, water.D_OH, water.D_HH)
    dev = torch.device("cuda:0")
    pos = torch.tensor(d["pos"], dtype=torch.float64, device=dev)
    vel = torch.tensor(d["vel"], dtype=torch.float64, device=dev)
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device=dev)
    f.leapfrog_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), 1.0, 20,
                      out.data_ptr(), _lib.PMB200_ENERGY)
    f.sync()
    p, v = pos.cpu().numpy(), vel.cpu().numpy()
    f.close()
    x = p[w]
    assert np.abs(np.linalg.norm(x[:, 1] - x[:, 0], axis=1) - water.D_OH).max() < 1e-10
    assert np.abs(np.linalg.norm(x[:, 2] - x[:, 1], axis=1) - water.D_HH).max() < 1e-10
    assert np.abs(p - p_ref).max() <= tol
    assert rms_rel(v, v_ref) <= 10 * tol
    assert np.allclose(out.cpu().numpy()[:2], e_ref, rtol=0, atol=5e-3)


def test_step_device_matches_leapfrog_body(water648):
    """pmb200_step_device (graph replay) equals kick + drift + SETTLE + force."""
    import torch
    d = water648
    w = water.rigid_waters(d)
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"],
                                       precision="fp64")
    f.set_rigid_waters(topo, w, water.D_OH, water.D_HH)
    st = torch.cuda.Stream()
    pos = torch.tensor(d["pos"], dtype=torch.float64, device="cuda:0")
    vel = torch.tensor(d["vel"], dtype=torch.float64, device="cuda:0")
    frc = torch.tensor(d["ref_forces"], dtype=torch.float64, device="cuda:0")
    for _ in range(3):
        f.step_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), 1.0, st.cuda_stream)
    st.synchronize()
    f.sync()
    from protomoladdon_b200 import rigid
    P, V, F = d["pos"].copy(), d["vel"].copy(), d["ref_forces"].copy()
    for _ in range(3):
        rigid.kick_drift_settle(P, V, F, d["mass"], 1.0, w, water.D_OH, water.D_HH)
        F, _, _, _ = O.restate_eval(d, P, 0)
    f.close()
    assert np.abs(pos.cpu().numpy() - P).max() < 1e-10
    assert rms_rel(frc.cpu().numpy(), F) < 1e-11


def test_pinned_host_positions_equal_pageable(water648):
    """pmb200_eval transfers page-locked positions directly and pageable ones
    through its staging copy: the same forces and energies either way."""
    import torch
    d = water648
    topo = PeriodicTopology.from_dict(d)
    f = NonbondedCutoffB200SystemForce(d["ron"], d["rc_lj"], d["rc_coul"], d["rc_alg"])
    pinned = torch.empty(d["pos"].shape, dtype=torch.float64, pin_memory=True).numpy()
    pinned[...] = d["pos"]
    out = []
    for pos in (np.ascontiguousarray(d["pos"]), pinned):
        F = np.zeros_like(d["pos"])
        E = ScalarStructure()
        f.evaluate(topo, pos, F, E)
        out.append((F, E[0], E[1]))
    f.close()
    assert np.array_equal(out[0][0], out[1][0])
    assert out[0][1:] == out[1][1:]


@pytest.mark.parametrize("cellsize", [0.0, 3.4, 4.2, 7.0, 10.5, 16.0])
def test_cell_sizes_keep_every_pair(cellsize):
    """The mixed kernel drops a staged atom that lies beyond the cutoff of the
    box around the chunk's i atoms.  At every cell size (rc/3 cells with 1 to 2
    atoms, cells wider than the cutoff holding several 32-atom chunks and home
    cells whose atoms can be farther apart than the cutoff) it must still find
    the oracle's pair set and forces."""
    s = water.water_box(11, rc=10.0, ron=9.0, seed=11)
    f, e, v, _ = O.restate_eval(s, s["pos"], virial_mode=1)
    ref_pairs = O.restate_count_pairs(s, s["pos"])
    topo = PeriodicTopology.from_dict(s)
    force = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                           precision="mixed", cellsize=cellsize)
    F = np.zeros_like(s["pos"])
    E = ScalarStructure(virial=True)
    force.evaluate(topo, s["pos"], F, E)
    pairs = force.last_pair_count()
    force.close()
    # the FP32 cutoff test may decide a pair within ~1e-7 of r = rc either way
    assert abs(pairs - ref_pairs) <= 2, (pairs, ref_pairs)
    assert rms_rel(F, f) <= 1e-5
    # cutoff-form Coulomb energy from FP64 distances, LJ energy in FP32
    assert abs(E[0] - e[0]) <= 1e-6 * abs(e[0])
    assert abs(E[1] - e[1]) <= 1e-6 * abs(e[1])


@pytest.mark.parametrize("fx", ["water423", "water648", "modified648"])
def test_mixed_energies_relative(fx, request):
    """The cutoff-form Coulomb energy of the mixed kernel is summed from FP64
    distances: within 1e-6 of the reference's own value even on the small
    lattice-start boxes (whose total cancels to ~1e-4 of the pair sum)."""
    d = request.getfixturevalue(fx)
    F, E, _ = run(d, "mixed")
    e = d["ref_energies"]
    assert abs(E[0] - e[0]) <= 1e-6 * abs(e[0])
    assert abs(E[1] - e[1]) <= 1e-6 * abs(e[1])
