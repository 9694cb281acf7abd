"""The supercluster pair kernel (PMB200_KERNEL_CLUSTERS) against the oracle
and the search kernel: the same pair set (up to FP32 ties at r = rc), forces
within 1e-5 RMS and energies within 1e-6 of the reference's FP64 arithmetic,
bitwise-reproducible results, the box shapes and positions it accepts, the
device step, and the configurations it leaves to the search kernel."""
from __future__ import annotations

import numpy as np
import pytest

from oracle import oracle as O
from protomoladdon_b200 import _lib, water
from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def evaluate(s, kernel, pos=None, flags_energy=True, F0=None):
    topo = PeriodicTopology.from_dict(s)
    f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                       precision="mixed")
    f.set_pair_kernel(kernel)
    F = np.zeros_like(s["pos"]) if F0 is None else F0.copy()
    E = ScalarStructure()
    f.evaluate(topo, s["pos"] if pos is None else pos, F, E)
    pairs = f.last_pair_count()
    f.close()
    return F, E, pairs


def check_vs_oracle(s, pos=None):
    p = s["pos"] if pos is None else pos
    fo, eo, _, _ = O.restate_eval(s, p, virial_mode=0)
    ref_pairs = O.restate_count_pairs(s, p)
    F, E, pairs = evaluate(s, "clusters", pos=pos)
    assert rms_rel(F, fo) <= 1e-5
    assert abs(E[0] - eo[0]) <= 1e-6 * abs(eo[0])
    assert abs(E[1] - eo[1]) <= 1e-6 * abs(eo[1])
    # the FP32 cutoff test may decide a pair within ~1e-7 of r = rc either way
    assert abs(pairs - ref_pairs) <= max(2, 1e-6 * ref_pairs), (pairs, ref_pairs)
    return F, E


@pytest.fixture(scope="module")
def medium():
    return water.medium_41k()


def test_water_41k_vs_oracle(medium):
    check_vs_oracle(medium)


def test_water_41k_deterministic_and_accumulates(medium):
    F1, E1, p1 = evaluate(medium, "clusters")
    F2, E2, p2 = evaluate(medium, "clusters")
    assert np.array_equal(F1, F2) and E1[0] == E2[0] and E1[1] == E2[1] and p1 == p2
    F3, _, _ = evaluate(medium, "clusters", F0=F1)
    assert np.allclose(F3, 2 * F1, rtol=1e-15, atol=1e-12)


def test_water_41k_close_to_search_kernel(medium):
    Fc, Ec, pc = evaluate(medium, "clusters")
    Fs, Es, ps = evaluate(medium, "search")
    assert rms_rel(Fc, Fs) <= 3e-6
    assert abs(Ec[0] - Es[0]) <= 1e-7 * abs(Es[0])
    assert abs(pc - ps) <= 4


def test_ions_four_types():
    s = water.water_box(16, rc=10.0, ron=9.0, ion_fraction=0.04, seed=5)
    check_vs_oracle(s)


def test_non_cubic_box_and_unwrapped_positions():
    s = water.water_box(18, rc=9.0, ron=8.0, seed=3)
    scale = np.array([1.0, 1.13, 0.97])
    s["box"] = s["box"] * scale
    s["pos"] = s["pos"] * scale
    s["origin"] = 0.5 * s["box"]
    F0, _ = check_vs_oracle(s)
    L = s["box"]
    rng = np.random.default_rng(4)
    shift = rng.integers(-3, 4, size=s["pos"].shape) * L
    F1, _, _ = evaluate(s, "clusters", pos=s["pos"] + shift)
    assert rms_rel(F1, F0) <= 1e-5


def test_forces_only_launch_equals_energy_launch(medium):
    """Forces of a forces-only device evaluation equal those of an energy
    evaluation bit for bit (the same lists and sums)."""
    import torch
    topo = PeriodicTopology.from_dict(medium)
    f = NonbondedCutoffB200SystemForce(medium["ron"], medium["rc_lj"], medium["rc_coul"],
                                       medium["rc_alg"], precision="mixed")
    f.set_pair_kernel("clusters")
    pos = torch.tensor(medium["pos"], dtype=torch.float64, device="cuda:0")
    fa = torch.zeros_like(pos)
    fb = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device="cuda:0")
    st = torch.cuda.current_stream().cuda_stream
    f.evaluate_device(topo, pos.data_ptr(), fa.data_ptr(), out.data_ptr(), _lib.PMB200_ENERGY, st)
    f.evaluate_device(topo, pos.data_ptr(), fb.data_ptr(), None, 0, st)
    torch.cuda.synchronize()
    f.sync()
    f.close()
    assert torch.equal(fa, fb)


def test_device_steps_follow_search_kernel(medium):
    """Five graph-replayed leapfrog steps with SETTLE: the trajectory stays
    within FP32 rounding of the search kernel's."""
    import torch
    topo = PeriodicTopology.from_dict(medium)
    widx = water.rigid_waters(medium)
    stream = torch.cuda.Stream()
    res = {}
    for kern in ("clusters", "search"):
        f = NonbondedCutoffB200SystemForce(medium["ron"], medium["rc_lj"], medium["rc_coul"],
                                           medium["rc_alg"], precision="mixed")
        f.set_rigid_waters(topo, widx, water.D_OH, water.D_HH)
        f.set_pair_kernel(kern)
        pos = torch.tensor(medium["pos"], dtype=torch.float64, device="cuda:0")
        vel = torch.tensor(medium["vel"], dtype=torch.float64, device="cuda:0")
        frc = torch.zeros_like(pos)
        out = torch.zeros(20, dtype=torch.float64, device="cuda:0")
        torch.cuda.synchronize()
        st = stream.cuda_stream
        f.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(),
                          _lib.PMB200_ENERGY, st)
        for _ in range(5):
            f.step_device(topo, pos.data_ptr(), vel.data_ptr(), frc.data_ptr(), 1.0, st,
                          out_ptr=out.data_ptr(), flags=_lib.PMB200_ENERGY)
        stream.synchronize()
        torch.cuda.synchronize()
        f.sync()
        res[kern] = (pos.cpu().numpy(), frc.cpu().numpy(), out.cpu().numpy())
        f.close()
    pc, fc, oc = res["clusters"]
    ps, fs, os_ = res["search"]
    assert np.abs(pc - ps).max() <= 1e-6
    assert rms_rel(fc, fs) <= 1e-5
    assert abs(oc[0] - os_[0]) <= 1e-6 * abs(os_[0])


def test_configurations_left_to_search_kernel(water648, modified648):
    """A box too small for five columns across the cutoff, and a topology with
    modified pairs, run on the search kernel: the results equal its own."""
    for d in (water648, modified648):
        Fc, Ec, _ = evaluate(d, "clusters")
        Fs, Es, _ = evaluate(d, "search")
        assert np.array_equal(Fc, Fs) and Ec[0] == Es[0] and Ec[1] == Es[1]


def test_autotune_may_choose_it(medium):
    import torch
    topo = PeriodicTopology.from_dict(medium)
    f = NonbondedCutoffB200SystemForce(medium["ron"], medium["rc_lj"], medium["rc_coul"],
                                       medium["rc_alg"], precision="mixed")
    pos = torch.tensor(medium["pos"], dtype=torch.float64, device="cuda:0")
    choice = f.autotune(topo, pos.data_ptr(), reps=3)
    assert choice["kernel_energy"] in ("search", "tiles", "clusters")
    fo, eo, _, _ = O.restate_eval(medium, medium["pos"], virial_mode=0)
    F = np.zeros_like(medium["pos"])
    E = ScalarStructure()
    f.evaluate(topo, medium["pos"], F, E)
    f.close()
    assert rms_rel(F, fo) <= 1e-5
    assert abs(E[0] - eo[0]) <= 1e-6 * abs(eo[0])


def test_dense_system_reports_list_overflow():
    """Atoms packed ~5x denser than water: a supercluster's list outgrows its
    buffer, the list kernel stops writing at the bound and flags it, and the
    evaluation reports PMB200_EDEVICE; the search kernel then serves the same
    context."""
    from protomoladdon_b200._lib import PmbError
    s = water.water_box(16, rc=10.0, ron=9.0, seed=5)
    scale = 0.6
    s["pos"] = s["pos"] * scale
    s["box"] = s["box"] * scale
    s["origin"] = s["origin"] * scale
    topo = PeriodicTopology.from_dict(s)
    f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                       precision="mixed")
    f.set_pair_kernel("clusters")
    F = np.zeros_like(s["pos"])
    E = ScalarStructure()
    with pytest.raises(PmbError) as ei:
        f.evaluate(topo, s["pos"], F, E)
    assert ei.value.code == _lib.PMB200_EDEVICE and "supercluster kernel" in str(ei.value)
    f.set_pair_kernel("search")
    F = np.zeros_like(s["pos"])
    E = ScalarStructure()
    f.evaluate(topo, s["pos"], F, E)
    f.close()
    fo, eo, _, _ = O.restate_eval(s, s["pos"], virial_mode=0)
    assert rms_rel(F, fo) <= 1e-5
