"""The large and batched benchmark systems themselves, through the C ABI,
against the FP64 CPU oracle on the same inputs.

* The 327,352-atom ion box (110,592 lattice sites, 2% Na+/Cl-, rc 12): the
  LJ(C2) + Coulomb(C1) mixed kernel and the real-space Ewald mixed kernel
  (alpha 0.30, rc 12), each against the oracle's restatement of the
  reference force.
* The 512 uneven boxes of the batched benchmark: the batch's forces match
  each system's own single-context evaluation, and a seeded sample of systems
  matches the oracle.

Tolerances (written here, checked below): forces RMS relative <= 1e-5 (the
mixed-precision bound); energies within 1e-6 of the sum over pairs of the
pair-energy magnitudes -- on these lattice-start boxes the Coulomb total
cancels to ~1e-4 of that sum, so a relative bound on the total would measure
the cancellation, not the kernel; the sum is n times its per-atom value,
measured by brute force on a 3,000-atom box of the same recipe and cutoff.
"""
import numpy as np
import pytest
import torch
from scipy.special import erfc

from oracle import oracle as O
from protomoladdon_b200 import _lib, water
from protomoladdon_b200.batch import SystemBatch
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology, ScalarStructure)

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


def abs_pair_energy_per_atom(d, form, alpha=0.0):
    """Per-atom sum over pairs within the cutoff of |E_LJ| + |E_Coulomb|
    (switched as the force switches them), brute force in numpy."""
    pos, q, box = d["pos"], d["qscaled"], np.asarray(d["box"], float)
    typ, lj = d["type"], np.asarray(d["lj"])
    rc, ron = d["rc_lj"], d["ron"]
    n = len(q)
    full = np.zeros((n, n), bool)
    for a, b, k in np.asarray(d["excl"]).reshape(-1, 3):
        if k == 2:
            full[a, b] = full[b, a] = True
    tot = 0.0
    for i in range(n - 1):
        dv = pos[i + 1:] - pos[i]
        dv -= box * np.rint(dv / box)
        r2 = (dv ** 2).sum(1)
        m = (r2 <= rc * rc) & ~full[i, i + 1:]
        r2 = r2[m]
        r = np.sqrt(r2)
        qq = q[i] * q[i + 1:][m]
        if form == "ewald":
            tot += np.abs(qq * erfc(alpha * r) / r).sum()
            continue
        A = lj[typ[i], typ[i + 1:][m], 0]
        B = lj[typ[i], typ[i + 1:][m], 1]
        r6 = 1.0 / r2 ** 3
        s2 = np.where(r2 <= ron * ron, 1.0,
                      (rc * rc - r2) ** 2 * (rc * rc + 2 * r2 - 3 * ron * ron)
                      / (rc * rc - ron * ron) ** 3)
        c1 = 1.0 - r * (1.5 / rc - 0.5 * r2 / rc ** 3)
        tot += np.abs((A * r6 * r6 - B * r6) * s2).sum() + np.abs(qq / r * c1).sum()
    return tot / n


@pytest.fixture(scope="module")
def large():
    return water.large_331k()


@pytest.fixture(scope="module")
def scale_box():
    # the same recipe and cutoff as the large box, small enough for n^2
    return water.water_box(10, rc=12.0, ron=11.0, seed=7, ion_fraction=0.02)


def eval_host(force, d):
    topo = PeriodicTopology.from_dict(d)
    F = np.zeros_like(d["pos"])
    E = ScalarStructure()
    force.evaluate(topo, d["pos"], F, E)
    pairs = force.last_pair_count()
    force.close()
    return F, E, pairs


def test_large_box_lj_c1_mixed_vs_oracle(large, scale_box):
    s = large
    F, E, pairs = eval_host(
        NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"]), s)
    fo, eo, _, _ = O.restate_eval(s, s["pos"], virial_mode=0)
    assert rms_rel(F, fo) <= 1e-5
    bound = 1e-6 * abs_pair_energy_per_atom(scale_box, "cutoff") * s["n"]
    assert abs(E[0] - eo[0]) <= bound
    assert abs(E[1] - eo[1]) <= bound
    # the pair set is the oracle's up to FP32 ties at the cutoff
    po = O.restate_count_pairs(s, s["pos"])
    assert abs(pairs - po) <= 1e-6 * po


def test_large_box_ewald_mixed_vs_oracle(large, scale_box):
    s = large
    acc = float(np.exp(-(0.30 * 12.0) ** 2))  # rc = 12 A
    F, E, _ = eval_host(EwaldRealB200SystemForce(0.30, acc), s)
    fo, eo, _, _ = O.restate_ewald_real(s, s["pos"], 0.30, acc, False, virial_mode=0)
    assert rms_rel(F, fo) <= 1e-5
    bound = 1e-6 * abs_pair_energy_per_atom(scale_box, "ewald", 0.30) * s["n"]
    assert abs(E[0] - eo) <= bound


@pytest.fixture(scope="module")
def batch512():
    return water.batch_boxes(count=512, seed=1234)


def test_batch_of_512_boxes_equals_single_contexts_and_oracle(batch512):
    boxes = batch512
    mem = []
    for s in boxes:
        mem.append((NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"],
                                                   s["rc_alg"]), PeriodicTopology.from_dict(s)))
    b = SystemBatch(mem)
    b.set_schedule(parts=4, order=1)
    pos = torch.tensor(np.concatenate([s["pos"] for s in boxes]), dtype=torch.float64,
                       device="cuda")
    frc = torch.zeros_like(pos)
    out = torch.zeros((len(boxes), 20), dtype=torch.float64, device="cuda")
    b.eval_device(pos.data_ptr(), frc.data_ptr(), out.data_ptr(), _lib.PMB200_ENERGY, None)
    b.sync()
    torch.cuda.synchronize()
    F = frc.cpu().numpy()
    out = out.cpu().numpy()
    counts = b.pair_counts()
    off = b.offsets
    for k, (s, (f, t)) in enumerate(zip(boxes, mem)):
        p = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
        fr = torch.zeros_like(p)
        o = torch.zeros(20, dtype=torch.float64, device="cuda")
        f.evaluate_device(t, p.data_ptr(), fr.data_ptr(), o.data_ptr(), _lib.PMB200_ENERGY, None)
        f.sync()
        assert np.array_equal(F[off[k]:off[k + 1]], fr.cpu().numpy()), k
        e = o.cpu().numpy()
        # the per-warp FP64 partial sums are added in another order (per
        # system in the batch); the Coulomb total cancels to ~1e-4 of its
        # terms, so the bound is 1e-12 of their scale (~1e4 x the total)
        assert np.allclose(out[k, :2], e[:2], rtol=0, atol=1e-8 * np.abs(e[:2]).max()), k
        assert counts[k] == f.last_pair_count(), k
    # a seeded sample against the FP64 oracle
    rng = np.random.default_rng(512)
    for k in rng.choice(len(boxes), size=8, replace=False):
        s = boxes[k]
        fo, eo, _, _ = O.restate_eval(s, s["pos"], virial_mode=0)
        assert rms_rel(F[off[k]:off[k + 1]], fo) <= 1e-5, k
        assert abs(out[k, 1] - eo[1]) <= 1e-5 * max(1.0, abs(eo[1])), k
        assert abs(out[k, 0] - eo[0]) <= 2e-3 * max(1.0, s["n"] / 648), k
    b.close()
    for f, _ in mem:
        f.close()
