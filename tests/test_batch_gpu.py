"""Batched evaluation (pmb200_batch_*) against the same systems evaluated one
by one through their own contexts, and against the CPU oracle.

Tolerances (written here, checked below):
* schedule parts = 4: forces bit-identical to the single-system mixed path
  of an energy evaluation, which splits each cell's stencil four ways too
  (same cells, same stencil order and split, same staging, integer force
  sums); energies within 1e-12 relative (the partial sums are added in a
  different order); pair counts equal.
* other schedules: forces within 1e-6 RMS relative of that (the FP32 i-force
  partial sums group differently); energies within 1e-6 relative or 2e-3
  kcal/mol (the per-atom FP32 Coulomb sums are split across tasks; the same
  bound the single-system tests use on boxes of this size).
* against the FP64 oracle: forces RMS relative <= 1e-5.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from protomoladdon_b200 import _lib, water
from protomoladdon_b200.batch import SystemBatch
from protomoladdon_b200.force import (EwaldRealB200SystemForce, NonbondedCutoffB200SystemForce,
                                      PeriodicTopology)

pytestmark = pytest.mark.gpu


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.fixture(scope="module")
def boxes():
    return water.batch_boxes(count=14, seed=99)


def single(s, topo, force):
    pos = torch.tensor(s["pos"], dtype=torch.float64, device="cuda")
    frc = torch.zeros_like(pos)
    out = torch.zeros(20, dtype=torch.float64, device="cuda")
    force.evaluate_device(topo, pos.data_ptr(), frc.data_ptr(), out.data_ptr(),
                          _lib.PMB200_ENERGY | _lib.PMB200_VIRIAL, None)
    force.sync()
    return frc.cpu().numpy(), out.cpu().numpy(), force.last_pair_count()


def make_members(boxes, kind="cutoff"):
    mem = []
    for s in boxes:
        t = PeriodicTopology.from_dict(s)
        if kind == "cutoff":
            f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"])
        else:
            f = EwaldRealB200SystemForce(0.35, float(np.exp(-(0.35 * 9.0) ** 2)))
        mem.append((f, t))
    return mem


def batch_eval(batch, boxes, flags=_lib.PMB200_ENERGY | _lib.PMB200_VIRIAL, stream=None,
               times=1):
    pos = torch.tensor(np.concatenate([s["pos"] for s in boxes]), dtype=torch.float64,
                       device="cuda")
    frc = torch.zeros_like(pos)
    out = torch.zeros((len(boxes), 20), dtype=torch.float64, device="cuda")
    for _ in range(times):
        batch.eval_device(pos.data_ptr(), frc.data_ptr(), out.data_ptr(), flags, stream)
    batch.sync()  # raises on a device-side error
    torch.cuda.synchronize()
    return frc.cpu().numpy(), out.cpu().numpy()


@pytest.mark.parametrize("kind", ["cutoff", "ewald"])
def test_batch_equals_one_by_one(boxes, kind):
    mem = make_members(boxes, kind)
    ref = [single(s, t, f) for s, (f, t) in zip(boxes, mem)]
    b = SystemBatch(mem)
    b.set_schedule(parts=4, order=1)
    F, out = batch_eval(b, boxes)
    counts = b.pair_counts()
    off = b.offsets
    for k, (fr, er, pr) in enumerate(ref):
        fb = F[off[k]:off[k + 1]]
        assert np.array_equal(fb, fr), k
        assert np.allclose(out[k, :11], er[:11], rtol=1e-12, atol=1e-12 * np.abs(er[:11]).max())
        assert counts[k] == pr
    # every other schedule: same physics
    for parts, order in ((1, 0), (2, 0), (8, 1), (3, 0)):
        b.set_schedule(parts=parts, order=order, blocks_per_sm=1)
        F2, out2 = batch_eval(b, boxes)
        assert rms_rel(F2, F) <= 1e-6, (parts, order)
        assert np.allclose(out2[:, :2], out[:, :2], rtol=1e-6, atol=2e-3), (parts, order)
    b.close()
    for f, _ in mem:
        f.close()


def test_batch_against_oracle(boxes):
    mem = make_members(boxes)
    b = SystemBatch(mem)
    F, out = batch_eval(b, boxes)
    for k in (0, 5, 13):
        s = boxes[k]
        fo, eo, _, _ = O.restate_eval(s, s["pos"], virial_mode=0)
        assert rms_rel(F[b.offsets[k]:b.offsets[k + 1]], fo) <= 1e-5
        assert abs(out[k, 1] - eo[1]) <= 1e-5 * max(1.0, abs(eo[1]))
    b.close()


def test_graph_replay_and_autotune(boxes):
    mem = make_members(boxes)
    b = SystemBatch(mem)
    F1, out1 = batch_eval(b, boxes, flags=0)
    st = torch.cuda.Stream()
    F2, _ = batch_eval(b, boxes, flags=0, stream=st.cuda_stream, times=3)  # captured once
    assert rms_rel(F2, 3 * F1) <= 1e-12
    pos = torch.tensor(np.concatenate([s["pos"] for s in boxes]), dtype=torch.float64,
                       device="cuda")
    best = b.autotune(pos.data_ptr(), st.cuda_stream, reps=2)
    assert best["parts"] in (1, 2, 4, 8) and best["order"] in (0, 1) and best["pair_kernel_ms"] > 0
    assert b.schedule()["parts"] == best["parts"]
    F3, _ = batch_eval(b, boxes, flags=0)
    assert rms_rel(F3, F1) <= 1e-6
    b.close()


def test_batch_rejects_mixed_kinds_and_fp64(boxes):
    from protomoladdon_b200._lib import PmbError
    a = make_members(boxes[:2])
    e = make_members(boxes[2:3], "ewald")
    with pytest.raises(PmbError):
        SystemBatch(a + e)
    s = boxes[0]
    f64 = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"],
                                         precision="fp64")
    with pytest.raises(PmbError) as ei:
        SystemBatch([(f64, PeriodicTopology.from_dict(s))])
    assert ei.value.code == _lib.PMB200_EUNSUPPORTED


def test_batch_reports_non_finite_positions(boxes):
    from protomoladdon_b200._lib import PmbError
    mem = make_members(boxes[:3])
    b = SystemBatch(mem)
    pos = torch.tensor(np.concatenate([s["pos"] for s in boxes[:3]]), dtype=torch.float64,
                       device="cuda")
    pos[5, 1] = float("nan")
    frc = torch.zeros_like(pos)
    b.eval_device(pos.data_ptr(), frc.data_ptr(), None, 0, None)
    with pytest.raises(PmbError) as ei:
        b.sync()
    assert ei.value.code == _lib.PMB200_EDEVICE
    b.sync()  # the flag is cleared once reported
    b.close()
