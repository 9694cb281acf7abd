"""pmb200_eval_noalloc: the evaluation for callers that cannot allocate
device memory (hosts whose own pool allocator owns all device memory, or
that must not hit cudaFree's device synchronisation mid-step).  It keeps its
scratch in one static device array inside libpmb200, so it is checked here
against the regular allocating entry point and against the reference's own
forces and energies (committed fixtures) on the same inputs, twice in a row
(the array keeps the previous call's contents, so the second call shows that
everything that must start at zero is cleared), with and without energies.
The energy output is exactly two doubles: the test places it inside a larger
buffer and checks that the doubles after it are untouched.  A non-finite
position must come back as PMB200_EDEVICE through the status word.  This
file is collected last on purpose.

Tolerances: the mixed-precision ones of the other GPU tests -- forces RMS
relative <= 1e-5; energies within 2e-3 kcal/mol on these 648-atom boxes
(1e-6 of the summed pair magnitudes)."""
import ctypes

import numpy as np
import pytest

from protomoladdon_b200 import _lib
from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)

pytestmark = pytest.mark.gpu
MAX_ATOMS = 32768  # the static scratch's stated limit
SENTINEL = -12345.678


def exclusion_lists(n, excl):
    """Per-atom partner lists sorted by partner ({partner, kind} pairs), with
    later duplicates overriding earlier ones like ExclusionTable::add."""
    kinds = {}
    for a, b, k in np.asarray(excl).reshape(-1, 3):
        if a != b:
            kinds[(min(a, b), max(a, b))] = int(k)
    per = [[] for _ in range(n)]
    for (a, b), k in kinds.items():
        if k:
            per[a].append((b, k))
            per[b].append((a, k))
    start = np.zeros(n + 1, np.int32)
    flat = []
    for i in range(n):
        per[i].sort()
        start[i + 1] = start[i] + len(per[i])
        flat.extend(per[i])
    return start, np.asarray(flat or [(0, 0)], np.int32).reshape(-1, 2)


def params(s):
    return _lib.Params(_lib.PMB200_MIXED, 0, s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"], 0.0)


def device_arrays(s, pos=None):
    import torch
    dev = torch.device("cuda:0")
    n = int(s["type"].size)
    exs, exl = exclusion_lists(n, s["excl"])
    return (torch.tensor(s["pos"] if pos is None else pos, dtype=torch.float64, device=dev),
            torch.tensor(s["type"], dtype=torch.int32, device=dev),
            torch.tensor(s["qscaled"], dtype=torch.float64, device=dev),
            torch.tensor(s["mol"], dtype=torch.int32, device=dev),
            torch.tensor(exs, dtype=torch.int32, device=dev),
            torch.tensor(exl, dtype=torch.int32, device=dev))


def call_noalloc(s, dev_arrays, forces, energy, status):
    """One call through the C ABI; energy / status may be None (NULL)."""
    import torch
    L = _lib.lib()
    pos, typ, q, mol, exs, exl = dev_arrays
    lj = np.ascontiguousarray(s["lj"], dtype=np.float64).reshape(-1)
    box = np.ascontiguousarray(s["box"], dtype=np.float64)
    org = np.ascontiguousarray(s["origin"], dtype=np.float64)
    P = ctypes.c_void_p
    rc = L.pmb200_eval_noalloc(
        ctypes.byref(params(s)), int(s["type"].size), P(pos.data_ptr()), P(typ.data_ptr()),
        P(q.data_ptr()), P(mol.data_ptr()), P(exs.data_ptr()), P(exl.data_ptr()),
        int(s["lj"].shape[0]), P(lj.ctypes.data), float(s["coulomb_scaling"]),
        P(box.ctypes.data), P(org.ctypes.data), P(forces.data_ptr()),
        None if energy is None else P(energy.data_ptr()),
        None if status is None else P(status.data_ptr()),
        P(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc


def allocating_path(s):
    topo = PeriodicTopology.from_dict(s)
    f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"])
    F = np.zeros_like(s["pos"])
    E = ScalarStructure()
    f.evaluate(topo, s["pos"], F, E)
    f.close()
    return F, E


def rms_rel(a, b):
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))


@pytest.mark.parametrize("fx", ["water648", "modified648"])
def test_noalloc_matches_allocating_path_and_reference_twice(fx, request):
    import torch
    s = request.getfixturevalue(fx)
    n = int(s["type"].size)
    F_alloc, E_alloc = allocating_path(s)
    arrays = device_arrays(s)
    dev = arrays[0].device
    for _ in range(2):  # two calls in a row share the static scratch
        forces = torch.full((n, 3), 7.0, dtype=torch.float64, device=dev)  # overwritten
        # the two energies, then sentinels the call must not touch
        buf = torch.full((20,), SENTINEL, dtype=torch.float64, device=dev)
        status = torch.full((1,), -1, dtype=torch.int32, device=dev)
        assert call_noalloc(s, arrays, forces, buf, status) == _lib.PMB200_OK
        assert int(status.item()) == _lib.PMB200_OK
        F = forces.cpu().numpy()
        E = buf.cpu().numpy()
        assert np.all(E[2:] == SENTINEL), "energy output wrote past its two doubles"
        assert rms_rel(F, F_alloc) <= 1e-5
        assert abs(E[0] - E_alloc[0]) <= 2e-3 and abs(E[1] - E_alloc[1]) <= 2e-3
        assert rms_rel(F, s["ref_forces"]) <= 1e-5
        e = s["ref_energies"]
        assert abs(E[0] - e[0]) <= 2e-3 and abs(E[1] - e[1]) <= 2e-3


@pytest.mark.parametrize("fx", ["water648", "modified648"])
def test_noalloc_forces_only_twice(fx, request):
    import torch
    s = request.getfixturevalue(fx)
    n = int(s["type"].size)
    arrays = device_arrays(s)
    dev = arrays[0].device
    F_prev = None
    for _ in range(2):
        forces = torch.full((n, 3), -3.0, dtype=torch.float64, device=dev)
        status = torch.full((1,), -1, dtype=torch.int32, device=dev)
        assert call_noalloc(s, arrays, forces, None, status) == _lib.PMB200_OK
        assert int(status.item()) == _lib.PMB200_OK
        F = forces.cpu().numpy()
        assert rms_rel(F, s["ref_forces"]) <= 1e-5
        if F_prev is not None:  # integer force sums: the same bits every call
            assert np.array_equal(F, F_prev)
        F_prev = F


def test_noalloc_reports_non_finite_position(water648):
    import torch
    s = water648
    n = int(s["type"].size)
    pos = s["pos"].copy()
    pos[17, 1] = np.nan
    arrays = device_arrays(s, pos)
    dev = arrays[0].device
    forces = torch.zeros((n, 3), dtype=torch.float64, device=dev)
    buf = torch.full((20,), SENTINEL, dtype=torch.float64, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    assert call_noalloc(s, arrays, forces, buf, status) == _lib.PMB200_OK  # queued fine
    assert int(status.item()) == _lib.PMB200_EDEVICE
    assert np.all(buf.cpu().numpy()[2:] == SENTINEL)
    # the next clean call clears the error word again
    arrays = device_arrays(s)
    assert call_noalloc(s, arrays, forces, buf, status) == _lib.PMB200_OK
    assert int(status.item()) == _lib.PMB200_OK
    assert rms_rel(forces.cpu().numpy(), s["ref_forces"]) <= 1e-5


def test_noalloc_rejects_sizes_beyond_its_scratch(water648):
    s = water648
    L = _lib.lib()
    lj = np.ascontiguousarray(s["lj"]).reshape(-1)
    box = np.ascontiguousarray(s["box"])
    org = np.ascontiguousarray(s["origin"])
    P = ctypes.c_void_p
    dummy = P(16)  # never dereferenced: the size check comes first
    rc = L.pmb200_eval_noalloc(ctypes.byref(params(s)), MAX_ATOMS + 1, dummy, dummy, dummy,
                               dummy, dummy, dummy, 2, P(lj.ctypes.data), 1.0,
                               P(box.ctypes.data), P(org.ctypes.data), dummy, None, None, None)
    assert rc == _lib.PMB200_ENOMEM
    bad = lj.copy()
    bad[0] = np.inf  # a non-finite LJ entry is refused before anything is queued
    rc = L.pmb200_eval_noalloc(ctypes.byref(params(s)), 8, dummy, dummy, dummy,
                               dummy, dummy, dummy, 2, P(bad.ctypes.data), 1.0,
                               P(box.ctypes.data), P(org.ctypes.data), dummy, None, None, None)
    assert rc == _lib.PMB200_EINVAL
