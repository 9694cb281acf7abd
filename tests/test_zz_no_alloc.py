"""pmb200_eval_noalloc: the evaluation for callers that cannot allocate
device memory (hosts whose own pool allocator owns all device memory, or
that must not hit cudaFree's device synchronisation mid-step).  It keeps its
scratch in one static device array inside libpmb200, so it is checked here
against the regular allocating entry point on the same inputs, twice in a
row (the array keeps the previous call's contents, so the second call shows
that everything that must start at zero is cleared).  This file is collected
last on purpose."""
import ctypes

import numpy as np
import pytest

from protomoladdon_b200 import _lib, water
from protomoladdon_b200.force import (NonbondedCutoffB200SystemForce, PeriodicTopology,
                                      ScalarStructure)

pytestmark = pytest.mark.gpu
MAX_ATOMS = 32768  # the static scratch's stated limit


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


def call_noalloc(s, dev_arrays, forces, energy):
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
        P(box.ctypes.data), P(org.ctypes.data), P(forces.data_ptr()), P(energy.data_ptr()),
        P(torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    return rc


@pytest.mark.parametrize("system", ["water648", "modified"])
def test_noalloc_matches_allocating_path_twice(system):
    import torch
    s = water.small_648()
    if system == "modified":  # 1-4 style pairs and a Coulomb scaling factor
        ex = s["excl"].copy()
        ex[s["type"][ex[:, 0]] == water.T_O, 2] = 1
        s["excl"] = ex
        s["coulomb_scaling"] = 0.5
    n = s["type"].size
    topo = PeriodicTopology.from_dict(s)
    f = NonbondedCutoffB200SystemForce(s["ron"], s["rc_lj"], s["rc_coul"], s["rc_alg"])
    F_ref = np.zeros_like(s["pos"])
    E_ref = ScalarStructure()
    f.evaluate(topo, s["pos"], F_ref, E_ref)
    f.close()

    dev = torch.device("cuda:0")
    exs, exl = exclusion_lists(n, s["excl"])
    arrays = (torch.tensor(s["pos"], dtype=torch.float64, device=dev),
              torch.tensor(s["type"], dtype=torch.int32, device=dev),
              torch.tensor(s["qscaled"], dtype=torch.float64, device=dev),
              torch.tensor(s["mol"], dtype=torch.int32, device=dev),
              torch.tensor(exs, dtype=torch.int32, device=dev),
              torch.tensor(exl, dtype=torch.int32, device=dev))
    for _ in range(2):  # two calls in a row share the static scratch
        forces = torch.full((n, 3), 7.0, dtype=torch.float64, device=dev)  # overwritten
        energy = torch.zeros(20, dtype=torch.float64, device=dev)
        assert call_noalloc(s, arrays, forces, energy) == _lib.PMB200_OK
        F = forces.cpu().numpy()
        E = energy.cpu().numpy()
        # the mixed-precision tolerance used throughout the GPU tests
        assert np.sqrt(((F - F_ref) ** 2).sum() / (F_ref ** 2).sum()) <= 1e-5
        assert abs(E[0] - E_ref[0]) <= 2e-3 and abs(E[1] - E_ref[1]) <= 2e-3


def test_noalloc_rejects_sizes_beyond_its_scratch():
    s = water.small_648()
    L = _lib.lib()
    lj = np.ascontiguousarray(s["lj"]).reshape(-1)
    box = np.ascontiguousarray(s["box"])
    org = np.ascontiguousarray(s["origin"])
    P = ctypes.c_void_p
    dummy = P(16)  # never dereferenced: the size check comes first
    rc = L.pmb200_eval_noalloc(ctypes.byref(params(s)), MAX_ATOMS + 1, dummy, dummy, dummy,
                               dummy, dummy, dummy, 2, P(lj.ctypes.data), 1.0,
                               P(box.ctypes.data), P(org.ctypes.data), dummy, None, None)
    assert rc == _lib.PMB200_ENOMEM
