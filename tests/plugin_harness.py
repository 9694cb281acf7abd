"""ctypes front end of tests/plugin/_build/libplugin_harness.so (test only)."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "plugin", "_build", "libplugin_harness.so")
_P, _D, _I = ctypes.c_void_p, ctypes.c_double, ctypes.c_int


def available():
    return os.path.exists(SO)


def lib():
    from oracle import oracle as O
    O.ref_lib()  # libpmref.so first, with its symbols global
    L = ctypes.CDLL(SO, mode=ctypes.RTLD_GLOBAL)
    L.harness_eval.argtypes = [_P, _I, _I, _P, _D, _D, _D, _D, _P, _P, _P, _P]
    L.harness_eval.restype = _I
    L.harness_message.restype = ctypes.c_char_p
    L.harness_set_parallel.argtypes = [_I]
    L.harness_last_blocks.restype = ctypes.c_uint
    return L


def set_parallel(on):
    """Call the forces through SystemForce::parallelEvaluate (after
    Force::numberOfBlocks, as ForceGroup does) instead of evaluate."""
    lib().harness_set_parallel(1 if on else 0)


def last_blocks():
    return int(lib().harness_last_blocks())


def evaluate(ref_force, which, sysd, pos):
    """which: 0 reference prototype, 1 B200 plugin, 2 plugin under 'time'.
    Returns (rc, message, forces, energies, virial, molvirial)."""
    L = lib()
    p = np.ascontiguousarray(pos, dtype=np.float64)
    n = p.shape[0]
    f = np.zeros((n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    rc = L.harness_eval(ref_force.h, which, n, p.ctypes.data, float(sysd["ron"]),
                        float(sysd["rc_lj"]), float(sysd["rc_coul"]), float(sysd["rc_alg"]),
                        f.ctypes.data, e.ctypes.data, v.ctypes.data, mv.ctypes.data)
    return rc, L.harness_message().decode(), f, e, v, mv


def evaluate_ewald(ref_force, which, sysd, pos, alpha, accuracy):
    """The Ewald real-space term through the factory: which 0 reference
    prototype ("Coulomb -algorithm FullEwald -real"), 1 B200 plugin.
    Returns (rc, message, forces, energies, virial, molvirial)."""
    L = lib()
    L.harness_ewald_eval.argtypes = [_P, _I, _I, _P, _D, _D, _P, _P, _P, _P]
    L.harness_ewald_eval.restype = _I
    p = np.ascontiguousarray(pos, dtype=np.float64)
    n = p.shape[0]
    f = np.zeros((n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    rc = L.harness_ewald_eval(ref_force.h, which, n, p.ctypes.data, float(alpha),
                              float(accuracy), f.ctypes.data, e.ctypes.data, v.ctypes.data,
                              mv.ctypes.data)
    return rc, L.harness_message().decode(), f, e, v, mv


def evaluate_pair(ref_force, vacuum, force_id, values, pos):
    """A switch-policy force made by the factory from its config id and
    values: on the reference topology of ref_force (vacuum 0) or on a vacuum
    copy of it (1).  Returns (rc, message, forces, energies, virial,
    molvirial)."""
    L = lib()
    L.harness_pair_eval.argtypes = [_P, _I, ctypes.c_char_p, _I, _P, _I, _P, _P, _P, _P, _P]
    L.harness_pair_eval.restype = _I
    p = np.ascontiguousarray(pos, dtype=np.float64)
    n = p.shape[0]
    vals = np.ascontiguousarray(values, dtype=np.float64)
    f = np.zeros((n, 3))
    e = np.zeros(2)
    v = np.zeros(9)
    mv = np.zeros(9)
    rc = L.harness_pair_eval(ref_force.h, int(vacuum), force_id.encode(), vals.size,
                             vals.ctypes.data, n, p.ctypes.data, f.ctypes.data, e.ctypes.data,
                             v.ctypes.data, mv.ctypes.data)
    return rc, L.harness_message().decode(), f, e, v, mv
