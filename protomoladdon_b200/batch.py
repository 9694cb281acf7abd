"""Batches of independent periodic systems on one GPU (pmb200_batch_*).

``SystemBatch(forces_and_topologies)`` builds one batch from per-system
forces (NonbondedCutoffB200SystemForce or EwaldRealB200SystemForce, mixed
precision) after each has seen its topology; ``eval_device`` evaluates all of
them with one persistent pair launch (a CUDA-graph replay when a stream is
given); ``autotune`` picks the schedule (stencil parts per cell, task order,
blocks per SM) by timing the candidates.  Positions and forces are the
systems' (n_s, 3) arrays back to back in system order.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import PmbError

_P = ctypes.c_void_p


class SystemBatch:
    def __init__(self, members):
        """members: list of (force, topology) pairs; the forces are created
        on the device here if needed and stay owned by the caller."""
        self.members = list(members)
        for f, t in self.members:
            f._ensure(t)
        arr = (_P * len(self.members))(*[f._ctx for f, _ in self.members])
        h = _P()
        rc = _lib.lib().pmb200_batch_create(arr, len(self.members), ctypes.byref(h))
        if rc != _lib.PMB200_OK:
            raise PmbError(rc, "pmb200_batch_create failed")
        self._b = h
        self.sizes = np.array([t.n for _, t in self.members], dtype=np.int64)
        self.offsets = np.concatenate([[0], np.cumsum(self.sizes)])

    @property
    def n_atoms(self):
        return int(self.offsets[-1])

    def _check(self, rc):
        if rc != _lib.PMB200_OK:
            msg = _lib.lib().pmb200_batch_last_error(self._b) if self._b else b""
            raise PmbError(rc, (msg or b"").decode())

    def eval_device(self, pos_ptr, force_ptr, out_ptr=None, flags=0, stream=None):
        self._check(_lib.lib().pmb200_batch_eval_device(
            self._b, _P(pos_ptr), _P(force_ptr), _P(out_ptr) if out_ptr else None, int(flags),
            _P(stream) if stream else None))

    def sync(self, stream=None):
        """Waits for the stream (None: the device) and raises PmbError for a
        device-side error of the batch's evaluations."""
        self._check(_lib.lib().pmb200_batch_sync(self._b, _P(stream) if stream else None))

    def set_schedule(self, parts=1, order=1, blocks_per_sm=0):
        self._check(_lib.lib().pmb200_batch_set_schedule(self._b, parts, order, blocks_per_sm))

    def schedule(self):
        s = (ctypes.c_int * 4)()
        self._check(_lib.lib().pmb200_batch_get_schedule(self._b, s))
        return {"parts": s[0], "order": s[1], "blocks_per_sm": s[2], "tasks": s[3]}

    def autotune(self, pos_ptr, stream=None, reps=5):
        s = (ctypes.c_int * 4)()
        ms = ctypes.c_float()
        self._check(_lib.lib().pmb200_batch_autotune(self._b, _P(pos_ptr),
                                                     _P(stream) if stream else None, int(reps),
                                                     s, ctypes.byref(ms)))
        return {"parts": s[0], "order": s[1], "blocks_per_sm": s[2], "tasks": s[3],
                "pair_kernel_ms": ms.value}

    def set_kernel_timing(self, on):
        self._check(_lib.lib().pmb200_batch_set_kernel_timing(self._b, 1 if on else 0))

    def last_kernel_ms(self):
        v = ctypes.c_float()
        self._check(_lib.lib().pmb200_batch_last_kernel_ms(self._b, ctypes.byref(v)))
        return float(v.value)

    def pair_counts(self):
        v = (ctypes.c_longlong * len(self.members))()
        self._check(_lib.lib().pmb200_batch_pair_counts(self._b, v))
        return np.array(v[:], dtype=np.int64)

    def close(self):
        if self._b is not None:
            _lib.lib().pmb200_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
