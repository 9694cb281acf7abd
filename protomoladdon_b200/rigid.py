"""Host-side rigid-water integrator pieces (numpy, FP64).

``settle`` is SETTLE (Miyamoto & Kollman, J. Comput. Chem. 13, 952 (1992))
vectorised over waters: it puts 3-site waters back on their O-H / H-H
lengths after an unconstrained drift, the role ProtoMol's SHAKE position
modifier plays in its leapfrog (protomol/src/protomol/modifier/
ModifierShake.cpp).  The device integrator runs the same algorithm in
libpmb200 (k_kick_drift_settle); this copy serves host integrators that call
the force through the host-buffer C ABI.
"""
from __future__ import annotations

import numpy as np

INV_TIMEFACTOR = 0.02045482828087295  # ProtoMol Constant::INV_TIMEFACTOR


def settle(widx, mass, d_oh, d_hh, old_pos, new_pos):
    """Constrains new_pos (n,3, modified in place) given constrained old_pos."""
    w = np.asarray(widx).reshape(-1, 3)
    if w.size == 0:
        return new_pos
    mo, mh = float(mass[w[0, 0]]), float(mass[w[0, 1]])
    M = mo + 2.0 * mh
    rc = 0.5 * d_hh
    t = np.sqrt(d_oh * d_oh - rc * rc)
    ra = 2.0 * mh * t / M
    rb = t - ra
    A0, B0, C0 = old_pos[w[:, 0]], old_pos[w[:, 1]], old_pos[w[:, 2]]
    A1, B1, C1 = new_pos[w[:, 0]], new_pos[w[:, 1]], new_pos[w[:, 2]]
    com = (mo * A1 + mh * B1 + mh * C1) / M
    a1, b1, c1 = A1 - com, B1 - com, C1 - com
    b0, c0 = B0 - A0, C0 - A0
    ez = np.cross(b0, c0)
    ex = np.cross(a1, ez)
    ey = np.cross(ez, ex)
    ex /= np.linalg.norm(ex, axis=1)[:, None]
    ey /= np.linalg.norm(ey, axis=1)[:, None]
    ez /= np.linalg.norm(ez, axis=1)[:, None]

    def d(u, v):
        return np.einsum("ij,ij->i", u, v)

    xb0, yb0, xc0, yc0 = d(ex, b0), d(ey, b0), d(ex, c0), d(ey, c0)
    za1 = d(ez, a1)
    xb1, yb1, zb1 = d(ex, b1), d(ey, b1), d(ez, b1)
    xc1, yc1, zc1 = d(ex, c1), d(ey, c1), d(ez, c1)
    sphi = za1 / ra
    cphi = np.sqrt(1.0 - sphi * sphi)
    spsi = (zb1 - zc1) / (2.0 * rc * cphi)
    cpsi = np.sqrt(1.0 - spsi * spsi)
    ya2 = ra * cphi
    xb2 = -rc * cpsi
    t1, t2 = -rb * cphi, rc * spsi * sphi
    yb2, yc2 = t1 - t2, t1 + t2
    al = xb2 * (xb0 - xc0) + yb0 * yb2 + yc0 * yc2
    be = xb2 * (yc0 - yb0) + xb0 * yb2 + xc0 * yc2
    ga = xb0 * yb1 - xb1 * yb0 + xc0 * yc1 - xc1 * yc0
    ab = al * al + be * be
    sth = (al * ga - be * np.sqrt(ab - ga * ga)) / ab
    cth = np.sqrt(1.0 - sth * sth)
    xa3, ya3, za3 = -ya2 * sth, ya2 * cth, za1
    xb3, yb3, zb3 = xb2 * cth - yb2 * sth, xb2 * sth + yb2 * cth, zb1
    xc3, yc3, zc3 = -xb2 * cth - yc2 * sth, -xb2 * sth + yc2 * cth, zc1

    def back(x, y, z):
        return com + x[:, None] * ex + y[:, None] * ey + z[:, None] * ez

    new_pos[w[:, 0]] = back(xa3, ya3, za3)
    new_pos[w[:, 1]] = back(xb3, yb3, zb3)
    new_pos[w[:, 2]] = back(xc3, yc3, zc3)
    return new_pos


def kick_drift_settle(pos, vel, forces, mass, dt_fs, widx, d_oh, d_hh, kick=1.0):
    """One leapfrog kick + drift with rigid waters, in place (ProtoMol's
    doKickdoDrift followed by the constraint modifier)."""
    h = dt_fs * INV_TIMEFACTOR
    old = pos.copy()
    vel += forces * (kick * h) / mass[:, None]
    pos += vel * h
    if len(widx):
        settle(widx, mass, d_oh, d_hh, old, pos)
        w = np.asarray(widx).reshape(-1)
        vel[w] = (pos[w] - old[w]) / h


def host_kick_drift(pos, vel, forces, mass, dt_fs, widx, d_oh, d_hh, kick=1.0,
                    clear_forces=False):
    """kick_drift_settle through libpmb200's native host helper
    (pmb200_host_kick_drift); arrays are C-contiguous float64, updated in place.
    clear_forces: zero ``forces`` once used (for the next evaluation to add into)."""
    import ctypes
    from . import _lib
    w = np.ascontiguousarray(widx, dtype=np.int32).reshape(-1)
    m = np.ascontiguousarray(mass, dtype=np.float64)
    P = ctypes.c_void_p
    rc = _lib.lib().pmb200_host_kick_drift(
        int(pos.shape[0]), P(pos.ctypes.data), P(vel.ctypes.data), P(forces.ctypes.data),
        P(m.ctypes.data), float(dt_fs), float(kick), w.size // 3,
        P(w.ctypes.data) if w.size else None, float(d_oh), float(d_hh), int(bool(clear_forces)))
    if rc:
        raise _lib.PmbError(rc, "pmb200_host_kick_drift")
