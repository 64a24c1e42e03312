"""Rotation helpers used by the emitter (genesis/utils/geom.py), numpy, one frame at a time."""

from __future__ import annotations

import numpy as np

from . import _globals


def normalize(v):
    v = np.asarray(v, dtype=np.float64)
    return v / np.linalg.norm(v)


def z_up_to_R(z):
    """Rotation whose z column is the unit vector along z; x is horizontal (utils/geom.py:1194-1240,
    no `up` argument): x = (z_y, -z_x, 0) unless z is vertical, then x = (z_z, 0, -z_x)."""
    eps = _globals.EPS
    z = np.array(z, dtype=np.float64)
    n = np.linalg.norm(z)
    z = z / n if n > eps else np.array([0.0, 1.0, 0.0])
    if abs(z[2]) < 1.0 - eps:
        x = np.array([z[1], -z[0], 0.0])
    else:
        x = np.array([z[2], 0.0, -z[0]])
    xn = np.linalg.norm(x)
    R = np.empty((3, 3))
    R[:, 2] = z
    if xn > eps:
        x = x / xn
        R[:, 0] = x
        R[:, 1] = np.cross(z, x)
    else:
        R[:] = np.eye(3)
    return R


def axis_angle_to_R(axis, theta):
    """Rotation about `axis` by theta, built from cos(theta) with sin = sqrt(1 - cos^2)
    as utils/geom.py:1430-1467 does (so theta and -theta give the same matrix)."""
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.sqrt(np.sum(axis * axis))
    c = float(np.cos(theta))
    s = np.sqrt(1.0 - c * c)
    c1 = (1.0 - c) * axis
    sa = s * axis
    R = np.empty((3, 3))
    R[0, 1] = c1[0] * axis[1] - sa[2]
    R[1, 0] = c1[0] * axis[1] + sa[2]
    R[0, 2] = c1[0] * axis[2] + sa[1]
    R[2, 0] = c1[0] * axis[2] - sa[1]
    R[1, 2] = c1[1] * axis[2] - sa[0]
    R[2, 1] = c1[1] * axis[2] + sa[0]
    d = c1 * axis + c
    R[0, 0], R[1, 1], R[2, 2] = d
    return R


def transform_by_trans_R(pos, trans, R):
    """R @ p + trans for each row p of pos (utils/geom.py:1101-1148)."""
    return np.asarray(pos, dtype=np.float64) @ np.asarray(R).T + np.asarray(trans, dtype=np.float64)
