"""Shared helpers of the test suite (not a test module)."""
import os

import numpy as np

from pe_b200 import scenes

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name):
    d = dict(np.load(os.path.join(GOLDEN, name + ".npz")))
    d["scene"] = scenes.scene_from_bytes(d["scene"].tobytes(), name=name)
    return d


def load_golden_arrays(name):
    """A golden file without a scene record (numbers only)."""
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def rel_err(a, b):
    """Norm-wise relative error max|a-b| / max|b| (0 when both vanish)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.abs(b).max() if b.size else 0.0
    num = np.abs(a - b).max() if b.size else 0.0
    if den == 0.0:
        return float(num)
    return float(num / den)


def pair_set(ids):
    ids = np.asarray(ids).reshape(-1, 2)
    return set(map(tuple, ids.tolist()))


GOLDEN_NAMES = ["small64_boxes", "small64_planes", "lattice512", "dense512", "loose125_planes",
                "loose125_boxes"]
CONVERGED_NAMES = ["loose125_planes", "loose125_boxes"]


def rel_err_w(w, w_ref, v_ref, r):
    """Error of angular velocities relative to the surface-speed scale max(|w_ref|, |v_ref|/r_min).

    Centred contacts produce torques only through rounding (r x f with r parallel to f), so an
    angular velocity can be pure round-off; its error is measured against the velocity scale."""
    scale = max(float(np.abs(w_ref).max(initial=0.0)),
                float(np.abs(v_ref).max(initial=0.0)) / float(np.min(r)))
    if scale == 0.0:
        return float(np.abs(np.asarray(w) - w_ref).max(initial=0.0))
    return float(np.abs(np.asarray(w) - w_ref).max(initial=0.0) / scale)
