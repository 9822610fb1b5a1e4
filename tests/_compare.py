"""Comparison helpers for per-particle fields."""
import numpy as np


def field_error(got: np.ndarray, ref: np.ndarray, floor_frac: float = 1e-3) -> float:
    """Max over particles of |got - ref| / max(|ref|, floor), with floor = floor_frac * max|ref| over
    the field (vector fields: per-particle norm of the difference over the norm of the value).
    floor_frac = 0 is the plain per-particle relative error: where the reference value is exactly
    zero the compared value must be exactly zero too (otherwise the error is infinite)."""
    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    if ref.size == 0:
        return 0.0
    if ref.ndim == 2:
        diff = np.linalg.norm(got - ref, axis=1)
        mag = np.linalg.norm(ref, axis=1)
    else:
        diff = np.abs(got - ref)
        mag = np.abs(ref)
    if floor_frac == 0.0:
        zero = mag == 0.0
        if np.any(diff[zero] != 0.0):
            return float("inf")
        return float(np.max(diff[~zero] / mag[~zero])) if np.any(~zero) else 0.0
    floor = max(floor_frac * float(mag.max()), 1e-300)
    return float(np.max(diff / np.maximum(mag, floor)))


def assert_field(name: str, got, ref, rtol: float, floor_frac: float = 1e-3):
    err = field_error(got, ref, floor_frac)
    assert err <= rtol, f"{name}: max relative error {err:.3e} > {rtol:.1e}"
    return err


def neighbor_sets(counts: np.ndarray, lists: np.ndarray):
    """List of (fluid_set, boundary_set) frozensets per particle."""
    out = []
    for i in range(counts.shape[0]):
        nf, nb = int(counts[i, 0]), int(counts[i, 1])
        out.append((frozenset(lists[i, :nf].tolist()), frozenset(lists[i, nf:nf + nb].tolist())))
    return out
