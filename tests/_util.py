"""Helpers shared by the tests."""
import numpy as np


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if not (np.iscomplexobj(a) or np.iscomplexobj(b)):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / nb) if nb > 0 else float(np.linalg.norm(a - b))


def random_fields(shape, seed):
    """Seeded random E (V/m) and H (A/m) fields of vacuum-impedance ratio."""
    rng = np.random.default_rng(seed)
    return [rng.standard_normal(shape) * (1.0 if c < 3 else 1.0 / 376.73) for c in range(6)]
