"""Field comparison metric of the reference's plotfile comparator
(py_utils/compare_fields_from_twoplotfiles.py:40-46): absolute error
RMS(f1 - f2) and relative error RMS(f1 - f2) / mean(|f1|), on raw arrays
(no yt dependency)."""
from __future__ import annotations

import numpy as np


def field_error(f1: np.ndarray, f2: np.ndarray) -> tuple[float, float]:
    f1 = np.asarray(f1, dtype=np.float64)
    f2 = np.asarray(f2, dtype=np.float64)
    err = float(np.sqrt(np.mean((f1 - f2) ** 2)))
    avg = float(np.mean(np.abs(f1)))
    return err, (err / avg if avg > 0 else (0.0 if err == 0 else np.inf))


def rel_l2(f1: np.ndarray, f2: np.ndarray) -> float:
    """Relative L2 error |f1 - f2|_2 / |f1|_2 (0 when both are 0)."""
    f1 = np.asarray(f1, dtype=np.float64)
    f2 = np.asarray(f2, dtype=np.float64)
    n = float(np.linalg.norm(f1))
    d = float(np.linalg.norm(f1 - f2))
    return d / n if n > 0 else d
