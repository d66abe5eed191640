"""Accuracy metric of the reference's check (sample/exafmm-dev-13274dd4ac68/
include/verify.h:18-90, applied in examples/tapas_exafmm.cxx:369-381):
relative L2 errors of the potential and of the acceleration vector."""
from __future__ import annotations

import numpy as np


def rel_l2(approx: np.ndarray, ref: np.ndarray):
    dp = np.sum((approx[:, 0] - ref[:, 0]) ** 2)
    npot = np.sum(ref[:, 0] ** 2)
    da = np.sum((approx[:, 1:] - ref[:, 1:]) ** 2)
    na = np.sum(ref[:, 1:] ** 2)
    return float(np.sqrt(dp / npot)), float(np.sqrt(da / na))
