"""Parameter choice (expansion order P, MAC theta, leaf size ncrit) for a
requested relative-L2 potential tolerance.

``choose_params`` returns the setting a run should use and where it came
from.  The plain FP64 form uses the reference's fixed theta = 0.4 and
ncrit = 64 and raises P until the tolerance is met (measured on the
sphere-surface workload: P=10 -> 1.6e-5, P=12 -> 4.0e-6, P=14 -> 1.3e-6,
P=16 -> 7.5e-7).  The fixed fallback is the reference's default setting.
"""
from __future__ import annotations

FIXED = {"P": 10, "theta": 0.4, "ncrit": 64}

# (tol upper bound, P) for the plain form at theta=0.4, ncrit=64
_FP64_P_BY_TOL = [(1e-4, 8), (2e-5, 10), (5e-6, 12), (1.5e-6, 14), (0.0, 16)]
# mixed form before the learned chooser: the cheapest measured setting per tolerance
_MIXED_TABLE = [(1e-4, {"P": 8, "theta": 0.4, "ncrit": 64}),
                (2e-5, {"P": 10, "theta": 0.4, "ncrit": 64}),
                (0.0, {"P": 10, "theta": 0.3, "ncrit": 64})]


def choose_params(n: int, tol: float, precision: str = "mixed", features=None) -> dict:
    if precision == "fp64":
        for bound, P in _FP64_P_BY_TOL:
            if tol >= bound:
                return {"P": P, "theta": 0.4, "ncrit": 64, "source": "fixed-theta P rule"}
    for bound, prm in _MIXED_TABLE:
        if tol >= bound:
            return dict(prm, source="table")
    return dict(FIXED, source="fixed")
