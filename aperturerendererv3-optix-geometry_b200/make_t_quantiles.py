"""Generates csrc/t_quantile_table.h: the 0.9975 quantile of Student's t
distribution (two-sided level 0.005) for 1..1024 degrees of freedom, rounded to
float32, and for each the smallest float whose square root reaches it -- the table the denoiser's Welch t-test reads (the reference's
LookupTQuantile005, core/denoise/t_quantile.cuh:15-27, holds the same values;
tests/test_cpu_denoise.py checks them against a fixture of that table).

    python make_t_quantiles.py      (needs scipy; the header is committed)
"""
import os

import numpy as np
from scipy import stats

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "csrc", "t_quantile_table.h")


def table() -> np.ndarray:
    return stats.t.ppf(0.9975, np.arange(1, 1025)).astype(np.float32)


def sqrt_thresholds(q: np.ndarray) -> np.ndarray:
    """For each quantile q, the smallest float32 x with sqrtf(x) >= q (IEEE
    square root, correctly rounded): for x >= 0, sqrtf(x) < q exactly when
    x < threshold."""
    out = np.empty_like(q)
    for k, t in enumerate(q):
        x = np.float32(t) * np.float32(t)
        while np.sqrt(x) >= t:
            x = np.nextafter(x, np.float32(0))
        while np.sqrt(x) < t:
            x = np.nextafter(x, np.float32(np.inf))
        out[k] = x
    return out


def main() -> None:
    vals = table()
    thr = sqrt_thresholds(vals)
    lines = ["// Generated by make_t_quantiles.py: Student t quantile 0.9975 for nu = 1..1024 (float32).",
             "#pragma once", "", "namespace ar {", "", "constexpr int kTQuantiles = 1024;",
             "static __device__ const float kTQuantile005[kTQuantiles] = {"]
    for k in range(0, len(vals), 6):
        lines.append("    " + " ".join(f"{float(v).hex()}f," for v in vals[k:k + 6]))
    lines += ["};", "", "// smallest x with sqrtf(x) >= kTQuantile005[k]: sqrtf(x) < q  <=>  0 <= x < threshold",
              "static __device__ const float kTQuantileSqrtThreshold[kTQuantiles] = {"]
    for k in range(0, len(thr), 6):
        lines.append("    " + " ".join(f"{float(v).hex()}f," for v in thr[k:k + 6]))
    lines += ["};", "", "}  // namespace ar", ""]
    with open(OUT, "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
