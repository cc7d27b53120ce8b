"""Extracts the reference's t-quantile table (T005_LUT_INIT,
core/denoise/t_quantile.cu) as text into t_quantile_005_ref.npy, the fixture
that pins the denoiser's generated table.  Run where the reference sources
are present:

    python tests/golden/make_t_quantile_fixture.py <reference root>
"""
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main() -> None:
    if len(sys.argv) != 2:
        raise SystemExit("usage: make_t_quantile_fixture.py <reference root>")
    root = sys.argv[1]
    txt = open(os.path.join(root, "core", "denoise", "t_quantile.cu")).read()
    body = re.search(r"#define T005_LUT_INIT \{([^}]*)\}", txt).group(1)
    vals = np.array([float(v.strip().rstrip("f")) for v in body.split(",") if v.strip()], np.float64)
    assert len(vals) == 1024
    np.save(os.path.join(HERE, "t_quantile_005_ref.npy"), vals.astype(np.float32))


if __name__ == "__main__":
    main()
