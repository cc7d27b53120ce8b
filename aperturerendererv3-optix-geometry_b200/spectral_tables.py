"""Spectral rendering data: the reference's spectrum-basis network weights and
its CIE 1931 / D65 tables, extracted from the reference's sources at build
time.

The spectral mode upsamples RGB material colours with the reference's own
trained model (spectrum::query::RGBEncode / LambdaEncode,
core/spectrum/spectrum_basis.cuh: residual MLPs of width 32, 4-value output
kernels) and weights wavelengths with its tabulated CIE 1931 2-degree colour
matching functions and D65 spectrum (core/spectrum/ciexyz.cuh).  Those numbers
belong to the reference (GPL-3.0) and are not redistributed here: `build()`
reads them from the reference's headers and writes a git-ignored binary,
`_data/spectral_tables.bin`, which the library takes through
ar_scene_set_spectral().  Without the reference sources the spectral mode is
unavailable; RGB rendering does not need the file.

File layout: 8-byte magic b"ARSPEC01", uint32 float count, then float32 values
in the order of TABLE_LAYOUT (the layout ar_scene_set_spectral expects),
followed by the reference's 100 self-test cases (inputTest[4][100] and
gtTest[100], spectrum_basis.cuh:2472-2489).
"""
from __future__ import annotations

import os
import re
import struct
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
DATA = os.path.join(HERE, "_data", "spectral_tables.bin")
MAGIC = b"ARSPEC01"

# (name, float count) in ar_scene_set_spectral order
TABLE_LAYOUT = (
    [("CIEXYZ_CMF", 421 * 3), ("D65_SPD", 421), ("RGB_IN_W", 1024), ("RGB_IN_B", 32)]
    + [(f"RGB_BLK{i}_W", 1024) for i in range(7)] + [(f"RGB_BLK{i}_B", 32) for i in range(7)]
    + [("RGB_OUT_W", 128)]
    + [(f"LAM_BLK{i}_W", 1024) for i in range(7)] + [(f"LAM_BLK{i}_B", 32) for i in range(7)]
    + [("LAM_OUT_W", 128)]
)
TABLE_FLOATS = sum(n for _, n in TABLE_LAYOUT)   # 17780


def _array_body(text: str, name: str) -> str:
    m = re.search(r"\b" + re.escape(name) + r"\s*(\[[^\]]*\])+\s*=\s*(?:\n#else\n[^\n]*\n#endif\n)?\s*\{", text)
    if not m:
        raise KeyError(name)
    i, depth = m.end() - 1, 0
    for j in range(i, len(text)):
        if text[j] == "{":
            depth += 1
        elif text[j] == "}":
            depth -= 1
            if depth == 0:
                return text[i + 1:j]
    raise ValueError(name)


def _floats(body: str) -> np.ndarray:
    body = re.sub(r"//[^\n]*", "", body).replace("float3", "")
    vals = re.findall(r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?f?", body)
    return np.array([float(v.rstrip("f")) for v in vals], np.float32)


def extract(ref_core: str) -> dict:
    """Arrays of TABLE_LAYOUT (plus inputTest, gtTest) from the reference headers."""
    spec = os.path.join(ref_core, "spectrum")
    basis = open(os.path.join(spec, "spectrum_basis.cuh")).read()
    cie = open(os.path.join(spec, "ciexyz.cuh")).read()
    out = {}
    for name, count in TABLE_LAYOUT:
        src = cie if name in ("CIEXYZ_CMF", "D65_SPD") else basis
        a = _floats(_array_body(src, name))
        if a.size != count:
            raise ValueError(f"{name}: {a.size} values, expected {count}")
        out[name] = a
    out["inputTest"] = _floats(_array_body(basis, "inputTest"))
    out["gtTest"] = _floats(_array_body(basis, "gtTest"))
    assert out["inputTest"].size == 400 and out["gtTest"].size == 100
    return out


def write(ref_core: str, path: str = DATA) -> None:
    arrays = extract(ref_core)
    flat = np.concatenate([arrays[n] for n, _ in TABLE_LAYOUT]).astype(np.float32)
    os.makedirs(os.path.dirname(path), exist_ok=True)
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(struct.pack("<I", flat.size))
        f.write(flat.tobytes())
        f.write(arrays["inputTest"].tobytes())
        f.write(arrays["gtTest"].tobytes())


def available(path: str = DATA) -> bool:
    return os.path.exists(path)


def load(path: str = DATA):
    """(tables float32[TABLE_FLOATS], inputTest float32[4, 100], gtTest float32[100])."""
    raw = open(path, "rb").read()
    if raw[:8] != MAGIC:
        raise ValueError(f"{path}: not a spectral table file")
    n = struct.unpack("<I", raw[8:12])[0]
    if n != TABLE_FLOATS:
        raise ValueError(f"{path}: {n} table values, expected {TABLE_FLOATS}")
    v = np.frombuffer(raw[12:], np.float32)
    return v[:n].copy(), v[n:n + 400].reshape(4, 100).copy(), v[n + 400:n + 500].copy()


def build(ref_core: str | None) -> bool:
    """Write the table file from the reference's core/ directory (given, or
    from the environment variable AR_REFERENCE_CORE); False when neither names
    an existing directory (the file already written, if any, stays)."""
    ref_core = ref_core or os.environ.get("AR_REFERENCE_CORE")
    if not ref_core or not os.path.isdir(ref_core):
        return False
    write(ref_core)
    return True


if __name__ == "__main__":
    if len(sys.argv) != 2:
        raise SystemExit("usage: spectral_tables.py <reference core/ directory>")
    ok = build(sys.argv[1])
    print(DATA if ok else "reference sources not found: spectral tables not written")
