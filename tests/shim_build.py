"""Builds tests/native/shim_render.cpp (a caller of the reference's C++ API
compiled against include/aperture_b200_renderer.hpp) and runs it."""
import os
import shutil
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
PKG = os.path.join(ROOT, "aperturerendererv3-optix-geometry_b200")
CUDA = "/usr/local/cuda"


def available() -> bool:
    return shutil.which("g++") is not None and os.path.exists(os.path.join(CUDA, "include", "vector_types.h"))


def build(outdir: str) -> str:
    exe = os.path.join(outdir, "shim_render")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I" + os.path.join(ROOT, "include"),
                    "-I" + os.path.join(CUDA, "include"), "-o", exe, os.path.join(HERE, "native", "shim_render.cpp"),
                    "-L" + PKG, "-laperture_b200", "-Wl,-rpath," + PKG, "-L" + os.path.join(CUDA, "lib64"),
                    "-lcudart", "-Wl,-rpath," + os.path.join(CUDA, "lib64")], check=True)
    return exe


def run(outdir: str, w: int, h: int, spp: int) -> str:
    exe = build(outdir)
    out = subprocess.run([exe, outdir, str(w), str(h), str(spp)], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    return out.stdout


def read_bmp(path: str):
    """(width, height, rgba[h, w, 4]) of a 32-bit top-down BMP."""
    raw = open(path, "rb").read()
    assert raw[:2] == b"BM"
    size, off = int.from_bytes(raw[2:6], "little"), int.from_bytes(raw[10:14], "little")
    w = int.from_bytes(raw[18:22], "little", signed=True)
    h = int.from_bytes(raw[22:26], "little", signed=True)
    assert size == len(raw) and off == 54 and raw[28] == 32 and h < 0
    bgra = np.frombuffer(raw[54:], np.uint8).reshape(-h, w, 4)
    return w, -h, bgra[..., [2, 1, 0, 3]]
