"""Build-time copy of the reference's core/ with the mechanical edits that let
its path loop (CalculateRadiance, core/render/render.cuh:460-999) run on the
host.  TEST INFRASTRUCTURE ONLY: run by `make -C oracle ref-path`; the output
goes to the git-ignored oracle/_ref/src/ and is compiled there together with
ref_path_harness.cu into oracle/_ref/libref_path.so.  Nothing of the reference
is committed; this script holds only the anchors of each edit.

    python ref_path_patch.py --src <reference>/core --dst _ref/src/core

Edits (each must match exactly once, else the script fails):
  0. The device-only function qualifiers FUNCTION_MODIFIER_DEVICE_INLINE and
     FUNCTION_MODIFIER_DEVICE (vector.cuh:35-36) become __host__ __device__,
     so that Trace, NEE, SampleBSDF, EvaluateMaterial, the NEE samplers and
     CalculateRadiance compile for the host.
  1. RGB build of Trace and NEE: the spectral signatures carry `const int
     depth`, the RGB ones do not, yet both bodies use it (render.cuh:76-84,
     207-212) and the RGB build fails to compile.  The RGB signatures get the
     same parameter; CalculateRadiance's RGB call of NEE passes the loop depth,
     as its spectral call does (render.cuh:788-790).  Trace is already called
     with nonDeltaDepth in both builds (render.cuh:547-553).
  2. Random numbers: Rand1/Rand2/Rand3 (random.cuh:41-53) draw through
     ref_uniform(seed), which the harness defines (curand_uniform on the
     device, a recorded tape or a host generator on the host); InitRand's
     body (threadIdx, curand_init) is compiled for the device only.
  3. Textures: tex2D<float4> in EvaluateBSDFWithCos / SampleBSDF
     (material.cuh:71, 200) goes through ref_tex2d_float4 (device: tex2D;
     host: never reached, the harness's materials have no texture).
  4. Two observation hooks for per-path records, placed where the reference's
     own control flow already is: after Trace has produced its result
     (render.cuh:162) and after NEE's shadow segment query (render.cuh:253).
     They read values and change nothing.
  5. thrust's `cuda::par` in guiding.cuh is spelled `thrust::cuda::par`
     (CCCL 2.8 makes the bare name ambiguous; guiding.cuh:84-111).
  6. The one `[&] __device__` lambda of the guiding debug view
     (guiding_debug.cuh:188) loses its annotation: a lambda inside a
     __host__ __device__ function takes that function's execution space.
Everything else -- the globals block, the 32-bit BVH layout, RGB mode and the
run-time MAX_TRACING_DEPTH -- is selected by ref_path_prelude.h without edits.
"""
from __future__ import annotations

import argparse
import os
import re
import shutil


def _sub_once(text: bytes, pattern: bytes, repl: bytes, what: str, count: int = 1) -> bytes:
    new, n = re.subn(pattern, repl, text)
    if n != count:
        raise SystemExit(f"ref_path_patch: {what}: expected {count} match(es), found {n}")
    return new


def patch(dst: str) -> None:
    def rw(rel, fn):
        path = os.path.join(dst, rel)
        with open(path, "rb") as f:
            text = f.read()
        text = fn(text)
        with open(path, "wb") as f:
            f.write(text)

    NL = rb"(\r?\n)"

    def render(t: bytes) -> bytes:
        # 1. RGB Trace / NEE signatures and the RGB NEE call
        t = _sub_once(t, rb"(#else" + NL + rb"FUNCTION_MODIFIER_DEVICE_INLINE TraceContext Trace\()" + NL + rb"#endif",
                      rb"\1\3    const int depth,\3#endif", "RGB Trace signature")
        t = _sub_once(t, rb"(#else" + NL + rb"FUNCTION_MODIFIER_DEVICE float3 NEE\()" + NL + rb"#endif",
                      rb"\1\3    const int depth,\3#endif", "RGB NEE signature")
        t = _sub_once(t, rb"(#else" + NL + rb"(\s*)const float3 radianceNEE = NEE<bUseBVH, bUsePathGuiding>\()" + NL
                      + rb"#endif", rb"\1\4\3    depth,\4#endif", "RGB NEE call")
        # 4. observation hooks
        t = _sub_once(t, rb"(\r?\n)(\s*)return traceResult;", rb"\1\2REF_HOOK_TRACE(seed, traceResult);\1\2return traceResult;",
                      "Trace hook")
        t = _sub_once(t, rb"(const IntersectionContext segmentTraceResult = SegmentTrace<bUseBVH>\([^;]*;)",
                      rb"\1 REF_HOOK_SHADOW(seed, depth);", "shadow hook")
        return t

    def vector(t: bytes) -> bytes:
        t = _sub_once(t, rb"#define FUNCTION_MODIFIER_DEVICE_INLINE __device__ __forceinline__",
                      b"#define FUNCTION_MODIFIER_DEVICE_INLINE __host__ __device__ __forceinline__", "DEVICE_INLINE")
        t = _sub_once(t, rb"#define FUNCTION_MODIFIER_DEVICE __device__(?=\s)",
                      b"#define FUNCTION_MODIFIER_DEVICE __host__ __device__", "DEVICE")
        return t

    def random(t: bytes) -> bytes:
        t = _sub_once(t, rb"curand_uniform\(seed\)", b"ref_uniform(seed)", "Rand1/2/3", count=6)
        t = _sub_once(t, rb"(void InitRand\(curandState\* seed\)" + NL + rb"\{)",
                      rb"\1\2#ifdef __CUDA_ARCH__", "InitRand begin")
        t = _sub_once(t, rb"(curand_init\(GLOBAL_SEED, pixelIndex, [^;]*;)" + NL + rb"\}",
                      rb"\1\2#endif\2}", "InitRand end")
        return t

    def material(t: bytes) -> bytes:
        return _sub_once(t, rb"tex2D<float4>\(", b"ref_tex2d_float4(", "tex2D", count=2)

    def guiding(t: bytes) -> bytes:
        return _sub_once(t, rb"(?<![:\w])cuda::par\b", b"thrust::cuda::par", "cuda::par", count=5)

    def guiding_debug(t: bytes) -> bytes:
        return _sub_once(t, rb"\[&\] __device__ \(", b"[&] (", "device lambda")

    rw("vector.cuh", vector)
    rw("guiding/guiding_debug.cuh", guiding_debug)
    rw("render/render.cuh", render)
    rw("random.cuh", random)
    rw("render/material.cuh", material)
    rw("guiding/guiding.cuh", guiding)
    # case-sensitive file systems: the sources include object/AABB.cuh and object/Sphere.cuh
    for a, b in (("aabb.cuh", "AABB.cuh"), ("sphere.cuh", "Sphere.cuh")):
        src = os.path.join(dst, "object", a)
        alias = os.path.join(dst, "object", b)
        if not os.path.exists(alias):
            with open(alias, "w") as f:
                f.write(f'#pragma once\n#include "{a}"\n')


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--src", required=True, help="the reference's core/ directory")
    ap.add_argument("--dst", required=True, help="output directory (git-ignored)")
    a = ap.parse_args()
    if not os.path.isdir(a.src):
        raise SystemExit(f"ref_path_patch: {a.src} is not a directory")
    if os.path.exists(a.dst):
        shutil.rmtree(a.dst)
    shutil.copytree(a.src, a.dst)
    patch(a.dst)


if __name__ == "__main__":
    main()
