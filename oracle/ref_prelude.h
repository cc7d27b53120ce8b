/*
 * ref_prelude.h -- pre-included (nvcc -include) into ref_harness.cu, before any
 * of the reference's own headers.  TEST INFRASTRUCTURE ONLY.
 *
 * It selects the reference configuration used for pinning without editing the
 * reference's files: the reference's config.cuh is included here first, its
 * `#pragma once` keeps it from being read again, and the switches below are
 * then changed.
 *   - USE_SPECTRUM_RENDERING off: the RGB build, which is what this project's
 *     CUDA core computes (config.cuh:61).
 *   - BVH_USE_16_BITS_NODE / BVH_PACK_NODE off: the reference's own 32-bit
 *     node layout (bvh.cuh:36-42), needed above 32767 primitives; it changes
 *     the node storage only, not the build or traversal algorithm.
 * <cfloat> and <climits> are included because some reference headers use
 * FLT_MAX / INT_MAX without including them.
 */
#pragma once
#include <cfloat>
#include <climits>

#include "config.cuh"

#undef USE_SPECTRUM_RENDERING
#undef BVH_USE_16_BITS_NODE
#undef BVH_PACK_NODE
