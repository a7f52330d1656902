// Internal types shared by the host launchers and the kernels.
#pragma once
#include <stdint.h>

#include "../../include/pyexner_b200.h"

#define PXB_MAX_SED 8
// Halo columns on each side of a warp strip (a three-deep dependency chain per stage).
#define PXB_HALO 3
// Consecutive columns per lane of the fused stage kernel (strip = 32 x CPT columns).
// float64: 1.  float32: 1 by default; 2 (a 64-column strip, 58 owned: half the halo
// columns and half the shuffles per cell) is a build knob, measured 15-20% slower on
// B200 because its ~200 registers per thread leave 8-12 warps per SM, too few to hide
// the latencies of the face arithmetic.
#ifndef PXB_STAGE_CPT_F32
#define PXB_STAGE_CPT_F32 1
#endif
static inline constexpr __host__ __device__ int pxb_stage_cpt(int esize) { return esize == 4 ? PXB_STAGE_CPT_F32 : 1; }
// Owned columns of one stage strip.
static inline constexpr __host__ __device__ int pxb_stage_strip_out(int esize) {
    return 32 * pxb_stage_cpt(esize) - 2 * PXB_HALO;
}

// Work items of the fused stage kernel in one band of rows: the interior strips one item
// each; the first and last strips, which also carry the boundary passes (more work per
// row), two half-height items each so that they are not the longest items of a launch.
// Order within a band: first strip (upper, lower half), interior strips, last strip
// (upper, lower half).
static inline __host__ __device__ int pxb_stage_items_per_band(int nstrips) { return nstrips >= 2 ? nstrips + 2 : 1; }
