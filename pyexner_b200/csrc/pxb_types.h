// Internal types shared by the host launchers and the kernels.
#pragma once
#include <stdint.h>

#include "../../include/pyexner_b200.h"

#define PXB_MAX_SED 8
// Columns of one warp strip: 32 lanes = 3 halo + 26 owned + 3 halo.
#define PXB_STRIP_OUT 26
#define PXB_HALO 3

// Work items of the fused stage kernel in one band of rows: the interior strips one item
// each; the first and last strips, which also carry the boundary passes (more work per
// row), two half-height items each so that they are not the longest items of a launch.
// Order within a band: first strip (upper, lower half), interior strips, last strip
// (upper, lower half).
static inline __host__ __device__ int pxb_stage_items_per_band(int nstrips) { return nstrips >= 2 ? nstrips + 2 : 1; }
