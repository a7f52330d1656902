// Internal types shared by the host launchers and the kernels.
#pragma once
#include <stdint.h>

#include "../../include/pyexner_b200.h"

#define PXB_MAX_SED 8
// Columns of one warp strip: 32 lanes = 3 halo + 26 owned + 3 halo.
#define PXB_STRIP_OUT 26
#define PXB_HALO 3
