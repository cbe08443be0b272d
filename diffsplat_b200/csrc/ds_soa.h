// Host/device structs of device pointers for the three splat SoA types.
// Field order matches the reference types (src/types/gaussian3d.h:34-74,
// src/types/splat3d.h:14-30, src/types/splat2d.h:13-26) and the public C ABI
// in include/diffsplat_b200.h, which uses the same layouts.
#pragma once
#include "../../include/diffsplat_b200.h"
