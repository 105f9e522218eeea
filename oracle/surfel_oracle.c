/*
 * TEST INFRASTRUCTURE ONLY — the checker for the UltraGS-baseline surfel rasteriser tests;
 * nothing in the product links or calls it.
 *
 * Restatement of ops/ultrags_baseline_renderer/cuda_rasterizer in C, in fp32 (suffix _f32)
 * and fp64 (suffix _f64): preprocess (near cull, splat homography, dual-visible normal,
 * screen AABB, SH colour), tile lists ordered by (view depth, Gaussian) like the reference's
 * stable radix sort of (tile << 32 | depth bits), front-to-back compositing with the
 * auxiliary maps, and the back-to-front backward with the preprocess backward.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define REAL float
#define SUFFIX _f32
#define SQRT sqrtf
#define CEIL ceilf
#define EXP expf
#include "surfel_oracle_impl.h"
#undef REAL
#undef SUFFIX
#undef SQRT
#undef CEIL
#undef EXP

#define REAL double
#define SUFFIX _f64
#define SQRT sqrt
#define CEIL ceil
#define EXP exp
#include "surfel_oracle_impl.h"
