// demosaic_simple.cuh -- the reference's 3x3 same-colour mean
// (pichromatic/src/demosaic.rs:108-186) for other translation units.
#pragma once

#include "color.cuh"
#include "common.cuh"

namespace imops {
namespace simple {

// The mean of a (w, h) f32 mosaic into interleaved RGB; when epi is given,
// each pixel's RGB goes through it before the store (the same operations
// as color::run_epilogue over the stored mean).  Validates its arguments and
// reports failures through fail().
int mean3x3(const float* mosaic, int w, int h, const CfaDev& c, const color::Epilogue* epi, float* rgb,
            cudaStream_t s);

}  // namespace simple
}  // namespace imops
