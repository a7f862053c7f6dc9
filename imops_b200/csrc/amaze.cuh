// amaze.cuh -- AMaZE launchers used by the fused pipeline.
#pragma once

#include "color.cuh"
#include "common.cuh"

namespace imops {
namespace amaze {

bool size_supported(int W, int H);

// AMaZE on an f32 mosaic, colour epilogue applied per pixel, RGB out.
int demosaic_color_f32(const float* mosaic, int W, int H, const CfaDev& cfa, float clip, const color::Epilogue& e,
                       float* rgb, cudaStream_t s);

// AMaZE reading a u16 sensor frame (crop origin cx, cy; per-cell black /
// white levels over a pw x ph period), scaled on load.
int demosaic_color_u16(const uint16_t* raw, int raw_w, int raw_h, int cx, int cy, int W, int H, const float* black,
                       const float* white, int pw, int ph, const CfaDev& cfa, float clip, const color::Epilogue& e,
                       float* rgb, cudaStream_t s);

}  // namespace amaze
}  // namespace imops
