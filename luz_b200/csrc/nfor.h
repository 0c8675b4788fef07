// NFOR denoiser entry shared by the render path (integrator.cu) and nfor.cu.
#pragma once

#include <cstdint>
#include <string>

#include "luz_gpu.h"

// Denoise::applyNFOR (src/core/Denoise/NFOR.cpp:977-1102) on device-resident
// NFOR buffers laid out as LuzNforBuffers; writes width*height*3 doubles to
// d_out on `stream` and synchronizes it. settings NULL = NFORSettings defaults.
// Returns LUZ_OK, or a LUZ_E_* code with its message in msg.
int luz_nfor_on_device(const double* color_a, const double* color_b, const double* color_variance,
                       const double* features_a, const double* features_b, const double* feature_variance,
                       int32_t width, int32_t height, const LuzNforSettings* settings, double* d_out, void* stream,
                       std::string& msg);
