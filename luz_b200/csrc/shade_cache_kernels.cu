// shade_cache_kernels.cu — the radiance-cache instantiation of the shade kernel
// (luz_gpu_render_cached), built like shade_kernels.cu (FMA contraction) but with the
// sampler, light sampling and hit record out of line: its larger shading body spilled
// with them inlined (Cornell 300x300, 256 spp: cached render 33.7 -> 39.0 ms).
#define LUZ_NO_CACHE_KERNELS
#include "shade_kernels.cuh"

namespace luz {

ShadeKernel shade_kernel_cached()
{
    return k_shade<2>;
}

}  // namespace luz
