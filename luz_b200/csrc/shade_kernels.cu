// shade_kernels.cu — the shade stage of the wavefront integrator, in a
// translation unit of its own built with FMA contraction (-fmad=true).
//
// Traversal (trace.cuh), ray generation and the film stay in integrator.cu,
// built with -fmad=false: there every FP32 expression rounds as written, so
// the GPU hits equal the FP32 restatement's bit for bit. Shading is compared
// with the FP64 reference within a relative tolerance, where contracting a
// product and a sum into one rounding only removes error; the sampler's FP64
// lattice arithmetic (dmath.cuh) is written with explicit round-to-nearest
// intrinsics, so it stays bit-exact with the reference in either unit.
#define LUZ_NO_CACHE_KERNELS
// Inlined here, out of line elsewhere: the sampler, the environment and light
// sampling / pdf functions and the hit record. With the paths binned by material
// class the shade kernel's instruction footprint no longer stalls it, and these
// calls' argument traffic through local memory cost more (1080p glossy frame, 16
// spp: shade stage 29.5 -> 25.8 ms). Inlining the BSDF functions as well made it
// slower (37.7 ms: 128 registers could no longer hold the larger body).
#define LUZ_SAMPLER_ATTR __forceinline__
#define LUZ_LIGHT_ATTR __forceinline__
#define LUZ_HIT_ATTR __forceinline__
#include "shade_kernels.cuh"

namespace luz {

BatchShadeKernel batch_shade_kernel(int mode)
{
    return mode == 1 ? k_shade_batch<1> : k_shade_batch<0>;
}

ShadeKernel shade_kernel(int mode)
{
    switch (mode) {
    case 1: return k_shade<1>;
    case 2: return shade_kernel_cached();
    case 3: return k_shade<3>;
    default: return k_shade<0>;
    }
}

}  // namespace luz
