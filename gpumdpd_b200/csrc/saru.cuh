// saru.cuh -- the Saru counter-based random number of the DPD random force.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// The stream must be bit-identical to the reference's (src/force/pair_dpd.cu:203-236),
// so the published steps and constants are kept; the float tail is evaluated with one
// rounding per operation exactly as the reference's -DSINGLE build does:
// u = (float)s * 2^-31 - 1, theta = sqrt(3)f * u.
__device__ __forceinline__ uint32_t saru_bits(uint32_t seed1, uint32_t seed2, uint32_t seed,
                                              uint32_t timestep)
{
    uint32_t seed3 = seed + timestep;
    seed3 ^= (seed1 << 7) ^ (seed2 >> 6);
    seed2 += (seed1 >> 4) ^ (seed3 >> 15);
    seed1 ^= (seed2 << 9) + (seed3 << 8);
    seed3 ^= 0xA5366B4Du * ((seed2 >> 11) ^ (seed1 << 1));
    seed2 += 0x72BE1579u * ((seed1 << 4) ^ (seed3 >> 16));
    seed1 ^= 0x3F38A6EDu * ((seed3 >> 5) ^ (uint32_t)(((int32_t)seed2) >> 22));
    seed2 += seed1 * seed3;
    seed1 += seed3 ^ (seed2 >> 2);
    seed2 ^= (uint32_t)(((int32_t)seed2) >> 17);
    uint32_t state = 0x79dedea3u * (seed1 ^ (uint32_t)(((int32_t)seed1) >> 14));
    uint32_t wstate = (state + seed2) ^ (uint32_t)(((int32_t)state) >> 8);
    state = state + (wstate * (wstate ^ 0xdddf97f5u));
    wstate = 0xABCB96F7u + (wstate >> 1);
    uint32_t sum = 0;
#pragma unroll
    for (int r = 0; r < 8; r++) {
        sum += 0x9e3779b9u;
        state += ((wstate << 4) + 0xA341316Cu) ^ (wstate + sum) ^ ((wstate >> 5) + 0xC8013EA4u);
        wstate += ((state << 4) + 0xAD90777Du) ^ (state + sum) ^ ((state >> 5) + 0x7E95761Eu);
    }
    uint32_t v = (state ^ (state >> 26)) + wstate;
    return (v ^ (v >> 20)) * 0x6957f5a7u;
}

__device__ __forceinline__ float saru_theta(uint32_t seed1, uint32_t seed2, uint32_t seed,
                                            uint32_t timestep)
{
    const uint32_t s = saru_bits(seed1, seed2, seed, timestep);
    float u = __fmaf_rn(__uint2float_rn(s), 4.6566128730773926e-10f, -1.0f);
    return __fmul_rn(1.7320508075688772f, u);
}

// The tail of the reference's -DDOUBLE build (the same line with numtyp = double): the
// product s * 2^-32 stays float (its constant is a float literal), an exact scaling of
// (float)s; the affine map and sqrt(3) are double.
__device__ __forceinline__ double saru_theta_f64(uint32_t seed1, uint32_t seed2, uint32_t seed,
                                                 uint32_t timestep)
{
    const uint32_t s = saru_bits(seed1, seed2, seed, timestep);
    const float a = __fmul_rn(__uint2float_rn(s), 2.3283064365386963e-10f);
    return __dmul_rn(1.7320508075688772935274463, __fma_rn((double)a, 2.0, -1.0));
}
