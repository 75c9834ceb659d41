// FP32 issue peak of the device: a kernel of independent FMA chains over every SM, timed with CUDA events.  It is
// the denominator of the pair and triple kernels' roofline (their bound is FP32 issue, not HBM or tensor cores).
#pragma once

namespace ix {

constexpr int kProbeChains = 8;
constexpr int kProbeIters = 16384;   // one wave of blocks that each run ~1 ms, so that the ramp and tail are negligible

__global__ void kFmaPeak(float* sink, float seed) {
    float v[kProbeChains];
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) v[c] = seed + threadIdx.x * 1e-7f + c;
    // the multiplier is a kernel argument's function, so that every FMA reads registers only
    const float a = 1.0f - 1e-6f * seed, b = 1e-7f;
    for (int it = 0; it < kProbeIters; it++) {
#pragma unroll
        for (int c = 0; c < kProbeChains; c++) v[c] = fmaf(v[c], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kProbeChains; c++) s += v[c];
    if (s == 123.456f) sink[threadIdx.x] = s;   // keeps the chains live; practically never true
}

}  // namespace ix
