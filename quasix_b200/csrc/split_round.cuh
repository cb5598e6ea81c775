// Rounding of the hi/lo operand split used by every tcgen05 split form.
//
// A value v (FP64, already scaled) becomes hi = rn16(f) and lo = rn16(f - hi)
// with f = rn32(v) and rn16 the round-to-nearest conversion to fp16 or bf16.
// f - hi is exact in FP32 (hi lies within half a 16-bit ulp of f, so the two
// are within a factor of two of each other, or both are multiples of f's ulp
// in the fp16 subnormal range), so hi + lo represents f to half a 16-bit ulp
// of the residual and v to that plus half an FP32 ulp.  The FP64 value is
// converted once; the rest is FP32 and packed 16-bit arithmetic, which keeps
// the splits off the slow FP64 conversion path.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <stdint.h>

namespace qx {

template <bool FP16>
__device__ __forceinline__ void split_round(double v, uint16_t& h, uint16_t& l) {
  const float f = (float)v;
  if (FP16) {
    const __half hh = __float2half_rn(f);
    h = __half_as_ushort(hh);
    l = __half_as_ushort(__float2half_rn(f - __half2float(hh)));
  } else {
    const __nv_bfloat16 hh = __float2bfloat16_rn(f);
    h = __bfloat16_as_ushort(hh);
    l = __bfloat16_as_ushort(__float2bfloat16_rn(f - __bfloat162float(hh)));
  }
}

// split_round of two values at once, packed as (first in the low 16 bits) the
// hi word and the lo word.
template <bool FP16>
__device__ __forceinline__ void split_round2(double v0, double v1, uint32_t& hw, uint32_t& lw) {
  const float f0 = (float)v0, f1 = (float)v1;
  if (FP16) {
    const __half2 hh = __floats2half2_rn(f0, f1);
    const float2 hf = __half22float2(hh);
    const __half2 ll = __floats2half2_rn(f0 - hf.x, f1 - hf.y);
    hw = (uint32_t)__half_as_ushort(__low2half(hh)) | ((uint32_t)__half_as_ushort(__high2half(hh)) << 16);
    lw = (uint32_t)__half_as_ushort(__low2half(ll)) | ((uint32_t)__half_as_ushort(__high2half(ll)) << 16);
  } else {
    const __nv_bfloat162 hh = __floats2bfloat162_rn(f0, f1);
    const float2 hf = __bfloat1622float2(hh);
    const __nv_bfloat162 ll = __floats2bfloat162_rn(f0 - hf.x, f1 - hf.y);
    hw = (uint32_t)__bfloat16_as_ushort(__low2bfloat16(hh)) |
         ((uint32_t)__bfloat16_as_ushort(__high2bfloat16(hh)) << 16);
    lw = (uint32_t)__bfloat16_as_ushort(__low2bfloat16(ll)) |
         ((uint32_t)__bfloat16_as_ushort(__high2bfloat16(ll)) << 16);
  }
}

}  // namespace qx
