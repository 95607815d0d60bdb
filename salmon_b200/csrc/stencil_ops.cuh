// Device helpers shared by the stencil kernels (k_pass.cu, k_resident.cu):
// vector loads and stores of a thread's run of RZ consecutive z points, and the
// arithmetic of one +-n neighbour pair of the finite-difference stencil.
#pragma once

#include <cuda_runtime.h>

#include <type_traits>

#include "sgpu_internal.cuh"

namespace sgpu {

// asynchronous copy of N complex elements (8- or 16-byte aligned runs)
template <typename R, int N>
__device__ __forceinline__ void cp_run(C2<R>* dst, const C2<R>* src) {
  constexpr int BYTES = N * (int)sizeof(C2<R>);
  if constexpr (BYTES == 8) {
    cp_async8(dst, src);
  } else {
#pragma unroll
    for (int k = 0; k < BYTES / 16; ++k)
      cp_async16(reinterpret_cast<char*>(dst) + 16 * k, reinterpret_cast<const char*>(src) + 16 * k);
  }
}

template <typename R, int RZ>
__device__ __forceinline__ void ld_run(C2<R> (&d)[RZ], const C2<R>* p) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    const float4 t = __ldg(reinterpret_cast<const float4*>(p));
    d[0] = make_float2(t.x, t.y);
    d[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) d[r] = __ldg(p + r);
  }
}
template <typename R, int RZ>
__device__ __forceinline__ void ld_run_rw(C2<R> (&d)[RZ], const C2<R>* p) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    d[0] = make_float2(t.x, t.y);
    d[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) d[r] = p[r];
  }
}
template <typename R, int RZ>
__device__ __forceinline__ void st_run(C2<R>* p, const C2<R> (&d)[RZ]) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    *reinterpret_cast<float4*>(p) = make_float4(d[0].x, d[0].y, d[1].x, d[1].y);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) p[r] = d[r];
  }
}
template <typename R, int RZ>
__device__ __forceinline__ void lds_run(C2<R> (&d)[RZ], const C2<R>* p) {
  if constexpr (RZ == 2 && std::is_same<R, float>::value) {
    const float4 t = *reinterpret_cast<const float4*>(p);
    d[0] = make_float2(t.x, t.y);
    d[1] = make_float2(t.z, t.w);
  } else {
#pragma unroll
    for (int r = 0; r < RZ; ++r) d[r] = p[r];
  }
}
// the RZ local sphere indices of this thread's points (-1: not a sphere point)
template <int RZ>
__device__ __forceinline__ void ld_lq(int (&d)[RZ], const short* p) {
  if constexpr (RZ == 2) {
    const int v = __ldg(reinterpret_cast<const int*>(p));
    d[0] = (int)(short)(v & 0xffff);
    d[1] = v >> 16;
  } else {
    d[0] = __ldg(p);
  }
}

__device__ __forceinline__ int wrapi(int a, int n) { a %= n; return a < 0 ? a + n : a; }

// v += cl (p + m), wa += cn (p - m).  Complex(4) runs on packed FP32 pairs
// (sm_100 f32x2 add/fma: one instruction updates both parts of a complex
// value; cl, cn are broadcast pairs); complex(8) on scalar FP64.
__device__ __forceinline__ void stencil_pair(float2& v, float2& wa, float2 p, float2 m, float2 cl, float2 cn) {
  const float2 sum = __fadd2_rn(p, m);
  const float2 dif = __ffma2_rn(m, make_float2(-1.f, -1.f), p);  // p - m (exact negation)
  v = __ffma2_rn(cl, sum, v);
  wa = __ffma2_rn(cn, dif, wa);
}
__device__ __forceinline__ void stencil_pair(double2& v, double2& wa, double2 p, double2 m, double cl, double cn) {
  v.x = fma(cl, p.x + m.x, v.x);
  v.y = fma(cl, p.y + m.y, v.y);
  wa.x = fma(cn, p.x - m.x, wa.x);
  wa.y = fma(cn, p.y - m.y, wa.y);
}
template <typename R> __device__ __forceinline__ auto kpair(double k) {
  if constexpr (std::is_same<R, float>::value) return make_float2((float)k, (float)k); else return k;
}
// w = k wa (first axis) or w += k wa
__device__ __forceinline__ float2 kscale(float2 k, float2 wa, float2 w) { return __ffma2_rn(k, wa, w); }
__device__ __forceinline__ double2 kscale(double k, double2 wa, double2 w) {
  return make_double2(fma(k, wa.x, w.x), fma(k, wa.y, w.y));
}


}  // namespace sgpu
