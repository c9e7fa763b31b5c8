// Shared host/device helpers for the pymdp_b200 sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <string>

#include "../../include/pymdp_b200.h"

namespace b2 {

// float32 image of the reference's clip floor MINVAL = finfo(float64).eps
// (pymdp/maths.py:15); the reference's float32 path clips at this value.
constexpr float kMinVal = 2.220446049250313e-16f;

// ----------------------------------------------------------------- errors
int32_t fail(int32_t code, const std::string& msg);
int32_t cuda_fail(const char* op, cudaError_t err);
void note_launches(uint64_t n);

#define B2_TRY(expr)                       \
  do {                                     \
    int32_t _b2_rc = (expr);               \
    if (_b2_rc != B2_OK) return _b2_rc;    \
  } while (0)

#define B2_CUDA_TRY(op, expr)                          \
  do {                                                 \
    cudaError_t _b2_e = (expr);                        \
    if (_b2_e != cudaSuccess) return ::b2::cuda_fail(op, _b2_e); \
  } while (0)

// Check the launch that just happened (configuration errors surface here).
inline int32_t check_launch(const char* op, uint64_t n = 1) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(op, e);
  note_launches(n);
  return B2_OK;
}

// Opt a kernel into `bytes` of dynamic shared memory once per process/device.
int32_t ensure_smem_attr(const void* kernel, int bytes, const char* op);

// Programmatic dependent launch: the grid is launched with programmatic stream
// serialization, so the GPU can schedule it while its predecessor on the
// stream drains; a kernel launched this way calls grid_dependency_wait() before
// it reads anything its predecessor wrote (a no-op under an ordinary launch).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream,
                       Args&&... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}

// ---------------------------------------------------------------- device
// Waits until the grids this one depends on have completed and their writes
// are visible (griddepcontrol.wait; returns at once without a programmatic
// dependency).
__device__ __forceinline__ void grid_dependency_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

__device__ __forceinline__ float log_stable(float x) { return logf(fmaxf(x, kMinVal)); }

// The same clip with the hardware base-2 logarithm (__logf: two instructions;
// absolute error about 1e-7 near 1, relative about 2^-22 elsewhere), for x log x
// terms whose products with x leave that error far below the FP32 sums they feed.
__device__ __forceinline__ float log_fast(float x) { return __logf(fmaxf(x, kMinVal)); }

// Two FP32 fused multiply-adds in one instruction (fma.rn.f32x2 on sm_100):
// d = a * b + c lane by lane, each rounded as fmaf rounds it.
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

}  // namespace b2
