// b2_neg_efe_noalloc: the SIMT FP32 neg-EFE evaluation (the same two kernels
// b2_neg_efe runs at FP32 precision) with its per-(agent, t) linear-row
// workspace taken from a fixed array in device memory instead of the
// stream-ordered pool.
//
// Who needs it: callers that must not allocate device memory while they run,
// e.g. a host framework that owns every byte of the GPU through its own
// arena (and would see a cudaMallocAsync as memory it cannot account for),
// a real-time control loop that has to keep allocator latency and pool
// growth out of its step, or a caller sitting inside a custom-call handler
// whose runtime forbids allocation there. This entry point calls no
// cudaMalloc / cudaMallocAsync / cudaFree and no allocating library routine.
//
// The scratch is one file-scope array shared by every call in the process on
// a given device (every device that loads the library holds it until exit).
// Consequences:
//  * Bn * T * (sum_m K_m) floats must fit in B2_NOALLOC_SCRATCH_BYTES
//    (16 MiB); larger calls are rejected with B2_ERR_UNSUPPORTED before any
//    launch.
//  * Calls that overlap on the GPU (two streams, or two host threads without
//    ordering) race on the array and give wrong results. Serialise them, e.g.
//    issue all of them on one stream.
//  * The array keeps the last call's contents. Nothing has to start at zero:
//    the linear-row kernel writes every element that the policy kernel reads
//    in the same call.
//  * The first call on each device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current) and caches it. Make that
//    first call before any stream capture begins.
#include <mutex>
#include <string>

#include "common.cuh"
#include "efe.cuh"

namespace b2 {
namespace {

constexpr size_t kNoAllocScratchBytes = B2_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;
const char* const kNoAllocName = "efe_noalloc";

static __device__ __align__(256) float g_efe_lin_scratch[kNoAllocScratchBytes / sizeof(float)];

std::mutex g_scratch_mu;
float* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (looked up once
// per device; the array's host-side name is not a device address).
int32_t scratch_for_current_device(float** out) {
  int dev = 0;
  B2_CUDA_TRY(kNoAllocName, cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices)
    return fail(B2_ERR_UNSUPPORTED, std::string(kNoAllocName) + ": device ordinal " + std::to_string(dev) +
                                        " above " + std::to_string(kMaxDevices - 1));
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_ptr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_efe_lin_scratch);
    if (e != cudaSuccess) return cuda_fail(kNoAllocName, e);
    if (!ptr) return fail(B2_ERR_CUDA, std::string(kNoAllocName) + ": scratch symbol has no device address");
    g_scratch_ptr[dev] = static_cast<float*>(ptr);
  }
  *out = g_scratch_ptr[dev];
  return B2_OK;
}

int32_t noalloc_bad(const std::string& msg) {
  return fail(B2_ERR_INVALID_ARGUMENT, std::string(kNoAllocName) + ": " + msg);
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_neg_efe_noalloc(
    void* stream_, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched, const float* qs_init,
    int64_t qs_count, const float* A, int64_t A_count, const float* B, int64_t B_count, const float* C,
    int64_t C_count, const float* I, int64_t I_count, const float* pA, int64_t pA_count, const float* pB,
    int64_t pB_count, const float* inductive_epsilon, int64_t eps_count, float* neg_efe_out, int64_t out_count,
    int64_t Bn, int64_t P, int64_t T, int64_t F, int64_t M, const int64_t* S, const int64_t* O, const int64_t* U,
    const int64_t* qs_offsets, const int64_t* A_offsets, const int64_t* B_offsets, const int64_t* C_offsets,
    const int64_t* I_offsets, const int64_t* I_depths, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
    const int64_t* A_dep_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets,
    int32_t flags) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (Bn < 0) return noalloc_bad("negative Bn");
  EfeParams p;
  B2_TRY(build_efe_params(&p, P, T, F, M, S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_offsets,
                          I_depths, A_dep_flat, A_dep_flat_len, A_dep_offsets, B_dep_flat, B_dep_flat_len,
                          B_dep_offsets, flags));
  const struct {
    const char* name;
    int64_t actual, expected;
  } chks[] = {
      {"policy_matrix", pm_count, (pm_batched ? Bn : 1) * P * T * F},
      {"qs_init", qs_count, Bn * (int64_t)p.S_tot},
      {"A", A_count, Bn * p.A_stride},
      {"B", B_count, Bn * p.B_stride},
      {"C", C_count, Bn * p.C_stride},
      {"I", I_count, Bn * I_offsets[F]},
      {"out", out_count, Bn * P},
  };
  for (const auto& c : chks)
    if (c.actual != c.expected)
      return noalloc_bad(std::string(c.name) + " element_count = " + std::to_string(c.actual) + ", expected " +
                         std::to_string(c.expected));
  if (eps_count != 1 && eps_count != Bn) return noalloc_bad("inductive_epsilon must have 1 or Bn elements");
  if (((flags >> B2_PRECISION_SHIFT) & 3) > B2_PRECISION_BF16) return noalloc_bad("unknown precision selector");
  if (flags & (B2_FLAG_USE_PARAM_INFO_GAIN | B2_FLAG_USE_INDUCTIVE))
    return fail(B2_ERR_UNSUPPORTED,
                std::string(kNoAllocName) + ": only the utility and state-information-gain terms are built");
  if (((flags >> B2_PRECISION_SHIFT) & 3) != B2_PRECISION_FP32)
    return fail(B2_ERR_UNSUPPORTED, std::string(kNoAllocName) + ": only B2_PRECISION_FP32 is available here");
  if (Bn == 0) return B2_OK;
  if (!policy_matrix || !qs_init || !A || !B || !C || !neg_efe_out) return noalloc_bad("null buffer");
  if (Bn > 65535) return fail(B2_ERR_UNSUPPORTED, std::string(kNoAllocName) + ": Bn > 65535");
  const uint64_t need = (uint64_t)Bn * (uint64_t)p.T * (uint64_t)p.K_tot * sizeof(float);
  if (need > kNoAllocScratchBytes)
    return fail(B2_ERR_UNSUPPORTED, std::string(kNoAllocName) + ": needs " + std::to_string(need) +
                                        " bytes of scratch (Bn * T * sum_m K_m floats); the fixed scratch holds " +
                                        std::to_string(kNoAllocScratchBytes) +
                                        " bytes. Split the batch or use b2_neg_efe");
  (void)I;
  (void)pA;
  (void)pB;
  (void)inductive_epsilon;
  float* lin = nullptr;
  B2_TRY(scratch_for_current_device(&lin));
  B2_TRY(launch_linear_rows(p, Bn, A, C, lin, stream));
  return launch_efe_plain(p, Bn, policy_matrix, pm_batched, qs_init, A, B, lin, neg_efe_out, stream);
}
