// Error plumbing, launch accounting and small exported entry points.
#include <map>
#include <mutex>
#include <utility>

#include "common.cuh"

namespace b2 {

namespace {
thread_local std::string g_last_error;
std::atomic<uint64_t> g_launches{0};
std::mutex g_attr_mu;
std::map<std::pair<const void*, int>, int> g_attr_bytes;  // (kernel, device) -> bytes opted in
}  // namespace

int32_t fail(int32_t code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int32_t cuda_fail(const char* op, cudaError_t err) {
  const int32_t code = (err == cudaErrorNoKernelImageForDevice || err == cudaErrorNoDevice ||
                        err == cudaErrorInsufficientDriver)
                           ? B2_ERR_NO_DEVICE
                           : B2_ERR_CUDA;
  return fail(code, std::string(op) + ": CUDA error " + cudaGetErrorName(err) + ": " + cudaGetErrorString(err));
}

void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

int32_t ensure_smem_attr(const void* kernel, int bytes, const char* op) {
  int dev = 0;
  B2_CUDA_TRY(op, cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_attr_mu);
  int& have = g_attr_bytes[{kernel, dev}];
  if (bytes <= have) return B2_OK;
  if (bytes > 48 * 1024) {
    B2_CUDA_TRY(op, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  }
  have = bytes;
  return B2_OK;
}

}  // namespace b2

extern "C" const char* b2_last_error(void) { return b2::g_last_error.c_str(); }

extern "C" int32_t b2_abi_version(void) { return 1; }

extern "C" int32_t b2_capabilities(void) { return 1 << 2; }

extern "C" uint64_t b2_launch_count(void) { return b2::g_launches.load(std::memory_order_relaxed); }
