// C entry points over the reference's own CPU FFI handlers, compiled from
// the reference's sources with the project-written xla::ffi stand-in in
// ./include. Test infrastructure: the CPU timing baseline and a cross-check,
// never part of the product path.
//
//   ref_neg_efe_cpu -> pymdp_ffi::NegEfeCpu (pymdp/ffi/neg_efe/neg_efe_cpu_entry.cc:25-117)
//   ref_fpi_cpu     -> pymdp_ffi::FpiCpu    (pymdp/ffi/fpi/fpi_cpu_runner.cc:110-117)
//
// Buffers are host arrays. Every buffer is passed with its dimensions,
// because the handlers read the batch from the policy matrix's rank
// (pymdp/ffi/neg_efe/neg_efe_layout.h:194-209) and the epsilon layout from
// its rank. Attribute spans are (pointer, length) pairs in the reference's
// order. Returns 0 on success, else the handler's error code, with the
// message in ref_last_error().
#include <cstdint>
#include <string>

#include "fpi/fpi.h"
#include "neg_efe/neg_efe.h"

namespace {
thread_local std::string g_err;

int finish(const xla::ffi::Error& e) {
  if (e.success()) return 0;
  g_err = e.message();
  return static_cast<int>(e.errc());
}

pymdp_ffi::FfiInt64Span span(const int64_t* p, int64_t n) { return pymdp_ffi::FfiInt64Span(p, (size_t)n); }
}  // namespace

extern "C" const char* ref_last_error(void) { return g_err.c_str(); }

extern "C" int ref_neg_efe_cpu(const int32_t* pm, const int64_t* pm_dims, int32_t pm_rank,  //
                               const float* qs, int64_t qs_n, const float* A, int64_t A_n, const float* B, int64_t B_n,
                               const float* C, int64_t C_n, const float* I, int64_t I_n, const float* pA,
                               int64_t pA_n, const float* pB, int64_t pB_n, const float* eps,
                               const int64_t* eps_dims, int32_t eps_rank, float* out, int64_t out_n,
                               const int64_t* const* spans, const int64_t* span_lens, int32_t flags) {
  using namespace xla::ffi;
  using F32 = Buffer<DataType::F32>;
  using S32 = Buffer<DataType::S32>;
  auto flat = [](const float* p, const int64_t* n) { return F32(const_cast<float*>(p), n, 1); };
  const int64_t zero = 0;
  return finish(pymdp_ffi::NegEfeCpu(
      S32(const_cast<int32_t*>(pm), pm_dims, (size_t)pm_rank), flat(qs, &qs_n), flat(A, &A_n), flat(B, &B_n),
      flat(C, &C_n), flat(I, &I_n), pA ? flat(pA, &pA_n) : flat(nullptr, &zero),
      pB ? flat(pB, &pB_n) : flat(nullptr, &zero), F32(const_cast<float*>(eps), eps_dims, (size_t)eps_rank),
      Result<F32>(F32(out, &out_n, 1)), span(spans[0], span_lens[0]), span(spans[1], span_lens[1]),
      span(spans[2], span_lens[2]), span(spans[3], span_lens[3]), span(spans[4], span_lens[4]),
      span(spans[5], span_lens[5]), span(spans[6], span_lens[6]), span(spans[7], span_lens[7]),
      span(spans[8], span_lens[8]), span(spans[9], span_lens[9]), span(spans[10], span_lens[10]),
      span(spans[11], span_lens[11]), span(spans[12], span_lens[12]), flags));
}

extern "C" int ref_fpi_cpu(const float* ll, int64_t ll_n, const float* lp, int64_t lp_n, float* q, int64_t q_n,
                           const int64_t* const* spans, const int64_t* span_lens, int32_t num_iter) {
  using namespace xla::ffi;
  using F32 = Buffer<DataType::F32>;
  return finish(pymdp_ffi::FpiCpu(F32(const_cast<float*>(ll), &ll_n, 1), F32(const_cast<float*>(lp), &lp_n, 1),
                                  Result<F32>(F32(q, &q_n, 1)), span(spans[0], span_lens[0]),
                                  span(spans[1], span_lens[1]), span(spans[2], span_lens[2]),
                                  span(spans[3], span_lens[3]), span(spans[4], span_lens[4]), num_iter));
}
