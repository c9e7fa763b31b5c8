// Project-written stand-in for the few `xla::ffi` types that the reference's
// CPU kernels use (pymdp/ffi/common/error_helpers.h:16-20): Error and
// ErrorCode, Buffer<F32> / Buffer<S32> (typed_data, element_count,
// dimensions), Result<Buffer> (pointer-like access to the output buffer) and
// Span<const int64_t>. It lets the reference's NegEfeCpu
// (pymdp/ffi/neg_efe/neg_efe_cpu_entry.cc) and FpiCpu
// (pymdp/ffi/fpi/fpi_cpu_runner.cc) be compiled unchanged from their own
// sources as a CPU timing baseline and cross-check. It is NOT jaxlib's header
// and implements only what those sources call.
//
// Test infrastructure: only the checker / CPU-baseline legs load the library
// built from it.
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <utility>

namespace xla {
namespace ffi {

enum class ErrorCode : int32_t { kOk = 0, kInvalidArgument = 3, kInternal = 13, kUnimplemented = 12 };

class Error {
 public:
  Error() = default;
  Error(ErrorCode code, std::string message) : code_(code), message_(std::move(message)) {}
  static Error Success() { return Error(); }
  bool success() const { return code_ == ErrorCode::kOk; }
  bool failure() const { return code_ != ErrorCode::kOk; }
  ErrorCode errc() const { return code_; }
  const std::string& message() const { return message_; }

 private:
  ErrorCode code_ = ErrorCode::kOk;
  std::string message_;
};

template <typename T>
class Span {
 public:
  Span() = default;
  Span(T* data, size_t size) : data_(data), size_(size) {}
  T* begin() const { return data_; }
  T* end() const { return data_ + size_; }
  size_t size() const { return size_; }
  bool empty() const { return size_ == 0; }
  T& operator[](size_t i) const { return data_[i]; }
  T& front() const { return data_[0]; }
  T& back() const { return data_[size_ - 1]; }
  T* data() const { return data_; }

 private:
  T* data_ = nullptr;
  size_t size_ = 0;
};

enum class DataType { F32, S32 };
constexpr DataType F32 = DataType::F32;
constexpr DataType S32 = DataType::S32;

template <DataType D>
struct NativeType;
template <>
struct NativeType<DataType::F32> {
  using type = float;
};
template <>
struct NativeType<DataType::S32> {
  using type = int32_t;
};

// A dense buffer: data pointer plus its dimensions (row-major).
template <DataType D>
class Buffer {
 public:
  using T = typename NativeType<D>::type;
  Buffer() = default;
  Buffer(T* data, const int64_t* dims, size_t rank) : data_(data), dims_(dims, rank) {
    count_ = 1;
    for (size_t i = 0; i < rank; ++i) count_ *= (size_t)dims[i];
  }
  T* typed_data() const { return data_; }
  void* untyped_data() const { return data_; }
  size_t element_count() const { return count_; }
  Span<const int64_t> dimensions() const { return dims_; }

 private:
  T* data_ = nullptr;
  Span<const int64_t> dims_;
  size_t count_ = 0;
};

// The handler's output: pointer-like access to the buffer it writes.
template <typename B>
class Result {
 public:
  explicit Result(B buf) : buf_(buf) {}
  B* operator->() { return &buf_; }
  const B* operator->() const { return &buf_; }
  B& operator*() { return buf_; }

 private:
  B buf_;
};

}  // namespace ffi
}  // namespace xla
