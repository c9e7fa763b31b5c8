// Kernel-parameter layout shared by the EFE kernels.
#pragma once

#include <cstring>

#include "common.cuh"

namespace b2 {

constexpr int kEfeMaxF = B2_MAX_FACTORS;

// The action index as jnp indexing reads B_f[..., u] (pymdp/control.py:386):
// a negative index counts from the end, then an out-of-range index clamps to
// [0, U - 1] (JAX's gather semantics for out-of-bounds indices).
__host__ __device__ __forceinline__ int jnp_action(int u, int U) {
  if (u < 0) u += U;
  return u < 0 ? 0 : (u >= U ? U - 1 : u);
}
constexpr int kEfeMaxM = B2_MAX_MODALITIES;
constexpr int kEfePlainMaxStot = 256;  // per-policy state vector kept per thread
constexpr int kEfePlainMaxO = 128;

struct EfeFactor {
  int64_t B_off;  // offset of B_f inside one agent's flat B
  int32_t K;      // prod of parent state counts
  int32_t rank;
  int8_t dep[B2_MAX_DEP_RANK];
};

struct EfeModality {
  int64_t A_off;    // offset of A_m inside one agent's flat A
  int64_t C_off;    // offset of C_m (T, O_m) inside one agent's flat C
  int64_t lin_off;  // offset of modality m inside one (agent, t) linear row
  int32_t O, K, rank;
  int8_t dep[B2_MAX_DEP_RANK];
};

struct EfeParams {
  int32_t P, T, F, M, S_tot, flags;
  int64_t K_tot;  // sum_m K_m
  int64_t A_stride, B_stride, C_stride;
  int32_t S[kEfeMaxF];
  int32_t U[kEfeMaxF];
  int32_t qs_off[kEfeMaxF + 1];
  int32_t I_off[kEfeMaxF + 1];  // inductive matrix I_f (depth_f, S_f) inside one agent's flat I
  int32_t I_depth[kEfeMaxF];
  int64_t I_stride;
  EfeFactor fac[kEfeMaxF];
  EfeModality mod[kEfeMaxM];
};

extern const char* const kEfeName;

int32_t build_efe_params(EfeParams* p, int64_t P, int64_t T, int64_t F, int64_t M, const int64_t* S,
                         const int64_t* O, const int64_t* U, const int64_t* qs_offsets, const int64_t* A_offsets,
                         const int64_t* B_offsets, const int64_t* C_offsets, const int64_t* I_offsets,
                         const int64_t* I_depths, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                         const int64_t* A_dep_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                         const int64_t* B_dep_offsets, int32_t flags);

int32_t launch_linear_rows(const EfeParams& p, int64_t Bn, const float* A, const float* C, float* lin,
                           cudaStream_t stream);
int32_t launch_efe_plain(const EfeParams& p, int64_t Bn, const int32_t* pm, int pm_batched, const float* qs,
                         const float* A, const float* B, const float* lin, float* G, cudaStream_t stream,
                         const float* wA = nullptr, const float* wB = nullptr, const float* wI = nullptr);
int32_t ws_alloc(void** ptr, size_t bytes, cudaStream_t stream, const char* op);
// Tensor-core path (efe_tc.cu); *used = false when the model is outside its
// limits and nothing was launched.
// Small-model path (efe_small.cu): one CTA per agent with every policy's
// roll-out in shared memory; used when that working set fits kEfeSmallMaxSmem.
constexpr int64_t kEfeSmallMaxSmem = 96 * 1024;
int64_t efe_small_smem_bytes(const EfeParams& p);
int32_t launch_efe_small(const EfeParams& p, int64_t Bn, bool bwd, const int32_t* pm, int pm_batched,
                         const float* qs, const float* A, const float* B, const float* C, float* G, const float* dG,
                         float* dqs, float* dA, float* dB, float* dC, cudaStream_t stream, bool* used);

// Caller-owned cache of the tensor-core operand images (b2_neg_efe_cached).
struct PackCache {
  uint8_t* buf;
  int64_t bytes;
  int32_t* valid;  // host flag: 0 = pack into buf (then set to 1), 1 = reuse
};
int32_t launch_efe_tc(const EfeParams& p, int prec, int64_t Bn, const int32_t* pm, int pm_batched, const float* qs,
                      const float* A, const float* B, const float* C, float* G, cudaStream_t stream, bool* used,
                      const PackCache* cache = nullptr);
// Factored path (efe_fact.cu): the contraction factor by factor over the
// distinct per-factor marginals of the policy tree; *used = false when the
// model is outside it (transitions not factor-local, a dependency tuple of
// rank above 3, a factor above 64 states, ...) and nothing was launched.
// wA / wB / wI: the parameter-information-gain weights (laid out like A / B)
// and the inductive weights per factor state (efe_wnorm_kernel,
// efe_inductive_kernel), null when the term is off.
int32_t launch_efe_fact(const EfeParams& p, int64_t Bn, const float* qs, const float* A, const float* B,
                        const float* C, float* G, cudaStream_t stream, bool* used, const float* wA = nullptr,
                        const float* wB = nullptr, const float* wI = nullptr);
bool efe_fact_applies(const EfeParams& p, int64_t Bn);
// Bytes of the tensor-core operand images for Bn agents at precision prec
// (0 when the model takes the SIMT path).
int64_t efe_tc_pack_bytes(const EfeParams& p, int prec, int64_t Bn);

}  // namespace b2
