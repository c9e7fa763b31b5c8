// The agent loop's glue between steps, on the GPU:
//  * b2_expected_state: the empirical prior of the next step,
//    Agent.update_empirical_prior (pymdp/agent.py:825-851) =
//    compute_expected_state (pymdp/control.py:351-389) on the last posterior
//    and the sampled action, batched over agents.
//  * b2_multiaction_probabilities: Agent.multiaction_probabilities
//    (pymdp/agent.py:908-937): probabilities of the unique first-step joint
//    actions, by summing q_pi over the policies that start with each one
//    ("full") or as the outer product of the per-factor action marginals
//    (get_marginals, pymdp/control.py:42-67; "marginal").
#include <string>

#include "common.cuh"
#include "efe.cuh"

namespace b2 {
namespace {

constexpr int kPriorMaxF = B2_MAX_FACTORS;

struct PriorParams {
  int32_t F, S_tot;
  int32_t S[kPriorMaxF], U[kPriorMaxF];
  int32_t qs_off[kPriorMaxF + 1];
  int64_t B_off[kPriorMaxF + 1];
  int32_t K[kPriorMaxF], rank[kPriorMaxF];
  int8_t dep[kPriorMaxF][B2_MAX_DEP_RANK];
};

// One thread per (agent, factor state): sum_k B_f[s, k, u] prod_i q_{dep_i}[digit_i(k)],
// the parents' joint in row-major order over B_dependencies[f] (the flattening
// of B_f's parent axes), u read as jnp indexing reads B_f[..., u].
__global__ void expected_state_kernel(const __grid_constant__ PriorParams p, const float* __restrict__ qs,
                                      const float* __restrict__ B, const int32_t* __restrict__ action,
                                      float* __restrict__ out, int64_t Bn) {
  const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= Bn * p.S_tot) return;
  const int64_t b = e / p.S_tot;
  const int j = (int)(e - b * p.S_tot);
  int f = 0;
  while (f + 1 < p.F && j >= p.qs_off[f + 1]) ++f;
  const int s = j - p.qs_off[f], U = p.U[f], K = p.K[f];
  const int u = jnp_action(action[b * p.F + f], U);
  const float* q = qs + b * p.S_tot;
  const float* Bs = B + b * p.B_off[p.F] + p.B_off[f] + (int64_t)s * K * U + u;
  int dig[B2_MAX_DEP_RANK];
  for (int i = 0; i < B2_MAX_DEP_RANK; ++i) dig[i] = 0;
  float acc = 0.f;
  for (int k = 0; k < K; ++k) {
    float w = 1.f;
    for (int i = 0; i < p.rank[f]; ++i) w *= q[p.qs_off[p.dep[f][i]] + dig[i]];
    acc = fmaf(__ldg(Bs + (int64_t)k * U), w, acc);
    for (int i = p.rank[f] - 1; i >= 0; --i) {
      if (++dig[i] < p.S[p.dep[f][i]]) break;
      dig[i] = 0;
    }
  }
  out[e] = acc;
}

// One CTA per agent. full: thread per unique joint action, the sum of q_pi
// over the policies whose first step is that action (in policy order, FP64);
// marginal: per-factor action marginals in shared memory, then their outer
// product in row-major factor order.
__global__ void multiaction_kernel(const float* __restrict__ q_pi, const int32_t* __restrict__ pm,
                                   const int32_t* __restrict__ uniq, int n_uniq, int marginal, int P, int T, int F,
                                   const __grid_constant__ PriorParams pp, float* __restrict__ out) {
  extern __shared__ double marg[];  // marginal mode: sum_f U_f values
  const int64_t b = blockIdx.x;
  const float* q = q_pi + b * (int64_t)P;
  if (!marginal) {
    for (int i = threadIdx.x; i < n_uniq; i += blockDim.x) {
      double acc = 0.0;
      for (int p = 0; p < P; ++p) {
        bool eq = true;
        for (int f = 0; f < F && eq; ++f) eq = pm[(int64_t)p * T * F + f] == uniq[i * F + f];
        if (eq) acc += q[p];
      }
      out[b * n_uniq + i] = (float)acc;
    }
    return;
  }
  int off[kPriorMaxF + 1];
  off[0] = 0;
  for (int f = 0; f < F; ++f) off[f + 1] = off[f] + pp.U[f];
  for (int e = threadIdx.x; e < off[F]; e += blockDim.x) {
    int f = 0;
    while (e >= off[f + 1]) ++f;
    const int a = e - off[f];
    double acc = 0.0;
    for (int p = 0; p < P; ++p)
      if (pm[(int64_t)p * T * F + f] == a) acc += q[p];
    marg[e] = acc;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n_uniq; i += blockDim.x) {
    int rem = i;
    double v = 1.0;
    for (int f = F - 1; f >= 0; --f) {
      const int a = rem % pp.U[f];
      rem /= pp.U[f];
      v *= marg[off[f] + a];
    }
    out[b * n_uniq + i] = (float)v;
  }
}

int32_t build_prior_params(const char* op, int64_t F, const int64_t* S, const int64_t* U, const int64_t* qs_offsets,
                           const int64_t* B_offsets, const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                           const int64_t* B_dep_offsets, PriorParams* p) {
  if (F < 1 || F > kPriorMaxF) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": F outside [1, 16]");
  if (!S || !U || !qs_offsets || !B_offsets || !B_dep_offsets || (B_dep_flat_len > 0 && !B_dep_flat))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute array");
  p->F = (int32_t)F;
  if (qs_offsets[0] != 0 || B_offsets[0] != 0 || B_dep_offsets[0] != 0)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": offsets must start at 0");
  for (int f = 0; f < F; ++f) {
    if (S[f] < 1 || U[f] < 1 || S[f] > 4096 || U[f] > 4096)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": S and U must lie in [1, 4096]");
    p->S[f] = (int32_t)S[f];
    p->U[f] = (int32_t)U[f];
    if (qs_offsets[f + 1] - qs_offsets[f] != S[f])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": qs_offsets inconsistent with S");
    const int64_t r = B_dep_offsets[f + 1] - B_dep_offsets[f];
    if (r < 1 || r > B2_MAX_DEP_RANK || B_dep_offsets[f + 1] > B_dep_flat_len)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B dependency ranks must lie in [1, 8]");
    int64_t K = 1;
    for (int64_t i = 0; i < r; ++i) {
      const int64_t d = B_dep_flat[B_dep_offsets[f] + i];
      if (d < 0 || d >= F) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B dependency out of range");
      p->dep[f][i] = (int8_t)d;
      K *= S[d];
    }
    if (K > (1 << 24)) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": B parent joint too large");
    p->rank[f] = (int32_t)r;
    p->K[f] = (int32_t)K;
    if (B_offsets[f + 1] - B_offsets[f] != S[f] * K * U[f])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_offsets inconsistent with S, U, B_dependencies");
  }
  for (int f = 0; f <= F; ++f) {
    p->qs_off[f] = (int32_t)qs_offsets[f];
    p->B_off[f] = B_offsets[f];
  }
  p->S_tot = (int32_t)qs_offsets[F];
  return B2_OK;
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_expected_state(void* stream, const float* qs, int64_t qs_count, const float* B,
                                     int64_t B_count, const int32_t* action, int64_t action_count, float* out,
                                     int64_t Bn, int64_t F, const int64_t* S, const int64_t* U,
                                     const int64_t* qs_offsets, const int64_t* B_offsets, const int64_t* B_dep_flat,
                                     int64_t B_dep_flat_len, const int64_t* B_dep_offsets) {
  const char* op = "expected_state";
  PriorParams p{};
  B2_TRY(build_prior_params(op, F, S, U, qs_offsets, B_offsets, B_dep_flat, B_dep_flat_len, B_dep_offsets, &p));
  if (Bn < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": negative Bn");
  if (qs_count != Bn * p.S_tot || B_count != Bn * p.B_off[F] || action_count != Bn * F)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": qs / B / action element counts do not match Bn");
  if (Bn == 0) return B2_OK;
  if (!qs || !B || !action || !out) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  const int64_t n = Bn * p.S_tot;
  expected_state_kernel<<<(unsigned)((n + 127) / 128), 128, 0, (cudaStream_t)stream>>>(p, qs, B, action, out, Bn);
  return check_launch(op);
}

extern "C" int32_t b2_multiaction_probabilities(void* stream, const float* q_pi, const int32_t* policy_matrix,
                                                const int32_t* unique_actions, int64_t n_unique, int32_t marginal,
                                                int64_t Bn, int64_t P, int64_t T, int64_t F, const int64_t* U,
                                                float* out) {
  const char* op = "multiaction_probabilities";
  if (Bn < 0 || P < 1 || T < 1 || F < 1 || F > kPriorMaxF || n_unique < 1 || !U)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (P > 0x7fffffff || n_unique > 0x7fffffff || Bn > 0x7fffffff)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": sizes above 2^31");
  PriorParams pp{};
  int64_t nu = 1;
  for (int f = 0; f < F; ++f) {
    if (U[f] < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": U must be positive");
    pp.U[f] = (int32_t)U[f];
    nu *= U[f];
  }
  if (marginal && n_unique != nu)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": marginal mode writes prod(U) probabilities");
  if (Bn == 0) return B2_OK;
  if (!q_pi || !policy_matrix || !out || (!marginal && !unique_actions))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  int64_t su = 0;
  for (int f = 0; f < F; ++f) su += U[f];
  const size_t smem = marginal ? (size_t)su * sizeof(double) : 0;
  if (smem > 48 * 1024) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too many controls");
  multiaction_kernel<<<(unsigned)Bn, 128, smem, (cudaStream_t)stream>>>(q_pi, policy_matrix, unique_actions,
                                                                       (int)n_unique, marginal, (int)P, (int)T,
                                                                       (int)F, pp, out);
  return check_launch(op);
}
