// Adjoint of the neg-EFE evaluation (utility + state information gain), for
// gradients of a loss on G with respect to qs_init, A, B and C.
//
// The reference differentiates its JAX path (pymdp/ffi/_core.py:282-310
// `with_jax_grad`, i.e. jax.grad of pymdp/control.py:604-690); its native
// kernels have no backward. This file is the hand-written reverse pass of the
// same arithmetic. With x_t = outer product of the step-t predicted marginals,
//   G = sum_t sum_m [ -sum_o qo log clip qo + sum_k x[k] lin_t[k] ],
//   qo = A_m x, lin_t[k] = sum_o A[o,k] (log clip A[o,k] [ig] + C_t[o] [ut]),
// and the JAX derivative of x log clip(x) being log clip(x) + [x >= eps]:
//   dG/dqo[o]   = -(log clip qo[o] + [qo[o] >= eps])                 (ig)
//   dG/dx[k]    = sum_o A[o,k] dG/dqo[o] + lin_t[k]
//   dG/dA[o,k] += x[k] (dG/dqo[o] + ig (log clip A + [A >= eps]) + ut C_t[o])
//   dG/dC_t[o] += qo[o]                                              (ut)
// then back through x = prod of marginals and the rollout
// qs_{t+1, f} = B_f[..., u_t] . (outer product of qs_t over B_deps[f]).
// One thread per (agent, policy): it recomputes its rollout, walks the steps
// backwards and adds w * (its gradient) into the per-agent outputs with
// atomics, w = dL/dG for that policy.
#include <string>
#include <vector>

#include "common.cuh"
#include "efe.cuh"

namespace b2 {
namespace {

constexpr int kBwdMaxHist = 1024;  // (T + 1) * S_tot floats of rollout history per thread
constexpr float kEps = 2.220446049250313e-16f;

// x[k] and, for axis j, the product of the other marginals at k.
__device__ __forceinline__ void digits_of(int k, const int8_t* dep, int rank, const int32_t* S, int* dig) {
  for (int i = rank - 1; i >= 0; --i) {
    const int d = S[dep[i]];
    const int q = k / d;
    dig[i] = k - q * d;
    k = q;
  }
}

__global__ void __launch_bounds__(128)
    efe_bwd_kernel(const __grid_constant__ EfeParams p, const int32_t* __restrict__ pm, int pm_batched,
                   const float* __restrict__ qs_init, const float* __restrict__ A, const float* __restrict__ B,
                   const float* __restrict__ C, const float* __restrict__ dG, float* __restrict__ dqs,
                   float* __restrict__ dA, float* __restrict__ dB, float* __restrict__ dC) {
  const int64_t b = blockIdx.y;
  const int pol = blockIdx.x * blockDim.x + threadIdx.x;
  if (pol >= p.P) return;
  const float w = dG[b * p.P + pol];
  if (w == 0.f) return;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const bool ut = (p.flags & B2_FLAG_USE_UTILITY) != 0;
  const int32_t* u_pol = pm + (pm_batched ? b * (int64_t)p.P * p.T * p.F : 0) + (int64_t)pol * p.T * p.F;
  const float* Ab = A + b * p.A_stride;
  const float* Bb = B + b * p.B_stride;
  const float* Cb = C + b * p.C_stride;
  float* dAb = dA + b * p.A_stride;
  float* dBb = dB + b * p.B_stride;
  float* dCb = dC + b * p.C_stride;

  // forward: rollout history hist[t] = qs_t, t = 0..T
  float hist[kBwdMaxHist];
  const int St = p.S_tot;
  for (int i = 0; i < St; ++i) hist[i] = __ldg(qs_init + b * St + i);
  for (int t = 0; t < p.T; ++t) {
    const float* qc = hist + t * St;
    float* qn = hist + (t + 1) * St;
    for (int f = 0; f < p.F; ++f) {
      const EfeFactor& fb = p.fac[f];
      const int U = p.U[f], u = jnp_action(u_pol[t * p.F + f], U);
      const float* Bf = Bb + fb.B_off;
      for (int s = 0; s < p.S[f]; ++s) {
        float acc = 0.f;
        int dig[B2_MAX_DEP_RANK];
        for (int k = 0; k < fb.K; ++k) {
          digits_of(k, fb.dep, fb.rank, p.S, dig);
          float x = 1.f;
          for (int i = 0; i < fb.rank; ++i) x *= qc[p.qs_off[fb.dep[i]] + dig[i]];
          acc = fmaf(__ldg(Bf + ((int64_t)s * fb.K + k) * U + u), x, acc);
        }
        qn[p.qs_off[f] + s] = acc;
      }
    }
  }

  // backward
  float gq[kEfePlainMaxStot];   // dG/dqs_{t+1}
  float gqp[kEfePlainMaxStot];  // dG/dqs_t
  float qo[kEfePlainMaxO], gqo[kEfePlainMaxO];
  for (int i = 0; i < St; ++i) gq[i] = 0.f;
  for (int t = p.T - 1; t >= 0; --t) {
    const float* q = hist + (t + 1) * St;
    // step-t terms on qs_{t+1}
    for (int m = 0; m < p.M; ++m) {
      const EfeModality& md = p.mod[m];
      const float* Am = Ab + md.A_off;
      const float* Cm = Cb + md.C_off + (int64_t)t * md.O;
      int dig[B2_MAX_DEP_RANK];
      for (int o = 0; o < md.O; ++o) qo[o] = 0.f;
      for (int k = 0; k < md.K; ++k) {
        digits_of(k, md.dep, md.rank, p.S, dig);
        float x = 1.f;
        for (int i = 0; i < md.rank; ++i) x *= q[p.qs_off[md.dep[i]] + dig[i]];
        for (int o = 0; o < md.O; ++o) qo[o] = fmaf(__ldg(Am + (int64_t)o * md.K + k), x, qo[o]);
      }
      for (int o = 0; o < md.O; ++o) {
        gqo[o] = ig ? -(log_stable(qo[o]) + (qo[o] >= kEps ? 1.f : 0.f)) : 0.f;
        if (ut) atomicAdd(dCb + md.C_off + (int64_t)t * md.O + o, w * qo[o]);
      }
      for (int k = 0; k < md.K; ++k) {
        digits_of(k, md.dep, md.rank, p.S, dig);
        float x = 1.f;
        for (int i = 0; i < md.rank; ++i) x *= q[p.qs_off[md.dep[i]] + dig[i]];
        float gx = 0.f;
        for (int o = 0; o < md.O; ++o) {
          const float a = __ldg(Am + (int64_t)o * md.K + k);
          const float la = (ig ? log_stable(a) : 0.f) + (ut ? __ldg(Cm + o) : 0.f);  // lin_t contribution
          gx = fmaf(a, gqo[o] + la, gx);
          const float ga = gqo[o] + la + (ig && a >= kEps ? 1.f : 0.f);
          atomicAdd(dAb + md.A_off + (int64_t)o * md.K + k, w * x * ga);
        }
        // back through x = prod_i q_{dep i}[dig i]
        for (int j = 0; j < md.rank; ++j) {
          float other = 1.f;
          for (int i = 0; i < md.rank; ++i)
            if (i != j) other *= q[p.qs_off[md.dep[i]] + dig[i]];
          gq[p.qs_off[md.dep[j]] + dig[j]] += gx * other;
        }
      }
    }
    // back through the rollout qs_{t+1} = B(u_t) . qs_t
    const float* qc = hist + t * St;
    for (int i = 0; i < St; ++i) gqp[i] = 0.f;
    for (int f = 0; f < p.F; ++f) {
      const EfeFactor& fb = p.fac[f];
      const int U = p.U[f], u = jnp_action(u_pol[t * p.F + f], U);
      const float* Bf = Bb + fb.B_off;
      float* dBf = dBb + fb.B_off;
      int dig[B2_MAX_DEP_RANK];
      for (int k = 0; k < fb.K; ++k) {
        digits_of(k, fb.dep, fb.rank, p.S, dig);
        float x = 1.f;
        for (int i = 0; i < fb.rank; ++i) x *= qc[p.qs_off[fb.dep[i]] + dig[i]];
        float gx = 0.f;
        for (int s = 0; s < p.S[f]; ++s) {
          const float g = gq[p.qs_off[f] + s];
          const int64_t e = ((int64_t)s * fb.K + k) * U + u;
          gx = fmaf(__ldg(Bf + e), g, gx);
          if (g != 0.f) atomicAdd(dBf + e, w * g * x);
        }
        for (int j = 0; j < fb.rank; ++j) {
          float other = 1.f;
          for (int i = 0; i < fb.rank; ++i)
            if (i != j) other *= qc[p.qs_off[fb.dep[i]] + dig[i]];
          gqp[p.qs_off[fb.dep[j]] + dig[j]] += gx * other;
        }
      }
    }
    for (int i = 0; i < St; ++i) gq[i] = gqp[i];
  }
  for (int i = 0; i < St; ++i)
    if (gq[i] != 0.f) atomicAdd(dqs + b * St + i, w * gq[i]);
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_neg_efe_bwd(void* stream_, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                                  const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                                  const float* B, int64_t B_count, const float* C, int64_t C_count,
                                  const float* d_neg_efe, int64_t dG_count, float* d_qs_init, float* d_A,
                                  float* d_B, float* d_C, int64_t Bn, int64_t P, int64_t T, int64_t F, int64_t M,
                                  const int64_t* S, const int64_t* O, const int64_t* U, const int64_t* qs_offsets,
                                  const int64_t* A_offsets, const int64_t* B_offsets, const int64_t* C_offsets,
                                  const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets,
                                  const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets,
                                  int32_t flags) {
  const char* op = "efe_ffi bwd";
  cudaStream_t stream = (cudaStream_t)stream_;
  if (Bn < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": negative Bn");
  if (flags & (B2_FLAG_USE_INDUCTIVE | B2_FLAG_USE_PARAM_INFO_GAIN))
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": only the utility and state-information-gain terms");
  // I is not used by these terms: a depth-1 layout of zeros
  std::vector<int64_t> I_off(F + 1), I_dep(F, 1);
  I_off[0] = 0;
  for (int64_t f = 0; f < F && S; ++f) I_off[f + 1] = I_off[f] + S[f];
  EfeParams p;
  B2_TRY(build_efe_params(&p, P, T, F, M, S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_off.data(),
                          I_dep.data(), A_dep_flat, A_dep_flat_len, A_dep_offsets, B_dep_flat, B_dep_flat_len,
                          B_dep_offsets, flags & 3));
  const struct {
    const char* name;
    int64_t actual, expected;
  } chks[] = {
      {"policy_matrix", pm_count, (pm_batched ? Bn : 1) * P * T * F},
      {"qs_init", qs_count, Bn * (int64_t)p.S_tot},
      {"A", A_count, Bn * p.A_stride},
      {"B", B_count, Bn * p.B_stride},
      {"C", C_count, Bn * p.C_stride},
      {"d_neg_efe", dG_count, Bn * P},
  };
  for (const auto& c : chks)
    if (c.actual != c.expected)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": " + c.name + " element_count = " +
                                               std::to_string(c.actual) + ", expected " + std::to_string(c.expected));
  const bool small = efe_small_smem_bytes(p) <= kEfeSmallMaxSmem;
  if (!small && (int64_t)(T + 1) * p.S_tot > kBwdMaxHist)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": (T + 1) * total states exceeds " +
                                        std::to_string(kBwdMaxHist));
  if (Bn == 0) return B2_OK;
  if (!policy_matrix || !qs_init || !A || !B || !C || !d_neg_efe || !d_qs_init || !d_A || !d_B || !d_C)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  if (Bn > 65535) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": Bn > 65535");
  // outputs accumulate with atomics: start from zero
  B2_CUDA_TRY(op, cudaMemsetAsync(d_qs_init, 0, (size_t)Bn * p.S_tot * sizeof(float), stream));
  B2_CUDA_TRY(op, cudaMemsetAsync(d_A, 0, (size_t)Bn * p.A_stride * sizeof(float), stream));
  B2_CUDA_TRY(op, cudaMemsetAsync(d_B, 0, (size_t)Bn * p.B_stride * sizeof(float), stream));
  B2_CUDA_TRY(op, cudaMemsetAsync(d_C, 0, (size_t)Bn * p.C_stride * sizeof(float), stream));
  if (small) {
    bool used = false;
    B2_TRY(launch_efe_small(p, Bn, true, policy_matrix, pm_batched, qs_init, A, B, C, nullptr, d_neg_efe, d_qs_init,
                            d_A, d_B, d_C, stream, &used));
    if (used) return B2_OK;
  }
  dim3 grid((unsigned)((P + 127) / 128), (unsigned)Bn);
  efe_bwd_kernel<<<grid, 128, 0, stream>>>(p, policy_matrix, pm_batched, qs_init, A, B, C, d_neg_efe, d_qs_init,
                                           d_A, d_B, d_C);
  return check_launch(op);
}
