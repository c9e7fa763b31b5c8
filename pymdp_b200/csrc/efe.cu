// Expected free energy (neg-EFE, "G") over all policies — reference-ABI entry,
// validation, the per-(agent, policy) SIMT FP32 kernel, and the policy
// posterior / action-selection kernels.
//
// Semantics: pymdp/control.py:604-690 (compute_neg_efe_policy) vmapped over
// policies (control.py:347), i.e. for each policy, from G = 0 and qs = qs_init:
//   for t < T: qs_f <- factor_dot(B_f[..., u_{t,f}], qs[B_deps[f]])   (:351-389)
//              qo_m  = factor_dot(A_m, qs[A_deps[m]])                  (:420-447)
//              G    += sum_m [ H(qo_m) - H_A_m . x_m ]   (if states info gain, :449-481)
//                    + sum_m qo_m . C_m[t]               (if utility, :483-509)
// with x_m = outer product of the dependency marginals and
// H_A_m[k] = -sum_o A_m[o,k] log(clip(A_m[o,k])).
//
// Both linear terms collapse into one per-(t, m) row computed once per agent
// (the reference's own trick, neg_efe_cuda_kernels.cu:1426-1445):
//   lin[t,m,k] = sum_o A_m[o,k] * (log(clip(A_m[o,k])) [ig] + C_m[t,o] [util])
// so the only per-policy nonlinearity is H(qo_m).
#include <mutex>
#include <set>
#include <string>
#include <vector>

#include "common.cuh"
#include "efe.cuh"

namespace b2 {

const char* const kEfeName = "efe_ffi";

namespace {

int32_t bad(const std::string& msg) { return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": " + msg); }

}  // namespace

// Mirrors parse_call_shape / validate_attr_spans / validate_layout /
// validate_buffer_counts (pymdp/ffi/neg_efe/neg_efe_layout.h:209-363).
int32_t build_efe_params(EfeParams* p, int64_t P, int64_t T, int64_t F, int64_t M, const int64_t* S,
                         const int64_t* O, const int64_t* U, const int64_t* qs_offsets,
                         const int64_t* A_offsets, const int64_t* B_offsets, const int64_t* C_offsets,
                         const int64_t* I_offsets, const int64_t* I_depths, const int64_t* A_dep_flat,
                         int64_t A_dep_flat_len, const int64_t* A_dep_offsets, const int64_t* B_dep_flat,
                         int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int32_t flags) {
  std::memset(p, 0, sizeof(*p));
  if (!S || !O || !U || !qs_offsets || !A_offsets || !B_offsets || !C_offsets || !I_offsets || !I_depths ||
      !A_dep_flat || !A_dep_offsets || !B_dep_flat || !B_dep_offsets)
    return bad("null attribute array");
  if (F <= 0 || M <= 0 || P <= 0 || T <= 0) return bad("F/M/P/T must all be positive");
  if (F > kEfeMaxF || M > kEfeMaxM)
    return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": F or M exceeds this build's limits");
  if (P > 0x7fffffff / 4 || T > 64) return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": P or T too large");
  if (qs_offsets[0] != 0 || A_offsets[0] != 0 || B_offsets[0] != 0 || C_offsets[0] != 0 || I_offsets[0] != 0 ||
      A_dep_offsets[0] != 0 || B_dep_offsets[0] != 0)
    return bad("offset tables must start at zero");
  if (A_dep_flat_len != A_dep_offsets[M]) return bad("A_dep_flat size inconsistent with A_dep_offsets");
  if (B_dep_flat_len != B_dep_offsets[F]) return bad("B_dep_flat size inconsistent with B_dep_offsets");
  p->P = (int32_t)P;
  p->T = (int32_t)T;
  p->F = (int32_t)F;
  p->M = (int32_t)M;
  p->flags = flags;
  uint64_t total_actions = 1;
  for (int64_t f = 0; f < F; ++f) {
    if (S[f] <= 0 || U[f] <= 0) return bad("S[f] and U[f] must be positive");
    if (total_actions > 0xffffffffull / (uint64_t)U[f])
      return bad("action encoding overflows 32 bits (prod(U[f]) > UINT32_MAX)");
    total_actions *= (uint64_t)U[f];
    if (qs_offsets[f + 1] < qs_offsets[f]) return bad("qs_off must be monotonic");
    if (qs_offsets[f + 1] - qs_offsets[f] != S[f]) return bad("qs_off inconsistent with S");
    if (B_offsets[f + 1] < B_offsets[f]) return bad("B_off must be monotonic");
    if (B_dep_offsets[f + 1] < B_dep_offsets[f]) return bad("B_dep_off must be monotonic");
    const int64_t r = B_dep_offsets[f + 1] - B_dep_offsets[f];
    if (r < 1 || r > B2_MAX_DEP_RANK) return bad("B_dep rank of factor " + std::to_string(f) + " outside [1, 8]");
    EfeFactor& fb = p->fac[f];
    fb.rank = (int32_t)r;
    int64_t K = 1;
    for (int64_t i = 0; i < r; ++i) {
      const int64_t d = B_dep_flat[B_dep_offsets[f] + i];
      if (d < 0 || d >= F) return bad("B_dep factor index out of range");
      fb.dep[i] = (int8_t)d;
      K *= S[d];
    }
    if (B_offsets[f + 1] - B_offsets[f] != S[f] * K * U[f]) return bad("B_off inconsistent with S/U/deps");
    fb.K = (int32_t)K;
    fb.B_off = B_offsets[f];
    p->S[f] = (int32_t)S[f];
    p->U[f] = (int32_t)U[f];
    p->qs_off[f] = (int32_t)qs_offsets[f];
  }
  p->qs_off[F] = (int32_t)qs_offsets[F];
  p->S_tot = (int32_t)qs_offsets[F];
  if (p->S_tot > kEfePlainMaxStot)
    return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": total states exceed this build's limit");
  int64_t koff = 0;
  for (int64_t m = 0; m < M; ++m) {
    if (O[m] <= 0) return bad("O[m] must be positive");
    if (A_offsets[m + 1] < A_offsets[m]) return bad("A_off must be monotonic");
    if (C_offsets[m + 1] < C_offsets[m]) return bad("C_off must be monotonic");
    if (C_offsets[m + 1] - C_offsets[m] != T * O[m]) return bad("C_off inconsistent with T/O");
    if (A_dep_offsets[m + 1] < A_dep_offsets[m]) return bad("A_dep_off must be monotonic");
    const int64_t r = A_dep_offsets[m + 1] - A_dep_offsets[m];
    if (r < 1 || r > B2_MAX_DEP_RANK) return bad("A_dep rank of modality " + std::to_string(m) + " outside [1, 8]");
    EfeModality& md = p->mod[m];
    md.rank = (int32_t)r;
    int64_t K = 1;
    for (int64_t i = 0; i < r; ++i) {
      const int64_t d = A_dep_flat[A_dep_offsets[m] + i];
      if (d < 0 || d >= F) return bad("A_dep factor index out of range");
      md.dep[i] = (int8_t)d;
      K *= S[d];
    }
    if (A_offsets[m + 1] - A_offsets[m] != O[m] * K) return bad("A_off inconsistent with O/deps");
    if (O[m] > kEfePlainMaxO)
      return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": O[m] exceeds this build's limit");
    if (K > (1 << 26)) return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": modality too large");
    md.O = (int32_t)O[m];
    md.K = (int32_t)K;
    md.A_off = A_offsets[m];
    md.C_off = C_offsets[m];
    md.lin_off = koff;
    koff += K;
  }
  p->K_tot = koff;
  for (int64_t f = 0; f < F; ++f) {
    if (I_depths[f] <= 0) return bad("I_depths[f] must be positive");
    if (I_offsets[f + 1] < I_offsets[f]) return bad("I_off must be monotonic");
    if (I_offsets[f + 1] - I_offsets[f] != I_depths[f] * S[f]) return bad("I_off inconsistent with depth/S");
    if (I_offsets[f + 1] > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": I too large");
    p->I_off[f] = (int32_t)I_offsets[f];
    p->I_depth[f] = (int32_t)I_depths[f];
  }
  p->I_off[F] = (int32_t)I_offsets[F];
  p->I_stride = I_offsets[F];
  p->A_stride = A_offsets[M];
  p->B_stride = B_offsets[F];
  p->C_stride = C_offsets[M];
  return B2_OK;
}

// ------------------------------------------------------------------ kernels
// lin[b, t, koff_m + k] for every agent, step and modality (one thread per k).
__global__ void efe_linear_rows_kernel(const __grid_constant__ EfeParams p, const float* __restrict__ A,
                                       const float* __restrict__ C, float* __restrict__ lin) {
  const int64_t b = blockIdx.z;
  const int t = blockIdx.y;
  const int64_t kk = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (kk >= p.K_tot) return;
  int m = 0;
  while (m + 1 < p.M && p.mod[m + 1].lin_off <= kk) ++m;
  const EfeModality& md = p.mod[m];
  const int64_t k = kk - md.lin_off;
  const float* Am = A + b * p.A_stride + md.A_off;
  const float* Cm = C + b * p.C_stride + md.C_off + (int64_t)t * md.O;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const bool ut = (p.flags & B2_FLAG_USE_UTILITY) != 0;
  float acc = 0.f;
  for (int o = 0; o < md.O; ++o) {
    const float a = __ldg(Am + (int64_t)o * md.K + k);
    float w = 0.f;
    if (ig) w += log_stable(a);
    if (ut) w += __ldg(Cm + o);
    acc = fmaf(a, w, acc);
  }
  lin[(b * p.T + t) * p.K_tot + kk] = acc;
}

// One thread = one (agent, policy): the plain per-policy SIMT evaluation.
// Optional terms (null pointers when unused): wA / wB = parameter
// information-gain weights (laid out like A / B, see efe_wnorm_kernel), wI =
// inductive weights per factor state (efe_inductive_kernel). Per step:
// G += info_gain + utility - (pA term + pB term) + inductive value
// (pymdp/control.py:772-787).
__global__ void __launch_bounds__(128)
    efe_plain_kernel(const __grid_constant__ EfeParams p, const int32_t* __restrict__ pm, int pm_batched,
                     const float* __restrict__ qs_init, const float* __restrict__ A, const float* __restrict__ B,
                     const float* __restrict__ lin, float* __restrict__ G, const float* __restrict__ wA,
                     const float* __restrict__ wB, const float* __restrict__ wI) {
  const int64_t b = blockIdx.y;
  const int pol = blockIdx.x * blockDim.x + threadIdx.x;
  if (pol >= p.P) return;
  float qs[2][kEfePlainMaxStot];
  float qo[kEfePlainMaxO];
  float fd[kEfePlainMaxO];  // pA term: factor_dot(wA_m, qs) per observation
  int cur = 0;
  for (int i = 0; i < p.S_tot; ++i) qs[0][i] = __ldg(qs_init + b * p.S_tot + i);
  const int32_t* u_pol = pm + (pm_batched ? b * (int64_t)p.P * p.T * p.F : 0) + (int64_t)pol * p.T * p.F;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  double g = 0.0;  // G summed over steps and terms in FP64
  for (int t = 0; t < p.T; ++t) {
    // expected states
    const float* qc = qs[cur];
    float* qn = qs[cur ^ 1];
    for (int f = 0; f < p.F; ++f) {
      const EfeFactor& fb = p.fac[f];
      const int u = jnp_action(u_pol[t * p.F + f], p.U[f]);
      const float* Bf = B + b * p.B_stride + fb.B_off;
      const float* wBf = wB ? wB + b * p.B_stride + fb.B_off : nullptr;
      const int U = p.U[f];
      for (int s = 0; s < p.S[f]; ++s) {
        float acc = 0.f, accw = 0.f;
        int dig[B2_MAX_DEP_RANK] = {0};
        for (int k = 0; k < fb.K; ++k) {
          float w = 1.f;
          for (int i = 0; i < fb.rank; ++i) w *= qc[p.qs_off[fb.dep[i]] + dig[i]];
          const int64_t e = ((int64_t)s * fb.K + k) * U + u;
          acc = fmaf(__ldg(Bf + e), w, acc);
          if (wBf) accw = fmaf(__ldg(wBf + e), w, accw);
          for (int i = fb.rank - 1; i >= 0; --i) {
            if (++dig[i] < p.S[fb.dep[i]]) break;
            dig[i] = 0;
          }
        }
        qn[p.qs_off[f] + s] = acc;
        // pB term: qs_next_f[s] * factor_dot(wB_f[..., u], qs_prev[B_deps])[s] (control.py:555-602)
        if (wBf) g -= (double)acc * accw;
      }
    }
    cur ^= 1;
    const float* q = qs[cur];
    // inductive value: linear in the predicted marginals (control.py:1021-1061)
    if (wI)
      for (int i = 0; i < p.S_tot; ++i) g += (double)__ldg(wI + b * p.S_tot + i) * q[i];
    // expected observations, entropy and the linear row
    for (int m = 0; m < p.M; ++m) {
      const EfeModality& md = p.mod[m];
      const float* Am = A + b * p.A_stride + md.A_off;
      const float* Lm = lin + (b * p.T + t) * p.K_tot + md.lin_off;
      const float* wAm = wA ? wA + b * p.A_stride + md.A_off : nullptr;
      for (int o = 0; o < md.O; ++o) qo[o] = fd[o] = 0.f;
      float la = 0.f;
      int dig[B2_MAX_DEP_RANK] = {0};
      for (int k = 0; k < md.K; ++k) {
        float w = 1.f;
        for (int i = 0; i < md.rank; ++i) w *= q[p.qs_off[md.dep[i]] + dig[i]];
        for (int o = 0; o < md.O; ++o) qo[o] = fmaf(__ldg(Am + (int64_t)o * md.K + k), w, qo[o]);
        if (wAm)
          for (int o = 0; o < md.O; ++o) fd[o] = fmaf(__ldg(wAm + (int64_t)o * md.K + k), w, fd[o]);
        la = fmaf(__ldg(Lm + k), w, la);
        for (int i = md.rank - 1; i >= 0; --i) {
          if (++dig[i] < p.S[md.dep[i]]) break;
          dig[i] = 0;
        }
      }
      float h = 0.f;
      if (ig)
        for (int o = 0; o < md.O; ++o) h -= qo[o] * log_stable(qo[o]);
      // pA term: qo_m . factor_dot(wA_m, qs) (control.py:511-553)
      if (wAm)
        for (int o = 0; o < md.O; ++o) h -= qo[o] * fd[o];
      g += (double)h + (double)la;
    }
  }
  G[b * p.P + pol] = (float)g;
}

// digamma(x) for x > 0 in FP64: the recurrence psi(x) = psi(x + 1) - 1/x up
// to x >= 10, then the asymptotic series psi(x) ~ ln x - 1/(2x) -
// sum_k B_2k / (2k x^2k) through B_14 (truncation below 1e-16 relative).
__device__ double digamma_fp64(double x) {
  double acc = 0.0;
  while (x < 10.0) {
    acc -= 1.0 / x;
    x += 1.0;
  }
  const double r = 1.0 / x, r2 = r * r;
  // B2/2 = 1/12, B4/4 = -1/120, B6/6 = 1/252, B8/8 = -1/240, B10/10 = 1/132,
  // B12/12 = -691/32760, B14/14 = 1/12
  const double series =
      r2 * (1.0 / 12 - r2 * (1.0 / 120 - r2 * (1.0 / 252 - r2 * (1.0 / 240 - r2 * (1.0 / 132 -
                                                                                   r2 * (691.0 / 32760 - r2 / 12))))));
  return acc + log(x) - 0.5 * r - series;
}

// Parameter information-gain weights (pymdp/control.py:543-544, :594):
// w = spm_wnorm(p) * (p > 0) with the exact Dirichlet form of
// pymdp/maths.py:783-808, -(log S - log a + 1/a - 1/S + digamma(a) -
// digamma(S)), a = clip(p, eps), S = clip(sum over axis 0 of a, eps).
// One thread per column: pA columns (modality m, joint state k) sum over the
// observations; pB columns (factor f, parent state k, action u) over the
// next states. Output laid out like pA / pB.
__global__ void efe_wnorm_kernel(const __grid_constant__ EfeParams p, const float* __restrict__ src, int is_B,
                                 float* __restrict__ w) {
  const int64_t b = blockIdx.y;
  const int64_t col = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  int64_t base, stride;
  int rows;
  if (!is_B) {
    if (col >= p.K_tot) return;
    int m = 0;
    while (m + 1 < p.M && p.mod[m + 1].lin_off <= col) ++m;
    const EfeModality& md = p.mod[m];
    base = b * p.A_stride + md.A_off + (col - md.lin_off);
    stride = md.K;
    rows = md.O;
  } else {
    int64_t c = col;
    int f = 0;
    for (; f < p.F; ++f) {
      const int64_t n = (int64_t)p.fac[f].K * p.U[f];
      if (c < n) break;
      c -= n;
    }
    if (f >= p.F) return;
    base = b * p.B_stride + p.fac[f].B_off + c;  // (k, u) column of (S_f, K_f, U_f)
    stride = (int64_t)p.fac[f].K * p.U[f];
    rows = p.S[f];
  }
  const double eps = 2.220446049250313e-16;
  double s = 0.0;
  for (int r = 0; r < rows; ++r) s += fmax((double)__ldg(src + base + r * stride), eps);
  s = fmax(s, eps);
  const double ls = log(s), ps = digamma_fp64(s), is = 1.0 / s;
  for (int r = 0; r < rows; ++r) {
    const float raw = __ldg(src + base + r * stride);
    const double a = fmax((double)raw, eps);
    const double wv = ls - log(a) + 1.0 / a - is + digamma_fp64(a) - ps;
    w[base + r * stride] = raw > 0.f ? (float)(-wv) : 0.f;
  }
}

// Inductive weights (pymdp/control.py:1021-1061, anchored to qs_init as in
// :775-777): per factor, idx = first argmax of qs_init_f, m = max(first argmax
// of I_f[:, idx] - 1, 0), path = clip(sum_i I_f[i, idx], 0, 1) and
// w_f[s] = path * (1 - I_f[m, s]) * log(clip(eps)). One thread per (agent, factor).
__global__ void efe_inductive_kernel(const __grid_constant__ EfeParams p, const float* __restrict__ qs_init,
                                     const float* __restrict__ I, const float* __restrict__ eps, int eps_batched,
                                     float* __restrict__ wI, int64_t Bn) {
  const int64_t idx_all = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx_all >= Bn * p.F) return;
  const int64_t b = idx_all / p.F;
  const int f = (int)(idx_all - b * p.F);
  const int S = p.S[f], D = p.I_depth[f];
  const float* q = qs_init + b * p.S_tot + p.qs_off[f];
  int idx = 0;
  for (int s = 1; s < S; ++s)
    if (q[s] > q[idx]) idx = s;
  const float* If = I + b * p.I_stride + p.I_off[f];
  int am = 0;
  double colsum = 0.0;
  for (int i = 0; i < D; ++i) {
    const float v = If[(int64_t)i * S + idx];
    if (v > If[(int64_t)am * S + idx]) am = i;
    colsum += v;
  }
  const int m = am - 1 > 0 ? am - 1 : 0;
  const double path = fmin(fmax(colsum, 0.0), 1.0);
  const double log_eps = log(fmax((double)eps[eps_batched ? b : 0], 2.220446049250313e-16));
  for (int s = 0; s < S; ++s)
    wI[b * p.S_tot + p.qs_off[f] + s] = (float)(path * (1.0 - (double)If[(int64_t)m * S + s]) * log_eps);
}

// q_pi[b] = softmax(gamma_b * G[b] + log(clip(E_b))) — one CTA per agent.
__global__ void __launch_bounds__(256)
    policy_posterior_kernel(const float* __restrict__ G, const float* __restrict__ E, int E_batched,
                            const float* __restrict__ gamma, int gamma_batched, float* __restrict__ q_pi, int P) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  __shared__ float red[32];
  const int64_t b = blockIdx.x;
  const float gm = gamma[gamma_batched ? b : 0];
  const float* g = G + b * P;
  const float* e = E + (E_batched ? b * P : 0);
  float mx = -INFINITY;
  for (int i = threadIdx.x; i < P; i += blockDim.x) mx = fmaxf(mx, gm * g[i] + log_stable(e[i]));
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
    v = warp_max(v);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  mx = red[0];
  __syncthreads();
  float sum = 0.f;
  for (int i = threadIdx.x; i < P; i += blockDim.x) sum += expf(gm * g[i] + log_stable(e[i]) - mx);
  sum = warp_sum(sum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    v = warp_sum(v);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  sum = red[0];
  for (int i = threadIdx.x; i < P; i += blockDim.x) q_pi[b * P + i] = expf(gm * g[i] + log_stable(e[i]) - mx) / sum;
}

// The same with every policy of the agent in registers (P <= 256 EPT): one
// pass over G and E; the same per-thread and block summation order, so the
// results equal the kernel above bit for bit.
template <int EPT>
__global__ void __launch_bounds__(256)
    policy_posterior_reg_kernel(const float* __restrict__ G, const float* __restrict__ E, int E_batched,
                                const float* __restrict__ gamma, int gamma_batched, float* __restrict__ q_pi, int P) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  __shared__ float red[32];
  const int64_t b = blockIdx.x;
  const float gm = gamma[gamma_batched ? b : 0];
  const float* g = G + b * P;
  const float* e = E + (E_batched ? b * P : 0);
  float z[EPT];
  float mx = -INFINITY;
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    const int i = threadIdx.x + k * 256;
    z[k] = i < P ? gm * g[i] + log_stable(e[i]) : -INFINITY;
    mx = fmaxf(mx, z[k]);
  }
  mx = warp_max(mx);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = mx;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : -INFINITY;
    v = warp_max(v);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  mx = red[0];
  __syncthreads();
  float sum = 0.f;
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    z[k] = threadIdx.x + k * 256 < P ? expf(z[k] - mx) : 0.f;
    sum += z[k];
  }
  sum = warp_sum(sum);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
    v = warp_sum(v);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  sum = red[0];
#pragma unroll
  for (int k = 0; k < EPT; ++k) {
    const int i = threadIdx.x + k * 256;
    if (i < P) q_pi[b * P + i] = z[k] / sum;
  }
}

// action[b, :] = policy_matrix[first argmax q_pi[b], 0, :] — one CTA per agent.
__global__ void __launch_bounds__(256)
    select_action_kernel(const float* __restrict__ q_pi, const int32_t* __restrict__ pm, int32_t* __restrict__ action,
                         int P, int T, int F) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  __shared__ float sv[32];
  __shared__ int si[32];
  const int64_t b = blockIdx.x;
  float best = -INFINITY;
  int bi = 0x7fffffff;
  // eight loads in flight, then the scan in index order
  for (int i0 = threadIdx.x; i0 < P; i0 += 8 * blockDim.x) {
    float v8[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = i0 + k * blockDim.x;
      v8[k] = i < P ? q_pi[b * P + i] : -INFINITY;
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int i = i0 + k * blockDim.x;
      const float v = v8[k];
      if (i < P && (v > best || (v == best && i < bi) || (bi == 0x7fffffff && v != v))) {
        best = v;
        bi = i;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, best, o);
    const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
    if (ov > best || (ov == best && oi < bi)) {
      best = ov;
      bi = oi;
    }
  }
  if ((threadIdx.x & 31) == 0) {
    sv[threadIdx.x >> 5] = best;
    si[threadIdx.x >> 5] = bi;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w)
      if (sv[w] > best || (sv[w] == best && si[w] < bi)) {
        best = sv[w];
        bi = si[w];
      }
    if (bi == 0x7fffffff) bi = 0;
    si[0] = bi;
  }
  __syncthreads();
  bi = si[0];
  for (int f = threadIdx.x; f < F; f += blockDim.x) action[b * F + f] = pm[(int64_t)bi * T * F + f];
}

int32_t launch_linear_rows(const EfeParams& p, int64_t Bn, const float* A, const float* C, float* lin,
                           cudaStream_t stream) {
  dim3 grid((unsigned)((p.K_tot + 127) / 128), (unsigned)p.T, (unsigned)Bn);
  efe_linear_rows_kernel<<<grid, 128, 0, stream>>>(p, A, C, lin);
  return check_launch("efe_ffi linear rows");
}

int32_t launch_efe_plain(const EfeParams& p, int64_t Bn, const int32_t* pm, int pm_batched, const float* qs,
                         const float* A, const float* B, const float* lin, float* G, cudaStream_t stream,
                         const float* wA, const float* wB, const float* wI) {
  dim3 grid((unsigned)((p.P + 127) / 128), (unsigned)Bn);
  efe_plain_kernel<<<grid, 128, 0, stream>>>(p, pm, pm_batched, qs, A, B, lin, G, wA, wB, wI);
  return check_launch("efe_ffi plain");
}

// Workspace from the device's stream-ordered pool; freed stream-ordered.
int32_t ws_alloc(void** ptr, size_t bytes, cudaStream_t stream, const char* op) {
  static std::mutex mu;
  static std::set<int> tuned;
  int dev = 0;
  B2_CUDA_TRY(op, cudaGetDevice(&dev));
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!tuned.count(dev)) {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t keep = ~0ull;  // keep freed blocks cached in this process
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
      }
      tuned.insert(dev);
    }
  }
  B2_CUDA_TRY(op, cudaMallocAsync(ptr, bytes, stream));
  return B2_OK;
}

}  // namespace b2

using namespace b2;

namespace b2 {
namespace {

int32_t neg_efe_impl(void* stream_, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                              const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                              const float* B, int64_t B_count, const float* C, int64_t C_count, const float* I,
                              int64_t I_count, const float* pA, int64_t pA_count, const float* pB,
                              int64_t pB_count, const float* inductive_epsilon, int64_t eps_count,
                              float* neg_efe_out, int64_t out_count, int64_t Bn, int64_t P, int64_t T, int64_t F,
                              int64_t M, const int64_t* S, const int64_t* O, const int64_t* U,
                              const int64_t* qs_offsets, const int64_t* A_offsets, const int64_t* B_offsets,
                              const int64_t* C_offsets, const int64_t* I_offsets, const int64_t* I_depths,
                              const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets,
                              const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets,
                              int32_t flags, const PackCache* cache) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (Bn < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": negative Bn");
  EfeParams p;
  B2_TRY(build_efe_params(&p, P, T, F, M, S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_offsets,
                          I_depths, A_dep_flat, A_dep_flat_len, A_dep_offsets, B_dep_flat, B_dep_flat_len,
                          B_dep_offsets, flags));
  const int64_t I_stride = I_offsets[F];
  struct Chk {
    const char* name;
    int64_t actual, expected;
  } chks[] = {
      {"policy_matrix", pm_count, (pm_batched ? Bn : 1) * P * T * F},
      {"qs_init", qs_count, Bn * (int64_t)p.S_tot},
      {"A", A_count, Bn * p.A_stride},
      {"B", B_count, Bn * p.B_stride},
      {"C", C_count, Bn * p.C_stride},
      {"I", I_count, Bn * I_stride},
      {"out", out_count, Bn * P},
  };
  for (const Chk& c : chks)
    if (c.actual != c.expected)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": " + c.name + " element_count = " +
                                               std::to_string(c.actual) + ", expected " + std::to_string(c.expected));
  if (eps_count != 1 && eps_count != Bn)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": inductive_epsilon must have 1 or Bn elements");
  const bool use_pig = (flags & B2_FLAG_USE_PARAM_INFO_GAIN) != 0;
  const bool use_ind = (flags & B2_FLAG_USE_INDUCTIVE) != 0;
  if (use_pig) {
    if (pA_count == 0 && pB_count == 0)
      return fail(B2_ERR_INVALID_ARGUMENT,
                  std::string(kEfeName) + ": use_param_info_gain=true requires at least one of pA, pB");
    if (pA_count != 0 && pA_count != Bn * p.A_stride)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": pA element_count = " +
                                               std::to_string(pA_count) + ", expected 0 or " +
                                               std::to_string(Bn * p.A_stride));
    if (pB_count != 0 && pB_count != Bn * p.B_stride)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": pB element_count = " +
                                               std::to_string(pB_count) + ", expected 0 or " +
                                               std::to_string(Bn * p.B_stride));
  }
  const int prec = (flags >> B2_PRECISION_SHIFT) & 3;
  if (prec > B2_PRECISION_BF16)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": unknown precision selector");
  if (Bn == 0) return B2_OK;
  if (!policy_matrix || !qs_init || !A || !B || !C || !neg_efe_out)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": null buffer");
  if (Bn > 65535) return fail(B2_ERR_UNSUPPORTED, std::string(kEfeName) + ": Bn > 65535");
  if ((use_pig && ((pA_count && !pA) || (pB_count && !pB))) || (use_ind && (!I || !inductive_epsilon)))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": null buffer");
  if (use_pig || use_ind) {
    // the flag-gated terms: weights first (FP64 digamma / inductive paths),
    // then the factored path where it applies, else the SIMT FP32 kernel
    const size_t lin_bytes = (size_t)Bn * p.T * p.K_tot * sizeof(float);
    const size_t wa_bytes = (use_pig && pA_count) ? (size_t)Bn * p.A_stride * sizeof(float) : 0;
    const size_t wb_bytes = (use_pig && pB_count) ? (size_t)Bn * p.B_stride * sizeof(float) : 0;
    const size_t wi_bytes = use_ind ? (size_t)Bn * p.S_tot * sizeof(float) : 0;
    auto up = [](size_t x) { return (x + 255) / 256 * 256; };
    uint8_t* ws = nullptr;
    B2_TRY(ws_alloc((void**)&ws, up(lin_bytes) + up(wa_bytes) + up(wb_bytes) + up(wi_bytes), stream, kEfeName));
    float* lin = reinterpret_cast<float*>(ws);
    float* wA = wa_bytes ? reinterpret_cast<float*>(ws + up(lin_bytes)) : nullptr;
    float* wB = wb_bytes ? reinterpret_cast<float*>(ws + up(lin_bytes) + up(wa_bytes)) : nullptr;
    float* wI = wi_bytes ? reinterpret_cast<float*>(ws + up(lin_bytes) + up(wa_bytes) + up(wb_bytes)) : nullptr;
    int32_t rc = B2_OK;
    if (wA) {
      efe_wnorm_kernel<<<dim3((unsigned)((p.K_tot + 127) / 128), (unsigned)Bn), 128, 0, stream>>>(p, pA, 0, wA);
      rc = check_launch("efe_ffi pA weights");
    }
    if (rc == B2_OK && wB) {
      int64_t cols = 0;
      for (int f = 0; f < p.F; ++f) cols += (int64_t)p.fac[f].K * p.U[f];
      efe_wnorm_kernel<<<dim3((unsigned)((cols + 127) / 128), (unsigned)Bn), 128, 0, stream>>>(p, pB, 1, wB);
      rc = check_launch("efe_ffi pB weights");
    }
    if (rc == B2_OK && wI) {
      const int64_t n = Bn * p.F;
      efe_inductive_kernel<<<(unsigned)((n + 127) / 128), 128, 0, stream>>>(p, qs_init, I, inductive_epsilon,
                                                                           eps_count == Bn && Bn > 1, wI, Bn);
      rc = check_launch("efe_ffi inductive weights");
    }
    bool done = false;
    if (rc == B2_OK && (flags & B2_FLAG_FACTORED) && (flags & B2_FLAG_POLICY_TREE) && !pm_batched)
      rc = launch_efe_fact(p, Bn, qs_init, A, B, C, neg_efe_out, stream, &done, wA, wB, wI);
    if (rc == B2_OK && !done) rc = launch_linear_rows(p, Bn, A, C, lin, stream);
    if (rc == B2_OK && !done)
      rc = launch_efe_plain(p, Bn, policy_matrix, pm_batched, qs_init, A, B, lin, neg_efe_out, stream, wA, wB, wI);
    cudaError_t fe = cudaFreeAsync(ws, stream);
    if (rc == B2_OK && fe != cudaSuccess) return cuda_fail(kEfeName, fe);
    return rc;
  }
  if ((flags & B2_FLAG_FACTORED) && (flags & B2_FLAG_POLICY_TREE) && !pm_batched) {
    // factored contraction over the per-factor marginals of the policy tree
    bool used = false;
    B2_TRY(launch_efe_fact(p, Bn, qs_init, A, B, C, neg_efe_out, stream, &used));
    if (used) return B2_OK;
  }
  if (prec != B2_PRECISION_FP32) {
    // tensor-core path; models outside its limits take the SIMT FP32 path
    bool used = false;
    B2_TRY(launch_efe_tc(p, prec, Bn, policy_matrix, pm_batched, qs_init, A, B, C, neg_efe_out, stream, &used,
                         cache));
    if (used) return B2_OK;
  }
  {
    // small models: all of an agent's policies in one CTA
    bool used = false;
    B2_TRY(launch_efe_small(p, Bn, false, policy_matrix, pm_batched, qs_init, A, B, C, neg_efe_out, nullptr,
                            nullptr, nullptr, nullptr, nullptr, stream, &used));
    if (used) return B2_OK;
  }
  float* lin = nullptr;
  const size_t bytes = (size_t)Bn * p.T * p.K_tot * sizeof(float);
  B2_TRY(ws_alloc((void**)&lin, bytes, stream, kEfeName));
  int32_t rc = launch_linear_rows(p, Bn, A, C, lin, stream);
  if (rc == B2_OK) rc = launch_efe_plain(p, Bn, policy_matrix, pm_batched, qs_init, A, B, lin, neg_efe_out, stream);
  cudaError_t fe = cudaFreeAsync(lin, stream);
  if (rc == B2_OK && fe != cudaSuccess) return cuda_fail(kEfeName, fe);
  return rc;
}

}  // namespace
}  // namespace b2

extern "C" int32_t b2_neg_efe(void* stream_, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                              const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                              const float* B, int64_t B_count, const float* C, int64_t C_count, const float* I,
                              int64_t I_count, const float* pA, int64_t pA_count, const float* pB,
                              int64_t pB_count, const float* inductive_epsilon, int64_t eps_count,
                              float* neg_efe_out, int64_t out_count, int64_t Bn, int64_t P, int64_t T, int64_t F,
                              int64_t M, const int64_t* S, const int64_t* O, const int64_t* U,
                              const int64_t* qs_offsets, const int64_t* A_offsets, const int64_t* B_offsets,
                              const int64_t* C_offsets, const int64_t* I_offsets, const int64_t* I_depths,
                              const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets,
                              const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets,
                              int32_t flags) {
  return neg_efe_impl(stream_, policy_matrix, pm_count, pm_batched, qs_init, qs_count, A, A_count, B, B_count, C, C_count, I,
                      I_count, pA, pA_count, pB, pB_count, inductive_epsilon, eps_count, neg_efe_out, out_count, Bn, P,
                      T, F, M, S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_offsets, I_depths, A_dep_flat,
                      A_dep_flat_len, A_dep_offsets, B_dep_flat, B_dep_flat_len, B_dep_offsets, flags, nullptr);
}

extern "C" int32_t b2_neg_efe_cached(void* stream_, const int32_t* policy_matrix, int64_t pm_count, int32_t pm_batched,
                              const float* qs_init, int64_t qs_count, const float* A, int64_t A_count,
                              const float* B, int64_t B_count, const float* C, int64_t C_count, const float* I,
                              int64_t I_count, const float* pA, int64_t pA_count, const float* pB,
                              int64_t pB_count, const float* inductive_epsilon, int64_t eps_count,
                              float* neg_efe_out, int64_t out_count, int64_t Bn, int64_t P, int64_t T, int64_t F,
                              int64_t M, const int64_t* S, const int64_t* O, const int64_t* U,
                              const int64_t* qs_offsets, const int64_t* A_offsets, const int64_t* B_offsets,
                              const int64_t* C_offsets, const int64_t* I_offsets, const int64_t* I_depths,
                              const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets,
                              const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets,
                              int32_t flags, uint8_t* pack_cache, int64_t pack_cache_bytes,
                                     int32_t* pack_cache_valid) {
  if (!pack_cache || !pack_cache_valid)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": null pack cache");
  const PackCache cache{pack_cache, pack_cache_bytes, pack_cache_valid};
  return neg_efe_impl(stream_, policy_matrix, pm_count, pm_batched, qs_init, qs_count, A, A_count, B, B_count, C, C_count, I,
                      I_count, pA, pA_count, pB, pB_count, inductive_epsilon, eps_count, neg_efe_out, out_count, Bn, P,
                      T, F, M, S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_offsets, I_depths, A_dep_flat,
                      A_dep_flat_len, A_dep_offsets, B_dep_flat, B_dep_flat_len, B_dep_offsets, flags, &cache);
}

extern "C" int32_t b2_neg_efe_pack_bytes(int64_t Bn, int64_t P, int64_t T, int64_t F, int64_t M, const int64_t* S,
                                         const int64_t* O, const int64_t* U, const int64_t* qs_offsets,
                                         const int64_t* A_offsets, const int64_t* B_offsets,
                                         const int64_t* C_offsets, const int64_t* I_offsets,
                                         const int64_t* I_depths, const int64_t* A_dep_flat,
                                         int64_t A_dep_flat_len, const int64_t* A_dep_offsets,
                                         const int64_t* B_dep_flat, int64_t B_dep_flat_len,
                                         const int64_t* B_dep_offsets, int32_t flags, int64_t* bytes) {
  if (!bytes || Bn < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": null bytes or negative Bn");
  EfeParams p;
  B2_TRY(build_efe_params(&p, P, T, F, M, S, O, U, qs_offsets, A_offsets, B_offsets, C_offsets, I_offsets,
                          I_depths, A_dep_flat, A_dep_flat_len, A_dep_offsets, B_dep_flat, B_dep_flat_len,
                          B_dep_offsets, flags));
  const bool simt_terms = (flags & (B2_FLAG_USE_PARAM_INFO_GAIN | B2_FLAG_USE_INDUCTIVE)) != 0;
  // the factored path packs nothing
  const bool factored = (flags & B2_FLAG_FACTORED) && (flags & B2_FLAG_POLICY_TREE) && efe_fact_applies(p, Bn);
  *bytes = simt_terms || factored ? 0 : efe_tc_pack_bytes(p, (flags >> B2_PRECISION_SHIFT) & 3, Bn);
  return B2_OK;
}

extern "C" int32_t b2_policy_posterior(void* stream, const float* neg_efe, const float* E, int32_t E_batched,
                                       const float* gamma, int32_t gamma_batched, float* q_pi, int64_t Bn,
                                       int64_t P) {
  if (Bn < 0 || P <= 0 || P > 0x7fffffff)
    return fail(B2_ERR_INVALID_ARGUMENT, "policy_posterior: invalid Bn or P");
  if (Bn == 0) return B2_OK;
  if (!neg_efe || !E || !gamma || !q_pi) return fail(B2_ERR_INVALID_ARGUMENT, "policy_posterior: null buffer");
  if (Bn > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, "policy_posterior: Bn too large");
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid((unsigned)Bn), blk(256);
  const int Pi = (int)P;
  const cudaError_t e =
      P <= 256 * 4    ? launch_pdl(policy_posterior_reg_kernel<4>, grid, blk, 0, st, neg_efe, E, E_batched, gamma,
                                   gamma_batched, q_pi, Pi)
      : P <= 256 * 16 ? launch_pdl(policy_posterior_reg_kernel<16>, grid, blk, 0, st, neg_efe, E, E_batched, gamma,
                                   gamma_batched, q_pi, Pi)
      : P <= 256 * 64 ? launch_pdl(policy_posterior_reg_kernel<64>, grid, blk, 0, st, neg_efe, E, E_batched, gamma,
                                   gamma_batched, q_pi, Pi)
                      : launch_pdl(policy_posterior_kernel, grid, blk, 0, st, neg_efe, E, E_batched, gamma,
                                   gamma_batched, q_pi, Pi);
  if (e != cudaSuccess) return cuda_fail("policy_posterior", e);
  return check_launch("policy_posterior");
}

extern "C" int32_t b2_select_action(void* stream, const float* q_pi, const int32_t* policy_matrix,
                                    int32_t* action, int64_t Bn, int64_t P, int64_t T, int64_t F) {
  if (Bn < 0 || P <= 0 || T <= 0 || F <= 0 || P > 0x7fffffff)
    return fail(B2_ERR_INVALID_ARGUMENT, "select_action: invalid sizes");
  if (Bn == 0) return B2_OK;
  if (!q_pi || !policy_matrix || !action) return fail(B2_ERR_INVALID_ARGUMENT, "select_action: null buffer");
  const cudaError_t e = launch_pdl(select_action_kernel, dim3((unsigned)Bn), dim3(256), 0, (cudaStream_t)stream, q_pi,
                                   policy_matrix, action, (int)P, (int)T, (int)F);
  if (e != cudaSuccess) return cuda_fail("select_action", e);
  return check_launch("select_action");
}

// -------------------------------------------------------------------------
// Action selection with the reference's four modes (pymdp/agent.py:939-967):
// sampling_mode "full" picks a policy (control.py:115-150) and returns its
// first step; "marginal" forms each control factor's first-step action
// marginal (get_marginals, control.py:42-67) and picks from it
// (control.py:69-113). Deterministic selection takes the first maximum;
// stochastic selection draws from the categorical with logits
// alpha * log clip(x) by the Gumbel-max trick (argmax of logits + Gumbel
// noise, the method jax.random.categorical uses), with u from SplitMix64 over
// (seed, agent, factor, index) instead of JAX's PRNG.
namespace b2 {
namespace {

__device__ __forceinline__ uint64_t sa_mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// Gumbel(0, 1) from u in (0, 1): u = (top 24 bits + 0.5) / 2^24.
__device__ __forceinline__ float sa_gumbel(uint64_t seed, int64_t agent, int factor, int index) {
  uint64_t h = sa_mix(seed);
  h = sa_mix(h ^ (uint64_t)agent);
  h = sa_mix(h ^ (uint64_t)(uint32_t)factor);
  h = sa_mix(h ^ (uint64_t)(uint32_t)index);
  const float u = ((float)(h >> 40) + 0.5f) * (1.0f / 16777216.0f);
  return -logf(-logf(u));
}

// argmax over a block (first index on ties); s_v / s_i: 32 slots each.
__device__ int sa_block_argmax(float v, int i, float* s_v, int* s_i) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const float ov = __shfl_xor_sync(0xffffffffu, v, o);
    const int oi = __shfl_xor_sync(0xffffffffu, i, o);
    if (ov > v || (ov == v && oi < i)) {
      v = ov;
      i = oi;
    }
  }
  if (lane == 0) {
    s_v[wid] = v;
    s_i[wid] = i;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w)
      if (s_v[w] > s_v[0] || (s_v[w] == s_v[0] && s_i[w] < s_i[0])) {
        s_v[0] = s_v[w];
        s_i[0] = s_i[w];
      }
  }
  __syncthreads();
  const int r = s_i[0];
  __syncthreads();
  return r;
}

struct SampleDims {
  int32_t U[B2_MAX_FACTORS];
};

__global__ void sample_action_kernel(const float* __restrict__ q_pi, const int32_t* __restrict__ pm,
                                     const __grid_constant__ SampleDims U, int32_t* __restrict__ action, int P,
                                     int T, int F, int marginal, int stochastic, const float* __restrict__ alpha_p,
                                     int alpha_batched, uint64_t seed) {
  __shared__ float s_v[32];
  __shared__ int s_i[32];
  __shared__ float s_m[B2_SAMPLE_MAX_U];
  const int64_t b = blockIdx.x;
  const float* q = q_pi + b * P;
  const float alpha = stochastic ? alpha_p[alpha_batched ? b : 0] : 0.f;
  if (!marginal) {
    float best = -INFINITY;
    int bi = 0x7fffffff;
    for (int p = threadIdx.x; p < P; p += blockDim.x) {
      const float v = stochastic ? alpha * log_stable(q[p]) + sa_gumbel(seed, b, -1, p) : q[p];
      if (v > best || (v == best && p < bi) || (bi == 0x7fffffff && v != v)) {
        best = v;
        bi = p;
      }
    }
    int p = sa_block_argmax(best, bi, s_v, s_i);
    if (p == 0x7fffffff) p = 0;
    for (int f = threadIdx.x; f < F; f += blockDim.x) action[b * F + f] = pm[(int64_t)p * T * F + f];
    return;
  }
  for (int f = 0; f < F; ++f) {
    const int Uf = U.U[f];
    // first-step action marginal of factor f, summed in policy order (deterministic)
    for (int a = threadIdx.x; a < Uf; a += blockDim.x) {
      float acc = 0.f;
      for (int p = 0; p < P; ++p)
        if (pm[(int64_t)p * T * F + f] == a) acc += q[p];
      s_m[a] = acc;
    }
    __syncthreads();
    float best = -INFINITY;
    int bi = 0x7fffffff;
    for (int a = threadIdx.x; a < Uf; a += blockDim.x) {
      const float v = stochastic ? alpha * log_stable(s_m[a]) + sa_gumbel(seed, b, f, a) : s_m[a];
      if (v > best || (v == best && a < bi)) {
        best = v;
        bi = a;
      }
    }
    int a = sa_block_argmax(best, bi, s_v, s_i);
    if (threadIdx.x == 0) action[b * F + f] = a == 0x7fffffff ? 0 : a;
    __syncthreads();
  }
}

}  // namespace
}  // namespace b2

extern "C" int32_t b2_sample_action(void* stream, const float* q_pi, const int32_t* policy_matrix, const int64_t* U,
                                    int32_t* action, int64_t Bn, int64_t P, int64_t T, int64_t F,
                                    int32_t sampling_mode, int32_t action_selection, const float* alpha,
                                    int32_t alpha_batched, uint64_t seed) {
  const char* op = "sample_action";
  if (Bn < 0 || P <= 0 || T <= 0 || F <= 0 || P > 0x7fffffff || T * F > 0x7fffffff)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (sampling_mode != 0 && sampling_mode != 1)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": sampling_mode must be 0 (full) or 1 (marginal)");
  if (action_selection != 0 && action_selection != 1)
    return fail(B2_ERR_INVALID_ARGUMENT,
                std::string(op) + ": action_selection must be 0 (deterministic) or 1 (stochastic)");
  if (F > B2_MAX_FACTORS) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": more than 16 factors");
  b2::SampleDims dims{};
  if (sampling_mode == 1) {
    if (!U) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": marginal mode needs U");
    for (int64_t f = 0; f < F; ++f) {
      if (U[f] < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": U must be positive");
      if (U[f] > B2_SAMPLE_MAX_U) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": U above 1024");
      dims.U[f] = (int32_t)U[f];
    }
  }
  if (Bn == 0) return B2_OK;
  if (!q_pi || !policy_matrix || !action || (action_selection == 1 && !alpha))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  if (Bn > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": Bn too large");
  b2::sample_action_kernel<<<(unsigned)Bn, 256, 0, (cudaStream_t)stream>>>(
      q_pi, policy_matrix, dims, action, (int)P, (int)T, (int)F, sampling_mode, action_selection, alpha,
      alpha_batched, seed);
  return check_launch(op);
}
