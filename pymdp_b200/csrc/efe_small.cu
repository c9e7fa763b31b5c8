// neg-EFE (utility + state information gain) and its reverse pass for small
// models: one CTA per agent holds every policy's roll-out in shared memory.
//
// Same arithmetic as efe_plain_kernel / efe_bwd_kernel (pymdp/control.py:
// 604-690 forward; the derivative of that arithmetic backward, see
// efe_bwd.cu for the formulas), organised for models whose policies and
// joint states are few (the model-fitting regime: P = 16, K = 32): threads
// run over (policy, state) and (observation, joint state) pairs; every
// gradient entry in global memory is owned by one thread that sums over the
// policies (no global atomics), and the per-policy state gradients gather in
// shared memory. With w_p = dL/dG_p:
//   gqo[p][o] = -w_p (log clip qo + [qo >= eps])                      (ig)
//   gx[p][k]  = sum_o A[o,k] (gqo[p][o] + w_p la[o,k]),  la = ig log clip A + ut C_t
//   dA[o,k]  += sum_p x[p][k] (gqo[p][o] + w_p (la[o,k] + ig [A >= eps]))
//   dC_t[o]  += sum_p w_p qo[p][o]                                     (ut)
// then back through x = prod of marginals and qs_{t+1,f} = B_f[..., u] . joint.
#include <string>

#include "common.cuh"
#include "efe.cuh"

namespace b2 {
namespace {

constexpr int kSmallThreads = 256;
constexpr float kEpsS = 2.220446049250313e-16f;

__device__ __forceinline__ void small_digits(int k, const int8_t* dep, int rank, const int32_t* S, int* dig) {
  for (int i = rank - 1; i >= 0; --i) {
    const int d = S[dep[i]];
    const int q = k / d;
    dig[i] = k - q * d;
    k = q;
  }
}

__device__ __forceinline__ int small_factor_of(const EfeParams& p, int j) {
  int f = 0;
  while (f + 1 < p.F && j >= p.qs_off[f + 1]) ++f;
  return f;
}

// x[p][k] = prod_i q[p][dep_i][k_i] for one dependency list (rank, dep, K).
__device__ void small_joint(const EfeParams& p, const int8_t* dep, int rank, int K, const float* q, int St,
                            float* x, int Kx) {
  const int P = p.P;
  for (int e = threadIdx.x; e < P * K; e += blockDim.x) {
    const int pp = e / K, k = e - pp * K;
    int dig[B2_MAX_DEP_RANK];
    small_digits(k, dep, rank, p.S, dig);
    float v = 1.f;
    for (int i = 0; i < rank; ++i) v *= q[pp * St + p.qs_off[dep[i]] + dig[i]];
    x[pp * Kx + k] = v;
  }
}

// acc[p][dep_j state k_j] += g[p][k] * prod_{i != j} q[p][dep_i][k_i] for every
// (p, k): one digit decomposition per pair, shared-memory atomics into acc.
__device__ void small_scatter(const EfeParams& p, const int8_t* dep, int rank, int K, const float* q, int St,
                              const float* g, int Kx, float* acc) {
  const int P = p.P;
  for (int e = threadIdx.x; e < P * K; e += blockDim.x) {
    const int pp = e / K, k = e - pp * K;
    const float gv = g[pp * Kx + k];
    if (gv == 0.f) continue;
    int dig[B2_MAX_DEP_RANK];
    small_digits(k, dep, rank, p.S, dig);
    float qv[B2_MAX_DEP_RANK];
    for (int i = 0; i < rank; ++i) qv[i] = q[pp * St + p.qs_off[dep[i]] + dig[i]];
    for (int j = 0; j < rank; ++j) {
      float other = 1.f;
      for (int i = 0; i < rank; ++i)
        if (i != j) other *= qv[i];
      atomicAdd(&acc[pp * St + p.qs_off[dep[j]] + dig[j]], gv * other);
    }
  }
  __syncthreads();
}

template <bool BWD>
__global__ void __launch_bounds__(kSmallThreads)
    efe_small_kernel(const __grid_constant__ EfeParams p, int Kx, int Omax, const int32_t* __restrict__ pm,
                     int pm_batched, const float* __restrict__ qs_init, const float* __restrict__ A,
                     const float* __restrict__ B, const float* __restrict__ C, float* __restrict__ G,
                     const float* __restrict__ dG, float* __restrict__ dqs, float* __restrict__ dA,
                     float* __restrict__ dB, float* __restrict__ dC) {
  extern __shared__ float sm[];
  const int P = p.P, T = p.T, St = p.S_tot, F = p.F, tid = threadIdx.x, NT = blockDim.x;
  const int64_t b = blockIdx.x;
  float* hist = sm;                    // (T + 1) x P x St
  float* x = hist + (T + 1) * P * St;  // P x Kx
  float* gx = x + P * Kx;              // P x Kx
  float* qo = gx + P * Kx;             // P x Omax
  float* gqo = qo + P * Omax;          // P x Omax
  float* gq = gqo + P * Omax;          // P x St
  float* gqp = gq + P * St;            // P x St
  float* wv = gqp + P * St;            // P
  float* lin = wv + P;                 // Kx
  float* la = lin + Kx;                // Omax x Kx: log clip A [ig] + C_t [ut] of one (step, modality)
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const bool ut = (p.flags & B2_FLAG_USE_UTILITY) != 0;
  const int32_t* pmb = pm + (pm_batched ? b * (int64_t)P * T * F : 0);
  const float* Ab = A + b * p.A_stride;
  const float* Bb = B + b * p.B_stride;
  const float* Cb = C + b * p.C_stride;

  for (int pp = tid; pp < P; pp += NT) wv[pp] = BWD ? dG[b * P + pp] : 0.f;
  for (int e = tid; e < P * St; e += NT) hist[e] = __ldg(qs_init + b * St + e % St);
  __syncthreads();
  // forward roll-out of every policy: hist[t + 1] = B(u_t) . joint(hist[t])
  for (int t = 0; t < T; ++t) {
    const float* qc = hist + t * P * St;
    float* qn = hist + (t + 1) * P * St;
    for (int e = tid; e < P * St; e += NT) {
      const int pp = e / St, j = e - pp * St;
      const int f = small_factor_of(p, j), s = j - p.qs_off[f], U = p.U[f];
      const int u = jnp_action(pmb[((int64_t)pp * T + t) * F + f], U);
      const EfeFactor& fb = p.fac[f];
      const float* Bs = Bb + fb.B_off + (int64_t)s * fb.K * U + u;
      float acc = 0.f;
      for (int k = 0; k < fb.K; ++k) {
        int dig[B2_MAX_DEP_RANK];
        small_digits(k, fb.dep, fb.rank, p.S, dig);
        float v = 1.f;
        for (int i = 0; i < fb.rank; ++i) v *= qc[pp * St + p.qs_off[fb.dep[i]] + dig[i]];
        acc = fmaf(__ldg(Bs + (int64_t)k * U), v, acc);
      }
      qn[e] = acc;
    }
    __syncthreads();
  }

  if (!BWD) {
    for (int t = 0; t < T; ++t) {
      const float* q = hist + (t + 1) * P * St;
      for (int m = 0; m < p.M; ++m) {
        const EfeModality& md = p.mod[m];
        const float* Am = Ab + md.A_off;
        const float* Cm = Cb + md.C_off + (int64_t)t * md.O;
        // linear row of step t: sum_o A[o,k] (log clip A [ig] + C_t[o] [ut])
        for (int k = tid; k < md.K; k += NT) {
          float l = 0.f;
          for (int o = 0; o < md.O; ++o) {
            const float a = __ldg(Am + (int64_t)o * md.K + k);
            l = fmaf(a, (ig ? log_stable(a) : 0.f) + (ut ? __ldg(Cm + o) : 0.f), l);
          }
          lin[k] = l;
        }
        small_joint(p, md.dep, md.rank, md.K, q, St, x, Kx);
        __syncthreads();
        for (int e = tid; e < P * md.O; e += NT) {
          const int pp = e / md.O, o = e - pp * md.O;
          float acc = 0.f;
          for (int k = 0; k < md.K; ++k) acc = fmaf(__ldg(Am + (int64_t)o * md.K + k), x[pp * Kx + k], acc);
          qo[pp * Omax + o] = acc;
        }
        __syncthreads();
        for (int pp = tid; pp < P; pp += NT) {
          float h = 0.f;
          if (ig)
            for (int o = 0; o < md.O; ++o) {
              const float v = qo[pp * Omax + o];
              h -= v * log_stable(v);
            }
          float l = 0.f;
          for (int k = 0; k < md.K; ++k) l = fmaf(lin[k], x[pp * Kx + k], l);
          wv[pp] += h + l;
        }
        __syncthreads();
      }
    }
    for (int pp = tid; pp < P; pp += NT) G[b * P + pp] = wv[pp];
    return;
  }

  // ------------------------------------------------------------- reverse pass
  float* dAb = dA + b * p.A_stride;
  float* dBb = dB + b * p.B_stride;
  float* dCb = dC + b * p.C_stride;
  for (int e = tid; e < P * St; e += NT) gq[e] = 0.f;
  __syncthreads();
  for (int t = T - 1; t >= 0; --t) {
    const float* q = hist + (t + 1) * P * St;
    for (int m = 0; m < p.M; ++m) {
      const EfeModality& md = p.mod[m];
      const float* Am = Ab + md.A_off;
      const float* Cm = Cb + md.C_off + (int64_t)t * md.O;
      small_joint(p, md.dep, md.rank, md.K, q, St, x, Kx);
      for (int e = tid; e < md.O * md.K; e += NT) {
        const int o = e / md.K;
        la[e] = (ig ? log_stable(__ldg(Am + e)) : 0.f) + (ut ? __ldg(Cm + o) : 0.f);
      }
      __syncthreads();
      for (int e = tid; e < P * md.O; e += NT) {
        const int pp = e / md.O, o = e - pp * md.O;
        float acc = 0.f;
        for (int k = 0; k < md.K; ++k) acc = fmaf(__ldg(Am + (int64_t)o * md.K + k), x[pp * Kx + k], acc);
        qo[pp * Omax + o] = acc;
        gqo[pp * Omax + o] = ig ? -wv[pp] * (log_stable(acc) + (acc >= kEpsS ? 1.f : 0.f)) : 0.f;
      }
      __syncthreads();
      if (ut)
        for (int o = tid; o < md.O; o += NT) {
          float acc = 0.f;
          for (int pp = 0; pp < P; ++pp) acc = fmaf(wv[pp], qo[pp * Omax + o], acc);
          dCb[md.C_off + (int64_t)t * md.O + o] += acc;
        }
      for (int e = tid; e < P * md.K; e += NT) {
        const int pp = e / md.K, k = e - pp * md.K;
        float acc = 0.f;
        const float wp = wv[pp];
        for (int o = 0; o < md.O; ++o)
          acc = fmaf(__ldg(Am + (int64_t)o * md.K + k), gqo[pp * Omax + o] + wp * la[o * md.K + k], acc);
        gx[pp * Kx + k] = acc;
      }
      for (int e = tid; e < md.O * md.K; e += NT) {
        const int o = e / md.K, k = e - o * md.K;
        const float a = __ldg(Am + e);
        const float lae = la[e] + (ig && a >= kEpsS ? 1.f : 0.f);
        float acc = 0.f;
        for (int pp = 0; pp < P; ++pp) acc = fmaf(x[pp * Kx + k], gqo[pp * Omax + o] + wv[pp] * lae, acc);
        dAb[md.A_off + e] += acc;
      }
      __syncthreads();
      small_scatter(p, md.dep, md.rank, md.K, q, St, gx, Kx, gq);
    }
    // back through the roll-out of step t
    const float* qc = hist + t * P * St;
    for (int e = tid; e < P * St; e += NT) gqp[e] = 0.f;
    __syncthreads();
    for (int f = 0; f < F; ++f) {
      const EfeFactor& fb = p.fac[f];
      const int S = p.S[f], U = p.U[f], K = fb.K;
      const float* Bf = Bb + fb.B_off;
      small_joint(p, fb.dep, fb.rank, K, qc, St, x, Kx);
      __syncthreads();
      for (int e = tid; e < P * K; e += NT) {
        const int pp = e / K, k = e - pp * K;
        const int u = jnp_action(pmb[((int64_t)pp * T + t) * F + f], U);
        float acc = 0.f;
        for (int s = 0; s < S; ++s) acc = fmaf(__ldg(Bf + ((int64_t)s * K + k) * U + u), gq[pp * St + p.qs_off[f] + s], acc);
        gx[pp * Kx + k] = acc;
      }
      for (int e = tid; e < S * K * U; e += NT) {
        const int u = e % U, sk = e / U, k = sk % K, s = sk / K;
        float acc = 0.f;
        for (int pp = 0; pp < P; ++pp) {
          const int up = jnp_action(pmb[((int64_t)pp * T + t) * F + f], U);
          if (up == u) acc = fmaf(gq[pp * St + p.qs_off[f] + s], x[pp * Kx + k], acc);
        }
        dBb[fb.B_off + e] += acc;
      }
      __syncthreads();
      small_scatter(p, fb.dep, fb.rank, K, qc, St, gx, Kx, gqp);
    }
    for (int e = tid; e < P * St; e += NT) gq[e] = gqp[e];
    __syncthreads();
  }
  for (int j = tid; j < St; j += NT) {
    float acc = 0.f;
    for (int pp = 0; pp < P; ++pp) acc += gq[pp * St + j];
    dqs[b * St + j] += acc;
  }
}

void small_dims(const EfeParams& p, int* Kx, int* Omax) {
  int k = 1, o = 1;
  for (int m = 0; m < p.M; ++m) {
    k = p.mod[m].K > k ? p.mod[m].K : k;
    o = p.mod[m].O > o ? p.mod[m].O : o;
  }
  for (int f = 0; f < p.F; ++f) k = p.fac[f].K > k ? p.fac[f].K : k;
  *Kx = k;
  *Omax = o;
}

}  // namespace

int64_t efe_small_smem_bytes(const EfeParams& p) {
  int Kx = 0, Omax = 0;
  small_dims(p, &Kx, &Omax);
  const int64_t P = p.P, St = p.S_tot;
  return ((p.T + 1) * P * St + 2 * P * Kx + 2 * P * Omax + 2 * P * St + P + Kx + (int64_t)Omax * Kx) * 4;
}

int32_t launch_efe_small(const EfeParams& p, int64_t Bn, bool bwd, const int32_t* pm, int pm_batched,
                         const float* qs, const float* A, const float* B, const float* C, float* G, const float* dG,
                         float* dqs, float* dA, float* dB, float* dC, cudaStream_t stream, bool* used) {
  *used = false;
  const int64_t smem = efe_small_smem_bytes(p);
  if (smem > kEfeSmallMaxSmem || Bn > 0x7fffffff || (p.flags & (B2_FLAG_USE_INDUCTIVE | B2_FLAG_USE_PARAM_INFO_GAIN)))
    return B2_OK;
  int Kx = 0, Omax = 0;
  small_dims(p, &Kx, &Omax);
  const void* kern = bwd ? (const void*)efe_small_kernel<true> : (const void*)efe_small_kernel<false>;
  B2_TRY(ensure_smem_attr(kern, (int)smem, kEfeName));
  if (bwd)
    efe_small_kernel<true><<<(unsigned)Bn, kSmallThreads, (size_t)smem, stream>>>(p, Kx, Omax, pm, pm_batched, qs, A,
                                                                                  B, C, G, dG, dqs, dA, dB, dC);
  else
    efe_small_kernel<false><<<(unsigned)Bn, kSmallThreads, (size_t)smem, stream>>>(p, Kx, Omax, pm, pm_batched, qs,
                                                                                   A, B, C, G, dG, dqs, dA, dB, dC);
  B2_TRY(check_launch(bwd ? "efe_ffi small bwd" : "efe_ffi small"));
  *used = true;
  return B2_OK;
}

}  // namespace b2
