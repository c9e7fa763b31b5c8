// Sequence inference over a window of T steps for a batch of agents:
// run_mmp / run_vmp (pymdp/algos.py:392-430, :512-571), both through
// update_marginals (:170-238). Per iteration, for every step t and factor f:
//   ln q      = log clip q                               (log-marginals of the previous iterate)
//   ln A      = all_marginal_log_likelihood (:30-51): the step's log-likelihood
//               tensors contracted with every other dependency's marginal
//   future    = ln prior at t = 0; for t >= 1 the forward message of the
//               transition into t: MMP log(B_{t-1} . q_{t-1}[deps]), VMP
//               (log B_{t-1}) . q_{t-1}[deps]; MMP halves it for t < T - 1
//               (get_mmp_messages :432-510 / get_vmp_messages :312-390)
//   past      = for t < T - 1, the backward messages of the transitions out of
//               t into every factor i whose B depends on f: MMP 1/2 log(q_{t+1}^i
//               . Bn) with Bn the contraction normalised over f's axis, VMP
//               q_{t+1}^i . (log B) contracted
//   q         = softmax(u - mean u), u = ln q + tau (ln A - ln q + past + future)
//               (mirror_gradient_descent_step :157-168)
// All of it in FP64 on chip: one CTA per agent; log-likelihoods of the whole
// window and five [T][S_tot] planes in shared memory. The agent's transition
// sequence is staged there too when it fits (VMP: log-clipped FP64; MMP: the
// FP32 entries themselves, with reciprocal row sums for factor-local
// transitions), else read from global memory; single-parent transitions take
// a direct S x S path. An iteration is three passes over the window, one
// thread per (factor, step, state) in factor-major order so that a warp's
// lanes share a factor: the messages folded into u; each (step, factor)
// segment's mean, maximum and exponentials; the normaliser, q and log q.
#include <algorithm>
#include <string>
#include <type_traits>

#include "common.cuh"

namespace b2 {
namespace {

constexpr int kSeqMaxF = B2_MAX_FACTORS;
constexpr int kSeqMaxM = B2_MAX_MODALITIES;
constexpr int kSeqMaxRank = B2_MAX_DEP_RANK;
constexpr double kMinD = 2.220446049250313e-16;

struct SeqParams {
  int32_t F, M, T, num_iter, vmp, distr;
  double tau;
  int32_t S_tot;
  int32_t S[kSeqMaxF];
  int32_t qs_off[kSeqMaxF + 1];
  // modalities
  int32_t O[kSeqMaxM], K[kSeqMaxM], rank[kSeqMaxM];
  int8_t dep[kSeqMaxM][kSeqMaxRank];
  int64_t A_off[kSeqMaxM];  // per-agent offset of A_m
  int32_t O_off[kSeqMaxM + 1];  // distribution observations: offset of modality m in one step's row
  int32_t ll_off[kSeqMaxM + 1];  // per step: offset of modality m's log-likelihood in shared memory
  int64_t A_stride;             // 0: A shared by the batch
  // transitions, the action-conditioned sequence (T - 1, S_f, *S[B_deps f]) per factor
  int32_t Kb[kSeqMaxF], brank[kSeqMaxF];
  int8_t bdep[kSeqMaxF][kSeqMaxRank];
  int64_t B_off[kSeqMaxF];
  int64_t B_stride;
  int32_t smem_words;  // doubles of shared memory per agent
  int32_t bstage;      // 1: B (and MMP row sums) staged in shared memory
  int32_t b_sm, rs_sm; // their double offsets in the agent's shared memory
  int32_t kbp[kSeqMaxF];      // staged rows of factor f: odd stride Kb | 1 (conflict-free when lanes walk rows)
  int64_t bsm_off[kSeqMaxF];  // factor f's staged block past b_sm: [(T - 1) S_f][kbp]
  int32_t rs_off[kSeqMaxF];  // factor f's row sums: rs_sm + rs_off[f] + t * S_f + s
};

// 4-byte asynchronous copy global -> shared (no register round trip); completed by cp_async_wait_all
__device__ __forceinline__ void cp_async4(void* smem_dst, const void* gsrc) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// joint of the marginals q[dep_0] x ... x q[dep_{r-1}] at flattened index k
// (row-major), skipping position `skip` (-1: none).
__device__ __forceinline__ double joint_at(const double* __restrict__ q, const int32_t* qs_off, const int32_t* S,
                                           const int8_t* dep, int rank, int k, int skip) {
  double w = 1.0;
  for (int i = rank - 1; i >= 0; --i) {
    const int d = S[dep[i]];
    const int dig = k % d;
    k /= d;
    if (i != skip) w *= q[qs_off[dep[i]] + dig];
  }
  return w;
}

// VMP stages log B in FP64; MMP stages B itself, whose FP32 entries a float holds exactly (half the shared memory)
template <bool VMP>
__global__ void __launch_bounds__(256, 4) seq_kernel(const __grid_constant__ SeqParams p, const float* __restrict__ A,
                                                  const int32_t* __restrict__ obs_idx,
                                                  const float* __restrict__ obs_distr, const float* __restrict__ B,
                                                  const float* __restrict__ prior, float* __restrict__ qs_out) {
  extern __shared__ double sm[];
  __shared__ SeqParams ps;  // fields indexed per lane read from here, not from the constant bank
  const int64_t b = blockIdx.x;
  const int T = p.T, St = p.S_tot, nthr = blockDim.x, tid = threadIdx.x;
  static_assert(sizeof(SeqParams) % 4 == 0, "SeqParams copies in words");
  for (int w = tid; w < (int)(sizeof(SeqParams) / 4); w += nthr)
    reinterpret_cast<int32_t*>(&ps)[w] = reinterpret_cast<const int32_t*>(&p)[w];
  const int ll_step = p.ll_off[p.M];
  double* ll = sm;                      // [T][ll_step]
  double* q = ll + (int64_t)T * ll_step;  // [T][St]
  double* lnq = q + T * St;
  double* fut = lnq + T * St;
  double* past = fut + T * St;
  double* la = past + T * St;
  double* lnp = la + T * St;  // [St]
  // entry x of a pass over the window, factor-major (f, t, s), so that a warp's lanes share one factor:
  // f << 26 | t << 13 | s (t and s < 8192 since 5 T S_tot doubles fit in shared memory, F <= 16)
  int32_t* emap = reinterpret_cast<int32_t*>(lnp + St);
  const float* Ab = A + b * p.A_stride;
  const float* Bb = B + b * p.B_stride;

  __syncthreads();  // ps
  // Every global read of the prologue is issued before any is waited on: cp.async for the observed rows
  // of A (index observations) and for MMP's transitions, plain loads for the rest.
  const int nll = T * ll_step;
  // raw A entries of the observed rows, 4 bytes each, in the upper half of the ll plane shifted by 8 bytes
  // (the last 8 run into q, written only after they are read): converting batch by batch in place, the
  // doubles of a batch land on raw entries of that batch or earlier ones only
  float* raw = reinterpret_cast<float*>(ll) + nll + 2;
  if (!p.distr) {
    for (int e = tid; e < nll; e += nthr) {
      const int t = e / ll_step, r = e - t * ll_step;
      int m = 0;
      while (m + 1 < p.M && r >= ps.ll_off[m + 1]) ++m;
      const int o = __ldg(obs_idx + (b * T + t) * p.M + m), Om = ps.O[m];
      // an index outside [0, O) selects no row: jnp clamps it (A_m[o_m]), as here
      const int oc = o < 0 ? (o + Om < 0 ? 0 : o + Om) : (o >= Om ? Om - 1 : o);
      cp_async4(raw + e, Ab + ps.A_off[m] + (int64_t)oc * ps.K[m] + (r - ps.ll_off[m]));
    }
  }
  // the transition sequence in shared memory when it fits: VMP's log-clipped in FP64, MMP's entries as they are
  using BT = typename std::conditional<VMP, double, float>::type;
  const BT* bsm = reinterpret_cast<const BT*>(sm + p.b_sm);
  double* rsm = sm + p.rs_sm;
  if (p.bstage && !VMP) {
    for (int f = 0; f < p.F; ++f) {
      const int Kb = p.Kb[f], kbp = p.kbp[f];
      const int n = (T - 1) * p.S[f] * Kb;
      const float* Bf = Bb + p.B_off[f];
      BT* dst = reinterpret_cast<BT*>(sm + p.b_sm) + p.bsm_off[f];
      for (int e = tid; e < n; e += nthr) {
        const int row = e / Kb;
        cp_async4(dst + (int64_t)row * kbp + (e - row * Kb), Bf + e);
      }
    }
  }
  // log-likelihoods of every step (compute_log_likelihood_single_modality, pymdp/maths.py:214-238)
  if (p.distr) {
    for (int t = 0; t < T; ++t)
      for (int m = 0; m < p.M; ++m) {
        const float* Am = Ab + p.A_off[m];
        const float* o = obs_distr + (b * T + t) * p.O_off[p.M] + p.O_off[m];
        for (int k = tid; k < p.K[m]; k += nthr) {
          double v = 0.0;
          for (int x = 0; x < p.O[m]; ++x) {
            const double ov = (double)o[x];
            if (ov != 0.0) v += ov * log(fmax((double)__ldg(Am + (int64_t)x * p.K[m] + k), kMinD));
          }
          ll[t * ll_step + p.ll_off[m] + k] = v;
        }
      }
  }
  for (int j = tid; j < St; j += nthr) lnp[j] = log(fmax((double)__ldg(prior + b * St + j), kMinD));
  if (p.bstage && VMP) {
    for (int f = 0; f < p.F; ++f) {
      const int Kb = p.Kb[f], kbp = p.kbp[f];
      const int n = (T - 1) * p.S[f] * Kb;
      const float* Bf = Bb + p.B_off[f];
      BT* dst = reinterpret_cast<BT*>(sm + p.b_sm) + p.bsm_off[f];
      for (int e0 = tid; e0 < n; e0 += 4 * nthr) {
        float bv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) bv[u] = e0 + u * nthr < n ? __ldg(Bf + e0 + u * nthr) : 0.0f;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int e = e0 + u * nthr;
          if (e < n) {
            const int row = e / Kb, k = e - row * Kb;
            dst[(int64_t)row * kbp + k] = (BT)log(fmax((double)bv[u], kMinD));
          }
        }
      }
    }
  }
  for (int x = tid; x < T * St; x += nthr) {
    int f = 0;
    while (f + 1 < p.F && x >= T * p.qs_off[f + 1]) ++f;
    const int local = x - T * p.qs_off[f], t = local / p.S[f];
    emap[x] = f << 26 | t << 13 | (local - t * p.S[f]);
  }
  cp_async_wait_all();
  __syncthreads();
  if (!p.distr) {
    // in place, four entries per thread per batch: the whole batch read before any of it is written
    for (int base = 0; base < nll; base += 4 * nthr) {
      float av[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = base + u * nthr + tid;
        av[u] = e < nll ? raw[e] : 1.0f;
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = base + u * nthr + tid;
        if (e < nll) ll[e] = log(fmax((double)av[u], kMinD));
      }
    }
  }
  if (p.bstage && !VMP) {
    // MMP's normaliser of a single-parent transition: the reciprocal of the row sum over the parent's states
    for (int f = 0; f < p.F; ++f) {
      if (p.brank[f] != 1) continue;
      const int Sf = p.S[f], Kb = p.Kb[f];
      for (int e = tid; e < (T - 1) * Sf; e += nthr) {
        const BT* row = bsm + p.bsm_off[f] + (int64_t)e * p.kbp[f];
        double acc = 0.0;
        for (int k = 0; k < Kb; ++k) acc += (double)row[k];
        rsm[p.rs_off[f] + e] = 1.0 / fmax(acc, kMinD);
      }
    }
  }
  for (int e = tid; e < T * St; e += nthr) {
    const int j = e % St;
    int f = 0;
    while (f + 1 < p.F && j >= p.qs_off[f + 1]) ++f;
    q[e] = 1.0 / p.S[f];
    lnq[e] = log(q[e]);  // afterwards the softmax below writes log q directly
  }
  __syncthreads();
  const double lmin = log(kMinD);
  for (int it = 0; it < p.num_iter; ++it) {
    // messages and marginal log-likelihoods from the previous iterate; factor-indexed fields come from
    // the shared copy of the parameters (a warp's lanes can straddle two factors)
    for (int ei = tid; ei < T * St; ei += nthr) {
      const int32_t em = emap[ei];
      const int f = em >> 26, t = (em >> 13) & 8191, j = ps.qs_off[f] + (em & 8191), e = t * St + j;
      const int s = em & 8191;
      // future message
      double fv;
      if (t == 0) {
        fv = lnp[j];
      } else {
        const int64_t row = ps.B_off[f] + ((int64_t)(t - 1) * ps.S[f] + s) * ps.Kb[f];
        const int64_t srow = ps.bsm_off[f] + ((int64_t)(t - 1) * ps.S[f] + s) * ps.kbp[f];  // staged copy
        const double* qp = q + (t - 1) * St;
        double acc = 0.0;
        if (p.bstage && ps.brank[f] == 1) {
          // single parent: M_{t-1}[s, :] . q_{t-1}[parent]
          const BT* Ms = bsm + srow;
          const double* qd = qp + ps.qs_off[ps.bdep[f][0]];
          double a1 = 0.0;
          int k = 0;
          for (; k + 2 <= ps.Kb[f]; k += 2) {
            acc = fma((double)Ms[k], qd[k], acc);
            a1 = fma((double)Ms[k + 1], qd[k + 1], a1);
          }
          if (k < ps.Kb[f]) acc = fma((double)Ms[k], qd[k], acc);
          acc += a1;
        } else {
          for (int k = 0; k < ps.Kb[f]; ++k) {
            const double w = joint_at(qp, ps.qs_off, ps.S, ps.bdep[f], ps.brank[f], k, -1);
            double mv;
            if (p.bstage) {
              mv = (double)bsm[srow + k];
            } else {
              const double bv = (double)__ldg(Bb + row + k);
              mv = VMP ? log(fmax(bv, kMinD)) : bv;
            }
            acc += mv * w;
          }
        }
        fv = VMP ? acc : log(fmax(acc, kMinD));
      }
      if (!VMP && t < T - 1) fv *= 0.5;
      // past message: transitions out of step t into every factor i whose B depends on f
      double pv = 0.0;
      if (t < T - 1) {
        const double* qt = q + t * St;
        const double* qn = q + (t + 1) * St;
        for (int i = 0; i < p.F; ++i) {
          int pos = -1;
          for (int x = 0; x < ps.brank[i]; ++x)
            if (ps.bdep[i][x] == f) pos = x;
          if (pos < 0) continue;
          const int Si = ps.S[i], Kb = ps.Kb[i];
          // stride of f's axis inside B_i's parent index, and the number of other-parent combinations
          int stf = 1;
          for (int x = ps.brank[i] - 1; x > pos; --x) stf *= ps.S[ps.bdep[i][x]];
          const int64_t bi0 = ps.B_off[i] + (int64_t)t * Si * Kb;
          double acc = 0.0;
          if (p.bstage && ps.brank[i] == 1) {
            // single parent (f itself): M_t[si, s], MMP normalised by the row sum
            const BT* Mi = bsm + ps.bsm_off[i] + (int64_t)t * Si * ps.kbp[i] + s;
            const double* rs = rsm + ps.rs_off[i] + t * Si;
            for (int si = 0; si < Si; ++si) {
              const double mv = (double)Mi[(int64_t)si * ps.kbp[i]];
              acc += qn[ps.qs_off[i] + si] * (VMP ? mv : mv * rs[si]);
            }
            pv += VMP ? acc : 0.5 * log(fmax(acc, kMinD));
            continue;
          }
          const float* Bi = Bb + bi0;
          for (int si = 0; si < Si; ++si) {
            // bm[si][s] = sum over the other parents' states of M_i[si, k] prod q (k with digit_pos = s)
            double bm_s = 0.0, bm_sum = 0.0;
            for (int k = 0; k < Kb; ++k) {
              const int dig = (k / stf) % ps.S[f];
              const double w = joint_at(qt, ps.qs_off, ps.S, ps.bdep[i], ps.brank[i], k, pos);
              double mv;
              if (p.bstage) {
                mv = (double)bsm[ps.bsm_off[i] + ((int64_t)t * Si + si) * ps.kbp[i] + k];
              } else {
                const double bv = (double)__ldg(Bi + (int64_t)si * Kb + k);
                mv = VMP ? log(fmax(bv, kMinD)) : bv;
              }
              if (dig == s) bm_s += mv * w;
              if (!VMP) bm_sum += mv * w;
            }
            if (VMP)
              acc += qn[ps.qs_off[i] + si] * bm_s;
            else
              acc += qn[ps.qs_off[i] + si] * (bm_s / fmax(bm_sum, kMinD));
          }
          pv += VMP ? acc : 0.5 * log(fmax(acc, kMinD));
        }
      }
      // marginal log-likelihood of factor f's state s at step t
      double lv = 0.0;
      const double* qt = q + t * St;
      for (int m = 0; m < p.M; ++m) {
        int pos = -1;
        for (int x = 0; x < ps.rank[m]; ++x)
          if (ps.dep[m][x] == f) pos = x;
        if (pos < 0) continue;
        const double* L = ll + t * ll_step + ps.ll_off[m];
        if (ps.rank[m] == 1) {
          lv += L[s];
          continue;
        }
        if (ps.rank[m] == 2) {
          // one other parent o: a row (f first) or a column (f second) of L_m against q_t[o]
          const int o = ps.dep[m][1 - pos], n = ps.S[o];
          const double* qo = qt + ps.qs_off[o];
          if (pos == 0) {
            // lanes walk rows of length n: each starts at its own column so they spread over the banks
            const double* Lr = L + s * n;
            int c = s % n;
            double acc = 0.0;
            for (int x = 0; x < n; ++x) {
              acc = fma(Lr[c], qo[c], acc);
              c = c + 1 == n ? 0 : c + 1;
            }
            lv += acc;
          } else {
            const int Sf = ps.S[f];
            double acc = 0.0;
            for (int x = 0; x < n; ++x) acc = fma(L[x * Sf + s], qo[x], acc);
            lv += acc;
          }
          continue;
        }
        int stf = 1;
        for (int x = ps.rank[m] - 1; x > pos; --x) stf *= ps.S[ps.dep[m][x]];
        const int Km = ps.K[m], outer = Km / (stf * ps.S[f]);
        for (int a = 0; a < outer; ++a)
          for (int c = 0; c < stf; ++c) {
            const int k = (a * ps.S[f] + s) * stf + c;
            lv += L[k] * joint_at(qt, ps.qs_off, ps.S, ps.dep[m], ps.rank[m], k, pos);
          }
      }
      // mirror-descent step (pymdp/algos.py:157-168): u = ln q + tau (ll - ln q + past + future)
      fut[e] = lnq[e] + p.tau * (lv - lnq[e] + pv + fv);
    }
    __syncthreads();
    // softmax of every (t, f) segment, one thread per entry: each reads its segment's mean and max back
    // from shared memory, then the segment's exponentials for the normaliser
    for (int ei = tid; ei < T * St; ei += nthr) {
      const int32_t em = emap[ei];
      const int f = em >> 26, t = (em >> 13) & 8191, j = ps.qs_off[f] + (em & 8191), e = t * St + j;
      const int o = t * St + ps.qs_off[f], n = ps.S[f];
      double sum = 0.0;
      for (int x = 0; x < n; ++x) sum += fut[o + x];
      const double mean = sum / n;
      double mx = -INFINITY;
      for (int x = 0; x < n; ++x) mx = fmax(mx, fut[o + x] - mean);
      const double d = fut[e] - mean - mx;
      past[e] = d;
      la[e] = exp(d);
    }
    __syncthreads();
    // q = e / z, and log(max(q, eps)) for the next iteration as d - log z, clipped at log eps
    for (int ei = tid; ei < T * St; ei += nthr) {
      const int32_t em = emap[ei];
      const int f = em >> 26, t = (em >> 13) & 8191, j = ps.qs_off[f] + (em & 8191), e = t * St + j;
      const int o = t * St + ps.qs_off[f], n = ps.S[f];
      double z = 0.0;
      for (int x = 0; x < n; ++x) z += la[o + x];
      q[e] = la[e] / z;
      lnq[e] = fmax(past[e] - log(z), lmin);
    }
    __syncthreads();
  }
  for (int e = tid; e < T * St; e += nthr) qs_out[b * T * St + e] = (float)q[e];
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_sequence_infer(void* stream, int32_t vmp, const float* A, int64_t A_count, int32_t A_batched,
                                     const int64_t* O, int64_t M, const int32_t* obs_idx, const float* obs_distr,
                                     int64_t obs_count, const float* B_seq, int64_t B_count, const float* prior,
                                     int64_t prior_count, float* qs_out, int64_t qs_count, int64_t Bn, int64_t T,
                                     int64_t F, const int64_t* S, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                                     const int64_t* A_dep_offsets, const int64_t* B_dep_flat,
                                     int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int32_t num_iter,
                                     float tau) {
  const char* op = vmp ? "run_vmp" : "run_mmp";
  auto bad = [&](const std::string& m) { return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": " + m); };
  if (F < 1 || F > kSeqMaxF || M < 1 || M > kSeqMaxM) return bad("F and M must lie in [1, 16] and [1, 32]");
  if (T < 1 || T > 4096 || num_iter < 0 || Bn < 0) return bad("invalid T, num_iter or Bn");
  if (!S || !O || !A_dep_offsets || !B_dep_offsets || (A_dep_flat_len && !A_dep_flat) ||
      (B_dep_flat_len && !B_dep_flat))
    return bad("null attribute array");
  if ((obs_idx == nullptr) == (obs_distr == nullptr)) return bad("pass exactly one of obs_idx, obs_distr");
  SeqParams p{};
  p.F = (int32_t)F;
  p.M = (int32_t)M;
  p.T = (int32_t)T;
  p.num_iter = num_iter;
  p.vmp = vmp ? 1 : 0;
  p.distr = obs_distr ? 1 : 0;
  p.tau = (double)tau;
  int St = 0;
  for (int f = 0; f < F; ++f) {
    if (S[f] < 1 || S[f] > 1024) return bad("S must lie in [1, 1024]");
    p.S[f] = (int32_t)S[f];
    p.qs_off[f] = St;
    St += (int)S[f];
  }
  p.qs_off[F] = St;
  p.S_tot = St;
  if (A_dep_offsets[0] != 0 || B_dep_offsets[0] != 0) return bad("dependency offsets must start at 0");
  int64_t aoff = 0, ll = 0, ooff = 0;
  for (int m = 0; m < M; ++m) {
    const int64_t r = A_dep_offsets[m + 1] - A_dep_offsets[m];
    if (r < 1 || r > kSeqMaxRank || A_dep_offsets[m + 1] > A_dep_flat_len) return bad("A dependency ranks in [1, 8]");
    if (O[m] < 1) return bad("O must be positive");
    int64_t K = 1;
    for (int64_t x = 0; x < r; ++x) {
      const int64_t d = A_dep_flat[A_dep_offsets[m] + x];
      if (d < 0 || d >= F) return bad("A dependency out of range");
      for (int64_t y = 0; y < x; ++y)
        if (A_dep_flat[A_dep_offsets[m] + y] == d) return bad("duplicate factor in A_dependencies");
      p.dep[m][x] = (int8_t)d;
      K *= S[d];
    }
    if (K > (1 << 20)) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": A modality too large");
    p.O[m] = (int32_t)O[m];
    p.K[m] = (int32_t)K;
    p.rank[m] = (int32_t)r;
    p.A_off[m] = aoff;
    p.O_off[m] = (int32_t)ooff;
    p.ll_off[m] = (int32_t)ll;
    aoff += O[m] * K;
    ooff += O[m];
    ll += K;
  }
  p.O_off[M] = (int32_t)ooff;
  p.ll_off[M] = (int32_t)ll;
  p.A_stride = A_batched ? aoff : 0;
  int64_t boff = 0;
  for (int f = 0; f < F; ++f) {
    const int64_t r = B_dep_offsets[f + 1] - B_dep_offsets[f];
    if (r < 1 || r > kSeqMaxRank || B_dep_offsets[f + 1] > B_dep_flat_len) return bad("B dependency ranks in [1, 8]");
    int64_t K = 1;
    for (int64_t x = 0; x < r; ++x) {
      const int64_t d = B_dep_flat[B_dep_offsets[f] + x];
      if (d < 0 || d >= F) return bad("B dependency out of range");
      p.bdep[f][x] = (int8_t)d;
      K *= S[d];
    }
    if (K > (1 << 20)) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": B parent joint too large");
    p.Kb[f] = (int32_t)K;
    p.brank[f] = (int32_t)r;
    p.B_off[f] = boff;
    boff += (T - 1) * S[f] * K;
  }
  p.B_stride = boff;
  const int64_t words = T * ll + 5 * T * St + St + (T * St + 1) / 2;  // + the int32 entry map
  if (words * 8 > 200 * 1024)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": window of " + std::to_string(words * 8) +
                                        " bytes of FP64 state exceeds 200 KB of shared memory");
  // stage B (and MMP's single-parent row sums) when the whole state stays under 200 KB
  int64_t rs_words = 0, bs_elems = 0;
  for (int f = 0; f < F; ++f) {
    p.rs_off[f] = (int32_t)rs_words;
    if (p.brank[f] == 1) rs_words += (T - 1) * S[f];
    p.kbp[f] = p.Kb[f] | 1;
    p.bsm_off[f] = bs_elems;
    bs_elems += (T - 1) * S[f] * p.kbp[f];
  }
  const int64_t bs_words = vmp ? bs_elems : (bs_elems + 1) / 2;  // MMP stages floats
  const int64_t staged = words + bs_words + rs_words;
  p.bstage = staged * 8 <= 200 * 1024 && boff < (1 << 30) ? 1 : 0;
  p.b_sm = (int32_t)words;
  p.rs_sm = (int32_t)(words + bs_words);
  p.smem_words = (int32_t)(p.bstage ? staged : words);
  if (A_count != (A_batched ? Bn : 1) * aoff) return bad("A element_count mismatch");
  if (obs_count != Bn * T * (obs_distr ? ooff : M)) return bad("observation element_count mismatch");
  if (B_count != Bn * boff) return bad("B element_count mismatch");
  if (prior_count != Bn * St || qs_count != Bn * T * St) return bad("prior / qs element_count mismatch");
  if (Bn == 0) return B2_OK;
  if (!A || (boff > 0 && !B_seq) || !prior || !qs_out) return bad("null buffer");
  if (Bn > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
  const int bytes = (int)((int64_t)p.smem_words * 8);
  const auto kernel = vmp ? seq_kernel<true> : seq_kernel<false>;
  B2_TRY(ensure_smem_attr((const void*)kernel, bytes, op));
  // one thread per (step, state) up to 256: idle warps would only hold registers that other agents could use
  const int nthr = (int)std::min<int64_t>(256, (T * St + 31) / 32 * 32);
  kernel<<<(unsigned)Bn, nthr, bytes, (cudaStream_t)stream>>>(p, A, obs_idx, obs_distr, B_seq, prior, qs_out);
  return check_launch(op);
}
