// Exact single-factor HMM filtering and smoothing for a batch of agents:
// the reference's run_exact_single_factor_hmm_scan (pymdp/algos.py:1132-1208)
// = hmm_filter_scan_colstoch (:959-988) + hmm_smoother_from_filtered_colstoch
// (:1049-1130), and smoothing_exact (pymdp/inference.py:595-634).
//
// The reference parallelises over time with lax.associative_scan because one
// sequence is its unit of work. Here the unit is one agent's sequence, and a
// batch holds thousands of them: one warp (K <= 32) or CTA per agent runs the recurrences in
// time order (each step a K x K matrix-vector product in FP64 from shared
// memory), which is the same algebra as the scan without its log2(T) extra
// matrix products. B lives in shared memory (all actions of a stationary B
// once per agent; a time-varying B step by step), rows padded by one float so
// both the row and the column walks are conflict-free.
//
// Forward (filter), with p_0 = prior and, for t >= 1, p_t = B_{t-1} f_{t-1}:
//   ll_t[k] = sum_m log clip(A_m[o_{m,t}, k])   (or sum_o o[o] log clip(A_m[o, k]))
//   w = exp(ll_t - max ll_t), u = p_t * w, c = sum u
//   f_t = u / c,  mll += log c + max ll_t        (_condition_on, algos.py:750-775)
// Backward (smoother from filtered), s_{T-1} = f_{T-1}:
//   pn_t = B_t f_t, cond_t[j, i] = B_t[j, i] f_t[i] / clip(pn_t[j])
//   s_t[i] = sum_j cond_t[j, i] s_{t+1}[j]; smoothed_t = s_t / clip(sum s_t)
//   joint_t[j, i] = cond_t[j, i] * smoothed_{t+1}[j]
#include "common.cuh"

namespace b2 {
namespace {

constexpr int kHmmThreads = 128;
constexpr int kHmmMaxK = 128;
constexpr double kHmmMinVal = 2.220446049250313e-16;

struct HmmParams {
  int32_t T, K, U;       // U = 0: time-varying B [T-1, K, K]
  int32_t M;             // modalities (forward only)
  int32_t obs_stride;    // M (index observations) or sum O (distributions)
  int32_t action_mode;   // 0: jnp indexing (negative from the end, clamped); 1: negative -> identity
  int32_t stage_all;     // stationary B staged once per agent
  int32_t wstage;        // warp kernels: A, observations and actions staged in shared memory
  int64_t A_stride;      // A floats per agent (0: shared by every agent)
  int64_t B_stride;      // B floats per agent (0: shared)
  int32_t O[B2_MAX_MODALITIES];
  int64_t A_off[B2_MAX_MODALITIES];
  int32_t O_off[B2_MAX_MODALITIES];  // start of modality m in a distribution row
};

__device__ __forceinline__ double block_sum(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = 0.0;
  for (int i = 0; i < kHmmThreads / 32; ++i) s += red[i];
  return s;
}

__device__ __forceinline__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  double s = red[0];
  for (int i = 1; i < kHmmThreads / 32; ++i) s = fmax(s, red[i]);
  return s;
}

// Action of transition t of agent b as an index into B's last axis, or -1 for
// the identity transition.
__device__ __forceinline__ int hmm_action(const HmmParams& p, const int32_t* act, int64_t b, int t) {
  if (p.U <= 0) return 0;
  int u = act ? act[b * (p.T - 1) + t] : 0;
  if (p.action_mode == 1) return u < 0 ? -1 : (u >= p.U ? p.U - 1 : u);
  if (u < 0) u += p.U;  // jnp indexing: negative from the end, then clamped
  return u < 0 ? 0 : (u >= p.U ? p.U - 1 : u);
}

// Shared tile of transition t: pointer to a K x (K+1) padded [next][current]
// matrix, staging it first when B is time-varying or not staged whole. Ends
// with a barrier when it stages. Returns nullptr for the identity transition.
__device__ const float* hmm_stage(const HmmParams& p, const float* Bb, float* tile, const int32_t* act, int64_t b,
                                  int t) {
  const int K = p.K, ld = K + 1;
  const int u = hmm_action(p, act, b, t);
  if (u < 0) return nullptr;
  if (p.U > 0 && p.stage_all) return tile + (int64_t)u * K * ld;
  __syncthreads();  // the previous step's readers are done with the tile
  if (p.U == 0) {
    const float* src = Bb + (int64_t)t * K * K;
    for (int e = threadIdx.x; e < K * K; e += kHmmThreads) tile[(e / K) * ld + e % K] = src[e];
  } else {
    for (int e = threadIdx.x; e < K * K; e += kHmmThreads) tile[(e / K) * ld + e % K] = Bb[(int64_t)e * p.U + u];
  }
  __syncthreads();
  return tile;
}

// One agent's backward pass from its filtered marginals (global, FP32; each
// thread reads back only the entries it wrote in the forward pass).
__device__ void hmm_backward(const HmmParams& p, const float* Bb, float* tile, const int32_t* act, int64_t b,
                             const float* filt, float* smoothed, float* joint, float* cond, double* f, double* inv_pn,
                             double* s_next, double* red) {
  const int K = p.K, ld = K + 1, T = p.T, j = threadIdx.x;
  const bool own = j < K;
  double s = own ? (double)filt[(int64_t)(T - 1) * K + j] : 0.0;  // s_{T-1} = f_{T-1}
  double tot = block_sum(s, red);
  if (own) {
    s_next[j] = s;
    if (smoothed) smoothed[(int64_t)(T - 1) * K + j] = (float)(s / fmax(tot, kHmmMinVal));
  }
  double sn_norm = tot;  // normaliser of s_{t+1}
  for (int t = T - 2; t >= 0; --t) {
    const float* Bt = hmm_stage(p, Bb, tile, act, b, t);
    if (own) f[j] = (double)filt[(int64_t)t * K + j];
    __syncthreads();
    if (own) {
      double pn = 0.0;  // pn_t[j] = sum_i B_t[j, i] f_t[i]
      if (Bt) {
        for (int i = 0; i < K; ++i) pn += (double)Bt[j * ld + i] * f[i];
      } else {
        pn = f[j];
      }
      inv_pn[j] = 1.0 / fmax(pn, kHmmMinVal);
    }
    __syncthreads();
    double si = 0.0;
    if (own) {  // s_t[i] = f_t[i] * sum_j B_t[j, i] inv_pn[j] s_{t+1}[j]  (thread = i)
      double acc = 0.0;
      if (Bt) {
        for (int jj = 0; jj < K; ++jj) acc += (double)Bt[jj * ld + j] * inv_pn[jj] * s_next[jj];
      } else {
        acc = inv_pn[j] * s_next[j];
      }
      si = f[j] * acc;
    }
    // pairwise outputs of step t use the normalised s_{t+1}
    const double inv_sn = 1.0 / fmax(sn_norm, kHmmMinVal);
    if (joint || cond) {
      float* jo = joint ? joint + (int64_t)t * K * K : nullptr;
      float* co = cond ? cond + (int64_t)t * K * K : nullptr;
      for (int e = threadIdx.x; e < K * K; e += kHmmThreads) {
        const int r = e / K, c = e % K;  // [next r][current c]
        const double bt = Bt ? (double)Bt[r * ld + c] : (r == c ? 1.0 : 0.0);
        const double cd = bt * f[c] * inv_pn[r];
        if (co) co[e] = (float)cd;
        if (jo) jo[e] = (float)(cd * (s_next[r] * inv_sn));
      }
    }
    tot = block_sum(si, red);  // its barriers order the reads of s_next / f / tile above before the writes below
    if (own) {
      s_next[j] = si;
      if (smoothed) smoothed[(int64_t)t * K + j] = (float)(si / fmax(tot, kHmmMinVal));
    }
    sn_norm = tot;
  }
}

// Stages every action of a stationary B once (ends with a barrier).
__device__ void hmm_stage_all(const HmmParams& p, const float* Bb, float* tile) {
  const int K = p.K, ld = K + 1;
  const int64_t n = (int64_t)K * K * p.U;
  for (int64_t e = threadIdx.x; e < n; e += kHmmThreads) {
    const int u = (int)(e % p.U);
    const int64_t jk = e / p.U;  // B[j, i, u] at (j * K + i) * U + u
    tile[(int64_t)u * K * ld + (jk / K) * ld + jk % K] = Bb[e];
  }
  __syncthreads();
}

size_t hmm_smem_bytes(const HmmParams& p) {
  const int64_t tiles = (p.U > 0 && p.stage_all) ? p.U : 1;
  return (size_t)(tiles * p.K * (p.K + 1)) * sizeof(float) + 4 * kHmmMaxK * sizeof(double) + 64 * sizeof(double);
}

__device__ __forceinline__ double* hmm_vectors(unsigned char* smem, const HmmParams& p) {
  const int64_t tiles = (p.U > 0 && p.stage_all) ? p.U : 1;
  return reinterpret_cast<double*>(smem + ((tiles * p.K * (p.K + 1) * sizeof(float) + 15) & ~size_t(15)));
}

__global__ void __launch_bounds__(kHmmThreads)
hmm_smoother_kernel(const HmmParams p, const float* __restrict__ A, const int32_t* __restrict__ obs,
                    const float* __restrict__ obs_dist, const float* __restrict__ prior, const float* __restrict__ B,
                    const int32_t* __restrict__ act, float* __restrict__ mll, float* __restrict__ filtered,
                    float* __restrict__ predicted, float* __restrict__ smoothed, float* __restrict__ joint,
                    float* __restrict__ cond) {
  extern __shared__ __align__(16) unsigned char hmm_smem[];
  const int64_t b = blockIdx.x;
  const int K = p.K, ld = K + 1, T = p.T, j = threadIdx.x;
  const bool own = j < K;
  float* tile = reinterpret_cast<float*>(hmm_smem);
  double* vec = hmm_vectors(hmm_smem, p);
  double* f = vec;
  double* red = vec + 4 * kHmmMaxK;
  const float* Ab = A + b * p.A_stride;
  const float* Bb = B + b * p.B_stride;
  float* filt = filtered + b * (int64_t)T * K;
  if (p.U > 0 && p.stage_all) hmm_stage_all(p, Bb, tile);
  double m_ll = 0.0;
  for (int t = 0; t < T; ++t) {
    const float* Bt = t > 0 ? hmm_stage(p, Bb, tile, act, b, t - 1) : nullptr;
    double pj = 0.0;
    if (own) {
      if (t == 0) {
        pj = (double)prior[b * K + j];
      } else if (Bt) {
        for (int i = 0; i < K; ++i) pj += (double)Bt[j * ld + i] * f[i];
      } else {
        pj = f[j];
      }
    }
    // log-likelihood of state j (compute_log_likelihood, maths.py:214-263)
    double ll = -INFINITY;
    if (own) {
      ll = 0.0;
      for (int m = 0; m < p.M; ++m) {
        const float* Am = Ab + p.A_off[m];
        if (obs_dist) {
          const float* od = obs_dist + (b * T + t) * p.obs_stride + p.O_off[m];
          double s = 0.0;
          for (int o = 0; o < p.O[m]; ++o) s += (double)od[o] * log(fmax((double)Am[(int64_t)o * K + j], kHmmMinVal));
          ll += s;
        } else {
          int o = obs[(b * T + t) * p.obs_stride + m];
          if (o < 0) o += p.O[m];  // jnp indexing: negative from the end, then clamped
          o = o < 0 ? 0 : (o >= p.O[m] ? p.O[m] - 1 : o);
          ll += log(fmax((double)Am[(int64_t)o * K + j], kHmmMinVal));
        }
      }
    }
    const double lmax = block_max(ll, red);
    const double u = own ? pj * exp(ll - lmax) : 0.0;
    double c = block_sum(u, red);
    if (c == 0.0) c = 1.0;  // _normalize_preserve_zeros: an all-zero row stays zero
    m_ll += log(fmax(c, kHmmMinVal)) + lmax;
    if (own) {
      const double fj = u / c;
      f[j] = fj;  // every read of f for this step happened before block_max's barriers
      filt[(int64_t)t * K + j] = (float)fj;
      if (predicted) predicted[(b * T + t) * K + j] = (float)pj;
    }
    __syncthreads();
  }
  if (mll && threadIdx.x == 0) mll[b] = (float)m_ll;
  if (!smoothed && !joint && !cond) return;
  hmm_backward(p, Bb, tile, act, b, filt, smoothed ? smoothed + b * (int64_t)T * K : nullptr,
               joint ? joint + b * (int64_t)(T - 1) * K * K : nullptr,
               cond ? cond + b * (int64_t)(T - 1) * K * K : nullptr, vec + 3 * kHmmMaxK, vec + kHmmMaxK,
               vec + 2 * kHmmMaxK, red);
}

__global__ void __launch_bounds__(kHmmThreads)
hmm_from_filtered_kernel(const HmmParams p, const float* __restrict__ filtered, const float* __restrict__ B,
                         const int32_t* __restrict__ act, float* __restrict__ smoothed, float* __restrict__ joint,
                         float* __restrict__ cond) {
  extern __shared__ __align__(16) unsigned char hmm_smem[];
  const int64_t b = blockIdx.x;
  const int K = p.K, T = p.T;
  float* tile = reinterpret_cast<float*>(hmm_smem);
  double* vec = hmm_vectors(hmm_smem, p);
  const float* Bb = B + b * p.B_stride;
  if (p.U > 0 && p.stage_all) hmm_stage_all(p, Bb, tile);
  hmm_backward(p, Bb, tile, act, b, filtered + b * (int64_t)T * K, smoothed ? smoothed + b * (int64_t)T * K : nullptr,
               joint ? joint + b * (int64_t)(T - 1) * K * K : nullptr,
               cond ? cond + b * (int64_t)(T - 1) * K * K : nullptr, vec + 3 * kHmmMaxK, vec + kHmmMaxK,
               vec + 2 * kHmmMaxK, vec + 4 * kHmmMaxK);
}

// ------------------------------------------------------------ K <= 32
// One warp per agent: lane j owns state j, the vectors live in registers and
// move between lanes by shuffles, so a step has no block barrier (the CTA
// kernel above spends most of its time waiting at them when K <= 32, where
// only one of its four warps does the K x K products). Pairwise outputs are
// written a row per iteration, lane = column: coalesced, no index division.
constexpr size_t kHmmWarpStageMax = 48 * 1024;  // all actions of B per agent, else one tile per step

__device__ __forceinline__ double warp_sum_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max_d(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Padded [next][current] tile of transition t (nullptr = identity).
// Action of transition t from one agent's action row (nullptr = action 0).
__device__ __forceinline__ int hmm_waction(const HmmParams& p, const int32_t* ab, int t) {
  if (p.U <= 0) return 0;
  int u = ab ? ab[t] : 0;
  if (p.action_mode == 1) return u < 0 ? -1 : (u >= p.U ? p.U - 1 : u);
  if (u < 0) u += p.U;  // jnp indexing: negative from the end, then clamped
  return u < 0 ? 0 : (u >= p.U ? p.U - 1 : u);
}

template <bool ALL>
__device__ __forceinline__ const float* hmm_wtile(const HmmParams& p, const float* Bb, float* tile,
                                                  const int32_t* ab, int t) {
  const int K = p.K, ld = K + 1, c = threadIdx.x;
  const int u = hmm_waction(p, ab, t);
  if (u < 0) return nullptr;
  if (ALL && p.U > 0) return tile + (int64_t)u * K * ld;
  __syncwarp();  // the lanes are done reading the previous tile
  if (c < K) {
    if (p.U == 0) {
      const float* src = Bb + (int64_t)t * K * K;
      for (int r = 0; r < K; ++r) tile[r * ld + c] = src[r * K + c];
    } else {
      for (int r = 0; r < K; ++r) tile[r * ld + c] = Bb[((int64_t)r * K + c) * p.U + u];
    }
  }
  __syncwarp();
  return tile;
}

// Backward pass of one agent from its filtered marginals (each lane reads
// back only its own entries).
template <bool ALL>
__device__ void hmm_wbackward(const HmmParams& p, const float* Bb, float* tile, const int32_t* ab,
                              const float* filt, float* smoothed, float* joint, float* cond) {
  const int K = p.K, ld = K + 1, T = p.T, j = threadIdx.x;
  const bool own = j < K;
  double s_next = own ? (double)filt[(int64_t)(T - 1) * K + j] : 0.0;  // s_{T-1} = f_{T-1}
  double ft_next = (own && T >= 2) ? (double)filt[(int64_t)(T - 2) * K + j] : 0.0;
  double sn_norm = warp_sum_d(s_next);
  if (own && smoothed) smoothed[(int64_t)(T - 1) * K + j] = (float)(s_next / fmax(sn_norm, kHmmMinVal));
  for (int t = T - 2; t >= 0; --t) {
    const double ft = ft_next;
    if (own && t > 0) ft_next = (double)filt[(int64_t)(t - 1) * K + j];  // one step ahead: hides its latency
    const float* Bt = hmm_wtile<ALL>(p, Bb, tile, ab, t);
    double pn = ft;  // pn_t[j] = sum_i B_t[j, i] f_t[i]
    if (Bt) {
      pn = 0.0;
      for (int i = 0; i < K; ++i) {
        const double fi = __shfl_sync(0xffffffffu, ft, i);
        if (own) pn += (double)Bt[j * ld + i] * fi;
      }
    }
    const double ipn = own ? 1.0 / fmax(pn, kHmmMinVal) : 0.0;
    const double w = ipn * s_next;  // row weight of s_t = cond^T s_{t+1}
    double acc = w;                 // s_t[i] = f_t[i] * sum_j B_t[j, i] w_j  (lane = i)
    if (Bt) {
      acc = 0.0;
      for (int r = 0; r < K; ++r) {
        const double wr = __shfl_sync(0xffffffffu, w, r);
        if (own) acc += (double)Bt[r * ld + j] * wr;
      }
    }
    const double si = own ? ft * acc : 0.0;
    if (joint || cond) {  // cond[t, r, c] = B[r, c] f[c] / pn[r]; joint = cond * smoothed_{t+1}[r]
      float* co = cond ? cond + (int64_t)t * K * K : nullptr;
      float* jo = joint ? joint + (int64_t)t * K * K : nullptr;
      const double inv_sn = 1.0 / fmax(sn_norm, kHmmMinVal);
      const float fc = (float)ft;
      for (int r = 0; r < K; ++r) {
        const float rc = (float)__shfl_sync(0xffffffffu, ipn, r);
        const float rj = (float)(__shfl_sync(0xffffffffu, w, r) * inv_sn);
        if (own) {
          const float base = (Bt ? Bt[r * ld + j] : (r == j ? 1.f : 0.f)) * fc;
          if (co) co[r * K + j] = base * rc;
          if (jo) jo[r * K + j] = base * rj;
        }
      }
    }
    const double tot = warp_sum_d(si);
    if (own && smoothed) smoothed[(int64_t)t * K + j] = (float)(si / fmax(tot, kHmmMinVal));
    s_next = si;
    sn_norm = tot;
  }
}

template <bool ALL>
__device__ void hmm_wstage_all(const HmmParams& p, const float* Bb, float* tile) {
  const int K = p.K, ld = K + 1, c = threadIdx.x;
  if (ALL && p.U > 0 && c < K)
    for (int u = 0; u < p.U; ++u)
      for (int r = 0; r < K; ++r) tile[((int64_t)u * K + r) * ld + c] = Bb[((int64_t)r * K + c) * p.U + u];
  __syncwarp();
}

template <bool ALL>
__global__ void __launch_bounds__(32)
hmm_smoother_warp_kernel(const HmmParams p, const float* __restrict__ A, const int32_t* __restrict__ obs,
                         const float* __restrict__ obs_dist, const float* __restrict__ prior,
                         const float* __restrict__ B, const int32_t* __restrict__ act, float* __restrict__ mll,
                         float* __restrict__ filtered, float* __restrict__ predicted, float* __restrict__ smoothed,
                         float* __restrict__ joint, float* __restrict__ cond) {
  extern __shared__ __align__(16) unsigned char hmm_smem[];
  float* tile = reinterpret_cast<float*>(hmm_smem);
  const int64_t b = blockIdx.x;
  const int K = p.K, ld = K + 1, T = p.T, j = threadIdx.x;
  const bool own = j < K;
  const float* Ab = A + b * p.A_stride;
  const float* Bb = B + b * p.B_stride;
  float* filt = filtered + b * (int64_t)T * K;
  hmm_wstage_all<ALL>(p, Bb, tile);
  // this agent's A, observations and actions: staged once, so no step waits on
  // a chain of global loads (observation -> row of A, action -> tile)
  const int64_t a_words = p.A_off[p.M - 1] + (int64_t)p.O[p.M - 1] * K;
  const int64_t o_words = (int64_t)T * p.obs_stride;
  const float* Aw = Ab;
  const int32_t* obw = obs ? obs + b * o_words : nullptr;
  const float* odw = obs_dist ? obs_dist + b * o_words : nullptr;
  const int32_t* aw = act ? act + b * (T - 1) : nullptr;
  if (p.wstage) {
    const size_t tile_bytes = ((size_t)((ALL && p.U > 0) ? p.U : 1) * K * ld * sizeof(float) + 15) & ~size_t(15);
    float* As = reinterpret_cast<float*>(hmm_smem + tile_bytes);
    uint32_t* Os = reinterpret_cast<uint32_t*>(As + a_words);
    int32_t* Ws = reinterpret_cast<int32_t*>(Os + o_words);
    for (int64_t e = j; e < a_words; e += 32) As[e] = Ab[e];
    const uint32_t* osrc = obs_dist ? reinterpret_cast<const uint32_t*>(odw) : reinterpret_cast<const uint32_t*>(obw);
    for (int64_t e = j; e < o_words; e += 32) Os[e] = osrc[e];
    if (aw)
      for (int e = j; e < T - 1; e += 32) Ws[e] = aw[e];
    __syncwarp();
    Aw = As;
    if (obs_dist) odw = reinterpret_cast<const float*>(Os); else obw = reinterpret_cast<const int32_t*>(Os);
    if (aw) aw = Ws;
  }
  double f = 0.0, m_ll = 0.0;
  for (int t = 0; t < T; ++t) {
    double pj;
    if (t == 0) {
      pj = own ? (double)prior[b * K + j] : 0.0;
    } else {
      const float* Bt = hmm_wtile<ALL>(p, Bb, tile, aw, t - 1);
      pj = f;
      if (Bt) {
        pj = 0.0;
        for (int i = 0; i < K; ++i) {
          const double fi = __shfl_sync(0xffffffffu, f, i);
          if (own) pj += (double)Bt[j * ld + i] * fi;
        }
      }
    }
    double ll = -INFINITY;
    if (own) {
      ll = 0.0;
      for (int m = 0; m < p.M; ++m) {
        const float* Am = Aw + p.A_off[m];
        if (obs_dist) {
          const float* od = odw + (int64_t)t * p.obs_stride + p.O_off[m];
          double s = 0.0;
          for (int o = 0; o < p.O[m]; ++o) s += (double)od[o] * log(fmax((double)Am[(int64_t)o * K + j], kHmmMinVal));
          ll += s;
        } else {
          int o = obw[(int64_t)t * p.obs_stride + m];
          if (o < 0) o += p.O[m];  // jnp indexing: negative from the end, then clamped
          o = o < 0 ? 0 : (o >= p.O[m] ? p.O[m] - 1 : o);
          ll += log(fmax((double)Am[(int64_t)o * K + j], kHmmMinVal));
        }
      }
    }
    const double lmax = warp_max_d(ll);
    const double u = own ? pj * exp(ll - lmax) : 0.0;
    double c = warp_sum_d(u);
    if (c == 0.0) c = 1.0;  // _normalize_preserve_zeros: an all-zero row stays zero
    m_ll += log(fmax(c, kHmmMinVal)) + lmax;
    f = u / c;
    if (own) {
      filt[(int64_t)t * K + j] = (float)f;
      if (predicted) predicted[(b * T + t) * K + j] = (float)pj;
    }
  }
  if (mll && j == 0) mll[b] = (float)m_ll;
  if (!smoothed && !joint && !cond) return;
  hmm_wbackward<ALL>(p, Bb, tile, aw, filt, smoothed ? smoothed + b * (int64_t)T * K : nullptr,
                     joint ? joint + b * (int64_t)(T - 1) * K * K : nullptr,
                     cond ? cond + b * (int64_t)(T - 1) * K * K : nullptr);
}

template <bool ALL>
__global__ void __launch_bounds__(32)
hmm_from_filtered_warp_kernel(const HmmParams p, const float* __restrict__ filtered, const float* __restrict__ B,
                              const int32_t* __restrict__ act, float* __restrict__ smoothed,
                              float* __restrict__ joint, float* __restrict__ cond) {
  extern __shared__ __align__(16) unsigned char hmm_smem[];
  float* tile = reinterpret_cast<float*>(hmm_smem);
  const int64_t b = blockIdx.x;
  const int K = p.K, T = p.T;
  const float* Bb = B + b * p.B_stride;
  hmm_wstage_all<ALL>(p, Bb, tile);
  hmm_wbackward<ALL>(p, Bb, tile, act ? act + b * (T - 1) : nullptr, filtered + b * (int64_t)T * K,
                     smoothed ? smoothed + b * (int64_t)T * K : nullptr,
                     joint ? joint + b * (int64_t)(T - 1) * K * K : nullptr,
                     cond ? cond + b * (int64_t)(T - 1) * K * K : nullptr);
}

constexpr size_t kHmmWarpInputMax = 40 * 1024;  // staged A + observations + actions per agent

// Shared memory of the warp kernels; *all = every action of B staged once.
// With `inputs`, also decides p.wstage (A, observations and actions staged).
size_t hmm_warp_smem(HmmParams& p, bool* all, bool inputs) {
  const size_t one = (size_t)p.K * (p.K + 1) * sizeof(float);
  *all = p.U > 0 && one * p.U <= kHmmWarpStageMax;
  const size_t tile = ((*all ? one * p.U : one) + 15) & ~size_t(15);
  p.wstage = 0;
  if (!inputs) return tile;
  const size_t a_words = (size_t)(p.A_off[p.M - 1] + (int64_t)p.O[p.M - 1] * p.K);
  const size_t extra = 4 * (a_words + (size_t)p.T * p.obs_stride + (size_t)p.T);
  p.wstage = extra <= kHmmWarpInputMax ? 1 : 0;
  return tile + (p.wstage ? extra : 0);
}

constexpr size_t kHmmMaxSmem = 200 * 1024;

// Validates the transition layout; fills p.U / p.B_stride / p.stage_all.
int32_t hmm_transitions(const char* op, HmmParams& p, int64_t Bn, int64_t U, int32_t B_batched, int64_t B_count,
                        const int32_t* actions, int64_t actions_count) {
  const int64_t K = p.K, T = p.T;
  if (U < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": U must be >= 0");
  const int64_t per = U == 0 ? (T - 1) * K * K : K * K * U;
  p.U = (int32_t)U;
  p.B_stride = B_batched ? per : 0;
  if (B_count != (B_batched ? Bn : 1) * per)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_count mismatch");
  if (U > 0 && actions && actions_count != Bn * (T - 1))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": actions_count mismatch (expected Bn * (T-1))");
  if (U > 1 && !actions && T > 1)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": actions are required when B has an action axis");
  p.stage_all = 0;
  if (U > 0) {
    HmmParams q = p;
    q.stage_all = 1;
    p.stage_all = hmm_smem_bytes(q) <= kHmmMaxSmem ? 1 : 0;
  }
  if (hmm_smem_bytes(p) > kHmmMaxSmem) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": K too large");
  return B2_OK;
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_hmm_smoother(void* stream, const float* A, int64_t A_count, int32_t A_batched, const int64_t* O,
                                   int64_t M, const int32_t* obs, const float* obs_dist, int64_t obs_count,
                                   const float* prior, int64_t prior_count, const float* B, int64_t B_count,
                                   int32_t B_batched, int64_t U, const int32_t* actions, int64_t actions_count,
                                   int32_t action_mode, int64_t Bn, int64_t T, int64_t K, float* mll,
                                   float* filtered, float* predicted, float* smoothed, float* joint, float* cond) {
  const char* op = "hmm_smoother";
  if (Bn < 0 || T < 1 || K < 1 || M < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (K > kHmmMaxK) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": K above 128");
  if (M > B2_MAX_MODALITIES) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too many modalities");
  if (Bn > 0x7fffffff || T * K > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too large");
  if (action_mode != 0 && action_mode != 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": action_mode");
  if (!O) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null O");
  HmmParams p{};
  p.T = (int32_t)T;
  p.K = (int32_t)K;
  p.M = (int32_t)M;
  p.action_mode = action_mode;
  int64_t a_off = 0, o_tot = 0;
  for (int64_t m = 0; m < M; ++m) {
    if (O[m] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": num_obs must be positive");
    p.O[m] = (int32_t)O[m];
    p.A_off[m] = a_off;
    p.O_off[m] = (int32_t)o_tot;
    a_off += O[m] * K;
    o_tot += O[m];
  }
  p.A_stride = A_batched ? a_off : 0;
  p.obs_stride = (int32_t)(obs_dist ? o_tot : M);
  if (A_count != (A_batched ? Bn : 1) * a_off)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_count mismatch");
  if (obs_count != Bn * T * p.obs_stride)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": obs_count mismatch");
  if (prior_count != Bn * K) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": prior_count mismatch");
  B2_TRY(hmm_transitions(op, p, Bn, U, B_batched, B_count, actions, actions_count));
  if (Bn == 0) return B2_OK;
  if (!A || !prior || !B || !filtered || (!obs && !obs_dist))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer (filtered is required)");
  if (K <= 32) {
    bool all = false;
    const size_t wsmem = hmm_warp_smem(p, &all, true);
    const int wmax = (int)(kHmmWarpStageMax + kHmmWarpInputMax + 16);
    B2_TRY(ensure_smem_attr((const void*)hmm_smoother_warp_kernel<true>, wmax, op));
    B2_TRY(ensure_smem_attr((const void*)hmm_smoother_warp_kernel<false>, wmax, op));
    if (all)
      hmm_smoother_warp_kernel<true><<<(unsigned)Bn, 32, wsmem, (cudaStream_t)stream>>>(
          p, A, obs_dist ? nullptr : obs, obs_dist, prior, B, actions, mll, filtered, predicted, smoothed,
          T > 1 ? joint : nullptr, T > 1 ? cond : nullptr);
    else
      hmm_smoother_warp_kernel<false><<<(unsigned)Bn, 32, wsmem, (cudaStream_t)stream>>>(
          p, A, obs_dist ? nullptr : obs, obs_dist, prior, B, actions, mll, filtered, predicted, smoothed,
          T > 1 ? joint : nullptr, T > 1 ? cond : nullptr);
    return check_launch(op);
  }
  const size_t smem = hmm_smem_bytes(p);
  B2_TRY(ensure_smem_attr((const void*)hmm_smoother_kernel, (int)kHmmMaxSmem, op));
  hmm_smoother_kernel<<<(unsigned)Bn, kHmmThreads, smem, (cudaStream_t)stream>>>(
      p, A, obs_dist ? nullptr : obs, obs_dist, prior, B, actions, mll, filtered, predicted, smoothed,
      T > 1 ? joint : nullptr, T > 1 ? cond : nullptr);
  return check_launch(op);
}

extern "C" int32_t b2_hmm_smoother_from_filtered(void* stream, const float* filtered, int64_t filtered_count,
                                                 const float* B, int64_t B_count, int32_t B_batched, int64_t U,
                                                 const int32_t* actions, int64_t actions_count, int32_t action_mode,
                                                 int64_t Bn, int64_t T, int64_t K, float* smoothed, float* joint,
                                                 float* cond) {
  const char* op = "hmm_smoother_from_filtered";
  if (Bn < 0 || T < 1 || K < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (K > kHmmMaxK) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": K above 128");
  if (Bn > 0x7fffffff || T * K > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too large");
  if (action_mode != 0 && action_mode != 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": action_mode");
  HmmParams p{};
  p.T = (int32_t)T;
  p.K = (int32_t)K;
  p.action_mode = action_mode;
  if (filtered_count != Bn * T * K)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": filtered_count mismatch");
  B2_TRY(hmm_transitions(op, p, Bn, U, B_batched, B_count, actions, actions_count));
  if (Bn == 0) return B2_OK;
  if (!filtered || !B) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  if (K <= 32) {
    bool all = false;
    const size_t wsmem = hmm_warp_smem(p, &all, false);
    if (all)
      hmm_from_filtered_warp_kernel<true><<<(unsigned)Bn, 32, wsmem, (cudaStream_t)stream>>>(
          p, filtered, B, actions, smoothed, T > 1 ? joint : nullptr, T > 1 ? cond : nullptr);
    else
      hmm_from_filtered_warp_kernel<false><<<(unsigned)Bn, 32, wsmem, (cudaStream_t)stream>>>(
          p, filtered, B, actions, smoothed, T > 1 ? joint : nullptr, T > 1 ? cond : nullptr);
    return check_launch(op);
  }
  const size_t smem = hmm_smem_bytes(p);
  B2_TRY(ensure_smem_attr((const void*)hmm_from_filtered_kernel, (int)kHmmMaxSmem, op));
  hmm_from_filtered_kernel<<<(unsigned)Bn, kHmmThreads, smem, (cudaStream_t)stream>>>(
      p, filtered, B, actions, smoothed, T > 1 ? joint : nullptr, T > 1 ? cond : nullptr);
  return check_launch(op);
}
