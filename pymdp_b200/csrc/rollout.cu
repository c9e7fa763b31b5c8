// Uneven-size closed-loop rollout in one cooperative persistent launch.
//
// Thousands of agents, each with its own factor / modality / policy sizes,
// run `steps` steps of the reference's rollout loop (pymdp/envs/rollout.py:
// 468-700 with infer_and_plan, :370-466): env reset, then per step
//   phase T (policy tiles):  neg-EFE of policies [p_lo, p_hi) of one agent;
//   phase A (agents):        q_pi, action, env step, empirical prior, FPI.
// A grid-wide barrier separates the phases; inside a phase CTAs pull work
// items from an atomic queue (tiles are pre-sorted by cost, largest first).
//
// Policy tile. The policies of an agent form a tree (construct_policies,
// pymdp/control.py:152-195, enumerates action sequences with the last step
// fastest), so the prefixes of a tile's policies at depth t are a contiguous
// range; each distinct prefix is rolled out and evaluated once:
//   q_t[c]  = B[..., u_t(c)] . q_{t-1}[parent(c)]          (control.py:351-389)
//   out     = [A_m; lin_m] (R x K) * X (K x n),  X[k, c] = prod_i q_t[c][dep_i][k_i]
//   g_t[c]  = g_{t-1}[parent] + sum_m ( H(out[:O, c]) + out[O, c] )
// with lin_m[k] = sum_o A_m[o, k] (C_m[o] + log A_m[o, k]) (utility and
// -H_A . x, control.py:449-509), a register-tiled SIMT contraction whose X
// operand is generated in shared memory from the prefix marginals. The BF16
// variant stores and reads the A rows in BF16 (half the bytes of the operand
// streamed per tile); X, lin and the accumulation stay FP32.
//
// Every spin (grid barrier) is bounded; on expiry the kernel raises the abort
// word sync[2] with a code in sync[3] and every CTA returns.
#include <cuda_bf16.h>
#include <math.h>

#include <algorithm>
#include <vector>

#include "common.cuh"

namespace b2 {
namespace {

constexpr int kF = B2_RO_MAX_F;
constexpr int kM = B2_RO_MAX_M;
constexpr int kRpad = 36;  // O + 1 <= 33 contraction rows, padded to a multiple of 4
constexpr int kCols = B2_RO_MAX_COLS;
constexpr double kMinValD = 2.220446049250313e-16;  // pymdp/maths.py:15
constexpr uint32_t kBarrierSpins = 1u << 24;

enum { kSyncCount = 0, kSyncGen = 1, kSyncAbort = 2, kSyncCode = 3, kSyncQueue = 16 };
enum { kErrBarrier = 1 };

struct RoArgs {
  b2_ro_buffers buf;
  int n_agents, n_tiles, steps, num_iter, flags, tab_floats;
  unsigned grid;
  uint64_t seed;
};

// SplitMix64 output function (Steele, Lea and Flood 2014): the environment's
// counter-based generator. u01 = top 24 bits of mix(mix(mix(mix(seed) ^ agent)
// ^ step) ^ stream) / 2^24, exact in float.
__host__ __device__ __forceinline__ uint64_t sm64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ float ro_u01(uint64_t seed, int agent, int hstep, int stream) {
  uint64_t h = sm64(seed);
  h = sm64(h ^ (uint64_t)(uint32_t)agent);
  h = sm64(h ^ (uint64_t)(uint32_t)hstep);
  h = sm64(h ^ (uint64_t)(uint32_t)stream);
  return (float)(h >> 40) * (1.0f / 16777216.0f);
}

// Inverse-CDF draw with sequential float32 sums (no contraction): the first
// i with cumsum[i] > u * total.
__device__ int ro_categorical(const float* p, int n, int64_t stride, float u) {
  float total = 0.f;
  for (int i = 0; i < n; ++i) total = __fadd_rn(total, p[i * stride]);
  const float thr = __fmul_rn(u, total);
  float c = 0.f;
  for (int i = 0; i < n; ++i) {
    c = __fadd_rn(c, p[i * stride]);
    if (c > thr) return i;
  }
  return n - 1;
}

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Grid-wide barrier (all CTAs are co-resident: cooperative launch). Returns
// false when the rollout is aborted.
__device__ bool ro_grid_sync(uint32_t* sync, unsigned grid) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* vs = sync;
    int ok = 1;
    if (vs[kSyncAbort]) {
      ok = 0;
    } else {
      const uint32_t gen = vs[kSyncGen];
      __threadfence();
      const uint32_t arrived = atomicAdd(&sync[kSyncCount], 1u);
      if (arrived == grid - 1) {
        atomicExch(&sync[kSyncCount], 0u);
        __threadfence();
        atomicAdd(&sync[kSyncGen], 1u);
      } else {
        uint32_t spins = 0;
        while (vs[kSyncGen] == gen) {
          if (vs[kSyncAbort]) {
            ok = 0;
            break;
          }
          if (++spins > kBarrierSpins) {
            atomicCAS(&sync[kSyncCode], 0u, (uint32_t)kErrBarrier);
            atomicExch(&sync[kSyncAbort], 1u);
            ok = 0;
            break;
          }
          __nanosleep(256);
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Next work item of a queue (INT_MAX once the rollout is aborted).
__device__ int ro_next(uint32_t* sync, int q, int* s_item) {
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile uint32_t* vs = sync;
    *s_item = vs[kSyncAbort] ? 0x7fffffff : (int)atomicAdd(&sync[kSyncQueue + q], 1u);
  }
  __syncthreads();
  return *s_item;
}

__device__ void ro_load_agent(b2_ro_agent& dst, const b2_ro_agent* src) {
  constexpr int n = (int)(sizeof(b2_ro_agent) / 4);
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    reinterpret_cast<int*>(&dst)[i] = __ldg(reinterpret_cast<const int*>(src) + i);
  __syncthreads();
}

__device__ __forceinline__ int ro_factor_of(const b2_ro_agent& ag, int j) {
  int f = 0;
  while (f + 1 < ag.F && j >= ag.qs_off[f + 1]) ++f;
  return f;
}

// ---------------------------------------------------------------- FPI (FP64)
// y_f = softmax(x_f) per factor, one warp per factor.
__device__ void ro_softmax_factors(const b2_ro_agent& ag, const double* x, double* y) {
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (w < ag.F) {
    const int S = ag.S[w], o = ag.qs_off[w];
    double mx = -INFINITY;
    for (int s = lane; s < S; s += 32) mx = fmax(mx, x[o + s]);
    mx = warp_max_d(mx);
    double sum = 0.0;
    for (int s = lane; s < S; s += 32) sum += exp(x[o + s] - mx);
    sum = warp_sum_d(sum);
    for (int s = lane; s < S; s += 32) y[o + s] = exp(x[o + s] - mx) / sum;
  }
}

// Messages of one modality to its factors (algos.py:26-51),
//   acc[dep_i][s] += sum_{k: k_i = s} ll[k] * prod_{j != i} q[dep_j][k_j],
// without atomics: v[k] = ll[k] * prod_j q[dep_j][k_j] goes to shared memory
// (each thread walks a contiguous chunk of k with mixed-radix digits, last
// axis fastest); then for each dependency axis i, viewing v as
// (pre, S_i, post), the R threads of state s sum a strided segment, combine
// by shuffles in a fixed order and divide by q[dep_i][s]. The division is
// safe: every log-likelihood and log-prior is >= log MINVAL, so log_q spans
// less than 745 and no softmax entry underflows to zero.
template <int NT>
__device__ void ro_fpi_modality(const b2_ro_agent& ag, int m, const double* ll, const double* q, double* acc,
                                double* v) {
  const int K = ag.K[m], r = ag.rank[m];
  {
    const int chunk = (K + NT - 1) / NT;
    const int k0 = threadIdx.x * chunk;
    const int k1 = min(K, k0 + chunk);
    if (k0 < k1) {
      int dig[kF], Sd[kF], base[kF];
#pragma unroll
      for (int i = 0; i < kF; ++i) {
        if (i < r) {
          const int f = ag.dep[m][i];
          Sd[i] = ag.S[f];
          base[i] = ag.qs_off[f];
          dig[i] = (k0 / ag.dstride[m][i]) % Sd[i];
        } else {
          Sd[i] = 1;
          base[i] = 0;
          dig[i] = 0;
        }
      }
      for (int k = k0;;) {
        double w = ll[k];
#pragma unroll
        for (int i = 0; i < kF; ++i)
          if (i < r) w *= q[base[i] + dig[i]];
        v[k] = w;
        if (++k >= k1) break;
        bool carry = true;
#pragma unroll
        for (int i = kF - 1; i >= 0; --i) {
          if (carry && i < r) {
            if (++dig[i] < Sd[i])
              carry = false;
            else
              dig[i] = 0;
          }
        }
      }
    }
  }
  __syncthreads();
  for (int i = 0; i < r; ++i) {
    const int f = ag.dep[m][i], S = ag.S[f], post = ag.dstride[m][i], pre = K / (S * post);
    int R = 1;
    while (R < 32 && S * R * 2 <= NT) R <<= 1;
    const int s = threadIdx.x / R, rr = threadIdx.x & (R - 1);
    double sum = 0.0;
    if (s < S) {
      if (post >= R) {
        for (int pp = 0; pp < pre; ++pp) {
          const double* row = v + ((int64_t)pp * S + s) * post;
          for (int j = rr; j < post; j += R) sum += row[j];
        }
      } else {
        for (int pp = rr; pp < pre; pp += R) {
          const double* row = v + ((int64_t)pp * S + s) * post;
          for (int j = 0; j < post; ++j) sum += row[j];
        }
      }
    }
    for (int o = R >> 1; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (s < S && rr == 0) acc[ag.qs_off[f] + s] += sum / q[ag.qs_off[f] + s];
  }
  __syncthreads();
}

// infer_states (algos.py:88-155): Jacobi sweeps from log_q = 0 with the log
// prior in sm[0:256]; writes qs (FP32 and FP64) and the optional record.
// Shared layout: lp | lq | q | acc (256 doubles each) | v (4096 doubles).
template <int NT>
__device__ void ro_fpi(const RoArgs& a, const b2_ro_agent& ag, const int* s_obs, double* sm, int rec_t) {
  double* lp = sm;
  double* lq = sm + B2_RO_MAX_STOT;
  double* q = sm + 2 * B2_RO_MAX_STOT;
  double* acc = sm + 3 * B2_RO_MAX_STOT;
  double* v = sm + 4 * B2_RO_MAX_STOT;
  double* ll = a.buf.ll + ag.ll_off;
  const int tid = threadIdx.x;
  int koff = 0;
  for (int m = 0; m < ag.M; ++m) {
    const int K = ag.K[m];
    const float* row = a.buf.Aprime + ag.A_off[m] + (int64_t)s_obs[m] * K;
    for (int k = tid; k < K; k += NT) ll[koff + k] = log(fmax((double)row[k], kMinValD));
    koff += K;
  }
  for (int j = tid; j < ag.S_tot; j += NT) lq[j] = 0.0;
  __syncthreads();
  for (int it = 0; it < a.num_iter; ++it) {
    ro_softmax_factors(ag, lq, q);
    for (int j = tid; j < ag.S_tot; j += NT) acc[j] = 0.0;
    __syncthreads();
    koff = 0;
    for (int m = 0; m < ag.M; ++m) {
      ro_fpi_modality<NT>(ag, m, ll + koff, q, acc, v);
      koff += ag.K[m];
    }
    for (int j = tid; j < ag.S_tot; j += NT) lq[j] = acc[j] + lp[j];
    __syncthreads();
  }
  ro_softmax_factors(ag, lq, q);
  __syncthreads();
  for (int j = tid; j < ag.S_tot; j += NT) {
    a.buf.qs[ag.qs_base + j] = (float)q[j];
    a.buf.qs64[ag.qs_base + j] = q[j];
    if (a.buf.rec_qs) a.buf.rec_qs[(int64_t)rec_t * a.buf.qs_count + ag.qs_base + j] = (float)q[j];
  }
}

// obs_m ~ A_m[:, state(deps)] for every modality (envs/env.py:380-400).
__device__ void ro_sample_obs(const RoArgs& a, const b2_ro_agent& ag, int agent, int hstep, const int* s_state,
                              int* s_obs) {
  if (threadIdx.x < ag.M) {
    const int m = threadIdx.x;
    int k = 0;
    for (int i = 0; i < ag.rank[m]; ++i) k += s_state[ag.dep[m][i]] * ag.dstride[m][i];
    s_obs[m] = ro_categorical(a.buf.Aprime + ag.A_off[m] + k, ag.O[m], ag.K[m],
                              ro_u01(a.seed, agent, hstep, 64 + m));
  }
}

template <int NT>
__device__ void ro_reset_agent(const RoArgs& a, const b2_ro_agent& ag, int agent, double* sm, int* s_state,
                               int* s_obs) {
  // state ~ D, first observation ~ A (envs/env.py:333-350)
  if (threadIdx.x < ag.F) {
    const int f = threadIdx.x;
    s_state[f] = ro_categorical(a.buf.D + ag.D_off + ag.qs_off[f], ag.S[f], 1, ro_u01(a.seed, agent, 0, f));
  }
  __syncthreads();
  ro_sample_obs(a, ag, agent, 0, s_state, s_obs);
  __syncthreads();
  if (threadIdx.x < kF) a.buf.env_state[agent * kF + threadIdx.x] = threadIdx.x < ag.F ? s_state[threadIdx.x] : 0;
  if (threadIdx.x < kM) a.buf.obs[agent * kM + threadIdx.x] = threadIdx.x < ag.M ? s_obs[threadIdx.x] : 0;
  for (int j = threadIdx.x; j < ag.S_tot; j += NT) sm[j] = log(fmax((double)a.buf.D[ag.D_off + j], kMinValD));
  __syncthreads();
  ro_fpi<NT>(a, ag, s_obs, sm, 0);
}

// Index of policy p in the reduced policy space (the observed factors'
// actions only; see b2_ro_agent).
__device__ __forceinline__ int ro_reduced_policy(const b2_ro_agent& ag, int p) {
  if (ag.P_r == ag.P) return p;
  int pr = 0, W = ag.w0;
  for (int t = 0; t < ag.T; ++t) {
    const int mt = (p / W) % ag.n_multi;
    int mr = 0;
    for (int f = 0; f < ag.F; ++f) mr += ((mt / ag.ustride[f]) % ag.U[f]) * ag.ustride_r[f];
    pr = pr * ag.n_multi_r + mr;
    W /= ag.n_multi;
  }
  return pr;
}

// q_pi, action, records, env step, empirical prior and the next FPI.
template <int NT>
__device__ void ro_step_agent(const RoArgs& a, const b2_ro_agent& ag, int agent, int t, double* sm, int* s_state,
                              int* s_obs, int* s_act) {
  __shared__ float s_rv[32];
  __shared__ int s_ri[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int nw = NT / 32;
  const float* G = a.buf.G + ag.G_off;
  const float gm = ag.gamma;
  if (tid < ag.F) s_state[tid] = a.buf.env_state[agent * kF + tid];
  if (tid < ag.M) s_obs[tid] = a.buf.obs[agent * kM + tid];
  // q_pi = softmax(gamma G + log E), E uniform (control.py:349)
  float mx = -INFINITY;
  for (int p = tid; p < ag.P; p += NT) mx = fmaxf(mx, gm * G[ro_reduced_policy(ag, p)]);
  mx = warp_max(mx);
  if (lane == 0) s_rv[wid] = mx;
  __syncthreads();
  if (wid == 0) {
    float v = lane < nw ? s_rv[lane] : -INFINITY;
    v = warp_max(v);
    if (lane == 0) s_rv[0] = v;
  }
  __syncthreads();
  mx = s_rv[0];
  __syncthreads();
  float sum = 0.f;
  for (int p = tid; p < ag.P; p += NT) sum += expf(gm * G[ro_reduced_policy(ag, p)] - mx);
  sum = warp_sum(sum);
  if (lane == 0) s_rv[wid] = sum;
  __syncthreads();
  if (wid == 0) {
    float v = lane < nw ? s_rv[lane] : 0.f;
    v = warp_sum(v);
    if (lane == 0) s_rv[0] = v;
  }
  __syncthreads();
  sum = s_rv[0];
  __syncthreads();
  // deterministic sample_policy: the first maximum of q_pi (control.py:115-150)
  float best = -INFINITY;
  int bi = 0x7fffffff;
  for (int p = tid; p < ag.P; p += NT) {
    const float v = expf(gm * G[ro_reduced_policy(ag, p)] - mx) / sum;
    if (v > best || (v == best && p < bi)) {
      best = v;
      bi = p;
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
  if (lane == 0) {
    s_rv[wid] = best;
    s_ri[wid] = bi;
  }
  __syncthreads();
  if (tid == 0) {
    float bv = s_rv[0];
    int bix = s_ri[0];
    for (int w = 1; w < nw; ++w)
      if (s_rv[w] > bv || (s_rv[w] == bv && s_ri[w] < bix)) {
        bv = s_rv[w];
        bix = s_ri[w];
      }
    if (bix == 0x7fffffff) bix = 0;
    const int mu = bix / ag.w0;  // first step of the chosen policy
    for (int f = 0; f < ag.F; ++f) s_act[f] = (mu / ag.ustride[f]) % ag.U[f];
  }
  __syncthreads();
  const int64_t rec = ((int64_t)t * a.n_agents + agent);
  if (tid < kM && a.buf.rec_obs) a.buf.rec_obs[rec * kM + tid] = (int16_t)(tid < ag.M ? s_obs[tid] : -1);
  if (tid < kF && a.buf.rec_state) a.buf.rec_state[rec * kF + tid] = (int16_t)(tid < ag.F ? s_state[tid] : -1);
  if (tid < kF && a.buf.rec_action) a.buf.rec_action[rec * kF + tid] = (int16_t)(tid < ag.F ? s_act[tid] : -1);
  if (a.buf.rec_G)
    for (int p = tid; p < ag.P; p += NT)
      a.buf.rec_G[(int64_t)t * a.buf.G_count + ag.G_off + p] = G[ro_reduced_policy(ag, p)];
  // env.step: state' ~ B[:, state, action], obs' ~ A[:, state'] (envs/env.py:352-378)
  const int hstep = t + 1;
  int* s_next = s_act + kF;
  if (tid < ag.F) {
    const int f = tid, S = ag.S[f], U = ag.U[f];
    s_next[f] = ro_categorical(a.buf.B + ag.B_off[f] + ((int64_t)s_act[f] * S + s_state[f]) * S, S, 1,
                               ro_u01(a.seed, agent, hstep, 128 + f));
  }
  __syncthreads();
  ro_sample_obs(a, ag, agent, hstep, s_next, s_obs);
  __syncthreads();
  if (tid < kF) a.buf.env_state[agent * kF + tid] = tid < ag.F ? s_next[tid] : 0;
  if (tid < kM) a.buf.obs[agent * kM + tid] = tid < ag.M ? s_obs[tid] : 0;
  if (t + 1 >= a.steps) return;
  // empirical prior B[..., a] . qs (agent.py:825-851), then FPI on obs'
  const double* qs64 = a.buf.qs64 + ag.qs_base;
  for (int j = tid; j < ag.S_tot; j += NT) {
    const int f = ro_factor_of(ag, j), S = ag.S[f], U = ag.U[f], s = j - ag.qs_off[f];
    (void)U;
    const float* Bf = a.buf.B + ag.B_off[f] + (int64_t)s_act[f] * S * S + s;
    double acc = 0.0;
    for (int s2 = 0; s2 < S; ++s2) acc = fma((double)Bf[(int64_t)s2 * S], qs64[ag.qs_off[f] + s2], acc);
    sm[j] = log(fmax(acc, kMinValD));
  }
  __syncthreads();
  ro_fpi<NT>(a, ag, s_obs, sm, t + 1);
}

// ------------------------------------------------------- policy evaluation
// Prefix tables are [state j][column c] with row stride NC = round_up(width, 8).
struct TileSmem {
  float *tab0, *tab1, *sA, *sW, *sOut, *g0, *g1;
  unsigned char* sFac;
};

template <int NT, int KC>
__device__ TileSmem ro_tile_smem(unsigned char* smem, int tab_floats) {
  TileSmem s;
  s.tab0 = reinterpret_cast<float*>(smem);
  s.tab1 = s.tab0 + tab_floats;
  s.sA = s.tab1 + tab_floats;
  s.sW = s.sA + KC * kRpad;
  s.sOut = s.sW + (KC + 1) * kCols;
  s.g0 = s.sOut + kRpad * kCols;
  s.g1 = s.g0 + kCols;
  s.sFac = reinterpret_cast<unsigned char*>(s.g1 + kCols);
  return s;
}

template <int NT, int KC, bool BF16>
__device__ __forceinline__ void ro_load_a(const float* Am, const __nv_bfloat16* Ab, int R, int K, int k0,
                                          float* pa) {
  constexpr int AE = (kRpad * KC + NT - 1) / NT;
#pragma unroll
  for (int j = 0; j < AE; ++j) {
    const int idx = threadIdx.x + j * NT, row = idx / KC, kk = idx % KC;
    float v = 0.f;
    if (idx < kRpad * KC && row < R && k0 + kk < K) {
      const int64_t g = (int64_t)row * K + k0 + kk;
      v = (BF16 && row + 1 < R) ? __bfloat162float(Ab[g]) : __ldg(Am + g);
    }
    pa[j] = v;
  }
}

// out[:R, :n] = [A_m; lin_m] (R x K) * X (K x n) into sOut (row stride kCols),
// with X[k, c] = prod_i q_c[dep_i][k_i] never formed: the innermost dependency
// axis (stride 1 in K) is contracted directly against the prefix table,
//   out[o, c] = sum_po w[po, c] * sum_s A[o, po * S_in + s] * q_c[dep_last][s],
// and the outer axes enter as per-column weights w[po, c] = prod of the other
// dependencies' marginals, S_in times fewer values than X. A thread owns 4 rows x
// CB columns of one contiguous k slice per chunk; the KG slices of a unit are
// adjacent lanes and combine by shuffles. The next A chunk is loaded into
// registers while the current one is multiplied.
template <int NT, int KC, bool BF16, int CB>
__device__ void ro_contract(const RoArgs& a, const b2_ro_agent& ag, int m, const float* tab, int NC, int n,
                            const TileSmem& s) {
  constexpr int NW = NT / 32;
  constexpr int AE = (kRpad * KC + NT - 1) / NT;
  const int K = ag.K[m], R = ag.O[m] + 1, r = ag.rank[m];
  const int f_in = ag.dep[m][r - 1], S_in = ag.S[f_in];
  const float* xin = tab + ag.qs_off[f_in] * NC;
  const int RG = (R + 3) >> 2, CG = (n + CB - 1) / CB, units = RG * CG;  // units <= 9 x 8 <= NT
  int KG = 1;
  while (KG < 16 && units * KG * 2 <= NT) KG <<= 1;
  const int L = KC / KG;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int unit = tid / KG, kg = tid & (KG - 1);
  const bool active = unit < units;
  const int cg = active ? unit / RG : 0, rg = active ? unit - (unit / RG) * RG : 0;
  const int colpad = CG * CB;
  const float* Am = a.buf.Aprime + ag.A_off[m];
  const __nv_bfloat16* Ab = BF16 ? reinterpret_cast<const __nv_bfloat16*>(a.buf.Aprime_bf16) + ag.A_off[m] : nullptr;
  int qo[kF - 1], So[kF - 1], ro[kF - 1];  // outer axes: table offset, size, stride in outer-index units
#pragma unroll
  for (int i = 0; i < kF - 1; ++i) {
    const bool on = i < r - 1;
    qo[i] = on ? ag.qs_off[ag.dep[m][i]] : 0;
    So[i] = on ? ag.S[ag.dep[m][i]] : 1;
    ro[i] = on ? ag.dstride[m][i] / S_in : 1;
  }
  float acc[4][CB];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < CB; ++j) acc[i][j] = 0.f;
  float pa[AE];
  ro_load_a<NT, KC, BF16>(Am, Ab, R, K, 0, pa);
  for (int k0 = 0; k0 < K; k0 += KC) {
    const int kn = min(KC, K - k0);
#pragma unroll
    for (int j = 0; j < AE; ++j) {
      const int idx = tid + j * NT;
      if (idx < kRpad * KC) s.sA[(idx % KC) * kRpad + idx / KC] = pa[j];
    }
    const int po0 = k0 / S_in, npo = (k0 + kn - 1) / S_in - po0 + 1;
    if (r > 1) {
      for (int pr = warp; pr < npo; pr += NW) {
        const int po = po0 + pr;
        int off[kF - 1];
#pragma unroll
        for (int i = 0; i < kF - 1; ++i) off[i] = (i < r - 1) ? (qo[i] + (po / ro[i]) % So[i]) * NC : 0;
        for (int c = lane; c < colpad; c += 32) {
          float w = 0.f;
          if (c < n) {
            w = tab[off[0] + c];
#pragma unroll
            for (int i = 1; i < kF - 1; ++i)
              if (i < r - 1) w *= tab[off[i] + c];
          }
          s.sW[pr * kCols + c] = w;
        }
      }
    }
    __syncthreads();
    if (k0 + KC < K) ro_load_a<NT, KC, BF16>(Am, Ab, R, K, k0 + KC, pa);
    const int kb = kg * L, ke = min(kn, kb + L);
    if (active && kb < ke) {
      int si = (k0 + kb) % S_in, pr = (k0 + kb) / S_in - po0;
      float inner[4][CB];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < CB; ++j) inner[i][j] = 0.f;
      for (int kk = kb; kk < ke; ++kk) {
        const float4 av = *reinterpret_cast<const float4*>(s.sA + kk * kRpad + 4 * rg);
        const float* xr = xin + si * NC + CB * cg;
        float xv[CB];
#pragma unroll
        for (int j = 0; j < CB; j += 4) {
          const float4 x4 = *reinterpret_cast<const float4*>(xr + j);
          xv[j] = x4.x;
          xv[j + 1] = x4.y;
          xv[j + 2] = x4.z;
          xv[j + 3] = x4.w;
        }
#pragma unroll
        for (int j = 0; j < CB; ++j) {
          inner[0][j] = fmaf(av.x, xv[j], inner[0][j]);
          inner[1][j] = fmaf(av.y, xv[j], inner[1][j]);
          inner[2][j] = fmaf(av.z, xv[j], inner[2][j]);
          inner[3][j] = fmaf(av.w, xv[j], inner[3][j]);
        }
        const bool wrap = ++si == S_in;
        if (wrap || kk + 1 == ke) {  // this outer index ends here (or the slice does): weight and flush
          if (r > 1) {
            const float* wr = s.sW + pr * kCols + CB * cg;
#pragma unroll
            for (int j = 0; j < CB; j += 4) {
              const float4 w4 = *reinterpret_cast<const float4*>(wr + j);
              const float wv[4] = {w4.x, w4.y, w4.z, w4.w};
#pragma unroll
              for (int jj = 0; jj < 4; ++jj)
#pragma unroll
                for (int i = 0; i < 4; ++i) acc[i][j + jj] = fmaf(inner[i][j + jj], wv[jj], acc[i][j + jj]);
            }
          } else {
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
              for (int j = 0; j < CB; ++j) acc[i][j] += inner[i][j];
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < CB; ++j) inner[i][j] = 0.f;
          if (wrap) {
            si = 0;
            ++pr;
          }
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < CB; ++j)
      for (int o = KG >> 1; o > 0; o >>= 1) acc[i][j] += __shfl_xor_sync(0xffffffffu, acc[i][j], o);
  if (active && kg == 0) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = 4 * rg + i;
#pragma unroll
      for (int j = 0; j < CB; ++j) {
        const int c = CB * cg + j;
        if (row < R && c < n) s.sOut[row * kCols + c] = acc[i][j];
      }
    }
  }
  __syncthreads();
}

// The same contraction for narrow tiles (n <= NCOL <= 8 columns): warps own
// 8-row groups and stream A straight from global memory, lanes over k
// (coalesced along the rows), with no shared-memory chunks or barriers inside
// the loop; each lane forms x[k, c] = w[po, c] q_c[dep_last][s] itself.
// Partial sums combine by shuffles and shared-memory atomics into sOut.
template <int NT, bool BF16, int NCOL>
__device__ void ro_contract_narrow(const RoArgs& a, const b2_ro_agent& ag, int m, const float* tab, int NC, int n,
                                   const TileSmem& s) {
  constexpr int NW = NT / 32;
  const int K = ag.K[m], R = ag.O[m] + 1, r = ag.rank[m];
  const int f_in = ag.dep[m][r - 1], S_in = ag.S[f_in];
  const float* xin = tab + ag.qs_off[f_in] * NC;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int RG8 = (R + 7) >> 3;
  const int KS = NW >= RG8 ? NW / RG8 : 1;  // k splits per row group
  const float* Am = a.buf.Aprime + ag.A_off[m];
  const __nv_bfloat16* Ab = BF16 ? reinterpret_cast<const __nv_bfloat16*>(a.buf.Aprime_bf16) + ag.A_off[m] : nullptr;
  int qo[kF - 1], So[kF - 1], ro[kF - 1];
#pragma unroll
  for (int i = 0; i < kF - 1; ++i) {
    const bool on = i < r - 1;
    qo[i] = on ? ag.qs_off[ag.dep[m][i]] : 0;
    So[i] = on ? ag.S[ag.dep[m][i]] : 1;
    ro[i] = on ? ag.dstride[m][i] / S_in : 1;
  }
  for (int e = tid; e < kRpad * kCols; e += NT) s.sOut[e] = 0.f;
  __syncthreads();
  for (int item = warp; item < RG8 * KS; item += NW) {
    const int rg8 = item % RG8, ks = item / RG8;
    float acc[8][NCOL];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int c = 0; c < NCOL; ++c) acc[i][c] = 0.f;
    for (int k = ks * 32 + lane; k < K; k += 32 * KS) {
      const int po = k / S_in, si = k - po * S_in;
      float xv[NCOL];
#pragma unroll
      for (int c = 0; c < NCOL; ++c) xv[c] = c < n ? xin[si * NC + c] : 0.f;
      if (r > 1) {
#pragma unroll
        for (int i = 0; i < kF - 1; ++i)
          if (i < r - 1) {
            const float* row = tab + (qo[i] + (po / ro[i]) % So[i]) * NC;
#pragma unroll
            for (int c = 0; c < NCOL; ++c) xv[c] *= c < n ? row[c] : 0.f;
          }
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int row = 8 * rg8 + i;
        float av = 0.f;
        if (row < R) {
          const int64_t g = (int64_t)row * K + k;
          av = (BF16 && row + 1 < R) ? __bfloat162float(Ab[g]) : __ldg(Am + g);
        }
#pragma unroll
        for (int c = 0; c < NCOL; ++c) acc[i][c] = fmaf(av, xv[c], acc[i][c]);
      }
    }
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int c = 0; c < NCOL; ++c) {
        float v = acc[i][c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        const int row = 8 * rg8 + i;
        if (lane == 0 && row < R && c < n) atomicAdd(&s.sOut[row * kCols + c], v);
      }
  }
  __syncthreads();
}

// neg-EFE of reduced policies [p_lo, p_hi) of one agent (control.py:604-690).
template <int NT, int KC, bool BF16>
__device__ void ro_tile(const RoArgs& a, const b2_ro_agent& ag, const b2_ro_tile& tile, unsigned char* smem) {
  constexpr int NW = NT / 32;
  const TileSmem s = ro_tile_smem<NT, KC>(smem, a.tab_floats);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int St = ag.S_tot, nu = ag.n_multi_r, NC = (tile.p_hi - tile.p_lo + 7) & ~7;
  const bool ig = (a.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  for (int j = tid; j < St; j += NT) {
    s.sFac[j] = (unsigned char)ro_factor_of(ag, j);
    s.tab1[j * NC] = a.buf.qs[ag.qs_base + j];  // the root (column 0): the posterior
  }
  __syncthreads();
  float *prev = s.tab1, *cur = s.tab0, *gp = s.g1, *gc = s.g0;
  int W = ag.w0_r, prev_lo = 0;
  for (int t = 0; t < ag.T; ++t) {
    const int c_lo = tile.p_lo / W, n = (tile.p_hi - 1) / W + 1 - c_lo;
    for (int c = warp; c < n; c += NW) {
      const int pc = t == 0 ? 0 : (c_lo + c) / nu - prev_lo;
      const int mu = (c_lo + c) % nu;
      for (int j = lane; j < St; j += 32) {
        const int f = s.sFac[j];
        if (!((ag.obs_mask >> f) & 1)) continue;  // unobserved: never read
        const int S = ag.S[f], U = ag.U[f], sj = j - ag.qs_off[f];
        const int u = (mu / ag.ustride_r[f]) % U;
        const float* Bf = a.buf.B + ag.B_off[f] + (int64_t)u * S * S + sj;  // lanes: consecutive next states
        const float* pf = prev + ag.qs_off[f] * NC + pc;
        float acc = 0.f;
        for (int s2 = 0; s2 < S; ++s2) acc = fmaf(__ldg(Bf + (int64_t)s2 * S), pf[s2 * NC], acc);
        cur[j * NC + c] = acc;
      }
    }
    for (int c = tid; c < n; c += NT) gc[c] = t == 0 ? 0.f : gp[(c_lo + c) / nu - prev_lo];
    __syncthreads();
    for (int m = 0; m < ag.M; ++m) {
      if (n <= 4)
        ro_contract_narrow<NT, BF16, 4>(a, ag, m, cur, NC, n, s);
      else if (n <= 8)
        ro_contract_narrow<NT, BF16, 8>(a, ag, m, cur, NC, n, s);
      else
        ro_contract<NT, KC, BF16, 8>(a, ag, m, cur, NC, n, s);
      const int O = ag.O[m];
      for (int c = tid; c < n; c += NT) {
        float h = 0.f;
        if (ig)
          for (int o = 0; o < O; ++o) {
            const float v = s.sOut[o * kCols + c];
            h -= v * log_stable(v);
          }
        gc[c] += h + s.sOut[O * kCols + c];
      }
      __syncthreads();
    }
    float* tp = prev;
    prev = cur;
    cur = tp;
    tp = gp;
    gp = gc;
    gc = tp;
    prev_lo = c_lo;
    W /= nu > 0 ? nu : 1;
  }
  for (int c = tid; c < tile.p_hi - tile.p_lo; c += NT) a.buf.G[ag.G_off + tile.p_lo + c] = gp[c];
}

template <int NT, int KC, bool BF16>
__global__ void __launch_bounds__(NT) ro_kernel(const __grid_constant__ RoArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ b2_ro_agent s_ag;
  __shared__ int s_item;
  __shared__ int s_obs[kM], s_state[kF], s_act[2 * kF];
  double* sm = reinterpret_cast<double*>(smem);
  uint32_t* sync = a.buf.sync;
  for (;;) {
    const int i = ro_next(sync, 0, &s_item);
    if (i >= a.n_agents) break;
    ro_load_agent(s_ag, a.buf.agents + i);
    ro_reset_agent<NT>(a, s_ag, i, sm, s_state, s_obs);
  }
  if (!ro_grid_sync(sync, a.grid)) return;
  for (int t = 0; t < a.steps; ++t) {
    for (;;) {
      const int i = ro_next(sync, 1 + 2 * t, &s_item);
      if (i >= a.n_tiles) break;
      const b2_ro_tile tile = a.buf.tiles[i];
      ro_load_agent(s_ag, a.buf.agents + tile.agent);
      ro_tile<NT, KC, BF16>(a, s_ag, tile, smem);
    }
    if (!ro_grid_sync(sync, a.grid)) return;
    for (;;) {
      const int i = ro_next(sync, 2 + 2 * t, &s_item);
      if (i >= a.n_agents) break;
      ro_load_agent(s_ag, a.buf.agents + i);
      ro_step_agent<NT>(a, s_ag, i, t, sm, s_state, s_obs, s_act);
    }
    if (t + 1 < a.steps && !ro_grid_sync(sync, a.grid)) return;
  }
}

// lin_m[k] = sum_o A_m[o, k] (C_m[o] + log A_m[o, k]) in FP64 (flags select the
// terms) and the optional BF16 image of [A_m; lin_m]. One CTA per agent.
__global__ void ro_setup_kernel(const b2_ro_agent* __restrict__ agents, float* __restrict__ Ap,
                                const float* __restrict__ C, __nv_bfloat16* __restrict__ Abf, int flags) {
  const b2_ro_agent* ag = agents + blockIdx.x;
  const bool util = (flags & B2_FLAG_USE_UTILITY) != 0, ig = (flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const int M = ag->M;
  for (int m = 0; m < M; ++m) {
    const int O = ag->O[m], K = ag->K[m];
    float* A = Ap + ag->A_off[m];
    const float* Cm = C + ag->C_off[m];
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      double lin = 0.0;
      for (int o = 0; o < O; ++o) {
        const double v = A[(int64_t)o * K + k];
        if (util) lin += (double)Cm[o] * v;
        if (ig) lin += v * log(fmax(v, kMinValD));
      }
      A[(int64_t)O * K + k] = (float)lin;
    }
  }
  if (!Abf) return;
  __syncthreads();
  for (int m = 0; m < M; ++m) {
    const int64_t n = (int64_t)(ag->O[m] + 1) * ag->K[m];
    for (int64_t e = threadIdx.x; e < n; e += blockDim.x)
      Abf[ag->A_off[m] + e] = __float2bfloat16_rn(Ap[ag->A_off[m] + e]);
  }
}

// ------------------------------------------------------------- validation
const char* const kRoName = "rollout";

int32_t ro_bad(const std::string& msg) { return fail(B2_ERR_INVALID_ARGUMENT, std::string(kRoName) + ": " + msg); }
int32_t ro_unsup(const std::string& msg) { return fail(B2_ERR_UNSUPPORTED, std::string(kRoName) + ": " + msg); }

bool in_range(int64_t off, int64_t len, int64_t count) { return off >= 0 && len >= 0 && off + len <= count; }

int32_t validate_agents(const b2_ro_agent* ags, int64_t n, const b2_ro_buffers& b, bool need_runtime) {
  for (int64_t i = 0; i < n; ++i) {
    const b2_ro_agent& g = ags[i];
    const std::string at = "agent " + std::to_string(i) + ": ";
    if (g.F < 1 || g.F > kF) return ro_unsup(at + "F must be in [1, 4]");
    if (g.M < 1 || g.M > kM) return ro_unsup(at + "M must be in [1, 8]");
    if (g.T < 1) return ro_bad(at + "T must be >= 1");
    int64_t st = 0, nu = 1;
    for (int f = 0; f < g.F; ++f) {
      if (g.S[f] < 1 || g.S[f] > B2_RO_MAX_S) return ro_unsup(at + "S_f must be in [1, 64]");
      if (g.U[f] < 1 || g.U[f] > B2_RO_MAX_S) return ro_unsup(at + "U_f must be in [1, 64]");
      if (g.qs_off[f] != st) return ro_bad(at + "qs_off inconsistent with S");
      st += g.S[f];
    }
    for (int f = g.F - 1; f >= 0; --f) {
      if (g.ustride[f] != nu) return ro_bad(at + "ustride inconsistent with U");
      nu *= g.U[f];
    }
    if (st != g.S_tot) return ro_bad(at + "S_tot != sum S");
    if (st > B2_RO_MAX_STOT) return ro_unsup(at + "sum S above 256");
    if (nu != g.n_multi) return ro_bad(at + "n_multi != prod U");
    int64_t P = 1, w0 = 1;
    for (int t = 0; t < g.T; ++t) {
      if (t + 1 < g.T) w0 *= nu;
      P *= nu;
      if (P > B2_RO_MAX_P) return ro_unsup(at + "prod(U)^T above 1024");
    }
    if (P != g.P || w0 != g.w0) return ro_bad(at + "P / w0 inconsistent with U and T");
    int mask = 0;
    for (int m = 0; m < g.M && m < kM; ++m)
      for (int j = 0; j < g.rank[m] && j < kF; ++j)
        if (g.dep[m][j] >= 0 && g.dep[m][j] < g.F) mask |= 1 << g.dep[m][j];
    if (mask != g.obs_mask) return ro_bad(at + "obs_mask != union of the dependencies");
    int64_t nr = 1;
    for (int f = g.F - 1; f >= 0; --f) {
      if ((mask >> f) & 1) {
        if (g.ustride_r[f] != nr) return ro_bad(at + "ustride_r inconsistent with U and obs_mask");
        nr *= g.U[f];
      } else if (g.ustride_r[f] != 0) {
        return ro_bad(at + "ustride_r of an unobserved factor must be 0");
      }
    }
    int64_t Pr = 1, w0r = 1;
    for (int t = 0; t < g.T; ++t) {
      if (t + 1 < g.T) w0r *= nr;
      Pr *= nr;
    }
    if (nr != g.n_multi_r || Pr != g.P_r || w0r != g.w0_r) return ro_bad(at + "n_multi_r / P_r / w0_r inconsistent");
    int64_t sumK = 0;
    for (int m = 0; m < g.M; ++m) {
      if (g.O[m] < 1 || g.O[m] > B2_RO_MAX_O) return ro_unsup(at + "O_m must be in [1, 32]");
      if (g.rank[m] < 1 || g.rank[m] > g.F) return ro_bad(at + "rank_m must be in [1, F]");
      int64_t K = 1;
      for (int j = g.rank[m] - 1; j >= 0; --j) {
        const int d = g.dep[m][j];
        if (d < 0 || d >= g.F) return ro_bad(at + "dependency out of range");
        if (j > 0 && g.dep[m][j - 1] >= d) return ro_bad(at + "dependencies must be strictly ascending");
        if (g.dstride[m][j] != K) return ro_bad(at + "dstride inconsistent with S");
        K *= g.S[d];
      }
      if (K > B2_RO_MAX_K) return ro_unsup(at + "K_m above 4096");
      if (K != g.K[m]) return ro_bad(at + "K_m != prod S_deps");
      sumK += K;
      if (!in_range(g.A_off[m], (int64_t)(g.O[m] + 1) * K, b.Aprime_count)) return ro_bad(at + "A_off out of range");
      if (!in_range(g.C_off[m], g.O[m], b.C_count)) return ro_bad(at + "C_off out of range");
    }
    if (sumK != g.sum_K) return ro_bad(at + "sum_K != sum K_m");
    for (int f = 0; f < g.F; ++f)
      if (!in_range(g.B_off[f], (int64_t)g.S[f] * g.S[f] * g.U[f], b.B_count)) return ro_bad(at + "B_off out of range");
    if (!need_runtime) continue;
    if (!in_range(g.D_off, st, b.D_count)) return ro_bad(at + "D_off out of range");
    if (!in_range(g.ll_off, sumK, b.ll_count)) return ro_bad(at + "ll_off out of range");
    if (!in_range(g.qs_base, st, b.qs_count)) return ro_bad(at + "qs_base out of range");
    if (!in_range(g.G_off, P, b.G_count)) return ro_bad(at + "G_off out of range");
    if (!(g.gamma == g.gamma)) return ro_bad(at + "gamma is NaN");
  }
  return B2_OK;
}

template <int NT, int KC, bool BF16>
int32_t ro_launch(const RoArgs& args, size_t smem, cudaStream_t stream, int n_sm) {
  auto kern = ro_kernel<NT, KC, BF16>;
  B2_TRY(ensure_smem_attr((const void*)kern, (int)smem, kRoName));
  int per_sm = 0;
  B2_CUDA_TRY(kRoName, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem));
  if (per_sm < 1) return ro_unsup("launch shape does not fit on an SM");
  RoArgs a = args;
  a.grid = (unsigned)(per_sm * n_sm);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(a.grid);
  cfg.blockDim = dim3(NT);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  B2_CUDA_TRY(kRoName, cudaLaunchKernelEx(&cfg, kern, a));
  return check_launch(kRoName);
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_rollout_setup(void* stream, const b2_ro_agent* agents_host, int64_t n_agents,
                                    const b2_ro_buffers* buffers, int32_t flags) {
  if (!agents_host || !buffers || n_agents < 0) return ro_bad("null descriptors or negative count");
  if (n_agents == 0) return B2_OK;
  if (n_agents > 0x7fffffff) return ro_unsup("too many agents");
  const b2_ro_buffers& b = *buffers;
  if (!b.agents || !b.Aprime || !b.C) return ro_bad("null buffer");
  B2_TRY(validate_agents(agents_host, n_agents, b, false));
  ro_setup_kernel<<<(unsigned)n_agents, 256, 0, (cudaStream_t)stream>>>(
      b.agents, b.Aprime, b.C, reinterpret_cast<__nv_bfloat16*>(b.Aprime_bf16), flags);
  return check_launch("rollout_setup");
}

extern "C" int32_t b2_rollout(void* stream_, const b2_ro_agent* agents_host, int64_t n_agents,
                              const b2_ro_tile* tiles_host, int64_t n_tiles, const b2_ro_buffers* buffers,
                              int64_t steps, uint64_t seed, int32_t num_iter, int32_t flags,
                              const b2_ro_config* config) {
  cudaStream_t stream = (cudaStream_t)stream_;
  if (!agents_host || !tiles_host || !buffers || !config) return ro_bad("null argument");
  if (n_agents < 1 || n_tiles < 1 || steps < 1 || num_iter < 1) return ro_bad("counts must be positive");
  if (n_agents > (1 << 24) || n_tiles > (1 << 28) || steps > (1 << 20)) return ro_unsup("too many agents / tiles / steps");
  const b2_ro_buffers& b = *buffers;
  if (!b.agents || !b.tiles || !b.Aprime || !b.B || !b.C || !b.D || !b.ll || !b.qs || !b.qs64 || !b.G ||
      !b.env_state || !b.obs || !b.sync)
    return ro_bad("null buffer");
  const b2_ro_config& c = *config;
  if (c.threads != 128 && c.threads != 256 && c.threads != 512) return ro_unsup("threads must be 128, 256 or 512");
  if (c.kc != 32 && c.kc != 64) return ro_unsup("kc must be 32 or 64");
  if (c.cols < 1 || c.cols > kCols) return ro_unsup("cols must be in [1, 64]");
  if (c.precision != B2_PRECISION_FP32 && c.precision != B2_PRECISION_BF16)
    return ro_unsup("precision must be FP32 or BF16");
  if (c.precision == B2_PRECISION_BF16 && !b.Aprime_bf16) return ro_bad("BF16 precision needs Aprime_bf16");
  if (b.sync_count < 2 * steps + 32) return ro_bad("sync needs at least 2 * steps + 32 words");
  B2_TRY(validate_agents(agents_host, n_agents, b, true));
  // tiles: bounds, shape, and an exact cover of every agent's policies
  int64_t tab = 8 * B2_RO_MAX_STOT;
  std::vector<int64_t> covered(n_agents, 0);
  for (int64_t i = 0; i < n_tiles; ++i) {
    const b2_ro_tile& t = tiles_host[i];
    if (t.agent < 0 || t.agent >= n_agents) return ro_bad("tile agent out of range");
    const b2_ro_agent& g = agents_host[t.agent];
    if (t.p_lo < 0 || t.p_hi <= t.p_lo || t.p_hi > g.P_r) return ro_bad("tile policy range out of range");
    const int64_t n = t.p_hi - t.p_lo, nc = (n + 7) & ~int64_t(7);
    if (n > c.cols) return ro_bad("tile wider than cols");
    if (nc * g.S_tot > B2_RO_TAB_FLOATS) return ro_unsup("round_up(tile width, 8) x S_tot above the table");
    tab = std::max(tab, nc * g.S_tot);
    covered[t.agent] += n;
  }
  for (int64_t i = 0; i < n_agents; ++i)
    if (covered[i] != agents_host[i].P_r)
      return ro_bad("tiles do not cover agent " + std::to_string(i) + " once");
  tab = (tab + 3) & ~int64_t(3);
  const size_t tile_bytes = (size_t)(2 * tab + c.kc * kRpad + (c.kc + 1) * kCols + kRpad * kCols + 2 * kCols) * 4 +
                            B2_RO_MAX_STOT;
  const size_t fpi_bytes = (size_t)(4 * B2_RO_MAX_STOT + B2_RO_MAX_K) * sizeof(double);
  const size_t smem = std::max(tile_bytes, fpi_bytes);
  int dev = 0, n_sm = 0, coop = 0;
  B2_CUDA_TRY(kRoName, cudaGetDevice(&dev));
  B2_CUDA_TRY(kRoName, cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, dev));
  B2_CUDA_TRY(kRoName, cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return ro_unsup("device has no cooperative launch");
  B2_CUDA_TRY(kRoName, cudaMemsetAsync(b.sync, 0, (size_t)b.sync_count * 4, stream));
  RoArgs a;
  a.buf = b;
  a.n_agents = (int)n_agents;
  a.n_tiles = (int)n_tiles;
  a.steps = (int)steps;
  a.num_iter = num_iter;
  a.flags = flags;
  a.tab_floats = (int)tab;
  a.grid = 0;
  a.seed = seed;
  const bool bf = c.precision == B2_PRECISION_BF16;
#define B2_RO_CASE(NT, KC)                                                                         \
  if (c.threads == NT && c.kc == KC)                                                               \
    return bf ? ro_launch<NT, KC, true>(a, smem, stream, n_sm) : ro_launch<NT, KC, false>(a, smem, stream, n_sm);
  B2_RO_CASE(128, 32)
  B2_RO_CASE(128, 64)
  B2_RO_CASE(256, 32)
  B2_RO_CASE(256, 64)
  B2_RO_CASE(512, 32)
  B2_RO_CASE(512, 64)
#undef B2_RO_CASE
  return ro_unsup("unsupported launch shape");
}
