// Online Dirichlet learning of the observation model (pA -> A) and of the
// transition model (pB -> B), run after inference on the device-resident
// flattened buffers the FPI and EFE kernels read.
//
// Observation model (pymdp/learning.py:11-55, :57-117):
//   pA_m += lr * sum_t  o_{m,t} (x) q_{dep_0,t} (x) q_{dep_1,t} (x) ...
//   A_m   = clip(pA_m, MINVAL) / sum_o clip(pA_m, MINVAL)
// Transition model (pymdp/learning.py:119-157, :159-233) with the joints of
// Agent.infer_parameters for filtering algorithms (pymdp/agent.py:539-543,
// :567, :588-607):
//   pB_f += lr * sum_t  mask_t q_{f,t+1} (x) q_{dep_0,t} (x) ... (x) onehot(a_{f,t})
//   B_f   = clip(pB_f, MINVAL) / sum_{s'} clip(pB_f, MINVAL)
// where mask_t = all_f(a_{f,t} >= 0) (agent.py:480-483, :502-511).
//
// Both updates stream each parameter once: one thread owns one column (every
// index but the leading outcome / next-state axis) of one agent's tensor,
// accumulates that column's contribution row by row, writes pA (pB), then
// writes the normalised column. Consecutive threads own consecutive columns,
// so every row access of a warp is one contiguous run. Algorithmic traffic:
// every pA element read and every A element written (8 bytes), plus the pA
// rows that take a count (the observed row of each column; for B the taken
// action's slice).
#include "common.cuh"

namespace b2 {
namespace {

constexpr int kLearnThreads = 256;
constexpr int kLearnMinBlocks = 4;  // <= 64 registers: 32 resident warps per SM, each with a row chunk in flight
constexpr int kLearnMaxSeg = B2_MAX_MODALITIES > B2_MAX_FACTORS ? B2_MAX_MODALITIES : B2_MAX_FACTORS;

// Division by a launch-constant divisor with a precomputed multiplier
// (Granlund & Montgomery, "Division by invariant integers using
// multiplication", 1994, fig. 4.1): q = (t + ((n - t) >> s1)) >> s2 with
// t = umulhi(m, n), exact for every 32-bit n and 1 <= d < 2^31.
struct FastDiv {
  uint32_t d, m;
  uint32_t s1, s2;
};

FastDiv make_fastdiv(uint32_t d) {
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  FastDiv f;
  f.d = d;
  f.m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
  f.s1 = l < 1 ? l : 1;
  f.s2 = l > 1 ? l - 1 : 0;
  return f;
}

__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
  const uint32_t t = __umulhi(f.m, n);
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

struct LearnSeg {
  uint32_t first;  // first work index of this segment in the launch (agent-major over its columns)
  int32_t rows;    // O_m (observation model) or S_f (transition model)
  int64_t off;     // segment offset inside one agent's parameter row
  int32_t cols;    // K_m, or K_f * U_f (the action axis innermost)
  int32_t rank;    // number of dependency axes
  int32_t row_q;   // transition model: qs offset of the next-state factor f
  int32_t obs_col;  // observation model: column of m in int obs (M wide) or
                    // start of m in categorical obs (sum_m O_m wide);
                    // transition model: column f of the action array
  FastDiv cols_div, u_div;          // cols; U (transition model)
  int64_t joff;                     // transition model from given joints: offset of factor f's (T-1, S_f, K_f)
  int32_t dep_q[B2_MAX_DEP_RANK];   // qs offset of each dependency factor
  FastDiv dep_div[B2_MAX_DEP_RANK];  // its number of states
};

struct LearnParams {
  uint32_t total;        // work items of this launch (< 2^31)
  int32_t nseg, T, S_tot, obs_stride, n_act;
  int32_t lanes;         // columns per work item: 1, or 4 on the float4 path
  int64_t agent_stride;  // parameter floats per agent
  int64_t joint_stride;  // transition model from given joints: joint floats per agent
  LearnSeg seg[kLearnMaxSeg];
};

__device__ __forceinline__ int find_seg(const LearnParams& p, uint32_t g) {
  int s = 0;
  while (s + 1 < p.nseg && g >= p.seg[s + 1].first) ++s;
  return s;
}

// Column of the dependency digits of k (row-major over the dependency axes,
// the last axis fastest) -> per-axis qs offsets relative to one time slice.
__device__ __forceinline__ void split_digits(const LearnSeg& sg, uint32_t k, int* idx) {
  for (int d = sg.rank - 1; d >= 0; --d) {
    const uint32_t q = fdiv(k, sg.dep_div[d]);
    idx[d] = sg.dep_q[d] + (int)(k - q * sg.dep_div[d].d);
    k = q;
  }
}

constexpr int kRowChunk = 16;
constexpr int kFastT = 4;  // windows of 1..kFastT steps: kernels specialised on the exact length

// Updates one column (rows x stride) and writes its normalised image. Rows
// are handled in chunks of kRowChunk held in registers, so a chunk's loads are
// all in flight at once (one load per thread at a time leaves HBM idle).
// contrib(row, d) returns whether the row takes a count update and sets d to
// the summed outer-product value; the row then becomes pcol + l * d
// (learning.py:54, :155). A column of at most kRowChunk rows is normalised
// from registers; a taller one re-reads its updated counts.
template <class Contrib>
__device__ __forceinline__ void update_column(float* __restrict__ pcol, float* __restrict__ ecol, int rows,
                                              int64_t stride, float l, Contrib contrib) {
  float sum = 0.f;
  float v[kRowChunk];
  float* pr = pcol;
  for (int r0 = 0; r0 < rows; r0 += kRowChunk) {
    const int n = rows - r0;
    const float* ld = pr;
#pragma unroll
    for (int i = 0; i < kRowChunk; ++i) {
      if (i < n) v[i] = *ld;
      ld += stride;
    }
    float* st = pr;
#pragma unroll
    for (int i = 0; i < kRowChunk; ++i) {
      if (i < n) {
        float d = 0.f;
        if (contrib(r0 + i, d)) {
          v[i] = v[i] + l * d;
          *st = v[i];
        }
        sum += fmaxf(v[i], kMinVal);
      }
      st += stride;
    }
    pr += kRowChunk * stride;
  }
  // one reciprocal per column: within 1.5 ulp of the per-element quotient
  const float inv = 1.f / sum;
  float* out = ecol;
  if (rows <= kRowChunk) {
#pragma unroll
    for (int i = 0; i < kRowChunk; ++i) {
      if (i < rows) *out = fmaxf(v[i], kMinVal) * inv;
      out += stride;
    }
  } else {
    const float* in = pcol;
    for (int r = 0; r < rows; ++r, in += stride, out += stride) *out = fmaxf(*in, kMinVal) * inv;
  }
}

// Observation model. obs: int32 [Bn, T, M] indices (an index outside [0, O_m)
// adds nothing, as jax.nn.one_hot of it is all zeros) or, when obs_cat is set,
// float [Bn, T, sum O] distributions. qs: [Bn, T, S_tot].
// NT = 1..kFastT: a window of exactly NT steps, per-step weights in
// registers; NT = 0: any window length.
template <int NT>
__global__ void __launch_bounds__(kLearnThreads, kLearnMinBlocks)
learn_obs_kernel(const LearnParams p, float* __restrict__ pA, float* __restrict__ A, const int32_t* __restrict__ obs,
                 const float* __restrict__ obs_cat, const float* __restrict__ qs, const float* __restrict__ lr,
                 int lr_batched) {
  const uint32_t g = blockIdx.x * kLearnThreads + threadIdx.x;
  if (g >= p.total) return;
  const LearnSeg& sg = p.seg[find_seg(p, g)];
  const uint32_t r = g - sg.first;
  const uint32_t b = fdiv(r, sg.cols_div);
  const uint32_t k = r - b * (uint32_t)sg.cols;
  int qi[B2_MAX_DEP_RANK];
  split_digits(sg, k, qi);
  const float l = lr[lr_batched ? b : 0];
  const float* qb = qs + (int64_t)b * p.T * p.S_tot;
  const int64_t base = (int64_t)b * p.agent_stride + sg.off + k;
  const int32_t* ob = obs_cat ? nullptr : obs + (int64_t)b * p.T * p.obs_stride + sg.obs_col;
  const float* oc = obs_cat ? obs_cat + (int64_t)b * p.T * p.obs_stride + sg.obs_col : nullptr;
  // dfda[o, k] = sum_t o_t[o] * (q_0[k_0] * q_1[k_1] * ...) (maths.py:763-781)
  if constexpr (NT > 0) {
    // the dependency product of each step is the same for every row, so it is
    // formed once and the rows only select
    int ot[NT];
    float wt[NT];
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      const float* qt = qb + t * p.S_tot;
      float w = 1.f;
      for (int a = 0; a < sg.rank; ++a) w *= qt[qi[a]];
      wt[t] = w;
      ot[t] = oc ? -1 : ob[t * p.obs_stride];
    }
    auto contrib = [&](int o, float& d) -> bool {
      bool hit = false;
#pragma unroll
      for (int t = 0; t < NT; ++t) {
        if (oc) {
          d += oc[t * p.obs_stride + o] * wt[t];
          hit = true;
        } else if (ot[t] == o) {
          d += wt[t];
          hit = true;
        }
      }
      return hit;
    };
    update_column(pA + base, A + base, sg.rows, sg.cols, l, contrib);
  } else {
    auto contrib = [&](int o, float& d) -> bool {
      bool hit = false;
      for (int t = 0; t < p.T; ++t) {
        float x;
        if (oc) {
          x = oc[(int64_t)t * p.obs_stride + o];
        } else {
          if (ob[(int64_t)t * p.obs_stride] != o) continue;
          x = 1.f;
        }
        const float* qt = qb + (int64_t)t * p.S_tot;
        float w = 1.f;
        for (int a = 0; a < sg.rank; ++a) w *= qt[qi[a]];
        d += x * w;
        hit = true;
      }
      return hit;
    };
    update_column(pA + base, A + base, sg.rows, sg.cols, l, contrib);
  }
}

// Observation model, four adjacent columns per thread as float4 (every
// segment's columns, offset and last dependency axis a multiple of 4, the
// buffers 16-byte aligned). The four columns share the agent, hence the
// observed row of each step; only their last dependency digit differs. Same
// arithmetic as learn_obs_kernel: per-element work is a select, an FMA, a
// clip, an add and the scaled store, the index math is paid once per 4x rows.
constexpr int kVecRows = 16;

__device__ __forceinline__ float4 f4_fma(float l, const float4& d, const float4& v) {
  return make_float4(v.x + l * d.x, v.y + l * d.y, v.z + l * d.z, v.w + l * d.w);
}

template <int NT>
__global__ void __launch_bounds__(kLearnThreads, 2)
learn_obs_vec_kernel(const LearnParams p, float* __restrict__ pA, float* __restrict__ A,
                     const int32_t* __restrict__ obs, const float* __restrict__ obs_cat,
                     const float* __restrict__ qs, const float* __restrict__ lr, int lr_batched) {
  const uint32_t g = blockIdx.x * kLearnThreads + threadIdx.x;
  if (g >= p.total) return;
  const LearnSeg& sg = p.seg[find_seg(p, g)];
  const uint32_t r = g - sg.first;
  const uint32_t b = fdiv(r, sg.cols_div);  // cols_div divides by cols / 4 here
  const uint32_t k = 4 * (r - b * sg.cols_div.d);
  int qi[B2_MAX_DEP_RANK];
  split_digits(sg, k, qi);
  const float l = lr[lr_batched ? b : 0];
  const float* qb = qs + (int64_t)b * p.T * p.S_tot;
  const int64_t base = (int64_t)b * p.agent_stride + sg.off + k;
  const int32_t* ob = obs_cat ? nullptr : obs + (int64_t)b * p.T * p.obs_stride + sg.obs_col;
  const float* oc = obs_cat ? obs_cat + (int64_t)b * p.T * p.obs_stride + sg.obs_col : nullptr;
  const int64_t stride = sg.cols / 4;  // row stride in float4
  float4* pcol = reinterpret_cast<float4*>(pA + base);
  float4* ecol = reinterpret_cast<float4*>(A + base);
  const int rows = sg.rows;
  float4 v[kVecRows];
  // the first chunk's loads go out before the per-step weights are formed, so
  // the belief / observation loads overlap them
  {
    const float4* ld = pcol;
#pragma unroll
    for (int i = 0; i < kVecRows; ++i) {
      if (i < rows) v[i] = *ld;
      ld += stride;
    }
  }
  float4 wt[NT];
  int ot[NT];
#pragma unroll
  for (int t = 0; t < NT; ++t) {
    const float* qt = qb + t * p.S_tot;
    float w = 1.f;
    for (int a = 0; a < sg.rank - 1; ++a) w *= qt[qi[a]];
    const float* ql = qt + qi[sg.rank - 1];
    wt[t] = make_float4(w * ql[0], w * ql[1], w * ql[2], w * ql[3]);
    ot[t] = oc ? -1 : ob[t * p.obs_stride];
  }
  float4 sum = make_float4(0.f, 0.f, 0.f, 0.f);
  float4* pr = pcol;
  for (int r0 = 0; r0 < rows; r0 += kVecRows) {
    const int n = rows - r0;
    if (r0 > 0) {
      const float4* ld = pr;
#pragma unroll
      for (int i = 0; i < kVecRows; ++i) {
        if (i < n) v[i] = *ld;
        ld += stride;
      }
    }
    float4* st = pr;
#pragma unroll
    for (int i = 0; i < kVecRows; ++i) {
      if (i < n) {
        const int o = r0 + i;
        float4 d = make_float4(0.f, 0.f, 0.f, 0.f);
        bool hit = false;
#pragma unroll
        for (int t = 0; t < NT; ++t) {
          if (oc) {
            const float e = oc[t * p.obs_stride + o];
            d = make_float4(d.x + e * wt[t].x, d.y + e * wt[t].y, d.z + e * wt[t].z, d.w + e * wt[t].w);
            hit = true;
          } else if (ot[t] == o) {
            d = make_float4(d.x + wt[t].x, d.y + wt[t].y, d.z + wt[t].z, d.w + wt[t].w);
            hit = true;
          }
        }
        if (hit) {
          v[i] = f4_fma(l, d, v[i]);
          *st = v[i];
        }
        sum.x += fmaxf(v[i].x, kMinVal);
        sum.y += fmaxf(v[i].y, kMinVal);
        sum.z += fmaxf(v[i].z, kMinVal);
        sum.w += fmaxf(v[i].w, kMinVal);
      }
      st += stride;
    }
    pr += kVecRows * stride;
  }
  const float4 inv = make_float4(1.f / sum.x, 1.f / sum.y, 1.f / sum.z, 1.f / sum.w);
  auto scaled = [&](const float4& x) {
    return make_float4(fmaxf(x.x, kMinVal) * inv.x, fmaxf(x.y, kMinVal) * inv.y, fmaxf(x.z, kMinVal) * inv.z,
                       fmaxf(x.w, kMinVal) * inv.w);
  };
  float4* out = ecol;
  if (rows <= kVecRows) {
#pragma unroll
    for (int i = 0; i < kVecRows; ++i) {
      if (i < rows) *out = scaled(v[i]);
      out += stride;
    }
  } else {
    const float4* in = pcol;
    for (int i = 0; i < rows; ++i, in += stride, out += stride) *out = scaled(*in);
  }
}

// Sets *flag to 1 when some transition t of some agent has every factor's
// action >= 0 (jnp.any(valid_transition_mask), agent.py:480-500), else 0.
// One block; every iteration ends early once any thread has found one.
__global__ void __launch_bounds__(1024)
learn_any_valid_kernel(const int32_t* __restrict__ act, int64_t n_trans, int n_act, int32_t* __restrict__ flag) {
  int found = 0;
  for (int64_t base = 0; base < n_trans; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    int ok = 0;
    if (i < n_trans) {
      ok = 1;
      for (int f = 0; f < n_act; ++f) ok &= act[i * n_act + f] >= 0;
    }
    found = __syncthreads_or(ok);
    if (found) break;
  }
  if (threadIdx.x == 0) *flag = found ? 1 : 0;
}

// Transition model. qs: [Bn, T, S_tot] (the belief sequence), act: int32
// [Bn, T-1, F]. update_mask bit f: factor f takes the count update; factors
// outside it are renormalised from their unchanged pB (learning.py:201-215).
// Nothing is written when *any_valid is 0 (agent.py:588-604 skip branch).
template <int NT>
__global__ void __launch_bounds__(kLearnThreads, kLearnMinBlocks)
learn_trans_kernel(const LearnParams p, float* __restrict__ pB, float* __restrict__ B, const float* __restrict__ qs,
                   const int32_t* __restrict__ act, const float* __restrict__ lr, int lr_batched, int64_t update_mask,
                   const int32_t* __restrict__ any_valid) {
  const uint32_t g = blockIdx.x * kLearnThreads + threadIdx.x;
  if (g >= p.total || *any_valid == 0) return;
  const LearnSeg& sg = p.seg[find_seg(p, g)];
  const uint32_t r = g - sg.first;
  const uint32_t b = fdiv(r, sg.cols_div);
  const uint32_t c = r - b * (uint32_t)sg.cols;
  const uint32_t kq = fdiv(c, sg.u_div);
  const int u = (int)(c - kq * sg.u_div.d);
  int qi[B2_MAX_DEP_RANK];
  split_digits(sg, kq, qi);
  const float l = lr[lr_batched ? b : 0];
  const float* qb = qs + (int64_t)b * p.T * p.S_tot;
  const int32_t* ab = act + (int64_t)b * (p.T - 1) * p.n_act;
  const bool learn = (update_mask >> sg.obs_col) & 1;
  const int64_t base = (int64_t)b * p.agent_stride + sg.off + c;
  const int n_tr = p.T - 1;
  // transition t adds to this column when it is valid and takes action u for f
  auto live_at = [&](int t) -> bool {
    const int32_t* at = ab + (int64_t)t * p.n_act;
    bool ok = at[sg.obs_col] == u;
    for (int f = 0; f < p.n_act && ok; ++f) ok = at[f] >= 0;
    return ok;
  };
  // d[s] = sum_t q_{f,t+1}[s] * (q_dep0,t[k0] * q_dep1,t[k1] * ...) * onehot[u]
  if constexpr (NT > 0) {
    float wt[NT];
    bool lt[NT];
    bool any = false;
#pragma unroll
    for (int t = 0; t < NT; ++t) {
      wt[t] = 0.f;
      lt[t] = learn && live_at(t);
      if (lt[t]) {
        const float* qt = qb + t * p.S_tot;
        float w = 1.f;
        for (int a = 0; a < sg.rank; ++a) w *= qt[qi[a]];
        wt[t] = w;
        any = true;
      }
    }
    const float* qn = qb + p.S_tot + sg.row_q;  // q_{f,t+1}
    auto contrib = [&](int s, float& d) -> bool {
      if (!any) return false;
#pragma unroll
      for (int t = 0; t < NT; ++t)
        if (lt[t]) d += qn[t * p.S_tot + s] * wt[t];
      return true;
    };
    update_column(pB + base, B + base, sg.rows, sg.cols, l, contrib);
  } else {
    auto contrib = [&](int s, float& d) -> bool {
      if (!learn) return false;
      bool hit = false;
      for (int t = 0; t < n_tr; ++t) {
        if (!live_at(t)) continue;
        const float* qt = qb + (int64_t)t * p.S_tot;
        float w = 1.f;
        for (int a = 0; a < sg.rank; ++a) w *= qt[qi[a]];
        d += qb[(int64_t)(t + 1) * p.S_tot + sg.row_q + s] * w;
        hit = true;
      }
      return hit;
    };
    update_column(pB + base, B + base, sg.rows, sg.cols, l, contrib);
  }
}

// pB += lr * sum_t joint_t (x) onehot(a_t) with the pairwise posteriors given
// (the smoothing algorithms' form: learning.py:119-157 fed by smoothing_ovf /
// smoothing_exact, agent.py:530-567): joint [Bn][per factor (T-1, S_f, K_f)],
// a transition counting only when it is valid (every action >= 0, the
// reference's _apply_transition_mask) and takes action u for f; then
// B = normalised pB as in learn_trans_kernel.
__global__ void __launch_bounds__(kLearnThreads, kLearnMinBlocks)
learn_trans_joint_kernel(const LearnParams p, float* __restrict__ pB, float* __restrict__ B,
                         const float* __restrict__ joint, const int32_t* __restrict__ act,
                         const float* __restrict__ lr, int lr_batched, int64_t update_mask,
                         const int32_t* __restrict__ any_valid) {
  const uint32_t g = blockIdx.x * kLearnThreads + threadIdx.x;
  if (g >= p.total || *any_valid == 0) return;
  const LearnSeg& sg = p.seg[find_seg(p, g)];
  const uint32_t r = g - sg.first;
  const uint32_t b = fdiv(r, sg.cols_div);
  const uint32_t c = r - b * (uint32_t)sg.cols;
  const uint32_t kq = fdiv(c, sg.u_div);
  const int u = (int)(c - kq * sg.u_div.d);
  const int K = sg.cols / (int)sg.u_div.d;
  const float l = lr[lr_batched ? b : 0];
  const int32_t* ab = act + (int64_t)b * (p.T - 1) * p.n_act;
  const bool learn = (update_mask >> sg.obs_col) & 1;
  const int64_t base = (int64_t)b * p.agent_stride + sg.off + c;
  const float* jb = joint + (int64_t)b * p.joint_stride + sg.joff + kq;
  const int n_tr = p.T - 1;
  auto contrib = [&](int s, float& d) -> bool {
    if (!learn) return false;
    bool hit = false;
    for (int t = 0; t < n_tr; ++t) {
      const int32_t* at = ab + (int64_t)t * p.n_act;
      bool ok = at[sg.obs_col] == u;
      for (int f = 0; f < p.n_act && ok; ++f) ok = at[f] >= 0;
      if (!ok) continue;
      d += __ldg(jb + ((int64_t)t * sg.rows + s) * K);
      hit = true;
    }
    return hit;
  };
  update_column(pB + base, B + base, sg.rows, sg.cols, l, contrib);
}

// Agents per launch so that every work index of the launch fits 31 bits;
// 0 when a single agent's columns do not.
int64_t agents_per_launch(const LearnParams& p) {
  int64_t items = 0;
  for (int i = 0; i < p.nseg; ++i) items += p.seg[i].cols / p.lanes;
  return items > 0x7fffffff ? 0 : 0x7fffffff / items;
}

// Sets the work ranges of a launch over nb agents; returns its block count.
unsigned plan_launch(LearnParams& p, int64_t nb) {
  uint32_t first = 0;
  for (int i = 0; i < p.nseg; ++i) {
    p.seg[i].first = first;
    first += (uint32_t)(nb * (p.seg[i].cols / p.lanes));
  }
  p.total = first;
  return (first + kLearnThreads - 1) / kLearnThreads;
}

// Shared validation of the dependency lists; fills seg[i].rank/dep_q/dep_div and
// returns the product of the dependency sizes in *K.
int32_t fill_deps(const char* op, LearnSeg& sg, int64_t i, int64_t F, const int64_t* S, const int64_t* qs_offsets,
                  const int64_t* dep_flat, int64_t dep_flat_len, const int64_t* dep_offsets, int64_t* K) {
  const int64_t d0 = dep_offsets[i], d1 = dep_offsets[i + 1];
  if (d0 < 0 || d1 < d0 || d1 > dep_flat_len)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": dependency offsets out of range");
  if (d1 - d0 > B2_MAX_DEP_RANK) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": dependency rank above 8");
  sg.rank = (int32_t)(d1 - d0);
  int64_t k = 1;
  for (int64_t j = d0; j < d1; ++j) {
    const int64_t f = dep_flat[j];
    if (f < 0 || f >= F) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": dependency factor out of range");
    sg.dep_q[j - d0] = (int32_t)qs_offsets[f];
    sg.dep_div[j - d0] = make_fastdiv((uint32_t)S[f]);
    k *= S[f];
    if (k > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": tensor too large");
  }
  *K = k;
  return B2_OK;
}

int32_t check_states(const char* op, int64_t F, const int64_t* S, const int64_t* qs_offsets, int64_t* S_tot) {
  if (qs_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": qs_offsets[0] must be 0");
  for (int64_t f = 0; f < F; ++f) {
    if (S[f] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": num_states must be positive");
    if (qs_offsets[f + 1] - qs_offsets[f] != S[f])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": qs_offsets inconsistent with S");
  }
  *S_tot = qs_offsets[F];
  if (*S_tot > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too many states");
  return B2_OK;
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_update_obs_likelihood_dirichlet(
    void* stream, float* pA, float* A, int64_t A_count, const int32_t* obs, const float* obs_cat, int64_t obs_count,
    const float* qs, int64_t qs_count, const float* lr, int32_t lr_batched, int64_t Bn, int64_t T, int64_t F,
    int64_t M, const int64_t* S, const int64_t* O, const int64_t* qs_offsets, const int64_t* A_offsets,
    const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets, int64_t modality_mask) {
  const char* op = "update_obs_likelihood_dirichlet";
  if (Bn < 0 || T < 1 || F < 1 || M < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (F > B2_MAX_FACTORS || M > B2_MAX_MODALITIES)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too many factors or modalities");
  if (!S || !O || !qs_offsets || !A_offsets || !A_dep_offsets || (A_dep_flat_len > 0 && !A_dep_flat))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute");
  int64_t S_tot = 0;
  B2_TRY(check_states(op, F, S, qs_offsets, &S_tot));
  LearnParams p{};
  p.lanes = 1;
  p.T = (int32_t)T;
  p.S_tot = (int32_t)S_tot;
  p.agent_stride = A_offsets[M];
  int64_t O_tot = 0;
  if (A_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets[0] must be 0");
  for (int64_t m = 0; m < M; ++m) {
    if (O[m] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": num_obs must be positive");
    LearnSeg sg{};
    int64_t K = 0;
    B2_TRY(fill_deps(op, sg, m, F, S, qs_offsets, A_dep_flat, A_dep_flat_len, A_dep_offsets, &K));
    if (A_offsets[m + 1] - A_offsets[m] != O[m] * K)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets inconsistent with O and S");
    if ((modality_mask >> m) & 1) {
      sg.rows = (int32_t)O[m];
      sg.cols = (int32_t)K;
      sg.cols_div = make_fastdiv((uint32_t)K);
      sg.u_div = make_fastdiv(1);
      sg.off = A_offsets[m];
      sg.obs_col = (int32_t)(obs_cat ? O_tot : m);
      p.seg[p.nseg++] = sg;
    }
    O_tot += O[m];
  }
  p.obs_stride = (int32_t)(obs_cat ? O_tot : M);
  if (A_count != Bn * p.agent_stride) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_count mismatch");
  if (qs_count != Bn * T * S_tot) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": qs_count mismatch");
  if (obs_count != Bn * T * p.obs_stride) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": obs_count mismatch");
  if (Bn == 0 || p.nseg == 0) return B2_OK;
  if (!pA || !A || !qs || !lr || (!obs && !obs_cat))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  // float4 path: every column quad inside one agent's segment and aligned
  bool vec = T <= kFastT && p.agent_stride % 4 == 0 && ((uintptr_t)pA % 16) == 0 && ((uintptr_t)A % 16) == 0;
  for (int i = 0; i < p.nseg && vec; ++i) {
    const LearnSeg& sg = p.seg[i];
    vec = sg.rank >= 1 && sg.cols % 4 == 0 && sg.off % 4 == 0 && sg.dep_div[sg.rank - 1].d % 4 == 0;
  }
  if (vec) {
    p.lanes = 4;
    for (int i = 0; i < p.nseg; ++i) p.seg[i].cols_div = make_fastdiv((uint32_t)(p.seg[i].cols / 4));
  }
  const int64_t per = agents_per_launch(p);
  if (per == 0) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": tensor too large");
  cudaStream_t st = (cudaStream_t)stream;
  for (int64_t b0 = 0; b0 < Bn; b0 += per) {
    const int64_t nb = Bn - b0 < per ? Bn - b0 : per;
    const unsigned blocks = plan_launch(p, nb);
    float* pa = pA + b0 * p.agent_stride;
    float* a = A + b0 * p.agent_stride;
    const int32_t* ob = obs_cat ? nullptr : obs + b0 * T * p.obs_stride;
    const float* oc = obs_cat ? obs_cat + b0 * T * p.obs_stride : nullptr;
    const float* q = qs + b0 * T * S_tot;
    const float* l = lr + (lr_batched ? b0 : 0);
    if (vec) {
      switch (T) {
        case 1: learn_obs_vec_kernel<1><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
        case 2: learn_obs_vec_kernel<2><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
        case 3: learn_obs_vec_kernel<3><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
        default: learn_obs_vec_kernel<4><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
      }
      B2_TRY(check_launch(op));
      continue;
    }
    switch (T) {
      case 1: learn_obs_kernel<1><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
      case 2: learn_obs_kernel<2><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
      case 3: learn_obs_kernel<3><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
      case 4: learn_obs_kernel<4><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
      default: learn_obs_kernel<0><<<blocks, kLearnThreads, 0, st>>>(p, pa, a, ob, oc, q, l, lr_batched); break;
    }
    B2_TRY(check_launch(op));
  }
  return B2_OK;
}

extern "C" int32_t b2_update_state_transition_dirichlet(
    void* stream, float* pB, float* B, int64_t B_count, const float* qs, int64_t qs_count, const int32_t* actions,
    int64_t actions_count, const float* lr, int32_t lr_batched, int32_t* workspace, int64_t Bn, int64_t T, int64_t F,
    const int64_t* S, const int64_t* U, const int64_t* qs_offsets, const int64_t* B_offsets,
    const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int64_t factor_mask) {
  const char* op = "update_state_transition_dirichlet";
  if (Bn < 0 || T < 1 || F < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (F > B2_MAX_FACTORS) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too many factors");
  if (!S || !U || !qs_offsets || !B_offsets || !B_dep_offsets || (B_dep_flat_len > 0 && !B_dep_flat))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute");
  int64_t S_tot = 0;
  B2_TRY(check_states(op, F, S, qs_offsets, &S_tot));
  LearnParams p{};
  p.lanes = 1;
  p.T = (int32_t)T;
  p.S_tot = (int32_t)S_tot;
  p.n_act = (int32_t)F;
  p.agent_stride = B_offsets[F];
  if (B_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_offsets[0] must be 0");
  for (int64_t f = 0; f < F; ++f) {
    if (U[f] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": num_controls must be positive");
    LearnSeg sg{};
    int64_t K = 0;
    B2_TRY(fill_deps(op, sg, f, F, S, qs_offsets, B_dep_flat, B_dep_flat_len, B_dep_offsets, &K));
    if (B_offsets[f + 1] - B_offsets[f] != S[f] * K * U[f])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_offsets inconsistent with S, U and dependencies");
    if (K * U[f] > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": tensor too large");
    sg.rows = (int32_t)S[f];
    sg.cols = (int32_t)(K * U[f]);
    sg.cols_div = make_fastdiv((uint32_t)sg.cols);
    sg.u_div = make_fastdiv((uint32_t)U[f]);
    sg.off = B_offsets[f];
    sg.row_q = (int32_t)qs_offsets[f];
    sg.obs_col = (int32_t)f;
    p.seg[p.nseg++] = sg;
  }
  if (B_count != Bn * p.agent_stride) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_count mismatch");
  if (qs_count != Bn * T * S_tot) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": qs_count mismatch");
  if (actions_count != Bn * (T - 1) * F)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": actions_count mismatch (expected Bn * (T-1) * F)");
  // no transition in the window: the reference keeps pB and B (agent.py:495-500, :603-604)
  if (T < 2 || Bn == 0) return B2_OK;
  if (!pB || !B || !qs || !lr || !actions || !workspace)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  const int64_t per = agents_per_launch(p);
  if (per == 0) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": tensor too large");
  cudaStream_t st = (cudaStream_t)stream;
  // the any-valid flag is over the whole batch, before any agent is updated
  learn_any_valid_kernel<<<1, 1024, 0, st>>>(actions, Bn * (T - 1), (int)F, workspace);
  B2_TRY(check_launch(op));
  for (int64_t b0 = 0; b0 < Bn; b0 += per) {
    const int64_t nb = Bn - b0 < per ? Bn - b0 : per;
    const unsigned blocks = plan_launch(p, nb);
    float* pb = pB + b0 * p.agent_stride;
    float* bb = B + b0 * p.agent_stride;
    const float* q = qs + b0 * T * S_tot;
    const int32_t* a = actions + b0 * (T - 1) * F;
    const float* l = lr + (lr_batched ? b0 : 0);
#define B2_LEARN_TRANS(NT) \
  learn_trans_kernel<NT><<<blocks, kLearnThreads, 0, st>>>(p, pb, bb, q, a, l, lr_batched, factor_mask, workspace)
    switch (T - 1) {
      case 1: B2_LEARN_TRANS(1); break;
      case 2: B2_LEARN_TRANS(2); break;
      case 3: B2_LEARN_TRANS(3); break;
      case 4: B2_LEARN_TRANS(4); break;
      default: B2_LEARN_TRANS(0); break;
    }
#undef B2_LEARN_TRANS
    B2_TRY(check_launch(op));
  }
  return B2_OK;
}

extern "C" int32_t b2_update_state_transition_from_joint(
    void* stream, float* pB, float* B, int64_t B_count, const float* joint, int64_t joint_count,
    const int32_t* actions, int64_t actions_count, const float* lr, int32_t lr_batched, int32_t* workspace, int64_t Bn,
    int64_t T, int64_t F, const int64_t* S, const int64_t* U, const int64_t* qs_offsets, const int64_t* B_offsets,
    const int64_t* B_dep_flat, int64_t B_dep_flat_len, const int64_t* B_dep_offsets, int64_t factor_mask) {
  const char* op = "update_state_transition_from_joint";
  if (Bn < 0 || T < 1 || F < 1) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": invalid sizes");
  if (F > B2_MAX_FACTORS) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": too many factors");
  if (!S || !U || !qs_offsets || !B_offsets || !B_dep_offsets || (B_dep_flat_len > 0 && !B_dep_flat))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute");
  int64_t S_tot = 0;
  B2_TRY(check_states(op, F, S, qs_offsets, &S_tot));
  LearnParams p{};
  p.lanes = 1;
  p.T = (int32_t)T;
  p.S_tot = (int32_t)S_tot;
  p.n_act = (int32_t)F;
  p.agent_stride = B_offsets[F];
  if (B_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_offsets[0] must be 0");
  int64_t joff = 0;
  for (int64_t f = 0; f < F; ++f) {
    if (U[f] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": num_controls must be positive");
    LearnSeg sg{};
    int64_t K = 0;
    B2_TRY(fill_deps(op, sg, f, F, S, qs_offsets, B_dep_flat, B_dep_flat_len, B_dep_offsets, &K));
    if (B_offsets[f + 1] - B_offsets[f] != S[f] * K * U[f])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_offsets inconsistent with S, U and dependencies");
    if (K * U[f] > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": tensor too large");
    sg.rows = (int32_t)S[f];
    sg.cols = (int32_t)(K * U[f]);
    sg.cols_div = make_fastdiv((uint32_t)sg.cols);
    sg.u_div = make_fastdiv((uint32_t)U[f]);
    sg.off = B_offsets[f];
    sg.row_q = (int32_t)qs_offsets[f];
    sg.obs_col = (int32_t)f;
    sg.joff = joff;
    joff += (T - 1) * S[f] * K;
    p.seg[p.nseg++] = sg;
  }
  p.joint_stride = joff;
  if (B_count != Bn * p.agent_stride) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": B_count mismatch");
  if (joint_count != Bn * joff)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": joint_count mismatch (expected Bn * sum_f (T-1) S_f K_f)");
  if (actions_count != Bn * (T - 1) * F)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": actions_count mismatch (expected Bn * (T-1) * F)");
  if (T < 2 || Bn == 0) return B2_OK;
  if (!pB || !B || !joint || !lr || !actions || !workspace)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  const int64_t per = agents_per_launch(p);
  if (per == 0) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": tensor too large");
  cudaStream_t st = (cudaStream_t)stream;
  learn_any_valid_kernel<<<1, 1024, 0, st>>>(actions, Bn * (T - 1), (int)F, workspace);
  B2_TRY(check_launch(op));
  for (int64_t b0 = 0; b0 < Bn; b0 += per) {
    const int64_t nb = Bn - b0 < per ? Bn - b0 : per;
    const unsigned blocks = plan_launch(p, nb);
    learn_trans_joint_kernel<<<blocks, kLearnThreads, 0, st>>>(
        p, pB + b0 * p.agent_stride, B + b0 * p.agent_stride, joint + b0 * joff, actions + b0 * (T - 1) * F,
        lr + (lr_batched ? b0 : 0), lr_batched, factor_mask, workspace);
    B2_TRY(check_launch(op));
  }
  return B2_OK;
}
