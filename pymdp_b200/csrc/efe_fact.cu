// Factored neg-EFE over the policy tree (B2_FLAG_FACTORED).
//
// With factor-local transitions (B_dependencies[f] == [f]) and the full
// product policy set of construct_policies, the predicted marginal of factor
// f after step t depends only on f's own actions u_{f,0..t}: there are
// H_f(t) = U_f^(t+1) distinct ones, its "histories" (efe_tree_rollout_kernel
// forms the joint prefixes instead: prod_f U_f^(t+1) of them). The expected
// observation of a policy prefix c at depth t is then
//   qo[c, n] = sum_{s_0..s_r-1} A[n, s] prod_i q_{f_i}^{h_{f_i}(c)}[s_i]
// (compute_expected_obs, pymdp/control.py:420-447), a multilinear form that
// is contracted one factor at a time over the distinct histories:
//   V1[h0][n][s1, s2]  = sum_{s0} q_{f0}^{h0}[s0]  A[n, s]          (level 1)
//   V2[h0,h1][n][s2]   = sum_{s1} q_{f1}^{h1}[s1]  V1[h0][n][s1, s2] (level 2)
//   qo[h0,h1,h2][n]    = sum_{s2} q_{f2}^{h2}[s2]  V2[h0,h1][n][s2] (level 3)
// The step's info gain + utility of the group's modalities (compute_info_gain
// + compute_expected_utility, pymdp/control.py:449-509) is H(qo) over the
// observation rows plus the linear row lin_t[k] = sum_o A[o,k] (log clip
// A[o,k] + C_t[o]) contracted the same way (the same linear-term collapse as
// efe_tc_pack_kernel). The per-group, per-depth tables T_g,t[h0,h1,h2] then
// sum into G[p] = sum_t sum_g T_g,t[histories of p at t].
//
// Same arithmetic as the per-policy evaluation, in another summation order:
// at the EFE benchmark model (S = [32,16,8], U = [4,4,1], T = 3, one group of
// 52 observation rows) depth 2 costs 1.7 M + 3.5 M multiply-adds per agent
// instead of 4096 x 55 x 4096 = 923 M, and the launch is bound by reading A
// once per agent. FP32 products and short FP32 dot products (at most the
// largest factor's size), entropies in FP32, G in FP64.
//
// Kernels: efe_fact_hist_kernel (history marginals), efe_fact_l1_kernel (one
// pass over A: level 1 for the observation rows, and the linear row of each
// depth through its information-gain and utility parts), efe_fact_tail_kernel
// (levels 2 and 3 and the entropy epilogue into the tables),
// efe_fact_combine_kernel (G per policy).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "efe.cuh"

namespace b2 {
namespace {

constexpr int kFactMaxRank = 3;
constexpr int kFactMaxT = 8;
constexpr int kFactMaxG = 8;
constexpr int kFactMaxS = 64;   // largest factor size on the factored path
constexpr int kFactCombo = 8;   // (depth, history) combinations per level-1 pass over A
constexpr int kFactTailThreads = 256;
constexpr int kTailTpi = 2;  // threads per last-level work item (they split its observation rows)
constexpr int kFactH1Tile = 8;  // level-2 histories per tail CTA (at least; 16 where shared memory allows)
constexpr int kFactTailSmem = 96 * 1024;  // tail shared memory: level-2 blocks of one h1 tile

struct FactGroup {
  int32_t rank;                         // 1..3
  int32_t f[kFactMaxRank];              // factors in contraction order (f[0] first)
  int32_t S[kFactMaxRank];              // their sizes (1 past rank)
  int32_t stA[kFactMaxRank];            // stride of the factor's axis in the modalities' A (state axes only)
  int32_t K, R;                         // prod of sizes; K / S[0] (one V1 row: s1 outer, s2 inner)
  int32_t vec4;                         // level-1 axis contiguous and every row start 16-byte aligned
  int32_t n_obs, m_begin, m_end;        // observation rows; modalities [m_begin, m_end) of mod_order
  int32_t n_w;                          // parameter-information-gain rows (wA, one per observation row) or 0;
                                        // V1 rows: [n_obs A rows][n_w wA rows][1 linear row]
  int32_t H[kFactMaxRank][kFactMaxT];   // histories of f[i] at depth t (1 past rank)
  int64_t v1_off[kFactMaxT];            // per-agent float offset of V1 at depth t: [H0][n_obs + n_w + 1][R]
  int64_t tab_off[kFactMaxT];           // per-agent double offset of the table at depth t: [H0][H1][H2]
};

struct FactParams {
  int32_t G, T, F, nu;
  int32_t ustride[kEfeMaxF];                // joint action a = sum_f u_f * ustride[f] (construct_policies order)
  int64_t qh_off[kEfeMaxF][kFactMaxT];      // per-agent float offset of factor f's histories at depth t
  int64_t qh_stride, v1_stride, tab_stride; // per-agent floats / floats / doubles
  int32_t hterm;                            // 1: per-factor history terms (pB information gain, inductive value)
  int64_t ht_off[kEfeMaxF][kFactMaxT];      // per-agent double offset of factor f's history terms at depth t
  int64_t ht_stride;                        // doubles per agent
  int32_t max_R, max_tiles;
  int32_t smax;                             // largest size among the factors the tail contracts
  int32_t tail_smem;                        // dynamic shared memory of the tail kernel (bytes)
  int32_t h1_tile;                          // level-2 histories per tail CTA: 8 or 16
  int32_t hist_smem;                        // dynamic shared memory of the history kernel (bytes; 0: global path)
  int32_t bt_off[kEfeMaxF], bt_plane[kEfeMaxF];  // staged B_f^T: plane u at bt_off + u * bt_plane, [k][s]
  int32_t bt_row[kEfeMaxF];                 // ... with row stride bt_row (odd)
  int32_t qi_sm, qh_sm, qh_words;           // staged qs_init and histories (float offsets); histories per agent
  int8_t mod_order[B2_MAX_MODALITIES];
  FactGroup grp[kFactMaxG];
};

__host__ __device__ __forceinline__ int ipow(int b, int e) {
  int r = 1;
  for (int i = 0; i < e; ++i) r *= b;
  return r;
}

// History marginals: Qh[f][t][h] = B_f[:, :, u] . Qh[f][t-1][h / U_f] with
// u = h % U_f (qs_init at t = 0): compute_expected_state (pymdp/control.py:
// 351-389) for a factor-local B, once per distinct action history. With the
// flag-gated terms, also the per-history step terms Ht[f][t][h]: minus the
// pB information gain q_next . (wB_f[..., u] . q_prev) (calc_negative_pB_info_gain,
// pymdp/control.py:555-602) plus the inductive value wI_f . q_next
// (calc_inductive_value_t, pymdp/control.py:1021-1061).
__global__ void __launch_bounds__(256) efe_fact_hist_kernel(const __grid_constant__ EfeParams p,
                                                            const __grid_constant__ FactParams fp,
                                                            const float* __restrict__ qs_init,
                                                            const float* __restrict__ B, float* __restrict__ Qh,
                                                            const float* __restrict__ wB,
                                                            const float* __restrict__ wI, double* __restrict__ Ht) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  extern __shared__ float hsm[];
  const int64_t b = blockIdx.x;
  float* Qb = Qh + b * fp.qh_stride;
  const float* Bb = B + b * p.B_stride;
  const float* qi = qs_init + b * p.S_tot;
  const bool staged = fp.hist_smem > 0;  // uniform over the grid
  if (staged) {
    // B_f transposed to [u][k][s] (planes padded so that the half-warps of
    // small factors fall on different banks) and qs_init, in shared memory
    for (int f = 0; f < p.F; ++f) {
      // one thread per (s, k): its U contiguous actions go to the U planes
      const int S = p.S[f], U = p.U[f];
      const float* src = Bb + p.fac[f].B_off;
      float* dst = hsm + fp.bt_off[f];
      const int plane = fp.bt_plane[f];
#pragma unroll 2
      for (int pr = threadIdx.x; pr < S * S; pr += blockDim.x) {
        const int s = pr / S, k = pr - s * S;
        const float* sp = src + (int64_t)pr * U;
        float* dp = dst + k * fp.bt_row[f] + s;
        if (U == 4 && (reinterpret_cast<uintptr_t>(sp) & 15) == 0) {
          const float4 v = __ldg(reinterpret_cast<const float4*>(sp));
          dp[0] = v.x;
          dp[plane] = v.y;
          dp[2 * plane] = v.z;
          dp[3 * plane] = v.w;
        } else {
          for (int u = 0; u < U; ++u) dp[u * plane] = __ldg(sp + u);
        }
      }
    }
    for (int i = threadIdx.x; i < p.S_tot; i += blockDim.x) hsm[fp.qi_sm + i] = __ldg(qi + i);
    __syncthreads();
  }
  float* Qw = staged ? hsm + fp.qh_sm : Qb;  // where this CTA writes (and reads back) the histories
  const float* q0 = staged ? hsm + fp.qi_sm : qi;
  for (int t = 0; t < p.T; ++t) {
    for (int f = 0; f < p.F; ++f) {
      const int S = p.S[f], U = p.U[f];
      const int H = ipow(U, t + 1);
      float* out = Qw + fp.qh_off[f][t];
      if (staged) {
        const float* qprev = t == 0 ? q0 + p.qs_off[f] : Qw + fp.qh_off[f][t - 1];
        const int br = fp.bt_row[f], plane = fp.bt_plane[f];
        const float* Bf = hsm + fp.bt_off[f];
        for (int e = threadIdx.x; e < H * S; e += blockDim.x) {
          const int h = e / S, s = e - h * S;
          const int u = h % U;
          const float* q = t == 0 ? qprev : qprev + (h / U) * S;
          const float* Bt = Bf + u * plane + s;
          float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
          int k = 0;
          for (; k + 4 <= S; k += 4) {
            a0 = fmaf(Bt[k * br], q[k], a0);
            a1 = fmaf(Bt[(k + 1) * br], q[k + 1], a1);
            a2 = fmaf(Bt[(k + 2) * br], q[k + 2], a2);
            a3 = fmaf(Bt[(k + 3) * br], q[k + 3], a3);
          }
          for (; k < S; ++k) a0 = fmaf(Bt[k * br], q[k], a0);
          out[e] = (a0 + a1) + (a2 + a3);
        }
      } else {
        const EfeFactor& fb = p.fac[f];
        for (int e = threadIdx.x; e < H * S; e += blockDim.x) {
          const int h = e / S, s = e - h * S;
          const int u = h % U;
          const float* q = t == 0 ? qi + p.qs_off[f] : Qb + fp.qh_off[f][t - 1] + (int64_t)(h / U) * S;
          const float* Bs = Bb + fb.B_off + (int64_t)s * S * U + u;
          float acc = 0.f;
          for (int k = 0; k < S; ++k) acc = fmaf(__ldg(Bs + (int64_t)k * U), q[k], acc);
          out[e] = acc;
        }
      }
    }
    __syncthreads();
    if (fp.hterm) {
      // one thread per history of each factor at this depth
      for (int f = 0; f < p.F; ++f) {
        const int S = p.S[f], U = p.U[f];
        const int H = ipow(U, t + 1);
        for (int h = threadIdx.x; h < H; h += blockDim.x) {
          const int u = h % U;
          const float* qn = Qw + fp.qh_off[f][t] + (int64_t)h * S;
          const float* qp = t == 0 ? q0 + p.qs_off[f] : Qw + fp.qh_off[f][t - 1] + (int64_t)(h / U) * S;
          double v = 0.0;
          if (wB) {
            const float* Ws = wB + b * p.B_stride + p.fac[f].B_off + u;
            for (int s = 0; s < S; ++s) {
              float fd = 0.f;
              for (int k = 0; k < S; ++k) fd = fmaf(__ldg(Ws + ((int64_t)s * S + k) * U), qp[k], fd);
              v -= (double)qn[s] * fd;
            }
          }
          if (wI)
            for (int s = 0; s < S; ++s) v += (double)__ldg(wI + b * p.S_tot + p.qs_off[f] + s) * qn[s];
          Ht[b * fp.ht_stride + fp.ht_off[f][t] + h] = v;
        }
      }
    }
  }
  if (staged)  // the last depth's barrier above orders every history write before this copy
    for (int i = threadIdx.x; i < fp.qh_words; i += blockDim.x) Qb[i] = hsm[fp.qh_sm + i];
}

// Level 1: one thread per (group, rest index r = (s1, s2)). For each
// observation row it streams the S0 entries A[row, s0, s1, s2] once and, for
// up to KC <= kFactCombo (depth, h0) combinations at a time (their marginals staged
// in shared memory), writes V1[h0][row][r] = sum_s0 q_{f0}^{h0}[s0] A and
// accumulates the depth's linear row sum_row [sum_s0 q xlogx(A)] + C_t[o] V1
// (information gain, utility).
// KC <= 4: registers capped for eight resident CTAs per SM (the 256-agent
// benchmark launch then fits in one wave)
template <int KC, int NJ>
__global__ void __launch_bounds__(128, KC <= 4 ? 8 : 4) efe_fact_l1_kernel(const __grid_constant__ EfeParams p,
                                                          const __grid_constant__ FactParams fp,
                                                          const float* __restrict__ A, const float* __restrict__ C,
                                                          const float* __restrict__ Qh, float* __restrict__ V1,
                                                          const float* __restrict__ wA) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  __shared__ __align__(16) float qsm[KC * kFactMaxS];  // [s][combination]
  const int64_t b = blockIdx.z;
  const int g = blockIdx.y;
  if (g >= fp.G) return;  // uniform over the CTA
  const FactGroup& gr = fp.grp[g];
  const int nrow = gr.n_obs + gr.n_w + 1;
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if ((int)(blockIdx.x * blockDim.x) >= gr.R) return;  // uniform over the CTA
  const bool active = r < gr.R;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const bool ut = (p.flags & B2_FLAG_USE_UTILITY) != 0;
  const int S0 = gr.S[0];
  const int s1 = gr.rank > 2 ? r / gr.S[2] : r;
  const int s2 = gr.rank > 2 ? r - s1 * gr.S[2] : 0;
  const int64_t base = active ? (int64_t)(gr.rank > 1 ? s1 : 0) * gr.stA[1] + (int64_t)s2 * gr.stA[2] : 0;
  const int64_t st0 = gr.stA[0];
  const float* Qb = Qh + b * fp.qh_stride;
  float* Vb = V1 + b * fp.v1_stride;
  // combinations of this group: depth-major, then h0
  int ncomb = 0;
  for (int t = 0; t < p.T; ++t) ncomb += gr.H[0][t];
  int t0 = 0, h0 = 0;  // first combination of the current chunk
  for (int c0 = 0; c0 < ncomb; c0 += KC) {
    const int nc = ncomb - c0 < KC ? ncomb - c0 : KC;
    int ct[KC], ch[KC];
    {
      int t = t0, h = h0;
#pragma unroll
      for (int i = 0; i < KC; ++i) {
        ct[i] = t;
        ch[i] = h;
        if (i < nc && ++h == gr.H[0][t] && t + 1 < p.T) {
          h = 0;
          ++t;
        }
      }
      t0 = t;
      h0 = h;
    }
    __syncthreads();  // the previous chunk's readers are done with qsm
    for (int e = threadIdx.x; e < nc * S0; e += blockDim.x) {
      const int i = e / S0, s = e - i * S0;
      int t = ct[0], h = ch[0];
      for (int k = 0; k < i; ++k)
        if (++h == gr.H[0][t]) {
          h = 0;
          ++t;
        }
      qsm[s * KC + i] = Qb[fp.qh_off[gr.f[0]][t] + (int64_t)h * S0 + s];
    }
    __syncthreads();
    if (!active) continue;
    float lin[KC];
#pragma unroll
    for (int i = 0; i < KC; ++i) lin[i] = 0.f;
    // each combination's V1 column for this thread (row 0), advanced by R per row
    float* vcol[KC];
#pragma unroll
    for (int i = 0; i < KC; ++i) vcol[i] = Vb + gr.v1_off[ct[i]] + (int64_t)ch[i] * nrow * gr.R + r;
    const int64_t Rg = gr.R;  // parameter fields read once: a capped register file would re-read them per row
    int row = 0;
    for (int mi = gr.m_begin; mi < gr.m_end; ++mi) {
      const EfeModality& md = p.mod[fp.mod_order[mi]];
      const int Om = md.O;
      const int64_t Km = md.K;
      const float* Am = A + b * p.A_stride + md.A_off + base;
      const float* Cm = C + b * p.C_stride + md.C_off;
      const float* crow[KC];  // each combination's C_t row of this modality
#pragma unroll
      for (int i = 0; i < KC; ++i) crow[i] = Cm + (int64_t)ct[i] * Om;
      // NJ > 0: every group's level-1 axis is 4 NJ contiguous, 16-byte aligned
      // entries; the next row's loads are issued before this row's
      // arithmetic, two rows in flight per thread
      constexpr bool pipe = NJ > 0;
      constexpr int NJ1 = NJ > 0 ? NJ : 1;
      float4 nx[NJ1];
      if (pipe) {
        const float4* A4 = reinterpret_cast<const float4*>(Am);
#pragma unroll
        for (int j = 0; j < NJ1; ++j) nx[j] = __ldg(A4 + j);
      }
      for (int o = 0; o < Om; ++o, ++row) {
        // combinations (2i, 2i + 1) in the halves of packed accumulators
        constexpr int KP = (KC + 1) / 2;
        float2 v2[KP], w2[KP];
#pragma unroll
        for (int i = 0; i < KP; ++i) v2[i] = w2[i] = make_float2(0.f, 0.f);
        const float* Ar = Am + (int64_t)o * Km;
        auto take = [&](float a, int s) {
          const float xl = ig ? a * log_fast(a) : 0.f;
          const float2 aa = make_float2(a, a), xx = make_float2(xl, xl);
          if (KC % 4 == 0) {
#pragma unroll
            for (int i = 0; i < KC / 4; ++i) {
              const float4 q4 = *reinterpret_cast<const float4*>(qsm + s * KC + 4 * i);
              const float2 qa = make_float2(q4.x, q4.y), qb = make_float2(q4.z, q4.w);
              v2[2 * i] = fma2(qa, aa, v2[2 * i]);
              w2[2 * i] = fma2(qa, xx, w2[2 * i]);
              v2[2 * i + 1] = fma2(qb, aa, v2[2 * i + 1]);
              w2[2 * i + 1] = fma2(qb, xx, w2[2 * i + 1]);
            }
          } else {
#pragma unroll
            for (int i = 0; i < KC; ++i) {
              const float q = qsm[s * KC + i];
              float2& vv = v2[i >> 1];
              float2& ww = w2[i >> 1];
              if (i & 1) {
                vv.y = fmaf(q, a, vv.y);
                ww.y = fmaf(q, xl, ww.y);
              } else {
                vv.x = fmaf(q, a, vv.x);
                ww.x = fmaf(q, xl, ww.x);
              }
            }
          }
        };
        if (pipe) {
          float4 cu[NJ1];
#pragma unroll
          for (int j = 0; j < NJ1; ++j) cu[j] = nx[j];
          if (o + 1 < Om) {
            const float4* A4 = reinterpret_cast<const float4*>(Ar + Km);
#pragma unroll
            for (int j = 0; j < NJ1; ++j) nx[j] = __ldg(A4 + j);
          }
#pragma unroll
          for (int j = 0; j < NJ1; ++j) {
            take(cu[j].x, 4 * j);
            take(cu[j].y, 4 * j + 1);
            take(cu[j].z, 4 * j + 2);
            take(cu[j].w, 4 * j + 3);
          }
        } else if (gr.vec4) {
          // contiguous, 16-byte aligned level-1 axis: four entries per load
          for (int s = 0; s < S0; s += 4) {
            const float4 a4 = __ldg(reinterpret_cast<const float4*>(Ar + s));
            take(a4.x, s);
            take(a4.y, s + 1);
            take(a4.z, s + 2);
            take(a4.w, s + 3);
          }
        } else {
          for (int s = 0; s < S0; ++s) take(__ldg(Ar + s * st0), s);
        }
#pragma unroll
        for (int i = 0; i < KC; ++i) {
          if (i < nc) {
            const float vi = i & 1 ? v2[i >> 1].y : v2[i >> 1].x;
            const float wi = i & 1 ? w2[i >> 1].y : w2[i >> 1].x;
            vcol[i][(int64_t)row * Rg] = vi;
            lin[i] += wi + (ut ? __ldg(crow[i] + o) * vi : 0.f);
          }
        }
      }
    }
    if (gr.n_w) {
      // parameter-information-gain weights: the same contraction, rows n_obs ..
      int wrow = gr.n_obs;
      for (int mi = gr.m_begin; mi < gr.m_end; ++mi) {
        const EfeModality& md = p.mod[fp.mod_order[mi]];
        const float* Wm = wA + b * p.A_stride + md.A_off + base;
        for (int o = 0; o < md.O; ++o, ++wrow) {
          float v[KC];
#pragma unroll
          for (int i = 0; i < KC; ++i) v[i] = 0.f;
          const float* Wr = Wm + (int64_t)o * md.K;
          for (int s = 0; s < S0; ++s) {
            const float a = __ldg(Wr + s * st0);
#pragma unroll
            for (int i = 0; i < KC; ++i) v[i] = fmaf(qsm[s * KC + i], a, v[i]);
          }
#pragma unroll
          for (int i = 0; i < KC; ++i)
            if (i < nc) vcol[i][(int64_t)wrow * Rg] = v[i];
        }
      }
    }
#pragma unroll
    for (int i = 0; i < KC; ++i)
      if (i < nc) vcol[i][(int64_t)(nrow - 1) * Rg] = lin[i];
  }
}

// Levels 2 and 3 and the epilogue. CTA (tile, b) covers one (group, depth t,
// h0, tile of up to TILE level-2 histories h1) of the tail work list.
// rank 3: V2[n][s2] = sum_s1 q1^{h1}[s1] V1[h0][n][s1,s2] in shared memory,
//         then qo[n] = sum_s2 q2^{h2}[s2] V2[n][s2] for every h2;
// rank 2: qo[n] = sum_s1 q1^{h1}[s1] V1[h0][n][s1] for every h1 of the tile;
// rank 1: qo[n] = V1[h0][n][0].
// Four threads per output column share the rows; their entropy sums meet by
// shuffles. Table entry = sum over observation rows of -qo log clip qo (when
// the information gain is on) + the linear row.
struct TailItem {
  int32_t g, t, h0, h1_begin;
};

__device__ __forceinline__ void tail_item(const FactParams& fp, int idx, TailItem* it) {
  for (int g = 0; g < fp.G; ++g) {
    const FactGroup& gr = fp.grp[g];
    for (int t = 0; t < fp.T; ++t) {
      const int h1n = gr.rank >= 3 ? gr.H[1][t] : 1;
      const int tiles = (h1n + fp.h1_tile - 1) / fp.h1_tile;
      const int n = gr.H[0][t] * tiles;
      if (idx < n) {
        it->g = g;
        it->t = t;
        it->h0 = idx / tiles;
        it->h1_begin = (idx - it->h0 * tiles) * fp.h1_tile;
        return;
      }
      idx -= n;
    }
  }
  it->g = -1;
}

// SMAX: a compile-time bound on the size of the factor of the last level (so
// a thread's marginals stay in registers); HPT of them per thread share each
// shared-memory load of the level's intermediate.
template <int SMAX>
struct TailShape {
  static constexpr int kHpt = SMAX <= 16 ? 4 : (SMAX <= 32 ? 2 : 1);
};

// Step value of one prefix from its rows of the last level: for each
// observation row o, -qo log clip qo (information gain on) and, with the
// parameter-information-gain rows, -qo * (wA . x)[o] (calc_negative_pA_info_gain,
// pymdp/control.py:511-553); plus the linear row (utility and the H_A part).
__device__ __forceinline__ double obs_term(bool ig, float d, bool w, float dw) {
  double v = ig ? -(double)d * (double)log_stable(d) : 0.0;
  if (w) v -= (double)d * dw;
  return v;
}

// The same in FP32, for the per-thread sums of the last level (at most a few
// dozen terms in [0, 0.37] each, FP64 from the pair sum on).
__device__ __forceinline__ float obs_term_f(bool ig, float d, bool w, float dw) {
  float v = ig ? -d * log_fast(d) : 0.f;
  if (w) v = fmaf(-d, dw, v);
  return v;
}

// Last level for HPT columns per thread: rows of X (shared memory, row stride
// xs, a multiple of 4 floats read as float4, zero past S; [n_obs A rows]
// [n_w wA rows][1 linear row]); observation rows o = part, part +
// kTailTpi, ..., the linear row by part 0; the parts of a column meet by
// shuffles within their kTailTpi consecutive lanes. `act` false: the thread
// only joins the shuffles.
template <int SMAX, bool FULL>
__device__ __forceinline__ void tail_final(const float* __restrict__ X, int xs, int n_obs, int n_w, bool ig,
                                           int S, const float2 (&qv)[TailShape<SMAX>::kHpt][SMAX / 2],
                                           int half, bool act, double (&out)[TailShape<SMAX>::kHpt]) {
  constexpr int HPT = TailShape<SMAX>::kHpt;
#pragma unroll
  for (int c = 0; c < HPT; ++c) out[c] = 0.0;
  // even and odd states in the two halves of a packed accumulator
  auto dot = [&](const float* xr, float (&d)[HPT]) {
    float2 a2[HPT];
#pragma unroll
    for (int c = 0; c < HPT; ++c) a2[c] = make_float2(0.f, 0.f);
#pragma unroll
    for (int s4 = 0; s4 < SMAX / 4; ++s4) {
      if (FULL || 4 * s4 < S) {  // FULL: S == SMAX, no guard
        const float4 x = *reinterpret_cast<const float4*>(xr + 4 * s4);
        const float2 x01 = make_float2(x.x, x.y), x23 = make_float2(x.z, x.w);
#pragma unroll
        for (int c = 0; c < HPT; ++c) {
          a2[c] = fma2(qv[c][2 * s4], x01, a2[c]);
          a2[c] = fma2(qv[c][2 * s4 + 1], x23, a2[c]);
        }
      }
    }
#pragma unroll
    for (int c = 0; c < HPT; ++c) d[c] = a2[c].x + a2[c].y;
  };
  float acc[HPT];
#pragma unroll
  for (int c = 0; c < HPT; ++c) acc[c] = 0.f;
  if (act) {
#pragma unroll 2
    for (int o = half; o < n_obs; o += kTailTpi) {
      float d[HPT], dw[HPT];
      dot(X + o * xs, d);
      if (n_w) dot(X + (n_obs + o) * xs, dw);
#pragma unroll
      for (int c = 0; c < HPT; ++c) acc[c] += obs_term_f(ig, d[c], n_w != 0, n_w ? dw[c] : 0.f);
    }
    if (half == 0) {
      float d[HPT];
      dot(X + (n_obs + n_w) * xs, d);
#pragma unroll
      for (int c = 0; c < HPT; ++c) out[c] = (double)d[c];
    }
  }
#pragma unroll
  for (int c = 0; c < HPT; ++c) {
    out[c] += (double)acc[c];
#pragma unroll
    for (int x = 1; x < kTailTpi; x <<= 1) out[c] += __shfl_xor_sync(0xffffffffu, out[c], x);
  }
}

template <int SMAX, int TILE, bool FULL>
__global__ void __launch_bounds__(kFactTailThreads) efe_fact_tail_kernel(const __grid_constant__ EfeParams p,
                                                                        const __grid_constant__ FactParams fp,
                                                                        const float* __restrict__ Qh,
                                                                        const float* __restrict__ V1,
                                                                        double* __restrict__ tab) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  constexpr int HPT = TailShape<SMAX>::kHpt;
  static_assert(TILE % 4 == 0, "level 2 reads the tile's marginals as float4");
  extern __shared__ float4 tsm4[];  // rank 3: [TILE][nrow][xs] level-2 blocks, then q1 tile [S1][TILE]
  float* tsm = reinterpret_cast<float*>(tsm4);
  TailItem it;
  tail_item(fp, blockIdx.x, &it);
  if (it.g < 0) return;  // uniform over the CTA
  const int64_t b = blockIdx.y;
  const FactGroup& gr = fp.grp[it.g];
  const int t = it.t, h0 = it.h0;
  const int n_obs = gr.n_obs, n_w = gr.n_w, nrow = n_obs + n_w + 1;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const float* Qb = Qh + b * fp.qh_stride;
  const float* V1b = V1 + b * fp.v1_stride + gr.v1_off[t] + (int64_t)h0 * nrow * gr.R;
  double* tb = tab + b * fp.tab_stride + gr.tab_off[t];
  const int tid = threadIdx.x;

  if (gr.rank == 1) {
    if (tid < 32) {
      double hs = 0.0;
      for (int o = tid; o < n_obs; o += 32)
        hs += obs_term(ig, __ldg(V1b + (int64_t)o * gr.R), n_w != 0,
                       n_w ? __ldg(V1b + (int64_t)(n_obs + o) * gr.R) : 0.f);
      if (tid == 0) hs += (double)__ldg(V1b + (int64_t)(nrow - 1) * gr.R);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) hs += __shfl_xor_sync(0xffffffffu, hs, o);
      if (tid == 0) tb[h0] = hs;
    }
    return;
  }
  // the last level contracts factor fl (size SL, HL histories) against X
  // ([nrow][SL] blocks in shared memory, row stride xs = SL rounded up to 4,
  // zero-filled past SL)
  const int rk = gr.rank;
  const int fl = gr.f[rk - 1], SL = gr.S[rk - 1], HL = gr.H[rk - 1][t];
  const int xs = (SL + 3) & ~3;
  const float* ql = Qb + fp.qh_off[fl][t];
  int nblk = 1, h1_begin = 0, H1 = 1;
  if (rk == 2) {
    // X = the V1 block itself
    for (int e = tid; e < nrow * xs; e += kFactTailThreads) {
      const int n = e / xs, s = e - n * xs;
      tsm[e] = s < SL ? __ldg(V1b + (int64_t)n * gr.R + s) : 0.f;
    }
  } else {
    // level 2 for the tile's h1 values at once: each V1 element read once
    const int S1 = gr.S[1];
    H1 = gr.H[1][t];
    h1_begin = it.h1_begin;
    nblk = H1 - h1_begin < TILE ? H1 - h1_begin : TILE;
    float* q1s = tsm + TILE * nrow * xs;  // [s1][h], h innermost
    const float* q1 = Qb + fp.qh_off[gr.f[1]][t] + (int64_t)h1_begin * S1;
    for (int e = tid; e < TILE * S1; e += kFactTailThreads) {
      const int h = e / S1, s1 = e - h * S1;
      q1s[s1 * TILE + h] = h < nblk ? __ldg(q1 + e) : 0.f;
    }
    __syncthreads();
    const float4* q1s4 = reinterpret_cast<const float4*>(q1s);
    const int64_t R1 = gr.R;  // read once (the loop below runs near the register cap)
    // two outputs (n, s2) per thread at a time: twice the V1 loads in flight
    constexpr int kStride = kFactTailThreads;
    for (int e0 = tid; e0 < nrow * xs; e0 += 2 * kStride) {
      float2 acc2[2][TILE / 2];  // [output][histories (2i, 2i + 1)]
#pragma unroll
      for (int u = 0; u < 2; ++u)
#pragma unroll
        for (int h = 0; h < TILE / 2; ++h) acc2[u][h] = make_float2(0.f, 0.f);
      const float* vr[2];
      bool ok[2];
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int e = e0 + u * kStride;
        const int n = e / xs, s2 = e - n * xs;
        ok[u] = e < nrow * xs && s2 < SL;
        vr[u] = V1b + (int64_t)(ok[u] ? n : 0) * R1 + (ok[u] ? s2 : 0);
      }
#pragma unroll 8
      for (int s1 = 0; s1 < S1; ++s1) {
        float v[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) v[u] = ok[u] ? __ldg(vr[u] + (int64_t)s1 * SL) : 0.f;
#pragma unroll
        for (int h4 = 0; h4 < TILE / 4; ++h4) {
          const float4 qa = q1s4[(TILE / 4) * s1 + h4];
#pragma unroll
          for (int u = 0; u < 2; ++u) {
            const float2 vv = make_float2(v[u], v[u]);
            acc2[u][2 * h4] = fma2(make_float2(qa.x, qa.y), vv, acc2[u][2 * h4]);
            acc2[u][2 * h4 + 1] = fma2(make_float2(qa.z, qa.w), vv, acc2[u][2 * h4 + 1]);
          }
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int e = e0 + u * kStride;
        if (e < nrow * xs) {
          const int n = e / xs, s2 = e - n * xs;
#pragma unroll
          for (int h = 0; h < TILE; ++h)
            if (h < nblk) tsm[(h * nrow + n) * xs + s2] = h & 1 ? acc2[u][h >> 1].y : acc2[u][h >> 1].x;
        }
      }
    }
  }
  __syncthreads();
  // final level: work items (block h, group of HPT histories of fl), two threads each
  const int groups = (HL + HPT - 1) / HPT;
  // histories as float4: SL a multiple of 4 and the depth's block 16-byte aligned
  const bool q4 = (SL & 3) == 0 && (fp.qh_off[fl][t] & 3) == 0;
  const int items = nblk * groups;
  for (int w0 = 0; w0 < items; w0 += kFactTailThreads / kTailTpi) {
    const int w = w0 + tid / kTailTpi, half = tid % kTailTpi;
    const bool act = w < items;  // uniform per lane pair; every lane still takes part in the shuffle
    const int hb = act ? w / groups : 0, hg = act ? w - hb * groups : 0;
    float2 qv[HPT][SMAX / 2];  // marginals of this thread's histories, zero past SL
    if (q4) {
#pragma unroll
      for (int c = 0; c < HPT; ++c) {
        const int hl = hg * HPT + c;
        const float4* q4p = reinterpret_cast<const float4*>(ql + (int64_t)hl * SL);
#pragma unroll
        for (int s4 = 0; s4 < SMAX / 4; ++s4) {
          const float4 v = (act && hl < HL && 4 * s4 < SL) ? __ldg(q4p + s4) : make_float4(0.f, 0.f, 0.f, 0.f);
          qv[c][2 * s4] = make_float2(v.x, v.y);
          qv[c][2 * s4 + 1] = make_float2(v.z, v.w);
        }
      }
    } else {
#pragma unroll
      for (int c = 0; c < HPT; ++c) {
        const int hl = hg * HPT + c;
        const bool ok = act && hl < HL;
#pragma unroll
        for (int s2 = 0; s2 < SMAX / 2; ++s2) {
          const int s = 2 * s2;
          qv[c][s2] = make_float2(ok && s < SL ? __ldg(ql + (int64_t)hl * SL + s) : 0.f,
                                  ok && s + 1 < SL ? __ldg(ql + (int64_t)hl * SL + s + 1) : 0.f);
        }
      }
    }
    double out[HPT];
    tail_final<SMAX, FULL>(tsm + hb * nrow * xs, xs, n_obs, n_w, ig, SL, qv, half, act, out);
    if (act && half == 0) {
#pragma unroll
      for (int c = 0; c < HPT; ++c) {
        const int hl = hg * HPT + c;
        if (hl < HL) {
          const int64_t base = rk == 2 ? (int64_t)h0 * HL : ((int64_t)h0 * H1 + h1_begin + hb) * HL;
          tb[base + hl] = out[c];
        }
      }
    }
  }
}

// G[b, pol] = sum_t sum_g T_g,t[histories of pol's prefix at t] (+ the
// per-factor history terms): the policy's actions come from its index in
// construct_policies order (mixed radix: the joint action of step t is digit
// T-1-t of pol in base nu). One CTA per agent with its tables staged in shared
// memory (when they fit); a work item is one prefix of the first T-1 steps
// and a run of up to kCombRun consecutive last actions, whose factor digits
// advance as a mixed-radix counter (no division per policy).
constexpr int kCombRun = 16;

__global__ void __launch_bounds__(256) efe_fact_combine_kernel(const __grid_constant__ EfeParams p,
                                                               const __grid_constant__ FactParams fp,
                                                               const double* __restrict__ tab,
                                                               const double* __restrict__ Ht, float* __restrict__ G,
                                                               int staged) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  extern __shared__ double ctab[];  // staged: tables [tab_stride], then history terms [ht_stride]
  const int64_t b = blockIdx.x;
  const double* tb = tab + b * fp.tab_stride;
  const double* hb = fp.hterm ? Ht + b * fp.ht_stride : nullptr;
  if (staged) {
    for (int i = threadIdx.x; i < fp.tab_stride; i += blockDim.x) ctab[i] = tb[i];
    if (fp.hterm)
      for (int i = threadIdx.x; i < fp.ht_stride; i += blockDim.x) ctab[fp.tab_stride + i] = hb[i];
    __syncthreads();
    tb = ctab;
    hb = fp.hterm ? ctab + fp.tab_stride : nullptr;
  }
  const int T = p.T, F = p.F, nu = fp.nu;
  int npre = 1;
  for (int t = 0; t + 1 < T; ++t) npre *= nu;
  const int runs = (nu + kCombRun - 1) / kCombRun;
  auto step_value = [&](int t, const int* hist) {
    double g = 0.0;
    for (int gi = 0; gi < fp.G; ++gi) {
      const FactGroup& gr = fp.grp[gi];
      int64_t idx = hist[gr.f[0]];
      if (gr.rank > 1) idx = idx * gr.H[1][t] + hist[gr.f[1]];
      if (gr.rank > 2) idx = idx * gr.H[2][t] + hist[gr.f[2]];
      g += tb[gr.tab_off[t] + idx];
    }
    if (fp.hterm)
      for (int f = 0; f < F; ++f) g += hb[fp.ht_off[f][t] + hist[f]];
    return g;
  };
  for (int item = threadIdx.x; item < npre * runs; item += blockDim.x) {
    const int pre = item / runs, a0 = (item - pre * runs) * kCombRun;
    // the prefix's actions, most significant (step 0) first
    int act[kFactMaxT];
    int rem = pre;
    for (int t = T - 2; t >= 0; --t) {
      act[t] = rem % nu;
      rem /= nu;
    }
    int hist[kEfeMaxF];
    for (int f = 0; f < F; ++f) hist[f] = 0;
    double g = 0.0;
    for (int t = 0; t + 1 < T; ++t) {
      for (int f = 0; f < F; ++f) hist[f] = hist[f] * p.U[f] + (act[t] / fp.ustride[f]) % p.U[f];
      g += step_value(t, hist);
    }
    // last step: the run's joint actions a0 .. a0 + kCombRun - 1 as per-factor digits
    int dig[kEfeMaxF], base[kEfeMaxF];
    for (int f = 0; f < F; ++f) {
      dig[f] = (a0 / fp.ustride[f]) % p.U[f];
      base[f] = hist[f] * p.U[f];
    }
    const int a1 = a0 + kCombRun < nu ? a0 + kCombRun : nu;
    float* out = G + b * p.P + (int64_t)pre * nu;
    for (int a = a0; a < a1; ++a) {
      int h[kEfeMaxF];
      for (int f = 0; f < F; ++f) h[f] = base[f] + dig[f];
      out[a] = (float)(g + step_value(T - 1, h));
      for (int f = F - 1; f >= 0; --f) {  // next joint action: the last factor's digit moves fastest
        if (++dig[f] < p.U[f]) break;
        dig[f] = 0;
      }
    }
  }
}


template <int SMAX, int TILE>
int32_t launch_tail_s(dim3 grid, int smem, cudaStream_t stream, const EfeParams& p, const FactParams& fp,
                      const float* Qh, const float* V1, double* tab) {
  // every group's last factor exactly SMAX states: the last level runs unguarded
  bool full = true;
  for (int g = 0; g < fp.G; ++g) {
    const FactGroup& gr = fp.grp[g];
    full = full && gr.rank >= 2 && gr.S[gr.rank - 1] == SMAX;
  }
  cudaError_t e;
  if (full) {
    B2_TRY(ensure_smem_attr((const void*)efe_fact_tail_kernel<SMAX, TILE, true>, smem, kEfeName));
    e = launch_pdl(efe_fact_tail_kernel<SMAX, TILE, true>, grid, dim3(kFactTailThreads), smem, stream, p, fp, Qh, V1,
                   tab);
  } else {
    B2_TRY(ensure_smem_attr((const void*)efe_fact_tail_kernel<SMAX, TILE, false>, smem, kEfeName));
    e = launch_pdl(efe_fact_tail_kernel<SMAX, TILE, false>, grid, dim3(kFactTailThreads), smem, stream, p, fp, Qh, V1,
                   tab);
  }
  return e != cudaSuccess ? cuda_fail(kEfeName, e) : check_launch("efe_ffi factored tail");
}

template <int TILE>
int32_t launch_tail(dim3 grid, int smem, cudaStream_t stream, const EfeParams& p, const FactParams& fp,
                    const float* Qh, const float* V1, double* tab) {
  if (fp.smax <= 8) return launch_tail_s<8, TILE>(grid, smem, stream, p, fp, Qh, V1, tab);
  if (fp.smax <= 16) return launch_tail_s<16, TILE>(grid, smem, stream, p, fp, Qh, V1, tab);
  if (fp.smax <= 32) return launch_tail_s<32, TILE>(grid, smem, stream, p, fp, Qh, V1, tab);
  return launch_tail_s<64, TILE>(grid, smem, stream, p, fp, Qh, V1, tab);
}

template <int KC>
cudaError_t launch_l1(int nj, dim3 grid, cudaStream_t stream, const EfeParams& p, const FactParams& fp, const float* A,
                      const float* C, const float* Qh, float* V1, const float* wA) {
  const dim3 blk(128);
  switch (nj) {
    case 1: return launch_pdl(efe_fact_l1_kernel<KC, 1>, grid, blk, 0, stream, p, fp, A, C, Qh, V1, wA);
    case 2: return launch_pdl(efe_fact_l1_kernel<KC, 2>, grid, blk, 0, stream, p, fp, A, C, Qh, V1, wA);
    case 3: return launch_pdl(efe_fact_l1_kernel<KC, 3>, grid, blk, 0, stream, p, fp, A, C, Qh, V1, wA);
    case 4: return launch_pdl(efe_fact_l1_kernel<KC, 4>, grid, blk, 0, stream, p, fp, A, C, Qh, V1, wA);
    default: return launch_pdl(efe_fact_l1_kernel<KC, 0>, grid, blk, 0, stream, p, fp, A, C, Qh, V1, wA);
  }
}

// Two-phase combine for models whose per-prefix and per-action offsets fit in
// shared memory (CTA per agent): phase 1, one thread per prefix of the first
// T-1 steps: its value (tables of steps 0..T-2) and, per group, the base of
// its last-step table index; phase 2, one thread per policy: G = prefix value
// + sum_g T_g,T-1[base_g(prefix) + off_g(last action)] (+ the last step's
// history terms), where off_g(a) = sum_k u_{f_k}(a) mult_gk depends on the
// last joint action alone.
struct CombLayout {
  int32_t npre, tab_w, ht_w;  // prefixes; staged table / history-term doubles
  int32_t pv, base, off, hb, ua;  // double offset of prefix values; int offsets (in ints past the doubles)
};

__global__ void __launch_bounds__(256) efe_fact_combine2_kernel(const __grid_constant__ EfeParams p,
                                                                const __grid_constant__ FactParams fp,
                                                                const CombLayout L, const double* __restrict__ tab,
                                                                const double* __restrict__ Ht, float* __restrict__ G) {
  grid_dependency_wait();  // inputs come from the previous launch on the stream
  extern __shared__ double csm[];
  const int64_t b = blockIdx.x;
  const int T = p.T, F = p.F, nu = fp.nu, NG = fp.G;
  double* tb = csm;
  double* hb = csm + L.tab_w;
  double* pv = csm + L.pv;
  int* ib = reinterpret_cast<int*>(csm + L.pv + L.npre);
  int* base = ib + L.base;  // [NG][npre]
  int* off = ib + L.off;    // [NG][nu]
  int* hbase = ib + L.hb;   // [F][npre] (history terms)
  int* ua = ib + L.ua;      // [F][nu]
  // staging: 16-byte loads, eight in flight per thread (tab_stride and ht_stride are multiples of 32 doubles)
  auto stage = [&](double* dst, const double* src, int n) {
    const double2* s2 = reinterpret_cast<const double2*>(src);
    double2* d2 = reinterpret_cast<double2*>(dst);
    const int n2 = n >> 1;
    for (int i0 = threadIdx.x; i0 < n2; i0 += 8 * blockDim.x) {
      double2 v[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int i = i0 + k * blockDim.x;
        if (i < n2) v[k] = s2[i];
      }
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        const int i = i0 + k * blockDim.x;
        if (i < n2) d2[i] = v[k];
      }
    }
  };
  stage(tb, tab + b * fp.tab_stride, L.tab_w);
  if (fp.hterm) stage(hb, Ht + b * fp.ht_stride, L.ht_w);
  // per last action: the factor digits and each group's index offset
  for (int a = threadIdx.x; a < nu; a += blockDim.x) {
    for (int gi = 0; gi < NG; ++gi) {
      const FactGroup& gr = fp.grp[gi];
      int o = 0;
      for (int k = 0; k < gr.rank; ++k) {
        int mult = 1;
        for (int j = k + 1; j < gr.rank; ++j) mult *= gr.H[j][T - 1];
        o += ((a / fp.ustride[gr.f[k]]) % p.U[gr.f[k]]) * mult;
      }
      off[gi * nu + a] = o;
    }
    if (fp.hterm)
      for (int f = 0; f < F; ++f) ua[f * nu + a] = (a / fp.ustride[f]) % p.U[f];
  }
  __syncthreads();
  // phase 1: prefixes
  for (int pre = threadIdx.x; pre < L.npre; pre += blockDim.x) {
    int act[kFactMaxT];
    int rem = pre;
    for (int t = T - 2; t >= 0; --t) {
      act[t] = rem % nu;
      rem /= nu;
    }
    int hist[kEfeMaxF];
    for (int f = 0; f < F; ++f) hist[f] = 0;
    double g = 0.0;
    for (int t = 0; t + 1 < T; ++t) {
      for (int f = 0; f < F; ++f) hist[f] = hist[f] * p.U[f] + (act[t] / fp.ustride[f]) % p.U[f];
      for (int gi = 0; gi < NG; ++gi) {
        const FactGroup& gr = fp.grp[gi];
        int64_t idx = hist[gr.f[0]];
        if (gr.rank > 1) idx = idx * gr.H[1][t] + hist[gr.f[1]];
        if (gr.rank > 2) idx = idx * gr.H[2][t] + hist[gr.f[2]];
        g += tb[gr.tab_off[t] + idx];
      }
      if (fp.hterm)
        for (int f = 0; f < F; ++f) g += hb[fp.ht_off[f][t] + hist[f]];
    }
    pv[pre] = g;
    for (int gi = 0; gi < NG; ++gi) {
      const FactGroup& gr = fp.grp[gi];
      int o = 0;
      for (int k = 0; k < gr.rank; ++k) {
        int mult = 1;
        for (int j = k + 1; j < gr.rank; ++j) mult *= gr.H[j][T - 1];
        o += hist[gr.f[k]] * p.U[gr.f[k]] * mult;
      }
      base[gi * L.npre + pre] = (int)gr.tab_off[T - 1] + o;
    }
    if (fp.hterm)
      for (int f = 0; f < F; ++f) hbase[f * L.npre + pre] = (int)fp.ht_off[f][T - 1] + hist[f] * p.U[f];
  }
  __syncthreads();
  // phase 2: one thread per policy, consecutive policies on consecutive threads
  float* Gb = G + b * p.P;
  for (int o = threadIdx.x; o < p.P; o += blockDim.x) {
    const int pre = o / nu, a = o - pre * nu;
    double g = pv[pre];
    for (int gi = 0; gi < NG; ++gi) g += tb[base[gi * L.npre + pre] + off[gi * nu + a]];
    if (fp.hterm)
      for (int f = 0; f < F; ++f) g += hb[hbase[f * L.npre + pre] + ua[f * nu + a]];
    Gb[o] = (float)g;
  }
}

// Host plan; false when the model is outside the factored path.
bool fact_plan(const EfeParams& p, FactParams* fp, bool with_wA = false, bool with_hterm = false) {
  std::memset(fp, 0, sizeof(*fp));
  if (p.T < 1 || p.T > kFactMaxT) return false;
  int64_t nu = 1, P = 1;
  for (int f = 0; f < p.F; ++f) {
    if (p.fac[f].rank != 1 || p.fac[f].dep[0] != f) return false;  // factor-local transitions only
    if (p.S[f] > kFactMaxS) return false;
    nu *= p.U[f];
  }
  for (int t = 0; t < p.T && P <= p.P; ++t) P *= nu;
  if (P != p.P || nu > (1 << 20)) return false;
  fp->T = p.T;
  fp->F = p.F;
  fp->nu = (int32_t)nu;
  int us = 1;
  for (int f = p.F - 1; f >= 0; --f) {
    fp->ustride[f] = us;
    us *= p.U[f];
  }
  // history marginals
  int64_t off = 0;
  for (int f = 0; f < p.F; ++f)
    for (int t = 0; t < p.T; ++t) {
      fp->qh_off[f][t] = off;
      const double h = std::pow((double)p.U[f], t + 1);
      if (h > (1 << 24)) return false;
      off += (int64_t)h * p.S[f];
    }
  fp->qh_stride = (off + 63) / 64 * 64;
  fp->qh_words = (int32_t)off;
  // the history kernel's staging: B_f^T planes, qs_init, every history
  int64_t hw = 0;
  for (int f = 0; f < p.F; ++f) {
    // rows of odd stride (the staging writes run down a column); planes of small
    // factors shifted by S banks, so the half-warps of consecutive histories
    // (consecutive actions, consecutive planes) read different banks
    const int S = p.S[f];
    fp->bt_row[f] = S | 1;
    int plane = S * fp->bt_row[f];
    if (S < 32) plane += ((S - plane) % 32 + 32) % 32;
    fp->bt_plane[f] = plane;
    fp->bt_off[f] = (int32_t)hw;
    hw += (int64_t)p.U[f] * fp->bt_plane[f];
  }
  fp->qi_sm = (int32_t)hw;
  hw += p.S_tot;
  fp->qh_sm = (int32_t)hw;
  hw += off;
  fp->hist_smem = hw * 4 <= 160 * 1024 ? (int32_t)(hw * 4) : 0;
  fp->hterm = with_hterm ? 1 : 0;
  int64_t hoff = 0;
  for (int f = 0; f < p.F; ++f)
    for (int t = 0; t < p.T; ++t) {
      fp->ht_off[f][t] = hoff;
      hoff += ipow(p.U[f], t + 1);
    }
  fp->ht_stride = with_hterm ? (hoff + 31) / 32 * 32 : 0;
  // groups: modalities sharing one dependency tuple
  std::vector<std::vector<int>> tuples, members;
  for (int m = 0; m < p.M; ++m) {
    std::vector<int> tup(p.mod[m].dep, p.mod[m].dep + p.mod[m].rank);
    size_t g = 0;
    while (g < tuples.size() && tuples[g] != tup) ++g;
    if (g == tuples.size()) {
      tuples.push_back(tup);
      members.emplace_back();
    }
    members[g].push_back(m);
  }
  if ((int)tuples.size() > kFactMaxG) return false;
  fp->G = (int32_t)tuples.size();
  int n_order = 0;
  int64_t v1 = 0, tab = 0;
  int max_R = 1;
  for (int g = 0; g < fp->G; ++g) {
    const std::vector<int>& tup = tuples[g];
    const int r = (int)tup.size();
    if (r < 1 || r > kFactMaxRank) return false;
    FactGroup& gr = fp->grp[g];
    gr.rank = r;
    // A-axis strides of the tuple's factors (row-major over the state axes)
    std::vector<int64_t> st(r);
    int64_t s_ = 1;
    for (int a = r - 1; a >= 0; --a) {
      st[a] = s_;
      s_ *= p.S[tup[a]];
    }
    int n_obs = 0;
    for (int m : members[g]) n_obs += p.mod[m].O;
    const int n_w = with_wA ? n_obs : 0;
    const int nrow = n_obs + n_w + 1;
    // contraction order: the cheapest permutation (summed over depths)
    std::vector<int> perm(r);
    for (int i = 0; i < r; ++i) perm[i] = i;
    std::vector<int> best;
    double best_cost = 0;
    do {
      double cost = 0;
      for (int t = 0; t < p.T; ++t) {
        double combos = 1, rest = (double)s_;
        for (int i = 0; i < r; ++i) {
          const int f = tup[perm[i]];
          combos *= std::pow((double)p.U[f], t + 1);
          cost += combos * nrow * rest;  // level i + 1: combos x rows x remaining size (incl. own axis)
          rest /= p.S[f];
        }
      }
      // level-1 intermediates live in global memory: prefer few level-1 histories
      cost += 4.0 * std::pow((double)p.U[tup[perm[0]]], p.T) * nrow * (double)s_ / p.S[tup[perm[0]]];
      if (best.empty() || cost < best_cost) {
        best = perm;
        best_cost = cost;
      }
    } while (std::next_permutation(perm.begin(), perm.end()));
    for (int i = 0; i < kFactMaxRank; ++i) {
      if (i < r) {
        gr.f[i] = tup[best[i]];
        gr.S[i] = p.S[gr.f[i]];
        gr.stA[i] = (int32_t)st[best[i]];
      } else {
        gr.f[i] = gr.f[0];
        gr.S[i] = 1;
        gr.stA[i] = 0;
      }
    }
    gr.K = (int32_t)s_;
    gr.R = (int32_t)(s_ / gr.S[0]);
    // float4 loads of the level-1 axis: stride 1, and every (agent, row, s1, s2)
    // start a multiple of four floats
    bool v4 = gr.stA[0] == 1 && gr.S[0] % 4 == 0 && p.A_stride % 4 == 0 && s_ % 4 == 0 &&
              (r < 2 || gr.stA[1] % 4 == 0) && (r < 3 || gr.stA[2] % 4 == 0);
    for (int m : members[g]) v4 = v4 && p.mod[m].A_off % 4 == 0;
    gr.vec4 = v4 ? 1 : 0;
    // the tail's shared memory: kFactH1Tile level-2 blocks (rank 3) or the V1 block (rank 2)
    const int last = r == 3 ? gr.S[2] : (r == 2 ? gr.S[1] : 1);
    const int64_t xs = (last + 3) / 4 * 4;
    const int64_t tail_words = (r == 3 ? (int64_t)kFactH1Tile * nrow * xs + kFactH1Tile * kFactMaxS
                                       : (int64_t)nrow * xs);  // with the smallest tile
    if (tail_words * 4 > kFactTailSmem) return false;
    max_R = gr.R > max_R ? gr.R : max_R;
    gr.n_obs = n_obs;
    gr.n_w = n_w;
    gr.m_begin = n_order;
    for (int m : members[g]) fp->mod_order[n_order++] = (int8_t)m;
    gr.m_end = n_order;
    for (int t = 0; t < p.T; ++t) {
      for (int i = 0; i < kFactMaxRank; ++i) gr.H[i][t] = i < r ? ipow(p.U[gr.f[i]], t + 1) : 1;
      gr.v1_off[t] = v1;
      v1 += (int64_t)gr.H[0][t] * nrow * gr.R;
      gr.tab_off[t] = tab;
      tab += (int64_t)gr.H[0][t] * gr.H[1][t] * gr.H[2][t];
    }
  }
  fp->v1_stride = (v1 + 63) / 64 * 64;
  fp->tab_stride = (tab + 31) / 32 * 32;
  fp->max_R = max_R;
  int smax = 1;
  for (int g = 0; g < fp->G; ++g) {
    const FactGroup& gr = fp->grp[g];
    const int last = gr.rank == 3 ? gr.S[2] : (gr.rank == 2 ? gr.S[1] : 1);
    smax = last > smax ? last : smax;
  }
  fp->smax = smax;
  // level-2 tile: 16 histories when their blocks fit, else 8
  auto tail_bytes = [&](int tile) {
    int64_t tsm = 0;
    for (int g = 0; g < fp->G; ++g) {
      const FactGroup& gr = fp->grp[g];
      const int last = gr.rank == 3 ? gr.S[2] : (gr.rank == 2 ? gr.S[1] : 1);
      const int nr = gr.n_obs + gr.n_w + 1;
      const int64_t xs = (last + 3) / 4 * 4;
      const int64_t w = gr.rank == 3 ? (int64_t)tile * nr * xs + (int64_t)tile * kFactMaxS : (int64_t)nr * xs;
      tsm = w > tsm ? w : tsm;
    }
    return tsm * 4;
  };
  fp->h1_tile = tail_bytes(2 * kFactH1Tile) <= kFactTailSmem ? 2 * kFactH1Tile : kFactH1Tile;
  fp->tail_smem = (int32_t)tail_bytes(fp->h1_tile);
  int items = 0;
  for (int g = 0; g < fp->G; ++g)
    for (int t = 0; t < p.T; ++t) {
      const FactGroup& gr = fp->grp[g];
      const int h1n = gr.rank >= 3 ? gr.H[1][t] : 1;
      items += gr.H[0][t] * ((h1n + fp->h1_tile - 1) / fp->h1_tile);
    }
  fp->max_tiles = items;
  return true;
}

}  // namespace

bool efe_fact_applies(const EfeParams& p, int64_t Bn) {
  FactParams fp;
  return Bn <= 65535 && fact_plan(p, &fp);
}

int32_t launch_efe_fact(const EfeParams& p, int64_t Bn, const float* qs, const float* A, const float* B,
                        const float* C, float* G, cudaStream_t stream, bool* used, const float* wA,
                        const float* wB, const float* wI) {
  *used = false;
  FactParams fp;
  const bool hterm = wB != nullptr || wI != nullptr;
  if (Bn > 65535 || !fact_plan(p, &fp, wA != nullptr, hterm)) return B2_OK;
  const size_t qh_bytes = (size_t)Bn * fp.qh_stride * sizeof(float);
  const size_t v1_bytes = (size_t)Bn * fp.v1_stride * sizeof(float);
  const size_t tab_bytes = (size_t)Bn * fp.tab_stride * sizeof(double);
  const size_t ht_bytes = (size_t)Bn * fp.ht_stride * sizeof(double);
  if (v1_bytes > ((size_t)8 << 30)) return B2_OK;  // level-1 intermediates above 8 GB: take another path
  uint8_t* ws = nullptr;
  B2_TRY(ws_alloc((void**)&ws, tab_bytes + ht_bytes + qh_bytes + v1_bytes, stream, kEfeName));
  double* tab = reinterpret_cast<double*>(ws);
  double* Ht = hterm ? reinterpret_cast<double*>(ws + tab_bytes) : nullptr;
  float* Qh = reinterpret_cast<float*>(ws + tab_bytes + ht_bytes);
  float* V1 = reinterpret_cast<float*>(ws + tab_bytes + ht_bytes + qh_bytes);
  int32_t rc = ensure_smem_attr((const void*)efe_fact_hist_kernel, fp.hist_smem, kEfeName);
  if (rc == B2_OK) {
    const cudaError_t e = launch_pdl(efe_fact_hist_kernel, dim3((unsigned)Bn), dim3(256), fp.hist_smem, stream, p, fp, qs,
                                     B, Qh, wB, wI, Ht);
    rc = e != cudaSuccess ? cuda_fail(kEfeName, e) : check_launch("efe_ffi factored histories");
  }
  if (rc == B2_OK) {
    dim3 grid((unsigned)((fp.max_R + 127) / 128), (unsigned)fp.G, (unsigned)Bn);
    // combinations per pass: enough for the group with the most, at most
    // kFactCombo (fewer live accumulators, more resident CTAs)
    int nc = 1;
    for (int g = 0; g < fp.G; ++g) {
      int n = 0;
      for (int t = 0; t < p.T; ++t) n += fp.grp[g].H[0][t];
      nc = n > nc ? n : nc;
    }
    // the pipelined form: every group's level-1 axis vec4 with one size <= 16
    int nj = fp.grp[0].vec4 && fp.grp[0].S[0] <= 16 ? fp.grp[0].S[0] / 4 : 0;
    for (int g = 1; g < fp.G; ++g)
      if (!fp.grp[g].vec4 || fp.grp[g].S[0] != fp.grp[0].S[0]) nj = 0;
    const cudaError_t e = nc <= 1   ? launch_l1<1>(nj, grid, stream, p, fp, A, C, Qh, V1, wA)
                          : nc <= 2 ? launch_l1<2>(nj, grid, stream, p, fp, A, C, Qh, V1, wA)
                          : nc <= 4 ? launch_l1<4>(nj, grid, stream, p, fp, A, C, Qh, V1, wA)
                                    : launch_l1<kFactCombo>(nj, grid, stream, p, fp, A, C, Qh, V1, wA);
    rc = e != cudaSuccess ? cuda_fail(kEfeName, e) : check_launch("efe_ffi factored level 1");
  }
  if (rc == B2_OK) {
    const dim3 grid((unsigned)fp.max_tiles, (unsigned)Bn);
    const int smem = fp.tail_smem;
    rc = fp.h1_tile == 2 * kFactH1Tile ? launch_tail<2 * kFactH1Tile>(grid, smem, stream, p, fp, Qh, V1, tab)
                                       : launch_tail<kFactH1Tile>(grid, smem, stream, p, fp, Qh, V1, tab);
  }
  CombLayout cl{};
  int64_t c2_bytes = 0;
  {
    int64_t npre = 1;
    for (int t = 0; t + 1 < p.T; ++t) npre *= fp.nu;
    const int64_t nhg = fp.G + (hterm ? p.F : 0);
    cl.npre = (int32_t)(npre < (1 << 20) ? npre : (1 << 20));
    cl.tab_w = (int32_t)fp.tab_stride;
    cl.ht_w = hterm ? (int32_t)fp.ht_stride : 0;
    cl.pv = cl.tab_w + cl.ht_w;
    cl.base = 0;
    cl.off = (int32_t)(fp.G * npre);
    cl.hb = cl.off + (int32_t)(fp.G * fp.nu);
    cl.ua = cl.hb + (hterm ? (int32_t)(p.F * npre) : 0);
    const int64_t ints = nhg * (npre + fp.nu);
    c2_bytes = (int64_t)(cl.pv + npre) * 8 + ints * 4;
    if (npre >= (1 << 20) || c2_bytes > 96 * 1024) c2_bytes = 0;  // too large: the one-phase kernel
  }
  if (rc == B2_OK && c2_bytes > 0) {
    rc = ensure_smem_attr((const void*)efe_fact_combine2_kernel, (int)c2_bytes, kEfeName);
    if (rc == B2_OK) {
      const cudaError_t e = launch_pdl(efe_fact_combine2_kernel, dim3((unsigned)Bn), dim3(256), (size_t)c2_bytes, stream,
                                       p, fp, cl, tab, Ht, G);
      rc = e != cudaSuccess ? cuda_fail(kEfeName, e) : check_launch("efe_ffi factored combine");
    }
  } else if (rc == B2_OK) {
    // the agent's tables in shared memory when they fit in 96 KB
    const int64_t words = fp.tab_stride + (hterm ? fp.ht_stride : 0);
    const int staged = words * 8 <= 96 * 1024 ? 1 : 0;
    const int smem = staged ? (int)(words * 8) : 0;
    rc = ensure_smem_attr((const void*)efe_fact_combine_kernel, smem, kEfeName);
    if (rc == B2_OK) {
      const cudaError_t e = launch_pdl(efe_fact_combine_kernel, dim3((unsigned)Bn), dim3(256), (size_t)smem, stream, p, fp,
                                       tab, Ht, G, staged);
      rc = e != cudaSuccess ? cuda_fail(kEfeName, e) : check_launch("efe_ffi factored combine");
    }
  }
  cudaError_t fe = cudaFreeAsync(ws, stream);
  if (rc == B2_OK && fe != cudaSuccess) return cuda_fail(kEfeName, fe);
  *used = rc == B2_OK;
  return rc;
}

}  // namespace b2
