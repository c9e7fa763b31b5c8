// Factorized fixed-point iteration (FPI) for sm_100a.
//
// Semantics: pymdp/algos.py:88-155 (`run_factorized_fpi`) — the JAX body the
// reference hands to its FFI (`_jax_fpi`, algos.py:121-133):
//   log_q <- 0
//   repeat num_iter: q_f = softmax(log_q_f)
//                    log_q_f = log_prior_f + sum_{m : f in deps(m)} mll_{m,f}(q)
//   return softmax(log_q)
// where mll_{m,f} contracts ll_m with every other dependency marginal of
// modality m (algos.py:26-51). No early stop (the reference's native kernels
// stop at max|d log q| < 1e-5, fpi/fpi_cpu_core.h:245-248; its JAX path,
// which defines the results, does not).
//
// Design (a team of 32, 128 or 256 threads per agent, by work size):
//  * Load phase: each modality's log-likelihood block is read once from HBM
//    with coalesced loads and written into shared memory in a padded layout
//    whose non-innermost strides are odd, so a sweep along ANY axis by the
//    lanes of a warp is bank-conflict free. In the fused observation form the
//    loaded values are the observed slice A_m[o_m] (K contiguous floats) and
//    log(clip(., eps)) is applied on the fly — ll never exists in HBM.
//  * Precision: FP32 inputs and outputs; the ll blocks, marginals and log q
//    live in FP64 on chip. The products of two FP32 numbers are exact in
//    FP64, so the marginal dot products and the per-factor sums carry FP64
//    accumulation error only (FP32 accumulation misses the 1e-5-relative
//    posterior target vs the FP64 reference on ill-conditioned Dirichlet(0.5)
//    models). The softmax is FP64. The log of each gathered A entry and
//    prior is taken as e ln 2 (FP64) + logf(m) for x = m 2^e, m in
//    [sqrt(1/2), sqrt(2)): absolute error about 4e-8 whatever the magnitude
//    of log x. On models with many coupled factors the Jacobi sweeps amplify
//    per-iteration rounding, and a plain FP32 logf/expf (absolute error
//    proportional to |log x|, up to ~1.4e-6 at the clip) moves some
//    posteriors by up to ~2e-5 relative after 16 iterations.
//  * Modalities with identical dependency tuples are merged at plan time
//    (their ll blocks are summed once at load), removing duplicate
//    contractions; the marginals are linear in ll so this is exact algebra.
//  * Iterations run entirely on-chip: phase A = warp-shuffle softmax per
//    factor, phase B = one output state per lane group (group size =
//    team/S_f rounded down to a power of two, at most 32), each group summing
//    the contributions of every (group, axis) pair that touches the factor,
//    then a butterfly reduction inside the group. No atomics: results are
//    deterministic.
//  * Final softmax is written straight to the caller's output.
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace b2 {
namespace {

constexpr int kMaxRank = B2_MAX_DEP_RANK;
constexpr int kMaxF = B2_MAX_FACTORS;
constexpr int kMaxM = B2_MAX_MODALITIES;
constexpr int kMaxContrib = 128;
constexpr int kMaxSmemPerCta = 227 * 1024;

// One caller modality (a source of a merged group).
struct FpiSource {
  int64_t src_off;  // ll form: ll_offsets[m]; fused form: A_offsets[m]
  int32_t O;        // observation count (fused form)
  int32_t K;        // elements of one observed slice (prod of dependency sizes)
};

// Modalities with an identical dependency tuple are merged into one group:
// their log-likelihoods are summed once at load time, which is exact algebra
// (every marginal is linear in ll) and removes their duplicate contractions.
struct FpiGroup {
  int32_t sm_off;  // double offset of the padded ll block inside the agent's smem
  int32_t K;       // prod_i S[dep[i]]
  int8_t rank, src_begin, src_end, pad;
  int8_t dep[kMaxRank];
  int16_t sst[kMaxRank];  // padded shared-memory stride of each axis (odd except innermost)
};

// One (factor, group axis) contraction with its addressing precomputed.
struct FpiContrib {
  int16_t sm_off, base_st;  // group block, stride of the output axis
  int16_t d0, st0, q0;      // first other axis: size, smem stride, offset of its q
  int16_t d1, st1, q1;      // second other axis (rank 3)
  int8_t rank, ax, g, pad;
};

struct FpiParams {
  int32_t F, M, G, num_iter, S_tot;
  int32_t agent_words;  // shared-memory doubles per agent
  int32_t ll_sm_total;  // doubles of padded ll blocks
  int32_t S[kMaxF];
  int32_t lp_off[kMaxF + 1];
  int32_t con_off[kMaxF + 1];
  int8_t src_order[kMaxM];  // modalities sorted by group
  FpiSource src[kMaxM];
  FpiGroup grp[kMaxM];
  FpiContrib con[kMaxContrib];
};

struct FpiIO {
  const float* src;    // ll_flat (ll form) or A_flat (fused form)
  int64_t src_stride;  // per-agent stride of src in floats
  const int32_t* obs;  // [batch, M] (fused form)
  const float* prior;  // [batch, S_tot]: log priors (ll form) or priors (fused form)
  float* q_out;        // [batch, S_tot]
  int64_t batch;
};

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

// log of a positive normal float to about 4e-8 absolute: x = m 2^e with m in
// [sqrt(1/2), sqrt(2)), log x = e ln 2 in FP64 plus logf(m) in FP32, where
// |log m| <= 0.35 keeps logf's relative error an absolute one that small.
__device__ __forceinline__ double log_split(float x) {
  int e;
  float m = frexpf(x, &e);  // x = m 2^e, m in [0.5, 1)
  if (m < 0.70710678f) {
    m *= 2.f;
    --e;
  }
  return (double)e * 0.69314718055994530942 + (double)logf(m);
}

// softmax(logq) of n values by one warp, in FP64 (max, shifted exponential, sum).
template <typename OutT>
__device__ __forceinline__ void softmax_warp(const double* __restrict__ logq, OutT* __restrict__ out, int n,
                                             int lane) {
  double mx = -INFINITY;
  for (int i = lane; i < n; i += 32) mx = fmax(mx, logq[i]);
  mx = warp_max_d(mx);
  auto ex = [&](double x) { return exp(x - mx); };
  double sum = 0.0;
  for (int i = lane; i < n; i += 32) sum += ex(logq[i]);
  sum = warp_sum_d(sum);
  const double inv = 1.0 / sum;
  for (int i = lane; i < n; i += 32) out[i] = (OutT)(ex(logq[i]) * inv);
}

// rank >= 4: mixed-radix counter over the other axes (innermost last).
__device__ __noinline__ double contract_generic(const FpiGroup& gr, const FpiParams& p,
                                                const double* __restrict__ ll, const double* __restrict__ q,
                                                int ax, int s, int j, int G) {
  const double* L = ll + gr.sm_off + s * gr.sst[ax];
  int dd[kMaxRank - 1], st[kMaxRank - 1], qoff[kMaxRank - 1], dig[kMaxRank - 1];
  int n = 0, total = 1;
  for (int x = 0; x < gr.rank; ++x) {
    if (x == ax) continue;
    dd[n] = p.S[gr.dep[x]];
    st[n] = gr.sst[x];
    qoff[n] = p.lp_off[gr.dep[x]];
    total *= dd[n];
    ++n;
  }
  int rem = j;
  for (int y = n - 1; y >= 0; --y) {
    dig[y] = rem % dd[y];
    rem /= dd[y];
  }
  double acc = 0.0;
  for (int t = j; t < total; t += G) {
    double w = 1.0;
    int addr = 0;
    for (int y = 0; y < n; ++y) {
      w *= q[qoff[y] + dig[y]];
      addr += dig[y] * st[y];
    }
    acc = fma(L[addr], w, acc);
    dig[n - 1] += G;
    for (int y = n - 1; y > 0 && dig[y] >= dd[y]; --y) {
      dig[y - 1] += dig[y] / dd[y];
      dig[y] %= dd[y];
    }
  }
  return acc;
}

// Contribution of one (factor, group axis) pair to output state `s`, summed
// over this lane's share (t = j, j+G, ...) of the other indices. FP64 FMA
// chains, four independent accumulators for ILP.
template <bool GENERIC>
__device__ __forceinline__ double contract(const FpiContrib& c, const FpiParams& p, const double* __restrict__ ll,
                                           const double* __restrict__ q, int s, int j, int G) {
  const double* L = ll + c.sm_off + s * c.base_st;
  if (c.rank == 1) return j == 0 ? L[0] : 0.0;
  if (c.rank == 2) {
    const double* qa = q + c.q0;
    const int d = c.d0, st = c.st0;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
    int t = j;
    for (; t + 3 * G < d; t += 4 * G) {
      a0 = fma(L[t * st], qa[t], a0);
      a1 = fma(L[(t + G) * st], qa[t + G], a1);
      a2 = fma(L[(t + 2 * G) * st], qa[t + 2 * G], a2);
      a3 = fma(L[(t + 3 * G) * st], qa[t + 3 * G], a3);
    }
    for (; t < d; t += G) a0 = fma(L[t * st], qa[t], a0);
    return (a0 + a1) + (a2 + a3);
  }
  if (c.rank == 3) {
    const double* qa = q + c.q0;
    const double* qb = q + c.q1;
    const int d1 = c.d1, st0 = c.st0, st1 = c.st1;
    const int total = c.d0 * d1;
    int i0 = j / d1, i1 = j - i0 * d1;
    double a0 = 0.0, a1 = 0.0;
    int t = j;
    for (; t + G < total; t += 2 * G) {
      a0 = fma(L[i0 * st0 + i1 * st1], qa[i0] * qb[i1], a0);
      i1 += G;
      while (i1 >= d1) { i1 -= d1; ++i0; }
      a1 = fma(L[i0 * st0 + i1 * st1], qa[i0] * qb[i1], a1);
      i1 += G;
      while (i1 >= d1) { i1 -= d1; ++i0; }
    }
    if (t < total) a0 = fma(L[i0 * st0 + i1 * st1], qa[i0] * qb[i1], a0);
    return a0 + a1;
  }
  if (GENERIC) return contract_generic(p.grp[c.g], p, ll, q, c.ax, s, j, G);
  return 0.0;
}

template <int TEAM>
__device__ __forceinline__ void team_sync() {
  if (TEAM == 32) __syncwarp(); else __syncthreads();
}

// TEAM threads per agent: TEAM = 32 runs APC agents (one per warp) per CTA;
// TEAM > 32 runs one agent per CTA of TEAM threads. GENERIC adds the
// rank >= 4 contraction path (kept out of the rank <= 3 instantiations so
// their hot loop has no call and no local memory).
// Bit m set when agent b's observation of modality m lies in [0, O_m).
__device__ __forceinline__ uint32_t obs_valid_mask(const FpiParams& p, const FpiIO& io, int64_t b) {
  uint32_t ok = 0;
  for (int m = 0; m < p.M; ++m) {
    const int o = io.obs[b * p.M + m];
    if (o >= 0 && o < p.src[m].O) ok |= 1u << m;
  }
  return ok;
}

template <int TEAM, int APC, bool FUSED, bool GENERIC>
__global__ void __launch_bounds__(TEAM * APC)
    fpi_kernel(const __grid_constant__ FpiParams p, const FpiIO io) {
  extern __shared__ double smem_d[];
  const int slot = threadIdx.x / TEAM;
  const int t = threadIdx.x % TEAM;
  const int lane = threadIdx.x & 31;
  const int wid = t >> 5;
  const int64_t b = (int64_t)blockIdx.x * APC + slot;
  if (b >= io.batch) return;  // TEAM > 32: APC == 1, uniform over the CTA
  double* ll = smem_d + slot * p.agent_words;
  double* lp = ll + p.ll_sm_total;
  double* logq = lp + p.S_tot;
  double* q = logq + p.S_tot;

  // ---- load phase: merged ll blocks (fused: observed log-A slices) + log prior
  // Each source's row start (agent offset + observed slice) is resolved once
  // into shared memory before the element loop.
  int64_t* rowoff = reinterpret_cast<int64_t*>(q + p.S_tot);
  // An observation outside [0, O_m) is the reference's all-zero one-hot
  // (jax.nn.one_hot, pymdp/agent.py:673): its log-likelihood tensordot is 0,
  // so that modality adds nothing (pymdp/maths.py:233-235).
  const uint32_t obs_ok = FUSED ? obs_valid_mask(p, io, b) : 0xffffffffu;
  for (int m = t; m < p.M; m += TEAM) {
    int64_t r = b * io.src_stride + p.src[m].src_off;
    if (FUSED) {
      int o = io.obs[b * p.M + m];
      o = (o < 0 || o >= p.src[m].O) ? 0 : o;
      r += (int64_t)o * p.src[m].K;
    }
    rowoff[m] = r;
  }
  team_sync<TEAM>();
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    for (int k = t; k < gr.K; k += TEAM) {
      double v = 0.0;
      for (int si = gr.src_begin; si < gr.src_end; ++si) {
        const int m = p.src_order[si];
        if (!((obs_ok >> m) & 1u)) continue;
        const float a = __ldg(io.src + rowoff[m] + k);
        v += FUSED ? log_split(fmaxf(a, kMinVal)) : (double)a;
      }
      int rem = k, addr = 0;
      for (int x = gr.rank - 1; x > 0; --x) {
        const int d = p.S[gr.dep[x]];
        const int qd = rem / d;
        addr += (rem - qd * d) * gr.sst[x];
        rem = qd;
      }
      addr += rem * gr.sst[0];
      ll[gr.sm_off + addr] = v;
    }
  }
  for (int i = t; i < p.S_tot; i += TEAM) {
    const float v = __ldg(io.prior + b * p.S_tot + i);
    lp[i] = FUSED ? log_split(fmaxf(v, kMinVal)) : (double)v;
    logq[i] = 0.0;
  }
  team_sync<TEAM>();

  // ---- fixed-point iterations (Jacobi: every factor uses the previous q)
  for (int it = 0; it < p.num_iter; ++it) {
    for (int f = wid; f < p.F; f += TEAM / 32) softmax_warp(logq + p.lp_off[f], q + p.lp_off[f], p.S[f], lane);
    team_sync<TEAM>();
    for (int f = 0; f < p.F; ++f) {
      const int Sf = p.S[f];
      int per = TEAM / Sf;
      per = per < 1 ? 1 : (per > 32 ? 32 : per);
      const int G = 1 << (31 - __clz(per));  // lanes per output, power of two <= 32
      const int groups = TEAM / G;
      const int c0 = p.con_off[f], c1 = p.con_off[f + 1];
      for (int s0 = 0; s0 < Sf; s0 += groups) {
        const int s = s0 + t / G;
        const int j = t & (G - 1);
        double acc = 0.0;
        if (s < Sf)
          for (int c = c0; c < c1; ++c) acc += contract<GENERIC>(p.con[c], p, ll, q, s, j, G);
        for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (s < Sf && j == 0) logq[p.lp_off[f] + s] = acc + lp[p.lp_off[f] + s];
      }
    }
    team_sync<TEAM>();
  }

  // ---- posterior marginals
  float* out = io.q_out + b * p.S_tot;
  for (int f = wid; f < p.F; f += TEAM / 32) softmax_warp(logq + p.lp_off[f], out + p.lp_off[f], p.S[f], lane);
}

// --------------------------------------------------------------- host side
const char* const kName = "fpi_ffi";

std::string idx(const char* name, int64_t i) { return std::string(name) + "[" + std::to_string(i) + "]"; }

// Build kernel parameters from the reference's attribute set. Mirrors
// validate_fpi_attrs / build_modality_dispatch / check_distinct_modality_factor
// (pymdp/ffi/fpi/fpi_entry.h:24-82, fpi/fpi_precompute.h:56-112) and in
// addition checks that offsets are the prefix sums the layout implies.
// Fills everything except p->src[m] (set by the entry point).
int32_t build_params(FpiParams* p, std::vector<int64_t>* Kmod, const int64_t* S, int64_t F,
                     const int64_t* lp_offsets, int64_t lp_offsets_len, const int64_t* A_dep_flat,
                     int64_t A_dep_flat_len, const int64_t* A_dep_offsets, int64_t A_dep_offsets_len,
                     int32_t num_iter, const char* op) {
  std::memset(p, 0, sizeof(*p));
  const int64_t M = A_dep_offsets_len - 1;
  if (F <= 0 || M <= 0)
    return fail(B2_ERR_INVALID_ARGUMENT,
                std::string(op) + ": invalid F=" + std::to_string(F) + " or M=" + std::to_string(M));
  if (lp_offsets && lp_offsets_len != F + 1)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": lp_offsets size = " +
                                             std::to_string(lp_offsets_len) + ", expected " +
                                             std::to_string(F + 1));
  if (num_iter <= 0)
    return fail(B2_ERR_INVALID_ARGUMENT,
                std::string(op) + ": num_iter = " + std::to_string(num_iter) + ", must be positive");
  if (F > kMaxF || M > kMaxM)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": F=" + std::to_string(F) + ", M=" +
                                        std::to_string(M) + " exceed this build's limits (" +
                                        std::to_string(kMaxF) + ", " + std::to_string(kMaxM) + ")");
  p->F = (int32_t)F;
  p->M = (int32_t)M;
  p->num_iter = num_iter;
  int64_t off = 0;
  for (int64_t f = 0; f < F; ++f) {
    if (S[f] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": " + idx("S", f) + " must be positive");
    if (lp_offsets && (lp_offsets[f] != off))
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": lp_offsets must be the prefix sums of S");
    p->S[f] = (int32_t)S[f];
    p->lp_off[f] = (int32_t)off;
    off += S[f];
    if (off > 16384) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": total_S exceeds 16384");
  }
  if (lp_offsets && lp_offsets[F] != off)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": lp_offsets must be the prefix sums of S");
  p->lp_off[F] = (int32_t)off;
  p->S_tot = (int32_t)off;
  if (A_dep_offsets[0] != 0)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_dep_offsets must start at zero");
  // validate modalities and group identical dependency tuples
  std::vector<std::vector<int64_t>> tuples;
  std::vector<int> group_of(M);
  Kmod->assign(M, 1);
  for (int64_t m = 0; m < M; ++m) {
    if (A_dep_offsets[m + 1] < A_dep_offsets[m])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_dep_offsets must be monotonic");
    const int64_t rank = A_dep_offsets[m + 1] - A_dep_offsets[m];
    if (rank < 1 || rank > kMaxRank)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": modality " + std::to_string(m) +
                                               " A_dep rank " + std::to_string(rank) + " outside [1, " +
                                               std::to_string(kMaxRank) + "]");
    if (A_dep_offsets[m + 1] > A_dep_flat_len)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_dep_flat shorter than A_dep_offsets");
    std::vector<int64_t> tup;
    int64_t K = 1;
    for (int64_t i = 0; i < rank; ++i) {
      const int64_t d = A_dep_flat[A_dep_offsets[m] + i];
      if (d < 0 || d >= F)
        return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": modality " + std::to_string(m) +
                                                 " A_dep factor " + std::to_string(d) + " out of range");
      for (int64_t d2 : tup)
        if (d2 == d)
          return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": modality " + std::to_string(m) +
                                                   " has duplicate factor in A_dependencies");
      tup.push_back(d);
      K *= S[d];
      if (K > (1 << 24)) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": modality too large");
    }
    (*Kmod)[m] = K;
    p->src[m].K = (int32_t)K;
    int g = -1;
    for (size_t i = 0; i < tuples.size(); ++i)
      if (tuples[i] == tup) g = (int)i;
    if (g < 0) {
      g = (int)tuples.size();
      tuples.push_back(tup);
    }
    group_of[m] = g;
  }
  p->G = (int32_t)tuples.size();
  int n_src = 0;
  int64_t sm = 0;
  std::vector<std::vector<FpiContrib>> con(F);
  for (int g = 0; g < p->G; ++g) {
    FpiGroup& gr = p->grp[g];
    const std::vector<int64_t>& tup = tuples[g];
    const int rank = (int)tup.size();
    gr.rank = (int8_t)rank;
    gr.src_begin = (int8_t)n_src;
    for (int64_t m = 0; m < M; ++m)
      if (group_of[m] == g) p->src_order[n_src++] = (int8_t)m;
    gr.src_end = (int8_t)n_src;
    int64_t K = 1;
    for (int i = 0; i < rank; ++i) {
      gr.dep[i] = (int8_t)tup[i];
      K *= S[tup[i]];
    }
    gr.K = (int32_t)K;
    int64_t st = 1;  // padded strides: innermost 1, every other stride odd
    for (int x = rank - 1; x >= 0; --x) {
      if (st > 32767) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": modality too large for shared memory");
      gr.sst[x] = (int16_t)st;
      st = st * S[tup[x]];
      if (x > 0 && (st % 2) == 0) st += 1;
    }
    const int64_t footprint = (int64_t)gr.sst[0] * S[tup[0]];
    gr.sm_off = (int32_t)sm;
    sm += (footprint + 1) / 2 * 2;  // 16-byte aligned blocks
    if (sm > 32767) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": log-likelihood blocks exceed shared memory");
    for (int ax = 0; ax < rank; ++ax) {
      FpiContrib c;
      std::memset(&c, 0, sizeof(c));
      c.sm_off = (int16_t)gr.sm_off;
      c.base_st = gr.sst[ax];
      c.rank = (int8_t)rank;
      c.ax = (int8_t)ax;
      c.g = (int8_t)g;
      int n_other = 0;
      for (int x = 0; x < rank && rank <= 3; ++x) {
        if (x == ax) continue;
        const int16_t d = (int16_t)S[tup[x]], stx = gr.sst[x], qx = (int16_t)p->lp_off[tup[x]];
        if (n_other == 0) {
          c.d0 = d; c.st0 = stx; c.q0 = qx;
        } else {
          c.d1 = d; c.st1 = stx; c.q1 = qx;
        }
        ++n_other;
      }
      con[tup[ax]].push_back(c);
    }
  }
  int n = 0;
  for (int64_t f = 0; f < F; ++f) {
    p->con_off[f] = n;
    for (const FpiContrib& c : con[f]) {
      if (n >= kMaxContrib)
        return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": more than " + std::to_string(kMaxContrib) +
                                            " (factor, modality) contractions");
      p->con[n++] = c;
    }
  }
  p->con_off[F] = n;
  p->ll_sm_total = (int32_t)sm;
  const int64_t agent = sm + 3 * off + M;  // ll | lp | logq | q | per-source row offsets
  p->agent_words = (int32_t)((agent + 1) / 2 * 2);
  if ((int64_t)p->agent_words * 8 > kMaxSmemPerCta)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": per-agent working set of " +
                                        std::to_string((int64_t)p->agent_words * 8) +
                                        " bytes exceeds shared memory (227 KB)");
  return B2_OK;
}

// Multiply-adds per agent per iteration: sum over groups of rank * K.
int64_t work_per_iter(const FpiParams& p) {
  int64_t w = 0;
  for (int g = 0; g < p.G; ++g) w += (int64_t)p.grp[g].rank * p.grp[g].K;
  return w;
}


// ------------------------------------------------------ rank <= 2 fast path
// Models whose modalities all depend on at most two factors of at most 16
// states each (the 4096-agent FPI benchmark: 4 x 16 states, 6 modalities on
// 2 factors each) run one warp per agent with every contraction a 16 x 16
// matrix-vector product:
//  * each rank-2 group's summed log-likelihood is one zero-padded 16 x 16
//    FP64 block in shared memory (row stride 18 doubles: conflict-free
//    16-byte row loads and 8-byte column loads);
//  * rank-1 groups are constant in the iteration and are folded into the
//    log prior at load time;
//  * lane (r, h) = (lane & 15, lane >> 4) multiplies row r (or column r, for
//    the group's second factor) segment [8h, 8h + 8) with the other factor's
//    q and one shuffle finishes the row; the products are sorted by output
//    factor, so each factor's new log q is accumulated in registers and
//    written once per iteration;
//  * the softmax handles two factors per step (one per half-warp).
// FP64 throughout, like the generic kernel.
constexpr int kR2MaxS = 16;
constexpr int kR2Stride = 18;                    // doubles per padded block row
constexpr int kR2Block = kR2MaxS * kR2Stride;    // doubles per block
constexpr int kR2MaxMv = 2 * kMaxM;

constexpr int kR2MaxWarps = 4;

struct FpiR2 {
  int32_t n_mv;         // matrix-vector products per iteration
  int32_t warps;        // warps per agent (one agent per CTA)
  int32_t vec4;         // 1: every observed row is 16-byte aligned, K % 4 == 0, <= 2 sources per group
  int16_t f_begin[kR2MaxWarps + 1];   // warp w owns output factors [f_begin[w], f_begin[w+1])
  int16_t mv_begin[kR2MaxWarps + 1];  // ... and their products [mv_begin[w], mv_begin[w+1])
  int32_t blk_words;    // doubles of one agent's blocks
  int32_t agent_words;  // blocks | lp' | log q | q | per-source row offsets
  int16_t g_blk[kMaxM]; // block offset of rank-2 group g (-1: rank 1)
  int16_t mv_blk[kR2MaxMv];
  int8_t mv_in[kR2MaxMv], mv_out[kR2MaxMv], mv_tr[kR2MaxMv];
};

// Builds the fast-path plan; false when the model is outside it.
bool build_r2(const FpiParams& p, FpiR2* r) {
  std::memset(r, 0, sizeof(*r));
  for (int f = 0; f < p.F; ++f)
    if (p.S[f] > kR2MaxS) return false;
  int nb = 0;
  std::vector<std::vector<int>> by_out(p.F);  // mv indices grouped by output factor
  struct Mv { int blk, in, out, tr; };
  std::vector<Mv> mvs;
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    if (gr.rank > 2) return false;
    if (gr.rank == 1) {
      r->g_blk[g] = -1;
      continue;
    }
    r->g_blk[g] = (int16_t)(nb * kR2Block);
    // block = ll[i0][i1] over (dep[0], dep[1]); row products feed dep[0]
    mvs.push_back({nb * kR2Block, gr.dep[1], gr.dep[0], 0});
    mvs.push_back({nb * kR2Block, gr.dep[0], gr.dep[1], 1});
    ++nb;
  }
  if ((int)mvs.size() > kR2MaxMv) return false;
  int n = 0;
  for (int f = 0; f < p.F; ++f)
    for (const Mv& m : mvs)
      if (m.out == f) {
        r->mv_blk[n] = (int16_t)m.blk;
        r->mv_in[n] = (int8_t)m.in;
        r->mv_out[n] = (int8_t)m.out;
        r->mv_tr[n] = (int8_t)m.tr;
        ++n;
      }
  r->n_mv = n;
  // warps per agent: about four products per warp, then split the output
  // factors into contiguous ranges with balanced product counts
  int W = (n + 3) / 4;
  W = W < 1 ? 1 : (W > kR2MaxWarps ? kR2MaxWarps : W);
  W = W > p.F ? p.F : W;
  std::vector<int> per_f(p.F, 0);
  for (int i = 0; i < n; ++i) per_f[r->mv_out[i]]++;
  r->warps = W;
  int f = 0, mv = 0;
  for (int w = 0; w < W; ++w) {
    r->f_begin[w] = (int16_t)f;
    r->mv_begin[w] = (int16_t)mv;
    const int target = (n * (w + 1) + W - 1) / W;
    const int f_left = p.F - f, w_left = W - w;
    // take factors while below the target, leaving at least one per later warp
    while (f < p.F && (f_left - (f - r->f_begin[w])) > w_left - 1 &&
           (f == r->f_begin[w] || mv + per_f[f] <= target || w == W - 1)) {
      mv += per_f[f];
      ++f;
    }
  }
  r->f_begin[W] = (int16_t)p.F;
  r->mv_begin[W] = (int16_t)n;
  r->blk_words = nb * kR2Block;
  const int64_t words = (int64_t)r->blk_words + 4LL * p.F * kR2MaxS + p.M;
  if (words * 8 > 48 * 1024 || words > 32767) return false;
  r->agent_words = (int32_t)((words + 1) / 2 * 2);
  return true;
}

template <bool FUSED>
__global__ void __launch_bounds__(32 * kR2MaxWarps) fpi_r2_kernel(const __grid_constant__ FpiParams p,
                                                                  const __grid_constant__ FpiR2 r,
                                                                  const FpiIO io) {
  extern __shared__ double smem_d[];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nthr = blockDim.x;
  const int64_t b = blockIdx.x;
  if (b >= io.batch) return;  // uniform over the CTA (one agent per CTA)
  const int F = p.F;
  double* blk = smem_d;
  double* lpp = blk + r.blk_words;  // log prior + rank-1 log-likelihoods, [F][16]
  double* logq = lpp + F * kR2MaxS;
  double* qbuf = logq + F * kR2MaxS;  // two q buffers, [2][F][16]
  int64_t* rowoff = reinterpret_cast<int64_t*>(qbuf + 2 * F * kR2MaxS);

  // ---- load phase
  // out-of-range observation: that modality adds nothing (see fpi_kernel)
  const uint32_t obs_ok = FUSED ? obs_valid_mask(p, io, b) : 0xffffffffu;
  for (int m = tid; m < p.M; m += nthr) {
    int64_t ro = b * io.src_stride + p.src[m].src_off;
    if (FUSED) {
      int o = io.obs[b * p.M + m];
      o = (o < 0 || o >= p.src[m].O) ? 0 : o;
      ro += (int64_t)o * p.src[m].K;
    }
    rowoff[m] = ro;
  }
  for (int i = tid; i < r.blk_words; i += nthr) blk[i] = 0.0;
  for (int i = tid; i < F * kR2MaxS; i += nthr) {
    const int f = i >> 4, s = i & 15;
    double v = 0.0;
    if (s < p.S[f]) {
      const float x = __ldg(io.prior + b * p.S_tot + p.lp_off[f] + s);
      v = FUSED ? log_split(fmaxf(x, kMinVal)) : (double)x;
    }
    lpp[i] = v;
    logq[i] = 0.0;  // log q starts at 0 (pymdp/algos.py:121-133)
  }
  __syncthreads();
  // Group blocks are disjoint and rank-1 groups fold into distinct factors, so
  // no barrier is needed between groups.
  auto store = [&](int g, int k, double v) {
    const FpiGroup& gr = p.grp[g];
    const int bo = r.g_blk[g];
    if (bo < 0) {
      lpp[gr.dep[0] * kR2MaxS + k] += v;  // one thread per state: no race
    } else {
      const int S1 = p.S[gr.dep[1]];
      const int i0 = k / S1, i1 = k - i0 * S1;
      blk[bo + i0 * kR2Stride + i1] = v;
    }
  };
  if (r.vec4) {
    // items (group, 4 consecutive elements): up to four items per thread per
    // batch, all their 16-byte loads issued before any log
    int g = 0, k4 = tid;
    while (g < p.G && 4 * k4 >= p.grp[g].K) {
      ++g;
      k4 = tid;
    }
    while (g < p.G) {
      float4 va[4][2];
      int gi[4], ki[4];
      int n = 0;
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        if (g < p.G) {
          const FpiGroup& gr = p.grp[g];
          gi[x] = g;
          ki[x] = k4;
          const int m0 = p.src_order[gr.src_begin];
          const int m1 = gr.src_end - gr.src_begin > 1 ? p.src_order[gr.src_begin + 1] : -1;
          va[x][0] = (obs_ok >> m0) & 1u ? __ldg(reinterpret_cast<const float4*>(io.src + rowoff[m0]) + k4)
                                        : make_float4(1.f, 1.f, 1.f, 1.f);
          va[x][1] = m1 >= 0 && ((obs_ok >> m1) & 1u)
                         ? __ldg(reinterpret_cast<const float4*>(io.src + rowoff[m1]) + k4)
                         : make_float4(1.f, 1.f, 1.f, 1.f);
          n = x + 1;
          k4 += nthr;
          while (g < p.G && 4 * k4 >= p.grp[g].K) {
            ++g;
            k4 = tid;
          }
        }
      }
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        if (x < n) {
          const bool two = p.grp[gi[x]].src_end - p.grp[gi[x]].src_begin > 1;
          const float a0[4] = {va[x][0].x, va[x][0].y, va[x][0].z, va[x][0].w};
          const float a1[4] = {va[x][1].x, va[x][1].y, va[x][1].z, va[x][1].w};
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            double v = FUSED ? log_split(fmaxf(a0[e], kMinVal)) : (double)a0[e];
            if (two) v += FUSED ? log_split(fmaxf(a1[e], kMinVal)) : (double)a1[e];
            store(gi[x], 4 * ki[x] + e, v);
          }
        }
      }
    }
  } else {
    for (int g = 0; g < p.G; ++g) {
      const FpiGroup& gr = p.grp[g];
      for (int k = tid; k < gr.K; k += nthr) {
        double v = 0.0;
        for (int si = gr.src_begin; si < gr.src_end; ++si) {
          const int m = p.src_order[si];
          if (!((obs_ok >> m) & 1u)) continue;
          const float a = __ldg(io.src + rowoff[m] + k);
          v += FUSED ? log_split(fmaxf(a, kMinVal)) : (double)a;
        }
        store(g, k, v);
      }
    }
  }
  __syncthreads();

  // ---- fixed-point iterations (Jacobi: every factor uses the previous q).
  // Warp wid owns output factors [f0w, f1w): their softmax and their log q.
  // q is double-buffered, so one CTA barrier per iteration separates the
  // softmax writes from the other warps' product reads.
  const int rr = lane & 15, h = lane >> 4;
  const int f0w = r.f_begin[wid], f1w = r.f_begin[wid + 1];
  const int m0w = r.mv_begin[wid], m1w = r.mv_begin[wid + 1];
  for (int it = 0; it <= p.num_iter; ++it) {
    double* q = qbuf + (it & 1) * F * kR2MaxS;
    // q = softmax(log q) for this warp's factors, two per step; after the
    // last iteration the same step writes the posterior
    for (int fa = f0w; fa < f1w; fa += 2) {
      const int f = fa + h;
      const bool fok = f < f1w;
      const bool valid = fok && rr < p.S[fok ? f : fa];
      const double x = valid ? logq[f * kR2MaxS + rr] : -INFINITY;
      double mx = x;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      const double e = valid ? exp(x - mx) : 0.0;
      double sum = e;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
      if (it == p.num_iter) {
        if (valid) io.q_out[b * p.S_tot + p.lp_off[f] + rr] = (float)(e / sum);
      } else if (fok) {
        q[f * kR2MaxS + rr] = e / sum;
      }
    }
    if (it == p.num_iter) break;
    __syncthreads();
    // new log q of this warp's factors: log prior + sum of its products
    double acc = 0.0;
    int i = m0w;
    for (int f = f0w; f < f1w; ++f) {
      for (; i < m1w && r.mv_out[i] == f; ++i) {
        const double* M = blk + r.mv_blk[i];
        const double* qv = q + r.mv_in[i] * kR2MaxS + 8 * h;
        double a0 = 0.0, a1 = 0.0;
        if (r.mv_tr[i]) {
          const double* col = M + (8 * h) * kR2Stride + rr;
#pragma unroll
          for (int k = 0; k < 8; k += 2) {
            a0 = fma(col[k * kR2Stride], qv[k], a0);
            a1 = fma(col[(k + 1) * kR2Stride], qv[k + 1], a1);
          }
        } else {
          const double2* row = reinterpret_cast<const double2*>(M + rr * kR2Stride + 8 * h);
          const double2* q2 = reinterpret_cast<const double2*>(qv);
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const double2 m2 = row[k], v2 = q2[k];
            a0 = fma(m2.x, v2.x, a0);
            a1 = fma(m2.y, v2.y, a1);
          }
        }
        acc += a0 + a1;
      }
      acc += __shfl_xor_sync(0xffffffffu, acc, 16);
      if (h == 0 && rr < p.S[f]) logq[f * kR2MaxS + rr] = lpp[f * kR2MaxS + rr] + acc;
      acc = 0.0;
    }
    __syncwarp();
  }
}


// ---------------------------------------------- rank <= 3 two-step path
// Models with a modality on three factors, no modality on more than three
// and no factor above 64 states (the agent-step model: S = [32, 16, 8], five
// modalities on all three factors, merged into one group) run one agent per
// CTA with each rank-3 contraction taken in two steps:
//   X_g[a][b] = sum_c L_g[a][b][c] q_c[c],   Y_g[a][c] = sum_b L_g[a][b][c] q_b[b]
// (2 K multiply-adds per group, spread over every thread of the CTA), then
//   m_a = X_g q_b,   m_b = X_g^T q_a,   m_c = Y_g^T q_a
// and the rank-2 groups' L q_b / L^T q_a, one warp per output factor, which
// goes on to that factor's softmax. The direct form takes 3 K three-term
// products per group and sweep. The same sums in another order, FP64 on
// chip like the generic kernel; two barriers per sweep.
//  * Load phase: each thread issues float4 loads of its columns of up to four
//    observed rows at a time, all in flight before the logs are taken.
//  * rank-1 groups are constant in the iteration and fold into the log prior.
constexpr int kR3MaxS = 64;
constexpr int kR3MaxTerm = 3 * kMaxM;

// One message term of output factor f: m_f[s] += sum_{k < n} M[s * rs + k * cs] q[q_off + k].
struct FpiR3Term {
  int16_t m_off;  // the matrix (an ll block, or a group's X or Y): double offset in the agent's shared memory
  int16_t rs, cs;
  int16_t n;
  int16_t q_off;
  int16_t pad;
};

struct FpiR3 {
  int32_t n_items;                // X and Y entries of every rank-3 group (one dot product each)
  int32_t n3;                     // rank-3 groups
  int32_t item_begin[kMaxM + 1];  // entries of the i-th rank-3 group: [item_begin[i], item_begin[i + 1])
  int16_t g3[kMaxM];              // its group index
  int16_t x_off[kMaxM], y_off[kMaxM];  // X_i [S_a][xs], Y_i [S_a][ys] (odd row strides)
  int16_t xs[kMaxM], ys[kMaxM];
  int32_t lp_sm, q_sm, row_sm;    // log prior (+ rank-1 terms) | q, two buffers | source row offsets (int64)
  int32_t agent_words;
  int32_t vec4;                   // float4 loads of the observed rows
  int16_t term_begin[kMaxF + 1];
  int8_t f_lg[kMaxF];             // S_f <= 32: log2 of the lanes that split each of its message sums
  FpiR3Term term[kR3MaxTerm];
};

// The two-step plan; false when the model is outside it.
bool build_r3(const FpiParams& p, FpiR3* r) {
  std::memset(r, 0, sizeof(*r));
  bool any3 = false;
  for (int g = 0; g < p.G; ++g) {
    if (p.grp[g].rank > 3) return false;
    any3 |= p.grp[g].rank == 3;
  }
  if (!any3) return false;
  for (int f = 0; f < p.F; ++f)
    if (p.S[f] > kR3MaxS) return false;
  int64_t sm = p.ll_sm_total;
  std::vector<std::vector<FpiR3Term>> terms(p.F);
  int items = 0;
  auto odd = [](int s) { return s % 2 ? s : s + 1; };
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    if (gr.rank == 2) {
      const int a = gr.dep[0], b = gr.dep[1];
      terms[a].push_back({(int16_t)gr.sm_off, gr.sst[0], gr.sst[1], (int16_t)p.S[b], (int16_t)p.lp_off[b], 0});
      terms[b].push_back({(int16_t)gr.sm_off, gr.sst[1], gr.sst[0], (int16_t)p.S[a], (int16_t)p.lp_off[a], 0});
    } else if (gr.rank == 3) {
      const int a = gr.dep[0], b = gr.dep[1], c = gr.dep[2];
      const int i = r->n3++;
      r->g3[i] = (int16_t)g;
      r->xs[i] = (int16_t)odd(p.S[b]);
      r->ys[i] = (int16_t)odd(p.S[c]);
      r->x_off[i] = (int16_t)sm;
      sm += (int64_t)p.S[a] * r->xs[i];
      r->y_off[i] = (int16_t)sm;
      sm += (int64_t)p.S[a] * r->ys[i];
      if (sm > 32767) return false;
      r->item_begin[i] = items;
      items += p.S[a] * (p.S[b] + p.S[c]);
      terms[a].push_back({r->x_off[i], r->xs[i], 1, (int16_t)p.S[b], (int16_t)p.lp_off[b], 0});
      terms[b].push_back({r->x_off[i], 1, r->xs[i], (int16_t)p.S[a], (int16_t)p.lp_off[a], 0});
      terms[c].push_back({r->y_off[i], 1, r->ys[i], (int16_t)p.S[a], (int16_t)p.lp_off[a], 0});
    }
  }
  r->item_begin[r->n3] = items;
  r->n_items = items;
  int n = 0;
  for (int f = 0; f < p.F; ++f) {
    r->term_begin[f] = (int16_t)n;
    for (const FpiR3Term& t : terms[f]) {
      if (n >= kR3MaxTerm) return false;
      r->term[n++] = t;
    }
  }
  r->term_begin[p.F] = (int16_t)n;
  for (int f = 0; f < p.F; ++f) {
    int lg = 5;  // 32 lanes per state, halved until every state has its lanes
    while (lg > 0 && (p.S[f] << lg) > 32) --lg;
    r->f_lg[f] = (int8_t)lg;
  }
  sm = (sm + 1) / 2 * 2;
  r->lp_sm = (int32_t)sm;
  sm += p.S_tot;
  r->q_sm = (int32_t)sm;
  sm += 2 * p.S_tot;
  r->row_sm = (int32_t)sm;
  sm += p.M;
  r->agent_words = (int32_t)((sm + 1) / 2 * 2);
  return (int64_t)r->agent_words * 8 <= kMaxSmemPerCta;
}

// One X or Y entry of a rank-3 group: a dot product of n shared-memory
// doubles at stride st from L (the group's block) with n consecutive q's.
struct R3Item {
  int32_t L, st, n, q, out;
};

__device__ __forceinline__ R3Item r3_item(const FpiParams& p, const FpiR3& r, int i) {
  int j = 0;
  while (i >= r.item_begin[j + 1]) ++j;
  const FpiGroup& gr = p.grp[r.g3[j]];
  const int Sa = p.S[gr.dep[0]], Sb = p.S[gr.dep[1]], Sc = p.S[gr.dep[2]];
  int li = i - r.item_begin[j];
  R3Item it;
  if (li < Sa * Sb) {  // X[a][b] = sum_c L[a][b][c] q_c[c]
    const int a = li / Sb, bb = li - a * Sb;
    it = {gr.sm_off + a * gr.sst[0] + bb * gr.sst[1], gr.sst[2], Sc, p.lp_off[gr.dep[2]], r.x_off[j] + a * r.xs[j] + bb};
  } else {  // Y[a][c] = sum_b L[a][b][c] q_b[b]
    li -= Sa * Sb;
    const int a = li / Sc, c = li - a * Sc;
    it = {gr.sm_off + a * gr.sst[0] + c * gr.sst[2], gr.sst[1], Sb, p.lp_off[gr.dep[1]], r.y_off[j] + a * r.ys[j] + c};
  }
  return it;
}

__device__ __forceinline__ double r3_dot(const double* __restrict__ L, int st, int n, const double* __restrict__ q) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int k = 0;
  for (; k + 4 <= n; k += 4) {
    a0 = fma(L[k * st], q[k], a0);
    a1 = fma(L[(k + 1) * st], q[k + 1], a1);
    a2 = fma(L[(k + 2) * st], q[k + 2], a2);
    a3 = fma(L[(k + 3) * st], q[k + 3], a3);
  }
  for (; k < n; ++k) a0 = fma(L[k * st], q[k], a0);
  return (a0 + a1) + (a2 + a3);
}

// Per-factor data of the message step, copied to shared memory once.
struct R3Factor {
  int32_t S, off, lg, t0, t1;
};

template <int TEAM, bool FUSED>
__global__ void __launch_bounds__(TEAM, TEAM >= 256 ? 2 : 4) fpi_r3_kernel(const __grid_constant__ FpiParams p,
                                                                         const __grid_constant__ FpiR3 r,
                                                                         const FpiIO io) {
  extern __shared__ double smem_d[];
  __shared__ uint32_t s_ok;
  __shared__ R3Factor s_fac[kMaxF];
  __shared__ FpiR3Term s_term[kR3MaxTerm];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  constexpr int kWarps = TEAM / 32;
  const int64_t b = blockIdx.x;
  if (b >= io.batch) return;  // uniform over the CTA (one agent per CTA)
  double* sm = smem_d;
  double* lpp = sm + r.lp_sm;
  double* qbuf = sm + r.q_sm;
  int64_t* rowoff = reinterpret_cast<int64_t*>(sm + r.row_sm);

  // ---- load phase: observations (one lane per modality; M <= 32) and the
  // prior are read side by side; an out-of-range observation adds nothing
  // (see fpi_kernel)
  if (wid == 0) {
    bool ok = false;
    if (lane < p.M) {
      int64_t ro = b * io.src_stride + p.src[lane].src_off;
      ok = true;
      if (FUSED) {
        const int o = io.obs[b * p.M + lane];
        ok = o >= 0 && o < p.src[lane].O;
        ro += (int64_t)(ok ? o : 0) * p.src[lane].K;
      }
      rowoff[lane] = ro;
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, ok);
    if (lane == 0) s_ok = bal;
  }
  for (int i = tid; i < p.S_tot; i += TEAM) {
    const float x = __ldg(io.prior + b * p.S_tot + i);
    lpp[i] = FUSED ? log_split(fmaxf(x, kMinVal)) : (double)x;
  }
  for (int f = wid; f < p.F; f += kWarps)  // q of the first sweep: softmax(log q = 0), uniform
    for (int s = lane; s < p.S[f]; s += 32) qbuf[p.lp_off[f] + s] = 1.0 / p.S[f];
  for (int f = tid; f < p.F; f += TEAM) s_fac[f] = {p.S[f], p.lp_off[f], r.f_lg[f], r.term_begin[f], r.term_begin[f + 1]};
  for (int i = tid; i < r.term_begin[p.F]; i += TEAM) s_term[i] = r.term[i];
  __syncthreads();
  const uint32_t obs_ok = s_ok;
  auto term_of = [&](float a) { return FUSED ? log_split(fmaxf(a, kMinVal)) : (double)a; };
  // shared-memory address of ll element k of a rank >= 2 group
  auto addr_of = [&](const FpiGroup& gr, int k) {
    int rem = k, addr = 0;
    for (int x = gr.rank - 1; x > 0; --x) {
      const int d = p.S[gr.dep[x]];
      const int qd = rem / d;
      addr += (rem - qd * d) * gr.sst[x];
      rem = qd;
    }
    return gr.sm_off + addr + rem * gr.sst[0];
  };
  // ll element k of group g into its padded block (rank >= 2) or the log prior (rank 1)
  auto put = [&](const FpiGroup& gr, int k, double v) {
    if (gr.rank == 1)
      lpp[p.lp_off[gr.dep[0]] + k] += v;  // one group per rank-1 tuple, one thread per state: no race
    else
      sm[addr_of(gr, k)] = v;
  };
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    if (r.vec4) {
      // two float4 columns per thread and up to four sources per batch of loads
      const int K4 = gr.K >> 2;
      const bool inner4 = gr.rank >= 2 && p.S[gr.dep[gr.rank - 1]] % 4 == 0;  // 4 columns share all outer digits
      for (int e0 = tid; e0 < K4; e0 += 2 * TEAM) {
        double v[2][4] = {{0.0, 0.0, 0.0, 0.0}, {0.0, 0.0, 0.0, 0.0}};
        for (int s0 = gr.src_begin; s0 < gr.src_end; s0 += 4) {
          float4 a[4][2];
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int si = s0 + j;
            const int m = si < gr.src_end ? p.src_order[si] : 0;
            const bool use = si < gr.src_end && ((obs_ok >> m) & 1u);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const int e4 = e0 + h * TEAM;
              a[j][h] = use && e4 < K4 ? __ldg(reinterpret_cast<const float4*>(io.src + rowoff[m]) + e4)
                                       : make_float4(1.f, 1.f, 1.f, 1.f);
            }
          }
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int si = s0 + j;
            if (si < gr.src_end && ((obs_ok >> p.src_order[si]) & 1u)) {
#pragma unroll
              for (int h = 0; h < 2; ++h) {
                v[h][0] += term_of(a[j][h].x);
                v[h][1] += term_of(a[j][h].y);
                v[h][2] += term_of(a[j][h].z);
                v[h][3] += term_of(a[j][h].w);
              }
            }
          }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int e4 = e0 + h * TEAM;
          if (e4 < K4) {
            if (inner4) {
              const int a0 = addr_of(gr, 4 * e4);
#pragma unroll
              for (int x = 0; x < 4; ++x) sm[a0 + x] = v[h][x];
            } else {
#pragma unroll
              for (int x = 0; x < 4; ++x) put(gr, 4 * e4 + x, v[h][x]);
            }
          }
        }
      }
    } else {
      for (int k = tid; k < gr.K; k += TEAM) {
        double v = 0.0;
        for (int si = gr.src_begin; si < gr.src_end; ++si) {
          const int m = p.src_order[si];
          if ((obs_ok >> m) & 1u) v += term_of(__ldg(io.src + rowoff[m] + k));
        }
        put(gr, k, v);
      }
    }
  }
  // this thread's first two X / Y entries, fixed for every sweep
  R3Item mine[2];
  int n_mine = 0;
#pragma unroll
  for (int c = 0; c < 2; ++c)
    if (tid + c * TEAM < r.n_items) {
      mine[c] = r3_item(p, r, tid + c * TEAM);
      n_mine = c + 1;
    }
  __syncthreads();

  // ---- sweeps (Jacobi: every factor uses the previous q)
  for (int it = 0; it < p.num_iter; ++it) {
    const double* q = qbuf + (it & 1) * p.S_tot;
    double* qn = qbuf + ((it + 1) & 1) * p.S_tot;
    // step 1: X and Y of every rank-3 group, one entry per thread
#pragma unroll
    for (int c = 0; c < 2; ++c)
      if (c < n_mine) sm[mine[c].out] = r3_dot(sm + mine[c].L, mine[c].st, mine[c].n, q + mine[c].q);
    for (int i = tid + 2 * TEAM; i < r.n_items; i += TEAM) {
      const R3Item e = r3_item(p, r, i);
      sm[e.out] = r3_dot(sm + e.L, e.st, e.n, q + e.q);
    }
    __syncthreads();
    // step 2: one warp per output factor: log q = log prior + its messages,
    // then the softmax (the posterior itself after the last sweep). S <= 32:
    // 2^lg lanes per state split each message sum; S > 32: every lane takes
    // states lane and lane + 32.
    for (int f = wid; f < p.F; f += kWarps) {
      const R3Factor fc = s_fac[f];
      const int S = fc.S, off = fc.off;
      double x0, x1 = 0.0;
      bool v0, v1 = false, w0;
      if (S <= 32) {
        const int G = 1 << fc.lg;
        const int s = lane >> fc.lg, j = lane & (G - 1);
        v0 = s < S;
        w0 = v0 && j == 0;  // the lane that writes state s
        double acc = 0.0;
        if (v0) {
          for (int ti = fc.t0; ti < fc.t1; ++ti) {
            const FpiR3Term tm = s_term[ti];
            const double* Ms = sm + tm.m_off + s * tm.rs;
            const double* qo = q + tm.q_off;
            double a0 = 0.0, a1 = 0.0;
            int k = j;
            for (; k + G < tm.n; k += 2 * G) {
              a0 = fma(Ms[k * tm.cs], qo[k], a0);
              a1 = fma(Ms[(k + G) * tm.cs], qo[k + G], a1);
            }
            if (k < tm.n) a0 = fma(Ms[k * tm.cs], qo[k], a0);
            acc += a0 + a1;
          }
        }
        for (int o = 1; o < G; o <<= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        x0 = v0 ? acc + lpp[off + s] : 0.0;
      } else {
        v0 = true;  // S > 32: lane < S always
        w0 = true;
        v1 = lane + 32 < S;
        x0 = lpp[off + lane];
        x1 = v1 ? lpp[off + lane + 32] : 0.0;
        for (int ti = fc.t0; ti < fc.t1; ++ti) {
          const FpiR3Term tm = s_term[ti];
          const double* M0 = sm + tm.m_off + lane * tm.rs;
          const double* M1 = M0 + 32 * tm.rs;
          const double* qo = q + tm.q_off;
          double a0 = 0.0, a1 = 0.0, c0 = 0.0, c1 = 0.0;
          int k = 0;
          for (; k + 2 <= tm.n; k += 2) {
            const double qa = qo[k], qb = qo[k + 1];
            a0 = fma(M0[k * tm.cs], qa, a0);
            a1 = fma(M0[(k + 1) * tm.cs], qb, a1);
            if (v1) {
              c0 = fma(M1[k * tm.cs], qa, c0);
              c1 = fma(M1[(k + 1) * tm.cs], qb, c1);
            }
          }
          if (k < tm.n) {
            a0 = fma(M0[k * tm.cs], qo[k], a0);
            if (v1) c0 = fma(M1[k * tm.cs], qo[k], c0);
          }
          x0 += a0 + a1;
          x1 += c0 + c1;
        }
      }
      // softmax: any shift near the maximum cancels, so the maximum is taken
      // in FP32; exponentials and their sum in FP64, the reciprocal as FP32
      // plus one Newton step
      float mf = fmaxf(v0 ? (float)x0 : -INFINITY, v1 ? (float)x1 : -INFINITY);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) mf = fmaxf(mf, __shfl_xor_sync(0xffffffffu, mf, o));
      const double mx = (double)mf;
      const double e0 = v0 ? exp(x0 - mx) : 0.0, e1 = v1 ? exp(x1 - mx) : 0.0;
      const double sum = warp_sum_d((w0 ? e0 : 0.0) + e1);
      double inv = (double)__frcp_rn((float)sum);
      inv = inv * fma(-sum, inv, 2.0);
      const int s_out = S <= 32 ? lane >> fc.lg : lane;
      if (it + 1 == p.num_iter) {
        float* out = io.q_out + b * p.S_tot + off;
        if (w0) out[s_out] = (float)(e0 * inv);
        if (v1) out[lane + 32] = (float)(e1 * inv);
      } else {
        if (w0) qn[off + s_out] = e0 * inv;
        if (v1) qn[off + lane + 32] = e1 * inv;
      }
    }
    __syncthreads();
  }
}

// ----------------------------------------- rank <= 2, blocks in registers
// The same models as the rank <= 2 path (every modality on at most two
// factors of at most 16 states), with each rank-2 group's 16 x 16 FP64 block
// held in registers across the sweeps: 16 lanes per block, lane i keeping row
// i and column i (32 doubles), so both of the block's mat-vecs are 16 FMAs per
// lane on broadcast q values and no block is re-read from shared memory.
// A sweep: (M) every block lane writes its row message L q_b and column
// message L^T q_a; barrier; (S) one lane per (factor, state) sums the messages
// into its factor with the log prior and the 16-lane softmax; barrier.
// APC agents per CTA, 32-lane aligned, so a warp never spans two agents.
constexpr int kRRMaxBlocks = 16;
constexpr int kRRMaxCon = 2 * kRRMaxBlocks;

struct FpiR2Reg {
  int32_t nb;     // rank-2 blocks per agent
  int32_t lanes;  // threads per agent: 16 * max(nb, F) rounded up to 32
  int32_t apc;    // agents per CTA
  int32_t vec4;   // 16-byte loads of the observed rows (two sources at most per group)
  int32_t stg_sm, lp_sm, q_sm, row_sm, agent_words;  // per agent: staging blocks | msg (reuses staging) | lp | q | rows
  int8_t blk_g[kRRMaxBlocks];                       // block -> group
  int8_t g_blk[kMaxM];                              // group -> block (-1: rank 1)
  int8_t con_n[kMaxF];                              // messages into factor f: (block, dir) pairs,
  int8_t con[kMaxF][kRRMaxCon];                     // 2 * block + dir (dir 0: rows -> dep 0, 1: columns -> dep 1)
};

bool build_r2reg(const FpiParams& p, FpiR2Reg* r) {
  std::memset(r, 0, sizeof(*r));
  for (int f = 0; f < p.F; ++f)
    if (p.S[f] > 16) return false;
  int nb = 0;
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    if (gr.rank > 2) return false;
    if (gr.rank == 1) {
      r->g_blk[g] = -1;
      continue;
    }
    if (nb >= kRRMaxBlocks) return false;
    r->g_blk[g] = (int8_t)nb;
    r->blk_g[nb] = (int8_t)g;
    const int a = gr.dep[0], b = gr.dep[1];
    r->con[a][r->con_n[a]++] = (int8_t)(2 * nb);
    r->con[b][r->con_n[b]++] = (int8_t)(2 * nb + 1);
    ++nb;
  }
  if (nb == 0) return false;
  r->nb = nb;
  const int need = 16 * (nb > p.F ? nb : p.F);
  r->lanes = (need + 31) / 32 * 32;
  r->apc = r->lanes <= 32 ? 8 : r->lanes <= 64 ? 4 : r->lanes <= 128 ? 2 : 1;
  r->stg_sm = 0;                                  // [nb][16][17] staging; later [nb][2][16] messages
  r->lp_sm = nb * 16 * 17;
  r->q_sm = r->lp_sm + 16 * p.F;
  r->row_sm = r->q_sm + 16 * p.F;
  r->agent_words = (r->row_sm + p.M + 1) / 2 * 2;
  return (int64_t)r->agent_words * 8 * r->apc <= 96 * 1024;
}

template <bool FUSED, int APC>
__global__ void __launch_bounds__(256) fpi_r2reg_kernel(const __grid_constant__ FpiParams p,
                                                        const __grid_constant__ FpiR2Reg r, const FpiIO io) {
  extern __shared__ __align__(16) double rr_smem[];  // 16-byte aligned: q rows are read as double2
  __shared__ uint32_t s_ok[APC];
  __shared__ int8_t s_con[kMaxF][kRRMaxCon];
  const int lanes = r.lanes;
  const int slot = threadIdx.x / lanes, t = threadIdx.x - slot * lanes;
  const int64_t b = (int64_t)blockIdx.x * APC + slot;
  const bool live = b < io.batch;  // a missing agent's lanes still join every barrier and shuffle
  double* sm = rr_smem + slot * r.agent_words;
  double* stg = sm + r.stg_sm;
  double* lp = sm + r.lp_sm;
  double* qs = sm + r.q_sm;
  int64_t* rowoff = reinterpret_cast<int64_t*>(sm + r.row_sm);

  // ---- load phase: observation rows (one lane per modality of the agent's
  // first warp, M <= 32; an out-of-range observation adds nothing, see
  // fpi_kernel), log prior and the uniform first q (zero past S_f), zeroed blocks
  if (t < 32) {
    bool ok = false;
    if (live && t < p.M) {
      int64_t ro = b * io.src_stride + p.src[t].src_off;
      ok = true;
      if (FUSED) {
        const int o = io.obs[b * p.M + t];
        ok = o >= 0 && o < p.src[t].O;
        ro += (int64_t)(ok ? o : 0) * p.src[t].K;
      }
      rowoff[t] = ro;
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, ok);
    if (t == 0) s_ok[slot] = bal;
  }
  for (int i = threadIdx.x; i < kMaxF * kRRMaxCon; i += blockDim.x) {
    const int f = i / kRRMaxCon, c = i - f * kRRMaxCon;
    s_con[f][c] = r.con[f][c];
  }
  for (int i = t; i < 16 * p.F; i += lanes) {
    const int f = i >> 4, s = i & 15;
    double v = 0.0, q0 = 0.0;
    if (s < p.S[f]) {
      if (live) {
        const float x = __ldg(io.prior + b * p.S_tot + p.lp_off[f] + s);
        v = FUSED ? log_split(fmaxf(x, kMinVal)) : (double)x;
      }
      q0 = 1.0 / p.S[f];
    }
    lp[i] = v;
    qs[i] = q0;
  }
  for (int i = t; i < r.nb * 16 * 17; i += lanes) stg[i] = 0.0;
  __syncthreads();
  const uint32_t obs_ok = s_ok[slot];
  // log-likelihoods: rank-2 groups into their zero-padded blocks, rank-1 groups
  // into the log prior (one group per rank-1 tuple, one thread per state: no race)
  if (live) {
    for (int g = 0; g < p.G; ++g) {
      const FpiGroup& gr = p.grp[g];
      const int blk = r.g_blk[g];
      const int S1 = gr.rank == 2 ? p.S[gr.dep[1]] : 1;
      for (int k0 = t; k0 < gr.K; k0 += 4 * lanes) {
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int si = gr.src_begin; si < gr.src_end; ++si) {
          const int m = p.src_order[si];
          if (!((obs_ok >> m) & 1u)) continue;
          float a[4];
#pragma unroll
          for (int x = 0; x < 4; ++x) {
            const int k = k0 + x * lanes;
            a[x] = k < gr.K ? __ldg(io.src + rowoff[m] + k) : 1.f;
          }
#pragma unroll
          for (int x = 0; x < 4; ++x) v[x] += FUSED ? log_split(fmaxf(a[x], kMinVal)) : (double)a[x];
        }
#pragma unroll
        for (int x = 0; x < 4; ++x) {
          const int k = k0 + x * lanes;
          if (k < gr.K) {
            if (blk < 0) {
              lp[16 * gr.dep[0] + k] += v[x];
            } else {
              const int i0 = k / S1, i1 = k - i0 * S1;
              stg[(blk * 16 + i0) * 17 + i1] = v[x];
            }
          }
        }
      }
    }
  }
  __syncthreads();
  // this lane's block row and column (lane t = 16 blk + i), in registers for every sweep
  const int blk = t >> 4, ri = t & 15;
  const bool has_blk = blk < r.nb;
  double row[16], col[16];
  int qa_off = 0, qb_off = 0;
  if (has_blk) {
    const FpiGroup& gr = p.grp[r.blk_g[blk]];
    qa_off = 16 * gr.dep[0];
    qb_off = 16 * gr.dep[1];
#pragma unroll
    for (int j = 0; j < 16; ++j) {
      row[j] = stg[(blk * 16 + ri) * 17 + j];
      col[j] = stg[(blk * 16 + j) * 17 + ri];
    }
  } else {
#pragma unroll
    for (int j = 0; j < 16; ++j) row[j] = col[j] = 0.0;
  }
  // this lane's (factor, state) for the softmax
  const int f = t >> 4, s = t & 15;
  const int Sf = f < p.F ? p.S[f] : 0;
  const bool vs = s < Sf;
  const int fcon = f < p.F ? r.con_n[f] : 0;
  const int fout = f < p.F ? p.lp_off[f] + s : 0;
  __syncthreads();  // the staging area now holds the messages [nb][2][16]
  double* msg = stg;

  // ---- sweeps (Jacobi: every factor uses the previous q)
  for (int it = 0; it < p.num_iter; ++it) {
    if (has_blk) {
      // q rows start at even doubles of a 16-byte aligned buffer: 16-byte loads
      const double2* qa = reinterpret_cast<const double2*>(qs + qa_off);
      const double2* qb = reinterpret_cast<const double2*>(qs + qb_off);
      double ra0 = 0.0, ra1 = 0.0, cb0 = 0.0, cb1 = 0.0;
#pragma unroll
      for (int j = 0; j < 16; j += 2) {
        const double2 vb = qb[j >> 1], va = qa[j >> 1];
        ra0 = fma(row[j], vb.x, ra0);
        ra1 = fma(row[j + 1], vb.y, ra1);
        cb0 = fma(col[j], va.x, cb0);
        cb1 = fma(col[j + 1], va.y, cb1);
      }
      msg[blk * 32 + ri] = ra0 + ra1;       // into dep 0, state ri
      msg[blk * 32 + 16 + ri] = cb0 + cb1;  // into dep 1, state ri
    }
    __syncthreads();
    double x = 0.0;
    if (vs) {
      x = lp[16 * f + s];
      for (int c = 0; c < fcon; ++c) x += msg[s_con[f][c] * 16 + s];
    }
    // 16-lane softmax: the maximum in FP32 (any shift near it cancels), the rest in FP64
    float mf = vs ? (float)x : -INFINITY;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) mf = fmaxf(mf, __shfl_xor_sync(0xffffffffu, mf, o));
    const double e = vs ? exp(x - (double)mf) : 0.0;
    double sum = e;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    double inv = (double)__frcp_rn((float)sum);
    inv = inv * fma(-sum, inv, 2.0);
    if (it + 1 == p.num_iter) {
      if (vs && live) io.q_out[b * p.S_tot + fout] = (float)(e * inv);
    } else if (vs) {
      qs[16 * f + s] = e * inv;
    }
    __syncthreads();
  }
}

template <bool FUSED, int APC>
int32_t launch_r2reg_t(const FpiParams& p, const FpiR2Reg& r, const FpiIO& io, cudaStream_t stream, const char* op) {
  const int64_t grid = (io.batch + APC - 1) / APC;
  if (grid > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
  const int bytes = APC * r.agent_words * 8;
  B2_TRY(ensure_smem_attr((const void*)fpi_r2reg_kernel<FUSED, APC>, bytes, op));
  fpi_r2reg_kernel<FUSED, APC><<<(unsigned)grid, APC * r.lanes, bytes, stream>>>(p, r, io);
  return check_launch(op);
}

template <bool FUSED>
int32_t launch_r2reg(const FpiParams& p, const FpiR2Reg& r, const FpiIO& io, cudaStream_t stream, const char* op) {
  switch (r.apc) {
    case 8: return launch_r2reg_t<FUSED, 8>(p, r, io, stream, op);
    case 4: return launch_r2reg_t<FUSED, 4>(p, r, io, stream, op);
    case 2: return launch_r2reg_t<FUSED, 2>(p, r, io, stream, op);
    default: return launch_r2reg_t<FUSED, 1>(p, r, io, stream, op);
  }
}

// ------------------------------------------------------------ adjoint
// Reverse pass of the fused-observation FPI for gradients of a loss on the
// posteriors with respect to the observed A rows and the prior. The reference
// differentiates its JAX scan (pymdp/ffi/_core.py:282-310 with_jax_grad over
// pymdp/algos.py:88-155); this is the hand-written unrolled adjoint of the
// same Jacobi sweeps, with every iterate recomputed and kept on chip:
//   q_i = softmax(logq_i), logq_{i+1} = lp + sum_(g,ax) M_(g,ax)(q_i),
//   M_(g,ax)(q)[s] = sum_{k: digit_ax(k) = s} ll_g[k] prod_{j != ax} q_{dep j}[digit_j(k)],
// output softmax(logq_n). Backward: softmax adjoint, then for i = n-1..0
// d lp += d logq_{i+1}, d ll_g[k] += c prod_{j != ax} q, d q_i += c ll_g[k]
// prod_{l != ax, j} q with c = d logq_{i+1}[dep ax][digit ax(k)], and the
// softmax adjoint for d logq_i. Finally d A[o_m, k] = d ll_g[k] / A (A >= eps)
// for every source m of group g, d prior = d lp / prior (prior >= eps). FP64
// throughout; one warp per agent; shared-memory double atomics for sums over k.
struct FpiBwd {
  int32_t ll_off[kMaxM + 1];  // group g's ll (and d ll) doubles inside the agent's smem block
  int32_t words;              // doubles per agent
};

__device__ __forceinline__ void softmax_bwd_warp(const double* __restrict__ q, const double* __restrict__ gq,
                                                 double* __restrict__ glogq, int n, int lane) {
  double dot = 0.0;
  for (int i = lane; i < n; i += 32) dot += q[i] * gq[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
  for (int i = lane; i < n; i += 32) glogq[i] = q[i] * (gq[i] - dot);
}

__global__ void __launch_bounds__(32)
    fpi_bwd_kernel(const __grid_constant__ FpiParams p, const __grid_constant__ FpiBwd bw, const FpiIO io,
                   const float* __restrict__ dq_out, float* __restrict__ dA, float* __restrict__ dprior) {
  extern __shared__ double smem_d[];
  const int lane = threadIdx.x;
  const int64_t b = blockIdx.x;
  if (b >= io.batch) return;
  const int F = p.F, St = p.S_tot, n = p.num_iter;
  double* ll = smem_d;                    // [sum_g K_g]
  double* dll = ll + bw.ll_off[p.G];      // [sum_g K_g]
  double* lp = dll + bw.ll_off[p.G];      // [St]
  double* dlp = lp + St;                  // [St]
  double* hist = dlp + St;                // [(n + 1) * St]: q_0 .. q_{n-1}, then softmax(logq_n)
  double* logq = hist + (n + 1) * St;     // [St]
  double* glogq = logq + St;              // [St]
  double* gq = glogq + St;                // [St]
  int64_t* rowoff = reinterpret_cast<int64_t*>(gq + St);  // [M]

  // out-of-range observation: that modality adds nothing and gets no gradient (see fpi_kernel)
  const uint32_t obs_ok = obs_valid_mask(p, io, b);
  for (int m = lane; m < p.M; m += 32) {
    int o = io.obs[b * p.M + m];
    o = (o < 0 || o >= p.src[m].O) ? 0 : o;
    rowoff[m] = b * io.src_stride + p.src[m].src_off + (int64_t)o * p.src[m].K;
  }
  for (int i = lane; i < St; i += 32) {
    lp[i] = log((double)fmaxf(__ldg(io.prior + b * St + i), kMinVal));
    dlp[i] = 0.0;
    logq[i] = 0.0;
  }
  __syncwarp();
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    for (int k = lane; k < gr.K; k += 32) {
      double v = 0.0;
      for (int si = gr.src_begin; si < gr.src_end; ++si) {
        const int m = p.src_order[si];
        if ((obs_ok >> m) & 1u) v += log((double)fmaxf(__ldg(io.src + rowoff[m] + k), kMinVal));
      }
      ll[bw.ll_off[g] + k] = v;
      dll[bw.ll_off[g] + k] = 0.0;
    }
  }
  __syncwarp();
  // forward with history
  for (int it = 0; it <= n; ++it) {
    for (int f = 0; f < F; ++f) softmax_warp(logq + p.lp_off[f], hist + it * St + p.lp_off[f], p.S[f], lane);
    __syncwarp();
    if (it == n) break;
    const double* q = hist + it * St;
    for (int i = lane; i < St; i += 32) logq[i] = lp[i];
    __syncwarp();
    for (int g = 0; g < p.G; ++g) {
      const FpiGroup& gr = p.grp[g];
      for (int k = lane; k < gr.K; k += 32) {
        int dig[kMaxRank];
        int rem = k;
        for (int x = gr.rank - 1; x >= 0; --x) {
          const int d = p.S[gr.dep[x]];
          const int qd = rem / d;
          dig[x] = rem - qd * d;
          rem = qd;
        }
        const double L = ll[bw.ll_off[g] + k];
        for (int ax = 0; ax < gr.rank; ++ax) {
          double other = L;
          for (int j = 0; j < gr.rank; ++j)
            if (j != ax) other *= q[p.lp_off[gr.dep[j]] + dig[j]];
          atomicAdd(&logq[p.lp_off[gr.dep[ax]] + dig[ax]], other);
        }
      }
    }
    __syncwarp();
  }
  // backward
  for (int i = lane; i < St; i += 32) gq[i] = (double)__ldg(dq_out + b * St + i);
  __syncwarp();
  for (int f = 0; f < F; ++f)
    softmax_bwd_warp(hist + n * St + p.lp_off[f], gq + p.lp_off[f], glogq + p.lp_off[f], p.S[f], lane);
  __syncwarp();
  for (int it = n - 1; it >= 0; --it) {
    const double* q = hist + it * St;
    for (int i = lane; i < St; i += 32) {
      dlp[i] += glogq[i];
      gq[i] = 0.0;
    }
    __syncwarp();
    for (int g = 0; g < p.G; ++g) {
      const FpiGroup& gr = p.grp[g];
      for (int k = lane; k < gr.K; k += 32) {
        int dig[kMaxRank];
        int rem = k;
        for (int x = gr.rank - 1; x >= 0; --x) {
          const int d = p.S[gr.dep[x]];
          const int qd = rem / d;
          dig[x] = rem - qd * d;
          rem = qd;
        }
        const double L = ll[bw.ll_off[g] + k];
        double dl = 0.0;
        for (int ax = 0; ax < gr.rank; ++ax) {
          const double c = glogq[p.lp_off[gr.dep[ax]] + dig[ax]];
          double prod = 1.0;
          for (int j = 0; j < gr.rank; ++j)
            if (j != ax) prod *= q[p.lp_off[gr.dep[j]] + dig[j]];
          dl += c * prod;
          for (int j = 0; j < gr.rank; ++j) {
            if (j == ax) continue;
            double pr = c * L;
            for (int l = 0; l < gr.rank; ++l)
              if (l != ax && l != j) pr *= q[p.lp_off[gr.dep[l]] + dig[l]];
            atomicAdd(&gq[p.lp_off[gr.dep[j]] + dig[j]], pr);
          }
        }
        dll[bw.ll_off[g] + k] += dl;  // one lane per k
      }
    }
    __syncwarp();
    for (int f = 0; f < F; ++f)
      softmax_bwd_warp(q + p.lp_off[f], gq + p.lp_off[f], glogq + p.lp_off[f], p.S[f], lane);
    __syncwarp();
  }
  // to the inputs
  for (int i = lane; i < St; i += 32) {
    const float pv = __ldg(io.prior + b * St + i);
    dprior[b * St + i] = pv >= kMinVal ? (float)(dlp[i] / (double)pv) : 0.f;
  }
  for (int g = 0; g < p.G; ++g) {
    const FpiGroup& gr = p.grp[g];
    for (int k = lane; k < gr.K; k += 32)
      for (int si = gr.src_begin; si < gr.src_end; ++si) {
        if (!((obs_ok >> p.src_order[si]) & 1u)) continue;
        const int64_t e = rowoff[p.src_order[si]] + k;
        const float a = __ldg(io.src + e);
        if (a >= kMinVal) atomicAdd(dA + e, (float)(dll[bw.ll_off[g] + k] / (double)a));
      }
  }
}

template <int TEAM, int APC, bool FUSED>
int32_t launch_one(const FpiParams& p, const FpiIO& io, cudaStream_t stream, const char* op) {
  const int bytes = APC * p.agent_words * 8;
  const int64_t grid = (io.batch + APC - 1) / APC;
  if (grid > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
  bool generic = false;
  for (int g = 0; g < p.G; ++g) generic |= p.grp[g].rank > 3;
  const void* k = generic ? (const void*)fpi_kernel<TEAM, APC, FUSED, true>
                          : (const void*)fpi_kernel<TEAM, APC, FUSED, false>;
  B2_TRY(ensure_smem_attr(k, bytes, op));
  if (generic)
    fpi_kernel<TEAM, APC, FUSED, true><<<(unsigned)grid, TEAM * APC, bytes, stream>>>(p, io);
  else
    fpi_kernel<TEAM, APC, FUSED, false><<<(unsigned)grid, TEAM * APC, bytes, stream>>>(p, io);
  return check_launch(op);
}

template <int TEAM, bool FUSED>
int32_t launch_r3(const FpiParams& p, const FpiR3& r, const FpiIO& io, cudaStream_t stream, const char* op) {
  const int bytes = r.agent_words * 8;
  B2_TRY(ensure_smem_attr((const void*)fpi_r3_kernel<TEAM, FUSED>, bytes, op));
  fpi_r3_kernel<TEAM, FUSED><<<(unsigned)io.batch, TEAM, bytes, stream>>>(p, r, io);
  return check_launch(op);
}

template <bool FUSED>
int32_t launch(const FpiParams& p, const FpiIO& io, cudaStream_t stream, const char* op) {
  if (io.batch <= 0) return B2_OK;
  FpiR2Reg rr;
  if (build_r2reg(p, &rr)) return launch_r2reg<FUSED>(p, rr, io, stream, op);
  FpiR2 r2;
  if (build_r2(p, &r2)) {
    bool v4 = (reinterpret_cast<uintptr_t>(io.src) % 16 == 0) && io.src_stride % 4 == 0;
    for (int m = 0; m < p.M; ++m) v4 = v4 && p.src[m].src_off % 4 == 0 && p.src[m].K % 4 == 0;
    for (int g = 0; g < p.G; ++g) v4 = v4 && p.grp[g].src_end - p.grp[g].src_begin <= 2;
    r2.vec4 = v4 ? 1 : 0;
    if (io.batch > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
    const int bytes = r2.agent_words * 8;
    B2_TRY(ensure_smem_attr((const void*)fpi_r2_kernel<FUSED>, bytes, op));
    fpi_r2_kernel<FUSED><<<(unsigned)io.batch, 32 * r2.warps, bytes, stream>>>(p, r2, io);
    return check_launch(op);
  }
  FpiR3 r3;
  if (build_r3(p, &r3)) {
    if (io.batch > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
    bool v4 = (reinterpret_cast<uintptr_t>(io.src) % 16 == 0) && io.src_stride % 4 == 0;
    for (int m = 0; m < p.M; ++m) v4 = v4 && p.src[m].src_off % 4 == 0 && p.src[m].K % 4 == 0;
    r3.vec4 = v4 ? 1 : 0;
    // threads: about two X / Y entries per thread and sweep
    if (r3.n_items > 512) return launch_r3<512, FUSED>(p, r3, io, stream, op);
    if (r3.n_items > 256) return launch_r3<256, FUSED>(p, r3, io, stream, op);
    return launch_r3<128, FUSED>(p, r3, io, stream, op);
  }
  const int64_t work = work_per_iter(p);
  const int bytes_agent = p.agent_words * 8;
  if (work >= 8192) return launch_one<256, 1, FUSED>(p, io, stream, op);
  if (work >= 4096 || bytes_agent > 48 * 1024) return launch_one<128, 1, FUSED>(p, io, stream, op);
  int apc = 8;
  while (apc > 1 && (apc * bytes_agent > 64 * 1024 || apc / 2 >= io.batch)) apc >>= 1;
  switch (apc) {
    case 8: return launch_one<32, 8, FUSED>(p, io, stream, op);
    case 4: return launch_one<32, 4, FUSED>(p, io, stream, op);
    case 2: return launch_one<32, 2, FUSED>(p, io, stream, op);
    default: return launch_one<32, 1, FUSED>(p, io, stream, op);
  }
}

}  // namespace
}  // namespace b2

using namespace b2;

extern "C" int32_t b2_fpi(void* stream, const float* ll_flat, int64_t ll_count, const float* lp_flat,
                          int64_t lp_count, float* q_out, int64_t q_count, const int64_t* S, int64_t S_len,
                          const int64_t* ll_offsets, int64_t ll_offsets_len, const int64_t* lp_offsets,
                          int64_t lp_offsets_len, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                          const int64_t* A_dep_offsets, int64_t A_dep_offsets_len, int32_t num_iter) {
  const char* op = kName;
  if (!S || !ll_offsets || !lp_offsets || !A_dep_flat || !A_dep_offsets)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute array");
  const int64_t M = A_dep_offsets_len - 1;
  if (ll_offsets_len != M + 1)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets size = " +
                                             std::to_string(ll_offsets_len) + ", expected " +
                                             std::to_string(M + 1));
  FpiParams p;
  std::vector<int64_t> K;
  B2_TRY(build_params(&p, &K, S, S_len, lp_offsets, lp_offsets_len, A_dep_flat, A_dep_flat_len, A_dep_offsets,
                      A_dep_offsets_len, num_iter, op));
  if (ll_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets must start at zero");
  for (int64_t m = 0; m < M; ++m) {
    if (ll_offsets[m + 1] < ll_offsets[m])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets must be monotonic");
    if (ll_offsets[m + 1] - ll_offsets[m] != K[m])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets inconsistent with S/A_dep for modality " +
                                               std::to_string(m));
    p.src[m].src_off = ll_offsets[m];
  }
  const int64_t total_S = p.S_tot, total_ll = ll_offsets[M];
  if (lp_count <= 0 || lp_count % total_S != 0)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": lp_flat size = " + std::to_string(lp_count) +
                                             " not divisible by total_S = " + std::to_string(total_S));
  const int64_t batch = lp_count / total_S;
  if (ll_count != batch * total_ll)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_flat element_count = " +
                                             std::to_string(ll_count) + ", expected " +
                                             std::to_string(batch * total_ll));
  if (q_count != batch * total_S)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": q_out element_count = " +
                                             std::to_string(q_count) + ", expected " +
                                             std::to_string(batch * total_S));
  if (!ll_flat || !lp_flat || !q_out) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  FpiIO io{ll_flat, total_ll, nullptr, lp_flat, q_out, batch};
  return launch<false>(p, io, (cudaStream_t)stream, op);
}

extern "C" int32_t b2_fpi_obs(void* stream, const float* A_flat, int64_t A_agent_stride,
                              const int64_t* A_offsets, int64_t A_offsets_len, const int64_t* O, int64_t O_len,
                              const int32_t* obs, const float* prior, float* q_out, int64_t batch,
                              const int64_t* S, int64_t S_len, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                              const int64_t* A_dep_offsets, int64_t A_dep_offsets_len, int32_t num_iter) {
  const char* op = "fpi_obs";
  if (!S || !A_offsets || !O || !A_dep_flat || !A_dep_offsets)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute array");
  const int64_t M = A_dep_offsets_len - 1;
  if (O_len != M || A_offsets_len != M + 1)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": O / A_offsets sizes inconsistent with M = " +
                                             std::to_string(M));
  FpiParams p;
  std::vector<int64_t> K;
  B2_TRY(build_params(&p, &K, S, S_len, nullptr, 0, A_dep_flat, A_dep_flat_len, A_dep_offsets, A_dep_offsets_len,
                      num_iter, op));
  if (A_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets must start at zero");
  for (int64_t m = 0; m < M; ++m) {
    if (O[m] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": " + idx("O", m) + " must be positive");
    if (A_offsets[m + 1] - A_offsets[m] != O[m] * K[m])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets inconsistent with O/deps for modality " +
                                               std::to_string(m));
    p.src[m].src_off = A_offsets[m];
    p.src[m].O = (int32_t)O[m];
  }
  if (batch < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": negative batch");
  if (A_agent_stride != 0 && A_agent_stride < A_offsets[M])
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_agent_stride smaller than one agent's A");
  if (batch > 0 && (!A_flat || !obs || !prior || !q_out))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  FpiIO io{A_flat, A_agent_stride, obs, prior, q_out, batch};
  return launch<true>(p, io, (cudaStream_t)stream, op);
}

extern "C" int32_t b2_fpi_obs_bwd(void* stream, const float* A_flat, int64_t A_agent_stride,
                                  const int64_t* A_offsets, int64_t A_offsets_len, const int64_t* O, int64_t O_len,
                                  const int32_t* obs, const float* prior, const float* d_q, float* d_A,
                                  float* d_prior, int64_t batch, const int64_t* S, int64_t S_len,
                                  const int64_t* A_dep_flat, int64_t A_dep_flat_len, const int64_t* A_dep_offsets,
                                  int64_t A_dep_offsets_len, int32_t num_iter) {
  const char* op = "fpi_obs bwd";
  if (!S || !A_offsets || !O || !A_dep_flat || !A_dep_offsets)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null attribute array");
  const int64_t M = A_dep_offsets_len - 1;
  if (O_len != M || A_offsets_len != M + 1)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": O / A_offsets sizes inconsistent with M = " +
                                             std::to_string(M));
  FpiParams p;
  std::vector<int64_t> K;
  B2_TRY(build_params(&p, &K, S, S_len, nullptr, 0, A_dep_flat, A_dep_flat_len, A_dep_offsets, A_dep_offsets_len,
                      num_iter, op));
  if (A_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets must start at zero");
  for (int64_t m = 0; m < M; ++m) {
    if (O[m] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": " + idx("O", m) + " must be positive");
    if (A_offsets[m + 1] - A_offsets[m] != O[m] * K[m])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets inconsistent with O/deps for modality " +
                                               std::to_string(m));
    p.src[m].src_off = A_offsets[m];
    p.src[m].O = (int32_t)O[m];
  }
  if (batch < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": negative batch");
  if (A_agent_stride != 0 && A_agent_stride < A_offsets[M])
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_agent_stride smaller than one agent's A");
  FpiBwd bw;
  std::memset(&bw, 0, sizeof(bw));
  int64_t off = 0;
  for (int g = 0; g < p.G; ++g) {
    bw.ll_off[g] = (int32_t)off;
    off += p.grp[g].K;
  }
  bw.ll_off[p.G] = (int32_t)off;
  const int64_t words = 2 * off + 2LL * p.S_tot + (int64_t)(num_iter + 1) * p.S_tot + 3LL * p.S_tot + M;
  if (words * 8 > kMaxSmemPerCta)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": per-agent working set of " + std::to_string(words * 8) +
                                        " bytes exceeds shared memory");
  bw.words = (int32_t)words;
  if (batch == 0) return B2_OK;
  if (!A_flat || !obs || !prior || !d_q || !d_A || !d_prior)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  if (batch > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
  const int64_t a_words = A_agent_stride == 0 ? A_offsets[M] : batch * A_agent_stride;
  B2_CUDA_TRY(op, cudaMemsetAsync(d_A, 0, (size_t)a_words * sizeof(float), (cudaStream_t)stream));
  FpiIO io{A_flat, A_agent_stride, obs, prior, nullptr, batch};
  const int bytes = (int)words * 8;
  B2_TRY(ensure_smem_attr((const void*)fpi_bwd_kernel, bytes, op));
  fpi_bwd_kernel<<<(unsigned)batch, 32, bytes, (cudaStream_t)stream>>>(p, bw, io, d_q, d_A, d_prior);
  return check_launch(op);
}
