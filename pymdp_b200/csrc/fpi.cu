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
// Design (one warp = one agent, several agents per CTA):
//  * Load phase: each modality's log-likelihood block is read once from HBM
//    with coalesced loads and written into shared memory in a padded layout
//    whose non-innermost strides are odd, so a sweep along ANY axis by the
//    lanes of a warp is bank-conflict free. In the fused observation form the
//    loaded values are the observed slice A_m[o_m] (K contiguous floats) and
//    log(clip(., eps)) is applied on the fly — ll never exists in HBM.
//  * Precision: FP32 inputs and outputs; on-chip values are FP64. The
//    products of two FP32 numbers are exact in FP64, so the marginal dot
//    products and the per-factor sums carry FP64 accumulation error only
//    (FP32 accumulation misses the 1e-5-relative posterior target vs the FP64
//    reference on ill-conditioned Dirichlet(0.5) models; FP64 accumulation
//    stays near 1e-6). B200 runs DFMA at half the FP32 FMA rate.
//  * Iterations run entirely on-chip: phase A = warp-shuffle softmax per
//    factor, phase B = one output state per lane group (group size = 32/S_f
//    rounded down to a power of two), each group summing the contributions of
//    every (modality, axis) pair that touches the factor, then a butterfly
//    reduction inside the group. No atomics: results are deterministic.
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
constexpr int kMaxSmemPerCta = 227 * 1024;

struct FpiModality {
  int32_t sm_off;  // double offset of the padded ll block inside the agent's smem
  int32_t K;       // prod_i S[dep[i]]
  int32_t rank;
  int32_t O;        // observation count (fused form only)
  int64_t src_off;  // ll form: ll_offsets[m]; fused form: A_offsets[m]
  int8_t dep[kMaxRank];
  int32_t sst[kMaxRank];  // padded shared-memory stride of each axis
};

struct FpiParams {
  int32_t F, M, num_iter, S_tot;
  int32_t agent_words;  // shared-memory doubles per agent
  int32_t ll_sm_total;  // doubles of padded ll blocks
  int32_t S[kMaxF];
  int32_t lp_off[kMaxF + 1];
  int32_t contrib_off[kMaxF + 1];
  int16_t contrib[kMaxM * kMaxRank];  // m * 8 + axis, grouped by factor
  FpiModality mod[kMaxM];
};

struct FpiIO {
  const float* src;    // ll_flat (ll form) or A_flat (fused form)
  int64_t src_stride;  // per-agent stride of src in floats
  const int32_t* obs;  // [batch, M] (fused form)
  const float* prior;  // [batch, S_tot]: log priors (ll form) or priors (fused form)
  float* q_out;        // [batch, S_tot]
  int64_t batch;
};

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Softmax of n values of `in` into `out` by one warp (FP64 on-chip).
template <typename OutT>
__device__ __forceinline__ void softmax_warp(const double* in, OutT* out, int n, int lane) {
  double mx = -INFINITY;
  for (int i = lane; i < n; i += 32) mx = fmax(mx, in[i]);
  mx = warp_max_d(mx);
  double sum = 0.0;
  for (int i = lane; i < n; i += 32) sum += exp(in[i] - mx);
  sum = warp_sum_d(sum);
  for (int i = lane; i < n; i += 32) out[i] = (OutT)(exp(in[i] - mx) / sum);
}

// Contribution of modality `md` to output state `s` of its axis `ax`, summed
// over the flattened "other" indices t = j, j+G, ... of this lane.
__device__ __forceinline__ double contract(const FpiModality& md, const FpiParams& p,
                                           const double* __restrict__ ll, const double* __restrict__ q,
                                           int ax, int s, int j, int G) {
  const double* L = ll + md.sm_off + s * md.sst[ax];
  if (md.rank == 1) return j == 0 ? L[0] : 0.0;
  if (md.rank == 2) {
    const int o = 1 - ax;
    const int d = p.S[md.dep[o]];
    const int st = md.sst[o];
    const double* qo = q + p.lp_off[md.dep[o]];
    double acc = 0.0;
    for (int t = j; t < d; t += G) acc = fma(L[t * st], qo[t], acc);
    return acc;
  }
  if (md.rank == 3) {
    const int a0 = ax == 0 ? 1 : 0;
    const int a1 = ax == 2 ? 1 : 2;
    const int d0 = p.S[md.dep[a0]], d1 = p.S[md.dep[a1]];
    const int st0 = md.sst[a0], st1 = md.sst[a1];
    const double* q0 = q + p.lp_off[md.dep[a0]];
    const double* q1 = q + p.lp_off[md.dep[a1]];
    const int total = d0 * d1;
    int i0 = j / d1, i1 = j - (j / d1) * d1;
    double acc = 0.0;
    for (int t = j; t < total; t += G) {
      acc = fma(L[i0 * st0 + i1 * st1], q0[i0] * q1[i1], acc);
      i1 += G;
      while (i1 >= d1) { i1 -= d1; ++i0; }
    }
    return acc;
  }
  // rank 4..8: mixed-radix counter over the other axes (innermost last).
  int dd[kMaxRank - 1], st[kMaxRank - 1], qoff[kMaxRank - 1], dig[kMaxRank - 1];
  int n = 0, total = 1;
  for (int x = 0; x < md.rank; ++x) {
    if (x == ax) continue;
    dd[n] = p.S[md.dep[x]];
    st[n] = md.sst[x];
    qoff[n] = p.lp_off[md.dep[x]];
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

template <int APC, bool FUSED>
__global__ void __launch_bounds__(32 * APC)
    fpi_warp_kernel(const __grid_constant__ FpiParams p, const FpiIO io) {
  extern __shared__ double smem_d[];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int64_t b = (int64_t)blockIdx.x * APC + warp;
  if (b >= io.batch) return;  // whole warp leaves; only warp-level syncs below
  double* ll = smem_d + warp * p.agent_words;
  double* lp = ll + p.ll_sm_total;
  double* logq = lp + p.S_tot;
  double* q = logq + p.S_tot;

  // ---- load phase: ll blocks (fused: observed log-A slices) and log prior
  bool bad_obs = false;
  for (int m = 0; m < p.M; ++m) {
    const FpiModality& md = p.mod[m];
    const float* src = io.src + b * io.src_stride + md.src_off;
    if (FUSED) {
      int o = io.obs[b * p.M + m];
      if (o < 0 || o >= md.O) {
        bad_obs = true;
        o = 0;
      }
      src += (int64_t)o * md.K;
    }
    for (int k = lane; k < md.K; k += 32) {
      double v = (double)__ldg(src + k);
      if (FUSED) v = log(fmax(v, (double)kMinVal));
      int rem = k, addr = 0;
      for (int x = md.rank - 1; x > 0; --x) {
        const int d = p.S[md.dep[x]];
        const int qd = rem / d;
        addr += (rem - qd * d) * md.sst[x];
        rem = qd;
      }
      addr += rem * md.sst[0];
      ll[md.sm_off + addr] = v;
    }
  }
  for (int i = lane; i < p.S_tot; i += 32) {
    const double v = (double)__ldg(io.prior + b * p.S_tot + i);
    lp[i] = FUSED ? log(fmax(v, (double)kMinVal)) : v;
    logq[i] = 0.0;
  }
  __syncwarp();

  // ---- fixed-point iterations (Jacobi: every factor uses the previous q)
  for (int it = 0; it < p.num_iter; ++it) {
    for (int f = 0; f < p.F; ++f) softmax_warp(logq + p.lp_off[f], q + p.lp_off[f], p.S[f], lane);
    __syncwarp();
    for (int f = 0; f < p.F; ++f) {
      const int Sf = p.S[f];
      const int per = Sf >= 32 ? 1 : 32 / Sf;
      const int G = 1 << (31 - __clz(per));  // lanes per output, power of two
      const int groups = 32 / G;
      const int c0 = p.contrib_off[f], c1 = p.contrib_off[f + 1];
      for (int s0 = 0; s0 < Sf; s0 += groups) {
        const int s = s0 + lane / G;
        const int j = lane & (G - 1);
        double acc = 0.0;
        if (s < Sf) {
          for (int c = c0; c < c1; ++c) {
            const int m = p.contrib[c] >> 3, ax = p.contrib[c] & 7;
            acc += contract(p.mod[m], p, ll, q, ax, s, j, G);
          }
        }
        for (int o = G >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (s < Sf && j == 0) logq[p.lp_off[f] + s] = acc + lp[p.lp_off[f] + s];
      }
    }
    __syncwarp();
  }

  // ---- posterior marginals
  float* out = io.q_out + b * p.S_tot;
  for (int f = 0; f < p.F; ++f) softmax_warp(logq + p.lp_off[f], out + p.lp_off[f], p.S[f], lane);
  if (FUSED && bad_obs) {
    __syncwarp();
    for (int i = lane; i < p.S_tot; i += 32) out[i] = __int_as_float(0x7fc00000);
  }
}

// --------------------------------------------------------------- host side
const char* const kName = "fpi_ffi";

std::string idx(const char* name, int64_t i) { return std::string(name) + "[" + std::to_string(i) + "]"; }

// Build kernel parameters from the reference's attribute set. Mirrors
// validate_fpi_attrs / build_modality_dispatch / check_distinct_modality_factor
// (pymdp/ffi/fpi/fpi_entry.h:24-82, fpi/fpi_precompute.h:56-112) and in
// addition checks that offsets are the prefix sums the layout implies.
int32_t build_params(FpiParams* p, const int64_t* S, int64_t F, const int64_t* lp_offsets,
                     int64_t lp_offsets_len, const int64_t* A_dep_flat, int64_t A_dep_flat_len,
                     const int64_t* A_dep_offsets, int64_t A_dep_offsets_len, int32_t num_iter,
                     const char* op) {
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
    if (off > 32767) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": total_S exceeds 32767");
  }
  if (lp_offsets && lp_offsets[F] != off)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": lp_offsets must be the prefix sums of S");
  p->lp_off[F] = (int32_t)off;
  p->S_tot = (int32_t)off;
  if (A_dep_offsets[0] != 0)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_dep_offsets must start at zero");
  std::vector<std::vector<int>> contrib(F);
  int64_t sm = 0;
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
    FpiModality& md = p->mod[m];
    md.rank = (int32_t)rank;
    int64_t K = 1;
    for (int64_t i = 0; i < rank; ++i) {
      const int64_t d = A_dep_flat[A_dep_offsets[m] + i];
      if (d < 0 || d >= F)
        return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": modality " + std::to_string(m) +
                                                 " A_dep factor " + std::to_string(d) + " out of range");
      for (int64_t i2 = 0; i2 < i; ++i2)
        if (md.dep[i2] == d)
          return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": modality " + std::to_string(m) +
                                                   " has duplicate factor in A_dependencies");
      md.dep[i] = (int8_t)d;
      K *= S[d];
      contrib[d].push_back((int)(m * 8 + i));
    }
    if (K > (1 << 24)) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": modality too large");
    md.K = (int32_t)K;
    // padded strides: innermost 1, every other stride odd
    int64_t st = 1;
    for (int64_t x = rank - 1; x >= 0; --x) {
      md.sst[x] = (int32_t)st;
      st = st * S[md.dep[x]];
      if (x > 0 && (st % 2) == 0) st += 1;
    }
    const int64_t footprint = (int64_t)md.sst[0] * S[md.dep[0]];
    md.sm_off = (int32_t)sm;
    sm += (footprint + 1) / 2 * 2;  // 16-byte aligned blocks
  }
  int n = 0;
  for (int64_t f = 0; f < F; ++f) {
    p->contrib_off[f] = n;
    for (int c : contrib[f]) p->contrib[n++] = (int16_t)c;
  }
  p->contrib_off[F] = n;
  p->ll_sm_total = (int32_t)sm;
  const int64_t agent = sm + 3 * off;
  p->agent_words = (int32_t)((agent + 1) / 2 * 2);
  if ((int64_t)p->agent_words * 8 > kMaxSmemPerCta)
    return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": per-agent working set of " +
                                        std::to_string((int64_t)p->agent_words * 8) +
                                        " bytes exceeds shared memory (227 KB)");
  return B2_OK;
}

template <bool FUSED>
int32_t launch(const FpiParams& p, const FpiIO& io, cudaStream_t stream, const char* op) {
  if (io.batch <= 0) return B2_OK;
  const int bytes_agent = p.agent_words * 8;
  int apc = 8;
  while (apc > 1 && (apc * bytes_agent > 64 * 1024 || apc / 2 >= io.batch)) apc >>= 1;
  const int bytes = apc * bytes_agent;
  const int64_t grid = (io.batch + apc - 1) / apc;
  if (grid > 0x7fffffff) return fail(B2_ERR_UNSUPPORTED, std::string(op) + ": batch too large");
  const void* k = nullptr;
  switch (apc) {
    case 8: k = (const void*)fpi_warp_kernel<8, FUSED>; break;
    case 4: k = (const void*)fpi_warp_kernel<4, FUSED>; break;
    case 2: k = (const void*)fpi_warp_kernel<2, FUSED>; break;
    default: k = (const void*)fpi_warp_kernel<1, FUSED>; break;
  }
  B2_TRY(ensure_smem_attr(k, bytes, op));
  switch (apc) {
    case 8: fpi_warp_kernel<8, FUSED><<<(unsigned)grid, 256, bytes, stream>>>(p, io); break;
    case 4: fpi_warp_kernel<4, FUSED><<<(unsigned)grid, 128, bytes, stream>>>(p, io); break;
    case 2: fpi_warp_kernel<2, FUSED><<<(unsigned)grid, 64, bytes, stream>>>(p, io); break;
    default: fpi_warp_kernel<1, FUSED><<<(unsigned)grid, 32, bytes, stream>>>(p, io); break;
  }
  return check_launch(op);
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
  B2_TRY(build_params(&p, S, S_len, lp_offsets, lp_offsets_len, A_dep_flat, A_dep_flat_len, A_dep_offsets,
                      A_dep_offsets_len, num_iter, op));
  if (ll_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets must start at zero");
  for (int64_t m = 0; m < M; ++m) {
    if (ll_offsets[m + 1] < ll_offsets[m])
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets must be monotonic");
    if (ll_offsets[m + 1] - ll_offsets[m] != p.mod[m].K)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": ll_offsets inconsistent with S/A_dep for modality " +
                                               std::to_string(m));
    p.mod[m].src_off = ll_offsets[m];
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
  B2_TRY(build_params(&p, S, S_len, nullptr, 0, A_dep_flat, A_dep_flat_len, A_dep_offsets, A_dep_offsets_len,
                      num_iter, op));
  if (A_offsets[0] != 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets must start at zero");
  for (int64_t m = 0; m < M; ++m) {
    if (O[m] <= 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": " + idx("O", m) + " must be positive");
    if (A_offsets[m + 1] - A_offsets[m] != O[m] * p.mod[m].K)
      return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_offsets inconsistent with O/deps for modality " +
                                               std::to_string(m));
    p.mod[m].src_off = A_offsets[m];
    p.mod[m].O = (int32_t)O[m];
  }
  if (batch < 0) return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": negative batch");
  if (A_agent_stride != 0 && A_agent_stride < A_offsets[M])
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": A_agent_stride smaller than one agent's A");
  if (batch > 0 && (!A_flat || !obs || !prior || !q_out))
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(op) + ": null buffer");
  FpiIO io{A_flat, A_agent_stride, obs, prior, q_out, batch};
  return launch<true>(p, io, (cudaStream_t)stream, op);
}
