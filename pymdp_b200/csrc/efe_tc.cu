// Dense tensor-core neg-EFE for sm_100a (tcgen05 + TMEM).
//
// For every agent, every step t and every group of modalities sharing one
// dependency tuple, the expected observations of ALL policies are one GEMM:
//   D[p, n] = sum_k X[p, k] * W[n, k]
//   X[p, k] = prod_{f in deps} qs_f^{(p,t)}[digit_f(k)]   (Kronecker of the
//             policy's predicted factor marginals, generated on chip)
//   W[n, :] = A_m[o, :]            for the obs rows n = (m, o) of the group
//           = lin_t                for the T linear rows (one per step)
//           = 0                    padding up to N (multiple of 16)
// with lin_t[k] = sum_m sum_o A_m[o,k] (log clip A_m[o,k] [info gain] +
// C_m[t,o] [utility]), the reference's own linear-term collapse
// (pymdp/ffi/neg_efe/neg_efe_cuda_kernels.cu:1426-1445). Then
//   G_p += sum_{obs rows n} -D[p,n] log clip D[p,n]  +  D[p, n_obs + t]
// which is compute_info_gain + compute_expected_utility
// (pymdp/control.py:449-509) summed over modalities.
//
// Mapping: one CTA = (agent, tile of 128 policies); M = 128 policies (TMEM
// lanes), N = rows of the group, K = joint states in 128-byte chunks.
//  * 256 threads generate the A operand (X, K-major, 128-byte swizzle) into
//    shared memory; each policy row is written by two threads (half a chunk
//    each). K is ordered with one factor innermost, padded to a power of two,
//    so a half chunk is a few runs of prefix * q_inner[0..DLP) with q_inner
//    in registers.
//  * W is packed once per call into ready-made shared-memory images (one per
//    128-byte K chunk, already swizzled) and each chunk arrives with ONE
//    cp.async.bulk (no multicast) on a transaction-count mbarrier.
//  * Stages are triple-buffered: a "full" mbarrier per stage (W landed) and
//    a "done" mbarrier per stage, armed by tcgen05.commit (MMAs reading the
//    stage finished).
//  * Thread 0 issues the UMMAs (kind::f16 BF16 operands, or kind::tf32 with
//    the 3xTF32 hi/lo split for FP32-level accuracy), accumulating in TMEM.
//  * Epilogue: warps 0-3 read their 32 TMEM lanes (= policies) with
//    tcgen05.ld, form the entropy of the obs rows and add the step's linear
//    row, accumulating G in FP64 registers.
// Every mbarrier wait is bounded; on timeout the CTA records an error in
// g_b2_device_error, stops issuing work, frees its TMEM and exits.
#include <cuda_bf16.h>

#include <cstring>
#include <string>
#include <vector>

#include "common.cuh"
#include "efe.cuh"
#include "tc.cuh"

namespace b2 {

__device__ int g_b2_device_error = 0;

namespace {

constexpr int kTcMaxGroups = 8;
constexpr int kTcThreads = 256;
constexpr int kTcTile = 128;
constexpr int kTcStages = 3;
constexpr uint32_t kWaitLimit = 1u << 22;

struct TcGroup {
  int64_t pack_off;  // per-agent byte offset of this group's W image
  int32_t K;         // prod of the dependency sizes
  int32_t outer;     // K / dim[rank-1]
  int32_t Kpad;      // padded K (innermost size rounded to a power of two, then to the chunk)
  int32_t nch;       // Kpad / chunk
  int32_t N, n_obs;  // rows: [0, n_obs) observations, then one linear row per step, then zeros
  int32_t rank, m_begin, m_end;
  int32_t lg;           // log2 of the padded innermost size
  int32_t chunk_bytes;  // bytes of one chunk image (all planes)
  uint32_t idesc;
  int8_t dep[B2_MAX_DEP_RANK];   // factor order used for K (innermost last)
  int8_t axis[B2_MAX_DEP_RANK];  // position of that factor in the modalities' A axes
  int16_t dim[B2_MAX_DEP_RANK];
};

struct TcParams {
  int32_t G, Nmax;
  int32_t nacc;       // TMEM accumulators the K chunks rotate over (summed in FP64)
  int32_t tmem_cols;  // allocated TMEM columns (power of two >= nacc * Nmax)
  int64_t pack_stride;  // bytes of W images per agent
  int8_t mod_order[B2_MAX_MODALITIES];
  TcGroup grp[kTcMaxGroups];
};

template <int PREC>
struct TcTraits;
template <>
struct TcTraits<B2_PRECISION_BF16> {
  static constexpr int kChunk = 64;  // K elements per 128-byte row
  static constexpr int kPlanes = 1;
  static constexpr int kEsz = 2;
};
template <>
struct TcTraits<B2_PRECISION_TF32X3> {
  static constexpr int kChunk = 32;
  static constexpr int kPlanes = 2;  // hi, lo
  static constexpr int kEsz = 4;
};

__device__ __forceinline__ uint16_t bf16_bits(float x) {
  __nv_bfloat16 h = __float2bfloat16_rn(x);
  return *reinterpret_cast<uint16_t*>(&h);
}

__device__ __forceinline__ uint32_t bf16x2_bits(float lo, float hi) {
  __nv_bfloat162 h = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<uint32_t*>(&h);
}

// Round-to-nearest TF32 (10 explicit mantissa bits) kept in an fp32 pattern.
__device__ __forceinline__ float tf32_round(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

__device__ __forceinline__ void bulk_g2s(uint32_t dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(tc::smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%1], %0;" ::"r"(bytes), "r"(tc::smem_u32(bar))
               : "memory");
}

// ---------------------------------------------------------- W packing
// Writes, per agent and group, the W operand as ready-to-copy shared-memory
// images: chunk c is planes x N rows x 128 bytes in the 128-byte-swizzled
// K-major layout, so the main kernel moves a whole chunk with one bulk copy.
// K is ordered with the group's chosen innermost factor last, its size padded
// to a power of two (padding columns are zero).
template <int PREC>
__global__ void efe_tc_pack_kernel(const __grid_constant__ EfeParams p, const __grid_constant__ TcParams tp,
                                   const float* __restrict__ A, const float* __restrict__ C, uint8_t* __restrict__ pack) {
  using Tr = TcTraits<PREC>;
  const int64_t b = blockIdx.z;
  const int g = blockIdx.y >> 8, n = blockIdx.y & 255;
  if (g >= tp.G) return;
  const TcGroup& gr = tp.grp[g];
  if (n >= gr.N) return;
  const int kp = blockIdx.x * blockDim.x + threadIdx.x;
  if (kp >= gr.Kpad) return;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const bool ut = (p.flags & B2_FLAG_USE_UTILITY) != 0;
  float v = 0.f;
  const int inner = kp & ((1 << gr.lg) - 1);
  int outer = kp >> gr.lg;
  if (inner < gr.dim[gr.rank - 1] && outer < gr.outer && n < gr.n_obs + p.T) {
    // original row-major index over the modalities' own axis order
    const EfeModality& m0 = p.mod[tp.mod_order[gr.m_begin]];
    int64_t stride[B2_MAX_DEP_RANK];
    int64_t st = 1;
    for (int a = gr.rank - 1; a >= 0; --a) {
      stride[a] = st;
      st *= p.S[m0.dep[a]];
    }
    int64_t k = (int64_t)inner * stride[gr.axis[gr.rank - 1]];
    for (int j = gr.rank - 2; j >= 0; --j) {
      const int d = gr.dim[j];
      const int qd = outer / d;
      k += (int64_t)(outer - qd * d) * stride[gr.axis[j]];
      outer = qd;
    }
    if (n < gr.n_obs) {
      int row = n;
      for (int mi = gr.m_begin; mi < gr.m_end; ++mi) {
        const EfeModality& md = p.mod[tp.mod_order[mi]];
        if (row < md.O) {
          v = __ldg(A + b * p.A_stride + md.A_off + (int64_t)row * md.K + k);
          break;
        }
        row -= md.O;
      }
    } else {
      const int t = n - gr.n_obs;
      for (int mi = gr.m_begin; mi < gr.m_end; ++mi) {
        const EfeModality& md = p.mod[tp.mod_order[mi]];
        const float* Am = A + b * p.A_stride + md.A_off;
        const float* Cm = C + b * p.C_stride + md.C_off + (int64_t)t * md.O;
        for (int o = 0; o < md.O; ++o) {
          const float a = __ldg(Am + (int64_t)o * md.K + k);
          float w = 0.f;
          if (ig) w += log_stable(a);
          if (ut) w += __ldg(Cm + o);
          v = fmaf(a, w, v);
        }
      }
    }
  }
  const int c = kp / Tr::kChunk;
  const int byte = (kp % Tr::kChunk) * Tr::kEsz;
  uint8_t* img = pack + b * tp.pack_stride + gr.pack_off + (int64_t)c * gr.chunk_bytes;
  const uint32_t off = tc::sw128_offset((uint32_t)n, (uint32_t)(byte >> 4)) + (byte & 15);
  if (PREC == B2_PRECISION_BF16) {
    *reinterpret_cast<uint16_t*>(img + off) = bf16_bits(v);
  } else {
    const float hi = tf32_round(v);
    *reinterpret_cast<float*>(img + off) = hi;
    *reinterpret_cast<float*>(img + (int64_t)gr.N * 128 + off) = tf32_round(v - hi);
  }
}

// ------------------------------------------------------ X generation
// This thread's H values of X[policy, k0 .. k0+H): the Kronecker product of
// the policy's factor marginals in the group's K order. q is laid out
// [state][128 policies]. DLP = padded innermost size when DLP <= H (then the
// H values are H/DLP runs of pre * ql[0..DLP) with ql held in registers);
// DLP = 0 selects the general path (padded innermost size > H).
template <int H, int DLP>
__device__ __forceinline__ void gen_x(const TcGroup& gr, const EfeParams& p, const float* __restrict__ q, int pl,
                                      int k0, const float (&ql)[DLP > 0 ? DLP : 1], float (&out)[H]) {
  const int r = gr.rank;
  const int lg = gr.lg;
  int ko = k0 >> lg;  // outer index of the first element
  // outer digits dig[0 .. r-2] of ko (row-major over dim[0 .. r-2])
  int dig[B2_MAX_DEP_RANK - 1];
  {
    int rem = ko;
#pragma unroll
    for (int j = B2_MAX_DEP_RANK - 2; j >= 0; --j) {
      dig[j] = 0;
      if (j < r - 1) {
        const int d = gr.dim[j];
        const int qd = rem / d;
        dig[j] = rem - qd * d;
        rem = qd;
      }
    }
  }
  // prefix product over dig[0 .. r-3] and the last outer factor's q base
  auto prefix2 = [&]() {
    float v = 1.f;
#pragma unroll
    for (int j = 0; j < B2_MAX_DEP_RANK - 2; ++j)
      if (j < r - 2) v *= q[(p.qs_off[gr.dep[j]] + dig[j]) * kTcTile + pl];
    return v;
  };
  float P2 = prefix2();
  const float* q_r2 = r >= 2 ? q + p.qs_off[gr.dep[r - 2]] * kTcTile + pl : nullptr;
  if (DLP > 0) {
    constexpr int kRuns = DLP > 0 ? H / DLP : 1;
#pragma unroll
    for (int run = 0; run < kRuns; ++run) {
      float pre = 0.f;
      if (ko + run < gr.outer) pre = r >= 2 ? P2 * q_r2[dig[r - 2] * kTcTile] : 1.f;
#pragma unroll
      for (int i = 0; i < (DLP > 0 ? DLP : 1); ++i) out[run * (DLP > 0 ? DLP : 1) + i] = pre * ql[i];
      if (run + 1 < kRuns && r >= 2) {
        // advance the outer index by one (carry through the outer digits)
        if (++dig[r - 2] >= gr.dim[r - 2]) {
          dig[r - 2] = 0;
          bool carry = true;
#pragma unroll
          for (int j = B2_MAX_DEP_RANK - 3; j >= 0; --j) {
            if (carry && j < r - 2) {
              if (++dig[j] < gr.dim[j]) carry = false;
              else dig[j] = 0;
            }
          }
          P2 = prefix2();
        }
      }
    }
  } else {
    const int off = k0 & ((1 << lg) - 1);
    const int dl = gr.dim[r - 1];
    float pre = 0.f;
    if (ko < gr.outer) pre = r >= 2 ? P2 * q_r2[dig[r - 2] * kTcTile] : 1.f;
    const float* qlp = q + p.qs_off[gr.dep[r - 1]] * kTcTile + pl;
#pragma unroll
    for (int i = 0; i < H; ++i) out[i] = (off + i < dl) ? pre * qlp[(off + i) * kTcTile] : 0.f;
  }
}

struct TcSmem {
  uint8_t* Xs;
  uint8_t* Ws;
  uint64_t* done;  // per stage: MMAs reading the stage finished
  uint64_t* full;  // per stage: W bulk copy landed
  volatile int* abort_flag;
  int xs_bytes, ws_bytes;
};

// All chunks of one (step, group) GEMM: produce X, bulk-copy W, issue UMMAs.
template <int PREC, int DLP>
__device__ __forceinline__ void run_group(const TcGroup& gr, const TcParams& tp, const EfeParams& p,
                                          const float* __restrict__ q, const uint8_t* __restrict__ wimg,
                                          const TcSmem& sm, uint32_t tmem, int tid, int pl, int half, bool active,
                                          uint32_t& it) {
  using Tr = TcTraits<PREC>;
  constexpr int H = Tr::kChunk / 2;
  constexpr int kQl = DLP > 0 ? DLP : 1;
  float ql[kQl];
  if (DLP > 0) {
    const float* qlp = q + p.qs_off[gr.dep[gr.rank - 1]] * kTcTile + pl;
    const int dl = gr.dim[gr.rank - 1];
#pragma unroll
    for (int i = 0; i < kQl; ++i) ql[i] = (i < dl && active) ? qlp[i * kTcTile] : 0.f;
  }
  for (int c = 0; c < gr.nch; ++c, ++it) {
    const int st = it % kTcStages;
    const uint32_t use = it / kTcStages;
    if (use > 0 && !tc::mbar_wait_bounded(&sm.done[st], (use - 1) & 1, kWaitLimit)) *sm.abort_flag = 1;
    uint8_t* xs = sm.Xs + st * sm.xs_bytes;
    uint8_t* ws = sm.Ws + st * sm.ws_bytes;
    if (tid == 0) {  // W chunk: one bulk copy of the pre-swizzled image
      mbar_expect_tx(&sm.full[st], (uint32_t)gr.chunk_bytes);
      bulk_g2s(tc::smem_u32(ws), wimg + (int64_t)c * gr.chunk_bytes, (uint32_t)gr.chunk_bytes, &sm.full[st]);
    }
    float v[H];
    gen_x<H, DLP>(gr, p, q, pl, c * Tr::kChunk + half * H, ql, v);
    if (!active)
#pragma unroll
      for (int i = 0; i < H; ++i) v[i] = 0.f;
    const uint32_t xa = tc::smem_u32(xs);
    if (PREC == B2_PRECISION_BF16) {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        tc::sts128(xa + tc::sw128_offset(pl, half * 4 + j), bf16x2_bits(v[j * 8 + 0], v[j * 8 + 1]),
                   bf16x2_bits(v[j * 8 + 2], v[j * 8 + 3]), bf16x2_bits(v[j * 8 + 4], v[j * 8 + 5]),
                   bf16x2_bits(v[j * 8 + 6], v[j * 8 + 7]));
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        float hi[4], lo[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          hi[e] = tf32_round(v[j * 4 + e]);
          lo[e] = tf32_round(v[j * 4 + e] - hi[e]);
        }
        const uint32_t off = tc::sw128_offset(pl, half * 4 + j);
        tc::sts128(xa + off, __float_as_uint(hi[0]), __float_as_uint(hi[1]), __float_as_uint(hi[2]),
                   __float_as_uint(hi[3]));
        tc::sts128(xa + kTcTile * 128 + off, __float_as_uint(lo[0]), __float_as_uint(lo[1]), __float_as_uint(lo[2]),
                   __float_as_uint(lo[3]));
      }
    }
    tc::fence_proxy_async_smem();
    __syncthreads();
    if (*sm.abort_flag) return;
    if (tid == 0) {
      if (!tc::mbar_wait_bounded(&sm.full[st], use & 1, kWaitLimit)) {
        *sm.abort_flag = 1;
      } else {
        tc::fence_after_sync();
        const uint32_t a0 = tc::smem_u32(xs), b0 = tc::smem_u32(ws);
        // chunk c accumulates into accumulator c % nacc: shorter FP32
        // accumulation chains inside the tensor core
        const uint32_t dt = tmem + (uint32_t)((c % tp.nacc) * gr.N);
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint32_t acc = (c >= tp.nacc || kk > 0) ? 1u : 0u;
          if (PREC == B2_PRECISION_BF16) {
            tc::mma_bf16(dt, tc::desc_kmajor_sw128(a0 + kk * 32), tc::desc_kmajor_sw128(b0 + kk * 32), gr.idesc, acc);
          } else {
            const uint32_t alo = a0 + kTcTile * 128, blo = b0 + gr.N * 128;
            tc::mma_tf32(dt, tc::desc_kmajor_sw128(a0 + kk * 32), tc::desc_kmajor_sw128(b0 + kk * 32), gr.idesc, acc);
            tc::mma_tf32(dt, tc::desc_kmajor_sw128(a0 + kk * 32), tc::desc_kmajor_sw128(blo + kk * 32), gr.idesc, 1u);
            tc::mma_tf32(dt, tc::desc_kmajor_sw128(alo + kk * 32), tc::desc_kmajor_sw128(b0 + kk * 32), gr.idesc, 1u);
          }
        }
        tc::mma_commit(&sm.done[st]);
      }
    }
  }
}

// ------------------------------------------------------------ main kernel
template <int PREC>
__global__ void __launch_bounds__(kTcThreads, 1)
    efe_tc_kernel(const __grid_constant__ EfeParams p, const __grid_constant__ TcParams tp,
                  const int32_t* __restrict__ pm, int pm_batched, const float* __restrict__ qs_init,
                  const float* __restrict__ B, const uint8_t* __restrict__ pack, float* __restrict__ G) {
  using Tr = TcTraits<PREC>;
  constexpr int kPl = Tr::kPlanes;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  TcSmem sm;
  sm.xs_bytes = kPl * kTcTile * 128;
  sm.ws_bytes = kPl * tp.Nmax * 128;
  sm.Xs = base;
  sm.Ws = sm.Xs + kTcStages * sm.xs_bytes;
  float* qsm = reinterpret_cast<float*>(sm.Ws + kTcStages * sm.ws_bytes);
  sm.done = reinterpret_cast<uint64_t*>(qsm + 2 * p.S_tot * kTcTile);
  sm.full = sm.done + kTcStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm.full + kTcStages);
  sm.abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5;
  const int pl = tid & (kTcTile - 1);
  const int half = tid >> 7;
  const int64_t b = blockIdx.y;
  const int pol = blockIdx.x * kTcTile + pl;
  const bool active = pol < p.P;

  if (warp == 0) tc::tmem_alloc(tmem_slot, (uint32_t)tp.tmem_cols);
  if (tid == 0) {
    for (int s = 0; s < kTcStages; ++s) {
      tc::mbar_init(&sm.done[s], 1);
      tc::mbar_init(&sm.full[s], 1);
    }
    tc::fence_mbar_init();
    *sm.abort_flag = 0;
  }
  for (int i = tid; i < p.S_tot * kTcTile; i += kTcThreads) qsm[i] = __ldg(qs_init + b * p.S_tot + i / kTcTile);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  double g_acc = 0.0;
  bool bad_action = false;
  int cur = 0;
  uint32_t it = 0;
  bool aborted = false;
  for (int t = 0; t < p.T && !aborted; ++t) {
    // ---- expected states (pymdp/control.py:351-389): policy pl, states s = half, half + 2, ...
    {
      const float* qc = qsm + cur * p.S_tot * kTcTile;
      float* qn = qsm + (cur ^ 1) * p.S_tot * kTcTile;
      const int32_t* u_pol = pm + (pm_batched ? b * (int64_t)p.P * p.T * p.F : 0) +
                             (int64_t)(active ? pol : 0) * p.T * p.F + t * p.F;
      for (int f = 0; f < p.F; ++f) {
        const EfeFactor& fb = p.fac[f];
        int u = u_pol[f];
        if (u < 0 || u >= p.U[f]) {
          bad_action = true;
          u = 0;
        }
        const float* Bf = B + b * p.B_stride + fb.B_off;
        const int U = p.U[f];
        for (int s = half; s < p.S[f]; s += 2) {
          float acc = 0.f;
          const float* Bs = Bf + (int64_t)s * fb.K * U + u;
          if (fb.rank == 1) {
            const float* qv = qc + p.qs_off[fb.dep[0]] * kTcTile + pl;
            for (int k = 0; k < fb.K; ++k) acc = fmaf(__ldg(Bs + (int64_t)k * U), qv[k * kTcTile], acc);
          } else {
            int dig[B2_MAX_DEP_RANK];
#pragma unroll
            for (int i = 0; i < B2_MAX_DEP_RANK; ++i) dig[i] = 0;
            for (int k = 0; k < fb.K; ++k) {
              float w = 1.f;
#pragma unroll
              for (int i = 0; i < B2_MAX_DEP_RANK; ++i)
                if (i < fb.rank) w *= qc[(p.qs_off[fb.dep[i]] + dig[i]) * kTcTile + pl];
              acc = fmaf(__ldg(Bs + (int64_t)k * U), w, acc);
              bool carry = true;
#pragma unroll
              for (int i = B2_MAX_DEP_RANK - 1; i >= 0; --i) {
                if (carry && i < fb.rank) {
                  if (++dig[i] < p.S[fb.dep[i]]) carry = false;
                  else dig[i] = 0;
                }
              }
            }
          }
          qn[(p.qs_off[f] + s) * kTcTile + pl] = acc;
        }
      }
    }
    __syncthreads();
    cur ^= 1;
    const float* q = qsm + cur * p.S_tot * kTcTile;

    for (int g = 0; g < tp.G && !aborted; ++g) {
      const TcGroup& gr = tp.grp[g];
      const uint8_t* wimg = pack + b * tp.pack_stride + gr.pack_off;
      constexpr int H = Tr::kChunk / 2;
      const int dlp = 1 << gr.lg;
      if (dlp > H) {
        run_group<PREC, 0>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it);
      } else {
        switch (gr.lg) {
          case 0: run_group<PREC, 1>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it); break;
          case 1: run_group<PREC, 2>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it); break;
          case 2: run_group<PREC, 4>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it); break;
          case 3: run_group<PREC, 8>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it); break;
          case 4: run_group<PREC, (H >= 16 ? 16 : 0)>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it); break;
          default: run_group<PREC, (H >= 32 ? 32 : 0)>(gr, tp, p, q, wimg, sm, tmem, tid, pl, half, active, it); break;
        }
      }
      __syncthreads();
      if (*sm.abort_flag) {
        aborted = true;
        break;
      }
      // ---- epilogue for (t, g): wait for the last chunk's MMAs
      {
        const uint32_t last = it - 1;
        if (!tc::mbar_wait_bounded(&sm.done[last % kTcStages], (last / kTcStages) & 1, kWaitLimit))
          *sm.abort_flag = 1;
      }
      tc::fence_after_sync();
      if (warp < 4) {
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16);
        double h = 0.0, lin = 0.0;
        const int nacc = gr.nch < tp.nacc ? gr.nch : tp.nacc;
        for (int n0 = 0; n0 < gr.N; n0 += 16) {
          double sum[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) sum[j] = 0.0;
          for (int a = 0; a < nacc; ++a) {
            uint32_t r[16];
            tc::tmem_ld16(taddr + (uint32_t)(a * gr.N + n0), r);
            tc::tmem_wait_ld();
#pragma unroll
            for (int j = 0; j < 16; ++j) sum[j] += (double)__uint_as_float(r[j]);
          }
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int n = n0 + j;
            if (n < gr.n_obs) {
              if (ig) h -= sum[j] * (double)logf(fmaxf((float)sum[j], kMinVal));
            } else if (n == gr.n_obs + t) {
              lin = sum[j];
            }
          }
        }
        g_acc += h + lin;
      }
      tc::fence_before_sync();
      __syncthreads();
      if (*sm.abort_flag) aborted = true;
    }
  }
  if (aborted && tid == 0) atomicExch(&g_b2_device_error, 1);
  if (tid < kTcTile && active && !aborted) G[b * p.P + pol] = bad_action ? __int_as_float(0x7fc00000) : (float)g_acc;
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)tp.tmem_cols);
}

}  // namespace

// Plan the tensor-core path; returns B2_ERR_UNSUPPORTED when the model falls
// outside its limits (the caller then uses the SIMT kernel).
int32_t tc_plan(const EfeParams& p, int prec, TcParams* tp, int* smem_bytes) {
  std::memset(tp, 0, sizeof(*tp));
  const int chunk = prec == B2_PRECISION_BF16 ? 64 : 32;
  const int H = chunk / 2;
  const int planes = prec == B2_PRECISION_BF16 ? 1 : 2;
  std::vector<std::vector<int>> groups;
  std::vector<std::vector<int>> tuples;
  for (int m = 0; m < p.M; ++m) {
    std::vector<int> tup(p.mod[m].dep, p.mod[m].dep + p.mod[m].rank);
    int g = -1;
    for (size_t i = 0; i < tuples.size(); ++i)
      if (tuples[i] == tup) g = (int)i;
    if (g < 0) {
      g = (int)tuples.size();
      tuples.push_back(tup);
      groups.emplace_back();
    }
    groups[g].push_back(m);
  }
  if ((int)groups.size() > kTcMaxGroups) return B2_ERR_UNSUPPORTED;
  tp->G = (int32_t)groups.size();
  int n_order = 0;
  int64_t off = 0;
  int Nmax = 16;
  for (int g = 0; g < tp->G; ++g) {
    TcGroup& gr = tp->grp[g];
    const std::vector<int>& tup = tuples[g];
    const int r = (int)tup.size();
    gr.rank = r;
    // innermost factor: the largest padded size that still fits a half chunk
    int best = r - 1, best_p = -1;
    for (int a = 0; a < r; ++a) {
      int pw = 1;
      while (pw < p.S[tup[a]]) pw <<= 1;
      const int score = pw <= H ? pw : 0;
      if (score > best_p) {
        best_p = score;
        best = a;
      }
    }
    int j = 0;
    int64_t K = 1;
    for (int a = 0; a < r; ++a) {
      K *= p.S[tup[a]];
      if (a == best) continue;
      gr.dep[j] = (int8_t)tup[a];
      gr.axis[j] = (int8_t)a;
      gr.dim[j] = (int16_t)p.S[tup[a]];
      ++j;
    }
    gr.dep[r - 1] = (int8_t)tup[best];
    gr.axis[r - 1] = (int8_t)best;
    gr.dim[r - 1] = (int16_t)p.S[tup[best]];
    int lg = 0;
    while ((1 << lg) < p.S[tup[best]]) ++lg;
    gr.lg = lg;
    if (K > (1 << 24)) return B2_ERR_UNSUPPORTED;
    gr.K = (int32_t)K;
    gr.outer = (int32_t)(K / p.S[tup[best]]);
    const int64_t Kp = (int64_t)gr.outer << lg;
    gr.Kpad = (int32_t)((Kp + chunk - 1) / chunk * chunk);
    gr.nch = gr.Kpad / chunk;
    gr.m_begin = n_order;
    int n_obs = 0;
    for (int m : groups[g]) {
      tp->mod_order[n_order++] = (int8_t)m;
      n_obs += p.mod[m].O;
    }
    gr.m_end = n_order;
    gr.n_obs = n_obs;
    gr.N = (n_obs + p.T + 15) / 16 * 16;
    if (gr.N > 256) return B2_ERR_UNSUPPORTED;
    Nmax = gr.N > Nmax ? gr.N : Nmax;
    gr.idesc = tc::idesc_f32acc(prec == B2_PRECISION_BF16 ? 1u : 2u, 128u, (uint32_t)gr.N);
    gr.chunk_bytes = planes * gr.N * 128;
    gr.pack_off = off;
    off += (int64_t)gr.nch * gr.chunk_bytes;
  }
  tp->Nmax = Nmax;
  int nacc = 512 / Nmax;
  nacc = nacc > 8 ? 8 : nacc;
  tp->nacc = nacc;
  int cols = 32;
  while (cols < nacc * Nmax) cols <<= 1;
  tp->tmem_cols = cols;
  tp->pack_stride = (off + 1023) / 1024 * 1024;
  const int xs_bytes = planes * kTcTile * 128;
  const int w_bytes = planes * Nmax * 128;
  const int64_t smem = 1024 + (int64_t)kTcStages * (xs_bytes + w_bytes) + 2LL * p.S_tot * kTcTile * 4 +
                       2 * kTcStages * 8 + 16;
  if (smem > 227 * 1024) return B2_ERR_UNSUPPORTED;
  *smem_bytes = (int)smem;
  return B2_OK;
}

int32_t launch_efe_tc(const EfeParams& p, int prec, int64_t Bn, const int32_t* pm, int pm_batched, const float* qs,
                      const float* A, const float* B, const float* C, float* G, cudaStream_t stream,
                      bool* used) {
  *used = false;
  TcParams tp;
  int smem = 0;
  if (tc_plan(p, prec, &tp, &smem) != B2_OK) return B2_OK;
  if (Bn > 65535) return B2_OK;
  const size_t bytes = (size_t)Bn * (size_t)tp.pack_stride;
  uint8_t* pack = nullptr;
  B2_TRY(ws_alloc((void**)&pack, bytes, stream, kEfeName));
  int32_t rc = B2_OK;
  int Kmax = 0;
  for (int g = 0; g < tp.G; ++g) Kmax = tp.grp[g].Kpad > Kmax ? tp.grp[g].Kpad : Kmax;
  dim3 pgrid((unsigned)((Kmax + 127) / 128), (unsigned)(tp.G * 256), (unsigned)Bn);
  dim3 grid((unsigned)((p.P + kTcTile - 1) / kTcTile), (unsigned)Bn);
  if (prec == B2_PRECISION_BF16) {
    efe_tc_pack_kernel<B2_PRECISION_BF16><<<pgrid, 128, 0, stream>>>(p, tp, A, C, pack);
    rc = check_launch("efe_ffi tc pack");
    if (rc == B2_OK) rc = ensure_smem_attr((const void*)efe_tc_kernel<B2_PRECISION_BF16>, smem, kEfeName);
    if (rc == B2_OK) {
      efe_tc_kernel<B2_PRECISION_BF16><<<grid, kTcThreads, smem, stream>>>(p, tp, pm, pm_batched, qs, B, pack, G);
      rc = check_launch("efe_ffi tc");
    }
  } else {
    efe_tc_pack_kernel<B2_PRECISION_TF32X3><<<pgrid, 128, 0, stream>>>(p, tp, A, C, pack);
    rc = check_launch("efe_ffi tc pack");
    if (rc == B2_OK) rc = ensure_smem_attr((const void*)efe_tc_kernel<B2_PRECISION_TF32X3>, smem, kEfeName);
    if (rc == B2_OK) {
      efe_tc_kernel<B2_PRECISION_TF32X3><<<grid, kTcThreads, smem, stream>>>(p, tp, pm, pm_batched, qs, B, pack,
                                                                               G);
      rc = check_launch("efe_ffi tc");
    }
  }
  cudaError_t fe = cudaFreeAsync(pack, stream);
  if (rc == B2_OK && fe != cudaSuccess) return cuda_fail(kEfeName, fe);
  *used = rc == B2_OK;
  return rc;
}

}  // namespace b2

// Reads and clears the device-side error word set by a kernel whose bounded
// wait ran out (synchronises the device; diagnostics and tests only).
extern "C" int32_t b2_device_error(void) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, b2::g_b2_device_error, sizeof(int)) != cudaSuccess) return -1;
  const int zero = 0;
  cudaMemcpyToSymbol(b2::g_b2_device_error, &zero, sizeof(int));
  return v;
}
