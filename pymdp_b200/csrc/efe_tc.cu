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
//  * 16 producer warps (four threads per policy) roll the policy's factor
//    marginals forward through B (staged in shared memory, transposed so a
//    thread's block of next states is one broadcast vector load per parent
//    state), build a per-policy table of the outer factors' products, and
//    write X straight into tensor memory (tcgen05.st): the MMA's A operand,
//    a ring of stages of kCps chunks.
//  * W is packed once per call into ready-made shared-memory images (one per
//    128-byte K chunk, already swizzled). One loader thread moves several
//    chunks per cp.async.bulk (no multicast) into a separate ring of large
//    shared-memory slots: a bulk copy costs about the same few hundred cycles
//    whether it moves 8 KB or 32 KB, so W arrives in big pieces.
//  * One thread issues the UMMAs (kind::f16 with a 3-pass BF16 hi/lo split,
//    or kind::tf32 with the 3xTF32 hi/lo split, A from tensor memory and B
//    from shared memory: hi*hi + hi*lo + lo*hi per K-step), accumulating in
//    TMEM. Where the accumulators fit (N <= 64), each pipeline stage's hi*hi
//    products go to a fresh accumulator that the producers fold into FP64
//    before the slot is reused ("drain mode"); otherwise stages rotate over
//    several accumulators. Either way the tensor core's FP32 accumulation
//    chains stay short.
//  * Epilogue: producer warp w reads TMEM lane quarter w % 4 (its 32
//    policies) with tcgen05.ld, forms the entropy of the obs rows and adds the
//    step's linear row, accumulating G in FP64 registers.
// Hand-offs are mbarriers: x_full (X written), done (MMAs of an A stage
// finished), w_full / w_free (W slot landed / consumed), acc_full / acc_free.
// Every wait is bounded; on timeout the CTA records an error in
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
constexpr int kTcTile = 128;
constexpr uint32_t kWaitLimit = 1u << 22;
constexpr int kTcMaxOuter = 3;       // tensor-core path: dependency rank <= 4
constexpr int kTcMaxAStages = 8;     // A (X) stages in tensor memory
constexpr int kTcWSlots = 2;         // W slots in shared memory
constexpr int kTcWSlotTarget = 32768;  // preferred bytes per W bulk copy
constexpr int kTcMaxT = 8;             // policy-tree mode: policy_len <= 8

struct TcGroup {
  int64_t pack_off;  // per-agent byte offset of this group's W image
  int32_t K;         // prod of the dependency sizes
  int32_t outer;     // K / dim[rank-1]
  int32_t Kpad;      // padded K (innermost size rounded to a power of two, then to the stage)
  int32_t nch;       // Kpad / chunk (a multiple of the chunks per A stage)
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
  int32_t nst;        // A stages in tensor memory (each kCps chunks)
  int32_t wch;        // chunks per W slot (a multiple of kCps)
  int32_t ws_bytes;   // bytes per W slot
  int32_t nacc;       // TMEM accumulators the A stages rotate over (summed in FP64)
  int32_t corr;       // 3xTF32: accumulator slot of the hi*lo + lo*hi correction products (-1: none, they
                      // go with the hi*hi products)
  int32_t drain;      // 1: each A stage's hi*hi products go to a fresh accumulator tied to its ring slot, which
                      // the producers fold into FP64 registers before reusing the slot (N <= 64)
  int32_t b_words;    // floats of B staged in shared memory per CTA (0 = read B from global)
  int32_t a_col;      // first TMEM column of the A (X) stages; accumulators start at column 0
  int32_t tmem_cols;  // allocated TMEM columns
  int32_t pre_cap;    // outer indices the shared prefix table holds (>= every group's outer)
  int64_t pack_stride;  // bytes of W images per agent
  int32_t b_off[kEfeMaxF];  // staged B of factor f: float offset in shared memory
  int8_t b_tr[kEfeMaxF];    // 1: staged transposed as [k][u][s] (rank-1 parents, S % 4 == 0)
  int8_t mod_order[B2_MAX_MODALITIES];
  TcGroup grp[kTcMaxGroups];
  // policy-tree mode (B2_FLAG_POLICY_TREE): CTA x of depth t covers prefixes
  // [(x - tree_tiles[t]) * 128, +128) of the prod(U)^(t+1) prefixes at depth t
  int32_t tree, tree_nu;
  int32_t tree_tiles[kTcMaxT + 1];  // cumulative 128-row tiles per depth
  int64_t tree_off[kTcMaxT + 1];    // cumulative prefixes per depth (per-agent offsets into Gt)
  int64_t tree_w[kTcMaxT];          // prod(U)^(T-1-t): policies per prefix at depth t
};

template <int PREC>
struct TcTraits;
// kChunk: K elements per 128-byte row (one chunk); kCps: chunks per A stage
// (the MMA issuer handles kCps * 4 K-steps per stage hand-off).
template <>
struct TcTraits<B2_PRECISION_BF16> {
  static constexpr int kChunk = 64;
  static constexpr int kPlanes = 2;  // hi, lo: the 3-pass BF16 split (hi*hi + hi*lo + lo*hi)
  static constexpr int kEsz = 2;
  static constexpr int kCps = 2;
  static constexpr int kMaxNst = 2;
};
template <>
struct TcTraits<B2_PRECISION_TF32X3> {
  static constexpr int kChunk = 32;
  static constexpr int kPlanes = 2;  // hi, lo
  static constexpr int kEsz = 4;
  static constexpr int kCps = 1;
  static constexpr int kMaxNst = 3;
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
// K-major layout, so the main kernel moves chunks with plain bulk copies.
// K is ordered with the group's chosen innermost factor last, its size padded
// to a power of two (padding columns are zero). One thread = one packed
// column kp of one group: it gathers the column's observation rows once,
// takes their logs once, and forms all T linear rows from them.
template <int PREC>
__global__ void efe_tc_pack_kernel(const __grid_constant__ EfeParams p, const __grid_constant__ TcParams tp,
                                   const float* __restrict__ A, const float* __restrict__ C, uint8_t* __restrict__ pack) {
  using Tr = TcTraits<PREC>;
  const int64_t b = blockIdx.z;
  const int g = blockIdx.y;
  if (g >= tp.G) return;
  const TcGroup& gr = tp.grp[g];
  const int kp = blockIdx.x * blockDim.x + threadIdx.x;
  if (kp >= gr.Kpad) return;
  const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
  const bool ut = (p.flags & B2_FLAG_USE_UTILITY) != 0;
  const int N = gr.N, n_obs = gr.n_obs, T = p.T;
  const int inner = kp & ((1 << gr.lg) - 1);
  int outer = kp >> gr.lg;
  const bool valid = inner < gr.dim[gr.rank - 1] && outer < gr.outer;
  int64_t k = 0;
  if (valid) {
    // original row-major index over the modalities' own axis order
    const EfeModality& m0 = p.mod[tp.mod_order[gr.m_begin]];
    int64_t stride[B2_MAX_DEP_RANK];
    int64_t st = 1;
    for (int a = gr.rank - 1; a >= 0; --a) {
      stride[a] = st;
      st *= p.S[m0.dep[a]];
    }
    k = (int64_t)inner * stride[gr.axis[gr.rank - 1]];
    for (int j = gr.rank - 2; j >= 0; --j) {
      const int d = gr.dim[j];
      const int qd = outer / d;
      k += (int64_t)(outer - qd * d) * stride[gr.axis[j]];
      outer = qd;
    }
  }
  const int c = kp / Tr::kChunk;
  const int byte = (kp % Tr::kChunk) * Tr::kEsz;
  uint8_t* img = pack + b * tp.pack_stride + gr.pack_off + (int64_t)c * gr.chunk_bytes;
  auto put = [&](int n, float v) {
    const uint32_t off = tc::sw128_offset((uint32_t)n, (uint32_t)(byte >> 4)) + (byte & 15);
    if (PREC == B2_PRECISION_BF16) {
      const __nv_bfloat16 hi = __float2bfloat16_rn(v);
      *reinterpret_cast<uint16_t*>(img + off) = bf16_bits(v);
      *reinterpret_cast<uint16_t*>(img + (int64_t)N * 128 + off) = bf16_bits(v - __bfloat162float(hi));
    } else {
      const float hi = tf32_round(v);
      *reinterpret_cast<float*>(img + off) = hi;
      *reinterpret_cast<float*>(img + (int64_t)N * 128 + off) = tf32_round(v - hi);
    }
  };
  // observation rows, and the information-gain part of the linear rows
  float hl = 0.f;
  int n = 0;
  for (int mi = gr.m_begin; mi < gr.m_end; ++mi) {
    const EfeModality& md = p.mod[tp.mod_order[mi]];
    const float* Am = A + b * p.A_stride + md.A_off + k;
    for (int o = 0; o < md.O; ++o, ++n) {
      const float a = valid ? __ldg(Am + (int64_t)o * md.K) : 0.f;
      if (ig) hl = fmaf(a, log_stable(a), hl);
      put(n, a);
    }
  }
  // one linear row per step: the utility part re-reads the column (cached)
  for (int t = 0; t < T; ++t) {
    float v = hl;
    if (ut && valid) {
      for (int mi = gr.m_begin; mi < gr.m_end; ++mi) {
        const EfeModality& md = p.mod[tp.mod_order[mi]];
        const float* Am = A + b * p.A_stride + md.A_off + k;
        const float* Cm = C + b * p.C_stride + md.C_off + (int64_t)t * md.O;
        for (int o = 0; o < md.O; ++o) v = fmaf(__ldg(Am + (int64_t)o * md.K), __ldg(Cm + o), v);
      }
    }
    put(n_obs + t, valid ? v : 0.f);
  }
  for (int r = n_obs + T; r < N; ++r) put(r, 0.f);
}

// Bounded mbarrier wait that also gives up as soon as another role of the
// CTA has flagged an abort (so one timeout cannot cascade into long waits).
__device__ __forceinline__ bool wait_or_abort(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  for (uint32_t i = 0; i < kWaitLimit; ++i) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    if ((i & 255) == 255 && *abort_flag) return false;
  }
  *abort_flag = 1;
  return false;
}

// One lane polls, the warp follows: keeps 512 producer threads from
// flooding the barrier unit that the MMA issuer also needs.
__device__ __forceinline__ void warp_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag, int lane) {
  if (lane == 0) wait_or_abort(bar, parity, abort_flag);
  __syncwarp();
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc::smem_u32(bar)) : "memory");
}

// Position in a ring of `n` slots: slot index and the parity of its use count.
struct Ring {
  int slot = 0;
  uint32_t phase = 0;  // parity of the current use of `slot`
  bool wrapped = false;  // every slot has been used at least once
  __device__ __forceinline__ void next(int n) {
    if (++slot == n) {
      slot = 0;
      phase ^= 1u;
      wrapped = true;
    }
  }
};

// One A stage of MMAs (kCps chunks x 4 K-steps; 3xTF32: three MMAs per
// K-step) in a single asm block that first starts non-blocking tests of the
// next stage's barriers: their latency overlaps the MMA issue, and the loop
// only blocks when a test found the next stage not ready yet. Operands:
// dt = accumulator, a0 = A stage in tensor memory, wd = descriptor of the
// stage's first W chunk, chunk16 / lo16 = descriptor steps to the next chunk
// / the lo plane, first = accumulate flag of the stage's first MMA.
// 3-pass BF16 stage (kCps = 2 chunks, 4 K-steps of 16 each): per K-step
// hi*hi into the accumulator dt (accumulate flag `first` on the stage's first
// K-step), hi*lo (W lo plane) and lo*hi (A lo plane, 32 columns on) into dc
// (`firstc` on the stage's first K-step).
__device__ __forceinline__ void issue_stage_bf16(uint32_t dt, uint32_t dc, uint32_t a0, uint64_t wd,
                                                 uint32_t chunk16, uint32_t idesc, uint32_t first, uint32_t firstc,
                                                 uint32_t nx, uint32_t nxp, uint32_t nw, uint32_t nwp, uint32_t lo16,
                                                 uint32_t& rx, uint32_t& rw) {
  asm volatile(
      "{\n\t"
      ".reg .pred px, pw, pa, pc, pt;\n\t"
      ".reg .b32 at, atl;\n\t"
      ".reg .b64 bh, bd, bdl, c16, cl;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 px, [%2], %3;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 pw, [%4], %5;\n\t"
      "setp.ne.b32 pa, %6, 0;\n\t"
      "setp.ne.b32 pc, %14, 0;\n\t"
      "setp.eq.b32 pt, 0, 0;\n\t"
      "cvt.u64.u32 c16, %10;\n\t"
      "cvt.u64.u32 cl, %12;\n\t"
      "mov.b64 bh, %9;\n\t"
      // chunk 0: K-steps at A columns 0, 8, 16, 24 (lo plane +32), W +0, +2, +4, +6
      "add.u32 at, %8, 0;\n\t"
      "add.u64 bd, bh, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pa;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pc;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 8;\n\t"
      "add.u64 bd, bh, 2;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 16;\n\t"
      "add.u64 bd, bh, 4;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 24;\n\t"
      "add.u64 bd, bh, 6;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      // chunk 1: A columns 64.. (a chunk is 64 columns: hi and lo planes), W one chunk on
      "add.u64 bh, bh, c16;\n\t"
      "add.u32 at, %8, 64;\n\t"
      "add.u64 bd, bh, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 72;\n\t"
      "add.u64 bd, bh, 2;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 80;\n\t"
      "add.u64 bd, bh, 4;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 88;\n\t"
      "add.u64 bd, bh, 6;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%13], [atl], bd, %11, pt;\n\t"
      "selp.u32 %0, 1, 0, px;\n\t"
      "selp.u32 %1, 1, 0, pw;\n\t"
      "}"
      : "=r"(rx), "=r"(rw)
      : "r"(nx), "r"(nxp), "r"(nw), "r"(nwp), "r"(first), "r"(dt), "r"(a0), "l"(wd), "r"(chunk16), "r"(idesc),
        "r"(lo16), "r"(dc), "r"(firstc)
      : "memory");
}

// 3xTF32 stage: per K-step hi*hi into the accumulator dt (accumulate flag
// `first` on the stage's first K-step), hi*lo and lo*hi into dc (`firstc` on
// the stage's first K-step). dc may equal dt.
__device__ __forceinline__ void issue_stage_tf32x3(uint32_t dt, uint32_t dc, uint32_t a0, uint64_t wd,
                                                   uint32_t chunk16, uint32_t idesc, uint32_t first, uint32_t firstc,
                                                   uint32_t nx, uint32_t nxp, uint32_t nw, uint32_t nwp,
                                                   uint32_t lo16, uint32_t& rx, uint32_t& rw) {
  asm volatile(
      "{\n\t"
      ".reg .pred px, pw, pa, pc, pt;\n\t"
      ".reg .b32 at, atl;\n\t"
      ".reg .b64 bh, bd, bdl, c16, cl;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 px, [%2], %3;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 pw, [%4], %5;\n\t"
      "setp.ne.b32 pa, %6, 0;\n\t"
      "setp.ne.b32 pc, %14, 0;\n\t"
      "setp.eq.b32 pt, 0, 0;\n\t"
      "cvt.u64.u32 c16, %10;\n\t"
      "cvt.u64.u32 cl, %12;\n\t"
      "mov.b64 bh, %9;\n\t"
      "add.u32 at, %8, 0;\n\t"
      "add.u64 bd, bh, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%7], [at], bd, %11, pa;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [at], bdl, %11, pc;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 8;\n\t"
      "add.u64 bd, bh, 2;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 16;\n\t"
      "add.u64 bd, bh, 4;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [atl], bd, %11, pt;\n\t"
      "add.u32 at, %8, 24;\n\t"
      "add.u64 bd, bh, 6;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%7], [at], bd, %11, pt;\n\t"
      "add.u64 bdl, bd, cl;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [at], bdl, %11, pt;\n\t"
      "add.u32 atl, at, 32;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%13], [atl], bd, %11, pt;\n\t"
      "selp.u32 %0, 1, 0, px;\n\t"
      "selp.u32 %1, 1, 0, pw;\n\t"
      "}"
      : "=r"(rx), "=r"(rw)
      : "r"(nx), "r"(nxp), "r"(nw), "r"(nwp), "r"(first), "r"(dt), "r"(a0), "l"(wd), "r"(chunk16), "r"(idesc),
        "r"(lo16), "r"(dc), "r"(firstc)
      : "memory");
}

struct TcSmem {
  uint8_t* Ws;         // W slots
  float* pre;          // [pre_cap][128]: prefix product over the outer factors per policy
  uint64_t* x_full;    // per A stage: the 16 producer warps wrote X into tensor memory
  uint64_t* done;      // per A stage: the MMAs reading the stage finished (tcgen05.commit)
  uint64_t* w_full;    // per W slot: the bulk copy landed (transaction count)
  uint64_t* w_free;    // per W slot: the MMAs reading the slot finished (tcgen05.commit)
  uint64_t* acc_full;  // all MMAs of a (step, group) GEMM finished
  uint64_t* acc_free;  // the epilogue has read the accumulators
  volatile int* abort_flag;
};

// ------------------------------------------------------ X generation
// X[p, k] for the group's K order (innermost factor last, its size padded to
// DLP = 2^lg) is pre[p][k >> lg] * q_inner[p][k & (DLP-1)], where pre is the
// product of the outer factors' marginals. Producers first write this
// policy's pre values into shared memory (once per step and group); a chunk
// is then one shared-memory read and Q multiplies per thread.
//   MODE 0: DLP <= Q: Q/DLP runs of pre * q_inner[0..DLP), q_inner in registers
//   MODE 1: Q < DLP <= chunk: one run segment at a fixed offset, in registers
//   MODE 2: DLP > chunk: one run segment at a varying offset, read per chunk
// Every parameter used inside the stage loop is copied to a register first:
// the tcgen05 / mbarrier asm statements clobber memory, so a value read from
// the kernel parameters (or any memory) inside the loop would be reloaded
// after each of them.
template <int PREC, int MODE, int DLP>
__device__ __forceinline__ void produce_group(const TcGroup& gr, const TcParams& tp, const EfeParams& p,
                                              const float* __restrict__ q, const TcSmem sm, uint32_t tmem, int warp,
                                              int pl, int qt, int lane, bool active, Ring& ring,
                                              double (&dsum)[16]) {
  using Tr = TcTraits<PREC>;
  constexpr int CH = Tr::kChunk;
  constexpr int Q = CH / 4;
  constexpr int CPS = Tr::kCps;
  constexpr int kPl = Tr::kPlanes;
  constexpr int kQl = MODE == 0 ? DLP : (MODE == 1 ? Q : 1);
  const int lg = gr.lg;
  const int dl = gr.dim[gr.rank - 1];
  const int outer = gr.outer;
  const int nst = tp.nst;
  const int a_col = tp.a_col;
  uint64_t* const done = sm.done;
  uint64_t* const x_full = sm.x_full;
  volatile int* const abort_flag = sm.abort_flag;
  const float* qin = q + p.qs_off[gr.dep[gr.rank - 1]] * kTcTile + pl;
  const float* pre = sm.pre + pl;
  float ql[kQl];
  if (MODE == 0) {
#pragma unroll
    for (int i = 0; i < kQl; ++i) ql[i] = (i < dl && active) ? qin[i * kTcTile] : 0.f;
  } else if (MODE == 1) {
    const int off = (qt * Q) & ((1 << lg) - 1);
#pragma unroll
    for (int i = 0; i < kQl; ++i) ql[i] = (off + i < dl && active) ? qin[(off + i) * kTcTile] : 0.f;
  }
  const uint32_t lane_base = tmem + ((uint32_t)((warp & 3) * 32) << 16);
  const int nstages = gr.nch / CPS;
  // drain mode: this warp's 16 accumulator columns (qt * 16 ..) exist when qt * 16 < N
  const bool drain = tp.drain && qt * 16 < gr.N;
  const uint32_t dcol = (uint32_t)(qt * 16);
  const int N = gr.N;
  for (int c = 0; c < nstages; ++c) {
    const int st = ring.slot;
    if (ring.wrapped) {
      warp_wait(&done[st], ring.phase ^ 1u, abort_flag, lane);
      tc::fence_after_sync();
    }
    if (drain && c >= nst) {
      // slot st holds the hi*hi partial sums of stage c - nst of this GEMM
      // (its MMAs are done): fold them into FP64 before stage c reuses it
      uint32_t r[16];
      tc::tmem_ld16(lane_base + (uint32_t)(st * N) + dcol, r);
      tc::tmem_wait_ld();
#pragma unroll
      for (int k = 0; k < 16; ++k) dsum[k] += (double)__uint_as_float(r[k]);
    }
    const uint32_t ta_st = lane_base + (uint32_t)(a_col + st * 32 * kPl * CPS + qt * 8);
#pragma unroll
    for (int h = 0; h < CPS; ++h) {
      const int k0 = (c * CPS + h) * CH + qt * Q;
      const int ko = k0 >> lg;
      float v[Q];
      if (MODE == 0) {
        constexpr int kRuns = Q / kQl;
#pragma unroll
        for (int run = 0; run < kRuns; ++run) {
          const float pr = (ko + run < outer) ? pre[(ko + run) * kTcTile] : 0.f;
#pragma unroll
          for (int i = 0; i < kQl; ++i) v[run * kQl + i] = pr * ql[i];
        }
      } else if (MODE == 1) {
        const float pr = ko < outer ? pre[ko * kTcTile] : 0.f;
#pragma unroll
        for (int i = 0; i < Q; ++i) v[i] = pr * ql[i];
      } else {
        const int off = k0 & ((1 << lg) - 1);
        const float pr = (ko < outer && active) ? pre[ko * kTcTile] : 0.f;
#pragma unroll
        for (int i = 0; i < Q; ++i) v[i] = (off + i < dl) ? pr * qin[(off + i) * kTcTile] : 0.f;
      }
      // this warp's 32 policy rows (TMEM lanes) x 8 columns of the A stage
      const uint32_t ta = ta_st + (uint32_t)(h * 32 * kPl);
      if (PREC == B2_PRECISION_BF16) {
        // hi = bf16(v), lo = bf16(v - hi): the two planes of the 3-pass split
        uint32_t r[8], rl[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const __nv_bfloat162 h2 = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
          r[e] = *reinterpret_cast<const uint32_t*>(&h2);
          rl[e] = bf16x2_bits(v[2 * e] - __low2float(h2), v[2 * e + 1] - __high2float(h2));
        }
        tc::tmem_st8(ta, r);
        tc::tmem_st8(ta + 32, rl);
      } else {
        uint32_t hi[8], lo[8];
#pragma unroll
        for (int e = 0; e < 8; ++e) {
          const float hv = tf32_round(v[e]);
          hi[e] = __float_as_uint(hv);
          lo[e] = __float_as_uint(tf32_round(v[e] - hv));
        }
        tc::tmem_st8(ta, hi);
        tc::tmem_st8(ta + 32, lo);
      }
    }
    tc::tmem_wait_st();
    tc::fence_before_sync();
    __syncwarp();
    if (lane == 0) mbar_arrive(&x_full[st]);
    ring.next(nst);
  }
}

template <int PREC>
__device__ __forceinline__ void produce_dispatch(const TcGroup& gr, const TcParams& tp, const EfeParams& p,
                                                 const float* __restrict__ q, const TcSmem sm, uint32_t tmem, int warp,
                                                 int pl, int qt, int lane, bool active, Ring& ring,
                                                 double (&dsum)[16]) {
  constexpr int CH = TcTraits<PREC>::kChunk;
  constexpr int Q = CH / 4;
  const int dlp = 1 << gr.lg;
  if (dlp > CH) {
    produce_group<PREC, 2, 1>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum);
  } else if (dlp > Q) {
    produce_group<PREC, 1, 1>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum);
  } else {
    switch (gr.lg) {
      case 0: produce_group<PREC, 0, 1>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum); break;
      case 1: produce_group<PREC, 0, 2>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum); break;
      case 2: produce_group<PREC, 0, 4>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum); break;
      case 3: produce_group<PREC, 0, (Q >= 8 ? 8 : 1)>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum); break;
      default: produce_group<PREC, 0, (Q >= 16 ? 16 : 1)>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum);
    }
  }
}

// Expected states of one policy for one step (pymdp/control.py:351-389):
// thread quarter qt computes next states of every factor. Factors staged
// transposed ([k][u][s], rank-1 parents, S % 4 == 0) are done in blocks of
// four next states: per parent state one broadcast 16-byte load of B and one
// load of the parent marginal. Other factors use the generic strided loop.
__device__ __forceinline__ void rollout_step(const EfeParams& p, const TcParams& tp, const float* __restrict__ Bag,
                                             bool b_staged, const int32_t* __restrict__ u_pol, const float* qc,
                                             float* qn, int pl, int qt) {
  for (int f = 0; f < p.F; ++f) {
    const EfeFactor& fb = p.fac[f];
    const int U = p.U[f];
    const int S = p.S[f];
    const int K = fb.K;
    const int u = jnp_action(u_pol[f], U);
    float* qnf = qn + p.qs_off[f] * kTcTile + pl;
    if (b_staged && tp.b_tr[f]) {
      const float* qv = qc + p.qs_off[fb.dep[0]] * kTcTile + pl;
      const float* Bt = Bag + tp.b_off[f] + u * S;
      const int row = U * S;
      for (int blk = qt * 4; blk < S; blk += 16) {
        float a0 = 0.f, a1 = 0.f, a2 = 0.f, a3 = 0.f;
        const float* bp = Bt + blk;
#pragma unroll 4
        for (int k = 0; k < K; ++k) {
          const float qk = qv[k * kTcTile];
          const float4 w = *reinterpret_cast<const float4*>(bp + k * row);
          a0 = fmaf(w.x, qk, a0);
          a1 = fmaf(w.y, qk, a1);
          a2 = fmaf(w.z, qk, a2);
          a3 = fmaf(w.w, qk, a3);
        }
        qnf[(blk + 0) * kTcTile] = a0;
        qnf[(blk + 1) * kTcTile] = a1;
        qnf[(blk + 2) * kTcTile] = a2;
        qnf[(blk + 3) * kTcTile] = a3;
      }
      continue;
    }
    const float* Bf = Bag + (b_staged ? (int64_t)tp.b_off[f] : fb.B_off);
    for (int s = qt; s < S; s += 4) {
      float acc = 0.f;
      const float* Bs = Bf + (int64_t)s * K * U + u;
      if (fb.rank == 1) {
        const float* qv = qc + p.qs_off[fb.dep[0]] * kTcTile + pl;
        for (int k = 0; k < K; ++k) acc = fmaf(Bs[k * U], qv[k * kTcTile], acc);
      } else {
        int dig[B2_MAX_DEP_RANK];
#pragma unroll
        for (int i = 0; i < B2_MAX_DEP_RANK; ++i) dig[i] = 0;
        for (int k = 0; k < K; ++k) {
          float w = 1.f;
#pragma unroll
          for (int i = 0; i < B2_MAX_DEP_RANK; ++i)
            if (i < fb.rank) w *= qc[(p.qs_off[fb.dep[i]] + dig[i]) * kTcTile + pl];
          acc = fmaf(Bs[k * U], w, acc);
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
      qnf[s * kTcTile] = acc;
    }
  }
}

// pre[ko][pl] = prod over the group's outer factors of q[digit(ko)], for the
// contiguous quarter qt of the ko range; digits advance by one per entry.
__device__ __forceinline__ void build_prefix(const TcGroup& gr, const EfeParams& p, const float* q, float* pre,
                                             int pl, int qt, bool active) {
  const int n = gr.rank - 1;
  const int outer = gr.outer;
  const int per = (outer + 3) >> 2;
  const int ko0 = qt * per;
  const int ko1 = ko0 + per < outer ? ko0 + per : outer;
  if (ko0 >= ko1) return;
  int d[kTcMaxOuter], o[kTcMaxOuter], dig[kTcMaxOuter];
#pragma unroll
  for (int x = 0; x < kTcMaxOuter; ++x) {
    d[x] = x < n ? gr.dim[x] : 1;
    o[x] = x < n ? p.qs_off[gr.dep[x]] * kTcTile + pl : 0;
  }
  int rem = ko0;
#pragma unroll
  for (int x = kTcMaxOuter - 1; x >= 0; --x) {
    const int qd = rem / d[x];
    dig[x] = rem - qd * d[x];
    rem = qd;
  }
  for (int ko = ko0; ko < ko1; ++ko) {
    float v = 1.f;
#pragma unroll
    for (int x = 0; x < kTcMaxOuter; ++x)
      if (x < n) v *= q[o[x] + dig[x] * kTcTile];
    pre[ko * kTcTile + pl] = active ? v : 0.f;
#pragma unroll
    for (int x = kTcMaxOuter - 1; x >= 0; --x) {
      if (++dig[x] < d[x]) break;
      dig[x] = 0;
    }
  }
}

// ------------------------------------------------------------ main kernel
// Warp roles: 0-15 producers (four threads per policy row: state rollout,
// prefix table, X generation into tensor memory, epilogue), 16 = W loader
// (large bulk copies into the W slots), 17 = MMA issuer (kCps * 4 K-steps
// back to back per A stage). The chunk loop has no CTA-wide barrier.
constexpr int kProducers = 512;
constexpr int kThreadsAll = kProducers + 64;

__device__ __forceinline__ void producers_sync() { asm volatile("bar.sync 1, %0;" ::"r"(kProducers) : "memory"); }

template <int PREC>
__global__ void __launch_bounds__(kThreadsAll, 1)
    efe_tc_kernel(const __grid_constant__ EfeParams p, const __grid_constant__ TcParams tp,
                  const int32_t* __restrict__ pm, int pm_batched, const float* __restrict__ qs_init,
                  const float* __restrict__ B, const uint8_t* __restrict__ pack, float* __restrict__ G,
                  double* __restrict__ Gt, const float* __restrict__ Qt) {
  using Tr = TcTraits<PREC>;
  constexpr int kPl = Tr::kPlanes;
  constexpr int CPS = Tr::kCps;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int nst = tp.nst;
  TcSmem sm;
  sm.Ws = base;
  double* red = reinterpret_cast<double*>(sm.Ws + kTcWSlots * tp.ws_bytes);  // [4][128] partial G
  float* qsm = reinterpret_cast<float*>(red + 4 * kTcTile);
  float* bsm = qsm + 2 * p.S_tot * kTcTile;  // this agent's B (when tp.b_words > 0)
  sm.pre = bsm + tp.b_words;                 // [pre_cap][128]
  sm.x_full = reinterpret_cast<uint64_t*>(sm.pre + tp.pre_cap * kTcTile);
  sm.done = sm.x_full + kTcMaxAStages;
  sm.w_full = sm.done + kTcMaxAStages;
  sm.w_free = sm.w_full + kTcWSlots;
  sm.acc_full = sm.w_free + kTcWSlots;
  sm.acc_free = sm.acc_full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sm.acc_free + 1);
  sm.abort_flag = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t b = blockIdx.y;
  // steps this CTA evaluates and its first row (a policy, or a prefix at depth t_lo in tree mode)
  int t_lo = 0, t_hi = p.T, row0 = blockIdx.x * kTcTile;
  if (tp.tree) {
    int t = 0;
    while (t + 1 < p.T && (int)blockIdx.x >= tp.tree_tiles[t + 1]) ++t;
    t_lo = t;
    t_hi = t + 1;
    row0 = ((int)blockIdx.x - tp.tree_tiles[t]) * kTcTile;
  }

  if (warp == 0) tc::tmem_alloc(tmem_slot, (uint32_t)tp.tmem_cols);
  if (tid == 0) {
    for (int s = 0; s < nst; ++s) {
      tc::mbar_init(&sm.x_full[s], kProducers / 32);
      tc::mbar_init(&sm.done[s], 1);
    }
    for (int s = 0; s < kTcWSlots; ++s) {
      tc::mbar_init(&sm.w_full[s], 1);
      tc::mbar_init(&sm.w_free[s], 1);
    }
    tc::mbar_init(sm.acc_full, 1);
    tc::mbar_init(sm.acc_free, kProducers / 32);
    tc::fence_mbar_init();
    *sm.abort_flag = 0;
  }
  for (int i = tid; i < p.S_tot * kTcTile; i += blockDim.x) qsm[i] = __ldg(qs_init + b * p.S_tot + i / kTcTile);
  if (tp.b_words > 0) {
    // stage B: transposed [k][u][s] where the rollout reads it that way
    for (int f = 0; f < p.F; ++f) {
      const EfeFactor& fb = p.fac[f];
      const int S = p.S[f], K = fb.K, U = p.U[f];
      const int n = S * K * U;
      const float* src = B + b * p.B_stride + fb.B_off;
      float* dst = bsm + tp.b_off[f];
      const bool tr = tp.b_tr[f] != 0;
      for (int i = tid; i < n; i += blockDim.x) {
        const float v = __ldg(src + i);
        if (tr) {
          const int s = i / (K * U);
          const int r = i - s * (K * U);
          const int k = r / U;
          const int u = r - k * U;
          dst[(k * U + u) * S + s] = v;
        } else {
          dst[i] = v;
        }
      }
    }
  }
  const float* Bag = tp.b_words > 0 ? bsm : B + b * p.B_stride;
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;

  if (warp == kProducers / 32) {
    // ---------------- W loader: large bulk copies into the W slots
    if (lane == 0) {
      const int G = tp.G, wch = tp.wch, ws_bytes = tp.ws_bytes;
      uint64_t* const w_full = sm.w_full;
      uint64_t* const w_free = sm.w_free;
      volatile int* const abort_flag = sm.abort_flag;
      const uint32_t ws0 = tc::smem_u32(sm.Ws);
      const uint8_t* const pack_b = pack + b * tp.pack_stride;
      Ring wr;
      for (int t = t_lo; t < t_hi; ++t)
        for (int g = 0; g < G; ++g) {
          const int nch = tp.grp[g].nch, chunk_bytes = tp.grp[g].chunk_bytes;
          const uint8_t* wimg = pack_b + tp.grp[g].pack_off;
          for (int c0 = 0; c0 < nch; c0 += wch) {
            const int cnt = nch - c0 < wch ? nch - c0 : wch;
            const uint32_t bytes = (uint32_t)(cnt * chunk_bytes);
            const int s = wr.slot;
            const bool ok = !wr.wrapped || wait_or_abort(&w_free[s], wr.phase ^ 1u, abort_flag);
            if (ok && !*abort_flag) {  // otherwise waiters give up through the abort flag
              mbar_expect_tx(&w_full[s], bytes);
              bulk_g2s(ws0 + (uint32_t)(s * ws_bytes), wimg + (int64_t)c0 * chunk_bytes, bytes, &w_full[s]);
            }
            wr.next(kTcWSlots);
          }
        }
    }
  } else if (warp == kProducers / 32 + 1) {
    // ---------------- MMA issuer
    if (lane == 0) {
      const uint64_t wdesc0 = tc::desc_kmajor_sw128(tc::smem_u32(sm.Ws));
      const uint32_t acol0 = tmem + (uint32_t)tp.a_col;
      const int G = tp.G, wch = tp.wch, nacc = tp.nacc, corr = tp.corr, drain = tp.drain;
      const uint32_t ws16 = (uint32_t)tp.ws_bytes >> 4;
      uint64_t* const x_full = sm.x_full;
      uint64_t* const done = sm.done;
      uint64_t* const w_full = sm.w_full;
      uint64_t* const w_free = sm.w_free;
      uint64_t* const acc_full = sm.acc_full;
      uint64_t* const acc_free = sm.acc_free;
      volatile int* const abort_flag = sm.abort_flag;
      static_assert(PREC != B2_PRECISION_BF16 || CPS == 2, "issue_stage_bf16 covers 2 chunks");
      static_assert(PREC != B2_PRECISION_TF32X3 || CPS == 1, "issue_stage_tf32x3 covers 1 chunk");
      Ring ar, wr;
      uint32_t j = 0;
      // results of the look-ahead barrier tests made while issuing the
      // previous stage (false: wait here)
      uint32_t x_ready = 0, w_ready = 0;
      for (int t = t_lo; t < t_hi; ++t)
        for (int g = 0; g < G; ++g, ++j) {
          const uint32_t idesc = tp.grp[g].idesc;
          const int N = tp.grp[g].N, nch = tp.grp[g].nch;
          const uint32_t chunk16 = (uint32_t)tp.grp[g].chunk_bytes >> 4;  // descriptor units per chunk tile
          const uint32_t lo16 = (uint32_t)(N * 128) >> 4;                 // descriptor units to the lo plane
          const int nstages = nch / CPS;
          if (j > 0) wait_or_abort(acc_free, (j - 1) & 1, abort_flag);
          int acc_slot = 0;
          bool w_ok = true;
          int wk = 0;  // position of the current A stage's first chunk in its W slot
          for (int c = 0; c < nstages; ++c) {
            const int kc = c * CPS;  // first chunk of this A stage (group-relative)
            if (wk == 0) w_ok = w_ready ? true : wait_or_abort(&w_full[wr.slot], wr.phase, abort_flag);
            const int st = ar.slot;
            const bool okx = x_ready ? true : wait_or_abort(&x_full[st], ar.phase, abort_flag);
            // where the next stage's X and (if it opens a W slot) W arrive
            const bool w_last = wk + CPS == wch || kc + CPS == nch;  // this stage ends its W slot
            Ring nar = ar, nwr = wr;
            nar.next(nst);
            if (w_last) nwr.next(kTcWSlots);
            const uint32_t nx = tc::smem_u32(&x_full[nar.slot]);
            const uint32_t nw = w_last ? tc::smem_u32(&w_full[nwr.slot]) : nx;
            uint32_t rx = 0, rw = 0;
            if (okx && w_ok && !*abort_flag) {
              tc::fence_after_sync();
              // stage c accumulates into accumulator c % nacc: shorter FP32
              // accumulation chains inside the tensor core
              // drain mode: a fresh accumulator per stage, the stage's own ring slot
              const uint32_t dt = tmem + (uint32_t)((drain ? st : acc_slot) * N);
              const uint32_t first = drain ? 0u : (c < nacc ? 0u : 1u);
              const uint64_t wd = wdesc0 + (uint64_t)((uint32_t)wr.slot * ws16 + (uint32_t)wk * chunk16);
              const uint32_t a0 = acol0 + (uint32_t)(st * 32 * kPl * CPS);
              // correction products: their own accumulator (first use at stage 0), or dt's chain
              const uint32_t dc = corr >= 0 ? tmem + (uint32_t)(corr * N) : dt;
              const uint32_t firstc = corr >= 0 ? (c == 0 ? 0u : 1u) : 1u;
              if (PREC == B2_PRECISION_BF16)
                issue_stage_bf16(dt, dc, a0, wd, chunk16, idesc, first, firstc, nx, nar.phase, nw, nwr.phase, lo16,
                                 rx, rw);
              else
                issue_stage_tf32x3(dt, dc, a0, wd, chunk16, idesc, first, firstc, nx, nar.phase, nw, nwr.phase,
                                   lo16, rx, rw);
            }
            x_ready = rx;
            w_ready = w_last ? rw : 1u;
            // always arm the barriers so every waiter makes progress
            tc::mma_commit(&done[st]);
            ar = nar;
            wk += CPS;
            if (w_last) {
              tc::mma_commit(&w_free[wr.slot]);
              wr = nwr;
              wk = 0;
            }
            if (++acc_slot == nacc) acc_slot = 0;
          }
          tc::mma_commit(acc_full);
        }
    }
  } else {
    // ---------------- producers (warps 0-15): policy pl, quarter qt
    const int pl = tid & (kTcTile - 1);
    const int qt = tid >> 7;
    const int pol = row0 + pl;  // policy, or prefix at depth t_lo in tree mode
    const int n_rows = tp.tree ? (int)(tp.tree_off[t_lo + 1] - tp.tree_off[t_lo]) : p.P;
    const bool active = pol < n_rows;
    // the row's actions: a prefix's are those of its first policy
    const int64_t pol_act = tp.tree ? (int64_t)pol * tp.tree_w[t_lo] : pol;
    const bool ig = (p.flags & B2_FLAG_USE_STATES_INFO_GAIN) != 0;
    double g_acc = 0.0;
    int cur = 0;
    Ring ring;
    uint32_t j = 0;
    const int32_t* u_base = pm + (pm_batched ? b * (int64_t)p.P * p.T * p.F : 0) + (active ? pol_act : 0) * p.T * p.F;
    for (int t = 0; t < t_hi; ++t) {
      if (tp.tree) {
        // the parents' marginals (depth t - 1) were rolled out once per agent by
        // efe_tree_rollout_kernel; qsm already holds qs_init for depth 0
        if (t < t_lo) continue;
        if (t > 0) {
          const int64_t prow = tp.tree_off[t - 1] + (active ? pol / tp.tree_nu : 0);
          const float* qrow = Qt + (b * tp.tree_off[p.T - 1] + prow) * p.S_tot;
          float* qd = qsm + cur * p.S_tot * kTcTile;
          for (int s2 = qt; s2 < p.S_tot; s2 += 4) qd[s2 * kTcTile + pl] = __ldg(qrow + s2);
          producers_sync();
        }
      }
      rollout_step(p, tp, Bag, tp.b_words > 0, u_base + t * p.F, qsm + cur * p.S_tot * kTcTile,
                   qsm + (cur ^ 1) * p.S_tot * kTcTile, pl, qt);
      producers_sync();
      cur ^= 1;
      if (t < t_lo) continue;  // (per-policy mode never skips)
      const float* q = qsm + cur * p.S_tot * kTcTile;
      for (int g = 0; g < tp.G; ++g, ++j) {
        const TcGroup& gr = tp.grp[g];
        build_prefix(gr, p, q, sm.pre, pl, qt, active);
        producers_sync();
        double dsum[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) dsum[k] = 0.0;
        const int s_first = ring.slot;  // ring slot of this GEMM's first A stage
        produce_dispatch<PREC>(gr, tp, p, q, sm, tmem, warp, pl, qt, lane, active, ring, dsum);
        // epilogue: warp w reads TMEM lane quarter (w & 3) = its 32 policies,
        // 16-column blocks qt*16, qt*16 + 64, ... of every accumulator
        const int N = gr.N, n_obs = gr.n_obs;
        // accumulators in use: main slots 0 .. nacc-1, then the correction slot
        const int nacc = gr.nch / CPS < tp.nacc ? gr.nch / CPS : tp.nacc;
        const int corr = tp.corr;
        const int nsum = nacc + (corr >= 0 ? 1 : 0);
        warp_wait(sm.acc_full, j & 1, sm.abort_flag, lane);
        tc::fence_after_sync();
        {
          const uint32_t taddr = tmem + ((uint32_t)((warp & 3) * 32) << 16);
          double h = 0.0, lin = 0.0;
          auto consume = [&](int n0, const double (&sum)[16]) {
#pragma unroll
            for (int k = 0; k < 16; ++k) {
              const int n = n0 + k;
              if (n < n_obs) {
                if (ig) h -= sum[k] * (double)logf(fmaxf((float)sum[k], kMinVal));
              } else if (n == n_obs + t) {
                lin = sum[k];
              }
            }
          };
          if (tp.drain) {
            if (qt * 16 < N) {
              // the stages still in their slots (the last nst), then the correction accumulator
              const int nst = tp.nst, nstages = gr.nch / CPS;
              for (int c = nstages > nst ? nstages - nst : 0; c < nstages; ++c) {
                uint32_t r[16];
                tc::tmem_ld16(taddr + (uint32_t)(((s_first + c) % nst) * N + qt * 16), r);
                tc::tmem_wait_ld();
#pragma unroll
                for (int k = 0; k < 16; ++k) dsum[k] += (double)__uint_as_float(r[k]);
              }
              uint32_t r[16];
              tc::tmem_ld16(taddr + (uint32_t)(corr * N + qt * 16), r);
              tc::tmem_wait_ld();
#pragma unroll
              for (int k = 0; k < 16; ++k) dsum[k] += (double)__uint_as_float(r[k]);
              consume(qt * 16, dsum);
            }
          } else {
          for (int n0 = qt * 16; n0 < N; n0 += 64) {
            double sum[16];
#pragma unroll
            for (int k = 0; k < 16; ++k) sum[k] = 0.0;
            int a = 0;
            for (; a + 1 < nsum; a += 2) {
              const int s0 = a, s1 = a + 1 < nacc ? a + 1 : corr;
              uint32_t r0[16], r1[16];
              tc::tmem_ld16(taddr + (uint32_t)(s0 * N + n0), r0);
              tc::tmem_ld16(taddr + (uint32_t)(s1 * N + n0), r1);
              tc::tmem_wait_ld();
#pragma unroll
              for (int k = 0; k < 16; ++k) sum[k] += (double)__uint_as_float(r0[k]) + (double)__uint_as_float(r1[k]);
            }
            if (a < nsum) {
              const int s0 = a < nacc ? a : corr;
              uint32_t r0[16];
              tc::tmem_ld16(taddr + (uint32_t)(s0 * N + n0), r0);
              tc::tmem_wait_ld();
#pragma unroll
              for (int k = 0; k < 16; ++k) sum[k] += (double)__uint_as_float(r0[k]);
            }
            consume(n0, sum);
          }
          }
          g_acc += h + lin;
        }
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) mbar_arrive(sm.acc_free);
        producers_sync();  // every producer is done with this group's prefix table
      }
    }
    red[qt * kTcTile + pl] = g_acc;
    producers_sync();
    if (qt == 0 && active && !*sm.abort_flag) {
      const double gsum = ((red[pl] + red[kTcTile + pl]) + red[2 * kTcTile + pl]) + red[3 * kTcTile + pl];
      if (tp.tree)
        Gt[b * tp.tree_off[p.T] + tp.tree_off[t_lo] + pol] = gsum;
      else
        G[b * p.P + pol] = (float)gsum;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (*sm.abort_flag && tid == 0) atomicExch(&g_b2_device_error, 1);
  if (warp == 0) tc::tmem_dealloc(tmem, (uint32_t)tp.tmem_cols);
}

}  // namespace

// Policy-tree mode: the marginals of every distinct policy prefix of depth
// 0 .. T-2, depth by depth, once per agent (one CTA): Qt[t][c][j] =
// (B_f[..., u_t(c)] . joint of the parent prefix's marginals over f's B
// dependencies)[s], the parent of prefix c at depth t being c / prod(U) at
// depth t - 1 (qs_init at t = 0). The deepest level is rolled out inside
// efe_tc_kernel, from these.
__global__ void __launch_bounds__(512) efe_tree_rollout_kernel(const __grid_constant__ EfeParams p,
                                                              const __grid_constant__ TcParams tp,
                                                              const float* __restrict__ qs_init,
                                                              const float* __restrict__ B, float* __restrict__ Qt) {
  const int64_t b = blockIdx.x;
  const int St = p.S_tot, nu = tp.tree_nu;
  float* Qb = Qt + b * tp.tree_off[p.T - 1] * St;
  const float* Bb = B + b * p.B_stride;
  int ustride[kEfeMaxF];
  int us = 1;
  for (int f = p.F - 1; f >= 0; --f) {
    ustride[f] = us;
    us *= p.U[f];
  }
  for (int t = 0; t + 1 < p.T; ++t) {
    const int n = (int)(tp.tree_off[t + 1] - tp.tree_off[t]);
    float* out = Qb + tp.tree_off[t] * St;
    for (int e = threadIdx.x; e < n * St; e += blockDim.x) {
      const int c = e / St;
      const int j = e - c * St;
      int f = 0;
      while (f + 1 < p.F && j >= p.qs_off[f + 1]) ++f;
      const int s = j - p.qs_off[f], U = p.U[f];
      const int u = ((c % nu) / ustride[f]) % U;
      const float* q = t == 0 ? qs_init + b * St : Qb + (tp.tree_off[t - 1] + c / nu) * St;
      const EfeFactor& fb = p.fac[f];
      const float* Bs = Bb + fb.B_off + (int64_t)s * fb.K * U + u;
      float acc = 0.f;
      if (fb.rank == 1) {
        const float* qv = q + p.qs_off[fb.dep[0]];
        for (int k = 0; k < fb.K; ++k) acc = fmaf(__ldg(Bs + (int64_t)k * U), qv[k], acc);
      } else {
        int dig[B2_MAX_DEP_RANK];
#pragma unroll
        for (int i = 0; i < B2_MAX_DEP_RANK; ++i) dig[i] = 0;
        for (int k = 0; k < fb.K; ++k) {
          float w = 1.f;
#pragma unroll
          for (int i = 0; i < B2_MAX_DEP_RANK; ++i)
            if (i < fb.rank) w *= q[p.qs_off[fb.dep[i]] + dig[i]];
          acc = fmaf(__ldg(Bs + (int64_t)k * U), w, acc);
          bool carry = true;
#pragma unroll
          for (int i = B2_MAX_DEP_RANK - 1; i >= 0; --i) {
            if (carry && i < fb.rank) {
              if (++dig[i] < p.S[fb.dep[i]])
                carry = false;
              else
                dig[i] = 0;
            }
          }
        }
      }
      out[(int64_t)c * St + j] = acc;
    }
    __syncthreads();
  }
}

// Policy-tree mode: G[p] = sum_t g_t[p / prod(U)^(T-1-t)] from the per-prefix
// step values (FP64).
__global__ void efe_tree_combine_kernel(const __grid_constant__ TcParams tp, int T, int P,
                                        const double* __restrict__ Gt, float* __restrict__ G) {
  const int64_t b = blockIdx.y;
  const int pol = blockIdx.x * blockDim.x + threadIdx.x;
  if (pol >= P) return;
  const double* g = Gt + b * tp.tree_off[T];
  double s = 0.0;
  for (int t = 0; t < T; ++t) s += g[tp.tree_off[t] + pol / tp.tree_w[t]];
  G[b * P + pol] = (float)s;
}

// Plan the tensor-core path; returns B2_ERR_UNSUPPORTED when the model falls
// outside its limits (the caller then uses the SIMT kernel).
template <int PREC>
int32_t tc_plan_t(const EfeParams& p, TcParams* tp, int* smem_bytes) {
  using Tr = TcTraits<PREC>;
  std::memset(tp, 0, sizeof(*tp));
  const int chunk = Tr::kChunk;
  const int planes = Tr::kPlanes;
  const int cps = Tr::kCps;
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
  int Nmax = 16, outer_max = 1;
  for (int g = 0; g < tp->G; ++g) {
    TcGroup& gr = tp->grp[g];
    const std::vector<int>& tup = tuples[g];
    const int r = (int)tup.size();
    if (r > kTcMaxOuter + 1) return B2_ERR_UNSUPPORTED;
    gr.rank = r;
    // innermost factor: the largest padded size that fits one chunk (its
    // marginal then stays in registers), else the largest overall; either way
    // the shared prefix table (K / innermost entries) is as small as possible
    int best = r - 1, best_p = -1;
    for (int a = 0; a < r; ++a) {
      int pw = 1;
      while (pw < p.S[tup[a]]) pw <<= 1;
      const int score = pw <= chunk ? 4 * pw : pw / 1024;
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
    outer_max = gr.outer > outer_max ? gr.outer : outer_max;
    const int64_t Kp = (int64_t)gr.outer << lg;
    const int64_t step = (int64_t)chunk * cps;
    gr.Kpad = (int32_t)((Kp + step - 1) / step * step);
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
    gr.idesc = tc::idesc_f32acc(PREC == B2_PRECISION_BF16 ? 1u : 2u, 128u, (uint32_t)gr.N);
    gr.chunk_bytes = planes * gr.N * 128;
    gr.pack_off = off;
    off += (int64_t)gr.nch * gr.chunk_bytes;
  }
  tp->Nmax = Nmax;
  // A stages in tensor memory: as many as leave room for at least 2
  // accumulators (BF16) / 5 (3xTF32, whose FP32 accumulation chains must stay
  // short), within the trait's maximum.
  const int stage_cols = 32 * planes * cps;  // 128 lanes x 128 bytes per plane per chunk
  tp->drain = 0;
  tp->corr = -1;
  tp->tmem_cols = 512;
  if (Nmax <= 64 && (Tr::kMaxNst + 1) * Nmax + Tr::kMaxNst * stage_cols <= 512) {
    // Drain mode (3xTF32 and 3-pass BF16): stage s's hi*hi products go to accumulator slot
    // (ring slot of s), fresh each stage, and the producers fold it into FP64
    // before the slot's next use; one more accumulator holds the correction
    // products (hi*lo + lo*hi, about 2^-11 of the result) of the whole GEMM.
    // The tensor core's FP32 accumulation (which does not round to nearest)
    // then runs over the 4 MMAs of one stage instead of the whole K range.
    tp->drain = 1;
    tp->nst = Tr::kMaxNst;
    tp->nacc = Tr::kMaxNst;
    tp->corr = Tr::kMaxNst;
    tp->a_col = ((Tr::kMaxNst + 1) * Nmax + 31) / 32 * 32;
  } else {
    // Rotation mode: A stages in tensor memory, as many as leave room for at
    // least 2 accumulators (BF16) / 5 (3xTF32) within the trait's maximum;
    // consecutive stages rotate over the accumulators (shorter FP32 chains).
    const int want_acc = PREC == B2_PRECISION_BF16 ? 2 : 5;
    int nst = Tr::kMaxNst;
    while (nst > 2 && 512 - nst * stage_cols < want_acc * Nmax) --nst;
    int nacc = (512 - nst * stage_cols) / Nmax;
    nacc = nacc > 8 ? 8 : nacc;
    if (nacc < 1) return B2_ERR_UNSUPPORTED;
    tp->nst = nst;
    tp->a_col = (nacc * Nmax + 31) / 32 * 32;
    // the correction products share one accumulator of their own when there
    // is room, so the main chains hold hi*hi products only (a third of the MMAs)
    if (nacc >= 3) {
      tp->corr = nacc - 1;
      nacc -= 1;
    }
    tp->nacc = nacc;
  }
  if (tp->a_col + tp->nst * stage_cols > 512) return B2_ERR_UNSUPPORTED;
  // W slots: whole A stages, about kTcWSlotTarget bytes per bulk copy
  const int chunk_max = planes * Nmax * 128;
  int wch = kTcWSlotTarget / chunk_max / cps * cps;
  if (wch < cps) wch = cps;
  tp->wch = wch;
  tp->ws_bytes = wch * chunk_max;
  tp->pre_cap = (outer_max + 1) / 2 * 2;
  tp->pack_stride = (off + 1023) / 1024 * 1024;
  int64_t smem = 1024 + (int64_t)kTcWSlots * tp->ws_bytes + 4LL * kTcTile * 8 + 2LL * p.S_tot * kTcTile * 4 +
                 (int64_t)tp->pre_cap * kTcTile * 4 + (2 * kTcMaxAStages + 2 * kTcWSlots + 2) * 8 + 16;
  if (smem > 227 * 1024) return B2_ERR_UNSUPPORTED;
  // B staged per factor at 16-byte aligned offsets (transposed where the
  // rollout's vector path applies)
  int64_t b_words = 0;
  for (int f = 0; f < p.F; ++f) {
    tp->b_off[f] = (int32_t)b_words;
    tp->b_tr[f] = (p.fac[f].rank == 1 && p.S[f] % 4 == 0) ? 1 : 0;
    b_words += ((int64_t)p.S[f] * p.fac[f].K * p.U[f] + 3) / 4 * 4;
  }
  if (smem + b_words * 4 <= 227 * 1024 && b_words < (1 << 30)) {
    tp->b_words = (int32_t)b_words;
    smem += b_words * 4;
  } else {
    tp->b_words = 0;
    std::memset(tp->b_tr, 0, sizeof(tp->b_tr));
  }
  *smem_bytes = (int)smem;
  return B2_OK;
}

template <int PREC>
int32_t launch_tc_t(const EfeParams& p, int64_t Bn, const int32_t* pm, int pm_batched, const float* qs,
                    const float* A, const float* B, const float* C, float* G, cudaStream_t stream, bool* used,
                    const PackCache* cache) {
  TcParams tp;
  int smem = 0;
  if (tc_plan_t<PREC>(p, &tp, &smem) != B2_OK) return B2_OK;
  // policy tree: a shared full product policy set with T >= 2
  if ((p.flags & B2_FLAG_POLICY_TREE) && !pm_batched && p.T >= 2 && p.T <= kTcMaxT) {
    int64_t nu = 1, P = 1;
    for (int f = 0; f < p.F; ++f) nu *= p.U[f];
    for (int t = 0; t < p.T && P <= p.P; ++t) P *= nu;
    if (P == p.P && nu > 1) {
      tp.tree = 1;
      tp.tree_nu = (int32_t)nu;
      int64_t n = 1;
      tp.tree_tiles[0] = 0;
      tp.tree_off[0] = 0;
      for (int t = 0; t < p.T; ++t) {
        n *= nu;
        tp.tree_tiles[t + 1] = tp.tree_tiles[t] + (int32_t)((n + kTcTile - 1) / kTcTile);
        tp.tree_off[t + 1] = tp.tree_off[t] + n;
        tp.tree_w[t] = p.P / n;
      }
      // the prefix roll-out kernel indexes (prefix, state) pairs of one depth in 32 bits
      if ((double)tp.tree_off[p.T - 1] * p.S_tot >= 2.0e9) tp.tree = 0;
    }
  }
  if (cache && (reinterpret_cast<uintptr_t>(cache->buf) & 255u) != 0)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": pack cache must be 256-byte aligned");
  if (cache && cache->bytes < Bn * tp.pack_stride)
    return fail(B2_ERR_INVALID_ARGUMENT, std::string(kEfeName) + ": pack cache of " + std::to_string(cache->bytes) +
                                             " bytes, needs " + std::to_string(Bn * tp.pack_stride));
  const size_t pack_bytes = cache ? 0 : (size_t)Bn * (size_t)tp.pack_stride;
  const size_t gt_bytes = tp.tree ? (size_t)Bn * (size_t)tp.tree_off[p.T] * sizeof(double) : 0;
  const size_t qt_bytes =
      tp.tree ? ((size_t)Bn * (size_t)tp.tree_off[p.T - 1] * (size_t)p.S_tot * sizeof(float) + 255) / 256 * 256 : 0;
  uint8_t* ws = nullptr;
  if (pack_bytes + gt_bytes + qt_bytes > 0)
    B2_TRY(ws_alloc((void**)&ws, pack_bytes + gt_bytes + qt_bytes, stream, kEfeName));
  uint8_t* pack = cache ? cache->buf : ws;
  double* Gt = tp.tree ? reinterpret_cast<double*>(ws + pack_bytes) : nullptr;
  float* Qt = tp.tree ? reinterpret_cast<float*>(ws + pack_bytes + gt_bytes) : nullptr;
  int Kmax = 0;
  for (int g = 0; g < tp.G; ++g) Kmax = tp.grp[g].Kpad > Kmax ? tp.grp[g].Kpad : Kmax;
  dim3 pgrid((unsigned)((Kmax + 127) / 128), (unsigned)tp.G, (unsigned)Bn);
  dim3 grid((unsigned)(tp.tree ? tp.tree_tiles[p.T] : (p.P + kTcTile - 1) / kTcTile), (unsigned)Bn);
  int32_t rc = B2_OK;
  if (!cache || *cache->valid == 0) {
    efe_tc_pack_kernel<PREC><<<pgrid, 128, 0, stream>>>(p, tp, A, C, pack);
    rc = check_launch("efe_ffi tc pack");
    if (rc == B2_OK && cache) *cache->valid = 1;
  }
  if (rc == B2_OK && tp.tree) {
    efe_tree_rollout_kernel<<<(unsigned)Bn, 512, 0, stream>>>(p, tp, qs, B, Qt);
    rc = check_launch("efe_ffi tc tree rollout");
  }
  if (rc == B2_OK) rc = ensure_smem_attr((const void*)efe_tc_kernel<PREC>, smem, kEfeName);
  if (rc == B2_OK) {
    efe_tc_kernel<PREC><<<grid, kThreadsAll, smem, stream>>>(p, tp, pm, pm_batched, qs, B, pack, G, Gt, Qt);
    rc = check_launch("efe_ffi tc");
  }
  if (rc == B2_OK && tp.tree) {
    efe_tree_combine_kernel<<<dim3((unsigned)((p.P + 255) / 256), (unsigned)Bn), 256, 0, stream>>>(tp, p.T, p.P, Gt,
                                                                                                   G);
    rc = check_launch("efe_ffi tc tree combine");
  }
  if (ws) {
    cudaError_t fe = cudaFreeAsync(ws, stream);
    if (rc == B2_OK && fe != cudaSuccess) return cuda_fail(kEfeName, fe);
  }
  *used = rc == B2_OK;
  return rc;
}

int64_t efe_tc_pack_bytes(const EfeParams& p, int prec, int64_t Bn) {
  TcParams tp;
  int smem = 0;
  if (Bn > 65535 || (prec != B2_PRECISION_BF16 && prec != B2_PRECISION_TF32X3)) return 0;
  const int32_t rc = prec == B2_PRECISION_BF16 ? tc_plan_t<B2_PRECISION_BF16>(p, &tp, &smem)
                                               : tc_plan_t<B2_PRECISION_TF32X3>(p, &tp, &smem);
  return rc == B2_OK ? Bn * tp.pack_stride : 0;
}

int32_t launch_efe_tc(const EfeParams& p, int prec, int64_t Bn, const int32_t* pm, int pm_batched, const float* qs,
                      const float* A, const float* B, const float* C, float* G, cudaStream_t stream,
                      bool* used, const PackCache* cache) {
  *used = false;
  if (Bn > 65535) return B2_OK;
  if (prec == B2_PRECISION_BF16)
    return launch_tc_t<B2_PRECISION_BF16>(p, Bn, pm, pm_batched, qs, A, B, C, G, stream, used, cache);
  return launch_tc_t<B2_PRECISION_TF32X3>(p, Bn, pm, pm_batched, qs, A, B, C, G, stream, used, cache);
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
