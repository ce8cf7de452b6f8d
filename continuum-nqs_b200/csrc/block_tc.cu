// block_tc.cu — one whole transformer block for single-channel (value) rows in one launch, on the
// tcgen05 tensor cores.
//
//   x += MHA(LN0(x));  x += Dense1(GELU(Dense0(LN1(x))))       (src/nqs/psiformer.py:50-81)
//
// Value rows are the Metropolis passes: one channel per token, so every token row is independent
// up to the attention, which mixes only the N tokens of one walker. A 128-row tile holds
// floor(128 / N) whole walkers. Per tile, the residual stream stays in registers (one row per
// thread), every Dense layer is one tcgen05.mma kind::tf32 chain over the tile (activations
// written by the threads into a 128B-swizzled K-major operand tile, the layer's W^T resident in
// shared memory for the CTA's lifetime, float32 accumulators in TMEM), and the attention runs on
// the CUDA cores from one head's K and V rows staged in shared memory. The only HBM traffic is
// the tile's rows in and out, instead of ~13 activation round trips for the unfused block.
//
// CTA: two warpgroups, each owning one tile at a time (their tiles interleave on the SM so one
// group's math hides the other's MMA and load latency) and its own TMEM columns; thread 0 of a
// group issues that group's MMAs and commits them to the group's mbarrier. All waits are bounded
// (tc_common.cuh); a timed-out wait aborts the CTA and sets *err.
//
// Operand precision: TF32 (float32 operand tiles and W^T, kind::tf32) or BF16 (the threads write
// the operand tiles in BF16 and W^T is staged in BF16, both rounded to nearest even; kind::f16,
// float32 accumulation; width 64 only, where every K is a multiple of 64).
#include <cuda_bf16.h>
#include <cstdio>
#include <algorithm>
#include <vector>

#include "net.cuh"
#include "tc_common.cuh"

namespace nqs {
namespace tc {

template <int D, int HD, bool BF = false>
struct BlkCfg {
  static constexpr int FF = 2 * D, H = D / HD, NQKV = 3 * D;
  static constexpr int ES = BF ? 2 : 4;                // operand element bytes
  static constexpr int KB = D * ES / 128;              // 128-byte K-blocks of a D-wide operand
  static constexpr int W_QKV = NQKV * D * ES, W_O = D * D * ES, W_0 = FF * D * ES,
                       W_1 = D * FF * ES;
  static constexpr int W_BYTES = W_QKV + W_O + W_0 + W_1;
  static constexpr int A_BYTES = 128 * D * 4;          // operand tile / row staging
  static constexpr int KV_BYTES = 2 * 128 * HD * 4;    // one head's K and V rows
  static constexpr int G_BYTES = A_BYTES + KV_BYTES;
  static constexpr int SMEM = W_BYTES + 2 * G_BYTES + 128 + 1024;
  static constexpr int TCOLS = D == 64 ? 256 : 128;    // TMEM columns per group
  // TMEM columns: QKV [0, 3D); attention projection [3D, 4D); up [0, FF); down [FF, FF + D)
  static constexpr int C_O = NQKV, C_UP = 0, C_DN = FF;
  static_assert(C_O + D <= TCOLS && C_DN + D <= TCOLS, "TMEM columns");
  static_assert(W_QKV % 1024 == 0 && W_O % 1024 == 0 && W_0 % 1024 == 0 && A_BYTES % 1024 == 0 &&
                    KV_BYTES % 1024 == 0,
                "1024-byte aligned operand regions");
  static_assert(SMEM <= 232448, "shared memory per CTA");
};

struct BlkArgs {
  const float *wqkv, *bqkv, *wo, *bo, *w0, *b0, *w1, *b1;
  const float *ln0_s, *ln0_b, *ln1_s, *ln1_b;
  float* X;  // [rows][D], updated in place
  int rows, N, rpt, ntiles;
  int* err;
  uint32_t wait_limit;
};

// TMEM -> registers, 32 lanes x NC columns (one column per register); completes with tmem_wait
template <int NC>
__device__ __forceinline__ void tmem_ld(uint32_t taddr, float (&v)[NC]) {
  uint32_t* r = reinterpret_cast<uint32_t*>(v);
  if constexpr (NC == 8) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
  } else if constexpr (NC == 16) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
  } else {
    static_assert(NC == 32, "8, 16 or 32 columns");
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
        "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
          "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
          "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
          "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
  }
}
__device__ __forceinline__ void tmem_wait() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void group_bar(int g) {
  asm volatile("bar.sync %0, 128;" ::"r"(1 + g) : "memory");
}
// group barrier that also ORs a predicate over the group's 128 threads (uniform decisions)
__device__ __forceinline__ bool group_bar_or(int g, bool pred) {
  uint32_t res;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}"
      : "=r"(res)
      : "r"((uint32_t)pred), "r"(1 + g)
      : "memory");
  return res != 0;
}
// read-only parameter loads kept inside the tile loop (not hoisted into registers across tiles)
// and kept in L1 (evict_last), where they stay hot for every tile of the CTA
__device__ __forceinline__ float4 ldp4(const float* p) {
  float4 v;
  asm volatile("ld.global.nc.L1::evict_last.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}
// activation rows are read once: no L1 allocation, so they do not evict the parameters
__device__ __forceinline__ float4 ld_stream4(const float4* p) {
  float4 v;
  asm volatile("ld.global.L1::no_allocate.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
               : "l"(p));
  return v;
}
// K / V staging rows: 16-byte chunk c of row r sits at chunk c ^ kv_sw(r), so that the 8 rows
// of one store phase hit 8 different bank groups
template <int HD>
__device__ __forceinline__ int kv_sw(int r) {
  return HD == 16 ? ((r >> 1) & 3) : ((r >> 2) & 1);
}
// tanh-GELU as x sigmoid(2w) = x / (1 + e^{-2w}), w = sqrt(2/pi) (x + 0.044715 x^3): the same
// function as x (1 + tanh w) / 2 (jax.nn.gelu, approximate=True), with one exponential and one
// reciprocal; relative error ~1e-6, far below the TF32 rounding of the operand it feeds
__device__ __forceinline__ float gelu_sig(float x) {
  const float w = 0.7978845608028654f * fmaf(0.044715f * x, x * x, x);
  return __fdividef(x, 1.0f + __expf(-2.0f * w));
}
__device__ __forceinline__ void proxy_fence() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// float4 chunk j (0..7) of row r in K-block kb of a 128B-swizzled K-major operand with nrows rows
__device__ __forceinline__ float4* sw_chunk(uint8_t* base, int nrows, int kb, int r, int j) {
  return reinterpret_cast<float4*>(base + (size_t)kb * nrows * 128 + r * 128 + ((j ^ (r & 7)) << 4));
}

// W^T [nrows][K] (row-major, K-major for the MMA) -> swizzled shared operand
__device__ __forceinline__ void load_wt(uint8_t* dst, const float* __restrict__ src, int nrows,
                                        int K) {
  const int q4 = K / 4, n4 = nrows * q4;
  for (int c = threadIdx.x; c < n4; c += blockDim.x) {
    const int n = c / q4, q = c - n * q4;
    *sw_chunk(dst, nrows, q >> 3, n, q & 7) = __ldg(reinterpret_cast<const float4*>(src) + c);
  }
}

// eight float32 values -> one 16-byte chunk of BF16 (round to nearest even)
__device__ __forceinline__ uint4 pack8_bf16(float a0, float a1, float a2, float a3, float a4,
                                            float a5, float a6, float a7) {
  __nv_bfloat162 h[4];
  h[0] = __floats2bfloat162_rn(a0, a1);
  h[1] = __floats2bfloat162_rn(a2, a3);
  h[2] = __floats2bfloat162_rn(a4, a5);
  h[3] = __floats2bfloat162_rn(a6, a7);
  return *reinterpret_cast<const uint4*>(h);
}
// 16-byte BF16 chunk j (0..7, eight elements) of row r in K-block kb (64 elements per row)
__device__ __forceinline__ uint4* sw_chunk16(uint8_t* base, int nrows, int kb, int r, int j) {
  return reinterpret_cast<uint4*>(base + (size_t)kb * nrows * 128 + r * 128 + ((j ^ (r & 7)) << 4));
}
// W^T [nrows][K] float32 -> swizzled BF16 shared operand
__device__ __forceinline__ void load_wt16(uint8_t* dst, const float* __restrict__ src, int nrows,
                                          int K) {
  const int q8 = K / 8, n8 = nrows * q8;
  for (int c = threadIdx.x; c < n8; c += blockDim.x) {
    const int n = c / q8, q = c - n * q8;
    const float4 a = __ldg(reinterpret_cast<const float4*>(src) + 2 * c);
    const float4 b = __ldg(reinterpret_cast<const float4*>(src) + 2 * c + 1);
    *sw_chunk16(dst, nrows, q >> 3, n, q & 7) = pack8_bf16(a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w);
  }
}

// row-major staging of a warp's 32 rows of width D (coalesced global <-> per-thread rows),
// chunk c of row r at r * D * 4 + 16 (c ^ (r mod D/4)) bytes
template <int D>
__device__ __forceinline__ float4* st_chunk(uint8_t* base, int r, int c) {
  return reinterpret_cast<float4*>(base + r * D * 4 + ((c ^ (r & (D / 4 - 1))) << 4));
}

// one 128 x N x (KBn * 32) TF32 MMA chain: A K-blocks from sa (128 rows), B K-blocks
// [kb0, kb0 + KBn) of a resident W^T with nrows rows. The descriptors are built here from 32-bit
// shared addresses made opaque to the compiler, so that they are not hoisted out of the tile loop
// and held in registers by every thread.
__device__ __forceinline__ uint64_t desc_u32(uint32_t u) {
  return (uint64_t)((u & 0x3FFFFu) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) |
         (2ull << 61);
}
// (BF: BF16 operands, kind::f16, K = 16 per MMA; otherwise TF32, K = 8: 32 bytes either way)
template <bool BF = false>
__device__ __forceinline__ void issue_chain(uint32_t tmem_d, const uint8_t* sa, const uint8_t* sw,
                                            int nrows, int kb0, int KBn, bool accumulate) {
  uint32_t ua = smem_u32(sa), ub = smem_u32(sw) + (uint32_t)(kb0 * nrows * 128);
  asm volatile("" : "+r"(ua), "+r"(ub));
  const uint32_t id = make_idesc(BF ? 0 : 1, 128, nrows);
#pragma unroll 1
  for (int kb = 0; kb < KBn; ++kb)
#pragma unroll
    for (int kk = 0; kk < 4; ++kk)
      mma<BF ? 0 : 1>(tmem_d, desc_u32(ua + (uint32_t)(kb * 128 * 128 + kk * 32)),
                      desc_u32(ub + (uint32_t)(kb * nrows * 128 + kk * 32)), id,
                      (accumulate || kb || kk) ? 1u : 0u);
}

template <int D, int HD, bool BF>
__global__ void __launch_bounds__(256, 1) k_block_value_tc(BlkArgs a) {
  using Cfg = BlkCfg<D, HD, BF>;
  constexpr int FF = Cfg::FF, H = Cfg::H, KB = Cfg::KB;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~(uintptr_t)1023);
  uint8_t* sWqkv = smem;
  uint8_t* sWo = sWqkv + Cfg::W_QKV;
  uint8_t* sW0 = sWo + Cfg::W_O;
  uint8_t* sW1 = sW0 + Cfg::W_0;
  const int g = threadIdx.x >> 7, r = threadIdx.x & 127, lane = threadIdx.x & 31;
  const int wq = r >> 5;  // warp within the group = TMEM lane quarter
  uint8_t* sA = sW1 + Cfg::W_1 + g * Cfg::G_BYTES;
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + Cfg::W_BYTES + 2 * Cfg::G_BYTES);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bars + 2);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  if (threadIdx.x == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(2 * Cfg::TCOLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if constexpr (BF) {
    load_wt16(sWqkv, a.wqkv, Cfg::NQKV, D);
    load_wt16(sWo, a.wo, D, D);
    load_wt16(sW0, a.w0, FF, D);
    load_wt16(sW1, a.w1, D, FF);
  } else {
    load_wt(sWqkv, a.wqkv, Cfg::NQKV, D);
    load_wt(sWo, a.wo, D, D);
    load_wt(sW0, a.w0, FF, D);
    load_wt(sW1, a.w1, D, FF);
  }
  proxy_fence();
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tm = *tmem_slot + (uint32_t)(g * Cfg::TCOLS);
  const uint32_t tlane = (uint32_t)(wq * 32) << 16;  // this warp's TMEM lane quarter
  uint64_t* bar = &bars[g];
  uint32_t phase = 0;
  const bool issuer = r == 0;
  const float sc = 1.0f / sqrtf((float)HD);
  const float inv_d = 1.0f / (float)D;

  // wait for this group's last commit; every thread of the group leaves together and takes the
  // same decision (an abort anywhere in the CTA ends the group's tile loop)
  auto wait_mma = [&]() -> bool {
    const bool ok = mbar_wait(bar, phase & 1, abort, a.wait_limit);
    ++phase;
    const bool bad = group_bar_or(g, !ok || *abort);
    fence_after();
    return !bad;
  };
  // make this thread's operand writes visible to the tensor core, then hand over to the issuer
  auto publish = [&]() {
    proxy_fence();
    fence_before();
    group_bar(g);
    fence_after();
  };
  // LayerNorm of the register row into the operand tile (K-blocks of 32 columns)
  auto ln_to_operand = [&](const float (&x)[D], const float* __restrict__ s,
                           const float* __restrict__ b, uint8_t* op) {
    float mu = 0.f;
#pragma unroll
    for (int f = 0; f < D; ++f) mu += x[f];
    mu *= inv_d;
    float var = 0.f;
#pragma unroll
    for (int f = 0; f < D; ++f) var += (x[f] - mu) * (x[f] - mu);
    const float rho = 1.0f / sqrtf(var * inv_d + 1e-6f);  // flax LayerNorm epsilon
    if constexpr (BF) {
#pragma unroll
      for (int q = 0; q < D / 8; ++q) {
        float o[8];
        const float4 sg0 = ldp4(s + 8 * q), sg1 = ldp4(s + 8 * q + 4);
        const float4 sb0 = ldp4(b + 8 * q), sb1 = ldp4(b + 8 * q + 4);
        const float sg[8] = {sg0.x, sg0.y, sg0.z, sg0.w, sg1.x, sg1.y, sg1.z, sg1.w};
        const float sb[8] = {sb0.x, sb0.y, sb0.z, sb0.w, sb1.x, sb1.y, sb1.z, sb1.w};
#pragma unroll
        for (int e = 0; e < 8; ++e) o[e] = ((x[8 * q + e] - mu) * rho) * sg[e] + sb[e];
        *sw_chunk16(op, 128, q >> 3, r, q & 7) =
            pack8_bf16(o[0], o[1], o[2], o[3], o[4], o[5], o[6], o[7]);
      }
    } else {
#pragma unroll
      for (int q = 0; q < D / 4; ++q) {
        float4 o;
        const float4 sg = ldp4(s + 4 * q), sb = ldp4(b + 4 * q);
        o.x = ((x[4 * q] - mu) * rho) * sg.x + sb.x;
        o.y = ((x[4 * q + 1] - mu) * rho) * sg.y + sb.y;
        o.z = ((x[4 * q + 2] - mu) * rho) * sg.z + sb.z;
        o.w = ((x[4 * q + 3] - mu) * rho) * sg.w + sb.w;
        *sw_chunk(op, 128, q >> 3, r, q & 7) = o;
      }
    }
  };

  for (int tile = blockIdx.x * 2 + g; tile < a.ntiles; tile += 2 * gridDim.x) {
    // shared addresses are re-derived from an opaque base every tile (cheap integer math) rather
    // than hoisted out of the loop into registers
    uint8_t* sAl = sA;
    asm volatile("" : "+l"(sAl));
    float* sKl = reinterpret_cast<float*>(sAl + Cfg::A_BYTES);
    float* sVl = sKl + 128 * HD;
    uint8_t* wstl = sAl + wq * 32 * D * 4;  // this warp's row staging (aliases the operand tile)
    const int row0 = tile * a.rpt;
    const int nrow = min(a.rpt, a.rows - row0);
    // ---- load: the warp's 32 rows, coalesced, through its staging rows ----
    float x[D];
    {
      const int wr0 = wq * 32;
      const int nw = max(0, min(32, nrow - wr0));
      const float4* src = reinterpret_cast<const float4*>(a.X + (size_t)(row0 + wr0) * D);
#pragma unroll
      for (int it = 0; it < D / 4; ++it) {
        const int f = it * 32 + lane, rr = f / (D / 4), c = f - rr * (D / 4);
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (rr < nw) v = ld_stream4(src + f);
        *st_chunk<D>(wstl, rr, c) = v;
      }
      __syncwarp();
#pragma unroll
      for (int c = 0; c < D / 4; ++c) {
        const float4 v = *st_chunk<D>(wstl, lane, c);
        x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
      }
      __syncwarp();
    }
    // the staging rows of one warp overlap the operand rows of others: all warps of the group
    // finish reading their staging before any thread writes the operand tile
    group_bar(g);
    // ---- attention: x += O(softmax(Q K^T / sqrt(hd)) V) with Q, K, V = LN0(x) Wqkv + b ----
    ln_to_operand(x, a.ln0_s, a.ln0_b, sAl);
    publish();
    if (issuer) {
      issue_chain<BF>(tm, sAl, sWqkv, Cfg::NQKV, 0, KB, false);
      mma_commit(bar);
    }
    if (!wait_mma()) break;
    const int wb = (r / a.N) * a.N;  // first row of this row's walker in the tile
    const bool attn = r < a.rpt;
#pragma unroll 1
    for (int h = 0; h < H; ++h) {
      float q[HD], k[HD], v[HD];
      float4 bq[HD / 4], bk[HD / 4], bv[HD / 4];
#pragma unroll
      for (int c = 0; c < HD / 4; ++c) {
        bq[c] = ldp4(a.bqkv + h * HD + 4 * c);
        bk[c] = ldp4(a.bqkv + D + h * HD + 4 * c);
        bv[c] = ldp4(a.bqkv + 2 * D + h * HD + 4 * c);
      }
      tmem_ld<HD>(tm + tlane + (uint32_t)(h * HD), q);
      tmem_ld<HD>(tm + tlane + (uint32_t)(D + h * HD), k);
      tmem_ld<HD>(tm + tlane + (uint32_t)(2 * D + h * HD), v);
      tmem_wait();
#pragma unroll
      for (int c = 0; c < HD / 4; ++c) {
        q[4 * c] += bq[c].x; q[4 * c + 1] += bq[c].y; q[4 * c + 2] += bq[c].z; q[4 * c + 3] += bq[c].w;
        k[4 * c] += bk[c].x; k[4 * c + 1] += bk[c].y; k[4 * c + 2] += bk[c].z; k[4 * c + 3] += bk[c].w;
        v[4 * c] += bv[c].x; v[4 * c + 1] += bv[c].y; v[4 * c + 2] += bv[c].z; v[4 * c + 3] += bv[c].w;
      }
#pragma unroll
      for (int c = 0; c < HD / 4; ++c) {
        const int cs = c ^ kv_sw<HD>(r);
        reinterpret_cast<float4*>(sKl + r * HD)[cs] =
            make_float4(k[4 * c], k[4 * c + 1], k[4 * c + 2], k[4 * c + 3]);
        reinterpret_cast<float4*>(sVl + r * HD)[cs] =
            make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
      }
      group_bar(g);
      float o[HD];
#pragma unroll
      for (int e = 0; e < HD; ++e) o[e] = 0.f;
      if (attn) {
        float s[16];
        float mx = -INFINITY;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          s[j] = -INFINITY;
          if (j < a.N) {
            const float4* kr = reinterpret_cast<const float4*>(sKl + (wb + j) * HD);
            const int sj = kv_sw<HD>(wb + j);
            float acc = 0.f;
#pragma unroll
            for (int c = 0; c < HD / 4; ++c) {
              const float4 kk = kr[c ^ sj];
              acc = fmaf(q[4 * c], kk.x, acc);
              acc = fmaf(q[4 * c + 1], kk.y, acc);
              acc = fmaf(q[4 * c + 2], kk.z, acc);
              acc = fmaf(q[4 * c + 3], kk.w, acc);
            }
            s[j] = acc * sc;
            mx = fmaxf(mx, s[j]);
          }
        }
        float ssum = 0.f;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          s[j] = j < a.N ? __expf(s[j] - mx) : 0.f;
          ssum += s[j];
        }
        const float inv = 1.0f / ssum;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          if (j < a.N) {
            const float p = s[j] * inv;
            const float4* vr = reinterpret_cast<const float4*>(sVl + (wb + j) * HD);
            const int sj = kv_sw<HD>(wb + j);
#pragma unroll
            for (int c = 0; c < HD / 4; ++c) {
              const float4 vv = vr[c ^ sj];
              o[4 * c] = fmaf(p, vv.x, o[4 * c]);
              o[4 * c + 1] = fmaf(p, vv.y, o[4 * c + 1]);
              o[4 * c + 2] = fmaf(p, vv.z, o[4 * c + 2]);
              o[4 * c + 3] = fmaf(p, vv.w, o[4 * c + 3]);
            }
          }
        }
      }
      // head output -> operand columns [h HD, (h + 1) HD) of the projection
      if constexpr (BF) {
#pragma unroll
        for (int c = 0; c < HD / 8; ++c) {
          const int col = h * HD + 8 * c;
          *sw_chunk16(sAl, 128, col >> 6, r, (col & 63) >> 3) =
              pack8_bf16(o[8 * c], o[8 * c + 1], o[8 * c + 2], o[8 * c + 3], o[8 * c + 4],
                         o[8 * c + 5], o[8 * c + 6], o[8 * c + 7]);
        }
      } else {
#pragma unroll
        for (int c = 0; c < HD / 4; ++c) {
          const int col = h * HD + 4 * c;
          *sw_chunk(sAl, 128, col >> 5, r, (col & 31) >> 2) =
              make_float4(o[4 * c], o[4 * c + 1], o[4 * c + 2], o[4 * c + 3]);
        }
      }
      group_bar(g);  // K / V rows of this head are no longer read
    }
    publish();
    if (issuer) {
      issue_chain<BF>(tm + Cfg::C_O, sAl, sWo, D, 0, KB, false);
      mma_commit(bar);
    }
    if (!wait_mma()) break;
#pragma unroll
    for (int c0 = 0; c0 < D; c0 += 32) {
      float t[32];
      tmem_ld<32>(tm + tlane + (uint32_t)(Cfg::C_O + c0), t);
      tmem_wait();
      float4 bb[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) bb[j] = ldp4(a.bo + c0 + 4 * j);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        x[c0 + 4 * j] += t[4 * j] + bb[j].x;
        x[c0 + 4 * j + 1] += t[4 * j + 1] + bb[j].y;
        x[c0 + 4 * j + 2] += t[4 * j + 2] + bb[j].z;
        x[c0 + 4 * j + 3] += t[4 * j + 3] + bb[j].w;
      }
    }
    // ---- MLP: x += W1 GELU(W0 LN1(x) + b0) + b1, the hidden layer in two halves of D ----
    ln_to_operand(x, a.ln1_s, a.ln1_b, sAl);
    publish();
    if (issuer) {
      issue_chain<BF>(tm + Cfg::C_UP, sAl, sW0, FF, 0, KB, false);
      mma_commit(bar);
    }
    if (!wait_mma()) break;
    bool ok = true;
#pragma unroll 1
    for (int half = 0; half < 2; ++half) {
#pragma unroll
      for (int c0 = 0; c0 < D; c0 += 32) {
        float t[32];
        tmem_ld<32>(tm + tlane + (uint32_t)(Cfg::C_UP + half * D + c0), t);
        tmem_wait();
        float4 bb[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) bb[j] = ldp4(a.b0 + half * D + c0 + 4 * j);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          t[4 * j] = gelu_sig(t[4 * j] + bb[j].x);
          t[4 * j + 1] = gelu_sig(t[4 * j + 1] + bb[j].y);
          t[4 * j + 2] = gelu_sig(t[4 * j + 2] + bb[j].z);
          t[4 * j + 3] = gelu_sig(t[4 * j + 3] + bb[j].w);
        }
        if constexpr (BF) {
#pragma unroll
          for (int j = 0; j < 4; ++j) {
            const int col = c0 + 8 * j;
            *sw_chunk16(sAl, 128, col >> 6, r, (col & 63) >> 3) =
                pack8_bf16(t[8 * j], t[8 * j + 1], t[8 * j + 2], t[8 * j + 3], t[8 * j + 4],
                           t[8 * j + 5], t[8 * j + 6], t[8 * j + 7]);
          }
        } else {
#pragma unroll
          for (int j = 0; j < 8; ++j)
            *sw_chunk(sAl, 128, c0 >> 5, r, j) =
                make_float4(t[4 * j], t[4 * j + 1], t[4 * j + 2], t[4 * j + 3]);
        }
      }
      publish();
      if (issuer) {
        issue_chain<BF>(tm + Cfg::C_DN, sAl, sW1, D, half * KB, KB, half != 0);
        mma_commit(bar);
      }
      if (!wait_mma()) {
        ok = false;
        break;
      }
    }
    if (!ok) break;
#pragma unroll
    for (int c0 = 0; c0 < D; c0 += 32) {
      float t[32];
      tmem_ld<32>(tm + tlane + (uint32_t)(Cfg::C_DN + c0), t);
      tmem_wait();
      float4 bb[8];
#pragma unroll
      for (int j = 0; j < 8; ++j) bb[j] = ldp4(a.b1 + c0 + 4 * j);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        x[c0 + 4 * j] += t[4 * j] + bb[j].x;
        x[c0 + 4 * j + 1] += t[4 * j + 1] + bb[j].y;
        x[c0 + 4 * j + 2] += t[4 * j + 2] + bb[j].z;
        x[c0 + 4 * j + 3] += t[4 * j + 3] + bb[j].w;
      }
    }
    // ---- store: per-thread rows -> staging -> coalesced rows ----
    {
#pragma unroll
      for (int c = 0; c < D / 4; ++c)
        *st_chunk<D>(wstl, lane, c) = make_float4(x[4 * c], x[4 * c + 1], x[4 * c + 2], x[4 * c + 3]);
      __syncwarp();
      const int wr0 = wq * 32;
      const int nw = max(0, min(32, nrow - wr0));
      float4* dst = reinterpret_cast<float4*>(a.X + (size_t)(row0 + wr0) * D);
#pragma unroll
      for (int it = 0; it < D / 4; ++it) {
        const int f = it * 32 + lane, rr = f / (D / 4), c = f - rr * (D / 4);
        if (rr < nw) dst[f] = *st_chunk<D>(wstl, rr, c);
      }
    }
    __syncwarp();  // the next tile's load reuses this warp's staging rows
  }
  fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0 && a.err) atomicExch(a.err, 1);
  if (threadIdx.x < 32) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot),
                 "r"(2 * Cfg::TCOLS));
  }
}

}  // namespace tc

bool g_block_fusion = true;

// ---- optional per-launch timing of the fused block (enabled together with nqs_profile_gemm) ----
namespace {
constexpr int kBlkProfCap = 16384;
std::vector<cudaEvent_t> g_blk_ev;  // pairs
int g_blk_n = 0;
double g_blk_bytes = 0.0, g_blk_flops = 0.0;
}  // namespace

extern "C" int nqs_profile_block_read(double* ms, double* bytes, double* flops,
                                      long long* launches) {
  double t = 0.0;
  for (int i = 0; i < g_blk_n; ++i) {
    float e = 0.f;
    if (cudaEventSynchronize(g_blk_ev[2 * i + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&e, g_blk_ev[2 * i], g_blk_ev[2 * i + 1]) != cudaSuccess) {
      set_error("nqs_profile_block_read: event %d", i);
      return NQS_ERR_CUDA;
    }
    t += e;
  }
  if (ms) *ms = t;
  if (bytes) *bytes = g_blk_bytes;
  if (flops) *flops = g_blk_flops;
  if (launches) *launches = g_blk_n;
  g_blk_n = 0;
  g_blk_bytes = g_blk_flops = 0.0;
  return NQS_OK;
}

extern "C" int nqs_set_block_fusion(int enable) {
  g_block_fusion = enable != 0;
  return NQS_OK;
}

bool block_value_tc_ok(int N, int d, int H, int ff) {
  return N >= 1 && N <= 16 && ff == 2 && ((d == 64 && (H == 4 || H == 8)) || (d == 32 && H == 4));
}

template <int D, int HD, bool BF>
static int launch_block_value(const tc::BlkArgs& a, cudaStream_t st) {
  using Cfg = tc::BlkCfg<D, HD, BF>;
  static int nsm = 0;
  if (!nsm) {
    cudaFuncSetAttribute(tc::k_block_value_tc<D, HD, BF>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    nsm = std::max(nsm, 1);
  }
  const int grid = std::min((a.ntiles + 1) / 2, nsm);
  const bool prof = profiling_enabled() && g_blk_n < kBlkProfCap;
  if (prof) {
    if ((int)g_blk_ev.size() < 2 * (g_blk_n + 1)) {
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      g_blk_ev.push_back(e0);
      g_blk_ev.push_back(e1);
    }
    cudaEventRecord(g_blk_ev[2 * g_blk_n], st);
  }
  tc::k_block_value_tc<D, HD, BF><<<grid, 256, Cfg::SMEM, st>>>(a);
  if (prof) {
    cudaEventRecord(g_blk_ev[2 * g_blk_n + 1], st);
    ++g_blk_n;
    // rows in and out, the weight panels and parameter vectors once; tensor-core flops of the
    // four Dense layers plus the attention's score and value products
    const double rows = a.rows;
    g_blk_bytes += 8.0 * rows * D + Cfg::W_BYTES + 4.0 * (3 * D + D + Cfg::FF + D + 4 * D);
    g_blk_flops += 2.0 * rows * D * (Cfg::NQKV + D + 2 * Cfg::FF) + 4.0 * rows * a.N * D;
  }
  NQS_CHECK_LAUNCH("k_block_value_tc");
  return NQS_OK;
}

int block_value_tc(float* X, int n_jobs, int N, int d, int H, const TcNet& tcn, int b,
                   const BlockW<float>& bw, cudaStream_t st, bool* done) {
  *done = false;
  if (n_jobs <= 0) {
    *done = true;
    return NQS_OK;
  }
  tc::BlkArgs a{};
  a.wqkv = tcn.wqkv[b]; a.bqkv = tcn.bqkv[b]; a.wo = tcn.wo[b]; a.bo = bw.bo;
  a.w0 = tcn.w0[b]; a.b0 = bw.b0; a.w1 = tcn.w1[b]; a.b1 = bw.b1;
  a.ln0_s = bw.ln0_s; a.ln0_b = bw.ln0_b; a.ln1_s = bw.ln1_s; a.ln1_b = bw.ln1_b;
  a.X = X;
  a.rows = n_jobs * N;
  a.N = N;
  a.rpt = (128 / N) * N;
  a.ntiles = (a.rows + a.rpt - 1) / a.rpt;
  a.err = tcn.err;
  a.wait_limit = wait_limit_or(tc::WAIT_LIMIT);
  // every operand is read as float4: a layout whose parameter vectors do not start on 16 bytes
  // is left to the unfused launches (*done stays false)
  uintptr_t al = reinterpret_cast<uintptr_t>(X);
  for (const float* q : {a.wqkv, a.bqkv, a.wo, a.bo, a.w0, a.b0, a.w1, a.b1, a.ln0_s, a.ln0_b,
                         a.ln1_s, a.ln1_b})
    al |= reinterpret_cast<uintptr_t>(q);
  if ((al & 15) || !block_value_tc_ok(N, d, H, 2)) return NQS_OK;
  *done = true;
  if (d == 64 && H == 4)
    return tcn.bf16 ? launch_block_value<64, 16, true>(a, st) : launch_block_value<64, 16, false>(a, st);
  if (d == 64 && H == 8)
    return tcn.bf16 ? launch_block_value<64, 8, true>(a, st) : launch_block_value<64, 8, false>(a, st);
  return launch_block_value<32, 8, false>(a, st);
}

}  // namespace nqs
