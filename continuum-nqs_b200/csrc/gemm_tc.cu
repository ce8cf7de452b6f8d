// gemm_tc.cu — network row GEMMs of the mixed-precision path on the tcgen05 tensor cores.
//
// Y[r, n] = sum_k X[r, k] W[k, n] (+ bias[n] on value rows r % C == 0) (+ Res[r, n]) with X the
// float32 activations read by TMA and W pre-transposed to K-major W^T[n][k] once per call.
// Persistent CTAs (one per SM) keep W^T resident in shared memory and stream 128-row tiles of X
// through a TMA ring; each tile's MMA covers the whole output width (N <= 256, padded to a
// multiple of 16) and K <= 128, float32 accumulation in TMEM. Two operand precisions:
//   TF32: the tensor core reads the float32 tiles as TF32 (kind::tf32);
//   BF16: W^T is a BF16 copy, and the MMA warp converts each float32 X tile into a BF16
//         operand tile (round to nearest even, K-major, 128B swizzle) before issuing
//         kind::f16 MMAs (K a multiple of 64).
// Waits are bounded (tc_common.cuh); an abort is recorded in *err.
#include <cuda_bf16.h>
#include <cstdio>
#include <algorithm>
#include <atomic>
#include <vector>

#include "net.cuh"
#include "tc_common.cuh"

namespace nqs {
namespace tc {

constexpr int RG_BM = 128;
constexpr int RG_KB = 32;  // float32 per 128-byte swizzle row

struct RowGemmArgs {
  int rows, K, Nout, Npad, C, res_inplace, stages, act;
  const float* bias;
  int* err;
  uint32_t wait_limit;
};

// Persistent, warp-specialised: warp 0 streams 128-row A tiles through an S-stage TMA ring (the
// weight panel W^T is loaded once per CTA and stays resident), warp 1 issues the MMAs into one of
// two TMEM accumulators, warps 2..5 drain the other accumulator (epilogue of tile i overlaps the
// MMAs of tile i+1). Tiles are dealt round-robin over the grid.
constexpr int RG_THREADS = 192;

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&r)[32]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]),
        "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]),
        "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]),
        "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// float32 tile (K-blocks of 32 floats, 128B swizzle) -> BF16 operand tile (K-blocks of 64, 128B
// swizzle), by one warp: lane l converts 16-byte chunk j of rows l, l + 32, ... (consecutive lanes
// take consecutive rows, so each phase of 8 lanes touches 8 different bank groups)
__device__ __forceinline__ void tile_to_bf16(const uint8_t* __restrict__ src, uint8_t* dst,
                                             int nkb16, int lane) {
  const int n = nkb16 * RG_BM * 8;
#pragma unroll 4
  for (int q = lane; q < n; q += 32) {
    const int row = q & (RG_BM - 1), j = (q >> 7) & 7, kb = q >> 10;
    const uint8_t* s32 = src + (size_t)(2 * kb + (j >> 2)) * RG_BM * 128 + row * 128;
    const int c0 = 2 * (j & 3);
    const float4 a = *reinterpret_cast<const float4*>(s32 + ((c0 ^ (row & 7)) << 4));
    const float4 b = *reinterpret_cast<const float4*>(s32 + (((c0 + 1) ^ (row & 7)) << 4));
    __nv_bfloat162 h[4];
    h[0] = __floats2bfloat162_rn(a.x, a.y);
    h[1] = __floats2bfloat162_rn(a.z, a.w);
    h[2] = __floats2bfloat162_rn(b.x, b.y);
    h[3] = __floats2bfloat162_rn(b.z, b.w);
    *reinterpret_cast<uint4*>(dst + (size_t)kb * RG_BM * 128 + row * 128 + ((j ^ (row & 7)) << 4)) =
        *reinterpret_cast<const uint4*>(h);
  }
}

template <bool BF>
__global__ void __launch_bounds__(RG_THREADS, 1) k_rowgemm_tc(const __grid_constant__ CUtensorMap tA,
                                                              const __grid_constant__ CUtensorMap tB,
                                                              const __grid_constant__ CUtensorMap tY,
                                                              RowGemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~(uintptr_t)1023);
  const int nkb = g.K / RG_KB, S = g.stages;
  const int nkb16 = g.K / 64;  // BF16 K-blocks (BF only)
  const int a_bytes = RG_BM * 128, b_bytes = g.Npad * 128;
  const int stage_bytes = nkb * a_bytes;
  // BF16 resident W^T: nkb16 blocks of Npad rows x 128 bytes (half the float32 panel)
  const int bpanel = BF ? nkb16 * b_bytes : nkb * b_bytes;
  uint8_t* sB = smem;
  uint8_t* sA = smem + bpanel;  // S stages of float32 tiles
  uint8_t* sC = sA + S * stage_bytes;  // BF16 operand tile (BF only)
  uint8_t* stage_out = sC + (BF ? nkb16 * a_bytes : 0);  // 4 warps x 2 x (32 x 32 floats)
  uint64_t* bfull = reinterpret_cast<uint64_t*>(stage_out + 4 * 2 * 4096);
  uint64_t* afull = bfull + 1;
  uint64_t* aempty = afull + S;
  uint64_t* accfull = aempty + S;
  uint64_t* accempty = accfull + 2;
  uint64_t* cempty = accempty + 2;  // BF16 operand tile free again (BF only)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(cempty + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t ncols = g.Npad <= 32 ? 32u : g.Npad <= 64 ? 64u : g.Npad <= 128 ? 128u : 256u;
  const int ntiles = (g.rows + RG_BM - 1) / RG_BM;
  const int my_tiles = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (threadIdx.x == 0) {
    mbar_init(bfull, 1);
    for (int s = 0; s < S; ++s) {
      mbar_init(&afull[s], 1);
      mbar_init(&aempty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&accfull[b], 1);
      mbar_init(&accempty[b], 4);
    }
    mbar_init(cempty, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(2 * ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0) {
    if (lane == 0) {
      mbar_expect_tx(bfull, (uint32_t)bpanel);
      if (BF) {
        for (int kb = 0; kb < nkb16; ++kb) tma_load_2d(sB + kb * b_bytes, &tB, kb * 64, 0, bfull);
      } else {
        for (int kb = 0; kb < nkb; ++kb) tma_load_2d(sB + kb * b_bytes, &tB, kb * RG_KB, 0, bfull);
      }
      int issued = 0;
      for (int i = 0; i < my_tiles; ++i) {
        const int s = i % S;
        if (i >= S && !mbar_wait(&aempty[s], ((i / S) - 1) & 1, abort, g.wait_limit)) break;
        const int m0 = (blockIdx.x + i * gridDim.x) * RG_BM;
        mbar_expect_tx(&afull[s], (uint32_t)stage_bytes);
        for (int kb = 0; kb < nkb; ++kb)
          tma_load_2d(sA + s * stage_bytes + kb * a_bytes, &tA, kb * RG_KB, m0, &afull[s]);
        issued = i + 1;
      }
      // drain: no bulk copy may still be writing shared memory when the CTA exits
      mbar_wait(bfull, 0, abort, g.wait_limit);
      for (int i = max(0, issued - S); i < issued; ++i)
        mbar_wait(&afull[i % S], (i / S) & 1, abort, g.wait_limit);
    }
  } else if (warp == 1 && BF) {
    // the whole warp converts tile i's float32 rows into the BF16 operand tile once the MMAs of
    // tile i - 1 have read it; lane 0 then frees the float32 stage and issues the BF16 MMAs
    const uint32_t id = make_idesc(0, RG_BM, g.Npad);
    bool ok = mbar_wait(bfull, 0, abort, g.wait_limit);
    for (int i = 0; i < my_tiles; ++i) {
      if (!__all_sync(0xffffffffu, ok)) break;
      const int s = i % S, b = i & 1;
      ok = mbar_wait(&afull[s], (i / S) & 1, abort, g.wait_limit);
      if (ok && i >= 1) ok = mbar_wait(cempty, (i - 1) & 1, abort, g.wait_limit);
      if (!__all_sync(0xffffffffu, ok)) break;
      fence_after();
      tile_to_bf16(sA + s * stage_bytes, sC, nkb16, lane);
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) {
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&aempty[s]))
                     : "memory");
        if (i >= 2) ok = mbar_wait(&accempty[b], ((i >> 1) - 1) & 1, abort, g.wait_limit);
        if (ok) {
          fence_after();
          const uint32_t td = tmem + (uint32_t)b * ncols;
          for (int kb = 0; kb < nkb16; ++kb)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)  // 4 x (K=16 BF16 = 32 bytes) per 128-byte row
              mma<0>(td, make_desc(sC + kb * a_bytes + kk * 32),
                     make_desc(sB + kb * b_bytes + kk * 32), id, (kb | kk) != 0 ? 1u : 0u);
          mma_commit(cempty);
          mma_commit(&accfull[b]);
        }
      }
      ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t id = make_idesc(1, RG_BM, g.Npad);
      if (mbar_wait(bfull, 0, abort, g.wait_limit)) {
        for (int i = 0; i < my_tiles; ++i) {
          const int s = i % S, b = i & 1;
          if (!mbar_wait(&afull[s], (i / S) & 1, abort, g.wait_limit)) break;
          if (i >= 2 && !mbar_wait(&accempty[b], ((i >> 1) - 1) & 1, abort, g.wait_limit)) break;
          fence_after();
          const uint32_t td = tmem + (uint32_t)b * ncols;
          const uint8_t* sa = sA + s * stage_bytes;
          for (int kb = 0; kb < nkb; ++kb)
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)  // 4 x (K=8 TF32 = 32 bytes) per 128-byte row
              mma<1>(td, make_desc(sa + kb * a_bytes + kk * 32), make_desc(sB + kb * b_bytes + kk * 32),
                     id, (kb | kk) != 0 ? 1u : 0u);
          mma_commit(&aempty[s]);
          mma_commit(&accfull[b]);
        }
      }
    }
  } else {
    // epilogue warps: TMEM lanes (warp % 4) * 32 .. +31 = tile rows. Each 32 x 32 chunk goes
    // registers (+ bias on value rows) -> 128B-swizzled shared staging -> one TMA bulk store, or a
    // bulk add-reduction into Y when Y already holds the residual (in-place Y += X W).
    const int ew = warp & 3;
    uint8_t* sbuf = stage_out + (warp - 2) * 8192;
    int nst = 0;
    for (int i = 0; i < my_tiles; ++i) {
      const int b = i & 1;
      const bool ok = mbar_wait(&accfull[b], (i >> 1) & 1, abort, g.wait_limit);
      fence_after();
      if (!__all_sync(0xffffffffu, ok && !*abort)) break;
      const int r0 = (blockIdx.x + i * gridDim.x) * RG_BM + ew * 32;
      const uint32_t tbase = tmem + (uint32_t)b * ncols + ((uint32_t)(ew * 32) << 16);
      const bool val = ((r0 + lane) % g.C) == 0;
#pragma unroll 1
      for (int c0 = 0; c0 < g.Nout; c0 += 32) {
        uint32_t r[32];
        tmem_ld32(tbase + (uint32_t)c0, r);
        if (c0 + 32 >= g.Nout) {
          // last TMEM read of this accumulator: hand it back to the MMA warp
          fence_before();
          __syncwarp();
          if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(
                                          smem_u32(&accempty[b]))
                                      : "memory");
        }
        uint8_t* buf = sbuf + (nst & 1) * 4096;
        if (nst >= 2) {  // the store that last read this buffer must be done reading it
          if (lane == 0) asm volatile("cp.async.bulk.wait_group.read 1;" ::: "memory");
          __syncwarp();
        }
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          float4 v;
          float* pv = reinterpret_cast<float*>(&v);
#pragma unroll
          for (int e = 0; e < 4; ++e) {
            const int col = c0 + 4 * j + e;
            pv[e] = __uint_as_float(r[4 * j + e]);
            if (val && g.bias && col < g.Nout) pv[e] += g.bias[col];
            if (g.act) pv[e] = gelu_value(pv[e], gelu_tanh_w(pv[e]));
          }
          *reinterpret_cast<float4*>(buf + lane * 128 + ((j ^ (lane & 7)) << 4)) = v;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0 && r0 < g.rows) {  // rows past the end are clipped by the tensor map
          if (g.res_inplace)
            asm volatile(
                "cp.reduce.async.bulk.tensor.2d.global.shared::cta.add.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                    reinterpret_cast<uint64_t>(&tY)),
                "r"(c0), "r"(r0), "r"(smem_u32(buf))
                : "memory");
          else
            asm volatile(
                "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(
                    reinterpret_cast<uint64_t>(&tY)),
                "r"(c0), "r"(r0), "r"(smem_u32(buf))
                : "memory");
          asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        }
        ++nst;
      }
    }
    if (lane == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    __syncwarp();
  }
  fence_before();
  __syncthreads();
  if (*abort && threadIdx.x == 0 && g.err) atomicExch(g.err, 1);
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(2 * ncols));
  }
}

}  // namespace tc

// ---- pipeline depth cap (nqs_set_rowgemm_stages) and optional per-launch timing ----
std::atomic<int> g_rowgemm_stages{4};
namespace {
constexpr int kGemmProfCap = 16384;
bool g_gemm_prof = false;
std::vector<cudaEvent_t> g_gemm_ev;  // pairs
int g_gemm_n = 0;
double g_gemm_bytes = 0.0;
}  // namespace

bool profiling_enabled() { return g_gemm_prof; }

// float32 -> BF16 (round to nearest even) copy of n values
__global__ void k_f32_to_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y,
                              size_t n) {
  const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = __float2bfloat16_rn(x[i]);
}

// one launch: K <= 128, Npad <= 256; W^T rows (K-major) have stride ldw elements
static int rowgemm_tc_piece(const float* X, int ldx, int rows, int K, const float* WT, int ldw,
                            int Npad, int Nout, const float* bias, int C, const float* Res,
                            int ldr, float* Y, int ldy, int* err, cudaStream_t st, int act,
                            const uint16_t* WT16) {
  if (rows <= 0) return NQS_OK;
  const bool bf = WT16 != nullptr && K % 64 == 0;
  if (act && C != 1) {
    set_error("rowgemm_tc: the fused activation needs single-channel rows");
    return NQS_ERR_INVALID_ARG;
  }
  tc::EncodeTiledFn enc = tc::encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return NQS_ERR_CUDA;
  }
  if ((reinterpret_cast<uintptr_t>(X) & 15) || (reinterpret_cast<uintptr_t>(WT) & 15) ||
      (ldx % 4) || (K % tc::RG_KB) || Npad % 16 || Npad > 256) {
    set_error("rowgemm_tc: operand layout not TMA-compatible");
    return NQS_ERR_INVALID_ARG;
  }
  CUtensorMap ta, tb;
  const cuuint32_t estr[2] = {1, 1};
  {
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ldx * 4};
    const cuuint32_t box[2] = {(cuuint32_t)tc::RG_KB, (cuuint32_t)tc::RG_BM};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(X), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      set_error("rowgemm_tc: tensor map (activations)");
      return NQS_ERR_CUDA;
    }
  }
  if (bf && (reinterpret_cast<uintptr_t>(WT16) & 15)) {
    set_error("rowgemm_tc: BF16 weights not 16-byte aligned");
    return NQS_ERR_INVALID_ARG;
  }
  {
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)Npad};
    const cuuint64_t strides[1] = {(cuuint64_t)ldw * (bf ? 2 : 4)};
    const cuuint32_t box[2] = {(cuuint32_t)(bf ? 64 : tc::RG_KB), (cuuint32_t)Npad};
    if (enc(&tb, bf ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
            bf ? (void*)WT16 : (void*)WT, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      set_error("rowgemm_tc: tensor map (weights)");
      return NQS_ERR_CUDA;
    }
  }
  // the residual, when given, is Y itself (Y += X W in place): the epilogue adds into Y with a
  // bulk reduction; Y rows must start on 16 bytes for the store tensor map
  if (Res && (Res != Y || ldr != ldy)) {
    set_error("rowgemm_tc: the residual must be the output itself (in-place Y += X W)");
    return NQS_ERR_INVALID_ARG;
  }
  if ((reinterpret_cast<uintptr_t>(Y) & 15) || (ldy % 4)) {
    set_error("rowgemm_tc: output rows not 16-byte aligned");
    return NQS_ERR_INVALID_ARG;
  }
  CUtensorMap ty;
  {
    const cuuint64_t dims[2] = {(cuuint64_t)Nout, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ldy * 4};
    const cuuint32_t box[2] = {32, 32};
    if (enc(&ty, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, Y, dims, strides, box, estr,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      set_error("rowgemm_tc: tensor map (output)");
      return NQS_ERR_CUDA;
    }
  }
  const int nkb = K / tc::RG_KB;
  // shared memory: resident W^T, S stages of A tiles, (BF16: the converted operand tile),
  // epilogue staging, barriers
  const size_t panel = bf ? (size_t)(K / 64) * Npad * 128 : (size_t)nkb * Npad * 128;
  const size_t conv = bf ? (size_t)(K / 64) * tc::RG_BM * 128 : 0;
  const size_t fixed = panel + conv + 4 * 2 * 4096 + 256 + 1024;
  const size_t stage = (size_t)nkb * tc::RG_BM * 128;
  const size_t cap = 227 * 1024;
  int S = (int)std::min<size_t>((size_t)g_rowgemm_stages.load(), (cap - fixed) / stage);
  if (S < 2) {
    set_error("rowgemm_tc: K=%d, N=%d leave room for %d pipeline stages", K, Npad, S);
    return NQS_ERR_UNSUPPORTED;
  }
  const size_t sm = fixed + (size_t)S * stage;
  static bool attr = false;
  static int nsm = 0;
  if (!attr) {
    cudaFuncSetAttribute(tc::k_rowgemm_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         227 * 1024);
    cudaFuncSetAttribute(tc::k_rowgemm_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         227 * 1024);
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    attr = true;
  }
  tc::RowGemmArgs a{rows, K, Nout, Npad, C, Res ? 1 : 0, S, act, bias, err,
                    wait_limit_or(tc::WAIT_LIMIT)};
  const int ntiles = (rows + tc::RG_BM - 1) / tc::RG_BM;
  const bool prof = g_gemm_prof && g_gemm_n < kGemmProfCap;
  if (prof) {
    if ((int)g_gemm_ev.size() < 2 * (g_gemm_n + 1)) {
      cudaEvent_t e0, e1;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      g_gemm_ev.push_back(e0);
      g_gemm_ev.push_back(e1);
    }
    cudaEventRecord(g_gemm_ev[2 * g_gemm_n], st);
  }
  if (bf)
    tc::k_rowgemm_tc<true><<<std::min(ntiles, std::max(nsm, 1)), tc::RG_THREADS, sm, st>>>(
        ta, tb, ty, a);
  else
    tc::k_rowgemm_tc<false><<<std::min(ntiles, std::max(nsm, 1)), tc::RG_THREADS, sm, st>>>(
        ta, tb, ty, a);
  if (prof) {
    cudaEventRecord(g_gemm_ev[2 * g_gemm_n + 1], st);
    ++g_gemm_n;
    // operand rows, weight panel, output rows (read again and written when accumulating in place)
    g_gemm_bytes += 4.0 * ((double)rows * K + (double)Npad * K + (double)rows * Nout * (Res ? 2 : 1));
  }
  NQS_CHECK_LAUNCH("k_rowgemm_tc");
  return NQS_OK;
}

// pipeline stages that fit one launch of K-piece kp and N-piece np (0: does not fit)
static int rowgemm_stages_for(int kp, int np, bool bf) {
  const size_t panel = bf ? (size_t)(kp / 64) * np * 128 : (size_t)(kp / tc::RG_KB) * np * 128;
  const size_t conv = bf ? (size_t)(kp / 64) * tc::RG_BM * 128 : 0;
  const size_t fixed = panel + conv + 4 * 2 * 4096 + 256 + 1024;
  const size_t stage = (size_t)(kp / tc::RG_KB) * tc::RG_BM * 128;
  const size_t cap = 227 * 1024;
  if (fixed + 2 * stage > cap) return 0;
  return (int)std::min<size_t>((size_t)g_rowgemm_stages.load(), (cap - fixed) / stage);
}

// Any K (a multiple of 32) and any output width: pieces of at most 128 K-columns and 256 output
// columns, one launch each, chosen among the splits that leave room for at least two pipeline
// stages by their HBM traffic (X is read once per N piece; Y is stored once and read + written
// again by every further K piece). The first K piece of an output slice stores (with the bias)
// or, when a residual is given, adds into Y; later K pieces add their partial products into Y
// with the bulk reduction. The fused activation needs a single K piece.
int rowgemm_tc(const float* X, int ldx, int rows, int K, const float* WT, int Npad, int Nout,
               const float* bias, int C, const float* Res, int ldr, float* Y, int ldy, int* err,
               cudaStream_t st, int act, const uint16_t* WT16) {
  const bool bf_all = WT16 != nullptr && K % 64 == 0;
  if (K <= 128 && Npad <= 256 && rowgemm_stages_for(K, Npad, bf_all) >= 2)
    return rowgemm_tc_piece(X, ldx, rows, K, WT, K, Npad, Nout, bias, C, Res, ldr, Y, ldy, err,
                            st, act, WT16);
  if (Res && (Res != Y || ldr != ldy)) {
    set_error("rowgemm_tc: the residual must be the output itself (in-place Y += X W)");
    return NQS_ERR_INVALID_ARG;
  }
  int best_k = 0, best_n = 0;
  double best = 0.0;
  for (int kp = 128; kp >= tc::RG_KB; kp -= tc::RG_KB) {
    if (act && kp < K) continue;
    for (int np = 256; np >= 16; np -= 16) {
      const bool bf = WT16 != nullptr && kp % 64 == 0;
      if (rowgemm_stages_for(kp, np, bf) < 2) continue;
      const int nk = (K + kp - 1) / kp, nn = (Npad + np - 1) / np;
      const double t = (double)K * nn + (double)Nout * (2 * nk - 1) + 1e-3 * nk * nn;
      if (!best_k || t < best) {
        best = t;
        best_k = kp;
        best_n = np;
      }
    }
  }
  if (!best_k) {
    set_error("rowgemm_tc: no piece of K=%d, N=%d fits shared memory", K, Npad);
    return NQS_ERR_UNSUPPORTED;
  }
  for (int n0 = 0; n0 < Npad && n0 < Nout; n0 += best_n) {
    const int np = std::min(best_n, Npad - n0), no = std::min(np, Nout - n0);
    for (int k0 = 0; k0 < K; k0 += best_k) {
      const int kp = std::min(best_k, K - k0);
      const bool first = k0 == 0;
      const float* res = (Res || !first) ? Y + n0 : nullptr;
      NQS_TRY(rowgemm_tc_piece(X + k0, ldx, rows, kp, WT + (size_t)n0 * K + k0, K, np, no,
                               first && bias ? bias + n0 : nullptr, C, res, ldy, Y + n0, ldy,
                               err, st, act, WT16 ? WT16 + (size_t)n0 * K + k0 : nullptr));
    }
  }
  return NQS_OK;
}

extern "C" int nqs_set_rowgemm_stages(int max_stages) {
  if (max_stages != 0 && (max_stages < 2 || max_stages > 4)) {
    set_error("nqs_set_rowgemm_stages: %d is not 0 or 2..4", max_stages);
    return NQS_ERR_INVALID_ARG;
  }
  g_rowgemm_stages.store(max_stages ? max_stages : 4);
  return NQS_OK;
}

extern "C" int nqs_profile_gemm(int enable) {
  g_gemm_prof = enable != 0;
  return NQS_OK;
}

extern "C" int nqs_profile_gemm_read(double* ms, double* bytes, long long* launches) {
  double t = 0.0;
  for (int i = 0; i < g_gemm_n; ++i) {
    float e = 0.f;
    if (cudaEventSynchronize(g_gemm_ev[2 * i + 1]) != cudaSuccess ||
        cudaEventElapsedTime(&e, g_gemm_ev[2 * i], g_gemm_ev[2 * i + 1]) != cudaSuccess) {
      set_error("nqs_profile_gemm_read: event %d", i);
      return NQS_ERR_CUDA;
    }
    t += e;
  }
  if (ms) *ms = t;
  if (bytes) *bytes = g_gemm_bytes;
  if (launches) *launches = g_gemm_n;
  g_gemm_n = 0;
  g_gemm_bytes = 0.0;
  return NQS_OK;
}

// ---------------------------------------------------------------------------------------------
// K-major weight copies: dst[row0 + n][k] = src[k][n] (src row-major [K][ld_src]), float32
// ---------------------------------------------------------------------------------------------
struct TransJob {
  const float* src;
  float* dst;
  int K, N, ld_src, row0;
};
struct TransBatch {
  TransJob j[8];
  int n;
};

__global__ void k_transpose_batch(TransBatch b) {
  const TransJob t = b.j[blockIdx.y];
  for (int idx = blockIdx.x * blockDim.x + threadIdx.x; idx < t.K * t.N;
       idx += gridDim.x * blockDim.x) {
    const int n = idx / t.K, k = idx - n * t.K;
    t.dst[(size_t)(t.row0 + n) * t.K + k] = t.src[(size_t)k * t.ld_src + n];
  }
}

int transpose_batch(const TransJob* jobs, int n, cudaStream_t st) {
  for (int i0 = 0; i0 < n; i0 += 8) {
    TransBatch b{};
    b.n = std::min(8, n - i0);
    for (int i = 0; i < b.n; ++i) b.j[i] = jobs[i0 + i];
    k_transpose_batch<<<dim3(64, b.n), 256, 0, st>>>(b);
    NQS_CHECK_LAUNCH("k_transpose_batch");
  }
  return NQS_OK;
}

static inline int pad16(int n) { return (n + 15) / 16 * 16; }

size_t tc_weights_bytes(const NqsModelDesc& d, bool bf16) {
  const size_t dd = d.embed_dim, D = (size_t)d.ff_mult * dd, KN = (size_t)d.n_dets * d.n_elec;
  const size_t per_block = (size_t)pad16(3 * (int)dd) * dd + 3 * dd + dd * dd + D * dd + dd * D;
  const size_t wts = (size_t)d.depth * per_block + (size_t)pad16(2 * (int)KN) * dd;
  return sizeof(float) * wts + (bf16 ? sizeof(uint16_t) * wts + (size_t)(5 * d.depth + 1) * 256
                                      : 0) +
         (size_t)(4 * d.depth + 4) * 256 + 64;
}

// BF16 copy of n float32 values in the workspace (nullptr when it does not fit)
static const uint16_t* bf16_copy(const float* x, size_t n, Arena& ws, cudaStream_t st) {
  __nv_bfloat16* y = reinterpret_cast<__nv_bfloat16*>(ws.take<uint16_t>(n));
  if (!y) return nullptr;
  k_f32_to_bf16<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(x, y, n);
  g_launches.fetch_add(1, std::memory_order_relaxed);
  return reinterpret_cast<const uint16_t*>(y);
}

int build_tc_weights(const NqsModelDesc& d, const float* th, Arena& ws, TcNet* out,
                     cudaStream_t st, bool bf16) {
  TcNet t{};
  const int dd = d.embed_dim, D = d.ff_mult * dd, KN = d.n_dets * d.n_elec;
  t.npad_qkv = pad16(3 * dd);
  t.npad_bf = pad16(2 * KN);
  // every Dense layer runs as row-GEMM pieces of K <= 128 and N <= 256 (rowgemm_tc)
  if (dd % tc::RG_KB || D % tc::RG_KB) {
    t.on = 0;
    *out = t;
    return NQS_OK;
  }
  std::vector<TransJob> jobs;
  for (int b = 0; b < d.depth; ++b) {
    const int64_t* o = d.off_block[b];
    float* wqkv = ws.take<float>((size_t)t.npad_qkv * dd);
    float* bqkv = ws.take<float>(3 * (size_t)dd);
    float* wo = ws.take<float>((size_t)dd * dd);
    float* w0 = ws.take<float>((size_t)D * dd);
    float* w1 = ws.take<float>((size_t)dd * D);
    if (!w1) return NQS_ERR_WORKSPACE;
    if (t.npad_qkv > 3 * dd)
      cudaMemsetAsync(wqkv + (size_t)3 * dd * dd, 0, sizeof(float) * (t.npad_qkv - 3 * dd) * dd, st);
    jobs.push_back({th + o[NQS_B_Q_KERNEL], wqkv, dd, dd, dd, 0});
    jobs.push_back({th + o[NQS_B_K_KERNEL], wqkv, dd, dd, dd, dd});
    jobs.push_back({th + o[NQS_B_V_KERNEL], wqkv, dd, dd, dd, 2 * dd});
    jobs.push_back({th + o[NQS_B_O_KERNEL], wo, dd, dd, dd, 0});
    jobs.push_back({th + o[NQS_B_DENSE0_KERNEL], w0, dd, D, D, 0});
    jobs.push_back({th + o[NQS_B_DENSE1_KERNEL], w1, D, dd, dd, 0});
    cudaMemcpyAsync(bqkv, th + o[NQS_B_Q_BIAS], sizeof(float) * dd, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(bqkv + dd, th + o[NQS_B_K_BIAS], sizeof(float) * dd, cudaMemcpyDeviceToDevice,
                    st);
    cudaMemcpyAsync(bqkv + 2 * dd, th + o[NQS_B_V_BIAS], sizeof(float) * dd,
                    cudaMemcpyDeviceToDevice, st);
    t.wqkv[b] = wqkv;
    t.bqkv[b] = bqkv;
    t.wo[b] = wo;
    t.w0[b] = w0;
    t.w1[b] = w1;
  }
  float* wbf = ws.take<float>((size_t)t.npad_bf * dd);
  if (!wbf) return NQS_ERR_WORKSPACE;
  if (t.npad_bf > 2 * KN)
    cudaMemsetAsync(wbf + (size_t)2 * KN * dd, 0, sizeof(float) * (t.npad_bf - 2 * KN) * dd, st);
  jobs.push_back({th + d.off_backflow_kernel, wbf, dd, KN, KN, 0});
  jobs.push_back({th + d.off_backflow_kernel + (int64_t)dd * KN, wbf, dd, KN, KN, KN});
  t.wbf = wbf;
  t.err = ws.take<int>(1);
  if (!t.err) return NQS_ERR_WORKSPACE;
  cudaMemsetAsync(t.err, 0, sizeof(int), st);
  NQS_TRY(transpose_batch(jobs.data(), (int)jobs.size(), st));
  if (bf16) {
    for (int b = 0; b < d.depth; ++b) {
      t.wqkv16[b] = bf16_copy(t.wqkv[b], (size_t)t.npad_qkv * dd, ws, st);
      t.wo16[b] = bf16_copy(t.wo[b], (size_t)dd * dd, ws, st);
      t.w016[b] = bf16_copy(t.w0[b], (size_t)D * dd, ws, st);
      t.w116[b] = bf16_copy(t.w1[b], (size_t)dd * D, ws, st);
      if (!t.w116[b]) return NQS_ERR_WORKSPACE;
    }
    t.wbf16 = bf16_copy(t.wbf, (size_t)t.npad_bf * dd, ws, st);
    if (!t.wbf16) return NQS_ERR_WORKSPACE;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(e, "k_f32_to_bf16");
    t.bf16 = 1;
  }
  t.on = 1;
  *out = t;
  return NQS_OK;
}

}  // namespace nqs
