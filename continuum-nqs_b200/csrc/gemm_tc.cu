// gemm_tc.cu — network row GEMMs of the mixed-precision path on the tcgen05 tensor cores.
//
// Y[r, n] = sum_k X[r, k] W[k, n] (+ bias[n] on value rows r % C == 0) (+ Res[r, n]) with X the
// float32 activations read by TMA as TF32 operands (kind::tf32, float32 accumulation in TMEM) and W
// pre-transposed to K-major W^T[n][k] once per call. One CTA = one 128-row tile and the whole
// output width (N <= 256, padded to a multiple of 16); K <= 128 fits in shared memory at once, so
// each CTA issues all its TMA loads on one mbarrier, one thread issues the MMAs, and four warps
// drain TMEM. Waits are bounded (tc_common.cuh); an abort is recorded in *err.
#include <cstdio>
#include <algorithm>
#include <vector>

#include "net.cuh"
#include "tc_common.cuh"

namespace nqs {
namespace tc {

constexpr int RG_BM = 128;
constexpr int RG_KB = 32;  // float32 per 128-byte swizzle row

struct RowGemmArgs {
  int rows, K, Nout, Npad, C, vec4;
  const float* bias;
  const float* Res;
  int ldr;
  float* Y;
  int ldy;
  int* err;
};

__global__ void __launch_bounds__(128, 1) k_rowgemm_tc(const __grid_constant__ CUtensorMap tA,
                                                       const __grid_constant__ CUtensorMap tB,
                                                       RowGemmArgs g) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~(uintptr_t)1023);
  const int nkb = g.K / RG_KB;
  const int a_bytes = RG_BM * 128, b_bytes = g.Npad * 128;
  uint8_t* sA = smem;
  uint8_t* sB = smem + nkb * a_bytes;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + nkb * b_bytes);
  uint64_t* done = full + 1;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int m0 = blockIdx.x * RG_BM;
  const uint32_t ncols = g.Npad <= 32 ? 32u : g.Npad <= 64 ? 64u : g.Npad <= 128 ? 128u : 256u;

  if (threadIdx.x == 0) {
    mbar_init(full, 1);
    mbar_init(done, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    mbar_expect_tx(full, (uint32_t)(nkb * (a_bytes + b_bytes)));
    for (int kb = 0; kb < nkb; ++kb) {
      tma_load_2d(sA + kb * a_bytes, &tA, kb * RG_KB, m0, full);
      tma_load_2d(sB + kb * b_bytes, &tB, kb * RG_KB, 0, full);
    }
    mbar_wait(full, 0, abort);  // drain before the CTA may exit
  } else if (warp == 1 && lane == 0) {
    const uint32_t id = make_idesc(1, RG_BM, g.Npad);
    if (mbar_wait(full, 0, abort)) {
      fence_after();
      for (int kb = 0; kb < nkb; ++kb)
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)  // 4 x (K=8 TF32 = 32 bytes) per 128-byte row
          mma<1>(tmem, make_desc(sA + kb * a_bytes + kk * 32), make_desc(sB + kb * b_bytes + kk * 32),
                 id, (kb | kk) != 0 ? 1u : 0u);
    }
    mma_commit(done);
  }
  __syncwarp();
  const bool ok = mbar_wait(done, 0, abort);
  fence_after();
  const bool go = __all_sync(0xffffffffu, ok && !*abort);
  if (go) {
    // Drain TMEM 32 columns at a time into a per-warp staging tile in the (now idle) operand
    // buffer, then write 4 rows x 128 bytes per warp instruction (coalesced float4 when every
    // row start is 16-byte aligned, scalar otherwise).
    float* stage = reinterpret_cast<float*>(sA) + warp * (32 * 33);
    const int r0 = m0 + warp * 32;
#pragma unroll 1
    for (int c0 = 0; c0 < g.Nout; c0 += 32) {
      uint32_t r[32];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
            "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
            "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
            "=r"(r[31])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      const int row_l = r0 + lane;
      const bool val = row_l < g.rows && (row_l % g.C) == 0;
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        const int col = c0 + q;
        float v = __uint_as_float(r[q]);
        if (val && g.bias && col < g.Nout) v += g.bias[col];
        stage[lane * 33 + q] = v;
      }
      __syncwarp();
      const int ncol = min(32, g.Nout - c0);
      if (g.vec4 && ncol == 32) {
#pragma unroll
        for (int rr = 0; rr < 32; rr += 4) {
          const int lr = rr + (lane >> 3), cg = (lane & 7) * 4;
          const int row = r0 + lr;
          if (row < g.rows) {
            const float* sv = stage + lr * 33 + cg;
            float4 v = make_float4(sv[0], sv[1], sv[2], sv[3]);
            if (g.Res) {
              const float4 rv =
                  *reinterpret_cast<const float4*>(g.Res + (size_t)row * g.ldr + c0 + cg);
              v = make_float4(rv.x + v.x, rv.y + v.y, rv.z + v.z, rv.w + v.w);
            }
            *reinterpret_cast<float4*>(g.Y + (size_t)row * g.ldy + c0 + cg) = v;
          }
        }
      } else {
        for (int rr = 0; rr < 32; ++rr) {
          const int row = r0 + rr;
          if (row >= g.rows) break;
          for (int q = lane; q < ncol; q += 32) {
            float v = stage[rr * 33 + q];
            if (g.Res) v = g.Res[(size_t)row * g.ldr + c0 + q] + v;
            g.Y[(size_t)row * g.ldy + c0 + q] = v;
          }
        }
      }
      __syncwarp();
    }
  }
  if (*abort && threadIdx.x == 0 && g.err) atomicExch(g.err, 1);
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
  }
}

}  // namespace tc

bool rowgemm_tc_ok(int K, int ldx, int Nout) {
  return K % tc::RG_KB == 0 && K <= 128 && ldx % 4 == 0 && Nout >= 1 && Nout <= 256;
}

int rowgemm_tc(const float* X, int ldx, int rows, int K, const float* WT, int Npad, int Nout,
               const float* bias, int C, const float* Res, int ldr, float* Y, int ldy, int* err,
               cudaStream_t st) {
  if (rows <= 0) return NQS_OK;
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
  {
    const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)Npad};
    const cuuint64_t strides[1] = {(cuuint64_t)K * 4};
    const cuuint32_t box[2] = {(cuuint32_t)tc::RG_KB, (cuuint32_t)Npad};
    if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(WT), dims, strides, box,
            estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
            CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
      set_error("rowgemm_tc: tensor map (weights)");
      return NQS_ERR_CUDA;
    }
  }
  const int nkb = K / tc::RG_KB;
  // at least 80 KB so at most two CTAs share an SM (2 x 256 TMEM columns <= 512)
  const size_t sm = std::max<size_t>((size_t)80 * 1024,
                                     (size_t)nkb * (tc::RG_BM * 128 + Npad * 128) + 1024 + 64);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(tc::k_rowgemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  // float4 row writes only when every row start of Y and Res is 16-byte aligned
  const int vec4 = ((reinterpret_cast<uintptr_t>(Y) & 15) == 0 && (ldy % 4) == 0 &&
                    (!Res || ((reinterpret_cast<uintptr_t>(Res) & 15) == 0 && (ldr % 4) == 0)))
                       ? 1
                       : 0;
  tc::RowGemmArgs a{rows, K, Nout, Npad, C, vec4, bias, Res, ldr, Y, ldy, err};
  tc::k_rowgemm_tc<<<(rows + tc::RG_BM - 1) / tc::RG_BM, 128, sm, st>>>(ta, tb, a);
  NQS_CHECK_LAUNCH("k_rowgemm_tc");
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

size_t tc_weights_bytes(const NqsModelDesc& d) {
  const size_t dd = d.embed_dim, D = (size_t)d.ff_mult * dd, KN = (size_t)d.n_dets * d.n_elec;
  const size_t per_block = (size_t)pad16(3 * (int)dd) * dd + 3 * dd + dd * dd + D * dd + dd * D;
  return sizeof(float) * ((size_t)d.depth * per_block + (size_t)pad16(2 * (int)KN) * dd) +
         (size_t)(4 * d.depth + 4) * 256 + 64;
}

int build_tc_weights(const NqsModelDesc& d, const float* th, Arena& ws, TcNet* out,
                     cudaStream_t st) {
  TcNet t{};
  const int dd = d.embed_dim, D = d.ff_mult * dd, KN = d.n_dets * d.n_elec;
  t.npad_qkv = pad16(3 * dd);
  t.npad_bf = pad16(2 * KN);
  if (!rowgemm_tc_ok(dd, dd, t.npad_qkv) || !rowgemm_tc_ok(D, D, dd) || !rowgemm_tc_ok(dd, dd, D) ||
      !rowgemm_tc_ok(dd, dd, t.npad_bf)) {
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
  t.on = 1;
  *out = t;
  return NQS_OK;
}

}  // namespace nqs
