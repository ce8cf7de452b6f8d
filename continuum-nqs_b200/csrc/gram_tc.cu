// gram_tc.cu — tensor-core Gram T = Otil Otil^T (lower triangle) on sm_100a.
//
// Otil (2W x P) is the centred per-sample Jacobian converted to BF16 (kind::f16) or kept in
// float32 (kind::tf32). One CTA computes one 128 x 256 tile of T:
//   * warp 0 / lane 0 issues TMA loads (128B-swizzled 128-row x 128-byte boxes, no multicast)
//     into a 4-stage shared-memory ring guarded by mbarriers;
//   * warp 1 / lane 0 issues tcgen05.mma (M=128, N=256, K=16 BF16 or K=8 TF32) with the
//     accumulator in tensor memory (256 float32 columns), and tcgen05.commit frees each stage;
//   * all 4 warps drain TMEM with tcgen05.ld (32 lanes x 16 columns per load) and write the
//     lower-triangular part of the tile to T in float64.
// Every wait is bounded: on time-out the CTA records an error flag, stops issuing, drains what
// it issued (bounded) and frees its tensor memory.
//
// The same pipeline, instantiated with SUB, is the trailing update T -= P P^T of the blocked
// Cholesky that preconditions the mixed-precision MinSR solve: P's float64 rows are split into a
// TF32 part and a float32 remainder, stored side by side as [hi | lo] (width 2K), and the k-blocks
// run over hi hi^T, lo hi^T and hi lo^T (three TF32 products: ~2^-22 relative error against the
// float64 update, instead of TF32's 2^-11); the epilogue subtracts from the float64 T.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cstdio>
#include <algorithm>

#include "minsr.cuh"
#include "tc_common.cuh"

namespace nqs {
namespace tc {

constexpr int BM = 128, BN = 256, STAGES = 4;
constexpr int ROW_BYTES = 128;                  // one 128B swizzle atom row per tile row
constexpr int A_BYTES = BM * ROW_BYTES;         // 16 KB
constexpr int B_BYTES = BN * ROW_BYTES;         // 32 KB
constexpr int SMEM_BYTES = STAGES * (A_BYTES + B_BYTES) + 1024 /*align*/ + 256 /*barriers*/;
constexpr uint32_t TMEM_COLS = 256;
// instruction descriptor: D f32, A/B format (1 = BF16, 2 = TF32), both K-major, M=128, N=256
template <int KIND>
__host__ __device__ constexpr uint32_t idesc() {
  return (1u << 4) | ((KIND == 0 ? 1u : 2u) << 7) | ((KIND == 0 ? 1u : 2u) << 10) |
         ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
}

// lower-triangular tile enumeration over 128-row x 256-col tiles (row tile ti needs col tiles
// 0 .. floor(ti/2)), grouped for L2 reuse: bands of 8 row tiles, inside a band column tile by
// column tile. Consecutive tiles share their 256-row B panel and cycle through the band's eight
// A panels, so the tiles of one launch round read a compact set of operand rows.
constexpr int GRAM_BAND = 8;
__device__ __forceinline__ void tile_coords(int t, int nrt, int* ti, int* tj) {
  *ti = 0;
  *tj = 0;
  for (int g0 = 0; g0 < nrt; g0 += GRAM_BAND) {
    const int g1 = min(nrt, g0 + GRAM_BAND);
    int cnt = 0;
    for (int i = g0; i < g1; ++i) cnt += i / 2 + 1;
    if (t >= cnt) {
      t -= cnt;
      continue;
    }
    for (int j = 0; 2 * j < g1; ++j) {
      const int lo = max(g0, 2 * j), c = g1 - lo;  // row tiles ti >= 2 j of the band
      if (t < c) {
        *ti = lo + t;
        *tj = j;
        return;
      }
      t -= c;
    }
    return;
  }
}

template <int KIND, bool SUB>
__global__ void __launch_bounds__(128, 1) k_gram_tc(const __grid_constant__ CUtensorMap tmap,
                                                    int M, int64_t K, double* __restrict__ T,
                                                    int64_t ldt, int* __restrict__ err,
                                                    uint32_t wait_limit, int t0) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~(uintptr_t)1023);
  uint8_t* sA = smem;
  uint8_t* sB = smem + STAGES * A_BYTES;
  uint64_t* full = reinterpret_cast<uint64_t*>(sB + STAGES * B_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* done = empty + STAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int ti, tj;
  tile_coords(t0 + (int)blockIdx.x, (M + BM - 1) / BM, &ti, &tj);
  const int i0 = ti * BM, j0 = tj * BN;
  constexpr int KE = (KIND == 0) ? 64 : 32;  // elements per 128-byte row
  const int nkh = (int)((K + KE - 1) / KE);  // k-blocks of one pass (SUB: of one half)
  const int nk = SUB ? 3 * nkh : nkh;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer ----------------
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1, abort, wait_limit)) break;
      int xa = kb * KE, xb = kb * KE;
      if constexpr (SUB) {  // passes hi.hi, lo.hi, hi.lo; the lo half starts at column K
        const int seg = kb / nkh, off = (kb - seg * nkh) * KE;
        xa = (seg == 1 ? (int)K : 0) + off;
        xb = (seg == 2 ? (int)K : 0) + off;
      }
      mbar_expect_tx(&full[s], A_BYTES + B_BYTES);
      tma_load_2d(sA + s * A_BYTES, &tmap, xa, i0, &full[s]);
      tma_load_2d(sB + s * B_BYTES, &tmap, xb, j0, &full[s]);
      tma_load_2d(sB + s * B_BYTES + A_BYTES, &tmap, xb, j0 + BM, &full[s]);
      issued = kb + 1;
    }
    // drain: every issued stage's loads must have landed before the CTA may exit
    for (int kb = (issued > STAGES ? issued - STAGES : 0); kb < issued; ++kb)
      mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1, abort, wait_limit);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer ----------------
    constexpr uint32_t id = idesc<KIND>();
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full[s], (kb / STAGES) & 1, abort, wait_limit)) break;
      fence_after();
      const uint8_t* a = sA + s * A_BYTES;
      const uint8_t* b = sB + s * B_BYTES;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk)  // 4 x 32 bytes = one 128-byte row of K
        mma<KIND>(tmem, make_desc(a + kk * 32), make_desc(b + kk * 32), id,
                  (kb | kk) != 0 ? 1u : 0u);
      mma_commit(&empty[s]);
    }
    mma_commit(done);  // tracks every MMA issued above, also on abort
  }
  // ---------------- epilogue (all 4 warps) ----------------
  __syncwarp();
  const bool ok = mbar_wait(done, 0, abort, wait_limit);
  fence_after();
  const bool go = __all_sync(0xffffffffu, ok && !*abort);  // tcgen05.ld is warp-collective
  if (go) {
    const int row = i0 + warp * 32 + lane;
    const int wrow_max = i0 + warp * 32 + 31;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      if (j0 + c0 > wrow_max) break;  // warp-uniform: no column of this chunk is on/below diag
      uint32_t r[16];
      const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0;
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
          "%14,%15}, [%16];"
          : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
            "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
            "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
          : "r"(taddr));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if constexpr (SUB) {
        // T -= acc; a chunk wholly on or below the diagonal as 16-byte read-modify-writes
        // (the host passes T 16-byte aligned with an even ldt)
        if (row < M) {
          double* tr = T + (size_t)row * ldt + j0 + c0;
          if (j0 + c0 + 15 <= row) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              double2 v = reinterpret_cast<double2*>(tr)[q];
              v.x -= (double)__uint_as_float(r[2 * q]);
              v.y -= (double)__uint_as_float(r[2 * q + 1]);
              reinterpret_cast<double2*>(tr)[q] = v;
            }
          } else {
#pragma unroll
            for (int q = 0; q < 16; ++q)
              if (j0 + c0 + q <= row) tr[q] -= (double)__uint_as_float(r[q]);
          }
        }
      } else if (row < M) {
#pragma unroll
        for (int q = 0; q < 16; ++q) {
          const int col = j0 + c0 + q;
          if (col <= row && col < M) T[(size_t)row * ldt + col] = (double)__uint_as_float(r[q]);
        }
      }
    }
  }
  if (*abort && threadIdx.x == 0) atomicExch(err, 1);
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(TMEM_COLS));
  }
}

// ---------------------------------------------------------------------------------------------
// Wide tiles: one CTA computes a 256 x 256 tile of T as two M = 128 accumulators (TMEM columns
// 0-255 and 256-511) against the same 256-row B panel, so every operand byte brought into shared
// memory feeds twice the MMA work of a 128 x 256 tile (L2 -> SM traffic per flop down by a
// third); 3-stage ring of 64 KB stages.
constexpr int WBM = 256, WSTAGES = 3;
constexpr int WA_BYTES = WBM * ROW_BYTES;  // 32 KB
constexpr int WSTAGE_BYTES = WA_BYTES + B_BYTES;
constexpr int WSMEM_BYTES = WSTAGES * WSTAGE_BYTES + 1024 + 256;
constexpr uint32_t WTMEM_COLS = 512;

// lower-triangular 256 x 256 tiles (row tile ti needs column tiles 0 .. ti), bands of GRAM_BAND
// row tiles, inside a band column tile by column tile
__device__ __forceinline__ void tile_coords_sq(int t, int nrt, int* ti, int* tj) {
  *ti = 0;
  *tj = 0;
  for (int g0 = 0; g0 < nrt; g0 += GRAM_BAND) {
    const int g1 = min(nrt, g0 + GRAM_BAND);
    int cnt = 0;
    for (int i = g0; i < g1; ++i) cnt += i + 1;
    if (t >= cnt) {
      t -= cnt;
      continue;
    }
    for (int j = 0; j < g1; ++j) {
      const int lo = max(g0, j), c = g1 - lo;
      if (t < c) {
        *ti = lo + t;
        *tj = j;
        return;
      }
      t -= c;
    }
    return;
  }
}

template <int KIND>
__global__ void __launch_bounds__(128, 1) k_gram_tc_wide(const __grid_constant__ CUtensorMap tmap,
                                                         int M, int64_t K, double* __restrict__ T,
                                                         int64_t ldt, int* __restrict__ err,
                                                         uint32_t wait_limit, int t0) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                             ~(uintptr_t)1023);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + WSTAGES * WSTAGE_BYTES);
  uint64_t* empty = full + WSTAGES;
  uint64_t* done = empty + WSTAGES;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(done + 1);
  volatile int* abort = reinterpret_cast<volatile int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int ti, tj;
  tile_coords_sq(t0 + (int)blockIdx.x, (M + WBM - 1) / WBM, &ti, &tj);
  const int i0 = ti * WBM, j0 = tj * BN;
  constexpr int KE = (KIND == 0) ? 64 : 32;
  const int nk = (int)((K + KE - 1) / KE);

  if (threadIdx.x == 0) {
    for (int s = 0; s < WSTAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(done, 1);
    *abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(WTMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tmem = *tmem_slot;

  if (warp == 0 && lane == 0) {
    // ---------------- TMA producer: A rows i0 .. i0 + 255, B rows j0 .. j0 + 255 ----------------
    int issued = 0;
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % WSTAGES;
      if (kb >= WSTAGES && !mbar_wait(&empty[s], ((kb / WSTAGES) - 1) & 1, abort, wait_limit))
        break;
      uint8_t* st = smem + s * WSTAGE_BYTES;
      mbar_expect_tx(&full[s], WSTAGE_BYTES);
      tma_load_2d(st, &tmap, kb * KE, i0, &full[s]);
      tma_load_2d(st + A_BYTES, &tmap, kb * KE, i0 + BM, &full[s]);
      tma_load_2d(st + WA_BYTES, &tmap, kb * KE, j0, &full[s]);
      tma_load_2d(st + WA_BYTES + A_BYTES, &tmap, kb * KE, j0 + BM, &full[s]);
      issued = kb + 1;
    }
    for (int kb = (issued > WSTAGES ? issued - WSTAGES : 0); kb < issued; ++kb)
      mbar_wait(&full[kb % WSTAGES], (kb / WSTAGES) & 1, abort, wait_limit);
  } else if (warp == 1 && lane == 0) {
    // ---------------- MMA issuer: two accumulators share each B operand ----------------
    constexpr uint32_t id = idesc<KIND>();
    for (int kb = 0; kb < nk; ++kb) {
      const int s = kb % WSTAGES;
      if (!mbar_wait(&full[s], (kb / WSTAGES) & 1, abort, wait_limit)) break;
      fence_after();
      const uint8_t* a = smem + s * WSTAGE_BYTES;
      const uint8_t* b = a + WA_BYTES;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const uint32_t acc = (kb | kk) != 0 ? 1u : 0u;
        const uint64_t db = make_desc(b + kk * 32);
        mma<KIND>(tmem, make_desc(a + kk * 32), db, id, acc);
        mma<KIND>(tmem + 256, make_desc(a + A_BYTES + kk * 32), db, id, acc);
      }
      mma_commit(&empty[s]);
    }
    mma_commit(done);
  }
  // ---------------- epilogue (all 4 warps, both halves) ----------------
  __syncwarp();
  const bool ok = mbar_wait(done, 0, abort, wait_limit);
  fence_after();
  const bool go = __all_sync(0xffffffffu, ok && !*abort);
  if (go) {
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
      const int rbase = i0 + h * BM + warp * 32;
      const int row = rbase + lane;
#pragma unroll 1
      for (int c0 = 0; c0 < BN; c0 += 16) {
        if (j0 + c0 > rbase + 31) break;  // warp-uniform: nothing on or below the diagonal
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(h * 256 + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
              "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
              "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < M) {
#pragma unroll
          for (int q = 0; q < 16; ++q) {
            const int col = j0 + c0 + q;
            if (col <= row) T[(size_t)row * ldt + col] = (double)__uint_as_float(r[q]);
          }
        }
      }
    }
  }
  if (*abort && threadIdx.x == 0) atomicExch(err, 1);
  fence_before();
  __syncthreads();
  if (warp == 0) {
    fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(WTMEM_COLS));
  }
}

// centre and convert: D[r][p] = O[r][p] - mu[half][p] (p < P), zero padding up to ldd
template <typename TO, typename TD>
__global__ void k_center_cvt(const TO* __restrict__ O, int W, int64_t P, int64_t ldd,
                             const double* __restrict__ mu, TD* __restrict__ D) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (p >= ldd) return;
  const int half = r >= W;
  double v = 0.0;
  if (p < P) v = (double)O[(size_t)r * P + p] - mu[(size_t)half * P + p];
  if constexpr (sizeof(TD) == 2)
    D[(size_t)r * ldd + p] = __double2bfloat16(v);
  else
    D[(size_t)r * ldd + p] = (TD)v;
}

// vectorised form: 8 consecutive columns x CVT_ROWS rows per thread (the column means are read
// once per thread); VEC: P % 4 == 0 so the 8 source columns are two 16-byte loads (float)
constexpr int CVT_ROWS = 16;
template <typename TO, typename TD, bool VEC>
__global__ void __launch_bounds__(256) k_center_cvt8(const TO* __restrict__ O, int W, int M,
                                                     int64_t P, int64_t ldd,
                                                     const double* __restrict__ mu,
                                                     TD* __restrict__ D) {
  const int64_t p0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 8;
  if (p0 >= ldd) return;
  const int r0 = blockIdx.y * CVT_ROWS, r1 = min(M, r0 + CVT_ROWS);
  double m0[8], m1[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const bool in = p0 + c < P;
    m0[c] = (in && r0 < W) ? mu[p0 + c] : 0.0;
    m1[c] = (in && r1 > W) ? mu[P + p0 + c] : 0.0;
  }
  for (int r = r0; r < r1; ++r) {
    const TO* src = O + (size_t)r * P + p0;
    double v[8];
    if (VEC && sizeof(TO) == 4 && p0 + 8 <= P) {
      const float4 a = reinterpret_cast<const float4*>(src)[0];
      const float4 b = reinterpret_cast<const float4*>(src)[1];
      v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
      v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    } else {
#pragma unroll
      for (int c = 0; c < 8; ++c) v[c] = p0 + c < P ? (double)src[c] : 0.0;
    }
    const bool hi = r >= W;
    TD out[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const double x = p0 + c < P ? v[c] - (hi ? m1[c] : m0[c]) : 0.0;
      if constexpr (sizeof(TD) == 2)
        out[c] = __double2bfloat16(x);
      else
        out[c] = (TD)x;
    }
    TD* dst = D + (size_t)r * ldd + p0;
    if (p0 + 8 <= ldd) {
#pragma unroll
      for (int c = 0; c < 8 * (int)sizeof(TD) / 16; ++c)
        reinterpret_cast<int4*>(dst)[c] = reinterpret_cast<const int4*>(out)[c];
    } else {  // row end (ldd a multiple of 4, not 8): element stores inside the row only
      for (int c = 0; c < 8 && p0 + c < ldd; ++c) dst[c] = out[c];
    }
  }
}

}  // namespace tc

static int64_t tc_ld(int64_t P, int prec) {
  const int64_t a = prec == 1 ? 8 : 4;  // 16-byte row stride
  return (P + a - 1) / a * a;
}

size_t gram_tc_workspace(int W, int64_t P, int prec) {
  const size_t es = prec == 1 ? 2 : 4;
  return (size_t)2 * W * tc_ld(P, prec) * es + 1024;
}

// centred copy of O in the Gram operand type (ldd: multiple of 8 elements, 16-byte rows)
template <typename TD>
static int center_cvt(const void* O, int o_dtype, int W, int M, int64_t P, int64_t ldd,
                      const double* mu, TD* d, cudaStream_t st) {
  const dim3 g((unsigned)(((ldd + 7) / 8 + 255) / 256),
               (unsigned)((M + tc::CVT_ROWS - 1) / tc::CVT_ROWS));
  const bool vec = (P % 4) == 0 && (reinterpret_cast<uintptr_t>(O) & 15) == 0;
  if (o_dtype == 0)
    tc::k_center_cvt8<double, TD, false><<<g, 256, 0, st>>>((const double*)O, W, M, P, ldd, mu, d);
  else if (vec)
    tc::k_center_cvt8<float, TD, true><<<g, 256, 0, st>>>((const float*)O, W, M, P, ldd, mu, d);
  else
    tc::k_center_cvt8<float, TD, false><<<g, 256, 0, st>>>((const float*)O, W, M, P, ldd, mu, d);
  NQS_CHECK_LAUNCH("k_center_cvt8");
  return NQS_OK;
}

bool g_gram_wide = true;  // nqs_set_gram_wide

// Encode the tensor map and launch the Gram on an operand already in D (rows M, ld ldd).
int gram_tc_launch(const void* D, int prec, int M, int64_t K, int64_t ldd, double* T, int64_t ldt,
                   int* err, cudaStream_t st) {
  tc::EncodeTiledFn enc = tc::encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return NQS_ERR_CUDA;
  }
  const size_t es = prec == 1 ? 2 : 4;
  if ((reinterpret_cast<uintptr_t>(D) & 15) || ((ldd * es) & 15)) {
    set_error("gram_tc: operand not 16-byte aligned");
    return NQS_ERR_INVALID_ARG;
  }
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)K, (cuuint64_t)M};
  const cuuint64_t strides[1] = {(cuuint64_t)(ldd * es)};
  const cuuint32_t box[2] = {(cuuint32_t)(128 / es), (cuuint32_t)tc::BM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(&map, prec == 1 ? CU_TENSOR_MAP_DATA_TYPE_BFLOAT16
                                         : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                         2, const_cast<void*>(D), dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return NQS_ERR_CUDA;
  }
  const bool wide = g_gram_wide && M > tc::WBM;
  const int nrt = (M + (wide ? tc::WBM : tc::BM) - 1) / (wide ? tc::WBM : tc::BM);
  int tiles = 0;
  for (int i = 0; i < nrt; ++i) tiles += wide ? i + 1 : i / 2 + 1;
  // every column tile must start inside the matrix: col tile tj <= floor(ti/2) => j0 <= i0
  // (wide: tj <= ti)
  if (g_prof_start) cudaEventRecord(g_prof_start, st);
  // one launch per round of one tile per SM: the CTAs of a round start together and stream K
  // in step, so the operand rows they share are read from DRAM about once per round
  static int nsm = 0;
  if (!nsm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaFuncSetAttribute(tc::k_gram_tc<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::SMEM_BYTES);
    cudaFuncSetAttribute(tc::k_gram_tc<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::SMEM_BYTES);
    cudaFuncSetAttribute(tc::k_gram_tc_wide<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::WSMEM_BYTES);
    cudaFuncSetAttribute(tc::k_gram_tc_wide<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::WSMEM_BYTES);
  }
  const int per = std::max(nsm, 1);
  const uint32_t wl = wait_limit_or(tc::WAIT_LIMIT);
  for (int t0 = 0; t0 < tiles; t0 += per) {
    const int nt = std::min(per, tiles - t0);
    if (wide && prec == 1)
      tc::k_gram_tc_wide<0><<<nt, 128, tc::WSMEM_BYTES, st>>>(map, M, K, T, ldt, err, wl, t0);
    else if (wide)
      tc::k_gram_tc_wide<1><<<nt, 128, tc::WSMEM_BYTES, st>>>(map, M, K, T, ldt, err, wl, t0);
    else if (prec == 1)
      tc::k_gram_tc<0, false><<<nt, 128, tc::SMEM_BYTES, st>>>(map, M, K, T, ldt, err, wl, t0);
    else
      tc::k_gram_tc<1, false><<<nt, 128, tc::SMEM_BYTES, st>>>(map, M, K, T, ldt, err, wl, t0);
    NQS_CHECK_LAUNCH("k_gram_tc");
  }
  if (g_prof_stop) cudaEventRecord(g_prof_stop, st);
  return NQS_OK;
}

namespace tc {
// Z[r] = [hi | lo] of the float64 row A[r][0..K): hi = v rounded to TF32 (cvt.rna), lo = the
// float32 of the remainder v - hi. One CTA per row, one thread per column.
__global__ void k_split_tf32(const double* __restrict__ A, int64_t lda, int K,
                             float* __restrict__ Z) {
  const int r = blockIdx.x;
  for (int c = threadIdx.x; c < K; c += blockDim.x) {
    const double v = A[(size_t)r * lda + c];
    uint32_t hb;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hb) : "f"((float)v));
    const float hi = __uint_as_float(hb);
    Z[(size_t)r * 2 * K + c] = hi;
    Z[(size_t)r * 2 * K + K + c] = (float)(v - (double)hi);
  }
}
}  // namespace tc

size_t syrk_split_tf32_scratch_floats(int M, int K) { return (size_t)M * 2 * K; }

// C (lower, float64, M x M, ldc) -= A A^T for A (M x K float64, lda) through the split-TF32
// tensor-core Gram; Z: syrk_split_tf32_scratch_floats(M, K) floats, 16-byte aligned.
int syrk_split_tf32(const double* A, int64_t lda, int M, int K, double* C, int64_t ldc, float* Z,
                    int* err, cudaStream_t st) {
  if (K % 32 || (reinterpret_cast<uintptr_t>(Z) & 15) || (reinterpret_cast<uintptr_t>(C) & 15) ||
      (ldc & 1)) {
    set_error("syrk_split_tf32: K %% 32, scratch or C alignment");
    return NQS_ERR_INVALID_ARG;
  }
  tc::EncodeTiledFn enc = tc::encode_fn();
  if (!enc) {
    set_error("cuTensorMapEncodeTiled unavailable");
    return NQS_ERR_CUDA;
  }
  tc::k_split_tf32<<<M, 256, 0, st>>>(A, lda, K, Z);
  NQS_CHECK_LAUNCH("k_split_tf32");
  CUtensorMap map;
  const cuuint64_t dims[2] = {(cuuint64_t)(2 * K), (cuuint64_t)M};
  const cuuint64_t strides[1] = {(cuuint64_t)(2 * K * sizeof(float))};
  const cuuint32_t box[2] = {32, (cuuint32_t)tc::BM};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = enc(&map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, Z, dims, strides, box, estr,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                         CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
    return NQS_ERR_CUDA;
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(tc::k_gram_tc<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         tc::SMEM_BYTES);
    attr = true;
  }
  const int nrt = (M + tc::BM - 1) / tc::BM;
  int tiles = 0;
  for (int i = 0; i < nrt; ++i) tiles += i / 2 + 1;
  // K = 256: the tiles are bound by their read-modify-write of C, so one launch of all of them
  tc::k_gram_tc<1, true><<<tiles, 128, tc::SMEM_BYTES, st>>>(map, M, K, C, ldc, err,
                                                              wait_limit_or(tc::WAIT_LIMIT), 0);
  NQS_CHECK_LAUNCH("k_gram_tc<sub>");
  return NQS_OK;
}

int gram_tc(const void* O, int o_dtype, const double* mu, int W, int64_t P, int prec, double* T,
            Arena& ws, int nsm, cudaStream_t st, int* err) {
  (void)nsm;
  const int64_t ldd = tc_ld(P, prec);
  const int M = 2 * W;
  void* D;
  if (prec == 1) {
    __nv_bfloat16* d = ws.take<__nv_bfloat16>((size_t)M * ldd);
    if (!d) return NQS_ERR_WORKSPACE;
    NQS_TRY(center_cvt(O, o_dtype, W, M, P, ldd, mu, d, st));
    D = d;
  } else {
    float* d = ws.take<float>((size_t)M * ldd);
    if (!d) return NQS_ERR_WORKSPACE;
    NQS_TRY(center_cvt(O, o_dtype, W, M, P, ldd, mu, d, st));
    D = d;
  }
  return gram_tc_launch(D, prec, M, P, ldd, T, M, err, st);
}

}  // namespace nqs

extern "C" int nqs_set_gram_wide(int enable) {
  nqs::g_gram_wide = enable != 0;
  return NQS_OK;
}

extern "C" int nqs_gram(const void* A, int a_dtype, int M, int64_t K, int64_t lda, double* T,
                        int64_t ldt, int* err_dev, void* stream) {
  using namespace nqs;
  if (!A || !T || M < 1 || K < 1 || lda < K || ldt < M || (a_dtype != 1 && a_dtype != 2)) {
    set_error("nqs_gram: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  return gram_tc_launch(A, a_dtype, M, K, lda, T, ldt, err_dev, (cudaStream_t)stream);
}
