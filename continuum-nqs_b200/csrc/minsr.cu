// minsr.cu — MinSR natural-gradient direction in the sample space (src/nqs/minsr.py:68-88) and
// the median-MAD energy clip of the training loop (src/nqs/minsr.py:142-153).
//
//   Otil = [Re(O - mean O); Im(O - mean O)]  (2W x P),  etil = [Re(e - mean e); Im(...)]
//   T = Otil Otil^T (lower triangle),  (T + lam I) = L L^T (float64 Cholesky),
//   y = L^-T L^-1 etil,  dtheta = Otil^T y  (optionally theta -= lr dtheta, fused)
//
// The Gram runs either in float64 (SIMT, 128x128 tiles, register-blocked 8x8 per thread) or in
// BF16 on the tcgen05 tensor cores with float32 accumulation (gram_tc.cu). Everything after the
// Gram is float64.
#include <cstdio>
#include <algorithm>
#include <cmath>
#include <mutex>

#include <cooperative_groups.h>

#include "minsr.cuh"

namespace cg = cooperative_groups;

namespace nqs {

// ============================================================================================
// centering
// ============================================================================================
// column means of each half of O [2W][P] (TO = double or float) -> mu [2][P] (float64)
template <typename TO>
__global__ void k_colmean(const TO* __restrict__ O, int W, int64_t P, double* __restrict__ mu) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int half = blockIdx.y;
  if (p >= P) return;
  const TO* base = O + (size_t)half * W * P + p;
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
  int w = 0;
  for (; w + 3 < W; w += 4) {
    s0 += (double)base[(size_t)w * P];
    s1 += (double)base[(size_t)(w + 1) * P];
    s2 += (double)base[(size_t)(w + 2) * P];
    s3 += (double)base[(size_t)(w + 3) * P];
  }
  for (; w < W; ++w) s0 += (double)base[(size_t)w * P];
  mu[(size_t)half * P + p] = ((s0 + s1) + (s2 + s3)) / (double)W;
}

// Otil = O - mu (per half), written in place (float64) or converted to the Gram operand type
template <typename TO, typename TD>
__global__ void k_center(const TO* __restrict__ O, int W, int64_t P, const double* __restrict__ mu,
                         TD* __restrict__ D, int64_t ldd) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;  // row of the 2W rows
  if (p >= P) return;
  const int half = r >= W;
  D[(size_t)r * ldd + p] = (TD)((double)O[(size_t)r * P + p] - mu[(size_t)half * P + p]);
}

__global__ void k_center_eps(const cplx* __restrict__ e, int W, double* __restrict__ et) {
  // single block: mean then centre
  __shared__ double red[2][32];
  double sr = 0, si = 0;
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    sr += e[w].re;
    si += e[w].im;
  }
  sr = warp_sum(sr);
  si = warp_sum(si);
  if ((threadIdx.x & 31) == 0) {
    red[0][threadIdx.x >> 5] = sr;
    red[1][threadIdx.x >> 5] = si;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      a += red[0][i];
      b += red[1][i];
    }
    red[0][0] = a / W;
    red[1][0] = b / W;
  }
  __syncthreads();
  const double mr = red[0][0], mi = red[1][0];
  for (int w = threadIdx.x; w < W; w += blockDim.x) {
    et[w] = e[w].re - mr;
    et[W + w] = e[w].im - mi;
  }
}

// ============================================================================================
// float64 GEMM on lower-triangular tiles: C[i][j] = alpha sum_k A[i][k] B[j][k] + beta C[i][j]
// for the 128x128 tiles with tile_j <= tile_i (both operands K-contiguous). Split-K over
// blockIdx.z writes partial sums to Cpart[z] (beta ignored) when nsplit > 1.
// ============================================================================================
struct DTile {
  const double* A;
  int64_t lda;
  const double* B;
  int64_t ldb;
  double* C;
  int64_t ldc;
  int M;       // rows = cols of the lower-triangular block region
  int64_t K;
  double alpha, beta;
  int nsplit;
  int64_t kchunk;
  double* Cpart;  // [nsplit][M][M] when nsplit > 1
};

__device__ __forceinline__ void tile_of(int t, int* ti, int* tj) {
  // lower-triangular enumeration: t -> (i, j), j <= i
  int i = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
  while ((i + 1) * (i + 2) / 2 <= t) ++i;
  while (i * (i + 1) / 2 > t) --i;
  *ti = i;
  *tj = t - i * (i + 1) / 2;
}

__global__ void __launch_bounds__(256) k_dsyrk_lower(DTile a) {
  constexpr int BM = 128, BK = 8;
  __shared__ __align__(16) double As[2][BK][BM];
  __shared__ __align__(16) double Bs[2][BK][BM];
  int ti, tj;
  tile_of(blockIdx.x, &ti, &tj);
  const int i0 = ti * BM, j0 = tj * BM;
  const int64_t kb = (int64_t)blockIdx.z * a.kchunk;
  const int64_t ke = min(a.K, kb + a.kchunk);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  // loader: row = tid / 2, k-quad = (tid & 1) * 4
  const int lr = tid >> 1, lk = (tid & 1) * 4;
  double ra[4], rb[4];
  auto gload = [&](int64_t k0) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int64_t k = k0 + lk + q;
      const int gi = i0 + lr, gj = j0 + lr;
      ra[q] = (gi < a.M && k < ke) ? a.A[(size_t)gi * a.lda + k] : 0.0;
      rb[q] = (gj < a.M && k < ke) ? a.B[(size_t)gj * a.ldb + k] : 0.0;
    }
  };
  auto sstore = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      As[buf][lk + q][lr] = ra[q];
      Bs[buf][lk + q][lr] = rb[q];
    }
  };
  gload(kb);
  sstore(0);
  __syncthreads();
  int buf = 0;
  for (int64_t k0 = kb; k0 < ke; k0 += BK) {
    const bool more = k0 + BK < ke;
    if (more) gload(k0 + BK);
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      double av[8], bv[8];
      const double2* pa = reinterpret_cast<const double2*>(&As[buf][kk][0]);
      const double2* pb = reinterpret_cast<const double2*>(&Bs[buf][kk][0]);
      double2 t0 = pa[ty * 2], t1 = pa[ty * 2 + 1], t2 = pa[32 + ty * 2], t3 = pa[32 + ty * 2 + 1];
      av[0] = t0.x; av[1] = t0.y; av[2] = t1.x; av[3] = t1.y;
      av[4] = t2.x; av[5] = t2.y; av[6] = t3.x; av[7] = t3.y;
      t0 = pb[tx * 2]; t1 = pb[tx * 2 + 1]; t2 = pb[32 + tx * 2]; t3 = pb[32 + tx * 2 + 1];
      bv[0] = t0.x; bv[1] = t0.y; bv[2] = t1.x; bv[3] = t1.y;
      bv[4] = t2.x; bv[5] = t2.y; bv[6] = t3.x; bv[7] = t3.y;
#pragma unroll
      for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
    }
    if (more) {
      sstore(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
  // epilogue, one output row at a time: that row's C values are all loaded before any of them is
  // stored (loads may not move above stores to the same array, so element-wise read-modify-write
  // would serialise 64 memory round trips per thread)
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gi = i0 + (i < 4 ? ty * 4 + i : 64 + ty * 4 + (i - 4));
    if (gi >= a.M) continue;
    double cv[8];
    if (a.nsplit == 1 && a.beta != 0.0) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int gj = j0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
        cv[j] = (gj < a.M && gj <= gi) ? a.C[(size_t)gi * a.ldc + gj] : 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gj = j0 + (j < 4 ? tx * 4 + j : 64 + tx * 4 + (j - 4));
      if (gj >= a.M || gj > gi) continue;
      if (a.nsplit > 1)
        a.Cpart[((size_t)blockIdx.z * a.M + gi) * a.M + gj] = acc[i][j];
      else if (a.beta == 0.0)  // C is not read
        a.C[(size_t)gi * a.ldc + gj] = a.alpha * acc[i][j];
      else
        a.C[(size_t)gi * a.ldc + gj] = a.alpha * acc[i][j] + a.beta * cv[j];
    }
  }
}

// ---- same contraction with a 3-stage cp.async pipeline (operand rows 16-byte aligned) ----
// 128 x 128 tile, K in chunks of 16 doubles; thread (ty, tx) owns rows ty + 16 i and columns
// tx + 16 j (i, j < 8): a warp's A reads are broadcasts, its B reads at most 2-way bank conflicts.
// The shared row stride (18 doubles = 144 bytes) keeps every cp.async destination 16-byte aligned.
constexpr int DK = 16, DSTAGES = 3, DLD = DK + 2;
static_assert((DLD * sizeof(double)) % 16 == 0, "cp.async rows must start on 16 bytes");
// copies n_src (0, 8 or 16) bytes and zero-fills the rest of the 16
__device__ __forceinline__ void cp_async16_zfill(void* smem, const void* gmem, int n_src) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = n_src;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n)
               : "memory");
}

__global__ void __launch_bounds__(256) k_dsyrk_cp(DTile a) {
  extern __shared__ __align__(16) double dsm[];
  double* As = dsm;                                  // [DSTAGES][128][DLD]
  double* Bs = dsm + DSTAGES * 128 * DLD;            // [DSTAGES][128][DLD]
  int ti, tj;
  tile_of(blockIdx.x, &ti, &tj);
  const int i0 = ti * 128, j0 = tj * 128;
  const int64_t kb = (int64_t)blockIdx.z * a.kchunk;
  const int64_t ke = min(a.K, kb + a.kchunk);
  const int nk = (int)((ke - kb + DK - 1) / DK);
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // stage loader: 128 rows x 8 chunks of 2 doubles for A and for B = 2048 copies, 8 per thread
  auto load_stage = [&](int st, int kc) {
    const int64_t k0 = kb + (int64_t)kc * DK;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + 256 * q, r = idx >> 3, c = (idx & 7) * 2;
      const int64_t k = k0 + c;
      const int gi = i0 + r, gj = j0 + r;
      const int nb = k < ke ? (int)min((int64_t)16, (ke - k) * 8) : 0;
      const bool va = gi < a.M && nb > 0, vb = gj < a.M && nb > 0;
      cp_async16_zfill(As + ((size_t)st * 128 + r) * DLD + c,
                       va ? a.A + (size_t)gi * a.lda + k : a.A, va ? nb : 0);
      cp_async16_zfill(Bs + ((size_t)st * 128 + r) * DLD + c,
                       vb ? a.B + (size_t)gj * a.ldb + k : a.B, vb ? nb : 0);
    }
  };
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
#pragma unroll
  for (int s = 0; s < DSTAGES - 1; ++s) {
    if (s < nk) load_stage(s, s);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int kc = 0; kc < nk; ++kc) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(DSTAGES - 2) : "memory");
    __syncthreads();
    const int nxt = kc + DSTAGES - 1;
    if (nxt < nk) load_stage(nxt % DSTAGES, nxt);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    const double* as = As + (size_t)(kc % DSTAGES) * 128 * DLD;
    const double* bs = Bs + (size_t)(kc % DSTAGES) * 128 * DLD;
    // two k per step: one 16-byte shared load per row gives (k, k + 1) (rows start on 16 bytes:
    // DLD * 8 = 144)
#pragma unroll
    for (int kk = 0; kk < DK; kk += 2) {
      double2 av[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)
        av[i] = *reinterpret_cast<const double2*>(as + (ty + 16 * i) * DLD + kk);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double2 bv = *reinterpret_cast<const double2*>(bs + (tx + 16 * j) * DLD + kk);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][j] = fma(av[i].x, bv.x, acc[i][j]);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][j] = fma(av[i].y, bv.y, acc[i][j]);
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  // epilogue, one output row at a time (its C values loaded before any is stored)
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int gi = i0 + ty + 16 * i;
    if (gi >= a.M) continue;
    double cv[8];
    if (a.nsplit == 1 && a.beta != 0.0) {
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const int gj = j0 + tx + 16 * j;
        cv[j] = (gj < a.M && gj <= gi) ? a.C[(size_t)gi * a.ldc + gj] : 0.0;
      }
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int gj = j0 + tx + 16 * j;
      if (gj >= a.M || gj > gi) continue;
      if (a.nsplit > 1)
        a.Cpart[((size_t)blockIdx.z * a.M + gi) * a.M + gj] = acc[i][j];
      else if (a.beta == 0.0)
        a.C[(size_t)gi * a.ldc + gj] = a.alpha * acc[i][j];
      else
        a.C[(size_t)gi * a.ldc + gj] = a.alpha * acc[i][j] + a.beta * cv[j];
    }
  }
}

__global__ void k_splitk_reduce(const double* __restrict__ part, int nsplit, int M,
                                double* __restrict__ C, int64_t ldc, double alpha, double beta) {
  const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (int64_t)M * M) return;
  const int i = (int)(idx / M), j = (int)(idx - (int64_t)i * M);
  if (j > i) return;
  double s = 0;
  for (int z = 0; z < nsplit; ++z) s += part[(size_t)z * M * M + idx];
  double* c = C + (size_t)i * ldc + j;
  *c = alpha * s + (beta == 0.0 ? 0.0 : beta * (*c));
}

int dsyrk_lower(const double* A, int64_t lda, int M, int64_t K, double alpha, double beta,
                double* C, int64_t ldc, double* part, size_t part_elems, int nsm,
                cudaStream_t st) {
  if (M <= 0) return NQS_OK;
  const int nt = (M + 127) / 128;
  const int tiles = nt * (nt + 1) / 2;
  int nsplit = 1;
  if (part && tiles < 2 * nsm && K >= 4096) {
    nsplit = std::min<int>(16, (2 * nsm + tiles - 1) / tiles);
    while (nsplit > 1 && (size_t)nsplit * M * M > part_elems) --nsplit;
  }
  DTile a{A, lda, A, lda, C, ldc, M, K, alpha, beta, nsplit, 0, part};
  const bool cp = (reinterpret_cast<uintptr_t>(A) & 15) == 0 && (lda % 2) == 0;
  if (cp) {
    a.kchunk = ((K + nsplit - 1) / nsplit + DK - 1) / DK * DK;
    const size_t sm = sizeof(double) * 2 * DSTAGES * 128 * DLD;
    static bool attr = false;
    if (!attr) {
      cudaFuncSetAttribute(k_dsyrk_cp, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      attr = true;
    }
    k_dsyrk_cp<<<dim3(tiles, 1, nsplit), 256, sm, st>>>(a);
    NQS_CHECK_LAUNCH("k_dsyrk_cp");
  } else {
    a.kchunk = ((K + nsplit - 1) / nsplit + 7) / 8 * 8;
    k_dsyrk_lower<<<dim3(tiles, 1, nsplit), 256, 0, st>>>(a);
    NQS_CHECK_LAUNCH("k_dsyrk_lower");
  }
  if (nsplit > 1) {
    const int64_t n = (int64_t)M * M;
    k_splitk_reduce<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(part, nsplit, M, C, ldc, alpha,
                                                                  beta);
    NQS_CHECK_LAUNCH("k_splitk_reduce");
  }
  return NQS_OK;
}

// ============================================================================================
// Cholesky (right-looking, block 64) and triangular solves, float64
// ============================================================================================
constexpr int CB = 64;

// *floor = rel * max_i A[i][i]  (one CTA)
__global__ void k_pivot_floor(const double* __restrict__ A, int64_t lda, int n, double rel,
                              double* __restrict__ floor_out) {
  __shared__ double red[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, A[(size_t)i * lda + i]);
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t = fmax(t, red[i]);
    *floor_out = rel * t;
  }
}

__global__ void k_add_diag(double* A, int64_t lda, int n, double lam) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(size_t)i * lda + i] += lam;
}

// extra[0] = u * (mean diagonal), added to the diagonal together with lam
__global__ void k_add_diag_noise(double* A, int64_t lda, int n, double lam, double u,
                                 const double* __restrict__ mean_diag, double* __restrict__ extra) {
  const double x = u * (*mean_diag);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) A[(size_t)i * lda + i] += lam + x;
  if (i == 0 && extra) *extra = x;
}

// Diagonal-block Cholesky + panel solve of one right-looking step, fused. Every CTA factors the
// b x b diagonal block [k0, k0+b) redundantly in shared memory, in 8-column sub-panels: warp 0
// factors a sub-panel with its rows in registers (shuffles carry the pivot row's entries), the
// whole CTA then applies the sub-panel's rank-8 update a_ik -= sum_c a_ic a_kc / d_c to the
// trailing block (unscaled columns, square roots deferred to the end). The CTA then solves its
// share of the panel rows r in [k0+b, n): A[r][k0:k0+b] <- A[r][k0:k0+b] L^-T, four rows per warp
// side by side. The factor is written to Ld rather than into A (other CTAs may still be reading
// the block); the next step's CTA 0 (or k_store_diag after the last step) copies it into A.
// Pivots d_j below *floor_p are raised to it (counted in bad[2]); a non-positive pivot sets
// bad[0] (CTA 0 records both).

__global__ void __launch_bounds__(256) k_potrf_trsm(double* __restrict__ A, int64_t lda, int k0,
                                                    int n, const double* __restrict__ floor_p,
                                                    int* __restrict__ bad, int rpc,
                                                    double* __restrict__ Ld, int prev_k0) {
  __shared__ double L[CB][CB + 1];
  __shared__ double rdiag[CB];
  const int b = min(CB, n - k0);
  const int tid = threadIdx.x, lane = tid & 31;
  if (blockIdx.x == 0 && prev_k0 >= 0) {  // previous step's diagonal factor into A
    const int bp = min(CB, n - prev_k0);
    for (int idx = tid; idx < bp * bp; idx += blockDim.x) {
      const int i = idx / bp, j = idx - i * bp;
      if (j <= i) A[(size_t)(prev_k0 + i) * lda + prev_k0 + j] = Ld[idx];
    }
    __syncthreads();  // Ld is rewritten below by this CTA
  }
  const double fl = floor_p ? *floor_p : 0.0;
  __shared__ double dval[CB], dinv[CB];
  // working copy of the diagonal block (lower triangle) in L; it becomes the factor in place
  for (int idx = tid; idx < CB * CB; idx += blockDim.x) {
    const int i = idx / CB, k = idx - i * CB;
    L[i][k] = (i < b && k <= i) ? A[(size_t)(k0 + i) * lda + k0 + k] : 0.0;
  }
  __syncthreads();
  // eight 8-column sub-panels: warp 0 factors sub-panel [j0, j0 + jw) of rows [j0, b) with the
  // rows in registers (lane l: rows j0 + l and j0 + l + 32), unscaled columns a_ik -= a_ic a_kc / d_c
  // and pivots d_c (raised to the floor when below it); then every thread applies the sub-panel's
  // rank-jw update to the trailing block, four threads per row.
  for (int j0 = 0; j0 < b; j0 += 8) {
    const int jw = min(8, b - j0);
    if (tid < 32) {
      const int ra = j0 + lane, rb = j0 + lane + 32;
      double pa[8], pb[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        pa[c] = (ra < b && c < jw) ? L[ra][j0 + c] : 0.0;
        pb[c] = (rb < b && c < jw) ? L[rb][j0 + c] : 0.0;
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < jw) {
          double d = __shfl_sync(0xffffffffu, pa[c], c);  // row j0 + c, column c
          const bool floored = floor_p && !(d > fl);
          if (floored) d = fl;
          const bool pos = d > 0.0;
          if (lane == 0) {
            if (blockIdx.x == 0) {
              if (floored) atomicAdd(bad + 2, 1);
              if (!pos) bad[0] = 1;
            }
            dval[j0 + c] = d;
          }
          const double inv = pos ? 1.0 / d : NAN;
          if (lane == 0) dinv[j0 + c] = inv;
          if (lane == c) pa[c] = d;  // the (floored) pivot is the stored diagonal
#pragma unroll
          for (int k = c + 1; k < 8; ++k) {
            const double akc = __shfl_sync(0xffffffffu, pa[c], k) * inv;  // row j0 + k, column c
            if (k < jw) {
              pa[k] -= pa[c] * akc;
              pb[k] -= pb[c] * akc;
            }
          }
        }
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < jw && ra < b && ra >= j0 + c) L[ra][j0 + c] = pa[c];
        if (c < jw && rb < b) L[rb][j0 + c] = pb[c];
      }
    }
    __syncthreads();
    // trailing update: rows i, columns k in [j0 + jw, i]
    const int t0 = j0 + jw, m = b - t0;
    if (m > 0) {
      const int i = t0 + (tid >> 2), q = tid & 3;
      if (tid >> 2 < m) {
        double pi[8];
#pragma unroll
        for (int c = 0; c < 8; ++c) pi[c] = c < jw ? L[i][j0 + c] * dinv[j0 + c] : 0.0;
        for (int k = t0 + q; k <= i; k += 4) {
          double acc = 0.0;
#pragma unroll
          for (int c = 0; c < 8; ++c) acc = fma(pi[c], L[k][j0 + c], acc);
          L[i][k] -= acc;
        }
      }
    }
    __syncthreads();
  }
  // L[i][k] = a_ik / sqrt(d_k) (i > k), L[k][k] = sqrt(d_k): one square root and one
  // reciprocal per column, then products
  if (tid < b) {
    const double d = dval[tid];
    const double sd = d > 0.0 ? sqrt(d) : NAN;
    rdiag[tid] = 1.0 / sd;
    dval[tid] = sd;
  }
  __syncthreads();
  for (int idx = tid; idx < b * b; idx += blockDim.x) {
    const int i = idx / b, k = idx - i * b;
    if (k <= i) L[i][k] = (i == k) ? dval[k] : L[i][k] * rdiag[k];
  }
  __syncthreads();
  if (blockIdx.x == 0)
    for (int idx = tid; idx < b * b; idx += blockDim.x) {
      const int i = idx / b, j = idx - i * b;
      Ld[idx] = j <= i ? L[i][j] : 0.0;
    }
  // panel rows of this CTA, four per warp at once: x L^T = a ->
  //   x_j = (a_j - sum_{m<j} x_m L[j][m]) / L[j][j]
  const int w = tid >> 5, nw = blockDim.x >> 5;
  const int r_lo = k0 + b + blockIdx.x * rpc, r_hi = min(n, r_lo + rpc);
  for (int r0 = r_lo + 4 * w; r0 < r_hi; r0 += 4 * nw) {
    double x0[4], x1[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r0 + u;
      const double* row = A + (size_t)r * lda + k0;
      x0[u] = (r < r_hi && lane < b) ? row[lane] : 0.0;
      x1[u] = (r < r_hi && lane + 32 < b) ? row[lane + 32] : 0.0;
    }
    for (int j = 0; j < b; ++j) {
      const double rd = rdiag[j];
      const double l0 = (lane > j && lane < b) ? L[lane][j] : 0.0;
      const double l1 = (lane + 32 > j && lane + 32 < b) ? L[lane + 32][j] : 0.0;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double xj = __shfl_sync(0xffffffffu, j < 32 ? x0[u] : x1[u], j & 31) * rd;
        if (lane == (j & 31)) {
          if (j < 32)
            x0[u] = xj;
          else
            x1[u] = xj;
        }
        x0[u] -= xj * l0;
        x1[u] -= xj * l1;
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = r0 + u;
      if (r >= r_hi) break;
      double* row = A + (size_t)r * lda + k0;
      if (lane < b) row[lane] = x0[u];
      if (lane + 32 < b) row[lane + 32] = x1[u];
    }
  }
}

__global__ void k_store_diag(double* __restrict__ A, int64_t lda, int k0, int n,
                             const double* __restrict__ Ld) {
  const int b = min(CB, n - k0);
  for (int idx = threadIdx.x; idx < b * b; idx += blockDim.x) {
    const int i = idx / b, j = idx - i * b;
    if (j <= i) A[(size_t)(k0 + i) * lda + k0 + j] = Ld[idx];
  }
}

// Update of ncb consecutive 64-column blocks by a kw-wide panel (kw a multiple of 64):
//   block y (columns c0 + 64 y of the caller's frame): C_y[r][c] -= sum_j P_y[r][j] P_y[c][j]
//   for r in [0, rest - 64 y), c in [0, min(64, rest - 64 y)), c <= r,
// with P_y = P + 64 y ldp (rows 0.. of P_y are the rows matching block y's columns) and
// C_y = C + 64 y (ldc + 1). One CTA per (64 rows, block), 4 x 4 outputs per thread; the sum runs
// over the panel's 64-column chunks in order.
__global__ void __launch_bounds__(256) k_panel_update(const double* __restrict__ P, int64_t ldp,
                                                      int rest, double* __restrict__ C,
                                                      int64_t ldc, int kw) {
  extern __shared__ double pu_sm[];
  double(*Pr)[CB + 1] = reinterpret_cast<double(*)[CB + 1]>(pu_sm);
  double(*Pc)[CB + 1] = Pr + CB;
  const int y = blockIdx.y;
  const int rest_y = rest - CB * y;
  const int r0 = blockIdx.x * CB;
  if (r0 >= rest_y) return;  // whole CTA
  P += (size_t)CB * y * ldp;
  C += (size_t)CB * y * (ldc + 1);
  const int nr = min(CB, rest_y - r0), nc = min(CB, rest_y);
  const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
  double acc[4][4] = {};
  for (int kc = 0; kc < kw; kc += CB) {
    if (kc) __syncthreads();  // the previous chunk is no longer read
    for (int idx = threadIdx.x; idx < CB * CB; idx += blockDim.x) {
      const int i = idx / CB, j = idx - i * CB;
      Pr[i][j] = i < nr ? P[(size_t)(r0 + i) * ldp + kc + j] : 0.0;
      Pc[i][j] = i < nc ? P[(size_t)i * ldp + kc + j] : 0.0;
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < CB; ++k) {
      double a4[4], b4[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        a4[u] = Pr[ty + 16 * u][k];
        b4[u] = Pc[tx + 16 * u][k];
      }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) acc[u][v] = fma(a4[u], b4[v], acc[u][v]);
    }
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int r = r0 + ty + 16 * u;
    if (r >= rest_y) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int c = tx + 16 * v;
      if (c < nc && c <= r) C[(size_t)r * ldc + c] -= acc[u][v];
    }
  }
}

bool g_chol_tc = true;  // split-TF32 tensor-core trailing updates of a preconditioner factor

// Right-looking blocked Cholesky A = L L^T (lower triangle, in place), two-level: 64-column
// panels inside 256-column outer blocks. A panel updates only the columns of its own outer block
// (k_panel_update); the trailing matrix beyond an outer block is updated once, by all of its
// panels together (dsyrk with K = 256), so the trailing matrix is read and written once per
// outer block instead of once per panel. One step of look-ahead: after a panel, the next 64
// columns are updated first (at an outer-block end, by the whole outer block) and the next
// diagonal factor + panel solve run on a side stream while the rest of the step's updates run on
// the caller's stream (they touch disjoint columns).
// part: scratch of at least 64 x 64 doubles for the diagonal factor.
int cholesky_lower(double* A, int64_t lda, int n, int* bad, double* part, size_t part_elems,
                   int nsm, cudaStream_t st, const double* floor_p = nullptr) {
  if (!part || part_elems < (size_t)CB * CB) {
    set_error("cholesky_lower: scratch of %zu doubles < %d", part_elems, CB * CB);
    return NQS_ERR_WORKSPACE;
  }
  // side stream and two fork / join events per device, created once
  static cudaStream_t side[64] = {};
  static cudaEvent_t ev_fork[64] = {}, ev_join[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) return NQS_ERR_UNSUPPORTED;
  if (!side[dev]) {
    // highest priority: the look-ahead CTAs are scheduled as soon as trailing-update CTAs retire
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);
    if (cudaStreamCreateWithPriority(&side[dev], cudaStreamNonBlocking, hi) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_fork[dev], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&ev_join[dev], cudaEventDisableTiming) != cudaSuccess) {
      set_error("cholesky_lower: side stream / events");
      return NQS_ERR_CUDA;
    }
  }
  cudaStream_t s2 = side[dev];
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_panel_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)(sizeof(double) * 2 * CB * (CB + 1)));
    attr = true;
  }
  auto potrf = [&](int k0, int prev, cudaStream_t s) -> int {
    const int b = std::min(CB, n - k0);
    const int rest = n - k0 - b;
    const int rpc = rest > 0 ? std::max(32, (rest + 2 * nsm - 1) / (2 * nsm)) : 1;
    const int grid = rest > 0 ? (rest + rpc - 1) / rpc : 1;
    k_potrf_trsm<<<grid, 256, 0, s>>>(A, lda, k0, n, floor_p, bad, rpc, part, prev);
    NQS_CHECK_LAUNCH("k_potrf_trsm");
    return NQS_OK;
  };
  constexpr int NB = 4 * CB;  // outer block
  // columns [c0, c0 + 64 ncb) updated by the panel of columns [p0, p0 + kw)
  auto pupd = [&](int p0, int kw, int c0, int ncb) {
    const int rest = n - c0;
    k_panel_update<<<dim3((rest + CB - 1) / CB, ncb), 256, sizeof(double) * 2 * CB * (CB + 1),
                     st>>>(A + (size_t)c0 * lda + p0, lda, rest, A + (size_t)c0 * lda + c0, lda,
                           kw);
    NQS_CHECK_LAUNCH("k_panel_update");
    return NQS_OK;
  };
  NQS_TRY(potrf(0, -1, st));
  int last = 0;
  for (int k0 = 0; k0 + CB < n; k0 += CB) {
    const int ob = (k0 / NB) * NB, oe = std::min(n, ob + NB);  // this panel's outer block
    const int cs = k0 + CB;  // the next panel's first column
    const bool boundary = cs == oe;
    // (a) the next 64 columns: by this panel, or at an outer-block end by the whole outer block
    //     (whose updates of later columns were deferred)
    if (boundary)
      NQS_TRY(pupd(ob, oe - ob, cs, 1));
    else
      NQS_TRY(pupd(k0, CB, cs, 1));
    // next diagonal factor + panel solve on the side stream
    cudaEventRecord(ev_fork[dev], st);
    cudaStreamWaitEvent(s2, ev_fork[dev], 0);
    NQS_TRY(potrf(cs, k0, s2));
    cudaEventRecord(ev_join[dev], s2);
    last = cs;
    if (!boundary) {
      // (b) the rest of this outer block's columns, by this panel
      const int nb = (oe - cs - CB + CB - 1) / CB;
      if (nb > 0) NQS_TRY(pupd(k0, CB, cs + CB, nb));
    } else if (cs + CB < n) {
      // (c) the deferred trailing update beyond the next panel, by the whole outer block; for
      //     a preconditioner (pivot floor given) on the tensor cores with split-TF32 operands,
      //     staged past the diagonal factor's share of the scratch
      const int m0 = cs + CB, M = n - m0;
      double* C = A + (size_t)m0 * lda + m0;
      if (floor_p && g_chol_tc && oe - ob == NB && (lda & 1) == 0 &&
          (reinterpret_cast<uintptr_t>(C) & 15) == 0 &&
          part_elems >= (size_t)CB * CB + (syrk_split_tf32_scratch_floats(M, NB) + 1) / 2)
        NQS_TRY(syrk_split_tf32(A + (size_t)m0 * lda + ob, lda, M, NB, C, lda,
                                reinterpret_cast<float*>(part + CB * CB), bad + 1, st));
      else
        NQS_TRY(dsyrk_lower(A + (size_t)m0 * lda + ob, lda, M, oe - ob, -1.0, 1.0, C, lda,
                            nullptr, 0, nsm, st));
    }
    cudaStreamWaitEvent(st, ev_join[dev], 0);
  }
  k_store_diag<<<1, 256, 0, st>>>(A, lda, last, n, part);
  NQS_CHECK_LAUNCH("k_store_diag");
  return NQS_OK;
}

// the task-graph factorization (chol_dag.cu) where its operand layout and scratch allow, the
// launch-per-panel one otherwise (or when switched off)
static int cholesky_any(double* A, int64_t lda, int n, int* bad, double* part, size_t part_elems,
                        int nsm, cudaStream_t st, const double* floor_p = nullptr) {
  if (g_chol_dag && lda % 2 == 0 && (reinterpret_cast<uintptr_t>(A) & 15) == 0 &&
      part_elems >= cholesky_dag_scratch_elems(n))
    return cholesky_dag(A, lda, n, bad, part, part_elems, nsm, st, floor_p);
  return cholesky_lower(A, lda, n, bad, part, part_elems, nsm, st, floor_p);
}

// Inverses of the 64x64 diagonal blocks of a lower-triangular L: dinv[s] = L_ss^-1 (row-major
// 64x64 per block, zero-padded past n). One CTA per block, one thread per column of the inverse
// (forward substitution against e_j in shared memory).
__global__ void __launch_bounds__(CB) k_trtri_diag(const double* __restrict__ L, int64_t ldl, int n,
                                                   double* __restrict__ dinv) {
  extern __shared__ double trtri_sm[];
  double(*Ls)[CB + 1] = reinterpret_cast<double(*)[CB + 1]>(trtri_sm);
  double(*X)[CB + 1] = Ls + CB;
  const int s = blockIdx.x, k0 = s * CB, b = min(CB, n - k0);
  for (int idx = threadIdx.x; idx < CB * CB; idx += blockDim.x) {
    const int i = idx / CB, j = idx - i * CB;
    Ls[i][j] = (i < b && j <= i) ? L[(size_t)(k0 + i) * ldl + k0 + j] : 0.0;
    X[i][j] = 0.0;
  }
  __syncthreads();
  const int j = threadIdx.x;
  if (j < b) {
    X[j][j] = 1.0 / Ls[j][j];
    for (int i = j + 1; i < b; ++i) {
      double a0 = 0.0, a1 = 0.0;
      int k = j;
      for (; k + 1 < i; k += 2) {
        a0 = fma(Ls[i][k], X[k][j], a0);
        a1 = fma(Ls[i][k + 1], X[k + 1][j], a1);
      }
      if (k < i) a0 = fma(Ls[i][k], X[k][j], a0);
      X[i][j] = -(a0 + a1) / Ls[i][i];
    }
  }
  __syncthreads();
  double* D = dinv + (size_t)s * CB * CB;
  for (int idx = threadIdx.x; idx < CB * CB; idx += blockDim.x) {
    const int i = idx / CB, jj = idx - i * CB;
    D[idx] = X[i][jj];
  }
}

// doubles of the triangular-solve scratch for order n: 2 x 64 exchange + one 64x64 inverse per block
inline size_t trsv_elems(size_t n) { return 2 * CB + ((n + CB - 1) / CB) * CB * CB; }

static int trtri_diag(const double* L, int64_t ldl, int n, double* dinv, cudaStream_t st) {
  const size_t sm = sizeof(double) * 2 * CB * (CB + 1);
  cudaFuncSetAttribute(k_trtri_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  k_trtri_diag<<<(n + CB - 1) / CB, CB, sm, st>>>(L, ldl, n, dinv);
  NQS_CHECK_LAUNCH("k_trtri_diag");
  return NQS_OK;
}

// Triangular solves on the whole GPU (cooperative launch, one grid barrier per 64-block):
//   forward   L x = v:   x_s = D_s (v_s - sum_{t<s} L_st x_t)
//   transposed L^T x = v: x_s = D_s^T (v_s - sum_{t>s} L_ts^T x_t),   D_s = L_ss^-1 (k_trtri_diag)
// In step s the first CTA applies x_s to block s+1 and multiplies by D_{s+1} (two 64x64 mat-vecs
// whose operands it loaded into registers before the previous barrier), while every other CTA
// applies x_s to the blocks beyond s+1. v is overwritten with x; xb: 2 x 64 doubles.
__global__ void __launch_bounds__(256) k_trsv_grid(const double* __restrict__ L, int64_t ldl,
                                                   int n, const double* __restrict__ dinv,
                                                   double* __restrict__ v,
                                                   double* __restrict__ xb, int transposed,
                                                   const int* __restrict__ skip) {
  if (skip && *skip) return;  // uniform over the grid: written by an earlier launch
  cg::grid_group grid = cg::this_grid();
  const int nblk = (n + CB - 1) / CB;
  const int tid = threadIdx.x, lane = tid & 31;
  __shared__ double xs[CB];
  __shared__ double vs[CB];
  __shared__ double red[4][CB];
  auto blk = [&](int s) { return transposed ? nblk - 1 - s : s; };
  // CTA 0's thread layout for a 64x64 mat-vec y = A x: forward (row-major A): row = tid / 4,
  // columns q*16 .. q*16+15 (q = tid % 4); transposed: column m = tid % 64, rows q*16.. (q = tid / 64)
  double lreg[16], dreg[16];
  auto load_next = [&](int s1) {  // operands of step s1-1 -> block s1 (L panel) and D_{s1}
    const int kb = blk(s1) * CB, bb = min(CB, n - kb);
    const double* D = dinv + (size_t)blk(s1) * CB * CB;
    if (!transposed) {
      const int r = tid >> 2, q = tid & 3;
#pragma unroll
      for (int c = 0; c < 16; ++c) dreg[c] = D[r * CB + q * 16 + c];
      if (s1 > 0) {
        const int kp = blk(s1 - 1) * CB, bp = min(CB, n - kp);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int col = q * 16 + c;
          lreg[c] = (r < bb && col < bp) ? L[(size_t)(kb + r) * ldl + kp + col] : 0.0;
        }
      }
    } else {
      const int m = tid & 63, q = tid >> 6;
#pragma unroll
      for (int c = 0; c < 16; ++c) dreg[c] = D[(q * 16 + c) * CB + m];
      if (s1 > 0) {
        const int kp = blk(s1 - 1) * CB, bp = min(CB, n - kp);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int row = q * 16 + c;
          lreg[c] = (m < bb && row < bp) ? L[(size_t)(kp + row) * ldl + kb + m] : 0.0;
        }
      }
    }
  };
  // y = A_reg . x (x in shared memory, 64 long) reduced over the 4 partial sums -> out[64]
  auto matvec = [&](const double* reg, const double* x, double* out) {
    double acc = 0.0;
    if (!transposed) {
      const int q = tid & 3;
#pragma unroll
      for (int c = 0; c < 16; ++c) acc = fma(reg[c], x[q * 16 + c], acc);
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      if (q == 0) out[tid >> 2] = acc;
    } else {
      const int q = tid >> 6;
#pragma unroll
      for (int c = 0; c < 16; ++c) acc = fma(reg[c], x[q * 16 + c], acc);
      red[q][tid & 63] = acc;
      __syncthreads();
      if (tid < CB) out[tid] = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
    }
  };
  if (blockIdx.x == 0) {
    const int k0 = blk(0) * CB, b = min(CB, n - k0);
    load_next(0);
    if (tid < CB) vs[tid] = tid < b ? v[k0 + tid] : 0.0;
    __syncthreads();
    matvec(dreg, vs, xs);
    __syncthreads();
    if (tid < b) {
      v[k0 + tid] = xs[tid];
      xb[tid] = xs[tid];
    }
    if (nblk > 1) load_next(1);
  }
  grid.sync();
  for (int s = 0; s < nblk; ++s) {
    const int k0 = blk(s) * CB, b = min(CB, n - k0);
    const double* xcur = xb + (s & 1) * CB;
    if (tid < CB) xs[tid] = tid < b ? xcur[tid] : 0.0;
    __syncthreads();
    const bool more = s + 1 < nblk;
    const int k1 = more ? blk(s + 1) * CB : 0, b1 = more ? min(CB, n - k1) : 0;
    if (blockIdx.x == 0) {
      if (more) {
        matvec(lreg, xs, vs);  // vs = L-panel . x_s
        __syncthreads();
        if (tid < CB) vs[tid] = tid < b1 ? v[k1 + tid] - vs[tid] : 0.0;
        __syncthreads();
        matvec(dreg, vs, xs);  // x_{s+1} = D_{s+1} v
        __syncthreads();
        double* xn = xb + ((s + 1) & 1) * CB;
        if (tid < b1) {
          v[k1 + tid] = xs[tid];
          xn[tid] = xs[tid];
        }
        if (s + 2 < nblk) load_next(s + 2);
      }
    } else {
      // every other CTA: apply x_s to the rows (columns) beyond block s+1
      const int gw = ((blockIdx.x - 1) * blockDim.x + tid) >> 5;
      const int nwk = ((gridDim.x - 1) * blockDim.x) >> 5;
      if (!transposed) {
        for (int r = k0 + b + b1 + gw; r < n; r += nwk) {
          const double* lr = L + (size_t)r * ldl + k0;
          double acc = 0.0;
          for (int jj = lane; jj < b; jj += 32) acc = fma(lr[jj], xs[jj], acc);
          acc = warp_sum(acc);
          if (lane == 0) v[r] -= acc;
        }
      } else {
        const int lim = more ? k1 : 0;  // columns below block s+1's start
        for (int m = (blockIdx.x - 1) * blockDim.x + tid; m < lim;
             m += (gridDim.x - 1) * blockDim.x) {
          double acc = 0.0;
          for (int jj = 0; jj < b; ++jj) acc = fma(L[(size_t)(k0 + jj) * ldl + m], xs[jj], acc);
          v[m] -= acc;
        }
      }
    }
    grid.sync();
  }
}

// Triangular solves as a wavefront over 64-row blocks (one CTA per block row, all CTAs resident
// through a cooperative launch), without grid barriers:
//   forward    CTA s:  x_s = D_s (v_s - sum_{t<s} L_st x_t)        (t ascending)
//   transposed CTA s:  x_s = D_s^T (v_s - sum_{t>s} L_ts^T x_t)    (t descending)
// CTA s walks its dependencies in groups of four blocks: the group's operand panels L_st are
// loaded into registers first, then one wait on the flag of the group's last block (a block
// publishes only after all of its own dependencies, so that flag covers the group; release /
// acquire at GPU scope) and the four x_t are applied in order. The walk thus takes a quarter of
// the flag round trips, and the chain costs one flag hop and two 64 x 64 mat-vecs per block.
// Every wait is bounded: a CTA that gives up records the timeout in flag[kTrsvErrSlot],
// publishes NaN for its block (its dependants then finish at once) and
// returns. v is overwritten with x. Sums run in a fixed order (deterministic).
constexpr int kTrsvErrSlot = 255;  // flags[0..254]: blocks; flags[255]: timeout record
constexpr uint32_t kTrsvWaitLimit = 1u << 21;

__device__ __forceinline__ int ld_acquire_gpu(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__global__ void __launch_bounds__(256) k_trsv_flags(const double* __restrict__ L, int64_t ldl,
                                                    int n, const double* __restrict__ dinv,
                                                    double* v, int* flags, int transposed,
                                                    const int* __restrict__ skip,
                                                    uint32_t wait_limit, int dead_block) {
  // skip: uniform over the grid (written by an earlier launch), so no CTA is left waiting
  if (skip && *skip) return;
  const int nblk = (n + CB - 1) / CB;
  const int s = blockIdx.x;
  const int k0 = s * CB, bs = min(CB, n - k0);
  const int tid = threadIdx.x;
  __shared__ double red[4][CB];
  __shared__ double rhs[CB];
  // the wait's outcome, double-buffered by iteration parity: thread 0 writes iteration it+1's
  // slot only after every thread has passed iteration it+1's barrier, i.e. has read slot it
  __shared__ int give_up_buf[2];
  bool give_up = false;
  // forward: output row r = tid / 4, columns q, q+4, .., q+60 (q = tid % 4) of each 64-block
  // (a warp's load covers eight rows' 32-byte segments);
  // transposed: output m = tid % 64 (a column of L), rows q*16 .. q*16+15 (q = tid / 64)
  const int r = transposed ? (tid & 63) : (tid >> 2);
  const int q = transposed ? (tid >> 6) : (tid & 3);
  double dreg[16];
  {
    const double* D = dinv + (size_t)s * CB * CB;
#pragma unroll
    for (int c = 0; c < 16; ++c)
      dreg[c] = transposed ? D[(q * 16 + c) * CB + r] : D[r * CB + q + 4 * c];
  }
  double acc = 0.0;
  const int nt = transposed ? nblk - 1 - s : s;  // blocks this row depends on
  // this block's right-hand side: written by no other CTA, read before the wait chain
  const double vs = (tid < bs) ? v[k0 + tid] : 0.0;
  __syncthreads();
  constexpr int G = 4;
  for (int it0 = 0, gi = 0; it0 < nt; it0 += G, ++gi) {
    const int g = min(G, nt - it0);
    double lreg[G][16];
#pragma unroll
    for (int u = 0; u < G; ++u) {
      const int t = transposed ? nblk - 1 - (it0 + u) : it0 + u;
      const int kt = t * CB, bt = u < g ? min(CB, n - kt) : 0;
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        const int jj = transposed ? q * 16 + c : q + 4 * c;
        lreg[u][c] = 0.0;
        if (!transposed && r < bs && jj < bt) lreg[u][c] = L[(size_t)(k0 + r) * ldl + kt + jj];
        if (transposed && r < bs && jj < bt) lreg[u][c] = L[(size_t)(kt + jj) * ldl + k0 + r];
      }
    }
    const int t = transposed ? nblk - 1 - (it0 + g - 1) : it0 + g - 1;  // the group's last
    if (tid == 0) {
      int gu = 0;
      uint32_t w = 0;
      while (ld_acquire_gpu(flags + t) == 0) {
        if (++w >= wait_limit || ld_acquire_gpu(flags + kTrsvErrSlot) != 0) {
          gu = 1;
          break;
        }
        if (w > 64) __nanosleep(64);
      }
      give_up_buf[gi & 1] = gu;
    }
    __syncthreads();
    give_up = give_up_buf[gi & 1] != 0;
    if (give_up) break;
#pragma unroll
    for (int u = 0; u < G; ++u) {
      if (u < g) {
        const int tu = transposed ? nblk - 1 - (it0 + u) : it0 + u;
        const int kt = tu * CB, bt = min(CB, n - kt);
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int jj = transposed ? q * 16 + c : q + 4 * c;
          const double xj = jj < bt ? __ldcg(v + kt + jj) : 0.0;
          acc = fma(lreg[u][c], xj, acc);
        }
      }
    }
  }
  if (give_up) {
    if (tid == 0) atomicExch(flags + kTrsvErrSlot, 1);
    if (tid < bs) v[k0 + tid] = __longlong_as_double(0x7ff8000000000000ll);
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      st_release_gpu(flags + s, 1);
    }
    return;
  }
  // rhs = v_s - (sum over the four column quarters)
  if (!transposed) {
    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
    if (q == 0) red[0][r] = acc;  // the row sums, handed to thread r below
  }
  __syncthreads();
  if (!transposed) {
    if (tid < CB) rhs[tid] = tid < bs ? vs - red[0][tid] : 0.0;
  } else {
    red[q][r] = acc;
    __syncthreads();
    if (tid < CB)
      rhs[tid] = tid < bs ? vs - ((red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid])) : 0.0;
  }
  __syncthreads();
  // x_s = D rhs (forward) or D^T rhs (transposed)
  double xs = 0.0;
#pragma unroll
  for (int c = 0; c < 16; ++c) xs = fma(dreg[c], rhs[transposed ? q * 16 + c : q + 4 * c], xs);
  if (!transposed) {
    xs += __shfl_xor_sync(0xffffffffu, xs, 1);
    xs += __shfl_xor_sync(0xffffffffu, xs, 2);
    if (q == 0 && r < bs) v[k0 + r] = xs;
  } else {
    red[q][r] = xs;
    __syncthreads();
    if (tid < bs) v[k0 + tid] = (red[0][tid] + red[1][tid]) + (red[2][tid] + red[3][tid]);
  }
  __syncthreads();
  // dead_block (self-test of the bounded waits only; -1 otherwise): that block never publishes,
  // so its dependants run into their wait limit
  if (tid == 0 && s != dead_block) {
    __threadfence();
    st_release_gpu(flags + s, 1);
  }
}

static int trsv_grid(const double* L, int64_t ldl, int n, const double* dinv, double* v,
                     double* xb, int transposed, cudaStream_t st, const int* skip = nullptr,
                     uint32_t wait_limit = 0, int dead_block = -1) {
  if (!wait_limit) wait_limit = wait_limit_or(kTrsvWaitLimit);
  static int grid = 0;
  if (!grid) {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trsv_grid, 256, 0);
    grid = per >= 1 ? nsm : 1;  // one CTA per SM keeps the grid barrier cheap
  }
  // the wavefront form while its flags fit the 2 x 64 exchange buffer and every block row's CTA
  // can be resident at once; the grid-barrier form otherwise
  static int max_resident = 0;
  if (!max_resident) {
    int dev = 0, nsm = 0, per = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_trsv_flags, 256, 0);
    max_resident = std::max(1, nsm * per);
  }
  const int nblk = (n + CB - 1) / CB;
  static_assert(sizeof(int) * (kTrsvErrSlot + 1) <= sizeof(double) * 2 * CB, "flag slots");
  if (nblk <= kTrsvErrSlot && nblk <= max_resident) {
    int* flags = reinterpret_cast<int*>(xb);
    cudaMemsetAsync(flags, 0, sizeof(int) * (kTrsvErrSlot + 1), st);
    void* fargs[] = {(void*)&L,         (void*)&ldl,   (void*)&n,
                     (void*)&dinv,      (void*)&v,     (void*)&flags,
                     (void*)&transposed, (void*)&skip, (void*)&wait_limit,
                     (void*)&dead_block};
    const cudaError_t e =
        cudaLaunchCooperativeKernel((const void*)k_trsv_flags, nblk, 256, fargs, 0, st);
    if (e != cudaSuccess) return cuda_status(e, "k_trsv_flags");
    NQS_CHECK_LAUNCH("k_trsv_flags");
    return NQS_OK;
  }
  void* args[] = {(void*)&L,  (void*)&ldl, (void*)&n,          (void*)&dinv,
                  (void*)&v, (void*)&xb,  (void*)&transposed, (void*)&skip};
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_trsv_grid, grid, 256, args, 0, st);
  if (e != cudaSuccess) return cuda_status(e, "k_trsv_grid");
  NQS_CHECK_LAUNCH("k_trsv_grid");
  return NQS_OK;
}

// Double centring of a symmetric Gram held in its lower triangle, per walker half:
//   T <- C T C,  C = blockdiag(I - 1 1^T / W, I - 1 1^T / W)
// (makes the two null vectors created by centring O exact again after a low-precision Gram).
__global__ void k_gram_rowsums(const double* __restrict__ T, int n, int W,
                               double* __restrict__ rs) {
  const int i = blockIdx.x;
  double s0 = 0.0, s1 = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double t = j <= i ? T[(size_t)i * n + j] : T[(size_t)j * n + i];
    if (j < W) s0 += t; else s1 += t;
  }
  __shared__ double r0[32], r1[32];
  s0 = warp_sum(s0);
  s1 = warp_sum(s1);
  if ((threadIdx.x & 31) == 0) {
    r0[threadIdx.x >> 5] = s0;
    r1[threadIdx.x >> 5] = s1;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += r0[w];
      b += r1[w];
    }
    rs[2 * i] = a / W;
    rs[2 * i + 1] = b / W;
  }
}

__global__ void k_gram_blocksums(const double* __restrict__ rs, int n, int W,
                                 double* __restrict__ S) {
  // S[2a + b] = mean over rows i in half a of rs[i][b]
  __shared__ double red[4][32];
  double acc[4] = {0, 0, 0, 0};
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int a = i >= W;
    acc[2 * a] += rs[2 * i];
    acc[2 * a + 1] += rs[2 * i + 1];
  }
  for (int q = 0; q < 4; ++q) {
    const double v = warp_sum(acc[q]);
    if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = v;
  }
  __syncthreads();
  if (threadIdx.x < 4) {
    double t = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[threadIdx.x][w];
    S[threadIdx.x] = t / W;
  }
}

// T <- C T C + (alpha / W) [same half]: alpha = mean diagonal of T (from S[4]) lifts the two
// exact null directions of the centred Gram to a well-conditioned eigenvalue, so the factor of a
// low-precision Gram is a uniform preconditioner there (the energies are centred, so the
// solution has no component along them and dtheta = Otil^T y ignores them).
__global__ void k_gram_center(double* __restrict__ T, int n, int W, const double* __restrict__ rs,
                              const double* __restrict__ S) {
  const int i = blockIdx.y;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j > i) return;
  const int a = i >= W, b = j >= W;
  double t = T[(size_t)i * n + j] - rs[2 * i + b] - rs[2 * j + a] + S[2 * a + b];
  if (a == b) t += S[4] / W;
  T[(size_t)i * n + j] = t;
}

__global__ void k_mean_diag(const double* __restrict__ T, int n, double* __restrict__ out) {
  __shared__ double red[32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += T[(size_t)i * n + i];
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    *out = t / n;
  }
}

// error-free transformations (Knuth TwoSum, FMA TwoProduct) for compensated dot products
struct DD {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add_prod(double a, double b) {
    const double p = a * b;
    const double pe = fma(a, b, -p);
    const double t = s + p;
    const double z = t - s;
    c += ((s - (t - z)) + (p - z)) + pe;
    s = t;
  }
  __device__ __forceinline__ void add(double a) {
    const double t = s + a;
    const double z = t - s;
    c += (s - (t - z)) + (a - z);
    s = t;
  }
};

// out[k] = sum_m (O[m][k] - mu[m >= Mh][k]) x[m]  (mu nullable), compensated; out_lo (nullable)
// receives the low word of the double-double result; theta[k] -= lr out[k] when theta given
template <typename TO>
__global__ void k_gemv_t(const TO* __restrict__ O, int M, int Mh, int64_t K,
                         const double* __restrict__ mu, const double* __restrict__ x,
                         double* __restrict__ out, double* __restrict__ out_lo,
                         double* __restrict__ theta, double lr,
                         const int* __restrict__ skip = nullptr) {
  if (skip && *skip) return;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  const double m0 = mu ? mu[k] : 0.0, m1 = mu ? mu[K + k] : 0.0;
  DD acc;
  for (int m = 0; m < M; ++m) {
    const double o = (double)O[(size_t)m * K + k] - (m < Mh ? m0 : m1);
    acc.add_prod(o, x[m]);
  }
  const double hi = acc.s + acc.c;
  if (out) out[k] = hi;
  if (out_lo) out_lo[k] = acc.c - (hi - acc.s);
  if (theta) theta[k] -= lr * hi;
}

// Split form of k_gemv_t for the large solves: each thread owns 4 consecutive columns and one
// slice of rows (blockIdx.y) and writes its slice's partial sum to part[y][k]; k_gemv_t_reduce
// adds the slices in slice order. Float64 accumulation (the products of float32 O entries and
// float64 weights, summed over at most 512 rows per slice, then over the slices): residuals to
// float64 working accuracy, which is what the refinement against the exact operator needs to
// reproduce a float64 solve. VEC: K % 4 == 0 (16-byte row starts).
template <typename TO, bool VEC>
__global__ void __launch_bounds__(256) k_gemv_t_split(const TO* __restrict__ O, int M, int Mh,
                                                      int64_t K, const double* __restrict__ mu,
                                                      const double* __restrict__ x, int mchunk,
                                                      double* __restrict__ part,
                                                      const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t k0 = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (k0 >= K) return;
  const int m_lo = blockIdx.y * mchunk, m_hi = min(M, m_lo + mchunk);
  double m0[4], m1[4];
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const bool in = k0 + c < K;
    m0[c] = (mu && in) ? mu[k0 + c] : 0.0;
    m1[c] = (mu && in) ? mu[K + k0 + c] : 0.0;
  }
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  // eight rows per step, all eight rows' loads issued before the first is used (rows past the
  // slice re-read row m_lo with weight 0)
  constexpr int RU = 8;
  for (int mb = m_lo; mb < m_hi; mb += RU) {
    TO o[RU][4];
    double xm[RU];
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const bool in = mb + u < m_hi;
      const TO* row = O + (size_t)(in ? mb + u : m_lo) * K + k0;
      xm[u] = in ? x[mb + u] : 0.0;
      if (VEC) {
        if (sizeof(TO) == 4) {
          const float4 f = *reinterpret_cast<const float4*>(row);
          o[u][0] = f.x; o[u][1] = f.y; o[u][2] = f.z; o[u][3] = f.w;
        } else {
          const double2 a = reinterpret_cast<const double2*>(row)[0];
          const double2 b = reinterpret_cast<const double2*>(row)[1];
          o[u][0] = a.x; o[u][1] = a.y; o[u][2] = b.x; o[u][3] = b.y;
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) o[u][c] = k0 + c < K ? row[c] : TO(0);
      }
    }
#pragma unroll
    for (int u = 0; u < RU; ++u) {
      const bool lo_half = mb + u < Mh;
#pragma unroll
      for (int c = 0; c < 4; ++c)
        acc[c] = fma((double)o[u][c] - (lo_half ? m0[c] : m1[c]), xm[u], acc[c]);
    }
  }
#pragma unroll
  for (int c = 0; c < 4; ++c)
    if (k0 + c < K) part[(size_t)blockIdx.y * K + k0 + c] = acc[c];
}

template <typename TO>
__global__ void k_gemv_t_reduce(const double* __restrict__ part, int nsplit, int64_t K,
                                double* __restrict__ out, double* __restrict__ out_lo,
                                double* __restrict__ theta, double lr,
                                const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  double acc = 0.0;
  for (int z = 0; z < nsplit; ++z) acc += part[(size_t)z * K + k];
  if (out) out[k] = acc;
  if (out_lo) out_lo[k] = 0.0;
  if (theta) theta[k] -= lr * acc;
}

// out = (O - mu)^T x through the split kernel when the scratch holds the slices, else k_gemv_t
template <typename TO>
static int gemv_t(const TO* O, int M, int Mh, int64_t K, const double* mu, const double* x,
                  double* out, double* out_lo, double* theta, double lr, double* part,
                  size_t part_elems, cudaStream_t st, const int* skip = nullptr) {
  int nsplit = std::max(1, std::min(16, M / 512));
  while (nsplit > 1 && (size_t)nsplit * K > part_elems) --nsplit;
  if (nsplit <= 1 || !part) {
    k_gemv_t<TO><<<(unsigned)((K + 255) / 256), 256, 0, st>>>(O, M, Mh, K, mu, x, out, out_lo,
                                                               theta, lr, skip);
    NQS_CHECK_LAUNCH("k_gemv_t");
    return NQS_OK;
  }
  const int mchunk = (M + nsplit - 1) / nsplit;
  const dim3 g((unsigned)((K + 1023) / 1024), (unsigned)nsplit);
  if (K % 4 == 0)
    k_gemv_t_split<TO, true><<<g, 256, 0, st>>>(O, M, Mh, K, mu, x, mchunk, part, skip);
  else
    k_gemv_t_split<TO, false><<<g, 256, 0, st>>>(O, M, Mh, K, mu, x, mchunk, part, skip);
  NQS_CHECK_LAUNCH("k_gemv_t_split");
  k_gemv_t_reduce<TO><<<(unsigned)((K + 255) / 256), 256, 0, st>>>(part, nsplit, K, out, out_lo,
                                                                   theta, lr, skip);
  NQS_CHECK_LAUNCH("k_gemv_t_reduce");
  return NQS_OK;
}

// Residual r = b - lam x - (O - mu) v for RB rows per CTA (v and mu read once per CTA for all
// its rows), float64 accumulation; 4 consecutive columns per thread when VEC.
template <typename TO, int RB, bool VEC>
__global__ void __launch_bounds__(256, sizeof(TO) == 4 ? 2 : 1) k_gemv_n_resid_rows(
    const TO* __restrict__ O, int M, int Mh, int64_t K, const double* __restrict__ mu,
    const double* __restrict__ v, const double* __restrict__ b, double lam0,
    const double* __restrict__ lam_extra, const double* __restrict__ x, double* __restrict__ r,
    const int* __restrict__ skip) {
  if (skip && *skip) return;
  const double lam = lam0 + (lam_extra ? *lam_extra : 0.0);
  const int m0 = blockIdx.x * RB;
  const int nr = min(RB, M - m0);
  double acc[RB];
  bool hi_half[RB];
#pragma unroll
  for (int i = 0; i < RB; ++i) {
    acc[i] = 0.0;
    hi_half[i] = m0 + i >= Mh;
  }
  // which column-mean halves this CTA's rows use (uniform per CTA)
  const bool need0 = mu && m0 < Mh, need1 = mu && m0 + nr - 1 >= Mh;
  const int64_t step = (int64_t)blockDim.x * 4;
  for (int64_t k = (int64_t)threadIdx.x * 4; k < K; k += step) {
    double vv[4], u0[4], u1[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const bool in = VEC || k + c < K;
      vv[c] = in ? v[k + c] : 0.0;
      u0[c] = (need0 && in) ? mu[k + c] : 0.0;
      u1[c] = (need1 && in) ? mu[K + k + c] : 0.0;
    }
    // all RB rows' loads are issued before any of them is used (rows past the end read row
    // m0 again and are never reduced)
    TO o[RB][4];
#pragma unroll
    for (int i = 0; i < RB; ++i) {
      const TO* row = O + (size_t)(m0 + (i < nr ? i : 0)) * K + k;
      if (VEC) {
        if (sizeof(TO) == 4) {
          const float4 f = *reinterpret_cast<const float4*>(row);
          o[i][0] = f.x; o[i][1] = f.y; o[i][2] = f.z; o[i][3] = f.w;
        } else {
          const double2 a = reinterpret_cast<const double2*>(row)[0];
          const double2 bb = reinterpret_cast<const double2*>(row)[1];
          o[i][0] = a.x; o[i][1] = a.y; o[i][2] = bb.x; o[i][3] = bb.y;
        }
      } else {
#pragma unroll
        for (int c = 0; c < 4; ++c) o[i][c] = k + c < K ? row[c] : TO(0);
      }
    }
#pragma unroll
    for (int i = 0; i < RB; ++i)
#pragma unroll
      for (int c = 0; c < 4; ++c)
        acc[i] = fma((double)o[i][c] - (hi_half[i] ? u1[c] : u0[c]), vv[c], acc[i]);
  }
  __shared__ double red[RB][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < RB; ++i) {
    double a = acc[i];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) a += __shfl_xor_sync(0xffffffffu, a, off);
    if (lane == 0) red[i][w] = a;
  }
  __syncthreads();
  if (threadIdx.x < nr) {
    const int i = threadIdx.x, m = m0 + i;
    double t = 0.0;
    for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[i][q];
    r[m] = ((b ? b[m] : 0.0) - lam * x[m]) - t;
  }
}

template <typename TO>
static int gemv_n_resid(const TO* O, int M, int Mh, int64_t K, const double* mu, const double* v,
                        const double* b, double lam0, const double* lam_extra, const double* x,
                        double* r, cudaStream_t st, const int* skip = nullptr) {
  constexpr int RB = 16;
  const unsigned g = (unsigned)((M + RB - 1) / RB);
  if (K % 4 == 0)
    k_gemv_n_resid_rows<TO, RB, true><<<g, 256, 0, st>>>(O, M, Mh, K, mu, v, b, lam0, lam_extra,
                                                         x, r, skip);
  else
    k_gemv_n_resid_rows<TO, RB, false><<<g, 256, 0, st>>>(O, M, Mh, K, mu, v, b, lam0,
                                                          lam_extra, x, r, skip);
  NQS_CHECK_LAUNCH("k_gemv_n_resid_rows");
  return NQS_OK;
}

__global__ void k_scale_vec(double* x, int64_t n, double s) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}

// Adam (Kingma & Ba 2015) with bias correction, as optax.adam: m <- b1 m + (1-b1) g,
// v <- b2 v + (1-b2) g^2, theta <- theta - lr (m/c1) / (sqrt(v/c2) + eps)
__global__ void k_adam(double* __restrict__ th, const double* __restrict__ g, double* __restrict__ m,
                       double* __restrict__ v, int64_t n, double lr, double b1, double b2,
                       double eps, double c1, double c2) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double gi = g[i];
  const double mi = b1 * m[i] + (1.0 - b1) * gi;
  const double vi = b2 * v[i] + (1.0 - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  th[i] -= lr * (mi / c1) / (sqrt(vi / c2) + eps);
}

// The same step with optax's treatment of complex leaves (the reference's train.py applies
// optax.adam to jax.grad of a real loss). For a complex leaf element c = a + i b JAX's gradient is
// the complex number G = dL/da - i dL/db, optax keeps one complex first moment m_c of G and one
// real second moment v of |G|^2, and c <- c - lr (m_c/c1) / (sqrt(v/c2) + eps). On the real ravel
// (re block, im block) that is: the re component's first moment tracks dL/da, the im component's
// tracks -dL/db, both share v (|G|^2 = (dL/da)^2 + (dL/db)^2). partner[k] is the index of the
// other component of k's complex element, or -1 for a real parameter; g is the real-ravel
// gradient (dL/da, dL/db). Both components compute the same v.
__global__ void k_adam_complex(double* __restrict__ th, const double* __restrict__ g,
                               double* __restrict__ m, double* __restrict__ v,
                               const int64_t* __restrict__ partner, int64_t n, double lr,
                               double b1, double b2, double eps, double c1, double c2) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  const double gk = g[k];
  const int64_t q = partner[k];
  double gm = gk, sq = gk * gk;
  if (q >= 0) {
    const double gq = g[q];
    if (q < k) gm = -gk;  // the imaginary component: G = dL/da - i dL/db
    sq = q < k ? gq * gq + gk * gk : gk * gk + gq * gq;  // same rounding on both components
  }
  const double mk_ = b1 * m[k] + (1.0 - b1) * gm;
  const double vk = b2 * v[k] + (1.0 - b2) * sq;
  m[k] = mk_;
  v[k] = vk;
  th[k] -= lr * (mk_ / c1) / (sqrt(vk / c2) + eps);
}

__global__ void k_axpy(int n, const double* __restrict__ a, double* __restrict__ y) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a[i];
}

// Solve (A A^T + lam I) y = b given the Cholesky factor L of (A A^T + lam I), with n_refine
// steps of iterative refinement against the exact operator y -> A (A^T y) + lam y, where
// A = O - mu (centred on the fly). On return tmpK holds A^T y (tmpK_lo is spare scratch).
template <typename TO>
static int solve_refined(const double* L, int M, int Mh, int64_t K, const TO* O,
                         const double* mu, double lam, const double* lam_extra, const double* b,
                         double* y, double* r,
                         double* tmpK, double* tmpK_lo, double* xb, int n_refine,
                         double* part, size_t part_elems, cudaStream_t st) {
  double* dinv = xb + 2 * CB;  // the diagonal-block inverses follow the 2 x 64 exchange buffer
  NQS_TRY(trtri_diag(L, M, M, dinv, st));
  cudaMemcpyAsync(y, b, sizeof(double) * M, cudaMemcpyDeviceToDevice, st);
  NQS_TRY(trsv_grid(L, M, M, dinv, y, xb, 0, st));
  NQS_TRY(trsv_grid(L, M, M, dinv, y, xb, 1, st));
  for (int it = 0; it < n_refine; ++it) {
    NQS_TRY(gemv_t<TO>(O, M, Mh, K, mu, y, tmpK, nullptr, nullptr, 0.0, part, part_elems, st));
    NQS_TRY(gemv_n_resid<TO>(O, M, Mh, K, mu, tmpK, b, lam, lam_extra, y, r, st));
    NQS_TRY(trsv_grid(L, M, M, dinv, r, xb, 0, st));
    NQS_TRY(trsv_grid(L, M, M, dinv, r, xb, 1, st));
    k_axpy<<<(M + 255) / 256, 256, 0, st>>>(M, r, y);
    NQS_CHECK_LAUNCH("k_axpy");
  }
  return NQS_OK;
}

// --------------------------------------------------------------------------------------------
// Preconditioned conjugate gradients for (A A^T + lam I) y = b at the caller's lam, A = O - mu
// applied from O itself (float64 accumulation, two passes over O per iteration), preconditioned
// by M = L L^T, the float64 Cholesky factor of a tensor-core Gram + (lam + delta) I. Scalars stay
// on the device (no host synchronisation). pcg[0] = r.z, pcg[1] = r0.z0; it_info[0] = stop flag
// (1 converged, 2 breakdown), it_info[1] = iterations done. Once the flag is set every later
// kernel of the loop returns at once.
// --------------------------------------------------------------------------------------------
constexpr int kPcgThreads = 1024;

__device__ double block_sum_1024(double v, double* red) {
  v = warp_sum(v);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) red[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    red[32] = t;
  }
  __syncthreads();
  t = red[32];
  __syncthreads();
  return t;
}

// p = z, pcg[0] = pcg[1] = r.z, flags cleared
__global__ void __launch_bounds__(kPcgThreads) k_pcg_init(int n, const double* __restrict__ r,
                                                          const double* __restrict__ z,
                                                          double* __restrict__ p,
                                                          double* __restrict__ pcg,
                                                          int* __restrict__ it_info) {
  __shared__ double red[33];
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    p[i] = z[i];
    a = fma(r[i], z[i], a);
  }
  const double rz = block_sum_1024(a, red);
  if (threadIdx.x == 0) {
    pcg[0] = rz;
    pcg[1] = rz;
    it_info[0] = (rz > 0.0 && isfinite(rz)) ? 0 : 1;  // b = 0 (or M r = 0): nothing to do
    it_info[1] = 0;
  }
}

// qn = -A p: alpha = r.z / (p.A p); y += alpha p; r -= alpha A p (= r + alpha qn)
__global__ void __launch_bounds__(kPcgThreads) k_pcg_alpha(int n, const double* __restrict__ p,
                                                           const double* __restrict__ qn,
                                                           double* __restrict__ y,
                                                           double* __restrict__ r,
                                                           double* __restrict__ pcg,
                                                           int* __restrict__ it_info) {
  if (it_info[0]) return;
  __shared__ double red[33];
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a = fma(p[i], -qn[i], a);
  const double pAp = block_sum_1024(a, red);
  if (!(pAp > 0.0) || !isfinite(pAp)) {  // loss of positivity: keep the current iterate
    if (threadIdx.x == 0) it_info[0] = 2;
    return;
  }
  const double alpha = pcg[0] / pAp;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    y[i] = fma(alpha, p[i], y[i]);
    r[i] = fma(alpha, qn[i], r[i]);
  }
  if (threadIdx.x == 0) pcg[2] = alpha;
}

// g += alpha (O - mu)^T p alongside y += alpha p, so that g = (O - mu)^T y at every step without
// a pass over O at the end (skipped exactly when k_pcg_alpha left y unchanged)
__global__ void k_pcg_push(int64_t K, const double* __restrict__ u, const double* __restrict__ pcg,
                           double* __restrict__ g, const int* __restrict__ it_info) {
  if (it_info[0]) return;
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < K) g[k] = fma(pcg[2], u[k], g[k]);
}

// the direction from g = (O - mu)^T y: out = g and / or theta -= lr g
__global__ void k_pcg_finish(int64_t K, const double* __restrict__ g, double* __restrict__ out,
                             double* __restrict__ theta, double lr) {
  const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= K) return;
  if (out) out[k] = g[k];
  if (theta) theta[k] -= lr * g[k];
}

// z <- r (the triangular solves then overwrite z with M^-1 r)
__global__ void k_pcg_copy(int n, const double* __restrict__ r, double* __restrict__ z,
                           const int* __restrict__ it_info) {
  if (it_info[0]) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) z[i] = r[i];
}

// beta = r.z / previous r.z; p = z + beta p; stop when sqrt(r.z / r0.z0) <= tol
__global__ void __launch_bounds__(kPcgThreads) k_pcg_beta(int n, const double* __restrict__ r,
                                                          const double* __restrict__ z,
                                                          double* __restrict__ p,
                                                          double* __restrict__ pcg,
                                                          int* __restrict__ it_info, double tol) {
  if (it_info[0]) return;
  __shared__ double red[33];
  double a = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a = fma(r[i], z[i], a);
  const double rz = block_sum_1024(a, red);
  const double beta = rz / pcg[0];
  for (int i = threadIdx.x; i < n; i += blockDim.x) p[i] = fma(beta, p[i], z[i]);
  __syncthreads();
  if (threadIdx.x == 0) {
    pcg[0] = rz;
    it_info[1] += 1;
    if (!(rz > tol * tol * pcg[1])) it_info[0] = 1;
  }
}

template <typename TO>
static int solve_pcg(const double* L, int M, int Mh, int64_t K, const TO* O, const double* mu,
                     double lam, const double* b, double* y, double* r, double* z, double* p,
                     double* q, double* pcg, int* it_info, double* tmpK, double* g, double* xb,
                     int max_it, double tol, double* part, size_t part_elems, cudaStream_t st) {
  double* dinv = xb + 2 * CB;
  const unsigned kb = (unsigned)((K + 255) / 256);
  NQS_TRY(trtri_diag(L, M, M, dinv, st));
  // y0 = M^-1 b, r0 = b - A y0, z0 = M^-1 r0
  cudaMemcpyAsync(y, b, sizeof(double) * M, cudaMemcpyDeviceToDevice, st);
  NQS_TRY(trsv_grid(L, M, M, dinv, y, xb, 0, st));
  NQS_TRY(trsv_grid(L, M, M, dinv, y, xb, 1, st));
  NQS_TRY(gemv_t<TO>(O, M, Mh, K, mu, y, g, nullptr, nullptr, 0.0, part, part_elems, st));
  NQS_TRY(gemv_n_resid<TO>(O, M, Mh, K, mu, g, b, lam, nullptr, y, r, st));
  cudaMemcpyAsync(z, r, sizeof(double) * M, cudaMemcpyDeviceToDevice, st);
  NQS_TRY(trsv_grid(L, M, M, dinv, z, xb, 0, st));
  NQS_TRY(trsv_grid(L, M, M, dinv, z, xb, 1, st));
  k_pcg_init<<<1, kPcgThreads, 0, st>>>(M, r, z, p, pcg, it_info);
  NQS_CHECK_LAUNCH("k_pcg_init");
  for (int it = 0; it < max_it; ++it) {
    // q = -(A A^T + lam I) p
    NQS_TRY(gemv_t<TO>(O, M, Mh, K, mu, p, tmpK, nullptr, nullptr, 0.0, part, part_elems, st,
                       it_info));
    NQS_TRY(gemv_n_resid<TO>(O, M, Mh, K, mu, tmpK, nullptr, lam, nullptr, p, q, st, it_info));
    k_pcg_alpha<<<1, kPcgThreads, 0, st>>>(M, p, q, y, r, pcg, it_info);
    NQS_CHECK_LAUNCH("k_pcg_alpha");
    k_pcg_push<<<kb, 256, 0, st>>>(K, tmpK, pcg, g, it_info);
    NQS_CHECK_LAUNCH("k_pcg_push");
    k_pcg_copy<<<(M + 255) / 256, 256, 0, st>>>(M, r, z, it_info);
    NQS_CHECK_LAUNCH("k_pcg_copy");
    NQS_TRY(trsv_grid(L, M, M, dinv, z, xb, 0, st, it_info));
    NQS_TRY(trsv_grid(L, M, M, dinv, z, xb, 1, st, it_info));
    k_pcg_beta<<<1, kPcgThreads, 0, st>>>(M, r, z, p, pcg, it_info, tol);
    NQS_CHECK_LAUNCH("k_pcg_beta");
  }
  return NQS_OK;
}

// ============================================================================================
// energy statistics and median-MAD clip (single CTA, bitonic sort in shared memory)
// ============================================================================================
__device__ void bitonic_sort(double* a, int n2) {
  for (int k = 2; k <= n2; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = threadIdx.x; i < n2; i += blockDim.x) {
        const int l = i ^ j;
        if (l > i) {
          const bool up = (i & k) == 0;
          const double x = a[i], y = a[l];
          if ((x > y) == up) {
            a[i] = y;
            a[l] = x;
          }
        }
      }
      __syncthreads();
    }
}

__device__ double median_sorted(const double* a, int n) {
  return (n & 1) ? a[n / 2] : 0.5 * (a[n / 2 - 1] + a[n / 2]);
}

// stats: [0] mean Re e, [1] std(Re e)/sqrt(W) (ddof 0), [2] var(Re e), [3] median, [4] MAD
__global__ void __launch_bounds__(1024) k_clip(const cplx* __restrict__ e, int W, double clip_k,
                                               cplx* __restrict__ out, double* __restrict__ stats) {
  extern __shared__ double sa[];
  int n2 = 1;
  while (n2 < W) n2 <<= 1;
  for (int i = threadIdx.x; i < n2; i += blockDim.x) sa[i] = i < W ? e[i].re : INFINITY;
  __syncthreads();
  bitonic_sort(sa, n2);
  const double med = median_sorted(sa, W);
  __syncthreads();
  for (int i = threadIdx.x; i < n2; i += blockDim.x) sa[i] = i < W ? fabs(e[i].re - med) : INFINITY;
  __syncthreads();
  bitonic_sort(sa, n2);
  const double mad = median_sorted(sa, W) + 1e-12;
  __syncthreads();
  // two roundings, as the reference's `med - clip_k * mad` (no fused multiply-add)
  const double kmad = __dmul_rn(clip_k, mad);
  const double lo = __dsub_rn(med, kmad), hi = __dadd_rn(med, kmad);
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    const double r = e[i].re;
    out[i] = mk(fmin(fmax(r, lo), hi), e[i].im);
  }
  // mean and variance (two-pass)
  __shared__ double red[32];
  double s = 0;
  for (int i = threadIdx.x; i < W; i += blockDim.x) s += e[i].re;
  s = warp_sum(s);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    red[0] = t / W;
  }
  __syncthreads();
  const double mean = red[0];
  __syncthreads();
  double v = 0;
  for (int i = threadIdx.x; i < W; i += blockDim.x) {
    const double dd = e[i].re - mean;
    v += dd * dd;
  }
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0 && stats) {
    double t = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
    const double var = t / W;
    stats[0] = mean;
    stats[1] = sqrt(var) / sqrt((double)W);
    stats[2] = var;
    stats[3] = med;
    stats[4] = mad;
  }
}

// ============================================================================================
// host driver
// ============================================================================================
// relative reduction of the preconditioned residual sqrt(r.z / r0.z0) at which the conjugate
// gradients stop by default
constexpr double kPcgDefaultTol = 1e-2;
// shift of the preconditioner factor, relative to mean(T_ii) (nqs_set_preconditioner_shift)
constexpr double kPrecondShiftDefault = 1e-4;
static double g_precond_shift = kPrecondShiftDefault;

// caller-facing status from the internal slots: [0] non-positive pivot, [1] Gram timeout,
// [2] floored pivots, [3] PCG iterations, [4] PCG stop reason (0 iteration limit, 1 converged,
// 2 breakdown); n_info of them are written
__global__ void k_pack_info(const int* __restrict__ bad, int* __restrict__ info, int n_info) {
  if (threadIdx.x != 0) return;
  const int v[5] = {bad[0], bad[1], bad[2], bad[5], bad[4]};
  for (int i = 0; i < n_info && i < 5; ++i) info[i] = v[i];
}
size_t minsr_part_elems(int W) {
  const size_t n = 2 * (size_t)W;
  return std::max<size_t>(std::min<size_t>(16 * n * n, (size_t)8 << 20), (size_t)CB * CB);
}

size_t minsr_workspace(int W, int64_t P, int odtype, int gram) {
  const size_t n = 2 * (size_t)W;
  size_t b = 0;
  auto add = [&](size_t x) { b += ((x + 255) / 256) * 256 + 256; };
  add(sizeof(double) * 2 * P);          // column means
  add(sizeof(double) * n);              // etil
  add(sizeof(double) * n);              // y
  add(sizeof(double) * n);              // refinement / PCG residual
  add(sizeof(double) * 3 * n);          // PCG z, p, q
  add(sizeof(double) * 4);              // PCG scalars
  add(sizeof(double) * 2 * P);          // Otil^T y and a spare P-vector
  add(sizeof(double) * n * n);          // T -> L
  add(sizeof(double) * (2 * n + 5));    // Gram row sums, block sums, mean diagonal
  add(sizeof(double) * trsv_elems(n));  // triangular-solve exchange + diagonal-block inverses
  add(sizeof(int) * 8);                 // status, PCG stop flag and iteration count
  add(sizeof(double) * 2);              // pivot floor, extra damping
  add(sizeof(double) * minsr_part_elems(W));  // split-K partials
  if (gram == 0 && odtype == 1) add(sizeof(double) * n * P);  // float64 Otil from float32 O
  if (gram != 0) add(gram_tc_workspace(W, P, gram));
  return b;
}

}  // namespace nqs

using namespace nqs;

extern "C" {

int nqs_minsr_workspace_size(int W, int64_t P, int o_dtype, int gram_prec, size_t* bytes) {
  if (!bytes || W < 1 || P < 1) return NQS_ERR_INVALID_ARG;
  *bytes = minsr_workspace(W, P, o_dtype, gram_prec);
  return NQS_OK;
}

static int minsr_direction_impl(void* O, int o_dtype, const double* eps, int W, int64_t P,
                                double lam, int gram_prec, int max_it, double tol,
                                double* out_dtheta, double* theta_io, double lr, int* info_dev,
                                int n_info, double* damping_out, void* wsp, size_t wsb,
                                cudaStream_t st) {
  if (!O || !eps || W < 1 || P < 1 || (o_dtype != 0 && o_dtype != 1) || gram_prec < 0 ||
      gram_prec > 2 || max_it < 0 || max_it > 64 || !(tol >= 0.0) ||
      (!out_dtheta && !theta_io)) {
    set_error("nqs_minsr_direction: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  const size_t need = minsr_workspace(W, P, o_dtype, gram_prec);
  if (wsb < need) {
    set_error("nqs_minsr_direction: workspace %zu < %zu", wsb, need);
    return NQS_ERR_WORKSPACE;
  }
  Arena ws{(char*)wsp, wsb, 0};
  const int n = 2 * W;
  double* mu = ws.take<double>(2 * P);
  double* et = ws.take<double>(n);
  double* y = ws.take<double>(n);
  double* r = ws.take<double>(n);
  double* zpq = ws.take<double>(3 * (size_t)n);
  double* pcg = ws.take<double>(4);
  double* tmpK = ws.take<double>(P);
  double* tmpK_lo = ws.take<double>(P);
  double* xb = ws.take<double>(trsv_elems(n));
  double* rsum = ws.take<double>(2 * (size_t)n + 5);
  double* T = ws.take<double>((size_t)n * n);
  int* bad = ws.take<int>(8);  // [0..2] status, [4] PCG stop reason, [5] PCG iterations
  const size_t part_elems = minsr_part_elems(W);
  double* part = ws.take<double>(part_elems);
  if (!part) return NQS_ERR_WORKSPACE;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaMemsetAsync(bad, 0, sizeof(int) * 8, st);
  const dim3 cg((unsigned)((P + 255) / 256), 2);
  if (o_dtype == 0)
    k_colmean<double><<<cg, 256, 0, st>>>((const double*)O, W, P, mu);
  else
    k_colmean<float><<<cg, 256, 0, st>>>((const float*)O, W, P, mu);
  NQS_CHECK_LAUNCH("k_colmean");
  k_center_eps<<<1, 1024, 0, st>>>((const cplx*)eps, W, et);
  NQS_CHECK_LAUNCH("k_center_eps");
  const dim3 ce((unsigned)((P + 255) / 256), (unsigned)n);
  const void* Oop = O;        // operand of the refinement / push-through
  int op_dtype = o_dtype;
  const double* mu_op = mu;
  if (gram_prec == 0) {
    double* Ot;
    if (o_dtype == 0) {  // centre in place
      k_center<double, double><<<ce, 256, 0, st>>>((const double*)O, W, P, mu, (double*)O, P);
      Ot = (double*)O;
    } else {
      Ot = ws.take<double>((size_t)n * P);
      if (!Ot) return NQS_ERR_WORKSPACE;
      k_center<float, double><<<ce, 256, 0, st>>>((const float*)O, W, P, mu, Ot, P);
    }
    NQS_CHECK_LAUNCH("k_center");
    if (g_prof_start) cudaEventRecord(g_prof_start, st);
    NQS_TRY(dsyrk_lower(Ot, P, n, P, 1.0, 0.0, T, n, part, part_elems, nsm, st));
    if (g_prof_stop) cudaEventRecord(g_prof_stop, st);
    Oop = Ot;
    op_dtype = 0;
    mu_op = nullptr;
  } else {
    NQS_TRY(gram_tc(O, o_dtype, mu, W, P, gram_prec, T, ws, nsm, st, bad + 1));
    k_gram_rowsums<<<n, 256, 0, st>>>(T, n, W, rsum);
    NQS_CHECK_LAUNCH("k_gram_rowsums");
    k_gram_blocksums<<<1, 1024, 0, st>>>(rsum, n, W, rsum + 2 * n);
    NQS_CHECK_LAUNCH("k_gram_blocksums");
    k_mean_diag<<<1, 1024, 0, st>>>(T, n, rsum + 2 * n + 4);
    NQS_CHECK_LAUNCH("k_mean_diag");
    k_gram_center<<<dim3((n + 255) / 256, n), 256, 0, st>>>(T, n, W, rsum, rsum + 2 * n);
    NQS_CHECK_LAUNCH("k_gram_center");
  }
  // A tensor-core Gram differs from Otil Otil^T by its operand rounding (a PSD perturbation of
  // the small eigenvalues) and by the float32 accumulation (a slightly indefinite one, of order
  // 1e-4 mean(T_ii) on the Jacobians of the wavefunction). Its Cholesky factor with the shift
  // lam + delta, delta = 1e-4 mean(T_ii), preconditions conjugate gradients on the exact system
  // (Otil Otil^T + lam I) y = etil, applied from O itself: the solve is at the caller's lam.
  const double* floor_p = nullptr;
  if (gram_prec == 0) {
    k_add_diag<<<(n + 255) / 256, 256, 0, st>>>(T, n, n, lam);
    NQS_CHECK_LAUNCH("k_add_diag");
    if (damping_out) cudaMemsetAsync(damping_out, 0, sizeof(double), st);
  } else {
    double* fl = ws.take<double>(2);
    if (!fl) return NQS_ERR_WORKSPACE;
    k_add_diag_noise<<<(n + 255) / 256, 256, 0, st>>>(T, n, n, lam, g_precond_shift,
                                                       rsum + 2 * n + 4,
                                                       fl + 1);
    NQS_CHECK_LAUNCH("k_add_diag_noise");
    k_pivot_floor<<<1, 1024, 0, st>>>(T, n, n, gram_prec == 1 ? 0x1p-16 : 0x1p-20, fl);
    NQS_CHECK_LAUNCH("k_pivot_floor");
    floor_p = fl;
    if (damping_out) cudaMemcpyAsync(damping_out, fl + 1, sizeof(double), cudaMemcpyDeviceToDevice, st);
  }
  NQS_TRY(cholesky_any(T, n, n, bad, part, part_elems, nsm, st, floor_p));
  double* z = zpq;
  double* pp = zpq + n;
  double* q = zpq + 2 * (size_t)n;
  if (gram_prec == 0) {
    if (op_dtype == 0)
      NQS_TRY(solve_refined<double>(T, n, W, P, (const double*)Oop, mu_op, lam, nullptr, et, y, r,
                                    tmpK, tmpK_lo, xb, max_it, part, part_elems, st));
    else
      NQS_TRY(solve_refined<float>(T, n, W, P, (const float*)Oop, mu_op, lam, nullptr, et, y, r,
                                   tmpK, tmpK_lo, xb, max_it, part, part_elems, st));
  } else {
    // the conjugate gradients keep tmpK_lo = (O - mu)^T y, so the direction needs no further
    // pass over O
    if (op_dtype == 0)
      NQS_TRY(solve_pcg<double>(T, n, W, P, (const double*)Oop, mu_op, lam, et, y, r, z, pp, q,
                                pcg, bad + 4, tmpK, tmpK_lo, xb, max_it, tol, part, part_elems,
                                st));
    else
      NQS_TRY(solve_pcg<float>(T, n, W, P, (const float*)Oop, mu_op, lam, et, y, r, z, pp, q, pcg,
                               bad + 4, tmpK, tmpK_lo, xb, max_it, tol, part, part_elems, st));
    k_pcg_finish<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(P, tmpK_lo, out_dtheta, theta_io,
                                                             lr);
    NQS_CHECK_LAUNCH("k_pcg_finish");
  }
  if (gram_prec == 0) {
    if (op_dtype == 0)
      NQS_TRY(gemv_t<double>((const double*)Oop, n, W, P, mu_op, y, out_dtheta, nullptr,
                             theta_io, lr, part, part_elems, st));
    else
      NQS_TRY(gemv_t<float>((const float*)Oop, n, W, P, mu_op, y, out_dtheta, nullptr, theta_io,
                            lr, part, part_elems, st));
  }
  if (info_dev) {
    k_pack_info<<<1, 32, 0, st>>>(bad, info_dev, n_info);
    NQS_CHECK_LAUNCH("k_pack_info");
  }
  return NQS_OK;
}

int nqs_minsr_direction(void* O, int o_dtype, const double* eps, int W, int64_t P, double lam,
                        int gram_prec, int n_refine, double* out_dtheta, double* theta_io,
                        double lr, int* status_dev, double* damping_out, void* wsp, size_t wsb,
                        void* stream) {
  return minsr_direction_impl(O, o_dtype, eps, W, P, lam, gram_prec, n_refine, kPcgDefaultTol,
                              out_dtheta, theta_io, lr, status_dev, 3, damping_out, wsp, wsb,
                              (cudaStream_t)stream);
}

int nqs_minsr_direction_ex(void* O, int o_dtype, const double* eps, int W, int64_t P,
                           double lam, int gram_prec, int max_iters, double tol,
                           double* out_dtheta, double* theta_io, double lr, int* info_dev,
                           double* damping_out, void* wsp, size_t wsb, void* stream) {
  return minsr_direction_impl(O, o_dtype, eps, W, P, lam, gram_prec, max_iters, tol, out_dtheta,
                              theta_io, lr, info_dev, 5, damping_out, wsp, wsb,
                              (cudaStream_t)stream);
}

int nqs_set_preconditioner_shift(double rel) {
  if (!(rel >= 0.0)) return NQS_ERR_INVALID_ARG;
  nqs::g_precond_shift = rel > 0.0 ? rel : nqs::kPrecondShiftDefault;
  return NQS_OK;
}

int nqs_set_cholesky_tc(int enable) {
  nqs::g_chol_tc = enable != 0;
  return NQS_OK;
}

int nqs_set_cholesky_dag(int enable) {
  g_chol_dag = enable != 0;
  return NQS_OK;
}

int nqs_selftest_bounded_wait(const double* L, int n, int dead_block, unsigned wait_limit,
                              double* v, void* wsp, size_t wsb, int* status_dev, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (!L || !v || !wsp || !status_dev || n < 1 || n > CB * kTrsvErrSlot || wait_limit < 1 ||
      dead_block < -1 || dead_block >= (n + CB - 1) / CB) {
    set_error("nqs_selftest_bounded_wait: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  if (wsb < sizeof(double) * trsv_elems(n)) {
    set_error("nqs_selftest_bounded_wait: workspace %zu < %zu", wsb,
              sizeof(double) * trsv_elems(n));
    return NQS_ERR_WORKSPACE;
  }
  double* xb = (double*)wsp;
  double* dinv = xb + 2 * CB;
  NQS_TRY(trtri_diag(L, n, n, dinv, st));
  NQS_TRY(trsv_grid(L, n, n, dinv, v, xb, 0, st, nullptr, wait_limit, dead_block));
  const cudaError_t e = cudaMemcpyAsync(status_dev, reinterpret_cast<int*>(xb) + kTrsvErrSlot,
                                        sizeof(int), cudaMemcpyDeviceToDevice, st);
  return e == cudaSuccess ? NQS_OK : cuda_status(e, "nqs_selftest_bounded_wait");
}

int nqs_gram_solve_workspace_size(int M, int64_t K, size_t* bytes) {
  if (!bytes || M < 1 || K < 1) return NQS_ERR_INVALID_ARG;
  const size_t m = (size_t)M;
  *bytes = sizeof(double) * (m * m + 2 * m + 2 * (size_t)K + trsv_elems(m) +
                             std::max<size_t>(std::min<size_t>(16 * m * m, (size_t)8 << 20),
                                              (size_t)CB * CB)) + 8192;
  return NQS_OK;
}

int nqs_gram_solve(const double* A, int M, int64_t K, double lam, const double* rhs, double* x,
                   void* wsp, size_t wsb, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  size_t need = 0;
  NQS_TRY(nqs_gram_solve_workspace_size(M, K, &need));
  if (!A || !rhs || !x) return NQS_ERR_INVALID_ARG;
  if (wsb < need) return NQS_ERR_WORKSPACE;
  Arena ws{(char*)wsp, wsb, 0};
  double* T = ws.take<double>((size_t)M * M);
  double* r = ws.take<double>(M);
  double* tmpK = ws.take<double>(K);
  double* tmpK_lo = ws.take<double>(K);
  const size_t pe = std::max<size_t>(std::min<size_t>(16 * (size_t)M * M, (size_t)8 << 20),
                                     (size_t)CB * CB);
  double* part = ws.take<double>(pe);
  int* bad = ws.take<int>(4);
  if (!bad) return NQS_ERR_WORKSPACE;
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaMemsetAsync(bad, 0, sizeof(int) * 4, st);
  NQS_TRY(dsyrk_lower(A, K, M, K, 1.0, 0.0, T, M, part, pe, nsm, st));
  k_add_diag<<<(M + 255) / 256, 256, 0, st>>>(T, M, M, lam);
  NQS_CHECK_LAUNCH("k_add_diag");
  NQS_TRY(cholesky_any(T, M, M, bad, part, pe, nsm, st));
  double* xb = ws.take<double>(trsv_elems(M));
  if (!xb) return NQS_ERR_WORKSPACE;
  NQS_TRY(solve_refined<double>(T, M, M, K, A, nullptr, lam, nullptr, rhs, x, r, tmpK, tmpK_lo, xb,
                                3, part, pe, st));
  return NQS_OK;
}

int nqs_energy_gradient(const void* O, int o_dtype, const double* e, int W, int64_t P,
                        double* out_grad, void* wsp, size_t wsb, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (!O || !e || !out_grad || W < 1 || P < 1 || (o_dtype != 0 && o_dtype != 1) || !wsp) {
    set_error("nqs_energy_gradient: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  if (wsb < sizeof(double) * 2 * (size_t)W + 256) {
    set_error("nqs_energy_gradient: workspace %zu < %zu", wsb, sizeof(double) * 2 * (size_t)W + 256);
    return NQS_ERR_WORKSPACE;
  }
  double* x = (double*)wsp;
  k_center_eps<<<1, 1024, 0, st>>>((const cplx*)e, W, x);
  NQS_CHECK_LAUNCH("k_center_eps");
  const unsigned gp = (unsigned)((P + 255) / 256);
  // g = (2/W) sum_w Re(conj(e_w - mean e) O_w) = (2/W) O_rows^T [Re eps; Im eps]
  if (o_dtype == 0)
    k_gemv_t<double><<<gp, 256, 0, st>>>((const double*)O, 2 * W, 2 * W, P, nullptr, x, out_grad,
                                         nullptr, nullptr, 0.0);
  else
    k_gemv_t<float><<<gp, 256, 0, st>>>((const float*)O, 2 * W, 2 * W, P, nullptr, x, out_grad,
                                        nullptr, nullptr, 0.0);
  NQS_CHECK_LAUNCH("k_gemv_t");
  k_scale_vec<<<gp, 256, 0, st>>>(out_grad, P, 2.0 / W);
  NQS_CHECK_LAUNCH("k_scale_vec");
  return NQS_OK;
}

// ---- nqs_energy_gradient_noalloc: the same computation with its 2W-double scratch in a
// file-scope device array instead of a caller workspace. Every call on a device shares the one
// array; the centred energies are written in full by k_center_eps before k_gemv_t reads them,
// so nothing in it has to start at zero. Calls that overlap in time on one device race.
static __device__ __align__(256) double g_eg_scratch[2 * NQS_NOALLOC_MAX_WALKERS];

namespace {
constexpr int kScratchDevices = 64;
std::mutex g_eg_scratch_mu;
double* g_eg_scratch_ptr[kScratchDevices];  // address of g_eg_scratch per device ordinal
}  // namespace

// Resolves the scratch address of the current device once (cudaGetSymbolAddress with that
// device current) and caches it per ordinal for the life of the process (a device reset while
// the library is loaded would leave the cached address stale; that is documented as unsupported).
static int eg_scratch(double** out) {
  int dev = -1;
  cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess) {
    set_error("nqs_energy_gradient_noalloc: cudaGetDevice: %s", cudaGetErrorString(rc));
    return NQS_ERR_CUDA;
  }
  if (dev < 0 || dev >= kScratchDevices) {
    set_error("nqs_energy_gradient_noalloc: device ordinal %d >= %d", dev, kScratchDevices);
    return NQS_ERR_UNSUPPORTED;
  }
  std::lock_guard<std::mutex> lock(g_eg_scratch_mu);
  if (!g_eg_scratch_ptr[dev]) {
    void* p = nullptr;
    rc = cudaGetSymbolAddress(&p, g_eg_scratch);
    if (rc != cudaSuccess || !p) {
      set_error("nqs_energy_gradient_noalloc: cudaGetSymbolAddress on device %d: %s", dev,
                cudaGetErrorString(rc));
      return NQS_ERR_CUDA;
    }
    g_eg_scratch_ptr[dev] = static_cast<double*>(p);
  }
  *out = g_eg_scratch_ptr[dev];
  return NQS_OK;
}

int nqs_energy_gradient_noalloc(const void* O, int o_dtype, const double* e, int W, int64_t P,
                                double* out_grad, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (!O || !e || !out_grad || W < 1 || P < 1 || (o_dtype != 0 && o_dtype != 1)) {
    set_error("nqs_energy_gradient_noalloc: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  if (W > NQS_NOALLOC_MAX_WALKERS) {
    set_error("nqs_energy_gradient_noalloc: n_walkers=%d exceeds the static scratch limit of %d "
              "walkers; use nqs_energy_gradient with a workspace",
              W, NQS_NOALLOC_MAX_WALKERS);
    return NQS_ERR_UNSUPPORTED;
  }
  double* x = nullptr;
  NQS_TRY(eg_scratch(&x));
  k_center_eps<<<1, 1024, 0, st>>>((const cplx*)e, W, x);
  NQS_CHECK_LAUNCH("k_center_eps");
  const unsigned gp = (unsigned)((P + 255) / 256);
  if (o_dtype == 0)
    k_gemv_t<double><<<gp, 256, 0, st>>>((const double*)O, 2 * W, 2 * W, P, nullptr, x, out_grad,
                                         nullptr, nullptr, 0.0);
  else
    k_gemv_t<float><<<gp, 256, 0, st>>>((const float*)O, 2 * W, 2 * W, P, nullptr, x, out_grad,
                                        nullptr, nullptr, 0.0);
  NQS_CHECK_LAUNCH("k_gemv_t");
  k_scale_vec<<<gp, 256, 0, st>>>(out_grad, P, 2.0 / W);
  NQS_CHECK_LAUNCH("k_scale_vec");
  return NQS_OK;
}

int nqs_adam_update(double* theta, const double* grad, double* m, double* v, int64_t P, double lr,
                    double b1, double b2, double eps, int t, void* stream) {
  if (!theta || !grad || !m || !v || P < 1 || t < 1) return NQS_ERR_INVALID_ARG;
  const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
  k_adam<<<(unsigned)((P + 255) / 256), 256, 0, (cudaStream_t)stream>>>(theta, grad, m, v, P, lr,
                                                                         b1, b2, eps, c1, c2);
  NQS_CHECK_LAUNCH("k_adam");
  return NQS_OK;
}

int nqs_adam_update_complex(double* theta, const double* grad, double* m, double* v,
                            const int64_t* partner, int64_t P, double lr, double b1, double b2,
                            double eps, int t, void* stream) {
  if (!theta || !grad || !m || !v || !partner || P < 1 || t < 1) {
    set_error("nqs_adam_update_complex: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  const double c1 = 1.0 - pow(b1, (double)t), c2 = 1.0 - pow(b2, (double)t);
  k_adam_complex<<<(unsigned)((P + 255) / 256), 256, 0, (cudaStream_t)stream>>>(
      theta, grad, m, v, partner, P, lr, b1, b2, eps, c1, c2);
  NQS_CHECK_LAUNCH("k_adam_complex");
  return NQS_OK;
}

int nqs_clip_energies(const double* e, int W, double clip_k, double* out_eclip, double* stats,
                      void* stream) {
  if (!e || !out_eclip || W < 1) return NQS_ERR_INVALID_ARG;
  if (W > 16384) {
    set_error("nqs_clip_energies: W=%d > 16384", W);
    return NQS_ERR_UNSUPPORTED;
  }
  int n2 = 1;
  while (n2 < W) n2 <<= 1;
  const size_t sm = sizeof(double) * n2;
  cudaFuncSetAttribute(k_clip, cudaFuncAttributeMaxDynamicSharedMemorySize, 132 * 1024);
  k_clip<<<1, 1024, sm, (cudaStream_t)stream>>>((const cplx*)e, W, clip_k, (cplx*)out_eclip, stats);
  NQS_CHECK_LAUNCH("k_clip");
  return NQS_OK;
}

}  // extern "C"
