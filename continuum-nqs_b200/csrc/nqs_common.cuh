// nqs_common.cuh — shared device/host helpers for libnqs (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>

#include "../../include/nqs.h"

#define NQS_WARP 32

// --------------------------------------------------------------------------------------------
// error plumbing (host)
// --------------------------------------------------------------------------------------------
#include <atomic>

namespace nqs {
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
extern std::atomic<unsigned long long> g_launches;  // kernels launched by this library
extern cudaEvent_t g_prof_start, g_prof_stop;      // optional events around the Gram kernel
// bound of every device-side wait, in polls (0: each wait's built-in default); nqs_set_wait_limit
extern std::atomic<unsigned> g_wait_limit;
inline unsigned wait_limit_or(unsigned dflt) {
  const unsigned v = g_wait_limit.load(std::memory_order_relaxed);
  return v ? v : dflt;
}
}  // namespace nqs

// every kernel launch is followed by exactly one NQS_CHECK_LAUNCH (it also counts the launch)
#define NQS_CHECK_LAUNCH(what)                                              \
  do {                                                                      \
    nqs::g_launches.fetch_add(1, std::memory_order_relaxed);                \
    cudaError_t _e = cudaGetLastError();                                    \
    if (_e != cudaSuccess) return nqs::cuda_status(_e, what);               \
  } while (0)

#define NQS_TRY(...)                                                        \
  do {                                                                      \
    int _s = (__VA_ARGS__);                                                 \
    if (_s != NQS_OK) return _s;                                            \
  } while (0)

// --------------------------------------------------------------------------------------------
// complex double
// --------------------------------------------------------------------------------------------
struct cplx {
  double re, im;
};
__host__ __device__ __forceinline__ cplx mk(double r, double i) { return cplx{r, i}; }
__host__ __device__ __forceinline__ cplx cadd(cplx a, cplx b) { return cplx{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cplx csub(cplx a, cplx b) { return cplx{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cplx cmul(cplx a, cplx b) {
  return cplx{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cplx cscale(cplx a, double s) { return cplx{a.re * s, a.im * s}; }
// a += b * c
__host__ __device__ __forceinline__ void cfma(cplx& a, cplx b, cplx c) {
  a.re = fma(b.re, c.re, fma(-b.im, c.im, a.re));
  a.im = fma(b.re, c.im, fma(b.im, c.re, a.im));
}
__device__ __forceinline__ cplx cdiv(cplx a, cplx b) {
  // Smith's algorithm (scaled by the larger component of b)
  if (fabs(b.re) >= fabs(b.im)) {
    double r = b.im / b.re, den = b.re + b.im * r;
    return cplx{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
  } else {
    double r = b.re / b.im, den = b.re * r + b.im;
    return cplx{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
  }
}
__device__ __forceinline__ cplx cexp_(cplx a) {
  double e = exp(a.re), s, c;
  sincos(a.im, &s, &c);
  return cplx{e * c, e * s};
}
__device__ __forceinline__ bool cfinite(cplx a) { return isfinite(a.re) && isfinite(a.im); }

// --------------------------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3",
// SC'11): 10 rounds of the 4x32 Philox S-box with the published multipliers and Weyl key bumps.
// --------------------------------------------------------------------------------------------
struct u32x4 {
  uint32_t x, y, z, w;
};
__host__ __device__ __forceinline__ void philox_round(u32x4& c, uint32_t k0, uint32_t k1) {
  const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
  const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
  const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
  const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
  c = u32x4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
}
__host__ __device__ __forceinline__ u32x4 philox4x32_10(u32x4 ctr, uint64_t key) {
  uint32_t k0 = (uint32_t)key, k1 = (uint32_t)(key >> 32);
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    philox_round(ctr, k0, k1);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return ctr;
}
// 53-bit uniform in [0, 1) from two words
__host__ __device__ __forceinline__ double u01_53(uint32_t a, uint32_t b) {
  const uint64_t v = (((uint64_t)a << 32) | b) >> 11;
  return (double)v * (1.0 / 9007199254740992.0);
}

// --------------------------------------------------------------------------------------------
// job batches: which (walker, spin flip, tangent set) each job of a network pass evaluates
// --------------------------------------------------------------------------------------------
enum JobKind { JOB_VALUE = 0, JOB_FLAP = 1, JOB_SOC = 2 };

struct JobBatch {
  int kind;
  int n_jobs;
  int N;        // electrons = tokens per job
  int C;        // channels per token: 1 + n_tan + has_lap
  int n_tan;    // tangent directions (pairs (electron, axis))
  int has_lap;  // Laplacian channel present (last channel)
  int w0;       // first walker of this chunk
  const double* R;    // [W][N][2] positions read by the jobs
  const int32_t* S;   // [W][N]
  const int32_t* flip;  // JOB_VALUE only: per-walker flipped electron (or -1), nullable
};

struct JobInfo {
  int walker, flip, tan_e0;
};

__device__ __forceinline__ JobInfo job_info(const JobBatch& jb, int j) {
  JobInfo ji;
  if (jb.kind == JOB_SOC) {
    ji.walker = jb.w0 + j / jb.N;
    ji.flip = j % jb.N;
    ji.tan_e0 = ji.flip;
  } else {
    ji.walker = jb.w0 + j;
    ji.flip = (jb.kind == JOB_VALUE && jb.flip) ? jb.flip[ji.walker] : -1;
    ji.tan_e0 = 0;
  }
  return ji;
}
__device__ __forceinline__ int job_spin(const JobBatch& jb, const JobInfo& ji, int tok) {
  int s = jb.S[(size_t)ji.walker * jb.N + tok];
  return (tok == ji.flip) ? (1 - s) : s;
}

// --------------------------------------------------------------------------------------------
// device model constants
// --------------------------------------------------------------------------------------------
struct ModelConst {
  int N, d, depth, H, ff, nf, K, nG;
  int learnable_env, use_jastrow, jastrow_kind, n_knots;
  int knots_uniform;  // rbf centres k * wdt (k = 0..n_knots-1): the Gaussians follow a recurrence
  double cusp;
  double A[4], Ainv[4];
  double rcut, wdt;
  const double* Gs;     // device [nG][2]
  const double* W;      // device [N][nG][2] complex interleaved
  const double* knots;  // device [n_knots]
};

// tanh(w) of the tanh-GELU (jax.nn.gelu, approximate=True): w = sqrt(2/pi) (x + 0.044715 x^3);
// gelu(x) = x * 0.5 (1 + tanh(w))
template <typename T>
__device__ __forceinline__ T gelu_tanh_w(T x) {
  return tanh(T(0.7978845608028654) * (x + T(0.044715) * (x * x * x)));
}
template <typename T>
__device__ __forceinline__ T gelu_value(T x, T th) {
  return x * (T(0.5) * (T(1) + th));
}

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// K independent warp sums in one butterfly (the same order per value as warp_sum)
template <typename T, int K>
__device__ __forceinline__ void warp_sum_n(T (&v)[K]) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
}
