// net_kernels.cuh — device kernels of the wavefunction network (shared by the forward and the
// reverse-mode translation units). See net_fwd.cu for the channel layout.
#pragma once
#include <algorithm>

#include "net.cuh"

namespace nqs {

// kernels of more than 16 electrons: one CTA per job (head) and per (job, head) (attention);
// off, the warp-per-task kernels (nqs_set_large_n_kernels)
extern bool g_large_n_cta;
// attention of 16 tokens or fewer through the CTA-per-(job, head) kernel as well
// (nqs_set_attention_cta_small; off by default)
extern bool g_attn_cta_small;
// attention of the multi-channel float32 batches on the tensor cores (nqs_set_attention_mma)
extern bool g_attn_mma;


constexpr double kPi = 3.141592653589793;
constexpr double kLnEps = 1e-6;  // flax.linen.LayerNorm default epsilon

// ============================================================================================
// embed: periodic features + spin one-hot -> Dense "embed" (psiformer.py:84-97,127-131)
// ============================================================================================
template <typename T>
__global__ void __launch_bounds__(256) k_embed(JobBatch jb, ModelConst mc,
                                               const T* __restrict__ Wemb,
                                               const T* __restrict__ bemb, T* __restrict__ X) {
  // With tangent / Laplacian channels: features and sums in float64. Value-only batches on the
  // float path: the angle is reduced to [-pi, pi] in float64, then sincosf and float sums.
  __shared__ double sf[8][4][4 * NQS_MAX_FREQ];
  const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = blockIdx.x * (blockDim.x >> 5) + wib;
  if (gw >= jb.n_jobs * jb.N) return;  // warp-uniform
  const int j = gw / jb.N, tok = gw - j * jb.N;
  const JobInfo ji = job_info(jb, j);
  const double* r = jb.R + ((size_t)ji.walker * jb.N + tok) * 2;
  const double r0 = r[0], r1 = r[1];
  const int nf = mc.nf, F = 4 * nf, d = mc.d;
  const int s = job_spin(jb, ji, tok);
  const int te = tok - ji.tan_e0;
  const bool is_tan = (te >= 0) && (2 * te < jb.n_tan);
  const bool derivs = jb.n_tan > 0 || jb.has_lap;  // uniform over the launch
  T* xrow = X + ((size_t)j * jb.N + tok) * jb.C * d;
  if (!derivs && sizeof(T) == 4) {
    T* sv = reinterpret_cast<T*>(&sf[wib][0][0]);
    for (int k = lane; k < F; k += 32) {
      const int al = k / (2 * nf), rem = k - al * 2 * nf, tau = rem / nf, m = rem - tau * nf + 1;
      const double sa = r0 * mc.Ainv[al * 2 + 0] + r1 * mc.Ainv[al * 2 + 1];
      const double ang = ((2.0 * kPi) * sa) * (double)m;
      const double red = ang - (2.0 * kPi) * rint(ang * (0.5 / kPi));
      float fs, fc;
      sincosf((float)red, &fs, &fc);
      sv[k] = (T)(tau == 0 ? fs : fc);
    }
    __syncwarp();
    for (int n = lane; n < d; n += 32) {
      T v = 0;
      for (int k = 0; k < F; ++k) v = fma(sv[k], Wemb[(size_t)k * d + n], v);
      v += Wemb[(size_t)(F + s) * d + n];
      v += bemb[n];
      xrow[n] = v;
    }
    return;
  }
  for (int k = lane; k < F; k += 32) {
    const int al = k / (2 * nf), rem = k - al * 2 * nf, tau = rem / nf, m = rem - tau * nf + 1;
    const double sa = r0 * mc.Ainv[al * 2 + 0] + r1 * mc.Ainv[al * 2 + 1];
    const double ph = (2.0 * kPi) * sa;
    const double ang = ph * (double)m;
    double sn, cs;
    sincos(ang, &sn, &cs);
    const double val = tau == 0 ? sn : cs;
    const double der = tau == 0 ? cs : -sn;
    const double c0 = 2.0 * kPi * m * mc.Ainv[al * 2 + 0], c1 = 2.0 * kPi * m * mc.Ainv[al * 2 + 1];
    sf[wib][0][k] = val;
    sf[wib][1][k] = c0 * der;
    sf[wib][2][k] = c1 * der;
    sf[wib][3][k] = -(c0 * c0 + c1 * c1) * val;
  }
  __syncwarp();
  for (int n = lane; n < d; n += 32) {
    double v = 0, dx = 0, dy = 0, lp = 0;
    // a token's derivative channels are non-zero only when it is a tangent electron (one token
    // of a spin-flip job): the other tokens need the value sum alone (warp-uniform branches)
    if (derivs && is_tan && jb.has_lap) {
      for (int k = 0; k < F; ++k) {
        const double w = (double)Wemb[(size_t)k * d + n];
        v = fma(sf[wib][0][k], w, v);
        dx = fma(sf[wib][1][k], w, dx);
        dy = fma(sf[wib][2][k], w, dy);
        lp = fma(sf[wib][3][k], w, lp);
      }
    } else if (derivs && is_tan) {
      for (int k = 0; k < F; ++k) {
        const double w = (double)Wemb[(size_t)k * d + n];
        v = fma(sf[wib][0][k], w, v);
        dx = fma(sf[wib][1][k], w, dx);
        dy = fma(sf[wib][2][k], w, dy);
      }
    } else if (derivs) {
      for (int k = 0; k < F; ++k) v = fma(sf[wib][0][k], (double)Wemb[(size_t)k * d + n], v);
    } else {
      for (int k = 0; k < F; ++k) v = fma(sf[wib][0][k], (double)Wemb[(size_t)k * d + n], v);
    }
    v += (double)Wemb[(size_t)(F + s) * d + n];
    v += (double)bemb[n];
    xrow[n] = (T)v;
    for (int t = 0; t < jb.n_tan; ++t) {
      double o = 0;
      if (is_tan && t == 2 * te) o = dx;
      if (is_tan && t == 2 * te + 1) o = dy;
      xrow[(size_t)(1 + t) * d + n] = (T)o;
    }
    if (jb.has_lap) xrow[(size_t)(jb.C - 1) * d + n] = (T)(is_tan ? lp : 0.0);
  }
}

// Value-only batches of the float32 path: one thread per token row. The embedding matrix and
// bias are staged in shared memory (every thread of a warp reads the same entry: broadcast), the
// 4 NF features live in registers, and each row leaves as float4 stores. Features and sums are
// the same operations in the same order as the value branch of k_embed (angle reduced to
// [-pi, pi] in float64, sincosf, float sums over k, then the spin row and the bias).
template <int NF>
__global__ void __launch_bounds__(128) k_embed_value(JobBatch jb, ModelConst mc,
                                                     const float* __restrict__ Wemb,
                                                     const float* __restrict__ bemb,
                                                     float* __restrict__ X) {
  constexpr int F = 4 * NF;
  extern __shared__ __align__(16) float sW[];  // (F + 2) rows of d, then the d biases
  const int d = mc.d;
  for (int i = threadIdx.x; i < (F + 2) * d; i += blockDim.x) sW[i] = Wemb[i];
  for (int i = threadIdx.x; i < d; i += blockDim.x) sW[(F + 2) * d + i] = bemb[i];
  __syncthreads();
  const int gt = blockIdx.x * blockDim.x + threadIdx.x;
  if (gt >= jb.n_jobs * jb.N) return;
  const int j = gt / jb.N, tok = gt - j * jb.N;
  const JobInfo ji = job_info(jb, j);
  const double* r = jb.R + ((size_t)ji.walker * jb.N + tok) * 2;
  const double r0 = r[0], r1 = r[1];
  const int s = job_spin(jb, ji, tok);
  float sv[F];
#pragma unroll
  for (int al = 0; al < 2; ++al) {
    const double sa = r0 * mc.Ainv[al * 2 + 0] + r1 * mc.Ainv[al * 2 + 1];
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      const double ang = ((2.0 * kPi) * sa) * (double)m;
      const double red = ang - (2.0 * kPi) * rint(ang * (0.5 / kPi));
      sincosf((float)red, &sv[al * 2 * NF + m - 1], &sv[al * 2 * NF + NF + m - 1]);
    }
  }
  float* xrow = X + ((size_t)j * jb.N + tok) * d;
  const float4* W4 = reinterpret_cast<const float4*>(sW);
  const int d4 = d / 4;
  for (int n4 = 0; n4 < d4; ++n4) {
    float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
    for (int k = 0; k < F; ++k) {
      const float4 w = W4[k * d4 + n4];
      acc.x = fmaf(sv[k], w.x, acc.x);
      acc.y = fmaf(sv[k], w.y, acc.y);
      acc.z = fmaf(sv[k], w.z, acc.z);
      acc.w = fmaf(sv[k], w.w, acc.w);
    }
    const float4 ws = W4[(F + s) * d4 + n4], b = W4[(F + 2) * d4 + n4];
    acc.x = (acc.x + ws.x) + b.x;
    acc.y = (acc.y + ws.y) + b.y;
    acc.z = (acc.z + ws.z) + b.z;
    acc.w = (acc.w + ws.w) + b.w;
    reinterpret_cast<float4*>(xrow)[n4] = acc;
  }
}

// ============================================================================================
// LayerNorm with tangent and Laplacian channels (flax LayerNorm: eps 1e-6, scale, bias)
//   u = x - mean(x), v = mean(u^2), rho = (v+eps)^-1/2, y = u rho g + b
//   d_t y = g (d_t u rho + u d_t rho),  d_t rho = -rho^3 mean(u d_t u)
//   Lap y = g (Lap u rho + 2 sum_t d_t u d_t rho + u Lap rho),
//   Lap rho = 3/4 rho^5 sum_t (d_t v)^2 - 1/2 rho^3 Lap v,  Lap v = 2 mean(u Lap u) + 2 sum_t mean((d_t u)^2)
// ============================================================================================
template <typename T, int Q = NQS_MAX_EMBED / 32>  // Q >= d / 32 features per lane
__global__ void __launch_bounds__(256) k_layernorm(int n_tok, int C, int n_tan, int has_lap, int d,
                                                   const T* __restrict__ X,
                                                   const T* __restrict__ g,
                                                   const T* __restrict__ b, T* __restrict__ Y) {
  const int lane = threadIdx.x & 31;
  const int tok = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (tok >= n_tok) return;
  const T* x = X + (size_t)tok * C * d;
  T* y = Y + (size_t)tok * C * d;
  const T inv_d = T(1) / T(d);
  T u[Q], gm[Q];
  T s = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int f = lane + 32 * q;
    u[q] = f < d ? x[f] : T(0);
    gm[q] = f < d ? g[f] : T(0);
    s += u[q];
  }
  const T mu = warp_sum(s) * inv_d;
  s = 0;
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int f = lane + 32 * q;
    if (f < d) {
      u[q] -= mu;
      s += u[q] * u[q];
    }
  }
  const T var = warp_sum(s) * inv_d;
  const T rho = T(1) / sqrt(var + T(kLnEps));
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int f = lane + 32 * q;
    if (f < d) y[f] = (u[q] * rho) * gm[q] + b[f];
  }
  T S1 = 0, S2 = 0, acc[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) acc[q] = 0;
  const T rho3 = rho * rho * rho;
  // tangent rows TP at a time: their loads are in flight before the first reduction (the narrow
  // instantiations, Q <= 2, keep the registers for this without losing occupancy)
  constexpr int TP = Q <= 2 ? 4 : 1;
  for (int t0 = 0; t0 < n_tan; t0 += TP) {
    T dus[TP][Q];
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      const T* xt = x + (size_t)(1 + t0 + tt) * d;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int f = lane + 32 * q;
        dus[tt][q] = (t0 + tt < n_tan && f < d) ? xt[f] : T(0);
      }
    }
    // the TP rows' sums reduce together: one butterfly for their means, one for their
    // (u . du, du . du) pairs (the same two-pass arithmetic per row as one row at a time)
    T mt[TP], s23[2 * TP];
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      mt[tt] = 0;
#pragma unroll
      for (int q = 0; q < Q; ++q) mt[tt] += dus[tt][q];
    }
    warp_sum_n<T, TP>(mt);
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      mt[tt] *= inv_d;
      T s2 = 0, s3 = 0;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int f = lane + 32 * q;
        if (f < d) {
          dus[tt][q] -= mt[tt];
          s2 += u[q] * dus[tt][q];
          s3 += dus[tt][q] * dus[tt][q];
        }
      }
      s23[2 * tt] = s2;
      s23[2 * tt + 1] = s3;
    }
    warp_sum_n<T, 2 * TP>(s23);
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      const int t = t0 + tt;
      if (t >= n_tan) break;  // warp-uniform
      const T dv = T(2) * s23[2 * tt] * inv_d;
      const T drho = T(-0.5) * rho3 * dv;
      T* yt = y + (size_t)(1 + t) * d;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int f = lane + 32 * q;
        if (f < d) {
          yt[f] = (dus[tt][q] * rho + u[q] * drho) * gm[q];
          acc[q] += dus[tt][q] * drho;
        }
      }
      S1 += dv * dv;
      S2 += s23[2 * tt + 1] * inv_d;
    }
  }
  if (has_lap) {
    const T* xl = x + (size_t)(C - 1) * d;
    T dl[Q];
    s = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int f = lane + 32 * q;
      dl[q] = f < d ? xl[f] : T(0);
      s += dl[q];
    }
    const T ml = warp_sum(s) * inv_d;
    T s2 = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int f = lane + 32 * q;
      if (f < d) {
        dl[q] -= ml;
        s2 += u[q] * dl[q];
      }
    }
    const T dvl = T(2) * warp_sum(s2) * inv_d + T(2) * S2;
    const T d2rho = T(0.75) * rho3 * rho * rho * S1 - T(0.5) * rho3 * dvl;
    T* yl = y + (size_t)(C - 1) * d;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int f = lane + 32 * q;
      if (f < d) yl[f] = (dl[q] * rho + T(2) * acc[q] + u[q] * d2rho) * gm[q];
    }
  }
}

// ============================================================================================
// Row GEMM: Y[r, off+n] = sum_k X[r,k] W[k,n] (+ bias[n] on value rows r % C == 0) (+ Res)
// Up to 3 column segments with their own weights (q|k|v, re|im backflow). SIMT, 64x64 tiles.
// ============================================================================================
template <typename T>
struct GemmSeg {
  const T* W;
  const T* b;
  int ldw, ncols, out_off, tile0;
};
template <typename T>
struct GemmArgs {
  const T* X;
  int ldx, rows, K, C;
  T* Y;
  int ldy;
  const T* Res;
  int ldr;
  int nseg, trans_w;
  GemmSeg<T> seg[3];
};

template <typename T>
__global__ void __launch_bounds__(256) k_gemm(GemmArgs<T> g) {
  constexpr int BM = 64, BN = 64, BK = 16;
  __shared__ T As[BK][BM + 1];
  __shared__ T Bs[BK][BN + 1];
  const int ct = blockIdx.y;
  int sidx = 0;
  while (sidx + 1 < g.nseg && ct >= g.seg[sidx + 1].tile0) ++sidx;
  const GemmSeg<T> sg = g.seg[sidx];
  const int n0 = (ct - sg.tile0) * BN;
  const int m0 = blockIdx.x * BM;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[i][jj] = T(0);
  for (int k0 = 0; k0 < g.K; k0 += BK) {
    for (int idx = threadIdx.x; idx < BM * BK; idx += 256) {
      const int r = idx / BK, kk = idx - r * BK;
      const int gr = m0 + r, gk = k0 + kk;
      As[kk][r] = (gr < g.rows && gk < g.K) ? g.X[(size_t)gr * g.ldx + gk] : T(0);
    }
    for (int idx = threadIdx.x; idx < BK * BN; idx += 256) {
      int kk, n;
      if (!g.trans_w) {
        kk = idx / BN;
        n = idx - kk * BN;
      } else {
        n = idx / BK;
        kk = idx - n * BK;
      }
      const int gk = k0 + kk, gn = n0 + n;
      T v = T(0);
      if (gk < g.K && gn < sg.ncols)
        v = g.trans_w ? sg.W[(size_t)gn * sg.ldw + gk] : sg.W[(size_t)gk * sg.ldw + gn];
      Bs[kk][n] = v;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; ++kk) {
      T a[4], bb[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) bb[jj] = Bs[kk][tx + 16 * jj];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int jj = 0; jj < 4; ++jj) acc[i][jj] = fma(a[i], bb[jj], acc[i][jj]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int r = m0 + ty + 16 * i;
    if (r >= g.rows) continue;
    const bool val = (r % g.C) == 0;
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) {
      const int n = n0 + tx + 16 * jj;
      if (n >= sg.ncols) continue;
      T v = acc[i][jj];
      if (val && sg.b) v += sg.b[n];
      const size_t o = (size_t)r * g.ldy + sg.out_off + n;
      if (g.Res) v = g.Res[(size_t)r * g.ldr + sg.out_off + n] + v;
      g.Y[o] = v;
    }
  }
}

template <typename T>
inline int launch_gemm(GemmArgs<T> g, cudaStream_t st) {
  int tiles = 0;
  for (int s = 0; s < g.nseg; ++s) {
    g.seg[s].tile0 = tiles;
    tiles += (g.seg[s].ncols + 63) / 64;
  }
  if (g.rows <= 0 || tiles == 0) return NQS_OK;
  k_gemm<T><<<dim3((g.rows + 63) / 64, tiles), 256, 0, st>>>(g);
  NQS_CHECK_LAUNCH("k_gemm");
  return NQS_OK;
}

// ============================================================================================
// Multi-head attention with tangent / Laplacian channels, one CTA per (job, head).
//   s = q.k/sqrt(hd), a = softmax_j(s), o = a v
//   d_t s = (d_t q.k + q.d_t k) sc, d_t lse_i = sum_l a_il d_t s_il, d_t a = a (d_t s - d_t lse)
//   d_t o = d_t a v + a d_t v
//   Lap s = (Lap q.k + q.Lap k + 2 P_qk) sc,  P_qk = sum_t d_t q . d_t k
//   Lap a = a (P_sq + Lap s - Lap lse), Lap lse_i = sum_l a_il (Lap s_il + P_sq_il),
//           P_sq = sum_t (d_t s - d_t lse)^2
//   Lap o = Lap a v + a Lap v + 2 P_av,  P_av = sum_t d_t a d_t v
// ============================================================================================
template <typename T>
__global__ void __launch_bounds__(256) k_attention(int n_jobs, int N, int C, int n_tan, int has_lap,
                                                   int d, int H, const T* __restrict__ QKV,
                                                   T* __restrict__ OUT) {
  // one warp per (job, head); every phase is warp-synchronous
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int pair = blockIdx.x * nwarp + wib;
  if (pair >= n_jobs * H) return;  // whole warp
  const int job = pair / H, h = pair - job * H;
  const int hd = d / H;
  const int per = 6 * N * hd + 4 * N * N + N + N * hd;  // elements of this warp's slot
  extern __shared__ __align__(16) unsigned char smraw[];
  T* q = reinterpret_cast<T*>(smraw) + (size_t)wib * per;
  T* k = q + N * hd;
  T* v = k + N * hd;
  T* a = v + N * hd;
  T* qt = a + N * N;
  T* kt = qt + N * hd;
  T* vt = kt + N * hd;
  T* st = vt + N * hd;
  T* lt = st + N * N;
  T* Pqk = lt + N;
  T* Psq = Pqk + N * N;
  T* Pav = Psq + N * N;
  const T sc = T(1) / sqrt(T(hd));
  const int ld = 3 * d;
  auto row = [&](int i, int c) -> size_t { return ((size_t)job * N + i) * C + c; };
  for (int idx = lane; idx < N * hd; idx += 32) {
    const int i = idx / hd, e = idx - i * hd;
    const T* p = QKV + row(i, 0) * ld + h * hd + e;
    q[idx] = p[0];
    k[idx] = p[d];
    v[idx] = p[2 * d];
  }
  if (has_lap) {
    for (int idx = lane; idx < N * N; idx += 32) Pqk[idx] = Psq[idx] = T(0);
    for (int idx = lane; idx < N * hd; idx += 32) Pav[idx] = T(0);
  }
  __syncwarp();
  for (int idx = lane; idx < N * N; idx += 32) {
    const int i = idx / N, jj = idx - i * N;
    T sacc = 0;
    for (int e = 0; e < hd; ++e) sacc = fma(q[i * hd + e], k[jj * hd + e], sacc);
    a[idx] = sacc * sc;
  }
  __syncwarp();
  for (int i = lane; i < N; i += 32) {
    T mx = a[i * N];
    for (int jj = 1; jj < N; ++jj) mx = max(mx, a[i * N + jj]);
    T ssum = 0;
    for (int jj = 0; jj < N; ++jj) {
      const T e = exp(a[i * N + jj] - mx);
      a[i * N + jj] = e;
      ssum += e;
    }
    for (int jj = 0; jj < N; ++jj) a[i * N + jj] = a[i * N + jj] / ssum;
  }
  __syncwarp();
  for (int idx = lane; idx < N * hd; idx += 32) {
    const int i = idx / hd, e = idx - i * hd;
    T o = 0;
    for (int jj = 0; jj < N; ++jj) o = fma(a[i * N + jj], v[jj * hd + e], o);
    OUT[row(i, 0) * d + h * hd + e] = o;
  }
  for (int t = 0; t < n_tan; ++t) {
    __syncwarp();
    for (int idx = lane; idx < N * hd; idx += 32) {
      const int i = idx / hd, e = idx - i * hd;
      const T* p = QKV + row(i, 1 + t) * ld + h * hd + e;
      qt[idx] = p[0];
      kt[idx] = p[d];
      vt[idx] = p[2 * d];
    }
    __syncwarp();
    for (int idx = lane; idx < N * N; idx += 32) {
      const int i = idx / N, jj = idx - i * N;
      T s1 = 0, s2 = 0;
      for (int e = 0; e < hd; ++e) {
        s1 = fma(qt[i * hd + e], k[jj * hd + e], s1);
        s1 = fma(q[i * hd + e], kt[jj * hd + e], s1);
        s2 = fma(qt[i * hd + e], kt[jj * hd + e], s2);
      }
      st[idx] = s1 * sc;
      if (has_lap) Pqk[idx] += s2;
    }
    __syncwarp();
    for (int i = lane; i < N; i += 32) {
      T l = 0;
      for (int jj = 0; jj < N; ++jj) l = fma(a[i * N + jj], st[i * N + jj], l);
      lt[i] = l;
    }
    __syncwarp();
    for (int idx = lane; idx < N * N; idx += 32) {
      const int i = idx / N;
      const T ds = st[idx] - lt[i];
      if (has_lap) Psq[idx] += ds * ds;
      st[idx] = a[idx] * ds;
    }
    __syncwarp();
    for (int idx = lane; idx < N * hd; idx += 32) {
      const int i = idx / hd, e = idx - i * hd;
      T o = 0, pav = 0;
      for (int jj = 0; jj < N; ++jj) {
        o = fma(st[i * N + jj], v[jj * hd + e], o);
        o = fma(a[i * N + jj], vt[jj * hd + e], o);
        pav = fma(st[i * N + jj], vt[jj * hd + e], pav);
      }
      OUT[row(i, 1 + t) * d + h * hd + e] = o;
      if (has_lap) Pav[idx] += pav;
    }
  }
  if (!has_lap) return;
  __syncwarp();
  for (int idx = lane; idx < N * hd; idx += 32) {
    const int i = idx / hd, e = idx - i * hd;
    const T* p = QKV + row(i, C - 1) * ld + h * hd + e;
    qt[idx] = p[0];
    kt[idx] = p[d];
    vt[idx] = p[2 * d];
  }
  __syncwarp();
  for (int idx = lane; idx < N * N; idx += 32) {
    const int i = idx / N, jj = idx - i * N;
    T s1 = 0;
    for (int e = 0; e < hd; ++e) {
      s1 = fma(qt[i * hd + e], k[jj * hd + e], s1);
      s1 = fma(q[i * hd + e], kt[jj * hd + e], s1);
    }
    st[idx] = (s1 + T(2) * Pqk[idx]) * sc;
  }
  __syncwarp();
  for (int i = lane; i < N; i += 32) {
    T l = 0;
    for (int jj = 0; jj < N; ++jj) l = fma(a[i * N + jj], st[i * N + jj] + Psq[i * N + jj], l);
    lt[i] = l;
  }
  __syncwarp();
  for (int idx = lane; idx < N * N; idx += 32) {
    const int i = idx / N;
    st[idx] = a[idx] * (Psq[idx] + st[idx] - lt[i]);
  }
  __syncwarp();
  for (int idx = lane; idx < N * hd; idx += 32) {
    const int i = idx / hd, e = idx - i * hd;
    T o = 0;
    for (int jj = 0; jj < N; ++jj) {
      o = fma(st[i * N + jj], v[jj * hd + e], o);
      o = fma(a[i * N + jj], vt[jj * hd + e], o);
    }
    OUT[row(i, C - 1) * d + h * hd + e] = o + T(2) * Pav[idx];
  }
}

// --------------------------------------------------------------------------------------------
// Register-tiled attention for N <= 16 tokens and head width HD in {4, 8, 16}: same arithmetic as
// k_attention, one warp per (job, head). Lane pair (2i, 2i+1) owns query row i; lane parity hh
// owns keys j = 2m + hh (m < 8) for scores / probabilities / P_qk / P_sq, and output features
// hh*HD/2 .. hh*HD/2 + HD/2-1 for outputs / P_av. Each channel's Q, K, V head tiles (16 x HD) are
// staged into shared memory with cp.async, double-buffered one channel ahead; the value channel's
// K, V stay resident. Interleaving the keys between the lanes of a pair keeps the two rows that a
// warp reads at one time in different banks, and every other lane reads the same address
// (broadcast).
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND) : "memory");
}

// NEL contiguous elements from shared memory; 16-byte loads when the row allows them
template <typename T, int NEL>
__device__ __forceinline__ void lds_row(const T* __restrict__ p, T* r) {
  if constexpr ((NEL * sizeof(T)) % 16 == 0) {
    constexpr int V = 16 / sizeof(T);
#pragma unroll
    for (int c = 0; c < NEL / V; ++c) {
      const int4 v = reinterpret_cast<const int4*>(p)[c];
      const T* t = reinterpret_cast<const T*>(&v);
#pragma unroll
      for (int e = 0; e < V; ++e) r[c * V + e] = t[e];
    }
  } else {
#pragma unroll
    for (int e = 0; e < NEL; ++e) r[e] = p[e];
  }
}
template <typename T, int NEL>
__device__ __forceinline__ void stg_row(T* __restrict__ p, const T* r) {
  if constexpr ((NEL * sizeof(T)) % 16 == 0) {
    constexpr int V = 16 / sizeof(T);
#pragma unroll
    for (int c = 0; c < NEL / V; ++c) {
      int4 v;
      T* t = reinterpret_cast<T*>(&v);
#pragma unroll
      for (int e = 0; e < V; ++e) t[e] = r[c * V + e];
      reinterpret_cast<int4*>(p)[c] = v;
    }
  } else {
#pragma unroll
    for (int e = 0; e < NEL; ++e) p[e] = r[e];
  }
}

constexpr int kAttnTok = 16;  // token slots of k_attention_rt

template <typename T, int HD, bool VAL = false>
__host__ __device__ constexpr size_t attention_rt_warp_bytes() {
  // resident K, V + two buffers of Q, K, V; value-only batches: K, V, Q
  return sizeof(T) * (VAL ? 3 : 8) * kAttnTok * HD;
}

template <typename T, int HD, bool LAP, bool VAL = false>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 2 : 1) k_attention_rt(int n_jobs, int N, int C, int n_tan,
                                                         int d, int H, const T* __restrict__ QKV,
                                                         T* __restrict__ OUT) {
  constexpr bool has_lap = LAP;  // VAL: single-channel batch (C == 1)
  constexpr int NT = kAttnTok, HE = HD / 2, V = 16 / sizeof(T), CH = HD / V;  // 16-B chunks/row
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int pair = blockIdx.x * nwarp + wib;
  if (pair >= n_jobs * H) return;  // whole warp; no block-level barrier below
  const int job = pair / H, h = pair - job * H;
  const int i = lane >> 1, hh = lane & 1;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* Kv = reinterpret_cast<T*>(smraw + (size_t)wib * attention_rt_warp_bytes<T, HD, VAL>());
  T* Vv = Kv + NT * HD;
  T* buf = Vv + NT * HD;  // buf + b * 3 * NT * HD: Q, K, V tiles of one channel
  const int ld = 3 * d;
  const T sc = T(1) / sqrt(T(HD));
  // rows >= N are never copied: zero them once (zero probabilities times zero values)
  if (N < NT) {
    for (int idx = lane; idx < (VAL ? 3 : 8) * (NT - N) * HD; idx += 32) {
      const int tile = idx / ((NT - N) * HD), r = idx - tile * (NT - N) * HD;
      Kv[tile * NT * HD + N * HD + r] = T(0);
    }
    __syncwarp();
  }
  // channel c -> buffer b (Q, K, V tiles); the value channel's K and V go straight to their
  // resident slots
  auto issue = [&](int c, int b) {
    if (c < C) {
      T* dst = buf + b * 3 * NT * HD;
      for (int q = lane; q < 3 * N * CH; q += 32) {
        const int t = q / (N * CH), r = q - t * (N * CH), tok = r / CH, ch = r - tok * CH;
        const T* src = QKV + (((size_t)job * N + tok) * C + c) * ld + t * d + h * HD + ch * V;
        T* tile = (c == 0 && t > 0) ? (t == 1 ? Kv : Vv) : dst + t * NT * HD;
        cp_async16(tile + tok * HD + ch * V, src);
      }
    }
    cp_async_commit();
  };
  auto out_row = [&](int c) { return OUT + (((size_t)job * N + i) * C + c) * d + h * HD + hh * HE; };
  const bool live = i < N;
  // ---- value channel ----
  issue(0, 0);
  if (VAL) {
    cp_async_wait<0>();
  } else {
    issue(1, 1);
    cp_async_wait<1>();
  }
  __syncwarp();
  T q[HD], a[8], ao[8];
  {
    const T* Q0 = buf;
    const T* K0 = Kv;
    const T* V0 = Vv;
    lds_row<T, HD>(Q0 + i * HD, q);
    T s[8];
    T mx = T(-INFINITY);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int j = 2 * m + hh;
      T k[HD];
      lds_row<T, HD>(K0 + j * HD, k);
      T acc = 0;
#pragma unroll
      for (int e = 0; e < HD; ++e) acc = fma(q[e], k[e], acc);
      s[m] = j < N ? acc * sc : T(-INFINITY);
      mx = max(mx, s[m]);
    }
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, 1));
    T ssum = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      a[m] = (2 * m + hh < N) ? exp(s[m] - mx) : T(0);
      ssum += a[m];
    }
    ssum += __shfl_xor_sync(0xffffffffu, ssum, 1);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      a[m] = a[m] / ssum;
      ao[m] = __shfl_xor_sync(0xffffffffu, a[m], 1);
    }
    T o[HE];
#pragma unroll
    for (int e = 0; e < HE; ++e) o[e] = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      T v0[HE], v1[HE];
      lds_row<T, HE>(V0 + (2 * m + hh) * HD + hh * HE, v0);
      lds_row<T, HE>(V0 + (2 * m + 1 - hh) * HD + hh * HE, v1);
#pragma unroll
      for (int e = 0; e < HE; ++e) o[e] = fma(a[m], v0[e], fma(ao[m], v1[e], o[e]));
    }
    if (live) stg_row<T, HE>(out_row(0), o);
  }
  if (VAL) return;
  __syncwarp();
  issue(2, 0);
  T Pqk[8], Psq[8], Pav[HE];
#pragma unroll
  for (int m = 0; m < 8; ++m) Pqk[m] = Psq[m] = T(0);
#pragma unroll
  for (int e = 0; e < HE; ++e) Pav[e] = T(0);
  // ---- tangent channels ----
  for (int t = 0; t < n_tan; ++t) {
    const int c = 1 + t, b = c & 1;
    cp_async_wait<1>();
    __syncwarp();
    const T* Qt = buf + b * 3 * NT * HD;
    const T* Kt = Qt + NT * HD;
    const T* Vt = Kt + NT * HD;
    T qt[HD], st[8];
    lds_row<T, HD>(Qt + i * HD, qt);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int j = 2 * m + hh;
      T k[HD], kt[HD];
      lds_row<T, HD>(Kv + j * HD, k);
      lds_row<T, HD>(Kt + j * HD, kt);
      T s1 = 0, s2 = 0;
#pragma unroll
      for (int e = 0; e < HD; ++e) {
        s1 = fma(qt[e], k[e], s1);
        s1 = fma(q[e], kt[e], s1);
        s2 = fma(qt[e], kt[e], s2);
      }
      st[m] = s1 * sc;
      if (has_lap) Pqk[m] += s2;
    }
    T lt = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) lt = fma(a[m], st[m], lt);
    lt += __shfl_xor_sync(0xffffffffu, lt, 1);
    T sto[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const T ds = st[m] - lt;
      if (has_lap) Psq[m] += ds * ds;
      st[m] = a[m] * ds;
      sto[m] = __shfl_xor_sync(0xffffffffu, st[m], 1);
    }
    T o[HE];
#pragma unroll
    for (int e = 0; e < HE; ++e) o[e] = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int j0 = 2 * m + hh, j1 = 2 * m + 1 - hh;
      T v0[HE], v1[HE], w0[HE], w1[HE];
      lds_row<T, HE>(Vv + j0 * HD + hh * HE, v0);
      lds_row<T, HE>(Vv + j1 * HD + hh * HE, v1);
      lds_row<T, HE>(Vt + j0 * HD + hh * HE, w0);
      lds_row<T, HE>(Vt + j1 * HD + hh * HE, w1);
#pragma unroll
      for (int e = 0; e < HE; ++e) {
        o[e] = fma(st[m], v0[e], o[e]);
        o[e] = fma(a[m], w0[e], o[e]);
        o[e] = fma(sto[m], v1[e], o[e]);
        o[e] = fma(ao[m], w1[e], o[e]);
        if (has_lap) Pav[e] = fma(st[m], w0[e], fma(sto[m], w1[e], Pav[e]));
      }
    }
    if (live) stg_row<T, HE>(out_row(c), o);
    __syncwarp();
    issue(c + 2, b);
  }
  if (!has_lap) {
    cp_async_wait<0>();
    return;
  }
  // ---- Laplacian channel (C - 1 = 1 + n_tan) ----
  {
    const int c = C - 1, b = c & 1;
    cp_async_wait<0>();
    __syncwarp();
    const T* Ql = buf + b * 3 * NT * HD;
    const T* Kl = Ql + NT * HD;
    const T* Vl = Kl + NT * HD;
    T ql[HD], sl[8];
    lds_row<T, HD>(Ql + i * HD, ql);
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int j = 2 * m + hh;
      T k[HD], kl[HD];
      lds_row<T, HD>(Kv + j * HD, k);
      lds_row<T, HD>(Kl + j * HD, kl);
      T s1 = 0;
#pragma unroll
      for (int e = 0; e < HD; ++e) {
        s1 = fma(ql[e], k[e], s1);
        s1 = fma(q[e], kl[e], s1);
      }
      sl[m] = (s1 + T(2) * Pqk[m]) * sc;
    }
    T ll = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) ll = fma(a[m], sl[m] + Psq[m], ll);
    ll += __shfl_xor_sync(0xffffffffu, ll, 1);
    T slo[8];
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      sl[m] = a[m] * (Psq[m] + sl[m] - ll);
      slo[m] = __shfl_xor_sync(0xffffffffu, sl[m], 1);
    }
    T o[HE];
#pragma unroll
    for (int e = 0; e < HE; ++e) o[e] = 0;
#pragma unroll
    for (int m = 0; m < 8; ++m) {
      const int j0 = 2 * m + hh, j1 = 2 * m + 1 - hh;
      T v0[HE], v1[HE], w0[HE], w1[HE];
      lds_row<T, HE>(Vv + j0 * HD + hh * HE, v0);
      lds_row<T, HE>(Vv + j1 * HD + hh * HE, v1);
      lds_row<T, HE>(Vl + j0 * HD + hh * HE, w0);
      lds_row<T, HE>(Vl + j1 * HD + hh * HE, w1);
#pragma unroll
      for (int e = 0; e < HE; ++e) {
        o[e] = fma(sl[m], v0[e], o[e]);
        o[e] = fma(a[m], w0[e], o[e]);
        o[e] = fma(slo[m], v1[e], o[e]);
        o[e] = fma(ao[m], w1[e], o[e]);
      }
    }
#pragma unroll
    for (int e = 0; e < HE; ++e) o[e] += T(2) * Pav[e];
    if (live) stg_row<T, HE>(out_row(c), o);
  }
}

// warps per CTA and dynamic shared memory of k_attention (each warp's slot rounded to 16 bytes)
template <typename T>
inline size_t attention_warp_bytes(int N, int hd) {
  return ((sizeof(T) * (size_t)(6 * N * hd + 4 * N * N + N + N * hd)) + 15) & ~(size_t)15;
}
template <typename T>
inline int attention_wpc(int N, int hd) {
  const size_t wb = attention_warp_bytes<T>(N, hd);
  int w = 8;
  while (w > 1 && (size_t)w * wb > 96 * 1024) w /= 2;
  return w;
}
template <typename T>
inline size_t attention_smem(int N, int hd) {
  return (size_t)attention_wpc<T>(N, hd) * attention_warp_bytes<T>(N, hd);
}

// k_attention_rt when N <= 16, the head width is 4, 8 or 16 and rows are 16-byte aligned,
// else k_attention
template <typename T, int HD>
inline int launch_attention_rt(int n_jobs, int N, int C, int n_tan, int has_lap, int d, int H,
                               const T* QKV, T* OUT, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_attention_rt<T, HD, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         96 * 1024);
    cudaFuncSetAttribute(k_attention_rt<T, HD, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         96 * 1024);
    cudaFuncSetAttribute(k_attention_rt<T, HD, false, true>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    attr = true;
  }
  const long long pairs = (long long)n_jobs * H;
  if (C == 1) {  // value-only batch: three tiles per warp, eight warps per CTA
    const size_t wbv = attention_rt_warp_bytes<T, HD, true>();
    k_attention_rt<T, HD, false, true><<<(unsigned)((pairs + 7) / 8), 256, 8 * wbv, st>>>(
        n_jobs, N, C, n_tan, d, H, QKV, OUT);
    NQS_CHECK_LAUNCH("k_attention_rt");
    return NQS_OK;
  }
  const size_t wb = attention_rt_warp_bytes<T, HD>();
  int wpc = 8;
  while (wpc > 1 && wpc * wb > 96 * 1024) wpc /= 2;
  const unsigned grid = (unsigned)((pairs + wpc - 1) / wpc);
  if (has_lap)
    k_attention_rt<T, HD, true><<<grid, 32 * wpc, wpc * wb, st>>>(n_jobs, N, C, n_tan, d, H, QKV,
                                                                   OUT);
  else
    k_attention_rt<T, HD, false><<<grid, 32 * wpc, wpc * wb, st>>>(n_jobs, N, C, n_tan, d, H, QKV,
                                                                    OUT);
  NQS_CHECK_LAUNCH("k_attention_rt");
  return NQS_OK;
}

// --------------------------------------------------------------------------------------------
// Attention for 16 < N <= 64 tokens: one CTA (256 threads) per (job, head), same arithmetic as
// k_attention. Thread (ty, tx) = (tid / 16, tid % 16) owns the score / probability entries of
// rows ty + 16u and columns tx + 16w (u, w < TS); a half-warp holds whole rows, so the softmax
// and every row sum (d_t lse, Lap lse) are 16-lane shuffles. P_qk and P_sq stay in the owners'
// registers across the channels, and so does P_av for the output entries: thread
// (tid / (HD/4), tid % (HD/4)) writes features 4 (tid % (HD/4)) .. + 3 of one token. Per channel:
// stage Q_c, K_c, V_c head tiles (rows past N are zero), scores, one barrier, outputs.
// Rows of the K-type tiles are HD + 4 long (16 rows of a half-warp fall in different banks); the
// probability tiles have an odd row length.
// --------------------------------------------------------------------------------------------
template <int HD>
constexpr int attn_cta_hdp() { return HD + 4; }

template <typename T, int TS, int HD>
__host__ __device__ constexpr size_t attention_cta_bytes() {
  return sizeof(T) * (6 * (size_t)(16 * TS) * attn_cta_hdp<HD>() +
                      2 * (size_t)(16 * TS) * (16 * TS + 1));
}

template <typename T>
__device__ __forceinline__ T hw_sum16(T v) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <typename T>
__device__ __forceinline__ T hw_max16(T v) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

template <typename T, int TS, int HD>
__global__ void __launch_bounds__(256) k_attention_cta(int n_jobs, int N, int C, int n_tan,
                                                       int has_lap, int d, int H,
                                                       const T* __restrict__ QKV,
                                                       T* __restrict__ OUT) {
  constexpr int NP = 16 * TS, HDP = attn_cta_hdp<HD>(), LDA = NP + 1, NQ = HD / 4;
  const int pair = blockIdx.x;
  const int job = pair / H, h = pair - job * H;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* q = reinterpret_cast<T*>(smraw);
  T* k = q + NP * HDP;
  T* v = k + NP * HDP;
  T* qt = v + NP * HDP;
  T* kt = qt + NP * HDP;
  T* vt = kt + NP * HDP;
  T* A = vt + NP * HDP;
  T* ST = A + NP * LDA;
  const T sc = T(1) / sqrt(T(HD));
  const int ld = 3 * d;
  auto row = [&](int i, int c) -> size_t { return ((size_t)job * N + i) * C + c; };
  // Q, K, V head tiles of channel c (rows >= N zero)
  auto stage = [&](int c, T* dq, T* dk, T* dv) {
    for (int idx = tid; idx < NP * HD; idx += 256) {
      const int i = idx / HD, e = idx - i * HD;
      T a = T(0), b = T(0), cc = T(0);
      if (i < N) {
        const T* p = QKV + row(i, c) * ld + h * HD + e;
        a = p[0];
        b = p[d];
        cc = p[2 * d];
      }
      dq[i * HDP + e] = a;
      dk[i * HDP + e] = b;
      dv[i * HDP + e] = cc;
    }
  };
  // output thread: token oi, features 4 oq .. 4 oq + 3
  const int oi = tid / NQ, oq = tid - (tid / NQ) * NQ;
  const bool out_on = oi < N;
  // sum_j P1[oi][j] V1[j][f] + P2[oi][j] V2[j][f] (and sum_j P1 V2 into pav when acc)
  auto outputs = [&](const T* P1, const T* V1, const T* P2, const T* V2, T (&o)[4], T* pav) {
#pragma unroll
    for (int f = 0; f < 4; ++f) o[f] = T(0);
    if (!out_on) return;
    const T* p1 = P1 + oi * LDA;
    const T* p2 = P2 ? P2 + oi * LDA : nullptr;
    for (int j = 0; j < N; ++j) {
      const T a1 = p1[j];
      const T* v1 = V1 + j * HDP + 4 * oq;
#pragma unroll
      for (int f = 0; f < 4; ++f) o[f] = fma(a1, v1[f], o[f]);
      if (p2) {
        const T a2 = p2[j];
        const T* v2 = V2 + j * HDP + 4 * oq;
#pragma unroll
        for (int f = 0; f < 4; ++f) {
          o[f] = fma(a2, v2[f], o[f]);
          if (pav) pav[f] = fma(a1, v2[f], pav[f]);
        }
      }
    }
  };
  auto store = [&](int c, const T (&o)[4]) {
    if (!out_on) return;
    T* p = OUT + row(oi, c) * d + h * HD + 4 * oq;
#pragma unroll
    for (int f = 0; f < 4; ++f) p[f] = o[f];
  };
  // ---- value channel: probabilities a (registers and shared), output ----
  stage(0, q, k, v);
  __syncthreads();
  T a[TS][TS];
#pragma unroll
  for (int u = 0; u < TS; ++u) {
    const int i = ty + 16 * u;
    T sv[TS];
#pragma unroll
    for (int w = 0; w < TS; ++w) sv[w] = T(0);
#pragma unroll
    for (int e = 0; e < HD; ++e) {
      const T qe = q[i * HDP + e];
#pragma unroll
      for (int w = 0; w < TS; ++w) sv[w] = fma(qe, k[(tx + 16 * w) * HDP + e], sv[w]);
    }
    T mx = -INFINITY;
#pragma unroll
    for (int w = 0; w < TS; ++w) {
      sv[w] = (tx + 16 * w < N) ? sv[w] * sc : T(-INFINITY);
      mx = max(mx, sv[w]);
    }
    mx = hw_max16(mx);
    T ssum = T(0);
#pragma unroll
    for (int w = 0; w < TS; ++w) {
      sv[w] = (tx + 16 * w < N) ? exp(sv[w] - mx) : T(0);
      ssum += sv[w];
    }
    ssum = hw_sum16(ssum);
#pragma unroll
    for (int w = 0; w < TS; ++w) {
      a[u][w] = sv[w] / ssum;
      A[i * LDA + tx + 16 * w] = a[u][w];
    }
  }
  __syncthreads();
  T o[4];
  outputs(A, v, nullptr, nullptr, o, nullptr);
  store(0, o);
  if (C == 1) return;
  T pqk[TS][TS], psq[TS][TS], pav[4];
#pragma unroll
  for (int u = 0; u < TS; ++u)
#pragma unroll
    for (int w = 0; w < TS; ++w) pqk[u][w] = psq[u][w] = T(0);
#pragma unroll
  for (int f = 0; f < 4; ++f) pav[f] = T(0);
  // scores of a channel: s1 = qt.k + q.kt (and s2 = qt.kt)
  auto scores = [&](T (&s1)[TS][TS], T (&s2)[TS][TS], bool want_s2) {
#pragma unroll
    for (int u = 0; u < TS; ++u)
#pragma unroll
      for (int w = 0; w < TS; ++w) s1[u][w] = s2[u][w] = T(0);
#pragma unroll 4
    for (int e = 0; e < HD; ++e) {
      T qa[TS], qb[TS], ka[TS], kb[TS];
#pragma unroll
      for (int u = 0; u < TS; ++u) {
        qa[u] = qt[(ty + 16 * u) * HDP + e];
        qb[u] = q[(ty + 16 * u) * HDP + e];
      }
#pragma unroll
      for (int w = 0; w < TS; ++w) {
        ka[w] = k[(tx + 16 * w) * HDP + e];
        kb[w] = kt[(tx + 16 * w) * HDP + e];
      }
#pragma unroll
      for (int u = 0; u < TS; ++u)
#pragma unroll
        for (int w = 0; w < TS; ++w) {
          s1[u][w] = fma(qa[u], ka[w], fma(qb[u], kb[w], s1[u][w]));
          if (want_s2) s2[u][w] = fma(qa[u], kb[w], s2[u][w]);
        }
    }
  };
  for (int t = 0; t < n_tan; ++t) {
    __syncthreads();  // the previous channel's outputs no longer read ST / vt
    stage(1 + t, qt, kt, vt);
    __syncthreads();
    T s1[TS][TS], s2[TS][TS];
    scores(s1, s2, has_lap != 0);
#pragma unroll
    for (int u = 0; u < TS; ++u) {
      T l = T(0);
#pragma unroll
      for (int w = 0; w < TS; ++w) {
        s1[u][w] *= sc;
        l = fma(a[u][w], s1[u][w], l);
      }
      l = hw_sum16(l);
#pragma unroll
      for (int w = 0; w < TS; ++w) {
        const T ds = s1[u][w] - l;
        if (has_lap) {
          pqk[u][w] += s2[u][w];
          psq[u][w] = fma(ds, ds, psq[u][w]);
        }
        ST[(ty + 16 * u) * LDA + tx + 16 * w] = a[u][w] * ds;
      }
    }
    __syncthreads();
    outputs(ST, v, A, vt, o, has_lap ? pav : nullptr);
    store(1 + t, o);
  }
  if (!has_lap) return;
  __syncthreads();
  stage(C - 1, qt, kt, vt);
  __syncthreads();
  {
    T s1[TS][TS], s2[TS][TS];
    scores(s1, s2, false);
#pragma unroll
    for (int u = 0; u < TS; ++u) {
      T l = T(0);
#pragma unroll
      for (int w = 0; w < TS; ++w) {
        s1[u][w] = (s1[u][w] + T(2) * pqk[u][w]) * sc;
        l = fma(a[u][w], s1[u][w] + psq[u][w], l);
      }
      l = hw_sum16(l);
#pragma unroll
      for (int w = 0; w < TS; ++w)
        ST[(ty + 16 * u) * LDA + tx + 16 * w] = a[u][w] * (psq[u][w] + s1[u][w] - l);
    }
  }
  __syncthreads();
  outputs(ST, v, A, vt, o, nullptr);
#pragma unroll
  for (int f = 0; f < 4; ++f) o[f] += T(2) * pav[f];
  store(C - 1, o);
}

template <typename T, int TS, int HD>
inline int launch_attention_cta(int n_jobs, int N, int C, int n_tan, int has_lap, int d, int H,
                                const T* QKV, T* OUT, cudaStream_t st) {
  constexpr size_t sm = attention_cta_bytes<T, TS, HD>();
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_attention_cta<T, TS, HD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sm);
    attr = true;
  }
  k_attention_cta<T, TS, HD><<<(unsigned)((long long)n_jobs * H), 256, sm, st>>>(
      n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT);
  NQS_CHECK_LAUNCH("k_attention_cta");
  return NQS_OK;
}

template <typename T, int HD>
inline int launch_attention_cta_ts(int n_jobs, int N, int C, int n_tan, int has_lap, int d, int H,
                                   const T* QKV, T* OUT, cudaStream_t st) {
  if (N <= 16)
    return launch_attention_cta<T, 1, HD>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
  if (N <= 32)
    return launch_attention_cta<T, 2, HD>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
  if (N <= 48)
    return launch_attention_cta<T, 3, HD>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
  return launch_attention_cta<T, 4, HD>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
}

// --------------------------------------------------------------------------------------------
// Attention of the multi-channel (forward-Laplacian, spin-flip) float32 batches on the tensor
// cores: head width 16, N <= 64 tokens, one CTA per (job, head) with one warp per 16 query rows.
// Every product of k_attention (Q_c K^T, Q K_c^T, Q_c K_c^T, P V, A V_c, P V_c) is a chain of
// mma.sync m16n8k8 TF32 MMAs with float32 accumulation; the probabilities A, P_qk, P_sq and P_av
// stay in accumulator fragments across the channels. A lane holds rows g, g + 8 (g = lane / 4) and
// columns 2t, 2t + 1 (t = lane % 4) of every 8-key tile; used as the A operand of the next product
// the pair (2t, 2t + 1) is read as keys (t, t + 4) of that tile, and V's rows are fetched in the
// same order, so no fragment changes lanes. Row sums (softmax, d_t lse, Lap lse) are 4-lane
// shuffles. Per channel: stage Q_c, K_c, V_c (rows past N zero), one barrier, products, outputs.
// --------------------------------------------------------------------------------------------
constexpr int kAttMmaHd = 16, kAttMmaLd = 20;  // head width; shared row stride (floats)

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

template <int NT>  // 16-row tiles of tokens (N <= 16 NT)
__global__ void __launch_bounds__(32 * NT) k_attention_mma(int n_jobs, int N, int C, int n_tan,
                                                          int has_lap, int d, int H,
                                                          const float* __restrict__ QKV,
                                                          float* __restrict__ OUT) {
  constexpr int NP = 16 * NT, NK = 2 * NT, LD = kAttMmaLd, HD = kAttMmaHd;
  const int pair = blockIdx.x;
  const int job = pair / H, h = pair - job * H;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int r0 = 16 * w;  // this warp's query rows r0 .. r0 + 15
  __shared__ __align__(16) float sm[6 * NP * LD];
  float* q = sm;
  float* k = q + NP * LD;
  float* v = k + NP * LD;
  float* qt = v + NP * LD;
  float* kt = qt + NP * LD;
  float* vt = kt + NP * LD;
  const float sc = 1.0f / sqrtf((float)HD);
  const int ld = 3 * d;
  auto row = [&](int i, int c) -> size_t { return ((size_t)job * N + i) * C + c; };
  auto stage = [&](int c, float* dq, float* dk, float* dv) {
    for (int idx = threadIdx.x; idx < NP * 4; idx += 32 * NT) {
      const int i = idx >> 2, e4 = (idx & 3) * 4;
      float4 a = make_float4(0.f, 0.f, 0.f, 0.f), b = a, cc = a;
      if (i < N) {
        const float* p = QKV + row(i, c) * ld + h * HD + e4;
        a = *reinterpret_cast<const float4*>(p);
        b = *reinterpret_cast<const float4*>(p + d);
        cc = *reinterpret_cast<const float4*>(p + 2 * d);
      }
      *reinterpret_cast<float4*>(dq + i * LD + e4) = a;
      *reinterpret_cast<float4*>(dk + i * LD + e4) = b;
      *reinterpret_cast<float4*>(dv + i * LD + e4) = cc;
    }
  };
  // A operand: rows r0.., features 8 ks .. 8 ks + 7 of X
  auto afrag_x = [&](const float* X, int ks, uint32_t (&a)[4]) {
    a[0] = to_tf32(X[(r0 + g) * LD + 8 * ks + t]);
    a[1] = to_tf32(X[(r0 + g + 8) * LD + 8 * ks + t]);
    a[2] = to_tf32(X[(r0 + g) * LD + 8 * ks + t + 4]);
    a[3] = to_tf32(X[(r0 + g + 8) * LD + 8 * ks + t + 4]);
  };
  // A operand from a score-shaped fragment of key tile j: columns (2t, 2t+1) read as keys (t, t+4)
  auto afrag_p = [&](const float (&P)[4], uint32_t (&a)[4]) {
    a[0] = to_tf32(P[0]);
    a[1] = to_tf32(P[2]);
    a[2] = to_tf32(P[1]);
    a[3] = to_tf32(P[3]);
  };
  // S[j] += X Y^T over the 16 features: X rows of this warp, Y rows = keys of tile j
  auto scores = [&](const float* X, const float* Y, float (&S)[NK][4]) {
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      uint32_t a[4];
      afrag_x(X, ks, a);
#pragma unroll
      for (int j = 0; j < NK; ++j) {
        const uint32_t b0 = to_tf32(Y[(8 * j + g) * LD + 8 * ks + t]);
        const uint32_t b1 = to_tf32(Y[(8 * j + g) * LD + 8 * ks + t + 4]);
        mma_tf32(S[j], a, b0, b1);
      }
    }
  };
  // O[f] += P V over the keys: P score-shaped, V rows in the (t, t+4) <- (2t, 2t+1) key order
  auto pv = [&](const float (&P)[NK][4], const float* V, float (&O)[2][4]) {
#pragma unroll
    for (int j = 0; j < NK; ++j) {
      uint32_t a[4];
      afrag_p(P[j], a);
#pragma unroll
      for (int f = 0; f < 2; ++f) {
        const uint32_t b0 = to_tf32(V[(8 * j + 2 * t) * LD + 8 * f + g]);
        const uint32_t b1 = to_tf32(V[(8 * j + 2 * t + 1) * LD + 8 * f + g]);
        mma_tf32(O[f], a, b0, b1);
      }
    }
  };
  auto store = [&](int c, const float (&O)[2][4], float add_scale, const float (&Add)[2][4]) {
    const int i0 = r0 + g, i1 = r0 + g + 8;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const int col = h * HD + 8 * f + 2 * t;
      if (i0 < N)
        *reinterpret_cast<float2*>(OUT + row(i0, c) * d + col) =
            make_float2(O[f][0] + add_scale * Add[f][0], O[f][1] + add_scale * Add[f][1]);
      if (i1 < N)
        *reinterpret_cast<float2*>(OUT + row(i1, c) * d + col) =
            make_float2(O[f][2] + add_scale * Add[f][2], O[f][3] + add_scale * Add[f][3]);
    }
  };
  auto quad_sum = [](float x) {
    x += __shfl_xor_sync(0xffffffffu, x, 1);
    x += __shfl_xor_sync(0xffffffffu, x, 2);
    return x;
  };
  auto quad_max = [](float x) {
    x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 1));
    x = fmaxf(x, __shfl_xor_sync(0xffffffffu, x, 2));
    return x;
  };
  // key column of fragment element e of tile j
  auto key = [&](int j, int e) { return 8 * j + 2 * t + (e & 1); };
  const float zero24[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  // ---- value channel ----
  stage(0, q, k, v);
  __syncthreads();
  float A[NK][4];
#pragma unroll
  for (int j = 0; j < NK; ++j) A[j][0] = A[j][1] = A[j][2] = A[j][3] = 0.f;
  scores(q, k, A);
  {
    float mx0 = -INFINITY, mx1 = -INFINITY;
#pragma unroll
    for (int j = 0; j < NK; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        A[j][e] = key(j, e) < N ? A[j][e] * sc : -INFINITY;
        if (e < 2) mx0 = fmaxf(mx0, A[j][e]); else mx1 = fmaxf(mx1, A[j][e]);
      }
    mx0 = quad_max(mx0);
    mx1 = quad_max(mx1);
    float s0 = 0.f, s1 = 0.f;
#pragma unroll
    for (int j = 0; j < NK; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float x = key(j, e) < N ? expf(A[j][e] - (e < 2 ? mx0 : mx1)) : 0.f;
        A[j][e] = x;
        if (e < 2) s0 += x; else s1 += x;
      }
    s0 = quad_sum(s0);
    s1 = quad_sum(s1);
    const float i0 = 1.f / s0, i1 = 1.f / s1;
#pragma unroll
    for (int j = 0; j < NK; ++j) {
      A[j][0] *= i0;
      A[j][1] *= i0;
      A[j][2] *= i1;
      A[j][3] *= i1;
    }
  }
  float O[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  pv(A, v, O);
  store(0, O, 0.f, zero24);
  if (C == 1) return;
  float Pqk[NK][4], Psq[NK][4], Pav[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
#pragma unroll
  for (int j = 0; j < NK; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) Pqk[j][e] = Psq[j][e] = 0.f;
  for (int c = 0; c < n_tan; ++c) {
    __syncthreads();  // the previous channel's products no longer read qt / kt / vt
    stage(1 + c, qt, kt, vt);
    __syncthreads();
    float S[NK][4];
#pragma unroll
    for (int j = 0; j < NK; ++j) S[j][0] = S[j][1] = S[j][2] = S[j][3] = 0.f;
    scores(qt, k, S);
    scores(q, kt, S);
    if (has_lap) scores(qt, kt, Pqk);
    float l0 = 0.f, l1 = 0.f;
#pragma unroll
    for (int j = 0; j < NK; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        S[j][e] *= sc;
        if (e < 2) l0 = fmaf(A[j][e], S[j][e], l0); else l1 = fmaf(A[j][e], S[j][e], l1);
      }
    l0 = quad_sum(l0);
    l1 = quad_sum(l1);
#pragma unroll
    for (int j = 0; j < NK; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) {
        const float ds = S[j][e] - (e < 2 ? l0 : l1);
        if (has_lap) Psq[j][e] = fmaf(ds, ds, Psq[j][e]);
        S[j][e] = A[j][e] * ds;
      }
    float Ot[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
    pv(S, v, Ot);
    pv(A, vt, Ot);
    if (has_lap) pv(S, vt, Pav);
    store(1 + c, Ot, 0.f, zero24);
  }
  if (!has_lap) return;
  __syncthreads();
  stage(C - 1, qt, kt, vt);
  __syncthreads();
  float S[NK][4];
#pragma unroll
  for (int j = 0; j < NK; ++j) S[j][0] = S[j][1] = S[j][2] = S[j][3] = 0.f;
  scores(qt, k, S);
  scores(q, kt, S);
  float l0 = 0.f, l1 = 0.f;
#pragma unroll
  for (int j = 0; j < NK; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      S[j][e] = (S[j][e] + 2.f * Pqk[j][e]) * sc;
      const float x = A[j][e] * (S[j][e] + Psq[j][e]);
      if (e < 2) l0 += x; else l1 += x;
    }
  l0 = quad_sum(l0);
  l1 = quad_sum(l1);
#pragma unroll
  for (int j = 0; j < NK; ++j)
#pragma unroll
    for (int e = 0; e < 4; ++e) S[j][e] = A[j][e] * (Psq[j][e] + S[j][e] - (e < 2 ? l0 : l1));
  float Ol[2][4] = {{0.f, 0.f, 0.f, 0.f}, {0.f, 0.f, 0.f, 0.f}};
  pv(S, v, Ol);
  pv(A, vt, Ol);
  store(C - 1, Ol, 2.f, Pav);
}

template <int NT>
inline int launch_attention_mma(int n_jobs, int N, int C, int n_tan, int has_lap, int d, int H,
                                const float* QKV, float* OUT, cudaStream_t st) {
  k_attention_mma<NT><<<(unsigned)((long long)n_jobs * H), 32 * NT, 0, st>>>(
      n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT);
  NQS_CHECK_LAUNCH("k_attention_mma");
  return NQS_OK;
}

template <typename T>
inline int launch_attention(int n_jobs, int N, int C, int n_tan, int has_lap, int d, int H,
                            const T* QKV, T* OUT, cudaStream_t st, bool tc = false) {
  const int hd = d / H;
  const bool aligned = ((uintptr_t)QKV % 16 == 0) && ((uintptr_t)OUT % 16 == 0) &&
                       ((size_t)d * sizeof(T)) % 16 == 0;
  if constexpr (sizeof(T) == 4) {
    if (tc && g_attn_mma && C > 1 && hd == kAttMmaHd && N <= 64 && aligned &&
        C == 1 + n_tan + has_lap) {
      const float* qf = (const float*)QKV;
      float* of = (float*)OUT;
      if (N <= 16) return launch_attention_mma<1>(n_jobs, N, C, n_tan, has_lap, d, H, qf, of, st);
      if (N <= 32) return launch_attention_mma<2>(n_jobs, N, C, n_tan, has_lap, d, H, qf, of, st);
      if (N <= 48) return launch_attention_mma<3>(n_jobs, N, C, n_tan, has_lap, d, H, qf, of, st);
      return launch_attention_mma<4>(n_jobs, N, C, n_tan, has_lap, d, H, qf, of, st);
    }
  }
  if (g_attn_cta_small && N <= kAttnTok && C == 1 + n_tan + has_lap) {
    if (hd == 16)
      return launch_attention_cta_ts<T, 16>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
    if (hd == 8)
      return launch_attention_cta_ts<T, 8>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
  }
  if (N <= kAttnTok && aligned && C == 1 + n_tan + has_lap) {
    if (hd == 16) return launch_attention_rt<T, 16>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
    if (hd == 8) return launch_attention_rt<T, 8>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
    if (hd == 4)
      return launch_attention_rt<T, 4>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
  }
  if (g_large_n_cta && N > kAttnTok && N <= 64 && C == 1 + n_tan + has_lap) {
    if (hd == 16)
      return launch_attention_cta_ts<T, 16>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
    if (hd == 8)
      return launch_attention_cta_ts<T, 8>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT, st);
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_attention<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  const int awpc = attention_wpc<T>(N, hd);
  k_attention<T><<<(unsigned)(((long long)n_jobs * H + awpc - 1) / awpc), 32 * awpc,
                   attention_smem<T>(N, hd), st>>>(n_jobs, N, C, n_tan, has_lap, d, H, QKV, OUT);
  NQS_CHECK_LAUNCH("k_attention");
  return NQS_OK;
}

// LayerNorm of single-channel rows (no tangents): R tokens per warp with every load issued
// before the reductions. Same arithmetic as the value channel of k_layernorm.
template <typename T, int R>
__global__ void __launch_bounds__(256) k_layernorm1(int n_tok, int d, const T* __restrict__ X,
                                                    const T* __restrict__ g,
                                                    const T* __restrict__ b, T* __restrict__ Y) {
  constexpr int Q = NQS_MAX_EMBED / 32;
  const int lane = threadIdx.x & 31;
  const int tok0 = (blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5)) * R;
  if (tok0 >= n_tok) return;
  const T inv_d = T(1) / T(d);
  T u[R][Q];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int f = lane + 32 * q;
      u[r][q] = (f < d && tok0 + r < n_tok) ? X[(size_t)(tok0 + r) * d + f] : T(0);
    }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    T s = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) s += u[r][q];
    const T mu = warp_sum(s) * inv_d;
    s = 0;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int f = lane + 32 * q;
      if (f < d) {
        u[r][q] -= mu;
        s += u[r][q] * u[r][q];
      }
    }
    const T var = warp_sum(s) * inv_d;
    const T rho = T(1) / sqrt(var + T(kLnEps));
    if (tok0 + r < n_tok) {
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int f = lane + 32 * q;
        if (f < d) Y[(size_t)(tok0 + r) * d + f] = (u[r][q] * rho) * g[f] + b[f];
      }
    }
  }
}

// LayerNorm launcher: single-channel rows take k_layernorm1
// The same LayerNorm for float32 rows of width 64: half a warp per token, four consecutive
// features per lane (16-byte loads and stores), 16-lane butterflies, tangent rows four at a time.
// Same formulas as k_layernorm; the sums run in a different order.
__device__ __forceinline__ float hw16_sum(float v) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
template <int K>
__device__ __forceinline__ void hw16_sum_n(float (&v)[K]) {
#pragma unroll
  for (int o = 8; o > 0; o >>= 1)
#pragma unroll
    for (int k = 0; k < K; ++k) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
}
__device__ __forceinline__ float4 ld4(const float* p) { return *reinterpret_cast<const float4*>(p); }
__device__ __forceinline__ void st4(float* p, float a, float b, float c, float d) {
  *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
}

static __global__ void __launch_bounds__(256) k_layernorm_w64(int n_tok, int C, int n_tan, int has_lap,
                                                       const float* __restrict__ X,
                                                       const float* __restrict__ g,
                                                       const float* __restrict__ b,
                                                       float* __restrict__ Y) {
  constexpr int d = 64, TP = 4;
  const int hl = threadIdx.x & 15;
  const int tok = blockIdx.x * (blockDim.x >> 4) + (threadIdx.x >> 4);
  // both half-warps run every shuffle: a token past the end works on the last token, writes nothing
  const bool live = tok < n_tok;
  const int tk = live ? tok : n_tok - 1;
  const float* x = X + (size_t)tk * C * d + 4 * hl;
  float* y = Y + (size_t)tk * C * d + 4 * hl;
  const float inv_d = 1.0f / d;
  const float4 xv = ld4(x), gv = ld4(g + 4 * hl), bv = ld4(b + 4 * hl);
  float u[4] = {xv.x, xv.y, xv.z, xv.w};
  const float gm[4] = {gv.x, gv.y, gv.z, gv.w};
  const float mu = hw16_sum((u[0] + u[1]) + (u[2] + u[3])) * inv_d;
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    u[q] -= mu;
    s += u[q] * u[q];
  }
  const float var = hw16_sum(s) * inv_d;
  const float rho = 1.0f / sqrtf(var + (float)kLnEps);
  if (live)
    st4(y, u[0] * rho * gm[0] + bv.x, u[1] * rho * gm[1] + bv.y, u[2] * rho * gm[2] + bv.z,
        u[3] * rho * gm[3] + bv.w);
  const float rho3 = rho * rho * rho;
  float S1 = 0.f, S2 = 0.f, acc[4] = {0.f, 0.f, 0.f, 0.f};
  for (int t0 = 0; t0 < n_tan; t0 += TP) {
    float du[TP][4];
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      if (t0 + tt < n_tan) {
        const float4 v = ld4(x + (size_t)(1 + t0 + tt) * d);
        du[tt][0] = v.x;
        du[tt][1] = v.y;
        du[tt][2] = v.z;
        du[tt][3] = v.w;
      } else {
        du[tt][0] = du[tt][1] = du[tt][2] = du[tt][3] = 0.f;
      }
    }
    float mt[TP], s23[2 * TP];
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) mt[tt] = (du[tt][0] + du[tt][1]) + (du[tt][2] + du[tt][3]);
    hw16_sum_n<TP>(mt);
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      mt[tt] *= inv_d;
      float s2 = 0.f, s3 = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        du[tt][q] -= mt[tt];
        s2 += u[q] * du[tt][q];
        s3 += du[tt][q] * du[tt][q];
      }
      s23[2 * tt] = s2;
      s23[2 * tt + 1] = s3;
    }
    hw16_sum_n<2 * TP>(s23);
#pragma unroll
    for (int tt = 0; tt < TP; ++tt) {
      const int t = t0 + tt;
      if (t >= n_tan) break;  // uniform over the warp (both tokens share n_tan)
      const float dv = 2.f * s23[2 * tt] * inv_d;
      const float drho = -0.5f * rho3 * dv;
      float o[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        o[q] = (du[tt][q] * rho + u[q] * drho) * gm[q];
        acc[q] += du[tt][q] * drho;
      }
      if (live) st4(y + (size_t)(1 + t) * d, o[0], o[1], o[2], o[3]);
      S1 += dv * dv;
      S2 += s23[2 * tt + 1] * inv_d;
    }
  }
  if (has_lap) {
    const float4 lv = ld4(x + (size_t)(C - 1) * d);
    float dl[4] = {lv.x, lv.y, lv.z, lv.w};
    const float ml = hw16_sum((dl[0] + dl[1]) + (dl[2] + dl[3])) * inv_d;
    float s2 = 0.f;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      dl[q] -= ml;
      s2 += u[q] * dl[q];
    }
    const float dvl = 2.f * hw16_sum(s2) * inv_d + 2.f * S2;
    const float d2rho = 0.75f * rho3 * rho * rho * S1 - 0.5f * rho3 * dvl;
    float o[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) o[q] = (dl[q] * rho + 2.f * acc[q] + u[q] * d2rho) * gm[q];
    if (live) st4(y + (size_t)(C - 1) * d, o[0], o[1], o[2], o[3]);
  }
}

template <typename T>
inline int launch_layernorm(int n_tok, int C, int n_tan, int has_lap, int d, const T* X,
                            const T* g, const T* b, T* Y, cudaStream_t st) {
  if (C == 1) {
    constexpr int R = 4;
    const int nw = (n_tok + R - 1) / R;
    k_layernorm1<T, R><<<(nw + 7) / 8, 256, 0, st>>>(n_tok, d, X, g, b, Y);
    NQS_CHECK_LAUNCH("k_layernorm1");
  } else {
    if constexpr (sizeof(T) == 4) {
      if (d == 64 && ((uintptr_t)X % 16 == 0) && ((uintptr_t)Y % 16 == 0) &&
          ((uintptr_t)g % 16 == 0) && ((uintptr_t)b % 16 == 0)) {
        k_layernorm_w64<<<(unsigned)((n_tok + 15) / 16), 256, 0, st>>>(
            n_tok, C, n_tan, has_lap, (const float*)X, (const float*)g, (const float*)b,
            (float*)Y);
        NQS_CHECK_LAUNCH("k_layernorm_w64");
        return NQS_OK;
      }
    }
    const unsigned grid = (unsigned)((n_tok + 7) / 8);
    if (d <= 32)
      k_layernorm<T, 1><<<grid, 256, 0, st>>>(n_tok, C, n_tan, has_lap, d, X, g, b, Y);
    else if (d <= 64)
      k_layernorm<T, 2><<<grid, 256, 0, st>>>(n_tok, C, n_tan, has_lap, d, X, g, b, Y);
    else
      k_layernorm<T><<<grid, 256, 0, st>>>(n_tok, C, n_tan, has_lap, d, X, g, b, Y);
    NQS_CHECK_LAUNCH("k_layernorm");
  }
  return NQS_OK;
}

// ============================================================================================
// tanh-GELU (jax.nn.gelu, approximate=True) with tangent / Laplacian channels, in place.
//   g = x cdf, cdf = 0.5 (1 + tanh(w)), w = c (x + 0.044715 x^3)
//   g' = cdf + 0.5 x sech^2 w',  g'' = sech^2 (w' - x tanh(w) w'^2 + 0.5 x w'')
// ============================================================================================
template <typename T>
__global__ void __launch_bounds__(256) k_gelu(size_t n_tok, int C, int n_tan, int has_lap, int D,
                                              T* __restrict__ X) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_tok * (size_t)D) return;
  const size_t tok = idx / D;
  const int f = (int)(idx - tok * D);
  T* x = X + tok * (size_t)C * D + f;
  const T xv = x[0];
  const T c = T(0.7978845608028654);  // sqrt(2/pi)
  const T b3 = T(0.044715);
  const T th = gelu_tanh_w(xv);
  const T cdf = T(0.5) * (T(1) + th);
  const T sech2 = T(1) - th * th;
  const T w1 = c * (T(1) + T(3) * b3 * xv * xv);
  const T w2 = c * T(6) * b3 * xv;
  const T g1 = cdf + T(0.5) * xv * sech2 * w1;
  const T g2 = sech2 * (w1 - xv * th * w1 * w1 + T(0.5) * xv * w2);
  // pass 1: independent loads of the tangents (sum of squares for the Laplacian); pass 2 rescales
  // them in place (the second reads hit L1)
  T acc = 0;
  if (has_lap) {
    T a4[4] = {0, 0, 0, 0};
    int t = 0;
    for (; t + 3 < n_tan; t += 4) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const T xt = x[(size_t)(1 + t + u) * D];
        a4[u] += xt * xt;
      }
    }
    for (; t < n_tan; ++t) {
      const T xt = x[(size_t)(1 + t) * D];
      a4[0] += xt * xt;
    }
    acc = (a4[0] + a4[1]) + (a4[2] + a4[3]);
  }
  x[0] = gelu_value(xv, th);
  int t = 0;
  for (; t + 3 < n_tan; t += 4) {
    T v4[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) v4[u] = x[(size_t)(1 + t + u) * D];
#pragma unroll
    for (int u = 0; u < 4; ++u) x[(size_t)(1 + t + u) * D] = g1 * v4[u];
  }
  {
    T v4[4];
    const int nr = n_tan - t;
#pragma unroll
    for (int u = 0; u < 3; ++u)
      if (u < nr) v4[u] = x[(size_t)(1 + t + u) * D];
#pragma unroll
    for (int u = 0; u < 3; ++u)
      if (u < nr) x[(size_t)(1 + t + u) * D] = g1 * v4[u];
  }
  if (has_lap) {
    T* p = x + (size_t)(C - 1) * D;
    *p = g1 * (*p) + g2 * acc;
  }
}

// The same GELU for float32 rows, four consecutive features per thread (16-byte loads and
// stores): same formulas as k_gelu, and the same two passes over the tangents.
static __global__ void __launch_bounds__(256) k_gelu4(size_t n_tok, int C, int n_tan, int has_lap, int D,
                                               float* __restrict__ X) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int D4 = D >> 2;
  if (idx >= n_tok * (size_t)D4) return;
  const size_t tok = idx / D4;
  const int f = 4 * (int)(idx - tok * D4);
  float* x = X + tok * (size_t)C * D + f;
  const float4 x4 = *reinterpret_cast<const float4*>(x);
  const float xv[4] = {x4.x, x4.y, x4.z, x4.w};
  const float c = 0.7978845608028654f, b3 = 0.044715f;
  float th[4], g1[4], g2[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    th[q] = gelu_tanh_w(xv[q]);
    const float cdf = 0.5f * (1.f + th[q]);
    const float sech2 = 1.f - th[q] * th[q];
    const float w1 = c * (1.f + 3.f * b3 * xv[q] * xv[q]);
    const float w2 = c * 6.f * b3 * xv[q];
    g1[q] = cdf + 0.5f * xv[q] * sech2 * w1;
    g2[q] = sech2 * (w1 - xv[q] * th[q] * w1 * w1 + 0.5f * xv[q] * w2);
  }
  float acc[4] = {0.f, 0.f, 0.f, 0.f};
  if (has_lap) {
    for (int t = 0; t < n_tan; ++t) {
      const float4 v = *reinterpret_cast<const float4*>(x + (size_t)(1 + t) * D);
      acc[0] += v.x * v.x;
      acc[1] += v.y * v.y;
      acc[2] += v.z * v.z;
      acc[3] += v.w * v.w;
    }
  }
  *reinterpret_cast<float4*>(x) = make_float4(gelu_value(xv[0], th[0]), gelu_value(xv[1], th[1]),
                                              gelu_value(xv[2], th[2]), gelu_value(xv[3], th[3]));
  for (int t = 0; t < n_tan; ++t) {
    float4* p = reinterpret_cast<float4*>(x + (size_t)(1 + t) * D);
    const float4 v = *p;
    *p = make_float4(g1[0] * v.x, g1[1] * v.y, g1[2] * v.z, g1[3] * v.w);
  }
  if (has_lap) {
    float4* p = reinterpret_cast<float4*>(x + (size_t)(C - 1) * D);
    const float4 v = *p;
    *p = make_float4(g1[0] * v.x + g2[0] * acc[0], g1[1] * v.y + g2[1] * acc[1],
                     g1[2] * v.z + g2[2] * acc[2], g1[3] * v.w + g2[3] * acc[3]);
  }
}

// ============================================================================================
// Head: envelope, K generalized spinor determinants (complex, partial pivoting, float64),
// complex log-sum-exp over dets with det_logw, optional pair Jastrow; with tangents:
//   d_t log det M = tr(M^-1 d_t M),   Lap log det M = tr(M^-1 Lap M) - sum_t tr((M^-1 d_t M)^2)
//   LSE: d L = sum_k p_k d L_k,  Lap L = sum_k p_k (Lap L_k + sum_t (d_t L_k)^2) - sum_t (d_t L)^2
// (psiformer.py:139-189). One CTA per job.
// ============================================================================================
// Shared-memory plan of k_head (complex entries unless noted):
//   env[N*N] Wk[N*N] (inv[N*N] Bm[N*N] when tangents) ph[nG*N] G[n_tan] dLk[n_tan] fcol[N]
//   red[40] | rx[N] ry[N] (double) | sp[N] piv sing (int)
__host__ __device__ inline size_t head_smem_bytes(int N, int nG, int n_tan, bool tan) {
  const size_t n2 = (size_t)N * N;
  const size_t nc = (tan ? 4 : 2) * n2 + (size_t)nG * N + 2 * (size_t)n_tan + N + 40;
  return nc * sizeof(cplx) + 2 * N * sizeof(double) + (N + 2) * sizeof(int);
}

__device__ __forceinline__ double cabs1(cplx z) { return fabs(z.re) + fabs(z.im); }

// Block-wide complex sum; red needs >= 32 entries. All threads must call it.
__device__ __forceinline__ cplx block_sum_c(cplx v, cplx* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v.re = warp_sum(v.re);
  v.im = warp_sum(v.im);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  if (threadIdx.x < 32) {
    cplx r = threadIdx.x < nw ? red[threadIdx.x] : mk(0, 0);
    r.re = warp_sum(r.re);
    r.im = warp_sum(r.im);
    if (threadIdx.x == 0) red[0] = r;
  }
  __syncthreads();
  const cplx r = red[0];
  __syncthreads();
  return r;
}

// Gauss-Jordan (inv != nullptr) or LU (value only) with partial pivoting (largest |re|+|im|,
// first index on ties, as LAPACK getrf) on Wk (N x N row-major, rows = orbitals a,
// cols = electrons j). Writes log det (principal arg) to *out_logdet and a singular flag;
// inv receives M^-1 indexed [j][a]. All threads must call it.
__device__ __noinline__ static void det_factor(cplx* Wk, cplx* inv, int N, int* piv_s, cplx* fcol, cplx* out_logdet,
                           int* out_sing) {
  const int tid = threadIdx.x, nth = blockDim.x;
  if (inv)
    for (int idx = tid; idx < N * N; idx += nth) {
      const int r = idx / N, c = idx - r * N;
      inv[idx] = mk(r == c ? 1.0 : 0.0, 0.0);
    }
  double logabs = 0.0;
  cplx sgn = mk(1.0, 0.0);
  int sing = 0;
  __syncthreads();
  for (int c = 0; c < N; ++c) {
    if (tid < 32) {
      double best = -1.0;
      int bi = c;
      for (int r = c + tid; r < N; r += 32) {
        const double v = cabs1(Wk[r * N + c]);
        if (v > best) {
          best = v;
          bi = r;
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      if (tid == 0) *piv_s = bi;
    }
    __syncthreads();
    const int p = *piv_s;
    if (p != c) {
      for (int col = tid; col < N; col += nth) {
        cplx t = Wk[c * N + col];
        Wk[c * N + col] = Wk[p * N + col];
        Wk[p * N + col] = t;
        if (inv) {
          t = inv[c * N + col];
          inv[c * N + col] = inv[p * N + col];
          inv[p * N + col] = t;
        }
      }
      sgn = mk(-sgn.re, -sgn.im);
    }
    __syncthreads();
    const cplx pv = Wk[c * N + c];
    const double apv = hypot(pv.re, pv.im);
    if (apv == 0.0) {
      sing = 1;
    } else {
      logabs += log(apv);
      sgn = cmul(sgn, mk(pv.re / apv, pv.im / apv));
    }
    const cplx ipv = (apv == 0.0) ? mk(0.0, 0.0) : cdiv(mk(1.0, 0.0), pv);
    for (int r = tid; r < N; r += nth) {
      if (r == c || (!inv && r < c)) continue;
      fcol[r] = cmul(Wk[r * N + c], ipv);
    }
    __syncthreads();
    const int ncol = N - c - 1;
    if (inv) {
      const int wdt = ncol + N;
      const int tot = N * wdt;
      for (int idx = tid; idx < tot; idx += nth) {
        const int r = idx / wdt, cc = idx - r * wdt;
        if (r == c) continue;
        const cplx f = fcol[r];
        if (cc < ncol) {
          const int col = c + 1 + cc;
          Wk[r * N + col] = csub(Wk[r * N + col], cmul(f, Wk[c * N + col]));
        } else {
          const int col = cc - ncol;
          inv[r * N + col] = csub(inv[r * N + col], cmul(f, inv[c * N + col]));
        }
      }
      __syncthreads();
      for (int col = tid; col < N; col += nth) {
        if (col > c) Wk[c * N + col] = cmul(Wk[c * N + col], ipv);
        inv[c * N + col] = cmul(inv[c * N + col], ipv);
      }
    } else {
      const int tot = (N - c - 1) * ncol;
      for (int idx = tid; idx < tot; idx += nth) {
        const int rr = idx / ncol, cc = idx - rr * ncol;
        const int r = c + 1 + rr, col = c + 1 + cc;
        Wk[r * N + col] = csub(Wk[r * N + col], cmul(fcol[r], Wk[c * N + col]));
      }
    }
    __syncthreads();
  }
  if (tid == 0) {
    *out_logdet = sing ? mk(-INFINITY, 0.0) : mk(logabs, atan2(sgn.im, sgn.re));
    *out_sing = sing;
  }
  __syncthreads();
}

// Pair Jastrow u(r), u'(r), u''(r) (psiformer.py:168-186).
__device__ __forceinline__ void jastrow_u(const ModelConst& mc, const HeadParams& hp, double r,
                                          bool same, double* u, double* u1, double* u2) {
  if (mc.jastrow_kind == 0 && mc.knots_uniform) {
    // centres mu_k = k w, width w: with t = r / w, g_k = exp(-(t - k)^2) satisfies
    //   g_{k+1} = g_k exp(2 (t - k) - 1),   g_{k-1} = g_k exp(-2 (t - k) - 1),
    // and each factor changes by exp(-2) per step; started at the knot nearest t (g = O(1)),
    // so tails underflow harmlessly. 3 exponentials per pair instead of n_knots.
    const double* c = same ? hp.jas_same : hp.jas_opp;
    const double iw = 1.0 / mc.wdt;
    const double t = r * iw;
    const int nk = mc.n_knots;
    const int k0 = min(max((int)rint(t), 0), nk - 1);
    const double e2 = 0.1353352832366127;  // exp(-2)
    double a0 = 0, a1 = 0, a2 = 0;
    auto acc = [&](int k, double g) {
      const double z = t - (double)k;
      const double ce = c[k] * g;
      a0 += ce;
      a1 += ce * (-2.0 * z * iw);
      a2 += ce * (4.0 * z * z - 2.0) * iw * iw;
    };
    const double z0 = t - (double)k0;
    const double g0 = exp(-(z0 * z0));
    acc(k0, g0);
    double g = g0, q = exp(2.0 * z0 - 1.0);  // upward factor
    for (int k = k0 + 1; k < nk; ++k) {
      g *= q;
      q *= e2;
      acc(k, g);
    }
    g = g0;
    q = exp(-2.0 * z0 - 1.0);  // downward factor
    for (int k = k0 - 1; k >= 0; --k) {
      g *= q;
      q *= e2;
      acc(k, g);
    }
    *u = a0;
    *u1 = a1;
    *u2 = a2;
  } else if (mc.jastrow_kind == 0) {
    const double* c = same ? hp.jas_same : hp.jas_opp;
    double a0 = 0, a1 = 0, a2 = 0;
    const double iw = 1.0 / mc.wdt;
    for (int k = 0; k < mc.n_knots; ++k) {
      const double z = (r - mc.knots[k]) / mc.wdt;
      const double ce = c[k] * exp(-(z * z));
      a0 += ce;
      a1 += ce * (-2.0 * z * iw);
      a2 += ce * (4.0 * z * z - 2.0) * iw * iw;
    }
    *u = a0;
    *u1 = a1;
    *u2 = a2;
  } else {
    const double la = hp.jas_loga[0];
    const double a = (la > 0 ? la + log1p(exp(-la)) : log1p(exp(la))) + 0.05;  // softplus + .05
    const double al = same ? mc.cusp / 3.0 : mc.cusp;
    const double e = exp(-r / a);
    *u = al * a * (1.0 - e);
    *u1 = al * e;
    *u2 = -(al / a) * e;
  }
}

// Nearest-image displacement (psiformer.py:164-166): round-half-even as jnp.round.
__device__ __forceinline__ void min_image(const ModelConst& mc, double dx, double dy, double* ox,
                                          double* oy) {
  double f0 = dx * mc.Ainv[0] + dy * mc.Ainv[1];
  double f1 = dx * mc.Ainv[2] + dy * mc.Ainv[3];
  f0 -= rint(f0);
  f1 -= rint(f1);
  *ox = f0 * mc.A[0] + f1 * mc.A[1];
  *oy = f0 * mc.A[2] + f1 * mc.A[3];
}

// --------------------------------------------------------------------------------------------
// warp-synchronous complex LU (value) / Gauss-Jordan (with inverse) on one N x N matrix in shared
// memory; partial pivoting on |re|+|im| with the first index on ties (as LAPACK getrf).
// M rows = orbitals a, columns = electrons j; inv (nullable) receives M^-1 indexed [j][a].
// --------------------------------------------------------------------------------------------
__device__ __forceinline__ void warp_factor(cplx* M, cplx* inv, int N, cplx* fcol, cplx* logdet,
                                            int* singular) {
  const int lane = threadIdx.x & 31;
  if (inv)
    for (int idx = lane; idx < N * N; idx += 32) {
      const int r = idx / N, c = idx - r * N;
      inv[idx] = mk(r == c ? 1.0 : 0.0, 0.0);
    }
  double logabs = 0.0;
  cplx sgn = mk(1.0, 0.0);
  int sing = 0;
  __syncwarp();
  for (int c = 0; c < N; ++c) {
    double best = -1.0;
    int bi = c;
    for (int r = c + lane; r < N; r += 32) {
      const double v = cabs1(M[r * N + c]);
      if (v > best) {
        best = v;
        bi = r;
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (bi != c) {
      for (int col = lane; col < N; col += 32) {
        cplx t = M[c * N + col];
        M[c * N + col] = M[bi * N + col];
        M[bi * N + col] = t;
        if (inv) {
          t = inv[c * N + col];
          inv[c * N + col] = inv[bi * N + col];
          inv[bi * N + col] = t;
        }
      }
      sgn = mk(-sgn.re, -sgn.im);
    }
    __syncwarp();
    const cplx pv = M[c * N + c];
    const double apv = hypot(pv.re, pv.im);
    if (apv == 0.0) {
      sing = 1;
    } else {
      logabs += log(apv);
      sgn = cmul(sgn, mk(pv.re / apv, pv.im / apv));
    }
    const cplx ipv = (apv == 0.0) ? mk(0.0, 0.0) : cdiv(mk(1.0, 0.0), pv);
    for (int r = lane; r < N; r += 32)
      if (r != c && (inv || r > c)) fcol[r] = cmul(M[r * N + c], ipv);
    __syncwarp();
    const int nc = N - c - 1;
    if (inv) {
      const int wd = nc + N;
      for (int idx = lane; idx < N * wd; idx += 32) {
        const int r = idx / wd, cc = idx - r * wd;
        if (r == c) continue;
        if (cc < nc) {
          const int col = c + 1 + cc;
          M[r * N + col] = csub(M[r * N + col], cmul(fcol[r], M[c * N + col]));
        } else {
          const int col = cc - nc;
          inv[r * N + col] = csub(inv[r * N + col], cmul(fcol[r], inv[c * N + col]));
        }
      }
      __syncwarp();
      for (int col = lane; col < N; col += 32) {
        if (col > c) M[c * N + col] = cmul(M[c * N + col], ipv);
        inv[c * N + col] = cmul(inv[c * N + col], ipv);
      }
    } else {
      for (int idx = lane; idx < nc * nc; idx += 32) {
        const int r = c + 1 + idx / nc, col = c + 1 + idx % nc;
        M[r * N + col] = csub(M[r * N + col], cmul(fcol[r], M[c * N + col]));
      }
    }
    __syncwarp();
  }
  *logdet = sing ? mk(-INFINITY, 0.0) : mk(logabs, atan2(sgn.im, sgn.re));
  *singular = sing;
}

// Shared-memory plan of k_head: per job slot env[N*N], ph[nG*N], per-det results
// (logdet, lap part, sum of squares, singular flag) and dL_k[K][n_tan]; per warp M[N*N]
// (+ inv[N*N], B[N*N] with tangents) and fcol[N].
struct HeadPlan {
  int wpc, jpc;
  size_t job_bytes, warp_bytes, bytes;
};
// slot sizes are rounded to 128 bytes so every job / warp slot (and the complex arrays at its
// start) stays 16-byte aligned for vector shared-memory access
__host__ __device__ inline size_t round128(size_t b) { return (b + 127) & ~(size_t)127; }
__host__ __device__ inline size_t head_job_bytes(int N, int nG, int K, int n_tan) {
  return round128(16 * ((size_t)N * N + (size_t)nG * N + 3 * (size_t)K + (size_t)K * n_tan) +
                  8 * 2 * (size_t)N + 4 * ((size_t)N + K) + 16);
}
__host__ __device__ inline size_t head_warp_bytes(int N, bool tan) {
  return round128(16 * ((tan ? 3 : 1) * (size_t)N * N + (size_t)N));
}
inline HeadPlan head_plan(int N, int nG, int K, int n_tan, bool tan) {
  HeadPlan p;
  p.wpc = tan ? 4 : 8;
  p.job_bytes = head_job_bytes(N, nG, K, tan ? n_tan : 0);
  p.warp_bytes = head_warp_bytes(N, tan);
  for (;;) {
    p.jpc = std::max(1, p.wpc / K);
    p.bytes = p.jpc * p.job_bytes + p.wpc * p.warp_bytes;
    if (p.bytes <= 200 * 1024 || p.wpc == 1) break;
    p.wpc /= 2;
  }
  return p;
}

template <typename TIN, bool TAN>
__global__ void __launch_bounds__(256) k_head(JobBatch jb, ModelConst mc, const TIN* __restrict__ BF,
                                              int ldbf, HeadParams hp, HeadOut out, int j_out0,
                                              int jpc, size_t job_bytes, size_t warp_bytes) {
  const int N = jb.N, C = jb.C, nG = mc.nG, K = mc.K;
  const int n_tan = TAN ? jb.n_tan : 0;
  const bool has_lap = TAN && jb.has_lap;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int job0 = blockIdx.x * jpc;
  const int njob = min(jpc, jb.n_jobs - job0);
  extern __shared__ __align__(16) unsigned char smraw[];
  // ---- carve ----
  auto jbase = [&](int j) -> unsigned char* { return smraw + (size_t)j * job_bytes; };
  auto j_env = [&](int j) { return reinterpret_cast<cplx*>(jbase(j)); };
  auto j_ph = [&](int j) { return j_env(j) + N * N; };
  auto j_ld = [&](int j) { return j_ph(j) + nG * N; };     // K
  auto j_lapk = [&](int j) { return j_ld(j) + K; };         // K
  auto j_sq = [&](int j) { return j_lapk(j) + K; };         // K
  auto j_dLk = [&](int j) { return j_sq(j) + K; };          // K * n_tan
  auto j_rx = [&](int j) { return reinterpret_cast<double*>(j_dLk(j) + K * n_tan); };
  auto j_ry = [&](int j) { return j_rx(j) + N; };
  auto j_sp = [&](int j) { return reinterpret_cast<int*>(j_ry(j) + N); };
  auto j_sing = [&](int j) { return j_sp(j) + N; };         // K
  unsigned char* wbase = smraw + (size_t)jpc * job_bytes + (size_t)warp * warp_bytes;
  cplx* Mw = reinterpret_cast<cplx*>(wbase);
  cplx* Iw = TAN ? Mw + N * N : nullptr;
  cplx* Bw = TAN ? Iw + N * N : nullptr;
  cplx* fw = (TAN ? Bw : Mw) + N * N;
  // ---- phase 1: positions, spins, phases, envelopes of this CTA's jobs ----
  for (int idx = threadIdx.x; idx < njob * N; idx += blockDim.x) {
    const int j = idx / N, i = idx - j * N;
    const JobInfo ji = job_info(jb, job0 + j);
    const double* r = jb.R + ((size_t)ji.walker * N + i) * 2;
    j_rx(j)[i] = r[0];
    j_ry(j)[i] = r[1];
    j_sp(j)[i] = job_spin(jb, ji, i);
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < njob * nG * N; idx += blockDim.x) {
    const int j = idx / (nG * N), r = idx - j * nG * N, g = r / N, i = r - g * N;
    double sn, cs;
    sincos(mc.Gs[2 * g] * j_rx(j)[i] + mc.Gs[2 * g + 1] * j_ry(j)[i], &sn, &cs);
    j_ph(j)[r] = mk(cs, sn);
  }
  __syncthreads();
  auto Weff = [&](int a, int g, int s) -> cplx {
    const size_t o = ((size_t)a * nG + g) * 2 + s;
    cplx w = mk(mc.W[2 * o], mc.W[2 * o + 1]);
    if (mc.learnable_env) w = cadd(w, mk(hp.dW[o], hp.dW[(size_t)N * nG * 2 + o]));
    return w;
  };
  for (int idx = threadIdx.x; idx < njob * N * N; idx += blockDim.x) {
    const int j = idx / (N * N), r = idx - j * N * N, a = r / N, i = r - a * N;
    const int s = j_sp(j)[i];
    const cplx* ph = j_ph(j);
    cplx e = mk(0, 0);
    for (int g = 0; g < nG; ++g) cfma(e, ph[g * N + i], Weff(a, g, s));
    j_env(j)[r] = e;
  }
  __syncthreads();
  // ---- phase 2: one warp per (job, determinant) ----
  for (int q = warp; q < njob * K; q += nwarp) {
    const int j = q / K, k = q - j * K;
    const int job = job0 + j;
    const JobInfo ji = job_info(jb, job);
    const int te_lo = ji.tan_e0, te_hi = ji.tan_e0 + n_tan / 2;
    const cplx* env = j_env(j);
    const cplx* ph = j_ph(j);
    const int* sp = j_sp(j);
    auto bfval = [&](int c, int a, int i) -> cplx {
      const TIN* p = BF + (((size_t)job * N + i) * C + c) * ldbf;
      return mk((double)p[k * N + a], (double)p[K * N + k * N + a]);
    };
    for (int idx = lane; idx < N * N; idx += 32) {
      const int a = idx / N, i = idx - a * N;
      const cplx b0 = bfval(0, a, i);
      Mw[idx] = cmul(env[idx], mk(1.0 + b0.re, b0.im));
    }
    __syncwarp();
    cplx logdet;
    int sing;
    warp_factor(Mw, Iw, N, fw, &logdet, &sing);
    cplx lapk = mk(0, 0), sq = mk(0, 0);
    if (TAN && !sing) {
      if (has_lap) {  // tr(M^-1 Lap M)
        cplx acc = mk(0, 0);
        for (int idx = lane; idx < N * N; idx += 32) {
          const int a = idx / N, i = idx - a * N;
          cplx lm = cmul(env[idx], bfval(C - 1, a, i));
          if (i >= te_lo && i < te_hi) {
            cplx dxe = mk(0, 0), dye = mk(0, 0), le = mk(0, 0);
            for (int g = 0; g < nG; ++g) {
              const cplx pw = cmul(ph[g * N + i], Weff(a, g, sp[i]));
              const double gx = mc.Gs[2 * g], gy = mc.Gs[2 * g + 1];
              cfma(dxe, pw, mk(0, gx));
              cfma(dye, pw, mk(0, gy));
              le = cadd(le, cscale(pw, -(gx * gx + gy * gy)));
            }
            const cplx b0 = bfval(0, a, i);
            const int tx = 2 * (i - te_lo);
            lm = cadd(lm, cmul(le, mk(1.0 + b0.re, b0.im)));
            lm = cadd(lm, cscale(cmul(dxe, bfval(1 + tx, a, i)), 2.0));
            lm = cadd(lm, cscale(cmul(dye, bfval(2 + tx, a, i)), 2.0));
          }
          cfma(acc, Iw[i * N + a], lm);
        }
        acc.re = warp_sum(acc.re);
        acc.im = warp_sum(acc.im);
        lapk = acc;
      }
      for (int t = 0; t < n_tan && !has_lap; ++t) {
        // without the Laplacian only tr(M^-1 D_t) = sum_{a,i} M^-1[i][a] D_t[a][i] is needed
        const int e = te_lo + t / 2, bax = t & 1;
        cplx trb = mk(0, 0);
        for (int idx = lane; idx < N * N; idx += 32) {
          const int a = idx / N, i = idx - a * N;
          cplx dm = cmul(env[idx], bfval(1 + t, a, i));
          if (i == e) {
            cplx de = mk(0, 0);
            for (int g = 0; g < nG; ++g)
              cfma(de, cmul(ph[g * N + i], Weff(a, g, sp[i])), mk(0, mc.Gs[2 * g + bax]));
            const cplx b0 = bfval(0, a, i);
            dm = cadd(dm, cmul(de, mk(1.0 + b0.re, b0.im)));
          }
          cfma(trb, Iw[i * N + a], dm);
        }
        trb.re = warp_sum(trb.re);
        trb.im = warp_sum(trb.im);
        if (lane == 0) j_dLk(j)[k * n_tan + t] = trb;
        cfma(sq, trb, trb);
      }
      for (int t = 0; t < n_tan && has_lap; ++t) {
        const int e = te_lo + t / 2, bax = t & 1;
        for (int idx = lane; idx < N * N; idx += 32) {  // D_t = d_t M
          const int a = idx / N, i = idx - a * N;
          cplx dm = cmul(env[idx], bfval(1 + t, a, i));
          if (i == e) {
            cplx de = mk(0, 0);
            for (int g = 0; g < nG; ++g)
              cfma(de, cmul(ph[g * N + i], Weff(a, g, sp[i])), mk(0, mc.Gs[2 * g + bax]));
            const cplx b0 = bfval(0, a, i);
            dm = cadd(dm, cmul(de, mk(1.0 + b0.re, b0.im)));
          }
          Mw[idx] = dm;
        }
        __syncwarp();
        cplx trb = mk(0, 0);
        for (int idx = lane; idx < N * N; idx += 32) {  // B = M^-1 D_t
          const int i = idx / N, i2 = idx - i * N;
          cplx s2 = mk(0, 0);
          for (int a = 0; a < N; ++a) cfma(s2, Iw[i * N + a], Mw[a * N + i2]);
          Bw[idx] = s2;
          if (i == i2) trb = cadd(trb, s2);
        }
        __syncwarp();
        cplx trb2 = mk(0, 0);
        for (int idx = lane; idx < N * N; idx += 32) {
          const int i = idx / N, i2 = idx - i * N;
          cfma(trb2, Bw[idx], Bw[i2 * N + i]);
        }
        trb.re = warp_sum(trb.re);
        trb.im = warp_sum(trb.im);
        trb2.re = warp_sum(trb2.re);
        trb2.im = warp_sum(trb2.im);
        if (lane == 0) j_dLk(j)[k * n_tan + t] = trb;
        lapk = csub(lapk, trb2);
        cfma(sq, trb, trb);
        __syncwarp();
      }
    }
    if (lane == 0) {
      j_ld(j)[k] = logdet;
      j_lapk(j)[k] = lapk;
      j_sq(j)[k] = sq;
      j_sing(j)[k] = sing;
    }
    __syncwarp();
  }
  __syncthreads();
  // ---- phase 3: one warp per job: log-sum-exp over dets (max-Re shift), Jastrow, outputs ----
  for (int j = warp; j < njob; j += nwarp) {
    const int job = job0 + j;
    const JobInfo ji = job_info(jb, job);
    const int te_lo = ji.tan_e0, te_hi = ji.tan_e0 + n_tan / 2;
    const int jo = j_out0 + job;
    const cplx* ld = j_ld(j);
    const int* sg = j_sing(j);
    const double* rx = j_rx(j);
    const double* ry = j_ry(j);
    const int* sp = j_sp(j);
    double m = -INFINITY;
    for (int k = 0; k < K; ++k) {
      const double zr = ld[k].re + ((K > 1 && hp.det_logw) ? hp.det_logw[k] : 0.0);
      if (!sg[k] && zr > m) m = zr;
    }
    const bool all_sing = (m == -INFINITY);
    cplx ssum = mk(0, 0);
    cplx p[NQS_MAX_DETS];
    for (int k = 0; k < K; ++k) {
      if (sg[k]) {
        p[k] = mk(0, 0);
        continue;
      }
      const cplx wk = (K > 1 && hp.det_logw) ? mk(hp.det_logw[k], hp.det_logw[K + k]) : mk(0, 0);
      p[k] = cexp_(mk(ld[k].re + wk.re - m, ld[k].im + wk.im));
      ssum = cadd(ssum, p[k]);
    }
    cplx L;
    if (K == 1) {
      L = ld[0];
    } else {
      L = all_sing ? mk(-INFINITY, 0.0)
                   : mk(m + log(hypot(ssum.re, ssum.im)), atan2(ssum.im, ssum.re));
      if (!all_sing) {
        const cplx inv_s = cdiv(mk(1.0, 0.0), ssum);
        for (int k = 0; k < K; ++k) p[k] = cmul(p[k], inv_s);
      }
    }
    if (K == 1) p[0] = mk(1.0, 0.0);
    // Jastrow value and Laplacian
    double J = 0.0, lapJ = 0.0;
    if (mc.use_jastrow) {
      for (int idx = lane; idx < N * N; idx += 32) {
        const int i = idx / N, jj = idx - i * N;
        if (jj <= i) continue;
        double dx, dy;
        min_image(mc, rx[i] - rx[jj], ry[i] - ry[jj], &dx, &dy);
        const double d2 = dx * dx + dy * dy;
        const double r = sqrt(d2 + 1e-12);
        double u, u1, u2;
        jastrow_u(mc, hp, r, sp[i] == sp[jj], &u, &u1, &u2);
        J += u;
        if (has_lap) {
          const int cnt = (i >= te_lo && i < te_hi) + (jj >= te_lo && jj < te_hi);
          lapJ += (u2 * d2 / (r * r) + u1 * (2.0 / r - d2 / (r * r * r))) * cnt;
        }
      }
      J = warp_sum(J);
      lapJ = warp_sum(lapJ);
    }
    cplx sumsq = mk(0, 0);
    for (int t = lane; t < n_tan; t += 32) {
      cplx g = mk(0, 0);
      if (all_sing) {
        g = mk(NAN, NAN);
      } else {
        for (int k = 0; k < K; ++k)
          if (!sg[k]) cfma(g, p[k], j_dLk(j)[k * n_tan + t]);
      }
      cfma(sumsq, g, g);
      if (mc.use_jastrow) {
        const int e = te_lo + t / 2, bax = t & 1;
        double gj = 0.0;
        for (int jj = 0; jj < N; ++jj) {
          if (jj == e) continue;
          double dx, dy;
          min_image(mc, rx[e] - rx[jj], ry[e] - ry[jj], &dx, &dy);
          const double r = sqrt(dx * dx + dy * dy + 1e-12);
          double u, u1, u2;
          jastrow_u(mc, hp, r, sp[e] == sp[jj], &u, &u1, &u2);
          gj += u1 * (bax == 0 ? dx : dy) / r;
        }
        g.re += gj;
      }
      if (out.dL) out.dL[(size_t)jo * jb.n_tan + t] = g;
    }
    sumsq.re = warp_sum(sumsq.re);
    sumsq.im = warp_sum(sumsq.im);
    if (lane == 0) {
      if (mc.use_jastrow) L.re += J;
      if (out.L) out.L[jo] = L;
      if (has_lap && out.lap) {
        cplx lap;
        if (all_sing) {
          lap = mk(NAN, NAN);
        } else if (K == 1) {
          lap = j_lapk(j)[0];
        } else {
          lap = mk(0, 0);
          for (int k = 0; k < K; ++k)
            if (!sg[k]) cfma(lap, p[k], cadd(j_lapk(j)[k], j_sq(j)[k]));
          lap = csub(lap, sumsq);
        }
        lap.re += lapJ;
        out.lap[jo] = lap;
      }
    }
  }
}

inline size_t head_smem(int N, int nG, int n_tan, bool tan) {
  (void)N; (void)nG; (void)n_tan; (void)tan;
  return 0;
}


}  // namespace nqs
