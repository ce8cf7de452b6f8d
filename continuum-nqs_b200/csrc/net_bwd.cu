// net_bwd.cu — hand-written reverse mode of the wavefunction: per-sample Jacobian
//   O[w][k] = d log psi(R_w, S_w) / d theta_k   (src/nqs/minsr.py:56-65)
// written as two real rows per walker (Re O in row w, Im O in row W + w of a [2W][P] matrix).
//
// log psi is complex and holomorphic in the complex parameters, the backbone is real, so every
// real activation carries a complex adjoint stored as two channels (re, im) and pushed through the
// real layers independently. For a complex leaf c = a + i b, dL/da = dL/dc and dL/db = i dL/dc.
// The forward pass is recomputed per chunk of walkers. By default every block's activations are
// kept; with per-block checkpointing only each block's input is kept and the block's forward is
// recomputed from it just before its reverse step (same kernels, same inputs: the recomputed
// activations are bit-identical, so is O). Attention probabilities are always recomputed from
// q, k inside the attention backward.
//
// The adjoints reach the parameters through a writer: ORows stores each walker's two Jacobian
// rows; VjpAcc contracts them with a per-walker complex cotangent c_w on the fly,
//   grad_k += Re(c_w O[w][k]),
// so a vector-Jacobian product never materialises O (src/nqs/train.py:53-59 differentiates the
// surrogate 2 mean Re[conj(e - mean e) log psi] this way).
#include <cstdio>
#include <algorithm>

#include "net_kernels.cuh"

namespace nqs {

// --------------------------------------------------------------------------------------------
// O row writer
// --------------------------------------------------------------------------------------------
template <typename TO>
struct ORows {
  static constexpr bool kVjp = false;
  TO* O;
  int64_t P;
  int W;  // total walkers (Im rows start at W)
  __device__ __forceinline__ void put(int w, int64_t col, double re, double im) const {
    O[(size_t)w * P + col] = (TO)re;
    O[((size_t)W + w) * P + col] = (TO)im;
  }
  // complex leaf at theta offset `off` with `n` elements: element e gets dL/dc = g
  __device__ __forceinline__ void put_c(int w, int64_t off, int64_t n, int64_t e, double gre,
                                        double gim) const {
    put(w, off + e, gre, gim);        // d/d Re c = g
    put(w, off + n + e, -gim, gre);   // d/d Im c = i g
  }
};

// contraction writer of the vector-Jacobian product: grad[col] += Re(c_w (re + i im)), double
// atomics (grad zeroed by the caller)
struct VjpAcc {
  static constexpr bool kVjp = true;
  double* grad;
  const cplx* ct;  // cotangent per walker (global walker index)
  __device__ __forceinline__ void put(int w, int64_t col, double re, double im) const {
    const cplx c = ct[w];
    atomicAdd(grad + col, c.re * re - c.im * im);
  }
  __device__ __forceinline__ void put_c(int w, int64_t off, int64_t n, int64_t e, double gre,
                                        double gim) const {
    put(w, off + e, gre, gim);
    put(w, off + n + e, -gim, gre);
  }
};

// --------------------------------------------------------------------------------------------
// per-walker weight gradient of a Dense layer: G[i][o] = sum_tok X[tok][i] Ybar[tok][ch][o]
// grid (walker, ceil(d_out / 128)); X rows ld ldx (+ col offset folded in the pointer);
// Ybar rows [tok][2][ldy]
// --------------------------------------------------------------------------------------------
template <typename T, typename TO>
__global__ void __launch_bounds__(256) k_wgrad(int N, int d_in, int d_out, const T* __restrict__ X,
                                               int ldx, const T* __restrict__ Yb, int ldy,
                                               ORows<TO> o, int w0, int64_t off_k, int64_t off_b,
                                               int is_complex) {
  constexpr int OT = 128;
  const int wl = blockIdx.x, o0 = blockIdx.y * OT;
  const int w = w0 + wl;
  const int ot = min(OT, d_out - o0);
  extern __shared__ __align__(16) unsigned char smraw[];
  T* xs = reinterpret_cast<T*>(smraw);  // [N][d_in]
  T* ys = xs + (size_t)N * d_in;        // [N][2][ot]
  const T* Xw = X + (size_t)wl * N * ldx;
  const T* Yw = Yb + (size_t)wl * N * 2 * ldy;
  for (int idx = threadIdx.x; idx < N * d_in; idx += blockDim.x) {
    const int t = idx / d_in, i = idx - t * d_in;
    xs[idx] = Xw[(size_t)t * ldx + i];
  }
  for (int idx = threadIdx.x; idx < N * 2 * ot; idx += blockDim.x) {
    const int t = idx / (2 * ot), r = idx - t * 2 * ot, ch = r / ot, oo = r - ch * ot;
    ys[idx] = Yw[((size_t)t * 2 + ch) * ldy + o0 + oo];
  }
  __syncthreads();
  // register blocks of 4 inputs x 4 outputs x 2 channels: lane -> outputs lane + 32 u, warp ->
  // inputs w + 8 (4 c + v) of chunk c; accumulation in T (the activations' type)
  const int64_t nK = (int64_t)d_in * d_out;
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nwp = blockDim.x >> 5;
  for (int i0 = wp; i0 < d_in; i0 += 4 * nwp) {
    T ar[4][4], ai[4][4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int u = 0; u < 4; ++u) ar[v][u] = ai[v][u] = T(0);
    for (int t = 0; t < N; ++t) {
      T xv[4], yr[4], yi[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) {
        const int i = i0 + v * nwp;
        xv[v] = i < d_in ? xs[t * d_in + i] : T(0);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int oo = lane + 32 * u;
        yr[u] = oo < ot ? ys[(t * 2) * ot + oo] : T(0);
        yi[u] = oo < ot ? ys[(t * 2 + 1) * ot + oo] : T(0);
      }
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          ar[v][u] = fma(xv[v], yr[u], ar[v][u]);
          ai[v][u] = fma(xv[v], yi[u], ai[v][u]);
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int i = i0 + v * nwp;
      if (i >= d_in) continue;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int oo = lane + 32 * u;
        if (oo >= ot) continue;
        const int64_t e = (int64_t)i * d_out + o0 + oo;
        if (is_complex)
          o.put_c(w, off_k, nK, e, (double)ar[v][u], (double)ai[v][u]);
        else
          o.put(w, off_k + e, (double)ar[v][u], (double)ai[v][u]);
      }
    }
  }
  if (off_b >= 0) {
    for (int oo = threadIdx.x; oo < ot; oo += blockDim.x) {
      double gr = 0, gi = 0;
      for (int t = 0; t < N; ++t) {
        gr += (double)ys[(t * 2) * ot + oo];
        gi += (double)ys[(t * 2 + 1) * ot + oo];
      }
      if (is_complex)
        o.put_c(w, off_b, d_out, o0 + oo, gr, gi);
      else
        o.put(w, off_b + o0 + oo, gr, gi);
    }
  }
}

template <typename T, typename TO>
static int launch_wgrad(int nw, int N, int d_in, int d_out, const T* X, int ldx, const T* Yb,
                        int ldy, ORows<TO> o, int w0, int64_t off_k, int64_t off_b, int is_c,
                        cudaStream_t st) {
  const int ot = std::min(128, d_out);
  const size_t sm = sizeof(T) * ((size_t)N * d_in + (size_t)N * 2 * ot);
  if (sm > 48 * 1024)
    cudaFuncSetAttribute(k_wgrad<T, TO>, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024);
  k_wgrad<T, TO><<<dim3(nw, (d_out + 127) / 128), 256, sm, st>>>(N, d_in, d_out, X, ldx, Yb, ldy,
                                                                  o, w0, off_k, off_b, is_c);
  NQS_CHECK_LAUNCH("k_wgrad");
  return NQS_OK;
}

// --------------------------------------------------------------------------------------------
// weight gradient of a Dense layer contracted with the cotangent and summed over walkers:
//   H[i][o] = sum_rows X[row][i] (c_w(row) Ybar[row][o])   (complex; i == d_in is the bias, X = 1)
// grid (ceil((d_in + 1) / 32), ceil(d_out / 64), row slices); each CTA reduces its rows in
// registers (4 inputs x 4 outputs x 2 parts per thread, operands staged 32 rows at a time) and
// adds to grad with double atomics: real leaf += Re H, complex leaf Re part += Re H, Im part
// -= Im H (d/d Im c = i d/dc).
// --------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_wgrad_vjp(int rows, int N, int d_in, int d_out,
                                                   const T* __restrict__ X, int ldx,
                                                   const T* __restrict__ Yb, int ldy,
                                                   const cplx* __restrict__ ct, int w0,
                                                   double* __restrict__ grad, int64_t off_k,
                                                   int64_t off_b, int is_complex,
                                                   int rows_per_cta) {
  constexpr int TI = 32, TO = 64, RB = 32;
  __shared__ T xs[RB][TI];
  __shared__ T ysr[RB][TO], ysi[RB][TO];
  const int i0 = blockIdx.x * TI, o0 = blockIdx.y * TO;
  const int r0 = blockIdx.z * rows_per_cta, r1 = min(rows, r0 + rows_per_cta);
  const int tid = threadIdx.x, ti = tid >> 4, to = tid & 15;  // inputs 4 ti + v, outputs to + 16 u
  T ar[4][4], ai[4][4];
#pragma unroll
  for (int v = 0; v < 4; ++v)
#pragma unroll
    for (int u = 0; u < 4; ++u) ar[v][u] = ai[v][u] = T(0);
  for (int rb = r0; rb < r1; rb += RB) {
    for (int idx = tid; idx < RB * TI; idx += blockDim.x) {
      const int r = idx / TI, i = idx - r * TI, row = rb + r, ii = i0 + i;
      T v = T(0);
      if (row < r1) v = ii < d_in ? X[(size_t)row * ldx + ii] : (ii == d_in ? T(1) : T(0));
      xs[r][i] = v;
    }
    for (int idx = tid; idx < RB * TO; idx += blockDim.x) {
      const int r = idx / TO, o = idx - r * TO, row = rb + r, oo = o0 + o;
      T vr = T(0), vi = T(0);
      if (row < r1 && oo < d_out) {
        const cplx c = ct[w0 + row / N];
        const T a = Yb[((size_t)row * 2) * ldy + oo], b = Yb[((size_t)row * 2 + 1) * ldy + oo];
        vr = (T)c.re * a - (T)c.im * b;
        vi = (T)c.re * b + (T)c.im * a;
      }
      ysr[r][o] = vr;
      ysi[r][o] = vi;
    }
    __syncthreads();
#pragma unroll 4
    for (int r = 0; r < RB; ++r) {
      T xv[4], yr[4], yi[4];
#pragma unroll
      for (int v = 0; v < 4; ++v) xv[v] = xs[r][4 * ti + v];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        yr[u] = ysr[r][to + 16 * u];
        yi[u] = ysi[r][to + 16 * u];
      }
#pragma unroll
      for (int v = 0; v < 4; ++v)
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          ar[v][u] = fma(xv[v], yr[u], ar[v][u]);
          ai[v][u] = fma(xv[v], yi[u], ai[v][u]);
        }
    }
    __syncthreads();
  }
  if (r0 >= r1) return;
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const int i = i0 + 4 * ti + v;
    if (i > d_in) continue;
    const int64_t base = i < d_in ? off_k : off_b;
    if (base < 0) continue;
    const int64_t n = i < d_in ? (int64_t)d_in * d_out : (int64_t)d_out;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int o = o0 + to + 16 * u;
      if (o >= d_out) continue;
      const int64_t e = i < d_in ? (int64_t)i * d_out + o : (int64_t)o;
      atomicAdd(grad + base + e, (double)ar[v][u]);
      if (is_complex) atomicAdd(grad + base + n + e, -(double)ai[v][u]);
    }
  }
}

template <typename T>
static int launch_wgrad_vjp(int nw, int N, int d_in, int d_out, const T* X, int ldx,
                            const T* Yb, int ldy, const VjpAcc& o, int w0, int64_t off_k,
                            int64_t off_b, int is_c, cudaStream_t st) {
  const int rows = nw * N;
  const int gi = (d_in + 1 + 31) / 32, go = (d_out + 63) / 64;
  // about four CTAs per SM in total, at least 64 rows per slice
  int slices = std::max(1, std::min((rows + 63) / 64, 592 / std::max(1, gi * go)));
  const int per = (rows + slices - 1) / slices;
  slices = (rows + per - 1) / per;
  k_wgrad_vjp<T><<<dim3(gi, go, slices), 128, 0, st>>>(rows, N, d_in, d_out, X, ldx, Yb, ldy, o.ct,
                                                       w0, o.grad, off_k, off_b, is_c, per);
  NQS_CHECK_LAUNCH("k_wgrad_vjp");
  return NQS_OK;
}

// the weight-gradient step of either writer
template <typename T, typename TO>
static int wgrad(const ORows<TO>& o, int nw, int N, int d_in, int d_out, const T* X, int ldx,
                 const T* Yb, int ldy, int w0, int64_t off_k, int64_t off_b, int is_c,
                 cudaStream_t st) {
  return launch_wgrad<T, TO>(nw, N, d_in, d_out, X, ldx, Yb, ldy, o, w0, off_k, off_b, is_c, st);
}
template <typename T>
static int wgrad(const VjpAcc& o, int nw, int N, int d_in, int d_out, const T* X, int ldx,
                 const T* Yb, int ldy, int w0, int64_t off_k, int64_t off_b, int is_c,
                 cudaStream_t st) {
  return launch_wgrad_vjp<T>(nw, N, d_in, d_out, X, ldx, Yb, ldy, o, w0, off_k, off_b, is_c, st);
}

// --------------------------------------------------------------------------------------------
// LayerNorm backward (one CTA per walker): x rows [tok][d], Ybar [tok][2][d]
//   z = (x - mu) rho, zbar = ybar g, xbar = rho (zbar - mean(zbar) - z mean(zbar z))
//   dL/dscale = sum_tok ybar z, dL/dbias = sum_tok ybar
// --------------------------------------------------------------------------------------------
template <typename T, class Wr>
__global__ void __launch_bounds__(256) k_ln_bwd(int N, int d, const T* __restrict__ X,
                                                const T* __restrict__ Yb, const T* __restrict__ g,
                                                T* __restrict__ Xb, int accumulate, Wr o,
                                                int w0, int64_t off_scale, int64_t off_bias) {
  constexpr int Q = NQS_MAX_EMBED / 32;
  const int wl = blockIdx.x, w = w0 + wl;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* zs = reinterpret_cast<T*>(smraw);  // [N][d]
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const T inv_d = T(1) / T(d);
  for (int t = wid; t < N; t += nwarp) {
    const size_t tok = (size_t)wl * N + t;
    const T* x = X + tok * d;
    T u[Q], gm[Q], s = 0;
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
    const T rho = T(1) / sqrt(warp_sum(s) * inv_d + T(kLnEps));
#pragma unroll
    for (int q = 0; q < Q; ++q) {
      const int f = lane + 32 * q;
      u[q] *= rho;  // z
      if (f < d) zs[t * d + f] = u[q];
    }
    for (int ch = 0; ch < 2; ++ch) {
      const T* yb = Yb + (tok * 2 + ch) * d;
      T zb[Q], s1 = 0, s2 = 0;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int f = lane + 32 * q;
        zb[q] = f < d ? yb[f] * gm[q] : T(0);
        s1 += zb[q];
        s2 += zb[q] * u[q];
      }
      const T m1 = warp_sum(s1) * inv_d, m2 = warp_sum(s2) * inv_d;
      T* xb = Xb + (tok * 2 + ch) * d;
#pragma unroll
      for (int q = 0; q < Q; ++q) {
        const int f = lane + 32 * q;
        if (f < d) {
          const T v = rho * (zb[q] - m1 - u[q] * m2);
          xb[f] = accumulate ? xb[f] + v : v;
        }
      }
    }
  }
  __syncthreads();
  for (int f = threadIdx.x; f < d; f += blockDim.x) {
    double sr = 0, si = 0, br = 0, bi = 0;
    for (int t = 0; t < N; ++t) {
      const size_t tok = (size_t)wl * N + t;
      const double y0 = (double)Yb[(tok * 2) * d + f], y1 = (double)Yb[(tok * 2 + 1) * d + f];
      const double z = (double)zs[t * d + f];
      sr = fma(y0, z, sr);
      si = fma(y1, z, si);
      br += y0;
      bi += y1;
    }
    o.put(w, off_scale + f, sr, si);
    o.put(w, off_bias + f, br, bi);
  }
}

// --------------------------------------------------------------------------------------------
// GELU backward: abar[r][ch][f] = gbar[r][ch][f] * gelu'(a[r][f])
// --------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_gelu_bwd(size_t n_tok, int D, const T* __restrict__ A, T* __restrict__ Gb) {
  const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= n_tok * D) return;
  const size_t tok = idx / D;
  const int f = (int)(idx - tok * D);
  const T x = A[idx];
  const T c = T(0.7978845608028654), b3 = T(0.044715);
  const T th = tanh(c * (x + b3 * (x * x * x)));
  const T g1 = T(0.5) * (T(1) + th) + T(0.5) * x * (T(1) - th * th) * c * (T(1) + T(3) * b3 * x * x);
  Gb[(tok * 2) * D + f] *= g1;
  Gb[(tok * 2 + 1) * D + f] *= g1;
}

// --------------------------------------------------------------------------------------------
// attention backward, one CTA per (walker, head). QKV rows [tok][3d] (value), Ob [tok][2][d],
// QKVb out [tok][2][3d].
// --------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) k_attn_bwd(int N, int d, int H, const T* __restrict__ QKV,
                                                  const T* __restrict__ Ob, T* __restrict__ QKVb) {
  const int wl = blockIdx.x / H, h = blockIdx.x - wl * H;
  const int hd = d / H;
  extern __shared__ __align__(16) unsigned char smraw[];
  T* q = reinterpret_cast<T*>(smraw);
  T* k = q + N * hd;
  T* v = k + N * hd;
  T* a = v + N * hd;   // N*N
  T* ob = a + N * N;   // N*hd
  T* ab = ob + N * hd; // N*N
  T* rs = ab + N * N;  // N
  const T sc = T(1) / sqrt(T(hd));
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int idx = tid; idx < N * hd; idx += nth) {
    const int i = idx / hd, e = idx - i * hd;
    const T* p = QKV + ((size_t)wl * N + i) * 3 * d + h * hd + e;
    q[idx] = p[0];
    k[idx] = p[d];
    v[idx] = p[2 * d];
  }
  __syncthreads();
  for (int idx = tid; idx < N * N; idx += nth) {
    const int i = idx / N, j = idx - i * N;
    T s = 0;
    for (int e = 0; e < hd; ++e) s = fma(q[i * hd + e], k[j * hd + e], s);
    a[idx] = s * sc;
  }
  __syncthreads();
  for (int i = tid; i < N; i += nth) {
    T mx = a[i * N];
    for (int j = 1; j < N; ++j) mx = max(mx, a[i * N + j]);
    T ssum = 0;
    for (int j = 0; j < N; ++j) {
      const T e = exp(a[i * N + j] - mx);
      a[i * N + j] = e;
      ssum += e;
    }
    for (int j = 0; j < N; ++j) a[i * N + j] = a[i * N + j] / ssum;
  }
  for (int ch = 0; ch < 2; ++ch) {
    __syncthreads();
    for (int idx = tid; idx < N * hd; idx += nth) {
      const int i = idx / hd, e = idx - i * hd;
      ob[idx] = Ob[(((size_t)wl * N + i) * 2 + ch) * d + h * hd + e];
    }
    __syncthreads();
    for (int idx = tid; idx < N * hd; idx += nth) {  // vbar
      const int j = idx / hd, e = idx - j * hd;
      T s = 0;
      for (int i = 0; i < N; ++i) s = fma(a[i * N + j], ob[i * hd + e], s);
      QKVb[(((size_t)wl * N + j) * 2 + ch) * 3 * d + 2 * d + h * hd + e] = s;
    }
    for (int idx = tid; idx < N * N; idx += nth) {  // abar
      const int i = idx / N, j = idx - i * N;
      T s = 0;
      for (int e = 0; e < hd; ++e) s = fma(ob[i * hd + e], v[j * hd + e], s);
      ab[idx] = s;
    }
    __syncthreads();
    for (int i = tid; i < N; i += nth) {
      T s = 0;
      for (int j = 0; j < N; ++j) s = fma(a[i * N + j], ab[i * N + j], s);
      rs[i] = s;
    }
    __syncthreads();
    for (int idx = tid; idx < N * N; idx += nth) {  // sbar (scaled)
      const int i = idx / N;
      ab[idx] = a[idx] * (ab[idx] - rs[i]) * sc;
    }
    __syncthreads();
    for (int idx = tid; idx < N * hd; idx += nth) {
      const int i = idx / hd, e = idx - i * hd;
      T sq = 0, sk = 0;
      for (int j = 0; j < N; ++j) {
        sq = fma(ab[i * N + j], k[j * hd + e], sq);
        sk = fma(ab[j * N + i], q[j * hd + e], sk);
      }
      T* p = QKVb + (((size_t)wl * N + i) * 2 + ch) * 3 * d + h * hd + e;
      p[0] = sq;
      p[d] = sk;
    }
  }
}

// --------------------------------------------------------------------------------------------
// features of the embedding input ([pos features | one-hot spin], value only) per token
// --------------------------------------------------------------------------------------------
template <typename T>
__global__ void k_features(JobBatch jb, ModelConst mc, T* __restrict__ Fo) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  const int F = 4 * mc.nf, Fp = F + 2;
  if (idx >= jb.n_jobs * jb.N * Fp) return;
  const int tokg = idx / Fp, k = idx - tokg * Fp;
  const int j = tokg / jb.N, tok = tokg - j * jb.N;
  const JobInfo ji = job_info(jb, j);
  if (k >= F) {
    Fo[idx] = (T)((k - F) == job_spin(jb, ji, tok) ? 1.0 : 0.0);
    return;
  }
  const double* r = jb.R + ((size_t)ji.walker * jb.N + tok) * 2;
  const int nf = mc.nf;
  const int al = k / (2 * nf), rem = k - al * 2 * nf, tau = rem / nf, m = rem - tau * nf + 1;
  const double sa = r[0] * mc.Ainv[al * 2 + 0] + r[1] * mc.Ainv[al * 2 + 1];
  const double ang = ((2.0 * kPi) * sa) * (double)m;
  double sn, cs;
  sincos(ang, &sn, &cs);
  Fo[idx] = (T)(tau == 0 ? sn : cs);
}

// --------------------------------------------------------------------------------------------
// head backward (one CTA per walker): dL/dbf, and O of det_logw, Jastrow, dW
// X1[tok][ch][KN] = (Re, Im) dL/dbf; X2[tok][ch][KN] = (-Im, Re) dL/dbf
// --------------------------------------------------------------------------------------------
struct HeadOffsets {
  int64_t logw, jas_same, jas_opp, loga, dW;
};

inline size_t head_bwd_smem(int N, int nG, int K, bool env_grad) {
  const size_t n2 = (size_t)N * N;
  const size_t nc = (3 + (env_grad ? 1 : 0)) * n2 + (size_t)nG * N + N + 40 + 2 * (size_t)K;
  return nc * 16 + 2 * N * sizeof(double) + (N + 2) * sizeof(int);
}

template <typename TIN, typename T, class Wr>
__global__ void __launch_bounds__(256) k_head_bwd(JobBatch jb, ModelConst mc,
                                                  const TIN* __restrict__ BF, int ldbf,
                                                  HeadParams hp, T* __restrict__ X1,
                                                  T* __restrict__ X2, Wr o,
                                                  HeadOffsets off) {
  const int wl = blockIdx.x;
  const int N = jb.N, nG = mc.nG, K = mc.K, KN = K * N;
  const JobInfo ji = job_info(jb, wl);
  const int w = ji.walker;
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* env = reinterpret_cast<cplx*>(smraw);
  cplx* Wk = env + N * N;
  cplx* inv = Wk + N * N;
  cplx* denv = inv + N * N;  // only when learnable_env
  cplx* ph = (mc.learnable_env ? denv + N * N : denv);
  cplx* fcol = ph + nG * N;
  cplx* red = fcol + N;
  cplx* pk = red + 40;     // K
  cplx* ldk = pk + K;      // K
  double* rx = reinterpret_cast<double*>(ldk + K);
  double* ry = rx + N;
  int* sp = reinterpret_cast<int*>(ry + N);
  int* piv_s = sp + N;
  int* sing_s = piv_s + 1;
  const int tid = threadIdx.x, nth = blockDim.x;
  for (int i = tid; i < N; i += nth) {
    const double* r = jb.R + ((size_t)w * N + i) * 2;
    rx[i] = r[0];
    ry[i] = r[1];
    sp[i] = job_spin(jb, ji, i);
  }
  __syncthreads();
  for (int idx = tid; idx < nG * N; idx += nth) {
    const int g = idx / N, i = idx - g * N;
    double s, c;
    sincos(mc.Gs[2 * g] * rx[i] + mc.Gs[2 * g + 1] * ry[i], &s, &c);
    ph[idx] = mk(c, s);
  }
  __syncthreads();
  const size_t nW = (size_t)N * nG * 2;
  for (int idx = tid; idx < N * N; idx += nth) {
    const int a = idx / N, i = idx - a * N;
    cplx e = mk(0, 0);
    for (int g = 0; g < nG; ++g) {
      const size_t oo = ((size_t)a * nG + g) * 2 + sp[i];
      cplx wv = mk(mc.W[2 * oo], mc.W[2 * oo + 1]);
      if (mc.learnable_env) wv = cadd(wv, mk(hp.dW[oo], hp.dW[nW + oo]));
      cfma(e, ph[g * N + i], wv);
    }
    env[idx] = e;
    if (mc.learnable_env) denv[idx] = mk(0, 0);
  }
  __syncthreads();
  auto bf0 = [&](int k, int a, int i) -> cplx {
    const TIN* p = BF + ((size_t)wl * N + i) * ldbf;
    return mk((double)p[k * N + a], (double)p[KN + k * N + a]);
  };
  // pass 1: log dets
  for (int k = 0; k < K; ++k) {
    for (int idx = tid; idx < N * N; idx += nth) {
      const int a = idx / N, i = idx - a * N;
      const cplx b = bf0(k, a, i);
      Wk[idx] = cmul(env[idx], mk(1.0 + b.re, b.im));
    }
    __syncthreads();
    det_factor(Wk, nullptr, N, piv_s, fcol, red + 33, sing_s);
    if (tid == 0) ldk[k] = *sing_s ? mk(-INFINITY, 0.0) : red[33];
    __syncthreads();
  }
  // p_k = d L / d logdet_k
  if (tid == 0) {
    if (K == 1) {
      pk[0] = isfinite(ldk[0].re) ? mk(1.0, 0.0) : mk(0.0, 0.0);
    } else {
      double m = -INFINITY;
      for (int k = 0; k < K; ++k) {
        const double zr = ldk[k].re + hp.det_logw[k];
        if (zr > m) m = zr;
      }
      cplx s = mk(0, 0);
      for (int k = 0; k < K; ++k) {
        if (!isfinite(ldk[k].re)) continue;
        s = cadd(s, cexp_(mk(ldk[k].re + hp.det_logw[k] - m, ldk[k].im + hp.det_logw[K + k])));
      }
      const cplx L = mk(m + log(hypot(s.re, s.im)), atan2(s.im, s.re));
      for (int k = 0; k < K; ++k) {
        pk[k] = isfinite(ldk[k].re)
                    ? cexp_(csub(mk(ldk[k].re + hp.det_logw[k], ldk[k].im + hp.det_logw[K + k]), L))
                    : mk(0.0, 0.0);
      }
    }
  }
  __syncthreads();
  // pass 2: inverses -> dL/dbf
  for (int k = 0; k < K; ++k) {
    for (int idx = tid; idx < N * N; idx += nth) {
      const int a = idx / N, i = idx - a * N;
      const cplx b = bf0(k, a, i);
      Wk[idx] = cmul(env[idx], mk(1.0 + b.re, b.im));
    }
    __syncthreads();
    det_factor(Wk, inv, N, piv_s, fcol, red + 33, sing_s);
    const cplx p = pk[k];
    for (int idx = tid; idx < N * N; idx += nth) {
      const int i = idx / N, a = idx - i * N;  // a fastest: coalesced writes along KN
      const cplx gM = cmul(p, inv[i * N + a]);  // dL/dM[a][i]
      const cplx gb = (p.re == 0.0 && p.im == 0.0) ? mk(0, 0) : cmul(gM, env[a * N + i]);
      const size_t row = ((size_t)wl * N + i) * 2;
      const int col = k * N + a;
      X1[row * KN + col] = (T)gb.re;
      X1[(row + 1) * KN + col] = (T)gb.im;
      X2[row * KN + col] = (T)(-gb.im);
      X2[(row + 1) * KN + col] = (T)gb.re;
      if (mc.learnable_env && !(p.re == 0.0 && p.im == 0.0)) {
        const cplx b = bf0(k, a, i);
        denv[a * N + i] = cadd(denv[a * N + i], cmul(gM, mk(1.0 + b.re, b.im)));
      }
    }
    __syncthreads();
  }
  // det_logw
  if (K > 1)
    for (int k = tid; k < K; k += nth) o.put_c(w, off.logw, K, k, pk[k].re, pk[k].im);
  // dW: dL/dW[a][g][s] = sum_{i: s_i = s} denv[a][i] ph[g][i]
  if (mc.learnable_env) {
    for (int idx = tid; idx < (int)nW; idx += nth) {
      const int a = idx / (nG * 2), r = idx - a * nG * 2, g = r / 2, s = r - g * 2;
      cplx acc = mk(0, 0);
      for (int i = 0; i < N; ++i)
        if (sp[i] == s) cfma(acc, denv[a * N + i], ph[g * N + i]);
      o.put_c(w, off.dW, (int64_t)nW, idx, acc.re, acc.im);
    }
  }
  // Jastrow
  if (mc.use_jastrow) {
    if (mc.jastrow_kind == 0) {
      for (int q = tid; q < 2 * mc.n_knots; q += nth) {
        const bool same = q < mc.n_knots;
        const int kk = same ? q : q - mc.n_knots;
        double acc = 0.0;
        for (int i = 0; i < N; ++i)
          for (int j = i + 1; j < N; ++j) {
            if ((sp[i] == sp[j]) != same) continue;
            double dx, dy;
            min_image(mc, rx[i] - rx[j], ry[i] - ry[j], &dx, &dy);
            const double r = sqrt(dx * dx + dy * dy + 1e-12);
            const double z = (r - mc.knots[kk]) / mc.wdt;
            acc += exp(-(z * z));
          }
        o.put(w, (same ? off.jas_same : off.jas_opp) + kk, acc, 0.0);
      }
    } else if (tid == 0) {
      const double la = hp.jas_loga[0];
      const double a = (la > 0 ? la + log1p(exp(-la)) : log1p(exp(la))) + 0.05;
      const double sig = 1.0 / (1.0 + exp(-la));
      double acc = 0.0;
      for (int i = 0; i < N; ++i)
        for (int j = i + 1; j < N; ++j) {
          double dx, dy;
          min_image(mc, rx[i] - rx[j], ry[i] - ry[j], &dx, &dy);
          const double r = sqrt(dx * dx + dy * dy + 1e-12);
          const double al = sp[i] == sp[j] ? mc.cusp / 3.0 : mc.cusp;
          const double e = exp(-r / a);
          acc += al * ((1.0 - e) - (r / a) * e);
        }
      o.put(w, off.loga, acc * sig, 0.0);
    }
  }
}

// --------------------------------------------------------------------------------------------
// orchestration
// --------------------------------------------------------------------------------------------
template <typename T>
struct SaveBufs {
  // per block: the block input; with all activations kept, also every intermediate (with
  // checkpointing the intermediates live in slot 0 and are recomputed per block)
  T *xin[NQS_MAX_DEPTH], *h0[NQS_MAX_DEPTH], *qkv[NQS_MAX_DEPTH], *ao[NQS_MAX_DEPTH];
  T *xmid[NQS_MAX_DEPTH], *h1[NQS_MAX_DEPTH], *a0[NQS_MAX_DEPTH], *g0[NQS_MAX_DEPTH];
  T *xL, *hf, *bf, *feat;
  T *xb, *hb, *big, *X1, *X2;
};

// elements per activation row of one block's intermediates (h0 qkv(3d) ao xmid h1 a0 g0)
static size_t block_inter_elems(const ModelConst& mc) {
  const size_t d = mc.d, D = (size_t)mc.ff * d;
  return 7 * d + 2 * D;
}

template <typename T>
size_t bwd_row_elems(const ModelConst& mc, bool ckpt) {
  const size_t d = mc.d, D = (size_t)mc.ff * d, KN = (size_t)mc.K * mc.N;
  const size_t inter = block_inter_elems(mc);
  const size_t blocks = (size_t)mc.depth * d + (ckpt ? (mc.depth ? inter : 0) : mc.depth * inter);
  const size_t big = std::max({6 * d, 2 * D, 2 * KN});
  return blocks + d /* xL */ + d /* hf */ + 2 * KN /* bf */ + (4 * mc.nf + 2) + 2 * d + 2 * d +
         big + 4 * KN;
}

// walkers per chunk: 2^17 activation rows with every block kept; with checkpointing the rows
// that fit in the same bytes, at most 2^18 (the two-channel adjoint GEMMs then see at most 2^19
// rows, the forward network's chunk limit)
template <typename T>
size_t bwd_chunk_walkers(const ModelConst& mc, int W, bool ckpt) {
  size_t rows = (size_t)1 << 17;
  if (ckpt)
    rows = std::min<size_t>((size_t)1 << 18,
                            rows * bwd_row_elems<T>(mc, false) / bwd_row_elems<T>(mc, true));
  return std::max<size_t>(1, std::min<size_t>((size_t)W, rows / mc.N));
}

template <typename T>
size_t backward_scratch(const ModelConst& mc, int W, bool ckpt) {
  const size_t nw = bwd_chunk_walkers<T>(mc, W, ckpt);
  return nw * mc.N * bwd_row_elems<T>(mc, ckpt) * sizeof(T) + 64 * 256;
}

template <typename T>
size_t per_sample_O_scratch(const ModelConst& mc, int W) {
  return backward_scratch<T>(mc, W, false);
}

static inline bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// Y (+)= X W^T of a reverse-pass layer. Float32 with the tensor-core weights on: a tcgen05 row
// GEMM that reads the stored [d_in][d_out] kernel as the K-major operand of the product (no copy);
// otherwise, or for an operand layout the TMA cannot take, the SIMT GEMM.
template <typename T>
static int gemm_wt(GemmArgs<T>& g, const TcNet& tc, cudaStream_t st) {
  if constexpr (sizeof(T) == 4) {
    const GemmSeg<T>& s0 = g.seg[0];
    const bool ok = tc.on && g.nseg == 1 && g.trans_w && !s0.b && s0.out_off == 0 &&
                    s0.ldw == g.K && g.K % 32 == 0 && s0.ncols % 16 == 0 && g.ldx % 4 == 0 &&
                    g.ldy % 4 == 0 && aligned16(g.X) && aligned16(g.Y) && aligned16(s0.W) &&
                    (!g.Res || (g.Res == g.Y && g.ldr == g.ldy));
    if (ok)
      return rowgemm_tc((const float*)g.X, g.ldx, g.rows, g.K, (const float*)s0.W, s0.ncols,
                        s0.ncols, nullptr, g.C, (const float*)g.Res, g.ldr, (float*)g.Y, g.ldy,
                        tc.err, st);
  }
  return launch_gemm<T>(g, st);
}

// forward of block l from x = b.xin[l] into the block's intermediates (slot s), and, when y is
// given, its output y = xmid + W1 GELU(W0 LN1 xmid) + b1
template <typename T>
static int block_forward(const ModelConst& mc, const BlockW<T>& bw, const TcNet& tc,
                         SaveBufs<T>& b, int l, int s, int nw, T* y, cudaStream_t st) {
  const int N = mc.N, d = mc.d, D = mc.ff * d, H = mc.H, nt = nw * N;
  const T* x = b.xin[l];
  NQS_TRY(launch_layernorm<T>(nt, 1, 0, 0, d, x, bw.ln0_s, bw.ln0_b, b.h0[s], st));
  if constexpr (sizeof(T) == 4) {
    if (tc.on) {  // the Dense layers on the tensor cores, as in the forward passes
      auto w16 = [&](const uint16_t* p) { return tc.bf16 ? p : nullptr; };
      NQS_TRY(rowgemm_tc(b.h0[s], d, nt, d, tc.wqkv[l], tc.npad_qkv, 3 * d, tc.bqkv[l], 1,
                         nullptr, 0, b.qkv[s], 3 * d, tc.err, st, 0, w16(tc.wqkv16[l])));
      NQS_TRY(launch_attention<T>(nw, N, 1, 0, 0, d, H, b.qkv[s], b.ao[s], st));
      cudaMemcpyAsync(b.xmid[s], x, sizeof(T) * (size_t)nt * d, cudaMemcpyDeviceToDevice, st);
      NQS_TRY(rowgemm_tc(b.ao[s], d, nt, d, tc.wo[l], d, d, bw.bo, 1, b.xmid[s], d, b.xmid[s], d,
                         tc.err, st, 0, w16(tc.wo16[l])));
      NQS_TRY(launch_layernorm<T>(nt, 1, 0, 0, d, b.xmid[s], bw.ln1_s, bw.ln1_b, b.h1[s], st));
      NQS_TRY(rowgemm_tc(b.h1[s], d, nt, d, tc.w0[l], D, D, bw.b0, 1, nullptr, 0, b.a0[s], D,
                         tc.err, st, 0, w16(tc.w016[l])));
      cudaMemcpyAsync(b.g0[s], b.a0[s], sizeof(T) * (size_t)nt * D, cudaMemcpyDeviceToDevice, st);
      const size_t nel = (size_t)nt * D;
      k_gelu<T><<<(unsigned)((nel + 255) / 256), 256, 0, st>>>((size_t)nt, 1, 0, 0, D, b.g0[s]);
      NQS_CHECK_LAUNCH("k_gelu");
      if (y) {
        cudaMemcpyAsync(y, b.xmid[s], sizeof(T) * (size_t)nt * d, cudaMemcpyDeviceToDevice, st);
        NQS_TRY(rowgemm_tc(b.g0[s], D, nt, D, tc.w1[l], d, d, bw.b1, 1, y, d, y, d, tc.err, st, 0,
                           w16(tc.w116[l])));
      }
      return NQS_OK;
    }
  }
  GemmArgs<T> g{};
  g.X = b.h0[s]; g.ldx = d; g.rows = nt; g.K = d; g.C = 1;
  g.Y = b.qkv[s]; g.ldy = 3 * d; g.nseg = 3;
  g.seg[0] = GemmSeg<T>{bw.wq, bw.bq, d, d, 0, 0};
  g.seg[1] = GemmSeg<T>{bw.wk, bw.bk, d, d, d, 0};
  g.seg[2] = GemmSeg<T>{bw.wv, bw.bv, d, d, 2 * d, 0};
  NQS_TRY(launch_gemm<T>(g, st));
  NQS_TRY(launch_attention<T>(nw, N, 1, 0, 0, d, H, b.qkv[s], b.ao[s], st));
  g = GemmArgs<T>{};
  g.X = b.ao[s]; g.ldx = d; g.rows = nt; g.K = d; g.C = 1;
  g.Y = b.xmid[s]; g.ldy = d; g.Res = x; g.ldr = d; g.nseg = 1;
  g.seg[0] = GemmSeg<T>{bw.wo, bw.bo, d, d, 0, 0};
  NQS_TRY(launch_gemm<T>(g, st));
  NQS_TRY(launch_layernorm<T>(nt, 1, 0, 0, d, b.xmid[s], bw.ln1_s, bw.ln1_b, b.h1[s], st));
  g = GemmArgs<T>{};
  g.X = b.h1[s]; g.ldx = d; g.rows = nt; g.K = d; g.C = 1;
  g.Y = b.a0[s]; g.ldy = D; g.nseg = 1;
  g.seg[0] = GemmSeg<T>{bw.w0, bw.b0, D, D, 0, 0};
  NQS_TRY(launch_gemm<T>(g, st));
  cudaMemcpyAsync(b.g0[s], b.a0[s], sizeof(T) * (size_t)nt * D, cudaMemcpyDeviceToDevice, st);
  const size_t nel = (size_t)nt * D;
  k_gelu<T><<<(unsigned)((nel + 255) / 256), 256, 0, st>>>((size_t)nt, 1, 0, 0, D, b.g0[s]);
  NQS_CHECK_LAUNCH("k_gelu");
  if (y) {
    g = GemmArgs<T>{};
    g.X = b.g0[s]; g.ldx = D; g.rows = nt; g.K = D; g.C = 1;
    g.Y = y; g.ldy = d; g.Res = b.xmid[s]; g.ldr = d;
    g.nseg = 1;
    g.seg[0] = GemmSeg<T>{bw.w1, bw.b1, d, d, 0, 0};
    NQS_TRY(launch_gemm<T>(g, st));
  }
  return NQS_OK;
}

template <typename T, class Wr>
static int backward_run(const HostModel& hm, const NetW<T>& w, const HeadParams& hp,
                        const double* R, const int32_t* S, int W, const Wr& wr, bool ckpt,
                        Arena& ws, cudaStream_t st) {
  const ModelConst& mc = hm.mc;
  const NqsModelDesc& dsc = hm.desc;
  const int N = mc.N, d = mc.d, D = mc.ff * d, KN = mc.K * N, H = mc.H;
  const int Fp = 4 * mc.nf + 2;
  const int nwc = (int)bwd_chunk_walkers<T>(mc, W, ckpt);
  const size_t rows = (size_t)nwc * N;
  const size_t save = ws.used;
  SaveBufs<T> b{};
  for (int l = 0; l < mc.depth; ++l) {
    b.xin[l] = ws.take<T>(rows * d);
    if (ckpt && l > 0) continue;
    b.h0[l] = ws.take<T>(rows * d);
    b.qkv[l] = ws.take<T>(rows * 3 * d);
    b.ao[l] = ws.take<T>(rows * d);
    b.xmid[l] = ws.take<T>(rows * d);
    b.h1[l] = ws.take<T>(rows * d);
    b.a0[l] = ws.take<T>(rows * D);
    b.g0[l] = ws.take<T>(rows * D);
  }
  b.xL = ws.take<T>(rows * d);
  b.hf = ws.take<T>(rows * d);
  b.bf = ws.take<T>(rows * 2 * KN);
  b.feat = ws.take<T>(rows * Fp);
  b.xb = ws.take<T>(rows * 2 * d);
  b.hb = ws.take<T>(rows * 2 * d);
  b.big = ws.take<T>(rows * std::max({6 * d, 2 * D, 2 * KN}));
  b.X1 = ws.take<T>(rows * 2 * KN);
  b.X2 = ws.take<T>(rows * 2 * KN);
  if (!b.X2) {
    set_error("workspace too small for the reverse pass");
    return NQS_ERR_WORKSPACE;
  }
  const size_t hsm = head_bwd_smem(N, mc.nG, mc.K, mc.learnable_env);
  const size_t absm = sizeof(T) * (size_t)(5 * N * (d / H) + 2 * N * N + N);
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_head_bwd<T, T, Wr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         220 * 1024);
    cudaFuncSetAttribute(k_attn_bwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    cudaFuncSetAttribute(k_ln_bwd<T, Wr>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr = true;
  }
  const HeadOffsets hoff{dsc.off_det_logw, dsc.off_jas_c_same, dsc.off_jas_c_opp,
                         dsc.off_jastrow_loga, dsc.off_dW};
  for (int w0 = 0; w0 < W; w0 += nwc) {
    const int nw = std::min(nwc, W - w0);
    const int nt = nw * N;
    JobBatch jb{JOB_VALUE, nw, N, 1, 0, 0, w0, R, S, nullptr};
    // ---------------- forward, keeping what the reverse pass needs ----------------
    k_embed<T><<<(nt + 7) / 8, 256, 0, st>>>(jb, mc, w.emb_w, w.emb_b, mc.depth ? b.xin[0] : b.xL);
    NQS_CHECK_LAUNCH("k_embed");
    for (int l = 0; l < mc.depth; ++l)
      NQS_TRY(block_forward<T>(mc, w.blk[l], w.tc, b, l, ckpt ? 0 : l, nw,
                               (l + 1 < mc.depth) ? b.xin[l + 1] : b.xL, st));
    NQS_TRY(launch_layernorm<T>(nt, 1, 0, 0, d, b.xL, w.lnf_s, w.lnf_b, b.hf, st));
    bool bf_done = false;
    if constexpr (sizeof(T) == 4) {
      if (w.tc.on) {
        NQS_TRY(rowgemm_tc(b.hf, d, nt, d, w.tc.wbf, w.tc.npad_bf, 2 * KN, w.bf_b_re, 1, nullptr,
                           0, b.bf, 2 * KN, w.tc.err, st, 0, w.tc.bf16 ? w.tc.wbf16 : nullptr));
        bf_done = true;
      }
    }
    if (!bf_done) {
      GemmArgs<T> g{};
      g.X = b.hf; g.ldx = d; g.rows = nt; g.K = d; g.C = 1;
      g.Y = b.bf; g.ldy = 2 * KN; g.nseg = 2;
      g.seg[0] = GemmSeg<T>{w.bf_w_re, w.bf_b_re, KN, KN, 0, 0};
      g.seg[1] = GemmSeg<T>{w.bf_w_im, w.bf_b_im, KN, KN, KN, 0};
      NQS_TRY(launch_gemm<T>(g, st));
    }
    // ---------------- reverse ----------------
    k_head_bwd<T, T, Wr><<<nw, 256, hsm, st>>>(jb, mc, b.bf, 2 * KN, hp, b.X1, b.X2, wr, hoff);
    NQS_CHECK_LAUNCH("k_head_bwd");
    // backflow: hbar = X1 Wr^T + X2 Wi^T ; the complex kernel / bias
    {
      GemmArgs<T> g{};
      g.X = b.X1; g.ldx = KN; g.rows = 2 * nt; g.K = KN; g.C = 2; g.trans_w = 1;
      g.Y = b.hb; g.ldy = d; g.nseg = 1;
      g.seg[0] = GemmSeg<T>{w.bf_w_re, nullptr, KN, d, 0, 0};
      NQS_TRY(gemm_wt<T>(g, w.tc, st));
      g.X = b.X2; g.Res = b.hb; g.ldr = d;
      g.seg[0] = GemmSeg<T>{w.bf_w_im, nullptr, KN, d, 0, 0};
      NQS_TRY(gemm_wt<T>(g, w.tc, st));
    }
    NQS_TRY(wgrad<T>(wr, nw, N, d, KN, b.hf, d, b.X1, KN, w0, dsc.off_backflow_kernel,
                     dsc.off_backflow_bias, 1, st));
    // final LayerNorm
    k_ln_bwd<T, Wr><<<nw, 256, sizeof(T) * (size_t)N * d, st>>>(
        N, d, b.xL, b.hb, w.lnf_s, b.xb, 0, wr, w0, dsc.off_final_ln_scale,
        dsc.off_final_ln_bias);
    NQS_CHECK_LAUNCH("k_ln_bwd");
    for (int l = mc.depth - 1; l >= 0; --l) {
      const BlockW<T>& bw = w.blk[l];
      const int64_t* of = dsc.off_block[l];
      const int s = ckpt ? 0 : l;
      if (ckpt) NQS_TRY(block_forward<T>(mc, bw, w.tc, b, l, 0, nw, nullptr, st));  // recompute
      // MLP: x_out = xmid + g0 W1 + b1
      GemmArgs<T> g{};
      g.X = b.xb; g.ldx = d; g.rows = 2 * nt; g.K = d; g.C = 2; g.trans_w = 1;
      g.Y = b.big; g.ldy = D; g.nseg = 1;
      g.seg[0] = GemmSeg<T>{bw.w1, nullptr, d, D, 0, 0};
      NQS_TRY(gemm_wt<T>(g, w.tc, st));  // gbar0 = xbar W1^T
      NQS_TRY(wgrad<T>(wr, nw, N, D, d, b.g0[s], D, b.xb, d, w0, of[NQS_B_DENSE1_KERNEL],
                       of[NQS_B_DENSE1_BIAS], 0, st));
      const size_t nel = (size_t)nt * D;
      k_gelu_bwd<T><<<(unsigned)((nel + 255) / 256), 256, 0, st>>>((size_t)nt, D, b.a0[s], b.big);
      NQS_CHECK_LAUNCH("k_gelu_bwd");
      g = GemmArgs<T>{};
      g.X = b.big; g.ldx = D; g.rows = 2 * nt; g.K = D; g.C = 2; g.trans_w = 1;
      g.Y = b.hb; g.ldy = d; g.nseg = 1;
      g.seg[0] = GemmSeg<T>{bw.w0, nullptr, D, d, 0, 0};
      NQS_TRY(gemm_wt<T>(g, w.tc, st));  // hbar1 = abar0 W0^T
      NQS_TRY(wgrad<T>(wr, nw, N, d, D, b.h1[s], d, b.big, D, w0, of[NQS_B_DENSE0_KERNEL],
                       of[NQS_B_DENSE0_BIAS], 0, st));
      k_ln_bwd<T, Wr><<<nw, 256, sizeof(T) * (size_t)N * d, st>>>(
          N, d, b.xmid[s], b.hb, bw.ln1_s, b.xb, 1, wr, w0, of[NQS_B_LN1_SCALE],
          of[NQS_B_LN1_BIAS]);
      NQS_CHECK_LAUNCH("k_ln_bwd");
      // attention: xmid = xin + ao Wo + bo
      g = GemmArgs<T>{};
      g.X = b.xb; g.ldx = d; g.rows = 2 * nt; g.K = d; g.C = 2; g.trans_w = 1;
      g.Y = b.hb; g.ldy = d; g.nseg = 1;
      g.seg[0] = GemmSeg<T>{bw.wo, nullptr, d, d, 0, 0};
      NQS_TRY(gemm_wt<T>(g, w.tc, st));  // aobar
      NQS_TRY(wgrad<T>(wr, nw, N, d, d, b.ao[s], d, b.xb, d, w0, of[NQS_B_O_KERNEL],
                       of[NQS_B_O_BIAS], 0, st));
      k_attn_bwd<T><<<nw * H, 128, absm, st>>>(N, d, H, b.qkv[s], b.hb, b.big);
      NQS_CHECK_LAUNCH("k_attn_bwd");
      // h0bar = qbar Wq^T + kbar Wk^T + vbar Wv^T
      const T* wts[3] = {bw.wq, bw.wk, bw.wv};
      for (int q = 0; q < 3; ++q) {
        g = GemmArgs<T>{};
        g.X = b.big + q * d; g.ldx = 3 * d; g.rows = 2 * nt; g.K = d; g.C = 2; g.trans_w = 1;
        g.Y = b.hb; g.ldy = d; g.Res = q ? b.hb : nullptr; g.ldr = d; g.nseg = 1;
        g.seg[0] = GemmSeg<T>{wts[q], nullptr, d, d, 0, 0};
        NQS_TRY(gemm_wt<T>(g, w.tc, st));
      }
      const int kk[3] = {NQS_B_Q_KERNEL, NQS_B_K_KERNEL, NQS_B_V_KERNEL};
      const int kb[3] = {NQS_B_Q_BIAS, NQS_B_K_BIAS, NQS_B_V_BIAS};
      for (int q = 0; q < 3; ++q)
        NQS_TRY(wgrad<T>(wr, nw, N, d, d, b.h0[s], d, b.big + q * d, 3 * d, w0, of[kk[q]],
                         of[kb[q]], 0, st));
      k_ln_bwd<T, Wr><<<nw, 256, sizeof(T) * (size_t)N * d, st>>>(
          N, d, b.xin[l], b.hb, bw.ln0_s, b.xb, 1, wr, w0, of[NQS_B_LN0_SCALE],
          of[NQS_B_LN0_BIAS]);
      NQS_CHECK_LAUNCH("k_ln_bwd");
    }
    // embedding
    k_features<T><<<(nt * Fp + 255) / 256, 256, 0, st>>>(jb, mc, b.feat);
    NQS_CHECK_LAUNCH("k_features");
    NQS_TRY(wgrad<T>(wr, nw, N, Fp, d, b.feat, Fp, b.xb, d, w0, dsc.off_embed_kernel,
                     dsc.off_embed_bias, 0, st));
  }
  ws.used = save;
  return NQS_OK;
}

// a tensor-core GEMM of the pass that gave up a bounded wait recorded it in *err: the result is
// then incomplete, and its first entry becomes NaN so that the caller sees it
template <typename X>
__global__ void k_poison_first_on_timeout(const int* __restrict__ err, X* p) {
  if (*err) p[0] = (X)NAN;
}

template <typename T, typename TO>
int per_sample_O_run(const HostModel& hm, const NetW<T>& w, const HeadParams& hp,
                     const double* R, const int32_t* S, int W, TO* O, bool ckpt, Arena& ws,
                     cudaStream_t st) {
  const ORows<TO> orows{O, hm.desc.n_params, W};
  NQS_TRY(backward_run<T, ORows<TO>>(hm, w, hp, R, S, W, orows, ckpt, ws, st));
  if (w.tc.on && w.tc.err) {
    k_poison_first_on_timeout<TO><<<1, 1, 0, st>>>(w.tc.err, O);
    NQS_CHECK_LAUNCH("k_poison_first_on_timeout");
  }
  return NQS_OK;
}

template <typename T>
int logpsi_vjp_run(const HostModel& hm, const NetW<T>& w, const HeadParams& hp,
                   const double* R, const int32_t* S, int W, const cplx* ct, double* grad,
                   bool ckpt, Arena& ws, cudaStream_t st) {
  const cudaError_t e = cudaMemsetAsync(grad, 0, sizeof(double) * hm.desc.n_params, st);
  if (e != cudaSuccess) return cuda_status(e, "nqs_logpsi_vjp: clear");
  const VjpAcc acc{grad, ct};
  NQS_TRY(backward_run<T, VjpAcc>(hm, w, hp, R, S, W, acc, ckpt, ws, st));
  if (w.tc.on && w.tc.err) {
    k_poison_first_on_timeout<double><<<1, 1, 0, st>>>(w.tc.err, grad);
    NQS_CHECK_LAUNCH("k_poison_first_on_timeout");
  }
  return NQS_OK;
}

template size_t backward_scratch<double>(const ModelConst&, int, bool);
template size_t backward_scratch<float>(const ModelConst&, int, bool);
template size_t per_sample_O_scratch<double>(const ModelConst&, int);
template size_t per_sample_O_scratch<float>(const ModelConst&, int);
template int per_sample_O_run<double, double>(const HostModel&, const NetW<double>&,
                                              const HeadParams&, const double*, const int32_t*,
                                              int, double*, bool, Arena&, cudaStream_t);
template int per_sample_O_run<float, float>(const HostModel&, const NetW<float>&,
                                            const HeadParams&, const double*, const int32_t*, int,
                                            float*, bool, Arena&, cudaStream_t);
template int per_sample_O_run<float, double>(const HostModel&, const NetW<float>&,
                                             const HeadParams&, const double*, const int32_t*,
                                             int, double*, bool, Arena&, cudaStream_t);
template int per_sample_O_run<double, float>(const HostModel&, const NetW<double>&,
                                             const HeadParams&, const double*, const int32_t*,
                                             int, float*, bool, Arena&, cudaStream_t);
template int logpsi_vjp_run<double>(const HostModel&, const NetW<double>&, const HeadParams&,
                                    const double*, const int32_t*, int, const cplx*, double*,
                                    bool, Arena&, cudaStream_t);
template int logpsi_vjp_run<float>(const HostModel&, const NetW<float>&, const HeadParams&,
                                   const double*, const int32_t*, int, const cplx*, double*,
                                   bool, Arena&, cudaStream_t);

}  // namespace nqs
