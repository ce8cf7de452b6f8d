// ewald.cu — 2D Ewald Coulomb energy on a general periodic cell (float64).
//
// Reference: src/nqs/ewald.py:26-73. For one configuration
//   E_C = sum_{i<j} alpha [ sum_img erfc(eta|r_ij + R|)/|r_ij + R|
//                           + sum_G RECIP(G) cos(G.r_ij) + V_G0 ] + N zeta_M / 2,
// images R = A n (|n_x|,|n_y| <= n_real), G = B m over the square index box (m != 0),
// RECIP(G) = (2 pi/area) erfc(|G|/2eta)/|G|, V_G0 = -2 sqrt(pi)/(area eta).
// The reciprocal pair sum is evaluated through the structure factor
//   sum_{i<j} cos(G.r_ij) = (|S(G)|^2 - N)/2,  S(G) = sum_i exp(i G.r_i)
// (algebraically identical, N*nG instead of N^2*nG/2 sincos). The real-space part is a
// warp-strided sum over (pair, image); all partial sums are compensated (TwoSum).
#include <cstdio>
#include <cstdlib>
#include <vector>
#include <cmath>

#include "nqs_common.cuh"

struct NqsEwald {
  double A[4], Ainv[4];
  double alpha, eta, area, V_G0, zeta_M;
  int n_img, n_G;
  double* d_img;    // [n_img][2]
  double* d_G;      // [n_G][2]
  double* d_recip;  // [n_G]
};

namespace nqs {

// Knuth TwoSum accumulation
struct KSum {
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double x) {
    const double t = s + x;
    const double bp = t - s;
    c += (s - (t - bp)) + (x - bp);
    s = t;
  }
  __device__ __forceinline__ double value() const { return s + c; }
};

__device__ double block_sum_kahan(double s, double c, double* red) {
  // reduce (s, c) pairs across the block with TwoSum at each step
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  KSum k;
  k.s = s;
  k.c = c;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const double os = __shfl_xor_sync(0xffffffffu, k.s, o);
    const double oc = __shfl_xor_sync(0xffffffffu, k.c, o);
    k.add(os);
    k.c += oc;
  }
  __syncthreads();
  if (lane == 0) {
    red[2 * wid] = k.s;
    red[2 * wid + 1] = k.c;
  }
  __syncthreads();
  double out = 0.0;
  if (threadIdx.x == 0) {
    KSum t;
    for (int w = 0; w < nw; ++w) {
      t.add(red[2 * w]);
      t.c += red[2 * w + 1];
    }
    red[0] = t.value();
  }
  __syncthreads();
  out = red[0];
  __syncthreads();
  return out;
}

// one CTA per walker
__global__ void __launch_bounds__(256) k_ewald_energy(NqsEwald ew, const double* __restrict__ R,
                                                      int n_walkers, int N,
                                                      double* __restrict__ out) {
  const int w = blockIdx.x;
  extern __shared__ double sm[];
  double* rx = sm;
  double* ry = rx + N;
  double* red = ry + N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    rx[i] = R[((size_t)w * N + i) * 2];
    ry[i] = R[((size_t)w * N + i) * 2 + 1];
  }
  __syncthreads();
  KSum acc;
  // real space: (pair, image)
  const int npair = N * (N - 1) / 2;
  const long long tot = (long long)npair * ew.n_img;
  for (long long idx = threadIdx.x; idx < tot; idx += blockDim.x) {
    const int p = (int)(idx / ew.n_img), m = (int)(idx - (long long)p * ew.n_img);
    // pair index p -> (i, j), i < j (row-major upper triangle)
    int i = 0, rem = p;
    while (rem >= N - 1 - i) {
      rem -= N - 1 - i;
      ++i;
    }
    const int j = i + 1 + rem;
    const double dx = rx[i] - rx[j] + ew.d_img[2 * m];
    const double dy = ry[i] - ry[j] + ew.d_img[2 * m + 1];
    const double d = sqrt(dx * dx + dy * dy);
    acc.add(erfc(ew.eta * d) / d);
  }
  // reciprocal space via the structure factor
  for (int g = threadIdx.x; g < ew.n_G; g += blockDim.x) {
    const double gx = ew.d_G[2 * g], gy = ew.d_G[2 * g + 1];
    KSum sr, si;
    for (int i = 0; i < N; ++i) {
      double s, c;
      sincos(gx * rx[i] + gy * ry[i], &s, &c);
      sr.add(c);
      si.add(s);
    }
    const double a = sr.value(), b = si.value();
    acc.add(ew.d_recip[g] * 0.5 * ((a * a + b * b) - (double)N));
  }
  const double tot_sum = block_sum_kahan(acc.s, acc.c, red);
  if (threadIdx.x == 0) {
    KSum e;
    e.add(ew.alpha * tot_sum);
    e.add(ew.alpha * ew.V_G0 * (double)npair);
    e.add((double)N * ew.zeta_M / 2.0);
    out[w] = e.value();
  }
}

// one thread per displacement vector
__global__ void k_ewald_pair(NqsEwald ew, const double* __restrict__ r, int M,
                             double* __restrict__ out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= M) return;
  const double x = r[2 * t], y = r[2 * t + 1];
  KSum re, rc;
  for (int m = 0; m < ew.n_img; ++m) {
    const double dx = x + ew.d_img[2 * m], dy = y + ew.d_img[2 * m + 1];
    const double d = sqrt(dx * dx + dy * dy);
    re.add(erfc(ew.eta * d) / d);
  }
  for (int g = 0; g < ew.n_G; ++g) rc.add(ew.d_recip[g] * cos(ew.d_G[2 * g] * x + ew.d_G[2 * g + 1] * y));
  out[t] = ew.alpha * (re.value() + rc.value() + ew.V_G0);
}

}  // namespace nqs

extern "C" {

int nqs_ewald_create(const double A_in[4], double alpha, double ewald_alpha, int n_real,
                     int n_recip, NqsEwald** out) {
  if (!A_in || !out || n_real < 0 || n_recip < 1) {
    nqs::set_error("nqs_ewald_create: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  NqsEwald e{};
  for (int i = 0; i < 4; ++i) e.A[i] = A_in[i];
  const double det = e.A[0] * e.A[3] - e.A[1] * e.A[2];
  if (det == 0.0) {
    nqs::set_error("nqs_ewald_create: singular cell");
    return NQS_ERR_INVALID_ARG;
  }
  e.Ainv[0] = e.A[3] / det;
  e.Ainv[1] = -e.A[1] / det;
  e.Ainv[2] = -e.A[2] / det;
  e.Ainv[3] = e.A[0] / det;
  e.area = std::fabs(det);
  e.eta = ewald_alpha > 0 ? ewald_alpha : std::sqrt(M_PI) / std::sqrt(e.area);
  e.alpha = alpha;
  // B = 2 pi A^-T : B[r][c] = 2 pi Ainv[c][r]
  const double B[4] = {2 * M_PI * e.Ainv[0], 2 * M_PI * e.Ainv[2], 2 * M_PI * e.Ainv[1],
                       2 * M_PI * e.Ainv[3]};
  std::vector<double> img, G, rec;
  for (int nx = -n_real; nx <= n_real; ++nx)
    for (int ny = -n_real; ny <= n_real; ++ny) {
      img.push_back(e.A[0] * nx + e.A[1] * ny);
      img.push_back(e.A[2] * nx + e.A[3] * ny);
    }
  for (int mx = -n_recip; mx <= n_recip; ++mx)
    for (int my = -n_recip; my <= n_recip; ++my) {
      if (mx == 0 && my == 0) continue;
      const double gx = B[0] * mx + B[1] * my, gy = B[2] * mx + B[3] * my;
      G.push_back(gx);
      G.push_back(gy);
      const double gm = std::sqrt(gx * gx + gy * gy);
      rec.push_back((2.0 * M_PI / e.area) * std::erfc(gm / (2.0 * e.eta)) / gm);
    }
  e.n_img = (int)img.size() / 2;
  e.n_G = (int)G.size() / 2;
  e.V_G0 = -2.0 * std::sqrt(M_PI) / (e.area * e.eta);
  // Madelung constant (ewald.py:53-58)
  double real_nz = 0.0, rsum = 0.0;
  for (int m = 0; m < e.n_img; ++m) {
    const double d = std::sqrt(img[2 * m] * img[2 * m] + img[2 * m + 1] * img[2 * m + 1]);
    if (d > 1e-10) real_nz += std::erfc(e.eta * d) / d;
  }
  for (double v : rec) rsum += v;
  e.zeta_M = alpha * (real_nz + (-2.0 * e.eta / std::sqrt(M_PI)) + rsum + e.V_G0);
  cudaError_t ce;
  if ((ce = cudaMalloc(&e.d_img, img.size() * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&e.d_G, G.size() * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&e.d_recip, rec.size() * sizeof(double))) != cudaSuccess)
    return nqs::cuda_status(ce, "nqs_ewald_create: cudaMalloc");
  cudaMemcpy(e.d_img, img.data(), img.size() * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(e.d_G, G.data(), G.size() * sizeof(double), cudaMemcpyHostToDevice);
  if ((ce = cudaMemcpy(e.d_recip, rec.data(), rec.size() * sizeof(double),
                       cudaMemcpyHostToDevice)) != cudaSuccess)
    return nqs::cuda_status(ce, "nqs_ewald_create: cudaMemcpy");
  *out = new NqsEwald(e);
  return NQS_OK;
}

int nqs_ewald_destroy(NqsEwald* e) {
  if (!e) return NQS_OK;
  cudaFree(e->d_img);
  cudaFree(e->d_G);
  cudaFree(e->d_recip);
  delete e;
  return NQS_OK;
}

int nqs_ewald_zeta(const NqsEwald* e, double* z) {
  if (!e || !z) return NQS_ERR_INVALID_ARG;
  *z = e->zeta_M;
  return NQS_OK;
}

int nqs_ewald_pair(const NqsEwald* e, const double* r, int M, double* out, void* stream) {
  if (!e || (M > 0 && (!r || !out)) || M < 0) return NQS_ERR_INVALID_ARG;
  if (M == 0) return NQS_OK;
  nqs::k_ewald_pair<<<(M + 127) / 128, 128, 0, (cudaStream_t)stream>>>(*e, r, M, out);
  NQS_CHECK_LAUNCH("k_ewald_pair");
  return NQS_OK;
}

int nqs_ewald_energy(const NqsEwald* e, const double* R, int W, int N, double* out,
                     void* stream) {
  if (!e || W < 0 || N < 1 || (W > 0 && (!R || !out))) return NQS_ERR_INVALID_ARG;
  if (N > 4096) return NQS_ERR_UNSUPPORTED;
  if (W == 0) return NQS_OK;
  const size_t sm = (2 * (size_t)N + 64) * sizeof(double);
  nqs::k_ewald_energy<<<W, 256, sm, (cudaStream_t)stream>>>(*e, R, W, N, out);
  NQS_CHECK_LAUNCH("k_ewald_energy");
  return NQS_OK;
}

}  // extern "C"
