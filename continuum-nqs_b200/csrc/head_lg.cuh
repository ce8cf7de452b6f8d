// head_lg.cuh — determinant head for more than 16 electrons: one CTA of 256 threads per job, the
// K determinants of the job one after the other, every step spread over the whole CTA.
//
// Same quantities as k_head / k_head_rt (psiformer.py:118-189: envelope, backflow-dressed
// orbitals, log-sum-exp over determinants, Jastrow; forward-mode tangents and Laplacian of
// log psi), organised for large N:
//   phase 1 (per job): positions, spins, phases e^{i G.r}, envelope env[a][i], the pair Jastrow
//     (value, per-tangent-electron gradient, Laplacian), reduced in a fixed order.
//   phase 2 (per determinant k): M[a][i] = env[a][i] (1 + b0[a][i]) in shared memory; in-place
//     Gauss-Jordan with implicit partial pivoting (largest |re| + |im| among the rows not used yet,
//     first index on ties), two barriers per column: warp 0 picks the pivot and stages the scaled
//     pivot row and the elimination column, then every thread updates its entries. Afterwards
//     storage row piv[c] holds row c of M^-1 and storage column c' belongs to orbital piv[c'].
//     Values only: the same pivots with the elimination restricted to the rows not used yet.
//     Tangents without the Laplacian: tr(M^-1 D_t) = sum_{i,c'} M^-1[i][piv c'] D_t[piv c'][i].
//     With the Laplacian: the rows are permuted once into Minv[i][c'] = M^-1[i][piv c'] and every
//     tangent is one complex GEMM of the CTA, B_t = Minv X_t with X_t[c'][j] = D_t[piv c'][j]
//     (16 x 16 threads, a TS x TS tile of B each: rows ty + 16u, columns tx + 16v, operands
//     zero-padded to 16 TS); tr B_t from the diagonal tiles and tr B_t^2 through B_t stored in
//     shared memory. Two barriers per tangent (X_t and B_t have their own buffers).
//       d_t log det M = tr B_t,  Lap log det M = tr(M^-1 Lap M) - sum_t tr B_t^2
//   phase 3 (warp 0): log-sum-exp over determinants with det_logw, Jastrow, outputs.
// D_t = d_t M = env (d_t b) + [column of the tangent electron] (d_t env) (1 + b0); Lap M adds
// env (Lap b) + (Lap env) (1 + b0) + 2 (d env).(d b) on the tangent electrons' columns. The
// envelope derivatives are summed from the phases where they are used.
#pragma once

#include "net_kernels.cuh"

namespace nqs {

constexpr int kHeadLgThreads = 256;
constexpr int kHeadLgMaxN = 64;        // values and gradients
constexpr int kHeadLgMaxNLap = 48;     // with the Laplacian (TS <= 3)

struct HeadLgLayout {
  int rows, ld;  // matrix rows (N, or 16 TS with the Laplacian) and row stride (complex)
  size_t ph, env, G, X, Y, dlk, total;
};

// mode: 0 values, 1 tangents, 2 tangents + Laplacian
__host__ __device__ inline HeadLgLayout head_lg_layout(int N, int nG, int K, int n_tan, int mode,
                                                       int ts) {
  HeadLgLayout L;
  L.rows = mode == 2 ? 16 * ts : N;
  L.ld = L.rows + 1;  // odd row stride: a column of 16-byte entries spreads over the banks
  const size_t mat = 16 * (size_t)L.rows * L.ld;
  size_t o = 0;
  L.ph = o;
  o += round128(16 * (size_t)nG * N);
  L.env = o;
  o += round128(16 * (size_t)N * L.ld);
  L.G = o;
  o += round128(mat);
  L.X = o;
  if (mode == 2) o += round128(mat);
  L.Y = o;
  if (mode == 2) o += round128(mat);
  L.dlk = o;
  o += round128(16 * (size_t)K * (mode ? n_tan : 0));
  L.total = o;
  return L;
}

inline int head_lg_ts(int N) { return (N + 15) / 16; }

// The static shared arrays of k_head_lg (bytes), for the host's fit check.
constexpr size_t kHeadLgStaticBytes = 8 * (3 * kHeadLgMaxN + 2 * kHeadLgMaxN + 4) +
                                      4 * (5 * kHeadLgMaxN + NQS_MAX_DETS + 4) +
                                      16 * (3 * NQS_MAX_DETS + 2 * kHeadLgMaxN + 2) + 8 * 64 + 256;

// four doubles summed over the CTA's 8 warps, written to red8[warp][4] by lane 0
__device__ __forceinline__ void head_lg_warp4(double (&v)[4], double (*red8)[4]) {
  warp_sum_n<double, 4>(v);
  if ((threadIdx.x & 31) == 0) {
    double* r = red8[threadIdx.x >> 5];
    r[0] = v[0];
    r[1] = v[1];
    r[2] = v[2];
    r[3] = v[3];
  }
}
// the CTA sum of the partials (fixed order), valid after a barrier
__device__ __forceinline__ void head_lg_total4(const double (*red8)[4], double (&o)[4]) {
  o[0] = o[1] = o[2] = o[3] = 0.0;
  for (int w = 0; w < kHeadLgThreads / 32; ++w)
    for (int q = 0; q < 4; ++q) o[q] += red8[w][q];
}

template <typename TIN, int MODE, int TS>
__global__ void __launch_bounds__(kHeadLgThreads, TS >= 3 ? 1 : 2) k_head_lg(JobBatch jb, ModelConst mc,
                                                            const TIN* __restrict__ BF, int ldbf,
                                                            HeadParams hp, HeadOut out,
                                                            int j_out0) {
  constexpr bool TAN = MODE >= 1, LAP = MODE == 2;
  const int N = jb.N, C = jb.C, nG = mc.nG, K = mc.K;
  const int n_tan = TAN ? jb.n_tan : 0;
  const bool has_lap = LAP && jb.has_lap;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int job = blockIdx.x;
  const HeadLgLayout lay = head_lg_layout(N, nG, K, n_tan, MODE, TS);
  const int LD = lay.ld, NR = lay.rows;
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* ph = reinterpret_cast<cplx*>(smraw + lay.ph);
  cplx* env = reinterpret_cast<cplx*>(smraw + lay.env);
  cplx* G = reinterpret_cast<cplx*>(smraw + lay.G);
  cplx* X = reinterpret_cast<cplx*>(smraw + lay.X);
  cplx* Y = reinterpret_cast<cplx*>(smraw + lay.Y);
  cplx* dlk = reinterpret_cast<cplx*>(smraw + lay.dlk);
  __shared__ double rx[kHeadLgMaxN], ry[kHeadLgMaxN], gj[2 * kHeadLgMaxN], jas[4];
  __shared__ int sp[kHeadLgMaxN], piv[kHeadLgMaxN], pinv[kHeadLgMaxN], used[kHeadLgMaxN];
  __shared__ int sing[NQS_MAX_DETS], s_p;
  __shared__ cplx s_ld[NQS_MAX_DETS], s_lapk[NQS_MAX_DETS], s_sq[NQS_MAX_DETS];
  __shared__ __align__(16) cplx prow[kHeadLgMaxN], fcol[kHeadLgMaxN];
  __shared__ double red[2][kHeadLgThreads / 32][4];

  const JobInfo ji = job_info(jb, job);
  const int te_lo = ji.tan_e0, n_te = n_tan / 2;
  auto is_te = [&](int i) { return TAN && i >= te_lo && i < te_lo + n_te; };
  auto Weff = [&](int a, int g, int s) -> cplx {
    const size_t o = ((size_t)a * nG + g) * 2 + s;
    cplx w = mk(mc.W[2 * o], mc.W[2 * o + 1]);
    if (mc.learnable_env) w = cadd(w, mk(hp.dW[o], hp.dW[(size_t)N * nG * 2 + o]));
    return w;
  };
  // ======================= phase 1: per-job tables =======================
  for (int i = tid; i < N; i += kHeadLgThreads) {
    const double* r = jb.R + ((size_t)ji.walker * N + i) * 2;
    rx[i] = r[0];
    ry[i] = r[1];
    sp[i] = job_spin(jb, ji, i);
  }
  __syncthreads();
  for (int idx = tid; idx < nG * N; idx += kHeadLgThreads) {
    const int g = idx / N, i = idx - g * N;
    double sn, cs;
    sincos(mc.Gs[2 * g] * rx[i] + mc.Gs[2 * g + 1] * ry[i], &sn, &cs);
    ph[idx] = mk(cs, sn);
  }
  __syncthreads();
  for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
    const int a = idx / N, i = idx - a * N;
    const int s = sp[i];
    cplx e = mk(0, 0);
    for (int g = 0; g < nG; ++g) cfma(e, ph[g * N + i], Weff(a, g, s));
    env[a * LD + i] = e;
  }
  if (LAP) {  // padding columns of the tangent staging buffer stay zero for the whole job
    for (int idx = tid; idx < N * (NR - N); idx += kHeadLgThreads) {
      const int r = idx / (NR - N), j = N + idx % (NR - N);
      G[r * LD + j] = mk(0, 0);
    }
  }
  // Jastrow: value over pairs, Laplacian and gradient per tangent electron (thread = (tangent
  // electron, group of 4 partners)); every sum in a fixed order
  if (mc.use_jastrow) {
    double v[4] = {0.0, 0.0, 0.0, 0.0};
    const int npair = N * (N - 1) / 2;
    for (int p = tid; p < npair; p += kHeadLgThreads) {
      int i = 0, rem = p;
      while (rem >= N - 1 - i) {
        rem -= N - 1 - i;
        ++i;
      }
      const int jj = i + 1 + rem;
      double dx, dy;
      min_image(mc, rx[i] - rx[jj], ry[i] - ry[jj], &dx, &dy);
      const double r = sqrt(dx * dx + dy * dy + 1e-12);
      double u, u1, u2;
      jastrow_u(mc, hp, r, sp[i] == sp[jj], &u, &u1, &u2);
      v[0] += u;
    }
    for (int base = 0; base < n_te; base += kHeadLgThreads / 4) {
      const int e = te_lo + base + (tid >> 2), g4 = tid & 3;
      const bool has_e = base + (tid >> 2) < n_te;
      double gx = 0.0, gy = 0.0, le = 0.0;
      if (has_e) {
        for (int jj = g4; jj < N; jj += 4) {
          if (jj == e) continue;
          double dx, dy;
          min_image(mc, rx[e] - rx[jj], ry[e] - ry[jj], &dx, &dy);
          const double d2 = dx * dx + dy * dy;
          const double r = sqrt(d2 + 1e-12);
          double u, u1, u2;
          jastrow_u(mc, hp, r, sp[e] == sp[jj], &u, &u1, &u2);
          gx += u1 * dx / r;
          gy += u1 * dy / r;
          le += u2 * d2 / (r * r) + u1 * (2.0 / r - d2 / (r * r * r));
        }
      }
      gx += __shfl_xor_sync(0xffffffffu, gx, 1);
      gx += __shfl_xor_sync(0xffffffffu, gx, 2);
      gy += __shfl_xor_sync(0xffffffffu, gy, 1);
      gy += __shfl_xor_sync(0xffffffffu, gy, 2);
      le += __shfl_xor_sync(0xffffffffu, le, 1);
      le += __shfl_xor_sync(0xffffffffu, le, 2);
      if (g4 == 0 && has_e) {
        gj[e - te_lo] = gx;
        gj[kHeadLgMaxN + e - te_lo] = gy;
        v[1] += le;
      }
    }
    head_lg_warp4(v, red[0]);
    __syncthreads();
    if (tid == 0) {
      double o[4];
      head_lg_total4(red[0], o);
      jas[0] = o[0];
      jas[1] = o[1];
    }
  }
  __syncthreads();
  // ======================= phase 2: the determinants =======================
  const int ty = tid >> 4, tx = tid & 15;
  for (int k = 0; k < K; ++k) {
    // bf(c, a, i): backflow channel c of orbital a (det k) at electron i; a is contiguous
    auto bf = [&](int c, int a, int i) -> cplx {
      const TIN* p = BF + (((size_t)job * N + i) * C + c) * ldbf;
      return mk((double)p[k * N + a], (double)p[K * N + k * N + a]);
    };
    // d env[a][e] / d r_e (axis bax) and its Laplacian, summed from the phases
    auto denv = [&](int a, int e, int bax) -> cplx {
      cplx d = mk(0, 0);
      const int s = sp[e];
      for (int g = 0; g < nG; ++g)
        cfma(d, cmul(ph[g * N + e], Weff(a, g, s)), mk(0, mc.Gs[2 * g + bax]));
      return d;
    };
    for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
      const int i = idx / N, a = idx - i * N;
      const cplx b0 = bf(0, a, i);
      G[a * LD + i] = cmul(env[a * LD + i], mk(1.0 + b0.re, b0.im));
    }
    for (int r = tid; r < N; r += kHeadLgThreads) used[r] = 0;
    __syncthreads();
    // ---- elimination (warp 0 keeps the pivot product) ----
    cplx prod = mk(1.0, 0.0);
    int pexp = 0, sg = 0;
#pragma unroll 1
    for (int c = 0; c < N; ++c) {
      if (warp == 0) {
        const int r0 = lane, r1 = lane + 32;
        const bool u0 = r0 >= N || used[r0], u1 = r1 >= N || used[r1];
        // |re| + |im| with NaN read as 0: the winner is always a row not used yet
        auto mag = [](cplx z) {
          const double v = cabs1(z);
          return v >= 0.0 ? v : 0.0;
        };
        double best = u0 ? -1.0 : mag(G[r0 * LD + c]);
        int bi = r0;
        if (!u1) {
          const double v1 = mag(G[r1 * LD + c]);
          if (v1 > best) {
            best = v1;
            bi = r1;
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
        const int p = bi;
        const cplx pv = G[p * LD + c];
        const bool zero = pv.re == 0.0 && pv.im == 0.0;
        const cplx ipv = zero ? mk(0.0, 0.0) : cdiv(mk(1.0, 0.0), pv);
        if (zero) {
          sg = 1;
        } else {
          prod = cmul(prod, pv);
          int ex;
          frexp(fmax(fabs(prod.re), fabs(prod.im)), &ex);
          prod = mk(ldexp(prod.re, -ex), ldexp(prod.im, -ex));
          pexp += ex;
        }
        if (TAN) {
          for (int j = lane; j < N; j += 32) prow[j] = cmul(j == c ? mk(1.0, 0.0) : G[p * LD + j], ipv);
          for (int r = lane; r < N; r += 32) fcol[r] = r == p ? mk(0.0, 0.0) : G[r * LD + c];
        } else {
          for (int j = lane; j < N; j += 32) prow[j] = G[p * LD + j];
          if (r0 < N) fcol[r0] = (!u0 && r0 != p) ? cmul(G[r0 * LD + c], ipv) : mk(0.0, 0.0);
          if (r1 < N) fcol[r1] = (!u1 && r1 != p) ? cmul(G[r1 * LD + c], ipv) : mk(0.0, 0.0);
        }
        __syncwarp();
        if (lane == 0) {
          piv[c] = p;
          used[p] = 1;
          s_p = p;
        }
      }
      __syncthreads();
      const int p = s_p;
      if (TAN) {
        for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
          const int r = idx / N, j = idx - r * N;
          cplx v;
          if (r == p) {
            v = prow[j];
          } else {
            v = j == c ? mk(0.0, 0.0) : G[r * LD + j];
            const cplx f = fcol[r];
            v = csub(v, cmul(f, prow[j]));
          }
          G[r * LD + j] = v;
        }
      } else {
        const int w = N - c - 1;  // columns c + 1 .. N - 1 of the rows not used yet
        for (int idx = tid; idx < N * w; idx += kHeadLgThreads) {
          const int r = idx / w, j = c + 1 + (idx - r * w);
          const cplx f = fcol[r];
          if (f.re != 0.0 || f.im != 0.0) G[r * LD + j] = csub(G[r * LD + j], cmul(f, prow[j]));
        }
      }
      __syncthreads();
    }
    // ---- log det: pivot product and the parity of the pivot order (warp 0) ----
    if (warp == 0) {
      int inv_cnt = 0;
      for (int c = lane; c < N; c += 32)
        for (int c2 = c + 1; c2 < N; ++c2)
          if (piv[c] > piv[c2]) ++inv_cnt;
      inv_cnt = warp_sum(inv_cnt);
      if (inv_cnt & 1) prod = mk(-prod.re, -prod.im);
      if (lane == 0) {
        s_ld[k] = sg ? mk(-INFINITY, 0.0)
                     : mk(log(hypot(prod.re, prod.im)) + pexp * 0.6931471805599453,
                          atan2(prod.im, prod.re));
        sing[k] = sg;
        s_lapk[k] = mk(0, 0);
        s_sq[k] = mk(0, 0);
      }
    }
    if (!TAN) continue;  // the next determinant's first barrier orders s_ld / sing
    // ---- tangents (also for singular matrices, whose results phase 3 discards) ----
    if (!LAP) {
      // tr(M^-1 D_t) for the two axes of each tangent electron in one pass over (i, c')
      for (int et = 0; et < n_te; ++et) {
        const int e = te_lo + et;
        double v[4] = {0.0, 0.0, 0.0, 0.0};
        for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
          const int i = idx / N, c2 = idx - i * N;
          const int a = piv[c2];
          const cplx m = G[piv[i] * LD + c2];
          const cplx en = env[a * LD + i];
          cplx dx = cmul(en, bf(1 + 2 * et, a, i)), dy = cmul(en, bf(2 + 2 * et, a, i));
          if (i == e) {
            const cplx b0 = bf(0, a, e), w1 = mk(1.0 + b0.re, b0.im);
            dx = cadd(dx, cmul(denv(a, e, 0), w1));
            dy = cadd(dy, cmul(denv(a, e, 1), w1));
          }
          const cplx tx_ = cmul(m, dx), ty_ = cmul(m, dy);
          v[0] += tx_.re;
          v[1] += tx_.im;
          v[2] += ty_.re;
          v[3] += ty_.im;
        }
        head_lg_warp4(v, red[et & 1]);
        __syncthreads();
        if (tid == 0) {
          double o[4];
          head_lg_total4(red[et & 1], o);
          const cplx tx_ = mk(o[0], o[1]), ty_ = mk(o[2], o[3]);
          dlk[k * n_tan + 2 * et] = tx_;
          dlk[k * n_tan + 2 * et + 1] = ty_;
          cfma(s_sq[k], tx_, tx_);
          cfma(s_sq[k], ty_, ty_);
        }
      }
      __syncthreads();
      continue;
    }
    // Laplacian: Minv[i][c'] = G[piv[i]][c'] (zero-padded to NR x NR) into X, pinv
    for (int idx = tid; idx < NR * NR; idx += kHeadLgThreads) {
      const int i = idx / NR, c2 = idx - i * NR;
      X[i * LD + c2] = (i < N && c2 < N) ? G[piv[i] * LD + c2] : mk(0.0, 0.0);
    }
    for (int c2 = tid; c2 < N; c2 += kHeadLgThreads) pinv[piv[c2]] = c2;
    __syncthreads();
    // tr(M^-1 Lap M): sum over (i, a) of Minv[i][pinv a] LapM[a][i]
    if (has_lap) {
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
        const int i = idx / N, a = idx - i * N;
        cplx lm = cmul(env[a * LD + i], bf(C - 1, a, i));
        if (is_te(i)) {
          const int txc = 2 * (i - te_lo);
          cplx dxe = mk(0, 0), dye = mk(0, 0), le = mk(0, 0);
          const int s = sp[i];
          for (int g = 0; g < nG; ++g) {
            const cplx pw = cmul(ph[g * N + i], Weff(a, g, s));
            const double gx = mc.Gs[2 * g], gy = mc.Gs[2 * g + 1];
            cfma(dxe, pw, mk(0, gx));
            cfma(dye, pw, mk(0, gy));
            le = cadd(le, cscale(pw, -(gx * gx + gy * gy)));
          }
          const cplx b0 = bf(0, a, i);
          lm = cadd(lm, cmul(le, mk(1.0 + b0.re, b0.im)));
          lm = cadd(lm, cscale(cmul(dxe, bf(1 + txc, a, i)), 2.0));
          lm = cadd(lm, cscale(cmul(dye, bf(2 + txc, a, i)), 2.0));
        }
        const cplx t = cmul(X[i * LD + pinv[a]], lm);
        v[0] += t.re;
        v[1] += t.im;
      }
      head_lg_warp4(v, red[1]);
      __syncthreads();
      if (tid == 0) {
        double o[4];
        head_lg_total4(red[1], o);
        s_lapk[k] = mk(o[0], o[1]);
      }
    }
    // B_t = Minv X_t, t = (tangent electron e, axis): X_t staged in G, B_t in Y
    for (int t = 0; t < n_tan; ++t) {
      const int e = te_lo + t / 2, bax = t & 1;
      for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
        const int j = idx / N, a = idx - j * N;
        cplx dm = cmul(env[a * LD + j], bf(1 + t, a, j));
        if (j == e) {
          const cplx b0 = bf(0, a, e);
          dm = cadd(dm, cmul(denv(a, e, bax), mk(1.0 + b0.re, b0.im)));
        }
        G[pinv[a] * LD + j] = dm;
      }
      __syncthreads();
      if (tid == 0 && t > 0) {  // the previous tangent's CTA sums
        double o[4];
        head_lg_total4(red[(t - 1) & 1], o);
        const cplx tr = mk(o[0], o[1]);
        dlk[k * n_tan + t - 1] = tr;
        cfma(s_sq[k], tr, tr);
        s_lapk[k] = csub(s_lapk[k], mk(o[2], o[3]));
      }
      cplx acc[TS][TS];
#pragma unroll
      for (int u = 0; u < TS; ++u)
#pragma unroll
        for (int w = 0; w < TS; ++w) acc[u][w] = mk(0.0, 0.0);
      const cplx* xa = X + ty * LD;
      const cplx* gb = G + tx;
#pragma unroll 2
      for (int c2 = 0; c2 < N; ++c2) {
        cplx av[TS], bv[TS];
#pragma unroll
        for (int u = 0; u < TS; ++u) av[u] = xa[16 * u * LD + c2];
#pragma unroll
        for (int w = 0; w < TS; ++w) bv[w] = gb[c2 * LD + 16 * w];
#pragma unroll
        for (int u = 0; u < TS; ++u)
#pragma unroll
          for (int w = 0; w < TS; ++w) cfma(acc[u][w], av[u], bv[w]);
      }
      double v[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
      for (int u = 0; u < TS; ++u) {
#pragma unroll
        for (int w = 0; w < TS; ++w) Y[(ty + 16 * u) * LD + tx + 16 * w] = acc[u][w];
        if (ty == tx) {
          v[0] += acc[u][u].re;
          v[1] += acc[u][u].im;
        }
      }
      __syncthreads();
#pragma unroll
      for (int u = 0; u < TS; ++u)
#pragma unroll
        for (int w = 0; w < TS; ++w) {
          const cplx bt = Y[(tx + 16 * w) * LD + ty + 16 * u];
          v[2] = fma(acc[u][w].re, bt.re, fma(-acc[u][w].im, bt.im, v[2]));
          v[3] = fma(acc[u][w].re, bt.im, fma(acc[u][w].im, bt.re, v[3]));
        }
      head_lg_warp4(v, red[t & 1]);
    }
    __syncthreads();
    if (tid == 0 && n_tan > 0) {
      double o[4];
      head_lg_total4(red[(n_tan - 1) & 1], o);
      const cplx tr = mk(o[0], o[1]);
      dlk[k * n_tan + n_tan - 1] = tr;
      cfma(s_sq[k], tr, tr);
      s_lapk[k] = csub(s_lapk[k], mk(o[2], o[3]));
    }
  }
  __syncthreads();
  // ======================= phase 3: log-sum-exp over determinants (warp 0) =======================
  if (warp != 0) return;
  const int jo = j_out0 + job;
  double mx = -INFINITY;
  for (int k = 0; k < K; ++k) {
    const double zr = s_ld[k].re + ((K > 1 && hp.det_logw) ? hp.det_logw[k] : 0.0);
    if (!sing[k] && zr > mx) mx = zr;
  }
  const bool all_sing = (mx == -INFINITY);
  cplx ssum = mk(0, 0);
  cplx p[NQS_MAX_DETS];
  for (int k = 0; k < K; ++k) {
    if (sing[k]) {
      p[k] = mk(0, 0);
      continue;
    }
    const cplx wk = (K > 1 && hp.det_logw) ? mk(hp.det_logw[k], hp.det_logw[K + k]) : mk(0, 0);
    p[k] = cexp_(mk(s_ld[k].re + wk.re - mx, s_ld[k].im + wk.im));
    ssum = cadd(ssum, p[k]);
  }
  cplx L;
  if (K == 1) {
    L = s_ld[0];
  } else {
    L = all_sing ? mk(-INFINITY, 0.0)
                 : mk(mx + log(hypot(ssum.re, ssum.im)), atan2(ssum.im, ssum.re));
    if (!all_sing) {
      const cplx inv_s = cdiv(mk(1.0, 0.0), ssum);
      for (int k = 0; k < K; ++k) p[k] = cmul(p[k], inv_s);
    }
  }
  if (K == 1) p[0] = mk(1.0, 0.0);
  cplx sumsq = mk(0, 0);
  for (int t = lane; t < n_tan; t += 32) {
    cplx g = mk(0, 0);
    if (all_sing) {
      g = mk(NAN, NAN);
    } else {
      for (int k = 0; k < K; ++k)
        if (!sing[k]) cfma(g, p[k], dlk[k * n_tan + t]);
    }
    cfma(sumsq, g, g);
    if (mc.use_jastrow) g.re += gj[(t & 1) * kHeadLgMaxN + t / 2];
    if (out.dL) out.dL[(size_t)jo * jb.n_tan + t] = g;
  }
  sumsq.re = warp_sum(sumsq.re);
  sumsq.im = warp_sum(sumsq.im);
  if (lane == 0) {
    if (mc.use_jastrow) L.re += jas[0];
    if (out.L) out.L[jo] = L;
    if (has_lap && out.lap) {
      cplx lap;
      if (all_sing) {
        lap = mk(NAN, NAN);
      } else if (K == 1) {
        lap = s_lapk[0];
      } else {
        lap = mk(0, 0);
        for (int k = 0; k < K; ++k)
          if (!sing[k]) cfma(lap, p[k], cadd(s_lapk[k], s_sq[k]));
        lap = csub(lap, sumsq);
      }
      if (mc.use_jastrow) lap.re += jas[1];
      out.lap[jo] = lap;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Values only (log psi of single-channel jobs: the sampler's proposals, the flipped-spin values),
// 16 < N <= 64: one CTA of 256 threads per job in four 64-thread groups, each factoring its own
// determinants (k = group, group + 4, ...) with the same pivot rule as k_head_lg; a group
// synchronises on its own named barrier, so four eliminations proceed at once. The phases live
// in the groups' matrix buffers while the envelope is built. Thread (tid % 64) of a group owns
// the entries of rows r = tid % 64 / 16 + 4 u and columns tx + 16 v of the trailing block.
// ---------------------------------------------------------------------------------------------
constexpr int kHeadValGroups = 4;
// static shared arrays of k_head_val_lg (bytes), for the host's fit check
constexpr size_t kHeadValStaticBytes = 8 * (2 * kHeadLgMaxN + kHeadLgThreads / 32 + 1) +
                                       4 * (kHeadLgMaxN + 2 * kHeadValGroups * kHeadLgMaxN +
                                            kHeadValGroups + NQS_MAX_DETS) +
                                       16 * (2 * kHeadValGroups * kHeadLgMaxN + NQS_MAX_DETS) +
                                       256;

struct HeadValLayout {
  int ld;
  size_t env, G, total;
};
__host__ __device__ inline HeadValLayout head_val_layout(int N, int nG) {
  HeadValLayout L;
  L.ld = N + 1;
  const size_t mat = round128(16 * (size_t)N * L.ld);
  L.env = 0;
  L.G = mat;
  L.total = mat + kHeadValGroups * mat;
  // the phases (nG x N complex) are staged in the group buffers before the envelope exists
  const size_t ph = 16 * (size_t)nG * N;
  if (ph > kHeadValGroups * mat) L.total = 0;  // does not fit: caller takes k_head_lg
  return L;
}

__device__ __forceinline__ void group_bar(int id) {
  asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory");
}

template <typename TIN>
__global__ void __launch_bounds__(kHeadLgThreads, 1) k_head_val_lg(JobBatch jb, ModelConst mc,
                                                                  const TIN* __restrict__ BF,
                                                                  int ldbf, HeadParams hp,
                                                                  HeadOut out, int j_out0) {
  const int N = jb.N, C = jb.C, nG = mc.nG, K = mc.K;
  const int tid = threadIdx.x, lane = tid & 31;
  const int grp = tid >> 6, gt = tid & 63, gw = gt >> 5;  // group, thread in group, warp in group
  const int job = blockIdx.x;
  const HeadValLayout lay = head_val_layout(N, nG);
  const int LD = lay.ld;
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* env = reinterpret_cast<cplx*>(smraw + lay.env);
  const size_t gstride = (lay.total - lay.G) / kHeadValGroups;
  cplx* G = reinterpret_cast<cplx*>(smraw + lay.G + grp * gstride);
  cplx* ph = reinterpret_cast<cplx*>(smraw + lay.G);  // phase 1 only
  __shared__ double rx[kHeadLgMaxN], ry[kHeadLgMaxN], red[kHeadLgThreads / 32];
  __shared__ int sp[kHeadLgMaxN];
  __shared__ int used[kHeadValGroups][kHeadLgMaxN], piv[kHeadValGroups][kHeadLgMaxN];
  __shared__ int s_p[kHeadValGroups], sing[NQS_MAX_DETS];
  __shared__ __align__(16) cplx prow[kHeadValGroups][kHeadLgMaxN],
      fcol[kHeadValGroups][kHeadLgMaxN];
  __shared__ cplx s_ld[NQS_MAX_DETS];
  __shared__ double s_jas;
  const JobInfo ji = job_info(jb, job);
  auto Weff = [&](int a, int g, int s) -> cplx {
    const size_t o = ((size_t)a * nG + g) * 2 + s;
    cplx w = mk(mc.W[2 * o], mc.W[2 * o + 1]);
    if (mc.learnable_env) w = cadd(w, mk(hp.dW[o], hp.dW[(size_t)N * nG * 2 + o]));
    return w;
  };
  // ---- phase 1 ----
  for (int i = tid; i < N; i += kHeadLgThreads) {
    const double* r = jb.R + ((size_t)ji.walker * N + i) * 2;
    rx[i] = r[0];
    ry[i] = r[1];
    sp[i] = job_spin(jb, ji, i);
  }
  __syncthreads();
  for (int idx = tid; idx < nG * N; idx += kHeadLgThreads) {
    const int g = idx / N, i = idx - g * N;
    double sn, cs;
    sincos(mc.Gs[2 * g] * rx[i] + mc.Gs[2 * g + 1] * ry[i], &sn, &cs);
    ph[idx] = mk(cs, sn);
  }
  __syncthreads();
  for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
    const int a = idx / N, i = idx - a * N;
    const int s = sp[i];
    cplx e = mk(0, 0);
#pragma unroll 4
    for (int g = 0; g < nG; ++g) cfma(e, ph[g * N + i], Weff(a, g, s));
    env[a * LD + i] = e;
  }
  double J = 0.0;
  if (mc.use_jastrow) {
    const int npair = N * (N - 1) / 2;
    for (int p = tid; p < npair; p += kHeadLgThreads) {
      int i = 0, rem = p;
      while (rem >= N - 1 - i) {
        rem -= N - 1 - i;
        ++i;
      }
      const int jj = i + 1 + rem;
      double dx, dy;
      min_image(mc, rx[i] - rx[jj], ry[i] - ry[jj], &dx, &dy);
      const double r = sqrt(dx * dx + dy * dy + 1e-12);
      double u, u1, u2;
      jastrow_u(mc, hp, r, sp[i] == sp[jj], &u, &u1, &u2);
      J += u;
    }
    J = warp_sum(J);
    if (lane == 0) red[tid >> 5] = J;
  }
  __syncthreads();  // env complete, phases no longer read: the group buffers are free
  if (tid == 0) {
    double t = 0.0;
    if (mc.use_jastrow)
      for (int w = 0; w < kHeadLgThreads / 32; ++w) t += red[w];
    s_jas = t;
  }
  // ---- phase 2: determinants k = grp, grp + 4, ... ----
  const int bar = 1 + grp;
  const int ty = gt >> 4, tx = gt & 15;  // 4 x 16 threads over the trailing block
  for (int k = grp; k < K; k += kHeadValGroups) {
    for (int idx = gt; idx < N * N; idx += 64) {
      const int i = idx / N, a = idx - i * N;
      const TIN* pb = BF + (((size_t)job * N + i) * C) * ldbf;
      const cplx b0 = mk((double)pb[k * N + a], (double)pb[K * N + k * N + a]);
      G[a * LD + i] = cmul(env[a * LD + i], mk(1.0 + b0.re, b0.im));
    }
    for (int r = gt; r < N; r += 64) used[grp][r] = 0;
    group_bar(bar);
    cplx prod = mk(1.0, 0.0);
    int pexp = 0, sg = 0;
#pragma unroll 1
    for (int c = 0; c < N; ++c) {
      if (gw == 0) {
        const int r0 = lane, r1 = lane + 32;
        const bool u0 = r0 >= N || used[grp][r0], u1 = r1 >= N || used[grp][r1];
        auto mag = [](cplx z) {
          const double v = cabs1(z);
          return v >= 0.0 ? v : 0.0;
        };
        double best = u0 ? -1.0 : mag(G[r0 * LD + c]);
        int bi = r0;
        if (!u1) {
          const double v1 = mag(G[r1 * LD + c]);
          if (v1 > best) {
            best = v1;
            bi = r1;
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
        const int p = bi;
        const cplx pv = G[p * LD + c];
        const bool zero = pv.re == 0.0 && pv.im == 0.0;
        const cplx ipv = zero ? mk(0.0, 0.0) : cdiv(mk(1.0, 0.0), pv);
        if (zero) {
          sg = 1;
        } else {
          prod = cmul(prod, pv);
          int ex;
          frexp(fmax(fabs(prod.re), fabs(prod.im)), &ex);
          prod = mk(ldexp(prod.re, -ex), ldexp(prod.im, -ex));
          pexp += ex;
        }
        for (int j = c + 1 + lane; j < N; j += 32) prow[grp][j] = G[p * LD + j];
        if (r0 < N) fcol[grp][r0] = (!u0 && r0 != p) ? cmul(G[r0 * LD + c], ipv) : mk(0.0, 0.0);
        if (r1 < N) fcol[grp][r1] = (!u1 && r1 != p) ? cmul(G[r1 * LD + c], ipv) : mk(0.0, 0.0);
        __syncwarp();
        if (lane == 0) {
          piv[grp][c] = p;
          used[grp][p] = 1;
          s_p[grp] = p;
        }
      }
      group_bar(bar);
      // rows not used yet, columns c + 1 .. N - 1
      for (int r = ty; r < N; r += 4) {
        const cplx f = fcol[grp][r];
        if (f.re == 0.0 && f.im == 0.0) continue;
        for (int j = c + 1 + tx; j < N; j += 16) G[r * LD + j] = csub(G[r * LD + j], cmul(f, prow[grp][j]));
      }
      group_bar(bar);
    }
    if (gw == 0) {
      int inv_cnt = 0;
      for (int c = lane; c < N; c += 32)
        for (int c2 = c + 1; c2 < N; ++c2)
          if (piv[grp][c] > piv[grp][c2]) ++inv_cnt;
      inv_cnt = warp_sum(inv_cnt);
      if (inv_cnt & 1) prod = mk(-prod.re, -prod.im);
      if (lane == 0) {
        s_ld[k] = sg ? mk(-INFINITY, 0.0)
                     : mk(log(hypot(prod.re, prod.im)) + pexp * 0.6931471805599453,
                          atan2(prod.im, prod.re));
        sing[k] = sg;
      }
    }
    group_bar(bar);  // piv / used / G of this group are rewritten by its next determinant
  }
  __syncthreads();
  // ---- phase 3: log-sum-exp over determinants ----
  if (tid != 0) return;
  double mx = -INFINITY;
  for (int k = 0; k < K; ++k) {
    const double zr = s_ld[k].re + ((K > 1 && hp.det_logw) ? hp.det_logw[k] : 0.0);
    if (!sing[k] && zr > mx) mx = zr;
  }
  cplx L;
  if (K == 1) {
    L = s_ld[0];
  } else if (mx == -INFINITY) {
    L = mk(-INFINITY, 0.0);
  } else {
    cplx ssum = mk(0, 0);
    for (int k = 0; k < K; ++k) {
      if (sing[k]) continue;
      const cplx wk = (K > 1 && hp.det_logw) ? mk(hp.det_logw[k], hp.det_logw[K + k]) : mk(0, 0);
      ssum = cadd(ssum, cexp_(mk(s_ld[k].re + wk.re - mx, s_ld[k].im + wk.im)));
    }
    L = mk(mx + log(hypot(ssum.re, ssum.im)), atan2(ssum.im, ssum.re));
  }
  if (mc.use_jastrow) L.re += s_jas;
  if (out.L) out.L[j_out0 + job] = L;
}

// ---------------------------------------------------------------------------------------------
// Gradient-only jobs with few tangent electrons (the spin-flip batch: one electron, two tangents),
// 16 < N <= 64: as k_head_val_lg, four 64-thread groups each invert their own determinants
// (in-place Gauss-Jordan, same pivot rule as k_head_lg) on named barriers; the tangent
// electrons' envelope derivatives are summed from the phases before the groups reuse that
// memory, so tr(M^-1 D_t) needs only the envelope, the backflow channels and those columns.
// ---------------------------------------------------------------------------------------------
constexpr int kHeadSocMaxTe = 4;
constexpr size_t kHeadSocStaticBytes =
    kHeadValStaticBytes + 16 * (2 * kHeadSocMaxTe * kHeadLgMaxN + NQS_MAX_DETS * 2 * kHeadSocMaxTe +
                                2 * NQS_MAX_DETS) +
    8 * (2 * kHeadSocMaxTe + kHeadValGroups * 2 * 4 + 4) + 256;

template <typename TIN>
__global__ void __launch_bounds__(kHeadLgThreads, 1) k_head_soc_lg(JobBatch jb, ModelConst mc,
                                                                  const TIN* __restrict__ BF,
                                                                  int ldbf, HeadParams hp,
                                                                  HeadOut out, int j_out0) {
  const int N = jb.N, C = jb.C, nG = mc.nG, K = mc.K;
  const int n_tan = jb.n_tan, n_te = n_tan / 2;
  const int tid = threadIdx.x, lane = tid & 31;
  const int grp = tid >> 6, gt = tid & 63, gw = gt >> 5;
  const int job = blockIdx.x;
  const HeadValLayout lay = head_val_layout(N, nG);
  const int LD = lay.ld;
  extern __shared__ __align__(16) unsigned char smraw[];
  cplx* env = reinterpret_cast<cplx*>(smraw + lay.env);
  const size_t gstride = (lay.total - lay.G) / kHeadValGroups;
  cplx* G = reinterpret_cast<cplx*>(smraw + lay.G + grp * gstride);
  cplx* ph = reinterpret_cast<cplx*>(smraw + lay.G);  // phase 1 only
  __shared__ double rx[kHeadLgMaxN], ry[kHeadLgMaxN], red[kHeadLgThreads / 32];
  __shared__ double gj[2 * kHeadSocMaxTe], s_jas;
  __shared__ double gred[kHeadValGroups][2][4];
  __shared__ int sp[kHeadLgMaxN];
  __shared__ int used[kHeadValGroups][kHeadLgMaxN], piv[kHeadValGroups][kHeadLgMaxN];
  __shared__ int sing[NQS_MAX_DETS];
  __shared__ __align__(16) cplx prow[kHeadValGroups][kHeadLgMaxN],
      fcol[kHeadValGroups][kHeadLgMaxN];
  __shared__ cplx dE[2 * kHeadSocMaxTe][kHeadLgMaxN];  // [axis + 2 et][orbital a]
  __shared__ cplx s_ld[NQS_MAX_DETS], s_sq[NQS_MAX_DETS], dlk[NQS_MAX_DETS][2 * kHeadSocMaxTe];
  const JobInfo ji = job_info(jb, job);
  const int te_lo = ji.tan_e0;
  auto Weff = [&](int a, int g, int s) -> cplx {
    const size_t o = ((size_t)a * nG + g) * 2 + s;
    cplx w = mk(mc.W[2 * o], mc.W[2 * o + 1]);
    if (mc.learnable_env) w = cadd(w, mk(hp.dW[o], hp.dW[(size_t)N * nG * 2 + o]));
    return w;
  };
  // ---- phase 1 ----
  for (int i = tid; i < N; i += kHeadLgThreads) {
    const double* r = jb.R + ((size_t)ji.walker * N + i) * 2;
    rx[i] = r[0];
    ry[i] = r[1];
    sp[i] = job_spin(jb, ji, i);
  }
  __syncthreads();
  for (int idx = tid; idx < nG * N; idx += kHeadLgThreads) {
    const int g = idx / N, i = idx - g * N;
    double sn, cs;
    sincos(mc.Gs[2 * g] * rx[i] + mc.Gs[2 * g + 1] * ry[i], &sn, &cs);
    ph[idx] = mk(cs, sn);
  }
  __syncthreads();
  for (int idx = tid; idx < N * N; idx += kHeadLgThreads) {
    const int a = idx / N, i = idx - a * N;
    const int s = sp[i];
    cplx e = mk(0, 0);
#pragma unroll 4
    for (int g = 0; g < nG; ++g) cfma(e, ph[g * N + i], Weff(a, g, s));
    env[a * LD + i] = e;
  }
  for (int idx = tid; idx < n_te * N; idx += kHeadLgThreads) {
    const int et = idx / N, a = idx - et * N, e = te_lo + et, s = sp[e];
    cplx dx = mk(0, 0), dy = mk(0, 0);
    for (int g = 0; g < nG; ++g) {
      const cplx pw = cmul(ph[g * N + e], Weff(a, g, s));
      cfma(dx, pw, mk(0, mc.Gs[2 * g]));
      cfma(dy, pw, mk(0, mc.Gs[2 * g + 1]));
    }
    dE[2 * et][a] = dx;
    dE[2 * et + 1][a] = dy;
  }
  double J = 0.0;
  if (mc.use_jastrow) {
    const int npair = N * (N - 1) / 2;
    for (int p = tid; p < npair; p += kHeadLgThreads) {
      int i = 0, rem = p;
      while (rem >= N - 1 - i) {
        rem -= N - 1 - i;
        ++i;
      }
      const int jj = i + 1 + rem;
      double dx, dy;
      min_image(mc, rx[i] - rx[jj], ry[i] - ry[jj], &dx, &dy);
      const double r = sqrt(dx * dx + dy * dy + 1e-12);
      double u, u1, u2;
      jastrow_u(mc, hp, r, sp[i] == sp[jj], &u, &u1, &u2);
      J += u;
    }
    J = warp_sum(J);
    if (lane == 0) red[tid >> 5] = J;
    // gradient of the tangent electrons: warp et, lanes over partners, fixed-order butterflies
    const int w = tid >> 5;
    if (w < n_te) {
      const int e = te_lo + w;
      double gx = 0.0, gy = 0.0;
      for (int jj = lane; jj < N; jj += 32) {
        if (jj == e) continue;
        double dx, dy;
        min_image(mc, rx[e] - rx[jj], ry[e] - ry[jj], &dx, &dy);
        const double r = sqrt(dx * dx + dy * dy + 1e-12);
        double u, u1, u2;
        jastrow_u(mc, hp, r, sp[e] == sp[jj], &u, &u1, &u2);
        gx += u1 * dx / r;
        gy += u1 * dy / r;
      }
      gx = warp_sum(gx);
      gy = warp_sum(gy);
      if (lane == 0) {
        gj[2 * w] = gx;
        gj[2 * w + 1] = gy;
      }
    }
  }
  __syncthreads();  // env / dE complete, phases no longer read: the group buffers are free
  if (tid == 0) {
    double t = 0.0;
    if (mc.use_jastrow)
      for (int w = 0; w < kHeadLgThreads / 32; ++w) t += red[w];
    s_jas = t;
  }
  // ---- phase 2: determinants k = grp, grp + 4, ... ----
  const int bar = 1 + grp;
  const int ty = gt >> 4, tx = gt & 15;
  for (int k = grp; k < K; k += kHeadValGroups) {
    auto bf = [&](int c, int a, int i) -> cplx {
      const TIN* p = BF + (((size_t)job * N + i) * C + c) * ldbf;
      return mk((double)p[k * N + a], (double)p[K * N + k * N + a]);
    };
    for (int idx = gt; idx < N * N; idx += 64) {
      const int i = idx / N, a = idx - i * N;
      const cplx b0 = bf(0, a, i);
      G[a * LD + i] = cmul(env[a * LD + i], mk(1.0 + b0.re, b0.im));
    }
    for (int r = gt; r < N; r += 64) used[grp][r] = 0;
    group_bar(bar);
    cplx prod = mk(1.0, 0.0);
    int pexp = 0, sg = 0;
#pragma unroll 1
    for (int c = 0; c < N; ++c) {
      if (gw == 0) {
        const int r0 = lane, r1 = lane + 32;
        const bool u0 = r0 >= N || used[grp][r0], u1 = r1 >= N || used[grp][r1];
        auto mag = [](cplx z) {
          const double v = cabs1(z);
          return v >= 0.0 ? v : 0.0;
        };
        double best = u0 ? -1.0 : mag(G[r0 * LD + c]);
        int bi = r0;
        if (!u1) {
          const double v1 = mag(G[r1 * LD + c]);
          if (v1 > best) {
            best = v1;
            bi = r1;
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
        const int p = bi;
        const cplx pv = G[p * LD + c];
        const bool zero = pv.re == 0.0 && pv.im == 0.0;
        const cplx ipv = zero ? mk(0.0, 0.0) : cdiv(mk(1.0, 0.0), pv);
        if (zero) {
          sg = 1;
        } else {
          prod = cmul(prod, pv);
          int ex;
          frexp(fmax(fabs(prod.re), fabs(prod.im)), &ex);
          prod = mk(ldexp(prod.re, -ex), ldexp(prod.im, -ex));
          pexp += ex;
        }
        for (int j = lane; j < N; j += 32)
          prow[grp][j] = cmul(j == c ? mk(1.0, 0.0) : G[p * LD + j], ipv);
        for (int r = lane; r < N; r += 32) fcol[grp][r] = r == p ? mk(0.0, 0.0) : G[r * LD + c];
        __syncwarp();
        if (lane == 0) {
          piv[grp][c] = p;
          used[grp][p] = 1;
        }
      }
      group_bar(bar);
      const int p = piv[grp][c];
      for (int r = ty; r < N; r += 4) {
        const cplx f = fcol[grp][r];
        for (int j = tx; j < N; j += 16) {
          cplx v;
          if (r == p) {
            v = prow[grp][j];
          } else {
            v = j == c ? mk(0.0, 0.0) : G[r * LD + j];
            v = csub(v, cmul(f, prow[grp][j]));
          }
          G[r * LD + j] = v;
        }
      }
      group_bar(bar);
    }
    if (gw == 0) {
      int inv_cnt = 0;
      for (int c = lane; c < N; c += 32)
        for (int c2 = c + 1; c2 < N; ++c2)
          if (piv[grp][c] > piv[grp][c2]) ++inv_cnt;
      inv_cnt = warp_sum(inv_cnt);
      if (inv_cnt & 1) prod = mk(-prod.re, -prod.im);
      if (lane == 0) {
        s_ld[k] = sg ? mk(-INFINITY, 0.0)
                     : mk(log(hypot(prod.re, prod.im)) + pexp * 0.6931471805599453,
                          atan2(prod.im, prod.re));
        sing[k] = sg;
        s_sq[k] = mk(0, 0);
      }
    }
    // tr(M^-1 D_t) for both axes of each tangent electron: sum over (i, c') of
    // M^-1[i][piv c'] D_t[piv c'][i] (rows of the inverse at storage rows piv[i])
    for (int et = 0; et < n_te; ++et) {
      const int e = te_lo + et;
      double v[4] = {0.0, 0.0, 0.0, 0.0};
      for (int idx = gt; idx < N * N; idx += 64) {
        const int i = idx / N, c2 = idx - i * N;
        const int a = piv[grp][c2];
        const cplx m = G[piv[grp][i] * LD + c2];
        const cplx en = env[a * LD + i];
        cplx dx = cmul(en, bf(1 + 2 * et, a, i)), dy = cmul(en, bf(2 + 2 * et, a, i));
        if (i == e) {
          const cplx b0 = bf(0, a, e), w1 = mk(1.0 + b0.re, b0.im);
          dx = cadd(dx, cmul(dE[2 * et][a], w1));
          dy = cadd(dy, cmul(dE[2 * et + 1][a], w1));
        }
        const cplx tx_ = cmul(m, dx), ty_ = cmul(m, dy);
        v[0] += tx_.re;
        v[1] += tx_.im;
        v[2] += ty_.re;
        v[3] += ty_.im;
      }
      warp_sum_n<double, 4>(v);
      if (lane == 0) {
        gred[grp][gw][0] = v[0];
        gred[grp][gw][1] = v[1];
        gred[grp][gw][2] = v[2];
        gred[grp][gw][3] = v[3];
      }
      group_bar(bar);
      if (gt == 0) {
        const cplx tx_ = mk(gred[grp][0][0] + gred[grp][1][0], gred[grp][0][1] + gred[grp][1][1]);
        const cplx ty_ = mk(gred[grp][0][2] + gred[grp][1][2], gred[grp][0][3] + gred[grp][1][3]);
        dlk[k][2 * et] = tx_;
        dlk[k][2 * et + 1] = ty_;
        cfma(s_sq[k], tx_, tx_);
        cfma(s_sq[k], ty_, ty_);
      }
      group_bar(bar);  // gred is rewritten by the next tangent electron
    }
  }
  __syncthreads();
  // ---- phase 3: log-sum-exp over determinants, gradients (warp 0) ----
  if (tid >= 32) return;
  const int jo = j_out0 + job;
  double mx = -INFINITY;
  for (int k = 0; k < K; ++k) {
    const double zr = s_ld[k].re + ((K > 1 && hp.det_logw) ? hp.det_logw[k] : 0.0);
    if (!sing[k] && zr > mx) mx = zr;
  }
  const bool all_sing = (mx == -INFINITY);
  cplx ssum = mk(0, 0);
  cplx p[NQS_MAX_DETS];
  for (int k = 0; k < K; ++k) {
    if (sing[k]) {
      p[k] = mk(0, 0);
      continue;
    }
    const cplx wk = (K > 1 && hp.det_logw) ? mk(hp.det_logw[k], hp.det_logw[K + k]) : mk(0, 0);
    p[k] = cexp_(mk(s_ld[k].re + wk.re - mx, s_ld[k].im + wk.im));
    ssum = cadd(ssum, p[k]);
  }
  cplx L;
  if (K == 1) {
    L = s_ld[0];
  } else {
    L = all_sing ? mk(-INFINITY, 0.0)
                 : mk(mx + log(hypot(ssum.re, ssum.im)), atan2(ssum.im, ssum.re));
    if (!all_sing) {
      const cplx inv_s = cdiv(mk(1.0, 0.0), ssum);
      for (int k = 0; k < K; ++k) p[k] = cmul(p[k], inv_s);
    }
  }
  if (K == 1) p[0] = mk(1.0, 0.0);
  for (int t = lane; t < n_tan; t += 32) {
    cplx g = mk(0, 0);
    if (all_sing) {
      g = mk(NAN, NAN);
    } else {
      for (int k = 0; k < K; ++k)
        if (!sing[k]) cfma(g, p[k], dlk[k][t]);
    }
    if (mc.use_jastrow) g.re += gj[t];
    if (out.dL) out.dL[(size_t)jo * jb.n_tan + t] = g;
  }
  if (lane == 0) {
    if (mc.use_jastrow) L.re += s_jas;
    if (out.L) out.L[jo] = L;
  }
}

}  // namespace nqs
