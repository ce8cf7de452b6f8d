// head_rt.cuh — determinant head for N <= 16 electrons with the orbital matrices in registers.
//
// Same quantities as k_head (psiformer.py:118-189: envelope, backflow-dressed orbitals,
// log-sum-exp over determinants, Jastrow; forward-mode tangents and Laplacian of log psi),
// organised for the SIMT FP64 pipes:
//   phase 1 (whole CTA, per job): phases e^{i G.r}, envelope env[a][i], its derivatives for the
//     tangent electrons (d/dx, d/dy, Laplacian), the Jastrow value, gradient and Laplacian.
//   phase 2 (half a warp per (job, determinant)): lane a holds row a of the orbital matrix M in
//     registers; elimination with partial pivoting on |re|+|im| picks the pivot row among the
//     rows not yet used (no row swaps: the pivot order piv[c] is kept instead). Values only:
//     LU elimination below the pivot. With tangents: in-place Gauss-Jordan, after which the
//     lane whose row was the pivot of column c holds row c of M^-1 with its entry c' belonging
//     to orbital piv[c'].
//       tr(M^-1 D) = sum_lanes sum_c' m[c'] D[piv[c']][step]        (step = lane's pivot column)
//       B_t = M^-1 D_t row by row: B[step][j2] = sum_c' m[c'] D_t[piv[c']][j2], with D_t staged
//       in shared memory by rows (lane a writes row a), and tr(B_t^2) through a transpose in the
//       same buffer.
//   phase 3 (half a warp per job): log-sum-exp over determinants, outputs.
// The determinant sign is the product of the pivot phases times the parity of piv.
#pragma once

#include "net_kernels.cuh"

namespace nqs {

constexpr int kHeadTok = 16;  // electron slots (register columns)
constexpr int kHeadLd = 17;   // row stride (complex) of the per-job and per-half-warp matrices

struct HeadRtPlan {
  int jpc;  // jobs per CTA (64 threads = 4 half-warps)
  size_t job_bytes, hw_bytes, bytes;
};

__host__ __device__ inline size_t head_rt_job_bytes(int N, int nG, int K, int n_tan, bool tan,
                                                    bool lap) {
  const size_t mat = 16 * (size_t)N * kHeadLd;
  size_t b = mat;                                   // env
  if (tan) b += 2 * mat;                            // d env / dx, dy (tangent electrons' columns)
  if (lap) b += mat;                                // Laplacian of env
  b += 16 * (size_t)nG * N;                         // phases
  b += (size_t)K * 16 * (3 + (size_t)n_tan);        // per det: logdet, lapk, sq, dLk[n_tan]
  b += 8 * 2 * (size_t)N;                           // rx, ry
  b += 8 * (4 + 2 * (size_t)N);                     // J, lapJ, (pad), gJ[2][N]
  b += 4 * (size_t)N + 4 * (size_t)K;               // spins, singular flags
  return round128(b);
}

inline HeadRtPlan head_rt_plan(int N, int nG, int K, int n_tan, bool tan, bool lap) {
  HeadRtPlan p;
  p.jpc = std::max(1, 4 / K);
  p.job_bytes = head_rt_job_bytes(N, nG, K, tan ? n_tan : 0, tan, lap);
  // per half-warp: pivot-row broadcast (and, with tangents, the D_t / B_t matrix), pivot order
  p.hw_bytes = round128(16 * (size_t)(tan ? kHeadTok * kHeadLd : 2 * kHeadTok) + 4 * kHeadTok);
  p.bytes = p.jpc * p.job_bytes + 4 * p.hw_bytes;
  while (p.jpc > 1 && p.bytes > 200 * 1024) {  // large envelopes (many plane waves): fewer jobs
    --p.jpc;
    p.bytes = p.jpc * p.job_bytes + 4 * p.hw_bytes;
  }
  return p;
}

template <typename TIN, bool TAN, bool LAP>
__global__ void __launch_bounds__(64) k_head_rt(JobBatch jb, ModelConst mc,
                                                const TIN* __restrict__ BF, int ldbf,
                                                HeadParams hp, HeadOut out, int j_out0, int jpc,
                                                size_t job_bytes, size_t hw_bytes) {
  constexpr int NP = kHeadTok, LD = kHeadLd;
  const int N = jb.N, C = jb.C, nG = mc.nG, K = mc.K;
  const int n_tan = TAN ? jb.n_tan : 0;
  const int tid = threadIdx.x, lane = tid & 31, hw = tid >> 4, l = lane & 15;
  const int job0 = blockIdx.x * jpc;
  const int njob = min(jpc, jb.n_jobs - job0);
  extern __shared__ __align__(16) unsigned char smraw[];
  // ---- carve ----
  struct JobMem {
    cplx *env, *dex, *dey, *lape, *ph;
    double *rx, *ry, *jas, *gj;
    int* sp;
    cplx *ld, *lapk, *sq, *dlk;
    int* sing;
  };
  auto jm = [&](int j) {
    JobMem m;
    unsigned char* p = smraw + (size_t)j * job_bytes;
    const size_t mat = (size_t)N * LD;
    m.env = reinterpret_cast<cplx*>(p);
    cplx* q = m.env + mat;
    m.dex = q;
    m.dey = q + (TAN ? mat : 0);
    q = m.dey + (TAN ? mat : 0);
    m.lape = q;
    q += LAP ? mat : 0;
    m.ph = q;
    q += (size_t)nG * N;
    m.ld = q;
    m.lapk = m.ld + K;
    m.sq = m.lapk + K;
    m.dlk = m.sq + K;
    q = m.dlk + (size_t)K * n_tan;
    m.rx = reinterpret_cast<double*>(q);
    m.ry = m.rx + N;
    m.jas = m.ry + N;  // [0] J, [1] lapJ
    m.gj = m.jas + 4;  // [2][N]
    m.sp = reinterpret_cast<int*>(m.gj + 2 * N);
    m.sing = m.sp + N;
    return m;
  };
  cplx* hbuf = reinterpret_cast<cplx*>(smraw + (size_t)jpc * job_bytes + (size_t)hw * hw_bytes);
  __shared__ double red[2][4];
  auto Weff = [&](int a, int g, int s) -> cplx {
    const size_t o = ((size_t)a * nG + g) * 2 + s;
    cplx w = mk(mc.W[2 * o], mc.W[2 * o + 1]);
    if (mc.learnable_env) w = cadd(w, mk(hp.dW[o], hp.dW[(size_t)N * nG * 2 + o]));
    return w;
  };
  // ======================= phase 1: per-job tables (all threads) =======================
  for (int j = 0; j < njob; ++j) {
    const JobMem m = jm(j);
    const JobInfo ji = job_info(jb, job0 + j);
    const int te_lo = ji.tan_e0, te_hi = ji.tan_e0 + n_tan / 2;
    for (int i = tid; i < N; i += blockDim.x) {
      const double* r = jb.R + ((size_t)ji.walker * N + i) * 2;
      m.rx[i] = r[0];
      m.ry[i] = r[1];
      m.sp[i] = job_spin(jb, ji, i);
    }
    __syncthreads();
    for (int idx = tid; idx < nG * N; idx += blockDim.x) {
      const int g = idx / N, i = idx - g * N;
      double sn, cs;
      sincos(mc.Gs[2 * g] * m.rx[i] + mc.Gs[2 * g + 1] * m.ry[i], &sn, &cs);
      m.ph[idx] = mk(cs, sn);
    }
    __syncthreads();
    for (int idx = tid; idx < N * N; idx += blockDim.x) {
      const int a = idx / N, i = idx - a * N;
      const int s = m.sp[i];
      const bool te = TAN && i >= te_lo && i < te_hi;
      cplx e = mk(0, 0), dx = mk(0, 0), dy = mk(0, 0), le = mk(0, 0);
      for (int g = 0; g < nG; ++g) {
        const cplx pw = cmul(m.ph[g * N + i], Weff(a, g, s));
        e = cadd(e, pw);
        if (te) {
          const double gx = mc.Gs[2 * g], gy = mc.Gs[2 * g + 1];
          cfma(dx, pw, mk(0, gx));
          cfma(dy, pw, mk(0, gy));
          if (LAP) le = cadd(le, cscale(pw, -(gx * gx + gy * gy)));
        }
      }
      m.env[a * LD + i] = e;
      if (te) {
        m.dex[a * LD + i] = dx;
        m.dey[a * LD + i] = dy;
        if (LAP) m.lape[a * LD + i] = le;
      }
    }
    // Jastrow: value over pairs; gradient / Laplacian per tangent electron
    if (mc.use_jastrow) {
      double Jp = 0.0;
      const int npair = N * (N - 1) / 2;
      for (int p = tid; p < npair; p += blockDim.x) {
        int i = 0, rem = p;
        while (rem >= N - 1 - i) {
          rem -= N - 1 - i;
          ++i;
        }
        const int jj = i + 1 + rem;
        double dx, dy;
        min_image(mc, m.rx[i] - m.rx[jj], m.ry[i] - m.ry[jj], &dx, &dy);
        const double r = sqrt(dx * dx + dy * dy + 1e-12);
        double u, u1, u2;
        jastrow_u(mc, hp, r, m.sp[i] == m.sp[jj], &u, &u1, &u2);
        Jp += u;
      }
      Jp = warp_sum(Jp);
      if (lane == 0) red[0][tid >> 5] = Jp;
      double lp = 0.0;
      if (TAN) {
        // thread = (tangent electron e, group g of 4): partners jj = g, g+4, ...
        const int n_te = n_tan / 2;
        for (int base = 0; base < n_te; base += 16) {
          const bool has_e = base + (tid >> 2) < n_te;
          const int e = te_lo + base + (tid >> 2), g = tid & 3;
          double gx = 0.0, gy = 0.0, le = 0.0;
          if (has_e) {
            for (int jj = g; jj < N; jj += 4) {
              if (jj == e) continue;
              double dx, dy;
              min_image(mc, m.rx[e] - m.rx[jj], m.ry[e] - m.ry[jj], &dx, &dy);
              const double d2 = dx * dx + dy * dy;
              const double r = sqrt(d2 + 1e-12);
              double u, u1, u2;
              jastrow_u(mc, hp, r, m.sp[e] == m.sp[jj], &u, &u1, &u2);
              gx += u1 * dx / r;
              gy += u1 * dy / r;
              if (LAP) le += u2 * d2 / (r * r) + u1 * (2.0 / r - d2 / (r * r * r));
            }
          }
          gx += __shfl_xor_sync(0xffffffffu, gx, 1);
          gx += __shfl_xor_sync(0xffffffffu, gx, 2);
          gy += __shfl_xor_sync(0xffffffffu, gy, 1);
          gy += __shfl_xor_sync(0xffffffffu, gy, 2);
          le += __shfl_xor_sync(0xffffffffu, le, 1);
          le += __shfl_xor_sync(0xffffffffu, le, 2);
          if (g == 0 && has_e) {
            m.gj[e] = gx;
            m.gj[N + e] = gy;
            lp += le;
          }
        }
      }
      lp = warp_sum(lp);
      if (lane == 0) red[1][tid >> 5] = lp;
      __syncthreads();
      if (tid == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
          a += red[0][w];
          b += red[1][w];
        }
        m.jas[0] = a;
        m.jas[1] = b;
      }
    }
    __syncthreads();
  }
  // ======================= phase 2: half a warp per (job, determinant) =======================
  // Both halves of a warp run every shuffle below: inactive halves work on a valid job / det
  // and write nothing.
  const int ntask = njob * K;
  const int nround = (jpc * K + 3) / 4;
  for (int rnd = 0; rnd < nround; ++rnd) {
    const int task = rnd * 4 + hw;
    const bool active = task < ntask;
    const int j = active ? task / K : 0, k = active ? task - (task / K) * K : 0;
    const JobMem m = jm(j);
    const int job = job0 + j;
    const JobInfo ji = job_info(jb, job);
    const int te_lo = ji.tan_e0;
    auto bf = [&](int c, int a, int i) -> cplx {
      const TIN* p = BF + (((size_t)job * N + i) * C + c) * ldbf;
      return mk((double)p[k * N + a], (double)p[K * N + k * N + a]);
    };
    // ---- row l of M (rows / columns past N: identity) ----
    cplx mr[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      if (l < N && i < N) {
        const cplx b0 = bf(0, l, i);
        mr[i] = cmul(m.env[l * LD + i], mk(1.0 + b0.re, b0.im));
      } else {
        mr[i] = mk(i == l ? 1.0 : 0.0, 0.0);
      }
    }
    // ---- elimination: register 0 always holds the current column (the row rotates left by one
    // register per step), so the step loop is not unrolled ----
    int* piv = reinterpret_cast<int*>(hbuf + (TAN ? NP * LD : 2 * NP));  // pivot row per column
    bool used = false;
    int step = l;  // the column this lane's row pivots (padding rows keep their own index)
    // product of the pivots, kept as prod * 2^pexp with max(|re|, |im|) of prod in [0.5, 1)
    cplx prod = mk(1.0, 0.0);
    int pexp = 0;
    int sing = 0;
#pragma unroll 1
    for (int c = 0; c < N; ++c) {
      double best = used ? -1.0 : cabs1(mr[0]);
      int bi = l;
#pragma unroll
      for (int o = 8; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) {
          best = ob;
          bi = oi;
        }
      }
      const int p = bi;
      if (l == 0) piv[c] = p;
      const int src = (lane & 16) | p;
      const cplx pv = mk(__shfl_sync(0xffffffffu, mr[0].re, src),
                         __shfl_sync(0xffffffffu, mr[0].im, src));
      const bool zero = (pv.re == 0.0 && pv.im == 0.0);
      if (zero) {
        sing = 1;
      } else {
        prod = cmul(prod, pv);
        int e;
        frexp(fmax(fabs(prod.re), fabs(prod.im)), &e);
        prod = mk(ldexp(prod.re, -e), ldexp(prod.im, -e));
        pexp += e;
      }
      const cplx ipv = zero ? mk(0.0, 0.0) : cdiv(mk(1.0, 0.0), pv);
      const bool me = (l == p);
      if (me) {
        used = true;
        step = c;
      }
      cplx* prow = hbuf + (c & 1) * NP;  // double-buffered broadcast of the scaled pivot row
      if (TAN) {
        if (me) {
          mr[0] = mk(1.0, 0.0);
#pragma unroll
          for (int col = 0; col < NP; ++col) {
            mr[col] = cmul(mr[col], ipv);
            prow[col] = mr[col];
          }
        }
        __syncwarp();
        if (!me) {
          const cplx f = mr[0];
          mr[0] = mk(0.0, 0.0);
#pragma unroll
          for (int col = 0; col < NP; ++col) mr[col] = csub(mr[col], cmul(f, prow[col]));
        }
      } else {
        if (me) {
#pragma unroll
          for (int col = 1; col < NP; ++col) prow[col] = cmul(mr[col], ipv);
        }
        __syncwarp();
        if (!used) {
          const cplx f = mr[0];
#pragma unroll
          for (int col = 1; col < NP; ++col) mr[col] = csub(mr[col], cmul(f, prow[col]));
        }
      }
      const cplx t0 = mr[0];
#pragma unroll
      for (int col = 0; col < NP - 1; ++col) mr[col] = mr[col + 1];
      mr[NP - 1] = t0;
    }
    if (TAN) {  // complete the rotation to NP registers: mr[c'] = slot c' of the in-place inverse
#pragma unroll 1
      for (int r = N; r < NP; ++r) {
        const cplx t0 = mr[0];
#pragma unroll
        for (int col = 0; col < NP - 1; ++col) mr[col] = mr[col + 1];
        mr[NP - 1] = t0;
      }
    }
    __syncwarp();
    // parity of the pivot order: inversions (c < c', piv[c] > piv[c']) counted by the row
    // pivoting column c
    int inv_cnt = 0;
    if (l < N)
      for (int c2 = step + 1; c2 < N; ++c2)
        if (piv[c2] < l) ++inv_cnt;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) inv_cnt += __shfl_xor_sync(0xffffffffu, inv_cnt, o);
    if (inv_cnt & 1) prod = mk(-prod.re, -prod.im);
    const cplx logdet = sing ? mk(-INFINITY, 0.0)
                             : mk(log(hypot(prod.re, prod.im)) + pexp * 0.6931471805599453,
                                  atan2(prod.im, prod.re));
    __syncwarp();
    // ---- tangents (also for singular matrices, whose results phase 3 discards) ----
    cplx lapk = mk(0, 0), sq = mk(0, 0);
    if (TAN) {
      const bool row = l < N;  // lane holds row `step` of M^-1
      const int e_me = step;   // electron of this lane's M^-1 row
      if (LAP) {
        // tr(M^-1 Lap M) = sum_lanes sum_c' m[c'] LapM[piv[c']][e_me]
        cplx acc = mk(0, 0);
        if (row) {
          const bool te = e_me >= te_lo && e_me < te_lo + n_tan / 2;
          const int tx = 2 * (e_me - te_lo);
#pragma unroll
          for (int c2 = 0; c2 < NP; ++c2) {
            if (c2 >= N) break;
            const int a = piv[c2];
            cplx lm = cmul(m.env[a * LD + e_me], bf(C - 1, a, e_me));
            if (te) {
              const cplx b0 = bf(0, a, e_me);
              lm = cadd(lm, cmul(m.lape[a * LD + e_me], mk(1.0 + b0.re, b0.im)));
              lm = cadd(lm, cscale(cmul(m.dex[a * LD + e_me], bf(1 + tx, a, e_me)), 2.0));
              lm = cadd(lm, cscale(cmul(m.dey[a * LD + e_me], bf(2 + tx, a, e_me)), 2.0));
            }
            cfma(acc, mr[c2], lm);
          }
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
          acc.re += __shfl_xor_sync(0xffffffffu, acc.re, o);
          acc.im += __shfl_xor_sync(0xffffffffu, acc.im, o);
        }
        lapk = acc;
        cplx trb2 = mk(0, 0);  // this lane's part of sum_t tr(B_t^2)
        for (int t = 0; t < n_tan; ++t) {
          const int e = te_lo + t / 2, bax = t & 1;
          const cplx* dE = bax ? m.dey : m.dex;
          // D_t row l -> hbuf (rows: orbitals, columns: electrons)
          if (row) {
            const cplx b0e = bf(0, l, e);
            for (int i = 0; i < N; ++i) {
              cplx dm = cmul(m.env[l * LD + i], bf(1 + t, l, i));
              if (i == e) dm = cadd(dm, cmul(dE[l * LD + e], mk(1.0 + b0e.re, b0e.im)));
              hbuf[l * LD + i] = dm;
            }
          }
          __syncwarp();
          cplx b[NP];
#pragma unroll
          for (int j2 = 0; j2 < NP; ++j2) b[j2] = mk(0, 0);
#pragma unroll
          for (int c2 = 0; c2 < NP; ++c2) {
            if (c2 >= N) break;
            const cplx* drow = hbuf + piv[c2] * LD;
            const cplx mv = mr[c2];
#pragma unroll
            for (int j2 = 0; j2 < NP; ++j2)
              if (j2 < N) cfma(b[j2], mv, drow[j2]);
          }
          cplx trb = mk(0, 0);
#pragma unroll
          for (int j2 = 0; j2 < NP; ++j2)
            if (j2 == e_me) trb = b[j2];
          if (!row) trb = mk(0, 0);
          __syncwarp();
          if (row) {
#pragma unroll
            for (int j2 = 0; j2 < NP; ++j2)
              if (j2 < N) hbuf[e_me * LD + j2] = b[j2];
          }
          __syncwarp();
          if (row) {
#pragma unroll
            for (int j2 = 0; j2 < NP; ++j2)
              if (j2 < N) cfma(trb2, b[j2], hbuf[j2 * LD + e_me]);
          }
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) {
            trb.re += __shfl_xor_sync(0xffffffffu, trb.re, o);
            trb.im += __shfl_xor_sync(0xffffffffu, trb.im, o);
          }
          if (active && l == 0) m.dlk[k * n_tan + t] = trb;
          cfma(sq, trb, trb);
          __syncwarp();
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) {
          trb2.re += __shfl_xor_sync(0xffffffffu, trb2.re, o);
          trb2.im += __shfl_xor_sync(0xffffffffu, trb2.im, o);
        }
        lapk = csub(lapk, trb2);
      } else {
        // tr(M^-1 D_t) only: sum_lanes sum_c' m[c'] D_t[piv[c']][e_me]
        for (int t = 0; t < n_tan; ++t) {
          const int e = te_lo + t / 2, bax = t & 1;
          const cplx* dE = bax ? m.dey : m.dex;
          cplx trb = mk(0, 0);
          if (row) {
#pragma unroll
            for (int c2 = 0; c2 < NP; ++c2) {
              if (c2 >= N) break;
              const int a = piv[c2];
              cplx dm = cmul(m.env[a * LD + e_me], bf(1 + t, a, e_me));
              if (e_me == e) {
                const cplx b0 = bf(0, a, e);
                dm = cadd(dm, cmul(dE[a * LD + e], mk(1.0 + b0.re, b0.im)));
              }
              cfma(trb, mr[c2], dm);
            }
          }
#pragma unroll
          for (int o = 8; o > 0; o >>= 1) {
            trb.re += __shfl_xor_sync(0xffffffffu, trb.re, o);
            trb.im += __shfl_xor_sync(0xffffffffu, trb.im, o);
          }
          if (active && l == 0) m.dlk[k * n_tan + t] = trb;
          cfma(sq, trb, trb);
        }
      }
    }
    if (active && l == 0) {
      m.ld[k] = logdet;
      m.lapk[k] = lapk;
      m.sq[k] = sq;
      m.sing[k] = sing;
    }
    __syncwarp();
  }
  __syncthreads();
  // ======================= phase 3: half a warp per job (jpc <= 4) =======================
  {
    const bool act = hw < njob;
    const int j = act ? hw : 0;
    const JobMem m = jm(j);
    const int job = job0 + j;
    const JobInfo ji = job_info(jb, job);
    const int te_lo = ji.tan_e0;
    const int jo = j_out0 + job;
    double mx = -INFINITY;
    for (int k = 0; k < K; ++k) {
      const double zr = m.ld[k].re + ((K > 1 && hp.det_logw) ? hp.det_logw[k] : 0.0);
      if (!m.sing[k] && zr > mx) mx = zr;
    }
    const bool all_sing = (mx == -INFINITY);
    cplx ssum = mk(0, 0);
    cplx p[NQS_MAX_DETS];
    for (int k = 0; k < K; ++k) {
      if (m.sing[k]) {
        p[k] = mk(0, 0);
        continue;
      }
      const cplx wk = (K > 1 && hp.det_logw) ? mk(hp.det_logw[k], hp.det_logw[K + k]) : mk(0, 0);
      p[k] = cexp_(mk(m.ld[k].re + wk.re - mx, m.ld[k].im + wk.im));
      ssum = cadd(ssum, p[k]);
    }
    cplx L;
    if (K == 1) {
      L = m.ld[0];
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
    for (int t = l; t < n_tan; t += 16) {
      cplx g = mk(0, 0);
      if (all_sing) {
        g = mk(NAN, NAN);
      } else {
        for (int k = 0; k < K; ++k)
          if (!m.sing[k]) cfma(g, p[k], m.dlk[k * n_tan + t]);
      }
      cfma(sumsq, g, g);
      if (mc.use_jastrow) g.re += m.gj[(t & 1) * N + te_lo + t / 2];
      if (act && out.dL) out.dL[(size_t)jo * jb.n_tan + t] = g;
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) {
      sumsq.re += __shfl_xor_sync(0xffffffffu, sumsq.re, o);
      sumsq.im += __shfl_xor_sync(0xffffffffu, sumsq.im, o);
    }
    if (act && l == 0) {
      if (mc.use_jastrow) L.re += m.jas[0];
      if (out.L) out.L[jo] = L;
      if (LAP && out.lap) {
        cplx lap;
        if (all_sing) {
          lap = mk(NAN, NAN);
        } else if (K == 1) {
          lap = m.lapk[0];
        } else {
          lap = mk(0, 0);
          for (int k = 0; k < K; ++k)
            if (!m.sing[k]) cfma(lap, p[k], cadd(m.lapk[k], m.sq[k]));
          lap = csub(lap, sumsq);
        }
        if (mc.use_jastrow) lap.re += m.jas[1];
        out.lap[jo] = lap;
      }
    }
  }
}

}  // namespace nqs
