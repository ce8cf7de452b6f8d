// net_fwd.cu — forward passes of the continuum spinor Psiformer over batches of "jobs".
//
// A job is one walker's configuration (optionally with one spin flipped) evaluated with C
// channels per electron token: channel 0 = value, channels 1..n_tan = tangents d/dr_t (forward
// mode), and optionally a last channel carrying the partial Laplacian sum_t d^2/dr_t^2 (the
// forward Laplacian of Li et al. 2023, restated per layer below). Activations are row-major
// [job][token][channel][feature]; every Dense layer is one row GEMM over all channels with its
// bias added to value rows only.
//
// Reference semantics: src/nqs/psiformer.py:38-196 (periodic_features :84-97, MultiHeadAttention
// :50-64, TransformerBlock :67-81, backflow/envelope/determinants/LSE/Jastrow :118-189).
#include <cstdio>
#include <algorithm>

#include "net_kernels.cuh"
#include "head_rt.cuh"
#include "head_lg.cuh"

namespace nqs {

// ============================================================================================
// host orchestration
// ============================================================================================
template <typename T>
size_t net_scratch_bytes(const ModelConst& mc, size_t rows) {
  const size_t d = mc.d;
  const size_t big = std::max({3 * d, (size_t)mc.ff * d, (size_t)2 * mc.K * mc.N});
  return rows * (3 * d + big) * sizeof(T) + 4 * 256;
}

bool g_large_n_cta = true;
bool g_attn_cta_small = false;
bool g_attn_mma = true;

extern "C" int nqs_set_attention_mma(int enable) {
  g_attn_mma = enable != 0;
  return NQS_OK;
}

extern "C" int nqs_set_attention_cta_small(int enable) {
  g_attn_cta_small = enable != 0;
  return NQS_OK;
}

extern "C" int nqs_set_large_n_kernels(int enable) {
  g_large_n_cta = enable != 0;
  return NQS_OK;
}

// one CTA per job for 16 < N (head_lg.cuh); false when the job's tables do not fit
template <typename T>
static bool launch_head_lg(const ModelConst& mc, const JobBatch& cb, const T* BF, int ldbf,
                           const HeadParams& hp, const HeadOut& out, int jout, cudaStream_t st) {
  const int N = cb.N;
  const bool tan = cb.n_tan > 0, lap = tan && cb.has_lap;
  const int mode = lap ? 2 : (tan ? 1 : 0);
  const int ts = head_lg_ts(N);
  if (N > kHeadLgMaxN || (lap && N > kHeadLgMaxNLap) || mc.K > NQS_MAX_DETS) return false;
  const HeadLgLayout lay = head_lg_layout(N, mc.nG, mc.K, cb.n_tan, mode, mode == 2 ? ts : 1);
  if (lay.total + kHeadLgStaticBytes > 227 * 1024) return false;
  static bool attr = false;  // one-time opt-in to large dynamic shared memory, per instantiation
  if (!attr) {
    const int mx = 227 * 1024 - (int)kHeadLgStaticBytes;
    cudaFuncSetAttribute(k_head_lg<T, 0, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_head_lg<T, 1, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_head_lg<T, 2, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    cudaFuncSetAttribute(k_head_lg<T, 2, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize, mx);
    attr = true;
  }
  const unsigned grid = (unsigned)cb.n_jobs;
  const size_t sm = lay.total;
  if (mode == 0) {
    const HeadValLayout vl = head_val_layout(N, mc.nG);
    if (vl.total && vl.total + kHeadValStaticBytes <= 227 * 1024) {
      static bool vattr = false;
      if (!vattr) {
        cudaFuncSetAttribute(k_head_val_lg<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024 - (int)kHeadValStaticBytes);
        vattr = true;
      }
      k_head_val_lg<T><<<grid, kHeadLgThreads, vl.total, st>>>(cb, mc, BF, ldbf, hp, out, jout);
    } else {
      k_head_lg<T, 0, 1><<<grid, kHeadLgThreads, sm, st>>>(cb, mc, BF, ldbf, hp, out, jout);
    }
  } else if (mode == 1) {
    const HeadValLayout vl = head_val_layout(N, mc.nG);
    if (cb.n_tan <= 2 * kHeadSocMaxTe && vl.total && vl.total + kHeadSocStaticBytes <= 227 * 1024) {
      static bool sattr = false;
      if (!sattr) {
        cudaFuncSetAttribute(k_head_soc_lg<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024 - (int)kHeadSocStaticBytes);
        sattr = true;
      }
      k_head_soc_lg<T><<<grid, kHeadLgThreads, vl.total, st>>>(cb, mc, BF, ldbf, hp, out, jout);
    } else {
      k_head_lg<T, 1, 1><<<grid, kHeadLgThreads, sm, st>>>(cb, mc, BF, ldbf, hp, out, jout);
    }
  } else if (ts == 2) {
    k_head_lg<T, 2, 2><<<grid, kHeadLgThreads, sm, st>>>(cb, mc, BF, ldbf, hp, out, jout);
  } else {
    k_head_lg<T, 2, 3><<<grid, kHeadLgThreads, sm, st>>>(cb, mc, BF, ldbf, hp, out, jout);
  }
  return true;
}

template <typename T>
int net_forward(const HostModel& hm, const NetW<T>& w, const HeadParams& hp, JobBatch jb,
                HeadOut out, Arena& ws, size_t max_rows, cudaStream_t st) {
  const ModelConst& mc = hm.mc;
  const int N = jb.N, C = jb.C, d = mc.d;
  const size_t rpj = job_rows(N, C);
  if (jb.n_jobs <= 0) return NQS_OK;
  int jobs_per_chunk = (int)std::max<size_t>(1, max_rows / rpj);
  if (jb.kind == JOB_SOC) jobs_per_chunk = std::max(N, (jobs_per_chunk / N) * N);
  jobs_per_chunk = std::min(jobs_per_chunk, jb.n_jobs);
  const size_t rows_cap = (size_t)jobs_per_chunk * rpj;
  const size_t big = std::max({(size_t)3 * d, (size_t)mc.ff * d, (size_t)2 * mc.K * N});
  const size_t save = ws.used;
  T* X = ws.take<T>(rows_cap * d);
  T* Hb = ws.take<T>(rows_cap * d);
  T* Att = ws.take<T>(rows_cap * d);
  T* Big = ws.take<T>(rows_cap * big);
  if (!X || !Hb || !Att || !Big) {
    set_error("workspace too small for a network chunk of %zu rows", rows_cap);
    return NQS_ERR_WORKSPACE;
  }
  const bool tan = jb.n_tan > 0;
  const bool tcn = sizeof(T) == 4 && w.tc.on;
  static bool attr_set = false;  // per-instantiation one-time opt-in to large shared memory
  if (!attr_set) {
    cudaFuncSetAttribute(k_head<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
    cudaFuncSetAttribute(k_head<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
    cudaFuncSetAttribute(k_head_rt<T, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    cudaFuncSetAttribute(k_head_rt<T, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    cudaFuncSetAttribute(k_head_rt<T, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         200 * 1024);
    attr_set = true;
  }
  for (int j0 = 0; j0 < jb.n_jobs; j0 += jobs_per_chunk) {
    JobBatch cb = jb;
    cb.n_jobs = std::min(jobs_per_chunk, jb.n_jobs - j0);
    if (jb.kind == JOB_SOC) {
      // SOC jobs are N per walker; chunks always hold whole walkers' worth of flips
      cb.w0 = jb.w0 + j0 / N;
    } else {
      cb.w0 = jb.w0 + j0;
    }
    const int rows = (int)(cb.n_jobs * rpj);
    const int ntok = cb.n_jobs * N;
    if constexpr (sizeof(T) == 4) {
      if (C == 1 && (mc.nf == 4 || mc.nf == 8) && d % 4 == 0) {
        const size_t smem = sizeof(float) * ((size_t)(4 * mc.nf + 3) * d);
        if (mc.nf == 8)
          k_embed_value<8><<<(ntok + 127) / 128, 128, smem, st>>>(cb, mc, w.emb_w, w.emb_b, X);
        else
          k_embed_value<4><<<(ntok + 127) / 128, 128, smem, st>>>(cb, mc, w.emb_w, w.emb_b, X);
        NQS_CHECK_LAUNCH("k_embed_value");
      } else {
        k_embed<T><<<(ntok + 7) / 8, 256, 0, st>>>(cb, mc, w.emb_w, w.emb_b, X);
        NQS_CHECK_LAUNCH("k_embed");
      }
    } else {
      k_embed<T><<<(ntok + 7) / 8, 256, 0, st>>>(cb, mc, w.emb_w, w.emb_b, X);
      NQS_CHECK_LAUNCH("k_embed");
    }
    // single-channel rows of the float32 path: each block is one fused launch (block_tc.cu)
    const bool fused = tcn && C == 1 && g_block_fusion && block_value_tc_ok(N, d, mc.H, mc.ff);
    for (int b = 0; b < mc.depth; ++b) {
      const BlockW<T>& bw = w.blk[b];
      if constexpr (sizeof(T) == 4) {
        if (fused) {
          bool done = false;
          NQS_TRY(block_value_tc((float*)X, cb.n_jobs, N, d, mc.H, w.tc, b, bw, st, &done));
          if (done) continue;
        }
      }
      NQS_TRY(launch_layernorm<T>(ntok, C, cb.n_tan, cb.has_lap, d, X, bw.ln0_s, bw.ln0_b, Hb,
                                  st));
      GemmArgs<T> g{};
      if (tcn) {
        NQS_TRY(rowgemm_tc((const float*)Hb, d, rows, d, w.tc.wqkv[b], w.tc.npad_qkv, 3 * d,
                           w.tc.bqkv[b], C, nullptr, 0, (float*)Big, 3 * d, w.tc.err, st, 0,
                           w.tc.bf16 ? w.tc.wqkv16[b] : nullptr));
      } else {
        g.X = Hb; g.ldx = d; g.rows = rows; g.K = d; g.C = C;
        g.Y = Big; g.ldy = 3 * d; g.Res = nullptr; g.ldr = 0; g.trans_w = 0; g.nseg = 3;
        g.seg[0] = GemmSeg<T>{bw.wq, bw.bq, d, d, 0, 0};
        g.seg[1] = GemmSeg<T>{bw.wk, bw.bk, d, d, d, 0};
        g.seg[2] = GemmSeg<T>{bw.wv, bw.bv, d, d, 2 * d, 0};
        NQS_TRY(launch_gemm<T>(g, st));
      }
      NQS_TRY(launch_attention<T>(cb.n_jobs, N, C, cb.n_tan, cb.has_lap, d, mc.H, Big, Att, st,
                                  tcn));
      if (tcn) {
        NQS_TRY(rowgemm_tc((const float*)Att, d, rows, d, w.tc.wo[b], d, d, (const float*)bw.bo,
                           C, (const float*)X, d, (float*)X, d, w.tc.err, st, 0,
                           w.tc.bf16 ? w.tc.wo16[b] : nullptr));
      } else {
        g = GemmArgs<T>{};
        g.X = Att; g.ldx = d; g.rows = rows; g.K = d; g.C = C;
        g.Y = X; g.ldy = d; g.Res = X; g.ldr = d; g.nseg = 1;
        g.seg[0] = GemmSeg<T>{bw.wo, bw.bo, d, d, 0, 0};
        NQS_TRY(launch_gemm<T>(g, st));
      }
      NQS_TRY(launch_layernorm<T>(ntok, C, cb.n_tan, cb.has_lap, d, X, bw.ln1_s, bw.ln1_b, Hb,
                                  st));
      const int D = mc.ff * d;
      // single-channel rows: the GELU runs in the GEMM epilogue
      const bool fuse_act = tcn && C == 1;
      if (tcn) {
        NQS_TRY(rowgemm_tc((const float*)Hb, d, rows, d, w.tc.w0[b], D, D, (const float*)bw.b0, C,
                           nullptr, 0, (float*)Big, D, w.tc.err, st, fuse_act ? 1 : 0,
                           w.tc.bf16 ? w.tc.w016[b] : nullptr));
      } else {
        g = GemmArgs<T>{};
        g.X = Hb; g.ldx = d; g.rows = rows; g.K = d; g.C = C;
        g.Y = Big; g.ldy = D; g.nseg = 1;
        g.seg[0] = GemmSeg<T>{bw.w0, bw.b0, D, D, 0, 0};
        NQS_TRY(launch_gemm<T>(g, st));
      }
      if (!fuse_act) {
        const size_t nel = (size_t)ntok * D;
        if (sizeof(T) == 4 && D % 4 == 0 && ((uintptr_t)Big % 16) == 0) {
          k_gelu4<<<(unsigned)((nel / 4 + 255) / 256), 256, 0, st>>>(
              (size_t)ntok, C, cb.n_tan, cb.has_lap, D, (float*)Big);
          NQS_CHECK_LAUNCH("k_gelu4");
        } else {
          k_gelu<T><<<(unsigned)((nel + 255) / 256), 256, 0, st>>>((size_t)ntok, C, cb.n_tan,
                                                                   cb.has_lap, D, Big);
          NQS_CHECK_LAUNCH("k_gelu");
        }
      }
      if (tcn) {
        NQS_TRY(rowgemm_tc((const float*)Big, D, rows, D, w.tc.w1[b], d, d, (const float*)bw.b1,
                           C, (const float*)X, d, (float*)X, d, w.tc.err, st, 0,
                           w.tc.bf16 ? w.tc.w116[b] : nullptr));
      } else {
        g = GemmArgs<T>{};
        g.X = Big; g.ldx = D; g.rows = rows; g.K = D; g.C = C;
        g.Y = X; g.ldy = d; g.Res = X; g.ldr = d; g.nseg = 1;
        g.seg[0] = GemmSeg<T>{bw.w1, bw.b1, d, d, 0, 0};
        NQS_TRY(launch_gemm<T>(g, st));
      }
    }
    NQS_TRY(launch_layernorm<T>(ntok, C, cb.n_tan, cb.has_lap, d, X, w.lnf_s, w.lnf_b, Hb, st));
    const int KN = mc.K * N;
    if (tcn) {
      NQS_TRY(rowgemm_tc((const float*)Hb, d, rows, d, w.tc.wbf, w.tc.npad_bf, 2 * KN,
                         (const float*)w.bf_b_re, C, nullptr, 0, (float*)Big, 2 * KN, w.tc.err,
                         st, 0, w.tc.bf16 ? w.tc.wbf16 : nullptr));
    } else {
      GemmArgs<T> g{};
      g.X = Hb; g.ldx = d; g.rows = rows; g.K = d; g.C = C;
      g.Y = Big; g.ldy = 2 * KN; g.nseg = 2;
      g.seg[0] = GemmSeg<T>{w.bf_w_re, w.bf_b_re, KN, KN, 0, 0};
      g.seg[1] = GemmSeg<T>{w.bf_w_im, w.bf_b_im, KN, KN, KN, 0};
      NQS_TRY(launch_gemm<T>(g, st));
    }
    const int jout = j0;
    if (N <= kHeadTok) {
      const bool lap = tan && cb.has_lap;
      const HeadRtPlan rp = head_rt_plan(N, mc.nG, mc.K, cb.n_tan, tan, lap);
      const unsigned rg = (unsigned)((cb.n_jobs + rp.jpc - 1) / rp.jpc);
      if (rp.bytes > 200 * 1024) {
        set_error("head: %zu bytes of shared memory per CTA", rp.bytes);
        return NQS_ERR_UNSUPPORTED;
      }
      if (lap)
        k_head_rt<T, true, true><<<rg, 64, rp.bytes, st>>>(cb, mc, Big, 2 * KN, hp, out, jout,
                                                           rp.jpc, rp.job_bytes, rp.hw_bytes);
      else if (tan)
        k_head_rt<T, true, false><<<rg, 64, rp.bytes, st>>>(cb, mc, Big, 2 * KN, hp, out, jout,
                                                            rp.jpc, rp.job_bytes, rp.hw_bytes);
      else
        k_head_rt<T, false, false><<<rg, 64, rp.bytes, st>>>(cb, mc, Big, 2 * KN, hp, out, jout,
                                                             rp.jpc, rp.job_bytes, rp.hw_bytes);
      NQS_CHECK_LAUNCH("k_head_rt");
      continue;
    }
    if (g_large_n_cta && launch_head_lg<T>(mc, cb, Big, 2 * KN, hp, out, jout, st)) {
      NQS_CHECK_LAUNCH("k_head_lg");
      continue;
    }
    const HeadPlan hpl = head_plan(N, mc.nG, mc.K, cb.n_tan, tan);
    const unsigned hgrid = (unsigned)((cb.n_jobs + hpl.jpc - 1) / hpl.jpc);
    if (tan) {
      k_head<T, true><<<hgrid, 32 * hpl.wpc, hpl.bytes, st>>>(cb, mc, Big, 2 * KN, hp, out, jout,
                                                              hpl.jpc, hpl.job_bytes,
                                                              hpl.warp_bytes);
    } else {
      k_head<T, false><<<hgrid, 32 * hpl.wpc, hpl.bytes, st>>>(cb, mc, Big, 2 * KN, hp, out, jout,
                                                               hpl.jpc, hpl.job_bytes,
                                                               hpl.warp_bytes);
    }
    NQS_CHECK_LAUNCH("k_head");
  }
  ws.used = save;
  return NQS_OK;
}

// ============================================================================================
// parameter pointers
// ============================================================================================
template <typename T>
NetW<T> make_netw(const NqsModelDesc& d, const T* th, const double* theta64) {
  NetW<T> w{};
  auto P = [&](int64_t off) -> const T* { return off >= 0 ? th + off : nullptr; };
  w.emb_w = P(d.off_embed_kernel);
  w.emb_b = P(d.off_embed_bias);
  for (int b = 0; b < d.depth; ++b) {
    const int64_t* o = d.off_block[b];
    BlockW<T>& bw = w.blk[b];
    bw.ln0_s = P(o[NQS_B_LN0_SCALE]);
    bw.ln0_b = P(o[NQS_B_LN0_BIAS]);
    bw.ln1_s = P(o[NQS_B_LN1_SCALE]);
    bw.ln1_b = P(o[NQS_B_LN1_BIAS]);
    bw.wq = P(o[NQS_B_Q_KERNEL]);
    bw.bq = P(o[NQS_B_Q_BIAS]);
    bw.wk = P(o[NQS_B_K_KERNEL]);
    bw.bk = P(o[NQS_B_K_BIAS]);
    bw.wv = P(o[NQS_B_V_KERNEL]);
    bw.bv = P(o[NQS_B_V_BIAS]);
    bw.wo = P(o[NQS_B_O_KERNEL]);
    bw.bo = P(o[NQS_B_O_BIAS]);
    bw.w0 = P(o[NQS_B_DENSE0_KERNEL]);
    bw.b0 = P(o[NQS_B_DENSE0_BIAS]);
    bw.w1 = P(o[NQS_B_DENSE1_KERNEL]);
    bw.b1 = P(o[NQS_B_DENSE1_BIAS]);
  }
  w.lnf_s = P(d.off_final_ln_scale);
  w.lnf_b = P(d.off_final_ln_bias);
  const int64_t KN = (int64_t)d.n_dets * d.n_elec;
  const int64_t nk = (int64_t)d.embed_dim * KN;
  w.bf_w_re = P(d.off_backflow_kernel);
  w.bf_w_im = P(d.off_backflow_kernel + nk);
  w.bf_b_re = P(d.off_backflow_bias);
  w.bf_b_im = P(d.off_backflow_bias + KN);
  w.theta = theta64;
  return w;
}

HeadParams make_head_params(const NqsModelDesc& d, const double* th) {
  HeadParams h{};
  auto P = [&](int64_t off) -> const double* { return off >= 0 ? th + off : nullptr; };
  h.det_logw = P(d.off_det_logw);
  h.jas_same = P(d.off_jas_c_same);
  h.jas_opp = P(d.off_jas_c_opp);
  h.jas_loga = P(d.off_jastrow_loga);
  h.dW = P(d.off_dW);
  return h;
}

__global__ void k_theta_f32(const double* __restrict__ a, float* __restrict__ b, int64_t n) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}
int theta_to_f32(const double* theta, float* out, int64_t n, cudaStream_t st) {
  k_theta_f32<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(theta, out, n);
  NQS_CHECK_LAUNCH("k_theta_f32");
  return NQS_OK;
}

template size_t net_scratch_bytes<double>(const ModelConst&, size_t);
template size_t net_scratch_bytes<float>(const ModelConst&, size_t);
template int net_forward<double>(const HostModel&, const NetW<double>&, const HeadParams&,
                                 JobBatch, HeadOut, Arena&, size_t, cudaStream_t);
template int net_forward<float>(const HostModel&, const NetW<float>&, const HeadParams&, JobBatch,
                                HeadOut, Arena&, size_t, cudaStream_t);
template NetW<double> make_netw<double>(const NqsModelDesc&, const double*, const double*);
template NetW<float> make_netw<float>(const NqsModelDesc&, const float*, const double*);

}  // namespace nqs
