// vmc.cu — C ABI entry points of libnqs: model handle, log psi, forward-Laplacian local energy,
// fused Metropolis sweeps. Reference semantics are cited per function in include/nqs.h.
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <algorithm>
#include <vector>
#include <cmath>
#include <atomic>

#include "net_kernels.cuh"

struct NqsModel {
  nqs::HostModel hm;
  bool fl_ok;  // forward-Laplacian head fits in shared memory
};

namespace nqs {

static thread_local char g_err[512] = "";
std::atomic<unsigned long long> g_launches{0};
std::atomic<unsigned> g_wait_limit{0};
cudaEvent_t g_prof_start = nullptr, g_prof_stop = nullptr;

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

int cuda_status(cudaError_t e, const char* what) {
  set_error("%s: %s", what, cudaGetErrorString(e));
  return NQS_ERR_CUDA;
}

size_t head_smem_host(int N, int nG, int K, int n_tan, bool tan) {
  return head_job_bytes(N, nG, K, tan ? n_tan : 0) + head_warp_bytes(N, tan);
}

// rows of one chunk for a batch (whole jobs; SOC chunks hold whole walkers)
static size_t chunk_rows(int kind, int n_jobs, int N, int C, size_t max_rows) {
  const size_t rpj = job_rows(N, C);
  size_t jpc = std::max<size_t>(1, max_rows / rpj);
  if (kind == JOB_SOC) jpc = std::max<size_t>((size_t)N, (jpc / N) * N);
  jpc = std::min<size_t>(jpc, (size_t)std::max(n_jobs, 1));
  return jpc * rpj;
}

// ============================================================================================
// Metropolis kernels (src/nqs/sampler.py:36-57)
// ============================================================================================
__device__ __forceinline__ double jmod1(double x) {
  double r = fmod(x, 1.0);  // jnp.mod(x, 1.0) semantics
  if (r != 0.0 && r < 0.0) r += 1.0;
  return r;
}

struct McArgs {
  int W, N, n_flips;
  double step;
  uint64_t seed, sweep;  // global sweep index = counter + s
  int s;                 // sweep index within the call (for injected buffers)
  const uint64_t* counter_dev;  // nullable: sweep = *counter_dev + s, read at run time
  double A[4], Ainv[4];
  const double* inj_normals;
  const double* inj_u_pos;
  const int32_t* inj_flip;
  const double* inj_u_flip;
};

__device__ __forceinline__ u32x4 mc_draw(const McArgs& a, int w, uint32_t draw) {
  const uint64_t sw = a.counter_dev ? *a.counter_dev + (uint64_t)a.s : a.sweep;
  return philox4x32_10(u32x4{(uint32_t)w, draw, (uint32_t)sw, (uint32_t)(sw >> 32)}, a.seed);
}

__global__ void k_counter_add(uint64_t* c, uint64_t n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *c += n;
}

__global__ void k_propose_pos(McArgs a, const double* __restrict__ R, double* __restrict__ Rp) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;  // (walker, electron)
  if (idx >= a.W * a.N) return;
  const int w = idx / a.N, i = idx - w * a.N;
  double n0, n1;
  if (a.inj_normals) {
    const double* p = a.inj_normals + (((size_t)a.s * a.W + w) * a.N + i) * 2;
    n0 = p[0];
    n1 = p[1];
  } else {
    const u32x4 r = mc_draw(a, w, (uint32_t)i);
    const double u1 = u01_53(r.x, r.y), u2 = u01_53(r.z, r.w);
    const double rad = sqrt(-2.0 * log(1.0 - u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    n0 = rad * c;
    n1 = rad * s;
  }
  // R + step*N(0,1), wrapped: mod(r A^-T, 1) A^T, every product rounded separately (no FMA)
  const double x = __dadd_rn(R[(size_t)idx * 2], __dmul_rn(a.step, n0));
  const double y = __dadd_rn(R[(size_t)idx * 2 + 1], __dmul_rn(a.step, n1));
  const double f0 = jmod1(__dadd_rn(__dmul_rn(x, a.Ainv[0]), __dmul_rn(y, a.Ainv[1])));
  const double f1 = jmod1(__dadd_rn(__dmul_rn(x, a.Ainv[2]), __dmul_rn(y, a.Ainv[3])));
  Rp[(size_t)idx * 2] = __dadd_rn(__dmul_rn(f0, a.A[0]), __dmul_rn(f1, a.A[1]));
  Rp[(size_t)idx * 2 + 1] = __dadd_rn(__dmul_rn(f0, a.A[2]), __dmul_rn(f1, a.A[3]));
}

__device__ __forceinline__ bool mh_accept(double d, double u) {
  return u < exp(fmin(0.0, d));  // sampler.py:41,52 (strict <)
}

__global__ void k_accept_pos(McArgs a, double* __restrict__ R, const double* __restrict__ Rp,
                             cplx* __restrict__ Lc, const cplx* __restrict__ Lp,
                             double* __restrict__ acc_pos, double* __restrict__ out_d) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= a.W) return;
  const double d = __dsub_rn(2.0 * Lp[w].re, 2.0 * Lc[w].re);
  double u;
  if (a.inj_u_pos) {
    u = a.inj_u_pos[(size_t)a.s * a.W + w];
  } else {
    const u32x4 r = mc_draw(a, w, (uint32_t)a.N);
    u = u01_53(r.x, r.y);
  }
  const bool acc = mh_accept(d, u);
  if (out_d) out_d[((size_t)a.s * (1 + a.n_flips)) * a.W + w] = d;
  if (acc) {
    for (int i = 0; i < 2 * a.N; ++i) R[(size_t)w * 2 * a.N + i] = Rp[(size_t)w * 2 * a.N + i];
    Lc[w] = Lp[w];
    if (acc_pos) acc_pos[w] += 1.0;
  }
}

__global__ void k_propose_flip(McArgs a, int j, int32_t* __restrict__ flip) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= a.W) return;
  int i;
  if (a.inj_flip) {
    i = a.inj_flip[((size_t)a.s * a.n_flips + j) * a.W + w];
  } else {
    const u32x4 r = mc_draw(a, w, (uint32_t)(a.N + 1 + j));
    i = (int)(((uint64_t)r.z * (uint64_t)a.N) >> 32);
  }
  flip[w] = i;
}

__global__ void k_accept_flip(McArgs a, int j, int32_t* __restrict__ S,
                              const int32_t* __restrict__ flip, cplx* __restrict__ Lc,
                              const cplx* __restrict__ Lp, double* __restrict__ acc_spin,
                              double* __restrict__ out_d) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= a.W) return;
  const double d = __dsub_rn(2.0 * Lp[w].re, 2.0 * Lc[w].re);
  double u;
  if (a.inj_u_flip) {
    u = a.inj_u_flip[((size_t)a.s * a.n_flips + j) * a.W + w];
  } else {
    const u32x4 r = mc_draw(a, w, (uint32_t)(a.N + 1 + j));
    u = u01_53(r.x, r.y);
  }
  const bool acc = mh_accept(d, u);
  if (out_d) out_d[((size_t)a.s * (1 + a.n_flips) + 1 + j) * a.W + w] = d;
  if (acc) {
    const int i = flip[w];
    S[(size_t)w * a.N + i] = 1 - S[(size_t)w * a.N + i];
    Lc[w] = Lp[w];
    if (acc_spin) acc_spin[w] += 1.0;
  }
}

__global__ void k_scale(double* x, int n, double s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) x[i] *= s;
}

// ============================================================================================
// local energy assembly (src/nqs/local_energy.py:63-115)
// ============================================================================================
__global__ void k_eloc_assemble(int W, int N, const cplx* __restrict__ L0,
                                const cplx* __restrict__ g, const cplx* __restrict__ lap,
                                const cplx* __restrict__ Lf, const cplx* __restrict__ gf,
                                const int32_t* __restrict__ S, const double* __restrict__ coul,
                                const double* __restrict__ field, double m_star, double lambda_r,
                                double h_z, cplx* __restrict__ out) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= W) return;
  cplx g2 = mk(0, 0);
  for (int t = 0; t < 2 * N; ++t) cfma(g2, g[(size_t)w * 2 * N + t], g[(size_t)w * 2 * N + t]);
  const cplx kin = cscale(cadd(lap[w], g2), -1.0 / (2.0 * m_star));
  double sg = 0.0, fz = 0.0;
  for (int i = 0; i < N; ++i) {
    const double sz = 1.0 - 2.0 * (double)S[(size_t)w * N + i];
    sg += sz;
    if (field) fz += field[((size_t)w * N + i) * 3 + 2] * sz;  // sum_i f_z(r_i) (sigma_z)_ss
  }
  const double ez = -0.5 * h_z * sg - fz;
  cplx soc = mk(0, 0);
  if (Lf) {
    const cplx l0 = L0[w];
    for (int i = 0; i < N; ++i) {
      const size_t j = (size_t)w * N + i;
      const cplx ratio = cexp_(csub(Lf[j], l0));
      cplx ax = cmul(ratio, gf[2 * j]);
      cplx ay = cmul(ratio, gf[2 * j + 1]);
      if (!cfinite(ax)) ax = mk(0, 0);
      if (!cfinite(ay)) ay = mk(0, 0);
      // lambda (sx (-i) ampgy + sy (-i) ampgx), sx = 1, sy = -i (s=0) / +i (s=1)
      const double sgy = S[j] == 0 ? -1.0 : 1.0;
      const cplx e = cadd(cmul(mk(0, -1), ay), cscale(ax, sgy));
      soc = cadd(soc, cscale(e, lambda_r));
      if (field) {  // -(f_x sigma_x + f_y sigma_y)_{s s'} Psi(s')/Psi(s): sigma_y = i sgy
        const double* f = field + j * 3;
        soc = csub(soc, cmul(mk(f[0], f[1] * sgy), ratio));
      }
    }
  }
  cplx e = cadd(cadd(kin, mk(ez, 0.0)), soc);
  if (coul) e.re += coul[w];
  out[w] = e;
}

// single-particle spin estimators from the flip ratios (observables.py:31-45):
// ratio_i = exp(L(flip i) - L) (non-finite -> 0), sx = ratio, sy = -i sz ratio, sz = 1 - 2 s_i
__global__ void k_spin_estimators(int W, int N, const cplx* __restrict__ L0,
                                  const cplx* __restrict__ Lf, const int32_t* __restrict__ S,
                                  cplx* __restrict__ sx, cplx* __restrict__ sy,
                                  double* __restrict__ sz) {
  const size_t j = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= (size_t)W * N) return;
  cplx r = cexp_(csub(Lf[j], L0[j / N]));
  if (!cfinite(r)) r = mk(0, 0);
  const double z = 1.0 - 2.0 * (double)S[j];
  sx[j] = r;
  sy[j] = mk(z * r.im, -z * r.re);  // -i z r
  sz[j] = z;
}

}  // namespace nqs

using namespace nqs;

// ============================================================================================
// model handle
// ============================================================================================
static int validate_desc(const NqsModelDesc* d) {
  if (!d) return NQS_ERR_INVALID_ARG;
  if (d->n_elec < 1 || d->embed_dim < 1 || d->depth < 0 || d->n_heads < 1 || d->ff_mult < 1 ||
      d->n_freq < 1 || d->n_dets < 1 || d->n_g < 1 || d->n_params < 1) {
    set_error("model descriptor: non-positive size");
    return NQS_ERR_INVALID_ARG;
  }
  if (d->n_elec > NQS_MAX_ELEC || d->embed_dim > NQS_MAX_EMBED || d->depth > NQS_MAX_DEPTH ||
      d->n_freq > NQS_MAX_FREQ || d->n_dets > NQS_MAX_DETS ||
      (d->use_jastrow && d->jastrow_kind == 0 && d->n_knots > NQS_MAX_KNOTS) ||
      (d->embed_dim % d->n_heads) != 0) {
    set_error("model descriptor outside compiled limits (N<=%d, d<=%d, depth<=%d, n_freq<=%d, "
              "K<=%d, heads | d)",
              NQS_MAX_ELEC, NQS_MAX_EMBED, NQS_MAX_DEPTH, NQS_MAX_FREQ, NQS_MAX_DETS);
    return NQS_ERR_UNSUPPORTED;
  }
  if (!d->Gs_host || !d->W_host) {
    set_error("model descriptor: envelope pointers are null");
    return NQS_ERR_INVALID_ARG;
  }
  const int64_t P = d->n_params;
  const int64_t dd = d->embed_dim, D = (int64_t)d->ff_mult * dd, KN = (int64_t)d->n_dets * d->n_elec;
  auto chk = [&](int64_t off, int64_t n) { return off >= 0 && off + n <= P; };
  bool ok = chk(d->off_final_ln_bias, dd) && chk(d->off_final_ln_scale, dd) &&
            chk(d->off_embed_bias, dd) && chk(d->off_embed_kernel, (4 * d->n_freq + 2) * dd) &&
            chk(d->off_backflow_bias, 2 * KN) && chk(d->off_backflow_kernel, 2 * dd * KN);
  for (int b = 0; b < d->depth && ok; ++b) {
    const int64_t* o = d->off_block[b];
    ok = chk(o[NQS_B_DENSE0_BIAS], D) && chk(o[NQS_B_DENSE0_KERNEL], dd * D) &&
         chk(o[NQS_B_DENSE1_BIAS], dd) && chk(o[NQS_B_DENSE1_KERNEL], D * dd) &&
         chk(o[NQS_B_LN0_BIAS], dd) && chk(o[NQS_B_LN0_SCALE], dd) && chk(o[NQS_B_LN1_BIAS], dd) &&
         chk(o[NQS_B_LN1_SCALE], dd);
    for (int q = NQS_B_K_BIAS; q <= NQS_B_V_KERNEL && ok; q += 2)
      ok = chk(o[q], dd) && chk(o[q + 1], dd * dd);
  }
  if (ok && d->n_dets > 1) ok = chk(d->off_det_logw, 2 * d->n_dets);
  if (ok && d->learnable_env) ok = chk(d->off_dW, 2LL * d->n_elec * d->n_g * 2);
  if (ok && d->use_jastrow) {
    if (d->jastrow_kind == 0)
      ok = chk(d->off_jas_c_same, d->n_knots) && chk(d->off_jas_c_opp, d->n_knots) && d->knots_host;
    else
      ok = chk(d->off_jastrow_loga, 1);
  }
  if (!ok) {
    set_error("model descriptor: a parameter offset is missing or out of range");
    return NQS_ERR_INVALID_ARG;
  }
  const double det = d->A[0] * d->A[3] - d->A[1] * d->A[2];
  if (det == 0.0) {
    set_error("model descriptor: singular cell");
    return NQS_ERR_INVALID_ARG;
  }
  if (head_smem_host(d->n_elec, d->n_g, d->n_dets, 0, false) > 210 * 1024) {
    set_error("model: N=%d, n_g=%d exceeds the determinant kernel's shared memory", d->n_elec,
              d->n_g);
    return NQS_ERR_UNSUPPORTED;
  }
  return NQS_OK;
}

extern "C" {

int nqs_version(void) { return 1; }

const char* nqs_status_string(int s) {
  switch (s) {
    case NQS_OK: return "ok";
    case NQS_ERR_INVALID_ARG: return "invalid argument";
    case NQS_ERR_UNSUPPORTED: return "unsupported shape";
    case NQS_ERR_WORKSPACE: return "workspace too small";
    case NQS_ERR_CUDA: return "CUDA error";
    case NQS_ERR_NONFINITE: return "non-finite value";
    case NQS_ERR_TIMEOUT: return "device wait timed out";
    case NQS_ERR_NOT_SPD: return "matrix not positive definite";
    default: return "unknown status";
  }
}

const char* nqs_last_error(void) { return g_err; }

unsigned long long nqs_kernel_launches(void) { return g_launches.load(); }

int nqs_set_wait_limit(unsigned polls) {
  g_wait_limit.store(polls, std::memory_order_relaxed);
  return NQS_OK;
}

int nqs_profile_events(void* start, void* stop) {
  g_prof_start = (cudaEvent_t)start;
  g_prof_stop = (cudaEvent_t)stop;
  return NQS_OK;
}

int nqs_model_create(const NqsModelDesc* d, NqsModel** out) {
  if (!out) return NQS_ERR_INVALID_ARG;
  NQS_TRY(validate_desc(d));
  NqsModel* m = new NqsModel();
  HostModel& hm = m->hm;
  hm.desc = *d;
  hm.desc.Gs_host = hm.desc.W_host = hm.desc.knots_host = nullptr;
  ModelConst& mc = hm.mc;
  mc.N = d->n_elec;
  mc.d = d->embed_dim;
  mc.depth = d->depth;
  mc.H = d->n_heads;
  mc.ff = d->ff_mult;
  mc.nf = d->n_freq;
  mc.K = d->n_dets;
  mc.nG = d->n_g;
  mc.learnable_env = d->learnable_env;
  mc.use_jastrow = d->use_jastrow;
  mc.jastrow_kind = d->jastrow_kind;
  mc.n_knots = d->n_knots;
  mc.cusp = d->cusp;
  for (int i = 0; i < 4; ++i) mc.A[i] = d->A[i];
  const double det = d->A[0] * d->A[3] - d->A[1] * d->A[2];
  if (d->A[1] == 0.0 && d->A[2] == 0.0) {  // diagonal cell: 1/a exactly, as LAPACK's inverse
    mc.Ainv[0] = 1.0 / d->A[0];
    mc.Ainv[1] = mc.Ainv[2] = 0.0;
    mc.Ainv[3] = 1.0 / d->A[3];
  } else {
    mc.Ainv[0] = d->A[3] / det;
    mc.Ainv[1] = -d->A[1] / det;
    mc.Ainv[2] = -d->A[2] / det;
    mc.Ainv[3] = d->A[0] / det;
  }
  const double area = std::fabs(det);
  mc.rcut = 0.5 * std::sqrt(area);
  mc.wdt = mc.rcut / std::max(d->n_knots - 1, 1);
  const size_t nGs = (size_t)d->n_g * 2, nW = (size_t)d->n_elec * d->n_g * 2 * 2;
  const size_t nk = (d->use_jastrow && d->jastrow_kind == 0) ? (size_t)d->n_knots : 1;
  cudaError_t ce;
  if ((ce = cudaMalloc(&hm.d_Gs, nGs * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&hm.d_W, nW * sizeof(double))) != cudaSuccess ||
      (ce = cudaMalloc(&hm.d_knots, nk * sizeof(double))) != cudaSuccess) {
    delete m;
    return cuda_status(ce, "nqs_model_create: cudaMalloc");
  }
  cudaMemcpy(hm.d_Gs, d->Gs_host, nGs * sizeof(double), cudaMemcpyHostToDevice);
  cudaMemcpy(hm.d_W, d->W_host, nW * sizeof(double), cudaMemcpyHostToDevice);
  std::vector<double> kn(nk, 0.0);
  if (nk > 1 || (d->use_jastrow && d->jastrow_kind == 0 && d->knots_host))
    for (size_t i = 0; i < nk; ++i) kn[i] = d->knots_host[i];
  mc.knots_uniform = nk > 1;
  for (size_t i = 0; i < nk && mc.knots_uniform; ++i)
    if (std::fabs(kn[i] - (double)i * mc.wdt) > 1e-12 * mc.rcut) mc.knots_uniform = 0;
  ce = cudaMemcpy(hm.d_knots, kn.data(), nk * sizeof(double), cudaMemcpyHostToDevice);
  if (ce != cudaSuccess) {
    nqs_model_destroy(m);
    return cuda_status(ce, "nqs_model_create: cudaMemcpy");
  }
  mc.Gs = hm.d_Gs;
  mc.W = hm.d_W;
  mc.knots = hm.d_knots;
  m->fl_ok = head_smem_host(d->n_elec, d->n_g, d->n_dets, 2 * d->n_elec, true) <= 210 * 1024;
  *out = m;
  return NQS_OK;
}

int nqs_model_destroy(NqsModel* m) {
  if (!m) return NQS_OK;
  cudaFree(m->hm.d_Gs);
  cudaFree(m->hm.d_W);
  cudaFree(m->hm.d_knots);
  delete m;
  return NQS_OK;
}

int64_t nqs_model_n_params(const NqsModel* m) { return m ? m->hm.desc.n_params : -1; }

}  // extern "C"

// ============================================================================================
// workspace planning
// ============================================================================================
namespace {

struct Plan {
  size_t bytes = 0;
  void add(size_t n) { bytes += ((n + 255) / 256) * 256 + 256; }
};

size_t net_bytes(const ModelConst& mc, int prec, size_t rows) {
  return prec == NQS_PREC_FP64 ? net_scratch_bytes<double>(mc, rows)
                               : net_scratch_bytes<float>(mc, rows);
}

size_t plan_bytes(const NqsModel* m, int op, int W, int prec) {
  const ModelConst& mc = m->hm.mc;
  const int N = mc.N;
  Plan p;
  if (prec != NQS_PREC_FP64) p.add(sizeof(float) * m->hm.desc.n_params);
  if (prec == NQS_PREC_MIXED || prec == NQS_PREC_MIXED_BF16)
    p.add(tc_weights_bytes(m->hm.desc, prec == NQS_PREC_MIXED_BF16));
  switch (op) {
    case NQS_OP_LOGPSI:
      p.add(net_bytes(mc, prec, chunk_rows(JOB_VALUE, W, N, 1, kMaxRows)));
      break;
    case NQS_OP_LOCAL_E: {
      p.add(sizeof(cplx) * (size_t)W * (2 * N + 2));  // L0, g, lap
      p.add(sizeof(cplx) * (size_t)W * N * 3);        // Lf, gf
      p.add(sizeof(double) * W);                      // coulomb
      const size_t r1 = chunk_rows(JOB_FLAP, W, N, 2 * N + 2, kMaxRows);
      const size_t r2 = chunk_rows(JOB_SOC, W * N, N, 3, kMaxRows);
      p.add(net_bytes(mc, prec, std::max(r1, r2)));
      break;
    }
    case NQS_OP_MCMC:
      p.add(sizeof(double) * (size_t)W * N * 2);  // proposal positions
      p.add(sizeof(cplx) * (size_t)W * 2);        // current / proposed log psi
      p.add(sizeof(int32_t) * (size_t)W);         // flip indices
      p.add(net_bytes(mc, prec, chunk_rows(JOB_VALUE, W, N, 1, kMaxRows)));
      break;
    case NQS_OP_PER_SAMPLE_O:
    case NQS_OP_PER_SAMPLE_O_CKPT:
    case NQS_OP_LOGPSI_VJP:
    case NQS_OP_LOGPSI_VJP_CKPT: {
      const bool ckpt = op == NQS_OP_PER_SAMPLE_O_CKPT || op == NQS_OP_LOGPSI_VJP_CKPT;
      p.add(prec == NQS_PREC_FP64 ? backward_scratch<double>(mc, W, ckpt)
                                  : backward_scratch<float>(mc, W, ckpt));
      break;
    }
    default:
      return 0;
  }
  return p.bytes;
}

struct Ctx {
  Arena ws;
  const double* theta64;
  const float* theta32;
  TcNet tc;
};

int begin(NqsModel* m, const double* theta, int prec, void* wsp, size_t wsb, cudaStream_t st,
          Ctx* c) {
  if (!m || !theta) {
    set_error("null model or theta");
    return NQS_ERR_INVALID_ARG;
  }
  if (prec != NQS_PREC_FP64 && prec != NQS_PREC_MIXED && prec != NQS_PREC_MIXED_SIMT &&
      prec != NQS_PREC_MIXED_BF16) {
    set_error("unknown precision %d", prec);
    return NQS_ERR_INVALID_ARG;
  }
  c->ws = Arena{(char*)wsp, wsb, 0};
  c->theta64 = theta;
  c->theta32 = nullptr;
  if (prec != NQS_PREC_FP64) {
    float* t32 = c->ws.take<float>(m->hm.desc.n_params);
    if (!t32) {
      set_error("workspace too small");
      return NQS_ERR_WORKSPACE;
    }
    NQS_TRY(theta_to_f32(theta, t32, m->hm.desc.n_params, st));
    c->theta32 = t32;
  }
  c->tc = TcNet{};
  if (prec == NQS_PREC_MIXED || prec == NQS_PREC_MIXED_BF16)
    NQS_TRY(build_tc_weights(m->hm.desc, c->theta32, c->ws, &c->tc, st,
                             prec == NQS_PREC_MIXED_BF16));
  return NQS_OK;
}

// A bounded wait that ran out in a tensor-core row GEMM or fused block of this call (*err set)
// leaves that pass's activations incomplete: every log psi, gradient and Laplacian the batch
// produced becomes NaN, so the entry point's outputs (log psi, E_loc, O's forward inputs, the
// Metropolis ratios, which then reject) carry the failure to the caller instead of wrong numbers.
__global__ void k_poison_on_timeout(const int* __restrict__ err, cplx* __restrict__ L, size_t nL,
                                    cplx* __restrict__ dL, size_t ndL, cplx* __restrict__ lap) {
  if (!*err) return;
  const double nan = __longlong_as_double(0x7ff8000000000000ll);
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nL; i += stride) {
    if (L) L[i] = cplx{nan, nan};
    if (lap) lap[i] = cplx{nan, nan};
  }
  if (dL)
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < ndL; i += stride)
      dL[i] = cplx{nan, nan};
}

int run_net(NqsModel* m, Ctx& c, int prec, const JobBatch& jb, HeadOut out, cudaStream_t st) {
  const HeadParams hp = make_head_params(m->hm.desc, c.theta64);
  if (prec == NQS_PREC_FP64) {
    const NetW<double> w = make_netw<double>(m->hm.desc, c.theta64, c.theta64);
    return net_forward<double>(m->hm, w, hp, jb, out, c.ws, kMaxRows, st);
  }
  NetW<float> w = make_netw<float>(m->hm.desc, c.theta32, c.theta64);
  w.tc = c.tc;
  NQS_TRY(net_forward<float>(m->hm, w, hp, jb, out, c.ws, kMaxRows, st));
  if (c.tc.err) {
    k_poison_on_timeout<<<64, 256, 0, st>>>(c.tc.err, out.L, (size_t)jb.n_jobs, out.dL,
                                            (size_t)jb.n_jobs * jb.n_tan, out.lap);
    NQS_CHECK_LAUNCH("k_poison_on_timeout");
  }
  return NQS_OK;
}

int check_ws(NqsModel* m, int op, int W, int prec, size_t wsb) {
  const size_t need = plan_bytes(m, op, W, prec);
  if (wsb < need) {
    set_error("workspace %zu bytes < required %zu", wsb, need);
    return NQS_ERR_WORKSPACE;
  }
  return NQS_OK;
}

}  // namespace

extern "C" {

int nqs_workspace_size(const NqsModel* m, int op, int W, int prec, size_t* bytes) {
  if (!m || !bytes || W < 0) return NQS_ERR_INVALID_ARG;
  *bytes = plan_bytes(m, op, W, prec);
  return NQS_OK;
}

int nqs_logpsi(NqsModel* m, const double* theta, const double* R, const int32_t* S, int W,
               double* out_logpsi, int prec, void* wsp, size_t wsb, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (W < 0 || (W > 0 && (!R || !S || !out_logpsi))) return NQS_ERR_INVALID_ARG;
  if (W == 0) return NQS_OK;
  NQS_TRY(check_ws(m, NQS_OP_LOGPSI, W, prec, wsb));
  Ctx c;
  NQS_TRY(begin(m, theta, prec, wsp, wsb, st, &c));
  JobBatch jb{JOB_VALUE, W, m->hm.mc.N, 1, 0, 0, 0, R, S, nullptr};
  return run_net(m, c, prec, jb, HeadOut{(cplx*)out_logpsi, nullptr, nullptr}, st);
}

int nqs_spin_estimators(NqsModel* m, const double* theta, const double* R, const int32_t* S,
                        int W, double* out_sx, double* out_sy, double* out_sz, int prec,
                        void* wsp, size_t wsb, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (W < 0 || (W > 0 && (!R || !S || !out_sx || !out_sy || !out_sz)))
    return NQS_ERR_INVALID_ARG;
  if (W == 0) return NQS_OK;
  NQS_TRY(check_ws(m, NQS_OP_LOCAL_E, W, prec, wsb));
  Ctx c;
  NQS_TRY(begin(m, theta, prec, wsp, wsb, st, &c));
  const int N = m->hm.mc.N;
  cplx* L0 = c.ws.take<cplx>(W);
  cplx* Lf = c.ws.take<cplx>((size_t)W * N);
  if (!Lf) return NQS_ERR_WORKSPACE;
  JobBatch jb{JOB_VALUE, W, N, 1, 0, 0, 0, R, S, nullptr};
  NQS_TRY(run_net(m, c, prec, jb, HeadOut{L0, nullptr, nullptr}, st));
  // the N single-spin flips of every walker, values only
  JobBatch fb{JOB_SOC, W * N, N, 1, 0, 0, 0, R, S, nullptr};
  NQS_TRY(run_net(m, c, prec, fb, HeadOut{Lf, nullptr, nullptr}, st));
  const size_t n = (size_t)W * N;
  k_spin_estimators<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(
      W, N, L0, Lf, S, (cplx*)out_sx, (cplx*)out_sy, out_sz);
  NQS_CHECK_LAUNCH("k_spin_estimators");
  return NQS_OK;
}

static int local_energy_impl(NqsModel* m, const double* theta, const double* R, const int32_t* S,
                             int W, double m_star, double lambda_r, double h_z,
                             const NqsEwald* ewald, const double* field, double* out_eloc,
                             double* out_logpsi, double* out_grad, double* out_lap, int prec,
                             void* wsp, size_t wsb, cudaStream_t st, bool energy) {
  if (W < 0 || (W > 0 && (!R || !S))) return NQS_ERR_INVALID_ARG;
  if (W == 0) return NQS_OK;
  if (!m->fl_ok) {
    set_error("forward-Laplacian head does not fit in shared memory for N=%d", m->hm.mc.N);
    return NQS_ERR_UNSUPPORTED;
  }
  NQS_TRY(check_ws(m, NQS_OP_LOCAL_E, W, prec, wsb));
  Ctx c;
  NQS_TRY(begin(m, theta, prec, wsp, wsb, st, &c));
  const int N = m->hm.mc.N;
  cplx* L0 = c.ws.take<cplx>(W);
  cplx* g = c.ws.take<cplx>((size_t)W * 2 * N);
  cplx* lap = c.ws.take<cplx>(W);
  cplx* Lf = c.ws.take<cplx>((size_t)W * N);
  cplx* gf = c.ws.take<cplx>((size_t)W * N * 2);
  double* coul = c.ws.take<double>(W);
  if (!coul) return NQS_ERR_WORKSPACE;
  JobBatch fl{JOB_FLAP, W, N, 2 * N + 2, 2 * N, 1, 0, R, S, nullptr};
  NQS_TRY(run_net(m, c, prec, fl, HeadOut{L0, g, lap}, st));
  if (!energy) {
    if (out_logpsi) cudaMemcpyAsync(out_logpsi, L0, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st);
    if (out_grad)
      cudaMemcpyAsync(out_grad, g, sizeof(cplx) * W * 2 * N, cudaMemcpyDeviceToDevice, st);
    if (out_lap) cudaMemcpyAsync(out_lap, lap, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st);
    NQS_CHECK_LAUNCH("copy outputs");
    return NQS_OK;
  }
  const bool soc = lambda_r != 0.0 || field;  // the field's sigma_x, sigma_y need the flips too
  if (soc) {
    JobBatch sb{JOB_SOC, W * N, N, 3, 2, 0, 0, R, S, nullptr};
    NQS_TRY(run_net(m, c, prec, sb, HeadOut{Lf, gf, nullptr}, st));
  }
  if (ewald) NQS_TRY(nqs_ewald_energy(ewald, R, W, N, coul, st));
  k_eloc_assemble<<<(W + 127) / 128, 128, 0, st>>>(W, N, L0, g, lap, soc ? Lf : nullptr, gf, S,
                                                    ewald ? coul : nullptr, field, m_star,
                                                    lambda_r, h_z, (cplx*)out_eloc);
  NQS_CHECK_LAUNCH("k_eloc_assemble");
  if (out_logpsi) cudaMemcpyAsync(out_logpsi, L0, sizeof(cplx) * W, cudaMemcpyDeviceToDevice, st);
  return NQS_OK;
}

int nqs_local_energy(NqsModel* m, const double* theta, const double* R, const int32_t* S, int W,
                     double m_star, double lambda_r, double h_z, const NqsEwald* ewald,
                     double* out_eloc, double* out_logpsi, int prec, void* wsp, size_t wsb,
                     void* stream) {
  if (!out_eloc && W > 0) return NQS_ERR_INVALID_ARG;
  return local_energy_impl(m, theta, R, S, W, m_star, lambda_r, h_z, ewald, nullptr, out_eloc,
                           out_logpsi, nullptr, nullptr, prec, wsp, wsb, (cudaStream_t)stream,
                           true);
}

int nqs_local_energy_field(NqsModel* m, const double* theta, const double* R, const int32_t* S,
                           int W, double m_star, double lambda_r, double h_z,
                           const NqsEwald* ewald, const double* field, double* out_eloc,
                           double* out_logpsi, int prec, void* wsp, size_t wsb, void* stream) {
  if ((!out_eloc || !field) && W > 0) return NQS_ERR_INVALID_ARG;
  return local_energy_impl(m, theta, R, S, W, m_star, lambda_r, h_z, ewald, field, out_eloc,
                           out_logpsi, nullptr, nullptr, prec, wsp, wsb, (cudaStream_t)stream,
                           true);
}

int nqs_grad_laplacian(NqsModel* m, const double* theta, const double* R, const int32_t* S,
                       int W, double* out_logpsi, double* out_grad, double* out_lap, int prec,
                       void* wsp, size_t wsb, void* stream) {
  return local_energy_impl(m, theta, R, S, W, 1.0, 0.0, 0.0, nullptr, nullptr, nullptr,
                           out_logpsi, out_grad, out_lap, prec, wsp, wsb, (cudaStream_t)stream,
                           false);
}

static int mcmc_impl(NqsModel* m, const double* theta, double* R, int32_t* S,
                     double* logpsi_io, int W, int n_sweeps, int n_flips, double step,
                     uint64_t seed, uint64_t counter, uint64_t* counter_dev,
                     const double* inj_normals, const double* inj_u_pos,
                     const int32_t* inj_flip_idx, const double* inj_u_flip, double* out_acc_pos,
                     double* out_acc_spin, double* out_d, int prec, void* wsp, size_t wsb,
                     cudaStream_t st) {
  if (W < 0 || n_sweeps < 0 || n_flips < 0 || (W > 0 && (!R || !S))) return NQS_ERR_INVALID_ARG;
  if (W == 0) return NQS_OK;
  NQS_TRY(check_ws(m, NQS_OP_MCMC, W, prec, wsb));
  Ctx c;
  NQS_TRY(begin(m, theta, prec, wsp, wsb, st, &c));
  const int N = m->hm.mc.N;
  double* Rp = c.ws.take<double>((size_t)W * N * 2);
  cplx* Lc = c.ws.take<cplx>(W);
  cplx* Lp = c.ws.take<cplx>(W);
  int32_t* flip = c.ws.take<int32_t>(W);
  if (!flip) return NQS_ERR_WORKSPACE;
  McArgs a{};
  a.W = W;
  a.N = N;
  a.n_flips = n_flips;
  a.step = step;
  a.seed = seed;
  for (int i = 0; i < 4; ++i) {
    a.A[i] = m->hm.mc.A[i];
    a.Ainv[i] = m->hm.mc.Ainv[i];
  }
  a.inj_normals = inj_normals;
  a.inj_u_pos = inj_u_pos;
  a.inj_flip = inj_flip_idx;
  a.inj_u_flip = inj_u_flip;
  a.counter_dev = counter_dev;
  if (out_acc_pos) cudaMemsetAsync(out_acc_pos, 0, sizeof(double) * W, st);
  if (out_acc_spin) cudaMemsetAsync(out_acc_spin, 0, sizeof(double) * W, st);
  // current log psi (the reference recomputes it per proposal; the forward is deterministic,
  // so caching it gives identical decisions)
  JobBatch cur{JOB_VALUE, W, N, 1, 0, 0, 0, R, S, nullptr};
  NQS_TRY(run_net(m, c, prec, cur, HeadOut{Lc, nullptr, nullptr}, st));
  const int nb = (W + 127) / 128;
  for (int s = 0; s < n_sweeps; ++s) {
    a.s = s;
    a.sweep = counter + (uint64_t)s;
    k_propose_pos<<<(W * N + 127) / 128, 128, 0, st>>>(a, R, Rp);
    NQS_CHECK_LAUNCH("k_propose_pos");
    JobBatch pj{JOB_VALUE, W, N, 1, 0, 0, 0, Rp, S, nullptr};
    NQS_TRY(run_net(m, c, prec, pj, HeadOut{Lp, nullptr, nullptr}, st));
    k_accept_pos<<<nb, 128, 0, st>>>(a, R, Rp, Lc, Lp, out_acc_pos, out_d);
    NQS_CHECK_LAUNCH("k_accept_pos");
    for (int j = 0; j < n_flips; ++j) {
      k_propose_flip<<<nb, 128, 0, st>>>(a, j, flip);
      NQS_CHECK_LAUNCH("k_propose_flip");
      JobBatch fj{JOB_VALUE, W, N, 1, 0, 0, 0, R, S, flip};
      NQS_TRY(run_net(m, c, prec, fj, HeadOut{Lp, nullptr, nullptr}, st));
      k_accept_flip<<<nb, 128, 0, st>>>(a, j, S, flip, Lc, Lp, out_acc_spin, out_d);
      NQS_CHECK_LAUNCH("k_accept_flip");
    }
  }
  if (n_sweeps > 0) {
    if (out_acc_pos) {
      k_scale<<<nb, 128, 0, st>>>(out_acc_pos, W, 1.0 / n_sweeps);
      NQS_CHECK_LAUNCH("k_scale");
    }
    if (out_acc_spin && n_flips > 0) {
      k_scale<<<nb, 128, 0, st>>>(out_acc_spin, W, 1.0 / ((double)n_sweeps * n_flips));
      NQS_CHECK_LAUNCH("k_scale");
    }
  }
  if (logpsi_io) {
    const cudaError_t e = cudaMemcpyAsync(logpsi_io, Lc, sizeof(cplx) * W,
                                          cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return cuda_status(e, "nqs_mcmc_sweeps: copy");
  }
  if (counter_dev && n_sweeps > 0) {
    k_counter_add<<<1, 32, 0, st>>>(counter_dev, (uint64_t)n_sweeps);
    NQS_CHECK_LAUNCH("k_counter_add");
  }
  return NQS_OK;
}

int nqs_mcmc_sweeps(NqsModel* m, const double* theta, double* R, int32_t* S, double* logpsi_io,
                    int W, int n_sweeps, int n_flips, double step, uint64_t seed,
                    uint64_t counter, const double* inj_normals, const double* inj_u_pos,
                    const int32_t* inj_flip_idx, const double* inj_u_flip, double* out_acc_pos,
                    double* out_acc_spin, double* out_d, int prec, void* wsp, size_t wsb,
                    void* stream) {
  return mcmc_impl(m, theta, R, S, logpsi_io, W, n_sweeps, n_flips, step, seed, counter, nullptr,
                   inj_normals, inj_u_pos, inj_flip_idx, inj_u_flip, out_acc_pos, out_acc_spin,
                   out_d, prec, wsp, wsb, (cudaStream_t)stream);
}

int nqs_mcmc_sweeps_devctr(NqsModel* m, const double* theta, double* R, int32_t* S,
                           double* logpsi_io, int W, int n_sweeps, int n_flips, double step,
                           uint64_t seed, uint64_t* counter_dev, double* out_acc_pos,
                           double* out_acc_spin, int prec, void* wsp, size_t wsb, void* stream) {
  if (!counter_dev) {
    set_error("nqs_mcmc_sweeps_devctr: null counter");
    return NQS_ERR_INVALID_ARG;
  }
  return mcmc_impl(m, theta, R, S, logpsi_io, W, n_sweeps, n_flips, step, seed, 0, counter_dev,
                   nullptr, nullptr, nullptr, nullptr, out_acc_pos, out_acc_spin, nullptr, prec,
                   wsp, wsb, (cudaStream_t)stream);
}

}  // extern "C"

// Dense layers of the float32 Jacobian / VJP pass on the tensor cores (nqs_set_jacobian_tc)
static bool g_jacobian_tc = false;

extern "C" int nqs_set_jacobian_tc(int enable) {
  g_jacobian_tc = enable != 0;
  return NQS_OK;
}

static int per_sample_O_impl(NqsModel* m, const double* theta, const double* R,
                             const int32_t* S, int W, void* out_O, int out_dtype, int prec,
                             bool ckpt, void* wsp, size_t wsb, cudaStream_t st) {
  if (W < 0 || (W > 0 && (!R || !S || !out_O)) || (out_dtype != 0 && out_dtype != 1)) {
    set_error("nqs_per_sample_O: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  if (W == 0) return NQS_OK;
  NQS_TRY(check_ws(m, ckpt ? NQS_OP_PER_SAMPLE_O_CKPT : NQS_OP_PER_SAMPLE_O, W, prec, wsb));
  Ctx c;
  NQS_TRY(begin(m, theta, prec, wsp, wsb, st, &c));
  const HeadParams hp = make_head_params(m->hm.desc, c.theta64);
  if (prec == NQS_PREC_FP64) {
    const NetW<double> w = make_netw<double>(m->hm.desc, c.theta64, c.theta64);
    if (out_dtype == 0)
      return per_sample_O_run<double, double>(m->hm, w, hp, R, S, W, (double*)out_O, ckpt, c.ws,
                                              st);
    return per_sample_O_run<double, float>(m->hm, w, hp, R, S, W, (float*)out_O, ckpt, c.ws, st);
  }
  NetW<float> w = make_netw<float>(m->hm.desc, c.theta32, c.theta64);
  if (g_jacobian_tc) w.tc = c.tc;  // the pass's Dense layers on the tensor cores (opt-in)
  if (out_dtype == 0)
    return per_sample_O_run<float, double>(m->hm, w, hp, R, S, W, (double*)out_O, ckpt, c.ws, st);
  return per_sample_O_run<float, float>(m->hm, w, hp, R, S, W, (float*)out_O, ckpt, c.ws, st);
}

extern "C" int nqs_per_sample_O(NqsModel* m, const double* theta, const double* R,
                                const int32_t* S, int W, void* out_O, int out_dtype, int prec,
                                void* wsp, size_t wsb, void* stream) {
  return per_sample_O_impl(m, theta, R, S, W, out_O, out_dtype, prec, false, wsp, wsb,
                           (cudaStream_t)stream);
}

extern "C" int nqs_per_sample_O_ex(NqsModel* m, const double* theta, const double* R,
                                   const int32_t* S, int W, void* out_O, int out_dtype, int prec,
                                   int checkpoint_blocks, void* wsp, size_t wsb, void* stream) {
  return per_sample_O_impl(m, theta, R, S, W, out_O, out_dtype, prec, checkpoint_blocks != 0,
                           wsp, wsb, (cudaStream_t)stream);
}

extern "C" int nqs_logpsi_vjp(NqsModel* m, const double* theta, const double* R,
                              const int32_t* S, int W, const double* cotangent, double* out_grad,
                              int prec, int checkpoint_blocks, void* wsp, size_t wsb,
                              void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  if (!m || W < 0 || !out_grad || (W > 0 && (!R || !S || !cotangent))) {
    set_error("nqs_logpsi_vjp: invalid argument");
    return NQS_ERR_INVALID_ARG;
  }
  if (W == 0) {
    const cudaError_t e = cudaMemsetAsync(out_grad, 0, sizeof(double) * m->hm.desc.n_params, st);
    return e == cudaSuccess ? NQS_OK : cuda_status(e, "nqs_logpsi_vjp: clear");
  }
  const bool ckpt = checkpoint_blocks != 0;
  NQS_TRY(check_ws(m, ckpt ? NQS_OP_LOGPSI_VJP_CKPT : NQS_OP_LOGPSI_VJP, W, prec, wsb));
  Ctx c;
  NQS_TRY(begin(m, theta, prec, wsp, wsb, st, &c));
  const HeadParams hp = make_head_params(m->hm.desc, c.theta64);
  const cplx* ct = (const cplx*)cotangent;
  if (prec == NQS_PREC_FP64) {
    const NetW<double> w = make_netw<double>(m->hm.desc, c.theta64, c.theta64);
    return logpsi_vjp_run<double>(m->hm, w, hp, R, S, W, ct, out_grad, ckpt, c.ws, st);
  }
  NetW<float> w = make_netw<float>(m->hm.desc, c.theta32, c.theta64);
  if (g_jacobian_tc) w.tc = c.tc;
  return logpsi_vjp_run<float>(m->hm, w, hp, R, S, W, ct, out_grad, ckpt, c.ws, st);
}
