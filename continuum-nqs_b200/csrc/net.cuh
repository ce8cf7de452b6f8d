// net.cuh — host-side interface of the wavefunction network passes (forward, forward-Laplacian,
// spin-flip JVPs, reverse-mode per-sample Jacobian).
#pragma once

#include "nqs_common.cuh"

namespace nqs {

// Per-block weight pointers in the working precision T (row-major Dense kernels [in][out]).
template <typename T>
struct BlockW {
  const T *ln0_s, *ln0_b, *ln1_s, *ln1_b;
  const T *wq, *bq, *wk, *bk, *wv, *bv, *wo, *bo;
  const T *w0, *b0, *w1, *b1;
};

// K-major float32 weight copies for the tensor-core row GEMMs of the mixed path, and (BF16
// operands) their BF16 copies (raw bits, round to nearest even).
struct TcNet {
  int on;
  int bf16;  // Dense layers with BF16 operands where K is a multiple of 64
  const float *wqkv[NQS_MAX_DEPTH], *bqkv[NQS_MAX_DEPTH], *wo[NQS_MAX_DEPTH];
  const float *w0[NQS_MAX_DEPTH], *w1[NQS_MAX_DEPTH];
  const float *wbf;
  const uint16_t *wqkv16[NQS_MAX_DEPTH], *wo16[NQS_MAX_DEPTH], *w016[NQS_MAX_DEPTH],
      *w116[NQS_MAX_DEPTH], *wbf16;
  int npad_qkv, npad_bf;
  int* err;
};

template <typename T>
struct NetW {
  TcNet tc;
  const T *emb_w, *emb_b;
  BlockW<T> blk[NQS_MAX_DEPTH];
  const T *lnf_s, *lnf_b;
  const T *bf_w_re, *bf_w_im, *bf_b_re, *bf_b_im;  // backflow Dense (complex leaf split)
  const double* theta;                              // float64 theta (head parameters)
};

// Head parameters always read from float64 theta.
struct HeadParams {
  const double* det_logw;  // [2K] re block then im block (nullable when K == 1)
  const double* jas_same;  // [n_knots]
  const double* jas_opp;   // [n_knots]
  const double* jas_loga;  // [1]
  const double* dW;        // [2 * N * nG * 2] complex leaf (re block, im block), nullable
};

struct HostModel {
  NqsModelDesc desc;  // host copy (host pointers inside are not kept)
  ModelConst mc;      // device pointers
  double* d_Gs;
  double* d_W;
  double* d_knots;
};

// Scratch carved out of the caller's workspace.
struct Arena {
  char* base;
  size_t cap, used;
  template <typename X>
  X* take(size_t n) {
    size_t off = (used + 255) & ~(size_t)255;
    used = off + n * sizeof(X);
    return (used <= cap && base) ? reinterpret_cast<X*>(base + off) : nullptr;
  }
};

// Outputs of a network pass for each job of a batch, float64:
//   L[j] complex, dL[j][n_tan] complex, lap[j] complex (each nullable).
struct HeadOut {
  cplx* L;
  cplx* dL;
  cplx* lap;
};

// Rows per job (tokens * channels) for a batch shape.
inline size_t job_rows(int N, int C) { return (size_t)N * C; }

// Bytes of activation scratch for `rows` rows in precision T.
template <typename T>
size_t net_scratch_bytes(const ModelConst& mc, size_t rows);

// Run the network over jb.n_jobs jobs, chunked to at most max_rows rows per chunk.
template <typename T>
int net_forward(const HostModel& hm, const NetW<T>& w, const HeadParams& hp, JobBatch jb,
                HeadOut out, Arena& ws, size_t max_rows, cudaStream_t st);

// Build the per-layer pointers into theta (float64 or a float32 copy) from the descriptor.
template <typename T>
NetW<T> make_netw(const NqsModelDesc& d, const T* theta_T, const double* theta64);
HeadParams make_head_params(const NqsModelDesc& d, const double* theta64);

// theta float64 -> float32 copy
int theta_to_f32(const double* theta, float* out, int64_t n, cudaStream_t st);

// Reverse mode: per-sample Jacobian rows (Re in [0,W), Im in [W,2W)) of a [2W][P] matrix, or
// the vector-Jacobian product grad[k] = sum_w Re(ct_w O[w][k]) without O. ckpt: keep only each
// transformer block's input and recompute the block's activations before its reverse step.
template <typename T>
size_t backward_scratch(const ModelConst& mc, int W, bool ckpt);
template <typename T>
size_t per_sample_O_scratch(const ModelConst& mc, int W);
template <typename T, typename TO>
int per_sample_O_run(const HostModel& hm, const NetW<T>& w, const HeadParams& hp,
                     const double* R, const int32_t* S, int W, TO* O, bool ckpt, Arena& ws,
                     cudaStream_t st);
template <typename T>
int logpsi_vjp_run(const HostModel& hm, const NetW<T>& w, const HeadParams& hp,
                   const double* R, const int32_t* S, int W, const cplx* ct, double* grad,
                   bool ckpt, Arena& ws, cudaStream_t st);

// tensor-core row GEMM (gemm_tc.cu): K a multiple of 32, any width (pieces of K <= 128 and
// N <= 256, one launch each); act 1: tanh-GELU on the output (C == 1 and K <= 128 only); WT16
// (nullable): BF16 copy of W^T, which makes the operands BF16 (kind::f16) when K is a multiple
// of 64
int rowgemm_tc(const float* X, int ldx, int rows, int K, const float* WT, int Npad, int Nout,
               const float* bias, int C, const float* Res, int ldr, float* Y, int ldy, int* err,
               cudaStream_t st, int act = 0, const uint16_t* WT16 = nullptr);
// one whole transformer block of single-channel rows in one launch (block_tc.cu); *done is false
// when the shape or the operand alignment is not covered and the caller runs the unfused block
bool block_value_tc_ok(int N, int d, int H, int ff);
int block_value_tc(float* X, int n_jobs, int N, int d, int H, const TcNet& tcn, int b,
                   const BlockW<float>& bw, cudaStream_t st, bool* done);
extern bool g_block_fusion;
bool profiling_enabled();  // nqs_profile_gemm(1) is in force
size_t tc_weights_bytes(const NqsModelDesc& d, bool bf16);
int build_tc_weights(const NqsModelDesc& d, const float* theta32, Arena& ws, TcNet* out,
                     cudaStream_t st, bool bf16);

// Default row budget of one network chunk.
constexpr size_t kMaxRows = (size_t)1 << 19;

}  // namespace nqs
