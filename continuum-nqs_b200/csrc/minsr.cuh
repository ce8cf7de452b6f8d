// minsr.cuh — internal interface between the MinSR driver and the tensor-core Gram.
#pragma once
#include "net.cuh"

namespace nqs {

// float64 lower-triangular C = alpha A A^T + beta C (A: M x K, K-contiguous rows)
int dsyrk_lower(const double* A, int64_t lda, int M, int64_t K, double alpha, double beta,
                double* C, int64_t ldc, double* part, size_t part_elems, int nsm,
                cudaStream_t st);

// Tensor-core Gram of the centred O: T (lower, float64, 2W x 2W) = Otil Otil^T with Otil =
// O - mu converted to the operand type of `prec` (1 = BF16, 2 = TF32), float32 accumulation.
size_t gram_tc_workspace(int W, int64_t P, int prec);
int gram_tc(const void* O, int o_dtype, const double* mu, int W, int64_t P, int prec, double* T,
            Arena& ws, int nsm, cudaStream_t st, int* err);
// float64 Cholesky of the lower triangle in place as one persistent task-graph kernel of
// 128 x 128 tiles (chol_dag.cu); scratch: cholesky_dag_scratch_elems(n) doubles (tile counters)
size_t cholesky_dag_scratch_elems(int n);
int cholesky_dag(double* A, int64_t lda, int n, int* bad, double* scratch, size_t scratch_elems,
                 int nsm, cudaStream_t st, const double* floor_p);
extern bool g_chol_dag;  // nqs_set_cholesky_dag

int gram_tc_launch(const void* D, int prec, int M, int64_t K, int64_t ldd, double* T, int64_t ldt,
                   int* err, cudaStream_t st);
// C (lower, float64) -= A A^T (A: M x K float64, K a multiple of 32) on the tensor cores with
// TF32 hi/lo operand splitting (three products, ~2^-22 relative error); Z: scratch of
// syrk_split_tf32_scratch_floats(M, K) floats, 16-byte aligned; C 16-byte aligned, ldc even.
size_t syrk_split_tf32_scratch_floats(int M, int K);
int syrk_split_tf32(const double* A, int64_t lda, int M, int K, double* C, int64_t ldc, float* Z,
                    int* err, cudaStream_t st);
extern bool g_chol_tc;  // nqs_set_cholesky_tc
extern bool g_gram_wide;  // nqs_set_gram_wide

}  // namespace nqs
