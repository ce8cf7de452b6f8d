// chol_dag.cu — float64 Cholesky A = L L^T (lower triangle, in place) as one persistent kernel
// over a task graph of 128 x 128 tiles.
//
// Tasks (T = ceil(n / 128) tile rows):
//   POTRF(k):        L_kk = chol(A_kk), in shared memory (8-column sub-panels: warp 0 factors a
//                    sub-panel with its rows in registers, the CTA applies its rank-8 update)
//   TRSM(i, k):      L_ik = A_ik L_kk^-T, i > k (forward substitution, four rows per warp with
//                    their 128 columns in registers, L_kk in shared memory)
//   UPDATE(i, j, k): A_ij -= L_ik L_jk^T, k < j <= i (128 x 128 x 128 tile product, 8 x 8 per
//                    thread, operands staged by cp.async in a 3-stage ring)
// Two queues, each consumed in order:
//   critical: POTRF(0), TRSM(i, 0); for k = 0 .. T-2: UPDATE(i, k+1, k) [column k+1],
//             POTRF(k+1), TRSM(i, k+1)                         -- the factorization's spine
//   bulk:     UPDATE(i, j, k), j >= k+2, by k, then column j, then row i
// A CTA (its thread 0) takes the head of the critical queue when that task's inputs are complete,
// otherwise the head of the bulk queue once the two panel solves it reads have been taken, so the
// spine runs as soon as it can and the bulk fills the SMs around it. Tile (i, j) carries a counter
// of the operations applied to it (updates k = 0 .. j-1, then its POTRF or TRSM): a critical task
// is taken only when its counters are reached (acquire loads), a bulk task waits (bounded) for
// counters of tasks already taken; a finished task publishes its tile's counter with a release
// store after a barrier. Every task a CTA waits for is held by a running CTA whose own inputs are
// complete or in flight, so the graph drains. Every wait and every idle spin is bounded: a CTA
// that runs out of its limit sets the abort word (every CTA then leaves), the failure flag bad[0]
// and a NaN in L[0][0].
// Pivots below *floor_p are raised to it (counted in bad[2]); a non-positive pivot sets bad[0].
#include <cstdio>
#include <algorithm>

#include "minsr.cuh"

namespace nqs {
namespace {

constexpr int TB = 128;                           // tile
constexpr int GK = 16, GST = 3, GLD = GK + 2;     // product: k-chunk, stages, shared row stride
constexpr int LDT = TB + 1;                       // factor tile row stride in shared memory
constexpr uint32_t kDagWaitLimit = 1u << 22;
constexpr size_t kDagSmem = sizeof(double) * TB * LDT;
static_assert(sizeof(double) * 2 * GST * TB * GLD <= kDagSmem, "product stages fit the tile");
static_assert((GLD * sizeof(double)) % 16 == 0, "cp.async rows start on 16 bytes");

struct DagTask {
  int type, k, i, j;  // type 0 POTRF, 1 TRSM, 2 UPDATE; -1 none
};

__host__ __device__ inline int dag_ncrit(int T) { return T * T; }
__host__ __device__ inline long long dag_c3(long long x) { return x >= 3 ? x * (x - 1) * (x - 2) / 6 : 0; }
__host__ __device__ inline int dag_nbulk(int T) { return (int)dag_c3(T); }  // sum_k C(T-k-1, 2)

// critical queue: position of the first task of step k's block (k >= 0), after the T tasks
// POTRF(0), TRSM(i, 0)
__device__ __forceinline__ int dag_crit_base(int T, int k) { return T + 2 * k * (T - 1) - k * (k - 1); }
// position of TRSM(i, k) in the critical queue
__device__ __forceinline__ int dag_trsm_index(int T, int i, int k) {
  return k == 0 ? i : dag_crit_base(T, k - 1) + (T - k) + 1 + (i - k - 1);
}

// The two task lists, written once per factorization: critical entries (type, k, i, j); bulk
// entries UPDATE(i, j, k) as (k, i, j, position of TRSM(i, k) in the critical queue).
__global__ void k_dag_lists(int T, int4* __restrict__ crit, int4* __restrict__ bulk) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nc = (long long)T * T;
  if (gid < nc) {
    const int c = (int)gid;
    int4 e = make_int4(-1, 0, 0, 0);
    if (c < T) {
      e = c == 0 ? make_int4(0, 0, 0, 0) : make_int4(1, 0, c, 0);
    } else {
      for (int k = 0; k + 1 < T; ++k) {
        const int b0 = dag_crit_base(T, k), a = T - 1 - k;
        if (c < b0 + 2 * a) {
          const int o = c - b0;
          if (o < a)
            e = make_int4(2, k, k + 1 + o, k + 1);
          else if (o == a)
            e = make_int4(0, k + 1, k + 1, k + 1);
          else
            e = make_int4(1, k + 1, k + 2 + (o - a - 1), k + 1);
          break;
        }
      }
    }
    crit[c] = e;
    return;
  }
  // bulk: one thread per (k, j, i) with k + 2 <= j <= i < T
  const long long t = gid - nc;
  if (t >= (long long)T * T * T) return;
  const int k = (int)(t / ((long long)T * T)), j = (int)((t / T) % T), i = (int)(t % T);
  if (!(k + 2 <= j && j <= i)) return;
  const long long offk = dag_c3(T) - dag_c3(T - k);
  const long long offj = (long long)(j - k - 2) * T - ((long long)(j - 1) * j / 2 - (long long)(k + 1) * (k + 2) / 2);
  bulk[offk + offj + (i - j)] = make_int4(k, i, j, dag_trsm_index(T, i, k));
}

__device__ __forceinline__ int dag_ld_acquire(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void dag_st_release(int* p, int v) {
  asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// 0: reached; 1: own limit ran out; 2: another CTA aborted
__device__ int dag_wait(const int* p, int target, const int* abort_w, uint32_t limit) {
  uint32_t w = 0;
  while (dag_ld_acquire(p) < target) {
    if (dag_ld_acquire(abort_w) != 0) return 2;
    if (++w >= limit) return 1;
    if (w > 32) __nanosleep(w > 4096 ? 256 : 64);
  }
  return 0;
}

// inputs of a task complete (acquire loads, no waiting)
__device__ bool dag_ready(const int* state, int T, DagTask t) {
  if (t.type == 0) return dag_ld_acquire(state + t.k * T + t.k) >= t.k;
  if (t.type == 1)
    return dag_ld_acquire(state + t.k * T + t.k) >= t.k + 1 &&
           dag_ld_acquire(state + t.i * T + t.k) >= t.k;
  return dag_ld_acquire(state + t.i * T + t.j) >= t.k &&
         dag_ld_acquire(state + t.i * T + t.k) >= t.k + 1 &&
         dag_ld_acquire(state + t.j * T + t.k) >= t.k + 1;
}

__device__ __forceinline__ void cp16_zfill(void* smem, const void* gmem, int n_src) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(n_src)
               : "memory");
}

// ---- POTRF: the tile [k0, k0 + b)^2 in shared memory, factored, written back ----
__device__ void dag_potrf(double* A, int64_t lda, int k0, int b, double* sm, double* dval,
                          double* dinv, int* bad, const double* floor_p) {
  double(*L)[LDT] = reinterpret_cast<double(*)[LDT]>(sm);
  const int tid = threadIdx.x, lane = tid & 31;
  const double fl = floor_p ? *floor_p : 0.0;
  for (int idx = tid; idx < TB * TB; idx += blockDim.x) {
    const int i = idx / TB, c = idx - i * TB;
    L[i][c] = (i < b && c <= i) ? __ldcg(A + (size_t)(k0 + i) * lda + k0 + c) : 0.0;
  }
  __syncthreads();
  for (int j0 = 0; j0 < b; j0 += 8) {
    const int jw = min(8, b - j0);
    if (tid < 32) {
      // lane holds rows j0 + lane + 32 m (m < 4) of the sub-panel's 8 columns
      double p[4][8];
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int r = j0 + lane + 32 * m;
#pragma unroll
        for (int c = 0; c < 8; ++c) p[m][c] = (r < b && c < jw) ? L[r][j0 + c] : 0.0;
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        if (c < jw) {
          double d = __shfl_sync(0xffffffffu, p[0][c], c);  // row j0 + c, column c
          const bool floored = floor_p && !(d > fl);
          if (floored) d = fl;
          const bool pos = d > 0.0;
          if (lane == 0) {
            if (floored) atomicAdd(bad + 2, 1);
            if (!pos) atomicExch(bad, 1);
            dval[j0 + c] = d;
            dinv[j0 + c] = pos ? 1.0 / d : NAN;
          }
          const double inv = pos ? 1.0 / d : NAN;
          if (lane == c) p[0][c] = d;  // the (floored) pivot is the stored diagonal
#pragma unroll
          for (int kk = c + 1; kk < 8; ++kk) {
            const double akc = __shfl_sync(0xffffffffu, p[0][c], kk) * inv;  // row j0 + kk
            if (kk < jw) {
#pragma unroll
              for (int m = 0; m < 4; ++m) p[m][kk] -= p[m][c] * akc;
            }
          }
        }
      }
#pragma unroll
      for (int m = 0; m < 4; ++m) {
        const int r = j0 + lane + 32 * m;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c < jw && r < b && r >= j0 + c) L[r][j0 + c] = p[m][c];
      }
    }
    __syncthreads();
    // trailing update inside the tile: rows i, columns kk in [j0 + jw, i], four threads per row
    const int t0 = j0 + jw;
    for (int i = t0 + (tid >> 2); i < b; i += (int)(blockDim.x >> 2)) {
      const int q = tid & 3;
      double pi[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) pi[c] = c < jw ? L[i][j0 + c] * dinv[j0 + c] : 0.0;
      for (int kk = t0 + q; kk <= i; kk += 4) {
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < 8; ++c) acc = fma(pi[c], L[kk][j0 + c], acc);
        L[i][kk] -= acc;
      }
    }
    __syncthreads();
  }
  // L[i][c] = a_ic / sqrt(d_c) (i > c), L[c][c] = sqrt(d_c); written back
  for (int idx = tid; idx < b * b; idx += blockDim.x) {
    const int i = idx / b, c = idx - i * b;
    if (c <= i) {
      const double d = dval[c];
      const double sd = d > 0.0 ? sqrt(d) : NAN;
      A[(size_t)(k0 + i) * lda + k0 + c] = (i == c) ? sd : L[i][c] / sd;
    }
  }
}

// ---- TRSM: rows [r0, r0 + rows) of the column block [k0, k0 + 128): x L_kk^T = a ----
__device__ void dag_trsm(double* A, int64_t lda, int k0, int r0, int rows, double* sm,
                         double* rdiag) {
  double(*L)[LDT] = reinterpret_cast<double(*)[LDT]>(sm);
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  for (int idx = tid; idx < TB * TB; idx += blockDim.x) {
    const int i = idx / TB, c = idx - i * TB;
    L[i][c] = c <= i ? __ldcg(A + (size_t)(k0 + i) * lda + k0 + c) : 0.0;
  }
  __syncthreads();
  if (tid < TB) rdiag[tid] = 1.0 / L[tid][tid];
  __syncthreads();
  for (int rb = 4 * w; rb < rows; rb += 4 * nw) {
    double x[4][4];  // [row u][column lane + 32 q]
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = rb + u;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        x[u][q] = r < rows ? __ldcg(A + (size_t)(r0 + r) * lda + k0 + lane + 32 * q) : 0.0;
    }
#pragma unroll 1
    for (int q0 = 0; q0 < 4; ++q0) {
#pragma unroll 1
      for (int jl = 0; jl < 32; ++jl) {
        const int j = 32 * q0 + jl;
        const double rd = rdiag[j];
        double l[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) l[q] = (lane + 32 * q > j) ? L[lane + 32 * q][j] : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          double xs = 0.0;
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q == q0) xs = x[u][q];
          const double xj = __shfl_sync(0xffffffffu, xs, jl) * rd;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            if (q == q0 && lane == jl) x[u][q] = xj;
            x[u][q] -= xj * l[q];
          }
        }
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = rb + u;
      if (r < rows) {
#pragma unroll
        for (int q = 0; q < 4; ++q) A[(size_t)(r0 + r) * lda + k0 + lane + 32 * q] = x[u][q];
      }
    }
  }
}

// ---- UPDATE: C[r][c] -= sum_kk X[r][kk] Y[c][kk], r < mi, c < mj (c <= r on a diagonal tile) --
__device__ void dag_update(double* C, const double* X, const double* Y, int64_t lda, int mi,
                           int mj, bool diag, double* sm) {
  double* As = sm;                   // [GST][TB][GLD]
  double* Bs = sm + GST * TB * GLD;  // [GST][TB][GLD]
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  constexpr int nk = TB / GK;
  auto load_stage = [&](int s, int kc) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int idx = tid + 256 * q, r = idx >> 3, c = (idx & 7) * 2;
      const int kk = kc * GK + c;
      cp16_zfill(As + ((size_t)s * TB + r) * GLD + c, r < mi ? X + (size_t)r * lda + kk : X,
                 r < mi ? 16 : 0);
      cp16_zfill(Bs + ((size_t)s * TB + r) * GLD + c, r < mj ? Y + (size_t)r * lda + kk : Y,
                 r < mj ? 16 : 0);
    }
  };
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
#pragma unroll
  for (int s = 0; s < GST - 1; ++s) {
    load_stage(s, s);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
  }
  for (int kc = 0; kc < nk; ++kc) {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(GST - 2) : "memory");
    __syncthreads();
    const int nxt = kc + GST - 1;
    if (nxt < nk) load_stage(nxt % GST, nxt);
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    const double* as = As + (size_t)(kc % GST) * TB * GLD;
    const double* bs = Bs + (size_t)(kc % GST) * TB * GLD;
#pragma unroll
    for (int kk = 0; kk < GK; kk += 2) {
      double2 av[8];
#pragma unroll
      for (int i = 0; i < 8; ++i)
        av[i] = *reinterpret_cast<const double2*>(as + (ty + 16 * i) * GLD + kk);
#pragma unroll
      for (int j = 0; j < 8; ++j) {
        const double2 bv = *reinterpret_cast<const double2*>(bs + (tx + 16 * j) * GLD + kk);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][j] = fma(av[i].x, bv.x, acc[i][j]);
#pragma unroll
        for (int i = 0; i < 8; ++i) acc[i][j] = fma(av[i].y, bv.y, acc[i][j]);
      }
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int r = ty + 16 * i;
    if (r >= mi) continue;
    double cv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = tx + 16 * j;
      cv[j] = (c < mj && (!diag || c <= r)) ? __ldcg(C + (size_t)r * lda + c) : 0.0;
    }
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const int c = tx + 16 * j;
      if (c < mj && (!diag || c <= r)) C[(size_t)r * lda + c] = cv[j] - acc[i][j];
    }
  }
}

__global__ void __launch_bounds__(256, 1) k_chol_dag(double* __restrict__ A, int64_t lda, int n,
                                                     int T, int* __restrict__ state,
                                                     int* __restrict__ tickets,
                                                     int* __restrict__ abort_w,
                                                     int* __restrict__ bad,
                                                     const int4* __restrict__ crit_list,
                                                     const int4* __restrict__ bulk_list,
                                                     const double* __restrict__ floor_p,
                                                     uint32_t wait_limit) {
  extern __shared__ __align__(16) double dsm[];
  __shared__ int s_task[5];  // type, k, i, j, stop
  __shared__ double dval[TB], dinv[TB];
  const int tid = threadIdx.x;
  const int n_crit = dag_ncrit(T), n_bulk = dag_nbulk(T);
  int* crit = tickets;
  int* bulk = tickets + 1;
  int pending = -1;  // (thread 0) a bulk task dealt to this CTA, not yet admitted
  auto fail = [&]() {
    atomicExch(abort_w, 1);
    atomicExch(bad, 1);
    A[0] = __longlong_as_double(0x7ff8000000000000ll);
  };
  for (;;) {
    if (tid == 0) {
      DagTask pick{-1, 0, 0, 0};
      int stop = 0;
      uint32_t idle = 0;
      for (;;) {
        if (dag_ld_acquire(abort_w) != 0) {
          stop = 1;
          break;
        }
        const int c = dag_ld_acquire(crit);
        if (c < n_crit) {  // the spine first, whenever its head is ready
          const int4 e = __ldcg(crit_list + c);
          const DagTask t{e.x, e.y, e.z, e.w};
          if (dag_ready(state, T, t)) {
            if (atomicCAS(crit, c, c + 1) == c) {
              pick = t;
              break;
            }
            continue;
          }
        }
        if (pending >= 0) {
          const int4 e = __ldcg(bulk_list + pending);
          if (c > e.w) {  // both panel solves it reads are taken: its inputs are in flight
            const DagTask t{2, e.x, e.y, e.z};
            pending = -1;
            int st = dag_wait(state + t.i * T + t.j, t.k, abort_w, wait_limit);
            if (!st) st = dag_wait(state + t.i * T + t.k, t.k + 1, abort_w, wait_limit);
            if (!st) st = dag_wait(state + t.j * T + t.k, t.k + 1, abort_w, wait_limit);
            if (st) {
              if (st == 1) fail();
              stop = 1;
            } else {
              pick = t;
            }
            break;
          }
        } else {
          const int b = dag_ld_acquire(bulk);
          if (b < n_bulk) {
            if (c > __ldcg(bulk_list + b).w) {
              const int b2 = atomicAdd(bulk, 1);
              if (b2 < n_bulk) pending = b2;
              continue;
            }
          } else if (c >= n_crit) {
            stop = 1;
            break;
          }
        }
        if (++idle >= wait_limit) {  // nothing admissible for too long
          fail();
          stop = 1;
          break;
        }
        if (idle > 32) __nanosleep(idle > 4096 ? 256 : 64);
      }
      s_task[0] = pick.type;
      s_task[1] = pick.k;
      s_task[2] = pick.i;
      s_task[3] = pick.j;
      s_task[4] = stop;
    }
    __syncthreads();
    if (s_task[4]) break;
    const DagTask t{s_task[0], s_task[1], s_task[2], s_task[3]};
    int tile;
    if (t.type == 0) {
      dag_potrf(A, lda, t.k * TB, min(TB, n - t.k * TB), dsm, dval, dinv, bad, floor_p);
      tile = t.k * T + t.k;
    } else if (t.type == 1) {
      dag_trsm(A, lda, t.k * TB, t.i * TB, min(TB, n - t.i * TB), dsm, dval);
      tile = t.i * T + t.k;
    } else {
      const int i0 = t.i * TB, j0 = t.j * TB, k0 = t.k * TB;
      dag_update(A + (size_t)i0 * lda + j0, A + (size_t)i0 * lda + k0,
                 A + (size_t)j0 * lda + k0, lda, min(TB, n - i0), min(TB, n - j0), t.i == t.j,
                 dsm);
      tile = t.i * T + t.j;
    }
    __syncthreads();
    if (tid == 0) {
      __threadfence();
      dag_st_release(state + tile, t.k + 1);
    }
  }
}

}  // namespace

bool g_chol_dag = false;

// doubles: two queue tickets, abort word + pad, T^2 tile counters, rounded up to an even count
// so that the two task lists (int4) that follow start on 16 bytes
static size_t dag_counters_elems(size_t T) { return (2 + (T * T + 1) / 2 + 1) & ~(size_t)1; }
size_t cholesky_dag_scratch_elems(int n) {
  const size_t T = (size_t)(n + TB - 1) / TB;
  return dag_counters_elems(T) + 2 * (T * T + (size_t)dag_nbulk((int)T));
}

int cholesky_dag(double* A, int64_t lda, int n, int* bad, double* scratch, size_t scratch_elems,
                 int nsm, cudaStream_t st, const double* floor_p) {
  if (n <= 0) return NQS_OK;
  const int T = (n + TB - 1) / TB;
  if (lda % 2 || (reinterpret_cast<uintptr_t>(A) & 15)) {
    set_error("cholesky_dag: rows must start on 16 bytes (lda %lld)", (long long)lda);
    return NQS_ERR_INVALID_ARG;
  }
  if (!scratch || scratch_elems < cholesky_dag_scratch_elems(n)) {
    set_error("cholesky_dag: scratch of %zu doubles < %zu", scratch_elems,
              cholesky_dag_scratch_elems(n));
    return NQS_ERR_WORKSPACE;
  }
  int* tickets = reinterpret_cast<int*>(scratch);  // [0] critical, [1] bulk
  int* abort_w = reinterpret_cast<int*>(scratch + 1);
  int* state = reinterpret_cast<int*>(scratch + 2);
  int4* crit_list = reinterpret_cast<int4*>(scratch + dag_counters_elems(T));
  int4* bulk_list = crit_list + (size_t)T * T;
  if (reinterpret_cast<uintptr_t>(crit_list) & 15) {
    set_error("cholesky_dag: scratch not 16-byte aligned");
    return NQS_ERR_INVALID_ARG;
  }
  cudaMemsetAsync(scratch, 0, sizeof(double) * dag_counters_elems(T), st);
  {
    const long long nthreads = (long long)T * T + (long long)T * T * T;
    k_dag_lists<<<(unsigned)((nthreads + 255) / 256), 256, 0, st>>>(T, crit_list, bulk_list);
    NQS_CHECK_LAUNCH("k_dag_lists");
  }
  static bool attr = false;
  if (!attr) {
    cudaFuncSetAttribute(k_chol_dag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDagSmem);
    attr = true;
  }
  const int ntasks = dag_ncrit(T) + dag_nbulk(T);
  int grid = std::min(std::max(nsm, 1), ntasks);
  uint32_t wl = wait_limit_or(kDagWaitLimit);
  int nn = n;
  int TT = T;
  const int4* cl = crit_list;
  const int4* bl = bulk_list;
  void* args[] = {(void*)&A,       (void*)&lda,     (void*)&nn,      (void*)&TT,
                  (void*)&state,   (void*)&tickets, (void*)&abort_w, (void*)&bad,
                  (void*)&cl,      (void*)&bl,      (void*)&floor_p, (void*)&wl};
  const cudaError_t e = cudaLaunchCooperativeKernel((const void*)k_chol_dag, grid, 256, args,
                                                    kDagSmem, st);
  if (e != cudaSuccess) return cuda_status(e, "k_chol_dag");
  NQS_CHECK_LAUNCH("k_chol_dag");
  return NQS_OK;
}

}  // namespace nqs
