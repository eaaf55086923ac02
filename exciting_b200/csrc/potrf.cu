// Cholesky factorisation O = U^H U (upper) and the inverse factor U^-1.
//
// ZHEGVX starts with ZPOTRF('U') on the overlap matrix
// (external/LAPACK/zhegvx.f:410).  Here it is blocked right-looking with a
// 64-wide panel: one CTA factors the diagonal block in shared memory and
// also inverts it; the row panel is then one GEMM with the inverted diagonal
// block, and the trailing update one upper-triangle GEMM.  The inverse
// factor U^-1 (used for the two-sided reduction and the back-transform) is
// built block column by block column from the inverted diagonal blocks:
//   Ui(0:j, j) = -Ui(0:j, 0:j) * U(0:j, j) * inv(U_jj).
// A non-positive pivot records its 1-based position in status[ST_POTRF]; the
// remaining panels then return immediately.
#include "handle.cuh"

namespace {

constexpr int NBP = 64;

// One CTA of 32 x 32 threads factors the b x b diagonal block (b <= 64) and
// inverts the factor, as a 2 x 2 block recursion on 32 x 32 blocks held in
// shared memory (thread (r, c) owns element (r, c) of a 32-block):
//   U11 = chol(A11), X11 = U11^-1, U12 = X11^H A12, A22 -= U12^H U12,
//   U22 = chol(A22), X22 = U22^-1, X12 = -X11 U12 X22.
// FP64 vector throughput bounds this kernel, so the work is laid out such
// that whole warps (one row each) drop out of every elimination step.
// Rows/columns past b are padded with the identity.
constexpr int LDB = 65;

__device__ __forceinline__ bool chol32(cplx* A, double* rinv, int o, int tr, int tc, int* s_fail, int fail_base) {
  // A is the 64 x LDB shared block; factor A(o:o+32, o:o+32) in place (upper)
  if (tr == 0 && tc == 0) {
    const double a = A[o * LDB + o].x;
    rinv[o] = (a > 0.0) ? 1.0 / sqrt(a) : 0.0;
    if (!(a > 0.0)) *s_fail = fail_base + 1;
  }
  __syncthreads();
  for (int j = 0; j < 32; ++j) {
    if (*s_fail) return false;
    if (tr == j && tc >= j) A[(o + j) * LDB + o + tc] = cscale(A[(o + j) * LDB + o + tc], rinv[o + j]);
    __syncthreads();
    if (tr > j && tc >= tr) {
      cplx* x = &A[(o + tr) * LDB + o + tc];
      *x = csub(*x, cmulc(A[(o + j) * LDB + o + tr], A[(o + j) * LDB + o + tc]));
      if (tr == j + 1 && tc == j + 1) {
        const double a = x->x;
        rinv[o + j + 1] = (a > 0.0) ? 1.0 / sqrt(a) : 0.0;
        if (!(a > 0.0)) *s_fail = fail_base + j + 2;
      }
    }
    __syncthreads();
  }
  return true;
}

// X(o:o+32, o:o+32) = inverse of the upper factor U(o:o+32, o:o+32)
__device__ __forceinline__ void inv32(const cplx* A, cplx* X, const double* rinv, int o, int tr, int tc) {
  X[(o + tr) * LDB + o + tc] = cmk(tr == tc ? 1.0 : 0.0, 0.0);
  __syncthreads();
  for (int i = 31; i >= 0; --i) {
    if (tr == i && tc >= i) X[(o + i) * LDB + o + tc] = cscale(X[(o + i) * LDB + o + tc], rinv[o + i]);
    __syncthreads();
    if (tr < i && tc >= i)
      X[(o + tr) * LDB + o + tc] = csub(X[(o + tr) * LDB + o + tc],
                                        cmul(A[(o + tr) * LDB + o + i], X[(o + i) * LDB + o + tc]));
    __syncthreads();
  }
}

__device__ __forceinline__ void potrf_diag_block(int n, int kb, cplx* O, long long ld, cplx* Ui, int* status) {
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx* A = reinterpret_cast<cplx*>(dsm);   // 64 x LDB, row-major [r][c]
  cplx* X = A + NBP * LDB;
  __shared__ double rinv[NBP];
  __shared__ int s_fail;
  if (status[ST_POTRF] != 0) return;
  const int b = min(NBP, n - kb);
  const int tc = threadIdx.x & 31, tr = threadIdx.x >> 5;
  for (int t = threadIdx.x; t < NBP * NBP; t += 1024) {
    const int r = t % NBP, c = t / NBP;  // coalesced along r
    cplx a = cmk(r == c ? 1.0 : 0.0, 0.0);
    if (r < b && c < b && r <= c) a = O[(kb + r) + ld * (kb + c)];
    A[r * LDB + c] = a;
    X[r * LDB + c] = cmk(0.0, 0.0);
  }
  if (threadIdx.x == 0) s_fail = 0;
  __syncthreads();
  if (!chol32(A, rinv, 0, tr, tc, &s_fail, 0)) {
    if (threadIdx.x == 0 && s_fail <= b) atomicCAS(&status[ST_POTRF], 0, kb + s_fail);
    return;
  }
  inv32(A, X, rinv, 0, tr, tc);
  // U12 = X11^H A12 (thread (r, c): column 32 + c)
  {
    cplx acc = cmk(0.0, 0.0);
    for (int k = 0; k <= tr; ++k) acc = cadd(acc, cmulc(X[k * LDB + tr], A[k * LDB + 32 + tc]));
    __syncthreads();
    A[tr * LDB + 32 + tc] = acc;
    __syncthreads();
  }
  // A22 -= U12^H U12 (upper)
  if (tc >= tr) {
    cplx acc = cmk(0.0, 0.0);
    for (int k = 0; k < 32; ++k) acc = cadd(acc, cmulc(A[k * LDB + 32 + tr], A[k * LDB + 32 + tc]));
    A[(32 + tr) * LDB + 32 + tc] = csub(A[(32 + tr) * LDB + 32 + tc], acc);
  }
  __syncthreads();
  if (!chol32(A, rinv, 32, tr, tc, &s_fail, 32)) {
    if (threadIdx.x == 0 && s_fail <= b) atomicCAS(&status[ST_POTRF], 0, kb + s_fail);
    return;
  }
  inv32(A, X, rinv, 32, tr, tc);
  // X12 = -X11 (U12 X22): T = U12 X22 into X's lower-left block, then X12
  {
    cplx acc = cmk(0.0, 0.0);
    for (int k = 0; k <= tc; ++k) acc = cadd(acc, cmul(A[tr * LDB + 32 + k], X[(32 + k) * LDB + 32 + tc]));
    X[(32 + tr) * LDB + tc] = acc;  // scratch: lower-left block of X
    __syncthreads();
    cplx acc2 = cmk(0.0, 0.0);
    for (int k = tr; k < 32; ++k) acc2 = cadd(acc2, cmul(X[tr * LDB + k], X[(32 + k) * LDB + tc]));
    X[tr * LDB + 32 + tc] = cmk(-acc2.x, -acc2.y);
    __syncthreads();
  }
  for (int t = threadIdx.x; t < NBP * NBP; t += 1024) {
    const int r = t % NBP, c = t / NBP;
    if (r < b && c < b && r <= c) {
      O[(kb + r) + ld * (kb + c)] = A[r * LDB + c];
      Ui[(kb + r) + ld * (kb + c)] = X[r * LDB + c];
    }
  }
}

__global__ void __launch_bounds__(1024) k_potrf_diag(int n, int kb, cplx* O, long long ld, cplx* Ui,
                                                     int* status) {
  potrf_diag_block(n, kb, O, ld, Ui, status);
}

// Grouped form: CTA b factors diagonal block kb of problem b.
__global__ void __launch_bounds__(1024) k_potrf_diag_grouped(const PotrfProb* __restrict__ probs, int kb) {
  const PotrfProb p = probs[blockIdx.x];
  potrf_diag_block(p.n, kb, p.O, p.ld, p.Ui, p.status);
}

}  // namespace

int potrf_smem_bytes() { return (int)(2 * sizeof(cplx) * NBP * LDB); }
int potrf_block() { return NBP; }

int potrf_diag_grouped(cudaStream_t s, const PotrfProb* d_probs, int nprob, int kb) {
  if (nprob <= 0) return EXCFV_OK;
  const int smem = potrf_smem_bytes();
  CUDA_TRY(cudaFuncSetAttribute(k_potrf_diag_grouped, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_potrf_diag_grouped<<<nprob, 1024, smem, s>>>(d_probs, kb); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

int potrf_upper(excfv_handle* h, int n, cplx* O, cplx* Ui, long long ld) {
  cudaStream_t s = h->stream;
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0);
  const int smem = (int)(2 * sizeof(cplx) * NBP * LDB);
  CUDA_TRY(cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  for (int kb = 0; kb < n; kb += NBP) {
    const int b = min(NBP, n - kb);
    k_potrf_diag<<<1, 1024, smem, s>>>(n, kb, O, ld, Ui, h->ws.status); count_launch();
    CUDA_TRY(cudaGetLastError());
    const int rest = n - kb - b;
    if (rest <= 0) break;
    cplx* panel = O + kb + ld * (kb + b);
    // U(kb, rest) = inv(U_kk)^H A(kb, rest)   (in place: one row tile per CTA)
    int rc = zgemm1(s, OP_C, OP_N, b, rest, b, one, Ui + kb + ld * kb, ld, panel, ld,
                    cmk(0.0, 0.0), panel, ld, TRI_NONE, TRI_LOWER, TRI_NONE);
    if (rc) return rc;
    // A(rest, rest) -= U(kb, rest)^H U(kb, rest), upper triangle: an A^H B
    // product with K = 64 whose operand tiles a TMA ring brings three stages
    // ahead (zgemm_tma.cu), so the K loop is not bound by load latency
    const cplx* Pp[1] = {panel};
    cplx* Cp[1] = {O + (kb + b) + ld * (kb + b)};
    rc = zgemm_cn_tma(h, rest, rest, b, mone, Pp, ld, Pp, ld, one, Cp, ld, 1, TRI_UPPER);
    if (rc) return rc;
  }
  return EXCFV_OK;
}

// Ui = U^-1 (upper).  The diagonal NBP-blocks of Ui were written by
// k_potrf_diag; pairs of inverted blocks are merged level by level,
//   inv([[U11, U12], [0, U22]]) = [[X11, -X11 U12 X22], [0, X22]],
// with all pairs of one level in one batched GEMM (log2(n / NBP) levels).
// scratch: n x n complex.
int trtri_upper(excfv_handle* h, int n, const cplx* U, cplx* Ui, long long ld, cplx* scratch) {
  cudaStream_t s = h->stream;
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  for (int bs = NBP; bs < n; bs *= 2) {
    const int nfull = n / (2 * bs);             // pairs whose second block is complete
    const int rem = n - nfull * 2 * bs;          // rows left after the full pairs
    // full pairs, batched
    if (nfull > 0) {
      const long long step = 2LL * bs * (ld + 1);
      ZgemmArgs g;
      g.m = bs; g.n = bs; g.k = bs; g.kdec = 0; g.alpha = one; g.beta = zero;
      g.A = U + ld * bs; g.lda = ld; g.strideA = step;              // U12
      g.B = Ui + bs * (ld + 1); g.ldb = ld; g.strideB = step;        // X22
      g.C = scratch; g.ldc = bs; g.strideC = (long long)bs * bs;     // T = U12 X22
      g.batch = nfull; g.uplo_c = TRI_NONE; g.tri_a = TRI_NONE; g.tri_b = TRI_UPPER;
      g.splitk = 1; g.part = nullptr;
      int rc = zgemm(s, OP_N, OP_N, g);
      if (rc) return rc;
      g.alpha = mone;
      g.A = Ui; g.strideA = step;                                    // X11
      g.B = scratch; g.ldb = bs; g.strideB = (long long)bs * bs;     // T
      g.C = Ui + ld * bs; g.ldc = ld; g.strideC = step;              // X12
      g.tri_a = TRI_UPPER; g.tri_b = TRI_NONE;
      rc = zgemm(s, OP_N, OP_N, g);
      if (rc) return rc;
    }
    // a trailing pair whose second block is shorter than bs
    if (rem > bs) {
      const int a0 = nfull * 2 * bs, d0 = a0 + bs, sd = n - d0;
      cplx* T = scratch + (size_t)nfull * bs * bs;
      int rc = zgemm1(s, OP_N, OP_N, bs, sd, sd, one, U + a0 + ld * d0, ld, Ui + d0 + ld * d0, ld,
                      zero, T, bs, TRI_NONE, TRI_NONE, TRI_UPPER);
      if (rc) return rc;
      rc = zgemm1(s, OP_N, OP_N, bs, sd, bs, mone, Ui + a0 + ld * a0, ld, T, bs, zero,
                  Ui + a0 + ld * d0, ld, TRI_NONE, TRI_UPPER, TRI_NONE);
      if (rc) return rc;
    }
  }
  return EXCFV_OK;
}
