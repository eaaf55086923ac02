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
constexpr int PT = 256;

__global__ void __launch_bounds__(PT) k_potrf_diag(int n, int kb, cplx* O, long long ld, cplx* Ui,
                                                   int* status) {
  extern __shared__ cplx sm[];
  cplx* A = sm;                  // b x b, column-major, ld NBP
  cplx* X = sm + NBP * NBP;      // inverse
  __shared__ int fail;
  if (status[ST_POTRF] != 0) return;
  const int b = min(NBP, n - kb);
  const int tid = threadIdx.x;
  for (int t = tid; t < b * b; t += PT) {
    const int r = t % b, c = t / b;
    A[r + NBP * c] = (r <= c) ? O[(kb + r) + ld * (kb + c)] : cmk(0.0, 0.0);
    X[r + NBP * c] = cmk(r == c ? 1.0 : 0.0, 0.0);
  }
  if (tid == 0) fail = 0;
  __syncthreads();
  // right-looking unblocked Cholesky on the upper triangle
  for (int j = 0; j < b; ++j) {
    const double ajj = A[j + NBP * j].x;
    if (!(ajj > 0.0)) {  // also catches NaN
      if (tid == 0) { fail = j + 1; }
      __syncthreads();
      break;
    }
    const double ujj = sqrt(ajj);
    const double inv = 1.0 / ujj;
    __syncthreads();
    for (int c = j + 1 + tid; c < b; c += PT) A[j + NBP * c] = cscale(A[j + NBP * c], inv);
    if (tid == 0) A[j + NBP * j] = cmk(ujj, 0.0);
    __syncthreads();
    // trailing: A(r, c) -= conj(U(j, r)) U(j, c), j < r <= c
    const int m = b - j - 1;
    for (int t = tid; t < m * m; t += PT) {
      const int r = j + 1 + t % m, c = j + 1 + t / m;
      if (r <= c) A[r + NBP * c] = csub(A[r + NBP * c], cmulc(A[j + NBP * r], A[j + NBP * c]));
    }
    __syncthreads();
  }
  if (fail) {
    if (tid == 0) atomicCAS(&status[ST_POTRF], 0, kb + fail);
    return;
  }
  // X = U^-1 by backward elimination on [U | I]: for i = b-1..0:
  // row i of X /= U(i,i); rows r < i: X(r,:) -= U(r,i) X(i,:)
  for (int i = b - 1; i >= 0; --i) {
    const double uii = A[i + NBP * i].x;
    for (int c = i + tid; c < b; c += PT) X[i + NBP * c] = cscale(X[i + NBP * c], 1.0 / uii);
    __syncthreads();
    for (int t = tid; t < i * (b - i); t += PT) {
      const int r = t % i, c = i + t / i;
      X[r + NBP * c] = csub(X[r + NBP * c], cmul(A[r + NBP * i], X[i + NBP * c]));
    }
    __syncthreads();
  }
  for (int t = tid; t < b * b; t += PT) {
    const int r = t % b, c = t / b;
    if (r <= c) {
      O[(kb + r) + ld * (kb + c)] = A[r + NBP * c];
      Ui[(kb + r) + ld * (kb + c)] = X[r + NBP * c];
    }
  }
}

}  // namespace

int potrf_upper(excfv_handle* h, int n, cplx* O, cplx* Ui, long long ld) {
  cudaStream_t s = h->stream;
  const size_t smem = 2 * NBP * NBP * sizeof(cplx);
  static bool attr = false;
  if (!attr) {
    CUDA_TRY(cudaFuncSetAttribute(k_potrf_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0);
  for (int kb = 0; kb < n; kb += NBP) {
    const int b = min(NBP, n - kb);
    k_potrf_diag<<<1, PT, smem, s>>>(n, kb, O, ld, Ui, h->ws.status); count_launch();
    CUDA_TRY(cudaGetLastError());
    const int rest = n - kb - b;
    if (rest <= 0) break;
    cplx* panel = O + kb + ld * (kb + b);
    // U(kb, rest) = inv(U_kk)^H A(kb, rest)   (in place: one row tile per CTA)
    int rc = zgemm1(s, OP_C, OP_N, b, rest, b, one, Ui + kb + ld * kb, ld, panel, ld,
                    cmk(0.0, 0.0), panel, ld, TRI_NONE, TRI_LOWER, TRI_NONE);
    if (rc) return rc;
    // A(rest, rest) -= U(kb, rest)^H U(kb, rest), upper triangle
    rc = zgemm1(s, OP_C, OP_N, rest, rest, b, mone, panel, ld, panel, ld, one,
                O + (kb + b) + ld * (kb + b), ld, TRI_UPPER);
    if (rc) return rc;
  }
  return EXCFV_OK;
}

// Ui = U^-1 (upper); the diagonal blocks were written by k_potrf_diag.
// scratch: n x NBP, leading dimension ld.
int trtri_upper(excfv_handle* h, int n, const cplx* U, cplx* Ui, long long ld, cplx* scratch) {
  cudaStream_t s = h->stream;
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  for (int jb = NBP; jb < n; jb += NBP) {
    const int b = min(NBP, n - jb);
    // W = U(0:jb, jb:jb+b) * inv(U_jj)
    int rc = zgemm1(s, OP_N, OP_N, jb, b, b, one, U + ld * jb, ld, Ui + jb + ld * jb, ld, zero,
                    scratch, ld, TRI_NONE, TRI_NONE, TRI_UPPER);
    if (rc) return rc;
    // Ui(0:jb, jb:jb+b) = -Ui(0:jb, 0:jb) * W
    rc = zgemm1(s, OP_N, OP_N, jb, b, jb, mone, Ui, ld, scratch, ld, zero, Ui + ld * jb, ld,
                TRI_NONE, TRI_UPPER, TRI_NONE);
    if (rc) return rc;
  }
  return EXCFV_OK;
}
