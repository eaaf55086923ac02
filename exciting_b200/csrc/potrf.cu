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

// One CTA of DT threads factors the b x b diagonal block (b <= 64) and
// inverts the factor, blocked in four 16-wide steps held in shared memory:
//   step j:  U_jj = chol(A_jj), X_jj = U_jj^-1   (one warp, in registers)
//            U_jc = X_jj^H A_jc            (c > j, the row panel)
//            A_cd -= U_jc^H U_jd           (j < c <= d, the trailing update)
// then X = U^-1 by merging the inverted diagonal blocks pairwise,
//   inv([[U11, U12], [0, U22]]) = [[X11, -X11 U12 X22], [0, X22]],
// for the 16-blocks (0,1), (2,3) and then the two 32-blocks.  Each 16 x 16
// leaf is one warp: lane c (and lane c + 16, which repeats it) keeps column c
// of the leaf in registers and takes the pivot row from the other lanes by
// shuffles, so the whole block needs about twenty CTA barriers.  Rows and
// columns past b are padded with the identity.
constexpr int LDB = 65;
constexpr int DT = 256;   // threads of the diagonal-block kernel
constexpr int LB = 16;    // leaf order

// Factors A(o:o+16, o:o+16) in place (upper; zeros below the diagonal) and
// writes its inverse into X(o:o+16, o:o+16).  Returns the 1-based position
// within the 64-block of the first pivot that is not positive (0 if none).
// Lanes apply every step to their whole column with a 0/1 weight instead of
// a branch (entries below the diagonal are never read as part of U).
__device__ __forceinline__ int leaf16(cplx* A, cplx* X, int o, int lane) {
  const unsigned full = 0xffffffffu;
  const int l = lane & (LB - 1);
  cplx a[LB];
#pragma unroll
  for (int r = 0; r < LB; ++r) a[r] = A[(o + r) * LDB + o + l];
  double rv[LB];
  int fail = 0;
#pragma unroll
  for (int j = 0; j < LB; ++j) {
    const double p = __shfl_sync(full, a[j].x, j);
    const bool ok = p > 0.0;
    if (!ok && fail == 0) fail = o + j + 1;
    const double ri = ok ? 1.0 / sqrt(p) : 0.0;
    rv[j] = ri;
    a[j] = cscale(a[j], (l >= j) ? ri : 1.0);   // row j of U (columns c >= j)
#pragma unroll
    for (int r = j + 1; r < LB; ++r) {     // A(r, c) -= conj(U(j, r)) U(j, c), c >= r
      const double m = (l >= r) ? 1.0 : 0.0;
      const cplx u = cmk(m * __shfl_sync(full, a[j].x, r), m * __shfl_sync(full, a[j].y, r));
      a[r] = csub(a[r], cmulc(u, a[j]));
    }
  }
  // back substitution U x = e_c for column c of X
  cplx x[LB];
#pragma unroll
  for (int i = LB - 1; i >= 0; --i) {
    cplx t = cmk(i == l ? 1.0 : 0.0, 0.0);
#pragma unroll
    for (int k = i + 1; k < LB; ++k) {
      const cplx u = cmk(__shfl_sync(full, a[i].x, k), __shfl_sync(full, a[i].y, k));
      t = csub(t, cmul(u, x[k]));
    }
    x[i] = cscale(t, rv[i]);
  }
  if (lane < LB) {
#pragma unroll
    for (int r = 0; r < LB; ++r) {
      A[(o + r) * LDB + o + l] = (r <= l) ? a[r] : cmk(0.0, 0.0);
      X[(o + r) * LDB + o + l] = (r <= l) ? x[r] : cmk(0.0, 0.0);
    }
  }
  return fail;
}

__device__ __forceinline__ void potrf_diag_block(int n, int kb, cplx* O, long long ld, cplx* Ui, int* status) {
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx* A = reinterpret_cast<cplx*>(dsm);   // 64 x LDB, row-major [r][c]
  cplx* X = A + NBP * LDB;
  __shared__ int s_fail;
  if (status[ST_POTRF] != 0) return;
  const int b = min(NBP, n - kb);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int t = tid; t < NBP * NBP; t += DT) {
    const int r = t % NBP, c = t / NBP;  // coalesced along r
    cplx a = cmk(r == c ? 1.0 : 0.0, 0.0);
    if (r < b && c < b && r <= c) a = O[(kb + r) + ld * (kb + c)];
    A[r * LDB + c] = a;
    X[r * LDB + c] = cmk(0.0, 0.0);
  }
  __syncthreads();
  for (int j = 0; j < NBP / LB; ++j) {
    const int o = j * LB;
    if (warp == 0) {
      const int f = leaf16(A, X, o, lane);
      if (lane == 0) s_fail = f;
    }
    __syncthreads();
    if (s_fail) {
      if (tid == 0 && s_fail <= b) atomicCAS(&status[ST_POTRF], 0, kb + s_fail);
      return;
    }
    const int c0 = o + LB, nc = NBP - c0;
    if (nc == 0) break;
    // row panel U(o+r, c) = sum_{k <= r} conj(X(o+k, o+r)) A(o+k, c)
    {
      cplx acc[3];
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int t = tid + q * DT;
        acc[q] = cmk(0.0, 0.0);
        if (t < LB * nc) {
          const int r = t % LB, c = c0 + t / LB;
          for (int k = 0; k <= r; ++k)
            acc[q] = cadd(acc[q], cmulc(X[(o + k) * LDB + o + r], A[(o + k) * LDB + c]));
        }
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int t = tid + q * DT;
        if (t < LB * nc) A[(o + t % LB) * LDB + c0 + t / LB] = acc[q];
      }
      __syncthreads();
    }
    // trailing update A(i, jj) -= sum_k conj(U(o+k, i)) U(o+k, jj), c0 <= i <= jj
    for (int t = tid; t < nc * nc; t += DT) {
      const int i = c0 + t % nc, jj = c0 + t / nc;
      if (i > jj) continue;
      cplx acc = cmk(0.0, 0.0);
#pragma unroll
      for (int k = 0; k < LB; ++k) acc = cadd(acc, cmulc(A[(o + k) * LDB + i], A[(o + k) * LDB + jj]));
      A[i * LDB + jj] = csub(A[i * LDB + jj], acc);
    }
    __syncthreads();
  }
  // X = U^-1: 16-blocks (0,1) and (2,3), then the 32-blocks; T goes to the
  // (unused) lower part of X
  for (int w = LB; w < NBP; w *= 2) {
    const int npair = NBP / (2 * w);
    // T = U12 X22 into X(p0 + w + r, p0 + c)
    for (int t = tid; t < npair * w * w; t += DT) {
      const int pr = t / (w * w), e = t % (w * w), r = e % w, c = e / w;
      const int p0 = pr * 2 * w;
      cplx acc = cmk(0.0, 0.0);
      for (int k = 0; k <= c; ++k)
        acc = cadd(acc, cmul(A[(p0 + r) * LDB + p0 + w + k], X[(p0 + w + k) * LDB + p0 + w + c]));
      X[(p0 + w + r) * LDB + p0 + c] = acc;
    }
    __syncthreads();
    // X12 = -X11 T
    for (int t = tid; t < npair * w * w; t += DT) {
      const int pr = t / (w * w), e = t % (w * w), r = e % w, c = e / w;
      const int p0 = pr * 2 * w;
      cplx acc = cmk(0.0, 0.0);
      for (int k = r; k < w; ++k)
        acc = cadd(acc, cmul(X[(p0 + r) * LDB + p0 + k], X[(p0 + w + k) * LDB + p0 + c]));
      X[(p0 + r) * LDB + p0 + w + c] = cmk(-acc.x, -acc.y);
    }
    __syncthreads();
  }
  for (int t = tid; t < NBP * NBP; t += DT) {
    const int r = t % NBP, c = t / NBP;
    if (r < b && c < b && r <= c) {
      O[(kb + r) + ld * (kb + c)] = A[r * LDB + c];
      Ui[(kb + r) + ld * (kb + c)] = X[r * LDB + c];
    }
  }
}

__global__ void __launch_bounds__(DT) k_potrf_diag(int n, int kb, cplx* O, long long ld, cplx* Ui,
                                                     int* status) {
  potrf_diag_block(n, kb, O, ld, Ui, status);
}

// Grouped form: CTA b factors diagonal block kb of problem b.
__global__ void __launch_bounds__(DT) k_potrf_diag_grouped(const PotrfProb* __restrict__ probs, int kb) {
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
  k_potrf_diag_grouped<<<nprob, DT, smem, s>>>(d_probs, kb); count_launch();
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
    k_potrf_diag<<<1, DT, smem, s>>>(n, kb, O, ld, Ui, h->ws.status); count_launch();
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
