// Generalized Hermitian eigensolve H x = e O x for the lowest k states
// (ZHEGVX(1,'V','I','U'), src/src_eigensystem/modfvsystem.f90:691-693).
//
//   O = U^H U                      potrf_upper      (ZPOTRF)
//   Ui = U^-1                      trtri_upper
//   C = Ui^H (H Ui)                two GEMMs skipping the zero triangles (ZHEGST)
//   C = Q T Q^H                    tridiag_reduce   (ZHETRD)
//   T y = e y, lowest k            tridiag_eig      (DSTEBZ + DSTEIN)
//   Z = orth(y)                    Cholesky-QR on the k vectors
//   Z <- Q Z                       block reflectors (I - V Tf V^H), GEMMs (ZUNMTR)
//   X = Ui Z                       one GEMM (ZTRSM)
#include <algorithm>

#include "handle.cuh"

int potrf_upper(excfv_handle* h, int n, cplx* O, cplx* Ui, long long ld);
int trtri_upper(excfv_handle* h, int n, const cplx* U, cplx* Ui, long long ld, cplx* scratch);
int tridiag_reduce(excfv_handle* h, int n, cplx* C, long long ld);
int tridiag_nb();
int tridiag_eig(excfv_handle* h, int n, int k, double abstol, const double* d, const double* e,
                double* w, cplx* Z, long long ldz, double* scratch, int* iscratch);
int mirror_upper(cudaStream_t s, int n, cplx* M, long long ld);
int tridiag_reduce_f32(excfv_handle* h, int n, float2* C, long long ld);
int stage_reserve(excfv_handle* h, int nmatmax, int ngkmax, int kmax);

namespace {

constexpr int NBQ = 64;  // reflectors per block of the back-transform
constexpr int LT = 256;

// Triangular factor of the block reflector H_p ... H_{p+nb-1} = I - V T V^H
// (forward, columnwise: T(i,i) = tau_i, T(0:i,i) = -tau_i T(0:i,0:i) G(0:i,i)
// with G = V^H V from a batched GEMM).  One CTA per block; G and T live in
// shared memory, four threads share each row of the triangular product.
__global__ void __launch_bounds__(LT) k_larft(int n, const cplx* Gall, const cplx* tau, cplx* Tf) {
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx (*G)[NBQ + 1] = reinterpret_cast<cplx (*)[NBQ + 1]>(dsm);
  cplx (*T)[NBQ + 1] = reinterpret_cast<cplx (*)[NBQ + 1]>(dsm + sizeof(cplx) * NBQ * (NBQ + 1));
  const int blk = blockIdx.x;
  const int p = blk * NBQ;
  const int nb = min(NBQ, n - 1 - p);
  if (nb <= 0) return;
  const int tid = threadIdx.x;
  const cplx* Gb = Gall + (size_t)blk * NBQ * NBQ;
  for (int t = tid; t < NBQ * NBQ; t += LT) {
    const int r = t % NBQ, c = t / NBQ;
    G[r][c] = Gb[t];
    T[r][c] = cmk(0.0, 0.0);
  }
  __syncthreads();
  if (tid == 0) T[0][0] = tau[p];
  __syncthreads();
  const int row = tid >> 2, sub = tid & 3;
  for (int i = 1; i < nb; ++i) {
    const cplx ti = tau[p + i];
    cplx val = cmk(0.0, 0.0);
    if (row < i)
      for (int q = row + sub; q < i; q += 4) val = cadd(val, cmul(T[row][q], G[q][i]));
    val.x += __shfl_xor_sync(0xffffffffu, val.x, 1);
    val.y += __shfl_xor_sync(0xffffffffu, val.y, 1);
    val.x += __shfl_xor_sync(0xffffffffu, val.x, 2);
    val.y += __shfl_xor_sync(0xffffffffu, val.y, 2);
    __syncthreads();
    if (row < i && sub == 0) T[row][i] = cmul(cmk(-ti.x, -ti.y), val);
    if (tid == 0) T[i][i] = ti;
    __syncthreads();
  }
  cplx* out = Tf + (size_t)blk * NBQ * NBQ;
  for (int t = tid; t < NBQ * NBQ; t += LT) out[t] = T[t % NBQ][t / NBQ];
}

// n x n FP64 (leading dimension ldi) -> complex64 (leading dimension ldo)
__global__ void k_to_f32(int n, const cplx* __restrict__ in, long long ldi, float2* __restrict__ out,
                         long long ldo) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r >= n) return;
  const cplx v = in[r + ldi * c];
  out[r + ldo * c] = make_float2((float)v.x, (float)v.y);
}

// reflectors (below the diagonal) of an n x n complex64 matrix -> FP64
__global__ void k_lower_to_f64(int n, const float2* __restrict__ in, long long ldi,
                               cplx* __restrict__ out, long long ldo) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r >= n || r <= c) return;
  const float2 v = in[r + ldi * c];
  out[r + ldo * c] = cmk((double)v.x, (double)v.y);
}

// status words of the nested Rayleigh-Ritz solve added into the caller's
// (its Cholesky-QR word is not an overlap failure of the caller's problem)
__global__ void k_or_status(const int* from, int* to) {
  const int i = threadIdx.x;
  if (i < ST_NWORDS && i != ST_POTRF && from[i]) to[i] += from[i];
}

__global__ void k_copy_eval(int k, const double* w, double* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < k) out[j] = w[j];
}

}  // namespace

// Z (n x k) <- Q Z with Q = H_0 ... H_{n-2} from tridiag_reduce.
int apply_q(excfv_handle* h, int n, int k, const cplx* C, long long ld, cplx* Z, long long ldz) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (n < 2) return EXCFV_OK;
  const int nblk = (n - 1 + NBQ - 1) / NBQ;
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  cplx* Gall = ws.Tf + (size_t)nblk * NBQ * NBQ;
  // Gram matrices G_b = V_b^H V_b: the full blocks in one batched GEMM
  // (K shrinks by NBQ from block to block), the last partial block alone.
  const int nfull = (n - 1) / NBQ;
  if (nfull > 0) {
    ZgemmArgs g;
    g.m = NBQ; g.n = NBQ; g.k = n - 1; g.kdec = NBQ;
    g.alpha = one; g.beta = zero;
    g.A = C + 1; g.lda = ld; g.strideA = (long long)NBQ * (ld + 1);
    g.B = C + 1; g.ldb = ld; g.strideB = (long long)NBQ * (ld + 1);
    g.C = Gall; g.ldc = NBQ; g.strideC = (long long)NBQ * NBQ;
    g.batch = nfull; g.uplo_c = TRI_UPPER; g.tri_a = TRI_UPPER; g.tri_b = TRI_LOWER;
    g.splitk = 1; g.part = nullptr;
    int rc = zgemm(s, OP_C, OP_N, g);
    if (rc) return rc;
  }
  if (nfull < nblk) {
    const int p = nfull * NBQ;
    const int nb = n - 1 - p, m = n - p - 1;
    const cplx* V = C + (p + 1) + ld * p;
    int rc = zgemm1(s, OP_C, OP_N, nb, nb, m, one, V, ld, V, ld, zero, Gall + (size_t)nfull * NBQ * NBQ,
                    NBQ, TRI_UPPER, TRI_UPPER, TRI_LOWER);
    if (rc) return rc;
  }
  const int smem = (int)(2 * sizeof(cplx) * NBQ * (NBQ + 1));
  CUDA_TRY(cudaFuncSetAttribute(k_larft, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_larft<<<nblk, LT, smem, s>>>(n, Gall, ws.tau, ws.Tf); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* X1 = ws.Xs;
  cplx* X2 = ws.Xs + (size_t)NBQ * ws.kmax;
  for (int b = nblk - 1; b >= 0; --b) {
    const int p = b * NBQ;
    const int nb = min(NBQ, n - 1 - p);
    const int m = n - p - 1;
    const cplx* V = C + (p + 1) + ld * p;
    cplx* Zs = Z + (p + 1);
    int rc = zgemm1(s, OP_C, OP_N, nb, k, m, one, V, ld, Zs, ldz, zero, X1, NBQ, TRI_NONE,
                    TRI_UPPER, TRI_NONE);
    if (rc) return rc;
    rc = zgemm1(s, OP_N, OP_N, nb, k, nb, one, ws.Tf + (size_t)b * NBQ * NBQ, NBQ, X1, NBQ, zero,
                X2, NBQ, TRI_NONE, TRI_UPPER, TRI_NONE);
    if (rc) return rc;
    rc = zgemm1(s, OP_N, OP_N, m, k, nb, mone, V, ld, X2, NBQ, one, Zs, ldz, TRI_NONE, TRI_LOWER,
                TRI_NONE);
    if (rc) return rc;
  }
  return EXCFV_OK;
}

// Z (n x k) <- Z R^-1 with Z^H Z = R^H R (Cholesky-QR), scratch in ws.Gk/ws.Gki/ws.Z2.
int cholqr(excfv_handle* h, int n, int k, cplx*& Z, long long ldz) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc = zgemm1(s, OP_C, OP_N, k, k, n, one, Z, ldz, Z, ldz, zero, ws.Gk, k, TRI_UPPER);
  if (rc) return rc;
  if ((rc = potrf_upper(h, k, ws.Gk, ws.Gki, k))) return rc;
  if ((rc = trtri_upper(h, k, ws.Gk, ws.Gki, k, ws.Z2))) return rc;
  rc = zgemm1(s, OP_N, OP_N, n, k, k, one, Z, ldz, ws.Gki, k, zero, ws.Z2, ldz, TRI_NONE, TRI_NONE,
              TRI_UPPER);
  if (rc) return rc;
  cplx* t = Z;
  Z = ws.Z2;
  ws.Z2 = t;
  return EXCFV_OK;
}

// States carried through the complex64 reduction so that the Rayleigh-Ritz
// step has a buffer between the kept and the discarded part of the spectrum.
int mixed_states(int n, int k) { return std::min(n, k + std::max(16, k / 8)); }

static int stage_solve_mixed(excfv_handle* h, int n, int k, double evaltol, double* d_eval,
                             cplx* d_evec, long long ldevec);

int stage_solve(excfv_handle* h, int n, int k, double evaltol, double* d_eval, cplx* d_evec,
                long long ldevec) {
  if (h->prec == EXCFV_PREC_MIXED && n > 64)
    return stage_solve_mixed(h, n, k, evaltol, d_eval, d_evec, ldevec);
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const long long ld = n;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc;
  if (k < 1 || k > n) return EXCFV_ERR_ARG;
  bind_gemm_ctx(h);
  if (k > ws.kmax) return EXCFV_ERR_ARG;
  CUDA_TRY(cudaMemsetAsync(ws.status, 0, ST_NWORDS * sizeof(int), s));
  // O = U^H U, Ui = U^-1
  prof_begin(h, PROF_POTRF);
  if ((rc = potrf_upper(h, n, ws.O, ws.Ui, ld))) return rc;
  if ((rc = trtri_upper(h, n, ws.O, ws.Ui, ld, ws.T))) return rc;
  prof_end(h, PROF_POTRF);
  prof_begin(h, PROF_HEGST);
  // C = Ui^H H Ui (upper), then both triangles
  if ((rc = zgemm1(s, OP_N, OP_N, n, n, n, one, ws.H, ld, ws.Ui, ld, zero, ws.T, ld, TRI_NONE,
                   TRI_NONE, TRI_UPPER)))
    return rc;
  if ((rc = zgemm1(s, OP_C, OP_N, n, n, n, one, ws.Ui, ld, ws.T, ld, zero, ws.H, ld, TRI_UPPER,
                   TRI_LOWER, TRI_NONE)))
    return rc;
  if ((rc = mirror_upper(s, n, ws.H, ld))) return rc;
  prof_end(h, PROF_HEGST);
  // tridiagonal reduction
  if ((rc = tridiag_reduce(h, n, ws.H, ld))) return rc;
  // eigenpairs of T
  cplx* Z = ws.Z;
  prof_begin(h, PROF_STEIG);
  if ((rc = tridiag_eig(h, n, k, evaltol, ws.d, ws.e, ws.w, Z, ld, ws.stein_ws, ws.icl)))
    return rc;
  prof_end(h, PROF_STEIG);
  prof_begin(h, PROF_BACKTR);
  if ((rc = cholqr(h, n, k, Z, ld))) return rc;
  // back-transforms
  if ((rc = apply_q(h, n, k, ws.H, ld, Z, ld))) return rc;
  if ((rc = zgemm1(s, OP_N, OP_N, n, k, n, one, ws.Ui, ld, Z, ld, zero, d_evec, ldevec, TRI_NONE,
                   TRI_UPPER, TRI_NONE)))
    return rc;
  prof_end(h, PROF_BACKTR);
  ws.Z = Z;  // cholqr may have swapped the buffers
  k_copy_eval<<<(k + 127) / 128, 128, 0, s>>>(k, ws.w, d_eval); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// Standard Hermitian eigenproblem on ws.H (n x n, both triangles, destroyed):
// lowest k eigenpairs -> ws.w and Z (n x k, ld n; returned pointer, one of
// ws.Z / ws.Z2).  The k' x k' Rayleigh-Ritz problem of the precision form.
static int solve_standard(excfv_handle* h, int n, int k, double evaltol, cplx** Zout) {
  Workspace& ws = h->ws;
  int rc;
  if ((rc = tridiag_reduce(h, n, ws.H, n))) return rc;
  cplx* Z = ws.Z;
  if ((rc = tridiag_eig(h, n, k, evaltol, ws.d, ws.e, ws.w, Z, n, ws.stein_ws, ws.icl))) return rc;
  if ((rc = cholqr(h, n, k, Z, n))) return rc;
  if ((rc = apply_q(h, n, k, ws.H, n, Z, n))) return rc;
  ws.Z = Z;
  *Zout = Z;
  return EXCFV_OK;
}

// The precision form: FP64 Cholesky and reduction to C = U^-H H U^-1; the
// Householder tridiagonal reduction of a complex64 copy of C; eigenpairs of T
// for k' = k + extra states and their back-transform; then Rayleigh-Ritz in
// FP64: X0 = orth(Q Z_T), Hk = X0^H C X0 (k' x k') solved in FP64, X = X0 Y.
// The Ritz values' errors are second order in the FP32 perturbation of X0
// (relative to the gap between state k and the discarded states beyond k').
static int stage_solve_mixed(excfv_handle* h, int n, int k, double evaltol, double* d_eval,
                             cplx* d_evec, long long ldevec) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const long long ld = n;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc;
  const int kx = mixed_states(n, k);
  if (k < 1 || k > n) return EXCFV_ERR_ARG;
  if (kx > ws.kmax) {
    excfv_set_error("mixed solve: workspace holds %d states, needs %d", ws.kmax, kx);
    return EXCFV_ERR_ARG;
  }
  bind_gemm_ctx(h);
  CUDA_TRY(cudaMemsetAsync(ws.status, 0, ST_NWORDS * sizeof(int), s));
  prof_begin(h, PROF_POTRF);
  if ((rc = potrf_upper(h, n, ws.O, ws.Ui, ld))) return rc;
  if ((rc = trtri_upper(h, n, ws.O, ws.Ui, ld, ws.T))) return rc;
  prof_end(h, PROF_POTRF);
  prof_begin(h, PROF_HEGST);
  if ((rc = zgemm1(s, OP_N, OP_N, n, n, n, one, ws.H, ld, ws.Ui, ld, zero, ws.T, ld, TRI_NONE,
                   TRI_NONE, TRI_UPPER)))
    return rc;
  if ((rc = zgemm1(s, OP_C, OP_N, n, n, n, one, ws.Ui, ld, ws.T, ld, zero, ws.H, ld, TRI_UPPER,
                   TRI_LOWER, TRI_NONE)))
    return rc;
  if ((rc = mirror_upper(s, n, ws.H, ld))) return rc;
  // complex64 copy of C for the reduction (ws.T is free now); an even leading
  // dimension keeps its columns 16-byte aligned for the tile loads
  float2* Cf = reinterpret_cast<float2*>(ws.T);
  const long long ldf = (n + 1) & ~1;
  k_to_f32<<<dim3((n + 255) / 256, n), 256, 0, s>>>(n, ws.H, ld, Cf, ldf); count_launch();
  CUDA_TRY(cudaGetLastError());
  prof_end(h, PROF_HEGST);
  if ((rc = tridiag_reduce_f32(h, n, Cf, ldf))) return rc;
  // reflectors back to FP64 into ws.O (the Cholesky factor is no longer needed)
  k_lower_to_f64<<<dim3((n + 255) / 256, n), 256, 0, s>>>(n, Cf, ldf, ws.O, ld); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* Z = ws.Z;
  prof_begin(h, PROF_STEIG);
  if ((rc = tridiag_eig(h, n, kx, evaltol, ws.d, ws.e, ws.w, Z, ld, ws.stein_ws, ws.icl))) return rc;
  prof_end(h, PROF_STEIG);
  prof_begin(h, PROF_BACKTR);
  if ((rc = apply_q(h, n, kx, ws.O, ld, Z, ld))) return rc;
  if ((rc = cholqr(h, n, kx, Z, ld))) return rc;
  // R = C X0 (FP64, full C)
  cplx* R = ws.Z2;
  if ((rc = zgemm1(s, OP_N, OP_N, n, kx, n, one, ws.H, ld, Z, ld, zero, R, ld))) return rc;
  // the k' x k' problem runs on a nested context with its own workspace
  if (!h->sub) {
    h->sub = new excfv_handle();
    h->sub->owns_static = false;
  }
  excfv_handle* sub = h->sub;
  sub->device = h->device;
  sub->nsm = h->nsm;
  sub->grid_ctas = h->grid_ctas;
  sub->stream = s;
  sub->st = h->st;
  sub->have_static = h->have_static;
  sub->prec = EXCFV_PREC_FP64;
  sub->prof.on = false;
  if ((rc = stage_reserve(sub, kx, 1, k))) return rc;
  if ((rc = zgemm1(s, OP_C, OP_N, kx, kx, n, one, Z, ld, R, ld, zero, sub->ws.H, kx, TRI_UPPER)))
    return rc;
  if ((rc = mirror_upper(s, kx, sub->ws.H, kx))) return rc;
  CUDA_TRY(cudaMemsetAsync(sub->ws.status, 0, ST_NWORDS * sizeof(int), s));
  cplx* Y = nullptr;
  if ((rc = solve_standard(sub, kx, k, evaltol, &Y))) return rc;
  bind_gemm_ctx(h);
  // X = X0 Y (n x k) into R's buffer, then the back-transform with U^-1
  if ((rc = zgemm1(s, OP_N, OP_N, n, k, kx, one, Z, ld, Y, kx, zero, R, ld))) return rc;
  if ((rc = zgemm1(s, OP_N, OP_N, n, k, n, one, ws.Ui, ld, R, ld, zero, d_evec, ldevec, TRI_NONE,
                   TRI_UPPER, TRI_NONE)))
    return rc;
  ws.Z = Z;
  k_copy_eval<<<(k + 127) / 128, 128, 0, s>>>(k, sub->ws.w, d_eval); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_or_status<<<1, ST_NWORDS, 0, s>>>(sub->ws.status, ws.status); count_launch();
  CUDA_TRY(cudaGetLastError());
  prof_end(h, PROF_BACKTR);
  return EXCFV_OK;
}

int stage_status(excfv_handle* h, int n) {
  int st[ST_NWORDS];
  CUDA_TRY(cudaMemcpyAsync(st, h->ws.status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return status_to_info(st, n);
}

int status_to_info(const int* st, int n) {
  if (st[ST_BARRIER]) {
    excfv_set_error("grid barrier timed out in the tridiagonal reduction");
    return EXCFV_ERR_TIMEOUT;
  }
  if (st[ST_POTRF]) return n + st[ST_POTRF];
  if (st[ST_STEBZ]) {
    excfv_set_error("bisection did not converge for %d eigenvalues", st[ST_STEBZ]);
    return EXCFV_ERR_NOCONV;
  }
  if (st[ST_STEIN]) return st[ST_STEIN];
  return EXCFV_OK;
}
