// The second-variational solve for a collinear field on the device: seceqnsv
// (src/seceqnsv.f90) on its default path (realspace = false), without
// spin-orbit coupling and LDA+U, ndmag = 1.
//
//   ZWF  = A E_G                 (A: the packed matching coefficients, stacked
//                                 over atoms; E_G: the G rows of evecfv)
//   ZHWF = aa ZWF + loa^T E_LO   (per atom; alo = loa^T, mt_pot.f90:280)
//   ZHLO = loa ZWF + lolo E_LO
//   S    = ZWF^H ZHWF + E_LO^H ZHLO + E_G^H (M E_G)
// with M(G, G') = bhat((G - G') mod grid), bhat the forward transform of
// bir = (bxcir + ga4 bfieldc(3)) cfunir divided by the grid size: the
// product the reference forms per state by zfftifc(+1), a multiplication by
// bir and zfftifc(-1) (seceqnsv.f90:675-690) is exactly this circular
// convolution.  The up block is diag(evalfv) + S, the down block
// diag(evalfv) - S (beta = -alpha, zv(:,2) = -zfft2), each solved as a
// Hermitian eigenproblem from its upper triangle (ZHEEV('V','U')) by the
// library's FP64 eigensolver with the identity as overlap.  Every product
// is a DMMA GEMM of zgemm.cu.
#include <vector>

#include "handle.cuh"

namespace {

constexpr double Y00C = 0.28209479177387814347;

// E_LO(q + maxnlo ias, j) = evecfv(ngp + first(ias) + q, j) for the atom's LO functions, else 0
__global__ void k_sv_gather_lo(int natmtot, int maxnlo, int nst, int ngp, const int* lo_lm, const int* lo_first,
                               const cplx* evec, long long ldev, cplx* evlo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long rows = (long long)maxnlo * natmtot;
  if (t >= rows * nst) return;
  const int r = (int)(t % rows), j = (int)(t / rows);
  const int ias = r / maxnlo, q = r % maxnlo;
  cplx v = cmk(0.0, 0.0);
  if (lo_first[ias] >= 0 && lo_lm[q + maxnlo * ias] >= 0) v = evec[(size_t)(ngp + lo_first[ias] + q) + ldev * j];
  evlo[t] = v;
}

// M(g, g') = bhat(wrap(iv(g) - iv(g'))), iv the integer components of G+k's G
__global__ void k_sv_conv(int ngp, const int* igpig, const int* ivg, int n1, int n2, int n3, const cplx* bhat,
                          cplx* M) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)ngp * ngp) return;
  const int g = (int)(t % ngp), gp = (int)(t / ngp);
  const int* a = ivg + 3 * (size_t)(igpig[g] - 1);
  const int* b = ivg + 3 * (size_t)(igpig[gp] - 1);
  int d1 = (a[0] - b[0]) % n1, d2 = (a[1] - b[1]) % n2, d3 = (a[2] - b[2]) % n3;
  if (d1 < 0) d1 += n1;
  if (d2 < 0) d2 += n2;
  if (d3 < 0) d3 += n3;
  M[t] = bhat[(size_t)d1 + (size_t)n1 * (d2 + (size_t)n2 * d3)];
}

// the solver resets its status words per solve: keep the worse of both blocks
__global__ void k_sv_status_merge(int nwords, int* status, const int* saved) {
  const int i = threadIdx.x;
  if (i < nwords) status[i] = max(status[i], saved[i]);
}

// H = diag(evalfv) + sign S from S's upper triangle (the diagonal real), O = I
__global__ void k_sv_block(int n, double sign, const cplx* S, const double* evalfv, cplx* H, cplx* O) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)n * n) return;
  const int i = (int)(t % n), j = (int)(t / n);
  const int r = min(i, j), c = max(i, j);
  cplx v = S[r + (size_t)n * c];
  v = cmk(sign * v.x, sign * v.y);
  if (i == j) v = cmk(v.x + evalfv[i], 0.0);
  else if (i > j) v = cmk(v.x, -v.y);
  H[t] = v;
  O[t] = cmk(i == j ? 1.0 : 0.0, 0.0);
}

int gemm(cudaStream_t s, int opA, int opB, int m, int n, int k, const cplx* A, long long lda, long long sA,
         const cplx* B, long long ldb, long long sB, cplx* C, long long ldc, long long sC, int batch, double beta) {
  ZgemmArgs z;
  z.m = m; z.n = n; z.k = k;
  z.alpha = cmk(1.0, 0.0); z.beta = cmk(beta, 0.0);
  z.A = A; z.lda = lda; z.strideA = sA;
  z.B = B; z.ldb = ldb; z.strideB = sB;
  z.C = C; z.ldc = ldc; z.strideC = sC;
  z.batch = batch; z.uplo_c = TRI_NONE; z.tri_a = TRI_NONE; z.tri_b = TRI_NONE;
  z.splitk = 1; z.part = nullptr; z.kdec = 0;
  return zgemm(s, opA, opB, z);
}

}  // namespace

void free_sv(DevSV& v) {
  for (void* p : {(void*)v.aa, (void*)v.loa, (void*)v.lolo, (void*)v.birhat, (void*)v.evlo, (void*)v.zhlo,
                  (void*)v.S, (void*)v.evalfv, (void*)v.lo_first, (void*)v.status_save})
    if (p) cudaFree(p);
  v = DevSV();
}

int stage_set_bfield(excfv_handle* h, const excfv_bfield* b) {
  DevStatic& st = h->st;
  DevSV& v = h->sv;
  free_sv(v);
  if (!b->rad || !b->bxcmt || !b->bmtconst || !b->ngrid || !b->bxcir || !b->cfunir) {
    excfv_set_error("excfv_set_bfield: missing arrays");
    return EXCFV_ERR_ARG;
  }
  const excfv_mtrad* r = b->rad;
  const int lmvr = (r->lmaxvr + 1) * (r->lmaxvr + 1);
  const size_t nr = (size_t)r->nrmtmax;
  const size_t N = (size_t)b->ngrid[0] * b->ngrid[1] * b->ngrid[2];
  if (r->lmaxvr < 0 || r->nrmtmax < 3 || N == 0) {
    excfv_set_error("excfv_set_bfield: inconsistent sizes");
    return EXCFV_ERR_ARG;
  }
  // the constant field of each atom joins the spherical part (hmlint.f90:94)
  std::vector<double> field(b->bxcmt, b->bxcmt + (size_t)lmvr * nr * st.natmtot);
  for (int ias = 0; ias < st.natmtot; ++ias)
    for (size_t ir = 0; ir < nr; ++ir) field[(size_t)lmvr * (ir + nr * ias)] += b->bmtconst[ias] / Y00C;
  const size_t nlo1 = std::max(st.maxnlo, 1), nst = std::max(st.nstfv, 1);
  auto al = [](auto** p, size_t n) -> int {
    if (cudaMalloc(p, sizeof(**p) * std::max<size_t>(n, 1)) != cudaSuccess) {
      excfv_set_error("excfv_set_bfield: cudaMalloc failed");
      return EXCFV_ERR_ALLOC;
    }
    cudaMemset(*p, 0, sizeof(**p) * std::max<size_t>(n, 1));
    return EXCFV_OK;
  };
  int rc;
  if ((rc = al(&v.aa, (size_t)st.maxaa * st.maxaa * st.natmtot)) ||
      (rc = al(&v.loa, nlo1 * st.maxaa * st.natmtot)) || (rc = al(&v.lolo, nlo1 * nlo1 * st.natmtot)) ||
      (rc = al(&v.birhat, N)) || (rc = al(&v.evlo, nlo1 * st.natmtot * nst)) ||
      (rc = al(&v.zhlo, nlo1 * st.natmtot * nst)) || (rc = al(&v.S, nst * nst)) || (rc = al(&v.evalfv, nst)) ||
      (rc = al(&v.lo_first, (size_t)st.natmtot)) || (rc = al(&v.status_save, (size_t)ST_NWORDS))) {
    free_sv(v);
    return rc;
  }
  std::vector<int> first(st.natmtot, -1);
  for (int a = 0; a < st.natmtot && a < (int)st.h_lo_first.size(); ++a) first[a] = st.h_lo_first[a];
  CUDA_TRY(cudaMemcpy(v.lo_first, first.data(), sizeof(int) * st.natmtot, cudaMemcpyHostToDevice));
  if ((rc = stage_mt_field(h, r, field.data(), v.aa, v.loa, v.lolo, nullptr, nullptr, nullptr)) ||
      (rc = stage_grid_field(h, b->ngrid, b->bxcir, b->cfunir, b->birconst, v.birhat))) {
    free_sv(v);
    return rc;
  }
  for (int d = 0; d < 3; ++d) v.ngrid[d] = b->ngrid[d];
  v.ready = true;
  return EXCFV_OK;
}

// ws.Apk holds the k-point's packed matching coefficients and ws.igpig its
// G indices; evec (ld ldev) and d_evalfv on the device
int stage_seceqnsv(excfv_handle* h, int ngp, const cplx* evec, long long ldev, const double* d_evalfv,
                   double* d_evalsv, cplx* d_evecsv) {
  DevStatic& st = h->st;
  Workspace& ws = h->ws;
  DevSV& v = h->sv;
  cudaStream_t s = h->stream;
  const int n = st.nstfv;
  const long long AM = (long long)st.natmtot * st.maxaa;
  const int nlo1 = std::max(st.maxnlo, 1);
  const long long LM = (long long)nlo1 * st.natmtot;
  if (n > ws.ngkmax || ngp > ws.nmatmax || n > ws.kmax) {
    excfv_set_error("excfv_seceqnsv: nstfv = %d exceeds the reserved workspace", n);
    return EXCFV_ERR_ARG;
  }
  bind_gemm_ctx(h);
  int rc;
  // the muffin-tin part (seceqnsv.f90:239-560)
  if ((rc = gemm(s, OP_N, OP_N, (int)AM, n, ngp, ws.Apk, AM, 0, evec, ldev, 0, ws.Zpk, AM, 0, 1, 0.0))) return rc;
  k_sv_gather_lo<<<(unsigned)((LM * n + 255) / 256), 256, 0, s>>>(st.natmtot, nlo1, n, ngp, st.lo_lm,
                                                                   v.lo_first, evec, ldev, v.evlo);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  // ZHWF (into Apk, free after ZWF) = aa ZWF + loa^T E_LO per atom
  if ((rc = gemm(s, OP_N, OP_N, st.maxaa, n, st.maxaa, v.aa, st.maxaa, (long long)st.maxaa * st.maxaa, ws.Zpk,
                 AM, st.maxaa, ws.Apk, AM, st.maxaa, st.natmtot, 0.0)))
    return rc;
  if (st.maxnlo > 0) {
    if ((rc = gemm(s, OP_T, OP_N, st.maxaa, n, nlo1, v.loa, nlo1, (long long)nlo1 * st.maxaa, v.evlo, LM, nlo1,
                   ws.Apk, AM, st.maxaa, st.natmtot, 1.0)))
      return rc;
    // ZHLO = loa ZWF + lolo E_LO
    if ((rc = gemm(s, OP_N, OP_N, nlo1, n, st.maxaa, v.loa, nlo1, (long long)nlo1 * st.maxaa, ws.Zpk, AM,
                   st.maxaa, v.zhlo, LM, nlo1, st.natmtot, 0.0)))
      return rc;
    if ((rc = gemm(s, OP_N, OP_N, nlo1, n, nlo1, v.lolo, nlo1, (long long)nlo1 * nlo1, v.evlo, LM, nlo1, v.zhlo,
                   LM, nlo1, st.natmtot, 1.0)))
      return rc;
  }
  // S = ZWF^H ZHWF + E_LO^H ZHLO
  if ((rc = gemm(s, OP_C, OP_N, n, n, (int)AM, ws.Zpk, AM, 0, ws.Apk, AM, 0, v.S, n, 0, 1, 0.0))) return rc;
  if (st.maxnlo > 0 &&
      (rc = gemm(s, OP_C, OP_N, n, n, (int)LM, v.evlo, LM, 0, v.zhlo, LM, 0, v.S, n, 0, 1, 1.0)))
    return rc;
  // the interstitial part: S += E_G^H (M E_G)
  k_sv_conv<<<(unsigned)(((long long)ngp * ngp + 255) / 256), 256, 0, s>>>(ngp, ws.igpig, st.ivg, v.ngrid[0],
                                                                           v.ngrid[1], v.ngrid[2], v.birhat, ws.T);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  if ((rc = gemm(s, OP_N, OP_N, ngp, n, ngp, ws.T, ngp, 0, evec, ldev, 0, ws.Z, ngp, 0, 1, 0.0))) return rc;
  if ((rc = gemm(s, OP_C, OP_N, n, n, ngp, evec, ldev, 0, ws.Z, ngp, 0, v.S, n, 0, 1, 1.0))) return rc;
  // one Hermitian eigensolve per spin block, in FP64
  const int prec = h->prec;
  h->prec = EXCFV_PREC_FP64;
  CUDA_TRY(cudaMemsetAsync(d_evecsv, 0, sizeof(cplx) * (size_t)4 * n * n, s));
  for (int blk = 0; blk < 2 && rc == EXCFV_OK; ++blk) {
    k_sv_block<<<(unsigned)(((long long)n * n + 255) / 256), 256, 0, s>>>(n, blk ? -1.0 : 1.0, v.S, d_evalfv,
                                                                         ws.H, ws.O);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) {
      rc = EXCFV_ERR_CUDA;
      break;
    }
    rc = stage_solve(h, n, n, st.evaltol, d_evalsv + (size_t)blk * n,
                     d_evecsv + (size_t)blk * n + (size_t)2 * n * blk * n, 2LL * n);
    if (rc == EXCFV_OK && blk == 0 &&
        cudaMemcpyAsync(v.status_save, ws.status, sizeof(int) * ST_NWORDS, cudaMemcpyDeviceToDevice, s) !=
            cudaSuccess)
      rc = EXCFV_ERR_CUDA;
  }
  if (rc == EXCFV_OK) {
    k_sv_status_merge<<<1, 32, 0, s>>>(ST_NWORDS, ws.status, v.status_save);
    count_launch();
    if (cudaGetLastError() != cudaSuccess) rc = EXCFV_ERR_CUDA;
  }
  h->prec = prec;
  return rc;
}
