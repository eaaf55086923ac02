// Hamiltonian and overlap setup (src/src_eigensystem/hamiltonsetup.f90,
// overlapsetup.f90, hmlistln.f90, olpistln.f90, hamiltonoverlapocopy_UL.f90).
//
// Layout.  The matching coefficients of all atoms are held packed and
// stacked, Apk((a*maxaa + f), G) with f = (l, m, io) exactly as the apwi
// arrays of hamiltonsetup.f90:62-71, leading dimension natmtot*maxaa.  Then
//   Z   = blockdiag(aa_a) * Apk                 (batched over atoms)
//   H_GG = Apk^H Z,  O_GG = Apk^H (I + H1) Apk   (one GEMM each, K = natmtot*maxaa,
//                                                 upper triangle only)
// so the sum over atoms happens inside the K loop of one contraction instead
// of natmtot separate zgemm pairs writing the full N x N block.
//
// Only the upper triangles are formed: the reference's lower triangle is
// overwritten by conj(upper) in hamiltonoverlapocopy_UL before anything
// reads it, and ZHEGVX('U') reads the upper triangle only.
#include "handle.cuh"

namespace {

// LO band: columns N..n-1, rows 0..j (assigned, not accumulated).
// H(G, lo) = conj(loa * apwi)^T (hamiltonsetup.f90:131-149),
// O(G, lo_m) = conj(A(G, io, lm) (oalo + h1loa)) (overlapsetup.f90:119-131),
// H(lo, lo') = lolo (:154-161), O(lo_m, lo'_m) = ololo + h1lolo (:136-148).
__global__ void k_lo_band(int N, int n, int natmtot, int maxaa, int maxnlo, int nlomax,
                          int apwordmax, const int* idxis, const int* lo_atom, const int* lo_local,
                          const int* lo_lm, const int* lo_ilo, const int* fofl, int lmmax,
                          const cplx* Apk, const cplx* loa, const cplx* lolo, const double* oalo,
                          const double* ololo, cplx* H, cplx* O, long long ld) {
  const int j = N + blockIdx.y;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n || i > j) return;
  const int jl = j - N;
  const int a = lo_atom[jl], jj = lo_local[jl];
  const int lmj = lo_lm[jj + maxnlo * a], iloj = lo_ilo[jj + maxnlo * a];
  cplx hv = cmk(0.0, 0.0), ov = cmk(0.0, 0.0);
  const long long AM = (long long)natmtot * maxaa;
  if (i < N) {
    const cplx* ac = Apk + (long long)a * maxaa + AM * i;
    const cplx* lr = loa + jj + (long long)maxnlo * maxaa * a;
    // (loa * apwi)(jj, i) = sum_f loa(jj, f) A(i, f); we need its conjugate
    double re = 0.0, im = 0.0;
    for (int f = 0; f < maxaa; ++f) {
      const cplx x = lr[(long long)maxnlo * f];
      const cplx y = ac[f];
      re += x.x * y.x - x.y * y.y;
      im += x.x * y.y + x.y * y.x;
    }
    hv = cmk(re, -im);
    const int is = idxis[a];
    for (int io = 0; io < apwordmax; ++io) {
      const int f = fofl[(lmj * apwordmax + io) + lmmax * apwordmax * is];
      if (f < 0) continue;
      const cplx y = ac[f];
      const double c = oalo[io + apwordmax * (iloj + (long long)nlomax * a)];
      ov.x += c * y.x;
      ov.y -= c * y.y;
    }
  } else {
    const int il = i - N;
    if (lo_atom[il] == a) {
      const int ii = lo_local[il];
      hv = lolo[ii + maxnlo * (jj + (long long)maxnlo * a)];
      if (lo_lm[ii + maxnlo * a] == lmj) {
        const int iloi = lo_ilo[ii + maxnlo * a];
        ov = cmk(ololo[iloi + nlomax * (iloj + (long long)nlomax * a)], 0.0);
      }
    }
  }
  H[i + ld * j] = hv;
  O[i + ld * j] = ov;
}

// Interstitial terms on the upper triangle of the G+k block
// (hmlistln.f90:61-84, olpistln.f90:53-82):
//   g = ivgig(ivg(:,igpig(i)) - ivg(:,igpig(j))); if 0 < g <= ngvec:
//   H(i,j) += veffig(g) + 1/2 (G_i+k).(G_j+k) X(g),   O(i,j) += cfunig(g)
//   (+ a2/2 (G_i+k).(G_j+k) m2effig(g) when h1on).
__global__ void k_interstitial(int N, const int* __restrict__ gk_iv, const double* __restrict__ vgpc,
                               int lo1, int lo2, int lo3, int e1, int e2, int e3,
                               const int* __restrict__ ivgig, int ngvec,
                               const cplx* __restrict__ veffig, const cplx* __restrict__ xig,
                               const cplx* __restrict__ cfunig, const cplx* __restrict__ m2effig,
                               int h1on, cplx* H, cplx* O, long long ld) {
  const int i = blockIdx.x * 32 + threadIdx.x;
  const int j0 = blockIdx.y * 32;
  if (blockIdx.x > blockIdx.y) return;
  if (i >= N) return;
  const int ai = gk_iv[3 * i], bi = gk_iv[3 * i + 1], ci = gk_iv[3 * i + 2];
  const double vx = vgpc[3 * i], vy = vgpc[3 * i + 1], vz = vgpc[3 * i + 2];
  const double a2 = 0.5 / (137.03599911 * 137.03599911);
  for (int jj = threadIdx.y; jj < 32; jj += blockDim.y) {
    const int j = j0 + jj;
    if (j >= N || i > j) continue;
    const int d1 = ai - gk_iv[3 * j] - lo1;
    const int d2 = bi - gk_iv[3 * j + 1] - lo2;
    const int d3 = ci - gk_iv[3 * j + 2] - lo3;
    if (d1 < 0 || d1 >= e1 || d2 < 0 || d2 >= e2 || d3 < 0 || d3 >= e3) continue;
    const int g = ivgig[d1 + (long long)e1 * (d2 + (long long)e2 * d3)];
    if (g <= 0 || g > ngvec) continue;
    const double t1 = 0.5 * (vx * vgpc[3 * j] + vy * vgpc[3 * j + 1] + vz * vgpc[3 * j + 2]);
    const cplx v = veffig[g - 1], x = xig[g - 1];
    cplx* hp = H + i + ld * j;
    cplx hv = *hp;
    hv.x += v.x + t1 * x.x;
    hv.y += v.y + t1 * x.y;
    *hp = hv;
    cplx* op = O + i + ld * j;
    cplx ov = *op;
    const cplx c = cfunig[g - 1];
    ov.x += c.x;
    ov.y += c.y;
    if (h1on) {
      const cplx m2 = m2effig[g - 1];
      ov.x += a2 * t1 * m2.x;
      ov.y += a2 * t1 * m2.y;
    }
    *op = ov;
  }
}

__global__ void k_gk_iv(int N, const int* igpig, const int* ivg, int* gk_iv) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const int g = igpig[i] - 1;
  gk_iv[3 * i] = ivg[3 * g];
  gk_iv[3 * i + 1] = ivg[3 * g + 1];
  gk_iv[3 * i + 2] = ivg[3 * g + 2];
}

// A1((lm,io2), G) = A((lm,io2), G) + sum_io1 h1aa(io1, io2, l) A((lm,io1), G)
// (the zm of overlapsetup.f90:82-94, conjugated).
__global__ void k_apply_h1(int ngp, int natmtot, int maxaa, int apwordmax, int lmaxapw,
                           const int* idxis, const int* flist, const int* fofl, int lmmax,
                           const double* h1aa, const cplx* Apk, cplx* A1) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long rows = (long long)natmtot * maxaa;
  if (t >= rows * ngp) return;
  const int r = (int)(t % rows);
  const int ig = (int)(t / rows);
  const int f = r % maxaa, a = r / maxaa;
  const int is = idxis[a];
  const int code = flist[f + maxaa * is];
  cplx v = Apk[t];
  if (code >= 0) {
    const int lm = code / apwordmax, io2 = code % apwordmax;
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    for (int io1 = 0; io1 < apwordmax; ++io1) {
      const int f1 = fofl[(lm * apwordmax + io1) + lmmax * apwordmax * is];
      if (f1 < 0) continue;
      const double c = h1aa[io1 + apwordmax * (io2 + apwordmax * (l + (lmaxapw + 1) * (long long)a))];
      const cplx y = Apk[(long long)a * maxaa + f1 + rows * ig];
      v.x += c * y.x;
      v.y += c * y.y;
    }
  }
  A1[t] = v;
}

}  // namespace

// lower <- conj(upper), 32x32 tiles through shared memory (coalesced both ways)
__global__ void k_mirror_upper(int n, cplx* M, long long ld) {
  __shared__ cplx tile[32][33];
  const int bi = blockIdx.x, bj = blockIdx.y;  // tile (bi, bj) with bi >= bj is a lower tile
  if (bi < bj) return;
  const int tx = threadIdx.x, ty = threadIdx.y;
  // read upper tile (bj, bi): rows bj*32.., cols bi*32..
  for (int y = ty; y < 32; y += blockDim.y) {
    const int r = bj * 32 + tx, c = bi * 32 + y;
    if (r < n && c < n) tile[y][tx] = M[r + ld * c];
  }
  __syncthreads();
  for (int y = ty; y < 32; y += blockDim.y) {
    const int r = bi * 32 + tx, c = bj * 32 + y;  // lower element (r, c) = conj(M(c, r))
    if (r < n && c < n && r > c) {
      const cplx v = tile[tx][y];
      M[r + ld * c] = cmk(v.x, -v.y);
    }
  }
}

int mirror_upper(cudaStream_t s, int n, cplx* M, long long ld) {
  dim3 grid((n + 31) / 32, (n + 31) / 32);
  k_mirror_upper<<<grid, dim3(32, 8), 0, s>>>(n, M, ld); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// Grouped form of k_mirror_upper over problems of different order
// (blockIdx.z), optionally writing the complex64 copy of the full matrix.
__global__ void k_mirror_grouped(const MirrorProb* __restrict__ probs) {
  __shared__ cplx tile[32][33];
  const MirrorProb p = probs[blockIdx.z];
  const int bi = blockIdx.x, bj = blockIdx.y;
  const int n = p.n;
  if (bi < bj || bi * 32 >= n) return;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int y = ty; y < 32; y += blockDim.y) {
    const int r = bj * 32 + tx, c = bi * 32 + y;  // upper tile (bj, bi)
    if (r < n && c < n) {
      const cplx v = p.M[r + p.ld * c];
      tile[y][tx] = v;
      if (p.F && r <= c) p.F[r + p.ldf * c] = make_float2((float)v.x, (float)v.y);
    }
  }
  __syncthreads();
  for (int y = ty; y < 32; y += blockDim.y) {
    const int r = bi * 32 + tx, c = bj * 32 + y;
    if (r < n && c < n && r > c) {
      const cplx v = tile[tx][y];
      p.M[r + p.ld * c] = cmk(v.x, -v.y);
      if (p.F) p.F[r + p.ldf * c] = make_float2((float)v.x, (float)-v.y);
    }
  }
}

int mirror_grouped(cudaStream_t s, const MirrorProb* d_probs, int nprob, int nmax) {
  if (nprob <= 0) return EXCFV_OK;
  dim3 grid((nmax + 31) / 32, (nmax + 31) / 32, nprob);
  k_mirror_grouped<<<grid, dim3(32, 8), 0, s>>>(d_probs); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

int stage_setup(excfv_handle* h, int nmatp, int ngp, bool mirror_o) {
  DevStatic& st = h->st;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const int N = ngp, n = nmatp;
  const long long ld = n;
  const long long AM = (long long)st.natmtot * st.maxaa;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc;
  bind_gemm_ctx(h);
  CUDA_TRY(cudaMemsetAsync(ws.status + ST_SETUP, 0, sizeof(int), s));

  // Z_a = aa_a * A_a for every atom (hamiltonsetup.f90:75-88)
  ZgemmArgs z;
  z.m = st.maxaa; z.n = N; z.k = st.maxaa; z.alpha = one; z.beta = zero;
  z.A = st.aa; z.lda = st.maxaa; z.strideA = (long long)st.maxaa * st.maxaa;
  z.B = ws.Apk; z.ldb = AM; z.strideB = st.maxaa;
  z.C = ws.Zpk; z.ldc = AM; z.strideC = st.maxaa;
  z.batch = st.natmtot; z.uplo_c = TRI_NONE; z.tri_a = TRI_NONE; z.tri_b = TRI_NONE;
  z.splitk = 1; z.part = nullptr; z.kdec = 0;
  prof_begin(h, PROF_SETUP_OTHER);
  if ((rc = zgemm(s, OP_N, OP_N, z))) return rc;
  prof_end(h, PROF_SETUP_OTHER);
  CUDA_TRY(cudaGetLastError());
  // H_GG = sum_a A_a^H Z_a (hamiltonsetup.f90:90-103), upper triangle
  // O_GG = sum_a A_a^H (I + H1) A_a (overlapsetup.f90:82-108), upper triangle
  // A^H B contractions with TMA-fed operand tiles (zgemm_tma.cu)
  const cplx* Aop[2] = {ws.Apk, ws.Apk};
  if (h->prec == EXCFV_PREC_MIXED && !st.have_h1aa) {
    // precision form: split-BF16 tensor-core products recombined to FP64 (setup_bf16.cu)
    prof_begin(h, PROF_SETUP_GEMM);
    if ((rc = zgemm_cn_bf16x(h, N, (int)AM, ws.Apk, ws.Zpk, AM, ws.H, ws.O, ld))) return rc;
    prof_end(h, PROF_SETUP_GEMM);
  } else if (!st.have_h1aa) {
    // both contractions share A^H: one grid over both outputs
    const cplx* Bop[2] = {ws.Zpk, ws.Apk};
    cplx* Cop[2] = {ws.H, ws.O};
    prof_begin(h, PROF_SETUP_GEMM);
    if ((rc = zgemm_cn_tma(h, N, N, (int)AM, one, Aop, AM, Bop, AM, zero, Cop, ld, 2, TRI_UPPER))) return rc;
    prof_end(h, PROF_SETUP_GEMM);
  } else {
    // IORA*: Z is overwritten by (I + H1) A after the H contraction
    const cplx* Bop[1] = {ws.Zpk};
    cplx* Cop[1] = {ws.H};
    prof_begin(h, PROF_SETUP_GEMM);
    if ((rc = zgemm_cn_tma(h, N, N, (int)AM, one, Aop, AM, Bop, AM, zero, Cop, ld, 1, TRI_UPPER))) return rc;
    prof_end(h, PROF_SETUP_GEMM);
    const long long tot = AM * N;
    k_apply_h1<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(
        N, st.natmtot, st.maxaa, st.apwordmax, st.lmaxapw, st.idxis, st.flist, st.fofl,
        st.lmmaxapw, st.h1aa, ws.Apk, ws.Zpk); count_launch();
    CUDA_TRY(cudaGetLastError());
    cplx* Cop2[1] = {ws.O};
    prof_begin(h, PROF_SETUP_GEMM);
    if ((rc = zgemm_cn_tma(h, N, N, (int)AM, one, Aop, AM, Bop, AM, zero, Cop2, ld, 1, TRI_UPPER))) return rc;
    prof_end(h, PROF_SETUP_GEMM);
  }
  CUDA_TRY(cudaGetLastError());
  prof_begin(h, PROF_SETUP_OTHER);
  // local-orbital band (columns N..n-1)
  if (n > N) {
    dim3 grid((n + 127) / 128, n - N);
    k_lo_band<<<grid, 128, 0, s>>>(N, n, st.natmtot, st.maxaa, st.maxnlo, st.nlomax, st.apwordmax,
                                   st.idxis, st.lo_atom, st.lo_local, st.lo_lm, st.lo_ilo,
                                   st.fofl, st.lmmaxapw, ws.Apk, st.loa, st.lolo, st.oalo,
                                   st.ololo, ws.H, ws.O, ld); count_launch();
    CUDA_TRY(cudaGetLastError());
  }
  // interstitial
  k_gk_iv<<<(N + 127) / 128, 128, 0, s>>>(N, ws.igpig, st.ivg, ws.gk_iv); count_launch();
  CUDA_TRY(cudaGetLastError());
  {
    const int e1 = st.intgv[3] - st.intgv[0] + 1;
    const int e2 = st.intgv[4] - st.intgv[1] + 1;
    const int e3 = st.intgv[5] - st.intgv[2] + 1;
    dim3 grid((N + 31) / 32, (N + 31) / 32);
    k_interstitial<<<grid, dim3(32, 8), 0, s>>>(N, ws.gk_iv, ws.vgpc, st.intgv[0], st.intgv[1],
                                                st.intgv[2], e1, e2, e3, st.ivgig, st.ngvec,
                                                st.veffig, st.xig, st.cfunig, st.m2effig, st.h1on,
                                                ws.H, ws.O, ld); count_launch();
    CUDA_TRY(cudaGetLastError());
  }
  if ((rc = mirror_upper(s, n, ws.H, ld))) return rc;
  if (mirror_o && (rc = mirror_upper(s, n, ws.O, ld))) return rc;
  prof_end(h, PROF_SETUP_OTHER);
  return EXCFV_OK;
}
