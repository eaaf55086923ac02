// The second-variational solve on the device: seceqnsv (src/seceqnsv.f90) on
// its default path (realspace = false), without LDA+U, for a collinear field
// (ndmag = 1: two eigenproblems of order nstfv) and for a non-collinear field
// with or without spin-orbit coupling (ndmag = 3: one of order 2 nstfv).
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
//
// Non-collinear (hmlint.f90:63-135): alpha from the z field, ab =
// mt_pot(x field) - i mt_pot(y field) with its alo kept explicitly (the
// spin-orbit terms break alo = loa^T), and the up-down block
//   Sud = ZWF^H (ab.aa ZWF + ab.alo E_LO) + E_LO^H (ab.loa ZWF + ab.lolo E_LO)
//       + E_G^H (M_xy E_G),   M_xy from bir1 - i bir2,
// then [[diag(evalfv) + S, Sud], [Sud^H, diag(evalfv) - S]] in one solve.
// The spin-orbit terms of mt_so.f90 are formed on the host (radial
// integrals of the spline rule, a few per atom) and added to alpha and ab;
// alpha's alo is then conj(loa)^T, as mt_so leaves it.
#include <tuple>
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

// the whole second-variational matrix of order 2n (ndmag = 3) from its up-up
// block S (upper triangle), the up-down block Sud and evalfv; O = I
__global__ void k_sv_full(int n, const cplx* S, const cplx* Sud, const double* evalfv, cplx* H, cplx* O) {
  const long long n2 = 2LL * n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n2 * n2) return;
  const int i = (int)(t % n2), j = (int)(t / n2);
  cplx v;
  if ((i < n) == (j < n)) {  // up-up, or down-down = -(up-up)
    const int a = i % n, b = j % n;
    const double sg = (i < n) ? 1.0 : -1.0;
    v = S[min(a, b) + (size_t)n * max(a, b)];
    v = cmk(sg * v.x, sg * v.y);
    if (a == b) v = cmk(v.x + evalfv[a], 0.0);
    else if (a > b) v = cmk(v.x, -v.y);
  } else if (i < n) {
    v = Sud[i + (size_t)n * (j - n)];
  } else {
    const cplx u = Sud[j + (size_t)n * (i - n)];
    v = cmk(u.x, -u.y);
  }
  H[t] = v;
  O[t] = cmk(i == j ? 1.0 : 0.0, 0.0);
}

// y += x (complex, n entries)
__global__ void k_sv_add(long long n, const cplx* x, cplx* y) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] = cadd(y[t], x[t]);
}

// y = y - i x: hmlint's ab = mt_pot(bx) - i mt_pot(by)
__global__ void k_sv_minus_i(long long n, const cplx* x, cplx* y) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[t] = cmk(y[t].x + x[t].y, y[t].y - x[t].x);
}

// alo(f, j, ias) = loa(j, f, ias): the transpose mt_pot leaves (mt_pot.f90:280)
__global__ void k_sv_transpose_lo(int maxaa, int nlo, int natmtot, const cplx* loa, cplx* alo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)maxaa * nlo * natmtot) return;
  const int f = (int)(t % maxaa), j = (int)((t / maxaa) % nlo), ias = (int)(t / ((long long)maxaa * nlo));
  alo[t] = loa[j + (size_t)nlo * (f + (size_t)maxaa * ias)];
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

// The spin-orbit terms of mt_so.f90 (InterstitialSO false; hmlint calls it at
// level_zora) on the host, added into dense host copies of the blocks: for
// radial functions p1, p2 of one l >= 1 and I = int p1 p2 rmtable2 r^2 with
// rmtable2 = d/dr [1 / (1 - alpha^2/2 V_00 y00)] / r (fderiv(1)),
//   alpha(l m, l m)  += m I / 2 (APW-APW, LO-APW, LO-LO; beta = -alpha),
//   ab(l m, l m+1)   += sqrt(l(l+1) - m(m+1)) I / 2 (APW-APW, APW-LO into
//                       ab.alo, LO-APW into ab.loa, LO-LO).
struct SoBlocks {
  std::vector<cplx> aa, loa, lolo, baa, bloa, balo, blolo;
};

void so_terms(const DevStatic& st, const excfv_mtrad* r, SoBlocks& o) {
  const int maxaa = st.maxaa, nlo1 = std::max(st.maxnlo, 1), nat = st.natmtot;
  const int L1 = st.lmaxapw + 1, nlm = std::max(1, st.nlomax), nrmax = r->nrmtmax;
  const int lmvr = (r->lmaxvr + 1) * (r->lmaxvr + 1);
  const double a = 0.5 / (137.03599911 * 137.03599911);
  o.aa.assign((size_t)maxaa * maxaa * nat, cmk(0.0, 0.0));
  o.baa = o.aa;
  o.loa.assign((size_t)nlo1 * maxaa * nat, cmk(0.0, 0.0));
  o.bloa = o.loa;
  o.balo.assign((size_t)maxaa * nlo1 * nat, cmk(0.0, 0.0));
  o.lolo.assign((size_t)nlo1 * nlo1 * nat, cmk(0.0, 0.0));
  o.blolo = o.lolo;
  std::vector<double> rm(nrmax), d1(nrmax), w(nrmax), prod(nrmax);
  auto cf = [](int l, int m) { return 0.5 * std::sqrt((double)(l * (l + 1) - m * (m + 1))); };
  auto add = [](std::vector<cplx>& v, size_t i, double x) { v[i].x += x; };
  for (int ias = 0; ias < nat; ++ias) {
    const int is = st.h_idxis[ias];
    const int nr = r->nrmt[is];
    const double* x = r->spr + (size_t)nrmax * is;
    for (int ir = 0; ir < nr; ++ir)
      rm[ir] = 1.0 / (1.0 - a * r->veffmt[(size_t)lmvr * (ir + (size_t)nrmax * ias)] * Y00C);
    host_spline(nr, x, rm.data(), d1.data());
    for (int ir = 0; ir < nr; ++ir) w[ir] = d1[ir] / x[ir] * x[ir] * x[ir];
    auto apw = [&](int io, int l) {
      return r->apwfr + (size_t)nrmax * 2 * (io + (size_t)st.apwordmax * (l + (size_t)L1 * ias));
    };
    auto lof = [&](int ilo) { return r->lofr + (size_t)nrmax * 2 * (ilo + (size_t)nlm * ias); };
    auto integral = [&](const double* p1, const double* p2) {
      for (int ir = 0; ir < nr; ++ir) prod[ir] = p1[ir] * p2[ir] * w[ir];
      return host_spline(nr, x, prod.data(), nullptr);
    };
    auto apword = [&](int l) { return st.h_apword[(size_t)l + (size_t)L1 * is]; };
    std::vector<int> off_l(st.lmaxmat + 2, 0);
    for (int l = 0; l <= st.lmaxmat; ++l) off_l[l + 1] = off_l[l] + apword(l) * (2 * l + 1);
    const int nlo = st.h_nlorb[is];
    std::vector<int> lol(nlo), lo_off(nlo + 1, 0);
    for (int ilo = 0; ilo < nlo; ++ilo) {
      lol[ilo] = st.h_lorbl[(size_t)ilo + (size_t)nlm * is];
      lo_off[ilo + 1] = lo_off[ilo] + 2 * lol[ilo] + 1;
    }
    const size_t oaa = (size_t)maxaa * maxaa * ias, oloa = (size_t)nlo1 * maxaa * ias;
    const size_t oalo = (size_t)maxaa * nlo1 * ias, ololo = (size_t)nlo1 * nlo1 * ias;
    // APW-APW (mt_so.f90:108-151)
    for (int l = 1; l <= st.lmaxmat; ++l) {
      const int no = apword(l);
      for (int io1 = 0; io1 < no; ++io1)
        for (int io2 = 0; io2 < no; ++io2) {
          const double v = integral(apw(io1, l), apw(io2, l));
          for (int m = -l; m <= l; ++m) {
            const int f1 = off_l[l] + (m + l) * no + io1;
            add(o.aa, oaa + f1 + (size_t)maxaa * (off_l[l] + (m + l) * no + io2), 0.5 * m * v);
            if (m != l) add(o.baa, oaa + f1 + (size_t)maxaa * (off_l[l] + (m + l + 1) * no + io2), cf(l, m) * v);
          }
        }
    }
    // APW-LO and LO-APW (:157-281)
    for (int ilo = 0; ilo < nlo; ++ilo) {
      const int l = lol[ilo];
      if (l == 0 || l > st.lmaxmat) continue;
      const int no = apword(l);
      for (int io = 0; io < no; ++io) {
        const double v = integral(apw(io, l), lof(ilo));
        for (int m = -l; m <= l; ++m) {
          const int j = lo_off[ilo] + m + l, f = off_l[l] + (m + l) * no + io;
          add(o.loa, oloa + j + (size_t)nlo1 * f, 0.5 * m * v);
          if (m != l) {
            add(o.balo, oalo + f + (size_t)maxaa * (j + 1), cf(l, m) * v);
            add(o.bloa, oloa + j + (size_t)nlo1 * (f + no), cf(l, m) * v);
          }
        }
      }
    }
    // LO-LO (:287-351)
    for (int ilo1 = 0; ilo1 < nlo; ++ilo1) {
      const int l = lol[ilo1];
      if (l == 0) continue;
      for (int ilo2 = 0; ilo2 < nlo; ++ilo2) {
        if (lol[ilo2] != l) continue;
        const double v = integral(lof(ilo1), lof(ilo2));
        for (int m = -l; m <= l; ++m) {
          const int j1 = lo_off[ilo1] + m + l, j2 = lo_off[ilo2] + m + l;
          add(o.lolo, ololo + j1 + (size_t)nlo1 * j2, 0.5 * m * v);
          if (m != l) add(o.blolo, ololo + j1 + (size_t)nlo1 * (j2 + 1), cf(l, m) * v);
        }
      }
    }
  }
}

}  // namespace

void free_sv(DevSV& v) {
  for (void* p : {(void*)v.aa, (void*)v.loa, (void*)v.lolo, (void*)v.birhat, (void*)v.evlo, (void*)v.zhlo,
                  (void*)v.S, (void*)v.evalfv, (void*)v.lo_first, (void*)v.status_save, (void*)v.ab_aa,
                  (void*)v.ab_loa, (void*)v.ab_alo, (void*)v.ab_lolo, (void*)v.birhat_xy, (void*)v.Sud})
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

namespace {

template <typename T>
int sv_alloc(T** p, size_t n) {
  if (cudaMalloc(p, sizeof(T) * std::max<size_t>(n, 1)) != cudaSuccess) {
    excfv_set_error("excfv_set_bfield_nc: cudaMalloc failed");
    return EXCFV_ERR_ALLOC;
  }
  cudaMemset(*p, 0, sizeof(T) * std::max<size_t>(n, 1));
  return EXCFV_OK;
}

// dst += the host array src (complex, n entries), through scratch
int sv_add_host(cudaStream_t s, cplx* dst, const std::vector<cplx>& src, cplx* scratch) {
  const long long n = (long long)src.size();
  if (n == 0) return EXCFV_OK;
  CUDA_TRY(cudaMemcpyAsync(scratch, src.data(), sizeof(cplx) * n, cudaMemcpyHostToDevice, s));
  k_sv_add<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(n, scratch, dst);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(s));  // the host array and the scratch are reused
  return EXCFV_OK;
}

}  // namespace

int stage_set_bfield_nc(excfv_handle* h, const excfv_bfield_nc* b) {
  DevStatic& st = h->st;
  DevSV& v = h->sv;
  free_sv(v);
  if (!b->rad || !b->bxcmt || !b->bmtconst || !b->ngrid || !b->bxcir || !b->cfunir ||
      (b->spinorb && !b->rad->veffmt)) {
    excfv_set_error("excfv_set_bfield_nc: missing arrays");
    return EXCFV_ERR_ARG;
  }
  const excfv_mtrad* r = b->rad;
  const int lmvr = (r->lmaxvr + 1) * (r->lmaxvr + 1);
  const size_t nr = (size_t)r->nrmtmax;
  const size_t N = (size_t)b->ngrid[0] * b->ngrid[1] * b->ngrid[2];
  if (r->lmaxvr < 0 || r->nrmtmax < 3 || N == 0) {
    excfv_set_error("excfv_set_bfield_nc: inconsistent sizes");
    return EXCFV_ERR_ARG;
  }
  cudaStream_t s = h->stream;
  const size_t nlo1 = std::max(st.maxnlo, 1), nst = std::max(st.nstfv, 1);
  const size_t naa = (size_t)st.maxaa * st.maxaa * st.natmtot, nloa = nlo1 * st.maxaa * st.natmtot;
  const size_t nlolo = nlo1 * nlo1 * st.natmtot;
  cplx *taa = nullptr, *tloa = nullptr, *tlolo = nullptr, *that = nullptr;
  int rc;
  if ((rc = sv_alloc(&v.aa, naa)) || (rc = sv_alloc(&v.loa, nloa)) || (rc = sv_alloc(&v.lolo, nlolo)) ||
      (rc = sv_alloc(&v.ab_aa, naa)) || (rc = sv_alloc(&v.ab_loa, nloa)) || (rc = sv_alloc(&v.ab_alo, nloa)) ||
      (rc = sv_alloc(&v.ab_lolo, nlolo)) || (rc = sv_alloc(&v.birhat, N)) || (rc = sv_alloc(&v.birhat_xy, N)) ||
      (rc = sv_alloc(&v.evlo, nlo1 * st.natmtot * nst)) || (rc = sv_alloc(&v.zhlo, nlo1 * st.natmtot * nst)) ||
      (rc = sv_alloc(&v.S, nst * nst)) || (rc = sv_alloc(&v.Sud, nst * nst)) || (rc = sv_alloc(&v.evalfv, nst)) ||
      (rc = sv_alloc(&v.lo_first, (size_t)st.natmtot)) || (rc = sv_alloc(&v.status_save, (size_t)ST_NWORDS)) ||
      (rc = sv_alloc(&taa, std::max(naa, N))) || (rc = sv_alloc(&tloa, nloa)) || (rc = sv_alloc(&tlolo, nlolo)) ||
      (rc = sv_alloc(&that, N))) {
    for (cplx* p : {taa, tloa, tlolo, that})
      if (p) cudaFree(p);
    free_sv(v);
    return rc;
  }
  auto fail = [&](int code) {
    cudaStreamSynchronize(s);
    for (cplx* p : {taa, tloa, tlolo, that})
      if (p) cudaFree(p);
    free_sv(v);
    return code;
  };
  std::vector<int> first(st.natmtot, -1);
  for (int a = 0; a < st.natmtot && a < (int)st.h_lo_first.size(); ++a) first[a] = st.h_lo_first[a];
  if (cudaMemcpy(v.lo_first, first.data(), sizeof(int) * st.natmtot, cudaMemcpyHostToDevice) != cudaSuccess)
    return fail(EXCFV_ERR_CUDA);
  // component d of the field with the atoms' constant field in its spherical part (hmlint.f90:63-135)
  auto component = [&](int d, std::vector<double>& field) {
    const size_t per = (size_t)lmvr * nr * st.natmtot;
    field.assign(b->bxcmt + per * d, b->bxcmt + per * (d + 1));
    for (int ias = 0; ias < st.natmtot; ++ias)
      for (size_t ir = 0; ir < nr; ++ir) field[(size_t)lmvr * (ir + nr * ias)] += b->bmtconst[d + 3 * ias] / Y00C;
  };
  std::vector<double> field;
  // alpha = mt_pot(z); ab = mt_pot(x) - i mt_pot(y); ab.alo = ab.loa^T
  component(2, field);
  if ((rc = stage_mt_field(h, r, field.data(), v.aa, v.loa, v.lolo, nullptr, nullptr, nullptr))) return fail(rc);
  component(0, field);
  if ((rc = stage_mt_field(h, r, field.data(), v.ab_aa, v.ab_loa, v.ab_lolo, nullptr, nullptr, nullptr)))
    return fail(rc);
  component(1, field);
  if ((rc = stage_mt_field(h, r, field.data(), taa, tloa, tlolo, nullptr, nullptr, nullptr))) return fail(rc);
  for (auto [x, y, n] : {std::make_tuple(taa, v.ab_aa, naa), std::make_tuple(tloa, v.ab_loa, nloa),
                         std::make_tuple(tlolo, v.ab_lolo, nlolo)}) {
    k_sv_minus_i<<<(unsigned)((n + 255) / 256), 256, 0, s>>>((long long)n, x, y);
    count_launch();
  }
  k_sv_transpose_lo<<<(unsigned)((nloa + 255) / 256), 256, 0, s>>>(st.maxaa, (int)nlo1, st.natmtot, v.ab_loa,
                                                                   v.ab_alo);
  count_launch();
  if (cudaGetLastError() != cudaSuccess) return fail(EXCFV_ERR_CUDA);
  // the spin-orbit terms of mt_so
  if (b->spinorb) {
    SoBlocks so;
    so_terms(st, r, so);
    if ((rc = sv_add_host(s, v.aa, so.aa, taa)) || (rc = sv_add_host(s, v.loa, so.loa, taa)) ||
        (rc = sv_add_host(s, v.lolo, so.lolo, taa)) || (rc = sv_add_host(s, v.ab_aa, so.baa, taa)) ||
        (rc = sv_add_host(s, v.ab_loa, so.bloa, taa)) || (rc = sv_add_host(s, v.ab_alo, so.balo, taa)) ||
        (rc = sv_add_host(s, v.ab_lolo, so.blolo, taa)))
      return fail(rc);
  }
  // the interstitial fields: bir3 and bir1 - i bir2 (seceqnsv.f90:660-665)
  if ((rc = stage_grid_field(h, b->ngrid, b->bxcir + 2 * N, b->cfunir, b->birconst[2], v.birhat)) ||
      (rc = stage_grid_field(h, b->ngrid, b->bxcir, b->cfunir, b->birconst[0], v.birhat_xy)) ||
      (rc = stage_grid_field(h, b->ngrid, b->bxcir + N, b->cfunir, b->birconst[1], that)))
    return fail(rc);
  k_sv_minus_i<<<(unsigned)((N + 255) / 256), 256, 0, s>>>((long long)N, that, v.birhat_xy);
  count_launch();
  if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) return fail(EXCFV_ERR_CUDA);
  for (cplx* p : {taa, tloa, tlolo, that}) cudaFree(p);
  for (int d = 0; d < 3; ++d) v.ngrid[d] = b->ngrid[d];
  v.nc = true;
  v.so = b->spinorb != 0;
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
  const int nsv = v.nc ? 2 * n : n;  // order of the eigenproblem(s)
  if (n > ws.ngkmax || ngp > ws.nmatmax || nsv > ws.kmax || nsv > ws.nmatmax) {
    excfv_set_error("excfv_seceqnsv: nstfv = %d exceeds the reserved workspace", n);
    return EXCFV_ERR_ARG;
  }
  // alpha's alo: loa^T as mt_pot leaves it, loa^H once mt_so has reset it
  const int alo_op = v.so ? OP_C : OP_T;
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
    if ((rc = gemm(s, alo_op, OP_N, st.maxaa, n, nlo1, v.loa, nlo1, (long long)nlo1 * st.maxaa, v.evlo, LM, nlo1,
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
  const int prec = h->prec;
  if (v.nc) {
    // the up-down block from ab (alo explicit) and the field bir1 - i bir2
    if ((rc = gemm(s, OP_N, OP_N, st.maxaa, n, st.maxaa, v.ab_aa, st.maxaa, (long long)st.maxaa * st.maxaa,
                   ws.Zpk, AM, st.maxaa, ws.Apk, AM, st.maxaa, st.natmtot, 0.0)))
      return rc;
    if (st.maxnlo > 0) {
      if ((rc = gemm(s, OP_N, OP_N, st.maxaa, n, nlo1, v.ab_alo, st.maxaa, (long long)nlo1 * st.maxaa, v.evlo, LM,
                     nlo1, ws.Apk, AM, st.maxaa, st.natmtot, 1.0)))
        return rc;
      if ((rc = gemm(s, OP_N, OP_N, nlo1, n, st.maxaa, v.ab_loa, nlo1, (long long)nlo1 * st.maxaa, ws.Zpk, AM,
                     st.maxaa, v.zhlo, LM, nlo1, st.natmtot, 0.0)))
        return rc;
      if ((rc = gemm(s, OP_N, OP_N, nlo1, n, nlo1, v.ab_lolo, nlo1, (long long)nlo1 * nlo1, v.evlo, LM, nlo1,
                     v.zhlo, LM, nlo1, st.natmtot, 1.0)))
        return rc;
    }
    if ((rc = gemm(s, OP_C, OP_N, n, n, (int)AM, ws.Zpk, AM, 0, ws.Apk, AM, 0, v.Sud, n, 0, 1, 0.0))) return rc;
    if (st.maxnlo > 0 &&
        (rc = gemm(s, OP_C, OP_N, n, n, (int)LM, v.evlo, LM, 0, v.zhlo, LM, 0, v.Sud, n, 0, 1, 1.0)))
      return rc;
    k_sv_conv<<<(unsigned)(((long long)ngp * ngp + 255) / 256), 256, 0, s>>>(
        ngp, ws.igpig, st.ivg, v.ngrid[0], v.ngrid[1], v.ngrid[2], v.birhat_xy, ws.T);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    if ((rc = gemm(s, OP_N, OP_N, ngp, n, ngp, ws.T, ngp, 0, evec, ldev, 0, ws.Z, ngp, 0, 1, 0.0))) return rc;
    if ((rc = gemm(s, OP_C, OP_N, n, n, ngp, evec, ldev, 0, ws.Z, ngp, 0, v.Sud, n, 0, 1, 1.0))) return rc;
    // one Hermitian eigensolve of order 2n (ZHEEV('V','U'), ndmag = 3), in FP64
    const long long n2 = 2LL * n;
    k_sv_full<<<(unsigned)((n2 * n2 + 255) / 256), 256, 0, s>>>(n, v.S, v.Sud, d_evalfv, ws.H, ws.O);
    count_launch();
    CUDA_TRY(cudaGetLastError());
    h->prec = EXCFV_PREC_FP64;
    rc = stage_solve(h, 2 * n, 2 * n, st.evaltol, d_evalsv, d_evecsv, n2);
    h->prec = prec;
    return rc;
  }
  // one Hermitian eigensolve per spin block, in FP64
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
