// The per-SCF-iteration muffin-tin Hamiltonian and radial overlaps on the
// device: hmlint = mt_kin + mt_pot (src/src_eigensystem/hmlint.f90:14-58,
// mt_kin.f90:64-230, mt_pot.f90:131-311) and olprad (olprad.f90:30-143),
// written straight into the handle's aa / loa / lolo / oalo / ololo / h1aa.
//
// Every radial integral of the reference is the spline integral of
// fderiv(-1) (src/src_lib/fderiv.f90 with spline.f90) over the species'
// mesh, a linear functional of the integrand: integral = sum_r w_r f(r), with
// weights w fixed by the mesh (the spline rule applied to the unit vectors,
// computed once per call on the host).  So the build is
//   radial integrals   one thread per integral, a weighted sum over r of
//                      products of radial functions (with r^2, the ZORA
//                      factor 1/(1 - a V_00 y00), the potential's lm);
//   Gaunt contraction  one thread per matrix element: aa(f1, f3) = kinetic
//                      (same lm) + sum_lm2 gntyry(lm1, lm2, lm3) haa(lm2),
//                      the same for loa and lolo.
// The Gaunt table gntyry(lm1, lm2, lm3) = integral of conj(Y_lm1) R_lm2
// Y_lm3 (R the real harmonics, lm2 up to lmaxvr) comes from Gauss-Legendre
// quadrature in cos(theta) of the Y_lm of specfun.cuh at phi = 0 (the phi
// integral is 2 pi delta(m1 = m2 + m3)); the nodes by Newton's method on the
// Legendre recurrence.
#include <cmath>
#include <vector>

#include "handle.cuh"
#include "specfun.cuh"

namespace {

constexpr double Y00C = 0.28209479177387814347;
constexpr double ALPHA_FS = 1.0 / 137.03599911;

// ---- host: spline integral weights -------------------------------------
// The integral of fderiv(-1) over the whole mesh for one integrand f: the
// spline coefficients by the recurrences of spline.f90, then the sum of the
// per-interval cubic integrals.
double spline_integral(int n, const double* x, const double* f, std::vector<double>& c1,
                       std::vector<double>& c2, std::vector<double>& c3, std::vector<double>& w) {
  for (int i = 0; i < n - 1; ++i) {
    w[i] = 1.0 / (x[i + 1] - x[i]);
    c1[i] = w[i] * (f[i + 1] - f[i]);
  }
  c2[0] = 1.0;
  c3[0] = (c1[1] - c1[0]) / (x[2] - x[0]);
  double t1 = (x[1] - x[0]) * w[1];
  double t2 = t1 * c2[0];
  double t3 = 1.0 / (2.0 * (t1 + 1.0));
  c2[1] = t3;
  double t4 = 3.0 * (c1[1] - c1[0]) * w[1] - t2 * c3[0];
  c3[1] = t4;
  for (int i = 2; i < n - 1; ++i) {
    t1 = (x[i] - x[i - 1]) * w[i];
    t2 = t1 * t3;
    t3 = 1.0 / (2.0 * t1 + 2.0 - t2);
    c2[i] = t3;
    t4 = 3.0 * (c1[i] - c1[i - 1]) * w[i] - t2 * t4;
    c3[i] = t4;
  }
  c2[n - 1] = 1.0;
  t1 = (c1[n - 2] - c1[n - 3]) / (x[n - 1] - x[n - 3]);
  c3[n - 1] = t1;
  for (int i = n - 2; i >= 1; --i) {
    t1 = c3[i] - t1 * c2[i + 1];
    c3[i] = t1;
  }
  for (int i = 0; i < n; ++i) c2[i] *= c3[i];
  double g = 0.0;
  for (int i = 0; i < n - 1; ++i) {
    const double d3 = (1.0 / 3.0) * (c2[i + 1] - c2[i]) * w[i];
    const double dx = x[i + 1] - x[i];
    const double d1 = c1[i] - (c2[i] + d3 * dx) * dx;
    g += (((0.25 * d3 * dx + (1.0 / 3.0) * c2[i]) * dx + 0.5 * d1) * dx + f[i]) * dx;
  }
  return g;
}

// weights w_j with integral(f) = sum_j w_j f_j (the rule is linear in f)
void spline_weights(int n, const double* x, double* wout) {
  std::vector<double> c1(n), c2(n), c3(n), w(n), e(n, 0.0);
  for (int j = 0; j < n; ++j) {
    e[j] = 1.0;
    wout[j] = spline_integral(n, x, e.data(), c1, c2, c3, w);
    e[j] = 0.0;
  }
}

// ---- host: Gaunt table ---------------------------------------------------
void gauss_legendre(int n, std::vector<double>& xq, std::vector<double>& wq) {
  xq.assign(n, 0.0);
  wq.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = cos(M_PI * (i + 0.75) / (n + 0.5));
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      const double dp = n * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) {
        xq[i] = z;
        wq[i] = 2.0 / ((1.0 - z * z) * dp * dp);
        break;
      }
      xq[i] = z;
      wq[i] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
  }
}

// gnt[(lm1 * lmmat + lm3) * lmvr + lm2] = integral conj(Y_lm1) R_lm2 Y_lm3
void gaunt_yry_table(int lmaxmat, int lmaxvr, std::vector<cplx>& gnt) {
  const int lmmat = (lmaxmat + 1) * (lmaxmat + 1), lmvr = (lmaxvr + 1) * (lmaxvr + 1);
  const int L = std::max(lmaxmat, lmaxvr);
  const int nq = (2 * lmaxmat + lmaxvr) / 2 + 2;
  std::vector<double> xq, wq;
  gauss_legendre(nq, xq, wq);
  const int lmL = (L + 1) * (L + 1);
  std::vector<cplx> y((size_t)nq * lmL);
  for (int q = 0; q < nq; ++q) sf_ylm(L, acos(xq[q]), 0.0, y.data() + (size_t)q * lmL, 1);
  auto lof = [](int lm) { int l = 0; while ((l + 1) * (l + 1) <= lm) ++l; return l; };
  auto yyy = [&](int a, int b, int c) -> double {
    const int l1 = lof(a), l2 = lof(b), l3 = lof(c);
    const int m1 = a - l1 * (l1 + 1), m2 = b - l2 * (l2 + 1), m3 = c - l3 * (l3 + 1);
    if (m1 != m2 + m3 || ((l1 + l2 + l3) & 1) || l1 > l2 + l3 || l2 > l1 + l3 || l3 > l1 + l2) return 0.0;
    double s = 0.0;
    for (int q = 0; q < nq; ++q)
      s += wq[q] * y[(size_t)q * lmL + a].x * y[(size_t)q * lmL + b].x * y[(size_t)q * lmL + c].x;
    return 2.0 * M_PI * s;
  };
  gnt.assign((size_t)lmmat * lmmat * lmvr, cmk(0.0, 0.0));
  const double sh = sqrt(0.5);
  for (int lm1 = 0; lm1 < lmmat; ++lm1)
    for (int lm3 = 0; lm3 < lmmat; ++lm3)
      for (int l2 = 0; l2 <= lmaxvr; ++l2)
        for (int m2 = -l2; m2 <= l2; ++m2) {
          const int lm2 = l2 * (l2 + 1) + m2, lmm = l2 * (l2 + 1) - m2;
          const double sg = (m2 & 1) ? -1.0 : 1.0;
          cplx v;
          if (m2 > 0) v = cmk(sh * (yyy(lm1, lm2, lm3) + sg * yyy(lm1, lmm, lm3)), 0.0);
          else if (m2 < 0) v = cmk(0.0, -sh * (yyy(lm1, lm2, lm3) - sg * yyy(lm1, lmm, lm3)));
          else v = cmk(yyy(lm1, lm2, lm3), 0.0);
          gnt[((size_t)lm1 * lmmat + lm3) * lmvr + lm2] = v;
        }
}

// ---- device ------------------------------------------------------------------
struct MtArgs {
  int natmtot, lmaxmat, lmaxapw, apwordmax, nlomax, lmvr, nrmtmax, maxaa, maxnlo;
  const int* idxis;     // (natmtot)
  const int* nrmt;      // (nspecies)
  const int* apword;    // (lmaxapw+1, nspecies)
  const int* nlorb;     // (nspecies)
  const int* lorbl;     // (nlomax, nspecies)
  const double* wts;    // (nrmtmax, nspecies) spline-integral weights times r^2
  const double* spr;    // (nrmtmax, nspecies)
  const double* apwfr;  // (nrmtmax, 2, apwordmax, lmaxapw+1, natmtot)
  const double* lofr;   // (nrmtmax, 2, nlomax, natmtot)
  const double* veff;   // (lmvr, nrmtmax, natmtot)
  double a;             // ZORA: alpha^2 / 2 (0 without valence relativity)
};

__device__ __forceinline__ const double* apw(const MtArgs& m, int ias, int d, int io, int l) {
  return m.apwfr + (size_t)m.nrmtmax * (d + 2 * (io + (size_t)m.apwordmax * (l + (size_t)(m.lmaxapw + 1) * ias)));
}
__device__ __forceinline__ const double* lof(const MtArgs& m, int ias, int d, int ilo) {
  return m.lofr + (size_t)m.nrmtmax * (d + 2 * (ilo + (size_t)m.nlomax * ias));
}

// potential integrals sum_r w_r r^2 p1(r) p2(r) V_lm2(r)
//   kind 0: (l1, io1, l3, io2, lm2) of two APWs
//   kind 1: (ilo, l3, io, lm2) of an LO and an APW
//   kind 2: (ilo1, ilo2, lm2) of two LOs
__global__ void k_mt_potint(MtArgs m, int kind, int per_atom, double* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)per_atom * m.natmtot) return;
  const int ias = (int)(t / per_atom);
  int q = (int)(t % per_atom);
  const int is = m.idxis[ias];
  const int lm2 = q % m.lmvr;
  q /= m.lmvr;
  const double *p1 = nullptr, *p2 = nullptr;
  const int L1 = m.lmaxmat + 1;
  if (kind == 0) {
    const int io2 = q % m.apwordmax; q /= m.apwordmax;
    const int l3 = q % L1; q /= L1;
    const int io1 = q % m.apwordmax; q /= m.apwordmax;
    const int l1 = q;
    if (io1 >= m.apword[l1 + (m.lmaxapw + 1) * is] || io2 >= m.apword[l3 + (m.lmaxapw + 1) * is]) {
      out[t] = 0.0;
      return;
    }
    p1 = apw(m, ias, 0, io1, l1);
    p2 = apw(m, ias, 0, io2, l3);
  } else if (kind == 1) {
    const int io = q % m.apwordmax; q /= m.apwordmax;
    const int l3 = q % L1; q /= L1;
    const int ilo = q;
    if (ilo >= m.nlorb[is] || io >= m.apword[l3 + (m.lmaxapw + 1) * is]) {
      out[t] = 0.0;
      return;
    }
    p1 = lof(m, ias, 0, ilo);
    p2 = apw(m, ias, 0, io, l3);
  } else {
    const int ilo2 = q % m.nlomax;
    const int ilo1 = q / m.nlomax;
    if (ilo1 >= m.nlorb[is] || ilo2 >= m.nlorb[is]) {
      out[t] = 0.0;
      return;
    }
    p1 = lof(m, ias, 0, ilo1);
    p2 = lof(m, ias, 0, ilo2);
  }
  const int nr = m.nrmt[is];
  const double* w = m.wts + (size_t)m.nrmtmax * is;
  const double* v = m.veff + (size_t)m.lmvr * m.nrmtmax * ias + lm2;
  double s = 0.0;
  for (int r = 0; r < nr; ++r) s += w[r] * p1[r] * p2[r] * v[(size_t)m.lmvr * r];
  out[t] = s;
}

// kinetic-type integrals sum_r w_r r^2 (1/2 p1' p2' f + 1/2 l(l+1) p1 p2 f / r^2),
// f = rm (kinetic, mode 0) or a rm^2 (IORA* h1, mode 1), rm = 1/(1 - a V_00 y00)
//   kind 0: (l, io1, io2); kind 1: (ilo, io) with l = lorbl(ilo); kind 2: (ilo1, ilo2), equal l
// and the plain overlaps sum_r w_r r^2 p1 p2 (mode 2; kinds 1 and 2)
__global__ void k_mt_radint(MtArgs m, int kind, int mode, int per_atom, double* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)per_atom * m.natmtot) return;
  const int ias = (int)(t / per_atom);
  int q = (int)(t % per_atom);
  const int is = m.idxis[ias];
  const int L1 = m.lmaxmat + 1;
  const double *p1 = nullptr, *d1 = nullptr, *p2 = nullptr, *d2 = nullptr;
  int l = 0;
  if (kind == 0) {
    const int io2 = q % m.apwordmax; q /= m.apwordmax;
    const int io1 = q % m.apwordmax;
    l = q / m.apwordmax;
    if (l >= L1 || io1 >= m.apword[l + (m.lmaxapw + 1) * is] || io2 >= m.apword[l + (m.lmaxapw + 1) * is]) {
      out[t] = 0.0;
      return;
    }
    p1 = apw(m, ias, 0, io1, l); d1 = apw(m, ias, 1, io1, l);
    p2 = apw(m, ias, 0, io2, l); d2 = apw(m, ias, 1, io2, l);
  } else if (kind == 1) {
    const int io = q % m.apwordmax;
    const int ilo = q / m.apwordmax;
    if (ilo >= m.nlorb[is]) { out[t] = 0.0; return; }
    l = m.lorbl[ilo + m.nlomax * is];
    if (l > m.lmaxapw || io >= m.apword[l + (m.lmaxapw + 1) * is]) { out[t] = 0.0; return; }
    p1 = apw(m, ias, 0, io, l); d1 = apw(m, ias, 1, io, l);
    p2 = lof(m, ias, 0, ilo); d2 = lof(m, ias, 1, ilo);
  } else {
    const int ilo2 = q % m.nlomax;
    const int ilo1 = q / m.nlomax;
    if (ilo1 >= m.nlorb[is] || ilo2 >= m.nlorb[is]) { out[t] = 0.0; return; }
    l = m.lorbl[ilo1 + m.nlomax * is];
    if (m.lorbl[ilo2 + m.nlomax * is] != l) { out[t] = 0.0; return; }
    p1 = lof(m, ias, 0, ilo1); d1 = lof(m, ias, 1, ilo1);
    p2 = lof(m, ias, 0, ilo2); d2 = lof(m, ias, 1, ilo2);
  }
  const int nr = m.nrmt[is];
  const double* w = m.wts + (size_t)m.nrmtmax * is;
  const double* r_ = m.spr + (size_t)m.nrmtmax * is;
  const double* v00 = m.veff + (size_t)m.lmvr * m.nrmtmax * ias;
  const double ll = (double)l * (l + 1);
  double s = 0.0;
  for (int r = 0; r < nr; ++r) {
    if (mode == 2) {
      s += w[r] * p1[r] * p2[r];
      continue;
    }
    const double rm = 1.0 / (1.0 - m.a * v00[(size_t)m.lmvr * r] * Y00C);
    const double f = (mode == 0) ? rm : m.a * rm * rm;
    const double rr = r_[r];
    s += w[r] * (0.5 * d1[r] * d2[r] * f + 0.5 * ll * p1[r] * p2[r] * f / (rr * rr));
  }
  out[t] = s;
}

// aa(f1, f3, ias) = kinetic (same lm) + sum_lm2 gnt(lm1, lm2, lm3) haa(l1, io1, l3, io2, lm2)
__global__ void k_mt_aa(MtArgs m, const int* flist, const cplx* gnt, const double* haa, const double* kaa,
                        cplx* aa) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)m.maxaa * m.maxaa * m.natmtot) return;
  const int f1 = (int)(t % m.maxaa);
  const int f3 = (int)((t / m.maxaa) % m.maxaa);
  const int ias = (int)(t / ((long long)m.maxaa * m.maxaa));
  const int is = m.idxis[ias];
  const int c1 = flist[f1 + m.maxaa * is], c3 = flist[f3 + m.maxaa * is];
  if (c1 < 0 || c3 < 0) { aa[t] = cmk(0.0, 0.0); return; }
  const int lm1 = c1 / m.apwordmax, io1 = c1 % m.apwordmax;
  const int lm3 = c3 / m.apwordmax, io2 = c3 % m.apwordmax;
  int l1 = 0; while ((l1 + 1) * (l1 + 1) <= lm1) ++l1;
  int l3 = 0; while ((l3 + 1) * (l3 + 1) <= lm3) ++l3;
  const int L1 = m.lmaxmat + 1, lmmat = L1 * L1;
  cplx s = cmk(0.0, 0.0);
  if (lm1 == lm3 && kaa) s.x = kaa[((size_t)ias * L1 + l1) * m.apwordmax * m.apwordmax + io1 * m.apwordmax + io2];
  const double* h = haa + ((((size_t)ias * L1 + l1) * m.apwordmax + io1) * L1 + l3) * m.apwordmax * m.lmvr +
                    (size_t)io2 * m.lmvr;
  const cplx* g = gnt + ((size_t)lm1 * lmmat + lm3) * m.lmvr;
  for (int lm2 = 0; lm2 < m.lmvr; ++lm2) s = cadd(s, cscale(g[lm2], h[lm2]));
  aa[t] = s;
}

// loa(j, f, ias): LO function j = (ilo, lm1) of the atom against APW f
__global__ void k_mt_loa(MtArgs m, const int* flist, const int* lo_lm, const int* lo_ilo, const cplx* gnt,
                         const double* halo, const double* kalo, cplx* loa) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)m.maxnlo * m.maxaa * m.natmtot) return;
  const int j = (int)(t % m.maxnlo);
  const int f = (int)((t / m.maxnlo) % m.maxaa);
  const int ias = (int)(t / ((long long)m.maxnlo * m.maxaa));
  const int is = m.idxis[ias];
  const int lm1 = lo_lm[j + m.maxnlo * ias], ilo = lo_ilo[j + m.maxnlo * ias];
  const int c3 = flist[f + m.maxaa * is];
  if (lm1 < 0 || ilo < 0 || c3 < 0) { loa[t] = cmk(0.0, 0.0); return; }
  const int lm3 = c3 / m.apwordmax, io = c3 % m.apwordmax;
  int l3 = 0; while ((l3 + 1) * (l3 + 1) <= lm3) ++l3;
  const int L1 = m.lmaxmat + 1, lmmat = L1 * L1;
  cplx s = cmk(0.0, 0.0);
  if (lm1 == lm3 && kalo) s.x = kalo[((size_t)ias * m.nlomax + ilo) * m.apwordmax + io];
  const double* h = halo + ((((size_t)ias * m.nlomax + ilo) * L1 + l3) * m.apwordmax + io) * m.lmvr;
  const cplx* g = gnt + ((size_t)lm1 * lmmat + lm3) * m.lmvr;
  for (int lm2 = 0; lm2 < m.lmvr; ++lm2) s = cadd(s, cscale(g[lm2], h[lm2]));
  loa[t] = s;
}

// lolo(j1, j3, ias)
__global__ void k_mt_lolo(MtArgs m, const int* lo_lm, const int* lo_ilo, const cplx* gnt, const double* hlolo,
                          const double* klolo, cplx* lolo) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)m.maxnlo * m.maxnlo * m.natmtot) return;
  const int j1 = (int)(t % m.maxnlo);
  const int j3 = (int)((t / m.maxnlo) % m.maxnlo);
  const int ias = (int)(t / ((long long)m.maxnlo * m.maxnlo));
  const int lm1 = lo_lm[j1 + m.maxnlo * ias], ilo1 = lo_ilo[j1 + m.maxnlo * ias];
  const int lm3 = lo_lm[j3 + m.maxnlo * ias], ilo2 = lo_ilo[j3 + m.maxnlo * ias];
  if (lm1 < 0 || ilo1 < 0 || lm3 < 0 || ilo2 < 0) { lolo[t] = cmk(0.0, 0.0); return; }
  const int lmmat = (m.lmaxmat + 1) * (m.lmaxmat + 1);
  cplx s = cmk(0.0, 0.0);
  if (lm1 == lm3 && klolo) s.x = klolo[((size_t)ias * m.nlomax + ilo1) * m.nlomax + ilo2];
  const double* h = hlolo + (((size_t)ias * m.nlomax + ilo1) * m.nlomax + ilo2) * m.lmvr;
  const cplx* g = gnt + ((size_t)lm1 * lmmat + lm3) * m.lmvr;
  for (int lm2 = 0; lm2 < m.lmvr; ++lm2) s = cadd(s, cscale(g[lm2], h[lm2]));
  lolo[t] = s;
}

// oalo(io, ilo, ias) = olap + h1 and ololo(ilo1, ilo2, ias) likewise (IORA* folded in),
// h1aa(io1, io2, l, ias) from the per-(l, io1, io2) integrals
__global__ void k_mt_olp(MtArgs m, const double* oalo_r, const double* h1loa_r, const double* ololo_r,
                         const double* h1lolo_r, const double* h1aa_r, double* oalo, double* ololo, double* h1aa,
                         int h1on) {
  const int ias = blockIdx.x;
  const int L1 = m.lmaxmat + 1;
  for (int e = threadIdx.x; e < m.apwordmax * m.nlomax; e += blockDim.x) {
    const int io = e % m.apwordmax, ilo = e / m.apwordmax;
    const size_t src = ((size_t)ias * m.nlomax + ilo) * m.apwordmax + io;
    oalo[io + (size_t)m.apwordmax * (ilo + (size_t)m.nlomax * ias)] = oalo_r[src] + (h1on ? h1loa_r[src] : 0.0);
  }
  for (int e = threadIdx.x; e < m.nlomax * m.nlomax; e += blockDim.x) {
    const int i1 = e % m.nlomax, i2 = e / m.nlomax;
    const size_t src = ((size_t)ias * m.nlomax + i1) * m.nlomax + i2;
    ololo[i1 + (size_t)m.nlomax * (i2 + (size_t)m.nlomax * ias)] = ololo_r[src] + (h1on ? h1lolo_r[src] : 0.0);
  }
  if (h1on && h1aa)
    for (int e = threadIdx.x; e < m.apwordmax * m.apwordmax * (m.lmaxapw + 1); e += blockDim.x) {
      const int io1 = e % m.apwordmax, io2 = (e / m.apwordmax) % m.apwordmax, l = e / (m.apwordmax * m.apwordmax);
      h1aa[io1 + (size_t)m.apwordmax * (io2 + (size_t)m.apwordmax * (l + (size_t)(m.lmaxapw + 1) * ias))] =
          (l < L1) ? h1aa_r[(((size_t)ias * L1 + l) * m.apwordmax + io1) * m.apwordmax + io2] : 0.0;
    }
}

template <typename T>
int upload(T** d, const void* h, size_t n) {
  if (n == 0) { *d = nullptr; return EXCFV_OK; }
  CUDA_TRY(cudaMalloc(d, sizeof(T) * n));
  if (h) CUDA_TRY(cudaMemcpy(*d, h, sizeof(T) * n, cudaMemcpyHostToDevice));
  return EXCFV_OK;
}

}  // namespace

// mt_kin (kinetic) + mt_pot of the field `pot` (host, veffmt's layout; NULL:
// veffmt) into dst_aa / dst_loa / dst_lolo (device, the handle's block
// layouts), and with `olp` olprad into the handle's oalo / ololo / h1 terms;
// the host copies (nullable) receive aa, loa, lolo (complex) and oalo, ololo
// (real, without the IORA* terms) in the reference layouts.
static int mt_build(excfv_handle* h, const excfv_mtrad* r, const double* pot, bool kinetic, bool olp,
                    cplx* dst_aa, cplx* dst_loa, cplx* dst_lolo, double* aa_out, double* loa_out,
                    double* lolo_out, double* oalo_out, double* ololo_out) {
  DevStatic& st = h->st;
  const int* nlorb_h = st.h_nlorb.data();
  const int* lorbl_h = st.h_lorbl.data();
  const int* apword_h = st.h_apword.data();
  if (r->lmaxvr < 0 || r->lmaxvr > SPECFUN_LMAX || r->nrmtmax < 3 || !r->nrmt || !r->spr || !r->apwfr ||
      (!pot && !r->veffmt) || (kinetic && !r->veffmt) || (st.nlotot > 0 && !r->lofr)) {
    excfv_set_error("muffin-tin build: missing or inconsistent radial data");
    return EXCFV_ERR_ARG;
  }
  if (!pot) pot = r->veffmt;
  if (olp && st.h1on && !st.h1aa) {
    CUDA_TRY(cudaMalloc(&st.h1aa, sizeof(double) * st.apwordmax * st.apwordmax * (st.lmaxapw + 1) * st.natmtot));
    CUDA_TRY(cudaMemset(st.h1aa, 0, sizeof(double) * st.apwordmax * st.apwordmax * (st.lmaxapw + 1) * st.natmtot));
  }
  cudaStream_t s = h->stream;
  const int lmvr = (r->lmaxvr + 1) * (r->lmaxvr + 1);
  const int nlomax = std::max(st.nlomax, 1);
  const int L1 = st.lmaxmat + 1;
  // host: spline weights (times r^2) per species and the Gaunt table
  std::vector<double> wts((size_t)r->nrmtmax * st.nspecies, 0.0);
  for (int is = 0; is < st.nspecies; ++is) {
    const int nr = r->nrmt[is];
    if (nr < 3 || nr > r->nrmtmax) {
      excfv_set_error("excfv_hmlint: species %d has %d mesh points (need 3..nrmtmax)", is + 1, nr);
      return EXCFV_ERR_ARG;
    }
    const double* x = r->spr + (size_t)r->nrmtmax * is;
    spline_weights(nr, x, wts.data() + (size_t)r->nrmtmax * is);
    for (int i = 0; i < nr; ++i) wts[(size_t)r->nrmtmax * is + i] *= x[i] * x[i];
  }
  std::vector<cplx> gnt;
  gaunt_yry_table(st.lmaxmat, r->lmaxvr, gnt);
  MtArgs m;
  m.natmtot = st.natmtot; m.lmaxmat = st.lmaxmat; m.lmaxapw = st.lmaxapw; m.apwordmax = st.apwordmax;
  m.nlomax = nlomax; m.lmvr = lmvr; m.nrmtmax = r->nrmtmax; m.maxaa = st.maxaa; m.maxnlo = std::max(st.maxnlo, 1);
  m.a = (st.vrel != 0) ? 0.5 * ALPHA_FS * ALPHA_FS : 0.0;
  int rc = EXCFV_OK;
  int *d_idxis = nullptr, *d_nrmt = nullptr, *d_apword = nullptr, *d_nlorb = nullptr, *d_lorbl = nullptr;
  double *d_wts = nullptr, *d_spr = nullptr, *d_apwfr = nullptr, *d_lofr = nullptr, *d_veff = nullptr;
  cplx* d_gnt = nullptr;
  const size_t nr2 = (size_t)r->nrmtmax;
  std::vector<int> lorbl_pad((size_t)nlomax * st.nspecies, 0);
  for (int is = 0; is < st.nspecies; ++is)
    for (int ilo = 0; ilo < nlorb_h[is]; ++ilo) lorbl_pad[ilo + (size_t)nlomax * is] = lorbl_h[ilo + (size_t)nlomax * is];
  if ((rc = upload(&d_idxis, st.h_idxis.data(), st.natmtot)) || (rc = upload(&d_nrmt, r->nrmt, st.nspecies)) ||
      (rc = upload(&d_apword, apword_h, (size_t)(st.lmaxapw + 1) * st.nspecies)) ||
      (rc = upload(&d_nlorb, nlorb_h, st.nspecies)) ||
      (rc = upload(&d_lorbl, lorbl_pad.data(), lorbl_pad.size())) ||
      (rc = upload(&d_wts, wts.data(), wts.size())) ||
      (rc = upload(&d_spr, r->spr, nr2 * st.nspecies)) ||
      (rc = upload(&d_apwfr, r->apwfr, nr2 * 2 * st.apwordmax * (st.lmaxapw + 1) * st.natmtot)) ||
      (rc = upload(&d_lofr, r->lofr, nr2 * 2 * nlomax * st.natmtot)) ||
      (rc = upload(&d_veff, pot, (size_t)lmvr * nr2 * st.natmtot)) ||
      (rc = upload(&d_gnt, gnt.data(), gnt.size()))) {
    cudaFree(d_idxis); cudaFree(d_nrmt); cudaFree(d_apword); cudaFree(d_nlorb); cudaFree(d_lorbl);
    cudaFree(d_wts); cudaFree(d_spr); cudaFree(d_apwfr); cudaFree(d_lofr); cudaFree(d_veff); cudaFree(d_gnt);
    return rc;
  }
  if (!r->lofr) CUDA_TRY(cudaMemset(d_lofr, 0, sizeof(double) * nr2 * 2 * nlomax * st.natmtot));
  m.idxis = d_idxis; m.nrmt = d_nrmt; m.apword = d_apword; m.nlorb = d_nlorb; m.lorbl = d_lorbl;
  m.wts = d_wts; m.spr = d_spr; m.apwfr = d_apwfr; m.lofr = d_lofr; m.veff = d_veff;
  // radial integrals
  const int A = st.apwordmax;
  const int per_aa = L1 * A * L1 * A * lmvr, per_loa = nlomax * L1 * A * lmvr, per_lolo = nlomax * nlomax * lmvr;
  const int per_kaa = L1 * A * A, per_kalo = nlomax * A, per_klolo = nlomax * nlomax;
  double *haa = nullptr, *halo = nullptr, *hlolo = nullptr, *kaa = nullptr, *kalo = nullptr, *klolo = nullptr;
  double *oalo_r = nullptr, *ololo_r = nullptr, *h1aa_r = nullptr, *h1loa_r = nullptr, *h1lolo_r = nullptr;
  const size_t N = st.natmtot;
  if ((rc = upload(&haa, nullptr, per_aa * N)) || (rc = upload(&halo, nullptr, per_loa * N)) ||
      (rc = upload(&hlolo, nullptr, per_lolo * N)) || (rc = upload(&kaa, nullptr, per_kaa * N)) ||
      (rc = upload(&kalo, nullptr, per_kalo * N)) || (rc = upload(&klolo, nullptr, per_klolo * N)) ||
      (rc = upload(&oalo_r, nullptr, per_kalo * N)) || (rc = upload(&ololo_r, nullptr, per_klolo * N)) ||
      (rc = upload(&h1aa_r, nullptr, per_kaa * N)) || (rc = upload(&h1loa_r, nullptr, per_kalo * N)) ||
      (rc = upload(&h1lolo_r, nullptr, per_klolo * N)))
    goto done;
  {
    auto grid = [](long long n) { return (unsigned)((n + 127) / 128); };
    k_mt_potint<<<grid(per_aa * N), 128, 0, s>>>(m, 0, per_aa, haa); count_launch();
    k_mt_potint<<<grid(per_loa * N), 128, 0, s>>>(m, 1, per_loa, halo); count_launch();
    k_mt_potint<<<grid(per_lolo * N), 128, 0, s>>>(m, 2, per_lolo, hlolo); count_launch();
    if (kinetic) {
      k_mt_radint<<<grid(per_kaa * N), 128, 0, s>>>(m, 0, 0, per_kaa, kaa); count_launch();
      k_mt_radint<<<grid(per_kalo * N), 128, 0, s>>>(m, 1, 0, per_kalo, kalo); count_launch();
      k_mt_radint<<<grid(per_klolo * N), 128, 0, s>>>(m, 2, 0, per_klolo, klolo); count_launch();
    }
    if (olp) {
      k_mt_radint<<<grid(per_kalo * N), 128, 0, s>>>(m, 1, 2, per_kalo, oalo_r); count_launch();
      k_mt_radint<<<grid(per_klolo * N), 128, 0, s>>>(m, 2, 2, per_klolo, ololo_r); count_launch();
    }
    if (olp && st.h1on) {
      k_mt_radint<<<grid(per_kaa * N), 128, 0, s>>>(m, 0, 1, per_kaa, h1aa_r); count_launch();
      k_mt_radint<<<grid(per_kalo * N), 128, 0, s>>>(m, 1, 1, per_kalo, h1loa_r); count_launch();
      k_mt_radint<<<grid(per_klolo * N), 128, 0, s>>>(m, 2, 1, per_klolo, h1lolo_r); count_launch();
    }
    // assembly into the static blocks
    const double* ka = kinetic ? kaa : nullptr;
    const double* kl = kinetic ? kalo : nullptr;
    const double* kll = kinetic ? klolo : nullptr;
    k_mt_aa<<<grid((long long)st.maxaa * st.maxaa * N), 128, 0, s>>>(m, st.flist, d_gnt, haa, ka, dst_aa);
    count_launch();
    if (st.maxnlo > 0) {
      k_mt_loa<<<grid((long long)st.maxnlo * st.maxaa * N), 128, 0, s>>>(m, st.flist, st.lo_lm, st.lo_ilo, d_gnt,
                                                                          halo, kl, dst_loa);
      count_launch();
      k_mt_lolo<<<grid((long long)st.maxnlo * st.maxnlo * N), 128, 0, s>>>(m, st.lo_lm, st.lo_ilo, d_gnt, hlolo,
                                                                            kll, dst_lolo);
      count_launch();
    }
    if (olp && (st.nlomax > 0 || st.h1on)) {
      k_mt_olp<<<st.natmtot, 128, 0, s>>>(m, oalo_r, h1loa_r, ololo_r, h1lolo_r, h1aa_r, st.oalo, st.ololo,
                                          st.h1aa, st.h1on);
      count_launch();
    }
    if (cudaGetLastError() != cudaSuccess) { rc = EXCFV_ERR_CUDA; goto done; }
    // optional host copies (reference layouts)
    if (aa_out) cudaMemcpyAsync(aa_out, dst_aa, sizeof(cplx) * st.maxaa * st.maxaa * N, cudaMemcpyDeviceToHost, s);
    if (loa_out && st.maxnlo > 0)
      cudaMemcpyAsync(loa_out, dst_loa, sizeof(cplx) * st.maxnlo * st.maxaa * N, cudaMemcpyDeviceToHost, s);
    if (lolo_out && st.maxnlo > 0)
      cudaMemcpyAsync(lolo_out, dst_lolo, sizeof(cplx) * st.maxnlo * st.maxnlo * N, cudaMemcpyDeviceToHost, s);
    std::vector<double> tmp;
    if (olp && (oalo_out || ololo_out) && st.nlomax > 0) {
      tmp.resize((size_t)(per_kalo + per_klolo) * N);
      cudaMemcpyAsync(tmp.data(), oalo_r, sizeof(double) * per_kalo * N, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(tmp.data() + per_kalo * N, ololo_r, sizeof(double) * per_klolo * N, cudaMemcpyDeviceToHost, s);
    }
    if (cudaStreamSynchronize(s) != cudaSuccess) { rc = EXCFV_ERR_CUDA; goto done; }
    if (!tmp.empty()) {
      for (size_t ias = 0; ias < N; ++ias) {
        for (int ilo = 0; ilo < st.nlomax; ++ilo)
          for (int io = 0; io < A; ++io)
            if (oalo_out)
              oalo_out[io + (size_t)A * (ilo + (size_t)st.nlomax * ias)] = tmp[(ias * nlomax + ilo) * A + io];
        for (int i1 = 0; i1 < st.nlomax; ++i1)
          for (int i2 = 0; i2 < st.nlomax; ++i2)
            if (ololo_out)
              ololo_out[i1 + (size_t)st.nlomax * (i2 + (size_t)st.nlomax * ias)] =
                  tmp[per_kalo * N + (ias * nlomax + i1) * nlomax + i2];
      }
    }
  }
done:
  cudaStreamSynchronize(s);
  for (void* p : {(void*)d_idxis, (void*)d_nrmt, (void*)d_apword, (void*)d_nlorb, (void*)d_lorbl, (void*)d_wts,
                  (void*)d_spr, (void*)d_apwfr, (void*)d_lofr, (void*)d_veff, (void*)d_gnt, (void*)haa, (void*)halo,
                  (void*)hlolo, (void*)kaa, (void*)kalo, (void*)klolo, (void*)oalo_r, (void*)ololo_r, (void*)h1aa_r,
                  (void*)h1loa_r, (void*)h1lolo_r})
    cudaFree(p);
  if (rc == EXCFV_OK && olp && st.h1on) st.have_h1aa = true;
  return rc;
}

int stage_hmlint(excfv_handle* h, const excfv_mtrad* r, double* aa_out, double* loa_out, double* lolo_out,
                 double* oalo_out, double* ololo_out) {
  DevStatic& st = h->st;
  return mt_build(h, r, nullptr, true, true, st.aa, st.loa, st.lolo, aa_out, loa_out, lolo_out, oalo_out,
                  ololo_out);
}

// mt_pot of a field without the kinetic term and without olprad (the spin
// blocks of hmlint.f90:88-108) into the given device blocks
int stage_mt_field(excfv_handle* h, const excfv_mtrad* r, const double* field, cplx* aa, cplx* loa, cplx* lolo,
                   double* aa_out, double* loa_out, double* lolo_out) {
  return mt_build(h, r, field, false, false, aa, loa, lolo, aa_out, loa_out, lolo_out, nullptr, nullptr);
}

// The cubic spline of spline.f90 on the host: d1 = cf(1, :), the first
// derivative at each mesh point (fderiv(1)); returns the integral over the
// whole mesh (fderiv(-1) at the last point) of f.
double host_spline(int n, const double* x, const double* f, double* d1) {
  std::vector<double> c1(n), c2(n), c3(n), w(n);
  const double g = spline_integral(n, x, f, c1, c2, c3, w);
  if (d1) {
    // spline_integral leaves c1 = the divided differences and c2 = the second
    // coefficients; the first coefficients follow as in spline.f90
    for (int i = 0; i < n - 1; ++i) {
      const double d3 = (1.0 / 3.0) * (c2[i + 1] - c2[i]) * w[i];
      const double dx = x[i + 1] - x[i];
      d1[i] = c1[i] - (c2[i] + d3 * dx) * dx;
    }
    const double dxl = x[n - 1] - x[n - 2];
    const double d3l = (1.0 / 3.0) * (c2[n - 1] - c2[n - 2]) * w[n - 2];
    d1[n - 1] = d1[n - 2] + (2.0 * c2[n - 2] + 3.0 * d3l * dxl) * dxl;
  }
  return g;
}
