// One task of the band -> tridiagonal bulge chase (the second stage of a
// two-stage Householder tridiagonal reduction), on compact lower band storage.
//
// Storage: a Hermitian matrix of lower bandwidth b plus room for the bulge,
// element (r, c) for c <= r <= c + 2b at AB[(r - c) + (2b + 1) c]; the upper
// triangle is the conjugate.
//
// A task (col, lo, hi), hi - lo <= b, builds the ZLARFG reflector
// H = I - tau v v^H (v[0] = 1) that maps rows [lo, hi) of column col to
// beta e_1 and applies H^H . H on rows and columns [lo, hi).  In lower
// storage that touches
//   column col                rows [lo, hi): beta, 0, ..., 0
//   columns (col, lo)         rows [lo, hi): y <- H^H y         (left)
//   the diagonal block        [lo, hi)^2:    A <- A - v q^H - q v^H,
//                             q = tau A v - 1/2 |tau|^2 (v^H A v) v
//   rows [hi, min(n, lo+2b))  columns [lo, hi): y^T <- y^T H    (right)
// Sweep i of the chase runs its tasks (col, lo) = (i, i+1), (i+1, i+1+b),
// (i+1+b, i+1+2b), ... until lo reaches n-1; with task (i, k) in time slot
// 3i + k the tasks of one slot touch disjoint entries.
//
// The routines are __host__ __device__: the same code runs in a host test
// against the dense restatement and inside a device kernel.
#pragma once

#include "common.cuh"

struct BandView {
  cplx* AB;
  int n, b;
  EXCFV_HD cplx& at(int r, int c) const { return AB[(r - c) + (size_t)(2 * b + 1) * c]; }
};

// ZLARFG on x[0..len): x becomes v (v[0] = 1); returns tau, beta.
EXCFV_HD void chase_larfg(int len, cplx* x, cplx* tau, double* beta) {
  const cplx alpha = x[0];
  double xn2 = 0.0;
  for (int t = 1; t < len; ++t) xn2 += cabs2(x[t]);
  x[0] = cmk(1.0, 0.0);
  if (xn2 == 0.0 && alpha.y == 0.0) {
    *tau = cmk(0.0, 0.0);
    *beta = alpha.x;
    return;
  }
  const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
  const double bt = (alpha.x >= 0.0) ? -nrm : nrm;
  *tau = cmk((bt - alpha.x) / bt, -alpha.y / bt);
  // 1 / (alpha - beta)
  const double dr = alpha.x - bt, di = alpha.y, den = dr * dr + di * di;
  const cplx sc = cmk(dr / den, -di / den);
  for (int t = 1; t < len; ++t) x[t] = cmul(x[t], sc);
  *beta = bt;
}

// One chase task; v (length hi - lo) and tau receive the reflector, work
// holds 2 (hi - lo) complex scratch values.
EXCFV_HD void chase_task(const BandView& B, int col, int lo, int hi, cplx* v, cplx* tau, cplx* work) {
  const int len = hi - lo;
  for (int t = 0; t < len; ++t) v[t] = B.at(lo + t, col);
  double beta;
  chase_larfg(len, v, tau, &beta);
  B.at(lo, col) = cmk(beta, 0.0);
  for (int t = 1; t < len; ++t) B.at(lo + t, col) = cmk(0.0, 0.0);
  const cplx tu = *tau;
  if (tu.x == 0.0 && tu.y == 0.0) return;
  // left: columns strictly between col and lo, rows [lo, hi)
  for (int c = col + 1; c < lo; ++c) {
    cplx s = cmk(0.0, 0.0);
    for (int t = 0; t < len; ++t) s = cadd(s, cmulc(v[t], B.at(lo + t, c)));
    const cplx f = cmulc(tu, s);  // conj(tau) s
    for (int t = 0; t < len; ++t) B.at(lo + t, c) = csub(B.at(lo + t, c), cmul(v[t], f));
  }
  // diagonal block: p = A v (Hermitian from the lower triangle), gamma = v^H p
  cplx* p = work;
  cplx* q = work + len;
  double gamma = 0.0;
  for (int r = 0; r < len; ++r) {
    cplx s = cmk(0.0, 0.0);
    for (int c = 0; c < len; ++c) {
      const cplx a = (r >= c) ? B.at(lo + r, lo + c) : cconj(B.at(lo + c, lo + r));
      s = cadd(s, cmul(a, v[c]));
    }
    p[r] = s;
  }
  for (int r = 0; r < len; ++r) gamma += cmulc(v[r], p[r]).x;
  const double h = 0.5 * cabs2(tu) * gamma;
  for (int r = 0; r < len; ++r) q[r] = csub(cmul(tu, p[r]), cscale(v[r], h));
  for (int c = 0; c < len; ++c)
    for (int r = c; r < len; ++r) {
      // A(r, c) -= v_r conj(q_c) + q_r conj(v_c)
      const cplx d = cadd(cmul(v[r], cconj(q[c])), cmul(q[r], cconj(v[c])));
      B.at(lo + r, lo + c) = csub(B.at(lo + r, lo + c), d);
    }
  // right: rows [hi, min(n, lo + 2b)), columns [lo, hi)
  const int rend = (lo + 2 * B.b < B.n) ? lo + 2 * B.b : B.n;
  for (int r = hi; r < rend; ++r) {
    cplx s = cmk(0.0, 0.0);
    for (int t = 0; t < len; ++t) s = cadd(s, cmul(B.at(r, lo + t), v[t]));
    const cplx f = cmul(tu, s);
    for (int t = 0; t < len; ++t) B.at(r, lo + t) = csub(B.at(r, lo + t), cmul(f, cconj(v[t])));
  }
}
