// Two-stage Householder reduction of a Hermitian matrix to real tridiagonal
// form, C = Q T Q^H (the ZHETRD step of ZHEEVX, external/LAPACK/zheevx.f:441,
// replaced by the two-stage scheme of LAPACK's ZHETRD_2STAGE: he2hb + hb2st).
//
// Stage 1, dense -> band of lower bandwidth BW.  Per block column j:
//   k_panel_qr   the QR of the panel C[j+BW:n, j:j+BW] by one thread-block
//                cluster: the panel's rows are split over the cluster's CTAs
//                and held in shared memory; every column takes one cluster
//                barrier, because the column's norm, its products with the
//                later panel columns and with the earlier reflectors come out
//                of one reduction through distributed shared memory (the
//                reflector's scale is applied after the reduction).  The
//                cluster also builds T of the compact-WY form I - V T V^H.
//   GEMMs        X = C22 V T, W = X - 1/2 V (T^H V^H X),
//                C22 -= [V W] [W V]^H (DMMA, the trailing block kept full).
// Stage 2, band -> tridiagonal by bulge chasing (k_chase) on compact band
//   storage: groups of two consecutive sweeps per CTA, round-robin over a
//   cooperative grid.  Within a group, step k of the second sweep runs three
//   slots after step k of the first, in the same CTA, on a ring of band
//   columns in shared memory; between groups, a group's first sweep waits
//   (bounded) until the previous group has written back the columns its last
//   sweep finished.  Every step's reflector is kept for the back-transform.
// A diagonal phase (a prefix product of unit complex numbers) makes the
// subdiagonal real and non-negative.
//
// Back-transform of the eigenvectors Z of T: Z <- diag(phase) Z, Z <- Q2 Z
// (k_apply_q2: groups of M2 consecutive sweeps at one step, applied in waves
// of groups whose rows are disjoint), Z <- Q1 Z (the blocked compact-WY
// back-transform of the one-stage path, with the reflectors starting BW rows
// below their column).
#include <cooperative_groups.h>

#include <algorithm>

#include "handle.cuh"

namespace cg = cooperative_groups;

int apply_q(excfv_handle* h, int n, int k, const cplx* C, long long ld, cplx* Z, long long ldz,
            int off);

namespace {

constexpr int BW = 32;           // bandwidth = panel width
constexpr int PT = 256;          // threads of the panel kernel: 8 warps x 32 columns
constexpr int LDP = BW + 1;      // shared-memory row stride of the panel (conflict-free)
constexpr int CLMAX = 16;        // largest cluster
constexpr int RSM = 352;         // panel rows per CTA held in shared memory
constexpr int LDB = 2 * BW + 1;  // diagonals of the compact band storage (band + bulge)
constexpr int M2 = 64;           // sweeps per group of the Q2 back-transform
constexpr int QT = 256;          // threads of the Q2 kernel: 32 columns x 8 row classes
constexpr int QCOL = 32;         // columns of Z per Q2 block
constexpr int PROG_DONE = 0x40000000;

__device__ __forceinline__ long long gtimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ int ld_acquire_s32(const int* p) {
  int v;
  asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_s32(int* p, int v) {
  asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// ---------------------------------------------------------------------------
// stage 1: panel QR in one cluster
// ---------------------------------------------------------------------------
struct PanelArgs {
  cplx* C;
  long long ld;
  int n, j;          // panel columns [j, j+BW), rows [j+BW, n)
  int rpc;           // panel rows per CTA
  cplx* tau;         // tau[j + t] (0 for t >= nb)
  cplx* V;           // explicit unit lower-trapezoidal reflectors, rows indexed as C's
  long long ldv;
  cplx* T;           // BW x BW upper triangular factor, column-major
};

size_t panel_smem_bytes(int rpc) {
  return sizeof(cplx) * ((size_t)rpc * LDP + 2 * CLMAX * BW + 2 * BW + 8 * BW + BW * BW);
}

// Householder QR of the panel: for column t, x = P[t:, t], alpha = x[0],
// beta = -sign(Re alpha) |x|, tau = (beta - alpha) / beta, v = x / (alpha -
// beta) with v[0] = 1 (ZLARFG), and P[t:, c] -= conj(tau) v (v^H P[t:, c])
// for c > t.  With S_c = sum over rows below t of conj(x_i) P_ic (one
// reduction, every column c at once) and row t's entries P_tc:
//   |x|^2 = |alpha|^2 + S_t,   v^H P_c = P_tc + conj(scale) S_c,
//   V_q^H v = conj(P_tq) + scale conj(S_q)  (q < t, for T's column t).
__global__ void __launch_bounds__(PT, 1) k_panel_qr(PanelArgs a) {
  cg::cluster_group cluster = cg::this_cluster();
  const int q = (int)cluster.block_rank();
  const int CL = (int)cluster.num_blocks();
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx* Ps = reinterpret_cast<cplx*>(dsm);          // [rpc][LDP]
  cplx* part = Ps + (size_t)a.rpc * LDP;            // [2][CLMAX][BW] pushed partial sums
  cplx* rowb = part + 2 * CLMAX * BW;               // [2][BW] pushed row t
  cplx* red = rowb + 2 * BW;                        // [8][BW]
  cplx* Tm = red + 8 * BW;                          // [BW][BW] column-major (CTA 0)
  __shared__ cplx s_w[BW], s_z[BW];
  __shared__ double s_sc[5];

  const int n = a.n, j = a.j, r0 = j + BW, m = n - r0;
  const int nb = min(BW, m - 1);
  const int lo = q * a.rpc;
  const int nr = max(0, min(m, lo + a.rpc) - lo);
  const int tid = threadIdx.x, lane = tid & 31, g = tid >> 5;
  const long long ld = a.ld;
  cplx* C = a.C;

  for (int e = tid; e < nr * BW; e += PT) {
    const int i = e % nr, c = e / nr;
    Ps[i * LDP + c] = C[(r0 + lo + i) + ld * (j + c)];
  }
  if (q == 0)
    for (int e = tid; e < BW * BW; e += PT) Tm[e] = cmk(0.0, 0.0);
  __syncthreads();

  for (int t = 0; t < nb; ++t) {
    const int buf = t & 1;
    // partial sums over this CTA's rows strictly below panel row t
    cplx acc = cmk(0.0, 0.0);
    for (int i = max(0, t + 1 - lo) + g; i < nr; i += 8)
      acc = cadd(acc, cmulc(Ps[i * LDP + t], Ps[i * LDP + lane]));
    red[g * BW + lane] = acc;
    __syncthreads();
    if (g == 0) {
      cplx s = cmk(0.0, 0.0);
      for (int gg = 0; gg < 8; ++gg) s = cadd(s, red[gg * BW + lane]);
      for (int d = 0; d < CL; ++d) cluster.map_shared_rank(part, d)[(buf * CLMAX + q) * BW + lane] = s;
    } else if (g == 1 && t >= lo && t < lo + nr) {
      const cplx rv = Ps[(t - lo) * LDP + lane];
      for (int d = 0; d < CL; ++d) cluster.map_shared_rank(rowb, d)[buf * BW + lane] = rv;
    }
    cluster.sync();
    if (g == 0) {
      cplx S = cmk(0.0, 0.0);
      for (int d = 0; d < CL; ++d) S = cadd(S, part[(buf * CLMAX + d) * BW + lane]);
      const cplx rv = rowb[buf * BW + lane];
      const double xn2 = __shfl_sync(0xffffffffu, S.x, t);
      const double ar = __shfl_sync(0xffffffffu, rv.x, t), ai = __shfl_sync(0xffffffffu, rv.y, t);
      double tr = 0.0, ti = 0.0, sr = 0.0, si = 0.0, beta;
      if (xn2 == 0.0 && ai == 0.0) {
        beta = ar;
      } else {
        const double nrm = sqrt(ar * ar + ai * ai + xn2);
        beta = (ar >= 0.0) ? -nrm : nrm;
        tr = (beta - ar) / beta;
        ti = -ai / beta;
        const double dr = ar - beta, di = ai, den = dr * dr + di * di;
        sr = dr / den;
        si = -di / den;
      }
      s_w[lane] = cadd(rv, cmul(cmk(sr, -si), S));
      s_z[lane] = cadd(cconj(rv), cmul(cmk(sr, si), cconj(S)));
      if (lane == 0) {
        s_sc[0] = tr; s_sc[1] = ti; s_sc[2] = sr; s_sc[3] = si; s_sc[4] = beta;
      }
    }
    __syncthreads();
    const cplx tau = cmk(s_sc[0], s_sc[1]);
    const cplx scale = cmk(s_sc[2], s_sc[3]);
    if (q == 0 && tid <= t) {
      // T(0:t, t) = -tau T(0:t, 0:t) (V(:, 0:t)^H v_t), T(t, t) = tau
      if (tid == t) {
        Tm[t * BW + t] = tau;
      } else {
        cplx z = cmk(0.0, 0.0);
        for (int p = tid; p < t; ++p) z = cadd(z, cmul(Tm[p * BW + tid], s_z[p]));
        Tm[t * BW + tid] = cmul(cmk(-tau.x, -tau.y), z);
      }
    }
    if (lane > t) {
      const cplx f = cmul(cconj(tau), s_w[lane]);
      for (int i = max(0, t - lo) + g; i < nr; i += 8) {
        const cplx vi = (lo + i == t) ? cmk(1.0, 0.0) : cmul(Ps[i * LDP + t], scale);
        Ps[i * LDP + lane] = csub(Ps[i * LDP + lane], cmul(vi, f));
      }
    }
    __syncthreads();
    for (int i = tid; i < nr; i += PT) {
      const int pr = lo + i;
      if (pr == t) Ps[i * LDP + t] = cmk(s_sc[4], 0.0);
      else if (pr > t) Ps[i * LDP + t] = cmul(Ps[i * LDP + t], scale);
    }
    __syncthreads();
  }

  for (int e = tid; e < nr * BW; e += PT) {
    const int i = e % nr, c = e / nr, pr = lo + i;
    const cplx p = Ps[i * LDP + c];
    C[(r0 + lo + i) + ld * (j + c)] = p;
    cplx v = cmk(0.0, 0.0);
    if (c < nb) v = (pr == c) ? cmk(1.0, 0.0) : (pr > c ? p : v);
    a.V[(r0 + lo + i) + a.ldv * c] = v;
  }
  if (q == 0) {
    for (int e = tid; e < BW * BW; e += PT) a.T[e] = Tm[e];
    if (tid < BW) a.tau[j + tid] = (tid < nb) ? Tm[tid * BW + tid] : cmk(0.0, 0.0);
  }
  cluster.sync();  // no CTA leaves while another may still address its shared memory
}

// [V | W] -> [W | V] (rows [r0, n)), W taken from the W slot of WV itself
// after the GEMMs left it there: VW(:, BW:2BW) = WV(:, 0:BW), WV(:, BW:2BW) = VW(:, 0:BW)
__global__ void k_swap_vw(int r0, int n, cplx* __restrict__ VW, cplx* __restrict__ WV, long long ld) {
  const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r >= n) return;
  VW[r + ld * (BW + c)] = WV[r + ld * c];
  WV[r + ld * (BW + c)] = VW[r + ld * c];
}

// compact band storage AB(o, c) = C(c + o, c), o <= BW; offsets BW+1..2BW
// (room for the bulge) zero
__global__ void k_band_extract(int n, const cplx* __restrict__ C, long long ld, cplx* __restrict__ AB) {
  const int c = blockIdx.x;
  for (int o = threadIdx.x; o < LDB; o += blockDim.x) {
    cplx v = cmk(0.0, 0.0);
    if (o <= BW && c + o < n) v = C[(c + o) + ld * c];
    AB[o + (size_t)LDB * c] = v;
  }
}

// The reflectors of stage 1 with their unit entries made explicit (the
// back-transform reads them in place); called after the band is extracted.
__global__ void k_unit_entries(int n, cplx* C, long long ld) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c < n - BW) C[(c + BW) + ld * c] = cmk(1.0, 0.0);
}

// ---------------------------------------------------------------------------
// stage 2: bulge chasing
// ---------------------------------------------------------------------------
constexpr int CS = 2;            // consecutive sweeps per CTA group
constexpr int TW = 8;            // warps per step
constexpr int CT = 32 * TW * CS; // threads of the chase kernel
constexpr int WIN = 192;         // band columns held in shared memory (a ring)

struct ChaseArgs {
  cplx* AB;          // (LDB, n) compact lower band with room for the bulge
  int n, ngrp;
  int* prog;         // per group: steps of its last sweep that are done and whose
                     // columns are back in AB (PROG_DONE at its end); zero at launch
  cplx* V2;          // reflector (i, k) at V2[BW * (toff(k) + i) + r]
  cplx* tau2;        // tau2[toff(k) + i]
  int* status;
  long long wait_ns;
  int planted;
};

// reflectors (sweeps) of the steps before step k: sum over k' < k of (n - 2 - k' BW)
__host__ __device__ __forceinline__ long long toff(int n, int k) {
  return (long long)k * (n - 2) - (long long)BW * k * (k - 1) / 2;
}
// steps of sweep i: k with i + 1 + k BW <= n - 2
__host__ __device__ __forceinline__ int chase_steps(int n, int i) {
  return (i <= n - 3) ? (n - 3 - i) / BW + 1 : 0;
}

// The window of a group at slot s (sweep i0 + a runs step s - 3a):
// need_hi(s) = end of the columns its running steps touch (the first sweep's
// step reaches furthest), need_lo(s) = first column a running or future
// step of the group touches.
__host__ __device__ __forceinline__ int win_need_hi(int n, int i0, const int* nt, int s) {
  int h = i0;
  for (int a = 0; a < CS; ++a) {
    const int k = s - 3 * a;
    if (k >= 0 && k < nt[a]) h = max(h, min(n, i0 + a + 1 + k * BW + BW));
  }
  return h;
}
__host__ __device__ __forceinline__ int win_need_lo(int n, int i0, const int* nt, int s) {
  int l = n;
  for (int a = 0; a < CS; ++a) {
    const int k = s - 3 * a;
    if (k >= nt[a]) continue;
    l = min(l, (k <= 0) ? i0 + a : i0 + a + 1 + k * BW - BW);
  }
  return l;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\ncp.async.wait_group 0;" ::: "memory");
}
// barrier of the threads of task group t (named barriers 1, 2)
__device__ __forceinline__ void tsync(int t) { asm volatile("bar.sync %0, %1;" ::"r"(t + 1), "n"(32 * TW) : "memory"); }

__device__ __forceinline__ cplx shfl_c(cplx v, int src) {
  return cmk(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}
__device__ __forceinline__ cplx wsum_c(cplx v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

size_t chase_smem_bytes() { return sizeof(cplx) * (size_t)WIN * LDB; }

// Step k of sweep i (lo = i + 1 + k BW, hi = min(lo + BW, n), len = hi - lo,
// column col = i for k = 0 and lo - BW after) on the shared-memory window:
// the reflector of rows [lo, hi) of column col; left update of the columns
// (col, lo) on those rows (block L); two-sided update of the diagonal block
// [lo, hi)^2 (lower storage, D); right update of the rows [hi, min(n, lo +
// 2 BW)) on the columns [lo, hi) (block R).  TW warps (task group t): every
// warp forms the reflector from the column itself (lane r holds v_r); warp w
// owns rows / columns 4w..4w+3 of p = D v, s = R v and w = v^H L, each a
// 32-lane shuffle reduction; after one barrier every thread has p, s, w and
// updates its four rows of D and R and four columns of L.  The reflector is
// kept in V2 / tau2.
__device__ void chase_step(const ChaseArgs& a, cplx* Wn, int t, int i, int k, cplx* s_p, cplx* s_s,
                           cplx* s_w) {
  const int n = a.n;
  const int tg = threadIdx.x % (32 * TW), w = tg >> 5, lane = tg & 31;
  const int lo = i + 1 + k * BW;
  const int hi = min(lo + BW, n), len = hi - lo;
  const int col = (k == 0) ? i : lo - BW;
  const int ncl = lo - col;
  const int nr = min(n, lo + 2 * BW) - hi;
  // ring slots: column col + j and lo + j of this lane (j = lane)
  const int sc0 = col % WIN, sd0 = lo % WIN;
  auto slot = [](int s0, int j) { const int q = s0 + j; return q >= WIN ? q - WIN : q; };
  cplx* Lcol = Wn + (size_t)slot(sc0, lane) * LDB;  // column col + lane
  cplx* Dcol = Wn + (size_t)slot(sd0, lane) * LDB;  // column lo + lane
  // reflector of column col, rows [lo, hi) (every warp)
  const cplx x = (lane < len) ? Wn[(size_t)sc0 * LDB + (lo + lane - col)] : cmk(0.0, 0.0);
  double xn2 = (lane >= 1) ? cabs2(x) : 0.0;
  for (int o = 16; o > 0; o >>= 1) xn2 += __shfl_xor_sync(0xffffffffu, xn2, o);
  const double ar = __shfl_sync(0xffffffffu, x.x, 0), ai = __shfl_sync(0xffffffffu, x.y, 0);
  double tr = 0.0, ti = 0.0, sr = 0.0, si = 0.0, beta;
  if (xn2 == 0.0 && ai == 0.0) {
    beta = ar;
  } else {
    const double nrm = sqrt(ar * ar + ai * ai + xn2);
    beta = (ar >= 0.0) ? -nrm : nrm;
    tr = (beta - ar) / beta;
    ti = -ai / beta;
    const double dr = ar - beta, di = ai, den = dr * dr + di * di;
    sr = dr / den;
    si = -di / den;
  }
  const cplx tau = cmk(tr, ti);
  const cplx v = (lane == 0) ? cmk(1.0, 0.0) : (lane < len ? cmul(x, cmk(sr, si)) : cmk(0.0, 0.0));
  if (w == 0) {
    const long long sl = toff(n, k) + i;
    a.V2[(size_t)BW * sl + lane] = v;
    if (lane == 0) a.tau2[sl] = tau;
  }
  const bool active = (tr != 0.0 || ti != 0.0);
  if (active) {
    // warp w: p_r = sum_c D(r, c) v_c and s_r = sum_c R(r, c) v_c for its rows
    // r = 4w + u (lane = c); w_j = sum_r conj(v_r) L(r, j) for its columns j = 4w + u (lane = r)
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int r = 4 * w + u;
      cplx dp = cmk(0.0, 0.0), rs = cmk(0.0, 0.0), lw = cmk(0.0, 0.0);
      if (r < len && lane < len) {
        // D(r, lane): lower storage, column min(r, lane)
        const cplx dv = (lane <= r) ? Dcol[r - lane] : cconj(Wn[(size_t)slot(sd0, r) * LDB + (lane - r)]);
        dp = cmul(dv, v);
      }
      if (r < nr && lane < len) rs = cmul(Dcol[hi + r - lo - lane], v);
      if (r >= 1 && r < ncl && lane < len) lw = cmulc(v, Wn[(size_t)slot(sc0, r) * LDB + (lo + lane - col - r)]);
      dp = wsum_c(dp);
      rs = wsum_c(rs);
      lw = wsum_c(lw);
      if (lane == 0) {
        s_p[r] = dp;
        s_s[r] = rs;
        s_w[r] = lw;
      }
    }
  }
  tsync(t);
  // column col: beta, then zeros (its readers are past the barrier)
  if (w == 0 && lane < len) Wn[(size_t)sc0 * LDB + (lo + lane - col)] = (lane == 0) ? cmk(beta, 0.0) : cmk(0.0, 0.0);
  if (active) {
    // q = tau p - 1/2 |tau|^2 (v^H p) v; lane r holds p_r, v_r
    const cplx pl = (lane < len) ? s_p[lane] : cmk(0.0, 0.0);
    double gm = cmulc(v, pl).x;
    for (int o = 16; o > 0; o >>= 1) gm += __shfl_xor_sync(0xffffffffu, gm, o);
    const cplx ql = csub(cmul(tau, pl), cscale(v, 0.5 * cabs2(tau) * gm));
    const cplx ctau = cconj(tau);
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int c = 4 * w + u;  // this warp's column c (D, R, L) ; lane = row
      const cplx vc = shfl_c(v, c & 31), qc = shfl_c(ql, c & 31);
      if (c < len) {
        cplx* Dc = Wn + (size_t)slot(sd0, c) * LDB;  // column lo + c
        // D(lane, c), lane >= c: -= v_lane conj(q_c) + q_lane conj(v_c)
        if (lane >= c && lane < len)
          Dc[lane - c] = csub(Dc[lane - c], cadd(cmul(v, cconj(qc)), cmul(ql, cconj(vc))));
        // R(lane, c) = A(hi + lane, lo + c): -= tau s_lane conj(v_c)
        if (lane < nr) Dc[hi + lane - lo - c] = csub(Dc[hi + lane - lo - c], cmul(cmul(tau, s_s[lane]), cconj(vc)));
      }
      if (c >= 1 && c < ncl && lane < len) {
        // L(lane, c) = A(lo + lane, col + c): -= v_lane conj(tau) w_c
        cplx* Lc = Wn + (size_t)slot(sc0, c) * LDB;
        const int off = lo + lane - col - c;
        Lc[off] = csub(Lc[off], cmul(v, cmul(ctau, s_w[c])));
      }
    }
  }
  tsync(t);
  (void)Lcol;
}

// Thread 0 polls, the block follows; false when the wait gave up (here or in
// another block of the launch).
__device__ bool wait_prog(const int* p, int target, int* seen, int* status, long long limit_ns) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    int ok = 1;
    if (*seen < target) {
      int v = ld_acquire_s32(p);
      if (v < target) {
        const long long t0 = gtimer();
        unsigned it = 0;
        while ((v = ld_acquire_s32(p)) < target) {
          if ((++it & 63u) == 0) {
            if (*(volatile int*)&status[ST_BARRIER] != 0) { ok = 0; break; }
            if (gtimer() - t0 > limit_ns) {
              atomicAdd(&status[ST_BARRIER], 1);
              ok = 0;
              break;
            }
          }
        }
      }
      *seen = v;
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

// Bulge chasing by groups of CS consecutive sweeps: group g (sweeps [g CS,
// g CS + CS)) runs in one CTA, round-robin over a cooperative grid; at slot s
// sweep i0 + a does step s - 3a, so the steps of a slot touch disjoint
// entries and each step finds the previous sweep's step k + 2 done.  The
// group's band columns live in a shared-memory ring: a column enters (cp.async
// from AB, one slot ahead) once the previous group has published that its
// last sweep finished the step that frees it, and leaves (back to AB) when no
// step of the group touches it again; then the group publishes its own last
// sweep's progress for the next group.
__global__ void __launch_bounds__(CT, 1) k_chase(ChaseArgs a) {
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx* Wn = reinterpret_cast<cplx*>(dsm);          // [WIN][LDB]
  __shared__ cplx s_p[CS][BW], s_s[CS][BW], s_w[CS][BW];
  __shared__ int s_seen;
  const int n = a.n;
  const int tid = threadIdx.x, t = tid / (32 * TW);
  cplx* AB = a.AB;
  bool first_wait = true;

  for (int grp = blockIdx.x; grp < a.ngrp; grp += gridDim.x) {
    const int i0 = grp * CS;
    int nt[CS];
    int nsw = 0, last = -1;
    for (int q = 0; q < CS; ++q) {
      nt[q] = chase_steps(n, i0 + q);
      if (nt[q] > 0) {
        nsw = q + 1;
        last = max(last, 3 * q + nt[q] - 1);
      }
    }
    if (nsw == 0) continue;
    if (tid == 0) s_seen = (grp == 0) ? PROG_DONE : 0;
    __syncthreads();
    const int* pprev = (grp > 0) ? a.prog + (grp - 1) : nullptr;
    // slot s of the first sweep needs the previous group's last sweep past
    // step s + 2; once the first sweep is done, columns that only the later
    // sweeps reach wait for the whole previous group
    auto need_prev = [&](int s) { return (s < nt[0]) ? s + 3 : PROG_DONE; };
    auto load_cols = [&](int c0, int c1) {
      for (int e = tid; e < (c1 - c0) * LDB; e += CT) {
        const int c = c0 + e / LDB, o = e % LDB;
        cp_async16(Wn + (size_t)(c % WIN) * LDB + o, AB + o + (size_t)LDB * c);
      }
    };
    int wlo = i0, whi = win_need_hi(n, i0, nt, 0);
    if (pprev) {
      int target = need_prev(0);
      if (first_wait && a.planted && blockIdx.x == 1) target += PROG_DONE;  // a test's planted stall
      first_wait = false;
      if (!wait_prog(pprev, target, &s_seen, a.status, a.wait_ns)) return;
    }
    load_cols(wlo, whi);
    for (int s = 0; s <= last; ++s) {
      cp_async_wait_all();
      __syncthreads();
      // one slot ahead: the columns slot s+1 adds
      const int nh = win_need_hi(n, i0, nt, s + 1);
      if (nh > whi) {
        if (pprev && !wait_prog(pprev, need_prev(s + 1), &s_seen, a.status, a.wait_ns)) {
          cp_async_wait_all();
          return;
        }
        load_cols(whi, nh);
        whi = nh;
      }
      const int k = s - 3 * t;
      if (t < nsw && k >= 0 && k < nt[t]) chase_step(a, Wn, t, i0 + t, k, s_p[t], s_s[t], s_w[t]);
      __syncthreads();
      // columns no step of the group touches again go back to AB
      const int nl = (s == last) ? whi : min(win_need_lo(n, i0, nt, s + 1), whi);
      if (nl > wlo) {
        for (int e = tid; e < (nl - wlo) * LDB; e += CT) {
          const int c = wlo + e / LDB, o = e % LDB;
          AB[o + (size_t)LDB * c] = Wn[(size_t)(c % WIN) * LDB + o];
        }
        wlo = nl;
      }
      __syncthreads();
      if (tid == 0) {
        const int kl = s - 3 * (nsw - 1);
        __threadfence();
        st_release_s32(a.prog + grp, (s == last) ? PROG_DONE : max(0, kl + 1));
      }
    }
    cp_async_wait_all();
    __syncthreads();
  }
}

// d = Re diag, e = |subdiag|, ph = prefix products of u_c = sub_c / |sub_c|
// (ph[0] = 1, ph[c+1] = u_c ph[c]): T = diag(ph)^H A diag(ph) is real with
// e >= 0.  One CTA: chunked prefix product, a block scan of the chunk
// products, renormalised to unit modulus.
__global__ void __launch_bounds__(1024) k_phase(int n, const cplx* __restrict__ AB, double* __restrict__ d,
                                                double* __restrict__ e, cplx* __restrict__ ph) {
  __shared__ cplx s_tot[1024];
  const int tid = threadIdx.x, nt = blockDim.x;
  const int per = (n + nt - 1) / nt;
  const int b = tid * per, en = min(n, b + per);
  cplx acc = cmk(1.0, 0.0);
  for (int c = b; c < en; ++c) {
    d[c] = AB[(size_t)LDB * c].x;
    if (c + 1 < n) {
      const cplx s = AB[1 + (size_t)LDB * c];
      const double a = sqrt(cabs2(s));
      e[c] = a;
      acc = cmul(acc, a > 0.0 ? cmk(s.x / a, s.y / a) : cmk(1.0, 0.0));
    }
  }
  s_tot[tid] = acc;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {  // inclusive scan (Hillis-Steele) of the chunk products
    const cplx v = (tid >= o) ? s_tot[tid - o] : cmk(1.0, 0.0);
    __syncthreads();
    s_tot[tid] = cmul(s_tot[tid], v);
    __syncthreads();
  }
  cplx p = (tid > 0) ? s_tot[tid - 1] : cmk(1.0, 0.0);  // product of the chunks before
  for (int c = b; c < en; ++c) {
    const double m = sqrt(cabs2(p));
    ph[c] = cmk(p.x / m, p.y / m);
    if (c + 1 < n) {
      const cplx s = AB[1 + (size_t)LDB * c];
      const double a = sqrt(cabs2(s));
      if (a > 0.0) p = cmul(p, cmk(s.x / a, s.y / a));
    }
  }
}

// Z(r, :) *= ph[r]
__global__ void k_scale_rows(int n, int k, const cplx* __restrict__ ph, cplx* __restrict__ Z, long long ldz) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r < n && c < k) Z[r + ldz * c] = cmul(ph[r], Z[r + ldz * c]);
}

size_t q2_smem_bytes() { return sizeof(cplx) * ((M2 + BW) * (QCOL + 1) + M2 * BW + M2); }

// One wave of the Q2 back-transform: the groups (k, g) with k - g = t, group
// (k, g) = the reflectors of step k of sweeps [g M2, (g+1) M2), applied by
// decreasing sweep.  Groups of one wave touch disjoint rows, and the waves in
// increasing t respect every overlap of the product Q2 = H(0,0) H(0,1) ...
// (sweep-major): the only reordered pairs are row-disjoint.  Block: one group,
// QCOL columns of Z; thread (column, row class mod 8) keeps to its rows, so
// only the dot product's 8-lane reduction crosses threads.
__global__ void __launch_bounds__(QT) k_apply_q2(int n, int t, int K2, const cplx* __restrict__ V2,
                                                 const cplx* __restrict__ tau2, cplx* __restrict__ Z,
                                                 long long ldz, int kz) {
  const int g = blockIdx.x, k = t + g;
  if (k < 0 || k >= K2) return;
  const int cnt = n - 2 - k * BW;  // sweeps with a step k
  const int i0 = g * M2;
  if (i0 >= cnt) return;
  const int i1 = min(cnt, i0 + M2);  // sweeps [i0, i1)
  const int c0 = blockIdx.y * QCOL;
  const int ncol = min(QCOL, kz - c0);
  if (ncol <= 0) return;
  const int rlo = i0 + 1 + k * BW;
  const int rhi = min(n, (i1 - 1) + 1 + (k + 1) * BW);
  const int nrow = rhi - rlo;
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx* Zs = reinterpret_cast<cplx*>(dsm);          // [M2 + BW][QCOL + 1]
  cplx* Vs = Zs + (M2 + BW) * (QCOL + 1);            // [M2][BW]
  cplx* Ts = Vs + M2 * BW;                           // [M2]
  const int tid = threadIdx.x;
  const long long base = toff(n, k);
  for (int e = tid; e < (i1 - i0) * BW; e += QT) Vs[e] = V2[(size_t)BW * (base + i0) + e];
  for (int e = tid; e < i1 - i0; e += QT) Ts[e] = tau2[base + i0 + e];
  for (int e = tid; e < nrow * ncol; e += QT) {
    const int r = e % nrow, c = e / nrow;
    Zs[r * (QCOL + 1) + c] = Z[(rlo + r) + ldz * (c0 + c)];
  }
  // columns >= ncol run on whatever their shared memory holds and are not
  // stored: every lane takes part in the 8-lane reductions
  for (int e = tid; e < nrow * (QCOL - ncol); e += QT) {
    const int r = e % nrow, c = ncol + e / nrow;
    Zs[r * (QCOL + 1) + c] = cmk(0.0, 0.0);
  }
  __syncthreads();
  const int c = tid >> 3, sub = tid & 7;
  {
    for (int ii = i1 - 1; ii >= i0; --ii) {
      const cplx tu = Ts[ii - i0];
      if (tu.x == 0.0 && tu.y == 0.0) continue;
      const int lo = ii + 1 + k * BW;
      const int len = min(BW, n - lo);
      const cplx* v = Vs + (ii - i0) * BW;
      // this thread's rows: absolute rows of class sub (mod 8) in [lo, lo+len)
      const int rfirst = lo + ((sub - lo) % 8 + 8) % 8;
      cplx dot = cmk(0.0, 0.0);
      for (int R = rfirst; R < lo + len; R += 8) dot = cadd(dot, cmulc(v[R - lo], Zs[(R - rlo) * (QCOL + 1) + c]));
      for (int o = 1; o < 8; o <<= 1) {
        dot.x += __shfl_xor_sync(0xffffffffu, dot.x, o);
        dot.y += __shfl_xor_sync(0xffffffffu, dot.y, o);
      }
      const cplx f = cmul(tu, dot);
      for (int R = rfirst; R < lo + len; R += 8) {
        cplx* zp = Zs + (R - rlo) * (QCOL + 1) + c;
        *zp = csub(*zp, cmul(v[R - lo], f));
      }
    }
  }
  __syncthreads();
  for (int e = tid; e < nrow * ncol; e += QT) {
    const int r = e % nrow, cc = e / nrow;
    Z[(rlo + r) + ldz * (c0 + cc)] = Zs[r * (QCOL + 1) + cc];
  }
}

int cluster_size_for(excfv_handle* h) {
  static int cached = 0;
  if (cached) return cached;
  int cl = 8;
  if (cudaFuncSetAttribute(k_panel_qr, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) == cudaSuccess) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(16);
    cfg.blockDim = dim3(PT);
    cfg.dynamicSmemBytes = panel_smem_bytes(RSM);
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 16;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int ncl = 0;
    if (cudaFuncSetAttribute(k_panel_qr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)panel_smem_bytes(RSM)) == cudaSuccess &&
        cudaOccupancyMaxActiveClusters(&ncl, k_panel_qr, &cfg) == cudaSuccess && ncl >= 1)
      cl = 16;
  }
  cudaGetLastError();  // an unsupported size leaves a sticky-free error: clear it
  (void)h;
  cached = cl;
  return cl;
}

}  // namespace

int band_bandwidth() { return BW; }

// Whether the two-stage path handles order n on this device: the panel of
// the first block column (n - BW rows) must fit the cluster's shared memory.
bool two_stage_supported(excfv_handle* h, int n) {
  if (n < 4 * BW) return false;
  const int cl = cluster_size_for(h);
  return (n - BW + cl - 1) / cl <= RSM;
}

// Size (complex elements) of the chase reflectors and their scalars.
size_t chase_reflector_elems(int n) {
  const int K2 = (n - 2 + BW - 1) / BW;
  return (size_t)(BW + 1) * (size_t)toff(n, K2);
}

// Stage 1 on C (n x n, both triangles, leading dimension ld): the band in C's
// lower band, the panel reflectors below it (unit entries explicit once
// two_stage_finish_band has run), tau[c] per column.
int he2hb(excfv_handle* h, int n, cplx* C, long long ld) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const int cl = cluster_size_for(h);
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0), mone = cmk(-1.0, 0.0), mhalf = cmk(-0.5, 0.0);
  // [V | W] and [W | V], n x 2BW each with leading dimension n, in ws.Wp
  const long long lv = n;
  cplx* VW = ws.Wp;
  cplx* WV = ws.Wp + (size_t)lv * 2 * BW;
  cplx* Tt = ws.Tf;                    // BW x BW
  cplx* Mb = ws.Tf + BW * BW;          // BW x BW
  cplx* Yb = ws.Tf + 2 * BW * BW;      // BW x BW
  CUDA_TRY(cudaMemsetAsync(VW, 0, sizeof(cplx) * (size_t)lv * 4 * BW, s));
  // columns past the last panel that still have a reflector slot (c + BW < n)
  // keep tau = 0: the back-transform runs over all n - BW slots
  CUDA_TRY(cudaMemsetAsync(ws.tau, 0, sizeof(cplx) * (size_t)n, s));
  CUDA_TRY(cudaFuncSetAttribute(k_panel_qr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)panel_smem_bytes(RSM)));
  for (int j = 0; j < n - BW - 1; j += BW) {
    const int r0 = j + BW, m = n - r0;
    const int rpc = (m + cl - 1) / cl;
    if (rpc > RSM) {
      excfv_set_error("two-stage reduction: panel of %d rows exceeds the cluster's shared memory", m);
      return EXCFV_ERR_UNSUPPORTED;
    }
    PanelArgs pa;
    pa.C = C; pa.ld = ld; pa.n = n; pa.j = j; pa.rpc = rpc;
    pa.tau = ws.tau; pa.V = VW; pa.ldv = lv; pa.T = Tt;
    const size_t smem = panel_smem_bytes(rpc);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(cl);
    cfg.blockDim = dim3(PT);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = cl;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    prof_begin(h, PROF_TRD_PANEL);
    CUDA_TRY(cudaLaunchKernelEx(&cfg, k_panel_qr, pa));
    count_launch();
    prof_end(h, PROF_TRD_PANEL);
    prof_begin(h, PROF_TRD_UPDATE);
    cplx* A22 = C + r0 + ld * r0;
    cplx* V = VW + r0;
    cplx* X = VW + r0 + lv * BW;   // W slot of [V | W] holds X first
    cplx* Xt = WV + r0;            // W slot of [W | V]
    int rc;
    // X = C22 V
    if ((rc = zgemm1(s, OP_N, OP_N, m, BW, m, one, A22, ld, V, lv, zero, X, lv))) return rc;
    // Xt = X T
    if ((rc = zgemm1(s, OP_N, OP_N, m, BW, BW, one, X, lv, Tt, BW, zero, Xt, lv, TRI_NONE, TRI_NONE,
                     TRI_UPPER)))
      return rc;
    // M = V^H Xt, Y = T^H M, W = Xt - 1/2 V Y
    if ((rc = zgemm1(s, OP_C, OP_N, BW, BW, m, one, V, lv, Xt, lv, zero, Mb, BW))) return rc;
    if ((rc = zgemm1(s, OP_C, OP_N, BW, BW, BW, one, Tt, BW, Mb, BW, zero, Yb, BW, TRI_NONE, TRI_LOWER,
                     TRI_NONE)))
      return rc;
    if ((rc = zgemm1(s, OP_N, OP_N, m, BW, BW, mhalf, V, lv, Yb, BW, one, Xt, lv))) return rc;
    k_swap_vw<<<dim3((m + 255) / 256, BW), 256, 0, s>>>(r0, n, VW, WV, lv); count_launch();
    CUDA_TRY(cudaGetLastError());
    // C22 -= [V W] [W V]^H
    if ((rc = zgemm1(s, OP_N, OP_C, m, m, 2 * BW, mone, VW + r0, lv, WV + r0, lv, one, A22, ld)))
      return rc;
    prof_end(h, PROF_TRD_UPDATE);
  }
  return EXCFV_OK;
}

// Band of C into compact storage AB (LDB x n) and the reflectors' unit entries.
int two_stage_finish_band(excfv_handle* h, int n, cplx* C, long long ld, cplx* AB) {
  cudaStream_t s = h->stream;
  k_band_extract<<<n, 128, 0, s>>>(n, C, ld, AB); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_unit_entries<<<(n + 255) / 256, 256, 0, s>>>(n, C, ld); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// Stage 2 on AB: d, e (real) into ws.d, ws.e, the phase into ph, the chase
// reflectors into V2 / tau2 (chase_reflector_elems(n) complex elements).
int hb2st(excfv_handle* h, int n, cplx* AB, cplx* V2, cplx* ph) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const int K2 = (n - 2 + BW - 1) / BW;
  cplx* tau2 = V2 + (size_t)BW * toff(n, K2);
  const int ngrp = (n - 2 + CS - 1) / CS;
  // groups in flight: a group starts about 3 CS slots after the previous one
  // and runs about n / BW + 3 CS slots
  const int budget = (h->grid_ctas > 0) ? h->grid_ctas : h->nsm;
  const int G = std::max(2, std::min(budget, std::min(ngrp, (n / BW + 3 * CS) / (3 * CS) + 3)));
  CUDA_TRY(cudaMemsetAsync(ws.prog, 0, sizeof(int) * (size_t)ngrp, s));
  const size_t smem = chase_smem_bytes();
  CUDA_TRY(cudaFuncSetAttribute(k_chase, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  ChaseArgs ca;
  ca.AB = AB; ca.n = n; ca.ngrp = ngrp; ca.prog = ws.prog; ca.V2 = V2; ca.tau2 = tau2;
  ca.status = ws.status;
  ca.wait_ns = wait_limit_ns();
  ca.planted = take_planted_stall() ? 1 : 0;
  void* args[] = {&ca};
  CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_chase, dim3(G), dim3(CT), args, smem, s));
  count_launch();
  k_phase<<<1, 1024, 0, s>>>(n, AB, ws.d, ws.e, ph); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// Z (n x k) <- Q Z for Q = Q1 Q2 diag(ph) of the two-stage reduction.
int two_stage_back(excfv_handle* h, int n, int k, const cplx* C, long long ld, const cplx* V2,
                   const cplx* ph, cplx* Z, long long ldz) {
  cudaStream_t s = h->stream;
  const int K2 = (n - 2 + BW - 1) / BW;
  const cplx* tau2 = V2 + (size_t)BW * toff(n, K2);
  k_scale_rows<<<dim3((n + 255) / 256, k), 256, 0, s>>>(n, k, ph, Z, ldz); count_launch();
  CUDA_TRY(cudaGetLastError());
  const int G2 = (n - 2 + M2 - 1) / M2;
  const size_t smem = q2_smem_bytes();
  CUDA_TRY(cudaFuncSetAttribute(k_apply_q2, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const dim3 grid(G2, (k + QCOL - 1) / QCOL);
  for (int t = -(G2 - 1); t < K2; ++t) {
    k_apply_q2<<<grid, QT, smem, s>>>(n, t, K2, V2, tau2, Z, ldz, k); count_launch();
  }
  CUDA_TRY(cudaGetLastError());
  return apply_q(h, n, k, C, ld, Z, ldz, BW);
}
