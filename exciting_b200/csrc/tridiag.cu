// Householder reduction of a Hermitian matrix to real symmetric tridiagonal
// form, C = Q T Q^H (the ZHETRD step of ZHEEVX, external/LAPACK/zheevx.f:441).
//
// Blocked in panels of NBT columns (the zlatrd/zher2k split of LAPACK's
// blocked ZHETRD, restated): one persistent cooperative kernel reduces the
// NBT columns of a panel, then two GEMMs apply the rank-2*NBT update
// C22 -= V W^H + W V^H to the trailing matrix.  Inside the panel kernel every
// column costs two grid-wide barriers:
//
//   phase 1 (row owners)  finish W(:, i-1); update column c with the panel's
//                         previous reflectors; partial |x|^2 for the norm
//   --- barrier ---
//   phase 2 (all)         reflector (beta, tau) from the norm; y = C22 v
//                         (the memory-bound Hermitian matrix-vector product,
//                         tiled 64x64 over all CTAs, row sums by atomics);
//                         partial v^H C v, V^H v, W^H v
//   --- barrier ---
//   phase 3 (row owners)  store v; every CTA derives alpha = -1/2 |tau|^2 (v^H w)
//                         from the reduced scalars, so the row of W needed by the
//                         next column is recomputed locally instead of synced.
//
// Rows are owned in chunks of 64 (four threads per row).  All loads of data
// written by other CTAs inside the kernel use ld.global.cg (L2), since L1 is
// not coherent across SMs.  Barrier waits are bounded in time; a timeout sets
// status[ST_BARRIER] and every CTA then leaves the kernel.
#include "handle.cuh"

namespace {

constexpr int NBT = 32;
constexpr int TT = 256;
constexpr int RCH = 64;
constexpr long long BARRIER_NS = 2000000000LL;  // 2 s

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ long long gtimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ cplx ldc(const cplx* p) { return __ldcg(p); }
__device__ __forceinline__ double ldd(const double* p) { return __ldcg(p); }

// Returns false when the barrier timed out (here or earlier in any CTA).
__device__ bool grid_barrier(unsigned* bar, int* status) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    if (atomicAdd(&status[ST_BARRIER], 0) != 0) {
      ok = 0;
    } else {
      const unsigned gen = ld_acquire(&bar[1]);
      __threadfence();
      const unsigned arrived = atomicAdd(&bar[0], 1u);
      if (arrived == gridDim.x - 1) {
        atomicExch(&bar[0], 0u);
        __threadfence();
        atomicAdd(&bar[1], 1u);
      } else {
        const long long t0 = gtimer();
        unsigned it = 0;
        while (ld_acquire(&bar[1]) == gen) {
          if ((++it & 63u) == 0) {
            if (gtimer() - t0 > BARRIER_NS || atomicAdd(&status[ST_BARRIER], 0) != 0) {
              atomicAdd(&status[ST_BARRIER], 1);
              ok = 0;
              break;
            }
          }
        }
      }
      __threadfence();
    }
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

struct TridArgs {
  int n;
  long long ld;
  cplx* C;
  cplx* W;       // n x NBT, leading dimension ld
  double* d;
  double* e;
  cplx* tau;
  cplx* ybuf;    // 2 x n
  double* red;   // norm[NBT] | vav[2 NBT] | s[2 NBT NBT] | t[2 NBT NBT]
  unsigned* bar;
  int* status;
  int p, nbp, final_panel;
};

__device__ __forceinline__ cplx shfl4_sum(cplx v) {
  v.x += __shfl_xor_sync(0xffffffffu, v.x, 1);
  v.y += __shfl_xor_sync(0xffffffffu, v.y, 1);
  v.x += __shfl_xor_sync(0xffffffffu, v.x, 2);
  v.y += __shfl_xor_sync(0xffffffffu, v.y, 2);
  return v;
}

__global__ void __launch_bounds__(TT, 1) k_tridiag_panel(TridArgs a) {
  __shared__ cplx s_vc[NBT], s_wc[NBT];   // row c of V and W
  __shared__ cplx s_sv[NBT], s_tv[NBT];   // V^H v, W^H v of the previous column
  __shared__ cplx s_acc_s[NBT], s_acc_t[NBT];
  __shared__ cplx s_v[64];
  __shared__ cplx s_part[TT];
  __shared__ double s_dred[TT / 32];
  __shared__ double s_scal[8];            // tau.re, tau.im, scale.re, scale.im, alpha, beta

  const int n = a.n;
  const long long ld = a.ld;
  cplx* __restrict__ C = a.C;
  cplx* __restrict__ W = a.W;
  const int tid = threadIdx.x, bid = blockIdx.x, G = gridDim.x;
  const int rsub = tid & 3, rloc = tid >> 2;
  const int lane = tid & 31, warp = tid >> 5;
  double* red_norm = a.red;
  double* red_vav = a.red + NBT;
  double* red_s = a.red + 3 * NBT;
  double* red_t = a.red + 3 * NBT + 2 * NBT * NBT;

  cplx tau_prev = cmk(0.0, 0.0);
  double alpha_prev = 0.0;

  for (int i = 0; i <= a.nbp; ++i) {
    const int c = a.p + i;
    const bool last = (i == a.nbp);
    cplx* yprev = a.ybuf + (size_t)((i + 1) & 1) * n;   // y of column i-1
    cplx* ycur = a.ybuf + (size_t)(i & 1) * n;

    // ---------------- phase 1 ----------------
    if (tid < i) {
      const int j = tid;
      s_vc[j] = (j == i - 1) ? cmk(1.0, 0.0) : ldc(C + c + ld * (a.p + j));
      if (j < i - 1) s_wc[j] = ldc(W + c + ld * j);
    }
    __syncthreads();
    if (i > 0 && tid == 0) {
      // W(c, i-1) = tau (y(c) - V(c,:) t - W(c,:) s) + alpha v(c), v(c) = 1
      cplx acc = cmk(0.0, 0.0);
      for (int j = 0; j < i - 1; ++j) {
        acc = cadd(acc, cmul(s_vc[j], s_tv[j]));
        acc = cadd(acc, cmul(s_wc[j], s_sv[j]));
      }
      const cplx y = ldc(yprev + c);
      cplx w = cmul(tau_prev, csub(y, acc));
      w.x += alpha_prev;
      s_wc[i - 1] = w;
    }
    __syncthreads();
    double nrm_part = 0.0;
    const bool do_update = (!last) || a.final_panel;
    for (int q = bid; q * RCH < n; q += G) {
      const int r = q * RCH + rloc;
      const bool act = (r >= c) && (r < n);
      cplx wnew = cmk(0.0, 0.0), vprev = cmk(0.0, 0.0);
      if (i > 0) {
        cplx acc = cmk(0.0, 0.0);
        if (act)
          for (int j = rsub; j < i - 1; j += 4) {
            acc = cadd(acc, cmul(ldc(C + r + ld * (a.p + j)), s_tv[j]));
            acc = cadd(acc, cmul(ldc(W + r + ld * j), s_sv[j]));
          }
        acc = shfl4_sum(acc);
        if (act) {
          vprev = (r == c) ? cmk(1.0, 0.0) : ldc(C + r + ld * (c - 1));
          const cplx y = ldc(yprev + r);
          wnew = cmul(tau_prev, csub(y, acc));
          wnew = cadd(wnew, cscale(vprev, alpha_prev));
          if (rsub == 0) W[r + ld * (i - 1)] = wnew;
        }
      }
      if (do_update) {
        cplx acc = cmk(0.0, 0.0);
        if (act)
          for (int j = rsub; j < i; j += 4) {
            const cplx vr = (j == i - 1) ? vprev : ldc(C + r + ld * (a.p + j));
            const cplx wr = (j == i - 1) ? wnew : ldc(W + r + ld * j);
            acc = cadd(acc, cmk(vr.x * s_wc[j].x + vr.y * s_wc[j].y, vr.y * s_wc[j].x - vr.x * s_wc[j].y));
            acc = cadd(acc, cmk(wr.x * s_vc[j].x + wr.y * s_vc[j].y, wr.y * s_vc[j].x - wr.x * s_vc[j].y));
          }
        acc = shfl4_sum(acc);
        if (act && rsub == 0) {
          cplx x = csub(ldc(C + r + ld * c), acc);
          if (r == c) {
            x.y = 0.0;
            a.d[c] = x.x;
          }
          C[r + ld * c] = x;
          if (r >= c + 2) nrm_part += cabs2(x);
        }
      }
      if (i == 0 && act && rsub == 0) ycur[r] = cmk(0.0, 0.0);
    }
    if (last) break;
    // block reduction of the norm
    for (int o = 16; o > 0; o >>= 1) nrm_part += __shfl_xor_sync(0xffffffffu, nrm_part, o);
    if (lane == 0) s_dred[warp] = nrm_part;
    __syncthreads();
    if (tid == 0) {
      double sacc = 0.0;
      for (int w = 0; w < TT / 32; ++w) sacc += s_dred[w];
      if (sacc != 0.0) atomicAdd(&red_norm[i], sacc);
    }
    if (!grid_barrier(a.bar, a.status)) return;

    // ---------------- phase 2 ----------------
    if (tid == 0) {
      const cplx alpha = ldc(C + (c + 1) + ld * c);
      const double xn2 = ldd(red_norm + i);
      double tr = 0.0, ti = 0.0, scr = 0.0, sci = 0.0, beta;
      if (xn2 == 0.0 && alpha.y == 0.0) {
        beta = alpha.x;
      } else {
        const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
        beta = (alpha.x >= 0.0) ? -nrm : nrm;
        tr = (beta - alpha.x) / beta;
        ti = -alpha.y / beta;
        // scale = 1 / (alpha - beta)
        const double dr = alpha.x - beta, di = alpha.y;
        const double den = dr * dr + di * di;
        scr = dr / den;
        sci = -di / den;
      }
      s_scal[0] = tr; s_scal[1] = ti; s_scal[2] = scr; s_scal[3] = sci; s_scal[5] = beta;
    }
    if (tid < NBT) { s_acc_s[tid] = cmk(0.0, 0.0); s_acc_t[tid] = cmk(0.0, 0.0); }
    __syncthreads();
    const cplx scale = cmk(s_scal[2], s_scal[3]);
    // own rows: clear y of the next column, V^H v and W^H v partials
    {
      cplx ps[NBT / 4], pt[NBT / 4];
#pragma unroll
      for (int u = 0; u < NBT / 4; ++u) { ps[u] = cmk(0.0, 0.0); pt[u] = cmk(0.0, 0.0); }
      for (int q = bid; q * RCH < n; q += G) {
        const int r = q * RCH + rloc;
        if (r >= c + 1 && r < n) {
          if (rsub == 0) yprev[r] = cmk(0.0, 0.0);
          const cplx vr = (r == c + 1) ? cmk(1.0, 0.0) : cmul(ldc(C + r + ld * c), scale);
#pragma unroll
          for (int u = 0; u < NBT / 4; ++u) {
            const int j = rsub + 4 * u;
            if (j < i) {
              ps[u] = cadd(ps[u], cmulc(ldc(C + r + ld * (a.p + j)), vr));
              pt[u] = cadd(pt[u], cmulc(ldc(W + r + ld * j), vr));
            }
          }
        }
      }
      // reduce lanes with the same rsub inside the warp, then across warps
#pragma unroll
      for (int u = 0; u < NBT / 4; ++u) {
        for (int o = 4; o < 32; o <<= 1) {
          ps[u].x += __shfl_xor_sync(0xffffffffu, ps[u].x, o);
          ps[u].y += __shfl_xor_sync(0xffffffffu, ps[u].y, o);
          pt[u].x += __shfl_xor_sync(0xffffffffu, pt[u].x, o);
          pt[u].y += __shfl_xor_sync(0xffffffffu, pt[u].y, o);
        }
      }
      if (lane < 4) {
#pragma unroll
        for (int u = 0; u < NBT / 4; ++u) {
          const int j = lane + 4 * u;
          if (j < i) {
            atomicAdd(&s_acc_s[j].x, ps[u].x);
            atomicAdd(&s_acc_s[j].y, ps[u].y);
            atomicAdd(&s_acc_t[j].x, pt[u].x);
            atomicAdd(&s_acc_t[j].y, pt[u].y);
          }
        }
      }
      __syncthreads();
      if (tid < i) {
        atomicAdd(&red_s[2 * (NBT * i + tid)], s_acc_s[tid].x);
        atomicAdd(&red_s[2 * (NBT * i + tid) + 1], s_acc_s[tid].y);
        atomicAdd(&red_t[2 * (NBT * i + tid)], s_acc_t[tid].x);
        atomicAdd(&red_t[2 * (NBT * i + tid) + 1], s_acc_t[tid].y);
      }
    }
    // y = C22 v on the trailing block [c+1, n)^2
    {
      const int r0g = c + 1;
      const int m2 = n - r0g;
      const int nt = (m2 + 63) / 64;
      int S = G / nt;
      if (S < 1) S = 1;
      if (S > nt) S = nt;
      const int per = (nt + S - 1) / S;
      const int items = nt * S;
      const int rr = tid & 63, cg = tid >> 6;
      double vav_re = 0.0, vav_im = 0.0;
      for (int it = bid; it < items; it += G) {
        const int I = it / S, seg = it % S;
        const int r = r0g + I * 64 + rr;
        cplx acc = cmk(0.0, 0.0);
        const int Jb = seg * per, Je = min(nt, Jb + per);
        for (int J = Jb; J < Je; ++J) {
          const int j0 = r0g + J * 64;
          __syncthreads();
          if (tid < 64) {
            const int j = j0 + tid;
            cplx v = cmk(0.0, 0.0);
            if (j < n) v = (j == c + 1) ? cmk(1.0, 0.0) : cmul(ldc(C + j + ld * c), scale);
            s_v[tid] = v;
          }
          __syncthreads();
          if (r < n) {
            const int jmax = min(16, n - (j0 + cg * 16));
            const cplx* col = C + r + ld * (j0 + cg * 16);
#pragma unroll 4
            for (int jj = 0; jj < jmax; ++jj) {
              const cplx x = ldc(col + ld * jj);
              const cplx v = s_v[cg * 16 + jj];
              acc.x += x.x * v.x - x.y * v.y;
              acc.y += x.x * v.y + x.y * v.x;
            }
          }
        }
        __syncthreads();
        s_part[tid] = acc;
        __syncthreads();
        if (tid < 64 && r < n) {
          cplx sum = cadd(cadd(s_part[tid], s_part[tid + 64]), cadd(s_part[tid + 128], s_part[tid + 192]));
          atomicAdd(&ycur[r].x, sum.x);
          atomicAdd(&ycur[r].y, sum.y);
          const cplx vr = (r == c + 1) ? cmk(1.0, 0.0) : cmul(ldc(C + r + ld * c), scale);
          // conj(v_r) * sum
          vav_re += vr.x * sum.x + vr.y * sum.y;
          vav_im += vr.x * sum.y - vr.y * sum.x;
        }
      }
      for (int o = 16; o > 0; o >>= 1) {
        vav_re += __shfl_xor_sync(0xffffffffu, vav_re, o);
        vav_im += __shfl_xor_sync(0xffffffffu, vav_im, o);
      }
      __syncthreads();
      if (lane == 0) { s_part[warp].x = vav_re; s_part[warp].y = vav_im; }
      __syncthreads();
      if (tid == 0) {
        double sr = 0.0, si = 0.0;
        for (int w = 0; w < TT / 32; ++w) { sr += s_part[w].x; si += s_part[w].y; }
        if (sr != 0.0) atomicAdd(&red_vav[2 * i], sr);
        if (si != 0.0) atomicAdd(&red_vav[2 * i + 1], si);
      }
    }
    if (!grid_barrier(a.bar, a.status)) return;

    // ---------------- phase 3 ----------------
    if (tid < i) {
      s_sv[tid] = cmk(ldd(red_s + 2 * (NBT * i + tid)), ldd(red_s + 2 * (NBT * i + tid) + 1));
      s_tv[tid] = cmk(ldd(red_t + 2 * (NBT * i + tid)), ldd(red_t + 2 * (NBT * i + tid) + 1));
    }
    __syncthreads();
    if (tid == 0) {
      const double vav = ldd(red_vav + 2 * i);
      double ts = 0.0;  // Re(t^H s)
      for (int j = 0; j < i; ++j) ts += s_tv[j].x * s_sv[j].x + s_tv[j].y * s_sv[j].y;
      const double t2 = s_scal[0] * s_scal[0] + s_scal[1] * s_scal[1];
      s_scal[4] = -0.5 * t2 * (vav - 2.0 * ts);
      if (bid == 0) {
        a.e[c] = s_scal[5];
        a.tau[c] = cmk(s_scal[0], s_scal[1]);
      }
    }
    for (int q = bid; q * RCH < n; q += G) {
      const int r = q * RCH + rloc;
      if (rsub == 0 && r >= c + 1 && r < n) {
        C[r + ld * c] = (r == c + 1) ? cmk(1.0, 0.0) : cmul(ldc(C + r + ld * c), scale);
      }
    }
    __syncthreads();
    tau_prev = cmk(s_scal[0], s_scal[1]);
    alpha_prev = s_scal[4];
  }
}

__global__ void k_tail_scalar(int n, cplx* C, long long ld, double* d) {
  // n == 1: nothing to reduce
  if (threadIdx.x == 0 && blockIdx.x == 0) d[0] = C[0].x;
}

}  // namespace

int tridiag_workspace_doubles() { return NBT + 2 * NBT + 4 * NBT * NBT; }
int tridiag_nb() { return NBT; }

// Reduces C (n x n, both triangles) to tridiagonal d, e with reflectors
// stored below the subdiagonal of C (unit entry stored explicitly).
int tridiag_reduce(excfv_handle* h, int n, cplx* C, long long ld) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (n == 1) {
    k_tail_scalar<<<1, 32, 0, s>>>(n, C, ld, ws.d); count_launch();
    CUDA_TRY(cudaGetLastError());
    return EXCFV_OK;
  }
  int per_sm = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tridiag_panel, TT, 0));
  if (per_sm < 1) {
    excfv_set_error("tridiag panel kernel cannot be resident");
    return EXCFV_ERR_CUDA;
  }
  const int G = h->nsm;  // one CTA per SM
  const cplx mone = cmk(-1.0, 0.0), one = cmk(1.0, 0.0);
  for (int p = 0; p < n - 1; p += NBT) {
    const int nbp = min(NBT, n - 1 - p);
    const int final_panel = (p + nbp == n - 1) ? 1 : 0;
    CUDA_TRY(cudaMemsetAsync(ws.red, 0, sizeof(double) * tridiag_workspace_doubles(), s));
    CUDA_TRY(cudaMemsetAsync(ws.bar, 0, 2 * sizeof(unsigned), s));
    TridArgs ta;
    ta.n = n; ta.ld = ld; ta.C = C; ta.W = ws.Wp; ta.d = ws.d; ta.e = ws.e; ta.tau = ws.tau;
    ta.ybuf = ws.ybuf;
    ta.red = ws.red; ta.bar = ws.bar; ta.status = ws.status;
    ta.p = p; ta.nbp = nbp; ta.final_panel = final_panel;
    void* args[] = {&ta};
    prof_begin(h, PROF_TRD_PANEL);
    CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_tridiag_panel, dim3(G), dim3(TT), args, 0, s));
    count_launch();
    prof_end(h, PROF_TRD_PANEL);
    if (!final_panel) {
      prof_begin(h, PROF_TRD_UPDATE);
      const int q = p + nbp;
      const int m2 = n - q;
      cplx* V2 = C + q + ld * p;
      cplx* W2 = ws.Wp + q;
      cplx* C22 = C + q + ld * q;
      int rc = zgemm1(s, OP_N, OP_C, m2, m2, nbp, mone, V2, ld, W2, ld, one, C22, ld);
      if (rc) return rc;
      rc = zgemm1(s, OP_N, OP_C, m2, m2, nbp, mone, W2, ld, V2, ld, one, C22, ld);
      if (rc) return rc;
      prof_end(h, PROF_TRD_UPDATE);
    }
  }
  return EXCFV_OK;
}
