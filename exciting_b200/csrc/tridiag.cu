// Householder reduction of a Hermitian matrix to real symmetric tridiagonal
// form, C = Q T Q^H (the ZHETRD step of ZHEEVX, external/LAPACK/zheevx.f:441).
//
// Blocked in panels of NBT columns (the zlatrd/zher2k split of LAPACK's
// blocked ZHETRD, restated): one persistent cooperative kernel reduces the
// NBT columns of a panel, then one GEMM applies the rank-2*NBT update
// C22 -= [V W] [W V]^H to the lower triangle of the trailing matrix (the only
// part the reduction reads).  Inside the panel kernel every column costs two
// grid-wide barriers:
//
//   phase 1 (row owners)  finish W(:, i-1); update column c with the panel's
//                         previous reflectors; partial |x|^2 for the norm
//   --- barrier ---
//   phase 2 (all)         reflector (beta, tau) from the norm; y = C22 v from
//                         the lower 64 x 64 tiles (row part A x and column part
//                         A^H x, equal tile counts per CTA in a folded row
//                         order), tiles streamed by TMA into a shared-memory
//                         ring by a producer warp; partial v^H C v, V^H v, W^H v
//   --- barrier ---
//   phase 3 (row owners)  store v; every CTA derives alpha = -1/2 |tau|^2 (v^H w)
//                         from the reduced scalars, so the row of W needed by the
//                         next column is recomputed locally instead of synced.
//
// Rows are owned in chunks of 64 (four threads per row); a CTA keeps the
// panel's V and W rows of the rows it owns in shared memory, so the row
// phases touch global memory once per row.  All loads of data written by
// other CTAs inside the kernel use ld.global.cg (L2), since L1 is not
// coherent across SMs.  Every wait (grid barrier, TMA tile, free ring slot) is
// bounded in time; a timeout sets status[ST_BARRIER] and every CTA then
// leaves the kernel.  The kernel is instantiated for FP64 storage and for
// complex64 storage (the precision form), with FP64 reflector arithmetic.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "handle.cuh"

namespace {

constexpr int NBT = 32;
constexpr int TT = 256;
constexpr int RCH = 64;
constexpr int MAXCH = 2;   // row chunks per CTA held in shared memory (FP64 storage)
constexpr int MAXCH_C64 = 3;  // complex64 storage: up to three, for more concurrent lanes

// Storage type T2 of C, V and W: double2 (FP64 form) or float2 (the precision
// form's complex64 copy).  Arithmetic is FP64 in both.
__device__ __forceinline__ cplx ldT(const double2* p) { return __ldcg(p); }
__device__ __forceinline__ cplx ldT(const float2* p) {
  const float2 v = __ldcg(p);
  return cmk((double)v.x, (double)v.y);
}
__device__ __forceinline__ void stT(double2* p, cplx v) { *p = v; }
__device__ __forceinline__ void stT(float2* p, cplx v) { *p = make_float2((float)v.x, (float)v.y); }
__device__ __forceinline__ cplx toD(double2 v) { return v; }
__device__ __forceinline__ cplx toD(float2 v) { return cmk((double)v.x, (double)v.y); }
template <typename T2> __device__ __forceinline__ T2 fromD(cplx v);
template <> __device__ __forceinline__ double2 fromD<double2>(cplx v) { return v; }
template <> __device__ __forceinline__ float2 fromD<float2>(cplx v) {
  return make_float2((float)v.x, (float)v.y);
}

template <typename T2, int MC>
struct PanelSmem {
  T2 V[MC][NBT][RCH];
  T2 W[MC][NBT][RCH];
  cplx X[MC][RCH];
};

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

// Tiles of the trailing matrix for y = C22 v: 64 rows x BC columns (16 KB),
// streamed through a ring of STAGES shared-memory slots by TMA.
template <typename T2, int MC>
struct Ring {
  static constexpr int BC = (sizeof(T2) == 16) ? 16 : 32;
  static constexpr int STAGES = (sizeof(T2) == 16) ? (MC == 1 ? 8 : 4) : (MC <= 2 ? 8 : 6);
  static constexpr int TILE = RCH * BC;  // elements
  static constexpr unsigned BYTES = TILE * sizeof(T2);
};
constexpr int MAX_STAGES = 8;

template <typename T2, int MC>
constexpr size_t panel_smem_bytes() {
  return sizeof(PanelSmem<T2, MC>) + 128 + (size_t)Ring<T2, MC>::STAGES * Ring<T2, MC>::BYTES;
}

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait for a TMA tile; gives up (status[ST_BARRIER] set) after
// limit_ns or as soon as another wait of the launch has given up.
__device__ __forceinline__ void mbar_wait(uint64_t* bar, unsigned parity, int* status,
                                          long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return;
  const long long t0 = gtimer();
  unsigned it = 0;
  while (!mbar_try_wait(bar, parity)) {
    if ((++it & 63u) == 0) {
      if (*(volatile int*)&status[ST_BARRIER] != 0) return;
      if (gtimer() - t0 > limit_ns) {
        atomicAdd(&status[ST_BARRIER], 1);
        return;
      }
    }
  }
}
// Bounded wait that reports whether the phase completed.
__device__ __forceinline__ bool mbar_wait_ok(uint64_t* bar, unsigned parity, int* status,
                                             long long limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = gtimer();
  unsigned it = 0;
  while (!mbar_try_wait(bar, parity)) {
    if ((++it & 63u) == 0) {
      if (*(volatile int*)&status[ST_BARRIER] != 0) return false;
      if (gtimer() - t0 > limit_ns) {
        atomicAdd(&status[ST_BARRIER], 1);
        return false;
      }
    }
  }
  return true;
}
// Before the producer leaves the kernel: every TMA copy it issued has landed
// (q copies issued round-robin over the slots), so no copy writes into the
// shared memory of a finished block.  Bounded by limit_ns per slot; this wait
// ignores the status word, since the copies land whether or not a wait of the
// launch gave up.
template <int STAGES>
__device__ __forceinline__ void drain_copies(uint64_t* full, unsigned q, long long limit_ns) {
  for (unsigned s = 0; s < (unsigned)STAGES && s < q; ++s) {
    const unsigned uses = q / STAGES + (s < q % STAGES ? 1u : 0u);
    const unsigned parity = (uses - 1u) & 1u;
    const long long t0 = gtimer();
    while (!mbar_try_wait(&full[s], parity))
      if (gtimer() - t0 > limit_ns) break;
  }
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
// Barrier of the TT consumer threads (named barrier 1; the producer warp does not take part).
__device__ __forceinline__ void csync() { asm volatile("bar.sync 1, %0;" ::"n"(TT) : "memory"); }

// 2-D tiled TMA load (no multicast) of one 64 x BC tile; x counts scalars
// (re and im separately) along the rows, y counts columns.
__device__ __forceinline__ void tma_tile(void* dst, const CUtensorMap* tm, int x, int y,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// Grid barrier on a monotonic arrival counter (zeroed before each launch):
// barrier number e completes when the counter reaches e * gridDim.x (plus
// `planted`, nonzero only when a test arms a target nothing reaches).
// Returns false when it timed out (here or in another CTA).
__device__ bool grid_barrier(unsigned* bar, unsigned& epoch, int* status, long long limit_ns,
                             unsigned planted = 0) {
  __shared__ int s_ok;
  csync();
  if (threadIdx.x == 0) {
    int ok = 1;
    epoch += 1;
    const unsigned target = epoch * gridDim.x + planted;
    // release this CTA's writes and arrive (no return value needed)
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(bar) : "memory");
    if (ld_acquire(&bar[0]) < target) {
      const long long t0 = gtimer();
      unsigned it = 0;
      while (ld_acquire(&bar[0]) < target) {
        if ((++it & 255u) == 0) {
          if (*(volatile int*)&status[ST_BARRIER] != 0 || gtimer() - t0 > limit_ns) {
            atomicAdd(&status[ST_BARRIER], 1);
            ok = 0;
            break;
          }
        }
      }
    }
    s_ok = ok;
  }
  csync();
  return s_ok != 0;
}

template <typename T2>
struct TridArgs {
  int n;
  long long ld;
  T2* C;
  T2* VW;        // n x 2NBT: [V | W] of the panel (leading dimension ld)
  T2* WV;        // n x 2NBT: [W | V]
  double* d;
  double* e;
  cplx* tau;
  cplx* ybuf;    // 2 x n
  double* red;   // norm[NBT] | vav[2 NBT] | s[2 NBT NBT] | t[2 NBT NBT], zero at launch
  double* red_next;  // the next panel's, zeroed by this launch
  unsigned* bar;
  int* status;
  int p, nbp, final_panel;
  long long wait_ns;  // limit of every bounded wait
  unsigned planted;   // extra arrivals the first barrier waits for (0; a test aid)
};

__device__ __forceinline__ cplx shfl4_sum(cplx v) {
  v.x += __shfl_xor_sync(0xffffffffu, v.x, 1);
  v.y += __shfl_xor_sync(0xffffffffu, v.y, 1);
  v.x += __shfl_xor_sync(0xffffffffu, v.x, 2);
  v.y += __shfl_xor_sync(0xffffffffu, v.y, 2);
  return v;
}

// a * conj(b)
__device__ __forceinline__ cplx cmul_cb(cplx a, cplx b) {
  return cmk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

__device__ __forceinline__ cplx warp_sum(cplx v) {
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

constexpr int JB = 8;  // column tiles whose x values are staged per round trip
constexpr int RED_DOUBLES = NBT + 2 * NBT + 4 * NBT * NBT;  // one panel's reduction slots

// Lower 64 x 64 tiles of an nt x nt tile grid in folded row order: row k is
// followed by row nt-1-k (k < nt/2; nt+1 tiles per pair), then the middle row
// when nt is odd, so that equal shares of tiles hold a similar number of runs
// (a run is the part of one row tile in a share).  Returns the run that starts
// at flat index t: row I, columns [Jb, Je), ending at t_end at the latest, and
// the flat index after it.
__device__ __forceinline__ long long tile_run(long long t, long long t_end, int nt, int& I, int& Jb,
                                              int& Je) {
  const long long P = nt + 1;
  const int npair = nt >> 1;
  long long rs, re;
  if (t < (long long)npair * P) {
    const int k = (int)(t / P);
    const long long base = (long long)k * P;
    if (t < base + k + 1) {
      I = k;
      rs = base;
      re = base + k + 1;
    } else {
      I = nt - 1 - k;
      rs = base + k + 1;
      re = base + P;
    }
  } else {
    I = npair;
    rs = (long long)npair * P;
    re = rs + npair + 1;
  }
  Jb = (int)(t - rs);
  const long long e = min(re, t_end);
  Je = Jb + (int)(e - t);
  return e;
}

template <typename T2, int MC>
__global__ void __launch_bounds__(TT + 32, 1)
    k_tridiag_panel(TridArgs<T2> a, const __grid_constant__ CUtensorMap tmap) {
  using R = Ring<T2, MC>;
  extern __shared__ __align__(128) unsigned char dsm[];
  PanelSmem<T2, MC>& S = *reinterpret_cast<PanelSmem<T2, MC>*>(dsm);
  T2* ring;
  {
    const unsigned b0 = smem_u32(dsm);
    const unsigned r0 = (b0 + (unsigned)sizeof(PanelSmem<T2, MC>) + 127u) & ~127u;
    ring = reinterpret_cast<T2*>(dsm + (r0 - b0));
  }
  __shared__ __align__(8) uint64_t s_full[MAX_STAGES];   // tile landed (TMA bytes)
  __shared__ __align__(8) uint64_t s_empty[MAX_STAGES];  // tile consumed by the 8 consumer warps
  __shared__ cplx s_vc[NBT], s_wc[NBT];   // row c+1 of V and W
  __shared__ cplx s_sv[NBT], s_tv[NBT];   // V^H v, W^H v of the current column
  __shared__ T2 s_x[JB * 64];             // staged x values of the trailing column
  __shared__ cplx s_xr[64];               // x values of the run's rows
  __shared__ cplx s_c1[64];               // C(r, c+1) of the run's rows
  __shared__ cplx s_red[TT / 32][64];     // row sums of the 8 warps
  __shared__ cplx s_part[TT / 32];        // v^H y partials of the 8 warps
  __shared__ double s_dred[TT / 32];
  __shared__ double s_scal[8];            // tau.re, tau.im, scale.re, scale.im, alpha, beta, vav, y(c+1)
  __shared__ cplx s_y1;

  const int n = a.n;
  const long long ld = a.ld;
  T2* __restrict__ C = a.C;
  const int tid = threadIdx.x, bid = blockIdx.x, G = gridDim.x;
  const int rsub = tid & 3, rloc = tid >> 2;
  const int lane = tid & 31, warp = tid >> 5;
  double* red_norm = a.red;
  double* red_vav = a.red + NBT;
  double* red_s = a.red + 3 * NBT;
  double* red_t = a.red + 3 * NBT + 2 * NBT * NBT;
  const int nch = (n + RCH - 1) / RCH;
  // the arrival counter runs on over the panels of one reduction: the
  // panels before column p took two barriers per column
  unsigned epoch = 2u * (unsigned)a.p;
  unsigned gtile = 0;  // tiles consumed by this CTA (ring slot and mbarrier phase)
  if (tid == 0) {
    for (int q = 0; q < R::STAGES; ++q) {
      mbar_init(&s_full[q], 1);
      mbar_init(&s_empty[q], TT / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  // ---- producer warp: TMA tiles of every column of the panel, in the order
  // the consumers read them, as far ahead as the ring allows.  The lower tiles
  // read for column c' (rows and columns >= c'+1, or c' for complex64) are not
  // written during the panel (only column c' itself, with zero weight), so the
  // tiles of the next column may land while the current one is finished.
  if (tid >= TT) {
    if (lane == 0) {
      unsigned q = 0;
      for (int i = 0; i < a.nbp; ++i) {
        const int r0g = a.p + i + 1;
        const int rb = (sizeof(T2) == 8) ? (r0g & ~1) : r0g;
        const int nt = (n - rb + 63) / 64;
        const long long ntri = (long long)nt * (nt + 1) / 2;
        const long long t_beg = ntri * bid / G, t_end = ntri * (bid + 1) / G;
        for (long long t = t_beg; t < t_end;) {
          int I, Jb, Je;
          t = tile_run(t, t_end, nt, I, Jb, Je);
          const int colb = rb + Jb * 64;
          const int ntile = (min(n, rb + Je * 64) - colb + R::BC - 1) / R::BC;
          for (int b = 0; b < ntile; ++b, ++q) {
            const unsigned slot = q % R::STAGES;
            if (q >= (unsigned)R::STAGES &&
                !mbar_wait_ok(&s_empty[slot], ((q / R::STAGES) - 1u) & 1u, a.status, a.wait_ns)) {
              drain_copies<R::STAGES>(s_full, q, a.wait_ns);
              return;
            }
            mbar_expect_tx(&s_full[slot], R::BYTES);
            tma_tile(ring + (size_t)slot * R::TILE, &tmap, 2 * (rb + I * 64), colb + b * R::BC,
                     &s_full[slot]);
          }
        }
      }
      drain_copies<R::STAGES>(s_full, q, a.wait_ns);
    }
    return;
  }

  if (bid == 0)  // the next launch's reduction slots (its launch is stream-ordered after this one)
    for (int t = tid; t < RED_DOUBLES; t += TT) a.red_next[t] = 0.0;

  // ---- prologue: column p needs no update; its norm and diagonal
  {
    const int c = a.p;
    double nrm_part = 0.0;
    for (int ch = 0; ch < MC; ++ch) {
      const int q = bid + ch * G;
      if (q >= nch) break;
      const int r = q * RCH + rloc;
      if (rsub == 0 && r >= c && r < n) {
        cplx x = ldT(C + r + ld * c);
        if (r == c) {
          x.y = 0.0;
          a.d[c] = x.x;
          stT(C + r + ld * c, x);
        }
        S.X[ch][rloc] = x;
        if (r >= c + 2) nrm_part += cabs2(x);
        a.ybuf[r] = cmk(0.0, 0.0);
      }
    }
    for (int o = 16; o > 0; o >>= 1) nrm_part += __shfl_xor_sync(0xffffffffu, nrm_part, o);
    if (lane == 0) s_dred[warp] = nrm_part;
    csync();
    if (tid == 0) {
      double sacc = 0.0;
      for (int w = 0; w < TT / 32; ++w) sacc += s_dred[w];
      if (sacc != 0.0) atomicAdd(&red_norm[0], sacc);
    }
  }

  for (int i = 0; i < a.nbp; ++i) {
    const int c = a.p + i;
    cplx* ycur = a.ybuf + (size_t)(i & 1) * n;
    cplx* ynext = a.ybuf + (size_t)((i + 1) & 1) * n;
    if (!grid_barrier(a.bar, epoch, a.status, a.wait_ns, i == 0 ? a.planted : 0u)) return;

    // ================= phase 2: reflector of column c, y = C22 v =================
    // y = C22 v with v(c+1) = 1, v(j) = scale x(j): accumulate C22 x~ (x~(c+1) = 0)
    // and the column c+1 separately, so that the tile loads do not wait for the
    // reflector.  Only the lower triangle of C22 is read: a 64 x 64 tile (I, J),
    // I >= J, adds A_IJ x~_J to y_I (row part) and A_IJ^H x~_I to y_J (column
    // part); diagonal tiles use r >= j for the row part and r > j for the
    // column part.  The tile grid starts at row and column rb (even for
    // complex64, as the TMA row coordinate needs 16-byte alignment); rows and
    // columns below c+1 carry zero weight.  CTA b takes the lower tiles
    // [b T / G, (b+1) T / G) in folded row order, as runs within one row tile.
    const int r0g = c + 1;
    const int rb = (sizeof(T2) == 8) ? (r0g & ~1) : r0g;
    const int nt = (n - rb + 63) / 64;
    const long long ntri = (long long)nt * (nt + 1) / 2;
    const long long t_beg = ntri * bid / G, t_end = ntri * (bid + 1) / G;
    constexpr int BPT = 64 / R::BC;    // TMA tiles (boxes) per 64-column tile
    constexpr int NPASS = R::BC / 16;  // 16-column passes per box
    const int rg = tid & 15, cq = tid >> 4;
    double vav_re = 0.0, vav_im = 0.0;
    if (tid == 0) {
      const cplx alpha = ldT(C + (c + 1) + ld * c);
      const double xn2 = ldd(red_norm + i);
      double tr = 0.0, ti = 0.0, scr = 0.0, sci = 0.0, beta;
      if (xn2 == 0.0 && alpha.y == 0.0) {
        beta = alpha.x;
      } else {
        // one square root, then two independent reciprocals (short dependent chain)
        const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
        beta = (alpha.x >= 0.0) ? -nrm : nrm;
        const double dr = alpha.x - beta, di = alpha.y;  // scale = 1 / (alpha - beta)
        const double rb = 1.0 / beta, rd = 1.0 / (dr * dr + di * di);
        tr = 1.0 - alpha.x * rb;
        ti = -alpha.y * rb;
        scr = dr * rd;
        sci = -di * rd;
      }
      s_scal[0] = tr; s_scal[1] = ti; s_scal[2] = scr; s_scal[3] = sci; s_scal[5] = beta;
    }
    for (long long t = t_beg; t < t_end;) {
      int I, Jb, Je;
      t = tile_run(t, t_end, nt, I, Jb, Je);
      const int row0 = rb + I * 64;
      const int colb = rb + Jb * 64;
      const int ntile = (min(n, rb + Je * 64) - colb + R::BC - 1) / R::BC;
      csync();  // the previous run's row sums are consumed
      if (tid < 64) {
        const int r2 = row0 + tid;
        s_xr[tid] = (r2 < n && r2 > c + 1) ? ldT(C + r2 + ld * c) : cmk(0.0, 0.0);
      } else if (tid < 128) {
        const int r2 = row0 + tid - 64;
        s_c1[tid - 64] = (Jb == 0 && r2 < n && r2 >= c + 1) ? ldT(C + r2 + ld * (c + 1)) : cmk(0.0, 0.0);
      }
      cplx rowp[4], xr[4];
      T2 xrT[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) rowp[u] = cmk(0.0, 0.0);
      cplx scale = cmk(0.0, 0.0);
      int b = 0;
      for (int g0 = Jb; g0 < Je; g0 += JB) {
        const int g1 = min(Je, g0 + JB);
        T2 rowf[4];  // complex64: row sums of this group in FP32 (at most 32 terms)
#pragma unroll
        for (int u = 0; u < 4; ++u) rowf[u] = fromD<T2>(cmk(0.0, 0.0));
        if (g0 != Jb) csync();  // the previous group's x values are consumed
        {
          const int j_a = rb + g0 * 64 + tid, j_b = j_a + TT;
          const int lim = min(n, rb + g1 * 64);
          s_x[tid] = fromD<T2>((j_a < lim && j_a > c + 1) ? ldT(C + j_a + ld * c) : cmk(0.0, 0.0));
          s_x[tid + TT] = fromD<T2>((j_b < lim && j_b > c + 1) ? ldT(C + j_b + ld * c) : cmk(0.0, 0.0));
        }
        csync();
        if (g0 == Jb) {
          scale = cmk(s_scal[2], s_scal[3]);
#pragma unroll
          for (int u = 0; u < 4; ++u) { xr[u] = s_xr[rg + 16 * u]; xrT[u] = fromD<T2>(xr[u]); }
        }
        const int bend = min(ntile, (g1 - Jb) * BPT);
        // Two tiles per step: their products and shuffle reductions are
        // independent, so each warp has two chains in flight.
        constexpr int NB = 2;
        for (; b < bend;) {
          const int nb = min(NB, bend - b);
          T2 cp[NB][NPASS];
          int jcol[NB][NPASS];
          T2 xjv[NB][NPASS];
#pragma unroll
          for (int z = 0; z < NB; ++z) {
            if (z >= nb) break;
            const unsigned q = gtile + b + z;
            mbar_wait(&s_full[q % R::STAGES], (q / R::STAGES) & 1u, a.status, a.wait_ns);
          }
#pragma unroll
          for (int z = 0; z < NB; ++z) {
#pragma unroll
            for (int ps = 0; ps < NPASS; ++ps) { cp[z][ps] = fromD<T2>(cmk(0.0, 0.0)); jcol[z][ps] = -1; }
            if (z >= nb) continue;
            const int bz = b + z;
            const T2* tile = ring + (size_t)((gtile + bz) % R::STAGES) * R::TILE;
            const int jt = Jb + bz / BPT;              // column tile of this box
            const bool diag = (jt == I);
#pragma unroll
            for (int ps = 0; ps < NPASS; ++ps) {
              const int cb = ps * 16 + cq;              // column within the box
              const int jl = (bz % BPT) * R::BC + cb;   // column within the 64-wide tile
              const T2 xj = s_x[(jt - g0) * 64 + jl];
              xjv[z][ps] = xj;
              jcol[z][ps] = rb + jt * 64 + jl;
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int rl = rg + 16 * u;
                const T2 av = tile[cb * RCH + rl];
                if (!diag || rl >= jl) {  // row part: A(r, j) x~(j)
                  if constexpr (sizeof(T2) == 16) {
                    rowp[u].x += av.x * xj.x - av.y * xj.y;
                    rowp[u].y += av.x * xj.y + av.y * xj.x;
                  } else {
                    rowf[u].x = fmaf(av.x, xj.x, fmaf(-av.y, xj.y, rowf[u].x));
                    rowf[u].y = fmaf(av.x, xj.y, fmaf(av.y, xj.x, rowf[u].y));
                  }
                }
                if (!diag || rl > jl) {   // column part: conj(A(r, j)) x~(r)
                  cp[z][ps].x += av.x * xrT[u].x + av.y * xrT[u].y;
                  cp[z][ps].y += av.x * xrT[u].y - av.y * xrT[u].x;
                }
              }
            }
          }
          // The slots are refilled by the async proxy (TMA): order this thread's
          // generic reads of them before that write, then release them (one
          // arrival per consumer warp).
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          __syncwarp();
          if (lane == 0) {
            for (int z = 0; z < nb; ++z) mbar_arrive(&s_empty[(gtile + b + z) % R::STAGES]);
          }
#pragma unroll
          for (int o = 1; o < 16; o <<= 1)
#pragma unroll
            for (int z = 0; z < NB; ++z)
#pragma unroll
              for (int ps = 0; ps < NPASS; ++ps) {
                cp[z][ps].x += __shfl_xor_sync(0xffffffffu, cp[z][ps].x, o);
                cp[z][ps].y += __shfl_xor_sync(0xffffffffu, cp[z][ps].y, o);
              }
          if (rg == 0) {
#pragma unroll
            for (int z = 0; z < NB; ++z)
#pragma unroll
              for (int ps = 0; ps < NPASS; ++ps) {
                const int j = jcol[z][ps];
                if (j >= r0g && j < n) {
                  const cplx sc = cmul(scale, toD(cp[z][ps]));
                  atomicAdd(&ycur[j].x, sc.x);
                  atomicAdd(&ycur[j].y, sc.y);
                  const cplx vj = (j == c + 1) ? cmk(1.0, 0.0) : cmul(toD(xjv[z][ps]), scale);
                  vav_re += vj.x * sc.x + vj.y * sc.y;  // conj(v_j) * contribution
                  vav_im += vj.x * sc.y - vj.y * sc.x;
                }
              }
          }
          b += nb;
        }
        if constexpr (sizeof(T2) == 8) {
#pragma unroll
          for (int u = 0; u < 4; ++u) rowp[u] = cadd(rowp[u], toD(rowf[u]));
        }
      }
      gtile += ntile;
      // row sums: the two column threads of a warp, then the 8 warps
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        rowp[u].x += __shfl_xor_sync(0xffffffffu, rowp[u].x, 16);
        rowp[u].y += __shfl_xor_sync(0xffffffffu, rowp[u].y, 16);
      }
      if (lane < 16) {
#pragma unroll
        for (int u = 0; u < 4; ++u) s_red[warp][rg + 16 * u] = rowp[u];
      }
      csync();
      if (tid < 64) {
        const int r = row0 + tid;
        if (r >= r0g && r < n) {
          cplx sum = s_red[0][tid];
#pragma unroll
          for (int w = 1; w < TT / 32; ++w) sum = cadd(sum, s_red[w][tid]);
          sum = cadd(cmul(scale, sum), s_c1[tid]);
          atomicAdd(&ycur[r].x, sum.x);
          atomicAdd(&ycur[r].y, sum.y);
          const cplx vr = (r == c + 1) ? cmk(1.0, 0.0) : cmul(s_xr[tid], scale);
          vav_re += vr.x * sum.x + vr.y * sum.y;  // conj(v_r) * sum
          vav_im += vr.x * sum.y - vr.y * sum.x;
        }
      }
    }
    csync();  // the scalars of thread 0 are visible
    const cplx scale = cmk(s_scal[2], s_scal[3]);
    for (int o = 16; o > 0; o >>= 1) {
      vav_re += __shfl_xor_sync(0xffffffffu, vav_re, o);
      vav_im += __shfl_xor_sync(0xffffffffu, vav_im, o);
    }
    csync();
    if (lane == 0) { s_part[warp].x = vav_re; s_part[warp].y = vav_im; }
    // own rows: clear y of the next column, V^H v and W^H v partials
    {
      cplx ps[NBT / 4], pt[NBT / 4];
#pragma unroll
      for (int u = 0; u < NBT / 4; ++u) { ps[u] = cmk(0.0, 0.0); pt[u] = cmk(0.0, 0.0); }
      for (int ch = 0; ch < MC; ++ch) {
        const int q = bid + ch * G;
        if (q >= nch) break;
        const int r = q * RCH + rloc;
        if (r >= c + 1 && r < n) {
          if (rsub == 0) ynext[r] = cmk(0.0, 0.0);
          if (i > 0) {
            const cplx vr = (r == c + 1) ? cmk(1.0, 0.0) : cmul(S.X[ch][rloc], scale);
#pragma unroll
            for (int u = 0; u < NBT / 4; ++u) {
              const int j = rsub + 4 * u;
              if (j < i) {
                ps[u] = cadd(ps[u], cmulc(toD(S.V[ch][j][rloc]), vr));
                pt[u] = cadd(pt[u], cmulc(toD(S.W[ch][j][rloc]), vr));
              }
            }
          }
        }
      }
      // Reduce over the 8 rows of the warp (lane bits 2..4) and scatter: after
      // three halving exchanges lane l holds the warp's sum for
      // j = rsub + 4 u(l), u(l) = 4 b4 + 2 b3 + b2 of its lane bits.
      const bool h1 = (lane >> 4) & 1, h2 = (lane >> 3) & 1, h3 = (lane >> 2) & 1;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const cplx sa = h1 ? ps[k] : ps[k + 4], ka = h1 ? ps[k + 4] : ps[k];
        const cplx ta = h1 ? pt[k] : pt[k + 4], kb = h1 ? pt[k + 4] : pt[k];
        ps[k] = cmk(ka.x + __shfl_xor_sync(0xffffffffu, sa.x, 16), ka.y + __shfl_xor_sync(0xffffffffu, sa.y, 16));
        pt[k] = cmk(kb.x + __shfl_xor_sync(0xffffffffu, ta.x, 16), kb.y + __shfl_xor_sync(0xffffffffu, ta.y, 16));
      }
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        const cplx sa = h2 ? ps[k] : ps[k + 2], ka = h2 ? ps[k + 2] : ps[k];
        const cplx ta = h2 ? pt[k] : pt[k + 2], kb = h2 ? pt[k + 2] : pt[k];
        ps[k] = cmk(ka.x + __shfl_xor_sync(0xffffffffu, sa.x, 8), ka.y + __shfl_xor_sync(0xffffffffu, sa.y, 8));
        pt[k] = cmk(kb.x + __shfl_xor_sync(0xffffffffu, ta.x, 8), kb.y + __shfl_xor_sync(0xffffffffu, ta.y, 8));
      }
      {
        const cplx sa = h3 ? ps[0] : ps[1], ka = h3 ? ps[1] : ps[0];
        const cplx ta = h3 ? pt[0] : pt[1], kb = h3 ? pt[1] : pt[0];
        ps[0] = cmk(ka.x + __shfl_xor_sync(0xffffffffu, sa.x, 4), ka.y + __shfl_xor_sync(0xffffffffu, sa.y, 4));
        pt[0] = cmk(kb.x + __shfl_xor_sync(0xffffffffu, ta.x, 4), kb.y + __shfl_xor_sync(0xffffffffu, ta.y, 4));
      }
      csync();  // the last run's row sums in s_red are consumed
      const int jl = rsub + 4 * (4 * (int)h1 + 2 * (int)h2 + (int)h3);
      s_red[warp][jl] = ps[0];
      s_red[warp][NBT + jl] = pt[0];
    }
    csync();
    if (tid < 2 * NBT && (tid & (NBT - 1)) < i) {
      cplx sum = s_red[0][tid];
#pragma unroll
      for (int w = 1; w < TT / 32; ++w) sum = cadd(sum, s_red[w][tid]);
      double* dst = (tid < NBT) ? red_s : red_t;
      const int j = tid & (NBT - 1);
      atomicAdd(&dst[2 * (NBT * i + j)], sum.x);
      atomicAdd(&dst[2 * (NBT * i + j) + 1], sum.y);
    }
    if (tid == 32) {
      double sr = 0.0, si = 0.0;
      for (int w = 0; w < TT / 32; ++w) { sr += s_part[w].x; si += s_part[w].y; }
      if (sr != 0.0) atomicAdd(&red_vav[2 * i], sr);
      if (si != 0.0) atomicAdd(&red_vav[2 * i + 1], si);
    }
    if (!grid_barrier(a.bar, epoch, a.status, a.wait_ns)) return;

    // ========== phase 3 (finish column c) merged with phase 1 (column c+1) ==========
    const bool upd = (i + 1 < a.nbp) || a.final_panel;  // column c+1 is updated here
    const int c1 = c + 1;
    // one round of independent loads
    if (warp == 0) {
      if (lane < i) {
        s_sv[lane] = cmk(ldd(red_s + 2 * (NBT * i + lane)), ldd(red_s + 2 * (NBT * i + lane) + 1));
        s_tv[lane] = cmk(ldd(red_t + 2 * (NBT * i + lane)), ldd(red_t + 2 * (NBT * i + lane) + 1));
      }
      if (lane == 31) s_scal[6] = ldd(red_vav + 2 * i);
    } else if (warp == 1) {
      if (lane < i) s_vc[lane] = ldT(a.VW + c1 + ld * lane);
      if (lane == i) s_vc[i] = cmk(1.0, 0.0);
    } else if (warp == 2) {
      if (lane < i) s_wc[lane] = ldT(a.VW + c1 + ld * (NBT + lane));
      if (lane == 31) s_y1 = ldc(ycur + c1);
    }
    cplx yr[MC], cn[MC];
    for (int ch = 0; ch < MC; ++ch) {
      yr[ch] = cmk(0.0, 0.0);
      cn[ch] = cmk(0.0, 0.0);
      const int q = bid + ch * G;
      if (q >= nch) break;
      const int r = q * RCH + rloc;
      if (r >= c1 && r < n) {
        yr[ch] = ldc(ycur + r);
        if (upd && rsub == 0) cn[ch] = ldT(C + r + ld * c1);
      }
    }
    csync();
    const cplx tau = cmk(s_scal[0], s_scal[1]);
    if (warp == 0) {
      // alpha = -1/2 |tau|^2 (v^H C v - 2 Re(t^H s))
      double ts = (lane < i) ? s_tv[lane].x * s_sv[lane].x + s_tv[lane].y * s_sv[lane].y : 0.0;
      for (int o = 16; o > 0; o >>= 1) ts += __shfl_xor_sync(0xffffffffu, ts, o);
      const double alpha = -0.5 * (tau.x * tau.x + tau.y * tau.y) * (s_scal[6] - 2.0 * ts);
      // W(c+1, i) = tau (y(c+1) - V(c+1,:) t - W(c+1,:) s) + alpha v(c+1), v(c+1) = 1
      cplx t = cmk(0.0, 0.0);
      if (lane < i) t = cadd(cmul(s_vc[lane], s_tv[lane]), cmul(s_wc[lane], s_sv[lane]));
      t = warp_sum(t);
      if (lane == 0) {
        s_scal[4] = alpha;
        cplx w = cmul(tau, csub(s_y1, t));
        w.x += alpha;
        s_wc[i] = w;
        if (bid == 0) {
          a.e[c] = s_scal[5];
          a.tau[c] = tau;
        }
      }
    }
    csync();
    const double alpha = s_scal[4];
    double nrm_part = 0.0;
    for (int ch = 0; ch < MC; ++ch) {
      const int q = bid + ch * G;
      if (q >= nch) break;
      const int r = q * RCH + rloc;
      const bool act = (r >= c1) && (r < n);
      cplx vr = cmk(0.0, 0.0), wr = cmk(0.0, 0.0);
      cplx acc = cmk(0.0, 0.0);
      if (act) {
        vr = (r == c1) ? cmk(1.0, 0.0) : cmul(S.X[ch][rloc], scale);
        for (int j = rsub; j < i; j += 4) {
          acc = cadd(acc, cmul(toD(S.V[ch][j][rloc]), s_tv[j]));
          acc = cadd(acc, cmul(toD(S.W[ch][j][rloc]), s_sv[j]));
        }
      }
      acc = shfl4_sum(acc);
      if (act) {
        wr = cadd(cmul(tau, csub(yr[ch], acc)), cscale(vr, alpha));
        if (rsub == 0) {
          stT(C + r + ld * c, vr);
          S.V[ch][i][rloc] = fromD<T2>(vr);
          S.W[ch][i][rloc] = fromD<T2>(wr);
          stT(a.VW + r + ld * i, vr);
          stT(a.WV + r + ld * (NBT + i), vr);
          stT(a.VW + r + ld * (NBT + i), wr);
          stT(a.WV + r + ld * i, wr);
        }
      }
      if (upd) {
        cplx u = cmk(0.0, 0.0);
        if (act)
          for (int j = rsub; j <= i; j += 4) {
            const cplx vj = (j == i) ? vr : toD(S.V[ch][j][rloc]);
            const cplx wj = (j == i) ? wr : toD(S.W[ch][j][rloc]);
            u = cadd(u, cmul_cb(vj, s_wc[j]));
            u = cadd(u, cmul_cb(wj, s_vc[j]));
          }
        u = shfl4_sum(u);
        if (act && rsub == 0) {
          cplx x = csub(cn[ch], u);
          if (r == c1) {
            x.y = 0.0;
            a.d[c1] = x.x;
          }
          stT(C + r + ld * c1, x);
          S.X[ch][rloc] = x;
          if (r >= c1 + 2) nrm_part += cabs2(x);
        }
      }
    }
    if (i + 1 < a.nbp) {
      for (int o = 16; o > 0; o >>= 1) nrm_part += __shfl_xor_sync(0xffffffffu, nrm_part, o);
      if (lane == 0) s_dred[warp] = nrm_part;
      csync();
      if (tid == 0) {
        double sacc = 0.0;
        for (int w = 0; w < TT / 32; ++w) sacc += s_dred[w];
        if (sacc != 0.0) atomicAdd(&red_norm[i + 1], sacc);
      }
    }
  }
}

template <typename T2>
__global__ void k_tail_scalar(const T2* C, double* d) {
  // n == 1: nothing to reduce
  if (threadIdx.x == 0 && blockIdx.x == 0) d[0] = toD(C[0]).x;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(smem_u32(dst)), "l"(src),
               "r"(src_bytes)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Lower 64 x 64 tiles of C (m x m, complex64) -= A B^H, A and B m x 2NBT
// (leading dimension ld, even): the trailing update of the complex64
// reduction, FP32 products.  Persistent, one CTA per SM: CTA b takes the
// lower tiles b, b + G, ... (row-major over the lower triangle).  A tile's
// 64 rows of A and B over the whole K = 2 NBT land in shared memory by
// cp.async (k-major, 64 KB), and the next tile's are copied into the other
// stage while this one is computed; the tile of C is read into registers
// before the products.  16 x 16 threads with 4 x 4 outputs each (rows on the
// fast thread index for coalesced accesses).
constexpr int HK = 2 * NBT;
constexpr int HER2K_SMEM = 2 * 2 * HK * 64 * (int)sizeof(float2);

__device__ __forceinline__ void lower_tile(int t, int& I, int& J) {
  int q = (int)((sqrtf(8.f * (float)t + 1.f) - 1.f) * 0.5f);
  while ((q + 1) * (q + 2) / 2 <= t) ++q;
  while (q * (q + 1) / 2 > t) --q;
  I = q;
  J = t - q * (q + 1) / 2;
}

__global__ void __launch_bounds__(256, 1) k_her2k_f32(int m, const float2* __restrict__ A,
                                                      const float2* __restrict__ B, long long ld,
                                                      float2* __restrict__ C) {
  extern __shared__ __align__(16) float2 hsm[];  // [stage][A | B][k][64 rows]
  const int nt = (m + 63) / 64;
  const int T = nt * (nt + 1) / 2;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  int t = blockIdx.x;
  if (t >= T) return;
  // rows r0.. of A and c0.. of B over all K into stage st; 16-byte chunks
  // (two rows), rows past m zero-filled
  auto issue = [&](int tt, int st) {
    int I, J;
    lower_tile(tt, I, J);
    float2* sA = hsm + (size_t)st * 2 * HK * 64;
    float2* sB = sA + HK * 64;
    for (int e = threadIdx.x; e < HK * 32; e += 256) {
      const int kk = e >> 5, ch = e & 31;
      const int ra = I * 64 + 2 * ch, cb = J * 64 + 2 * ch;
      const int na = max(0, min(2, m - ra)), nb = max(0, min(2, m - cb));
      cp_async16(sA + kk * 64 + 2 * ch, na ? (const void*)(A + ra + ld * kk) : (const void*)A, 8 * na);
      cp_async16(sB + kk * 64 + 2 * ch, nb ? (const void*)(B + cb + ld * kk) : (const void*)B, 8 * nb);
    }
  };
  issue(t, 0);
  cp_async_commit();
  for (int it = 0; t < T; t += gridDim.x, ++it) {
    const int st = it & 1;
    if (t + (int)gridDim.x < T) issue(t + gridDim.x, st ^ 1);
    cp_async_commit();
    int I, J;
    lower_tile(t, I, J);
    const int r0 = I * 64, c0 = J * 64;
    float2 cv[4][4];
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int rr = r0 + tx + 16 * u, cc = c0 + ty + 16 * v;
        cv[u][v] = (rr < m && cc < m) ? C[rr + ld * cc] : make_float2(0.f, 0.f);
      }
    float accr[4][4], acci[4][4];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) { accr[u][v] = 0.f; acci[u][v] = 0.f; }
    cp_async_wait1();  // this stage's copies (the newest group may still be in flight)
    __syncthreads();
    const float2* sA = hsm + (size_t)st * 2 * HK * 64;
    const float2* sB = sA + HK * 64;
#pragma unroll 8
    for (int kk = 0; kk < HK; ++kk) {
      float2 av[4], bv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) { av[u] = sA[kk * 64 + tx + 16 * u]; bv[u] = sB[kk * 64 + ty + 16 * u]; }
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {  // a * conj(b)
          accr[u][v] = fmaf(av[u].x, bv[v].x, fmaf(av[u].y, bv[v].y, accr[u][v]));
          acci[u][v] = fmaf(av[u].y, bv[v].x, fmaf(-av[u].x, bv[v].y, acci[u][v]));
        }
    }
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int cc = c0 + ty + 16 * v;
      if (cc >= m) continue;
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int rr = r0 + tx + 16 * u;
        if (rr < m) C[rr + ld * cc] = make_float2(cv[u][v].x - accr[u][v], cv[u][v].y - acci[u][v]);
      }
    }
    __syncthreads();  // this stage is refilled two tiles later
  }
}

// C22 -= [V W] [W V]^H: one K = 2 NBT GEMM in the storage precision
int her2k_update(excfv_handle* h, int m2, const double2* VW, const double2* WV, long long ld,
                 double2* C22) {
  const cplx mone = cmk(-1.0, 0.0), one = cmk(1.0, 0.0);
  return zgemm1(h->stream, OP_N, OP_C, m2, m2, 2 * NBT, mone, VW, ld, WV, ld, one, C22, ld,
                TRI_LOWER);
}
int her2k_update(excfv_handle* h, int m2, const float2* VW, const float2* WV, long long ld,
                 float2* C22) {
  if ((ld & 1) || (reinterpret_cast<uintptr_t>(VW) & 15) || (reinterpret_cast<uintptr_t>(WV) & 15)) {
    excfv_set_error("complex64 trailing update: panels not 16-byte aligned (ld=%lld)", ld);
    return EXCFV_ERR_ARG;
  }
  if (!h->her2k_smem_set) {  // once per handle (handles are per device)
    CUDA_TRY(cudaFuncSetAttribute(k_her2k_f32, cudaFuncAttributeMaxDynamicSharedMemorySize, HER2K_SMEM));
    h->her2k_smem_set = true;
  }
  // one CTA per SM of the handle's budget (a lane of a batch gets its share)
  const int nt = (m2 + 63) / 64;
  const int grid = min(nt * (nt + 1) / 2, (h->grid_ctas > 0) ? h->grid_ctas : h->nsm);
  k_her2k_f32<<<grid, 256, HER2K_SMEM, h->stream>>>(m2, VW, WV, ld, C22); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

}  // namespace

int tridiag_workspace_doubles() { return 2 * RED_DOUBLES; }
int tridiag_nb() { return NBT; }

// cuTensorMapEncodeTiled through the runtime's driver entry point
static PFN_cuTensorMapEncodeTiled_v12000 encode_tiled_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// Tensor map of the n x n matrix C (leading dimension ld) as real scalars:
// 2n rows of re/im pairs, n columns; tiles of 64 complex rows x BC columns.
template <typename T2>
static int make_tile_map(CUtensorMap* tm, const T2* C, int n, long long ld) {
  auto fn = encode_tiled_fn();
  if (!fn) {
    excfv_set_error("cuTensorMapEncodeTiled is not available from the driver");
    return EXCFV_ERR_CUDA;
  }
  if ((reinterpret_cast<uintptr_t>(C) & 15) || ((ld * sizeof(T2)) & 15)) {
    excfv_set_error("tridiagonal reduction: matrix base or column stride not 16-byte aligned");
    return EXCFV_ERR_ARG;
  }
  const cuuint64_t dims[2] = {2ull * (cuuint64_t)n, (cuuint64_t)n};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(T2)};
  const cuuint32_t box[2] = {2u * RCH, (cuuint32_t)Ring<T2, 2>::BC};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUtensorMapDataType dt =
      (sizeof(T2) == 16) ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  const CUresult r = fn(tm, dt, 2, const_cast<T2*>(C), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    excfv_set_error("cuTensorMapEncodeTiled failed (%d) for n=%d ld=%lld", (int)r, n, ld);
    return EXCFV_ERR_CUDA;
  }
  return EXCFV_OK;
}

template <typename T2>
int tridiag_tail_max();
template <typename T2>
int tridiag_tail(excfv_handle* h, int n, int c0, T2* C, long long ld);

int tridiag_tail_start(int n, bool complex64) {
  const int tail_max = complex64 ? tridiag_tail_max<float2>() : tridiag_tail_max<double2>();
  for (int p = 0; p < n - 1; p += NBT)
    if (n - p <= tail_max) return p;
  return n > 0 ? n - 1 : 0;
}

template <typename T2, int MC>
static int tridiag_reduce_t(excfv_handle* h, int n, T2* C, long long ld) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (n == 1) {
    k_tail_scalar<T2><<<1, 32, 0, s>>>(C, ws.d); count_launch();
    CUDA_TRY(cudaGetLastError());
    return EXCFV_OK;
  }
  const int G = (h->grid_ctas > 0) ? h->grid_ctas : h->nsm;  // one CTA per SM of the budget
  const int nch = (n + RCH - 1) / RCH;
  if (nch > MC * G) {
    excfv_set_error("tridiagonal reduction supports n <= %d with %d CTAs", MC * G * RCH, G);
    return EXCFV_ERR_UNSUPPORTED;
  }
  const int smem = (int)panel_smem_bytes<T2, MC>();
  CUtensorMap tmap;
  if (int rc = make_tile_map(&tmap, C, n, ld)) return rc;
  CUDA_TRY(cudaFuncSetAttribute(k_tridiag_panel<T2, MC>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int per_sm = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tridiag_panel<T2, MC>, TT + 32, smem));
  if (per_sm < 1) {
    excfv_set_error("tridiag panel kernel cannot be resident");
    return EXCFV_ERR_CUDA;
  }
  // [V W] and [W V] of the panel in the storage type, both with leading
  // dimension ld, inside ws.Wp (n_max x 4 NBT FP64 complex: room for ld <= n_max
  // in FP64 storage and ld <= 2 n_max in complex64)
  if ((size_t)ld * 2 * NBT * 2 * sizeof(T2) > (size_t)ws.nmatmax * 4 * NBT * sizeof(cplx)) {
    excfv_set_error("tridiagonal reduction: leading dimension %lld exceeds the panel workspace", ld);
    return EXCFV_ERR_ARG;
  }
  T2* VW = reinterpret_cast<T2*>(ws.Wp);
  T2* WV = VW + (size_t)ld * 2 * NBT;
  // once per reduction: both panels' reduction slots and the barrier counter;
  // each panel launch then zeroes the slots of the next
  CUDA_TRY(cudaMemsetAsync(ws.red, 0, sizeof(double) * tridiag_workspace_doubles(), s));
  CUDA_TRY(cudaMemsetAsync(ws.bar, 0, 2 * sizeof(unsigned), s));
  const long long wait_ns = wait_limit_ns();
  const unsigned planted = take_planted_stall() ? 1u : 0u;
  // the last columns (a trailing block the cluster's shared memory holds) go
  // to the cluster kernel (tridiag_tail.cu); a planted stall keeps the panels
  const int p_tail = planted ? n : tridiag_tail_start(n, sizeof(T2) == 8);
  for (int p = 0; p < n - 1; p += NBT) {
    if (p == p_tail) {
      prof_begin(h, PROF_TRD_TAIL);
      if (int rc = tridiag_tail<T2>(h, n, p, C, ld)) return rc;
      prof_end(h, PROF_TRD_TAIL);
      break;
    }
    const int nbp = min(NBT, n - 1 - p);
    const int final_panel = (p + nbp == n - 1) ? 1 : 0;
    const int pi = p / NBT;
    TridArgs<T2> ta;
    ta.n = n; ta.ld = ld; ta.C = C; ta.VW = VW; ta.WV = WV; ta.d = ws.d; ta.e = ws.e;
    ta.tau = ws.tau; ta.ybuf = ws.ybuf; ta.bar = ws.bar; ta.status = ws.status;
    ta.red = ws.red + (size_t)(pi & 1) * RED_DOUBLES;
    ta.red_next = ws.red + (size_t)((pi + 1) & 1) * RED_DOUBLES;
    ta.p = p; ta.nbp = nbp; ta.final_panel = final_panel;
    ta.wait_ns = wait_ns;
    ta.planted = (p == 0) ? planted : 0u;
    void* args[] = {&ta, &tmap};
    prof_begin(h, PROF_TRD_PANEL);
    CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_tridiag_panel<T2, MC>, dim3(G), dim3(TT + 32), args,
                                         (size_t)smem, s));
    count_launch();
    prof_end(h, PROF_TRD_PANEL);
    if (!final_panel) {
      prof_begin(h, PROF_TRD_UPDATE);
      const int q = p + nbp;
      // C22 -= [V W] [W V]^H on the lower triangle (all the next panel reads)
      int rc = her2k_update(h, n - q, VW + q, WV + q, ld, C + q + ld * q);
      if (rc) return rc;
      prof_end(h, PROF_TRD_UPDATE);
    }
  }
  return EXCFV_OK;
}

// Reduces C (n x n, both triangles) to tridiagonal d, e with reflectors
// stored below the diagonal of C (unit entry stored explicitly).
// One row chunk per CTA (eight ring stages, 128 KB of tiles in flight) when
// that covers n, else two (four stages).
int tridiag_reduce(excfv_handle* h, int n, cplx* C, long long ld) {
  const int G = (h->grid_ctas > 0) ? h->grid_ctas : h->nsm;
  if ((n + RCH - 1) / RCH <= G) return tridiag_reduce_t<double2, 1>(h, n, C, ld);
  return tridiag_reduce_t<double2, MAXCH>(h, n, C, ld);
}

// Rows one CTA of the reduction can own (its shared-memory row chunks).
int tridiag_rows_per_cta(bool complex64) { return (complex64 ? MAXCH_C64 : MAXCH) * RCH; }

// The same on a complex64 matrix (d, e and tau stay FP64).
// Two row chunks per CTA (eight ring stages) when they suffice, else three.
int tridiag_reduce_f32(excfv_handle* h, int n, float2* C, long long ld) {
  const int G = (h->grid_ctas > 0) ? h->grid_ctas : h->nsm;
  if ((n + RCH - 1) / RCH <= MAXCH * G) return tridiag_reduce_t<float2, MAXCH>(h, n, C, ld);
  return tridiag_reduce_t<float2, MAXCH_C64>(h, n, C, ld);
}
