// The setup contractions of the precision form on the 5th-generation tensor
// cores: C = A^H B (H = A^H (aa A), O = A^H A; hamiltonsetup.f90:90-103,
// overlapsetup.f90:82-108) as split-BF16 products with FP32 accumulation in
// TMEM, recombined to FP64 accuracy.
//
// Splitting.  Every row r of the operands (a column of the packed matching
// coefficients, contiguous along K) is scaled by a power of two 2^e_r with
// max_k |Re|, |Im| < 2^e_r, and its real and imaginary parts are cut into
// NSL slices of 7 bits: x / 2^e_r = sum_s a_s 2^-7(s+1) with integers
// |a_0| <= 128, |a_s| <= 64 (s >= 1), exact in BF16; the rest is below
// 2^-7 NSL - 1.  The product is then
//   C(i,j) = 2^(e_i + f_j) sum_{s+t <= NSL-1} 2^-7(s+t+2) sum_k a_s(k,i) b_t(k,j)
// (the slice pairs of level d = s + t, the pairs past the last level
// dropped).  Products of slices are integers below 2^14, so a level's FP32
// sum over 256 of K stays below 2^24 and is exact (level 0: 2 products of
// <= 2^14 per k; level 4: 2 pairs of <= 2^13 and 3 of <= 2^12, 4 products
// each: < 2^23.8 over 256 k); every 256 of K the level accumulators are
// flushed from TMEM into FP64 registers.  With NSL = 5 (15 slice pairs) the
// setup's relative error is ~1e-10 and the eigenvalues move by ~1e-11 Ha.
//
// Kernel.  One CTA per 128 x 48 output tile (upper triangle of H and of O,
// both in one grid), 10 warps: warp 0 issues the TMA copies (one 3-D box of
// the 2 NSL planes (Re, Im per slice) of A's 128 rows and one of the 3 NSL
// planes (Re, Im, -Re per slice) of B's 48 rows per 16 of K, into a 3-stage
// ring, 32-byte swizzle), warp 1 allocates the 512 TMEM columns and one of
// its threads issues tcgen05.mma (kind::f16, BF16 x BF16 -> F32, M 128,
// N 96, K 16; both operands K-major): with B's planes in that order [Br; Bi]
// and [Bi; -Br] are contiguous 96-row operands, so Ar [Br; Bi]^T + Ai [Bi;
// -Br]^T = [Re | Im] is two MMAs per slice pair into one accumulator of 96
// columns per level (NSL x 96 columns), warps 2..9 read the
// accumulators back with tcgen05.ld after each 256 of K (tcgen05.commit on
// an mbarrier) and keep the FP64 sums.  Every wait is bounded in time; a
// wait that gives up sets the status word, the CTA waits for its copies and
// MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "handle.cuh"

namespace {

constexpr int NSL = 5;                 // slices per part
constexpr int NPL = 2 * NSL;           // planes of the row (A) side: (slice, re/im)
constexpr int NPB = 3 * NSL;           // planes of the column (B) side: (slice, re/im/-re)
constexpr int BM = 128, BN = 48, KS = 16;
constexpr int CHUNK = 16;              // K steps (of 16) per exact FP32 chunk = 256 of K
constexpr int STAGES = 3;
constexpr int NEPI = 8;                // epilogue warps
constexpr int NWARP = 2 + NEPI;
constexpr unsigned A_PLANE = BM * KS * 2;            // 4096 B
constexpr unsigned B_PLANE = BN * KS * 2;            // 1536 B
constexpr unsigned STAGE_BYTES = NPL * A_PLANE + NPB * B_PLANE;
constexpr unsigned TMEM_COLS = 512;
constexpr int COLS_PER_LEVEL = 2 * BN; // Re then Im
constexpr int EPI_COLS = BN / 2;       // output columns per epilogue thread
static_assert(NSL * COLS_PER_LEVEL <= (int)TMEM_COLS, "TMEM holds one Re/Im accumulator per level");
static_assert(B_PLANE % 256 == 0 && A_PLANE % 256 == 0, "planes keep the 32-byte swizzle phase");

struct Bf16xArgs {
  int n;                 // C is n x n (upper triangle)
  int nsteps;            // K steps of KS
  int ntm, ntn;          // tile rows (of BM) and columns (of BN)
  int tpb;               // tiles per batch entry
  const double* scA[2];  // row scales of the A-side operand
  const double* scB[2];  // row scales of the B-side operand
  cplx* C[2];
  long long ldc;
  int* flag;
  long long wait_ns;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ long long gtimer() {
  long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned c) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(c) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}
// bounded wait; false when it (or another wait of the launch) gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity, int* flag, long long lim) {
  if (mbar_try(b, parity)) return true;
  const long long t0 = gtimer();
  unsigned it = 0;
  while (!mbar_try(b, parity)) {
    if ((++it & 63u) == 0) {
      if (*(volatile int*)flag != 0) return false;
      if (gtimer() - t0 > lim) {
        atomicAdd(flag, 1);
        return false;
      }
    }
  }
  return true;
}
// wait without giving up early on the flag (used to drain work in flight)
__device__ __forceinline__ void mbar_drain(uint64_t* b, unsigned parity, long long lim) {
  const long long t0 = gtimer();
  while (!mbar_try(b, parity))
    if (gtimer() - t0 > lim) break;
}
__device__ __forceinline__ void tma3d(void* dst, const CUtensorMap* tm, int x, int y, int z, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// shared-memory matrix descriptor: K-major, 32-byte swizzle, rows of 32 B,
// 8-row groups 256 B apart (SBO), LBO unused (1), version 1
__device__ __forceinline__ uint64_t sdesc(unsigned addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1u << 16) | ((uint64_t)(256u >> 4) << 32) |
         ((uint64_t)1u << 46) | ((uint64_t)6u << 61);
}
// instruction descriptor: F32 accumulator, BF16 A and B, both K-major,
// N = 2 BN (Re and Im side by side), M = BM
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)((2 * BN) >> 3) << 17) |
                           ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
      "l"(a), "l"(b), "r"(idesc), "r"(acc)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                   smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// 8 consecutive FP32 columns of this thread's TMEM lane
#define TMEM_LD8(addr, v, q)                                                                              \
  do {                                                                                                    \
    uint32_t r0, r1, r2, r3, r4, r5, r6, r7;                                                              \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"                  \
                 : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3), "=r"(r4), "=r"(r5), "=r"(r6), "=r"(r7)          \
                 : "r"(addr)                                                                              \
                 : "memory");                                                                             \
    v[q] = __uint_as_float(r0); v[q + 1] = __uint_as_float(r1); v[q + 2] = __uint_as_float(r2);         \
    v[q + 3] = __uint_as_float(r3); v[q + 4] = __uint_as_float(r4); v[q + 5] = __uint_as_float(r5);     \
    v[q + 6] = __uint_as_float(r6); v[q + 7] = __uint_as_float(r7);                                      \
  } while (0)
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// linear tile -> (batch entry, tile row, tile column) over the tiles that hold
// an upper-triangle element (row <= column)
__device__ __forceinline__ void tile_coords(const Bf16xArgs& a, int t, int& z, int& ti, int& tj) {
  z = t / a.tpb;
  int l = t - z * a.tpb;
  for (tj = 0; tj < a.ntn; ++tj) {
    const int rows = min(a.ntm, (BN * tj + BN - 1) / BM + 1);
    if (l < rows) break;
    l -= rows;
  }
  ti = l;
}

__global__ void __launch_bounds__(32 * NWARP, 1)
    k_zgemm_bf16x(Bf16xArgs a, const __grid_constant__ CUtensorMap tA0, const __grid_constant__ CUtensorMap tA1,
                  const __grid_constant__ CUtensorMap tB0, const __grid_constant__ CUtensorMap tB1) {
  extern __shared__ __align__(1024) unsigned char dsm[];
  unsigned char* ring;
  {
    const unsigned b0 = smem_u32(dsm);
    ring = dsm + (((b0 + 1023u) & ~1023u) - b0);
  }
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES], acc_full, acc_empty, mma_done;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int z, ti, tj;
  tile_coords(a, blockIdx.x, z, ti, tj);
  const int nchunks = (a.nsteps + CHUNK - 1) / CHUNK;

  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(&acc_full, 1);
    mbar_init(&acc_empty, NEPI);
    mbar_init(&mma_done, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_slot)),
                 "r"(TMEM_COLS)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = tmem_slot;

  if (warp == 0) {
    // ---- TMA producer -----------------------------------------------------
    if (lane == 0) {
      const CUtensorMap* mA = z ? &tA1 : &tA0;
      const CUtensorMap* mB = z ? &tB1 : &tB0;
      int issued = 0;
      for (int it = 0; it < a.nsteps; ++it) {
        const int s = it % STAGES;
        if (it >= STAGES && !mbar_wait(&empty[s], ((it / STAGES) - 1) & 1, a.flag, a.wait_ns)) break;
        unsigned char* st = ring + (size_t)s * STAGE_BYTES;
        mbar_expect_tx(&full[s], STAGE_BYTES);
        tma3d(st, mA, it * KS, ti * BM, 0, &full[s]);
        tma3d(st + NPL * A_PLANE, mB, it * KS, tj * BN, 0, &full[s]);
        ++issued;
      }
      // every issued copy lands before the CTA can finish
      for (int it = max(0, issued - STAGES); it < issued; ++it)
        mbar_drain(&full[it % STAGES], (it / STAGES) & 1, a.wait_ns);
    }
  } else if (warp == 1) {
    // ---- MMA issuer -------------------------------------------------------
    if (lane == 0) {
      bool ok = true;
      for (int it = 0; it < a.nsteps && ok; ++it) {
        const int c = it / CHUNK;
        const bool first = (it % CHUNK) == 0;
        if (first && c > 0) {
          if (!mbar_wait(&acc_empty, (c - 1) & 1, a.flag, a.wait_ns)) { ok = false; break; }
          tc_fence_after();
        }
        const int s = it % STAGES;
        if (!mbar_wait(&full[s], (it / STAGES) & 1, a.flag, a.wait_ns)) { ok = false; break; }
        tc_fence_after();
        const unsigned baseA = smem_u32(ring + (size_t)s * STAGE_BYTES);
        const unsigned baseB = baseA + NPL * A_PLANE;
#pragma unroll
        for (int d = 0; d < NSL; ++d) {
          const uint32_t dacc = tmem + d * COLS_PER_LEVEL;   // [Re | Im] of level d
#pragma unroll
          for (int sa = 0; sa <= d; ++sa) {
            const int tb = d - sa;
            const uint64_t aRe = sdesc(baseA + (2 * sa) * A_PLANE), aIm = sdesc(baseA + (2 * sa + 1) * A_PLANE);
            // [Br; Bi] and [Bi; -Br]: planes 3 tb, 3 tb + 1 and 3 tb + 1, 3 tb + 2
            const uint64_t bP = sdesc(baseB + (3 * tb) * B_PLANE), bQ = sdesc(baseB + (3 * tb + 1) * B_PLANE);
            const uint32_t acc = (first && sa == 0) ? 0u : 1u;
            // [Re | Im] += Ar [Br | Bi] + Ai [Bi | -Br]
            umma(dacc, aRe, bP, IDESC, acc);
            umma(dacc, aIm, bQ, IDESC, 1u);
          }
        }
        umma_commit(&empty[s]);
        if ((it % CHUNK) == CHUNK - 1 || it == a.nsteps - 1) umma_commit(&acc_full);
      }
      // every issued MMA completes before TMEM is freed
      umma_commit(&mma_done);
      mbar_drain(&mma_done, 0, a.wait_ns);
    }
  } else {
    // ---- epilogue: FP64 sums of the level accumulators --------------------
    const int ew = warp - 2;
    const int quarter = warp & 3;          // TMEM lanes 32*quarter .. +31
    const int half = ew >> 2;              // output columns EPI_COLS*half ..
    const int row = quarter * 32 + lane;   // tile row = TMEM lane
    const uint32_t lane_base = tmem + ((uint32_t)(quarter * 32) << 16);
    double are[EPI_COLS], aim[EPI_COLS];
#pragma unroll
    for (int q = 0; q < EPI_COLS; ++q) are[q] = aim[q] = 0.0;
    bool ok = true;
    for (int c = 0; c < nchunks; ++c) {
      if (!mbar_wait(&acc_full, c & 1, a.flag, a.wait_ns)) { ok = false; break; }
      tc_fence_after();
#pragma unroll
      for (int d = 0; d < NSL; ++d) {
        const double f = ldexp(1.0, -7 * (d + 2));
        float vr[EPI_COLS], vi[EPI_COLS];
        const uint32_t cre = lane_base + d * COLS_PER_LEVEL + EPI_COLS * half;
#pragma unroll
        for (int q = 0; q < EPI_COLS; q += 8) {
          TMEM_LD8(cre + q, vr, q);
          TMEM_LD8(cre + BN + q, vi, q);
        }
        tmem_wait_ld();
#pragma unroll
        for (int q = 0; q < EPI_COLS; ++q) {
          are[q] = fma(f, (double)vr[q], are[q]);
          aim[q] = fma(f, (double)vi[q], aim[q]);
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(&acc_empty);
    }
    if (ok) {
      const int i = ti * BM + row;
      if (i < a.n) {
        const double* scb = z ? a.scB[1] : a.scB[0];
        const double si = z ? a.scA[1][i] : a.scA[0][i];
        cplx* C = z ? a.C[1] : a.C[0];
#pragma unroll
        for (int q = 0; q < EPI_COLS; ++q) {
          const int j = tj * BN + EPI_COLS * half + q;
          if (j < a.n && i <= j) {
            const double sc = si * scb[j];
            // H and O are Hermitian: the diagonal is real (the truncated
            // slice pairs leave ~1e-11 of imaginary part there)
            C[i + a.ldc * j] = cmk(are[q] * sc, (i == j) ? 0.0 : aim[q] * sc);
          }
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
  }
}

// slices of one operand: X is K x R complex, column-major (leading dimension
// ld), contiguous along K.  outA (nullable) receives the row-side layout
// [NPL][rpad][kpad] BF16 (plane 2s + part), outB (nullable) the column-side
// layout [NPB][rpad][kpad] (planes 3s: Re, 3s + 1: Im, 3s + 2: -Re);
// sc[r] = 2^e_r.  Rows past R and k past K are zero.
__global__ void k_slice(const cplx* X, long long ld, int K, int R, int kpad, int rpad, __nv_bfloat16* outA,
                        __nv_bfloat16* outB, double* sc) {
  const int r = blockIdx.x;
  __shared__ double red[32];
  double m = 0.0;
  if (r < R)
    for (int k = threadIdx.x; k < K; k += blockDim.x) {
      const cplx x = X[k + ld * r];
      m = fmax(m, fmax(fabs(x.x), fabs(x.y)));
    }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  m = red[0];
  // 2^e > m, so every |x| / 2^e < 1
  const int e = (m > 0.0) ? ilogb(m) + 1 : 0;
  if (threadIdx.x == 0 && r < rpad) sc[r] = ldexp(1.0, e);
  const double inv = ldexp(1.0, 7 - e);   // scale, then the first slice's 2^7
  const size_t plane = (size_t)rpad * kpad;
  const size_t at = (size_t)r * kpad;
  for (int k = threadIdx.x; k < kpad; k += blockDim.x) {
    cplx x = cmk(0.0, 0.0);
    if (r < R && k < K) x = X[k + ld * r];
    double vr = x.x * inv, vi = x.y * inv;
#pragma unroll
    for (int s = 0; s < NSL; ++s) {
      const double qr = rint(vr), qi = rint(vi);
      const __nv_bfloat16 br = __float2bfloat16_rn((float)qr), bi = __float2bfloat16_rn((float)qi);
      if (outA) {
        outA[(size_t)(2 * s) * plane + at + k] = br;
        outA[(size_t)(2 * s + 1) * plane + at + k] = bi;
      }
      if (outB) {
        outB[(size_t)(3 * s) * plane + at + k] = br;
        outB[(size_t)(3 * s + 1) * plane + at + k] = bi;
        outB[(size_t)(3 * s + 2) * plane + at + k] = __float2bfloat16_rn((float)-qr);
      }
      vr = (vr - qr) * 128.0;
      vi = (vi - qi) * 128.0;
    }
  }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

// [np][rpad][kpad] BF16 planes as a 3-D map, boxes of 16 k x rows x np planes
int plane_map(CUtensorMap* tm, const __nv_bfloat16* P, int kpad, int rpad, int rows, int np) {
  auto fn = encode_fn();
  if (!fn) {
    excfv_set_error("cuTensorMapEncodeTiled is not available from the driver");
    return EXCFV_ERR_CUDA;
  }
  const cuuint64_t dims[3] = {(cuuint64_t)kpad, (cuuint64_t)rpad, (cuuint64_t)np};
  const cuuint64_t strides[2] = {(cuuint64_t)kpad * 2, (cuuint64_t)kpad * rpad * 2};
  const cuuint32_t box[3] = {(cuuint32_t)KS, (cuuint32_t)rows, (cuuint32_t)np};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 3, const_cast<__nv_bfloat16*>(P), dims, strides,
                        box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    excfv_set_error("cuTensorMapEncodeTiled failed (%d) for BF16 slice planes %d x %d", (int)r, kpad, rpad);
    return EXCFV_ERR_CUDA;
  }
  return EXCFV_OK;
}

}  // namespace

int bf16x_kpad(int K) { return (K + KS - 1) / KS * KS; }
int bf16x_rpad(int R) { return (R + BM - 1) / BM * BM; }
// BF16 elements of the slice planes of one k-point: A in both layouts, aa A
// in the column-side layout
size_t bf16x_plane_elems(int K, int R) { return (size_t)(NPL + 2 * NPB) * bf16x_kpad(K) * bf16x_rpad(R); }

// H = A^H Z and O = A^H A (upper triangles, n x n, leading dimension ldc)
// from the packed K x n operands A and Z (leading dimension ld) through the
// handle's slice buffers.
int zgemm_cn_bf16x(excfv_handle* h, int n, int K, const cplx* A, const cplx* Z, long long ld, cplx* H, cplx* O,
                   long long ldc) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (n <= 0 || K <= 0) return EXCFV_ERR_ARG;
  const int kpad = bf16x_kpad(K), rpad = bf16x_rpad(n);
  const size_t plane = (size_t)kpad * rpad;
  if (!ws.slices || ws.slices_elems < bf16x_plane_elems(K, n) || ws.slice_sc_n < 2 * (size_t)rpad) {
    excfv_set_error("split-BF16 setup: slice workspace not reserved for K = %d, n = %d", K, n);
    return EXCFV_ERR_STATE;
  }
  __nv_bfloat16* PA = ws.slices;                    // A, row side
  __nv_bfloat16* PAB = PA + (size_t)NPL * plane;    // A, column side
  __nv_bfloat16* PZB = PAB + (size_t)NPB * plane;   // aa A, column side
  double* scA = ws.slice_sc;
  double* scZ = ws.slice_sc + rpad;
  k_slice<<<rpad, 256, 0, s>>>(A, ld, K, n, kpad, rpad, PA, PAB, scA);
  count_launch();
  k_slice<<<rpad, 256, 0, s>>>(Z, ld, K, n, kpad, rpad, nullptr, PZB, scZ);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  CUtensorMap mA, mZ, mAb;
  int rc;
  if ((rc = plane_map(&mA, PA, kpad, rpad, BM, NPL)) || (rc = plane_map(&mZ, PZB, kpad, rpad, BN, NPB)) ||
      (rc = plane_map(&mAb, PAB, kpad, rpad, BN, NPB)))
    return rc;
  Bf16xArgs a;
  a.n = n;
  a.nsteps = kpad / KS;
  a.ntm = (n + BM - 1) / BM;
  a.ntn = (n + BN - 1) / BN;
  int tpb = 0;
  for (int tj = 0; tj < a.ntn; ++tj) tpb += std::min(a.ntm, (BN * tj + BN - 1) / BM + 1);
  a.tpb = tpb;
  // entry 0: H = A^H Z; entry 1: O = A^H A
  a.scA[0] = scA; a.scB[0] = scZ; a.C[0] = H;
  a.scA[1] = scA; a.scB[1] = scA; a.C[1] = O;
  a.ldc = ldc;
  a.flag = ws.status + ST_SETUP;
  a.wait_ns = wait_limit_ns();
  const size_t smem = (size_t)STAGES * STAGE_BYTES + 1024;
  static bool attr = false;
  if (!attr) {
    CUDA_TRY(cudaFuncSetAttribute(k_zgemm_bf16x, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    attr = true;
  }
  k_zgemm_bf16x<<<2 * tpb, 32 * NWARP, smem, s>>>(a, mA, mA, mZ, mAb);
  count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}
