// Complex FP64 GEMM C = alpha A^H B + beta C with TMA-fed tiles, for the
// setup contractions H = A^H (aa A) and O = A^H A (hamiltonsetup.f90:90-103,
// overlapsetup.f90:82-108): A is K x M and B is K x N, column-major and
// contiguous along K (the packed matching coefficients and aa A), C is
// M x N column-major; optionally only C's upper triangle is formed.
//
// Tiles: 64 x 64 complex outputs per CTA, four consumer warps (2 x 2) of
// 32 x 32, DMMA m8n8k4 on re/im operands as in zgemm.cu (tcgen05 has no FP64
// kind).  Operands: every pipeline stage holds 16 k of A^H and of B, brought
// by non-multicast cp.async.bulk.tensor.2d as four boxes of 64 rows x 4 k
// (64-byte rows: a lane's (re, im) fragment is one 16-byte shared-memory
// load, conflict-free), in a STAGES-deep ring of full/empty mbarriers that
// thread 0 refills once the four warps have released a slot.  Grid: the output tiles (upper triangle only when
// asked) of both batch entries; tiles past the last full wave of resident
// CTAs run with their K range split over several CTAs, whose partial sums a
// second kernel adds in a fixed order, so the last wave is full too.  Every
// wait is bounded in time; a wait that gives up sets the status word.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "handle.cuh"

namespace {

constexpr int TM = 64, TN = 64;   // output tile (complex)
constexpr int KB = 4;             // k per box (64-byte rows)
constexpr int KS = 16;            // k per stage = 4 boxes
constexpr int STAGES = 3;
constexpr int NCW = 4;            // warps (all consume; thread 0 also produces)
constexpr int GT = 32 * NCW;
constexpr unsigned BOX_BYTES = TM * KB * 16;             // 4 KB
constexpr unsigned STAGE_BYTES = 2 * (KS / KB) * BOX_BYTES;  // 32 KB: A^H and B

struct TmaGemmArgs {
  int m, n, nk;            // C is m x n; nk stages of KS along K
  cplx alpha, beta;
  cplx* C0;
  cplx* C1;
  long long ldc;
  int uplo;                // TRI_UPPER (square C) or TRI_NONE
  int ntm, ntn, tpb;       // tiles per dimension, tiles per batch entry
  int tile0;               // first tile of this launch
  int splitk;              // K pieces per tile
  cplx* part;              // splitk > 1: partial sums [tile - tile0][split][TM * TN]
  int* flag;               // set when a bounded wait gives up
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
__device__ __forceinline__ void tma_box(void* dst, const CUtensorMap* tm, int x, int y, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// linear tile -> (batch entry, tile row, tile column); upper triangle by columns
__device__ __forceinline__ void tile_coords(const TmaGemmArgs& a, int t, int& z, int& ti, int& tj) {
  z = t / a.tpb;
  const int l = t - z * a.tpb;
  if (a.uplo == TRI_UPPER) {
    int c = (int)((sqrt(8.0 * l + 1.0) - 1.0) * 0.5);
    while ((c + 1) * (c + 2) / 2 <= l) ++c;
    while (c * (c + 1) / 2 > l) --c;
    tj = c;
    ti = l - c * (c + 1) / 2;
  } else {
    ti = l % a.ntm;
    tj = l / a.ntm;
  }
}

__global__ void __launch_bounds__(GT) k_zgemm_cn_tma(TmaGemmArgs a, const __grid_constant__ CUtensorMap tA0,
                                                     const __grid_constant__ CUtensorMap tA1,
                                                     const __grid_constant__ CUtensorMap tB0,
                                                     const __grid_constant__ CUtensorMap tB1) {
  extern __shared__ __align__(128) unsigned char dsm[];
  // stage s: A^H boxes q = 0..3 then B boxes q = 0..3, each [64 rows][4 k] complex
  unsigned char* ring;
  {
    const unsigned b0 = smem_u32(dsm);
    ring = dsm + (((b0 + 127u) & ~127u) - b0);
  }
  __shared__ __align__(8) uint64_t full[STAGES], empty[STAGES];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t = a.tile0 + (int)blockIdx.x / a.splitk;
  const int split = (int)blockIdx.x % a.splitk;
  int z, ti, tj;
  tile_coords(a, t, z, ti, tj);
  const int i0 = ti * TM, j0 = tj * TN;
  const int chunk = (a.nk + a.splitk - 1) / a.splitk;
  const int kb = split * chunk, ke = min(a.nk, kb + chunk);
  const int nit = max(0, ke - kb);
  if (tid == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], NCW);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();

  const CUtensorMap* mA = z ? &tA1 : &tA0;
  const CUtensorMap* mB = z ? &tB1 : &tB0;
  int issued = 0;  // thread 0: stages issued
  auto issue = [&](int it) {
    const int s = it % STAGES;
    mbar_expect_tx(&full[s], STAGE_BYTES);
    unsigned char* st = ring + (size_t)s * STAGE_BYTES;
    const int k0 = (kb + it) * KS;
    for (int q = 0; q < KS / KB; ++q) {
      // x counts doubles along K (re, im interleaved): 16-byte aligned
      tma_box(st + q * BOX_BYTES, mA, 2 * (k0 + q * KB), i0, &full[s]);
      tma_box(st + (KS / KB + q) * BOX_BYTES, mB, 2 * (k0 + q * KB), j0, &full[s]);
    }
    ++issued;
  };
  // every issued copy lands before the block can finish (thread 0)
  auto drain = [&]() {
    for (int s = 0; s < STAGES && s < issued; ++s) {
      const int uses = issued / STAGES + (s < issued % STAGES ? 1 : 0);
      const long long t0 = gtimer();
      while (!mbar_try(&full[s], (uses - 1) & 1))
        if (gtimer() - t0 > a.wait_ns) break;
    }
  };
  if (tid == 0)
    for (int it = 0; it < STAGES && it < nit; ++it) issue(it);

  const int wm = (warp & 1) * 32, wn = (warp >> 1) * 32;
  double acc[4][4][2][2];
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
      for (int c = 0; c < 2; ++c) acc[x][y][c][0] = acc[x][y][c][1] = 0.0;

  const int fr = lane >> 2, fk = lane & 3;
  bool ok = true;
  for (int it = 0; it < nit; ++it) {
    const int s = it % STAGES;
    if (!mbar_wait(&full[s], (it / STAGES) & 1, a.flag, a.wait_ns)) { ok = false; break; }
    const double2* sA = reinterpret_cast<const double2*>(ring + (size_t)s * STAGE_BYTES);
    const double2* sB = sA + (KS / KB) * TM * KB;
#pragma unroll
    for (int q = 0; q < KS / KB; ++q) {
      double are[4], aim[4], bre[4], bim[4], bimn[4];
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const double2 va = sA[(q * TM + wm + 8 * x + fr) * KB + fk];  // A(k, i): A^H = conj
        are[x] = va.x;
        aim[x] = -va.y;
        const double2 vb = sB[(q * TN + wn + 8 * x + fr) * KB + fk];  // B(k, j)
        bre[x] = vb.x;
        bim[x] = vb.y;
        bimn[x] = -vb.y;
      }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) {
          dmma(acc[x][y][0][0], acc[x][y][0][1], are[x], bre[y]);
          dmma(acc[x][y][0][0], acc[x][y][0][1], aim[x], bimn[y]);
          dmma(acc[x][y][1][0], acc[x][y][1][1], are[x], bim[y]);
          dmma(acc[x][y][1][0], acc[x][y][1][1], aim[x], bre[y]);
        }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[s]);
    if (tid == 0 && it + STAGES < nit) {
      // refill this slot once all warps have released it
      if (!mbar_wait(&empty[s], (it / STAGES) & 1, a.flag, a.wait_ns)) { ok = false; break; }
      issue(it + STAGES);
    }
  }
  if (!ok) {
    if (tid == 0) drain();
    return;
  }

  if (a.splitk > 1) {
    cplx* P = a.part + ((size_t)(t - a.tile0) * a.splitk + split) * (TM * TN);
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      const int r = wm + 8 * x + (lane >> 2);
#pragma unroll
      for (int y = 0; y < 4; ++y)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int c = wn + 8 * y + (lane & 3) * 2 + e;
          P[r + TM * c] = cmk(acc[x][y][0][e], acc[x][y][1][e]);
        }
    }
    return;
  }
  cplx* C = z ? a.C1 : a.C0;
  const bool use_beta = (a.beta.x != 0.0 || a.beta.y != 0.0);
#pragma unroll
  for (int x = 0; x < 4; ++x) {
    const int row = i0 + wm + 8 * x + (lane >> 2);
    if (row >= a.m) continue;
#pragma unroll
    for (int y = 0; y < 4; ++y)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = j0 + wn + 8 * y + (lane & 3) * 2 + e;
        if (col >= a.n) continue;
        if (a.uplo == TRI_UPPER && row > col) continue;
        cplx out = cmul(a.alpha, cmk(acc[x][y][0][e], acc[x][y][1][e]));
        cplx* dst = C + row + a.ldc * col;
        if (use_beta) out = cadd(out, cmul(a.beta, *dst));
        *dst = out;
      }
  }
}

// C = alpha * (sum of the split partial sums, in split order) + beta C
__global__ void k_split_reduce(TmaGemmArgs a) {
  const int tl = blockIdx.x;
  const int t = a.tile0 + tl;
  int z, ti, tj;
  tile_coords(a, t, z, ti, tj);
  cplx* C = z ? a.C1 : a.C0;
  const bool use_beta = (a.beta.x != 0.0 || a.beta.y != 0.0);
  for (int e = threadIdx.x; e < TM * TN; e += blockDim.x) {
    const int r = e % TM, c = e / TM;
    const int row = ti * TM + r, col = tj * TN + c;
    if (row >= a.m || col >= a.n) continue;
    if (a.uplo == TRI_UPPER && row > col) continue;
    cplx s = cmk(0.0, 0.0);
    for (int p = 0; p < a.splitk; ++p) s = cadd(s, a.part[((size_t)tl * a.splitk + p) * (TM * TN) + e]);
    cplx out = cmul(a.alpha, s);
    cplx* dst = C + row + a.ldc * col;
    if (use_beta) out = cadd(out, cmul(a.beta, *dst));
    *dst = out;
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

// K x R column-major complex operand (leading dimension ld) as doubles:
// 2K x R, boxes of 8 doubles (4 complex) x 64 rows
int operand_map(CUtensorMap* tm, const cplx* X, int K, int R, long long ld) {
  auto fn = encode_fn();
  if (!fn) {
    excfv_set_error("cuTensorMapEncodeTiled is not available from the driver");
    return EXCFV_ERR_CUDA;
  }
  if ((reinterpret_cast<uintptr_t>(X) & 15) || ld < K) {
    excfv_set_error("TMA GEMM operand not 16-byte aligned or ld < K");
    return EXCFV_ERR_ARG;
  }
  const cuuint64_t dims[2] = {2ull * (cuuint64_t)K, (cuuint64_t)R};
  const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(cplx)};
  const cuuint32_t box[2] = {2u * KB, (cuuint32_t)TM};
  const cuuint32_t estr[2] = {1u, 1u};
  const CUresult r = fn(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<cplx*>(X), dims, strides, box,
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    excfv_set_error("cuTensorMapEncodeTiled failed (%d) for a %d x %d operand", (int)r, K, R);
    return EXCFV_ERR_CUDA;
  }
  return EXCFV_OK;
}

}  // namespace

// C_z = alpha A_z^H B_z + beta C_z for z < batch (<= 2); A_z K x m, B_z K x n
// (column-major, contiguous along K); uplo = TRI_UPPER forms only the upper
// triangle of the square C_z.
int zgemm_cn_tma(excfv_handle* h, int m, int n, int k, cplx alpha, const cplx* const* A, long long lda,
                 const cplx* const* B, long long ldb, cplx beta, cplx* const* C, long long ldc, int batch,
                 int uplo) {
  if (m <= 0 || n <= 0 || batch < 1 || batch > 2 || k <= 0) return EXCFV_ERR_ARG;
  if (uplo == TRI_UPPER && m != n) return EXCFV_ERR_ARG;
  cudaStream_t s = h->stream;
  CUtensorMap mA[2], mB[2];
  for (int zz = 0; zz < 2; ++zz) {
    const int zi = std::min(zz, batch - 1);
    if (int rc = operand_map(&mA[zz], A[zi], k, m, lda)) return rc;
    if (int rc = operand_map(&mB[zz], B[zi], k, n, ldb)) return rc;
  }
  TmaGemmArgs a;
  a.m = m; a.n = n; a.nk = (k + KS - 1) / KS;
  a.alpha = alpha; a.beta = beta;
  a.C0 = C[0]; a.C1 = C[std::min(1, batch - 1)]; a.ldc = ldc;
  a.uplo = uplo;
  a.ntm = (m + TM - 1) / TM; a.ntn = (n + TN - 1) / TN;
  a.tpb = (uplo == TRI_UPPER) ? a.ntm * (a.ntm + 1) / 2 : a.ntm * a.ntn;
  a.flag = h->ws.status + ST_SETUP;
  a.wait_ns = wait_limit_ns();
  const size_t smem = (size_t)STAGES * STAGE_BYTES + 128;
  CUDA_TRY(cudaFuncSetAttribute(k_zgemm_cn_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int per_sm = 0;
  CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_zgemm_cn_tma, GT, smem));
  const int budget = (h->grid_ctas > 0) ? h->grid_ctas : h->nsm;
  const long long R = (long long)std::max(1, per_sm) * budget;  // resident CTAs
  const long long total = (long long)a.tpb * batch;
  const long long full = (total / R) * R;
  if (full > 0) {
    a.tile0 = 0; a.splitk = 1; a.part = nullptr;
    k_zgemm_cn_tma<<<(unsigned)full, GT, smem, s>>>(a, mA[0], mA[1], mB[0], mB[1]); count_launch();
    CUDA_TRY(cudaGetLastError());
  }
  const long long rem = total - full;
  if (rem > 0) {
    const GemmCtx& g = gemm_ctx();
    int sk = (int)std::max(1LL, std::min<long long>(R / rem, a.nk / 4));
    while (sk > 1 && (size_t)rem * sk * TM * TN > g.cap) --sk;
    a.tile0 = (int)full; a.splitk = sk; a.part = (sk > 1) ? g.ws : nullptr;
    k_zgemm_cn_tma<<<(unsigned)(rem * sk), GT, smem, s>>>(a, mA[0], mA[1], mB[0], mB[1]); count_launch();
    CUDA_TRY(cudaGetLastError());
    if (sk > 1) {
      k_split_reduce<<<(unsigned)rem, 256, 0, s>>>(a); count_launch();
      CUDA_TRY(cudaGetLastError());
    }
  }
  return EXCFV_OK;
}
