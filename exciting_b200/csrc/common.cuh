// Common definitions for libexcfv (first-variational LAPW+lo on sm_100a).
//
// Complex numbers are double2 {re, im}: the same bytes as Fortran complex(8),
// so arrays cross the C ABI without conversion.  All matrices are
// column-major with an explicit leading dimension, as in the Fortran caller.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>
#include <vector>

typedef double2 cplx;

#define EXCFV_HD __host__ __device__ __forceinline__

EXCFV_HD cplx cmk(double r, double i) { cplx z; z.x = r; z.y = i; return z; }
EXCFV_HD cplx cadd(cplx a, cplx b) { return cmk(a.x + b.x, a.y + b.y); }
EXCFV_HD cplx csub(cplx a, cplx b) { return cmk(a.x - b.x, a.y - b.y); }
EXCFV_HD cplx cmul(cplx a, cplx b) { return cmk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
// conj(a) * b
EXCFV_HD cplx cmulc(cplx a, cplx b) { return cmk(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x); }
EXCFV_HD cplx cconj(cplx a) { return cmk(a.x, -a.y); }
EXCFV_HD cplx cscale(cplx a, double s) { return cmk(a.x * s, a.y * s); }
EXCFV_HD double cabs2(cplx a) { return a.x * a.x + a.y * a.y; }

// Status codes shared with include/excfv.h.
#define EXCFV_OK 0
#define EXCFV_ERR_ARG (-1)
#define EXCFV_ERR_UNSUPPORTED (-2)
#define EXCFV_ERR_CUDA (-3)
#define EXCFV_ERR_ALLOC (-4)
#define EXCFV_ERR_STATE (-5)
#define EXCFV_ERR_TIMEOUT (-6)
#define EXCFV_ERR_NOCONV (-7)

// Device-side status word written by kernels (0 = fine).  Layout of the
// per-handle status block (int32):
//   [0] potrf: first non-positive pivot, 1-based (0 = none)
//   [1] grid barrier timeout count
//   [2] stein: number of eigenvectors that failed to converge
//   [3] stebz: bisection did not converge for some eigenvalue
//   [4] refinement: cluster above the precision form's limit
//   [5] setup: a bounded wait of the setup contraction gave up (cleared by the
//       setup, not by the eigensolve)
enum { ST_POTRF = 0, ST_BARRIER = 1, ST_STEIN = 2, ST_STEBZ = 3, ST_REFINE = 4, ST_SETUP = 5, ST_NWORDS = 8 };

#define CUDA_TRY(expr)                                                          \
  do {                                                                          \
    cudaError_t _e = (expr);                                                    \
    if (_e != cudaSuccess) {                                                    \
      excfv_set_error("%s:%d: %s: %s", __FILE__, __LINE__, #expr,               \
                      cudaGetErrorString(_e));                                  \
      return EXCFV_ERR_CUDA;                                                    \
    }                                                                           \
  } while (0)

void excfv_set_error(const char* fmt, ...);
// Time limit of every bounded spin-wait in the kernels (default 2 s) and a
// one-shot planted stall: when armed, the next reduction's first wait gets a
// target that nothing reaches, so the limit runs out (a test aid; see
// excfv_test_set_wait_limit in include/excfv.h).
long long wait_limit_ns();
bool take_planted_stall();
// process-wide count of kernel launches made by this library
void count_launch(int n = 1);

// ---------------------------------------------------------------------------
// complex FP64 GEMM on the DMMA (mma.sync m8n8k4 f64) tensor path
// ---------------------------------------------------------------------------
enum { OP_N = 0, OP_C = 1, OP_T = 2 };
enum { TRI_NONE = 0, TRI_LOWER = 1, TRI_UPPER = 2 };

struct ZgemmArgs {
  int m, n, k;
  cplx alpha, beta;
  const cplx* A; long long lda, strideA;
  const cplx* B; long long ldb, strideB;
  cplx* C; long long ldc, strideC;
  int batch;
  // Structure hints.  uplo_c: write only C(i,j) with i<=j (TRI_UPPER) or
  // i>=j (TRI_LOWER).  tri_a / tri_b: op(A) / op(B) is triangular; elements
  // in the other triangle are treated as zero (never loaded) and whole
  // k-tiles outside the triangle are skipped.
  int uplo_c, tri_a, tri_b;
  // split-K: the K range of every tile is cut into splitk pieces whose
  // partial products go to part (splitk * batch * m * n) and are summed in a
  // fixed order by a second kernel (deterministic).  Set by zgemm().
  int splitk;
  cplx* part;
  // batch z uses K = k - kdec * z (0 = the same K for every batch entry)
  int kdec;
};

// Scratch for split-K partial products, owned by the calling handle and made
// current for the calling thread by the entry points (a handle is used by one
// thread at a time).
struct GemmCtx {
  cplx* ws = nullptr;
  size_t cap = 0;  // complex elements
  int nsm = 148;
};
void gemm_ctx_set(const GemmCtx& c);
const GemmCtx& gemm_ctx();

int zgemm(cudaStream_t s, int opA, int opB, const ZgemmArgs& a);

// Grouped products: many unbatched products of different sizes in one
// launch, one CTA per output tile.  The host appends each product and
// its tiles to shared lists (zgemm_group_add; tile entries carry the global
// product index), orders one launch's tiles heaviest first
// (zgemm_group_order), uploads both lists and launches zgemm_grouped with the
// device copies, the tiles as int4 {product, row tile, column tile, 0}.
struct GroupTile {
  int prob, ti, tj;
  long long klen;  // K range of the tile: the ordering key, not uploaded
};
// Tile shapes: tbm x 64 outputs per CTA, tbm = 64 or 128.
void zgemm_group_add(const ZgemmArgs& p, std::vector<ZgemmArgs>& probs, std::vector<GroupTile>& tiles,
                     int tbm);
void zgemm_group_order(std::vector<GroupTile>& tiles, size_t from);
int zgemm_grouped(cudaStream_t s, int opA, int opB, const ZgemmArgs* d_probs, const int4* d_tiles, int ntiles,
                  int tbm);

// convenience: single (non-batched) product
int zgemm1(cudaStream_t s, int opA, int opB, int m, int n, int k, cplx alpha,
           const cplx* A, long long lda, const cplx* B, long long ldb, cplx beta,
           cplx* C, long long ldc, int uplo_c = TRI_NONE, int tri_a = TRI_NONE,
           int tri_b = TRI_NONE);
