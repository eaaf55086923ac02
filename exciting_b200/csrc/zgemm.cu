// Complex FP64 GEMM on the FP64 tensor path (DMMA, mma.sync m8n8k4 f64).
//
// C = alpha * op(A) * op(B) + beta * C, column-major, op in {N, C, T},
// strided batch over blockIdx.z, optional triangular structure (see
// ZgemmArgs).  This is the workhorse of the plain-FP64 form: Z = aa A, the
// Cholesky row panels, the triangular inverse, the two-sided reduction
// U^-H H U^-1, the her2k update of the tridiagonal reduction and the
// eigenvector back-transforms (the A^H B products with long K — the setup
// contractions and the Cholesky trailing updates — have their TMA-fed
// kernel in zgemm_tma.cu).  Its grouped form runs many products of
// different sizes in one launch from a device tile list.
//
// tcgen05 has no FP64 kind, so the FP64 tensor instruction on sm_100a is
// DMMA.  A complex product is four real DMMAs on split re/im planes:
//   Cre += Are*Bre + Aim*(-Bim),  Cim += Are*Bim + Aim*Bre.
//
// Tiling: 64x64 complex outputs per CTA, 4 warps (2x2), 32x32 per warp =
// 4x4 m8n8 tiles x {re, im} (the grouped form also has 128x64 tiles, 4x2
// warps); k-tile 8 complex, two shared-memory stages
// with register-staged global loads (loads of tile t+1 overlap the DMMAs of
// tile t).  Shared rows are padded by 4 doubles so that fragment loads
// (lane%4 -> k row, lane/4 -> column) are bank-conflict free.
#include "common.cuh"

#include <algorithm>
#include <vector>

namespace {

constexpr int BM = 64, BN = 64, BK = 8, PAD = 4, NT = 128;
constexpr int LDS = BM + PAD;

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Two-stage operand buffers of a TBM x 64 tile: re/im planes of A (k-major,
// TBM rows) and of B (k-major, 64 columns).
template <int TBM>
struct TileSmem {
  double A[2][2][BK][TBM + PAD];
  double B[2][2][BK][BN + PAD];
};

// One TBM x 64 output tile (rows i0.., columns j0..) of batch entry bz and
// split-K piece split, by 2 TBM threads: (TBM / 32) x 2 warps of 32 x 32.
// TBM = 64 is the shape of every plain launch; the grouped launches also
// have TBM = 128 (eight warps, half the B loads per product).
template <int OPA, int OPB, int TBM>
__device__ __forceinline__ void zgemm_tile(const ZgemmArgs& p, int i0, int j0, long long bz, int split,
                                           TileSmem<TBM>& S) {
  constexpr int TNT = 2 * TBM;            // threads
  constexpr int BPER = BN * BK / TNT;     // B elements each thread stages
  auto& As = S.A;
  auto& Bs = S.B;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  if (p.uplo_c == TRI_UPPER && i0 > j0 + BN - 1) return;
  if (p.uplo_c == TRI_LOWER && j0 > i0 + TBM - 1) return;

  const cplx* __restrict__ A = p.A + bz * p.strideA;
  const cplx* __restrict__ B = p.B + bz * p.strideB;
  cplx* __restrict__ C = p.C + bz * p.strideC;

  int kbeg = 0, kend = p.k - p.kdec * (int)bz;
  if (p.tri_a == TRI_LOWER) kend = min(kend, i0 + TBM);
  if (p.tri_a == TRI_UPPER) kbeg = max(kbeg, i0);
  if (p.tri_b == TRI_UPPER) kend = min(kend, j0 + BN);
  if (p.tri_b == TRI_LOWER) kbeg = max(kbeg, j0);
  kbeg = (kbeg / BK) * BK;
  if (p.splitk > 1 && kend > kbeg) {
    const int span = kend - kbeg;
    const int chunk = ((span + p.splitk - 1) / p.splitk + BK - 1) / BK * BK;
    const int b0 = kbeg + split * chunk;
    kend = min(kend, b0 + chunk);
    kbeg = b0;
  }

  const int wm = (warp % (TBM / 32)) * 32;
  const int wn = (warp / (TBM / 32)) * 32;

  double acc[4][4][2][2];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b)
#pragma unroll
      for (int c = 0; c < 2; ++c) acc[a][b][c][0] = acc[a][b][c][1] = 0.0;

  cplx ra[4], rb[BPER];

  auto load_tile = [&](int kt) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int idx = tid + r * TNT;
      int ii, kk;
      if (OPA == OP_N) { ii = idx & (TBM - 1); kk = idx / TBM; }
      else { kk = idx & 7; ii = idx >> 3; }
      const int gi = i0 + ii, gk = kt + kk;
      bool ok = gi < p.m && gk < kend;
      if (p.tri_a == TRI_LOWER && gk > gi) ok = false;
      if (p.tri_a == TRI_UPPER && gk < gi) ok = false;
      cplx v = cmk(0.0, 0.0);
      if (ok) {
        if (OPA == OP_N) v = A[gi + (long long)gk * p.lda];
        else {
          v = A[gk + (long long)gi * p.lda];
          if (OPA == OP_C) v.y = -v.y;
        }
      }
      ra[r] = v;
    }
#pragma unroll
    for (int r = 0; r < BPER; ++r) {
      const int idx = tid + r * TNT;
      int jj, kk;
      if (OPB == OP_N) { kk = idx & 7; jj = idx >> 3; }
      else { jj = idx & 63; kk = idx >> 6; }
      const int gj = j0 + jj, gk = kt + kk;
      bool ok = gj < p.n && gk < kend;
      if (p.tri_b == TRI_UPPER && gk > gj) ok = false;
      if (p.tri_b == TRI_LOWER && gk < gj) ok = false;
      cplx v = cmk(0.0, 0.0);
      if (ok) {
        if (OPB == OP_N) v = B[gk + (long long)gj * p.ldb];
        else {
          v = B[gj + (long long)gk * p.ldb];
          if (OPB == OP_C) v.y = -v.y;
        }
      }
      rb[r] = v;
    }
  };

  auto store_tile = [&](int st) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int idx = tid + r * TNT;
      int ii, kk;
      if (OPA == OP_N) { ii = idx & (TBM - 1); kk = idx / TBM; }
      else { kk = idx & 7; ii = idx >> 3; }
      As[st][0][kk][ii] = ra[r].x;
      As[st][1][kk][ii] = ra[r].y;
    }
#pragma unroll
    for (int r = 0; r < BPER; ++r) {
      const int idx = tid + r * TNT;
      int jj, kk;
      if (OPB == OP_N) { kk = idx & 7; jj = idx >> 3; }
      else { jj = idx & 63; kk = idx >> 6; }
      Bs[st][0][kk][jj] = rb[r].x;
      Bs[st][1][kk][jj] = rb[r].y;
    }
  };

  if (kbeg < kend) {
    load_tile(kbeg);
    store_tile(0);
    __syncthreads();
    int st = 0;
    for (int kt = kbeg; kt < kend; kt += BK) {
      const bool more = kt + BK < kend;
      if (more) load_tile(kt + BK);
#pragma unroll
      for (int ks = 0; ks < BK; ks += 4) {
        const int kr = ks + (lane & 3);
        const int cc = lane >> 2;
        double are[4], aim[4], bre[4], bim[4], bimn[4];
#pragma unroll
        for (int t = 0; t < 4; ++t) {
          are[t] = As[st][0][kr][wm + t * 8 + cc];
          aim[t] = As[st][1][kr][wm + t * 8 + cc];
          bre[t] = Bs[st][0][kr][wn + t * 8 + cc];
          bim[t] = Bs[st][1][kr][wn + t * 8 + cc];
          bimn[t] = -bim[t];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            dmma(acc[a][b][0][0], acc[a][b][0][1], are[a], bre[b]);
            dmma(acc[a][b][0][0], acc[a][b][0][1], aim[a], bimn[b]);
            dmma(acc[a][b][1][0], acc[a][b][1][1], are[a], bim[b]);
            dmma(acc[a][b][1][0], acc[a][b][1][1], aim[a], bre[b]);
          }
      }
      if (more) store_tile(st ^ 1);
      __syncthreads();
      st ^= 1;
    }
  }

  if (p.splitk > 1) {
    // raw partial sums, leading dimension m, slab (split, batch)
    cplx* P = p.part + ((long long)split * p.batch + bz) * (long long)p.m * p.n;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int row = i0 + wm + a * 8 + (lane >> 2);
      if (row >= p.m) continue;
#pragma unroll
      for (int b = 0; b < 4; ++b)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          const int col = j0 + wn + b * 8 + (lane & 3) * 2 + e;
          if (col >= p.n) continue;
          P[row + (long long)col * p.m] = cmk(acc[a][b][0][e], acc[a][b][1][e]);
        }
    }
    return;
  }
  const bool use_beta = (p.beta.x != 0.0 || p.beta.y != 0.0);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int row = i0 + wm + a * 8 + (lane >> 2);
    if (row >= p.m) continue;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int col = j0 + wn + b * 8 + (lane & 3) * 2 + e;
        if (col >= p.n) continue;
        if (p.uplo_c == TRI_UPPER && row > col) continue;
        if (p.uplo_c == TRI_LOWER && row < col) continue;
        const cplx v = cmk(acc[a][b][0][e], acc[a][b][1][e]);
        cplx out = cmul(p.alpha, v);
        cplx* dst = C + row + (long long)col * p.ldc;
        if (use_beta) out = cadd(out, cmul(p.beta, *dst));
        *dst = out;
      }
    }
  }
}

template <int OPA, int OPB>
__global__ void __launch_bounds__(NT) zgemm_kernel(ZgemmArgs p) {
  __shared__ __align__(16) TileSmem<BM> S;
  // Tiles whose K range grows with the row (tri_a lower) or the column
  // (tri_b upper) index are dispatched heaviest first, so that the last wave
  // holds the short ones.
  const bool rev_x = p.tri_a == TRI_LOWER;
  const bool rev_y = p.tri_b == TRI_UPPER || (p.tri_a == TRI_LOWER && p.uplo_c == TRI_UPPER);
  const int i0 = (rev_x ? (int)(gridDim.x - 1 - blockIdx.x) : (int)blockIdx.x) * BM;
  const int j0 = (rev_y ? (int)(gridDim.y - 1 - blockIdx.y) : (int)blockIdx.y) * BN;
  const long long bz = (p.splitk > 1) ? blockIdx.z / p.splitk : blockIdx.z;
  const int split = (p.splitk > 1) ? (int)(blockIdx.z % p.splitk) : 0;
  zgemm_tile<OPA, OPB, BM>(p, i0, j0, bz, split, S);
}

// Grouped form: one launch over the TBM x 64 tiles of many independent
// products of different sizes.  tiles[b] = (problem, row tile, column tile, -) of CTA b,
// listed by the host heaviest first; probs[problem] is an unbatched product
// (batch 1, no split-K).
template <int OPA, int OPB, int TBM>
__global__ void __launch_bounds__(2 * TBM) zgemm_grouped_kernel(const ZgemmArgs* __restrict__ probs,
                                                                const int4* __restrict__ tiles) {
  extern __shared__ __align__(16) unsigned char gsm[];
  TileSmem<TBM>& S = *reinterpret_cast<TileSmem<TBM>*>(gsm);
  const int4 t = tiles[blockIdx.x];
  const ZgemmArgs p = probs[t.x];
  zgemm_tile<OPA, OPB, TBM>(p, t.y * TBM, t.z * BN, 0, 0, S);
}

// C = alpha * sum_s P_s + beta * C over the split-K slabs (fixed order).
__global__ void k_splitk_reduce(ZgemmArgs p) {
  const long long mn = (long long)p.m * p.n;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= mn * p.batch) return;
  const long long bz = t / mn, e = t % mn;
  const int row = (int)(e % p.m), col = (int)(e / p.m);
  if (p.uplo_c == TRI_UPPER && row > col) return;
  if (p.uplo_c == TRI_LOWER && row < col) return;
  cplx acc = cmk(0.0, 0.0);
  for (int sp = 0; sp < p.splitk; ++sp) acc = cadd(acc, p.part[((long long)sp * p.batch + bz) * mn + e]);
  cplx* dst = p.C + bz * p.strideC + row + (long long)col * p.ldc;
  cplx out = cmul(p.alpha, acc);
  if (p.beta.x != 0.0 || p.beta.y != 0.0) out = cadd(out, cmul(p.beta, *dst));
  *dst = out;
}

template <int OPA, int OPB>
int launch(cudaStream_t s, const ZgemmArgs& a) {
  dim3 grid((a.m + BM - 1) / BM, (a.n + BN - 1) / BN, a.batch * max(1, a.splitk));
  zgemm_kernel<OPA, OPB><<<grid, NT, 0, s>>>(a); count_launch();
  if (a.splitk > 1) {
    const long long tot = (long long)a.m * a.n * a.batch;
    k_splitk_reduce<<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(a); count_launch();
  }
  return 0;
}

thread_local GemmCtx g_ctx;

}  // namespace

void gemm_ctx_set(const GemmCtx& c) { g_ctx = c; }
const GemmCtx& gemm_ctx() { return g_ctx; }

int zgemm(cudaStream_t s, int opA, int opB, const ZgemmArgs& a_in) {
  ZgemmArgs a = a_in;
  if (a.m <= 0 || a.n <= 0 || a.batch <= 0) return 0;
  if (a.k <= 0 && a.beta.x == 1.0 && a.beta.y == 0.0) return 0;
  // split-K when the output has too few tiles to fill the GPU and K is long
  a.splitk = 1;
  a.part = nullptr;
  {
    const long long tm = (a.m + BM - 1) / BM, tn = (a.n + BN - 1) / BN;
    long long tiles = tm * tn * a.batch;
    if (a.uplo_c != TRI_NONE && a.m == a.n) tiles = (tiles + tm * a.batch) / 2;
    const int nsm = g_ctx.nsm;
    if (g_ctx.ws && tiles < nsm && a.k >= 256) {
      int sk = (int)((2 * nsm + tiles - 1) / tiles);
      sk = min(sk, a.k / 128);
      sk = min(sk, 32);
      const long long need = (long long)a.m * a.n * a.batch;
      while (sk > 1 && (size_t)(need * sk) > g_ctx.cap) --sk;
      if (sk > 1) {
        a.splitk = sk;
        a.part = g_ctx.ws;
      }
    }
  }
  switch (opA * 3 + opB) {
    case OP_N * 3 + OP_N: return launch<OP_N, OP_N>(s, a);
    case OP_N * 3 + OP_C: return launch<OP_N, OP_C>(s, a);
    case OP_N * 3 + OP_T: return launch<OP_N, OP_T>(s, a);
    case OP_C * 3 + OP_N: return launch<OP_C, OP_N>(s, a);
    case OP_C * 3 + OP_C: return launch<OP_C, OP_C>(s, a);
    case OP_C * 3 + OP_T: return launch<OP_C, OP_T>(s, a);
    case OP_T * 3 + OP_N: return launch<OP_T, OP_N>(s, a);
    case OP_T * 3 + OP_C: return launch<OP_T, OP_C>(s, a);
    case OP_T * 3 + OP_T: return launch<OP_T, OP_T>(s, a);
  }
  return EXCFV_ERR_ARG;
}

// Length of the K range tile (ti, tj) of p runs over (the same rules as
// zgemm_tile), or -1 for a tile outside the written triangle of C.
static long long group_tile_k(const ZgemmArgs& p, int ti, int tj, int tbm) {
  const int i0 = ti * tbm, j0 = tj * BN;
  if (p.uplo_c == TRI_UPPER && i0 > j0 + BN - 1) return -1;
  if (p.uplo_c == TRI_LOWER && j0 > i0 + tbm - 1) return -1;
  int kbeg = 0, kend = p.k;
  if (p.tri_a == TRI_LOWER) kend = std::min(kend, i0 + tbm);
  if (p.tri_a == TRI_UPPER) kbeg = std::max(kbeg, i0);
  if (p.tri_b == TRI_UPPER) kend = std::min(kend, j0 + BN);
  if (p.tri_b == TRI_LOWER) kbeg = std::max(kbeg, j0);
  return std::max(0, kend - (kbeg / BK) * BK);
}

void zgemm_group_add(const ZgemmArgs& p_in, std::vector<ZgemmArgs>& probs, std::vector<GroupTile>& tiles,
                     int tbm) {
  ZgemmArgs p = p_in;
  if (p.m <= 0 || p.n <= 0) return;
  p.batch = 1; p.splitk = 1; p.part = nullptr; p.kdec = 0;
  p.strideA = p.strideB = p.strideC = 0;
  const int pi = (int)probs.size();
  probs.push_back(p);
  const int tm = (p.m + tbm - 1) / tbm, tn = (p.n + BN - 1) / BN;
  for (int tj = 0; tj < tn; ++tj)
    for (int ti = 0; ti < tm; ++ti) {
      const long long kl = group_tile_k(p, ti, tj, tbm);
      if (kl >= 0) tiles.push_back(GroupTile{pi, ti, tj, kl});
    }
}

void zgemm_group_order(std::vector<GroupTile>& tiles, size_t from) {
  std::stable_sort(tiles.begin() + (long)from, tiles.end(),
                   [](const GroupTile& a, const GroupTile& b) { return a.klen > b.klen; });
}

template <int TBM>
static int launch_grouped(cudaStream_t s, int opA, int opB, const ZgemmArgs* d_probs, const int4* d_tiles,
                          int ntiles) {
  const int smem = (int)sizeof(TileSmem<TBM>);
  switch (opA * 3 + opB) {
#define EXCFV_GROUPED_CASE(A_, B_)                                                               \
  case A_ * 3 + B_:                                                                              \
    if (cudaFuncSetAttribute(zgemm_grouped_kernel<A_, B_, TBM>,                                  \
                             cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)  \
      return EXCFV_ERR_CUDA;                                                                     \
    zgemm_grouped_kernel<A_, B_, TBM><<<ntiles, 2 * TBM, smem, s>>>(d_probs, d_tiles);          \
    count_launch();                                                                              \
    return cudaGetLastError() == cudaSuccess ? 0 : EXCFV_ERR_CUDA;
    EXCFV_GROUPED_CASE(OP_N, OP_N)
    EXCFV_GROUPED_CASE(OP_N, OP_C)
    EXCFV_GROUPED_CASE(OP_C, OP_N)
    EXCFV_GROUPED_CASE(OP_C, OP_C)
#undef EXCFV_GROUPED_CASE
  }
  return EXCFV_ERR_ARG;
}

int zgemm_grouped(cudaStream_t s, int opA, int opB, const ZgemmArgs* d_probs, const int4* d_tiles, int ntiles,
                  int tbm) {
  if (ntiles <= 0) return 0;
  if (tbm == 128) return launch_grouped<128>(s, opA, opB, d_probs, d_tiles, ntiles);
  if (tbm == 64) return launch_grouped<64>(s, opA, opB, d_probs, d_tiles, ntiles);
  return EXCFV_ERR_ARG;
}

int zgemm1(cudaStream_t s, int opA, int opB, int m, int n, int k, cplx alpha,
           const cplx* A, long long lda, const cplx* B, long long ldb, cplx beta,
           cplx* C, long long ldc, int uplo_c, int tri_a, int tri_b) {
  ZgemmArgs a;
  a.m = m; a.n = n; a.k = k; a.alpha = alpha; a.beta = beta;
  a.A = A; a.lda = lda; a.strideA = 0;
  a.B = B; a.ldb = ldb; a.strideB = 0;
  a.C = C; a.ldc = ldc; a.strideC = 0;
  a.batch = 1; a.uplo_c = uplo_c; a.tri_a = tri_a; a.tri_b = tri_b;
  a.splitk = 1; a.part = nullptr; a.kdec = 0;
  return zgemm(s, opA, opB, a);
}
