// Generalized Hermitian eigensolve H x = e O x for the lowest k states
// (ZHEGVX(1,'V','I','U'), src/src_eigensystem/modfvsystem.f90:691-693).
//
//   O = U^H U                      potrf_upper      (ZPOTRF)
//   Ui = U^-1                      trtri_upper
//   C = Ui^H (H Ui)                two GEMMs skipping the zero triangles (ZHEGST)
//   C = Q T Q^H                    tridiag_reduce   (ZHETRD)
//   T y = e y, lowest k            tridiag_eig      (DSTEBZ + DSTEIN)
//   Z = orth(y)                    Cholesky-QR on the k vectors
//   Z <- Q Z                       block reflectors (I - V Tf V^H), GEMMs (ZUNMTR)
//   X = Ui Z                       one GEMM (ZTRSM)
#include <algorithm>

#include "handle.cuh"

int potrf_upper(excfv_handle* h, int n, cplx* O, cplx* Ui, long long ld);
int trtri_upper(excfv_handle* h, int n, const cplx* U, cplx* Ui, long long ld, cplx* scratch);
int tridiag_reduce(excfv_handle* h, int n, cplx* C, long long ld);
int tridiag_nb();
int tridiag_eig(excfv_handle* h, int n, int k, double abstol, const double* d, const double* e,
                double* w, cplx* Z, long long ldz, double* scratch, int* iscratch);
int mirror_upper(cudaStream_t s, int n, cplx* M, long long ld);
int tridiag_reduce_f32(excfv_handle* h, int n, float2* C, long long ld);

namespace {

constexpr int NBQ = 64;   // reflectors per block of k_larft's recurrence
constexpr int NBW = 256;  // reflectors per block of the back-transform
constexpr long long WST = (long long)NBW * (NBW + 1);  // storage stride of one NBW block
constexpr int LT = 256;

// The Gram matrices G = V^H V and the factors T of the NBW-wide blocks are
// stored with leading dimension NBW and a block stride of NBW (NBW + 1)
// elements: element (r, c) of block B at B NBW (NBW + 1) + r + NBW c.  The
// diagonal sub-block starting at reflector g (global index) then sits at
// g (NBW + 1), whichever block it belongs to, so every level of the T merge
// below is one batched GEMM with a uniform stride.

// Triangular factor of the block reflector H_p ... H_{p+nb-1} = I - V T V^H
// (forward, columnwise: T(i,i) = tau_i, T(0:i,i) = -tau_i T(0:i,0:i) G(0:i,i)
// with G = V^H V), for the NBQ-wide diagonal sub-blocks of the NBW blocks.
// One CTA per sub-block; G and T live in shared memory, four threads share
// each row of the triangular product.
__global__ void __launch_bounds__(LT) k_larft(int n, const cplx* Gbig, const cplx* tau, cplx* Tbig) {
  extern __shared__ __align__(16) unsigned char dsm[];
  cplx (*G)[NBQ + 1] = reinterpret_cast<cplx (*)[NBQ + 1]>(dsm);
  cplx (*T)[NBQ + 1] = reinterpret_cast<cplx (*)[NBQ + 1]>(dsm + sizeof(cplx) * NBQ * (NBQ + 1));
  const int blk = blockIdx.x;
  const int p = blk * NBQ;
  const int nb = min(NBQ, n - 1 - p);
  if (nb <= 0) return;
  const int tid = threadIdx.x;
  const cplx* Gb = Gbig + (size_t)p * (NBW + 1);
  for (int t = tid; t < NBQ * NBQ; t += LT) {
    const int r = t % NBQ, c = t / NBQ;
    G[r][c] = Gb[r + (size_t)NBW * c];
    T[r][c] = cmk(0.0, 0.0);
  }
  __syncthreads();
  if (tid == 0) T[0][0] = tau[p];
  __syncthreads();
  const int row = tid >> 2, sub = tid & 3;
  for (int i = 1; i < nb; ++i) {
    const cplx ti = tau[p + i];
    cplx val = cmk(0.0, 0.0);
    if (row < i)
      for (int q = row + sub; q < i; q += 4) val = cadd(val, cmul(T[row][q], G[q][i]));
    val.x += __shfl_xor_sync(0xffffffffu, val.x, 1);
    val.y += __shfl_xor_sync(0xffffffffu, val.y, 1);
    val.x += __shfl_xor_sync(0xffffffffu, val.x, 2);
    val.y += __shfl_xor_sync(0xffffffffu, val.y, 2);
    __syncthreads();
    if (row < i && sub == 0) T[row][i] = cmul(cmk(-ti.x, -ti.y), val);
    if (tid == 0) T[i][i] = ti;
    __syncthreads();
  }
  cplx* out = Tbig + (size_t)p * (NBW + 1);
  for (int t = tid; t < NBQ * NBQ; t += LT) out[t % NBQ + (size_t)NBW * (t / NBQ)] = T[t % NBQ][t / NBQ];
}

// n x n FP64 (leading dimension ldi) -> complex64 (leading dimension ldo)
__global__ void k_to_f32(int n, const cplx* __restrict__ in, long long ldi, float2* __restrict__ out,
                         long long ldo) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r >= n) return;
  const cplx v = in[r + ldi * c];
  out[r + ldo * c] = make_float2((float)v.x, (float)v.y);
}

// reflectors (below the diagonal) of an n x n complex64 matrix -> FP64
__global__ void k_lower_to_f64(int n, const float2* __restrict__ in, long long ldi,
                               cplx* __restrict__ out, long long ldo) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  const int c = blockIdx.y;
  if (r >= n || r <= c) return;
  const float2 v = in[r + ldi * c];
  out[r + ldo * c] = cmk((double)v.x, (double)v.y);
}

// ---------------------------------------------------------------------------
// Precision form: refinement of the k' x k' Rayleigh-Ritz matrix Hk = X0^H C X0.
// X0 comes from the complex64 reduction, so Hk = diag + E with |E| at the
// FP32 level.  States whose Rayleigh quotients lie within tau = max|E| / RR_RHO
// of each other form clusters (contiguous in sorted order), each diagonalised
// exactly by complex Jacobi rotations; between clusters every coupling is at
// most RR_RHO times the gap, and second-order perturbation theory gives the
// eigenvalues (error ~ |E| RR_RHO^2) and first-order the vectors, which a
// Cholesky-QR pass re-orthonormalises afterwards.
// ---------------------------------------------------------------------------
constexpr double RR_RHO = 1e-3;
constexpr int RR_MAXC = 64;  // largest cluster diagonalised by the Jacobi kernel

struct RRScratch {
  double* D;      // kx: Rayleigh quotients
  double* lam;    // kx: refined eigenvalues
  int* perm;      // kx: sorted position -> state
  int* cid;       // kx: cluster of each state
  int* cstart;    // kx: first sorted position of each cluster
  int* csize;     // kx
  int* sel;       // k : state of the r-th lowest refined eigenvalue
  int* nclust;    // 1
};

__device__ __forceinline__ double cabsd(cplx a) { return hypot(a.x, a.y); }

// Sort key of a total order on doubles: NaN ranks as +inf, ties go by index,
// so ranks computed by counting form a permutation whatever the values (a
// failed earlier stage may leave NaN here; the indices derived from the ranks
// must stay in range).
__device__ __forceinline__ double rank_key(double v) { return isnan(v) ? INFINITY : v; }

__device__ __forceinline__ double block_max(double v, double* red) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  __syncthreads();
  if (l == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = (l < (int)(blockDim.x >> 5)) ? red[l] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    if (l == 0) red[0] = v;
  }
  __syncthreads();
  return red[0];
}

// One CTA of 1024 threads: Rayleigh quotients, max coupling, sort, clusters.
__global__ void __launch_bounds__(1024) k_rr_clusters(int kx, const cplx* __restrict__ Hk, RRScratch s) {
  __shared__ double red[32];
  __shared__ int wsum[32];
  const int tid = threadIdx.x;
  double emax = 0.0, dmax = 0.0;
  for (int i = tid; i < kx; i += blockDim.x) {
    const double d = rank_key(Hk[i + (long long)kx * i].x);
    s.D[i] = d;
    dmax = fmax(dmax, fabs(d));
  }
  for (long long e = tid; e < (long long)kx * kx; e += blockDim.x) {
    const int i = (int)(e % kx), j = (int)(e / kx);
    if (i != j) emax = fmax(emax, cabsd(Hk[e]));
  }
  emax = block_max(emax, red);
  dmax = block_max(dmax, red);
  const double tau = fmax(emax / RR_RHO, 64.0 * 2.220446049250313e-16 * dmax);
  // rank of each state in ascending order (ties by index)
  for (int i = tid; i < kx; i += blockDim.x) {
    const double di = s.D[i];
    int r = 0;
    for (int j = 0; j < kx; ++j) {
      const double dj = s.D[j];
      r += (dj < di) || (dj == di && j < i);
    }
    s.perm[r] = i;
  }
  __syncthreads();
  // cluster ids: inclusive scan of the start flags over sorted positions
  const int per = (kx + blockDim.x - 1) / blockDim.x;
  const int r0 = tid * per;
  int cnt = 0;
  for (int r = r0; r < min(kx, r0 + per); ++r)
    cnt += (r == 0) || (s.D[s.perm[r]] - s.D[s.perm[r - 1]] > tau);
  int incl = cnt;
  const int lane = tid & 31, w = tid >> 5;
  for (int o = 1; o < 32; o <<= 1) {
    const int v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) wsum[w] = incl;
  __syncthreads();
  if (w == 0) {
    int v = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += u;
    }
    wsum[lane] = v;
  }
  __syncthreads();
  int c = (w > 0 ? wsum[w - 1] : 0) + incl - cnt - 1;  // cluster before this thread's range
  for (int r = r0; r < min(kx, r0 + per); ++r) {
    if ((r == 0) || (s.D[s.perm[r]] - s.D[s.perm[r - 1]] > tau)) {
      ++c;
      s.cstart[c] = r;
    }
    s.cid[s.perm[r]] = c;
  }
  if (tid == blockDim.x - 1) *s.nclust = wsum[(blockDim.x >> 5) - 1];
  __syncthreads();
  for (int r = tid; r < kx; r += blockDim.x) {
    const int cc = s.cid[s.perm[r]];
    if (r == s.cstart[cc]) {
      int e = r + 1;
      while (e < kx && s.cid[s.perm[e]] == cc) ++e;
      s.csize[cc] = e - r;
    }
  }
}

// Cyclic Jacobi on the Hermitian m x m matrix A (column-major, ld m); V gets
// the eigenvectors.  Rotation on (p, q): with A(p,q) = g e^{i phi} and
// t = tan(theta) from tau = (A(q,q) - A(p,p)) / 2g, U = [[c, s], [-s e^{-i phi},
// c e^{-i phi}]]; A <- U^H A U, V <- V U.
__device__ void jacobi_herm(int m, cplx* A, cplx* V) {
  for (int i = 0; i < m * m; ++i) V[i] = cmk(0.0, 0.0);
  for (int i = 0; i < m; ++i) V[i + m * i] = cmk(1.0, 0.0);
  for (int sweep = 0; sweep < 40; ++sweep) {
    double off = 0.0, sc = 0.0;
    for (int q = 0; q < m; ++q) {
      sc = fmax(sc, fabs(A[q + m * q].x));
      for (int p = 0; p < q; ++p) off = fmax(off, cabsd(A[p + m * q]));
    }
    if (off <= 1e-15 * sc || off == 0.0) break;
    for (int p = 0; p < m; ++p)
      for (int q = p + 1; q < m; ++q) {
        const cplx apq = A[p + m * q];
        const double g = cabsd(apq);
        if (g <= 1e-300) continue;
        const cplx ph = cmk(apq.x / g, apq.y / g);
        const double tu = (A[q + m * q].x - A[p + m * p].x) / (2.0 * g);
        const double t = (tu >= 0.0 ? 1.0 : -1.0) / (fabs(tu) + sqrt(1.0 + tu * tu));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = t * cs;
        const cplx phc = cmk(ph.x, -ph.y);
        const cplx up0 = cmk(cs, 0.0), up1 = cscale(phc, -sn);
        const cplx uq0 = cmk(sn, 0.0), uq1 = cscale(phc, cs);
        for (int k = 0; k < m; ++k) {
          const cplx akp = A[k + m * p], akq = A[k + m * q];
          A[k + m * p] = cadd(cmul(akp, up0), cmul(akq, up1));
          A[k + m * q] = cadd(cmul(akp, uq0), cmul(akq, uq1));
        }
        for (int k = 0; k < m; ++k) {
          const cplx apk = A[p + m * k], aqk = A[q + m * k];
          A[p + m * k] = cadd(cmulc(up0, apk), cmulc(up1, aqk));
          A[q + m * k] = cadd(cmulc(uq0, apk), cmulc(uq1, aqk));
        }
        for (int k = 0; k < m; ++k) {
          const cplx vkp = V[k + m * p], vkq = V[k + m * q];
          V[k + m * p] = cadd(cmul(vkp, up0), cmul(vkq, up1));
          V[k + m * q] = cadd(cmul(vkp, uq0), cmul(vkq, uq1));
        }
      }
  }
}

// One thread per cluster: Q (kx x kx, zeroed) gets the cluster rotations on
// the cluster's own state indices.  Scratch: the cluster at sorted start r
// uses A at sa + r kx and V at sv + r kx (m^2 <= (kx - r) kx entries).
__global__ void k_rr_jacobi(int kx, const cplx* __restrict__ Hk, RRScratch s, cplx* __restrict__ Q,
                            cplx* __restrict__ sa, cplx* __restrict__ sv, int* status) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= *s.nclust) return;
  const int r0 = s.cstart[c], m = s.csize[c];
  if (m == 1) {
    const int i = s.perm[r0];
    Q[i + (long long)kx * i] = cmk(1.0, 0.0);
    return;
  }
  if (m > RR_MAXC) {
    atomicMax(&status[ST_REFINE], m);
    for (int p = 0; p < m; ++p) {
      const int i = s.perm[r0 + p];
      Q[i + (long long)kx * i] = cmk(1.0, 0.0);
    }
    return;
  }
  cplx* A = sa + (long long)r0 * kx;
  cplx* V = sv + (long long)r0 * kx;
  for (int q = 0; q < m; ++q)
    for (int p = 0; p < m; ++p)
      A[p + m * q] = Hk[s.perm[r0 + p] + (long long)kx * s.perm[r0 + q]];
  jacobi_herm(m, A, V);
  for (int q = 0; q < m; ++q)
    for (int p = 0; p < m; ++p)
      Q[s.perm[r0 + p] + (long long)kx * s.perm[r0 + q]] = V[p + m * q];
}

// One warp per state a of the rotated basis (Hp = Q^H Hk Q): second-order
// eigenvalue and first-order vector T(:, a) from the couplings to other clusters.
__global__ void k_rr_perturb(int kx, const cplx* __restrict__ Hp, RRScratch s, cplx* __restrict__ T) {
  const int a = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (a >= kx) return;
  const double mua = Hp[a + (long long)kx * a].x;
  const int ca = s.cid[a];
  double corr = 0.0;
  for (int b = lane; b < kx; b += 32) {
    cplx t = cmk(b == a ? 1.0 : 0.0, 0.0);
    if (s.cid[b] != ca) {
      const cplx hba = Hp[b + (long long)kx * a];
      const double d = mua - Hp[b + (long long)kx * b].x;
      corr += (hba.x * hba.x + hba.y * hba.y) / d;
      t = cmk(hba.x / d, hba.y / d);
    }
    T[b + (long long)kx * a] = t;
  }
  for (int o = 16; o > 0; o >>= 1) corr += __shfl_xor_sync(0xffffffffu, corr, o);
  if (lane == 0) s.lam[a] = mua + corr;
}

// One CTA: the k lowest refined eigenvalues (ascending) and their states.
__global__ void __launch_bounds__(1024) k_rr_select(int kx, int k, RRScratch s, double* w) {
  for (int a = threadIdx.x; a < kx; a += blockDim.x) {
    const double la = rank_key(s.lam[a]);
    int r = 0;
    for (int b = 0; b < kx; ++b) {
      const double lb = rank_key(s.lam[b]);
      r += (lb < la) || (lb == la && b < a);
    }
    if (r < k) {
      s.sel[r] = a;
      w[r] = la;
    }
  }
}

// M (m x m, leading dimension ld) -= I
__global__ void k_sub_identity(int m, cplx* M, long long ld) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) M[i + ld * i].x -= 1.0;
}

// Tsel(:, r) = T(:, sel[r])
__global__ void k_rr_gather(int kx, int k, const cplx* __restrict__ T, const int* __restrict__ sel,
                            cplx* __restrict__ Ts) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int r = blockIdx.y;
  if (b < kx && r < k) Ts[b + (long long)kx * r] = T[b + (long long)kx * sel[r]];
}

__global__ void k_copy_eval(int k, const double* w, double* out) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < k) out[j] = w[j];
}

}  // namespace

// Z (n x k) <- Q Z with Q = H_0 ... H_{n-1-off}: reflector c stored in
// column c of C from row c + off down, unit entry explicit (off = 1 for the
// one-stage reduction, the bandwidth for stage 1 of the two-stage one).
size_t backtr_factor_elems(int nrefl) {
  const long long nblk = (nrefl + NBW - 1) / NBW;
  return (size_t)(2 * nblk * WST + nblk * (NBW / 2) * (NBW / 2) + NBW);
}

int apply_q(excfv_handle* h, int n, int k, const cplx* C, long long ld, cplx* Z, long long ldz,
            int off) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const int nrefl = n - off;
  if (nrefl < 1) return EXCFV_OK;
  const int nblk = (nrefl + NBW - 1) / NBW;
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  cplx* Tbig = ws.Tf;
  cplx* Gbig = ws.Tf + (size_t)nblk * WST;
  cplx* Xm = Gbig + (size_t)nblk * WST;  // scratch of the T merge
  const int nfull = nrefl / NBW;
  // a partial last block: the parts past nrefl must read as zero (identity
  // reflectors) in the T recurrence and the merge
  if (nfull < nblk) {
    CUDA_TRY(cudaMemsetAsync(Tbig + (size_t)nfull * WST, 0, sizeof(cplx) * WST, s));
    CUDA_TRY(cudaMemsetAsync(Gbig + (size_t)nfull * WST, 0, sizeof(cplx) * WST, s));
  }
  // Gram matrices G_B = V_B^H V_B (upper): the full blocks in one batched
  // GEMM (K shrinks by NBW from block to block), the last partial block alone
  if (nfull > 0) {
    ZgemmArgs g;
    g.m = NBW; g.n = NBW; g.k = n - off; g.kdec = NBW;
    g.alpha = one; g.beta = zero;
    g.A = C + off; g.lda = ld; g.strideA = (long long)NBW * (ld + 1);
    g.B = C + off; g.ldb = ld; g.strideB = (long long)NBW * (ld + 1);
    g.C = Gbig; g.ldc = NBW; g.strideC = WST;
    g.batch = nfull; g.uplo_c = TRI_UPPER; g.tri_a = TRI_UPPER; g.tri_b = TRI_LOWER;
    g.splitk = 1; g.part = nullptr;
    int rc = zgemm(s, OP_C, OP_N, g);
    if (rc) return rc;
  }
  if (nfull < nblk) {
    const int p = nfull * NBW;
    const int nb = nrefl - p, m = n - p - off;
    const cplx* V = C + (p + off) + ld * p;
    int rc = zgemm1(s, OP_C, OP_N, nb, nb, m, one, V, ld, V, ld, zero, Gbig + (size_t)nfull * WST, NBW,
                    TRI_UPPER, TRI_UPPER, TRI_LOWER);
    if (rc) return rc;
  }
  // T of the NBQ-wide diagonal sub-blocks, then merged level by level:
  //   T([V1 V2]) = [[T1, -T1 (V1^H V2) T2], [0, T2]]
  // (all pairs of one level in two batched GEMMs over the uniform stride)
  const int smem = (int)(2 * sizeof(cplx) * NBQ * (NBQ + 1));
  CUDA_TRY(cudaFuncSetAttribute(k_larft, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  k_larft<<<nblk * (NBW / NBQ), LT, smem, s>>>(nrefl + 1, Gbig, ws.tau, Tbig); count_launch();
  CUDA_TRY(cudaGetLastError());
  for (int bs = NBQ; bs < NBW; bs *= 2) {
    const long long step = 2LL * bs * (NBW + 1);
    const int npair = nblk * (NBW / (2 * bs));
    ZgemmArgs g;
    g.m = bs; g.n = bs; g.k = bs; g.kdec = 0; g.alpha = one; g.beta = zero;
    g.A = Gbig + (size_t)bs * NBW; g.lda = NBW; g.strideA = step;         // G12
    g.B = Tbig + (size_t)bs * (NBW + 1); g.ldb = NBW; g.strideB = step;  // T2
    g.C = Xm; g.ldc = bs; g.strideC = (long long)bs * bs;                 // G12 T2
    g.batch = npair; g.uplo_c = TRI_NONE; g.tri_a = TRI_NONE; g.tri_b = TRI_UPPER;
    g.splitk = 1; g.part = nullptr;
    int rc = zgemm(s, OP_N, OP_N, g);
    if (rc) return rc;
    g.alpha = mone;
    g.A = Tbig; g.strideA = step;                                         // T1
    g.B = Xm; g.ldb = bs; g.strideB = (long long)bs * bs;
    g.C = Tbig + (size_t)bs * NBW; g.ldc = NBW; g.strideC = step;         // T12
    g.tri_a = TRI_UPPER; g.tri_b = TRI_NONE;
    rc = zgemm(s, OP_N, OP_N, g);
    if (rc) return rc;
  }
  cplx* X1 = ws.Xs;
  cplx* X2 = ws.Xs + (size_t)NBW * ws.kmax;
  for (int b = nblk - 1; b >= 0; --b) {
    const int p = b * NBW;
    const int nb = min(NBW, nrefl - p);
    const int m = n - p - off;
    const cplx* V = C + (p + off) + ld * p;
    cplx* Zs = Z + (p + off);
    int rc = zgemm1(s, OP_C, OP_N, nb, k, m, one, V, ld, Zs, ldz, zero, X1, NBW, TRI_NONE,
                    TRI_UPPER, TRI_NONE);
    if (rc) return rc;
    rc = zgemm1(s, OP_N, OP_N, nb, k, nb, one, Tbig + (size_t)b * WST, NBW, X1, NBW, zero,
                X2, NBW, TRI_NONE, TRI_UPPER, TRI_NONE);
    if (rc) return rc;
    rc = zgemm1(s, OP_N, OP_N, m, k, nb, mone, V, ld, X2, NBW, one, Zs, ldz, TRI_NONE, TRI_LOWER,
                TRI_NONE);
    if (rc) return rc;
  }
  return EXCFV_OK;
}

// Z (n x k) <- Z R^-1 with Z^H Z = R^H R (Cholesky-QR), scratch in ws.Gk/ws.Gki/ws.Z2.
int cholqr(excfv_handle* h, int n, int k, cplx*& Z, long long ldz) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc = zgemm1(s, OP_C, OP_N, k, k, n, one, Z, ldz, Z, ldz, zero, ws.Gk, k, TRI_UPPER);
  if (rc) return rc;
  if ((rc = potrf_upper(h, k, ws.Gk, ws.Gki, k))) return rc;
  if ((rc = trtri_upper(h, k, ws.Gk, ws.Gki, k, ws.Z2))) return rc;
  rc = zgemm1(s, OP_N, OP_N, n, k, k, one, Z, ldz, ws.Gki, k, zero, ws.Z2, ldz, TRI_NONE, TRI_NONE,
              TRI_UPPER);
  if (rc) return rc;
  cplx* t = Z;
  Z = ws.Z2;
  ws.Z2 = t;
  return EXCFV_OK;
}

// The two-stage reduction when the handle asks for it and it supports n
// (its chase reflectors must fit ws.O); the one-stage panels otherwise.  On
// one B200 the one-stage panels are faster at the orders of the workloads
// (n = 316..5028): the chase's ~3n dependent steps each pay a hand-off
// between SMs, so EXCFV_REDUCTION_AUTO takes the one-stage reduction.
bool use_two_stage(excfv_handle* h, int n) {
  if (h->reduction != EXCFV_REDUCTION_TWO_STAGE) return false;
  if (!two_stage_supported(h, n)) return false;
  return chase_reflector_elems(n) <= (size_t)n * n;
}

// States carried through the complex64 reduction so that the Rayleigh-Ritz
// step has a buffer between the kept and the discarded part of the spectrum.
int mixed_states(int n, int k) { return std::min(n, k + std::max(16, k / 8)); }

static int stage_solve_mixed(excfv_handle* h, int n, int k, double evaltol, double* d_eval,
                             cplx* d_evec, long long ldevec);

// The front of the solve: O = U^H U, Ui = U^-1, C = Ui^H H Ui in ws.H (both
// triangles) and, in the precision form, C's complex64 copy in ws.T (leading
// dimension n rounded up to even).  The grouped batch runs this step for all
// of its k-points together and then only stage_solve_back per k-point.
static int solve_front(excfv_handle* h, int n, bool f32copy) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const long long ld = n;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc;
  bind_gemm_ctx(h);
  CUDA_TRY(cudaMemsetAsync(ws.status, 0, ST_SETUP * sizeof(int), s));
  prof_begin(h, PROF_POTRF);
  if ((rc = potrf_upper(h, n, ws.O, ws.Ui, ld))) return rc;
  if ((rc = trtri_upper(h, n, ws.O, ws.Ui, ld, ws.T))) return rc;
  prof_end(h, PROF_POTRF);
  prof_begin(h, PROF_HEGST);
  // C = Ui^H H Ui (upper), then both triangles
  if ((rc = zgemm1(s, OP_N, OP_N, n, n, n, one, ws.H, ld, ws.Ui, ld, zero, ws.T, ld, TRI_NONE,
                   TRI_NONE, TRI_UPPER)))
    return rc;
  if ((rc = zgemm1(s, OP_C, OP_N, n, n, n, one, ws.Ui, ld, ws.T, ld, zero, ws.H, ld, TRI_UPPER,
                   TRI_LOWER, TRI_NONE)))
    return rc;
  if ((rc = mirror_upper(s, n, ws.H, ld))) return rc;
  if (f32copy) {
    // complex64 copy of C for the reduction (ws.T is free now); an even
    // leading dimension keeps its columns 16-byte aligned for the tile loads
    float2* Cf = reinterpret_cast<float2*>(ws.T);
    const long long ldf = (n + 1) & ~1;
    k_to_f32<<<dim3((n + 255) / 256, n), 256, 0, s>>>(n, ws.H, ld, Cf, ldf); count_launch();
    CUDA_TRY(cudaGetLastError());
  }
  prof_end(h, PROF_HEGST);
  return EXCFV_OK;
}

static int solve_back_fp64(excfv_handle* h, int n, int k, double evaltol, double* d_eval, cplx* d_evec,
                           long long ldevec);

int stage_solve(excfv_handle* h, int n, int k, double evaltol, double* d_eval, cplx* d_evec,
                long long ldevec) {
  if (k < 1 || k > n) return EXCFV_ERR_ARG;
  const bool mixed = h->prec == EXCFV_PREC_MIXED && n > 64;
  if (mixed && mixed_states(n, k) > h->ws.kmax) {
    excfv_set_error("mixed solve: workspace holds %d states, needs %d", h->ws.kmax, mixed_states(n, k));
    return EXCFV_ERR_ARG;
  }
  if (!mixed && k > h->ws.kmax) return EXCFV_ERR_ARG;
  int rc = solve_front(h, n, mixed);
  if (rc) return rc;
  return stage_solve_back(h, n, k, evaltol, d_eval, d_evec, ldevec);
}

int solve_front_f32copy(excfv_handle* h, int n) { return h->prec == EXCFV_PREC_MIXED && n > 64; }

int stage_solve_back(excfv_handle* h, int n, int k, double evaltol, double* d_eval, cplx* d_evec,
                     long long ldevec) {
  if (h->prec == EXCFV_PREC_MIXED && n > 64)
    return stage_solve_mixed(h, n, k, evaltol, d_eval, d_evec, ldevec);
  return solve_back_fp64(h, n, k, evaltol, d_eval, d_evec, ldevec);
}

// From C (ws.H) and Ui onwards: tridiagonal reduction, eigenpairs of T,
// back-transforms.
static int solve_back_fp64(excfv_handle* h, int n, int k, double evaltol, double* d_eval, cplx* d_evec,
                           long long ldevec) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const long long ld = n;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc;
  if (k < 1 || k > n || k > ws.kmax) return EXCFV_ERR_ARG;
  bind_gemm_ctx(h);
  // tridiagonal reduction: C = Q T Q^H, Q's reflectors in C (and, two-stage,
  // the chase reflectors in ws.O, the band in ws.T, the phase in ws.ybuf)
  const bool two = use_two_stage(h, n);
  if (two) {
    if ((rc = he2hb(h, n, ws.H, ld))) return rc;
    if ((rc = two_stage_finish_band(h, n, ws.H, ld, ws.T))) return rc;
    prof_begin(h, PROF_TRD_CHASE);
    if ((rc = hb2st(h, n, ws.T, ws.O, ws.ybuf))) return rc;
    prof_end(h, PROF_TRD_CHASE);
  } else {
    if ((rc = tridiag_reduce(h, n, ws.H, ld))) return rc;
  }
  // eigenpairs of T
  cplx* Z = ws.Z;
  prof_begin(h, PROF_STEIG);
  if ((rc = tridiag_eig(h, n, k, evaltol, ws.d, ws.e, ws.w, Z, ld, ws.stein_ws, ws.icl)))
    return rc;
  prof_end(h, PROF_STEIG);
  prof_begin(h, PROF_BACKTR);
  if ((rc = cholqr(h, n, k, Z, ld))) return rc;
  // back-transforms
  if (two) {
    if ((rc = two_stage_back(h, n, k, ws.H, ld, ws.O, ws.ybuf, Z, ld))) return rc;
  } else {
    if ((rc = apply_q(h, n, k, ws.H, ld, Z, ld, 1))) return rc;
  }
  if ((rc = zgemm1(s, OP_N, OP_N, n, k, n, one, ws.Ui, ld, Z, ld, zero, d_evec, ldevec, TRI_NONE,
                   TRI_UPPER, TRI_NONE)))
    return rc;
  prof_end(h, PROF_BACKTR);
  ws.Z = Z;  // cholqr may have swapped the buffers
  k_copy_eval<<<(k + 127) / 128, 128, 0, s>>>(k, ws.w, d_eval); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

// The precision form: FP64 Cholesky and reduction to C = U^-H H U^-1; the
// Householder tridiagonal reduction of a complex64 copy of C; eigenpairs of T
// for k' = k + extra states and their back-transform; then Rayleigh-Ritz in
// FP64: X0 = orth(Q Z_T), Hk = X0^H C X0 (k' x k') solved in FP64, X = X0 Y.
// The Ritz values' errors are second order in the FP32 perturbation of X0
// (relative to the gap between state k and the discarded states beyond k').
static int stage_solve_mixed(excfv_handle* h, int n, int k, double evaltol, double* d_eval,
                             cplx* d_evec, long long ldevec) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const long long ld = n;
  const cplx one = cmk(1.0, 0.0), zero = cmk(0.0, 0.0);
  int rc;
  const int kx = mixed_states(n, k);
  if (k < 1 || k > n) return EXCFV_ERR_ARG;
  if (kx > ws.kmax) {
    excfv_set_error("mixed solve: workspace holds %d states, needs %d", ws.kmax, kx);
    return EXCFV_ERR_ARG;
  }
  bind_gemm_ctx(h);
  // C in ws.H, its complex64 copy in ws.T (solve_front)
  float2* Cf = reinterpret_cast<float2*>(ws.T);
  const long long ldf = (n + 1) & ~1;
  if ((rc = tridiag_reduce_f32(h, n, Cf, ldf))) return rc;
  // reflectors back to FP64 into ws.O (the Cholesky factor is no longer needed)
  k_lower_to_f64<<<dim3((n + 255) / 256, n), 256, 0, s>>>(n, Cf, ldf, ws.O, ld); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* Z = ws.Z;
  prof_begin(h, PROF_STEIG);
  // T's eigenvalues only seed inverse iteration and are replaced by the
  // refinement's, so bisection stops at 1e-10 (evaltol if looser)
  if ((rc = tridiag_eig(h, n, kx, fmax(evaltol, 1e-10), ws.d, ws.e, ws.w, Z, ld, ws.stein_ws, ws.icl)))
    return rc;
  prof_end(h, PROF_STEIG);
  prof_begin(h, PROF_BACKTR);
  if ((rc = apply_q(h, n, kx, ws.O, ld, Z, ld, 1))) return rc;
  // X0 = Z: orthonormal up to the complex64 rounding of the reflectors,
  // S = X0^H X0 = I + D with |D| ~ 1e-7.  Rayleigh-Ritz in FP64 on
  // S^-1/2 Hk S^-1/2 with S^-1/2 = I - D/2 (error O(D^2)):
  //   Hm = Hk - (D Hk + Hk D)/2,  refine Hm -> (lambda, Y),  Y <- (I - D/2) Y,
  // then one first-order Loewdin step Y <- Y (I - (Y^H S Y - I)/2) makes
  // X = X0 Y orthonormal (error O(|Y^H S Y - I|^2) ~ 1e-12).
  const cplx mhalf = cmk(-0.5, 0.0);
  cplx* R = ws.Z2;
  if ((rc = zgemm1(s, OP_N, OP_N, n, kx, n, one, ws.H, ld, Z, ld, zero, R, ld))) return rc;
  cplx* Hk = ws.T;
  if ((rc = zgemm1(s, OP_C, OP_N, kx, kx, n, one, Z, ld, R, ld, zero, Hk, kx, TRI_UPPER))) return rc;
  if ((rc = mirror_upper(s, kx, Hk, kx))) return rc;
  cplx* Dm = ws.Gk;  // S - I
  if ((rc = zgemm1(s, OP_C, OP_N, kx, kx, n, one, Z, ld, Z, ld, zero, Dm, kx, TRI_UPPER))) return rc;
  if ((rc = mirror_upper(s, kx, Dm, kx))) return rc;
  k_sub_identity<<<(kx + 127) / 128, 128, 0, s>>>(kx, Dm, kx); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* Hm = ws.O;   // the reflectors are consumed
  CUDA_TRY(cudaMemcpyAsync(Hm, Hk, sizeof(cplx) * (size_t)kx * kx, cudaMemcpyDeviceToDevice, s));
  if ((rc = zgemm1(s, OP_N, OP_N, kx, kx, kx, mhalf, Dm, kx, Hk, kx, one, Hm, kx))) return rc;
  if ((rc = zgemm1(s, OP_N, OP_N, kx, kx, kx, mhalf, Hk, kx, Dm, kx, one, Hm, kx))) return rc;
  // clusters, their exact rotations Q, Hp = Q^H Hm Q, perturbation
  RRScratch rs;
  {
    double* dp = ws.stein_ws;
    rs.D = dp; rs.lam = dp + kx;
    int* ip = reinterpret_cast<int*>(dp + 2 * kx);
    rs.perm = ip; rs.cid = ip + kx; rs.cstart = ip + 2 * kx; rs.csize = ip + 3 * kx;
    rs.sel = ip + 4 * kx; rs.nclust = ip + 5 * kx;
  }
  cplx* Q = ws.T;    // Hk is consumed
  CUDA_TRY(cudaMemsetAsync(Q, 0, sizeof(cplx) * (size_t)kx * kx, s));
  k_rr_clusters<<<1, 1024, 0, s>>>(kx, Hm, rs); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_rr_jacobi<<<(kx + 127) / 128, 128, 0, s>>>(kx, Hm, rs, Q, ws.Z2, ws.H, ws.status); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* W = ws.H;    // Jacobi scratch is consumed
  if ((rc = zgemm1(s, OP_N, OP_N, kx, kx, kx, one, Hm, kx, Q, kx, zero, W, kx))) return rc;
  cplx* Hp = ws.Z2;
  if ((rc = zgemm1(s, OP_C, OP_N, kx, kx, kx, one, Q, kx, W, kx, zero, Hp, kx))) return rc;
  cplx* Tm = ws.O;   // Hm is consumed
  k_rr_perturb<<<(kx * 32 + 255) / 256, 256, 0, s>>>(kx, Hp, rs, Tm); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_rr_select<<<1, 1024, 0, s>>>(kx, k, rs, d_eval); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* Ts = ws.H;   // W is consumed
  k_rr_gather<<<dim3((kx + 255) / 256, k), 256, 0, s>>>(kx, k, Tm, rs.sel, Ts); count_launch();
  CUDA_TRY(cudaGetLastError());
  cplx* Y = ws.Z2;   // Hp is consumed
  if ((rc = zgemm1(s, OP_N, OP_N, kx, k, kx, one, Q, kx, Ts, kx, zero, Y, kx))) return rc;
  // Y1 = (I - D/2) Y
  cplx* Y1 = ws.T;   // Q is consumed
  CUDA_TRY(cudaMemcpyAsync(Y1, Y, sizeof(cplx) * (size_t)kx * k, cudaMemcpyDeviceToDevice, s));
  if ((rc = zgemm1(s, OP_N, OP_N, kx, k, kx, mhalf, Dm, kx, Y, kx, one, Y1, kx))) return rc;
  // E = Y1^H S Y1 - I = Y1^H (Y1 + D Y1) - I
  cplx* SY = ws.O;   // Tm is consumed
  CUDA_TRY(cudaMemcpyAsync(SY, Y1, sizeof(cplx) * (size_t)kx * k, cudaMemcpyDeviceToDevice, s));
  if ((rc = zgemm1(s, OP_N, OP_N, kx, k, kx, one, Dm, kx, Y1, kx, one, SY, kx))) return rc;
  cplx* E = ws.H;    // Ts is consumed
  if ((rc = zgemm1(s, OP_C, OP_N, k, k, kx, one, Y1, kx, SY, kx, zero, E, k))) return rc;
  k_sub_identity<<<(k + 127) / 128, 128, 0, s>>>(k, E, k); count_launch();
  CUDA_TRY(cudaGetLastError());
  // Y2 = Y1 (I - E/2)
  cplx* Y2 = ws.Z2;  // Y is consumed
  CUDA_TRY(cudaMemcpyAsync(Y2, Y1, sizeof(cplx) * (size_t)kx * k, cudaMemcpyDeviceToDevice, s));
  if ((rc = zgemm1(s, OP_N, OP_N, kx, k, k, mhalf, Y1, kx, E, k, one, Y2, kx))) return rc;
  // X = X0 Y2 (n x k, into ws.O), back-transform with U^-1
  cplx* X = ws.O;    // SY is consumed
  if ((rc = zgemm1(s, OP_N, OP_N, n, k, kx, one, Z, ld, Y2, kx, zero, X, ld))) return rc;
  if ((rc = zgemm1(s, OP_N, OP_N, n, k, n, one, ws.Ui, ld, X, ld, zero, d_evec, ldevec, TRI_NONE,
                   TRI_UPPER, TRI_NONE)))
    return rc;
  prof_end(h, PROF_BACKTR);
  return EXCFV_OK;
}

int stage_status(excfv_handle* h, int n) {
  int st[ST_NWORDS];
  CUDA_TRY(cudaMemcpyAsync(st, h->ws.status, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return status_to_info(st, n);
}

int status_to_info(const int* st, int n) {
  if (st[ST_SETUP]) {
    excfv_set_error("a bounded wait of the setup contraction timed out");
    return EXCFV_ERR_TIMEOUT;
  }
  if (st[ST_BARRIER]) {
    excfv_set_error("grid barrier timed out in the tridiagonal reduction");
    return EXCFV_ERR_TIMEOUT;
  }
  if (st[ST_POTRF]) return n + st[ST_POTRF];
  if (st[ST_STEBZ]) {
    excfv_set_error("bisection did not converge for %d eigenvalues", st[ST_STEBZ]);
    return EXCFV_ERR_NOCONV;
  }
  if (st[ST_STEIN]) return st[ST_STEIN];
  if (st[ST_REFINE]) {
    excfv_set_error("precision form: %d near-degenerate states in one cluster exceed the "
                    "refinement's limit; solve this k-point with EXCFV_PREC_FP64", st[ST_REFINE]);
    return EXCFV_ERR_NOCONV;
  }
  return EXCFV_OK;
}
