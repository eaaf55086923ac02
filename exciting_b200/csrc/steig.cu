// Eigenpairs of the real symmetric tridiagonal T = tridiag(e, d, e).
//
// Eigenvalues (DSTEBZ, external/LAPACK/zheevx.f:490, range 'I'): one warp
// per requested eigenvalue index, multisection on the Sturm count (32
// points per step, the interval shrinks 33x per step) from the Gershgorin
// interval; stop when the width is below max(abstol, pivmin,
// 2 ulp max(|lo|,|hi|)) exactly as DSTEBZ's bisection test.
//
// Eigenvectors (DSTEIN, zheevx.f:496): inverse iteration with the shifted
// tridiagonal factored by Gaussian elimination with partial pivoting, at
// most five iterations, growth test sqrt(0.1/n) plus two extra iterations,
// unit 2-norm with the largest component positive.  Eigenvalues closer than
// CLUSTER_REL * ||T|| form a cluster: its shifts are separated by 10 ulp
// (DSTEIN's perturbation) and its vectors are Gram-Schmidt orthogonalised
// against the earlier members inside the iteration.  Residual loss of
// orthogonality between well-separated vectors is removed afterwards by a
// Cholesky-QR pass on the complex vectors (see solve.cu).
#include "handle.cuh"

namespace {

constexpr double CLUSTER_REL = 1e-9;

// 1/q from the hardware approximation refined by two Newton-Raphson steps
// r <- r (2 - q r) (each roughly doubles the correct bits).
__device__ __forceinline__ double recip_nr(double q) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(q));
  r = fma(r, fma(-q, r, 1.0), r);
  r = fma(r, fma(-q, r, 1.0), r);
  return r;
}

// Number of eigenvalues of T below x (Sturm sequence of the LDL^T pivots).
// The pivot recurrence q_i = d_i - x - e_{i-1}^2 / q_{i-1} uses recip_nr
// instead of a division: within an ulp or so of the quotient, i.e. a relative
// perturbation of e^2 of the order of the rounding the count already carries
// (the count stays that of a nearby tridiagonal matrix), on a dependent chain
// much shorter than a correctly rounded division.
__device__ __forceinline__ int sturm_count(int n, const double* __restrict__ d,
                                           const double* __restrict__ e2, double x, double pivmin) {
  double q = d[0] - x;
  if (fabs(q) <= pivmin) q = -pivmin;
  int cnt = q < 0.0;
  for (int i = 1; i < n; ++i) {
    q = fma(-e2[i - 1], recip_nr(q), d[i] - x);
    if (fabs(q) <= pivmin) q = -pivmin;
    cnt += q < 0.0;
  }
  return cnt;
}

// scal[0] = gl, [1] = gu, [2] = pivmin, [3] = tnorm; e2[i] = e[i]^2
__global__ void k_tridiag_prep(int n, const double* d, const double* e, double* e2, double* scal) {
  __shared__ double s_lo[256], s_hi[256], s_e2[256], s_nrm[256];
  double lo = 1e300, hi = -1e300, em = 0.0, nm = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double ea = (i > 0) ? fabs(e[i - 1]) : 0.0;
    const double eb = (i < n - 1) ? fabs(e[i]) : 0.0;
    lo = fmin(lo, d[i] - ea - eb);
    hi = fmax(hi, d[i] + ea + eb);
    nm = fmax(nm, fabs(d[i]) + ea + eb);
    if (i < n - 1) {
      e2[i] = e[i] * e[i];
      em = fmax(em, e[i] * e[i]);
    }
  }
  s_lo[threadIdx.x] = lo; s_hi[threadIdx.x] = hi; s_e2[threadIdx.x] = em; s_nrm[threadIdx.x] = nm;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) {
      s_lo[threadIdx.x] = fmin(s_lo[threadIdx.x], s_lo[threadIdx.x + o]);
      s_hi[threadIdx.x] = fmax(s_hi[threadIdx.x], s_hi[threadIdx.x + o]);
      s_e2[threadIdx.x] = fmax(s_e2[threadIdx.x], s_e2[threadIdx.x + o]);
      s_nrm[threadIdx.x] = fmax(s_nrm[threadIdx.x], s_nrm[threadIdx.x + o]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double safemin = 2.2250738585072014e-308;
    const double ulp = 2.220446049250313e-16;
    const double pivmin = safemin * fmax(1.0, s_e2[0]);
    const double tnorm = fmax(fabs(s_lo[0]), fabs(s_hi[0]));
    const double fudge = 2.1;
    scal[0] = s_lo[0] - fudge * tnorm * ulp * n - fudge * 2.0 * pivmin;
    scal[1] = s_hi[0] + fudge * tnorm * ulp * n + fudge * 2.0 * pivmin;
    scal[2] = pivmin;
    scal[3] = s_nrm[0];
  }
}

__global__ void k_stebz(int n, const double* d, const double* e2, const double* scal, int k,
                        double abstol, double* w, int* status) {
  const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (j >= k) return;
  const double pivmin = scal[2];
  const double ulp = 2.220446049250313e-16;
  const double atol = abstol > 0.0 ? abstol : ulp * scal[3];
  double lo = scal[0], hi = scal[1];
  bool conv = false;
  for (int it = 0; it < 200; ++it) {
    const double width = hi - lo;
    const double tol = fmax(fmax(atol, pivmin), 2.0 * ulp * fmax(fabs(lo), fabs(hi)));
    if (width <= tol) { conv = true; break; }
    const double step = width / 33.0;
    double x = lo + (lane + 1) * step;
    if (x >= hi) x = hi;
    const int cnt = sturm_count(n, d, e2, x, pivmin);
    const unsigned ball = __ballot_sync(0xffffffffu, cnt >= j + 1);
    if (ball == 0u) {
      lo = __shfl_sync(0xffffffffu, x, 31);
    } else {
      const int f = __ffs(ball) - 1;
      const double xf = __shfl_sync(0xffffffffu, x, f);
      const double xp = __shfl_sync(0xffffffffu, x, f > 0 ? f - 1 : 0);
      hi = xf;
      if (f > 0) lo = xp;
    }
    if (!(hi > lo)) { conv = true; break; }
  }
  if (lane == 0) {
    w[j] = 0.5 * (lo + hi);
    if (!conv) atomicAdd(&status[ST_STEBZ], 1);
  }
}

// cluster starts: cl[j] = 1 if j starts a cluster
__global__ void k_clusters(int k, const double* w, const double* scal, int* cl) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= k) return;
  const double tol = CLUSTER_REL * fmax(scal[3], 1e-300);
  cl[j] = (j == 0) || (w[j] - w[j - 1] > tol);
}

__device__ __forceinline__ double urand(unsigned long long a, unsigned long long b) {
  unsigned long long z = a * 0x9E3779B97F4A7C15ull + b * 0xBF58476D1CE4E5B9ull + 0x94D049BB133111EBull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  z ^= z >> 31;
  return ((double)(z >> 11) * (1.0 / 9007199254740992.0)) * 2.0 - 1.0;
}

// One thread per cluster.  Work arrays are interleaved by eigenvalue index
// (element i of slot j at [i*k + j]) so that neighbouring threads touch
// neighbouring addresses.  Y (interleaved too) receives the vectors.  The
// factorisation stores the pivots' reciprocals, so the solves' dependency
// chains hold only multiply-adds; the loops are unrolled so that loads run
// ahead of the recurrences.
__global__ void k_stein(int n, const double* __restrict__ d, const double* __restrict__ e,
                        const double* __restrict__ scal, int k, const double* __restrict__ w,
                        const int* __restrict__ cl, double* __restrict__ ua, double* __restrict__ ub,
                        double* __restrict__ uf, double* __restrict__ um, double* __restrict__ Yi,
                        int* status) {
  const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (j0 >= k || !cl[j0]) return;
  int j1 = j0 + 1;
  while (j1 < k && !cl[j1]) ++j1;
  const double eps = 1.1102230246251565e-16;
  const double tnorm = scal[3];
  const double dtpcrt = sqrt(0.1 / n);
  const double pert = fmax(eps * tnorm, 1e-300);
  double xprev = 0.0;
  for (int j = j0; j < j1; ++j) {
    double lam = w[j];
    if (j > j0) {
      const double pertol = 10.0 * fabs(eps * lam);
      if (lam - xprev < pertol) lam = xprev + pertol;
    }
    xprev = lam;
    // factor T - lam I (slot j); ua holds 1/pivot
    double a = d[0] - lam, b = (n > 1) ? e[0] : 0.0;
    double ulast = 0.0;
#pragma unroll 4
    for (int i = 0; i < n - 1; ++i) {
      const double c = e[i], dd = d[i + 1] - lam, ee = (i + 1 < n - 1) ? e[i + 1] : 0.0;
      const size_t o = (size_t)i * k + j;
      if (fabs(a) >= fabs(c)) {
        const double aa = (fabs(a) < pert) ? copysign(pert, a) : a;
        const double ra = 1.0 / aa;
        ua[o] = ra; ub[o] = b; uf[o] = 0.0;
        const double m = c * ra;
        um[o] = m;
        a = dd - m * b;
        b = ee;
      } else {
        const double rc = 1.0 / c;
        ua[o] = rc; ub[o] = dd; uf[o] = ee;
        const double m = a * rc;
        um[o] = -m - 2.0;  // encodes a swap (a multiplier |m| <= 1 never reaches below -1)
        a = b - m * dd;
        b = -m * ee;
      }
    }
    {
      const size_t o = (size_t)(n - 1) * k + j;
      const double aa = (fabs(a) < pert) ? copysign(pert, a) : a;
      ua[o] = 1.0 / aa;
      ub[o] = 0.0; uf[o] = 0.0; um[o] = 0.0;
      ulast = fabs(aa);
    }
    for (int i = 0; i < n; ++i) Yi[(size_t)i * k + j] = urand(j + 1, i + 1);
    int nrmchk = 0;
    bool conv = false;
    for (int its = 0; its < 5; ++its) {
      // scale the right-hand side: ||x||_1 = n ||T|| max(eps, |u_last|)
      double s1 = 0.0;
#pragma unroll 8
      for (int i = 0; i < n; ++i) s1 += fabs(Yi[(size_t)i * k + j]);
      const double scl = (s1 > 0.0) ? n * tnorm * fmax(eps, ulast) / s1 : 1.0;
      // forward elimination on the right-hand side
      double cur = Yi[j] * scl;
#pragma unroll 4
      for (int i = 0; i < n - 1; ++i) {
        const size_t o = (size_t)i * k + j;
        const double nx = Yi[o + k] * scl;
        const double m = um[o];
        if (m < -1.0) {  // swapped
          Yi[o] = nx;
          cur = cur + (m + 2.0) * nx;
        } else {
          Yi[o] = cur;
          cur = nx - m * cur;
        }
      }
      // back substitution with the stored reciprocals
      double x2 = 0.0, x1 = cur * ua[(size_t)(n - 1) * k + j];
      Yi[(size_t)(n - 1) * k + j] = x1;
      double nrm = fabs(x1);
#pragma unroll 4
      for (int i = n - 2; i >= 0; --i) {
        const size_t o = (size_t)i * k + j;
        const double x = (Yi[o] - ub[o] * x1 - uf[o] * x2) * ua[o];
        Yi[o] = x;
        nrm = fmax(nrm, fabs(x));
        x2 = x1;
        x1 = x;
      }
      // orthogonalise against the earlier members of the cluster
      if (j > j0) {
        for (int q = j0; q < j; ++q) {
          double dot = 0.0;
          for (int i = 0; i < n; ++i) dot += Yi[(size_t)i * k + q] * Yi[(size_t)i * k + j];
          for (int i = 0; i < n; ++i) Yi[(size_t)i * k + j] -= dot * Yi[(size_t)i * k + q];
        }
        nrm = 0.0;
        for (int i = 0; i < n; ++i) nrm = fmax(nrm, fabs(Yi[(size_t)i * k + j]));
      }
      if (!(nrm >= dtpcrt)) {
        if (nrm > 0.0 && nrm < 1e-200) {
          for (int i = 0; i < n; ++i) Yi[(size_t)i * k + j] *= 1e200;
        }
        continue;
      }
      ++nrmchk;
      if (nrmchk >= 3) { conv = true; break; }
    }
    if (!conv) atomicAdd(&status[ST_STEIN], 1);
    // normalise: unit 2-norm, largest component positive
    double s2 = 0.0, big = 0.0;
    int ib = 0;
    for (int i = 0; i < n; ++i) {
      const double v = Yi[(size_t)i * k + j];
      s2 += v * v;
      if (fabs(v) > big) { big = fabs(v); ib = i; }
    }
    double sc = (s2 > 0.0) ? 1.0 / sqrt(s2) : 0.0;
    if (Yi[(size_t)ib * k + j] < 0.0) sc = -sc;
    for (int i = 0; i < n; ++i) Yi[(size_t)i * k + j] *= sc;
  }
}

// The same inverse iteration with the factor and the working vector of one
// eigenvector in shared memory (40 n bytes): one warp per cluster, lane 0
// runs the recurrences (factorisation, forward elimination, back
// substitution) at shared-memory latency, the warp shares the element-wise
// passes.  The finished vectors go to Yi (interleaved as in k_stein) because
// later members of a cluster are orthogonalised against them.
__global__ void __launch_bounds__(32) k_stein_smem(int n, const double* __restrict__ d,
                                                   const double* __restrict__ e,
                                                   const double* __restrict__ scal, int k,
                                                   const double* __restrict__ w,
                                                   const int* __restrict__ cl, double* Yi,
                                                   int* status) {
  extern __shared__ double sm[];
  double* ra = sm;          // 1 / pivot
  double* rb = ra + n;      // first superdiagonal of U
  double* rf = rb + n;      // second superdiagonal (fill-in from swaps)
  double* rm = rf + n;      // multiplier (swap encoded as -m-2)
  double* y = rm + n;       // working vector
  const int j0 = blockIdx.x;
  const int lane = threadIdx.x;
  if (!cl[j0]) return;
  int j1 = j0 + 1;
  while (j1 < k && !cl[j1]) ++j1;
  const double eps = 1.1102230246251565e-16;
  const double tnorm = scal[3];
  const double dtpcrt = sqrt(0.1 / n);
  const double pert = fmax(eps * tnorm, 1e-300);
  double xprev = 0.0;
  for (int j = j0; j < j1; ++j) {
    double lam = w[j];
    if (j > j0) {
      const double pertol = 10.0 * fabs(eps * lam);
      if (lam - xprev < pertol) lam = xprev + pertol;
    }
    xprev = lam;
    __shared__ double s_ulast;
    if (lane == 0) {
      double a = d[0] - lam, b = (n > 1) ? e[0] : 0.0;
      for (int i = 0; i < n - 1; ++i) {
        const double c = e[i], dd = d[i + 1] - lam, ee = (i + 1 < n - 1) ? e[i + 1] : 0.0;
        if (fabs(a) >= fabs(c)) {
          const double aa = (fabs(a) < pert) ? copysign(pert, a) : a;
          const double r = 1.0 / aa;
          ra[i] = r; rb[i] = b; rf[i] = 0.0;
          const double m = c * r;
          rm[i] = m;
          a = dd - m * b;
          b = ee;
        } else {
          const double r = 1.0 / c;
          ra[i] = r; rb[i] = dd; rf[i] = ee;
          const double m = a * r;
          rm[i] = -m - 2.0;
          a = b - m * dd;
          b = -m * ee;
        }
      }
      const double aa = (fabs(a) < pert) ? copysign(pert, a) : a;
      ra[n - 1] = 1.0 / aa;
      rb[n - 1] = 0.0; rf[n - 1] = 0.0; rm[n - 1] = 0.0;
      s_ulast = fabs(aa);
    }
    for (int i = lane; i < n; i += 32) y[i] = urand(j + 1, i + 1);
    __syncwarp();
    const double ulast = s_ulast;
    int nrmchk = 0;
    bool conv = false;
    for (int its = 0; its < 5; ++its) {
      double s1 = 0.0;
      for (int i = lane; i < n; i += 32) s1 += fabs(y[i]);
      for (int o = 16; o > 0; o >>= 1) s1 += __shfl_xor_sync(0xffffffffu, s1, o);
      const double scl = (s1 > 0.0) ? n * tnorm * fmax(eps, ulast) / s1 : 1.0;
      if (lane == 0) {
        double cur = y[0] * scl;
        for (int i = 0; i < n - 1; ++i) {
          const double nx = y[i + 1] * scl;
          const double m = rm[i];
          if (m < -1.0) {
            y[i] = nx;
            cur = cur + (m + 2.0) * nx;
          } else {
            y[i] = cur;
            cur = nx - m * cur;
          }
        }
        double x2 = 0.0, x1 = cur * ra[n - 1];
        y[n - 1] = x1;
        for (int i = n - 2; i >= 0; --i) {
          const double x = (y[i] - rb[i] * x1 - rf[i] * x2) * ra[i];
          y[i] = x;
          x2 = x1;
          x1 = x;
        }
      }
      __syncwarp();
      for (int q = j0; q < j; ++q) {
        double dot = 0.0;
        for (int i = lane; i < n; i += 32) dot += Yi[(size_t)i * k + q] * y[i];
        for (int o = 16; o > 0; o >>= 1) dot += __shfl_xor_sync(0xffffffffu, dot, o);
        for (int i = lane; i < n; i += 32) y[i] -= dot * Yi[(size_t)i * k + q];
        __syncwarp();
      }
      double nrm = 0.0;
      for (int i = lane; i < n; i += 32) nrm = fmax(nrm, fabs(y[i]));
      for (int o = 16; o > 0; o >>= 1) nrm = fmax(nrm, __shfl_xor_sync(0xffffffffu, nrm, o));
      if (!(nrm >= dtpcrt)) {
        if (nrm > 0.0 && nrm < 1e-200)
          for (int i = lane; i < n; i += 32) y[i] *= 1e200;
        __syncwarp();
        continue;
      }
      ++nrmchk;
      if (nrmchk >= 3) { conv = true; break; }
    }
    if (!conv && lane == 0) atomicAdd(&status[ST_STEIN], 1);
    // normalise: unit 2-norm, largest component positive (lowest index on ties)
    double s2 = 0.0, big = -1.0;
    int ib = 0;
    for (int i = lane; i < n; i += 32) {
      const double v = y[i];
      s2 += v * v;
      if (fabs(v) > big) { big = fabs(v); ib = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      s2 += __shfl_xor_sync(0xffffffffu, s2, o);
      const double ob = __shfl_xor_sync(0xffffffffu, big, o);
      const int oi = __shfl_xor_sync(0xffffffffu, ib, o);
      if (ob > big || (ob == big && oi < ib)) { big = ob; ib = oi; }
    }
    double sc = (s2 > 0.0) ? 1.0 / sqrt(s2) : 0.0;
    if (y[ib] < 0.0) sc = -sc;
    for (int i = lane; i < n; i += 32) Yi[(size_t)i * k + j] = y[i] * sc;
    __syncwarp();
  }
}

// Z(i, j) = Yi[i*k + j] (interleaved real -> column-major complex, ld ldz)
__global__ void k_y_to_z(int n, int k, const double* Yi, cplx* Z, long long ldz) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  if (i >= n || j >= k) return;
  Z[i + ldz * j] = cmk(Yi[(size_t)i * k + j], 0.0);
}

}  // namespace

// Lowest k eigenvalues into w, eigenvectors as complex columns of Z (n x k).
// scratch: e2 (n), scal (4), cl (k ints), 4*n*k doubles for the factors, n*k for Yi.
int tridiag_eig(excfv_handle* h, int n, int k, double abstol, const double* d, const double* e,
                double* w, cplx* Z, long long ldz, double* scratch, int* iscratch) {
  cudaStream_t s = h->stream;
  double* e2 = scratch;
  double* scal = scratch + n;
  double* ua = scal + 8;
  double* ub = ua + (size_t)n * k;
  double* uf = ub + (size_t)n * k;
  double* um = uf + (size_t)n * k;
  double* Yi = um + (size_t)n * k;
  k_tridiag_prep<<<1, 256, 0, s>>>(n, d, e, e2, scal); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_stebz<<<(k * 32 + 127) / 128, 128, 0, s>>>(n, d, e2, scal, k, abstol, w, h->ws.status); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_clusters<<<(k + 127) / 128, 128, 0, s>>>(k, w, scal, iscratch); count_launch();
  CUDA_TRY(cudaGetLastError());
  const size_t sbytes = 40 * (size_t)n;
  if (sbytes <= 200 * 1024) {
    CUDA_TRY(cudaFuncSetAttribute(k_stein_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sbytes));
    k_stein_smem<<<k, 32, sbytes, s>>>(n, d, e, scal, k, w, iscratch, Yi, h->ws.status); count_launch();
  } else {
    k_stein<<<(k + 31) / 32, 32, 0, s>>>(n, d, e, scal, k, w, iscratch, ua, ub, uf, um, Yi,
                                         h->ws.status); count_launch();
  }
  CUDA_TRY(cudaGetLastError());
  k_y_to_z<<<dim3((n + 255) / 256, k), 256, 0, s>>>(n, k, Yi, Z, ldz); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

size_t tridiag_eig_scratch_doubles(int n, int k) { return (size_t)n + 8 + 5 * (size_t)n * k; }
