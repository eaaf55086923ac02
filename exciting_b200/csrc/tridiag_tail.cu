// The last columns of the Householder tridiagonal reduction (ZHETRD's tail,
// external/LAPACK/zhetd2.f: the unblocked reduction, lower storage) in one
// cluster of CL CTAs (16 where the device schedules a cluster that size at
// full shared memory, else 8) whose distributed shared memory holds the
// trailing block.
//
// Once the trailing block C22 is small, the panel kernel's per-column cost
// is set by its two grid barriers and the L2 round trips around them, not by
// the block's size.  Here the lower triangle of the m x m block is packed in
// the shared memory of the cluster's CTAs (row i in CTA i mod CL) and every
// column is one unblocked step.  Data another CTA needs is pushed into its
// shared memory (distributed-shared-memory stores) before a cluster barrier,
// never fetched, so no thread waits on a remote load:
//
//   S1  x = C22(c+1:m, c) has arrived in every CTA
//   B   one warp of every CTA: |x(c+2:m)|^2, beta, tau, scale by ZLARFG (the
//       panel kernel's formulas; the same operands and order everywhere, so
//       the same bits), e(c), tau(c); then v = [1; scale x] into vbuf and
//       into column c of own packed rows (unit entry explicit)
//   C   y = C22 v: the row part of own rows (a warp per row), the column part
//       sum_{own i > j} conj(C22_ij) v_i (a thread per column j, no atomics)
//       pushed to the owner of row j
//   S2
//   D   owners: y_i = row part + the CL column parts; w0_i = tau y_i to all,
//       and Re(v^H y) over own rows to all
//   S3
//   E   every CTA: alpha = -|tau|^2/2 v^H C22 v from the CL partials (the
//       panel kernel's real form), w = w0 + alpha v once per entry,
//       C22 -= v w^H + w v^H on own rows (the diagonal kept real, apart from
//       the off-diagonal loop); the updated column c+1 goes out at once: x of
//       the next column and d(c+1)
//
// with three cluster barriers per column.  All CTAs run the same loop, so
// every barrier is reached by all of them; the kernel has no other waits.
// The reflectors, d, e and tau it leaves are those of the panel kernel's
// convention, so the back-transform reads them unchanged.
#include <cooperative_groups.h>

#include "handle.cuh"

namespace cg = cooperative_groups;

namespace {

constexpr int TT = 512;                   // threads per CTA
constexpr int NW = TT / 32;
constexpr size_t SMEM_MAX = 226 * 1024;   // dynamic; the static part is under 1 KB of the 227 KB

__device__ __forceinline__ cplx ldT(const double2* p) { return *p; }
__device__ __forceinline__ cplx ldT(const float2* p) {
  const float2 v = *p;
  return cmk((double)v.x, (double)v.y);
}
__device__ __forceinline__ void stT(double2* p, cplx v) { *p = v; }
__device__ __forceinline__ void stT(float2* p, cplx v) { *p = make_float2((float)v.x, (float)v.y); }

// packed offset of local slot s of rank r (rows r, r + CL, ...; row i holds i + 1 entries)
template <int CL>
__device__ __forceinline__ long long row_off(int r, int s) {
  return (long long)s * (r + 1) + (long long)CL * s * (s - 1) / 2;
}

template <typename T2, int CL>
__global__ void __launch_bounds__(TT, 1) k_tridiag_tail(int n, int c0, T2* C, long long ld, double* d, double* e,
                                                        cplx* tau_out) {
  extern __shared__ __align__(16) unsigned char dsm[];
  cg::cluster_group cl = cg::this_cluster();
  const int rank = (int)cl.block_rank();
  const int m = n - c0;
  const int smax = (m + CL - 1) / CL;            // slots of rank 0, the most any rank has
  const int nslot = (m - rank + CL - 1) / CL;    // rows rank, rank + CL, ...
  // Offsets depend on m only, so they are the same in every CTA (a
  // map_shared_rank address keeps the offset); the packed rows come last.
  cplx* xbuf = reinterpret_cast<cplx*>(dsm);     // column c below the diagonal (pushed)
  cplx* vbuf = xbuf + m;                         // the reflector (local)
  cplx* wbuf = vbuf + m;                         // w0 = tau y (pushed by the row owners), then w
  cplx* ypart = wbuf + m;                        // [CL][smax]: column parts for own rows (pushed)
  cplx* yrow = ypart + (size_t)CL * smax;        // row parts of own rows (local)
  cplx* tau_loc = yrow + smax;                   // tau(c) of the columns c = rank mod CL (local)
  double* e_loc = reinterpret_cast<double*>(tau_loc + smax);  // e(c) of the same columns
  double* d_loc = e_loc + smax;                  // d(i) of own rows
  T2* A = reinterpret_cast<T2*>(d_loc + smax);  // 16-byte aligned: the last three take 32 smax bytes
  __shared__ double s_vav[CL];                   // Re(v^H y) of every rank's rows (pushed)
  __shared__ double s_scal[4];                   // tau, scale
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  // the trailing block's lower triangle into the packed rows
  for (int s = 0; s < nslot; ++s) {
    const int i = rank + CL * s;
    const long long o = row_off<CL>(rank, s);
    for (int j = tid; j <= i; j += TT) {
      cplx v = ldT(C + (c0 + i) + ld * (c0 + j));
      if (j == i) v.y = 0.0;
      stT(A + o + j, v);
    }
  }
  cl.sync();  // every CTA is running before the first remote store
  // column 0: x = C22(1:, 0) to every CTA (a thread per row and target), d(0)
  for (int t = tid; t < nslot * CL; t += TT) {
    const int s = t / CL, r = t % CL, i = rank + CL * s;
    const cplx x = ldT(A + row_off<CL>(rank, s));
    if (i == 0) {
      if (r == 0) d_loc[0] = x.x;
      continue;
    }
    cl.map_shared_rank(xbuf, r)[i] = x;
  }

  for (int c = 0; c < m - 1; ++c) {
    cl.sync();  // x of column c has arrived
    // ---- the reflector (one warp; every CTA derives the same bits from the
    //      same operands: |x(c+2:)|^2 summed in the same order), v into vbuf
    //      and into the packed rows ------------------------------------------
    if (warp == 0) {
      double xn2 = 0.0;
      for (int i = c + 2 + lane; i < m; i += 32) {
        const cplx x = xbuf[i];
        xn2 += x.x * x.x + x.y * x.y;
      }
      for (int o = 16; o > 0; o >>= 1) xn2 += __shfl_xor_sync(0xffffffffu, xn2, o);
      const cplx alpha = xbuf[c + 1];
      double tr = 0.0, ti = 0.0, scr = 0.0, sci = 0.0, beta;
      if (xn2 == 0.0 && alpha.y == 0.0) {
        beta = alpha.x;
      } else {
        const double nrm = sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2);
        beta = (alpha.x >= 0.0) ? -nrm : nrm;
        const double dr = alpha.x - beta, di = alpha.y;  // scale = 1 / (alpha - beta)
        const double rb = 1.0 / beta, rd = 1.0 / (dr * dr + di * di);
        tr = 1.0 - alpha.x * rb;
        ti = -alpha.y * rb;
        scr = dr * rd;
        sci = -di * rd;
      }
      if (lane == 0) {
        s_scal[0] = tr; s_scal[1] = ti; s_scal[2] = scr; s_scal[3] = sci;
        if (c % CL == rank) {
          e_loc[c / CL] = beta;
          tau_loc[c / CL] = cmk(tr, ti);
        }
      }
    }
    __syncthreads();
    const cplx tau = cmk(s_scal[0], s_scal[1]), scale = cmk(s_scal[2], s_scal[3]);
    // v also replaces column c of own packed rows (dead from here on): the
    // reflectors go to C once, at the end, so no global store is pending at a
    // cluster barrier
    for (int i = c + 1 + tid; i < m; i += TT) {
      const cplx v = (i == c + 1) ? cmk(1.0, 0.0) : cmul(xbuf[i], scale);
      vbuf[i] = v;
      if (i % CL == rank) stT(A + row_off<CL>(rank, i / CL) + c, v);  // unit entry explicit
    }
    __syncthreads();
    // own rows from slot s_lo on are the rows >= c + 1
    const int s_lo = (c + 1 > rank) ? (c + 1 - rank + CL - 1) / CL : 0;
    // ---- y = C22 v: the row part of own rows (a warp per row) ---------------
    for (int s = s_lo + warp; s < nslot; s += NW) {
      const int i = rank + CL * s;
      const T2* row = A + row_off<CL>(rank, s);
      // two independent chains per lane
      double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;
      int j = c + 1 + lane;
      for (; j + 32 < i; j += 64) {
        const cplx a0 = ldT(row + j), v0 = vbuf[j];
        const cplx a1 = ldT(row + j + 32), v1 = vbuf[j + 32];
        ar += a0.x * v0.x - a0.y * v0.y;
        ai += a0.x * v0.y + a0.y * v0.x;
        br += a1.x * v1.x - a1.y * v1.y;
        bi += a1.x * v1.y + a1.y * v1.x;
      }
      if (j < i) {
        const cplx a0 = ldT(row + j), v0 = vbuf[j];
        ar += a0.x * v0.x - a0.y * v0.y;
        ai += a0.x * v0.y + a0.y * v0.x;
      }
      ar += br;
      ai += bi;
      for (int o = 16; o > 0; o >>= 1) {
        ar += __shfl_xor_sync(0xffffffffu, ar, o);
        ai += __shfl_xor_sync(0xffffffffu, ai, o);
      }
      if (lane == 0) {
        const double aii = ldT(row + i).x;
        const cplx vi = vbuf[i];
        yrow[s] = cmk(ar + aii * vi.x, ai + aii * vi.y);
      }
    }
    // ---- and the column part: sum over own rows i > j of conj(A_ij) v_i, a
    //      thread per column j, pushed to the owner of row j -----------------
    for (int j = c + 1 + tid; j < m; j += TT) {
      int s = (j >= rank) ? (j - rank) / CL + 1 : 0;  // first own row below j
      long long o = row_off<CL>(rank, s);
      double ar = 0.0, ai = 0.0, br = 0.0, bi = 0.0;  // two rows per step
      for (; s + 1 < nslot; s += 2) {
        const int i0 = rank + CL * s, i1 = i0 + CL;
        const long long o1 = o + i0 + 1;
        const cplx a0 = ldT(A + o + j), v0 = vbuf[i0];
        const cplx a1 = ldT(A + o1 + j), v1 = vbuf[i1];
        ar += a0.x * v0.x + a0.y * v0.y;
        ai += a0.x * v0.y - a0.y * v0.x;
        br += a1.x * v1.x + a1.y * v1.y;
        bi += a1.x * v1.y - a1.y * v1.x;
        o = o1 + i1 + 1;
      }
      if (s < nslot) {
        const int i0 = rank + CL * s;
        const cplx a0 = ldT(A + o + j), v0 = vbuf[i0];
        ar += a0.x * v0.x + a0.y * v0.y;
        ai += a0.x * v0.y - a0.y * v0.x;
      }
      cl.map_shared_rank(ypart, j % CL)[rank * smax + j / CL] = cmk(ar + br, ai + bi);
    }
    cl.sync();
    // ---- own rows: y = row part + every rank's column part; w0 = tau y to
    //      every CTA (a thread per row and target) -----------------------------
    for (int t = s_lo * CL + tid; t < nslot * CL; t += TT) {
      const int s = t / CL, r = t % CL;
      cplx y = yrow[s];
      for (int q = 0; q < CL; ++q) y = cadd(y, ypart[q * smax + s]);
      cl.map_shared_rank(wbuf, r)[rank + CL * s] = cmul(tau, y);
    }
    // and the last warp: Re(v^H y) over own rows to every CTA
    if (warp == NW - 1) {
      double vy = 0.0;
      for (int s = s_lo + lane; s < nslot; s += 32) {
        cplx y = yrow[s];
        for (int q = 0; q < CL; ++q) y = cadd(y, ypart[q * smax + s]);
        const cplx v = vbuf[rank + CL * s];
        vy += v.x * y.x + v.y * y.y;
      }
      for (int o = 16; o > 0; o >>= 1) vy += __shfl_xor_sync(0xffffffffu, vy, o);
      if (lane < CL) cl.map_shared_rank(s_vav, lane)[rank] = vy;
    }
    cl.sync();
    // ---- alpha = -|tau|^2/2 v^H C22 v (real; the panel kernel's form), the
    //      same sum in every CTA; w = w0 + alpha v ------------------------------
    double vav = 0.0;
    for (int q = 0; q < CL; ++q) vav += s_vav[q];
    const double alpha = -0.5 * (tau.x * tau.x + tau.y * tau.y) * vav;
    for (int j = c + 1 + tid; j < m; j += TT) {
      const cplx w = wbuf[j], v = vbuf[j];
      wbuf[j] = cmk(w.x + alpha * v.x, w.y + alpha * v.y);
    }
    __syncthreads();
    // ---- C22 -= v w^H + w v^H on own rows; the updated column c + 1 goes out
    //      at once (x of the next column, d(c + 1)) ----------------------------
    for (int s = s_lo + warp; s < nslot; s += NW) {
      const int i = rank + CL * s;
      T2* row = A + row_off<CL>(rank, s);
      const cplx vi = vbuf[i], wi = wbuf[i];
      // v_i conj(w_j) + w_i conj(v_j) off the diagonal, two entries per step
      int j = c + 1 + lane;
      for (; j + 32 < i; j += 64) {
        const cplx v0 = vbuf[j], w0 = wbuf[j], v1 = vbuf[j + 32], w1 = wbuf[j + 32];
        cplx a0 = ldT(row + j), a1 = ldT(row + j + 32);
        a0.x -= vi.x * w0.x + vi.y * w0.y + wi.x * v0.x + wi.y * v0.y;
        a0.y -= vi.y * w0.x - vi.x * w0.y + wi.y * v0.x - wi.x * v0.y;
        a1.x -= vi.x * w1.x + vi.y * w1.y + wi.x * v1.x + wi.y * v1.y;
        a1.y -= vi.y * w1.x - vi.x * w1.y + wi.y * v1.x - wi.x * v1.y;
        stT(row + j, a0);
        stT(row + j + 32, a1);
      }
      if (j < i) {
        const cplx v0 = vbuf[j], w0 = wbuf[j];
        cplx a0 = ldT(row + j);
        a0.x -= vi.x * w0.x + vi.y * w0.y + wi.x * v0.x + wi.y * v0.y;
        a0.y -= vi.y * w0.x - vi.x * w0.y + wi.y * v0.x - wi.x * v0.y;
        stT(row + j, a0);
      }
      if (lane == 0) {
        cplx a = ldT(row + i);
        a.x -= 2.0 * (vi.x * wi.x + vi.y * wi.y);
        a.y = 0.0;
        stT(row + i, a);
      }
      // lane 0 wrote entry c + 1 of this row (the diagonal when i = c + 1)
      cplx x = cmk(0.0, 0.0);
      if (lane == 0) x = ldT(row + c + 1);  // as stored
      x.x = __shfl_sync(0xffffffffu, x.x, 0);
      x.y = __shfl_sync(0xffffffffu, x.y, 0);
      if (i == c + 1) {
        if (lane == 0) d_loc[s] = x.x;
      } else if (lane < CL) {
        cl.map_shared_rank(xbuf, lane)[i] = x;
      }
    }
  }
  cl.sync();  // no CTA leaves while another may still store into it
  // the reflectors (below the diagonal of own rows), d, e and tau to memory
  for (int s = 0; s < nslot; ++s) {
    const int i = rank + CL * s;
    const T2* row = A + row_off<CL>(rank, s);
    for (int j = tid; j < i; j += TT) {
      const T2 v = row[j];
      C[(c0 + i) + ld * (c0 + j)] = v;
    }
  }
  for (int s = tid; s < nslot; s += TT) {
    const int i = rank + CL * s;
    d[c0 + i] = d_loc[s];
    if (i < m - 1) {
      e[c0 + i] = e_loc[s];
      tau_out[c0 + i] = tau_loc[s];
    }
  }
}

template <typename T2, int CL>
size_t tail_smem(int m) {
  // the packed rows of the rank holding the most entries, and the vectors
  size_t best = 0;
  for (int r = 0; r < CL; ++r) {
    const int ns = (m - r + CL - 1) / CL;
    const long long P = (long long)ns * (r + 1) + (long long)CL * ns * (ns - 1) / 2;
    best = std::max(best, (size_t)P);
  }
  const size_t smax = (m + CL - 1) / CL;
  return sizeof(cplx) * (3 * (size_t)m + (CL + 3) * smax) + best * sizeof(T2);
}

template <typename T2, int CL>
cudaError_t tail_config(cudaLaunchConfig_t* cfg, cudaLaunchAttribute* at, size_t smem, cudaStream_t s) {
  cudaError_t err = cudaSuccess;
  if (CL > 8) err = cudaFuncSetAttribute(k_tridiag_tail<T2, CL>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(k_tridiag_tail<T2, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  *cfg = cudaLaunchConfig_t{};
  cfg->gridDim = dim3(CL);
  cfg->blockDim = dim3(TT);
  cfg->dynamicSmemBytes = smem;
  cfg->stream = s;
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = CL;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg->attrs = at;
  cfg->numAttrs = 1;
  return err;
}

// 16 when a cluster of 16 CTAs at the full shared memory can be resident on
// this device (both storage types), else the portable 8; decided once
int tail_cluster() {
  static const int cl = [] {
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    int n64 = 0, n32 = 0;
    const bool ok = tail_config<double2, 16>(&cfg, at, SMEM_MAX, 0) == cudaSuccess &&
                    cudaOccupancyMaxActiveClusters(&n64, k_tridiag_tail<double2, 16>, &cfg) == cudaSuccess &&
                    tail_config<float2, 16>(&cfg, at, SMEM_MAX, 0) == cudaSuccess &&
                    cudaOccupancyMaxActiveClusters(&n32, k_tridiag_tail<float2, 16>, &cfg) == cudaSuccess;
    cudaGetLastError();  // an unsupported cluster size is not an error of the caller's
    return (ok && n64 >= 1 && n32 >= 1) ? 16 : 8;
  }();
  return cl;
}

template <typename T2, int CL>
int tail_max_cl() {
  int m = 8;
  while (tail_smem<T2, CL>(m + 8) <= SMEM_MAX) m += 8;
  return m;
}

template <typename T2, int CL>
int tail_launch(excfv_handle* h, int n, int c0, T2* C, long long ld) {
  Workspace& ws = h->ws;
  const size_t smem = tail_smem<T2, CL>(n - c0);
  if (smem > SMEM_MAX) return EXCFV_ERR_ARG;
  cudaLaunchConfig_t cfg;
  cudaLaunchAttribute at[1];
  const cudaError_t cerr = tail_config<T2, CL>(&cfg, at, smem, h->stream);
  CUDA_TRY(cerr);
  auto* kern = k_tridiag_tail<T2, CL>;
  CUDA_TRY(cudaLaunchKernelEx(&cfg, kern, n, c0, C, ld, ws.d, ws.e, ws.tau));
  count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

}  // namespace

// the largest tail (m = n - c0) the cluster holds for this storage type
template <typename T2>
int tridiag_tail_max() {
  return tail_cluster() == 16 ? tail_max_cl<T2, 16>() : tail_max_cl<T2, 8>();
}
template int tridiag_tail_max<double2>();
template int tridiag_tail_max<float2>();

// reduces the trailing block C(c0:n, c0:n) (lower triangle, already updated
// by the panels before c0) and leaves reflectors, d, e, tau as the panels do
template <typename T2>
int tridiag_tail(excfv_handle* h, int n, int c0, T2* C, long long ld) {
  if (n - c0 < 2) return EXCFV_ERR_ARG;
  return tail_cluster() == 16 ? tail_launch<T2, 16>(h, n, c0, C, ld) : tail_launch<T2, 8>(h, n, c0, C, ld);
}
template int tridiag_tail<double2>(excfv_handle*, int, int, double2*, long long);
template int tridiag_tail<float2>(excfv_handle*, int, int, float2*, long long);
