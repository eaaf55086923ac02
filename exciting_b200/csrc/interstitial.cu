// Interstitial Fourier coefficients of the effective potential and the
// (scalar-relativistic) inverse mass on the device: genveffig
// (src/genveffig.f90:26-40) and genmeffig (src/genmeffig.f90:24-58).
//
//   veffig(G)  = FFT[ veffir cfunir ](G)
//   meffig(G)  = FFT[ cfunir / (1 - a2 veffir) ](G)        (ValenceRelativity != none)
//   m2effig(G) = FFT[ cfunir / (1 - a2 veffir)^2 ](G)      (IORA*)
// with a2 = alpha^2 / 2 and FFT the forward transform exp(-i G.r) over the
// real-space grid ngrid(3) divided by its size (zfftifc(3, ngrid, -1, .)),
// read at igfft(G) (gengvec.f90 genigfft: negative components wrapped by
// +ngrid).  The grid (tens of points per axis, any factorisation) is
// transformed axis by axis as a direct DFT: one block per line, the line in
// shared memory, one output per thread, exact twiddles exp(-2 pi i (k j mod
// n) / n) from sincospi.  The results go straight into the handle's veffig,
// meffig (the hmlistln kinetic factor when ValenceRelativity != none) and
// m2effig, which the next setup reads.
#include <vector>

#include "handle.cuh"

namespace {

constexpr double A2 = 0.5 / (137.03599911 * 137.03599911);
constexpr int DFT_NMAX = 1024;

// zfft = f(veffir, cfunir) on the whole grid; kind 3: (v + c0) cfunir (the
// interstitial magnetic field of seceqnsv.f90:660-668)
__global__ void k_ir_prepare(long long n, int kind, const double* veffir, const double* cfunir, double c0,
                             cplx* z) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = veffir[i], c = cfunir[i];
  double r;
  if (kind == 0) r = v * c;
  else if (kind == 1) r = c / (1.0 - v * A2);
  else if (kind == 2) {
    const double t = 1.0 - v * A2;
    r = c / (t * t);
  } else r = (v + c0) * c;
  z[i] = cmk(r, 0.0);
}

__global__ void k_ir_scale(long long n, double scale, const cplx* z, cplx* out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = cmk(z[i].x * scale, z[i].y * scale);
}

// forward DFT along one axis of the column-major grid: lines of length n with
// element stride `stride`; line l starts at (l % stride) + (l / stride) * stride * n
__global__ void k_dft_axis(int n, long long stride, long long nlines, const cplx* in, cplx* out) {
  __shared__ cplx line[DFT_NMAX];
  __shared__ cplx tw[DFT_NMAX];
  for (long long l = blockIdx.x; l < nlines; l += gridDim.x) {
    const long long base = (l % stride) + (l / stride) * stride * n;
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
      line[j] = in[base + j * stride];
      double s, c;
      sincospi(-2.0 * (double)j / (double)n, &s, &c);
      tw[j] = cmk(c, s);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
      double re = 0.0, im = 0.0;
      int e = 0;  // (k * j) mod n
      for (int j = 0; j < n; ++j) {
        const cplx a = line[j], w = tw[e];
        re += a.x * w.x - a.y * w.y;
        im += a.x * w.y + a.y * w.x;
        e += k;
        if (e >= n) e -= n;
      }
      out[base + k * stride] = cmk(re, im);
    }
    __syncthreads();
  }
}

// out(ig) = z(igfft(ig)) / N for ig < ngvec
__global__ void k_ir_gather(int ngvec, const int* ivg, int n1, int n2, int n3, double scale, const cplx* z,
                            cplx* out) {
  const int ig = blockIdx.x * blockDim.x + threadIdx.x;
  if (ig >= ngvec) return;
  int j1 = ivg[3 * ig], j2 = ivg[3 * ig + 1], j3 = ivg[3 * ig + 2];
  if (j1 < 0) j1 += n1;
  if (j2 < 0) j2 += n2;
  if (j3 < 0) j3 += n3;
  const cplx v = z[(long long)j1 + (long long)n1 * (j2 + (long long)n2 * j3)];
  out[ig] = cmk(v.x * scale, v.y * scale);
}

}  // namespace

// kinds: 0 veffig, 1 meffig, 2 m2effig; host copies optional
int stage_genfig(excfv_handle* h, const int* ngrid, const double* veffir, const double* cfunir, int nkinds,
                 const int* kinds, cplx* const* dst, cplx* const* host_out) {
  DevStatic& st = h->st;
  cudaStream_t s = h->stream;
  const int n1 = ngrid[0], n2 = ngrid[1], n3 = ngrid[2];
  if (n1 < 1 || n2 < 1 || n3 < 1 || n1 > DFT_NMAX || n2 > DFT_NMAX || n3 > DFT_NMAX) {
    excfv_set_error("genveffig: ngrid (%d %d %d) outside 1..%d", n1, n2, n3, DFT_NMAX);
    return EXCFV_ERR_ARG;
  }
  // every G vector of the list must land on the grid (genigfft)
  const int e[3] = {st.intgv[3] - st.intgv[0] + 1, st.intgv[4] - st.intgv[1] + 1, st.intgv[5] - st.intgv[2] + 1};
  for (int d = 0; d < 3; ++d)
    if (ngrid[d] < e[d] || st.intgv[d] < -(ngrid[d] - 1) || st.intgv[3 + d] > ngrid[d] - 1) {
      excfv_set_error("genveffig: ngrid(%d) = %d does not hold the G-vector box %d..%d", d + 1, ngrid[d],
                      st.intgv[d], st.intgv[3 + d]);
      return EXCFV_ERR_ARG;
    }
  const long long N = (long long)n1 * n2 * n3;
  double *d_v = nullptr, *d_c = nullptr;
  cplx *z0 = nullptr, *z1 = nullptr;
  int rc = EXCFV_OK;
  auto fail = [&](cudaError_t err) {
    excfv_set_error("genveffig: %s", cudaGetErrorString(err));
    rc = EXCFV_ERR_CUDA;
  };
  cudaError_t err;
  if ((err = cudaMalloc(&d_v, sizeof(double) * N)) != cudaSuccess ||
      (err = cudaMalloc(&d_c, sizeof(double) * N)) != cudaSuccess ||
      (err = cudaMalloc(&z0, sizeof(cplx) * N)) != cudaSuccess ||
      (err = cudaMalloc(&z1, sizeof(cplx) * N)) != cudaSuccess ||
      (err = cudaMemcpyAsync(d_v, veffir, sizeof(double) * N, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (err = cudaMemcpyAsync(d_c, cfunir, sizeof(double) * N, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
    fail(err);
  } else {
    const unsigned gb = (unsigned)((N + 255) / 256);
    for (int q = 0; q < nkinds && rc == EXCFV_OK; ++q) {
      k_ir_prepare<<<gb, 256, 0, s>>>(N, kinds[q], d_v, d_c, 0.0, z0);
      count_launch();
      const long long nl1 = N / n1, nl2 = N / n2, nl3 = N / n3;
      auto grid = [](long long nl) { return (unsigned)std::min<long long>(nl, 148LL * 16); };
      k_dft_axis<<<grid(nl1), 64, 0, s>>>(n1, 1, nl1, z0, z1);
      count_launch();
      k_dft_axis<<<grid(nl2), 64, 0, s>>>(n2, n1, nl2, z1, z0);
      count_launch();
      k_dft_axis<<<grid(nl3), 64, 0, s>>>(n3, (long long)n1 * n2, nl3, z0, z1);
      count_launch();
      k_ir_gather<<<(st.ngvec + 255) / 256, 256, 0, s>>>(st.ngvec, st.ivg, n1, n2, n3, 1.0 / (double)N, z1,
                                                         dst[q]);
      count_launch();
      if ((err = cudaGetLastError()) != cudaSuccess) {
        fail(err);
        break;
      }
      if (host_out && host_out[q] &&
          (err = cudaMemcpyAsync(host_out[q], dst[q], sizeof(cplx) * st.ngvec, cudaMemcpyDeviceToHost, s)) !=
              cudaSuccess)
        fail(err);
    }
  }
  cudaError_t serr = cudaStreamSynchronize(s);
  if (rc == EXCFV_OK && serr != cudaSuccess) fail(serr);
  cudaFree(d_v);
  cudaFree(d_c);
  cudaFree(z0);
  cudaFree(z1);
  return rc;
}

// the forward transform (divided by the grid size) of (f + c0) cfunir over
// the whole grid into dst (ngrtot complex, device): the Fourier coefficients
// of the interstitial field whose product with a wavefunction seceqnsv forms
// by zfftifc(+1), a multiplication and zfftifc(-1)
int stage_grid_field(excfv_handle* h, const int* ngrid, const double* f, const double* cfunir, double c0,
                     cplx* dst) {
  cudaStream_t s = h->stream;
  const int n1 = ngrid[0], n2 = ngrid[1], n3 = ngrid[2];
  if (n1 < 1 || n2 < 1 || n3 < 1 || n1 > DFT_NMAX || n2 > DFT_NMAX || n3 > DFT_NMAX) {
    excfv_set_error("interstitial field: ngrid (%d %d %d) outside 1..%d", n1, n2, n3, DFT_NMAX);
    return EXCFV_ERR_ARG;
  }
  const long long N = (long long)n1 * n2 * n3;
  double *d_v = nullptr, *d_c = nullptr;
  cplx *z0 = nullptr, *z1 = nullptr;
  int rc = EXCFV_OK;
  cudaError_t err;
  if ((err = cudaMalloc(&d_v, sizeof(double) * N)) != cudaSuccess ||
      (err = cudaMalloc(&d_c, sizeof(double) * N)) != cudaSuccess ||
      (err = cudaMalloc(&z0, sizeof(cplx) * N)) != cudaSuccess ||
      (err = cudaMalloc(&z1, sizeof(cplx) * N)) != cudaSuccess ||
      (err = cudaMemcpyAsync(d_v, f, sizeof(double) * N, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (err = cudaMemcpyAsync(d_c, cfunir, sizeof(double) * N, cudaMemcpyHostToDevice, s)) != cudaSuccess) {
    excfv_set_error("interstitial field: %s", cudaGetErrorString(err));
    rc = EXCFV_ERR_CUDA;
  } else {
    const unsigned gb = (unsigned)((N + 255) / 256);
    k_ir_prepare<<<gb, 256, 0, s>>>(N, 3, d_v, d_c, c0, z0);
    count_launch();
    const long long nl1 = N / n1, nl2 = N / n2, nl3 = N / n3;
    auto grid = [](long long nl) { return (unsigned)std::min<long long>(nl, 148LL * 16); };
    k_dft_axis<<<grid(nl1), 64, 0, s>>>(n1, 1, nl1, z0, z1);
    count_launch();
    k_dft_axis<<<grid(nl2), 64, 0, s>>>(n2, n1, nl2, z1, z0);
    count_launch();
    k_dft_axis<<<grid(nl3), 64, 0, s>>>(n3, (long long)n1 * n2, nl3, z0, z1);
    count_launch();
    k_ir_scale<<<gb, 256, 0, s>>>(N, 1.0 / (double)N, z1, dst);
    count_launch();
    if ((err = cudaGetLastError()) != cudaSuccess) {
      excfv_set_error("interstitial field: %s", cudaGetErrorString(err));
      rc = EXCFV_ERR_CUDA;
    }
  }
  if (cudaStreamSynchronize(s) != cudaSuccess && rc == EXCFV_OK) rc = EXCFV_ERR_CUDA;
  cudaFree(d_v);
  cudaFree(d_c);
  cudaFree(z0);
  cudaFree(z1);
  return rc;
}
