// G+k vectors of a k-point and their structure factors on the device
// (src/gengpvec.f90:43-68 with src/src_lib/sphcrd.f90, src/gensfacgp.f90:40-53),
// so that a k-point's inputs to match / seceqnfv can be formed where they are
// used.  The G vectors are kept in the reference's order (sorted by length);
// the G+k set is their stable compaction by |G + k| < gkmax: per block of
// GB vectors a count (k_gp_count), then each block adds the counts of the
// blocks before it and scans its own flags with warp ballots (k_gp_scatter).
#include "handle.cuh"

namespace {

constexpr int GB = 256;

__device__ __forceinline__ bool gp_inside(const double* vgc, int ig, double3 vpc, double t1, double3* v) {
  v->x = vgc[3 * ig] + vpc.x;
  v->y = vgc[3 * ig + 1] + vpc.y;
  v->z = vgc[3 * ig + 2] + vpc.z;
  const double t2 = v->x * v->x + v->y * v->y + v->z * v->z;
  return t2 < t1;
}

__global__ void __launch_bounds__(GB) k_gp_count(int ngvec, const double* __restrict__ vgc, double3 vpc,
                                                 double t1, int* __restrict__ bcount) {
  const int ig = blockIdx.x * GB + threadIdx.x;
  double3 v;
  const bool in = ig < ngvec && gp_inside(vgc, ig, vpc, t1, &v);
  const int c = __syncthreads_count(in);
  if (threadIdx.x == 0) bcount[blockIdx.x] = c;
}

// sphcrd: length, theta = acos(z / r) (argument clipped to [-1, 1]), phi =
// atan2(y, x) moved to [0, 2 pi); both angles 0 below r = 1e-14, phi 0 when
// |x| and |y| are both at most 1e-14
__device__ __forceinline__ void sphcrd_d(double3 v, double* r, double* th, double* ph) {
  const double eps = 1e-14;
  *r = sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
  *th = 0.0;
  *ph = 0.0;
  if (*r > eps) {
    double t = v.z / *r;
    t = (t > 0.0) ? fmin(t, 1.0) : fmax(t, -1.0);
    *th = acos(t);
    if (fabs(v.x) > eps || fabs(v.y) > eps) {
      *ph = atan2(v.y, v.x);
      if (*ph < 0.0) *ph += 6.2831853071795864769;
    }
  }
}

__global__ void __launch_bounds__(GB) k_gp_scatter(int ngvec, const double* __restrict__ vgc,
                                                   const int* __restrict__ ivg, double3 vpl, double3 vpc,
                                                   double t1, const int* __restrict__ bcount, int nblk,
                                                   int ngkmax, int* __restrict__ igpig, double* __restrict__ vgpl,
                                                   double* __restrict__ vgpc, double* __restrict__ gpc,
                                                   double* __restrict__ tpgpc, int* __restrict__ ngp) {
  __shared__ int s_warp[GB / 32];
  __shared__ int s_base;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  if (tid == 0) {
    int b = 0;
    for (int q = 0; q < (int)blockIdx.x; ++q) b += bcount[q];
    s_base = b;
  }
  const int ig = blockIdx.x * GB + tid;
  double3 v;
  const bool in = ig < ngvec && gp_inside(vgc, ig, vpc, t1, &v);
  const unsigned ball = __ballot_sync(0xffffffffu, in);
  if (lane == 0) s_warp[w] = __popc(ball);
  __syncthreads();
  int before = s_base;
  for (int q = 0; q < w; ++q) before += s_warp[q];
  before += __popc(ball & ((1u << lane) - 1u));
  if (in) {
    if (before < ngkmax) {
      igpig[before] = ig + 1;
      vgpl[3 * before] = (double)ivg[3 * ig] + vpl.x;
      vgpl[3 * before + 1] = (double)ivg[3 * ig + 1] + vpl.y;
      vgpl[3 * before + 2] = (double)ivg[3 * ig + 2] + vpl.z;
      vgpc[3 * before] = v.x;
      vgpc[3 * before + 1] = v.y;
      vgpc[3 * before + 2] = v.z;
      double r, th, ph;
      sphcrd_d(v, &r, &th, &ph);
      gpc[before] = r;
      tpgpc[2 * before] = th;
      tpgpc[2 * before + 1] = ph;
    }
  }
  // the count; negative when the set does not fit ngkmax
  if (blockIdx.x == nblk - 1 && tid == GB - 1) {
    int tot = s_base;
    for (int q = 0; q < GB / 32; ++q) tot += s_warp[q];
    *ngp = (tot > ngkmax) ? -tot : tot;
  }
}

// sfacgp(igp, ias) = exp(i (G+k) . r_ias)
__global__ void k_sfacgp(int ngp, int natmtot, const double* __restrict__ vgpc, const double* __restrict__ atposc,
                         long long ld, cplx* __restrict__ sfacgp) {
  const int igp = blockIdx.x * blockDim.x + threadIdx.x;
  const int ias = blockIdx.y;
  if (igp >= ngp || ias >= natmtot) return;
  const double t = vgpc[3 * igp] * atposc[3 * ias] + vgpc[3 * igp + 1] * atposc[3 * ias + 1] +
                   vgpc[3 * igp + 2] * atposc[3 * ias + 2];
  double sn, cs;
  sincos(t, &sn, &cs);
  sfacgp[igp + ld * ias] = cmk(cs, sn);
}

}  // namespace

// G vectors in Cartesian coordinates, vgc(3, ngvec), and atomic positions,
// atposc(3, natmtot) (mod_Gvector, mod_atoms), for the device G+k set.
int stage_set_lattice(excfv_handle* h, const double* vgc, const double* atposc) {
  DevStatic& st = h->st;
  if (st.ngvec <= 0 || st.natmtot <= 0) return EXCFV_ERR_STATE;
  cudaFree(st.vgc);
  cudaFree(st.atposc);
  cudaFree(st.gkcount);
  st.vgc = nullptr;
  st.atposc = nullptr;
  st.gkcount = nullptr;
  CUDA_TRY(cudaMalloc(&st.vgc, sizeof(double) * 3 * (size_t)st.ngvec));
  CUDA_TRY(cudaMalloc(&st.atposc, sizeof(double) * 3 * (size_t)st.natmtot));
  CUDA_TRY(cudaMemcpy(st.vgc, vgc, sizeof(double) * 3 * (size_t)st.ngvec, cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(st.atposc, atposc, sizeof(double) * 3 * (size_t)st.natmtot, cudaMemcpyHostToDevice));
  const int nblk = (st.ngvec + GB - 1) / GB;
  CUDA_TRY(cudaMalloc(&st.gkcount, sizeof(int) * (size_t)(nblk + 2)));
  st.have_lattice = true;
  return EXCFV_OK;
}

// The G+k set of k-point vpl (Cartesian vpc) into device arrays; *d_ngp
// (device) receives the count, negated when it exceeds ngkmax.
int stage_gengpvec(excfv_handle* h, const double* vpl, const double* vpc, double gkmax, int ngkmax,
                   int* d_ngp, int* igpig, double* vgpl, double* vgpc, double* gpc, double* tpgpc) {
  const DevStatic& st = h->st;
  cudaStream_t s = h->stream;
  const int nblk = (st.ngvec + GB - 1) / GB;
  const double t1 = gkmax * gkmax;
  const double3 pl = make_double3(vpl[0], vpl[1], vpl[2]);
  const double3 pc = make_double3(vpc[0], vpc[1], vpc[2]);
  k_gp_count<<<nblk, GB, 0, s>>>(st.ngvec, st.vgc, pc, t1, st.gkcount); count_launch();
  CUDA_TRY(cudaGetLastError());
  k_gp_scatter<<<nblk, GB, 0, s>>>(st.ngvec, st.vgc, st.ivg, pl, pc, t1, st.gkcount, nblk, ngkmax, igpig, vgpl,
                                   vgpc, gpc, tpgpc, d_ngp); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}

int stage_gensfacgp(excfv_handle* h, int ngp, const double* vgpc, long long ld, cplx* sfacgp) {
  const DevStatic& st = h->st;
  k_sfacgp<<<dim3((ngp + 127) / 128, st.natmtot), 128, 0, h->stream>>>(ngp, st.natmtot, vgpc, st.atposc, ld,
                                                                        sfacgp); count_launch();
  CUDA_TRY(cudaGetLastError());
  return EXCFV_OK;
}
