// The EVECFV file of first-variational eigenvectors (src/writers/putevecfv.f90,
// read by src/read/getevecfv.f90): a Fortran unformatted direct-access file
// with one fixed-length record per k-point, record ik at byte offset
// (ik - 1) * recl, no record markers, native byte order:
//   vkl(3) real(8) | nmatmax int(4) | nstfv int(4) | nspnfv int(4) |
//   evecfv(nmatmax, nstfv, nspnfv) complex(8)
// recl = 24 + 12 + 16 nmatmax nstfv nspnfv bytes (IoLength in bytes).  The
// writer keeps the reference's record so that files interchange with it; the
// device form copies evecfv from HBM through a pinned staging buffer.
#include <cstdio>
#include <cstring>
#include <vector>

#include "handle.cuh"

namespace {

long long evecfv_recl(int nmatmax, int nstfv, int nspnfv) {
  return 24LL + 12LL + 16LL * nmatmax * nstfv * nspnfv;
}

int write_record(const char* path, int ik, const double* vkl, int nmatmax, int nstfv, int nspnfv,
                 const void* evec) {
  const long long recl = evecfv_recl(nmatmax, nstfv, nspnfv);
  FILE* f = fopen(path, "r+b");
  if (!f) f = fopen(path, "w+b");
  if (!f) {
    excfv_set_error("putevecfv: cannot open %s", path);
    return EXCFV_ERR_ARG;
  }
  int rc = EXCFV_OK;
  const int32_t dims[3] = {nmatmax, nstfv, nspnfv};
  const size_t nev = (size_t)nmatmax * nstfv * nspnfv;
  if (fseeko(f, (off_t)(ik - 1) * recl, SEEK_SET) != 0 || fwrite(vkl, sizeof(double), 3, f) != 3 ||
      fwrite(dims, sizeof(int32_t), 3, f) != 3 || fwrite(evec, 16, nev, f) != nev) {
    excfv_set_error("putevecfv: write of record %d of %s failed", ik, path);
    rc = EXCFV_ERR_ARG;
  }
  if (fclose(f) != 0 && rc == EXCFV_OK) rc = EXCFV_ERR_ARG;
  return rc;
}

}  // namespace

extern "C" {

int excfv_putevecfv(const char* path, int32_t ik, const double* vkl, int32_t nmatmax, int32_t nstfv,
                    int32_t nspnfv, const double* evecfv) {
  if (!path || !vkl || !evecfv || ik < 1 || nmatmax < 1 || nstfv < 1 || nspnfv < 1) return EXCFV_ERR_ARG;
  return write_record(path, ik, vkl, nmatmax, nstfv, nspnfv, evecfv);
}

int excfv_putevecfv_dev(excfv_handle* h, const char* path, int32_t ik, const double* vkl, int32_t nmatmax,
                        int32_t nstfv, int32_t nspnfv, const double* d_evecfv) {
  if (!h || !path || !vkl || !d_evecfv || ik < 1 || nmatmax < 1 || nstfv < 1 || nspnfv < 1)
    return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  const size_t bytes = 16 * (size_t)nmatmax * nstfv * nspnfv;
  Workspace& ws = h->ws;
  if (ws.h_pinned_bytes < bytes) {
    if (ws.h_pinned) cudaFreeHost(ws.h_pinned);
    ws.h_pinned = nullptr;
    ws.h_pinned_bytes = 0;
    CUDA_TRY(cudaMallocHost(&ws.h_pinned, bytes));
    ws.h_pinned_bytes = bytes;
  }
  CUDA_TRY(cudaMemcpyAsync(ws.h_pinned, d_evecfv, bytes, cudaMemcpyDeviceToHost, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return write_record(path, ik, vkl, nmatmax, nstfv, nspnfv, ws.h_pinned);
}

int excfv_getevecfv(const char* path, int32_t ik, const double* vkl, int32_t nmatmax, int32_t nstfv,
                    int32_t nspnfv, double* evecfv) {
  if (!path || !evecfv || ik < 1 || nmatmax < 1 || nstfv < 1 || nspnfv < 1) return EXCFV_ERR_ARG;
  const long long recl = evecfv_recl(nmatmax, nstfv, nspnfv);
  FILE* f = fopen(path, "rb");
  if (!f) {
    excfv_set_error("getevecfv: cannot open %s", path);
    return EXCFV_ERR_ARG;
  }
  double v[3];
  int32_t dims[3];
  const size_t nev = (size_t)nmatmax * nstfv * nspnfv;
  int rc = EXCFV_OK;
  if (fseeko(f, (off_t)(ik - 1) * recl, SEEK_SET) != 0 || fread(v, sizeof(double), 3, f) != 3 ||
      fread(dims, sizeof(int32_t), 3, f) != 3) {
    excfv_set_error("getevecfv: record %d of %s is missing", ik, path);
    rc = EXCFV_ERR_ARG;
  } else if (dims[0] != nmatmax || dims[1] != nstfv || dims[2] != nspnfv) {
    // the reference stops on these mismatches (getevecfv.f90)
    excfv_set_error("getevecfv: record %d holds nmatmax/nstfv/nspnfv %d %d %d, expected %d %d %d", ik, dims[0],
                    dims[1], dims[2], nmatmax, nstfv, nspnfv);
    rc = EXCFV_ERR_ARG;
  } else if (vkl && fabs(v[0] - vkl[0]) + fabs(v[1] - vkl[1]) + fabs(v[2] - vkl[2]) > 1e-6) {
    excfv_set_error("getevecfv: record %d is for k-point (%g %g %g), expected (%g %g %g)", ik, v[0], v[1], v[2],
                    vkl[0], vkl[1], vkl[2]);
    rc = EXCFV_ERR_ARG;
  } else if (fread(evecfv, 16, nev, f) != nev) {
    excfv_set_error("getevecfv: record %d of %s is short", ik, path);
    rc = EXCFV_ERR_ARG;
  }
  fclose(f);
  return rc;
}

}  // extern "C"
