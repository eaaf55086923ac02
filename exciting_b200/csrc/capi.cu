// C ABI of libexcfv (include/excfv.h): handle lifetime, per-SCF-iteration
// data upload, workspace, and the drop-ins for match / hamiltonandoverlapsetup
// / solvewithlapack / seceqnfv / seceqn.
#include <cstdarg>
#include <cstring>
#include <vector>
#include <chrono>
#include <atomic>

#include <algorithm>
#include "handle.cuh"

int match_compute_zdinv(DevStatic& st, const double* d_sprwin, const double* d_apwfrwin,
                        cudaStream_t s);
int mirror_upper(cudaStream_t s, int n, cplx* M, long long ld);
size_t tridiag_eig_scratch_doubles(int n, int k);
int tridiag_workspace_doubles();
int tridiag_nb();

namespace {
thread_local char g_err[512] = "";

template <typename T>
int dalloc(T** p, size_t count) {
  *p = nullptr;
  if (count == 0) count = 1;
  cudaError_t e = cudaMalloc((void**)p, count * sizeof(T));
  if (e != cudaSuccess) {
    excfv_set_error("cudaMalloc of %zu bytes failed: %s", count * sizeof(T), cudaGetErrorString(e));
    *p = nullptr;
    return EXCFV_ERR_ALLOC;
  }
  return EXCFV_OK;
}

template <typename T>
int upload(T** p, const void* host, size_t count) {
  int rc = dalloc(p, count);
  if (rc) return rc;
  if (host) {
    cudaError_t e = cudaMemcpy(*p, host, count * sizeof(T), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      excfv_set_error("upload: %s", cudaGetErrorString(e));
      return EXCFV_ERR_CUDA;
    }
  } else {
    cudaMemset(*p, 0, count * sizeof(T));
  }
  return EXCFV_OK;
}

template <typename T>
void dfree(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}



double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

static std::atomic<long long> g_launches{0};
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

static std::atomic<long long> g_wait_ns{2000000000LL};
static std::atomic<int> g_planted{0};
long long wait_limit_ns() { return g_wait_ns.load(std::memory_order_relaxed); }
bool take_planted_stall() { return g_planted.exchange(0) != 0; }

void prof_begin(excfv_handle* h, int cls) {
  Prof& p = h->prof;
  if (!p.on) return;
  auto& v = p.ev[cls];
  while (v.size() < p.used[cls] + 2) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return;
    v.push_back(e);
  }
  cudaEventRecord(v[p.used[cls]], h->stream);
}

void prof_end(excfv_handle* h, int cls) {
  Prof& p = h->prof;
  if (!p.on || p.ev[cls].size() < p.used[cls] + 2) return;
  cudaEventRecord(p.ev[cls][p.used[cls] + 1], h->stream);
  p.used[cls] += 2;
}

void prof_collect(excfv_handle* h) {
  Prof& p = h->prof;
  cudaStreamSynchronize(h->stream);
  for (int c = 0; c < PROF_NCLS; ++c) {
    for (size_t i = 0; i + 1 < p.used[c]; i += 2) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, p.ev[c][i], p.ev[c][i + 1]) == cudaSuccess) p.ms[c] += ms;
      p.cnt[c] += 1;
    }
    p.used[c] = 0;
  }
}

void excfv_set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}

void free_static(DevStatic& st) {
  dfree(st.idxis); dfree(st.rmt); dfree(st.apword); dfree(st.flist); dfree(st.fofl);
  dfree(st.lo_atom); dfree(st.lo_local); dfree(st.lo_lm); dfree(st.lo_ilo);
  dfree(st.aa); dfree(st.loa); dfree(st.lolo); dfree(st.oalo); dfree(st.ololo); dfree(st.h1aa);
  dfree(st.ivg); dfree(st.ivgig); dfree(st.veffig); dfree(st.xig); dfree(st.cfunig);
  dfree(st.m2effig); dfree(st.zdinv);
  dfree(st.vgc); dfree(st.atposc); dfree(st.gkcount);
  st.have_lattice = false;
}

void free_workspace(Workspace& ws) {
  dfree(ws.H); dfree(ws.O); dfree(ws.Ui); dfree(ws.T); dfree(ws.Apk); dfree(ws.Zpk);
  dfree(ws.ylm); dfree(ws.djl); dfree(ws.apwalm); dfree(ws.igpig); dfree(ws.vgpc); dfree(ws.gpc);
  dfree(ws.tpgpc); dfree(ws.sfacgp); dfree(ws.gk_iv); dfree(ws.d); dfree(ws.e); dfree(ws.tau);
  dfree(ws.Wp); dfree(ws.red); dfree(ws.w); dfree(ws.stein_ws); dfree(ws.icl); dfree(ws.ybuf);
  dfree(ws.Z); dfree(ws.Z2); dfree(ws.Gk); dfree(ws.Gki); dfree(ws.Tf); dfree(ws.Xs);
  dfree(ws.status); dfree(ws.bar); dfree(ws.part); dfree(ws.prog); dfree(ws.slices); dfree(ws.slice_sc);
  ws.slices_elems = ws.slice_sc_n = 0;
  if (ws.h_pinned) cudaFreeHost(ws.h_pinned);
  ws.h_pinned = nullptr;
  ws.h_pinned_bytes = 0;
  ws.part_cap = 0;
  ws.nmatmax = ws.ngkmax = ws.kmax = 0;
}

int stage_set_static(excfv_handle* h, const excfv_static* s) {
  DevStatic& st = h->st;
  h->static_gen++;
  free_static(st);
  h->have_static = false;
  if (!s || s->natmtot <= 0 || s->nspecies <= 0 || s->lmaxapw < 0 || s->apwordmax <= 0 ||
      s->maxaa <= 0 || s->ngvec <= 0 || s->ngrtot < s->ngvec || s->nstfv <= 0 || !s->idxis ||
      !s->rmt || !s->apword || !s->ivg || !s->ivgig || !s->veffig || !s->cfunig ||
      !s->sprwin || !s->apwfrwin || s->npmatch <= 0) {
    excfv_set_error("excfv_set_static: missing or inconsistent arguments");
    return EXCFV_ERR_ARG;
  }
  if (s->lmaxmat > s->lmaxapw) {
    excfv_set_error("excfv_set_static: lmaxmat > lmaxapw");
    return EXCFV_ERR_ARG;
  }
  st.natmtot = s->natmtot; st.nspecies = s->nspecies; st.lmaxapw = s->lmaxapw;
  st.lmaxmat = s->lmaxmat; st.lmmaxapw = (s->lmaxapw + 1) * (s->lmaxapw + 1);
  st.apwordmax = s->apwordmax; st.nlomax = s->nlomax; st.lolmmax = (s->lolmax + 1) * (s->lolmax + 1);
  st.nlotot = s->nlotot; st.maxaa = s->maxaa; st.maxnlo = s->maxnlo; st.ngvec = s->ngvec;
  st.ngrtot = s->ngrtot; st.h1on = s->h1on; st.vrel = s->valence_relativity;
  st.npmatch = s->npmatch; st.omega = s->omega; st.nstfv = s->nstfv; st.evaltol = s->evaltol;
  for (int i = 0; i < 6; ++i) st.intgv[i] = s->intgv[i];
  const int na = st.natmtot, ns = st.nspecies;
  int rc;
  // species (0-based)
  std::vector<int> idxis(na);
  for (int a = 0; a < na; ++a) {
    idxis[a] = s->idxis[a] - 1;
    if (idxis[a] < 0 || idxis[a] >= ns) {
      excfv_set_error("excfv_set_static: idxis out of range");
      return EXCFV_ERR_ARG;
    }
  }
  // packed APW function list per species (hamiltonsetup.f90:62-71)
  const int L1 = st.lmaxapw + 1;
  std::vector<int> flist((size_t)st.maxaa * ns, -1), fofl((size_t)st.lmmaxapw * st.apwordmax * ns, -1);
  for (int is = 0; is < ns; ++is) {
    int f = 0;
    for (int l = 0; l <= st.lmaxmat; ++l)
      for (int m = -l; m <= l; ++m) {
        const int lm = l * (l + 1) + m;
        const int nap = s->apword[l + L1 * is];
        if (nap > st.apwordmax || nap < 0) {
          excfv_set_error("excfv_set_static: apword > apwordmax");
          return EXCFV_ERR_ARG;
        }
        for (int io = 0; io < nap; ++io) {
          if (f >= st.maxaa) {
            excfv_set_error("excfv_set_static: maxaa too small for apword/lmaxmat");
            return EXCFV_ERR_ARG;
          }
          flist[f + (size_t)st.maxaa * is] = lm * st.apwordmax + io;
          fofl[(lm * st.apwordmax + io) + (size_t)st.lmmaxapw * st.apwordmax * is] = f;
          ++f;
        }
      }
  }
  // local-orbital maps (genidxlo.f90:32-44)
  std::vector<int> lo_atom(std::max(1, st.nlotot), -1), lo_local(std::max(1, st.nlotot), -1);
  std::vector<int> lo_lm((size_t)std::max(1, st.maxnlo) * na, -1), lo_ilo((size_t)std::max(1, st.maxnlo) * na, -1);
  if (st.nlotot > 0) {
    if (!s->nlorb || !s->lorbl || !s->idxlo || !s->losize) {
      excfv_set_error("excfv_set_static: local-orbital arrays missing");
      return EXCFV_ERR_ARG;
    }
    st.h_lo_first.assign(na, -1);
    for (int a = 0; a < na; ++a) {
      const int is = idxis[a];
      int first = -1;
      for (int ilo = 0; ilo < s->nlorb[is]; ++ilo) {
        const int l = s->lorbl[ilo + st.nlomax * is];
        for (int m = -l; m <= l; ++m) {
          const int lm = l * (l + 1) + m;
          const int g = s->idxlo[lm + st.lolmmax * (ilo + (size_t)st.nlomax * a)] - 1;
          if (g < 0 || g >= st.nlotot) {
            excfv_set_error("excfv_set_static: idxlo out of range");
            return EXCFV_ERR_ARG;
          }
          if (first < 0 || g < first) first = g;
        }
      }
      for (int ilo = 0; ilo < s->nlorb[is]; ++ilo) {
        const int l = s->lorbl[ilo + st.nlomax * is];
        for (int m = -l; m <= l; ++m) {
          const int lm = l * (l + 1) + m;
          const int g = s->idxlo[lm + st.lolmmax * (ilo + (size_t)st.nlomax * a)] - 1;
          const int jj = g - first;
          if (jj >= st.maxnlo) {
            excfv_set_error("excfv_set_static: LO block larger than maxnlo");
            return EXCFV_ERR_ARG;
          }
          st.h_lo_first[a] = first;
          lo_atom[g] = a;
          lo_local[g] = jj;
          lo_lm[jj + (size_t)st.maxnlo * a] = lm;
          lo_ilo[jj + (size_t)st.maxnlo * a] = ilo;
        }
      }
    }
    for (int g = 0; g < st.nlotot; ++g)
      if (lo_atom[g] < 0) {
        excfv_set_error("excfv_set_static: idxlo does not cover 1..nlotot");
        return EXCFV_ERR_ARG;
      }
  }
  // overlap radial integrals with the IORA* terms folded in
  const size_t noalo = (size_t)st.apwordmax * std::max(1, st.nlomax) * na;
  const size_t nololo = (size_t)std::max(1, st.nlomax) * std::max(1, st.nlomax) * na;
  std::vector<double> oalo(noalo, 0.0), ololo(nololo, 0.0);
  if (st.nlotot > 0) {
    for (size_t i = 0; i < noalo; ++i) oalo[i] = (s->oalo ? s->oalo[i] : 0.0) + (s->h1loa ? s->h1loa[i] : 0.0);
    for (size_t i = 0; i < nololo; ++i)
      ololo[i] = (s->ololo ? s->ololo[i] : 0.0) + (s->h1lolo ? s->h1lolo[i] : 0.0);
  }
  st.have_h1aa = false;
  const size_t nh1 = (size_t)st.apwordmax * st.apwordmax * L1 * na;
  if (s->h1aa)
    for (size_t i = 0; i < nh1; ++i)
      if (s->h1aa[i] != 0.0) { st.have_h1aa = true; break; }
  const int e1 = s->intgv[3] - s->intgv[0] + 1, e2 = s->intgv[4] - s->intgv[1] + 1,
            e3 = s->intgv[5] - s->intgv[2] + 1;
  if (e1 <= 0 || e2 <= 0 || e3 <= 0) {
    excfv_set_error("excfv_set_static: empty intgv box");
    return EXCFV_ERR_ARG;
  }
  const size_t nbox = (size_t)e1 * e2 * e3;
  const size_t maxnlo1 = std::max(1, st.maxnlo);
  st.h_idxis = idxis;
  st.h_apword.assign(s->apword, s->apword + (size_t)L1 * ns);
  st.h_nlorb.assign(ns, 0);
  st.h_lorbl.assign((size_t)std::max(1, st.nlomax) * ns, 0);
  if (s->nlorb && s->lorbl)
    for (int is = 0; is < ns; ++is) {
      st.h_nlorb[is] = s->nlorb[is];
      for (int ilo = 0; ilo < s->nlorb[is] && ilo < st.nlomax; ++ilo)
        st.h_lorbl[ilo + (size_t)std::max(1, st.nlomax) * is] = s->lorbl[ilo + (size_t)st.nlomax * is];
    }
  if ((rc = upload(&st.idxis, idxis.data(), na))) return rc;
  if ((rc = upload(&st.rmt, s->rmt, ns))) return rc;
  if ((rc = upload(&st.apword, s->apword, (size_t)L1 * ns))) return rc;
  if ((rc = upload(&st.flist, flist.data(), flist.size()))) return rc;
  if ((rc = upload(&st.fofl, fofl.data(), fofl.size()))) return rc;
  if ((rc = upload(&st.lo_atom, lo_atom.data(), lo_atom.size()))) return rc;
  if ((rc = upload(&st.lo_local, lo_local.data(), lo_local.size()))) return rc;
  if ((rc = upload(&st.lo_lm, lo_lm.data(), lo_lm.size()))) return rc;
  if ((rc = upload(&st.lo_ilo, lo_ilo.data(), lo_ilo.size()))) return rc;
  if ((rc = upload(&st.aa, s->aa, (size_t)st.maxaa * st.maxaa * na))) return rc;
  if ((rc = upload(&st.loa, st.nlotot ? s->loa : nullptr, maxnlo1 * st.maxaa * na))) return rc;
  if ((rc = upload(&st.lolo, st.nlotot ? s->lolo : nullptr, maxnlo1 * maxnlo1 * na))) return rc;
  // upload(nullptr) zero-fills: a NULL aa / loa / lolo waits for excfv_hmlint
  if ((rc = upload(&st.oalo, oalo.data(), noalo))) return rc;
  if ((rc = upload(&st.ololo, ololo.data(), nololo))) return rc;
  if (st.have_h1aa && (rc = upload(&st.h1aa, s->h1aa, nh1))) return rc;
  if ((rc = upload(&st.ivg, s->ivg, (size_t)3 * st.ngrtot))) return rc;
  if ((rc = upload(&st.ivgig, s->ivgig, nbox))) return rc;
  if ((rc = upload(&st.veffig, s->veffig, st.ngvec))) return rc;
  const double* xsrc = (st.vrel != 0) ? s->meffig : s->cfunig;
  if (!xsrc) {
    excfv_set_error("excfv_set_static: meffig required when valence_relativity != 0");
    return EXCFV_ERR_ARG;
  }
  if ((rc = upload(&st.xig, xsrc, st.ngvec))) return rc;
  if ((rc = upload(&st.cfunig, s->cfunig, st.ngvec))) return rc;
  if (st.h1on && !s->m2effig) {
    excfv_set_error("excfv_set_static: m2effig required when h1on");
    return EXCFV_ERR_ARG;
  }
  if ((rc = upload(&st.m2effig, st.h1on ? s->m2effig : nullptr, st.ngvec))) return rc;
  if ((rc = dalloc(&st.zdinv, (size_t)st.apwordmax * st.apwordmax * L1 * na))) return rc;
  double *d_spr = nullptr, *d_apwfr = nullptr;
  if ((rc = upload(&d_spr, s->sprwin, (size_t)st.npmatch * ns))) return rc;
  if ((rc = upload(&d_apwfr, s->apwfrwin, (size_t)st.npmatch * st.apwordmax * L1 * na))) return rc;
  rc = match_compute_zdinv(st, d_spr, d_apwfr, h->stream);
  cudaStreamSynchronize(h->stream);
  cudaFree(d_spr);
  cudaFree(d_apwfr);
  if (rc) return rc;
  h->have_static = true;
  return EXCFV_OK;
}

int stage_reserve(excfv_handle* h, int nmatmax, int ngkmax, int kmax) {
  Workspace& ws = h->ws;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  // the precision form carries extra states through the eigensolver
  if (h->prec == EXCFV_PREC_MIXED) kmax = mixed_states(nmatmax, kmax);
  const bool want_slices = (h->prec == EXCFV_PREC_MIXED);
  if (nmatmax <= ws.nmatmax && ngkmax <= ws.ngkmax && kmax <= ws.kmax && ws.H && (!want_slices || ws.slices))
    return EXCFV_OK;
  nmatmax = std::max(nmatmax, ws.nmatmax);
  ngkmax = std::max(ngkmax, ws.ngkmax);
  kmax = std::max(kmax, ws.kmax);
  cudaStreamSynchronize(h->stream);
  free_workspace(ws);
  const DevStatic& st = h->st;
  const size_t n = nmatmax, n2 = n * n, AM = (size_t)st.natmtot * st.maxaa;
  const size_t K = kmax;
  int rc;
  if ((rc = dalloc(&ws.H, n2)) || (rc = dalloc(&ws.O, n2)) || (rc = dalloc(&ws.Ui, n2)) ||
      (rc = dalloc(&ws.T, n2)) || (rc = dalloc(&ws.Apk, AM * ngkmax)) ||
      (rc = dalloc(&ws.Zpk, AM * ngkmax)) || (rc = dalloc(&ws.ylm, (size_t)st.lmmaxapw * ngkmax)) ||
      (rc = dalloc(&ws.djl, (size_t)ngkmax * (st.lmaxapw + 1) * st.apwordmax * st.nspecies)) ||
      (rc = dalloc(&ws.apwalm, (size_t)ngkmax * st.apwordmax * st.lmmaxapw * st.natmtot)) ||
      (rc = dalloc(&ws.igpig, (size_t)ngkmax)) || (rc = dalloc(&ws.vgpc, (size_t)3 * ngkmax)) ||
      (rc = dalloc(&ws.gpc, (size_t)ngkmax)) || (rc = dalloc(&ws.tpgpc, (size_t)2 * ngkmax)) ||
      (rc = dalloc(&ws.sfacgp, (size_t)ngkmax * st.natmtot)) ||
      (rc = dalloc(&ws.gk_iv, (size_t)3 * ngkmax)) || (rc = dalloc(&ws.d, n)) ||
      (rc = dalloc(&ws.e, n)) || (rc = dalloc(&ws.tau, n)) ||
      (rc = dalloc(&ws.Wp, n * 4 * tridiag_nb())) ||
      (rc = dalloc(&ws.red, (size_t)tridiag_workspace_doubles())) || (rc = dalloc(&ws.w, n)) ||
      (rc = dalloc(&ws.stein_ws, tridiag_eig_scratch_doubles((int)n, (int)K))) ||
      (rc = dalloc(&ws.icl, K)) || (rc = dalloc(&ws.ybuf, 2 * n)) || (rc = dalloc(&ws.Z, n * K)) ||
      (rc = dalloc(&ws.Z2, n * K)) || (rc = dalloc(&ws.Gk, K * K)) || (rc = dalloc(&ws.Gki, K * K)) ||
      (rc = dalloc(&ws.Tf, backtr_factor_elems((int)n))) || (rc = dalloc(&ws.Xs, 2 * 256 * K)) ||
      (rc = dalloc(&ws.status, (size_t)ST_NWORDS)) || (rc = dalloc(&ws.bar, (size_t)4)) ||
      (rc = dalloc(&ws.prog, n)) ||
      (rc = dalloc(&ws.part, std::max((size_t)(8u << 20), n * 64 * 4)))) {
    free_workspace(ws);
    return rc;
  }
  ws.part_cap = std::max((size_t)(8u << 20), n * 64 * 4);
  if (want_slices) {
    // A and aa A as BF16 slice planes (setup_bf16.cu)
    const size_t pe = bf16x_plane_elems((int)AM, (int)ngkmax);
    const size_t nsc = 2 * (size_t)bf16x_rpad((int)ngkmax);
    if ((rc = dalloc(&ws.slices, pe)) || (rc = dalloc(&ws.slice_sc, nsc))) {
      free_workspace(ws);
      return rc;
    }
    ws.slices_elems = pe;
    ws.slice_sc_n = nsc;
  }
  // zeroed in the handle's stream order (lane streams do not wait for the legacy stream)
  CUDA_TRY(cudaMemsetAsync(ws.status, 0, ST_NWORDS * sizeof(int), h->stream));
  CUDA_TRY(cudaMemsetAsync(ws.bar, 0, 4 * sizeof(unsigned), h->stream));
  ws.nmatmax = (int)nmatmax;
  ws.ngkmax = (int)ngkmax;
  ws.kmax = (int)kmax;
  return EXCFV_OK;
}

// ---------------------------------------------------------------------------
// exported C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* excfv_last_error(void) { return g_err; }

int excfv_create(int device, excfv_handle** out) {
  if (!out) return EXCFV_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
    excfv_set_error("excfv_create: no CUDA device %d", device);
    return EXCFV_ERR_CUDA;
  }
  DeviceGuard g(device);
  cudaDeviceProp prop;
  CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10) {
    excfv_set_error("excfv_create: device %d is sm_%d%d; libexcfv is built for sm_100a", device,
                    prop.major, prop.minor);
    return EXCFV_ERR_UNSUPPORTED;
  }
  excfv_handle* h = new excfv_handle();
  h->device = device;
  h->nsm = prop.multiProcessorCount;
  if (cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete h;
    excfv_set_error("excfv_create: stream creation failed");
    return EXCFV_ERR_CUDA;
  }
  h->stream = h->own_stream;
  *out = h;
  return EXCFV_OK;
}

static void drop_graph(excfv_handle* h);

int excfv_destroy(excfv_handle* h) {
  if (!h) return EXCFV_OK;
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  for (int c = 0; c < PROF_NCLS; ++c)
    for (cudaEvent_t e : h->prof.ev[c]) cudaEventDestroy(e);
  for (excfv_handle* c : h->lanes) {
    cudaStreamSynchronize(c->stream);
    free_workspace(c->ws);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
    delete c;
  }
  h->lanes.clear();
  drop_graph(h);
  free_group(h->gplan);
  free_rho(h->rho);
  free_sv(h->sv);
  if (h->kinfo) cudaFree(h->kinfo);
  free_workspace(h->ws);
  if (h->owns_static) free_static(h->st);
  if (h->own_stream) cudaStreamDestroy(h->own_stream);
  delete h;
  return EXCFV_OK;
}

int excfv_set_precision(excfv_handle* h, int prec) {
  if (!h) return EXCFV_ERR_ARG;
  if (prec != EXCFV_PREC_FP64 && prec != EXCFV_PREC_MIXED) return EXCFV_ERR_ARG;
  h->prec = prec;
  return EXCFV_OK;
}

int excfv_set_reduction(excfv_handle* h, int reduction) {
  if (!h || reduction < 0 || reduction > 2) return EXCFV_ERR_ARG;
  h->reduction = reduction;
  for (excfv_handle* l : h->lanes) l->reduction = reduction;
  return EXCFV_OK;
}

int excfv_set_stream(excfv_handle* h, void* stream) {
  if (!h) return EXCFV_ERR_ARG;
  h->stream = stream ? (cudaStream_t)stream : h->own_stream;
  return EXCFV_OK;
}

int excfv_reserve(excfv_handle* h, int32_t nmatmax, int32_t ngkmax) {
  if (!h || nmatmax <= 0 || ngkmax <= 0) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  return stage_reserve(h, nmatmax, ngkmax, std::max(1, std::min(h->st.nstfv, nmatmax)));
}

int excfv_set_static(excfv_handle* h, const excfv_static* s) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  return stage_set_static(h, s);
}

int excfv_hmlint(excfv_handle* h, const excfv_mtrad* r, double* aa, double* loa, double* lolo, double* oalo,
                 double* ololo) {
  if (!h || !r) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  return stage_hmlint(h, r, aa, loa, lolo, oalo, ololo);
}

int excfv_genveffig(excfv_handle* h, const int32_t* ngrid, const double* veffir, const double* cfunir,
                    double* veffig) {
  if (!h || !ngrid || !veffir || !cfunir) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  const int kinds[1] = {0};
  cplx* dst[1] = {h->st.veffig};
  cplx* out[1] = {reinterpret_cast<cplx*>(veffig)};
  return stage_genfig(h, ngrid, veffir, cfunir, 1, kinds, dst, out);
}

int excfv_genmeffig(excfv_handle* h, const int32_t* ngrid, const double* veffir, const double* cfunir,
                    double* meffig, double* m2effig) {
  if (!h || !ngrid || !veffir || !cfunir) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  // meffig only with valence relativity, m2effig only for IORA* (genmeffig.f90:34,45)
  int kinds[2];
  cplx* dst[2];
  cplx* out[2];
  int nk = 0;
  if (h->st.vrel != 0) {
    kinds[nk] = 1; dst[nk] = h->st.xig; out[nk] = reinterpret_cast<cplx*>(meffig); ++nk;
  }
  if (h->st.h1on) {
    kinds[nk] = 2; dst[nk] = h->st.m2effig; out[nk] = reinterpret_cast<cplx*>(m2effig); ++nk;
  }
  if (nk == 0) return EXCFV_OK;
  return stage_genfig(h, ngrid, veffir, cfunir, nk, kinds, dst, out);
}

int excfv_set_rho(excfv_handle* h, const excfv_rhoset* r) {
  if (!h || !r) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  return stage_set_rho(h, r);
}

// G+k inputs of one k-point into the workspace; device or host pointers
static int rho_stage_k(excfv_handle* h, int ngp, int ngkmax, int nmatmax, const double* gpc,
                       const double* tpgpc, const double* sfacgp, cudaMemcpyKind kind) {
  int rc;
  if ((rc = stage_reserve(h, nmatmax, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  Workspace& ws = h->ws;
  if (ngkmax != ws.ngkmax) {
    // staged G+k arrays use the workspace leading dimension; re-reserve exactly
    cudaStreamSynchronize(h->stream);
    free_workspace(ws);
    if ((rc = stage_reserve(h, nmatmax, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  }
  cudaStream_t s = h->stream;
  CUDA_TRY(cudaMemcpyAsync(ws.gpc, gpc, sizeof(double) * ngp, kind, s));
  CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, tpgpc, sizeof(double) * 2 * ngp, kind, s));
  CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, sfacgp, sizeof(cplx) * (size_t)ngkmax * h->st.natmtot, kind, s));
  return stage_match(h, ngp, ngkmax, ws.apwalm);
}

static int check_rho(excfv_handle* h, int ngp, int ngkmax, int nmatmax) {
  if (!h) return EXCFV_ERR_ARG;
  if (!h->have_static || !h->rho.ready) {
    excfv_set_error("excfv_set_static and excfv_set_rho must be called first");
    return EXCFV_ERR_STATE;
  }
  if (ngp <= 0 || ngp > ngkmax || nmatmax < ngp + h->st.nlotot) {
    excfv_set_error("excfv_rhovalk: inconsistent sizes ngp=%d ngkmax=%d nmatmax=%d", ngp, ngkmax, nmatmax);
    return EXCFV_ERR_ARG;
  }
  return EXCFV_OK;
}

int excfv_rhovalk(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                  const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* wocc, double epsocc) {
  int rc = check_rho(h, ngp, ngkmax, nmatmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !evecfv || !wocc) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = rho_stage_k(h, ngp, ngkmax, nmatmax, gpc, tpgpc, sfacgp, cudaMemcpyHostToDevice))) return rc;
  Workspace& ws = h->ws;
  // evecfv(nmatmax, nstfv) into the eigenvector scratch (nmatmax x kmax, kmax >= nstfv)
  const size_t need = (size_t)nmatmax * h->st.nstfv;
  CUDA_TRY(cudaMemcpyAsync(ws.Z, evecfv, sizeof(cplx) * need, cudaMemcpyHostToDevice, h->stream));
  if ((rc = stage_rhovalk(h, ngp, ngkmax, ws.apwalm, ws.Z, nmatmax, wocc, epsocc))) return rc;
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EXCFV_OK;
}

int excfv_rhovalk_dev(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                      const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* wocc,
                      double epsocc) {
  int rc = check_rho(h, ngp, ngkmax, nmatmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !evecfv || !wocc) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = rho_stage_k(h, ngp, ngkmax, nmatmax, gpc, tpgpc, sfacgp, cudaMemcpyDeviceToDevice))) return rc;
  return stage_rhovalk(h, ngp, ngkmax, h->ws.apwalm, reinterpret_cast<const cplx*>(evecfv), nmatmax, wocc,
                       epsocc);
}

int excfv_set_bfield(excfv_handle* h, const excfv_bfield* b) {
  if (!h || !b) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  return stage_set_bfield(h, b);
}

int excfv_set_bfield_nc(excfv_handle* h, const excfv_bfield_nc* b) {
  if (!h || !b) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  cudaStreamSynchronize(h->stream);
  return stage_set_bfield_nc(h, b);
}

// the k-point's G+k data into the workspace and its packed matching coefficients
static int sv_stage_k(excfv_handle* h, int ngp, int ngkmax, int nmatmax, const double* gpc, const double* tpgpc,
                      const double* sfacgp, const int32_t* igpig, cudaMemcpyKind kind) {
  int rc;
  // the eigenproblem's order: nstfv per spin block, 2 nstfv for a non-collinear field
  const int nsv = std::max(1, h->st.nstfv) * (h->sv.nc ? 2 : 1);
  const int nmat = std::max(nmatmax, nsv);
  if ((rc = stage_reserve(h, nmat, ngkmax, nsv))) return rc;
  Workspace& ws = h->ws;
  if (ngkmax != ws.ngkmax) {
    cudaStreamSynchronize(h->stream);
    free_workspace(ws);
    if ((rc = stage_reserve(h, nmat, ngkmax, nsv))) return rc;
  }
  cudaStream_t s = h->stream;
  CUDA_TRY(cudaMemcpyAsync(ws.gpc, gpc, sizeof(double) * ngp, kind, s));
  CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, tpgpc, sizeof(double) * 2 * ngp, kind, s));
  CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, sfacgp, sizeof(cplx) * (size_t)ngkmax * h->st.natmtot, kind, s));
  CUDA_TRY(cudaMemcpyAsync(ws.igpig, igpig, sizeof(int) * ngp, kind, s));
  return stage_match(h, ngp, ngkmax, nullptr);
}

static int check_sv(excfv_handle* h, int ngp, int ngkmax, int nmatmax) {
  if (!h) return EXCFV_ERR_ARG;
  if (!h->have_static || !h->sv.ready) {
    excfv_set_error("excfv_set_static and excfv_set_bfield must be called first");
    return EXCFV_ERR_STATE;
  }
  if (ngp <= 0 || ngp > ngkmax || nmatmax < ngp + h->st.nlotot || h->st.nstfv > ngp) {
    excfv_set_error("excfv_seceqnsv: inconsistent sizes ngp=%d ngkmax=%d nmatmax=%d nstfv=%d", ngp, ngkmax,
                    nmatmax, h->st.nstfv);
    return EXCFV_ERR_ARG;
  }
  return EXCFV_OK;
}

int excfv_seceqnsv(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                   const double* sfacgp, const int32_t* igpig, int32_t nmatmax, const double* evalfv,
                   const double* evecfv, double* evalsv, double* evecsv) {
  int rc = check_sv(h, ngp, ngkmax, nmatmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !igpig || !evalfv || !evecfv || !evalsv || !evecsv) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = sv_stage_k(h, ngp, ngkmax, nmatmax, gpc, tpgpc, sfacgp, igpig, cudaMemcpyHostToDevice))) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const int n = h->st.nstfv;
  CUDA_TRY(cudaMemcpyAsync(ws.Z2, evecfv, sizeof(cplx) * (size_t)nmatmax * n, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(h->sv.evalfv, evalfv, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  double* dw = nullptr;
  cplx* dv = nullptr;
  if ((rc = dalloc(&dw, (size_t)2 * n)) || (rc = dalloc(&dv, (size_t)4 * n * n))) {
    if (dw) cudaFree(dw);
    return rc;
  }
  rc = stage_seceqnsv(h, ngp, ws.Z2, nmatmax, h->sv.evalfv, dw, dv);
  if (rc == EXCFV_OK) rc = stage_status(h, n);
  if (rc == EXCFV_OK) {
    cudaMemcpyAsync(evalsv, dw, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(evecsv, dv, sizeof(cplx) * 4 * (size_t)n * n, cudaMemcpyDeviceToHost, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) rc = EXCFV_ERR_CUDA;
  }
  cudaFree(dw);
  cudaFree(dv);
  return rc;
}

int excfv_seceqnsv_dev(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                       const double* sfacgp, const int32_t* igpig, int32_t nmatmax, const double* evalfv,
                       const double* evecfv, double* evalsv, double* evecsv) {
  int rc = check_sv(h, ngp, ngkmax, nmatmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !igpig || !evalfv || !evecfv || !evalsv || !evecsv) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = sv_stage_k(h, ngp, ngkmax, nmatmax, gpc, tpgpc, sfacgp, igpig, cudaMemcpyDeviceToDevice))) return rc;
  return stage_seceqnsv(h, ngp, reinterpret_cast<const cplx*>(evecfv), nmatmax, evalfv, evalsv,
                        reinterpret_cast<cplx*>(evecsv));
}

static int rhovalk_sv_host(excfv_handle* h, bool nc, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                     const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* evecsv,
                     const double* wocc, double epsocc) {
  int rc = check_rho(h, ngp, ngkmax, nmatmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !evecfv || !evecsv || !wocc) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = rho_stage_k(h, ngp, ngkmax, nmatmax, gpc, tpgpc, sfacgp, cudaMemcpyHostToDevice))) return rc;
  Workspace& ws = h->ws;
  const int n = h->st.nstfv;
  CUDA_TRY(cudaMemcpyAsync(ws.Z, evecfv, sizeof(cplx) * (size_t)nmatmax * n, cudaMemcpyHostToDevice, h->stream));
  cplx* dsv = nullptr;
  if ((rc = dalloc(&dsv, (size_t)4 * n * n))) return rc;
  rc = EXCFV_OK;
  if (cudaMemcpyAsync(dsv, evecsv, sizeof(cplx) * (size_t)4 * n * n, cudaMemcpyHostToDevice, h->stream) !=
      cudaSuccess)
    rc = EXCFV_ERR_CUDA;
  if (rc == EXCFV_OK)
    rc = nc ? stage_rhovalk_sv_nc(h, ngp, ngkmax, ws.apwalm, ws.Z, nmatmax, dsv, wocc, epsocc)
            : stage_rhovalk_sv(h, ngp, ngkmax, ws.apwalm, ws.Z, nmatmax, dsv, wocc, epsocc);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess && rc == EXCFV_OK) rc = EXCFV_ERR_CUDA;
  cudaFree(dsv);
  return rc;
}

int excfv_rhovalk_sv(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                     const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* evecsv,
                     const double* wocc, double epsocc) {
  return rhovalk_sv_host(h, false, ngp, ngkmax, gpc, tpgpc, sfacgp, nmatmax, evecfv, evecsv, wocc, epsocc);
}

int excfv_rhovalk_sv_nc(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc, const double* tpgpc,
                        const double* sfacgp, int32_t nmatmax, const double* evecfv, const double* evecsv,
                        const double* wocc, double epsocc) {
  return rhovalk_sv_host(h, true, ngp, ngkmax, gpc, tpgpc, sfacgp, nmatmax, evecfv, evecsv, wocc, epsocc);
}

int excfv_get_magmt3(excfv_handle* h, double* magmt, int32_t reset) {
  if (!h) return EXCFV_ERR_ARG;
  if (!h->rho.ready) {
    excfv_set_error("excfv_set_rho must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  const size_t n = (size_t)3 * h->rho.lmmaxvr * h->rho.nrmtmax * h->st.natmtot;
  if (magmt) CUDA_TRY(cudaMemcpyAsync(magmt, h->rho.magmt3, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  if (reset) CUDA_TRY(cudaMemsetAsync(h->rho.magmt3, 0, sizeof(double) * n, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EXCFV_OK;
}

int excfv_get_magmt(excfv_handle* h, double* magmt, int32_t reset) {
  if (!h) return EXCFV_ERR_ARG;
  if (!h->rho.ready) {
    excfv_set_error("excfv_set_rho must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  const size_t n = (size_t)h->rho.lmmaxvr * h->rho.nrmtmax * h->st.natmtot;
  if (magmt) CUDA_TRY(cudaMemcpyAsync(magmt, h->rho.magmt, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  if (reset) CUDA_TRY(cudaMemsetAsync(h->rho.magmt, 0, sizeof(double) * n, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EXCFV_OK;
}

int excfv_get_rhomt(excfv_handle* h, double* rhomt, int32_t reset) {
  if (!h) return EXCFV_ERR_ARG;
  if (!h->rho.ready) {
    excfv_set_error("excfv_set_rho must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  const size_t n = (size_t)h->rho.lmmaxvr * h->rho.nrmtmax * h->st.natmtot;
  if (rhomt) CUDA_TRY(cudaMemcpyAsync(rhomt, h->rho.rhomt, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
  if (reset) CUDA_TRY(cudaMemsetAsync(h->rho.rhomt, 0, sizeof(double) * n, h->stream));
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  return EXCFV_OK;
}

static int check_k(excfv_handle* h, int nmatp, int ngp, int ngkmax) {
  if (!h) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  if (ngp <= 0 || ngp > ngkmax || nmatp != ngp + h->st.nlotot) {
    excfv_set_error("inconsistent sizes: nmatp=%d ngp=%d ngkmax=%d nlotot=%d", nmatp, ngp, ngkmax,
                    h->st.nlotot);
    return EXCFV_ERR_ARG;
  }
  return EXCFV_OK;
}

int excfv_match(excfv_handle* h, int32_t ngp, int32_t ngkmax, const double* gpc,
                const double* tpgpc, const double* sfacgp, double* apwalm) {
  if (!h || !gpc || !tpgpc || !sfacgp || !apwalm) return EXCFV_ERR_ARG;
  int rc = check_k(h, ngp + h->st.nlotot, ngp, ngkmax);
  if (rc) return rc;
  DeviceGuard g(h->device);
  if ((rc = stage_reserve(h, ngp + h->st.nlotot, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (ngkmax != ws.ngkmax) {
    // staged arrays use the workspace leading dimension; re-reserve exactly
    free_workspace(ws);
    if ((rc = stage_reserve(h, ngp + h->st.nlotot, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  }
  CUDA_TRY(cudaMemcpyAsync(ws.gpc, gpc, sizeof(double) * ngkmax, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, tpgpc, sizeof(double) * 2 * ngkmax, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, sfacgp, sizeof(cplx) * (size_t)ngkmax * h->st.natmtot,
                           cudaMemcpyHostToDevice, s));
  if ((rc = stage_match(h, ngp, ngkmax, ws.apwalm))) return rc;
  const size_t na = (size_t)ngkmax * h->st.apwordmax * h->st.lmmaxapw * h->st.natmtot;
  CUDA_TRY(cudaMemcpyAsync(apwalm, ws.apwalm, sizeof(cplx) * na, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  return EXCFV_OK;
}

// G+k arrays (host) -> workspace, ld = ws.ngkmax
static int stage_gk_host(excfv_handle* h, int ngp, int ngkmax, const int32_t* igpig,
                         const double* vgpc) {
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  CUDA_TRY(cudaMemcpyAsync(ws.igpig, igpig, sizeof(int) * ngp, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.vgpc, vgpc, sizeof(double) * 3 * ngp, cudaMemcpyHostToDevice, s));
  (void)ngkmax;
  return EXCFV_OK;
}

int excfv_hamiltonandoverlapsetup(excfv_handle* h, int32_t nmatp, int32_t ngp, int32_t ngkmax,
                                  const double* apwalm, const int32_t* igpig, const double* vgpc,
                                  double* hmat, double* omat) {
  int rc = check_k(h, nmatp, ngp, ngkmax);
  if (rc) return rc;
  if (!apwalm || !igpig || !vgpc || !hmat || !omat) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = stage_reserve(h, nmatp, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const size_t na = (size_t)ngkmax * h->st.apwordmax * h->st.lmmaxapw * h->st.natmtot;
  if (ngkmax > ws.ngkmax) return EXCFV_ERR_STATE;
  CUDA_TRY(cudaMemcpyAsync(ws.apwalm, apwalm, sizeof(cplx) * na, cudaMemcpyHostToDevice, s));
  if ((rc = stage_gk_host(h, ngp, ngkmax, igpig, vgpc))) return rc;
  if ((rc = stage_pack_apwalm(h, ngp, ngkmax, ws.apwalm))) return rc;
  if ((rc = stage_setup(h, nmatp, ngp, true))) return rc;
  const size_t nn = (size_t)nmatp * nmatp;
  CUDA_TRY(cudaMemcpyAsync(hmat, ws.H, sizeof(cplx) * nn, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(omat, ws.O, sizeof(cplx) * nn, cudaMemcpyDeviceToHost, s));
  int setup_flag = 0;
  CUDA_TRY(cudaMemcpyAsync(&setup_flag, ws.status + ST_SETUP, sizeof(int), cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaStreamSynchronize(s));
  if (setup_flag) {
    excfv_set_error("a bounded wait of the setup contraction timed out");
    return EXCFV_ERR_TIMEOUT;
  }
  return EXCFV_OK;
}

int excfv_solvewithlapack(excfv_handle* h, int32_t nmatp, const double* hmat, const double* omat,
                          int32_t nstfv, double evaltol, double* evalfv, double* evecfv,
                          int32_t ldevec) {
  if (!h || nmatp <= 0 || !hmat || !omat || !evalfv || !evecfv || nstfv < 1 || nstfv > nmatp ||
      ldevec < nmatp)
    return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  int rc = stage_reserve(h, nmatp, std::max(1, h->ws.ngkmax), std::max(nstfv, h->st.nstfv));
  if (rc) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const double t0 = now_s();
  const size_t nn = (size_t)nmatp * nmatp;
  CUDA_TRY(cudaMemcpyAsync(ws.H, hmat, sizeof(cplx) * nn, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.O, omat, sizeof(cplx) * nn, cudaMemcpyHostToDevice, s));
  // ZHEGVX('U') reads the upper triangles only
  if ((rc = mirror_upper(s, nmatp, ws.H, nmatp))) return rc;
  cplx* outv = nullptr;
  double* outw = nullptr;
  if ((rc = dalloc(&outv, (size_t)nmatp * nstfv))) return rc;
  if ((rc = dalloc(&outw, (size_t)nstfv))) {
    cudaFree(outv);
    return rc;
  }
  rc = stage_solve(h, nmatp, nstfv, evaltol, outw, outv, nmatp);
  if (rc == 0) {
    CUDA_TRY(cudaMemcpy2DAsync(evecfv, sizeof(cplx) * ldevec, outv, sizeof(cplx) * nmatp,
                               sizeof(cplx) * nmatp, nstfv, cudaMemcpyDeviceToHost, s));
    CUDA_TRY(cudaMemcpyAsync(evalfv, outw, sizeof(double) * nstfv, cudaMemcpyDeviceToHost, s));
    rc = stage_status(h, nmatp);
  }
  cudaStreamSynchronize(s);
  cudaFree(outv);
  cudaFree(outw);
  h->timings[2] = now_s() - t0;
  return rc;
}

// evalfv/evecfv device outputs for the seceqn paths
static int solve_into(excfv_handle* h, int nmatp, double* d_eval, cplx* d_evec, long long ld) {
  return stage_solve(h, nmatp, h->st.nstfv, h->st.evaltol, d_eval, d_evec, ld);
}

int excfv_seceqnfv(excfv_handle* h, int32_t ispn, int32_t ik, int32_t nmatp, int32_t ngp,
                   int32_t ngkmax, const int32_t* igpig, const double* vgpc, const double* apwalm,
                   int32_t nmatmax, double* evalfv, double* evecfv) {
  (void)ik;
  if (ispn != 1) {
    excfv_set_error("excfv_seceqnfv: only one first-variational spin (ispn = 1) is supported");
    return EXCFV_ERR_UNSUPPORTED;
  }
  int rc = check_k(h, nmatp, ngp, ngkmax);
  if (rc) return rc;
  if (!igpig || !vgpc || !apwalm || !evalfv || !evecfv || nmatmax < nmatp) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = stage_reserve(h, nmatp, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  const int k = h->st.nstfv;
  if (k > nmatp) return EXCFV_ERR_ARG;
  const double t0 = now_s();
  const size_t na = (size_t)ngkmax * h->st.apwordmax * h->st.lmmaxapw * h->st.natmtot;
  if (ngkmax > ws.ngkmax) return EXCFV_ERR_STATE;
  CUDA_TRY(cudaMemcpyAsync(ws.apwalm, apwalm, sizeof(cplx) * na, cudaMemcpyHostToDevice, s));
  if ((rc = stage_gk_host(h, ngp, ngkmax, igpig, vgpc))) return rc;
  if ((rc = stage_pack_apwalm(h, ngp, ngkmax, ws.apwalm))) return rc;
  if ((rc = stage_setup(h, nmatp, ngp, false))) return rc;
  // outputs staged in Z2 (n x k, overwritten only by the Cholesky-QR before the
  // final product) -> use Ui-sized T buffer region past the solve instead
  cplx* outv = ws.apwalm;  // free after packing; holds >= n*k complex? check below
  const size_t need = (size_t)nmatp * k;
  bool own = false;
  if (need > na) {
    if ((rc = dalloc(&outv, need))) return rc;
    own = true;
  }
  if ((rc = solve_into(h, nmatp, ws.w + 0, outv, nmatp))) { if (own) cudaFree(outv); return rc; }
  CUDA_TRY(cudaMemcpy2DAsync(evecfv, sizeof(cplx) * nmatmax, outv, sizeof(cplx) * nmatp,
                             sizeof(cplx) * nmatp, k, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(evalfv, ws.w, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
  rc = stage_status(h, nmatp);
  if (own) cudaFree(outv);
  h->timings[2] = now_s() - t0;
  return rc;
}

int excfv_seceqn_dev(excfv_handle* h, int32_t nmatp, int32_t ngp, int32_t ngkmax, const double* gpc,
                     const double* tpgpc, const double* sfacgp, const int32_t* igpig,
                     const double* vgpc, int32_t nmatmax, double* evalfv, double* evecfv) {
  int rc = check_k(h, nmatp, ngp, ngkmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !igpig || !vgpc || !evalfv || !evecfv || nmatmax < nmatp)
    return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = stage_reserve(h, nmatp, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (ngkmax != ws.ngkmax) {
    excfv_set_error("excfv_seceqn_dev: ngkmax must equal the reserved ngkmax (%d)", ws.ngkmax);
    return EXCFV_ERR_ARG;
  }
  const int k = h->st.nstfv;
  if (k > nmatp) return EXCFV_ERR_ARG;
  CUDA_TRY(cudaMemcpyAsync(ws.gpc, gpc, sizeof(double) * ngp, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, tpgpc, sizeof(double) * 2 * ngp, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, sfacgp, sizeof(cplx) * (size_t)ngkmax * h->st.natmtot,
                           cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.igpig, igpig, sizeof(int) * ngp, cudaMemcpyDeviceToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.vgpc, vgpc, sizeof(double) * 3 * ngp, cudaMemcpyDeviceToDevice, s));
  if ((rc = stage_match(h, ngp, ngkmax, nullptr))) return rc;
  if ((rc = stage_setup(h, nmatp, ngp, false))) return rc;
  return solve_into(h, nmatp, evalfv, (cplx*)evecfv, nmatmax);
}

int excfv_seceqn(excfv_handle* h, int32_t ik, int32_t nmatp, int32_t ngp, int32_t ngkmax,
                 const double* gpc, const double* tpgpc, const double* sfacgp,
                 const int32_t* igpig, const double* vgpc, int32_t nmatmax, double* evalfv,
                 double* evecfv) {
  (void)ik;
  int rc = check_k(h, nmatp, ngp, ngkmax);
  if (rc) return rc;
  if (!gpc || !tpgpc || !sfacgp || !igpig || !vgpc || !evalfv || !evecfv || nmatmax < nmatp)
    return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if ((rc = stage_reserve(h, nmatp, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  if (ngkmax != ws.ngkmax) {
    free_workspace(ws);
    if ((rc = stage_reserve(h, nmatp, ngkmax, std::max(1, h->st.nstfv)))) return rc;
  }
  const int k = h->st.nstfv;
  if (k > nmatp) return EXCFV_ERR_ARG;
  const double t0 = now_s();
  CUDA_TRY(cudaMemcpyAsync(ws.gpc, gpc, sizeof(double) * ngp, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, tpgpc, sizeof(double) * 2 * ngp, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, sfacgp, sizeof(cplx) * (size_t)ngkmax * h->st.natmtot,
                           cudaMemcpyHostToDevice, s));
  if ((rc = stage_gk_host(h, ngp, ngkmax, igpig, vgpc))) return rc;
  if ((rc = stage_match(h, ngp, ngkmax, nullptr))) return rc;
  if ((rc = stage_setup(h, nmatp, ngp, false))) return rc;
  cplx* outv = ws.apwalm;
  const size_t na = (size_t)ngkmax * h->st.apwordmax * h->st.lmmaxapw * h->st.natmtot;
  const size_t need = (size_t)nmatp * k;
  bool own = false;
  if (need > na) {
    if ((rc = dalloc(&outv, need))) return rc;
    own = true;
  }
  if ((rc = solve_into(h, nmatp, ws.w, outv, nmatp))) { if (own) cudaFree(outv); return rc; }
  CUDA_TRY(cudaMemcpy2DAsync(evecfv, sizeof(cplx) * nmatmax, outv, sizeof(cplx) * nmatp,
                             sizeof(cplx) * nmatp, k, cudaMemcpyDeviceToHost, s));
  CUDA_TRY(cudaMemcpyAsync(evalfv, ws.w, sizeof(double) * k, cudaMemcpyDeviceToHost, s));
  rc = stage_status(h, nmatp);
  if (own) cudaFree(outv);
  h->timings[2] = now_s() - t0;
  return rc;
}

int excfv_sync(excfv_handle* h) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  if (!h->ws.status) {  // only batched calls so far: their status is read by excfv_batch_info
    CUDA_TRY(cudaStreamSynchronize(h->stream));
    return EXCFV_OK;
  }
  return stage_status(h, 0);
}

long long excfv_launch_count(void) { return g_launches.load(); }

int excfv_tridiag_tail_start(int n, int complex64) {
  if (n < 1) return 0;
  return tridiag_tail_start(n, complex64 != 0);
}

int excfv_set_lattice(excfv_handle* h, const double* vgc, const double* atposc) {
  if (!h || !vgc || !atposc) return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  return stage_set_lattice(h, vgc, atposc);
}

int excfv_gengpvec_dev(excfv_handle* h, const double* vpl, const double* vpc, double gkmax, int32_t ngkmax,
                       int32_t* d_ngp, int32_t* igpig, double* vgpl, double* vgpc, double* gpc, double* tpgpc) {
  if (!h || !vpl || !vpc || !d_ngp || !igpig || !vgpl || !vgpc || !gpc || !tpgpc || ngkmax < 1 || gkmax <= 0.0)
    return EXCFV_ERR_ARG;
  if (!h->have_static || !h->st.have_lattice) {
    excfv_set_error("excfv_set_static and excfv_set_lattice must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  return stage_gengpvec(h, vpl, vpc, gkmax, ngkmax, d_ngp, igpig, vgpl, vgpc, gpc, tpgpc);
}

int excfv_gengpvec(excfv_handle* h, const double* vpl, const double* vpc, double gkmax, int32_t ngkmax,
                   int32_t* ngp, int32_t* igpig, double* vgpl, double* vgpc, double* gpc, double* tpgpc) {
  if (!h || !ngp || !igpig || !vgpl || !vgpc || !gpc || !tpgpc || ngkmax < 1) return EXCFV_ERR_ARG;
  if (!h->have_static || !h->st.have_lattice) {
    excfv_set_error("excfv_set_static and excfv_set_lattice must be called first");
    return EXCFV_ERR_STATE;
  }
  DeviceGuard g(h->device);
  cudaStream_t s = h->stream;
  int* di = nullptr;
  double* dd = nullptr;
  int rc;
  if ((rc = dalloc(&di, (size_t)ngkmax + 1))) return rc;
  if ((rc = dalloc(&dd, (size_t)9 * ngkmax))) {
    cudaFree(di);
    return rc;
  }
  double* dvgpl = dd;
  double* dvgpc = dd + 3 * (size_t)ngkmax;
  double* dgpc = dd + 6 * (size_t)ngkmax;
  double* dtp = dd + 7 * (size_t)ngkmax;
  rc = stage_gengpvec(h, vpl, vpc, gkmax, ngkmax, di + ngkmax, di, dvgpl, dvgpc, dgpc, dtp);
  int n = 0;
  if (rc == EXCFV_OK && cudaMemcpyAsync(&n, di + ngkmax, sizeof(int), cudaMemcpyDeviceToHost, s) == cudaSuccess &&
      cudaStreamSynchronize(s) == cudaSuccess) {
    if (n < 0) {
      excfv_set_error("gengpvec: %d G+k vectors exceed ngkmax = %d", -n, ngkmax);
      rc = EXCFV_ERR_ARG;
    } else if (n > 0) {
      cudaMemcpyAsync(igpig, di, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(vgpl, dvgpl, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(vgpc, dvgpc, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(gpc, dgpc, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(tpgpc, dtp, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost, s);
      if (cudaStreamSynchronize(s) != cudaSuccess) rc = EXCFV_ERR_CUDA;
    }
    *ngp = n;
  } else if (rc == EXCFV_OK) {
    rc = EXCFV_ERR_CUDA;
  }
  cudaFree(di);
  cudaFree(dd);
  return rc;
}

int excfv_gensfacgp_dev(excfv_handle* h, int32_t ngp, const double* vgpc, int32_t ld, double* sfacgp) {
  if (!h || !vgpc || !sfacgp || ngp < 0 || ld < ngp) return EXCFV_ERR_ARG;
  if (!h->have_static || !h->st.have_lattice) {
    excfv_set_error("excfv_set_static and excfv_set_lattice must be called first");
    return EXCFV_ERR_STATE;
  }
  if (ngp == 0) return EXCFV_OK;
  DeviceGuard g(h->device);
  return stage_gensfacgp(h, ngp, vgpc, ld, reinterpret_cast<cplx*>(sfacgp));
}

int excfv_gensfacgp(excfv_handle* h, int32_t ngp, const double* vgpc, int32_t ld, double* sfacgp) {
  if (!h || !vgpc || !sfacgp || ngp < 0 || ld < ngp) return EXCFV_ERR_ARG;
  if (!h->have_static || !h->st.have_lattice) {
    excfv_set_error("excfv_set_static and excfv_set_lattice must be called first");
    return EXCFV_ERR_STATE;
  }
  if (ngp == 0) return EXCFV_OK;
  DeviceGuard g(h->device);
  cudaStream_t s = h->stream;
  double* dv = nullptr;
  cplx* ds = nullptr;
  int rc;
  if ((rc = dalloc(&dv, (size_t)3 * ngp))) return rc;
  if ((rc = dalloc(&ds, (size_t)ld * h->st.natmtot))) {
    cudaFree(dv);
    return rc;
  }
  if (cudaMemcpyAsync(dv, vgpc, sizeof(double) * 3 * ngp, cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(ds, 0, sizeof(cplx) * (size_t)ld * h->st.natmtot, s) != cudaSuccess)
    rc = EXCFV_ERR_CUDA;
  if (rc == EXCFV_OK) rc = stage_gensfacgp(h, ngp, dv, ld, ds);
  if (rc == EXCFV_OK &&
      (cudaMemcpyAsync(sfacgp, ds, sizeof(cplx) * (size_t)ld * h->st.natmtot, cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess))
    rc = EXCFV_ERR_CUDA;
  cudaFree(dv);
  cudaFree(ds);
  return rc;
}

int excfv_test_reduce_band(excfv_handle* h, int32_t n, const double* c, int32_t stages,
                           double* band, double* d, double* e, int32_t* bandwidth) {
  if (!h || !c || n < 1 || (stages != 1 && stages != 2) || (stages == 1 && !band) ||
      (stages == 2 && (!d || !e)))
    return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  const int bw = band_bandwidth();
  if (bandwidth) *bandwidth = bw;
  DeviceGuard g(h->device);
  if (!two_stage_supported(h, n)) {
    excfv_set_error("two-stage reduction does not support n = %d", n);
    return EXCFV_ERR_UNSUPPORTED;
  }
  int rc = stage_reserve(h, n, std::max(1, h->ws.ngkmax), std::max(1, h->st.nstfv));
  if (rc) return rc;
  Workspace& ws = h->ws;
  cudaStream_t s = h->stream;
  bind_gemm_ctx(h);
  CUDA_TRY(cudaMemcpyAsync(ws.H, c, sizeof(cplx) * (size_t)n * n, cudaMemcpyHostToDevice, s));
  CUDA_TRY(cudaMemsetAsync(ws.status, 0, ST_NWORDS * sizeof(int), s));
  if ((rc = he2hb(h, n, ws.H, n))) return rc;
  cplx* AB = ws.T;
  if ((rc = two_stage_finish_band(h, n, ws.H, n, AB))) return rc;
  if (stages == 1) {
    // compact (2 bw + 1, n) -> (bw + 1, n)
    CUDA_TRY(cudaMemcpy2DAsync(band, sizeof(cplx) * (bw + 1), AB, sizeof(cplx) * (2 * bw + 1),
                               sizeof(cplx) * (bw + 1), n, cudaMemcpyDeviceToHost, s));
  } else {
    if ((rc = hb2st(h, n, AB, ws.O, ws.ybuf))) return rc;
    CUDA_TRY(cudaMemcpyAsync(d, ws.d, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    if (n > 1) CUDA_TRY(cudaMemcpyAsync(e, ws.e, sizeof(double) * (n - 1), cudaMemcpyDeviceToHost, s));
  }
  CUDA_TRY(cudaStreamSynchronize(s));
  return stage_status(h, n);
}

int excfv_test_set_wait_limit(int64_t limit_ns, int32_t plant_stall) {
  if (limit_ns <= 0) limit_ns = 2000000000LL;
  if (limit_ns < 100000LL) limit_ns = 100000LL;  // at least 0.1 ms
  g_wait_ns.store(limit_ns);
  g_planted.store(plant_stall ? 1 : 0);
  return EXCFV_OK;
}

// ---------------------------------------------------------------------------
// batched k-points: lanes
// ---------------------------------------------------------------------------

// Largest lane count whose per-lane CTA budget still holds an n x n panel
// (a CTA of the reduction owns 128 rows, 192 in complex64 storage).
static int max_lanes_for(const excfv_handle* h, int nmax) {
  const int rows = tridiag_rows_per_cta(h->prec == EXCFV_PREC_MIXED);
  const int need = (nmax + rows - 1) / rows;
  return std::max(1, h->nsm / std::max(1, need));
}

static int ensure_lanes(excfv_handle* h, int L, int nmatmax, int ngkmax, int kmax) {
  while ((int)h->lanes.size() < L) {
    excfv_handle* c = new excfv_handle();
    c->device = h->device;
    c->nsm = h->nsm;
    c->owns_static = false;
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) {
      delete c;
      excfv_set_error("lane stream creation failed");
      return EXCFV_ERR_CUDA;
    }
    c->stream = c->own_stream;
    h->lanes.push_back(c);
  }
  for (int i = 0; i < L; ++i) {
    excfv_handle* c = h->lanes[i];
    c->st = h->st;
    c->have_static = h->have_static;
    c->prec = h->prec;
    c->grid_ctas = std::max(1, h->nsm / L);
    c->prof.on = h->prof.on;  // lanes report into the parent's profile
    if (c->ws.H && c->ws.ngkmax != ngkmax) free_workspace(c->ws);
    int rc = stage_reserve(c, nmatmax, ngkmax, kmax);
    if (rc) return rc;
  }
  return EXCFV_OK;
}

struct BatchArgs {
  int nk;
  const int32_t* nmatp;
  const int32_t* ngp;
  int ngkmax;
  const double* const* gpc;
  const double* const* tpgpc;
  const double* const* sfacgp;
  const int32_t* const* igpig;
  const double* const* vgpc;
  int nmatmax;
  double* const* evalfv;
  double* const* evecfv;
  bool host;  // pointers are host pointers (copies in/out on the lane streams)
};

static int check_batch(excfv_handle* h, const BatchArgs& b, int* nmax) {
  if (!h || b.nk <= 0 || !b.nmatp || !b.ngp || !b.gpc || !b.tpgpc || !b.sfacgp || !b.igpig ||
      !b.vgpc || !b.evalfv || !b.evecfv)
    return EXCFV_ERR_ARG;
  if (!h->have_static) {
    excfv_set_error("excfv_set_static must be called first");
    return EXCFV_ERR_STATE;
  }
  *nmax = 0;
  for (int k = 0; k < b.nk; ++k) {
    if (b.ngp[k] <= 0 || b.ngp[k] > b.ngkmax || b.nmatp[k] != b.ngp[k] + h->st.nlotot ||
        b.nmatp[k] > b.nmatmax || h->st.nstfv > b.nmatp[k]) {
      excfv_set_error("batch entry %d: inconsistent sizes", k);
      return EXCFV_ERR_ARG;
    }
    *nmax = std::max(*nmax, (int)b.nmatp[k]);
  }
  return EXCFV_OK;
}

static int enqueue_batch(excfv_handle* h, const BatchArgs& b, int L);
static int run_batch_graph(excfv_handle* h, const BatchArgs& b, int L);
static void group_segments(excfv_handle* h, const BatchArgs& b, int L, std::vector<std::vector<int>>& segs);

// Enqueues the whole batch on L lanes (largest k-points first, each to the
// least-loaded lane), fork/join on h->stream.
static int run_batch(excfv_handle* h, const BatchArgs& b, int L) {
  int nmax = 0;
  int rc = check_batch(h, b, &nmax);
  if (rc) return rc;
  L = std::max(1, std::min(L, std::min(b.nk, max_lanes_for(h, nmax))));
  if ((rc = ensure_lanes(h, L, b.nmatmax, b.ngkmax, std::max(1, h->st.nstfv)))) return rc;
  if (h->kinfo_cap < b.nk) {
    if (h->kinfo) cudaFree(h->kinfo);
    h->kinfo = nullptr;
    h->kinfo_cap = 0;
    if ((rc = dalloc(&h->kinfo, (size_t)b.nk * ST_NWORDS))) return rc;
    h->kinfo_cap = b.nk;
  }
  h->batch_nmat.assign(b.nmatp, b.nmatp + b.nk);
  h->last_nk = b.nk;
  h->batch_form = h->batch_mode;
  if (h->batch_mode == EXCFV_BATCH_AUTO) {
    size_t fr = 0, tot = 0;
    CUDA_TRY(cudaMemGetInfo(&fr, &tot));
    const double need = 4.0 * sizeof(cplx) * (double)nmax * nmax * b.nk;
    const bool have = group_slots_hold(h, b.nk, nmax);
    h->batch_form = (have || need <= 0.25 * (double)fr) ? EXCFV_BATCH_GROUPED : EXCFV_BATCH_LANES;
  }
  if (h->batch_form == EXCFV_BATCH_GROUPED || h->batch_form == EXCFV_BATCH_GROUPED_LANES) {
    std::vector<std::vector<int>> segs;
    group_segments(h, b, L, segs);
    bool rebuilt = false;
    if ((rc = group_plan_front(h, b.nk, b.nmatp, nmax, segs, &rebuilt))) return rc;
    // the plan's descriptors (and buffers) changed: no graph of an older plan may replay
    if (rebuilt) {
      drop_graph(h);
      h->gkey.clear();
      h->gseen = 0;
    }
  }
  if (!b.host && h->graph_on && !h->prof.on) return run_batch_graph(h, b, L);
  return enqueue_batch(h, b, L);
}

// Longest-processing-time-first: k-points by decreasing nmatp^3 (the
// eigensolver's cost), each to the lane with the least work so far, so the
// lanes finish together although the basis sizes differ.
static void deal_lanes(const BatchArgs& b, int L, std::vector<int>& order, std::vector<int>& lane_of) {
  order.resize(b.nk);
  lane_of.resize(b.nk);
  for (int k = 0; k < b.nk; ++k) order[k] = k;
  auto cost = [&](int k) { const double x = b.nmatp[k]; return x * x * x; };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
  std::vector<double> load(L, 0.0);
  for (int k : order) {
    const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
    lane_of[k] = l;
    load[l] += cost(k);
  }
}

// The k-points of each lane in the order the lane runs them.
static void lane_lists(const BatchArgs& b, int L, std::vector<std::vector<int>>& lists) {
  std::vector<int> order, lane_of;
  deal_lanes(b, L, order, lane_of);
  lists.assign(L, {});
  for (int k : order) lists[lane_of[k]].push_back(k);
}

// Segments of the grouped front: all k-points together (EXCFV_BATCH_GROUPED)
// or each lane's k-points (EXCFV_BATCH_GROUPED_LANES).
static void group_segments(excfv_handle* h, const BatchArgs& b, int L, std::vector<std::vector<int>>& segs) {
  if (h->batch_form == EXCFV_BATCH_GROUPED_LANES) {
    lane_lists(b, L, segs);
    return;
  }
  segs.assign(1, {});
  for (int k = 0; k < b.nk; ++k) segs[0].push_back(k);
}

static int fork_lanes(excfv_handle* h, int L) {
  cudaEvent_t fork;
  CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  CUDA_TRY(cudaEventRecord(fork, h->stream));
  for (int i = 0; i < L; ++i) CUDA_TRY(cudaStreamWaitEvent(h->lanes[i]->stream, fork, 0));
  cudaEventDestroy(fork);
  return EXCFV_OK;
}

static int join_lanes(excfv_handle* h, int L) {
  for (int i = 0; i < L; ++i) {
    cudaEvent_t join;
    CUDA_TRY(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(join, h->lanes[i]->stream));
    CUDA_TRY(cudaStreamWaitEvent(h->stream, join, 0));
    cudaEventDestroy(join);
  }
  return EXCFV_OK;
}

// The lane's matrices pointed at k-point k's slots of the grouped batch for
// the scope of one k-point's enqueue (launches take the pointers by value).
struct SlotScope {
  Workspace& ws;
  cplx *H, *O, *Ui, *T;
  SlotScope(excfv_handle* h, excfv_handle* c, int k) : ws(c->ws), H(ws.H), O(ws.O), Ui(ws.Ui), T(ws.T) {
    ws.H = group_slot(h, 0, k);
    ws.O = group_slot(h, 1, k);
    ws.Ui = group_slot(h, 2, k);
    ws.T = group_slot(h, 3, k);
  }
  ~SlotScope() { ws.H = H; ws.O = O; ws.Ui = Ui; ws.T = T; }
};

// One k-point's inputs, match and setup (H and O into its slots) on lane c;
// its status words (the setup's) are kept in the batch's status array.
static int grouped_setup_k(excfv_handle* h, excfv_handle* c, const BatchArgs& b, int k) {
  const cudaMemcpyKind in = b.host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  Workspace& ws = c->ws;
  cudaStream_t s = c->stream;
  const int ngp = b.ngp[k], n = b.nmatp[k];
  int rc;
  CUDA_TRY(cudaMemcpyAsync(ws.gpc, b.gpc[k], sizeof(double) * ngp, in, s));
  CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, b.tpgpc[k], sizeof(double) * 2 * ngp, in, s));
  CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, b.sfacgp[k], sizeof(cplx) * (size_t)b.ngkmax * h->st.natmtot, in, s));
  CUDA_TRY(cudaMemcpyAsync(ws.igpig, b.igpig[k], sizeof(int) * ngp, in, s));
  CUDA_TRY(cudaMemcpyAsync(ws.vgpc, b.vgpc[k], sizeof(double) * 3 * ngp, in, s));
  if ((rc = stage_match(c, ngp, b.ngkmax, nullptr))) return rc;
  {
    SlotScope sc(h, c, k);
    if ((rc = stage_setup(c, n, ngp, false))) return rc;
  }
  CUDA_TRY(cudaMemcpyAsync(h->kinfo + (size_t)k * ST_NWORDS, ws.status, sizeof(int) * ST_NWORDS,
                           cudaMemcpyDeviceToDevice, s));
  return EXCFV_OK;
}

// The rest of one k-point's solve after the grouped front, on lane c.
static int grouped_back_k(excfv_handle* h, excfv_handle* c, const BatchArgs& b, int k) {
  const cudaMemcpyKind out = b.host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const int k_st = h->st.nstfv;
  Workspace& ws = c->ws;
  cudaStream_t s = c->stream;
  const int n = b.nmatp[k];
  int rc;
  CUDA_TRY(cudaMemcpyAsync(ws.status, h->kinfo + (size_t)k * ST_NWORDS, sizeof(int) * ST_NWORDS,
                           cudaMemcpyDeviceToDevice, s));
  {
    SlotScope sc(h, c, k);
    if (b.host) {
      cplx* ov = ws.apwalm;
      const size_t na = (size_t)b.ngkmax * h->st.apwordmax * h->st.lmmaxapw * h->st.natmtot;
      if ((size_t)n * k_st > na) {
        excfv_set_error("batched host path: nmatp*nstfv exceeds the lane staging buffer");
        return EXCFV_ERR_UNSUPPORTED;
      }
      if ((rc = stage_solve_back(c, n, k_st, h->st.evaltol, ws.w, ov, n))) return rc;
      CUDA_TRY(cudaMemcpy2DAsync(b.evecfv[k], sizeof(cplx) * b.nmatmax, ov, sizeof(cplx) * n, sizeof(cplx) * n,
                                 k_st, out, s));
      CUDA_TRY(cudaMemcpyAsync(b.evalfv[k], ws.w, sizeof(double) * k_st, out, s));
    } else {
      if ((rc = stage_solve_back(c, n, k_st, h->st.evaltol, b.evalfv[k], (cplx*)b.evecfv[k], b.nmatmax)))
        return rc;
    }
  }
  CUDA_TRY(cudaMemcpyAsync(h->kinfo + (size_t)k * ST_NWORDS, ws.status, sizeof(int) * ST_NWORDS,
                           cudaMemcpyDeviceToDevice, s));
  return EXCFV_OK;
}

// The grouped batch.  EXCFV_BATCH_GROUPED: per lane match + setup into the
// k-points' slots; the grouped front (Cholesky, inverse factor, two-sided
// reduction) of all k-points on h->stream; per lane the rest of each
// k-point's solve.  EXCFV_BATCH_GROUPED_LANES: each lane sets up its own
// k-points, runs their grouped front on its stream and goes on with their
// solves, with no batch-wide join in between.
static int enqueue_grouped(excfv_handle* h, const BatchArgs& b, int L) {
  int rc = EXCFV_OK;
  std::vector<std::vector<int>> lists;
  lane_lists(b, L, lists);
  if ((rc = fork_lanes(h, L))) return rc;
  if (h->batch_form == EXCFV_BATCH_GROUPED_LANES) {
    for (int l = 0; l < L; ++l) {
      excfv_handle* c = h->lanes[l];
      for (int k : lists[l])
        if ((rc = grouped_setup_k(h, c, b, k))) return rc;
      if (!lists[l].empty() && (rc = group_enqueue_front(h, l, c->stream, c))) return rc;
      for (int k : lists[l])
        if ((rc = grouped_back_k(h, c, b, k))) return rc;
    }
    return join_lanes(h, L);
  }
  for (int l = 0; l < L; ++l)
    for (int k : lists[l])
      if ((rc = grouped_setup_k(h, h->lanes[l], b, k))) return rc;
  if ((rc = join_lanes(h, L))) return rc;
  if ((rc = group_enqueue_front(h, 0, h->stream, h))) return rc;
  if ((rc = fork_lanes(h, L))) return rc;
  for (int l = 0; l < L; ++l)
    for (int k : lists[l])
      if ((rc = grouped_back_k(h, h->lanes[l], b, k))) return rc;
  return join_lanes(h, L);
}

static int enqueue_batch(excfv_handle* h, const BatchArgs& b, int L) {
  if (h->batch_form == EXCFV_BATCH_GROUPED || h->batch_form == EXCFV_BATCH_GROUPED_LANES)
    return enqueue_grouped(h, b, L);
  int rc = EXCFV_OK;
  cudaEvent_t fork;
  CUDA_TRY(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  CUDA_TRY(cudaEventRecord(fork, h->stream));
  for (int i = 0; i < L; ++i) CUDA_TRY(cudaStreamWaitEvent(h->lanes[i]->stream, fork, 0));
  const cudaMemcpyKind in = b.host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  const cudaMemcpyKind out = b.host ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
  const int k_st = h->st.nstfv;
  // Longest-processing-time-first: k-points by decreasing nmatp^3 (the
  // eigensolver's cost), each to the lane with the least work so far, so the
  // lanes finish together although the basis sizes differ.
  std::vector<int> order(b.nk), lane_of(b.nk);
  for (int k = 0; k < b.nk; ++k) order[k] = k;
  auto cost = [&](int k) { const double x = b.nmatp[k]; return x * x * x; };
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost(x) > cost(y); });
  {
    std::vector<double> load(L, 0.0);
    for (int k : order) {
      const int l = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      lane_of[k] = l;
      load[l] += cost(k);
    }
  }
  for (int idx = 0; idx < b.nk && rc == EXCFV_OK; ++idx) {
    const int k = order[idx];
    excfv_handle* c = h->lanes[lane_of[k]];
    Workspace& ws = c->ws;
    cudaStream_t s = c->stream;
    const int ngp = b.ngp[k], n = b.nmatp[k];
    CUDA_TRY(cudaMemcpyAsync(ws.gpc, b.gpc[k], sizeof(double) * ngp, in, s));
    CUDA_TRY(cudaMemcpyAsync(ws.tpgpc, b.tpgpc[k], sizeof(double) * 2 * ngp, in, s));
    CUDA_TRY(cudaMemcpyAsync(ws.sfacgp, b.sfacgp[k], sizeof(cplx) * (size_t)b.ngkmax * h->st.natmtot,
                             in, s));
    CUDA_TRY(cudaMemcpyAsync(ws.igpig, b.igpig[k], sizeof(int) * ngp, in, s));
    CUDA_TRY(cudaMemcpyAsync(ws.vgpc, b.vgpc[k], sizeof(double) * 3 * ngp, in, s));
    if ((rc = stage_match(c, ngp, b.ngkmax, nullptr))) break;
    if ((rc = stage_setup(c, n, ngp, false))) break;
    if (b.host) {
      // outputs staged in the lane's (now free) reference-layout apwalm buffer
      cplx* ov = ws.apwalm;
      const size_t na = (size_t)b.ngkmax * h->st.apwordmax * h->st.lmmaxapw * h->st.natmtot;
      if ((size_t)n * k_st > na) {
        excfv_set_error("batched host path: nmatp*nstfv exceeds the lane staging buffer");
        rc = EXCFV_ERR_UNSUPPORTED;
        break;
      }
      if ((rc = stage_solve(c, n, k_st, h->st.evaltol, ws.w, ov, n))) break;
      CUDA_TRY(cudaMemcpy2DAsync(b.evecfv[k], sizeof(cplx) * b.nmatmax, ov, sizeof(cplx) * n,
                                 sizeof(cplx) * n, k_st, out, s));
      CUDA_TRY(cudaMemcpyAsync(b.evalfv[k], ws.w, sizeof(double) * k_st, out, s));
    } else {
      if ((rc = stage_solve(c, n, k_st, h->st.evaltol, b.evalfv[k], (cplx*)b.evecfv[k], b.nmatmax)))
        break;
    }
    CUDA_TRY(cudaMemcpyAsync(h->kinfo + (size_t)k * ST_NWORDS, ws.status, sizeof(int) * ST_NWORDS,
                             cudaMemcpyDeviceToDevice, s));
  }
  for (int i = 0; i < L; ++i) {
    cudaEvent_t join;
    CUDA_TRY(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
    CUDA_TRY(cudaEventRecord(join, h->lanes[i]->stream));
    CUDA_TRY(cudaStreamWaitEvent(h->stream, join, 0));
    cudaEventDestroy(join);
  }
  cudaEventDestroy(fork);
  return rc;
}

static int batch_info(excfv_handle* h, int nk, int32_t* info) {
  if (nk != h->last_nk || !h->kinfo) return EXCFV_ERR_STATE;
  std::vector<int> st((size_t)nk * ST_NWORDS);
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  CUDA_TRY(cudaMemcpy(st.data(), h->kinfo, sizeof(int) * st.size(), cudaMemcpyDeviceToHost));
  int worst = EXCFV_OK;
  for (int k = 0; k < nk; ++k) {
    const int v = status_to_info(&st[(size_t)k * ST_NWORDS], h->batch_nmat[k]);
    if (info) info[k] = v;
    if (worst == EXCFV_OK) worst = v;
  }
  return worst;
}

int excfv_set_lanes(excfv_handle* h, int32_t nlanes) {
  if (!h || nlanes < 0) return EXCFV_ERR_ARG;
  h->nlanes_pref = nlanes;
  return EXCFV_OK;
}

int excfv_get_lanes(excfv_handle* h) { return h ? h->nlanes_pref : EXCFV_ERR_ARG; }

int excfv_set_batch_mode(excfv_handle* h, int32_t mode) {
  if (!h || (mode != EXCFV_BATCH_LANES && mode != EXCFV_BATCH_GROUPED && mode != EXCFV_BATCH_AUTO &&
             mode != EXCFV_BATCH_GROUPED_LANES))
    return EXCFV_ERR_ARG;
  h->batch_mode = mode;
  return EXCFV_OK;
}

int excfv_get_batch_mode(excfv_handle* h) { return h ? h->batch_mode : EXCFV_ERR_ARG; }

long long excfv_group_launches(excfv_handle* h) { return h ? group_front_launches(h) : 0; }

int excfv_set_group_tile(excfv_handle* h, int32_t rows) {
  if (!h || (rows != 64 && rows != 128)) return EXCFV_ERR_ARG;
  h->group_tbm = rows;
  return EXCFV_OK;
}

int excfv_get_group_tile(excfv_handle* h) { return h ? h->group_tbm : EXCFV_ERR_ARG; }

static std::vector<unsigned long long> batch_key(const excfv_handle* h, const BatchArgs& b, int L) {
  std::vector<unsigned long long> k = {(unsigned long long)b.nk, (unsigned long long)L,
                                       (unsigned long long)h->prec, h->static_gen,
                                       (unsigned long long)h->batch_form,
                                       (unsigned long long)h->group_tbm,
                                       (unsigned long long)b.nmatmax, (unsigned long long)b.ngkmax,
                                       (unsigned long long)(uintptr_t)h->stream};
  for (int i = 0; i < b.nk; ++i) {
    k.push_back((unsigned long long)b.nmatp[i]);
    k.push_back((unsigned long long)b.ngp[i]);
    for (const void* ptr : {(const void*)b.gpc[i], (const void*)b.tpgpc[i], (const void*)b.sfacgp[i],
                            (const void*)b.igpig[i], (const void*)b.vgpc[i], (const void*)b.evalfv[i],
                            (const void*)b.evecfv[i]})
      k.push_back((unsigned long long)(uintptr_t)ptr);
  }
  return k;
}

static void drop_graph(excfv_handle* h) {
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  h->gexec = nullptr;
}

// A device-pointer batch that repeats the previous call exactly (same sizes,
// pointers, lanes, precision and per-SCF-iteration data) replays a CUDA graph
// captured on its second occurrence; the first occurrence runs eagerly and
// sizes every workspace.  If capture or instantiation fails, the batch runs
// eagerly and capture is not tried again for this key.
static int run_batch_graph(excfv_handle* h, const BatchArgs& b, int L) {
  std::vector<unsigned long long> key = batch_key(h, b, L);
  if (key != h->gkey) {
    drop_graph(h);
    h->gkey.swap(key);
    h->gseen = 0;
  }
  if (h->gexec) {
    CUDA_TRY(cudaGraphLaunch(h->gexec, h->stream));
    return EXCFV_OK;
  }
  if (h->gseen == 1) {
    h->gseen = 2;
    cudaGraph_t g = nullptr;
    if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      const int rc = enqueue_batch(h, b, L);
      const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
      cudaGraphExec_t ex = nullptr;
      if (rc == EXCFV_OK && e == cudaSuccess && g && cudaGraphInstantiate(&ex, g, 0) == cudaSuccess) {
        cudaGraphDestroy(g);
        h->gexec = ex;
        CUDA_TRY(cudaGraphLaunch(h->gexec, h->stream));
        return EXCFV_OK;
      }
      if (g) cudaGraphDestroy(g);
      (void)cudaGetLastError();
      g_err[0] = 0;
    }
    return enqueue_batch(h, b, L);
  }
  if (h->gseen < 2) h->gseen++;
  return enqueue_batch(h, b, L);
}

static BatchArgs make_batch(int32_t nk, const int32_t* nmatp, const int32_t* ngp, int32_t ngkmax,
                            const double* const* gpc, const double* const* tpgpc,
                            const double* const* sfacgp, const int32_t* const* igpig,
                            const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                            double* const* evecfv, bool host) {
  BatchArgs b;
  b.nk = nk; b.nmatp = nmatp; b.ngp = ngp; b.ngkmax = ngkmax; b.gpc = gpc; b.tpgpc = tpgpc;
  b.sfacgp = sfacgp; b.igpig = igpig; b.vgpc = vgpc; b.nmatmax = nmatmax; b.evalfv = evalfv;
  b.evecfv = evecfv; b.host = host;
  return b;
}

static int default_lanes(excfv_handle* h, const BatchArgs& b) {
  if (h->nlanes_pref > 0) return h->nlanes_pref;
  int nmax = 0;
  for (int k = 0; k < b.nk; ++k) nmax = std::max(nmax, (int)b.nmatp[k]);
  return std::min(8, max_lanes_for(h, nmax));
}

int excfv_seceqn_batched_dev(excfv_handle* h, int32_t nk, const int32_t* nmatp, const int32_t* ngp,
                             int32_t ngkmax, const double* const* gpc, const double* const* tpgpc,
                             const double* const* sfacgp, const int32_t* const* igpig,
                             const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                             double* const* evecfv) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  BatchArgs b = make_batch(nk, nmatp, ngp, ngkmax, gpc, tpgpc, sfacgp, igpig, vgpc, nmatmax, evalfv,
                           evecfv, false);
  return run_batch(h, b, default_lanes(h, b));
}

int excfv_seceqn_batched(excfv_handle* h, int32_t nk, const int32_t* nmatp, const int32_t* ngp,
                         int32_t ngkmax, const double* const* gpc, const double* const* tpgpc,
                         const double* const* sfacgp, const int32_t* const* igpig,
                         const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                         double* const* evecfv, int32_t* info) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  BatchArgs b = make_batch(nk, nmatp, ngp, ngkmax, gpc, tpgpc, sfacgp, igpig, vgpc, nmatmax, evalfv,
                           evecfv, true);
  int rc = run_batch(h, b, default_lanes(h, b));
  if (rc) return rc;
  return batch_info(h, nk, info);
}

int excfv_set_batch_graph(excfv_handle* h, int enable) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  h->graph_on = enable != 0;
  if (!h->graph_on) {
    drop_graph(h);
    h->gkey.clear();
    h->gseen = 0;
  }
  return EXCFV_OK;
}

int excfv_batch_info(excfv_handle* h, int32_t nk, int32_t* info) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  return batch_info(h, nk, info);
}

// Times the batch in every form (lanes; grouped front over the batch or per
// lane) with 1, 2, 4, 6, 8, 12, ... lanes (those the SM budget allows), then
// the winning grouped form with the other GEMM tile shape, and keeps the
// fastest form, lane count and tile shape for later batched calls.  Device pointers; the outputs of
// the last timed run are valid.  best_ms (optional) receives the winning time.
int excfv_autotune_lanes(excfv_handle* h, int32_t nk, const int32_t* nmatp, const int32_t* ngp,
                         int32_t ngkmax, const double* const* gpc, const double* const* tpgpc,
                         const double* const* sfacgp, const int32_t* const* igpig,
                         const double* const* vgpc, int32_t nmatmax, double* const* evalfv,
                         double* const* evecfv, double* best_ms) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  BatchArgs b = make_batch(nk, nmatp, ngp, ngkmax, gpc, tpgpc, sfacgp, igpig, vgpc, nmatmax, evalfv,
                           evecfv, false);
  int nmax = 0;
  int rc = check_batch(h, b, &nmax);
  if (rc) return rc;
  const int lmax = std::min(nk, max_lanes_for(h, nmax));
  cudaEvent_t e0, e1;
  CUDA_TRY(cudaEventCreate(&e0));
  CUDA_TRY(cudaEventCreate(&e1));
  float best = 1e30f;
  int bestL = 1, bestMode = EXCFV_BATCH_LANES, bestTbm = 64;
  const int cand[] = {1, 2, 4, 6, 8, 12, 16, 24, 32};
  h->group_tbm = 64;
  for (int mode : {EXCFV_BATCH_LANES, EXCFV_BATCH_GROUPED, EXCFV_BATCH_GROUPED_LANES}) {
    h->batch_mode = mode;
    for (int L : cand) {
      if (L > lmax) break;
      for (int rep = 0; rep < 2; ++rep) {  // the first run of a lane count sizes its workspaces
        CUDA_TRY(cudaEventRecord(e0, h->stream));
        if ((rc = run_batch(h, b, L))) break;
        CUDA_TRY(cudaEventRecord(e1, h->stream));
        CUDA_TRY(cudaEventSynchronize(e1));
      }
      if (rc) break;
      float ms = 0.f;
      CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) { best = ms; bestL = L; bestMode = mode; }
    }
    if (rc) break;
  }
  // the grouped forms' GEMM tile shape: 128 x 64 tiles against the 64 x 64 of
  // the search above, at the winning form and lane count
  if (rc == EXCFV_OK && bestMode != EXCFV_BATCH_LANES) {
    h->batch_mode = bestMode;
    h->group_tbm = 128;
    for (int rep = 0; rep < 2 && rc == EXCFV_OK; ++rep) {
      CUDA_TRY(cudaEventRecord(e0, h->stream));
      if ((rc = run_batch(h, b, bestL))) break;
      CUDA_TRY(cudaEventRecord(e1, h->stream));
      CUDA_TRY(cudaEventSynchronize(e1));
    }
    float ms = 0.f;
    if (rc == EXCFV_OK) {
      CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) { best = ms; bestTbm = 128; }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  h->nlanes_pref = bestL;
  h->batch_mode = bestMode;
  h->group_tbm = bestTbm;
  if (best_ms) *best_ms = best;
  rc = run_batch(h, b, bestL);
  if (rc) return rc;
  return batch_info(h, nk, nullptr);
}

int excfv_profile(excfv_handle* h, int enable) {
  if (!h) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  prof_collect(h);
  for (int c = 0; c < PROF_NCLS; ++c) { h->prof.ms[c] = 0.0; h->prof.cnt[c] = 0; }
  h->prof.on = enable != 0;
  for (excfv_handle* l : h->lanes) {
    prof_collect(l);
    for (int c = 0; c < PROF_NCLS; ++c) { l->prof.ms[c] = 0.0; l->prof.cnt[c] = 0; }
    l->prof.on = h->prof.on;
  }
  return EXCFV_OK;
}

int excfv_profile_read(excfv_handle* h, double* ms, long long* count, int nclasses) {
  if (!h || !ms || !count || nclasses < 0) return EXCFV_ERR_ARG;
  DeviceGuard g(h->device);
  prof_collect(h);
  for (excfv_handle* l : h->lanes) prof_collect(l);
  for (int c = 0; c < nclasses && c < PROF_NCLS; ++c) {
    ms[c] = h->prof.ms[c];
    count[c] = h->prof.cnt[c];
    h->prof.ms[c] = 0.0;
    h->prof.cnt[c] = 0;
    for (excfv_handle* l : h->lanes) {  // summed over lanes (their times overlap)
      ms[c] += l->prof.ms[c];
      count[c] += l->prof.cnt[c];
      l->prof.ms[c] = 0.0;
      l->prof.cnt[c] = 0;
    }
  }
  return EXCFV_OK;
}

int excfv_get_timings(excfv_handle* h, double* t4) {
  if (!h || !t4) return EXCFV_ERR_ARG;
  for (int i = 0; i < 4; ++i) t4[i] = h->timings[i];
  return EXCFV_OK;
}

}  // extern "C"
