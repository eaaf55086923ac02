// The grouped front of the batching form.
//
// A batch of k-points (the reference's k-loop, src/scf_cycle.f90:256-289)
// has one generalized eigenproblem per k-point, each of its own order n_k.
// The lanes of the batching form run every k-point's whole chain on its own
// stream; here the BLAS-3 front of the chain — ZPOTRF, the inverse factor
// and ZHEGST's two-sided reduction (external/LAPACK/zhegvx.f:410-418) — runs
// for all k-points of the batch together: each step is ONE launch over every
// k-point that has it (the diagonal Cholesky block of step j of all k-points,
// the row panels of all k-points, their trailing updates, ...), so a 64-k
// batch issues one launch where the lanes issue 64, and the latency-bound
// diagonal blocks of different k-points run side by side on different SMs.
//
// The batch's matrices live in four slot arrays (H, O, U^-1, scratch T) of
// nmax x nmax complex elements per k-point, leading dimension n_k.  The
// lanes' setup writes H and O into the slots, this front leaves C = U^-H H
// U^-1 (both triangles), U^-1 and, in the precision form, C's complex64 copy
// in T; the lanes then run the rest of each k-point's solve from the slots.
//
// Every launch's problems and tiles are known from the sizes alone, so the
// plan is built on the host and uploaded once per batch shape (before any
// stream capture); the launches read their descriptors from device memory.
#include <algorithm>

#include "handle.cuh"

struct GroupPlan {
  std::vector<unsigned long long> key;
  int nk = 0, nmax = 0;
  // slot arrays (capacity in k-points x nmax^2 complex elements)
  cplx* slot[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t slot_elems = 0;   // nmax * nmax of the allocation
  int slot_k = 0;
  // device descriptors
  ZgemmArgs* d_probs = nullptr;
  int4* d_tiles = nullptr;
  PotrfProb* d_potrf = nullptr;
  MirrorProb* d_mirror = nullptr;
  size_t cap_probs = 0, cap_tiles = 0, cap_potrf = 0, cap_mirror = 0;
  // the launch sequence
  enum { OPK_ZERO_STATUS, OPK_POTRF, OPK_GEMM, OPK_MIRROR, OPK_PROF_BEGIN, OPK_PROF_END };
  struct Op {
    int kind, a, b, off, cnt, kb;
  };
  std::vector<Op> ops;
  std::vector<int> seg_begin;  // ops of segment s: [seg_begin[s], seg_begin[s+1])
  std::vector<int> zero_k;     // k-points whose eigensolve status words a ZERO op clears
  long long launches = 0;
  int tbm = 64;                // rows of the grouped GEMM tiles
};

namespace {

template <typename T>
int grow(T** p, size_t* cap, size_t need) {
  if (need <= *cap) return EXCFV_OK;
  if (*p) cudaFree(*p);
  *p = nullptr;
  *cap = 0;
  const size_t n = std::max(need, (size_t)1);
  if (cudaMalloc((void**)p, n * sizeof(T)) != cudaSuccess) {
    *p = nullptr;
    (void)cudaGetLastError();
    excfv_set_error("grouped batch: device allocation of %zu bytes failed", n * sizeof(T));
    return EXCFV_ERR_ALLOC;
  }
  *cap = n;
  return EXCFV_OK;
}

ZgemmArgs gemm(int m, int n, int k, cplx alpha, const cplx* A, long long lda, const cplx* B, long long ldb,
               cplx beta, cplx* C, long long ldc, int uplo_c = TRI_NONE, int tri_a = TRI_NONE,
               int tri_b = TRI_NONE) {
  ZgemmArgs a;
  a.m = m; a.n = n; a.k = k; a.alpha = alpha; a.beta = beta;
  a.A = A; a.lda = lda; a.strideA = 0;
  a.B = B; a.ldb = ldb; a.strideB = 0;
  a.C = C; a.ldc = ldc; a.strideC = 0;
  a.batch = 1; a.uplo_c = uplo_c; a.tri_a = tri_a; a.tri_b = tri_b;
  a.splitk = 1; a.part = nullptr; a.kdec = 0;
  return a;
}

}  // namespace

void free_group(GroupPlan*& g) {
  if (!g) return;
  for (cplx*& p : g->slot)
    if (p) cudaFree(p);
  if (g->d_probs) cudaFree(g->d_probs);
  if (g->d_tiles) cudaFree(g->d_tiles);
  if (g->d_potrf) cudaFree(g->d_potrf);
  if (g->d_mirror) cudaFree(g->d_mirror);
  delete g;
  g = nullptr;
}

cplx* group_slot(excfv_handle* h, int which, int k) {
  GroupPlan* g = h->gplan;
  return g->slot[which] + g->slot_elems * (size_t)k;
}

long long group_front_launches(const excfv_handle* h) { return h->gplan ? h->gplan->launches : 0; }

bool group_slots_hold(const excfv_handle* h, int nk, int nmax) {
  const GroupPlan* g = h->gplan;
  return g && g->slot[0] && g->slot_elems == (size_t)nmax * nmax && g->slot_k >= nk;
}

// Builds (or keeps) the plan of the grouped front for a batch of nk k-points
// of orders nmatp[k] (status words of k-point k at h->kinfo + k ST_NWORDS),
// one op sequence per segment (a list of k-points grouped together).
// Allocates the slots and descriptors and uploads them; when the plan
// changes, the handle's stream is synchronised first (a previous batch may
// still read the old descriptors) and *rebuilt is set: a CUDA graph captured
// with the old plan must not be replayed.  Must not run inside a stream capture.
int group_plan_front(excfv_handle* h, int nk, const int32_t* nmatp, int nmax,
                     const std::vector<std::vector<int>>& segs, bool* rebuilt) {
  *rebuilt = false;
  if (!h->gplan) h->gplan = new GroupPlan();
  GroupPlan& P = *h->gplan;
  const int tbm = h->group_tbm;
  std::vector<unsigned long long> key = {(unsigned long long)nk, (unsigned long long)nmax,
                                         (unsigned long long)h->prec, (unsigned long long)tbm,
                                         (unsigned long long)(uintptr_t)h->kinfo};
  for (int k = 0; k < nk; ++k) key.push_back((unsigned long long)nmatp[k]);
  for (const std::vector<int>& ks : segs) {
    key.push_back(~0ull);
    for (int k : ks) key.push_back((unsigned long long)k);
  }
  const size_t S = (size_t)nmax * nmax;
  const bool slots_ok = P.slot[0] && P.slot_elems == S && P.slot_k >= nk;
  if (slots_ok && key == P.key) return EXCFV_OK;
  *rebuilt = true;
  CUDA_TRY(cudaStreamSynchronize(h->stream));
  int rc;
  if (!slots_ok) {
    for (cplx*& p : P.slot)
      if (p) { cudaFree(p); p = nullptr; }
    P.slot_k = 0;
    P.slot_elems = 0;
    for (cplx*& p : P.slot) {
      size_t cap = 0;
      if ((rc = grow(&p, &cap, S * (size_t)nk))) return rc;
    }
    P.slot_elems = S;
    P.slot_k = nk;
  }
  P.key.swap(key);
  P.nk = nk;
  P.nmax = nmax;
  P.tbm = tbm;
  P.ops.clear();
  P.seg_begin.clear();
  P.zero_k.clear();
  P.launches = 0;

  std::vector<ZgemmArgs> probs;
  std::vector<GroupTile> tiles;
  std::vector<PotrfProb> pp;
  std::vector<MirrorProb> mp;
  const cplx one = cmk(1.0, 0.0), mone = cmk(-1.0, 0.0), zero = cmk(0.0, 0.0);
  auto Hs = [&](int k) { return P.slot[0] + S * k; };
  auto Os = [&](int k) { return P.slot[1] + S * k; };
  auto Us = [&](int k) { return P.slot[2] + S * k; };
  auto Ts = [&](int k) { return P.slot[3] + S * k; };
  auto gemm_op = [&](int opA, int opB, size_t t0) {
    if (tiles.size() == t0) return;
    zgemm_group_order(tiles, t0);
    P.ops.push_back({GroupPlan::OPK_GEMM, opA, opB, (int)t0, (int)(tiles.size() - t0), 0});
    P.launches++;
  };
  const int NB = potrf_block();
  for (const std::vector<int>& ks : segs) {
    P.seg_begin.push_back((int)P.ops.size());
    int smax = 0;
    for (int k : ks) smax = std::max(smax, (int)nmatp[k]);
    const bool f32 = solve_front_f32copy(h, smax) != 0;
    P.ops.push_back({GroupPlan::OPK_ZERO_STATUS, 0, 0, (int)P.zero_k.size(), (int)ks.size(), 0});
    P.zero_k.insert(P.zero_k.end(), ks.begin(), ks.end());
    P.ops.push_back({GroupPlan::OPK_PROF_BEGIN, PROF_POTRF, 0, 0, 0, 0});
    // ZPOTRF, blocked right-looking: diagonal block, row panel, trailing update
    for (int kb = 0; kb < smax; kb += NB) {
      const size_t p0 = pp.size();
      for (int k : ks)
        if (nmatp[k] > kb)
          pp.push_back(PotrfProb{nmatp[k], (long long)nmatp[k], Os(k), Us(k), h->kinfo + (size_t)k * ST_NWORDS});
      if (pp.size() > p0) {
        P.ops.push_back({GroupPlan::OPK_POTRF, 0, 0, (int)p0, (int)(pp.size() - p0), kb});
        P.launches++;
      }
      size_t t0 = tiles.size();
      for (int k : ks) {
        const int n = nmatp[k];
        const long long ld = n;
        if (n <= kb) continue;
        const int b = std::min(NB, n - kb), rest = n - kb - b;
        if (rest <= 0) continue;
        cplx* panel = Os(k) + kb + ld * (kb + b);
        zgemm_group_add(gemm(b, rest, b, one, Us(k) + kb + ld * kb, ld, panel, ld, zero, panel, ld, TRI_NONE,
                             TRI_LOWER, TRI_NONE),
                        probs, tiles, tbm);
      }
      gemm_op(OP_C, OP_N, t0);
      t0 = tiles.size();
      for (int k : ks) {
        const int n = nmatp[k];
        const long long ld = n;
        if (n <= kb) continue;
        const int b = std::min(NB, n - kb), rest = n - kb - b;
        if (rest <= 0) continue;
        const cplx* panel = Os(k) + kb + ld * (kb + b);
        zgemm_group_add(gemm(rest, rest, b, mone, panel, ld, panel, ld, one, Os(k) + (kb + b) * (ld + 1), ld,
                             TRI_UPPER),
                        probs, tiles, tbm);
      }
      gemm_op(OP_C, OP_N, t0);
    }
    // U^-1: inverted diagonal blocks merged pairwise, level by level
    //   inv([[U11, U12], [0, U22]]) = [[X11, -X11 U12 X22], [0, X22]]
    for (int bs = NB; bs < smax; bs *= 2) {
      for (int half = 0; half < 2; ++half) {
        const size_t t0 = tiles.size();
        for (int k : ks) {
          const int n = nmatp[k];
          const long long ld = n;
          if (bs >= n) continue;
          const cplx* U = Os(k);
          cplx* Ui = Us(k);
          cplx* T = Ts(k);
          const int nfull = n / (2 * bs), rem = n - nfull * 2 * bs;
          const long long step = 2LL * bs * (ld + 1);
          for (int q = 0; q < nfull; ++q) {
            if (half == 0)  // T = U12 X22
              zgemm_group_add(gemm(bs, bs, bs, one, U + ld * bs + q * step, ld, Ui + bs * (ld + 1) + q * step, ld,
                                   zero, T + (size_t)q * bs * bs, bs, TRI_NONE, TRI_NONE, TRI_UPPER),
                              probs, tiles, tbm);
            else  // X12 = -X11 T
              zgemm_group_add(gemm(bs, bs, bs, mone, Ui + q * step, ld, T + (size_t)q * bs * bs, bs, zero,
                                   Ui + ld * bs + q * step, ld, TRI_NONE, TRI_UPPER, TRI_NONE),
                              probs, tiles, tbm);
          }
          if (rem > bs) {  // a trailing pair whose second block is shorter
            const int a0 = nfull * 2 * bs, d0 = a0 + bs, sd = n - d0;
            cplx* Tq = T + (size_t)nfull * bs * bs;
            if (half == 0)
              zgemm_group_add(gemm(bs, sd, sd, one, U + a0 + ld * d0, ld, Ui + d0 + ld * d0, ld, zero, Tq, bs,
                                   TRI_NONE, TRI_NONE, TRI_UPPER),
                              probs, tiles, tbm);
            else
              zgemm_group_add(gemm(bs, sd, bs, mone, Ui + a0 + ld * a0, ld, Tq, bs, zero, Ui + a0 + ld * d0, ld,
                                   TRI_NONE, TRI_UPPER, TRI_NONE),
                              probs, tiles, tbm);
          }
        }
        gemm_op(OP_N, OP_N, t0);
      }
    }
    P.ops.push_back({GroupPlan::OPK_PROF_END, PROF_POTRF, 0, 0, 0, 0});
    P.ops.push_back({GroupPlan::OPK_PROF_BEGIN, PROF_HEGST, 0, 0, 0, 0});
    // ZHEGST: T = H U^-1, C = U^-H T (upper), then both triangles
    size_t t0 = tiles.size();
    for (int k : ks) {
      const int n = nmatp[k];
      zgemm_group_add(gemm(n, n, n, one, Hs(k), n, Us(k), n, zero, Ts(k), n, TRI_NONE, TRI_NONE, TRI_UPPER), probs,
                      tiles, tbm);
    }
    gemm_op(OP_N, OP_N, t0);
    t0 = tiles.size();
    for (int k : ks) {
      const int n = nmatp[k];
      zgemm_group_add(gemm(n, n, n, one, Us(k), n, Ts(k), n, zero, Hs(k), n, TRI_UPPER, TRI_LOWER, TRI_NONE), probs,
                      tiles, tbm);
    }
    gemm_op(OP_C, OP_N, t0);
    const int m0 = (int)mp.size();
    for (int k : ks) {
      const int n = nmatp[k];
      const bool fk = f32 && solve_front_f32copy(h, n);
      mp.push_back(MirrorProb{n, (long long)n, Hs(k), fk ? reinterpret_cast<float2*>(Ts(k)) : nullptr,
                              (long long)((n + 1) & ~1)});
    }
    P.ops.push_back({GroupPlan::OPK_MIRROR, 0, 0, m0, (int)ks.size(), smax});
    P.launches++;
    P.ops.push_back({GroupPlan::OPK_PROF_END, PROF_HEGST, 0, 0, 0, 0});
  }
  P.seg_begin.push_back((int)P.ops.size());

  // upload
  std::vector<int4> t4(tiles.size());
  for (size_t i = 0; i < tiles.size(); ++i) t4[i] = make_int4(tiles[i].prob, tiles[i].ti, tiles[i].tj, 0);
  if ((rc = grow(&P.d_probs, &P.cap_probs, probs.size()))) return rc;
  if ((rc = grow(&P.d_tiles, &P.cap_tiles, t4.size()))) return rc;
  if ((rc = grow(&P.d_potrf, &P.cap_potrf, pp.size()))) return rc;
  if ((rc = grow(&P.d_mirror, &P.cap_mirror, mp.size()))) return rc;
  CUDA_TRY(cudaMemcpy(P.d_probs, probs.data(), sizeof(ZgemmArgs) * probs.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(P.d_tiles, t4.data(), sizeof(int4) * t4.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(P.d_potrf, pp.data(), sizeof(PotrfProb) * pp.size(), cudaMemcpyHostToDevice));
  CUDA_TRY(cudaMemcpy(P.d_mirror, mp.data(), sizeof(MirrorProb) * mp.size(), cudaMemcpyHostToDevice));
  return EXCFV_OK;
}

// Enqueues segment seg of the planned front on stream s; its stage events go
// to the profile of handle ph (no allocation, no host synchronisation: safe
// inside a stream capture).
int group_enqueue_front(excfv_handle* h, int seg, cudaStream_t s, excfv_handle* ph) {
  GroupPlan& P = *h->gplan;
  int rc;
  for (int i = P.seg_begin[seg]; i < P.seg_begin[seg + 1]; ++i) {
    const GroupPlan::Op& op = P.ops[i];
    switch (op.kind) {
      case GroupPlan::OPK_ZERO_STATUS:
        // eigensolve words of the segment's k-points (the setup's word is kept)
        for (int q = 0; q < op.cnt; ++q)
          CUDA_TRY(cudaMemsetAsync(h->kinfo + (size_t)P.zero_k[op.off + q] * ST_NWORDS, 0, sizeof(int) * ST_SETUP, s));
        break;
      case GroupPlan::OPK_POTRF:
        if ((rc = potrf_diag_grouped(s, P.d_potrf + op.off, op.cnt, op.kb))) return rc;
        break;
      case GroupPlan::OPK_GEMM:
        if ((rc = zgemm_grouped(s, op.a, op.b, P.d_probs, P.d_tiles + op.off, op.cnt, P.tbm))) return rc;
        break;
      case GroupPlan::OPK_MIRROR:
        if ((rc = mirror_grouped(s, P.d_mirror + op.off, op.cnt, op.kb))) return rc;
        break;
      case GroupPlan::OPK_PROF_BEGIN:
        prof_begin(ph, op.a);
        break;
      case GroupPlan::OPK_PROF_END:
        prof_end(ph, op.a);
        break;
    }
  }
  return EXCFV_OK;
}
