// C ABI of libanb.so: context, device memory, SIMPLE orchestration (include/anb.h).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "context.hpp"
#include "context_access.hpp"
#include "setup_gpu.hpp"

namespace anb {

// Message of the last failed anb_create on this thread (anb_last_error(NULL)).
thread_local std::string g_createError = "no context";

int fail(anb_ctx* c, const AnbError& e) {
  if (c) c->err = e.what();
  return e.code;
}


void permute_in(const anb_ctx* c, const double* src, std::vector<double>& dst, int comps) {
  dst.resize((size_t)comps * c->C);
  for (int q = 0; q < comps; ++q)
    for (int r = 0; r < c->C; ++r) dst[(size_t)q * c->C + r] = src[(size_t)q * c->C + c->L.new2old[r]];
}

// Cell fields cross the host/device boundary in input numbering.  Upload: the host copies the
// caller's arrays into the pinned staging buffer chunk by chunk, each chunk's DMA running while the
// next one is copied, and one kernel gathers the staged fields into layout numbering.  Download: the
// kernel gathers into input numbering, the DMAs go out chunk by chunk and each chunk is copied to
// the caller's array as soon as its event has completed.  No permutation runs on the host.
size_t stage_chunk(size_t C) { return std::max<size_t>((size_t)1 << 18, (C + 15) / 16); }

void host_copy(double* d, const double* s, size_t n) {
  constexpr size_t kB = 8192;
  const ptrdiff_t nb = (ptrdiff_t)((n + kB - 1) / kB);
#pragma omp parallel for schedule(static) if (nb > 8)
  for (ptrdiff_t b = 0; b < nb; ++b) {
    const size_t o = (size_t)b * kB;
    std::memcpy(d + o, s + o, sizeof(double) * std::min(kB, n - o));
  }
}

void upload_cells(anb_ctx* c, const double* const* src, double* const* dst, int comps) {
  if (comps < 1 || comps > 4) throw AnbError(ANB_ERR_INVALID, "upload of more than 4 cell fields");
  const size_t C = c->C, ch = stage_chunk(C);
  PermuteArgs a{};
  a.idx = c->dN2O;
  a.n = c->C;
  a.comps = comps;
  for (int q = 0; q < comps; ++q) {
    double* h = c->hStage + q * C;
    double* d = c->dStage + q * C;
    for (size_t o = 0; o < C; o += ch) {
      const size_t n = std::min(ch, C - o);
      host_copy(h + o, src[q] + o, n);
      CK(cudaMemcpyAsync(d + o, h + o, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    a.src[q] = d;
    a.dst[q] = dst[q];
  }
  launch_permute_cells(c->lc, a);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(c->stream));
}

void upload_cells(anb_ctx* c, const double* const* src, double* dst, int comps) {
  double* d[4] = {};
  for (int q = 0; q < comps && q < 4; ++q) d[q] = dst + (size_t)q * c->C;
  upload_cells(c, src, d, comps);
}

void download_cells(anb_ctx* c, const double* const* src, double* const* dst, int comps) {
  if (comps < 1 || comps > 4) throw AnbError(ANB_ERR_INVALID, "download of more than 4 cell fields");
  const size_t C = c->C, ch = stage_chunk(C);
  PermuteArgs a{};
  a.idx = c->dO2N;
  a.n = c->C;
  double* out[4] = {};
  for (int q = 0; q < comps; ++q) {
    if (!dst[q]) continue;
    a.src[a.comps] = src[q];
    a.dst[a.comps] = c->dStage + a.comps * C;
    out[a.comps++] = dst[q];
  }
  if (a.comps == 0) return;
  launch_permute_cells(c->lc, a);
  CK(cudaGetLastError());
  int ev = 0;
  for (int k = 0; k < a.comps; ++k)
    for (size_t o = 0; o < C; o += ch) {
      const size_t n = std::min(ch, C - o);
      CK(cudaMemcpyAsync(c->hStage + k * C + o, c->dStage + k * C + o, n * sizeof(double),
                         cudaMemcpyDeviceToHost, c->stream));
      CK(cudaEventRecord(c->stageEv[ev++], c->stream));
    }
  ev = 0;
  for (int k = 0; k < a.comps; ++k)
    for (size_t o = 0; o < C; o += ch) {
      CK(cudaEventSynchronize(c->stageEv[ev++]));
      host_copy(out[k] + o, c->hStage + k * C + o, std::min(ch, C - o));
    }
}

void download_cells(anb_ctx* c, const double* src, double* const* dst, int comps) {
  const double* s[4] = {};
  for (int q = 0; q < comps && q < 4; ++q) s[q] = src + (size_t)q * c->C;
  download_cells(c, s, dst, comps);
}

// Face array on the device (new order, new orientation) -> input order and orientation.
void download_faces(anb_ctx* c, const double* src, double* dst) {
  const int nF = c->nI + c->nB;
  std::vector<double> h(nF);
  CK(cudaMemcpyAsync(h.data(), src, nF * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int fi = 0; fi < c->nI; ++fi) dst[c->L.fOrig[fi]] = c->L.fFlip[fi] ? -h[fi] : h[fi];
  for (int b = 0; b < c->nB; ++b) dst[c->nI + b] = h[c->nI + b];
}

// Off-diagonal matrix values per input face in input orientation.
void download_offdiag(anb_ctx* c, const double* val, double* a_pn, double* a_np) {
  std::vector<double> h(c->nEnt);
  CK(cudaMemcpyAsync(h.data(), val, h.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  for (int fi = 0; fi < c->nI; ++fi) {
    const double own = h[c->slotOwn[fi]], nei = h[c->slotNei[fi]];
    const int f = c->L.fOrig[fi];
    const bool flip = c->L.fFlip[fi] != 0;
    if (a_pn) a_pn[f] = flip ? nei : own;
    if (a_np) a_np[f] = flip ? own : nei;
  }
}

DSell mom_sell(const anb_ctx* c) {
  return DSell{c->C, c->L.sliceOff.empty() ? nullptr : c->dm.sliceOff, c->dm.col, c->mval, c->mdiag, c->L.maxRowLen};
}
DSell p_sell(const anb_ctx* c) { return DSell{c->C, c->dm.sliceOff, c->dm.col, c->pval, c->pdiag, c->L.maxRowLen}; }

void grad(anb_ctx* c, int nf, const double* const* phi, const unsigned char* bits, double* const* out) {
  GradArgs a{};
  a.nf = nf;
  for (int f = 0; f < nf; ++f) {
    a.phi[f] = phi[f];
    a.bit[f] = bits[f];
    const int q = bits[f] == 1 ? 0 : bits[f] == 2 ? 1 : bits[f] == 4 ? 2 : 3;
    a.bval[f] = c->dBVal + (size_t)q * c->nB;
    a.g[f] = out[f];
  }
  launch_lsq_grad(c->lc, c->dm, a);
}

void poll(anb_ctx* c, const int* dflags, int count) {
  CK(cudaMemcpyAsync(c->hFlags, dflags, sizeof(int) * count, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

// Outcome of one linear solve: iterations and convergence per component, or, for a solve that ran
// as a loop graph with its read-back deferred, the hDefer slot its flags arrive in once the stream
// has synchronised (resolve_solve).
struct SolveOut {
  bool momentum = false;
  bool resolved = false;
  int slot = -1;
  int active[3] = {1, 1, 1};
  int its[3] = {0, 0, 0};
  bool conv[3] = {true, true, true};
  long long kernelsPerIteration = 0;  // loop-graph launch bookkeeping
};

// Queues the copy of a loop-graph solve's flags into the next hDefer slot; with every slot taken it
// polls instead (slot -1, flags in hFlags).
int defer_flags(anb_ctx* c, const int* dflags, int count) {
  if (c->nDefer >= kDeferSlots) {
    poll(c, dflags, count);
    return -1;
  }
  const int slot = c->nDefer++;
  CK(cudaMemcpyAsync(c->hDefer + slot * kDeferInts, dflags, sizeof(int) * count, cudaMemcpyDeviceToHost,
                     c->stream));
  return slot;
}

// Fills a solve's iterations and convergence from its flags (hDefer slot, after the stream has
// synchronised, or hFlags right after a poll) and books the kernels its loop graph ran: one
// condition kernel per evaluation, two iterations per body run.
void resolve_solve(anb_ctx* c, SolveOut& o) {
  if (o.resolved) return;
  o.resolved = true;
  const int* f = o.slot >= 0 ? c->hDefer + o.slot * kDeferInts : c->hFlags;
  if (o.momentum) {
    int mx = 0;
    for (int q = 0; q < 3; ++q) {
      o.its[q] = o.active[q] ? f[4 * q + 2] : 0;
      o.conv[q] = o.active[q] ? f[4 * q + 3] != 0 : true;
      mx = std::max(mx, o.its[q]);
    }
    c->lastMomIts = std::max(1, mx);
  } else {
    o.its[0] = f[1];
    o.conv[0] = f[2] != 0;
    c->lastPIts = std::max(1, o.its[0]);
  }
  if (o.kernelsPerIteration > 0) {
    const int trips = f[o.momentum ? 12 : 4];
    g_launches += trips + 2LL * std::max(trips - 1, 0) * o.kernelsPerIteration;
  }
}

// Momentum: nc-component BiCGSTAB + Jacobi on the shared matrix; comps with active[q]==0 are
// frozen.  Returns per-component iterations and convergence.
void solve_momentum_mixed(anb_ctx* c, const int* active, int its[3], bool conv[3]);
void solve_pressure_mixed(anb_ctx* c, const double* b, double* x, double rtol, int* its, bool* conv);

// Right preconditioner of the momentum BiCGSTAB with mom_amg: one V-cycle of the momentum
// hierarchy for component q after the p update (which = 0) or the s update (which = 1).
void mom_apply(void* ctx, int q, int which) {
  anb_ctx* c = static_cast<anb_ctx*>(ctx);
  amg_apply(c->lc, c->momArgs[2 * q + which], &c->amgMom, &c->momGraph[2 * q + which]);
}

// The BiCGSTAB iterations after bicg_init until every component is done: one launch of the loop
// graph when it applies (no preconditioner callback, no BiCGSTAB kernel family being timed), else
// batches of iterations (most of the previous solve's count, then two) with a poll after each.
// Iterations after convergence return at once either way.  Returns the iterations enqueued by the
// host loop (0 for the loop graph).  Afterwards the flags are in hFlags, or, for the loop graph
// with `out` given, on their way to out->slot.
template <class T>
int bicg_iterate(anb_ctx* c, const BicgArgsT<T>& a, BicgLoopT<T>& loop, SolveOut* out) {
  const int fam = c->prof.family;
  const bool timed = fam == kKfBicgSpmv || fam == kKfBicgVector;
  if (!timed && bicg_loop_launch(c->lc, a, loop)) {
    if (out) {
      out->kernelsPerIteration = 5;
      out->slot = defer_flags(c, a.fl, 13);
      return 0;
    }
    poll(c, a.fl, 13);
    const int trips = c->hFlags[12];
    g_launches += trips + 10LL * std::max(trips - 1, 0);
    return 0;
  }
  int done = 0;
  int batch = std::max(2, std::min(3 * c->lastMomIts / 4, 32));
  while (true) {
    for (int k = 0; k < batch; ++k) {
      if (a.precond) bicg_iteration_precond(c->lc, a, mom_apply, c);
      else bicg_iteration(c->lc, a);
    }
    done += batch;
    poll(c, a.fl, 12);
    bool all = true;
    for (int q = 0; q < a.nc; ++q) all = all && c->hFlags[4 * q];
    if (all || done > a.maxit + 2) break;
    batch = 2;
  }
  return done;
}

// Momentum solve.  With defer (and the loop graph), out is resolved after the step's
// synchronisation (resolve_solve); otherwise on return.
void solve_momentum(anb_ctx* c, const int* active, SolveOut* out, bool defer) {
  ProfScope whole(c->lc, kKfMomentumSolve, 0.0, 0);
  out->momentum = true;
  for (int q = 0; q < 3; ++q) out->active[q] = active[q];
  if (c->mixed) {
    solve_momentum_mixed(c, active, out->its, out->conv);
    out->resolved = true;
    return;
  }
  BicgArgs a{};
  a.A = mom_sell(c);
  a.nc = 3;
  a.b = c->rhs;
  a.x = c->Us;
  a.r = c->bw[0]; a.rh = c->bw[1]; a.p = c->bw[2]; a.v = c->bw[3];
  a.s = c->bw[4]; a.t = c->bw[5]; a.ph = c->bw[6]; a.sh = c->bw[7];
  a.sc = c->scal + kScalBicg;
  a.fl = c->flags + kFlagBicg;
  a.atol = c->prm.vel_tol;
  a.rtol = c->prm.vel_rel_tol;
  a.maxit = c->prm.vel_maxit;
  a.red = c->red;
  a.precond = (c->prm.mom_amg && c->momAmgBuilt && c->amgMom.nLevels >= 2) ? 1 : 0;
  bicg_init(c->lc, a);
  // freeze inactive components
  for (int q = 0; q < 3; ++q)
    if (!active[q]) {
      const int one[4] = {1, 0, 0, 1};
      CK(cudaMemcpyAsync(a.fl + 4 * q, one, sizeof(one), cudaMemcpyHostToDevice, c->stream));
    }
  const int done = bicg_iterate(c, a, c->momLoop, defer ? out : nullptr);
  if (defer && out->slot >= 0) return;
  resolve_solve(c, *out);
  const int* its = out->its;
  if (c->prof.family == kKfBicgSpmv) {  // count only the components each launch worked on
    double booked = 2.0 * done * c->ab.bicg_spmv(3), real = 0.0;
    long long realLaunches = 0;
    for (int k = 1; k <= done; ++k) {
      int n = 0;
      for (int q = 0; q < 3; ++q) n += its[q] >= k ? 1 : 0;
      if (n > 0) {
        real += 2.0 * c->ab.bicg_spmv(n);
        realLaunches += 2;
      }
    }
    c->prof.bytes += real - booked;
    c->prof.launches += realLaunches - 2LL * done;
  }
}

void ensure_amg(anb_ctx* c);

// FP64 PCG arguments; the iterate is the context's fixed work vector pxw (copy the caller's x in
// before pcg_init and out after the solve).
PcgArgs pcg_args(anb_ctx* c, const double* b, double rtol) {
  PcgArgs a{};
  a.A = p_sell(c);
  a.b = b;
  a.x = c->pxw;
  a.r = c->pr; a.z = c->pz; a.p0 = c->pp0; a.p1 = c->pp1; a.q = c->pq;
  a.r2 = c->pr2;
  a.sc = c->scal + kScalPcg;
  a.fl = c->flags + kFlagPcg;
  a.atol = c->prm.p_tol;
  a.rtol = rtol;
  a.maxit = c->prm.p_maxit;
  a.red = c->red;
  return a;
}

// The PCG iterations after pcg_init + pcg_precondition, until the solve is done: one launch of the
// hierarchy's loop graph when it holds one for these arguments (and no PCG or V-cycle kernel family
// is being timed), else batches of pcg_iteration, most of the expected iterations (previous
// solve's count) before the first poll, then small batches.  Iterations after convergence return
// at once either way.  Returns the iterations enqueued by the host loop (0 for the loop graph).
// Afterwards the PCG flags are in hFlags, or, for the loop graph with `out` given, on their way to
// out->slot.
template <class T>
int pcg_iterate(anb_ctx* c, const PcgArgsT<T>& a, const AmgDevT<T>* amg, SolveOut* out = nullptr) {
  const int fam = c->prof.family;
  const bool timed = fam >= kKfPcgSpmv && fam <= kKfPcgUpdate;
  if (amg && !timed && pcg_loop_launch(c->lc, a, *amg)) {
    if (out) {
      out->kernelsPerIteration = 1 + amg->graphKernels;
      out->slot = defer_flags(c, a.fl, 5);
      return 0;
    }
    poll(c, a.fl, 5);
    const int trips = c->hFlags[4];
    g_launches += trips + 2LL * std::max(trips - 1, 0) * (1 + amg->graphKernels);
    return 0;
  }
  int it = 0;
  int batch = std::max(2, std::min(3 * c->lastPIts / 4, 64));
  const int tail = std::max(2, c->lastPIts / 8);
  while (true) {
    for (int k = 0; k < batch; ++k) pcg_iteration(c->lc, a, it++, amg);
    poll(c, a.fl, 4);
    if (c->hFlags[0] || it > a.maxit + 2) break;
    batch = tail;
  }
  return it;
}

// Pressure: PCG with the AMG (or Jacobi) preconditioner; x holds the initial guess.  With defer
// (and the loop graph), out is resolved after the step's synchronisation (resolve_solve);
// otherwise on return.
void solve_pressure(anb_ctx* c, const double* b, double* x, double rtol, SolveOut* out, bool defer) {
  ProfScope whole(c->lc, kKfPressureSolve, 0.0, 0);
  if (c->mixed) {
    solve_pressure_mixed(c, b, x, rtol, &out->its[0], &out->conv[0]);
    out->resolved = true;
    return;
  }
  PcgArgs a = pcg_args(c, b, rtol);
  const AmgDev* amg = (c->prm.p_use_amg && c->amgBuilt && c->amg.nLevels >= 2) ? &c->amg : nullptr;
  CK(cudaMemcpyAsync(c->pxw, x, sizeof(double) * c->C, cudaMemcpyDeviceToDevice, c->stream));
  pcg_init(c->lc, a);
  pcg_precondition(c->lc, a, amg);
  const int it = pcg_iterate(c, a, amg, defer ? out : nullptr);
  CK(cudaMemcpyAsync(x, c->pxw, sizeof(double) * c->C, cudaMemcpyDeviceToDevice, c->stream));
  if (defer && out->slot >= 0) return;
  resolve_solve(c, *out);
  if (c->prof.family == kKfPcgSpmv) {  // launches after convergence returned at once: not counted
    c->prof.bytes -= (double)(it - out->its[0]) * c->ab.pcg_spmv();
    c->prof.launches -= it - out->its[0];
  }
}

void solve_pressure(anb_ctx* c, const double* b, double* x, double rtol, int* its, bool* conv) {
  SolveOut o;
  solve_pressure(c, b, x, rtol, &o, false);
  *its = o.its[0];
  *conv = o.conv[0];
}

PcgArgsT<float> pcg_args32(anb_ctx* c, const float* b, float* x, double atol, double rtol) {
  PcgArgsT<float> a{};
  a.A = DSellT<float>{c->C, c->dm.sliceOff, c->dm.col, c->pval32, c->pdiag32, c->L.maxRowLen};
  a.b = b;
  a.x = x;
  a.r = c->pr32; a.z = c->pz32; a.p0 = c->pp0_32; a.p1 = c->pp1_32; a.q = c->pq32;
  a.r2 = c->pr2_32;
  a.sc = c->scal + kScalPcg;
  a.fl = c->flags + kFlagPcg;
  a.atol = atol;
  a.rtol = rtol;
  a.maxit = c->prm.p_maxit;
  a.red = c->red;
  return a;
}

// Coarse levels of at most this many rows run as one cluster kernel (ANB_AMG_TAIL_ROWS overrides;
// 0 launches every level and sweep separately).  The arithmetic is the same either way.
constexpr int kAmgTailRows = 1024;
// CSR levels of at most this many rows run down sweep + restriction as one kernel
// (ANB_AMG_FUSED_DOWN_ROWS overrides; 0 = off).  Same values either way.
constexpr int kAmgFusedDownRows = 65536;

// Grid of the row-parallel kernels: at most this many 256-thread blocks per SM (grid-stride
// beyond); ANB_BLOCKS_PER_SM overrides.
constexpr int kBlocksPerSM = 8;

// Aggregation hierarchy for the current level-0 matrix (val0/diag0 on the device, storage type T),
// coarse levels in T, coarsest inverse in double, host structure in H, device arrays in ar.  For the
// pressure hierarchy (ga != nullptr) the PCG V-cycles are captured as graphs for *ga.
template <class T>
void build_amg(anb_ctx* c, AmgDevT<T>& A, std::vector<AmgLevelHost>& H, DevArena& ar, T* val0, T* diag0, T* wdinv0,
               const PcgArgsT<T>* ga) {
  std::vector<T> hv(c->nEnt), hd(c->C);
  CK(cudaMemcpyAsync(hv.data(), val0, hv.size() * sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaMemcpyAsync(hd.data(), diag0, hd.size() * sizeof(T), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  AmgSetupOptions opt;
  if (const char* sr = std::getenv("ANB_AMG_SELL_MIN_ROWS")) opt.sellMinRows = std::atoi(sr);
  if (const char* ps = std::getenv("ANB_AMG_PASSES")) {  // e.g. "2,2,3": passes per level
    for (const char* q = ps; *q;) {
      opt.passes.push_back(std::max(1, std::atoi(q)));
      while (*q && *q != ',') ++q;
      if (*q == ',') ++q;
    }
  }
  H = build_amg_hierarchy(c->L, std::vector<double>(hv.begin(), hv.end()),
                                   std::vector<double>(hd.begin(), hd.end()), opt);
  A.nLevels = (int)H.size();
  for (int l = 0; l < A.nLevels; ++l) {
    const AmgLevelHost& h = H[l];
    AmgLevelDevT<T>& d = A.lv[l];
    d = AmgLevelDevT<T>{};
    d.n = h.n;
    d.nc = h.nc;
    if (l == 0) {
      d.sliceOff = c->dm.sliceOff;
      d.col = c->dm.col;
      d.val = val0;
      d.diag = diag0;
      d.wdinv = wdinv0;
      d.maxW = c->L.maxRowLen;
    } else {
      if (!h.sliceOff.empty()) {
        d.sliceOff = ar.upload(h.sliceOff);
        d.maxW = h.maxW;
      } else {
        d.rowOff = ar.upload(h.rowOff);
      }
      d.col = ar.upload(h.col);
      d.val = ar.alloc<T>(std::max(h.nStore, 1));
      d.diag = ar.alloc<T>(h.n);
      d.b = ar.alloc<T>(h.n);
      d.wdinv = ar.alloc<T>(h.n);
    }
    d.x = ar.alloc<T>(h.n);
    d.x2 = ar.alloc<T>(h.n);
    if (l + 1 < A.nLevels) {
      d.agg = ar.upload(h.agg);
      d.memOff = ar.upload(h.memOff);
      d.mem = ar.upload(h.mem);
      if (l > 0 && h.sliceOff.empty()) {  // CSR level: the sweeps' shortcut indices
        std::vector<int> colAgg(h.col.size());
        for (size_t k = 0; k < h.col.size(); ++k) colAgg[k] = h.agg[h.col[k]];
        std::vector<int2> memRow(h.mem.size());
        for (size_t m = 0; m < h.mem.size(); ++m) memRow[m] = make_int2(h.rowOff[h.mem[m]], h.rowOff[h.mem[m] + 1]);
        d.colAgg = ar.upload(colAgg);
        d.memRow = ar.upload(memRow);
      }
      d.gOff = ar.upload(h.gOff);
      d.gIdx = ar.upload(h.gIdx);
      d.nEntNext = H[l + 1].nStore;
    }
  }
  const int nd = H.back().n;
  if (nd > 160) throw AnbError(ANB_ERR_UNSUPPORTED, "AMG coarsest level too large (" + std::to_string(nd) + ")");
  A.nDense = nd;
  A.dense = ar.alloc<double>((size_t)nd * nd);
  if (ga) c->amgBuilt = true;
  const char* tailEnv = std::getenv("ANB_AMG_TAIL_ROWS");
  amg_configure_tail(A, tailEnv ? std::atoi(tailEnv) : kAmgTailRows, c->stream);
  const char* fdEnv = std::getenv("ANB_AMG_FUSED_DOWN_ROWS");
  A.fusedDownRows = fdEnv ? std::atoi(fdEnv) : kAmgFusedDownRows;
  const char* verbose = std::getenv("ANB_AMG_VERBOSE");
  if (verbose && verbose[0] == '1') {
    std::fprintf(stderr, "AMG levels (rows/stored entries/max width):");
    for (int l = 0; l < A.nLevels; ++l)
      std::fprintf(stderr, " %d/%lld/%d", A.lv[l].n, l == 0 ? (long long)c->nEnt : (long long)H[l].nStore,
                   l == 0 ? c->L.maxRowLen : H[l].maxW);
    std::fprintf(stderr, " | tail rows %d, cluster %d\n", A.tailRows, A.tailCluster);
  }
  const char* noGraph = std::getenv("ANB_NO_GRAPH");
  if (ga && A.nLevels >= 2 && !(noGraph && noGraph[0] == '1')) CK(amg_capture_graph(c->lc, *ga, A));
}

// Momentum AMG (mom_amg): Jacobi weights of the freshly assembled matrix, the hierarchy on first
// use (its structure is kept; every full assembly refreshes the coarse values), and the arguments
// of the six V-cycle applications (component q, on p or on s) of the preconditioned BiCGSTAB.
void mom_amg_refresh(anb_ctx* c) {
  launch_jacobi_weights(c->lc, c->C, c->amgMom.omega, c->mdiag, c->mwdinv);
  if (!c->momAmgBuilt) {
    build_amg<double>(c, c->amgMom, c->amgMomHost, c->amgMomArena, c->mval, c->mdiag, c->mwdinv, nullptr);
    c->momAmgBuilt = true;
    const size_t C = c->C;
    for (int q = 0; q < 3; ++q)
      for (int which = 0; which < 2; ++which) {
        PcgArgs& m = c->momArgs[2 * q + which];
        m = PcgArgs{};
        m.A = mom_sell(c);
        m.mode = 1;
        m.r = (which ? c->bw[4] : c->bw[2]) + q * C;  // s or p of component q
        m.z = (which ? c->bw[7] : c->bw[6]) + q * C;  // sh or ph
        m.b = m.r;
        m.r2 = c->momScratch;
        m.x = m.q = m.p0 = m.p1 = c->momScratch;    // not read in mode 1
        m.fl = c->flags + kFlagBicg + 4 * q;          // the component's done flag
        m.sc = c->momSc;
        m.red = c->red;
      }
  }
  if (c->amgMom.nLevels >= 2) amg_refresh(c->lc, c->amgMom);
}

void ensure_amg(anb_ctx* c) {
  if (!c->prm.p_use_amg) return;
  if (c->mixed) {
    if (!c->amgBuilt) {
      const PcgArgsT<float> ga = pcg_args32(c, c->r32, c->dx32, 0.0, 0.0);
      build_amg<float>(c, c->amg32, c->amgHost, c->amgArena, c->pval32, c->pdiag32, c->pwdinv32, &ga);
    }
    if (c->amg32.nLevels >= 2) amg_refresh(c->lc, c->amg32);
    return;
  }
  if (!c->amgBuilt) {
    const PcgArgs ga = pcg_args(c, c->pb, 0.0);
    build_amg<double>(c, c->amg, c->amgHost, c->amgArena, c->pval, c->pdiag, c->pwdinv, &ga);
  }
  if (c->amg.nLevels >= 2) amg_refresh(c->lc, c->amg);
}

constexpr int kScalDefect = 32;  // 3 * 8
constexpr int kFlagDefect = 16;  // 3 * 4
constexpr int kFlagFrozen = 28;  // 3

// Mixed precision: FP64 defect correction around FP32 inner solves.  Each sweep forms the FP64
// residual r = b - A x with the float matrix and stops once |r| <= target = max(atol, rtol |b|);
// otherwise it solves A dx = r in FP32, down to half the target or to a relative reduction
// innerRtol, whichever is reached first (FP32 resolves about six digits of r), and adds dx to x.
// Returns per-component inner iterations and convergence.
void solve_momentum_mixed(anb_ctx* c, const int* active, int its[3], bool conv[3]) {
  const int C = c->C;
  DefectArgs d{};
  d.A = DSellT<float>{C, c->dm.sliceOff, c->dm.col, c->mval32, c->mdiag32, c->L.maxRowLen};
  d.nc = 3;
  d.b = c->rhs;
  d.x = c->Us;
  d.r32 = c->r32;
  d.sc = c->scal + kScalDefect;
  d.fl = c->flags + kFlagDefect;
  d.frozen = c->flags + kFlagFrozen;
  d.atol = c->prm.vel_tol;
  d.rtol = c->prm.vel_rel_tol;
  d.red = c->red;
  const int fr[3] = {!active[0], !active[1], !active[2]};
  CK(cudaMemcpyAsync(c->flags + kFlagFrozen, fr, sizeof(fr), cudaMemcpyHostToDevice, c->stream));
  BicgArgsT<float> a{};
  a.A = d.A;
  a.nc = 3;
  a.b = c->r32;
  a.x = c->dx32;
  a.r = c->bw32[0]; a.rh = c->bw32[1]; a.p = c->bw32[2]; a.v = c->bw32[3];
  a.s = c->bw32[4]; a.t = c->bw32[5]; a.ph = c->bw32[6]; a.sh = c->bw32[7];
  a.sc = c->scal + kScalBicg;
  a.fl = c->flags + kFlagBicg;
  a.rtol = c->innerRtol;
  a.maxit = c->prm.vel_maxit;
  a.red = c->red;
  int tot[3] = {0, 0, 0};
  bool outerConv[3] = {false, false, false};
  for (int sweep = 0;; ++sweep) {
    launch_defect(c->lc, d);
    CK(cudaMemcpyAsync(c->hScal, d.sc, sizeof(double) * 24, cudaMemcpyDeviceToHost, c->stream));
    poll(c, d.fl, 12);
    bool all = true;
    int innerFlags[12];
    double target = 1e300;
    for (int q = 0; q < 3; ++q) {
      outerConv[q] = c->hFlags[4 * q] != 0;
      all = all && outerConv[q];
      // converged (or frozen) components sit out the inner solve
      innerFlags[4 * q] = outerConv[q] ? 1 : 0;
      innerFlags[4 * q + 1] = 0;
      innerFlags[4 * q + 2] = 0;
      innerFlags[4 * q + 3] = outerConv[q] ? 1 : 0;
      if (!outerConv[q])
        target = std::min(target, std::max(d.atol, d.rtol * std::sqrt(c->hScal[8 * q + 1])));
    }
    const bool budget = tot[0] < a.maxit && tot[1] < a.maxit && tot[2] < a.maxit;
    if (all || !budget || sweep >= 50) break;
    a.atol = 0.5 * target;
    bicg_init(c->lc, a);
    CK(cudaMemcpyAsync(a.fl, innerFlags, sizeof(innerFlags), cudaMemcpyHostToDevice, c->stream));
    bicg_iterate(c, a, c->momLoop32, nullptr);
    int mx = 0;
    for (int q = 0; q < 3; ++q) {
      tot[q] += c->hFlags[4 * q + 2];
      mx = std::max(mx, c->hFlags[4 * q + 2]);
    }
    c->lastMomIts = std::max(1, mx);
    launch_apply_correction(c->lc, C, 3, c->Us, c->dx32);
    if (c->prm.mixed_refine == 1) {  // one inner solve per step: the SIMPLE iteration refines
      for (int q = 0; q < 3; ++q) outerConv[q] = true;
      break;
    }
  }
  for (int q = 0; q < 3; ++q) {
    its[q] = active[q] ? tot[q] : 0;
    conv[q] = active[q] ? outerConv[q] : true;
  }
}

void solve_pressure_mixed(anb_ctx* c, const double* b, double* x, double rtol, int* its, bool* conv) {
  DefectArgs d{};
  d.A = DSellT<float>{c->C, c->dm.sliceOff, c->dm.col, c->pval32, c->pdiag32, c->L.maxRowLen};
  d.nc = 1;
  d.b = b;
  d.x = x;
  d.r32 = c->r32;
  d.sc = c->scal + kScalDefect;
  d.fl = c->flags + kFlagDefect;
  d.frozen = nullptr;
  d.atol = c->prm.p_tol;
  d.rtol = rtol;
  d.red = c->red;
  const AmgDevT<float>* amg = (c->prm.p_use_amg && c->amgBuilt && c->amg32.nLevels >= 2) ? &c->amg32 : nullptr;
  int tot = 0;
  bool ok = false;
  for (int sweep = 0;; ++sweep) {
    launch_defect(c->lc, d);
    CK(cudaMemcpyAsync(c->hScal, d.sc, sizeof(double) * 2, cudaMemcpyDeviceToHost, c->stream));
    poll(c, d.fl, 1);
    ok = c->hFlags[0] != 0;
    if (ok || tot >= c->prm.p_maxit || sweep >= 50) break;
    const double target = std::max(d.atol, rtol * std::sqrt(c->hScal[1]));
    PcgArgsT<float> a = pcg_args32(c, c->r32, c->dx32, 0.5 * target, c->innerRtol);
    pcg_init(c->lc, a);
    pcg_precondition(c->lc, a, amg);
    const int it = pcg_iterate(c, a, amg);
    const int n = c->hFlags[1];
    tot += n;
    c->lastPIts = std::max(1, n);
    if (c->prof.family == kKfPcgSpmv) {  // launches after convergence returned at once
      c->prof.bytes -= (double)(it - n) * (20.0 * c->ab.C + 8.0 * c->ab.nnzOff);
      c->prof.launches -= it - n;
    }
    launch_apply_correction(c->lc, c->C, 1, x, c->dx32);
    if (c->prm.mixed_refine == 1) {  // one inner solve per step: the SIMPLE iteration refines
      ok = true;
      break;
    }
  }
  *its = tot;
  *conv = ok;
}

void check_ready(anb_ctx* c) {
  if (!c->bcSet) throw AnbError(ANB_ERR_INVALID, "boundary conditions not set (anb_set_bc)");
  if (!c->stateSet) throw AnbError(ANB_ERR_INVALID, "state not set (anb_set_state)");
  CK(cudaSetDevice(c->prm.device));
}

// Momentum assembly into the matrix storage of the context's precision; Q is the field of the
// relaxation term (the old velocity, or the current iterate for rhs-only re-assembly).
template <class M>
void launch_mom_t(anb_ctx* c, M* val, M* diag, const double* Q, int rhsOnly) {
  MomArgsT<M> ma{};
  ma.U = c->U;
  ma.Q = Q;
  ma.G = c->G;
  ma.rho = c->prm.rho;
  ma.mu = c->prm.mu;
  ma.uRelax = c->prm.u_relax;
  ma.relax = c->prm.u_relax < 0.999999 ? 1 : 0;
  ma.rhsOnly = rhsOnly;
  ma.val = val;
  ma.diag = diag;
  ma.rhs = c->rhs;
  ma.rau = c->rau;
  launch_momentum(c->lc, c->dm, ma);
}
void launch_mom(anb_ctx* c, const double* Q, int rhsOnly) {
  if (c->mixed) launch_mom_t<float>(c, c->mval32, c->mdiag32, Q, rhsOnly);
  else launch_mom_t<double>(c, c->mval, c->mdiag, Q, rhsOnly);
}

template <class M>
void launch_prc(anb_ctx* c, M* val, M* diag, M* wdinv) {
  PresArgsT<M> pa{};
  pa.Us = c->Us;
  pa.P = c->P;
  pa.Gp = c->G + 9 * (size_t)c->C;
  pa.rau = c->rau;
  pa.rho = c->prm.rho;
  pa.val = val;
  pa.diag = diag;
  pa.phiStar = c->phiStar;
  pa.divStar = c->divStar;
  pa.b = c->pb;
  pa.pc = c->Pc;
  pa.wdinv = wdinv;
  pa.omega = c->amg.omega;
  launch_pressure_rc(c->lc, c->dm, pa);
}

// One SIMPLE outer iteration, main.cu:3388-3634.
int simple_step(anb_ctx* c, anb_iter_stats* st) {
  const int C = c->C;
  const anb_params& p = c->prm;
  bool anyNC = false;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  CK(cudaEventRecord(e0, c->stream));
  ++c->outerStep;
  // solves whose flags are read back after the step's one synchronisation
  c->nDefer = 0;
  std::vector<SolveOut> pending;
  pending.reserve(8);
  // 1. gradients of the old fields (u, v, w with their BC sets, p)
  {
    const double* phi[4] = {c->U, c->U + C, c->U + 2 * C, c->P};
    const unsigned char bits[4] = {1, 2, 4, 8};
    double* out[4] = {c->G, c->G + 3 * C, c->G + 6 * C, c->G + 9 * C};
    grad(c, 4, phi, bits, out);
  }
  // 2. momentum matrix (u pass) + three right-hand sides + relaxation + rAU
  launch_mom(c, c->U, 0);
  if (p.mom_amg) mom_amg_refresh(c);
  CK(cudaMemcpyAsync(c->Us, c->U, sizeof(double) * 3 * C, cudaMemcpyDeviceToDevice, c->stream));
  int its[3] = {0, 0, 0};
  {
    const int nVel = std::max(p.n_vel_nonorth_corr, 0) + 1;
    if (nVel > 1 && !c->UsPrev)
      throw AnbError(ANB_ERR_INVALID, "n_vel_nonorth_corr changed after anb_create");
    int active[3] = {1, 1, 1};
    for (int it = 1; it <= nVel; ++it) {
      if (it > 1) {
        // rhs-only re-assembly on the current iterates (K26, K9, K7, K8, K10)
        const double* phi[3] = {c->Us, c->Us + C, c->Us + 2 * C};
        const unsigned char bits[3] = {1, 2, 4};
        double* out[3] = {c->G, c->G + 3 * C, c->G + 6 * C};
        grad(c, 3, phi, bits, out);
        launch_mom(c, c->Us, 1);
      }
      // keep the iterate for the relative-change test (main.cu:3377-3381)
      if (nVel > 1 && it < nVel)
        CK(cudaMemcpyAsync(c->UsPrev, c->Us, sizeof(double) * 3 * C, cudaMemcpyDeviceToDevice, c->stream));
      SolveOut mo;
      solve_momentum(c, active, &mo, nVel == 1);
      if (!mo.resolved) {
        pending.push_back(mo);  // the only momentum pass: its flags arrive with the step's sync
      } else {
        for (int q = 0; q < 3; ++q)
          if (active[q]) {
            its[q] = mo.its[q];
            anyNC = anyNC || !mo.conv[q];
          }
      }
      if (nVel > 1 && it < nVel) {
        // relchg = sqrt(sum (q_new - q_iter)^2 / (1 + sum q_new^2)) per component, reduced on the device
        launch_relchg3(c->lc, C, c->UsPrev, c->Us, c->red, c->scal + kScalRelchg);
        CK(cudaMemcpyAsync(c->hScal, c->scal + kScalRelchg, sizeof(double) * 6, cudaMemcpyDeviceToHost, c->stream));
        CK(cudaStreamSynchronize(c->stream));
        for (int q = 0; q < 3; ++q)
          if (active[q] && std::sqrt(c->hScal[2 * q] / (1.0 + c->hScal[2 * q + 1])) < p.corr_tol) active[q] = 0;
        if (!active[0] && !active[1] && !active[2]) break;
      }
    }
  }
  // 3. pressure matrix + Rhie-Chow flux + continuity, p' = 0
  if (c->mixed) launch_prc<float>(c, c->pval32, c->pdiag32, c->pwdinv32);
  else launch_prc<double>(c, c->pval, c->pdiag, c->pwdinv);
  // preconditioner refresh: at the rebuild cadence (main.cu:3409-3411), or before every pressure
  // solve with pAmgSetupScope 1 (main.cu:2594-2598; the fine matrix does not change between the
  // solves of one step, so the later refreshes reproduce the same hierarchy values)
  const int every = std::max(p.p_amg_rebuild_every, 1);
  const bool perSolve = p.p_amg_setup_scope == 1;
  if (perSolve || !c->amgBuilt || c->outerStep == 1 || ((c->outerStep - 1) % every) == 0) ensure_amg(c);
  // 4. non-orthogonal pressure passes
  const int nPS = std::max(p.n_nonorth_corr, 0) + 1, nExtra = std::max(p.n_pressure_corr, 0);
  const int total = nPS + nExtra;
  int counter = 0, pTot = 0, pLast = 0;
  NonOrthArgs na{c->rau, c->Gc, c->divStar, c->pb};
  FluxArgs fa{};
  fa.rau = c->rau;
  fa.Gc = c->Gc;
  fa.pc = c->Pc;
  fa.phiStar = c->phiStar;
  fa.phi = c->phi;
  fa.divCorr = c->divCorr;
  fa.pRelax = p.p_relax;
  fa.P = c->P;
  fa.U = c->U;
  fa.Us = c->Us;
  fa.red = c->red;
  fa.stats = c->stats;
  const unsigned char pbit[1] = {8};
  for (int pc = 1; pc <= nPS; ++pc) {
    if (pc > 1 || !c->pZeroBC) {
      const double* phi[1] = {c->Pc};
      double* out[1] = {c->Gc};
      grad(c, 1, phi, pbit, out);
      launch_nonorth_rhs(c->lc, c->dm, na);
    }
    ++counter;
    const double rtol = counter == total ? 0.0 : p.p_rel_tol;
    if (perSolve && pc > 1) ensure_amg(c);
    pending.emplace_back();
    solve_pressure(c, c->pb, c->Pc, rtol, &pending.back(), true);
    if (pc == nPS) {
      const double* phi[1] = {c->Pc};
      double* out[1] = {c->Gc};
      grad(c, 1, phi, pbit, out);
      fa.update = nExtra == 0 ? 1 : 0;
      launch_flux_final(c->lc, c->dm, fa);
    }
  }
  for (int k = 1; k <= nExtra; ++k) {  // main.cu:3521-3567
    // b = -divCorr ; dp' from zero ; p' += dp'
    launch_pass_rhs(c->lc, C, c->divCorr, c->pb, c->pdx);
    ++counter;
    const double rtol = counter == total ? 0.0 : p.p_rel_tol;
    if (perSolve) ensure_amg(c);
    pending.emplace_back();
    solve_pressure(c, c->pb, c->pdx, rtol, &pending.back(), true);
    launch_add_scaled(c->lc, C, 1.0, c->pdx, c->Pc);
    const double* phi[1] = {c->Pc};
    double* out[1] = {c->Gc};
    grad(c, 1, phi, pbit, out);
    fa.update = k == nExtra ? 1 : 0;
    launch_flux_final(c->lc, c->dm, fa);
  }
  CK(cudaEventRecord(e1, c->stream));
  CK(cudaMemcpyAsync(c->hScal, c->stats, sizeof(double) * 9, cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  CK(cudaGetLastError());
  for (SolveOut& o : pending) {
    resolve_solve(c, o);
    if (o.momentum) {
      for (int q = 0; q < 3; ++q)
        if (o.active[q]) {
          its[q] = o.its[q];
          anyNC = anyNC || !o.conv[q];
        }
    } else {
      pLast = o.its[0];
      pTot += pLast;
      anyNC = anyNC || !o.conv[0];
    }
  }
  c->prof.flush();
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double* s = c->hScal;
  st->mass_res = s[8];
  st->du_rel = std::sqrt(s[0] / (1.0 + s[1]));
  st->dv_rel = std::sqrt(s[2] / (1.0 + s[3]));
  st->dw_rel = std::sqrt(s[4] / (1.0 + s[5]));
  st->dp_rel = std::sqrt(s[6] / (1.0 + s[7]));
  st->its_u = its[0];
  st->its_v = its[1];
  st->its_w = its[2];
  st->its_p_last = pLast;
  st->its_p_total = pTot;
  st->iter_seconds = ms * 1e-3;
  st->status = anyNC ? ANB_NOT_CONVERGED : ANB_OK;
  return st->status;
}

void build_slot_lookup(anb_ctx* c) {
  c->slotOwn.assign(c->nI, -1);
  c->slotNei.assign(c->nI, -1);
  for (int s = 0; s < c->L.nSlices; ++s) {
    const int w = (c->L.sliceOff[s + 1] - c->L.sliceOff[s]) / kSlice;
    for (int lane = 0; lane < kSlice; ++lane) {
      const int r = s * kSlice + lane;
      if (r >= c->C) continue;
      for (int k = 0; k < w; ++k) {
        const int e = c->L.sliceOff[s] + k * kSlice + lane;
        const int f = c->L.slotFace[e];
        if (f < 0) continue;
        if (c->L.fOwner[f] == r) c->slotOwn[f] = e;
        else c->slotNei[f] = e;
      }
    }
  }
}

void release_amg(anb_ctx* c) {
  CK(cudaStreamSynchronize(c->stream));
  amg_release_graphs(c->amg);
  c->amg.nLevels = 0;
  c->amg.dense = nullptr;
  amg_release_graphs(c->amg32);
  c->amg32.nLevels = 0;
  c->amg32.dense = nullptr;
  c->amgArena.release();
  c->amgHost.clear();
  c->amgBuilt = false;
}

}  // namespace anb

extern "C" {

void anb_default_params(anb_params* p) {
  if (!p) return;
  std::memset(p, 0, sizeof(*p));
  p->rho = 1.0;
  p->mu = 0.05;
  p->u_relax = 0.7;
  p->p_relax = 1.0;
  p->n_nonorth_corr = 2;
  p->n_vel_nonorth_corr = 0;
  p->n_pressure_corr = 0;
  p->vel_maxit = 100;
  p->vel_tol = 1e-10;
  p->vel_rel_tol = 0.0;
  p->p_maxit = 4000;
  p->p_tol = 1e-10;
  p->p_rel_tol = 0.0;
  p->corr_tol = 1e-12;
  p->p_amg_rebuild_every = 1;
  p->p_use_amg = 1;
  p->precision = ANB_PRECISION_FP64;
  p->device = 0;
  p->mixed_refine = 0;
  p->mixed_inner_rtol = 1e-4;
}

const char* anb_last_error(const anb_ctx* c) { return c ? c->err.c_str() : g_createError.c_str(); }

int anb_setup_times(const anb_ctx* c, double* t) {
  if (!c || !t) return ANB_ERR_INVALID;
  for (int k = 0; k < 4; ++k) t[k] = c->setupSec[k];
  for (int k = 0; k < 6; ++k) t[4 + k] = c->L.seconds[k];
  return ANB_OK;
}

int anb_create(const anb_mesh_desc* md, const anb_params* prm, anb_ctx** out) {
  if (!out) return ANB_ERR_INVALID;
  *out = nullptr;
  if (!md || !prm) return ANB_ERR_INVALID;
  CallerDevice keep;
  auto c = std::make_unique<anb_ctx>();
  auto clk = std::chrono::steady_clock::now();
  auto lap = [&](int k) {
    const auto t = std::chrono::steady_clock::now();
    c->setupSec[k] = std::chrono::duration<double>(t - clk).count();
    clk = t;
    if (k == 2 && std::getenv("ANB_SETUP_VERBOSE")) {
      std::fprintf(stderr, "anb_create: copy-in+topology %.3f s, geometry %.3f s, layout %.3f s [", c->setupSec[0],
                   c->setupSec[1], c->setupSec[2]);
      for (double s : c->L.seconds) std::fprintf(stderr, " %.3f", s);
      std::fprintf(stderr, " ]\n");
    }
  };
  int rc = guarded(c.get(), [&]() -> int {
    c->prm = *prm;
    if (prm->precision != ANB_PRECISION_FP64 && prm->precision != ANB_PRECISION_MIXED)
      throw AnbError(ANB_ERR_INVALID, "unknown precision");
    if (md->n_points <= 0 || md->n_faces <= 0 || md->n_internal_faces < 0 || md->n_internal_faces > md->n_faces ||
        !md->points || !md->face_offsets || !md->face_points || !md->owner ||
        (md->n_internal_faces > 0 && !md->neighbour) || md->n_patches < 0)
      throw AnbError(ANB_ERR_INVALID, "invalid mesh description");
    HostMesh& m = c->hm;
    m.points.resize(md->n_points);
    for (int i = 0; i < md->n_points; ++i)
      m.points[i] = {md->points[3 * i], md->points[3 * i + 1], md->points[3 * i + 2]};
    m.faceOff.assign(md->face_offsets, md->face_offsets + md->n_faces + 1);
    if (m.faceOff[0] != 0) throw AnbError(ANB_ERR_INVALID, "face_offsets must start at 0");
    for (int f = 0; f < md->n_faces; ++f)
      if (m.faceOff[f + 1] - m.faceOff[f] < 3) throw AnbError(ANB_ERR_MESH, "face " + std::to_string(f) + " has fewer than 3 points");
    m.facePts.assign(md->face_points, md->face_points + m.faceOff.back());
    m.owner.assign(md->owner, md->owner + md->n_faces);
    m.neigh.assign(md->neighbour, md->neighbour + md->n_internal_faces);
    m.patches.resize(md->n_patches);
    std::vector<int> cover(md->n_faces, 0);
    for (int k = 0; k < md->n_patches; ++k) {
      m.patches[k].start = md->patch_start[k];
      m.patches[k].nFaces = md->patch_size[k];
      m.patches[k].name = "patch" + std::to_string(k);
      if (md->patch_size[k] < 0 || md->patch_start[k] < md->n_internal_faces ||
          md->patch_start[k] + md->patch_size[k] > md->n_faces)
        throw AnbError(ANB_ERR_MESH, "patch " + std::to_string(k) + " has an invalid face range");
      for (int f = md->patch_start[k]; f < md->patch_start[k] + md->patch_size[k]; ++f) cover[f]++;
    }
    for (int f = md->n_internal_faces; f < md->n_faces; ++f)
      if (cover[f] != 1) throw AnbError(ANB_ERR_MESH, "boundary face " + std::to_string(f) + " is not in exactly one patch");
    finalize_topology(m);
    for (int v : m.owner)
      if (v < 0) throw AnbError(ANB_ERR_MESH, "negative owner label");
    lap(0);
    CK(cudaSetDevice(prm->device));
    CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    if (nalloc_prepare_device(prm->device) != 0)
      throw AnbError(ANB_ERR_CUDA, "could not place the static scratch of anb_patch_force_nalloc on the device");
    // geometry, LSQ moments and slot-ordered face records on the device (bit-identical to the
    // host restatement; ANB_HOST_SETUP=1 builds them on the host instead)
    const char* hs = std::getenv("ANB_HOST_SETUP");
    const bool hostSetup = hs && hs[0] == '1';
    if (hostSetup || !compute_geometry_gpu(m, c->stream)) compute_geometry(m);
    lap(1);
    {
      auto t0 = std::chrono::steady_clock::now();
      std::vector<int> adjOff, adj;
      cell_adjacency(m, adjOff, adj);
      auto t1 = std::chrono::steady_clock::now();
      const std::vector<double> minv = hostSetup ? lsq_minv_host(m, adjOff, adj) : lsq_minv_gpu(m, adjOff, adj, c->stream);
      auto t2 = std::chrono::steady_clock::now();
      c->L = build_layout(m, adjOff, adj, minv);
      c->L.seconds[0] = std::chrono::duration<double>(t1 - t0).count();
      c->L.seconds[1] = std::chrono::duration<double>(t2 - t1).count();
    }
    Layout& L = c->L;
    c->C = L.nCells;
    c->nI = L.nInternal;
    c->nB = L.nBoundary;
    c->nEnt = L.sliceOff.back();
    build_slot_lookup(c.get());
    lap(2);

    int nSM = 148;
    CK(cudaDeviceGetAttribute(&nSM, cudaDevAttrMultiProcessorCount, prm->device));
    c->lc.stream = c->stream;
    {
      const char* bps = std::getenv("ANB_BLOCKS_PER_SM");
      const int perSM = bps ? std::max(1, std::min(64, std::atoi(bps))) : kBlocksPerSM;
      c->lc.rowBlocks = std::max(1, std::min((c->C + kBlock - 1) / kBlock, nSM * perSM));
      // the SELL row kernels get one full wave of resident blocks; ANB_GRID=fixed gives every row
      // kernel rowBlocks blocks instead
      const char* gp = std::getenv("ANB_GRID");
      c->lc.nSM = (gp && std::string(gp) == "fixed") ? 0 : nSM;
    }
    c->lc.prof = &c->prof;
    c->lc.ab = &c->ab;
    c->ab.C = c->C;
    c->ab.Fi = c->nI;
    c->ab.Fb = c->nB;
    c->ab.nnzOff = 2LL * c->nI;

    DevArena& A = c->arena;
    // faces
    std::vector<FaceRec> fr(c->nI);
    for (int f = 0; f < c->nI; ++f) {
      fr[f].lam = L.fLam[f];
      fr[f].g = L.fG[f];
      for (int k = 0; k < 3; ++k) {
        fr[f].t[k] = L.fT[3 * f + k];
        fr[f].d[k] = L.fD[3 * f + k];
      }
    }
    std::vector<BndRec> br(c->nB);
    std::vector<double> bA(c->nB), bN((size_t)3 * c->nB);
    for (int b = 0; b < c->nB; ++b) {
      const int f = c->nI + b;
      br[b].g = L.bG[b];
      for (int k = 0; k < 3; ++k) {
        br[b].t[k] = L.bT[3 * b + k];
        br[b].S[k] = L.bS[3 * b + k];
        br[b].d[k] = m.xf[f][k] - m.cc[m.owner[f]][k];
        bN[3 * b + k] = m.nf[f][k];
      }
      bA[b] = m.Af[f];
    }
    c->dFace = A.upload(fr);
    c->dBnd = A.upload(br);
    c->dBA = A.upload(bA);
    c->dBN = A.upload(bN);
    c->dBType = A.alloc<uint8_t>(c->nB);
    c->dBVal = A.alloc<double>((size_t)4 * c->nB);
    DMesh& dm = c->dm;
    dm.nCells = c->C;
    dm.nInternal = c->nI;
    dm.nBoundary = c->nB;
    dm.nSlices = L.nSlices;
    dm.maxW = L.maxRowLen;
    dm.sliceOff = A.upload(L.sliceOff);
    dm.col = A.upload(L.col);
    dm.slotFace = A.upload(L.slotFace);
    dm.fOwner = A.upload(L.fOwner);
    dm.fNeigh = A.upload(L.fNeigh);
    dm.face = c->dFace;
    dm.fFlags = A.upload(L.fFlags);
    c->dN2O = A.upload(L.new2old);
    c->dO2N = A.upload(L.old2new);
    c->dStage = A.alloc<double>((size_t)4 * c->C);
    {
      const size_t nE = (size_t)c->nEnt;
      dm.nEnt = c->nEnt;
      if (hostSetup) {
        std::vector<double> sg(8 * nE, 0.0);
        std::vector<uint8_t> sf(nE, 0);
        for (size_t e = 0; e < nE; ++e) {
          const int f = L.slotFace[e];
          if (f < 0) continue;
          const FaceRec& r = fr[f];
          const double v[8] = {r.lam, r.g, r.t[0], r.t[1], r.t[2], r.d[0], r.d[1], r.d[2]};
          for (int q = 0; q < 8; ++q) sg[q * nE + e] = v[q];
          sf[e] = L.fFlags[f];
        }
        dm.slotGeom = A.upload(sg);
        dm.slotFlags = A.upload(sf);
      } else {
        double* sg = A.alloc<double>(8 * nE);
        uint8_t* sf = A.alloc<uint8_t>(nE);
        build_slot_geometry(nE, dm.slotFace, c->dFace, dm.fFlags, sg, sf, c->stream);
        dm.slotGeom = sg;
        dm.slotFlags = sf;
      }
    }
    dm.bOwner = A.upload(L.bOwner);
    dm.bnd = c->dBnd;
    dm.bFlags = A.upload(L.bFlags);
    dm.cbOff = A.upload(L.cbOff);
    dm.cbList = A.upload(L.cbList);
    dm.vol = A.upload(L.vol);
    dm.cc = A.upload(L.cc);
    dm.minv = A.upload(L.minv);
    dm.bType = c->dBType;
    dm.bVal = c->dBVal;
    // fields and work
    const size_t C = c->C, F = (size_t)c->nI + c->nB;
    c->U = A.alloc<double>(3 * C);
    c->Us = A.alloc<double>(3 * C);
    c->P = A.alloc<double>(C);
    c->Pc = A.alloc<double>(C);
    c->rau = A.alloc<double>(C);
    c->G = A.alloc<double>(12 * C);
    c->Gc = A.alloc<double>(3 * C);
    c->mixed = prm->precision == ANB_PRECISION_MIXED;
    if (!c->mixed) {
      c->mval = A.alloc<double>(c->nEnt);
      c->mdiag = A.alloc<double>(C);
      c->pval = A.alloc<double>(c->nEnt);
      c->pdiag = A.alloc<double>(C);
    } else {
      c->mval32 = A.alloc<float>(c->nEnt);
      c->mdiag32 = A.alloc<float>(C);
      c->pval32 = A.alloc<float>(c->nEnt);
      c->pdiag32 = A.alloc<float>(C);
      c->pwdinv32 = A.alloc<float>(C);
      for (int k = 0; k < 8; ++k) c->bw32[k] = A.alloc<float>(3 * C);
      c->r32 = A.alloc<float>(3 * C);
      c->dx32 = A.alloc<float>(3 * C);
      c->pr32 = A.alloc<float>(C);
      c->pz32 = A.alloc<float>(C);
      c->pp0_32 = A.alloc<float>(C);
      c->pp1_32 = A.alloc<float>(C);
      c->pq32 = A.alloc<float>(C);
      c->pr2_32 = A.alloc<float>(C);
      CK(cudaMemset(c->mval32, 0, sizeof(float) * c->nEnt));
      CK(cudaMemset(c->pval32, 0, sizeof(float) * c->nEnt));
      CK(cudaMemset(c->dx32, 0, sizeof(float) * 3 * C));
      c->innerRtol = prm->mixed_inner_rtol > 0.0 ? prm->mixed_inner_rtol : 1e-4;
      if (const char* s = std::getenv("ANB_MIXED_INNER_RTOL")) c->innerRtol = std::atof(s);
      if (prm->mixed_refine != 0 && prm->mixed_refine != 1)
        throw AnbError(ANB_ERR_INVALID, "mixed_refine must be 0 or 1");
    }
    c->rhs = A.alloc<double>(3 * C);
    c->pb = A.alloc<double>(C);
    c->divStar = A.alloc<double>(C);
    c->divCorr = A.alloc<double>(C);
    c->phiStar = A.alloc<double>(F);
    c->phi = A.alloc<double>(F);
    if (!c->mixed) {
      for (int k = 0; k < 8; ++k) c->bw[k] = A.alloc<double>(3 * C);
      c->pr = A.alloc<double>(C);
      c->pz = A.alloc<double>(C);
      c->pp0 = A.alloc<double>(C);
      c->pp1 = A.alloc<double>(C);
      c->pq = A.alloc<double>(C);
      c->pr2 = A.alloc<double>(C);
      c->pxw = A.alloc<double>(C);
      c->pwdinv = A.alloc<double>(C);
    }
    c->pdx = A.alloc<double>(C);
    if (prm->n_vel_nonorth_corr > 0) c->UsPrev = A.alloc<double>(3 * C);
    if (prm->mom_amg) {
      if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "mom_amg needs an FP64 context");
      c->mwdinv = A.alloc<double>(C);
      c->momScratch = A.alloc<double>(C);
      c->momSc = A.alloc<double>(8);
      c->amgMom.corr = 1.0;
    }
    if (prm->p_amg_setup_scope != 0 && prm->p_amg_setup_scope != 1)
      throw AnbError(ANB_ERR_INVALID, "p_amg_setup_scope must be 0 (outer) or 1 (pressure)");
    if (const char* s = std::getenv("ANB_AMG_OMEGA")) c->amg.omega = std::atof(s);
    if (const char* s = std::getenv("ANB_AMG_CORR")) c->amg.corr = std::atof(s);
    c->amg32.omega = c->amg.omega;
    c->amg32.corr = c->amg.corr;
    c->scal = A.alloc<double>(64);
    c->flags = A.alloc<int>(kFlagCount);
    c->stats = A.alloc<double>(16);
    c->forceOut = A.alloc<double>(16);
    c->red.partials = A.alloc<double>((size_t)(c->lc.rowBlocks + 16) * 16);
    c->red.ticket = A.alloc<unsigned int>(1);
    CK(cudaMemset(c->red.ticket, 0, sizeof(unsigned int)));
    if (!c->mixed) {
      CK(cudaMemset(c->mval, 0, sizeof(double) * c->nEnt));
      CK(cudaMemset(c->pval, 0, sizeof(double) * c->nEnt));
    }
    CK(cudaMemset(c->phi, 0, sizeof(double) * F));
    CK(cudaMemset(c->Pc, 0, sizeof(double) * C));
    CK(cudaMallocHost(&c->hFlags, sizeof(int) * kFlagCount));
    CK(cudaMallocHost(&c->hScal, sizeof(double) * 64));
    CK(cudaMallocHost(&c->hStage, sizeof(double) * 4 * C));
    for (auto& e : c->stageEv) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    CK(cudaMallocHost(&c->hDefer, sizeof(int) * kDeferSlots * kDeferInts));
    CK(cudaDeviceSynchronize());
    lap(3);
    return ANB_OK;
  });
  if (rc != ANB_OK) {
    g_createError = c->err;
    c->arena.release();
    if (c->stream) cudaStreamDestroy(c->stream);
    if (c->hFlags) cudaFreeHost(c->hFlags);
    if (c->hScal) cudaFreeHost(c->hScal);
    if (c->hStage) cudaFreeHost(c->hStage);
    if (c->hDefer) cudaFreeHost(c->hDefer);
    for (auto e : c->stageEv)
      if (e) cudaEventDestroy(e);
    return rc;
  }
  *out = c.release();
  return ANB_OK;
}

void anb_destroy(anb_ctx* c) {
  if (!c) return;
  CallerDevice keep;
  cudaSetDevice(c->prm.device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  amg_release_graphs(c->amg);
  amg_release_graphs(c->amg32);
  amg_release_graphs(c->amgMom);
  bicg_loop_release(c->momLoop);
  bicg_loop_release(c->momLoop32);
  for (auto g : c->momGraph)
    if (g) cudaGraphExecDestroy(g);
  adjoint_release(c);
  c->amgArena.release();
  c->arena.release();
  if (c->hFlags) cudaFreeHost(c->hFlags);
  if (c->hScal) cudaFreeHost(c->hScal);
  if (c->hStage) cudaFreeHost(c->hStage);
  if (c->hDefer) cudaFreeHost(c->hDefer);
  for (auto e : c->stageEv)
    if (e) cudaEventDestroy(e);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
}

int anb_get_sizes(const anb_ctx* c, int* nc, int* nf, int* ni, int* np) {
  if (!c) return ANB_ERR_INVALID;
  if (nc) *nc = c->C;
  if (nf) *nf = c->nI + c->nB;
  if (ni) *ni = c->nI;
  if (np) *np = (int)c->hm.patches.size();
  return ANB_OK;
}

int anb_get_geometry(anb_ctx* c, double* cc, double* vol, double* xf, double* nf, double* area, double* mx) {
  if (!c) return ANB_ERR_INVALID;
  const HostMesh& m = c->hm;
  for (int i = 0; i < m.nCells; ++i) {
    if (cc) for (int k = 0; k < 3; ++k) cc[3 * i + k] = m.cc[i][k];
    if (vol) vol[i] = m.vol[i];
  }
  for (int f = 0; f < m.nFaces; ++f) {
    for (int k = 0; k < 3; ++k) {
      if (xf) xf[3 * f + k] = m.xf[f][k];
      if (nf) nf[3 * f + k] = m.nf[f][k];
    }
    if (area) area[f] = m.Af[f];
  }
  if (mx) *mx = m.maxNonOrthDeg;
  return ANB_OK;
}

int anb_set_bc(anb_ctx* c, const int* tu, const int* tv, const int* tw, const int* tp, const double* uf,
               const double* vf, const double* wf, const double* pf) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (!tu || !tv || !tw || !tp || !uf || !vf || !wf || !pf) throw AnbError(ANB_ERR_INVALID, "null BC array");
    CK(cudaSetDevice(c->prm.device));
    const int nB = c->nB, nI = c->nI;
    std::vector<uint8_t> ty(nB);
    std::vector<double> val((size_t)4 * nB);
    bool pZero = true;
    for (int b = 0; b < nB; ++b) {
      const int patch = c->L.bPatch[b];
      ty[b] = (uint8_t)((tu[patch] == 1 ? 1 : 0) | (tv[patch] == 1 ? 2 : 0) | (tw[patch] == 1 ? 4 : 0) |
                        (tp[patch] == 1 ? 8 : 0));
      val[b] = uf[nI + b];
      val[(size_t)nB + b] = vf[nI + b];
      val[(size_t)2 * nB + b] = wf[nI + b];
      val[(size_t)3 * nB + b] = pf[nI + b];
      if ((ty[b] & 8) && pf[nI + b] != 0.0) pZero = false;
    }
    CK(cudaMemcpy(c->dBType, ty.data(), nB, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c->dBVal, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice));
    c->pZeroBC = pZero;
    c->bcSet = true;
    return ANB_OK;
  });
}

int anb_set_state(anb_ctx* c, const double* u, const double* v, const double* w, const double* p) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (!u || !v || !w || !p) throw AnbError(ANB_ERR_INVALID, "null state array");
    CK(cudaSetDevice(c->prm.device));
    const double* s4[4] = {u, v, w, p};
    double* d4[4] = {c->U, c->U + c->C, c->U + 2 * (size_t)c->C, c->P};
    CK(cudaMemsetAsync(c->phi, 0, sizeof(double) * ((size_t)c->nI + c->nB), c->stream));
    upload_cells(c, s4, d4, 4);
    c->stateSet = true;
    return ANB_OK;
  });
}

int anb_get_state(anb_ctx* c, double* u, double* v, double* w, double* p, double* phi) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    CK(cudaSetDevice(c->prm.device));
    const double* s4[4] = {c->U, c->U + c->C, c->U + 2 * (size_t)c->C, c->P};
    double* d4[4] = {u, v, w, p};
    download_cells(c, s4, d4, 4);
    if (phi) download_faces(c, c->phi, phi);
    return ANB_OK;
  });
}

int anb_simple_iterate(anb_ctx* c, int nsteps, double tolMass, double tolVel, anb_iter_stats* stats, int* done) {
  if (!c) return ANB_ERR_INVALID;
  if (done) *done = 0;
  return guarded(c, [&]() -> int {
    check_ready(c);
    int status = ANB_OK;
    for (int k = 0; k < nsteps; ++k) {
      anb_iter_stats st{};
      st.step = k + 1;
      if (simple_step(c, &st) == ANB_NOT_CONVERGED) status = ANB_NOT_CONVERGED;
      if (stats) stats[k] = st;
      if (done) *done = k + 1;
      if (!std::isfinite(st.mass_res) || st.mass_res > 1e50 || !std::isfinite(st.du_rel) ||
          !std::isfinite(st.dv_rel) || !std::isfinite(st.dw_rel) || !std::isfinite(st.dp_rel)) {
        c->err = "SIMPLE-like steady solve diverged.";
        return ANB_ERR_DIVERGED;
      }
      if (st.mass_res < tolMass && std::max({st.du_rel, st.dv_rel, st.dw_rel}) < tolVel) break;
    }
    return status;
  });
}

int anb_patch_force(anb_ctx* c, int patch, int sign, anb_force_report* out) {
  if (!c || !out) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    std::memset(out, 0, sizeof(*out));
    if (patch < 0 || patch >= (int)c->hm.patches.size()) return ANB_OK;  // valid = 0
    CK(cudaSetDevice(c->prm.device));
    const int b0 = c->hm.patches[patch].start - c->nI;
    const int b1 = b0 + c->hm.patches[patch].nFaces;
    launch_patch_force(c->stream, c->dm, b0, b1, sign, c->prm.mu, c->dBA, c->dBN, c->U, c->P, c->forceOut);
    double h[16];
    CK(cudaMemcpyAsync(h, c->forceOut, sizeof(double) * 15, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    out->valid = 1;
    for (int k = 0; k < 3; ++k) {
      out->Fp[k] = h[k];
      out->Fv[k] = h[3 + k];
      out->F[k] = h[6 + k];
    }
    out->area = h[9];
    out->n_faces = (int)h[10];
    out->min_wall_distance = h[11];
    out->max_wall_distance = h[12];
    out->max_ut = h[13];
    out->max_shear_mag = h[14];
    return ANB_OK;
  });
}

// ---- scalar libraries -------------------------------------------------------------------------
namespace {

void ensure_scalar_buffers(anb_ctx* c) {
  if (c->sPhi) return;
  DevArena& A = c->scalarArena;
  const int C = c->C, nF = c->nI + c->nB;
  c->sMinv = A.alloc<double>((size_t)6 * C);
  c->sBcType = A.alloc<uint8_t>(c->nB);
  c->sBcVal = A.alloc<double>(c->nB);
  c->sGamma = A.alloc<double>(nF);
  c->sFlux = A.alloc<double>(nF);
  c->sSrc = A.alloc<double>(C);
  c->sSp = A.alloc<double>(C);
  c->sPhi = A.alloc<double>(C);
  c->sGrad = A.alloc<double>((size_t)3 * C);
}

// Face array in input order/orientation -> device (layout order; fluxes change sign on flipped
// internal faces).  src == nullptr uploads `fill`.
void upload_faces(anb_ctx* c, const double* src, double* dst, bool orientSign, double fill) {
  const int nF = c->nI + c->nB;
  std::vector<double> h(nF, fill);
  if (src) {
    for (int fi = 0; fi < c->nI; ++fi) {
      const double v = src[c->L.fOrig[fi]];
      h[fi] = (orientSign && c->L.fFlip[fi]) ? -v : v;
    }
    for (int b = 0; b < c->nB; ++b) h[c->nI + b] = src[c->nI + b];
  }
  CK(cudaMemcpyAsync(dst, h.data(), nF * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

void upload_cells1(anb_ctx* c, const double* src, double* dst, double fill) {
  if (src) {
    const double* s[1] = {src};
    upload_cells(c, s, dst, 1);
  } else {
    std::vector<double> h(c->C, fill);
    CK(cudaMemcpyAsync(dst, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
  }
}

// Boundary types/values (nFaces arrays, boundary entries read) -> device, LSQ inverse for them.
void upload_scalar_bc(anb_ctx* c, const int* type, const double* value, int maxType) {
  std::vector<uint8_t> t(c->nB), dir(c->nB);
  std::vector<double> v(c->nB);
  for (int b = 0; b < c->nB; ++b) {
    const int ty = type[c->nI + b];
    if (ty < 0 || ty > maxType)
      throw AnbError(ANB_ERR_INVALID, "invalid scalar boundary type " + std::to_string(ty) + " at face " +
                                          std::to_string(c->nI + b));
    t[b] = (uint8_t)ty;
    dir[b] = ty == ANB_SCALAR_DIRICHLET;
    v[b] = value[c->nI + b];
  }
  const std::vector<double> minv = scalar_lsq_minv(c->hm, c->L, dir);
  CK(cudaMemcpyAsync(c->sBcType, t.data(), t.size(), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->sBcVal, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaMemcpyAsync(c->sMinv, minv.data(), minv.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
  CK(cudaStreamSynchronize(c->stream));
}

ScalarArgs scalar_args(anb_ctx* c) {
  ScalarArgs a{};
  a.phi = c->sPhi;
  a.minv = c->sMinv;
  a.bcType = c->sBcType;
  a.bcVal = c->sBcVal;
  a.bA = c->dBA;
  a.bN = c->dBN;
  a.gammaF = c->sGamma;
  a.src = c->sSrc;
  a.grad = c->sGrad;
  a.g = c->sGrad;
  a.refCell = -1;
  a.omega = c->amg.omega;
  return a;
}

void download_cells1(anb_ctx* c, const double* src, double* dst) {
  double* d[1] = {dst};
  download_cells(c, src, d, 1);
}

}  // namespace

int anb_scalar_elliptic_solve(anb_ctx* c, const double* gammaFace, const double* source, const int* bcType,
                              const double* bcValue, int nonorth, int nNonOrthCorr, int useRef, int refCell,
                              double refValue, double absTol, double relTol, int maxIter, double* phi,
                              anb_solve_info* info) {
  if (!c || !source || !bcType || !bcValue || !phi) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
    CK(cudaSetDevice(c->prm.device));
    if (info) std::memset(info, 0, sizeof(*info));
    bool anyDirichlet = false;
    for (int b = 0; b < c->nB && !anyDirichlet; ++b) anyDirichlet = bcType[c->nI + b] == ANB_SCALAR_DIRICHLET;
    if (!anyDirichlet && !useRef)
      throw AnbError(ANB_ERR_INVALID, "Pure-Neumann scalar elliptic problem needs useReferenceCell=true.");
    if (useRef && (refCell < 0 || refCell >= c->C)) throw AnbError(ANB_ERR_INVALID, "Invalid reference cell");
    ensure_scalar_buffers(c);
    upload_scalar_bc(c, bcType, bcValue, ANB_SCALAR_NEUMANN);
    upload_faces(c, gammaFace, c->sGamma, false, 1.0);
    upload_cells1(c, source, c->sSrc, 0.0);
    CK(cudaMemsetAsync(c->sPhi, 0, sizeof(double) * c->C, c->stream));
    CK(cudaMemsetAsync(c->sGrad, 0, sizeof(double) * 3 * c->C, c->stream));
    ScalarArgs a = scalar_args(c);
    a.transport = 0;
    a.nonorth = nonorth != 0;
    a.refCell = useRef ? c->L.old2new[refCell] : -1;
    a.refValue = refValue;
    a.val = c->pval;
    a.diag = c->pdiag;
    a.rhs = c->pb;
    a.wdinv = c->pwdinv;
    const int nOuter = nonorth ? std::max(nNonOrthCorr, 0) + 1 : 1;
    // the matrix stays the same across passes (only the non-orthogonal rhs changes): one AMG set-up
    release_amg(c);
    const double saveTol = c->prm.p_tol;
    const int saveMaxit = c->prm.p_maxit;
    c->prm.p_tol = absTol;
    c->prm.p_maxit = maxIter;
    int its = 0;
    bool conv = true, allConv = true;
    try {
      for (int outer = 0; outer < nOuter; ++outer) {
        if (a.nonorth) launch_scalar_grad(c->lc, c->dm, a);
        launch_scalar_assemble(c->lc, c->dm, a);
        if (outer == 0) ensure_amg(c);
        CK(cudaMemsetAsync(c->sPhi, 0, sizeof(double) * c->C, c->stream));
        solve_pressure(c, c->pb, c->sPhi, relTol, &its, &conv);
        allConv = allConv && conv;
      }
    } catch (...) {
      c->prm.p_tol = saveTol;
      c->prm.p_maxit = saveMaxit;
      release_amg(c);
      throw;
    }
    c->prm.p_tol = saveTol;
    c->prm.p_maxit = saveMaxit;
    double sc[8];
    CK(cudaMemcpyAsync(sc, c->scal + kScalPcg, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    release_amg(c);  // the SIMPLE path rebuilds its own hierarchy
    download_cells1(c, c->sPhi, phi);
    if (info) {
      info->iterations = its;
      info->converged = allConv ? 1 : 0;
      info->outer = nOuter;
      info->final_res_norm = std::sqrt(std::max(sc[4], 0.0));
      // eps = max(atol, rtol |b|) is not |b|; recompute |b| on the host from the assembled rhs
      std::vector<double> hb(c->C);
      CK(cudaMemcpy(hb.data(), c->pb, sizeof(double) * c->C, cudaMemcpyDeviceToHost));
      double bn = 0.0;
      for (double x : hb) bn += x * x;
      info->final_rel_res = bn > 0.0 ? info->final_res_norm / std::sqrt(bn) : 0.0;
    }
    return allConv ? ANB_OK : ANB_NOT_CONVERGED;
  });
}

int anb_scalar_transport_solve(anb_ctx* c, const double* flux, const double* gammaFace, const double* su,
                               const double* sp, const int* bcType, const double* bcValue, int convection,
                               int nonorth, int nNonOrthCorr, double absTol, double relTol, int maxIter,
                               const double* x0, double* phi, anb_solve_info* info) {
  if (!c || !gammaFace || !su || !bcType || !bcValue || !phi) return ANB_ERR_INVALID;
  if (convection != ANB_CONVECTION_CENTRAL && convection != ANB_CONVECTION_UPWIND) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
    CK(cudaSetDevice(c->prm.device));
    if (info) std::memset(info, 0, sizeof(*info));
    ensure_scalar_buffers(c);
    upload_scalar_bc(c, bcType, bcValue, ANB_SCALAR_ZERO_GRADIENT);
    upload_faces(c, gammaFace, c->sGamma, false, 0.0);
    if (flux) upload_faces(c, flux, c->sFlux, true, 0.0);
    upload_cells1(c, su, c->sSrc, 0.0);
    upload_cells1(c, sp, c->sSp, 0.0);
    upload_cells1(c, x0, c->sPhi, 0.0);
    CK(cudaMemsetAsync(c->sGrad, 0, sizeof(double) * 3 * c->C, c->stream));
    ScalarArgs a = scalar_args(c);
    a.transport = 1;
    a.upwind = convection == ANB_CONVECTION_UPWIND;
    a.nonorth = nonorth != 0;
    a.flux = flux ? c->sFlux : nullptr;
    a.sp = c->sSp;
    a.val = c->mval;
    a.diag = c->mdiag;
    a.rhs = c->rhs;
    const int nOuter = nonorth ? std::max(nNonOrthCorr, 0) + 1 : 1;
    BicgArgs b{};
    b.A = mom_sell(c);
    b.nc = 1;
    b.b = c->rhs;
    b.x = c->sPhi;
    b.r = c->bw[0]; b.rh = c->bw[1]; b.p = c->bw[2]; b.v = c->bw[3];
    b.s = c->bw[4]; b.t = c->bw[5]; b.ph = c->bw[6]; b.sh = c->bw[7];
    b.sc = c->scal + kScalBicg;
    b.fl = c->flags + kFlagBicg;
    b.atol = absTol;
    b.rtol = relTol;
    b.maxit = maxIter;
    b.red = c->red;
    int its = 0;
    bool allConv = true;
    for (int outer = 0; outer < nOuter; ++outer) {
      if (a.nonorth) launch_scalar_grad(c->lc, c->dm, a);
      launch_scalar_assemble(c->lc, c->dm, a);
      bicg_init(c->lc, b);
      int done = 0;
      while (true) {
        for (int k = 0; k < 16; ++k) bicg_iteration(c->lc, b);
        done += 16;
        poll(c, b.fl, 4);
        if (c->hFlags[0] || done > maxIter + 2) break;
      }
      its = c->hFlags[2];
      allConv = allConv && c->hFlags[3] != 0;
    }
    double sc[8];
    CK(cudaMemcpyAsync(sc, c->scal + kScalBicg, sizeof(sc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    download_cells1(c, c->sPhi, phi);
    if (info) {
      info->iterations = its;
      info->converged = allConv ? 1 : 0;
      info->outer = nOuter;
      info->final_res_norm = sc[5];
      std::vector<double> hb(c->C);
      CK(cudaMemcpy(hb.data(), c->rhs, sizeof(double) * c->C, cudaMemcpyDeviceToHost));
      double bn = 0.0;
      for (double x : hb) bn += x * x;
      info->final_rel_res = bn > 0.0 ? sc[5] / std::sqrt(bn) : 0.0;
    }
    return allConv ? ANB_OK : ANB_NOT_CONVERGED;
  });
}

long long anb_launch_count(void) { return g_launches.load(); }

int anb_profile_select(anb_ctx* c, int family) {
  if (!c || family < 0 || family >= kKfCount) return ANB_ERR_INVALID;
  c->prof.flush();
  c->prof.family = family;
  c->prof.launches = 0;
  c->prof.seconds = 0.0;
  c->prof.bytes = 0.0;
  return ANB_OK;
}

int anb_profile_read(anb_ctx* c, long long* launches, double* seconds, double* bytes) {
  if (!c) return ANB_ERR_INVALID;
  if (launches) *launches = c->prof.launches;
  if (seconds) *seconds = c->prof.seconds;
  if (bytes) *bytes = c->prof.bytes;
  return ANB_OK;
}

int anb_debug_gradient(anb_ctx* c, int field, const double* phi, double* gx, double* gy, double* gz) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (!c->bcSet) throw AnbError(ANB_ERR_INVALID, "boundary conditions not set");
    if (field < 0 || field > 3) throw AnbError(ANB_ERR_INVALID, "field must be 0..3");
    CK(cudaSetDevice(c->prm.device));
    const double* s1[1] = {phi};
    upload_cells(c, s1, c->pdx, 1);
    const unsigned char bits[1] = {(unsigned char)(1u << field)};
    const double* in[1] = {c->pdx};
    double* outp[1] = {c->Gc};
    grad(c, 1, in, bits, outp);
    CK(cudaGetLastError());
    double* d[3] = {gx, gy, gz};
    download_cells(c, c->Gc, d, 3);
    return ANB_OK;
  });
}

int anb_debug_momentum(anb_ctx* c, const double* u, const double* v, const double* w, const double* p,
                       double* diag, double* a_pn, double* a_np, double* rhs, double* rau) {
  if (!c) return ANB_ERR_INVALID;
  int rc = anb_set_state(c, u, v, w, p);
  if (rc) return rc;
  return guarded(c, [&]() -> int {
    if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
    check_ready(c);
    const int C = c->C;
    const double* phi[4] = {c->U, c->U + C, c->U + 2 * C, c->P};
    const unsigned char bits[4] = {1, 2, 4, 8};
    double* out[4] = {c->G, c->G + 3 * C, c->G + 6 * C, c->G + 9 * C};
    grad(c, 4, phi, bits, out);
    MomArgs ma{};
    ma.U = c->U;
    ma.Q = c->U;
    ma.G = c->G;
    ma.rho = c->prm.rho;
    ma.mu = c->prm.mu;
    ma.uRelax = c->prm.u_relax;
    ma.relax = c->prm.u_relax < 0.999999 ? 1 : 0;
    ma.val = c->mval;
    ma.diag = c->mdiag;
    ma.rhs = c->rhs;
    ma.rau = c->rau;
    launch_momentum(c->lc, c->dm, ma);
    CK(cudaGetLastError());
    double* d1[1] = {diag};
    if (diag) download_cells(c, c->mdiag, d1, 1);
    double* r1[1] = {rau};
    if (rau) download_cells(c, c->rau, r1, 1);
    if (rhs) {
      double* d3[3] = {rhs, rhs + C, rhs + 2 * C};
      download_cells(c, c->rhs, d3, 3);
    }
    download_offdiag(c, c->mval, a_pn, a_np);
    return ANB_OK;
  });
}

int anb_debug_pressure(anb_ctx* c, const double* u, const double* v, const double* w, const double* p,
                       const double* rau, double* diag, double* a_pn, double* phi_star, double* div_star) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
    if (!c->bcSet) throw AnbError(ANB_ERR_INVALID, "boundary conditions not set");
    CK(cudaSetDevice(c->prm.device));
    const int C = c->C;
    const double* s3[3] = {u, v, w};
    upload_cells(c, s3, c->Us, 3);
    const double* s1[1] = {p};
    upload_cells(c, s1, c->P, 1);
    const double* s2[1] = {rau};
    upload_cells(c, s2, c->rau, 1);
    const double* phi[1] = {c->P};
    const unsigned char bits[1] = {8};
    double* out[1] = {c->G + 9 * C};
    grad(c, 1, phi, bits, out);
    PresArgs pa{};
    pa.Us = c->Us;
    pa.P = c->P;
    pa.Gp = c->G + 9 * C;
    pa.rau = c->rau;
    pa.rho = c->prm.rho;
    pa.val = c->pval;
    pa.diag = c->pdiag;
    pa.phiStar = c->phiStar;
    pa.divStar = c->divStar;
    pa.b = c->pb;
    pa.pc = c->Pc;
    pa.wdinv = c->pwdinv;
    pa.omega = c->amg.omega;
    launch_pressure_rc(c->lc, c->dm, pa);
    CK(cudaGetLastError());
    double* d1[1] = {diag};
    if (diag) download_cells(c, c->pdiag, d1, 1);
    double* d2[1] = {div_star};
    if (div_star) download_cells(c, c->divStar, d2, 1);
    if (a_pn) download_offdiag(c, c->pval, a_pn, nullptr);
    if (phi_star) download_faces(c, c->phiStar, phi_star);
    return ANB_OK;
  });
}

int anb_debug_nonorth(anb_ctx* c, const double* rau, const double* gx, const double* gy, const double* gz,
                      double* div_no) {
  if (!c || !div_no) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
    if (!c->bcSet) throw AnbError(ANB_ERR_INVALID, "boundary conditions not set");
    CK(cudaSetDevice(c->prm.device));
    const int C = c->C;
    const double* s1[1] = {rau};
    upload_cells(c, s1, c->rau, 1);
    const double* s3[3] = {gx, gy, gz};
    upload_cells(c, s3, c->Gc, 3);
    // b = -divBase + div(phi_NO): with a zero base the right-hand side is the divergence itself
    CK(cudaMemsetAsync(c->divCorr, 0, sizeof(double) * C, c->stream));
    NonOrthArgs na{c->rau, c->Gc, c->divCorr, c->pb};
    launch_nonorth_rhs(c->lc, c->dm, na);
    CK(cudaGetLastError());
    double* d1[1] = {div_no};
    download_cells(c, c->pb, d1, 1);
    return ANB_OK;
  });
}

int anb_debug_pressure_solve(anb_ctx* c, const double* b, double* x, int* iters, double* final_res) {
  if (!c) return ANB_ERR_INVALID;
  return guarded(c, [&]() -> int {
    if (c->mixed) throw AnbError(ANB_ERR_UNSUPPORTED, "this entry point needs an FP64 (ANB_PRECISION_FP64) context");
    CK(cudaSetDevice(c->prm.device));
    const double* s1[1] = {b};
    upload_cells(c, s1, c->pb, 1);
    const double* s2[1] = {x};
    upload_cells(c, s2, c->pdx, 1);
    ensure_amg(c);
    int its = 0;
    bool cv = true;
    solve_pressure(c, c->pb, c->pdx, c->prm.p_rel_tol, &its, &cv);
    CK(cudaGetLastError());
    double* d1[1] = {x};
    download_cells(c, c->pdx, d1, 1);
    double h[8];
    CK(cudaMemcpy(h, c->scal + kScalPcg, sizeof(double) * 8, cudaMemcpyDeviceToHost));
    if (iters) *iters = its;
    if (final_res) *final_res = std::sqrt(h[4]);
    return cv ? ANB_OK : ANB_NOT_CONVERGED;
  });
}

}  // extern "C"

namespace anb {

bool context_force_view(const anb_ctx* c, int patch, ForceView* v) {
  if (!c || patch < 0 || patch >= (int)c->hm.patches.size()) return false;
  v->dm = c->dm;
  v->b0 = c->hm.patches[patch].start - c->nI;
  v->b1 = v->b0 + c->hm.patches[patch].nFaces;
  v->mu = c->prm.mu;
  v->bA = c->dBA;
  v->bN = c->dBN;
  v->U = c->U;
  v->P = c->P;
  v->stream = c->stream;
  v->device = c->prm.device;
  return true;
}

void context_set_error(anb_ctx* c, const char* msg) {
  if (c) c->err = msg;
}

}  // namespace anb
