// Ensemble solve: many independent geometries (different body counts, node
// counts per body and wall sizes) solved together.  Every geometry runs its
// own GMRES (the same method as erosion_solve: flexible GMRES with the block
// preconditioner, relaxed mixed precision inside FP64 refinement), and the
// geometries advance in lockstep rounds of one Arnoldi iteration each:
//
//   * the far field of ALL geometries of a round is one persistent launch per
//     precision (k_far64_batch / k_far32_batch over a work list of
//     (geometry, target block, tile split) items), in a launch shape chosen
//     by timing the candidates on the ensemble;
//   * everything else of the round (preconditioner, strengths, self and near
//     sums, assembly, CGS2 Arnoldi, the Givens step, the residual read-back)
//     runs from one captured CUDA graph that is replayed every round; the
//     column count lives in device memory, so the graph only changes when a
//     geometry switches precision, finishes a cycle or outgrows its buffers;
//   * one host synchronisation per round reads every geometry's residual
//     estimate.
// End-of-cycle work (least squares, update, FP64 true residual, a new
// refinement sweep) is per geometry and rare.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "state.h"
#include <chrono>
#include <exception>
#include <thread>
#include "kernels.cuh"

namespace eb {
namespace ensemble {

constexpr double kBatchRelaxFactor = 1e5;   // same switch point as the single solve
constexpr double kBatchTuneMinPairs = 2e8;

struct Member {
  std::unique_ptr<State> s;
  long long ntot = 0, ldv = 0;
  DBuf<double> x, b, r, cur, zc, out, h1, h2, hn, cs, R, part, scal, y;
  DBuf<int> kdev, stdev;
  long long vcap = 0, zcap = 0, rcols = 0, cscap = 0, partcap = 0;
  int nb = 1, Rrows = 1;   // dot-product blocks and rows per block
  // host cycle state
  double bnrm = 0, r0nrm = 0, rho = 0, prev_tr = 1e300, abs_tol = 0, relax_abs = 0;
  double cyc_abs = 0;   // the current cycle's stopping point (tol, or sweep_decades below its start)
  long long kcyc = 0, total = 0, maxl = 0;
  int sweep = 0, prec = 0, status = EROSION_OK;
  bool in_cycle = false, done = false;
  double true_residual = -1;
  // the member's stream (its kernels run concurrently with the other
  // members') and its captured graphs: the part of a round before the far
  // field, and the part after it for each precision
  cudaStream_t side = nullptr;
  cudaEvent_t ev_pre = nullptr, ev_post = nullptr;
  cudaGraphExec_t pre = nullptr, post[2] = {nullptr, nullptr};
  long long launches_pre = 0, launches_post[2] = {0, 0};
};

struct Batch {
  std::vector<Member> m;
  std::vector<int> key;           // per member: -1 idle, else precision of its round
  int n64 = 0, n32 = 0;           // far-field jobs of the current key
  long long items64 = 0, items32 = 0;
  cudaEvent_t ev_far = nullptr, ev_start = nullptr;
  DBuf<FarJob64> jobs64;
  DBuf<FarJob32> jobs32;
  int shape64 = 0, shape32 = 0;   // indices into kFar64Shapes / kFar32Shapes
  double* pinned = nullptr;
  size_t pinned_cap = 0;
  erosion_batch_stats stats{};
  cudaEvent_t a = nullptr, b = nullptr;
  int occ64[4] = {0, 0, 0, 0}, occ32[4] = {0, 0, 0, 0};   // resident CTAs per SM of each shape
};

Batch& batch() {
  static Batch B;
  return B;
}

int dot_blocks_of(long long n, int* R) {
  int nb = (int)std::min<long long>((long long)eb_num_sms() * 8, nblk(n, 256));
  nb = std::max(nb, 1);
  *R = (int)((n + nb - 1) / nb);
  return (int)((n + *R - 1) / *R);
}

void init_member_state(State& m, const State& lib) {
  m.init = true;
  m.device = lib.device;
  m.st = lib.st;
  cudaEvent_t* evs[] = {&m.e0, &m.e1, &m.ef0, &m.ef1, &m.ew0, &m.ew1, &m.et0, &m.et1};
  for (auto* e : evs)
    if (!*e) EB_CK(cudaEventCreate(e));
}

void destroy_member_graphs(Member& mb) {
  if (mb.pre) cudaGraphExecDestroy(mb.pre);
  for (auto& g : mb.post)
    if (g) cudaGraphExecDestroy(g);
  mb.pre = mb.post[0] = mb.post[1] = nullptr;
}

void destroy_graph(Batch& B) {
  for (auto& mb : B.m) destroy_member_graphs(mb);
  B.key.clear();
}

// ---- far-field jobs of a round -------------------------------------------

FarJob64 job64(State& s, const int* sp, int nsplit, double2* partial, int nt_tpt) {
  FarJob64 J;
  J.G = s.geo();
  J.sq = s.sq64.p;
  J.tiles = s.tiles.p;
  J.split_ptr = sp;
  J.mask = s.near.npairs > 0 ? s.near.mask.p : nullptr;
  J.mw = s.near.mw;
  J.partial = partial;
  J.nbx = (int)nblk(s.pr.N, nt_tpt);
  J.nsplit = nsplit;
  J.item0 = 0;
  return J;
}

FarJob32 job32(State& s, int nt_tpt) {
  FarJob32 J;
  J.N = s.pr.N; J.nout = s.pr.nout; J.n = s.pr.n;
  J.src = s.src32.p; J.tgt = s.tgt32.p; J.anchor = s.anchor.p; J.tile_c = s.tile_c.p; J.sq32 = s.sq32.p;
  J.tiles = s.tiles.p;
  J.split_ptr = s.split_ptr32.p;
  J.mask = s.near.npairs > 0 ? s.near.mask.p : nullptr;
  J.mw = s.near.mw;
  J.partial = s.partial.p;
  J.nbx = (int)nblk(s.pr.N, nt_tpt);
  J.nsplit = s.nsplit32;
  J.item0 = 0;
  return J;
}

// Orders the jobs by work per item (largest first, for the tail of the
// persistent loop) and numbers their items.
template <class Job>
long long number_jobs(std::vector<Job>& jobs, const std::vector<double>& cost) {
  std::vector<size_t> idx(jobs.size());
  for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
  std::stable_sort(idx.begin(), idx.end(), [&](size_t a, size_t b) { return cost[a] > cost[b]; });
  std::vector<Job> out;
  long long item = 0;
  for (size_t i : idx) {
    Job J = jobs[i];
    J.item0 = item;
    item += (long long)J.nbx * J.nsplit;
    out.push_back(J);
  }
  jobs.swap(out);
  return item;
}

// Builds (and uploads) the job lists of a round; sizes returned.
void build_jobs(Batch& B, const std::vector<int>& key, int* n64, long long* items64, int* n32, long long* items32,
                double* pairs64, double* pairs32) {
  const FarShape s64 = kFar64Shapes[B.shape64], s32 = kFar32Shapes[B.shape32];
  std::vector<FarJob64> j64;
  std::vector<FarJob32> j32;
  std::vector<double> c64, c32;
  *pairs64 = *pairs32 = 0;
  for (size_t i = 0; i < B.m.size(); ++i) {
    if (key[i] < 0) continue;
    State& s = *B.m[i].s;
    const double srcs = (double)s.pr.N;
    if (key[i] == 0) {
      j64.push_back(job64(s, s.split_ptr64t.p, s.nsplit64t, s.partial.p, s64.nt * s64.tpt));
      c64.push_back(srcs / s.nsplit64t);
      *pairs64 += (double)s.far64_pairs;
    } else {
      if (s.nsplit32 > 0) {
        j32.push_back(job32(s, s32.nt * s32.tpt));
        c32.push_back(srcs / s.nsplit32);
        *pairs32 += (double)s.far32_pairs;
      }
      j64.push_back(job64(s, s.split_ptrw.p, s.nsplitw, s.partial.p + (size_t)s.nsplit32 * s.pr.N,
                          s64.nt * s64.tpt));
      c64.push_back((double)s.pr.nout / s.nsplitw);
      *pairs64 += (double)s.farw_pairs;
    }
  }
  *items64 = number_jobs(j64, c64);
  *items32 = number_jobs(j32, c32);
  *n64 = (int)j64.size();
  *n32 = (int)j32.size();
  cudaStream_t st = state().st;
  if (!j64.empty()) h2d(B.jobs64.ensure(j64.size()), j64.data(), j64.size(), st);
  if (!j32.empty()) h2d(B.jobs32.ensure(j32.size()), j32.data(), j32.size(), st);
  EB_CK(cudaStreamSynchronize(st));
}

// Persistent grid: every resident CTA slot of the GPU, or fewer items.
int persistent_grid(int occ, long long items) {
  long long g = (long long)std::max(occ, 1) * eb_num_sms();
  return (int)std::max<long long>(1, std::min<long long>(g, items));
}

void launch_batch64(Batch& B, int shape, int njobs, long long items, cudaStream_t st) {
  if (njobs == 0) return;
#define EB_B64(IDX, NT, TPT, RCP)                                                                      \
  case IDX: {                                                                                          \
    k_far64_batch<NT, TPT, RCP><<<persistent_grid(B.occ64[IDX], items), NT, 0, st>>>(B.jobs64.p, njobs,   \
                                                                                    items);            \
    break;                                                                                             \
  }
  switch (shape) {
    EB_B64(0, 256, 2, 1)
    EB_B64(1, 128, 4, 1)
    EB_B64(2, 256, 2, 3)
    EB_B64(3, 128, 4, 3)
    default: throw Error(EROSION_BAD_INPUT, "unknown FP64 batch shape");
  }
#undef EB_B64
  EB_LAUNCH_CHECK();
}

void launch_batch32(Batch& B, int shape, int njobs, long long items, cudaStream_t st) {
  if (njobs == 0) return;
#define EB_B32(IDX, NT, TPT, U, MB)                                                                        \
  case IDX: {                                                                                          \
    k_far32_batch<NT, TPT, U, MB><<<persistent_grid(B.occ32[IDX], items), NT, 0, st>>>(B.jobs32.p, njobs, items); \
    break;                                                                                             \
  }
  switch (shape) {
    EB_B32(0, 256, 4, 2, 2)
    EB_B32(1, 256, 4, 4, 2)
    EB_B32(2, 256, 4, 2, 3)
    EB_B32(3, 256, 4, 4, 3)
    default: throw Error(EROSION_BAD_INPUT, "unknown FP32 batch shape");
  }
#undef EB_B32
  EB_LAUNCH_CHECK();
}

static_assert(kFar64Shapes[0].nt == 256 && kFar64Shapes[0].tpt == 2 && kFar64Shapes[0].rcp == 1 &&
              kFar64Shapes[1].nt == 128 && kFar64Shapes[1].tpt == 4 && kFar64Shapes[1].rcp == 1 &&
              kFar64Shapes[2].nt == 256 && kFar64Shapes[2].tpt == 2 && kFar64Shapes[2].rcp == 3 &&
              kFar64Shapes[3].nt == 128 && kFar64Shapes[3].tpt == 4 && kFar64Shapes[3].rcp == 3 &&
              kFar32Shapes[0].nt == 256 && kFar32Shapes[0].tpt == 4 && kFar32Shapes[1].rcp == 4 &&
              kFar32Shapes[2].minb == 3 && kFar32Shapes[2].tpt == 4 && kFar32Shapes[3].rcp == 4 &&
              kFar32Shapes[3].minb == 3,
              "launch_batch shape tables");

// Chooses the ensemble launch shapes by timing each candidate on the jobs of
// an all-FP64 and an all-FP32 round (zeroed strengths: same work).
void occupancy(Batch& B) {
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ64[0], k_far64_batch<256, 2, 1>, 256, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ64[1], k_far64_batch<128, 4, 1>, 128, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ64[2], k_far64_batch<256, 2, 3>, 256, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ64[3], k_far64_batch<128, 4, 3>, 128, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ32[0], k_far32_batch<256, 4, 2, 2>, 256, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ32[1], k_far32_batch<256, 4, 4, 2>, 256, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ32[2], k_far32_batch<256, 4, 2, 3>, 256, 0));
  EB_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&B.occ32[3], k_far32_batch<256, 4, 4, 3>, 256, 0));
}

void tune_batch(Batch& B, double pairs_total) {
  occupancy(B);
  B.shape64 = 0;
  B.shape32 = 0;
  for (int k = 0; k < 8; ++k) B.stats.tune_ms[k] = 0.f;
  if (pairs_total < kBatchTuneMinPairs) return;
  cudaStream_t st = state().st;
  for (auto& mb : B.m) {
    State& s = *mb.s;
    EB_CK(cudaMemsetAsync(s.sq32.p, 0, sizeof(float4) * s.pr.N, st));
    EB_CK(cudaMemsetAsync(s.sq64.p, 0, sizeof(double4) * s.pr.N, st));
  }
  for (int kind = 0; kind < 2; ++kind) {
    const std::vector<int> key(B.m.size(), kind);
    float best = 1e30f;
    const int nsh = kind ? kNumFar32Shapes : kNumFar64Shapes;
    int bestsh = 0;
    for (int sh = 0; sh < nsh; ++sh) {
      if (kind) B.shape32 = sh;
      else B.shape64 = sh;
      int n64, n32;
      long long i64, i32;
      double p64, p32;
      build_jobs(B, key, &n64, &i64, &n32, &i32, &p64, &p32);
      float ms = 1e30f;
      for (int r = 0; r < 2; ++r) {
        EB_CK(cudaEventRecord(B.a, st));
        if (kind) launch_batch32(B, sh, n32, i32, st);
        else launch_batch64(B, sh, n64, i64, st);
        EB_CK(cudaEventRecord(B.b, st));
        EB_CK(cudaEventSynchronize(B.b));
        float t = 0;
        EB_CK(cudaEventElapsedTime(&t, B.a, B.b));
        if (r > 0) ms = std::min(ms, t);
      }
      B.stats.tune_ms[4 * kind + sh] = ms;
      if (ms < best) { best = ms; bestsh = sh; }
    }
    if (kind) B.shape32 = bestsh;
    else B.shape64 = bestsh;
  }
}

// ---- per-member buffers ---------------------------------------------------

// Capacity for the next round of a cycle that has run kcyc iterations.
// Returns true when a buffer the graph refers to moved.
bool ensure_capacity(Member& mb) {
  State& s = *mb.s;
  cudaStream_t st = s.st;
  bool moved = false;
  // the round reads V[:, 0..kcyc] and writes V[:, kcyc+1], Z[:, kcyc] and
  // column kcyc of R
  const long long need_v = mb.kcyc + 2;
  if (need_v > mb.vcap) {
    long long nc = std::min<long long>(mb.maxl + 1, std::max<long long>(2 * mb.vcap, std::max<long long>(need_v, 128)));
    double* old = s.V.p;
    s.V.grow_keep((size_t)nc * mb.ldv, (size_t)mb.vcap * mb.ldv, st);
    mb.vcap = nc;
    moved |= s.V.p != old;
    // the dot partials follow the basis size
    const size_t np = (size_t)nc * mb.nb;
    if (np > (size_t)mb.partcap) { mb.part.release(); mb.part.ensure(np); mb.partcap = (long long)np; moved = true; }
    if ((long long)mb.h1.cap < nc + 1) {
      mb.h1.release(); mb.h2.release();
      mb.h1.ensure(nc + 1); mb.h2.ensure(nc + 1);
      moved = true;
    }
  }
  if (s.pc_active && mb.kcyc + 1 > mb.zcap) {
    long long nc = std::min<long long>(mb.maxl, std::max<long long>(2 * mb.zcap, std::max<long long>(mb.kcyc + 1, 128)));
    double* old = s.Z.p;
    s.Z.grow_keep((size_t)nc * mb.ldv, (size_t)mb.zcap * mb.ldv, st);
    mb.zcap = nc;
    moved |= s.Z.p != old;
  }
  if (mb.kcyc + 1 > mb.rcols) {   // packed R (columns 0..kcyc) and the rotations
    long long nc = std::min<long long>(mb.maxl, std::max<long long>(2 * mb.rcols, std::max<long long>(mb.kcyc + 1, 128)));
    double* oldR = mb.R.p;
    mb.R.grow_keep((size_t)nc * (nc + 1) / 2, (size_t)mb.rcols * (mb.rcols + 1) / 2, st);
    double* oldc = mb.cs.p;
    mb.cs.grow_keep((size_t)2 * nc, (size_t)2 * mb.rcols, st);
    mb.rcols = nc;
    moved |= mb.R.p != oldR || mb.cs.p != oldc;
  }
  if (moved) destroy_member_graphs(mb);   // they refer to the old buffers
  return moved;
}

// ---- the round graph --------------------------------------------------------

void record_member_pre(Member& mb, int idx) {
  State& s = *mb.s;
  cudaStream_t st = s.st;
  const long long N = mb.ntot;
  k_col_get<<<nblk(N, 256), 256, 0, st>>>(s.V.p, mb.ldv, mb.kdev.p, -1, mb.cur.p, N);
  EB_LAUNCH_CHECK();
  const double* den = mb.cur.p;
  if (s.pc_active) {
    apply_preconditioner(s, mb.cur.p, mb.zc.p);
    k_col_put<<<nblk(N, 256), 256, 0, st>>>(s.Z.p, mb.ldv, mb.kdev.p, -1, mb.zc.p, nullptr, N);
    EB_LAUNCH_CHECK();
    den = mb.zc.p;
  }
  operator_prep(s, den, mb.out.p);
  (void)idx;
}

void record_member_post(Member& mb, int prec, double* pinned_slot) {
  State& s = *mb.s;
  cudaStream_t st = s.st;
  const long long N = mb.ntot;
  const double* den = s.pc_active ? mb.zc.p : mb.cur.p;
  operator_post(s, den, mb.out.p, far_slots(s, prec));
  const size_t smem = (size_t)mb.Rrows * sizeof(double);
  k_dot_part_dk<<<mb.nb, 256, smem, st>>>(s.V.p, mb.ldv, mb.kdev.p, mb.out.p, N, mb.Rrows, mb.part.p);
  EB_LAUNCH_CHECK();
  k_dot_reduce_dk<<<std::max(1, eb_num_sms()), 256, 0, st>>>(mb.part.p, mb.nb, mb.kdev.p, 0, mb.h1.p);
  EB_LAUNCH_CHECK();
  k_vh_dk<<<nblk(N, 256), 256, 0, st>>>(s.V.p, mb.ldv, mb.kdev.p, mb.h1.p, -1.0, mb.out.p, N);
  EB_LAUNCH_CHECK();
  k_dot_part_dk<<<mb.nb, 256, smem, st>>>(s.V.p, mb.ldv, mb.kdev.p, mb.out.p, N, mb.Rrows, mb.part.p);
  EB_LAUNCH_CHECK();
  k_dot_reduce_dk<<<std::max(1, eb_num_sms()), 256, 0, st>>>(mb.part.p, mb.nb, mb.kdev.p, 0, mb.h2.p);
  EB_LAUNCH_CHECK();
  k_vh_dk<<<nblk(N, 256), 256, 0, st>>>(s.V.p, mb.ldv, mb.kdev.p, mb.h2.p, -1.0, mb.out.p, N);
  EB_LAUNCH_CHECK();
  // ||w||^2 with the single-column forms
  k_dot_part<<<mb.nb, 256, smem, st>>>(mb.out.p, N, 1, mb.out.p, N, mb.Rrows, mb.part.p);
  EB_LAUNCH_CHECK();
  k_dot_reduce<<<1, 256, 0, st>>>(mb.part.p, mb.nb, 1, mb.hn.p, 0);
  EB_LAUNCH_CHECK();
  k_givens_step<<<1, 32, 0, st>>>(mb.kdev.p, mb.h1.p, mb.h2.p, mb.hn.p, mb.cs.p, mb.R.p, mb.scal.p, mb.scal.p + 1,
                                  mb.scal.p + 2, mb.scal.p + 3, mb.stdev.p);
  EB_LAUNCH_CHECK();
  k_col_put<<<nblk(N, 256), 256, 0, st>>>(s.V.p, mb.ldv, mb.kdev.p, 0, mb.out.p, mb.scal.p + 3, N);
  EB_LAUNCH_CHECK();
  k_inc<<<1, 32, 0, st>>>(mb.kdev.p);
  EB_LAUNCH_CHECK();
  EB_CK(cudaMemcpyAsync(pinned_slot, mb.scal.p + 2, sizeof(double), cudaMemcpyDeviceToHost, st));
  EB_CK(cudaMemcpyAsync(reinterpret_cast<int*>(pinned_slot + 1), mb.stdev.p, sizeof(int), cudaMemcpyDeviceToHost,
                        st));
}

// Captures one member's graphs on its stream (outside any other capture).
template <class F>
cudaGraphExec_t capture_on(cudaStream_t st, F&& record, long long* launches) {
  const long long l0 = g_launches;
  EB_CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
  cudaGraph_t g = nullptr;
  try {
    record();
  } catch (...) {
    cudaStreamEndCapture(st, &g);
    if (g) cudaGraphDestroy(g);
    throw;
  }
  EB_CK(cudaStreamEndCapture(st, &g));
  cudaGraphExec_t e = nullptr;
  cudaError_t err = cudaGraphInstantiate(&e, g, 0);
  cudaGraphDestroy(g);
  EB_CK(err);
  *launches = g_launches - l0;
  g_launches = l0;
  return e;
}

void capture_member(Batch& B, Member& mb, int idx) {
  destroy_member_graphs(mb);
  mb.pre = capture_on(mb.side, [&] { record_member_pre(mb, idx); }, &mb.launches_pre);
  for (int prec = 0; prec < 2; ++prec)
    mb.post[prec] = capture_on(mb.side, [&] { record_member_post(mb, prec, B.pinned + 2 * idx); },
                               &mb.launches_post[prec]);
  B.stats.graph_captures++;
}

// One round: every active member's pre-graph on its own stream, the
// ensemble far field on the library stream once they are all done, then the
// post-graphs, again concurrently.
void run_round(Batch& B, const std::vector<int>& key) {
  cudaStream_t st = state().st;
  EB_CK(cudaEventRecord(B.ev_start, st));
  for (size_t i = 0; i < B.m.size(); ++i) {
    if (key[i] < 0) continue;
    Member& mb = B.m[i];
    EB_CK(cudaStreamWaitEvent(mb.side, B.ev_start, 0));
    EB_CK(cudaGraphLaunch(mb.pre, mb.side));
    g_launches += mb.launches_pre;
    EB_CK(cudaEventRecord(mb.ev_pre, mb.side));
    EB_CK(cudaStreamWaitEvent(st, mb.ev_pre, 0));
  }
  launch_batch64(B, B.shape64, B.n64, B.items64, st);
  launch_batch32(B, B.shape32, B.n32, B.items32, st);
  EB_CK(cudaEventRecord(B.ev_far, st));
  for (size_t i = 0; i < B.m.size(); ++i) {
    if (key[i] < 0) continue;
    Member& mb = B.m[i];
    EB_CK(cudaStreamWaitEvent(mb.side, B.ev_far, 0));
    EB_CK(cudaGraphLaunch(mb.post[key[i]], mb.side));
    g_launches += mb.launches_post[key[i]];
    EB_CK(cudaEventRecord(mb.ev_post, mb.side));
    EB_CK(cudaStreamWaitEvent(st, mb.ev_post, 0));
  }
  EB_CK(cudaStreamSynchronize(st));
}

// ---- cycles ------------------------------------------------------------------

void least_squares_update(Member& mb) {
  State& s = *mb.s;
  cudaStream_t st = s.st;
  const long long L = mb.kcyc;
  if (L == 0) return;
  std::vector<double> R((size_t)L * (L + 1) / 2), cs((size_t)2 * L);
  d2h(R.data(), mb.R.p, R.size(), st);
  d2h(cs.data(), mb.cs.p, cs.size(), st);
  EB_CK(cudaStreamSynchronize(st));
  std::vector<double> y(L + 1, 0.0);
  y[0] = mb.r0nrm;
  for (long long kk = 1; kk <= L; ++kk) {
    const double c = cs[2 * (kk - 1)], sn = cs[2 * (kk - 1) + 1];
    const double a1 = y[kk - 1], a2 = y[kk];
    y[kk - 1] = c * a1 - sn * a2;
    y[kk] = sn * a1 + c * a2;
  }
  auto Rc = [&](long long col, long long row) { return R[(size_t)col * (col + 1) / 2 + row]; };
  for (long long kb = 1; kb <= L; ++kb) {
    const long long kk = L + 1 - kb;
    y[kk - 1] = y[kk - 1] / Rc(kk - 1, kk - 1);
    const double t = -y[kk - 1];
    for (long long i = 1; i <= kk - 1; ++i) y[i - 1] += t * Rc(kk - 1, i - 1);
  }
  h2d(mb.y.ensure((size_t)L + 1), y.data(), (size_t)L, st);
  const double* basis = s.pc_active ? s.Z.p : s.V.p;
  k_vh<<<nblk(mb.ntot, 256), 256, 0, st>>>(basis, mb.ldv, (int)L, mb.y.p, 1.0, mb.x.p, mb.ntot);
  EB_LAUNCH_CHECK();
  EB_CK(cudaStreamSynchronize(st));
}

// Starts a GMRES cycle on the residual in mb.r; false when it is already
// below the tolerance.
bool start_cycle(Member& mb) {
  State& s = *mb.s;
  cudaStream_t st = s.st;
  const long long N = mb.ntot;
  mb.r0nrm = device_norm(s, mb.r.p, N);
  if (!std::isfinite(mb.r0nrm)) throw Error(EROSION_BREAKDOWN, "non-finite initial residual");
  mb.rho = mb.r0nrm;
  mb.kcyc = 0;
  if (mb.r0nrm <= mb.abs_tol) return false;
  // as gmres_solve: a mixed-precision cycle stops sweep_decades below its
  // start unless that point lies within a decade of tol
  const int sd = s.pr.P.precision != 0 ? std::max(0, (int)s.pr.P.sweep_decades) : 0;
  mb.cyc_abs = (s.pr.P.precision != 0 ? 0.5 : 1.0) * mb.abs_tol;   // a mixed sweep to tol aims at half of it
  if (sd > 0 && mb.r0nrm * std::pow(10.0, -sd) > 10.0 * mb.abs_tol) mb.cyc_abs = mb.r0nrm * std::pow(10.0, -sd);
  ensure_capacity(mb);
  k_copy<<<nblk(N, 256), 256, 0, st>>>(mb.r.p, s.V.p, N);
  EB_LAUNCH_CHECK();
  k_scale<<<nblk(N, 256), 256, 0, st>>>(s.V.p, 1.0 / mb.r0nrm, N);
  EB_LAUNCH_CHECK();
  const int one = 1;
  const double sc[4] = {1.0, mb.r0nrm, mb.r0nrm, 0.0};
  h2d(mb.kdev.p, &one, 1, st);
  h2d(mb.scal.p, sc, 4, st);
  EB_CK(cudaStreamSynchronize(st));
  mb.in_cycle = true;
  return true;
}

// After a cycle: x += basis y; FP64 refinement bookkeeping (as gmres_solve).
void finish_cycle(Member& mb, int rc_cycle, double tol) {
  State& s = *mb.s;
  cudaStream_t st = s.st;
  mb.in_cycle = false;
  least_squares_update(mb);
  if (rc_cycle == EROSION_BREAKDOWN) { mb.status = EROSION_BREAKDOWN; mb.done = true; return; }
  if (s.pr.P.precision == 0 && !s.pc_active) {   // unpreconditioned FP64: one cycle, as gmres_solve
    mb.status = rc_cycle;
    mb.true_residual = mb.rho / mb.bnrm;
    mb.done = true;
    return;
  }
  mb.sweep++;
  apply_operator(s, mb.x.p, mb.r.p, 0);
  k_bminus<<<nblk(mb.ntot, 256), 256, 0, st>>>(mb.b.p, mb.r.p, mb.ntot);
  EB_LAUNCH_CHECK();
  const double tr = device_norm(s, mb.r.p, mb.ntot) / mb.bnrm;
  mb.true_residual = tr;
  if (!std::isfinite(tr)) throw Error(EROSION_BREAKDOWN, "non-finite true residual");
  const bool floor = mb.sweep > 1 && (tr <= 2.0 * tol || tr > 0.5 * mb.prev_tr);
  if (tr <= tol || floor) { mb.status = EROSION_OK; mb.done = true; return; }
  mb.prev_tr = tr;
  const int sd = std::max(0, (int)s.pr.P.sweep_decades);
  if (mb.total >= mb.maxl || mb.sweep >= 6 + 2 * sd) { mb.status = EROSION_MAXITER; mb.done = true; return; }
  if (!start_cycle(mb)) finish_cycle(mb, EROSION_OK, tol);
}

}  // namespace ensemble

using namespace ensemble;

void release_batch() {
  Batch& B = batch();
  destroy_graph(B);
  for (auto& mb : B.m) {
    if (mb.side) cudaStreamSynchronize(mb.side);
    release_state_buffers(*mb.s);
    DBuf<double>* bufs[] = {&mb.x, &mb.b, &mb.r, &mb.cur, &mb.zc, &mb.out, &mb.h1, &mb.h2, &mb.hn,
                            &mb.cs, &mb.R, &mb.part, &mb.scal, &mb.y};
    for (auto* q : bufs) q->release();
    mb.kdev.release();
    mb.stdev.release();
    if (mb.ev_pre) cudaEventDestroy(mb.ev_pre);
    if (mb.ev_post) cudaEventDestroy(mb.ev_post);
    if (mb.side) cudaStreamDestroy(mb.side);
    mb.ev_pre = mb.ev_post = nullptr;
    mb.side = nullptr;
  }
  B.m.clear();
  B.jobs64.release();
  B.jobs32.release();
}

}  // namespace eb

using namespace eb;
using namespace eb::ensemble;

extern "C" {

int erosion_solve_batch(const erosion_params* p, int32_t nbatch, const int64_t* npts, const int64_t* nbods,
                        const int64_t* nouter, const double* xx, const double* yy, double* density, int64_t* nits) {
  State& lib = state();
  std::lock_guard<std::mutex> lk(lib.mu);
  try {
    ensure_init(lib);
    if (nbatch <= 0 || !npts || !nbods || !nouter || !density || !nits)
      throw Error(EROSION_BAD_INPUT, "erosion_solve_batch: empty ensemble or null array");
    erosion_params P;
    if (p) P = *p;
    else erosion_default_params(&P);
    Batch& B = batch();
    release_batch();
    if (!B.a) { EB_CK(cudaEventCreate(&B.a)); EB_CK(cudaEventCreate(&B.b)); }
    B.stats = erosion_batch_stats{};
    B.m.resize(nbatch);
    if (B.pinned_cap < 2 * (size_t)nbatch) {
      if (B.pinned) cudaFreeHost(B.pinned);
      B.pinned = nullptr;
      EB_CK(cudaMallocHost((void**)&B.pinned, 2 * (size_t)nbatch * sizeof(double)));
      B.pinned_cap = 2 * (size_t)nbatch;
    }
    cudaStream_t st = lib.st;
    EB_CK(cudaEventRecord(B.a, st));
    // set-up: geometry, near lists, tiles, preconditioner, right-hand side.
    // Each member works on its own stream and buffers, so the members' set-ups
    // (host near-list construction included) run on a pool of host threads.
    std::vector<size_t> node_offs(nbatch), den_offs(nbatch);
    {
      size_t node_off = 0, den_off = 0;
      for (int g = 0; g < nbatch; ++g) {
        if (npts[g] < 0 || nbods[g] < 0 || nouter[g] < 0) throw Error(EROSION_BAD_INPUT, "negative sizes");
        node_offs[g] = node_off;
        den_offs[g] = den_off;
        node_off += (size_t)npts[g] * nbods[g];
        den_off += 2 * (size_t)nouter[g] + 2 * (size_t)npts[g] * nbods[g] + 3 * (size_t)nbods[g];
      }
    }
    for (int g = 0; g < nbatch; ++g) {
      Member& mb = B.m[g];
      mb.s = std::make_unique<State>();
      init_member_state(*mb.s, lib);
      EB_CK(cudaStreamCreateWithFlags(&mb.side, cudaStreamNonBlocking));
      EB_CK(cudaEventCreateWithFlags(&mb.ev_pre, cudaEventDisableTiming));
      EB_CK(cudaEventCreateWithFlags(&mb.ev_post, cudaEventDisableTiming));
      mb.s->st = mb.side;
    }
    const auto t_setup = std::chrono::steady_clock::now();
    auto setup_member = [&](int g) {
      Member& mb = B.m[g];
      State& s = *mb.s;
      // the ensemble's far field runs in the ensemble's own launch shapes
      // (tune_batch), so the members skip the per-geometry timing
      s.force_shape[0] = 0;
      s.force_shape[1] = 0;
      s.force_shape[2] = 0;
      Problem pr;
      pr.P = P;
      pr.n = (int)npts[g]; pr.M = (int)nbods[g]; pr.nout = (int)nouter[g];
      const size_t nb = (size_t)pr.n * pr.M;
      double* dx = s.d_xx.ensure(std::max<size_t>(nb, 1));
      double* dy = s.d_yy.ensure(std::max<size_t>(nb, 1));
      h2d(dx, xx + node_offs[g], nb, s.st);
      h2d(dy, yy + node_offs[g], nb, s.st);
      setup_problem(s, pr, dx, dy);
      mb.ntot = s.pr.ntot;
      mb.ldv = (mb.ntot + 31) & ~31LL;
      mb.maxl = std::min<long long>(P.maxl > 0 ? P.maxl : 10, mb.ntot);
      mb.nb = dot_blocks_of(mb.ntot, &mb.Rrows);
      mb.x.ensure(mb.ntot); mb.b.ensure(mb.ntot); mb.r.ensure(mb.ntot);
      mb.cur.ensure(mb.ntot); mb.zc.ensure(mb.ntot); mb.out.ensure(mb.ntot);
      mb.hn.ensure(1); mb.scal.ensure(4); mb.kdev.ensure(1); mb.stdev.ensure(1);
      mb.vcap = mb.zcap = mb.rcols = mb.partcap = 0;
      s.V.release(); s.Z.release();
      h2d(mb.x.p, density + den_offs[g], (size_t)mb.ntot, s.st);
      bool zero = true;
      for (long long i = 0; i < mb.ntot && zero; ++i) zero = density[den_offs[g] + i] == 0.0;
      build_rhs(s, mb.b.p);
      mb.bnrm = device_norm(s, mb.b.p, mb.ntot);
      if (mb.bnrm == 0.0) throw Error(EROSION_BAD_INPUT, "erosion_solve_batch: zero right-hand side");
      mb.abs_tol = P.tol * mb.bnrm;
      mb.relax_abs = P.precision == 1 ? (P.relax_tol > 0 ? P.relax_tol : P.tol * kBatchRelaxFactor) * mb.bnrm : 0.0;
      if (zero) {
        k_copy<<<nblk(mb.ntot, 256), 256, 0, s.st>>>(mb.b.p, mb.r.p, mb.ntot);
        EB_LAUNCH_CHECK();
      } else {
        apply_operator(s, mb.x.p, mb.r.p, 0);
        k_bminus<<<nblk(mb.ntot, 256), 256, 0, s.st>>>(mb.b.p, mb.r.p, mb.ntot);
        EB_LAUNCH_CHECK();
        // as gmres_solve: in the refinement forms a guess no better than zero
        // is replaced by zero
        const bool refine = P.precision != 0 || s.pc_active;
        if (refine && !(device_norm(s, mb.r.p, mb.ntot) < mb.bnrm)) {
          EB_CK(cudaMemsetAsync(mb.x.p, 0, (size_t)mb.ntot * sizeof(double), s.st));
          k_copy<<<nblk(mb.ntot, 256), 256, 0, s.st>>>(mb.b.p, mb.r.p, mb.ntot);
          EB_LAUNCH_CHECK();
        }
      }
      if (!start_cycle(mb)) finish_cycle(mb, EROSION_OK, P.tol);
      EB_CK(cudaStreamSynchronize(s.st));
    };
    {
      const int nthr = std::max(1, std::min<int>(nbatch, std::min(16u, std::max(1u, std::thread::hardware_concurrency()))));
      std::vector<std::thread> pool;
      std::vector<std::exception_ptr> errs(nthr);
      for (int t = 0; t < nthr; ++t)
        pool.emplace_back([&, t]() {
          try {
            EB_CK(cudaSetDevice(lib.device));
            for (int g = t; g < nbatch; g += nthr) setup_member(g);
          } catch (...) {
            errs[t] = std::current_exception();
          }
        });
      for (auto& th : pool) th.join();
      for (auto& e : errs)
        if (e) std::rethrow_exception(e);
    }
    B.stats.setup_host_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_setup).count();
    double pairs_total = 0;
    for (int g = 0; g < nbatch; ++g) pairs_total += (double)B.m[g].s->far64_pairs;
    if (!B.ev_far) {
      EB_CK(cudaEventCreateWithFlags(&B.ev_far, cudaEventDisableTiming));
      EB_CK(cudaEventCreateWithFlags(&B.ev_start, cudaEventDisableTiming));
    }
    tune_batch(B, pairs_total);
    B.stats.shape64 = B.shape64;
    B.stats.shape32 = B.shape32;
    // lockstep rounds
    std::vector<int> key(nbatch);
    while (true) {
      bool any = false;
      for (int g = 0; g < nbatch; ++g) {
        Member& mb = B.m[g];
        key[g] = -1;
        if (mb.done || !mb.in_cycle) continue;
        mb.prec = (mb.relax_abs > 0.0 && mb.rho <= mb.relax_abs) ? 1 : 0;
        key[g] = mb.prec;
        if (ensure_capacity(mb) || !mb.pre) capture_member(B, mb, g);
        any = true;
      }
      if (!any) break;
      if (key != B.key) {
        double p64, p32;
        build_jobs(B, key, &B.n64, &B.items64, &B.n32, &B.items32, &p64, &p32);
        B.stats.pairs64_per_round = p64;
        B.stats.pairs32_per_round = p32;
        B.key = key;
      }
      run_round(B, key);
      B.stats.rounds++;
      B.stats.pairs64_total += B.stats.pairs64_per_round;
      B.stats.pairs32_total += B.stats.pairs32_per_round;
      for (int g = 0; g < nbatch; ++g) {
        if (key[g] < 0) continue;
        Member& mb = B.m[g];
        const double rho = B.pinned[2 * g];
        int flag = 0;
        std::memcpy(&flag, &B.pinned[2 * g + 1], sizeof(int));
        mb.kcyc++;
        mb.total++;
        if (key[g] == 1) mb.s->stats.matvecs_fp32++;
        mb.s->stats.matvecs++;
        if (flag == 3) throw Error(EROSION_BREAKDOWN, "non-finite value in the Arnoldi process (ensemble)");
        if (flag == 2) { finish_cycle(mb, EROSION_BREAKDOWN, P.tol); continue; }
        mb.rho = rho;
        if (rho <= mb.cyc_abs) finish_cycle(mb, EROSION_OK, P.tol);
        else if (mb.kcyc >= mb.maxl || mb.total >= mb.maxl)
          finish_cycle(mb, rho < mb.r0nrm ? EROSION_MAXITER : EROSION_BREAKDOWN, P.tol);
      }
    }
    destroy_graph(B);
    EB_CK(cudaEventRecord(B.b, st));
    EB_CK(cudaEventSynchronize(B.b));
    float ms = 0;
    EB_CK(cudaEventElapsedTime(&ms, B.a, B.b));
    B.stats.ms_total = ms;
    int worst = EROSION_OK;
    for (int g = 0; g < nbatch; ++g) {
      Member& mb = B.m[g];
      d2h(density + den_offs[g], mb.x.p, (size_t)mb.ntot, st);
      nits[g] = mb.total;
      B.stats.iterations += mb.total;
      if (mb.status != EROSION_OK && worst == EROSION_OK) worst = mb.status;
      B.stats.max_true_residual = std::max(B.stats.max_true_residual, mb.true_residual);
    }
    B.stats.geometries = nbatch;
    EB_CK(cudaStreamSynchronize(st));
    set_status(worst, worst == EROSION_OK ? "" : "a geometry of the ensemble did not converge");
    return worst;
  } catch (const Error& e) {
    if (lib.st) cudaStreamSynchronize(lib.st);
    destroy_graph(batch());
    set_status(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    if (lib.st) cudaStreamSynchronize(lib.st);
    destroy_graph(batch());
    set_status(EROSION_CUDA_ERROR, e.what());
    return EROSION_CUDA_ERROR;
  }
}

void erosion_get_batch_stats(erosion_batch_stats* out) {
  if (out) *out = batch().stats;
}

}  // extern "C"
