// Host orchestration of the boundary operator and the GMRES solve, and the
// C ABI entry points that replace the reference's libstokes.so.
#include "state.h"
#include "kernels.cuh"
#include <chrono>
#include <cmath>
#include <cstring>

namespace eb {

State& state() {
  static State s;
  return s;
}

std::atomic<long long> g_launches{0};

thread_local int t_status = EROSION_OK;
thread_local std::string t_err;

void set_status(int code, const std::string& msg) {
  t_status = code;
  t_err = msg;
}
static int g_num_sms = 148;
int eb_num_sms() { return g_num_sms; }

void allow_max_dynamic_smem(const void* fn) {
  int dev = 0, optin = 0;
  EB_CK(cudaGetDevice(&dev));
  EB_CK(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  cudaFuncAttributes fa;
  EB_CK(cudaFuncGetAttributes(&fa, fn));   // the cap excludes the kernel's static shared memory
  EB_CK(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes));
}

void ensure_init(State& s) {
  if (s.init) return;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0)
    throw Error(EROSION_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
  EB_CK(cudaGetDevice(&s.device));
  cudaDeviceProp prop;
  EB_CK(cudaGetDeviceProperties(&prop, s.device));
  g_num_sms = prop.multiProcessorCount;
  EB_CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
  EB_CK(cudaEventCreate(&s.e0));
  EB_CK(cudaEventCreate(&s.e1));
  EB_CK(cudaEventCreate(&s.ef0));
  EB_CK(cudaEventCreate(&s.ef1));
  EB_CK(cudaEventCreate(&s.ew0));
  EB_CK(cudaEventCreate(&s.ew1));
  EB_CK(cudaEventCreate(&s.et0));
  EB_CK(cudaEventCreate(&s.et1));
  s.init = true;
}

// The circulant matrix of fourierDiff (stokesSolver.f:348-388) for even n:
// d[m] = (1/2)(-1)^m cot(pi m/n), d[0] = d[n/2] = 0.
static std::vector<double> spectral_kernel(int n) {
  std::vector<double> d(n, 0.0);
  const double pi = 4.0 * std::atan(1.0);
  for (int m = 1; m < n; ++m) {
    if (2 * m == n) continue;
    double t = pi * m / n;
    d[m] = 0.5 * ((m & 1) ? -1.0 : 1.0) * std::cos(t) / std::sin(t);
  }
  return d;
}

static void build_near(State& s, const std::vector<double2>& hxy, const std::vector<double>& hsp,
                       const std::vector<double2>& hcen, const std::vector<double>& hrb) {
  const Problem& pr = s.pr;
  const int n = pr.n, M = pr.M, nout = pr.nout, N = pr.N;
  const double TWOPI = 8.0 * std::atan(1.0);
  Near& nr = s.near;
  // matvec_DLP_fmmbary's wall length scale: 'lw' is an implicitly typed
  // INTEGER there (stokesSolver.f:705-709), so each partial sum truncates and
  // the mean is an integer division.
  long long lw = 0;
  for (int k = 0; k < nout; ++k) lw = (long long)((double)lw + hsp[k]);
  lw = lw / nout;
  nr.lw = lw;
  nr.wall_bodies.clear();

  std::vector<int> pc, pt;   // (source curve, target node) in the reference's order
  if (pr.P.ibary == 1 && pr.P.ifmm != 0) {
    const double alpha1 = 4.0, alpha2 = 4.0, bw = pr.P.wall_b;
    for (int b = 0; b < M; ++b) {   // :711-816
      double dsum = hrb[b] + alpha2 * (double)lw * TWOPI / nout;
      double dsum2 = bw - dsum;
      if (std::fabs(hcen[b].y) >= dsum2) {
        nr.wall_bodies.push_back(b);
        for (int k = 0; k < n; ++k) {
          int g = nout + b * n + k;
          if (std::fabs(hxy[g].y) >= dsum2) { pc.push_back(0); pt.push_back(g); }
        }
        double r = bw - std::fabs(hcen[b].y) + 2.0 * hrb[b];
        for (int j = 0; j < nout; ++j) {
          double dx = hcen[b].x - hxy[j].x, dy = hcen[b].y - hxy[j].y;
          if (dx * dx + dy * dy <= r * r) { pc.push_back(1 + b); pt.push_back(j); }
        }
      }
    }
    for (int sb = 0; sb < M; ++sb) {   // :838-926
      for (int t = 0; t < M; ++t) {
        if (t == sb) continue;
        double dx = hcen[sb].x - hcen[t].x, dy = hcen[sb].y - hcen[t].y;
        double d2 = dx * dx + dy * dy;
        double rsum = hrb[sb] + hrb[t] + alpha1 * (hrb[sb] + hrb[t]) * TWOPI / n;
        if (d2 <= rsum * rsum) {
          for (int k = 0; k < n; ++k) {
            int g = nout + t * n + k;
            double ex = hcen[sb].x - hxy[g].x, ey = hcen[sb].y - hxy[g].y;
            if (ex * ex + ey * ey <= rsum * rsum) { pc.push_back(1 + sb); pt.push_back(g); }
          }
        }
      }
    }
  } else if (pr.P.ibary == 1) {
    // matvec_DLP_bary (:1128-1516): every pair of distinct curves.
    for (int g = nout; g < N; ++g) { pc.push_back(0); pt.push_back(g); }
    for (int sb = 0; sb < M; ++sb) {
      for (int g = 0; g < N; ++g) {
        if (g >= nout && (g - nout) / n == sb) continue;
        pc.push_back(1 + sb); pt.push_back(g);
      }
    }
  }
  const long long P = (long long)pc.size();
  nr.npairs = P;
  nr.mw = (M + 1 + 31) / 32;
  if (P == 0) { nr.nsrc = 0; nr.n_bd_work = nr.n_bary_work = 0; return; }
  // group by source curve, stable
  std::vector<long long> cnt(M + 2, 0);
  for (long long p = 0; p < P; ++p) cnt[pc[p] + 1]++;
  for (int c = 0; c <= M; ++c) cnt[c + 1] += cnt[c];
  std::vector<int> order(P);
  {
    std::vector<long long> pos(cnt.begin(), cnt.end() - 1);
    for (long long p = 0; p < P; ++p) order[pos[pc[p]]++] = (int)p;
  }
  nr.h_src_curve.clear(); nr.h_src_ptr.clear(); nr.h_pair_tgt.assign(P, 0);
  std::vector<long long> hbdoff;
  std::vector<int2> hbdw;
  std::vector<int4> hbw;
  long long bdtot = 0;
  for (int c = 0; c <= M; ++c) {
    if (cnt[c + 1] == cnt[c]) continue;
    int sidx = (int)nr.h_src_curve.size();
    nr.h_src_curve.push_back(c);
    nr.h_src_ptr.push_back((int)cnt[c]);
    int len = c == 0 ? nout : n;
    hbdoff.push_back(bdtot);
    bdtot += 5LL * len;
    for (int j0 = 0; j0 < len; j0 += BD_NT) hbdw.push_back(make_int2(sidx, j0));
    for (long long p0 = cnt[c]; p0 < cnt[c + 1]; p0 += NEAR_NT)
      hbw.push_back(make_int4(sidx, (int)p0, (int)std::min<long long>(p0 + NEAR_NT, cnt[c + 1]), 0));
  }
  nr.h_src_ptr.push_back((int)P);
  for (long long q = 0; q < P; ++q) nr.h_pair_tgt[q] = pt[order[q]];
  nr.nsrc = (int)nr.h_src_curve.size();
  nr.bd_total = bdtot;
  nr.n_bd_work = (int)hbdw.size();
  nr.n_bary_work = (int)hbw.size();
  // per-target list of pair slots (pairs are now in grouped order)
  std::vector<int> tptr(N + 1, 0), tpairs(P);
  for (long long q = 0; q < P; ++q) tptr[nr.h_pair_tgt[q] + 1]++;
  for (int g = 0; g < N; ++g) tptr[g + 1] += tptr[g];
  {
    std::vector<int> pos(tptr.begin(), tptr.end() - 1);
    for (long long q = 0; q < P; ++q) tpairs[pos[nr.h_pair_tgt[q]]++] = (int)q;
  }
  std::vector<unsigned> mask((size_t)N * nr.mw, 0u);
  for (long long q = 0; q < P; ++q) {
    int g = nr.h_pair_tgt[q];
    int c = pc[order[q]];
    mask[(size_t)g * nr.mw + (c >> 5)] |= 1u << (c & 31);
  }
  cudaStream_t st = s.st;
  h2d(nr.src_curve.ensure(nr.nsrc), nr.h_src_curve.data(), nr.nsrc, st);
  h2d(nr.pair_tgt.ensure(P), nr.h_pair_tgt.data(), P, st);
  h2d(nr.tptr.ensure(N + 1), tptr.data(), N + 1, st);
  h2d(nr.tpairs.ensure(P), tpairs.data(), P, st);
  h2d(nr.bd_off.ensure(nr.nsrc), hbdoff.data(), nr.nsrc, st);
  h2d(nr.bd_work.ensure(hbdw.size()), hbdw.data(), hbdw.size(), st);
  h2d(nr.bary_work.ensure(hbw.size()), hbw.data(), hbw.size(), st);
  h2d(nr.mask.ensure(mask.size()), mask.data(), mask.size(), st);
  s.bd.ensure(bdtot);
  s.pair_out.ensure(P);
  EB_CK(cudaStreamSynchronize(st));   // host vectors go out of scope
}

// Split-K of the far-field sums: about 8 (target block, tile range) CTAs per
// SM, contiguous tile ranges of equal count.  With the kernel's resident CTAs
// per SM known (resident > 0), the count is chosen within [want/2, 2 want]
// so that the CTAs fill whole waves: W = CTAs / (SMs x resident) waves leave
// the SMs partly idle during the last ceil(W) - W of a wave, so the count
// with the largest W / ceil(W) wins (the smaller count within 0.5%).  At 400
// bodies the FP32 kernel (104 target blocks, 2 resident CTAs) goes from 12
// splits (4.2 waves) to 17 (5.97 waves).
static int far_split_count(int N, int ntile, int targets_per_cta, int resident = 0) {
  const int TB = (int)nblk(N, targets_per_cta);
  const int want = std::max(1, std::min((int)std::ceil(8.0 * g_num_sms / TB), ntile));
  if (resident <= 0) return want;
  const double conc = (double)g_num_sms * resident;
  int best = want;
  double beste = -1.0;
  for (int ns = std::max(1, want / 2); ns <= std::min(ntile, 2 * want); ++ns) {
    const double w = (double)TB * ns / conc;
    const double e = w / std::ceil(w);
    if (e > beste + 0.005) { beste = e; best = ns; }
  }
  return best;
}

// Tile ranges [t0 + q (t1-t0)/ns, ...) of equal count over tiles [t0, t1).
static void upload_splits(State& s, DBuf<int>& buf, int ns, int t0, int t1) {
  std::vector<int> sp(ns + 1);
  for (int q = 0; q <= ns; ++q) sp[q] = t0 + (int)((long long)q * (t1 - t0) / ns);
  h2d(buf.ensure(sp.size()), sp.data(), sp.size(), s.st);
  EB_CK(cudaStreamSynchronize(s.st));   // sp goes out of scope
}

static void build_tiles(State& s) {
  const Problem& pr = s.pr;
  std::vector<int4> tl;
  auto add = [&](int start, int len, int c, int ts) {
    for (int o = 0; o < len; o += ts) tl.push_back(make_int4(start + o, std::min(ts, len - o), c, 0));
  };
  add(0, pr.nout, 0, WALL_TS);
  s.nwall_tiles = (int)tl.size();
  for (int b = 0; b < pr.M; ++b) add(pr.nout + b * pr.n, pr.n, 1 + b, FAR_TS);
  s.ntile = (int)tl.size();
  h2d(s.tiles.ensure(tl.size()), tl.data(), tl.size(), s.st);
  // tile splits of the shear-stress and target sums (the far-field kernels
  // get theirs from plan_far, per launch shape)
  s.nsplit = far_split_count(pr.N, s.ntile, FAR_NT * FAR_TPT);
  upload_splits(s, s.split_ptr, s.nsplit, 0, s.ntile);
  s.partial.ensure((size_t)s.nsplit * pr.N);
  // self-curve tasks: (first target, count <= 256, curve, source chunk)
  std::vector<int4> st;
  s.n_self_slots = 1;
  s.n_self_wall = s.n_self_body = 1;
  for (int c = 0; c <= pr.M; ++c) {
    int start = c == 0 ? 0 : pr.nout + (c - 1) * pr.n, len = c == 0 ? pr.nout : pr.n;
    const int csz = c == 0 ? SELF_CHUNK : SELF_CHUNK_BODY;
    int nch = (len + csz - 1) / csz;
    if (c == 0) s.n_self_wall = nch;
    else s.n_self_body = nch;
    s.n_self_slots = std::max(s.n_self_slots, nch);
    for (int ch = 0; ch < nch; ++ch)
      for (int o = 0; o < len; o += 256) st.push_back(make_int4(start + o, std::min(256, len - o), c, ch));
  }
  s.n_self_tasks = (int)st.size();
  h2d(s.self_tasks.ensure(st.size()), st.data(), st.size(), s.st);
  // pairs of distinct curves, less the near-masked ones (counted per launch)
  long long same = (long long)pr.nout * (pr.nout - 1) + (long long)pr.M * pr.n * (pr.n - 1);
  long long masked = 0, masked_wall = 0;
  for (int q = 0; q < s.near.nsrc; ++q) {
    int c = s.near.h_src_curve[q];
    long long m = (long long)(s.near.h_src_ptr[q + 1] - s.near.h_src_ptr[q]) * (c == 0 ? pr.nout : pr.n);
    masked += m;
    if (c == 0) masked_wall += m;
  }
  s.far64_pairs = (long long)pr.N * (pr.N - 1) - same - masked;
  s.farw_pairs = (long long)pr.nout * (pr.N - pr.nout) - masked_wall;
  s.far32_pairs = s.far64_pairs - s.farw_pairs;
  EB_CK(cudaStreamSynchronize(s.st));
}

// ---------------------------------------------------------------------------
// Far-field launch shapes and their autotuner.

static int shape_targets(int kind, int shape) {
  const FarShape sh = far_shape_of(kind, shape);
  return sh.nt * sh.tpt;
}

static_assert(kFar64Shapes[0].nt == 256 && kFar64Shapes[0].tpt == 2 && kFar64Shapes[0].rcp == 1 &&
              kFar64Shapes[1].nt == 128 && kFar64Shapes[1].tpt == 4 && kFar64Shapes[1].rcp == 1 &&
              kFar64Shapes[2].nt == 256 && kFar64Shapes[2].tpt == 2 && kFar64Shapes[2].rcp == 3 &&
              kFar64Shapes[3].nt == 128 && kFar64Shapes[3].tpt == 4 && kFar64Shapes[3].rcp == 3,
              "launch_far's FP64 cases");
static_assert(kFar64FastShapes[0].nt == 256 && kFar64FastShapes[0].tpt == 2 && kFar64FastShapes[0].rcp == 2 &&
              kFar64FastShapes[1].nt == 128 && kFar64FastShapes[1].tpt == 4 && kFar64FastShapes[1].rcp == 2 &&
              kFar64FastShapes[2].nt == 256 && kFar64FastShapes[2].tpt == 2 && kFar64FastShapes[2].rcp == 4 &&
              kFar64FastShapes[3].nt == 128 && kFar64FastShapes[3].tpt == 4 && kFar64FastShapes[3].rcp == 4,
              "launch_far's fast FP64 cases");
static_assert(kFar32Shapes[0].nt == 256 && kFar32Shapes[0].tpt == 4 && kFar32Shapes[0].rcp == 2 &&
                  kFar32Shapes[0].minb == 2 &&
              kFar32Shapes[1].nt == 256 && kFar32Shapes[1].tpt == 4 && kFar32Shapes[1].rcp == 4 &&
                  kFar32Shapes[1].minb == 2 &&
              kFar32Shapes[2].nt == 256 && kFar32Shapes[2].tpt == 4 && kFar32Shapes[2].rcp == 2 &&
                  kFar32Shapes[2].minb == 3 &&
              kFar32Shapes[3].nt == 256 && kFar32Shapes[3].tpt == 4 && kFar32Shapes[3].rcp == 4 &&
                  kFar32Shapes[3].minb == 3,
              "launch_far's FP32 cases");

// One far-field launch of the given kind (0 accurate FP64 and 2 fast FP64 on
// sq64, 1 FP32 on sq32) and shape over the tile splits sp[0..nsplit], into
// out[split * N + i].
static void launch_far(State& s, int kind, int shape, const int* sp, int nsplit, double2* out) {
  const Problem& pr = s.pr;
  const Near& nr = s.near;
  const GeoDev G = s.geo();
  cudaStream_t st = s.st;
  const bool mk = nr.npairs > 0;
  const dim3 g((unsigned)nblk(pr.N, shape_targets(kind, shape)), (unsigned)nsplit);
#define EB_FAR32(IDX, NT, TPT, U, MB)                                                                           \
  case IDX:                                                                                                       \
    if (mk)                                                                                                       \
      k_far32<true, NT, TPT, U, MB><<<g, NT, 0, st>>>(pr.N, pr.nout, pr.n, s.src32.p, s.tgt32.p, s.anchor.p,        \
                                                   s.tile_c.p, s.sq32.p, s.tiles.p, sp, nr.mask.p, nr.mw, out);  \
    else                                                                                                          \
      k_far32<false, NT, TPT, U, MB><<<g, NT, 0, st>>>(pr.N, pr.nout, pr.n, s.src32.p, s.tgt32.p, s.anchor.p,       \
                                                    s.tile_c.p, s.sq32.p, s.tiles.p, sp, nullptr, 0, out);     \
    break;
#define EB_FAR64(IDX, NT, TPT, RCP)                                                                          \
  case IDX:                                                                                                  \
    if (mk)                                                                                                  \
      k_far64<true, NT, TPT, RCP><<<g, NT, 0, st>>>(G, s.sq64.p, s.tiles.p, sp, nr.mask.p, nr.mw, out);     \
    else                                                                                                     \
      k_far64<false, NT, TPT, RCP><<<g, NT, 0, st>>>(G, s.sq64.p, s.tiles.p, sp, nullptr, 0, out);          \
    break;
  if (kind == 1) {
    switch (shape) {
      EB_FAR32(0, 256, 4, 2, 2)
      EB_FAR32(1, 256, 4, 4, 2)
      EB_FAR32(2, 256, 4, 2, 3)
      EB_FAR32(3, 256, 4, 4, 3)
      default: throw Error(EROSION_BAD_INPUT, "unknown FP32 far-field shape");
    }
  } else if (kind == 0) {
    switch (shape) {
      EB_FAR64(0, 256, 2, 1)
      EB_FAR64(1, 128, 4, 1)
      EB_FAR64(2, 256, 2, 3)
      EB_FAR64(3, 128, 4, 3)
      default: throw Error(EROSION_BAD_INPUT, "unknown FP64 far-field shape");
    }
  } else {
    switch (shape) {
      EB_FAR64(0, 256, 2, 2)
      EB_FAR64(1, 128, 4, 2)
      EB_FAR64(2, 256, 2, 4)
      EB_FAR64(3, 128, 4, 4)
      default: throw Error(EROSION_BAD_INPUT, "unknown fast FP64 far-field shape");
    }
  }
#undef EB_FAR32
#undef EB_FAR64
  EB_LAUNCH_CHECK();
}

// The FP32 far-field kernel (the shape in use, no near mask) on the source
// tensors sq over the tile splits sp[0..nsplit]: the preconditioner's
// wall-to-body coupling, a far-field sum with the wall tiles as the only
// sources.
static void launch_far32_unmasked(State& s, const float4* sq, const int* sp, int nsplit, double2* out) {
  const Problem& pr = s.pr;
  cudaStream_t st = s.st;
  const int shape = s.far_shape[1];
  const dim3 g((unsigned)nblk(pr.N, shape_targets(1, shape)), (unsigned)nsplit);
#define EB_FAR32U(IDX, NT, TPT, U, MB)                                                                       \
  case IDX:                                                                                                 \
    k_far32<false, NT, TPT, U, MB><<<g, NT, 0, st>>>(pr.N, pr.nout, pr.n, s.src32.p, s.tgt32.p, s.anchor.p,  \
                                                  s.tile_c.p, sq, s.tiles.p, sp, nullptr, 0, out);        \
    break;
  switch (shape) {
    EB_FAR32U(0, 256, 4, 2, 2)
    EB_FAR32U(1, 256, 4, 4, 2)
    EB_FAR32U(2, 256, 4, 2, 3)
    EB_FAR32U(3, 256, 4, 4, 3)
    default: throw Error(EROSION_BAD_INPUT, "unknown FP32 far-field shape");
  }
#undef EB_FAR32U
  EB_LAUNCH_CHECK();
}

// Resident CTAs per SM of one far-field kernel instance (the occupancy the
// split count is sized for); 0 when the runtime cannot tell.
static int far_resident(int kind, int shape, bool masked) {
  const void* fn = nullptr;
  int nt = 0;
#define EB_R32(IDX, NT, TPT, U, MB)                                                                      \
  case IDX:                                                                                             \
    fn = masked ? (const void*)k_far32<true, NT, TPT, U, MB> : (const void*)k_far32<false, NT, TPT, U, MB>; \
    nt = NT;                                                                                            \
    break;
#define EB_R64(IDX, NT, TPT, RCP)                                                                        \
  case IDX:                                                                                             \
    fn = masked ? (const void*)k_far64<true, NT, TPT, RCP> : (const void*)k_far64<false, NT, TPT, RCP>; \
    nt = NT;                                                                                            \
    break;
  if (kind == 1) {
    switch (shape) { EB_R32(0, 256, 4, 2, 2) EB_R32(1, 256, 4, 4, 2) EB_R32(2, 256, 4, 2, 3) EB_R32(3, 256, 4, 4, 3) default: break; }
  } else if (kind == 0) {
    switch (shape) { EB_R64(0, 256, 2, 1) EB_R64(1, 128, 4, 1) EB_R64(2, 256, 2, 3) EB_R64(3, 128, 4, 3) default: break; }
  } else {
    switch (shape) { EB_R64(0, 256, 2, 2) EB_R64(1, 128, 4, 2) EB_R64(2, 256, 2, 4) EB_R64(3, 128, 4, 4) default: break; }
  }
#undef EB_R32
#undef EB_R64
  if (!fn) return 0;
  int r = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&r, fn, nt, 0) != cudaSuccess) {
    (void)cudaGetLastError();
    return 0;
  }
  return r;
}

// Problems below this many node pairs keep the first shape of each list (a
// launch is a few microseconds; timing would cost more than it saves).
constexpr double kTuneMinPairs = 2e8;

// Chooses the launch shape of each far-field kernel for the current tiles.
// A forced shape wins; otherwise, for large problems, every candidate is timed
// (one warm-up and two timed launches on zeroed strengths, CUDA events on the
// library stream) and the fastest kept.  The choice is cached per problem size
// (N, tile count, masking), so an erosion run tunes once until a body is
// deleted.  Kinds 0 and 2 (accurate and fast FP64) sum every tile; kind 1
// (FP32) the body tiles, and the mixed operator adds the wall tiles in the
// kind-0 shape.
static void plan_far(State& s) {
  const Problem& pr = s.pr;
  // the FP32 kernel sums the body tiles; the wall's tiles (first nwall_tiles)
  // always run in FP64 (their densities carry fields that cancel against the
  // bodies' to a few parts in 1e4, beyond FP32's reach)
  const int t32 = s.nwall_tiles, n32 = s.ntile - s.nwall_tiles;
  const int masked = s.near.npairs > 0;
  int maxs = s.nsplit, max32 = 0, maxw = 0;
  for (int kind = 0; kind < kFarKinds; ++kind)
    for (int sh = 0; sh < far_num_shapes(kind); ++sh) {
      const int res = far_resident(kind, sh, masked);
      if (kind == 1) {
        if (n32 > 0) max32 = std::max(max32, far_split_count(pr.N, n32, shape_targets(1, sh), res));
      } else {
        maxs = std::max(maxs, far_split_count(pr.N, s.ntile, shape_targets(kind, sh), res));
        maxw = std::max(maxw, far_split_count(pr.N, s.nwall_tiles, shape_targets(kind, sh), res));
      }
    }
  s.partial.ensure((size_t)std::max(maxs, max32 + maxw) * pr.N);
  const bool tune = (double)pr.N * (double)pr.N >= kTuneMinPairs;
  const bool cached = s.tune_N == pr.N && s.tune_ntile == s.ntile && s.tune_masked == masked;
  bool zeroed = false;
  for (int kind = 0; kind < kFarKinds; ++kind) {
    const int nsh = far_num_shapes(kind);
    const int tb = kind == 1 ? t32 : 0, tcount = kind == 1 ? n32 : s.ntile;
    if (tcount == 0) { s.nsplit32 = 0; s.far_shape[kind] = 0; continue; }
    int best = 0;
    if (s.force_shape[kind] >= 0) {
      best = s.force_shape[kind];
    } else if (tune && cached && s.tuned_shape[kind] >= 0) {
      best = s.tuned_shape[kind];
    } else if (tune) {
      if (!zeroed) {
        EB_CK(cudaMemsetAsync(s.sq32.p, 0, sizeof(float4) * pr.N, s.st));
        EB_CK(cudaMemsetAsync(s.sq64.p, 0, sizeof(double4) * pr.N, s.st));
        zeroed = true;
      }
      float bestms = 1e30f;
      for (int sh = 0; sh < nsh; ++sh) {
        const int ns = far_split_count(pr.N, tcount, shape_targets(kind, sh), far_resident(kind, sh, masked));
        upload_splits(s, s.split_tune, ns, tb, tb + tcount);
        launch_far(s, kind, sh, s.split_tune.p, ns, s.partial.p);
        float ms = 1e30f;
        for (int r = 0; r < 2; ++r) {
          EB_CK(cudaEventRecord(s.et0, s.st));
          launch_far(s, kind, sh, s.split_tune.p, ns, s.partial.p);
          EB_CK(cudaEventRecord(s.et1, s.st));
          EB_CK(cudaEventSynchronize(s.et1));
          float t = 0;
          EB_CK(cudaEventElapsedTime(&t, s.et0, s.et1));
          ms = std::min(ms, t);
        }
        s.tune_ms[kind][sh] = ms;
        if (ms < bestms) { bestms = ms; best = sh; }
      }
      s.tuned_shape[kind] = best;
    }
    s.far_shape[kind] = best;
    const int ns = far_split_count(pr.N, tcount, shape_targets(kind, best), far_resident(kind, best, masked));
    if (kind == 1) { s.nsplit32 = ns; upload_splits(s, s.split_ptr32, ns, tb, tb + tcount); }
    else if (kind == 0) { s.nsplit64t = ns; upload_splits(s, s.split_ptr64t, ns, 0, s.ntile); }
    else { s.nsplit64f = ns; upload_splits(s, s.split_ptr64f, ns, 0, s.ntile); }
  }
  // the wall-source FP64 launch of the mixed operator, in the FP64 shape
  // (the fast FP64 kind when allowed: these pairs need ~1e-9, not FP64 rounding)
  const int wk = pr.P.fast_fp64 ? 2 : 0;
  s.nsplitw = far_split_count(pr.N, s.nwall_tiles, shape_targets(wk, s.far_shape[wk]),
                              far_resident(wk, s.far_shape[wk], masked));
  upload_splits(s, s.split_ptrw, s.nsplitw, 0, s.nwall_tiles);
  if (tune) { s.tune_N = pr.N; s.tune_ntile = s.ntile; s.tune_masked = masked; }
}

void setup_problem(State& s, const Problem& in, const double* d_xx, const double* d_yy) {
  const auto t_start = std::chrono::steady_clock::now();
  Problem pr = in;
  if (pr.nout < 8 || (pr.nout & 1)) throw Error(EROSION_BAD_INPUT, "nouter must be even and >= 8");
  if (pr.M < 0) throw Error(EROSION_BAD_INPUT, "nbods must be >= 0");
  if (pr.M > 0 && (pr.n < 4 || (pr.n & 1))) throw Error(EROSION_BAD_INPUT, "npts must be even and >= 4");
  if (pr.M == 0) pr.n = std::max(pr.n, 2);
  if (!(pr.P.wall_a > 0 && pr.P.wall_b > 0 && pr.P.wall_order > 0))
    throw Error(EROSION_BAD_INPUT, "wall semi-axes and order must be positive");
  if ((long long)pr.nout + (long long)pr.n * pr.M > (1LL << 30)) throw Error(EROSION_BAD_INPUT, "too many nodes");
  pr.N = pr.nout + pr.n * pr.M;
  pr.ntot = 2LL * pr.N + 3LL * pr.M;
  s.pr = pr;
  s.geo_valid = false;
  cudaStream_t st = s.st;
  if (s.dker_wall_n != pr.nout) {
    auto d = spectral_kernel(pr.nout);
    h2d(s.dker_wall.ensure(pr.nout), d.data(), pr.nout, st);
    EB_CK(cudaStreamSynchronize(st));
    s.dker_wall_n = pr.nout;
  }
  if (pr.M > 0 && s.dker_body_n != pr.n) {
    auto d = spectral_kernel(pr.n);
    h2d(s.dker_body.ensure(pr.n), d.data(), pr.n, st);
    EB_CK(cudaStreamSynchronize(st));
    s.dker_body_n = pr.n;
  }
  const int N = pr.N;
  s.wx.ensure(pr.nout); s.wy.ensure(pr.nout);
  s.xy.ensure(N); s.nrm.ensure(N); s.dz.ensure(N); s.d1tmp.ensure(N);
  s.sp.ensure(N); s.cur.ensure(N); s.w.ensure(N);
  s.cen.ensure(std::max(pr.M, 1)); s.rb.ensure(std::max(pr.M, 1));
  s.ws.ensure(N); s.sq64.ensure(N); s.sigdotn.ensure(1);
  k_wall_nodes<<<nblk(pr.nout, 256), 256, 0, st>>>(pr.nout, pr.P.wall_a, pr.P.wall_b, pr.P.wall_order, s.wx.p, s.wy.p);
  EB_LAUNCH_CHECK();
  k_geom<<<1, 1024, 0, st>>>(s.wx.p, s.wy.p, pr.nout, s.dker_wall.p, 0, 1, s.xy.p, s.nrm.p, s.sp.p, s.cur.p, s.w.p,
                             s.dz.p, s.d1tmp.p);
  EB_LAUNCH_CHECK();
  if (pr.M > 0) {
    k_geom<<<pr.M, 256, 0, st>>>(d_xx, d_yy, pr.n, s.dker_body.p, pr.nout, 0, s.xy.p, s.nrm.p, s.sp.p, s.cur.p,
                                 s.w.p, s.dz.p, s.d1tmp.p + pr.nout);
    EB_LAUNCH_CHECK();
    k_body_stats<<<pr.M, 256, 0, st>>>(pr.n, pr.nout, s.xy.p, s.sp.p, s.cen.p, s.rb.p);
    EB_LAUNCH_CHECK();
  }
  std::vector<double2> hxy(N), hcen(pr.M);
  std::vector<double> hsp(pr.nout), hrb(pr.M);
  d2h(hxy.data(), s.xy.p, N, st);
  d2h(hsp.data(), s.sp.p, pr.nout, st);
  d2h(hcen.data(), s.cen.p, pr.M, st);
  d2h(hrb.data(), s.rb.p, pr.M, st);
  EB_CK(cudaStreamSynchronize(st));
  for (int g = 0; g < N; ++g)
    if (!std::isfinite(hxy[g].x) || !std::isfinite(hxy[g].y)) throw Error(EROSION_BAD_INPUT, "non-finite node coordinates");
  for (int k = 0; k < pr.nout; ++k)
    if (!(hsp[k] > 0) || !std::isfinite(hsp[k])) throw Error(EROSION_BAD_INPUT, "degenerate wall geometry");
  // Every body node must lie strictly inside the superellipse wall.
  for (int g = pr.nout; g < N; ++g) {
    double fx = std::pow(std::fabs(hxy[g].x) / pr.P.wall_a, pr.P.wall_order);
    double fy = std::pow(std::fabs(hxy[g].y) / pr.P.wall_b, pr.P.wall_order);
    if (!(fx + fy < 1.0)) throw Error(EROSION_BAD_INPUT, "a body node lies on or outside the wall");
  }
  build_near(s, hxy, hsp, hcen, hrb);
  build_tiles(s);
  s.src32.ensure(N);
  s.sq32.ensure(N);
  s.tgt32.ensure(N);
  s.anchor.ensure(N);
  s.selfsum.ensure((size_t)s.n_self_slots * N);
  s.tile_c.ensure(s.ntile);
  k_geom32<<<s.ntile, 256, 0, st>>>(s.ntile, s.tiles.p, s.xy.p, s.nrm.p, s.tile_c.p, s.src32.p, s.tgt32.p,
                                     s.anchor.p);
  EB_LAUNCH_CHECK();
  harvest_far_timing(s);
  plan_far(s);
  setup_preconditioner(s);
  s.geo_valid = true;
  s.setup_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  record_setup_stats(s);
}

void record_setup_stats(State& s) {
  s.stats.precond_active = s.pc_active ? 1 : 0;
  s.stats.precond_singular_blocks = s.pc_singular;
  s.stats.ms_setup = s.setup_ms;
  s.stats.ms_precond_setup = s.pc_setup_ms;
}

// The wall's own state (no bodies): its operator is the wall block A_ww of
// the full operator (wall sources at wall targets with the rank-one term).
static State& wall_state() {
  static State w;
  return w;
}

// Wall part of a candidate density given its bodies: c_wall += A_ww^{-1} r_wall
// for the residual r = b - A c of the full problem.  The body and wall
// densities carry fields that cancel against each other, so a body-only
// update of a density (the learned increment) is useless without the wall's
// answer to it (measured with the oracle on a 10-body channel: the exact body
// increment without the wall's raised the residual 25-fold; with the wall
// rows solved for, it lowered it 28-fold).  A_ww = -1/2 I + D_ww + the
// rank-one term is well conditioned (condition ~40 at 1024 wall nodes):
// plain FP64 GMRES to 1e-6 takes a few tens of iterations of an N_out^2 sum.
static void solve_wall_rows(State& s, const double* d_r, double* d_c) {
  State& w = wall_state();
  ensure_init(w);
  const Problem& pr = s.pr;
  const long long nw = 2LL * pr.nout;
  const bool same = w.geo_valid && w.pr.nout == pr.nout && w.pr.P.wall_a == pr.P.wall_a &&
                    w.pr.P.wall_b == pr.P.wall_b && w.pr.P.wall_order == pr.P.wall_order &&
                    w.pr.P.ibary == pr.P.ibary && w.pr.P.ifmm == pr.P.ifmm;
  EB_CK(cudaStreamSynchronize(s.st));   // r is complete before the wall state's stream reads it
  if (!same) {
    Problem pw = pr;
    pw.M = 0;
    pw.n = 2;
    pw.P.precision = 0;
    pw.P.precond = 0;
    pw.P.learned_guess = 0;
    pw.P.true_residual = 0;
    setup_problem(w, pw, w.d_xx.ensure(1), w.d_yy.ensure(1));
  }
  double* rb = w.d_rhs.ensure(nw);
  double* dx = w.d_den.ensure(nw);
  EB_CK(cudaMemcpyAsync(rb, d_r, nw * sizeof(double), cudaMemcpyDeviceToDevice, w.st));
  EB_CK(cudaMemsetAsync(dx, 0, nw * sizeof(double), w.st));
  long long it = 0;
  double est = 0;
  int rc = EROSION_OK;
  try {
    rc = gmres_solve(w, rb, dx, true, 200, 1e-6, &it, &est);
  } catch (const Error& e) {
    if (e.code != EROSION_BAD_INPUT) throw;   // a zero wall residual: nothing to add
    return;
  }
  if (rc == EROSION_BREAKDOWN) return;   // leave the candidate's wall part as it is
  k_axpy<<<nblk(nw, 256), 256, 0, w.st>>>(1.0, dx, d_c, nw);
  EB_LAUNCH_CHECK();
  EB_CK(cudaStreamSynchronize(w.st));
}

bool choose_initial_guess(State& s, const double* d_b, double* d_x, bool have_x, bool learned, const float* d_hist) {
  for (int q = 0; q < 3; ++q) s.stats.guess_residual[q] = -1.0;
  s.stats.guess_residual[0] = 1.0;
  const long long N = s.pr.ntot;
  cudaStream_t st = s.st;
  if (!learned) {
    s.stats.guess_used = have_x ? 1 : 0;
    return !have_x;
  }
  const double bnrm = device_norm(s, d_b, N);
  if (!(bnrm > 0)) { s.stats.guess_used = have_x ? 1 : 0; return !have_x; }
  double* r = s.d_r.ensure(N);
  auto rel_res = [&](const double* x) {
    apply_operator(s, x, r, 0);
    k_bminus<<<nblk(N, 256), 256, 0, st>>>(d_b, r, N);
    EB_LAUNCH_CHECK();
    return device_norm(s, r, N) / bnrm;
  };
  double best = 1.0;
  int used = 0;
  if (have_x) {
    const double rx = rel_res(d_x);
    s.stats.guess_residual[1] = rx;
    if (rx < best) { best = rx; used = 1; }
  }
  static DBuf<double> cand;
  double* c = cand.ensure(N);
  if (have_x) EB_CK(cudaMemcpyAsync(c, d_x, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
  if (have_x && lw_guess_increment(s, d_hist, c)) {
    // the network predicts the bodies' increment only: the wall's part
    // follows from the wall rows given the new body densities
    rel_res(c);
    solve_wall_rows(s, r, c);
    const double rl = rel_res(c);
    s.stats.guess_residual[2] = rl;
    if (rl < best) {
      best = rl;
      used = 2;
      EB_CK(cudaMemcpyAsync(d_x, c, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
    }
  }
  if (used == 0) EB_CK(cudaMemsetAsync(d_x, 0, N * sizeof(double), st));
  EB_CK(cudaStreamSynchronize(st));
  s.stats.guess_used = used;
  return used == 0;
}

// In-place inversion of count m x m FP32 matrices (one CTA each), a zero
// pivot flagged in bad[matrix].  Blocked Gauss-Jordan with the widest panel
// whose shared-memory working set (2 m pb + m floats, m ints) fits; the
// unblocked kernel past that.
static void invert_fp32(State& s, float* B, int m, int count, int* bad) {
  int pb = 32;
  auto gj_smem = [m](int b) { return (2 * (size_t)m * b + m) * sizeof(float) + (size_t)m * sizeof(int); };
  while (pb > 4 && gj_smem(pb) > 200 * 1024) pb /= 2;
  if (gj_smem(pb) <= 200 * 1024) {
    const size_t smem = gj_smem(pb);
    if (smem > 48 * 1024) allow_max_dynamic_smem((const void*)k_gj_inv32_blocked);
    k_gj_inv32_blocked<<<count, 512, smem, s.st>>>(m, pb, B, bad);
    EB_LAUNCH_CHECK();
  } else {
    const size_t smem = 3 * (size_t)m * sizeof(float);
    if (smem > 48 * 1024) allow_max_dynamic_smem((const void*)k_gj_inv32);
    k_gj_inv32<<<count, 1024, smem, s.st>>>(m, B, bad);
    EB_LAUNCH_CHECK();
  }
}

// The coarse correction of precond = 2 (kernels.cuh, k_cg_*): the constraint
// rows' 3 x 3 inverses and the inverse of the rigid moments of the
// completion fields, for the current geometry.  cg_ready is false when that
// matrix had a zero pivot (the block preconditioner then runs alone).
static void setup_coarse(State& s) {
  const Problem& pr = s.pr;
  s.cg_ready = false;
  if (pr.P.precond != 2 || pr.M == 0) return;
  const GeoDev G = s.geo();
  const int m3 = 3 * pr.M;
  k_cg_constraints<<<pr.M, 256, 0, s.st>>>(G, s.cg_Cinv.ensure(9LL * pr.M));
  EB_LAUNCH_CHECK();
  float* Bm = s.cg_B.ensure((size_t)m3 * m3);
  k_cg_moments<<<dim3(pr.M, pr.M), 128, 0, s.st>>>(G, Bm);
  EB_LAUNCH_CHECK();
  int* bad = s.cg_bad.ensure(1);
  EB_CK(cudaMemsetAsync(bad, 0, sizeof(int), s.st));
  invert_fp32(s, Bm, m3, 1, bad);
  s.cg_q.ensure(6LL * pr.M);
  s.cg_cs.ensure(3LL * pr.M);
  s.cg_cr.ensure(3LL * pr.M);
  s.pc_u.ensure(pr.ntot);
  int hbad = 0;
  d2h(&hbad, bad, 1, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
  s.cg_ready = hbad == 0;
}

void setup_preconditioner(State& s) {
  const Problem& pr = s.pr;
  s.pc_setup_ms = 0.0;
  if ((pr.P.precond != 1 && pr.P.precond != 2) || pr.M == 0) {
    s.pc_active = false;
    s.pc_singular = 0;
    s.cg_ready = false;
    return;
  }
  const int n = pr.n, m = 2 * n + 3;
  // the wall-to-body coupling runs the FP32 far-field kernel over the wall
  // tiles: its tile splits (whole waves, as the far field's own) and its
  // partial sums, one N-long slot per split
  {
    const int sh = s.far_shape[1];
    s.pc_wsplit = far_split_count(pr.N, s.nwall_tiles, shape_targets(1, sh), far_resident(1, sh, false));
    upload_splits(s, s.pc_split_ptr, s.pc_wsplit, 0, s.nwall_tiles);
    s.pc_tw.ensure((size_t)s.pc_wsplit * pr.N);
    s.pc_sq32.ensure(pr.nout);
  }
  // keep the previous inverses (a lagged preconditioner) when allowed
  if (pr.P.precond_refresh > 1 && s.pc_valid && s.pc_M == pr.M && s.pc_n == n && s.pc_nout == pr.nout &&
      s.pc_age + 1 < pr.P.precond_refresh) {
    s.pc_age++;
    s.pc_active = s.pc_singular < pr.M;
    setup_coarse(s);
    return;
  }
  s.pc_active = false;
  s.pc_singular = 0;
  s.pc_valid = false;
  const GeoDev G = s.geo();
  EB_CK(cudaEventRecord(s.et0, s.st));
  float* B = s.pcB.ensure((size_t)pr.M * m * m);
  k_pc_blocks<<<dim3(pr.M, m), 256, 0, s.st>>>(G, B);
  EB_LAUNCH_CHECK();
  int* bad = s.pc_bad.ensure(pr.M);
  EB_CK(cudaMemsetAsync(bad, 0, sizeof(int) * pr.M, s.st));
  invert_fp32(s, B, m, pr.M, bad);
  // a body whose block had a zero pivot gets the identity (left
  // unpreconditioned); the other bodies keep their inverses
  k_pc_identity_if_bad<<<dim3(pr.M, nblk(m, 8)), 256, 0, s.st>>>(m, bad, B);
  EB_LAUNCH_CHECK();
  EB_CK(cudaEventRecord(s.et1, s.st));
  std::vector<int> hbad(pr.M);
  d2h(hbad.data(), bad, pr.M, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
  {
    float t = 0;
    EB_CK(cudaEventElapsedTime(&t, s.et0, s.et1));
    s.pc_setup_ms = t;
  }
  for (int b = 0; b < pr.M; ++b) s.pc_singular += hbad[b] != 0;
  s.pc_z.ensure(pr.ntot);
  s.pc_u.ensure(pr.ntot);
  setup_coarse(s);
  s.pc_active = s.pc_singular < pr.M;
  s.pc_valid = true;
  s.pc_M = pr.M;
  s.pc_n = n;
  s.pc_nout = pr.nout;
  s.pc_age = 0;
}

static void apply_block_gs(State& s, const double* v, double* z);

// precond = 1: block Gauss-Seidel.  precond = 2: first the coarse problem
// Q^T A Q c = Q^T v (k_cg_*), then block Gauss-Seidel on the rest,
// z = Q c + P (v - A Q c).
void apply_preconditioner(State& s, const double* v, double* z) {
  const Problem& pr = s.pr;
  if (pr.P.precond != 2 || !s.cg_ready) {
    apply_block_gs(s, v, z);
    return;
  }
  const GeoDev G = s.geo();
  double* w = s.pc_u.p;
  EB_CK(cudaMemcpyAsync(w, v, pr.ntot * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  k_cg_restrict<<<pr.M, 256, 0, s.st>>>(G, v, s.cg_q.p);
  EB_LAUNCH_CHECK();
  k_cg_solve_s<<<(unsigned)nblk(3LL * pr.M, 8), 256, 0, s.st>>>(pr.M, s.cg_B.p, s.cg_q.p, s.cg_cs.p);
  EB_LAUNCH_CHECK();
  k_cg_solve_r<<<(unsigned)nblk(pr.M, 128), 128, 0, s.st>>>(G, s.cg_Cinv.p, s.cg_q.p, s.cg_cs.p, s.cg_cr.p, w);
  EB_LAUNCH_CHECK();
  k_cg_field<<<(unsigned)nblk(pr.N, 256), 256, 0, s.st>>>(G, s.cg_cs.p, w);
  EB_LAUNCH_CHECK();
  apply_block_gs(s, w, z);
  k_cg_prolong<<<pr.M, 256, 0, s.st>>>(G, s.cg_cr.p, s.cg_cs.p, z);
  EB_LAUNCH_CHECK();
}

static void apply_block_gs(State& s, const double* v, double* z) {
  const Problem& pr = s.pr;
  const GeoDev G = s.geo();
  const int n = pr.n, m = 2 * n + 3, nb = n * pr.M;
  k_pc_wall<<<nblk(pr.nout, 256), 256, 0, s.st>>>(G, v, z, s.pc_sq32.p);
  EB_LAUNCH_CHECK();
  launch_far32_unmasked(s, s.pc_sq32.p, s.pc_split_ptr.p, s.pc_wsplit, s.pc_tw.p);
  dim3 g(pr.M, (unsigned)std::max(1, (m + 63) / 64));
  k_pc_apply_bodies<<<g, 256, m * sizeof(float), s.st>>>(G, s.pcB.p, v, s.pc_tw.p + pr.nout, pr.N, s.pc_wsplit, z);
  EB_LAUNCH_CHECK();
}

void harvest_far_timing(State& s) {
  float ms = 0;
  if (s.far_pending) {
    EB_CK(cudaEventSynchronize(s.ef1));   // complete already on every path that calls this
    EB_CK(cudaEventElapsedTime(&ms, s.ef0, s.ef1));
    if (s.far_kind == 1) s.stats.ms_far32 += ms;
    else if (s.far_kind == 2) s.stats.ms_far64f += ms;
    else s.stats.ms_far += ms;
    s.far_pending = false;
  }
  if (s.farw_pending) {
    EB_CK(cudaEventSynchronize(s.ew1));
    EB_CK(cudaEventElapsedTime(&ms, s.ew0, s.ew1));
    s.stats.ms_farw += ms;
    s.farw_pending = false;
  }
}

void operator_prep(State& s, const double* d_den, double* d_vel) {
  const Problem& pr = s.pr;
  k_prep<<<pr.M + 1, 256, 0, s.st>>>(s.geo(), d_den, s.ws.p, s.sq64.p, s.sq32.p, d_vel, s.sigdotn.p,
                                      pr.P.ibary == 1);
  EB_LAUNCH_CHECK();
}

int far_slots(const State& s, int prec) {
  return prec == 1 ? s.nsplit32 + s.nsplitw : (prec == 2 ? s.nsplit64f : s.nsplit64t);
}

void operator_post(State& s, const double* d_den, double* d_vel, int nsplit) {
  const Problem& pr = s.pr;
  const GeoDev G = s.geo();
  const Near& nr = s.near;
  cudaStream_t st = s.st;
  k_self64<<<s.n_self_tasks, 256, 0, st>>>(G, s.ws.p, s.self_tasks.p, s.selfsum.p, SELF_CHUNK_BODY);
  EB_LAUNCH_CHECK();
  if (nr.npairs > 0) {
    k_bdval<<<nr.n_bd_work, BD_NT, 0, st>>>(G, d_den, nr.bd_work.p, nr.src_curve.p, nr.bd_off.p, s.dker_wall.p,
                                            s.dker_body.p, s.bd.p);
    EB_LAUNCH_CHECK();
    k_bary_list<<<nr.n_bary_work, NEAR_NT, 0, st>>>(G, nr.bary_work.p, nr.src_curve.p, nr.bd_off.p, s.bd.p,
                                                    nr.pair_tgt.p, s.xy.p, s.pair_out.p);
    EB_LAUNCH_CHECK();
  }
  k_combine<<<nblk((long long)pr.N * COMBINE_G, 256), 256, 0, st>>>(G, d_den, s.partial.p, nsplit, nr.npairs ? nr.tptr.p : nullptr,
                                             nr.npairs ? nr.tpairs.p : nullptr, s.pair_out.p, s.sigdotn.p,
                                             s.selfsum.p, s.n_self_wall, s.n_self_body, d_vel);
  EB_LAUNCH_CHECK();
}

void apply_operator(State& s, const double* d_den, double* d_vel, int prec) {
  harvest_far_timing(s);
  const Problem& pr = s.pr;
  cudaStream_t st = s.st;
  operator_prep(s, d_den, d_vel);
  const int kind = prec == 1 ? 1 : (prec == 2 ? 2 : 0);
  const int n1 = kind == 1 ? s.nsplit32 : (kind == 2 ? s.nsplit64f : s.nsplit64t);
  if (n1 > 0) {
    EB_CK(cudaEventRecord(s.ef0, st));
    launch_far(s, kind, s.far_shape[kind],
               kind == 1 ? s.split_ptr32.p : (kind == 2 ? s.split_ptr64f.p : s.split_ptr64t.p), n1, s.partial.p);
    EB_CK(cudaEventRecord(s.ef1, st));
    s.far_kind = kind;
    s.far_pending = true;
  }
  if (kind == 1) {
    // wall sources in FP64, into the partial slots after the FP32 ones
    EB_CK(cudaEventRecord(s.ew0, st));
    const int wk = pr.P.fast_fp64 ? 2 : 0;
    launch_far(s, wk, s.far_shape[wk], s.split_ptrw.p, s.nsplitw, s.partial.p + (size_t)n1 * pr.N);
    EB_CK(cudaEventRecord(s.ew1, st));
    s.farw_pending = true;
    s.stats.matvecs_fp32++;
    if (s.nsplit32 > 0) s.stats.far32_launches++;
    s.stats.farw_launches++;
  } else if (kind == 2) {
    s.stats.far64f_launches++;
  } else {
    s.stats.far_launches++;
  }
  operator_post(s, d_den, d_vel, far_slots(s, prec));
  s.stats.matvecs++;
  s.stats.far32_pairs = s.far32_pairs;
  s.stats.far64_pairs = s.far64_pairs;
  s.stats.farw_pairs = s.farw_pairs;
}

void build_rhs(State& s, double* d_rhs) {
  const GeoDev G = s.geo();
  k_rhs<<<nblk(std::max(s.pr.N, 3 * s.pr.M), 256), 256, 0, s.st>>>(G, s.pr.P.ibc, s.pr.P.rhs_mode, s.pr.P.wall_b, d_rhs);
  EB_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
// Krylov helpers.
static int dot_blocks(long long n, int* R) {
  int nb = (int)std::min<long long>((long long)g_num_sms * 8, nblk(n, 256));
  nb = std::max(nb, 1);
  *R = (int)((n + nb - 1) / nb);
  nb = (int)((n + *R - 1) / *R);
  return nb;
}

// h[0..k) (+)= V[0..k) . w
static void dots(State& s, const double* V, long long ldv, int k, const double* w, long long n, double* h,
                 int accumulate) {
  int R;
  int nb = dot_blocks(n, &R);
  double* part = s.part.ensure((size_t)k * nb);
  k_dot_part<<<nb, 256, R * sizeof(double), s.st>>>(V, ldv, k, w, n, R, part);
  EB_LAUNCH_CHECK();
  k_dot_reduce<<<nblk(k, 8), 256, 0, s.st>>>(part, nb, k, h, accumulate);
  EB_LAUNCH_CHECK();
}

double device_norm(State& s, const double* d_v, long long n) {
  double* h = s.hdev.ensure(8);
  dots(s, d_v, n, 1, d_v, n, h, 0);
  double r = 0;
  d2h(&r, h, 1, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
  return std::sqrt(r);
}

static double* pinned(State& s, size_t n) {
  if (n > s.h_pinned_cap) {
    if (s.h_pinned) cudaFreeHost(s.h_pinned);
    s.h_pinned = nullptr;
    size_t m = std::max<size_t>(n, 4096);
    EB_CK(cudaMallocHost((void**)&s.h_pinned, m * sizeof(double)));
    s.h_pinned_cap = m;
  }
  return s.h_pinned;
}

// One GMRES run with the semantics of SLATEC DGMRES as solveBIE calls it
// (stokesSolver.f:481-497, gmres_routines.f): no restart, MAXL = min(maxl, N),
// stop when the Givens estimate rho <= abs_tol, least squares by DHELS, x += V y.
// The Arnoldi step is classical Gram-Schmidt applied twice (two passes of
// tall-skinny products instead of DORTH's k sequential dot/axpy pairs).
// d_r holds the initial residual on entry.  Operator precision: FP64, or, when
// relax_abs > 0, FP32 far field once rho <= relax_abs (inexact Krylov: the
// operator error tolerated grows as the residual shrinks).
static int gmres_cycle(State& s, double* d_r, double* d_x, long long maxl_in, double abs_tol, double relax_abs,
                       long long* iters, double* rho_out) {
  const long long N = s.pr.ntot;
  const long long ldv = (N + 31) & ~31LL;
  long long MAXL = maxl_in;
  if (MAXL == 0) MAXL = 10;
  if (MAXL > N) MAXL = N;
  *iters = 0;
  cudaStream_t st = s.st;
  long long cap0 = std::min<long long>(MAXL + 1, 64);
  if ((long long)(s.V.cap / ldv) < cap0) s.V.ensure((size_t)cap0 * ldv);
  s.vcap = (long long)(s.V.cap / ldv);
  s.zcap = (long long)(s.Z.cap / ldv);
  k_copy<<<nblk(N, 256), 256, 0, st>>>(d_r, s.V.p, N);
  EB_LAUNCH_CHECK();
  const double r0nrm = device_norm(s, s.V.p, N);
  *rho_out = r0nrm;
  if (!std::isfinite(r0nrm)) throw Error(EROSION_BREAKDOWN, "non-finite initial residual");
  if (r0nrm <= abs_tol) return EROSION_OK;
  k_scale<<<nblk(N, 256), 256, 0, st>>>(s.V.p, 1.0 / r0nrm, N);
  EB_LAUNCH_CHECK();
  std::vector<std::vector<double>> HES;   // column ll-1 holds HES(1..ll+1, ll)
  std::vector<double> Q;
  double prod = 1.0, rho = r0nrm;
  long long lgmr = 0;
  int iflag = -1;
  double* hdev = s.hdev.ensure((size_t)MAXL + 2);
  double* hs = s.ydev.ensure((size_t)MAXL + 2);
  double* hp = pinned(s, 2 * (size_t)MAXL + 4);
  for (long long ll = 1; ll <= MAXL; ++ll) {
    lgmr = ll;
    if (ll + 1 > s.vcap) {
      long long nc = std::min<long long>(MAXL + 1, std::max<long long>(2 * s.vcap, ll + 1));
      s.V.grow_keep((size_t)nc * ldv, (size_t)ll * ldv, st);
      s.vcap = nc;
    }
    double* V = s.V.p;
    double* vnew = V + ll * ldv;
    // mixed precision: the fast FP64 operator while the residual is large,
    // the FP32 far field once it is below relax_abs
    const int prec = relax_abs > 0.0 ? (rho <= relax_abs ? 1 : (s.pr.P.fast_fp64 ? 2 : 0)) : 0;
    if (s.pc_active) {
      // flexible GMRES: keep z_k = P^{-1} v_k so that x = x0 + Z y is exactly
      // consistent with the Arnoldi relation A Z = V H whatever the
      // preconditioner's rounding
      if (ll > s.zcap) {
        long long nc = std::min<long long>(MAXL, std::max<long long>(2 * s.zcap, std::max<long long>(ll, 64)));
        s.Z.grow_keep((size_t)nc * ldv, (size_t)(ll - 1) * ldv, st);
        s.zcap = nc;
      }
      double* zk = s.Z.p + (ll - 1) * ldv;
      apply_preconditioner(s, V + (ll - 1) * ldv, zk);
      apply_operator(s, zk, vnew, prec);
    } else {
      apply_operator(s, V + (ll - 1) * ldv, vnew, prec);
    }
    const int k = (int)ll;
    dots(s, V, ldv, k, vnew, N, hdev, 0);
    k_vh<<<nblk(N, 256), 256, 0, st>>>(V, ldv, k, hdev, -1.0, vnew, N);
    EB_LAUNCH_CHECK();
    dots(s, V, ldv, k, vnew, N, hs, 0);
    k_vh<<<nblk(N, 256), 256, 0, st>>>(V, ldv, k, hs, -1.0, vnew, N);
    EB_LAUNCH_CHECK();
    dots(s, vnew, N, 1, vnew, N, hdev + k, 0);
    d2h(hp, hdev, (size_t)k + 1, st);
    d2h(hp + MAXL + 2, hs, (size_t)k, st);
    EB_CK(cudaStreamSynchronize(st));
    harvest_far_timing(s);
    const double snormw = std::sqrt(hp[k]);
    std::vector<double> col(ll + 1);
    for (int i = 0; i < k; ++i) col[i] = hp[i] + hp[MAXL + 2 + i];
    col[ll] = snormw;
    bool finite = std::isfinite(snormw);
    for (int i = 0; i < k && finite; ++i) finite = std::isfinite(col[i]);
    if (!finite) { iflag = 3; break; }
    // DHEQR (gmres_routines.f:1148), update of the last column.
    for (long long kk = 1; kk <= ll - 1; ++kk) {
      double c = Q[2 * (kk - 1)], sn = Q[2 * (kk - 1) + 1];
      double t1 = col[kk - 1], t2 = col[kk];
      col[kk - 1] = c * t1 - sn * t2;
      col[kk] = sn * t1 + c * t2;
    }
    double t1 = col[ll - 1], t2 = col[ll], c, sn;
    if (t2 == 0.0) { c = 1; sn = 0; }
    else if (std::fabs(t2) >= std::fabs(t1)) { double t = t1 / t2; sn = -1.0 / std::sqrt(1.0 + t * t); c = -sn * t; }
    else { double t = t2 / t1; c = 1.0 / std::sqrt(1.0 + t * t); sn = -c * t; }
    Q.push_back(c); Q.push_back(sn);
    col[ll - 1] = c * t1 - sn * t2;
    HES.push_back(col);
    if (col[ll - 1] == 0.0) { iflag = 2; break; }
    prod = prod * sn;
    rho = std::fabs(prod * r0nrm);
    if (rho <= abs_tol) { iflag = 0; break; }
    if (ll == MAXL) { iflag = (rho < r0nrm) ? 1 : 2; break; }
    k_scale<<<nblk(N, 256), 256, 0, st>>>(vnew, 1.0 / snormw, N);
    EB_LAUNCH_CHECK();
  }
  *iters = lgmr;
  *rho_out = rho;
  if (iflag == 3) throw Error(EROSION_BREAKDOWN, "non-finite value in the Arnoldi process");
  if (iflag == 2) return EROSION_BREAKDOWN;
  // DHELS (gmres_routines.f:1048) and x += V y.
  const long long L = lgmr;
  std::vector<double> y(L + 1, 0.0);
  y[0] = r0nrm;
  for (long long kk = 1; kk <= L; ++kk) {
    double c = Q[2 * (kk - 1)], sn = Q[2 * (kk - 1) + 1];
    double a1 = y[kk - 1], a2 = y[kk];
    y[kk - 1] = c * a1 - sn * a2;
    y[kk] = sn * a1 + c * a2;
  }
  for (long long kb = 1; kb <= L; ++kb) {
    long long kk = L + 1 - kb;
    y[kk - 1] = y[kk - 1] / HES[kk - 1][kk - 1];
    double t = -y[kk - 1];
    for (long long i = 1; i <= kk - 1; ++i) y[i - 1] += t * HES[kk - 1][i - 1];
  }
  double* yd = s.ydev.ensure((size_t)L + 1);
  h2d(yd, y.data(), (size_t)L, st);
  if (s.pc_active) {   // x += Z y
    k_vh<<<nblk(N, 256), 256, 0, st>>>(s.Z.p, ldv, (int)L, yd, 1.0, d_x, N);
    EB_LAUNCH_CHECK();
  } else {
    k_vh<<<nblk(N, 256), 256, 0, st>>>(s.V.p, ldv, (int)L, yd, 1.0, d_x, N);
    EB_LAUNCH_CHECK();
  }
  EB_CK(cudaStreamSynchronize(st));
  return iflag == 1 ? EROSION_MAXITER : EROSION_OK;
}

// Switch point of the mixed-precision operator when relax_tol is 0: FP32 far
// field once the GMRES residual estimate is below kRelaxFactor * tol (1e-3 at
// tol 1e-8).  erosion_default_params sets relax_tol = 1 with sweep_decades = 5
// instead: on the 400-body channel (block preconditioner, tol 1e-8, cold
// start) that solve takes 776 iterations in 5.28 s, all but 3 far-field sums
// in FP32, against 611 iterations in 6.09 s with 46% of them in FP64 at
// relax_tol = 1e-2, and 601 at 1e-3.
static const double kRelaxFactor = 1e5;

int gmres_solve(State& s, const double* d_b, double* d_x, bool x0_zero, long long maxl, double tol,
                long long* iters, double* est) {
  const long long N = s.pr.ntot;
  cudaStream_t st = s.st;
  *iters = 0;
  const double bnrm = device_norm(s, d_b, N);
  if (bnrm == 0.0) {
    EB_CK(cudaMemsetAsync(d_x, 0, N * sizeof(double), st));
    EB_CK(cudaStreamSynchronize(st));
    *est = 0.0;
    throw Error(EROSION_BAD_INPUT, "zero right-hand side: the zero density was returned");
  }
  double* r = s.d_r.ensure(N);
  auto residual = [&](bool zero) {   // r = b - A x with the FP64 operator
    if (zero) {
      k_copy<<<nblk(N, 256), 256, 0, st>>>(d_b, r, N);
      EB_LAUNCH_CHECK();
    } else {
      apply_operator(s, d_x, r, 0);
      k_bminus<<<nblk(N, 256), 256, 0, st>>>(d_b, r, N);
      EB_LAUNCH_CHECK();
    }
  };
  residual(x0_zero);
  if (s.pr.P.precision == 0 && !s.pc_active) {
    // the reference's algorithm: one unrestarted cycle, stop on the estimate
    long long it = 0;
    double rho = 0;
    int rc = gmres_cycle(s, r, d_x, maxl, tol * bnrm, 0.0, &it, &rho);
    *iters = it;
    *est = rho / bnrm;
    return rc;
  }
  // Mixed precision: relaxed FP32 cycles inside FP64 iterative refinement.
  // The preconditioned FP64 solve takes the same refinement loop with the
  // FP64 operator throughout: with the FP32 preconditioner the flexible
  // Arnoldi relation A Z = V H holds only to the rounding of A z, and the
  // preconditioned vectors z carry the bodies' large rigid modes, so the
  // estimate can fall orders of magnitude below the true residual (measured
  // on the 400-body channel: estimate 1e-11, true residual 1.6e-7); each sweep
  // restarts from the true FP64 residual until it meets tol or its rounding
  // floor.
  long long total = 0;
  double prev_tr = 1e300;
  const bool mixed = s.pr.P.precision != 0;
  double r_start = x0_zero ? bnrm : device_norm(s, r, N);   // residual the sweep starts from
  if (!x0_zero) {   // the supplied (or chosen) guess and its residual
    if (s.stats.guess_used < 1) s.stats.guess_used = 1;
    s.stats.guess_residual[s.stats.guess_used] = r_start / bnrm;
  }
  if (!x0_zero && !(r_start < bnrm)) {
    // An initial guess no better than zero would cost iterations just to get
    // back to ||b||; start from zero instead.
    EB_CK(cudaMemsetAsync(d_x, 0, N * sizeof(double), st));
    residual(true);
    r_start = bnrm;
    s.stats.guess_used = 0;
  }
  const int sd = mixed ? std::max(0, (int)s.pr.P.sweep_decades) : 0;
  for (int sweep = 0; sweep < 6 + 2 * sd; ++sweep) {
    long long it = 0;
    double rho = 0;
    const double relax = s.pr.P.relax_tol > 0 ? s.pr.P.relax_tol : tol * kRelaxFactor;
    // a sweep stops at tol, or sd decades below the residual it started from
    // when that point is more than a decade above tol (a sweep that would
    // stop within a decade of tol runs on to it: another restart would cost
    // more iterations than it saves).  A mixed sweep that runs to tol aims at
    // half of it: its FP32 operator leaves a residual whose shear stress is
    // about twice an FP64 solve's at the same residual (3 circles: 1.7e-7 of
    // max |tau| against 8e-8 with the FP64 solve to 1e-8).
    double cyc_tol = (mixed ? 0.5 : 1.0) * tol * bnrm;
    if (sd > 0 && r_start * std::pow(10.0, -sd) > 10.0 * tol * bnrm) cyc_tol = r_start * std::pow(10.0, -sd);
    int rc = gmres_cycle(s, r, d_x, std::max<long long>(maxl - total, 1), cyc_tol, mixed ? relax * bnrm : 0.0,
                         &it, &rho);
    total += it;
    s.stats.sweeps = sweep + 1;
    if (rc == EROSION_BREAKDOWN) { *iters = total; *est = rho / bnrm; return rc; }
    residual(false);
    const double tr = device_norm(s, r, N) / bnrm;
    s.stats.true_residual = tr;
    s.stats.true_residual_checks += 1;
    if (sweep < 8) { s.stats.sweep_residual[sweep] = tr; s.stats.sweep_iterations[sweep] = it; }
    *est = tr;
    if (!std::isfinite(tr)) throw Error(EROSION_BREAKDOWN, "non-finite true residual");
    if (tr <= tol) { *iters = total; return EROSION_OK; }
    r_start = tr * bnrm;
    // The true residual has a rounding floor ~ eps ||A|| ||x|| / ||b|| that
    // can exceed tol when the densities are large (small bodies: ~1.1e-8 on
    // the 400-body channel, where the FP64 form stops on its estimate with a
    // true residual of ~3e-8).  A refinement sweep whose true residual is
    // within 2 tol, or that does not halve it, has reached that floor.
    if (sweep > 0 && (tr <= 2.0 * tol || tr > 0.5 * prev_tr)) {
      *iters = total;
      s.stats.floor_accepted = 1;
      return EROSION_OK;
    }
    prev_tr = tr;
    if (total >= maxl) { *iters = total; return EROSION_MAXITER; }
  }
  *iters = total;
  return EROSION_MAXITER;
}

// Frees every device buffer a State holds (the next call sets it up again).
void release_state_buffers(State& s) {
  DBuf<double>* dbs[] = {&s.dker_body, &s.dker_wall, &s.wx, &s.wy, &s.sp, &s.cur, &s.w, &s.rb, &s.sigdotn,
                         &s.d_xx, &s.d_yy, &s.d_den, &s.d_rhs, &s.d_r, &s.d_w, &s.V, &s.Z, &s.part, &s.hdev,
                         &s.ydev, &s.pc_z, &s.pc_u};
  for (auto* b : dbs) b->release();
  DBuf<double2>* d2s[] = {&s.xy, &s.nrm, &s.dz, &s.cen, &s.d1tmp, &s.ws, &s.partial, &s.bd, &s.pair_out};
  s.sq64.release();
  for (auto* b : d2s) b->release();
  s.near.src_curve.release(); s.near.pair_tgt.release(); s.near.tptr.release(); s.near.tpairs.release();
  s.near.bd_off.release(); s.near.bd_work.release(); s.near.bary_work.release(); s.near.mask.release();
  s.tiles.release(); s.split_ptr.release();
  s.vcap = 0;
  s.zcap = 0;
  s.pcB.release(); s.pc_tw.release(); s.pc_sq32.release(); s.pc_split_ptr.release(); s.pc_bad.release();
  s.cg_B.release(); s.cg_Cinv.release(); s.cg_q.release(); s.cg_cs.release(); s.cg_cr.release(); s.cg_bad.release();
  s.cg_ready = false;
  s.pc_valid = false;
  s.src32.release(); s.sq32.release(); s.tgt32.release(); s.tile_c.release(); s.anchor.release();
  s.self_tasks.release(); s.selfsum.release(); s.split_ptr32.release(); s.split_ptr64t.release(); s.split_ptrw.release();
  s.split_tune.release(); s.split_ptr64f.release(); s.tune_N = -1;
  for (int k = 0; k < kFarKinds; ++k) s.tuned_shape[k] = -1;
  s.dker_body_n = s.dker_wall_n = -1;
  s.geo_valid = false;
}

}  // namespace eb

// ===========================================================================
// C ABI
using namespace eb;

namespace {

template <class F>
int guarded(F&& f) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  try {
    ensure_init(s);
    int rc = f(s);
    set_status(rc, rc == EROSION_OK ? "" : (rc == EROSION_MAXITER ? "GMRES reached maxl before the tolerance"
                                                            : (rc == EROSION_BREAKDOWN ? "GMRES stalled" : "error")));
    return rc;
  } catch (const Error& e) {
    set_status(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_status(EROSION_CUDA_ERROR, e.what());
    return EROSION_CUDA_ERROR;
  }
}

Problem make_problem(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter) {
  if (npts < 0 || nbods < 0 || nouter < 0 || npts > (1 << 24) || nbods > (1 << 24) || nouter > (1 << 26))
    throw Error(EROSION_BAD_INPUT, "negative or oversized sizes");
  Problem pr;
  if (p) pr.P = *p;
  else erosion_default_params(&pr.P);
  pr.n = (int)npts; pr.M = (int)nbods; pr.nout = (int)nouter;
  return pr;
}

// Copies body nodes to the device and sets the problem up.
void setup_from_host(State& s, const Problem& pr, const double* xx, const double* yy) {
  size_t nb = (size_t)pr.n * pr.M;
  double* dx = s.d_xx.ensure(std::max<size_t>(nb, 1));
  double* dy = s.d_yy.ensure(std::max<size_t>(nb, 1));
  h2d(dx, xx, nb, s.st);
  h2d(dy, yy, nb, s.st);
  setup_problem(s, pr, dx, dy);
}

int solve_device_impl(State& s, double* d_den, bool x0_zero, int64_t* nits) {
  const Problem& pr = s.pr;
  {
    const int64_t gu = s.stats.guess_used;
    double gr[3] = {s.stats.guess_residual[0], s.stats.guess_residual[1], s.stats.guess_residual[2]};
    s.stats = erosion_solve_stats{};
    s.stats.guess_used = gu;
    for (int q = 0; q < 3; ++q) s.stats.guess_residual[q] = gr[q];
    record_setup_stats(s);
  }
  EB_CK(cudaEventRecord(s.e0, s.st));
  double* rhs = s.d_rhs.ensure(pr.ntot);
  build_rhs(s, rhs);
  long long it = 0;
  double est = 0;
  int rc = gmres_solve(s, rhs, d_den, x0_zero, pr.P.maxl, pr.P.tol, &it, &est);
  s.stats.iterations = it;
  if (s.stats.sweeps == 0) s.stats.sweeps = 1;
  s.stats.est_residual = est;
  s.stats.near_pairs = s.near.npairs;
  if (pr.P.true_residual) {
    double* r = s.d_w.ensure(pr.ntot);
    apply_operator(s, d_den, r);
    k_bminus<<<nblk(pr.ntot, 256), 256, 0, s.st>>>(rhs, r, pr.ntot);
    EB_LAUNCH_CHECK();
    s.stats.true_residual = device_norm(s, r, pr.ntot) / device_norm(s, rhs, pr.ntot);
  }
  EB_CK(cudaEventRecord(s.e1, s.st));
  EB_CK(cudaEventSynchronize(s.e1));
  harvest_far_timing(s);
  float ms = 0;
  EB_CK(cudaEventElapsedTime(&ms, s.e0, s.e1));
  s.stats.ms_total = ms;
  if (nits) *nits = it;
  return rc;
}

}  // namespace

extern "C" {

void erosion_default_params(erosion_params* p) {
  std::memset(p, 0, sizeof(*p));
  p->wall_a = 3.0;
  p->wall_b = 1.0;
  p->wall_order = 8.0;
  p->tol = 1e-8;
  p->maxl = 8000;
  p->ibary = 1;
  p->ifmm = 1;
  p->ibc = 1;
  p->precision = 0;
  p->rhs_mode = 0;
  p->true_residual = 0;
  p->fast_fp64 = 1;
  p->sweep_decades = 5;
  p->relax_tol = 1.0;
}

int erosion_last_status(void) { return t_status; }
const char* erosion_last_error(void) { return t_err.c_str(); }

void erosion_get_solve_stats(erosion_solve_stats* out) { *out = state().stats; }

int erosion_solve(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                  const double* yy, double* density, int64_t* nits) {
  return guarded([&](State& s) {
    Problem pr = make_problem(p, npts, nbods, nouter);
    setup_from_host(s, pr, xx, yy);
    const long long ntot = s.pr.ntot;
    double* dd = s.d_den.ensure(ntot);
    h2d(dd, density, ntot, s.st);
    bool zero = true;
    for (long long i = 0; i < ntot && zero; ++i) zero = density[i] == 0.0;
    int rc = EROSION_OK;
    try {
      s.stats = erosion_solve_stats{};
      if (s.pr.P.learned_guess) {
        double* rhs = s.d_rhs.ensure(ntot);
        build_rhs(s, rhs);
        zero = choose_initial_guess(s, rhs, dd, !zero, true);
      }
      rc = solve_device_impl(s, dd, zero, nits);
    } catch (const Error& e) {
      if (e.code == EROSION_BAD_INPUT) {   // zero right-hand side: density zeroed
        d2h(density, dd, ntot, s.st);
        EB_CK(cudaStreamSynchronize(s.st));
      }
      throw;
    }
    d2h(density, dd, ntot, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return rc;
  });
}

int erosion_solve_device(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* d_xx,
                         const double* d_yy, double* d_density, int64_t* nits) {
  return guarded([&](State& s) {
    Problem pr = make_problem(p, npts, nbods, nouter);
    setup_problem(s, pr, d_xx, d_yy);
    return solve_device_impl(s, d_density, false, nits);
  });
}

void stokessolver_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter, const int64_t* ifmm,
                   const int64_t* ibary, const int64_t* ibc, const int64_t* maxl, const double* xx, const double* yy,
                   double* density, int64_t* nits) {
  erosion_params p;
  erosion_default_params(&p);
  p.ifmm = (int32_t)*ifmm;
  p.ibary = (int32_t)*ibary;
  p.ibc = (int32_t)*ibc;
  p.maxl = *maxl;
  int64_t it = 0;
  erosion_solve(&p, *npts, *nbods, *nouter, xx, yy, density, &it);
  *nits = it;
}

int erosion_matvec(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                   const double* yy, const double* density, double* vel) {
  return guarded([&](State& s) {
    Problem pr = make_problem(p, npts, nbods, nouter);
    setup_from_host(s, pr, xx, yy);
    const long long ntot = s.pr.ntot;
    double* dd = s.d_den.ensure(ntot);
    double* dv = s.d_w.ensure(ntot);
    h2d(dd, density, ntot, s.st);
    const int prec = s.pr.P.precision;
    if (prec < 0 || prec > 2) throw Error(EROSION_BAD_INPUT, "precision must be 0, 1 or 2");
    apply_operator(s, dd, dv, prec);
    d2h(vel, dv, ntot, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_rhs(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                const double* yy, double* rhs) {
  return guarded([&](State& s) {
    Problem pr = make_problem(p, npts, nbods, nouter);
    setup_from_host(s, pr, xx, yy);
    double* dr = s.d_rhs.ensure(s.pr.ntot);
    build_rhs(s, dr);
    d2h(rhs, dr, s.pr.ntot, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_geometry(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                     const double* yy, double* px, double* py, double* cur, double* speed, double* cx, double* cy,
                     double* xo, double* yo, double* px0, double* py0, double* cur0, double* speed0) {
  return guarded([&](State& s) {
    Problem pr = make_problem(p, npts, nbods, nouter);
    setup_from_host(s, pr, xx, yy);
    const int N = s.pr.N, nout = s.pr.nout, M = s.pr.M;
    std::vector<double2> hxy(N), hn(N), hc(std::max(M, 1));
    std::vector<double> hs(N), hk(N);
    d2h(hxy.data(), s.xy.p, N, s.st);
    d2h(hn.data(), s.nrm.p, N, s.st);
    d2h(hs.data(), s.sp.p, N, s.st);
    d2h(hk.data(), s.cur.p, N, s.st);
    d2h(hc.data(), s.cen.p, M, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    for (int g = nout; g < N; ++g) {
      int i = g - nout;
      if (px) px[i] = hn[g].x;
      if (py) py[i] = hn[g].y;
      if (cur) cur[i] = hk[g];
      if (speed) speed[i] = hs[g];
    }
    for (int b = 0; b < M; ++b) {
      if (cx) cx[b] = hc[b].x;
      if (cy) cy[b] = hc[b].y;
    }
    for (int g = 0; g < nout; ++g) {
      if (xo) xo[g] = hxy[g].x;
      if (yo) yo[g] = hxy[g].y;
      if (px0) px0[g] = hn[g].x;
      if (py0) py0[g] = hn[g].y;
      if (cur0) cur0[g] = hk[g];
      if (speed0) speed0[g] = hs[g];
    }
    return EROSION_OK;
  });
}

void* erosion_stream(void) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  try {
    ensure_init(s);
  } catch (const Error& e) {
    set_status(e.code, e.what());
    return nullptr;
  }
  return (void*)s.st;
}

int64_t erosion_launch_count(void) { return (int64_t)g_launches.load(); }

int erosion_set_far_shape(int32_t kind, int32_t shape) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  if (kind < 0 || kind >= kFarKinds || shape < -1 || shape >= far_num_shapes(kind)) {
    set_status(EROSION_BAD_INPUT, "unknown far-field kernel kind or shape");
    return EROSION_BAD_INPUT;
  }
  s.force_shape[kind] = shape;
  set_status(EROSION_OK, "");
  return EROSION_OK;
}

int erosion_get_far_shapes(int32_t* shape, int32_t* desc, float* ms, int32_t* num_shapes) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  for (int kind = 0; kind < kFarKinds; ++kind) {
    const int nsh = far_num_shapes(kind);
    if (shape) shape[kind] = s.far_shape[kind];
    if (num_shapes) num_shapes[kind] = nsh;
    for (int i = 0; i < nsh; ++i) {
      const FarShape sh = far_shape_of(kind, i);
      if (desc) {
        desc[12 * kind + 3 * i] = sh.nt;
        desc[12 * kind + 3 * i + 1] = sh.tpt;
        desc[12 * kind + 3 * i + 2] = sh.rcp + 10 * sh.minb;   // FP32: unroll + 10 x resident CTAs
      }
      if (ms) ms[8 * kind + i] = s.tune_ms[kind][i] < 1e29f ? s.tune_ms[kind][i] : 0.f;
    }
  }
  return EROSION_OK;
}

int64_t erosion_near_info(int64_t* lw, int64_t* wall_bodies, int64_t* near_pairs) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  if (lw) *lw = s.near.lw;
  if (wall_bodies)
    for (size_t i = 0; i < s.near.wall_bodies.size(); ++i) wall_bodies[i] = s.near.wall_bodies[i];
  if (near_pairs) *near_pairs = s.near.npairs;
  return (int64_t)s.near.wall_bodies.size();
}

void erosion_release(void) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  release_batch();
  release_state_buffers(s);
  release_state_buffers(wall_state());
}

}  // extern "C"
