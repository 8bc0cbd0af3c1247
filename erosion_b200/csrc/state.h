// Host-side state of the library: device buffers kept between calls, the
// current problem's geometry and near-field bookkeeping, and the status
// channel of the C ABI.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>
#include <cstdint>
#include <algorithm>
#include "erosion_b200.h"
#include "common.cuh"

namespace eb {

extern std::atomic<long long> g_launches;

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define EB_CK(x)                                                                               \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess)                                                                     \
      throw ::eb::Error(EROSION_CUDA_ERROR, std::string(#x) + ": " + cudaGetErrorString(e_));  \
  } while (0)

#define EB_LAUNCH_CHECK()  \
  do {                     \
    ++::eb::g_launches;    \
    EB_CK(cudaGetLastError()); \
  } while (0)

// Grow-only device buffer.
template <class T>
struct DBuf {
  T* p = nullptr;
  size_t cap = 0;
  T* ensure(size_t n) {
    if (n > cap) {
      release();
      size_t m = std::max<size_t>(n, 1);
      EB_CK(cudaMalloc((void**)&p, m * sizeof(T)));
      cap = m;
    }
    return p;
  }
  // Grows keeping the first `keep` elements.
  T* grow_keep(size_t n, size_t keep, cudaStream_t st) {
    if (n <= cap) return p;
    T* q = nullptr;
    EB_CK(cudaMalloc((void**)&q, n * sizeof(T)));
    if (p && keep) EB_CK(cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st));
    EB_CK(cudaStreamSynchronize(st));
    release();
    p = q;
    cap = n;
    return p;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

template <class T>
void h2d(T* d, const T* h, size_t n, cudaStream_t st) {
  if (n) EB_CK(cudaMemcpyAsync(d, h, n * sizeof(T), cudaMemcpyHostToDevice, st));
}
template <class T>
void d2h(T* h, const T* d, size_t n, cudaStream_t st) {
  if (n) EB_CK(cudaMemcpyAsync(h, d, n * sizeof(T), cudaMemcpyDeviceToHost, st));
}

inline unsigned nblk(long long n, int nt) { return (unsigned)((n + nt - 1) / nt); }

struct Problem {
  int n = 0, M = 0, nout = 0, N = 0;
  long long ntot = 0;
  erosion_params P{};
};

// Near-field bookkeeping of one geometry.
struct Near {
  long long lw = 0;
  std::vector<long long> wall_bodies;
  int nsrc = 0;              // source curves with at least one pair
  long long npairs = 0;
  int mw = 0;                // mask words per target
  int n_bd_work = 0, n_bary_work = 0;
  long long bd_total = 0;    // complex entries of the boundary-value buffer
  std::vector<int> h_src_curve, h_src_ptr, h_pair_tgt;
  DBuf<int> src_curve, pair_tgt, tptr, tpairs;
  DBuf<long long> bd_off;
  DBuf<int2> bd_work;
  DBuf<int4> bary_work;
  DBuf<unsigned> mask;
};

struct State {
  std::mutex mu;
  bool init = false;
  int device = -1;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr, ef0 = nullptr, ef1 = nullptr, ew0 = nullptr, ew1 = nullptr;

  Problem pr;
  bool geo_valid = false;

  // spectral derivative kernels
  int dker_body_n = -1, dker_wall_n = -1;
  DBuf<double> dker_body, dker_wall;

  // geometry
  DBuf<double> wx, wy, sp, cur, w, rb;
  DBuf<double2> xy, nrm, dz, cen, d1tmp;

  Near near;

  // far field
  DBuf<int4> tiles;
  DBuf<int> split_ptr, split_ptr32, split_ptr64t, split_ptr64f, split_ptrw, split_tune;
  int nsplit = 0, nsplit32 = 0, nsplit64t = 0, nsplit64f = 0, nsplitw = 0, ntile = 0;
  long long far64_pairs = 0, farw_pairs = 0;   // pairs per full FP64 / wall-source launch
  // far-field launch shapes: index into the candidate lists of kernels.cuh
  // (kind 0 FP64, 1 FP32), chosen by the autotuner or forced by the caller
  // (kind 0 accurate FP64, 1 FP32, 2 fast FP64)
  int far_shape[3] = {0, 0, 0};
  int force_shape[3] = {-1, -1, -1};
  int tuned_shape[3] = {-1, -1, -1};
  int tune_N = -1, tune_ntile = -1, tune_masked = -1;
  float tune_ms[3][8] = {};
  cudaEvent_t et0 = nullptr, et1 = nullptr;
  // mixed precision: FP32 geometry, strengths, self-curve tasks and sums
  DBuf<float4> src32;
  DBuf<float4> sq32;        // FP32 far-field source tensors (pair_tensor32)
  DBuf<float2> tgt32;
  DBuf<double2> tile_c, anchor;
  DBuf<int4> self_tasks;
  int n_self_tasks = 0, n_self_slots = 1, n_self_wall = 1, n_self_body = 1;
  int pc_wsplit = 1;        // wall-tile splits of the preconditioner's coupling sum
  DBuf<double2> selfsum;
  long long far32_pairs = 0;
  // block Gauss-Seidel preconditioner
  bool pc_active = false;
  int nwall_tiles = 0;
  DBuf<float> pcB;          // M inverse blocks of (2n+3)^2
  DBuf<double> pc_z, pc_u;  // scratch vectors
  DBuf<double2> pc_tw;      // A_bw z_wall: pc_wsplit partial sums, N long each (body nodes after the wall's)
  DBuf<float4> pc_sq32;     // wall source tensors of the coupling sum (pair_tensor32 of w z_wall)
  DBuf<int> pc_split_ptr;   // its splits of the wall tiles
  // coarse correction (precond = 2): inverse of the completion fields' rigid
  // moments (3M x 3M, FP32), the constraint rows' 3 x 3 inverses (FP64),
  // coarse coordinates
  DBuf<float> cg_B;
  DBuf<double> cg_Cinv, cg_q, cg_cs, cg_cr;
  DBuf<int> cg_bad;
  bool cg_ready = false;
  DBuf<int> pc_bad;         // per body: 1 when its block had a zero pivot
  int pc_singular = 0;      // bodies left unpreconditioned
  bool pc_valid = false;    // pcB holds inverses of a (pc_M, pc_n) problem
  int pc_M = -1, pc_n = -1, pc_nout = -1, pc_age = 0;   // ... built pc_age set-ups ago
  double pc_setup_ms = 0.0; // device time of block assembly + inversion
  double setup_ms = 0.0;    // host wall time of the last setup_problem
  int far_kind = 0;   // kind of the far launch bracketed by ef0/ef1: 0 FP64, 1 FP32, 2 fast FP64

  // work buffers
  DBuf<double2> ws, partial, bd, pair_out;
  DBuf<double4> sq64;        // FP64 far-field source tensors (pair_tensor64)
  DBuf<double> sigdotn;
  DBuf<double> d_xx, d_yy, d_den, d_rhs, d_r, d_w;

  // Krylov
  DBuf<double> V, Z, part, hdev, ydev;
  long long vcap = 0;   // vectors held by V
  long long zcap = 0;   // vectors held by Z (preconditioned basis, flexible GMRES)
  double* h_pinned = nullptr;
  size_t h_pinned_cap = 0;

  erosion_solve_stats stats{};
  bool farw_pending = false;  // ew0/ew1 bracket a wall-source FP64 launch not yet harvested
  bool far_pending = false;   // ef0/ef1 bracket a far-field launch not yet harvested

  GeoDev geo() const {
    GeoDev G;
    G.n = pr.n; G.M = pr.M; G.nout = pr.nout; G.N = pr.N; G.ntot = pr.ntot;
    G.xy = xy.p; G.nrm = nrm.p; G.sp = sp.p; G.cur = cur.p; G.w = w.p; G.dz = dz.p;
    G.cen = cen.p; G.rb = rb.p;
    return G;
  }
};

State& state();
int eb_num_sms();
// Raises a kernel's dynamic shared-memory cap to the device's opt-in maximum
// (less the kernel's static shared memory).  Every caller sets the same value, so set-ups running concurrently on host
// threads (the ensemble) that need different sizes never lower the cap under
// each other's launches.
void allow_max_dynamic_smem(const void* fn);
// The outcome of the last entry-point call made by the calling thread,
// read back by erosion_last_status / erosion_last_error.  Thread-local, so it
// takes no lock and one thread's call never overwrites another's outcome.
void set_status(int code, const std::string& msg);
void ensure_init(State& s);

// Geometry + near lists + far-field tiles for (xx, yy) already on the device.
void setup_problem(State& s, const Problem& pr, const double* d_xx, const double* d_yy);
// vel = A den, device pointers.  prec 0: FP64 far field; 1: FP32 far field
// between distinct curves + FP64 self-curve sums.
void apply_operator(State& s, const double* d_den, double* d_vel, int prec = 0);
// apply_operator in three parts, for callers that batch the far field of
// several geometries into one launch: k_prep (strengths), then the far field
// into s.partial (far_slots(s, prec) slots), then the self/near sums and the
// assembly.
void operator_prep(State& s, const double* d_den, double* d_vel);
int far_slots(const State& s, int prec);
void operator_post(State& s, const double* d_den, double* d_vel, int nsplit);
void build_rhs(State& s, double* d_rhs);
// GMRES (SLATEC DGMRES semantics, CGS2 Arnoldi); returns EROSION_* status.
int gmres_solve(State& s, const double* d_b, double* d_x, bool x0_zero, long long maxl, double tol,
                long long* iters, double* est);
// Initial guess selection: candidates zero, the supplied d_x (have_x: the
// previous step's density) and, with learned and have_x, that density plus
// the network's predicted increment (d_hist: the encoded previous
// increment, or null); d_x receives the one with the smallest FP64
// residual.  Returns true when that is the zero vector.
bool choose_initial_guess(State& s, const double* d_b, double* d_x, bool have_x, bool learned,
                          const float* d_hist = nullptr);
// Adds the learned density increment of every body to d_den (the previous
// step's density; wall untouched), given the encoding of the previous
// increment d_hist (nbods x lw_out_width(), or null); false when no trained
// network exists.
bool lw_guess_increment(State& s, const float* d_hist, double* d_den);
// The learned part's density encoding (lw_out_width() floats per body) of
// d_den on the current geometry.
void lw_encode_current(State& s, const double* d_den, float* d_out);
int lw_out_width();
// Builds (or disables) the block preconditioner for the current geometry.
void setup_preconditioner(State& s);
// Copies the last set-up's figures (time, preconditioner state) into s.stats.
void record_setup_stats(State& s);
// z = P^{-1} v (device vectors of length ntot).
void apply_preconditioner(State& s, const double* v, double* z);
double device_norm(State& s, const double* d_v, long long n);
// Adds the last far-field launch's event time to stats.ms_far (after a sync).
void harvest_far_timing(State& s);

void release_state_buffers(State& s);
// Frees the ensemble solver's members (batch.cu).
void release_batch();

// Shear stress / targets (stress.cu)
void shear_stress(State& s, const double* d_den, double* d_tau, double* d_E);
// Pressure on the body boundaries (computePressure).
void body_pressure(State& s, const double* d_den, double* d_p);
void qoi_targets(State& s, const double* d_den, long long ntar, const double* d_xt, const double* d_yt,
                 double* d_u, double* d_v, double* d_p, double* d_w);

}  // namespace eb
