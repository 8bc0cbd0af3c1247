// Erosion time step in theta-L form on the device: getxy (ThetaLen.jl:92-101),
// the spectral helpers of SpectralMethods.jl:10-67 as circulant convolutions,
// getstress! (DensityStress.jl:23-36), getderivs (TimeStepping.jl:63-95),
// delete_indices (:103-126), timestep! (:130-185) and rungekutta2 (:189-202).
//
// Every spectral helper is a Fourier multiplier m(k) applied to a real,
// n-periodic sequence; for even n it equals the circulant convolution with
// c[j] = Re((1/n) sum_k m(k) e^{2 pi i j k/n}), k over the kvec modes of
// SpectralMethods.jl:15-23:
//   specdiff  m = i k            (Nyquist zeroed)
//   specint   m = 1/(i k)        (k = 0 and Nyquist zeroed)
//   expsmooth m = exp(-f k^2)    (Nyquist kept with |k| = n/2)
#include "state.h"
#include "kernels.cuh"
#include <cmath>
#include <cstring>

// The kernels share the translation unit's anonymous namespace with
// kernels.cuh (internal linkage).
namespace {

constexpr int TL_NT = 256;

__device__ __forceinline__ double alpha_of(int j, int n) {
  const double d = EB_TWOPI / n;
  return 0.5 * d + d * j;   // getalpha, ThetaLen.jl:113-116
}

// y_j = sum_l c[(j - l) mod n] f_l, for the n values of one body, f and c in
// shared memory.
__device__ __forceinline__ double circ(const double* __restrict__ c, const double* __restrict__ f, int j, int n) {
  double a = 0.0;
  for (int l = 0; l < n; ++l) {
    int m = j - l;
    if (m < 0) m += n;
    a = fma(c[m], f[l], a);
  }
  return a;
}

// getxy: x = specint(L/2pi (cos th - mean cos th)) + xsm, same for y.
__global__ void __launch_bounds__(TL_NT)
k_tl_getxy(int n, const double* __restrict__ th, const double* __restrict__ len, const double* __restrict__ xsm,
           const double* __restrict__ ysm, const double* __restrict__ iker, double* __restrict__ xx,
           double* __restrict__ yy, int* __restrict__ flag) {
  extern __shared__ double sm[];
  __shared__ double red[32];
  double* dx = sm;
  double* dy = sm + n;
  double* ik = sm + 2 * n;
  const int b = blockIdx.x;
  const double* t = th + (size_t)b * n;
  double mc = 0, ms = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    mc += cos(t[j]);
    ms += sin(t[j]);
    ik[j] = iker[j];
  }
  mc = block_sum<TL_NT>(mc, red) / n;
  ms = block_sum<TL_NT>(ms, red) / n;
  const double L = len[b];
  if (threadIdx.x == 0 && !(L > 0.0)) atomicOr(flag, 1);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    dx[j] = L / EB_TWOPI * (cos(t[j]) - mc);
    dy[j] = L / EB_TWOPI * (sin(t[j]) - ms);
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    xx[(size_t)b * n + j] = circ(ik, dx, j, n) + xsm[b];
    yy[(size_t)b * n + j] = circ(ik, dy, j, n) + ysm[b];
  }
}

// getstress!: atau = gaussfilter(|tau|, sigma) per body, matau = mean(atau).
__global__ void __launch_bounds__(TL_NT)
k_tl_atau(int n, const double* __restrict__ tau, const double* __restrict__ gker, double* __restrict__ atau,
          double* __restrict__ matau) {
  extern __shared__ double sm[];
  __shared__ double red[32];
  double* f = sm;
  double* c = sm + n;
  const int b = blockIdx.x;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    f[j] = fabs(tau[(size_t)b * n + j]);
    c[j] = gker[j];
  }
  __syncthreads();
  double s = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double a = circ(c, f, j, n);
    atau[(size_t)b * n + j] = a;
    s += a;
  }
  s = block_sum<TL_NT>(s, red);
  if (threadIdx.x == 0) matau[b] = s / n;
}

// d = x - d (the density increment over the previous step), in place.
__global__ void k_lw_delta(long long n, const double* __restrict__ x, double* __restrict__ d) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < n) d[i] = x[i] - d[i];
}

// Warm start across a change of geometry: the previous solve's density,
// with each body's rigid part carried to the new nodes.  Per body (one
// block), on the old nodes: t1, t2 = the node means of the two components,
// t3 = the rotation coefficient about the node mean (xc, yc) (least squares
// on (-(y - yc), x - xc)); the remainder sigma - rigid stays attached to the
// node index and the rigid part is evaluated at the new nodes about their
// own mean.  A rigid-motion density is in the null space of the body's
// double-layer block, so its size (~6e5 for the smallest bodies of a dense
// packing) is set by the stokeslet/rotlet rows alone, while the nodes slide
// along the curves between solves (the theta-L update keeps them at equal
// arclength): index-aligned, that rigid part leaves a residual of ~1e3 ||b||
// (200 bodies); carried to the new nodes, 2e-2 ||b|| (10 bodies, dt 1e-5) to
// 0.3 ||b|| (200 bodies, dt 2e-6).  Nodes are at equal arclength, so
// node means are arclength means.  Wall and stokeslet/rotlet entries are
// copied unchanged.
__global__ void __launch_bounds__(TL_NT)
k_warm_reanchor(int n, int nout, const double* __restrict__ xo, const double* __restrict__ yo,
                const double* __restrict__ xn, const double* __restrict__ yn, const double* __restrict__ den_old,
                double* __restrict__ den_new) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  const size_t nodes = (size_t)b * n;
  const size_t off = 2 * (size_t)nout + 2 * (size_t)n * b;
  const double* sx = den_old + off;
  const double* sy = sx + n;
  double mx = 0, my = 0, mxn = 0, myn = 0, ax = 0, ay = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    mx += xo[nodes + j]; my += yo[nodes + j];
    mxn += xn[nodes + j]; myn += yn[nodes + j];
    ax += sx[j]; ay += sy[j];
  }
  mx = block_sum<TL_NT>(mx, red) / n;
  my = block_sum<TL_NT>(my, red) / n;
  mxn = block_sum<TL_NT>(mxn, red) / n;
  myn = block_sum<TL_NT>(myn, red) / n;
  const double t1 = block_sum<TL_NT>(ax, red) / n;
  const double t2 = block_sum<TL_NT>(ay, red) / n;
  double num = 0, den = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double fx = -(yo[nodes + j] - my), fy = xo[nodes + j] - mx;
    num += fx * sx[j] + fy * sy[j];
    den += fx * fx + fy * fy;
  }
  num = block_sum<TL_NT>(num, red);
  den = block_sum<TL_NT>(den, red);
  const double t3 = den > 0.0 ? num / den : 0.0;
  double* ox = den_new + off;
  double* oy = ox + n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const double fx = -(yo[nodes + j] - my), fy = xo[nodes + j] - mx;
    const double gx = -(yn[nodes + j] - myn), gy = xn[nodes + j] - mxn;
    ox[j] = sx[j] + t3 * (gx - fx);
    oy[j] = sy[j] + t3 * (gy - fy);
  }
}

// xyrot (DensityStress.jl:40): (x, y) -> (-y, x), in place.
__global__ void k_tl_xyrot(long long nb, double* __restrict__ xx, double* __restrict__ yy) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const double x = xx[i], y = yy[i];
  xx[i] = -y;
  yy[i] = x;
}

// drag (PostProcess.jl:131-162) per body: the pressure and viscous parts
//   pdrag = sum_k p_k n_k ds,  vdrag = sum_k tau_k s_k ds,  ds = L / n,
// with the tangent s = (cos th, sin th), rotated (-sin th, cos th) for the
// rotated flow, and the inward normal n = (-s_y, s_x) of getns
// (PostProcess.jl:23-33).  out[4 b + (0..3)] = pdragx, pdragy, vdragx, vdragy.
__global__ void __launch_bounds__(TL_NT)
k_tl_drag(int n, const double* __restrict__ th, const double* __restrict__ len, const double* __restrict__ press,
          const double* __restrict__ tau, int rotation, double* __restrict__ out) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    const size_t i = (size_t)b * n + j;
    const double c = cos(th[i]), sn = sin(th[i]);
    const double sx = rotation ? -sn : c, sy = rotation ? c : sn;
    const double nx = -sy, ny = sx;
    a0 += press[i] * nx;
    a1 += press[i] * ny;
    a2 += tau[i] * sx;
    a3 += tau[i] * sy;
  }
  const double ds = len[b] / n;
  a0 = block_sum<TL_NT>(a0, red);
  a1 = block_sum<TL_NT>(a1, red);
  a2 = block_sum<TL_NT>(a2, red);
  a3 = block_sum<TL_NT>(a3, red);
  if (threadIdx.x == 0) {
    out[4 * b] = a0 * ds;
    out[4 * b + 1] = a1 * ds;
    out[4 * b + 2] = a2 * ds;
    out[4 * b + 3] = a3 * ds;
  }
}

// getderivs for one body per CTA (TimeStepping.jl:42-83).
__global__ void __launch_bounds__(TL_NT)
k_tl_derivs(int n, const double* __restrict__ th, const double* __restrict__ len, const double* __restrict__ atau,
            const double* __restrict__ matau, double eps, int fixarea, const double* __restrict__ dker,
            const double* __restrict__ iker, double* __restrict__ mterm, double* __restrict__ nterm,
            double* __restrict__ xsd, double* __restrict__ ysd) {
  extern __shared__ double sm[];
  __shared__ double red[32];
  double* u = sm;            // theta - alpha, later dvtang
  double* a = sm + n;        // atau
  double* dk = sm + 2 * n;
  double* ik = sm + 3 * n;
  double* dth = sm + 4 * n;  // dtheta
  double* vn = sm + 5 * n;   // vnorm
  double* vt = sm + 6 * n;   // vtang
  const int b = blockIdx.x;
  const double* t = th + (size_t)b * n;
  const double mt = matau[b];
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    u[j] = t[j] - alpha_of(j, n);
    a[j] = atau[(size_t)b * n + j];
    dk[j] = dker[j];
    ik[j] = iker[j];
  }
  __syncthreads();
  double s = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double d = circ(dk, u, j, n) + 1.0;
    double ae = a[j] - fixarea * mt;
    double v = ae + eps * mt * (d - 1.0);
    dth[j] = d;
    vn[j] = v;
    s += d * v;
  }
  const double mdthvn = block_sum<TL_NT>(s, red) / n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) u[j] = dth[j] * vn[j] - mdthvn;
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) vt[j] = circ(ik, u, j, n);
  __syncthreads();
  const double L = len[b];
  double sx = 0, sy = 0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double datau = circ(dk, a, j, n);
    nterm[(size_t)b * n + j] = EB_TWOPI / L * (datau + dth[j] * vt[j]);
    double c = cos(t[j]), sn = sin(t[j]);
    sx += -vn[j] * sn + vt[j] * c;
    sy += vn[j] * c + vt[j] * sn;
  }
  sx = block_sum<TL_NT>(sx, red);
  sy = block_sum<TL_NT>(sy, red);
  if (threadIdx.x == 0) {
    mterm[b] = -EB_TWOPI * mdthvn;
    xsd[b] = sx / n;
    ysd[b] = sy / n;
  }
}

// expsmooth kernel for factor f into c[0..n): (1/n)(1 + 2 sum_{k<n/2} e^{-f k^2}
// cos(2 pi j k/n) + e^{-f n^2/4} (-1)^j).
__device__ void expsmooth_kernel(int n, double f, const double* __restrict__ cosT, double* c, double* e) {
  const int h = n / 2;
  for (int k = threadIdx.x; k <= h; k += blockDim.x) e[k] = exp(-f * (double)k * (double)k);
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double a = 1.0;
    for (int k = 1; k < h; ++k) a += 2.0 * e[k] * cosT[((long long)j * k) % n];
    a += e[h] * ((j & 1) ? -1.0 : 1.0);
    c[j] = a / n;
  }
  __syncthreads();
}

// timestep! body update (TimeStepping.jl:150-182).
__global__ void __launch_bounds__(TL_NT)
k_tl_advance(int n, const double* __restrict__ th0, const double* __restrict__ len0, const double* __restrict__ xsm0,
             const double* __restrict__ ysm0, const double* __restrict__ mat0, const double* __restrict__ lend,
             const double* __restrict__ matd, const double* __restrict__ mterm, const double* __restrict__ nterm,
             const double* __restrict__ xsd, const double* __restrict__ ysd, double eps, double dt1, double dt2,
             const double* __restrict__ cosT, double* __restrict__ th1, double* __restrict__ len1,
             double* __restrict__ xsm1, double* __restrict__ ysm1, int* __restrict__ flag) {
  extern __shared__ double sm[];
  double* c1 = sm;
  double* c2 = sm + n;
  double* u = sm + 2 * n;
  double* v = sm + 3 * n;
  double* e = sm + 4 * n;   // n/2 + 1
  const int b = blockIdx.x;
  const double L0 = len0[b];
  const double L1 = L0 + dt1 * mterm[b];
  const double z0 = EB_TWOPI / L0 * mat0[b];
  const double zd = EB_TWOPI / lend[b] * matd[b];
  const double fac1 = eps * dt1 * zd;
  const double fac2 = eps * dt2 * (2.0 * zd - z0);
  expsmooth_kernel(n, fac1, cosT, c1, e);
  expsmooth_kernel(n, fac2, cosT, c2, e);
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    u[j] = th0[(size_t)b * n + j] - alpha_of(j, n);
    v[j] = nterm[(size_t)b * n + j];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < n; j += blockDim.x)
    th1[(size_t)b * n + j] = circ(c1, u, j, n) + alpha_of(j, n) + dt1 * circ(c2, v, j, n);
  if (threadIdx.x == 0) {
    if (!(L1 > 0.0)) atomicOr(flag, 2);
    len1[b] = L1;
    xsm1[b] = xsm0[b] + dt1 * xsd[b];
    ysm1[b] = ysm0[b] + dt1 * ysd[b];
  }
}

// dst[b'] = src[map[b']] for per-body arrays of width w.
__global__ void k_tl_gather(int w, int Mnew, const int* __restrict__ map, const double* __restrict__ src,
                            double* __restrict__ dst) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)Mnew * w) return;
  int b = (int)(i / w), k = (int)(i % w);
  dst[i] = src[(long long)map[b] * w + k];
}

__global__ void k_scale_range(double* __restrict__ v, double a, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] *= a;
}

}  // namespace

namespace eb {

// ---------------------------------------------------------------------------
// Host side.

struct TL {
  int n = -1;
  double sigma = -1;
  DBuf<double> iker, cosT, gker;
  // state buffers: 0 = thld0, 1 = thld05, 2 = output
  DBuf<double> th[3], len[3], xsm[3], ysm[3], mat[2];
  DBuf<double> mterm, nterm, xsd, ysd, atau, tau, xx, yy, tmp;
  DBuf<double> den[2], den_prev;
  long long den_ntot[2] = {-1, -1};
  DBuf<double> sx[2], sy[2];   // node coordinates each stage's density was solved on
  long long s_nodes[2] = {-1, -1};
  // the most recent solve (either stage): density and node coordinates, the
  // warm start of the next solve
  DBuf<double> last_den, last_x, last_y;
  long long last_ntot = -1;
  // encoding of the most recent density increment (learned guess input)
  DBuf<float> hist;
  bool hist_valid = false;
  DBuf<int> flag, map;
  erosion_step_stats stats{};
};

static TL& tl() {
  static TL t;
  return t;
}

// Fourier-multiplier kernels for even n (see the header comment of this file).
static void tl_tables(State& s, TL& T, int n, double sigma) {
  const double pi = 4.0 * std::atan(1.0);
  if (T.n != n) {
    std::vector<double> ik(n, 0.0), ct(n);
    for (int j = 0; j < n; ++j) {
      long double a = 0.0L;
      for (int k = 1; k < n / 2; ++k) a += 2.0L * std::sin(2.0L * (long double)pi * j * k / n) / k;
      ik[j] = (double)(a / n);
      ct[j] = std::cos(2.0 * pi * j / n);
    }
    h2d(T.iker.ensure(n), ik.data(), n, s.st);
    h2d(T.cosT.ensure(n), ct.data(), n, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    T.n = n;
    T.sigma = -1;
  }
  if (T.sigma != sigma) {
    std::vector<double> gk(n);
    const double f = 0.5 * sigma * sigma;   // gaussfilter = expsmooth(., sigma^2/2)
    for (int j = 0; j < n; ++j) {
      long double a = 1.0L;
      for (int k = 1; k < n / 2; ++k)
        a += 2.0L * std::exp(-(long double)f * k * k) * std::cos(2.0L * (long double)pi * j * k / n);
      a += std::exp(-(long double)f * (n / 2) * (n / 2)) * ((j & 1) ? -1.0L : 1.0L);
      gk[j] = (double)(a / n);
    }
    h2d(T.gker.ensure(n), gk.data(), n, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    T.sigma = sigma;
  }
}

static void ensure_spectral(State& s, int n) {
  if (s.dker_body_n != n) {
    std::vector<double> d(n, 0.0);
    const double pi = 4.0 * std::atan(1.0);
    for (int m = 1; m < n; ++m) {
      if (2 * m == n) continue;
      double t = pi * m / n;
      d[m] = 0.5 * ((m & 1) ? -1.0 : 1.0) * std::cos(t) / std::sin(t);
    }
    h2d(s.dker_body.ensure(n), d.data(), n, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    s.dker_body_n = n;
  }
}

static float elapsed(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

// getpdrop/getumax (DensityStress.jl:129-167): mean pressure on 13 points of
// the slices x = -2 and x = 2, umax = 4 x0/(pdrop + 1e-4).
static double pressure_rescale(State& s, double* d_den) {
  const double x0 = 2.0;
  const int ny = 13;
  const double dy = 2.0 / ny;
  std::vector<double> hx(2 * ny), hy(2 * ny);
  for (int i = 0; i < ny; ++i) {
    hy[i] = hy[ny + i] = -1.0 + 0.5 * dy + dy * i;
    hx[i] = x0;
    hx[ny + i] = -x0;
  }
  static DBuf<double> buf;
  double* b = buf.ensure(6 * 2 * ny);
  h2d(b, hx.data(), 2 * ny, s.st);
  h2d(b + 2 * ny, hy.data(), 2 * ny, s.st);
  qoi_targets(s, d_den, 2 * ny, b, b + 2 * ny, b + 4 * ny, b + 6 * ny, b + 8 * ny, b + 10 * ny);
  std::vector<double> p(2 * ny);
  d2h(p.data(), b + 8 * ny, 2 * ny, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
  double pp = 0, pm = 0;
  for (int i = 0; i < ny; ++i) { pp += p[i]; pm += p[ny + i]; }
  const double pdrop = pm / ny - pp / ny;
  return 4.0 * x0 / (pdrop + 1e-4);
}

// One stage's derivatives: getderivs(thlenden) with getstress! inside.
static void stage_derivs(State& s, TL& T, const Problem& base, const erosion_step_params& sp, int M, int k,
                         double* th, double* len, double* xsm, double* ysm, double* mat, long long* iters,
                         double* resid, double* ms_solve, double* ms_stress, double* ms_tl) {
  const int n = base.n;
  cudaEvent_t ev[4];
  for (auto& e : ev) EB_CK(cudaEventCreate(&e));
  EB_CK(cudaEventRecord(ev[0], s.st));
  T.xx.ensure((size_t)M * n);
  T.yy.ensure((size_t)M * n);
  size_t smem = 3 * (size_t)n * sizeof(double);
  k_tl_getxy<<<M, TL_NT, smem, s.st>>>(n, th, len, xsm, ysm, T.iker.p, T.xx.p, T.yy.p, T.flag.p);
  EB_LAUNCH_CHECK();
  Problem pr = base;
  pr.M = M;
  setup_problem(s, pr, T.xx.p, T.yy.p);
  T.stats.ms_setup += s.setup_ms;
  T.stats.ms_precond_setup += s.pc_setup_ms;
  T.stats.precond_active[k] = s.pc_active ? 1 : 0;
  T.stats.precond_singular_blocks[k] = s.pc_singular;
  const long long ntot = s.pr.ntot;
  double* den = T.den[k].ensure(ntot);
  const bool have_prev = sp.warm_start && T.last_ntot == ntot;
  if (!have_prev) {
    EB_CK(cudaMemsetAsync(den, 0, ntot * sizeof(double), s.st));
    T.hist_valid = false;
  } else {
    // the most recent solve (half a step back), its bodies' rigid parts
    // carried to this stage's nodes
    EB_CK(cudaMemcpyAsync(den, T.last_den.p, ntot * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
    k_warm_reanchor<<<M, TL_NT, 0, s.st>>>(n, base.nout, T.last_x.p, T.last_y.p, T.xx.p, T.yy.p, T.last_den.p, den);
    EB_LAUNCH_CHECK();
    EB_CK(cudaMemcpyAsync(T.den_prev.ensure(ntot), den, ntot * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  }
  double* rhs = s.d_rhs.ensure(ntot);
  build_rhs(s, rhs);
  const bool zero = choose_initial_guess(s, rhs, den, have_prev, sp.warm_start == 2,
                                         T.hist_valid ? T.hist.p : nullptr);
  long long it = 0;
  double est = 0;
  const long long mv0 = s.stats.matvecs, mv32 = s.stats.matvecs_fp32;
  int rc = gmres_solve(s, rhs, den, zero, s.pr.P.maxl, s.pr.P.tol, &it, &est);
  // the solve may have replaced a guess no better than zero by zero
  T.stats.guess_used[k] = s.stats.guess_used;
  T.stats.guess_residual[k] = s.stats.guess_used > 0 ? s.stats.guess_residual[s.stats.guess_used]
                                                     : (have_prev ? s.stats.guess_residual[1] : 1.0);
  T.stats.matvecs[k] = s.stats.matvecs - mv0;
  T.stats.matvecs_fp32[k] = s.stats.matvecs_fp32 - mv32;
  if (rc == EROSION_BREAKDOWN) throw Error(EROSION_BREAKDOWN, "GMRES stalled inside the time step");
  T.den_ntot[k] = ntot;
  const size_t nbn = (size_t)M * n;
  EB_CK(cudaMemcpyAsync(T.sx[k].ensure(nbn), T.xx.p, nbn * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  EB_CK(cudaMemcpyAsync(T.sy[k].ensure(nbn), T.yy.p, nbn * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  T.s_nodes[k] = (long long)nbn;
  if (sp.warm_start) {
    EB_CK(cudaMemcpyAsync(T.last_den.ensure(ntot), den, ntot * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
    EB_CK(cudaMemcpyAsync(T.last_x.ensure(nbn), T.xx.p, nbn * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
    EB_CK(cudaMemcpyAsync(T.last_y.ensure(nbn), T.yy.p, nbn * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
    T.last_ntot = ntot;
  }
  if (have_prev && sp.warm_start == 2) {
    // encoding of this solve's increment over its warm start: the next
    // solve's network input
    k_lw_delta<<<nblk(ntot, 256), 256, 0, s.st>>>(ntot, den, T.den_prev.p);
    EB_LAUNCH_CHECK();
    lw_encode_current(s, T.den_prev.p, T.hist.ensure((size_t)M * lw_out_width()));
    T.hist_valid = true;
  } else if (sp.warm_start == 2) {
    T.hist_valid = false;
  }
  *iters = it;
  *resid = est;
  EB_CK(cudaEventRecord(ev[1], s.st));
  double* sden = den;
  if (sp.fixpdrop) {
    double umax = pressure_rescale(s, den);
    double* tmp = T.tmp.ensure(ntot);
    EB_CK(cudaMemcpyAsync(tmp, den, ntot * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
    k_scale_range<<<nblk(ntot, 256), 256, 0, s.st>>>(tmp, umax, ntot);
    EB_LAUNCH_CHECK();
    sden = tmp;
  }
  T.tau.ensure((size_t)M * n);
  shear_stress(s, sden, T.tau.p, nullptr);
  EB_CK(cudaEventRecord(ev[2], s.st));
  T.atau.ensure((size_t)M * n);
  k_tl_atau<<<M, TL_NT, 2 * n * sizeof(double), s.st>>>(n, T.tau.p, T.gker.p, T.atau.p, mat);
  EB_LAUNCH_CHECK();
  T.mterm.ensure(M); T.nterm.ensure((size_t)M * n); T.xsd.ensure(M); T.ysd.ensure(M);
  k_tl_derivs<<<M, TL_NT, 7 * n * sizeof(double), s.st>>>(n, th, len, T.atau.p, mat, sp.epsilon, sp.fixarea,
                                                           s.dker_body.p, T.iker.p, T.mterm.p, T.nterm.p, T.xsd.p,
                                                           T.ysd.p);
  EB_LAUNCH_CHECK();
  EB_CK(cudaEventRecord(ev[3], s.st));
  EB_CK(cudaEventSynchronize(ev[3]));
  *ms_solve += elapsed(ev[0], ev[1]);
  *ms_stress += elapsed(ev[1], ev[2]);
  *ms_tl += elapsed(ev[2], ev[3]);
  for (auto& e : ev) cudaEventDestroy(e);
}

// delete_indices (TimeStepping.jl:103-126) and the compaction of every
// per-body array that the step still uses.
static int delete_and_compact(State& s, TL& T, int M, int n, double dt1, const double* len_dev,
                              std::vector<double*>& body_arrays_n, std::vector<double*>& body_arrays_1,
                              std::vector<int>& orig, std::vector<long long>& deleted) {
  std::vector<double> mt(M), ln(M);
  d2h(mt.data(), T.mterm.p, M, s.st);
  d2h(ln.data(), len_dev, M, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
  const double ndts = 1.0, mthresh = 10.0;
  std::vector<int> keep;
  for (int b = 0; b < M; ++b) {
    double minlen = -std::sqrt(2.0) * mt[b] * ndts * dt1;
    if (ln[b] <= minlen || mt[b] > mthresh) deleted.push_back(orig[b]);
    else keep.push_back(b);
  }
  if ((int)keep.size() == M) return M;
  const int Mn = (int)keep.size();
  std::vector<int> neworig(Mn);
  for (int i = 0; i < Mn; ++i) neworig[i] = orig[keep[i]];
  orig.swap(neworig);
  if (Mn == 0) return 0;
  h2d(T.map.ensure(Mn), keep.data(), Mn, s.st);
  double* tmp = T.tmp.ensure((size_t)M * n);
  for (double* a : body_arrays_n) {
    k_tl_gather<<<nblk((long long)Mn * n, 256), 256, 0, s.st>>>(n, Mn, T.map.p, a, tmp);
    EB_LAUNCH_CHECK();
    EB_CK(cudaMemcpyAsync(a, tmp, (size_t)Mn * n * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  }
  for (double* a : body_arrays_1) {
    k_tl_gather<<<nblk(Mn, 256), 256, 0, s.st>>>(1, Mn, T.map.p, a, tmp);
    EB_LAUNCH_CHECK();
    EB_CK(cudaMemcpyAsync(a, tmp, (size_t)Mn * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  }
  EB_CK(cudaStreamSynchronize(s.st));
  T.den_ntot[0] = T.den_ntot[1] = -1;   // body count changed: no warm start
  T.last_ntot = -1;
  T.hist_valid = false;
  return Mn;
}

// rungekutta2 (TimeStepping.jl:189-202) on device state (in place).
static int rk2_device(State& s, const Problem& base, const erosion_step_params& sp, int64_t* nbods, double* th,
                      double* len, double* xsm, double* ysm, double* t, int64_t* deleted_out) {
  TL& T = tl();
  const int n = base.n;
  int M = (int)*nbods;
  if (n < 4 || (n & 1)) throw Error(EROSION_BAD_INPUT, "npts must be even and >= 4");
  if (M <= 0) throw Error(EROSION_BAD_INPUT, "no bodies to erode");
  ensure_spectral(s, n);
  tl_tables(s, T, n, sp.sigma);
  T.flag.ensure(1);
  EB_CK(cudaMemsetAsync(T.flag.p, 0, sizeof(int), s.st));
  for (int q = 0; q < 3; ++q) {
    T.th[q].ensure((size_t)M * n); T.len[q].ensure(M); T.xsm[q].ensure(M); T.ysm[q].ensure(M);
  }
  T.mat[0].ensure(M); T.mat[1].ensure(M);
  T.stats = erosion_step_stats{};
  cudaEvent_t a0, a1;
  EB_CK(cudaEventCreate(&a0));
  EB_CK(cudaEventCreate(&a1));
  EB_CK(cudaEventRecord(a0, s.st));
  // thld0 = the caller's state (copied so that deletions can compact it)
  EB_CK(cudaMemcpyAsync(T.th[0].p, th, (size_t)M * n * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  EB_CK(cudaMemcpyAsync(T.len[0].p, len, M * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  EB_CK(cudaMemcpyAsync(T.xsm[0].p, xsm, M * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  EB_CK(cudaMemcpyAsync(T.ysm[0].p, ysm, M * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
  std::vector<int> orig(M);
  for (int b = 0; b < M; ++b) orig[b] = b;
  std::vector<long long> deleted;
  double ms_solve = 0, ms_stress = 0, ms_tl = 0;
  const double dt = sp.dt;
  auto adv = [&](double dt1, double dt2, int src_d, int M_) {
    k_tl_advance<<<M_, TL_NT, (4 * n + n / 2 + 1) * sizeof(double), s.st>>>(
        n, T.th[0].p, T.len[0].p, T.xsm[0].p, T.ysm[0].p, T.mat[0].p, T.len[src_d].p, T.mat[src_d].p, T.mterm.p,
        T.nterm.p, T.xsd.p, T.ysd.p, sp.epsilon, dt1, dt2, T.cosT.p, T.th[2].p, T.len[2].p, T.xsm[2].p, T.ysm[2].p,
        T.flag.p);
    EB_LAUNCH_CHECK();
  };
  // Stage 1: timestep!(thld0, thld0, dt/2, dt/2)
  long long it = 0;
  double res = 0;
  stage_derivs(s, T, base, sp, M, 0, T.th[0].p, T.len[0].p, T.xsm[0].p, T.ysm[0].p, T.mat[0].p, &it, &res,
               &ms_solve, &ms_stress, &ms_tl);
  T.stats.gmres_iterations[0] = it;
  T.stats.max_residual = res;
  {
    std::vector<double*> an = {T.th[0].p, T.nterm.p}, a1v = {T.len[0].p, T.xsm[0].p, T.ysm[0].p, T.mat[0].p,
                                                              T.mterm.p, T.xsd.p, T.ysd.p};
    M = delete_and_compact(s, T, M, n, 0.5 * dt, T.len[0].p, an, a1v, orig, deleted);
  }
  if (M > 0) {
    adv(0.5 * dt, 0.5 * dt, 0, M);
    // thld05 <- output buffers
    std::swap(T.th[1], T.th[2]); std::swap(T.len[1], T.len[2]);
    std::swap(T.xsm[1], T.xsm[2]); std::swap(T.ysm[1], T.ysm[2]);
    // Stage 2: timestep!(thld0, thld05, dt, dt/2)
    stage_derivs(s, T, base, sp, M, 1, T.th[1].p, T.len[1].p, T.xsm[1].p, T.ysm[1].p, T.mat[1].p, &it, &res,
                 &ms_solve, &ms_stress, &ms_tl);
    T.stats.gmres_iterations[1] = it;
    T.stats.max_residual = std::max(T.stats.max_residual, res);
    std::vector<double*> an = {T.th[0].p, T.th[1].p, T.nterm.p},
                         a1v = {T.len[0].p, T.xsm[0].p, T.ysm[0].p, T.mat[0].p, T.len[1].p, T.xsm[1].p,
                                T.ysm[1].p, T.mat[1].p, T.mterm.p, T.xsd.p, T.ysd.p};
    M = delete_and_compact(s, T, M, n, dt, T.len[0].p, an, a1v, orig, deleted);
    if (M > 0) {
      adv(dt, 0.5 * dt, 1, M);
      EB_CK(cudaMemcpyAsync(th, T.th[2].p, (size_t)M * n * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
      EB_CK(cudaMemcpyAsync(len, T.len[2].p, M * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
      EB_CK(cudaMemcpyAsync(xsm, T.xsm[2].p, M * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
      EB_CK(cudaMemcpyAsync(ysm, T.ysm[2].p, M * sizeof(double), cudaMemcpyDeviceToDevice, s.st));
    }
  }
  EB_CK(cudaEventRecord(a1, s.st));
  EB_CK(cudaEventSynchronize(a1));
  int flag = 0;
  d2h(&flag, T.flag.p, 1, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
  T.stats.ms_total = elapsed(a0, a1);
  T.stats.ms_solve = ms_solve;
  T.stats.ms_stress = ms_stress;
  T.stats.ms_thetalen = T.stats.ms_total - ms_solve - ms_stress;
  T.stats.bodies_deleted = (int64_t)deleted.size();
  {
    std::vector<double> m0(std::max(M, 1));
    if (M > 0) {
      d2h(m0.data(), T.mat[0].p, M, s.st);
      EB_CK(cudaStreamSynchronize(s.st));
      double a = 0;
      for (int b = 0; b < M; ++b) a += m0[b];
      T.stats.matau[0] = a / M;
      d2h(m0.data(), T.mat[1].p, M, s.st);
      EB_CK(cudaStreamSynchronize(s.st));
      a = 0;
      for (int b = 0; b < M; ++b) a += m0[b];
      T.stats.matau[1] = a / M;
    }
  }
  cudaEventDestroy(a0);
  cudaEventDestroy(a1);
  for (size_t i = 0; i < deleted.size(); ++i) deleted_out[i] = deleted[i];
  *nbods = M;
  *t += dt;
  if (flag & 1) throw Error(EROSION_BAD_INPUT, "a body length is not positive (getxy)");
  if (flag & 2) throw Error(EROSION_BREAKDOWN, "a body length became non-positive (timestep!)");
  return EROSION_OK;
}

}  // namespace eb

using namespace eb;

namespace {
template <class F>
int guarded3(F&& f) {
  State& s = state();
  std::lock_guard<std::mutex> lk(s.mu);
  try {
    ensure_init(s);
    int rc = f(s);
    set_status(rc, "");
    return rc;
  } catch (const Error& e) {
    set_status(e.code, e.what());
    return e.code;
  } catch (const std::exception& e) {
    set_status(EROSION_CUDA_ERROR, e.what());
    return EROSION_CUDA_ERROR;
  }
}

Problem base_problem(const erosion_params* p, int64_t npts, int64_t nouter) {
  if (npts <= 0 || nouter <= 0 || npts > (1 << 20) || nouter > (1 << 26)) throw Error(EROSION_BAD_INPUT, "bad sizes");
  Problem pr;
  if (p) pr.P = *p;
  else erosion_default_params(&pr.P);
  pr.n = (int)npts;
  pr.nout = (int)nouter;
  return pr;
}
}  // namespace

extern "C" {

void erosion_default_step_params(erosion_step_params* sp, int64_t npts) {
  std::memset(sp, 0, sizeof(*sp));
  sp->dt = 1e-3;
  sp->epsilon = 15.0 / (double)npts;
  sp->sigma = 10.0 / (double)npts;
  sp->fixarea = 0;
  sp->fixpdrop = 1;
  sp->warm_start = 0;
}

void erosion_get_step_stats(erosion_step_stats* out) { *out = tl().stats; }

int erosion_rk2_step_device(const erosion_params* p, const erosion_step_params* sp, int64_t npts, int64_t* nbods,
                            int64_t nouter, double* d_theta, double* d_len, double* d_xsm, double* d_ysm, double* t,
                            int64_t* deleted) {
  return guarded3([&](State& s) {
    Problem base = base_problem(p, npts, nouter);
    return rk2_device(s, base, *sp, nbods, d_theta, d_len, d_xsm, d_ysm, t, deleted);
  });
}

int erosion_rk2_step(const erosion_params* p, const erosion_step_params* sp, int64_t npts, int64_t* nbods,
                     int64_t nouter, double* theta, double* len, double* xsm, double* ysm, double* t,
                     int64_t* deleted) {
  return guarded3([&](State& s) {
    Problem base = base_problem(p, npts, nouter);
    const int M = (int)*nbods, n = (int)npts;
    if (M <= 0) throw Error(EROSION_BAD_INPUT, "no bodies to erode");
    static DBuf<double> st;
    double* b = st.ensure((size_t)M * n + 3 * (size_t)M);
    h2d(b, theta, (size_t)M * n, s.st);
    h2d(b + (size_t)M * n, len, M, s.st);
    h2d(b + (size_t)M * n + M, xsm, M, s.st);
    h2d(b + (size_t)M * n + 2 * M, ysm, M, s.st);
    int64_t Mo = M;
    int rc = rk2_device(s, base, *sp, &Mo, b, b + (size_t)M * n, b + (size_t)M * n + M, b + (size_t)M * n + 2 * M,
                        t, deleted);
    d2h(theta, b, (size_t)Mo * n, s.st);
    d2h(len, b + (size_t)M * n, Mo, s.st);
    d2h(xsm, b + (size_t)M * n + M, Mo, s.st);
    d2h(ysm, b + (size_t)M * n + 2 * M, Mo, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    *nbods = Mo;
    return rc;
  });
}

int erosion_drag(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* theta,
                 const double* len, const double* xsm, const double* ysm, const double* density, int32_t rotation,
                 double sigma, double* drag, double* drag_bodies, double* tau_all, double* atau_all,
                 double* press_all) {
  return guarded3([&](State& s) {
    const int n = (int)npts, M = (int)nbods;
    if (n < 4 || (n & 1) || M <= 0 || nouter < 8 || (nouter & 1) || nouter > (1 << 26) || n > (1 << 20))
      throw Error(EROSION_BAD_INPUT, "erosion_drag: npts and nouter must be even, nbods > 0");
    if (!theta || !len || !xsm || !ysm || !density || !drag) throw Error(EROSION_BAD_INPUT, "erosion_drag: null array");
    if (!(sigma > 0)) throw Error(EROSION_BAD_INPUT, "erosion_drag: sigma must be positive");
    Problem pr = base_problem(p, npts, nouter);
    pr.M = M;
    pr.P.precond = 0;   // no solve here: skip the preconditioner's set-up
    pr.P.learned_guess = 0;
    TL& T = tl();
    ensure_spectral(s, n);
    tl_tables(s, T, n, sigma);
    T.flag.ensure(1);
    EB_CK(cudaMemsetAsync(T.flag.p, 0, sizeof(int), s.st));
    const size_t nb = (size_t)M * n;
    static DBuf<double> buf;
    double* b = buf.ensure(8 * nb + 8 * (size_t)M + 4);
    double* dth = b;
    double* dl = dth + nb;
    double* dxs = dl + M;
    double* dys = dxs + M;
    double* dx = dys + M;
    double* dy = dx + nb;
    double* dtau = dy + nb;
    double* datau = dtau + nb;
    double* dp = datau + nb;
    double* dmat = dp + nb;
    double* dper = dmat + M;   // 4 M
    h2d(dth, theta, nb, s.st);
    h2d(dl, len, M, s.st);
    h2d(dxs, xsm, M, s.st);
    h2d(dys, ysm, M, s.st);
    k_tl_getxy<<<M, TL_NT, 3 * n * sizeof(double), s.st>>>(n, dth, dl, dxs, dys, T.iker.p, dx, dy, T.flag.p);
    EB_LAUNCH_CHECK();
    if (rotation) {
      k_tl_xyrot<<<nblk((long long)nb, 256), 256, 0, s.st>>>((long long)nb, dx, dy);
      EB_LAUNCH_CHECK();
    }
    setup_problem(s, pr, dx, dy);
    const long long ntot = s.pr.ntot;
    double* dden = T.tmp.ensure(std::max<size_t>(ntot, nb));
    h2d(dden, density, ntot, s.st);
    shear_stress(s, dden, dtau, nullptr);
    body_pressure(s, dden, dp);
    k_tl_atau<<<M, TL_NT, 2 * n * sizeof(double), s.st>>>(n, dtau, T.gker.p, datau, dmat);
    EB_LAUNCH_CHECK();
    k_tl_drag<<<M, TL_NT, 0, s.st>>>(n, dth, dl, dp, dtau, rotation ? 1 : 0, dper);
    EB_LAUNCH_CHECK();
    std::vector<double> per(4 * (size_t)M);
    d2h(per.data(), dper, 4 * (size_t)M, s.st);
    if (tau_all) d2h(tau_all, dtau, nb, s.st);
    if (atau_all) d2h(atau_all, datau, nb, s.st);
    if (press_all) d2h(press_all, dp, nb, s.st);
    int flag = 0;
    d2h(&flag, T.flag.p, 1, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    if (flag) throw Error(EROSION_BAD_INPUT, "erosion_drag: a body length is not positive");
    // totals in body order, as the reference's loop accumulates them
    for (int q = 0; q < 4; ++q) drag[q] = 0.0;
    for (int bb = 0; bb < M; ++bb)
      for (int q = 0; q < 4; ++q) drag[q] += per[4 * (size_t)bb + q];
    if (drag_bodies) std::copy(per.begin(), per.end(), drag_bodies);
    return EROSION_OK;
  });
}

int erosion_get_step_density(int32_t stage, double* density, int64_t capacity) {
  return guarded3([&](State& s) {
    TL& T = tl();
    if (stage < 0 || stage > 1 || !density) throw Error(EROSION_BAD_INPUT, "stage must be 0 or 1");
    const long long n = T.den_ntot[stage];
    if (n <= 0) throw Error(EROSION_BAD_INPUT, "no solved density of that stage since the last body-count change");
    if (capacity < n) throw Error(EROSION_BAD_INPUT, "density capacity below the stage's unknown count");
    d2h(density, T.den[stage].p, n, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_get_step_nodes(int32_t stage, double* xx, double* yy, int64_t capacity) {
  return guarded3([&](State& s) {
    TL& T = tl();
    if (stage < 0 || stage > 1 || !xx || !yy) throw Error(EROSION_BAD_INPUT, "stage must be 0 or 1");
    if (T.den_ntot[stage] <= 0) throw Error(EROSION_BAD_INPUT, "no solve of that stage since the last body-count change");
    const long long nb = T.s_nodes[stage];
    if (capacity < nb) throw Error(EROSION_BAD_INPUT, "node capacity below the stage's node count");
    d2h(xx, T.sx[stage].p, nb, s.st);
    d2h(yy, T.sy[stage].p, nb, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_getxy(int64_t npts, int64_t nbods, const double* theta, const double* len, const double* xsm,
                  const double* ysm, double* xx, double* yy) {
  return guarded3([&](State& s) {
    const int n = (int)npts, M = (int)nbods;
    if (n < 4 || (n & 1) || M < 0) throw Error(EROSION_BAD_INPUT, "npts must be even and >= 4");
    if (M == 0) return EROSION_OK;
    TL& T = tl();
    tl_tables(s, T, n, T.sigma > 0 ? T.sigma : 10.0 / n);
    T.flag.ensure(1);
    EB_CK(cudaMemsetAsync(T.flag.p, 0, sizeof(int), s.st));
    static DBuf<double> buf;
    double* b = buf.ensure((size_t)M * n * 3 + 3 * (size_t)M);
    double* dth = b;
    double* dl = b + (size_t)M * n;
    double* dxs = dl + M;
    double* dys = dxs + M;
    double* dx = dys + M;
    double* dy = dx + (size_t)M * n;
    h2d(dth, theta, (size_t)M * n, s.st);
    h2d(dl, len, M, s.st);
    h2d(dxs, xsm, M, s.st);
    h2d(dys, ysm, M, s.st);
    k_tl_getxy<<<M, TL_NT, 3 * n * sizeof(double), s.st>>>(n, dth, dl, dxs, dys, T.iker.p, dx, dy, T.flag.p);
    EB_LAUNCH_CHECK();
    d2h(xx, dx, (size_t)M * n, s.st);
    d2h(yy, dy, (size_t)M * n, s.st);
    int flag = 0;
    d2h(&flag, T.flag.p, 1, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    if (flag) throw Error(EROSION_BAD_INPUT, "a body length is not positive");
    return EROSION_OK;
  });
}

}  // extern "C"
