// Learned GMRES initial guess.  A small network maps per-body geometry
// features, with the body's density increment over the previous time step,
// to its increment over the current one; the guess is the previous step's
// density plus the predicted increment.  It is trained on densities the
// solver produced and supplies the initial guess of the next solves (GMRES
// still iterates to the same tolerance, and the guess is used only when its
// residual beats the previous step's density).  Everything (features,
// forward, backward, Adam, encoding, decoding) runs in the kernels of this
// file.
//
// Geometry features of body b (LW_GEO = 68), with R_b the mean radius (mean
// speed):
//   32  Fourier modes +-2..+-9 of (z - c_b)/R_b on the offset grid (re, im)
//    4  log R_b, c_y/b, (b - |c_y| - R_b)/R_b, (a - |c_x| - R_b)/R_b
//   32  the 8 nearest bodies: (dx, dy)/R_b, log(R_j/R_b), gap/R_b (clipped)
// Density encoding (LW_OUT = 37): R_b * (modes -8..8 of sigma_x + i sigma_y),
//   (re, im), then lambda_1, lambda_2, xi/R_b^2.  It is linear, so the
//   encoding of an increment is the increment of the encodings.
// Network input (LW_IN = 105): the geometry features, then the encoding of
// the previous step's increment (zero when there is none); output: the
// encoding of the current increment.
// Network: 105 -> 256 -> 256 -> 256 -> 37, GELU on the hidden layers, weights
// stored in BF16 for the forward and backward products (FP32 master copy for
// Adam), FP32 accumulation.  Inputs and targets are standardised with the
// training set's mean and deviation, which are part of the model.
#include "state.h"
#include "kernels.cuh"
#include <cuda_bf16.h>
#include <cmath>
#include <cstring>
#include <random>

namespace {

constexpr int LW_GEO = 68, LW_H = 256, LW_OUT = 37, LW_K = 8, LW_KF = 9, LW_NN = 8;
constexpr int LW_IN = LW_GEO + LW_OUT;
constexpr int LW_LAYERS = 4;
__host__ __device__ constexpr int lw_in(int l) { return l == 0 ? LW_IN : LW_H; }
__host__ __device__ constexpr int lw_out(int l) { return l == LW_LAYERS - 1 ? LW_OUT : LW_H; }

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  const float cdf = 0.5f * (1.f + erff(z * 0.70710678118654752f));
  const float pdf = 0.39894228040143268f * expf(-0.5f * z * z);
  return cdf + z * pdf;
}

// Per-body geometry features into row b of feat (row stride ld), one CTA
// (128 threads) per body.
__global__ void __launch_bounds__(128)
k_lw_features(GeoDev G, double wall_a, double wall_b, float* __restrict__ feat, int ld) {
  __shared__ double re[2 * LW_KF + 1], im[2 * LW_KF + 1];
  const int b = blockIdx.x, n = G.n;
  const double2 c = G.cen[b];
  const double R = G.rb[b];
  float* f = feat + (size_t)b * ld;
  // Fourier modes m = -KF..KF of (z - c)/R: one warp per mode, strided
  for (int mi = threadIdx.x >> 5; mi < 2 * LW_KF + 1; mi += blockDim.x >> 5) {
    const int m = mi - LW_KF;
    double sr = 0, si = 0;
    for (int k = threadIdx.x & 31; k < n; k += 32) {
      const double2 z = G.xy[G.nout + b * n + k];
      const double zx = (z.x - c.x) / R, zy = (z.y - c.y) / R;
      const double th = EB_TWOPI * (k + 0.5) / n;
      double sn, cs;
      sincos(m * th, &sn, &cs);
      sr += zx * cs + zy * sn;   // (zx + i zy) e^{-i m th}
      si += zy * cs - zx * sn;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if ((threadIdx.x & 31) == 0) { re[mi] = sr / n; im[mi] = si / n; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int q = 0;
    for (int m = -LW_KF; m <= LW_KF; ++m) {
      if (m >= -1 && m <= 1) continue;
      f[q++] = (float)re[m + LW_KF];
      f[q++] = (float)im[m + LW_KF];
    }
    f[q++] = (float)log(R);
    f[q++] = (float)(c.y / wall_b);
    f[q++] = (float)fmin(50.0, (wall_b - fabs(c.y) - R) / R);
    f[q++] = (float)fmin(50.0, (wall_a - fabs(c.x) - R) / R);
    // 8 nearest bodies by centroid distance (insertion into a sorted list)
    double bd[LW_NN];
    int bi[LW_NN];
    for (int t = 0; t < LW_NN; ++t) { bd[t] = 1e300; bi[t] = -1; }
    for (int j = 0; j < G.M; ++j) {
      if (j == b) continue;
      const double2 cj = G.cen[j];
      const double d = (cj.x - c.x) * (cj.x - c.x) + (cj.y - c.y) * (cj.y - c.y);
      if (d >= bd[LW_NN - 1]) continue;
      int t = LW_NN - 1;
      while (t > 0 && bd[t - 1] > d) { bd[t] = bd[t - 1]; bi[t] = bi[t - 1]; --t; }
      bd[t] = d;
      bi[t] = j;
    }
    for (int t = 0; t < LW_NN; ++t) {
      if (bi[t] < 0) {
        f[q++] = 0.f; f[q++] = 0.f; f[q++] = 0.f; f[q++] = 50.f;
        continue;
      }
      const double2 cj = G.cen[bi[t]];
      const double Rj = G.rb[bi[t]];
      const double dx = cj.x - c.x, dy = cj.y - c.y;
      f[q++] = (float)(dx / R);
      f[q++] = (float)(dy / R);
      f[q++] = (float)log(Rj / R);
      f[q++] = (float)fmin(50.0, (sqrt(dx * dx + dy * dy) - R - Rj) / R);
    }
  }
}

// Targets from a density (encode) — one CTA per body.
__global__ void __launch_bounds__(128)
k_lw_encode(GeoDev G, const double* __restrict__ den, float* __restrict__ targ) {
  __shared__ double re[2 * LW_K + 1], im[2 * LW_K + 1];
  const int b = blockIdx.x, n = G.n;
  const double R = G.rb[b];
  for (int mi = threadIdx.x >> 5; mi < 2 * LW_K + 1; mi += blockDim.x >> 5) {
    const int m = mi - LW_K;
    double sr = 0, si = 0;
    for (int k = threadIdx.x & 31; k < n; k += 32) {
      const int g = G.nout + b * n + k;
      const double sx = den[ix_of(G, g)], sy = den[iy_of(G, g)];
      const double th = EB_TWOPI * (k + 0.5) / n;
      double sn, cs;
      sincos(m * th, &sn, &cs);
      sr += sx * cs + sy * sn;
      si += sy * cs - sx * sn;
    }
    sr = warp_sum(sr);
    si = warp_sum(si);
    if ((threadIdx.x & 31) == 0) { re[mi] = sr / n; im[mi] = si / n; }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    float* t = targ + (size_t)b * LW_OUT;
    for (int mi = 0; mi < 2 * LW_K + 1; ++mi) {
      t[2 * mi] = (float)(R * re[mi]);
      t[2 * mi + 1] = (float)(R * im[mi]);
    }
    t[34] = (float)den[ic_of(G, b, 0)];
    t[35] = (float)den[ic_of(G, b, 1)];
    t[36] = (float)(den[ic_of(G, b, 2)] / (R * R));
  }
}

// Density from targets (decode) into the unknown vector, or added to it
// (add = 1); wall entries untouched.
__global__ void __launch_bounds__(128)
k_lw_decode(GeoDev G, const float* __restrict__ targ, double* __restrict__ den, int add) {
  const int b = blockIdx.x, n = G.n;
  const double R = G.rb[b];
  const float* t = targ + (size_t)b * LW_OUT;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    const double th = EB_TWOPI * (k + 0.5) / n;
    double sx = 0, sy = 0;
    for (int mi = 0; mi < 2 * LW_K + 1; ++mi) {
      const int m = mi - LW_K;
      double sn, cs;
      sincos(m * th, &sn, &cs);
      const double ar = t[2 * mi] / R, ai = t[2 * mi + 1] / R;
      sx += ar * cs - ai * sn;   // (ar + i ai) e^{i m th}
      sy += ar * sn + ai * cs;
    }
    const int g = G.nout + b * n + k;
    den[ix_of(G, g)] = add ? den[ix_of(G, g)] + sx : sx;
    den[iy_of(G, g)] = add ? den[iy_of(G, g)] + sy : sy;
  }
  if (threadIdx.x == 0) {
    const double l1 = t[34], l2 = t[35], xi = (double)t[36] * R * R;
    den[ic_of(G, b, 0)] = add ? den[ic_of(G, b, 0)] + l1 : l1;
    den[ic_of(G, b, 1)] = add ? den[ic_of(G, b, 1)] + l2 : l2;
    den[ic_of(G, b, 2)] = add ? den[ic_of(G, b, 2)] + xi : xi;
  }
}

// Row b of the network input: column LW_GEO.. of x gets the history hist[b]
// (or zeros).
__global__ void k_lw_put_hist(int M, const float* __restrict__ hist, float* __restrict__ x) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= M * LW_OUT) return;
  const int b = i / LW_OUT, c = i - b * LW_OUT;
  x[(size_t)b * LW_IN + LW_GEO + c] = hist ? hist[i] : 0.f;
}

// ---------------------------------------------------------------------------
// Network kernels.  Activations are row-major [batch][features].

// Y[b][o] = sum_i X[b][i] W[o][i] + bias[o]; Z keeps the pre-activation and
// Y = GELU(Z) when act.  16x16 output tile per CTA, BF16 weights, FP32 sums.
__global__ void __launch_bounds__(256)
k_lw_fwd(int B, int nin, int nout, const float* __restrict__ X, const __nv_bfloat16* __restrict__ W,
         const float* __restrict__ bias, float* __restrict__ Z, float* __restrict__ Y, int act) {
  __shared__ float xs[16][17], wsh[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int row = blockIdx.y * 16 + ty, col = blockIdx.x * 16 + tx;
  float acc = 0.f;
  for (int k0 = 0; k0 < nin; k0 += 16) {
    const int xr = blockIdx.y * 16 + ty, xc = k0 + tx;
    xs[ty][tx] = (xr < B && xc < nin) ? X[(size_t)xr * nin + xc] : 0.f;
    const int wr = blockIdx.x * 16 + ty, wc = k0 + tx;
    wsh[ty][tx] = (wr < nout && wc < nin) ? __bfloat162float(W[(size_t)wr * nin + wc]) : 0.f;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) acc = fmaf(xs[ty][k], wsh[tx][k], acc);
    __syncthreads();
  }
  if (row < B && col < nout) {
    const float z = acc + bias[col];
    Z[(size_t)row * nout + col] = z;
    Y[(size_t)row * nout + col] = act ? gelu(z) : z;
  }
}

// dZ = dY * GELU'(Z) (or dY for the linear output layer), in place in dY.
__global__ void k_lw_act_back(long long n, const float* __restrict__ Z, float* __restrict__ dY, int act) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n && act) dY[i] *= gelu_grad(Z[i]);
}

// dX[b][i] = sum_o dZ[b][o] W[o][i]
__global__ void __launch_bounds__(256)
k_lw_bwd_x(int B, int nin, int nout, const float* __restrict__ dZ, const __nv_bfloat16* __restrict__ W,
           float* __restrict__ dX) {
  __shared__ float zs[16][17], wsh[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int row = blockIdx.y * 16 + ty, col = blockIdx.x * 16 + tx;
  float acc = 0.f;
  for (int k0 = 0; k0 < nout; k0 += 16) {
    const int zr = blockIdx.y * 16 + ty, zc = k0 + tx;
    zs[ty][tx] = (zr < B && zc < nout) ? dZ[(size_t)zr * nout + zc] : 0.f;
    const int wr = k0 + ty, wc = blockIdx.x * 16 + tx;
    wsh[ty][tx] = (wr < nout && wc < nin) ? __bfloat162float(W[(size_t)wr * nin + wc]) : 0.f;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) acc = fmaf(zs[ty][k], wsh[k][tx], acc);
    __syncthreads();
  }
  if (row < B && col < nin) dX[(size_t)row * nin + col] = acc;
}

// dW[o][i] = sum_b dZ[b][o] X[b][i] / B ; db[o] = sum_b dZ[b][o] / B
__global__ void __launch_bounds__(256)
k_lw_bwd_w(int B, int nin, int nout, const float* __restrict__ dZ, const float* __restrict__ X,
           float* __restrict__ dW, float* __restrict__ db) {
  __shared__ float zs[16][17], xs[16][17];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const int o = blockIdx.y * 16 + ty, i = blockIdx.x * 16 + tx;
  float acc = 0.f, accb = 0.f;
  for (int b0 = 0; b0 < B; b0 += 16) {
    const int zb = b0 + tx, zo = blockIdx.y * 16 + ty;
    zs[ty][tx] = (zb < B && zo < nout) ? dZ[(size_t)zb * nout + zo] : 0.f;   // zs[o][b]
    const int xb = b0 + ty, xi = blockIdx.x * 16 + tx;
    xs[ty][tx] = (xb < B && xi < nin) ? X[(size_t)xb * nin + xi] : 0.f;      // xs[b][i]
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      acc = fmaf(zs[ty][k], xs[k][tx], acc);
      accb += zs[ty][k];
    }
    __syncthreads();
  }
  if (o < nout && i < nin) dW[(size_t)o * nin + i] = acc / B;
  if (o < nout && blockIdx.x == 0 && tx == 0) db[o] = accb / B;
}

// loss = mean (Y - T)^2 ; dY = 2 (Y - T)/(B*OUT) * B (the 1/B lives in k_lw_bwd_w)
__global__ void k_lw_loss(long long n, int out, const float* __restrict__ Y, const float* __restrict__ T,
                          float* __restrict__ dY, double* __restrict__ loss) {
  __shared__ double sh[32];
  double s = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float d = Y[i] - T[i];
    dY[i] = 2.f * d / out;
    s += (double)d * d;
  }
  s = block_sum<256>(s, sh);
  if (threadIdx.x == 0) atomicAdd(loss, s);
}

// Adam step on the FP32 master weights; refreshes the BF16 copy.
__global__ void k_lw_adam(long long n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m1,
                          float* __restrict__ m2, __nv_bfloat16* __restrict__ pb, float lr, float b1, float b2,
                          float c1, float c2, float eps) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float a = b1 * m1[i] + (1.f - b1) * gi;
  const float v = b2 * m2[i] + (1.f - b2) * gi * gi;
  m1[i] = a;
  m2[i] = v;
  const float w = p[i] - lr * (a / c1) / (sqrtf(v / c2) + eps);
  p[i] = w;
  if (pb) pb[i] = __float2bfloat16(w);
}

// dst[r][:] = src[idx[r]][:] (mini-batch gather)
__global__ void k_lw_gather(int rows, int w, const long long* __restrict__ idx, const float* __restrict__ src,
                            float* __restrict__ dst) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (long long)rows * w) return;
  const int r = (int)(i / w), c = (int)(i % w);
  dst[i] = src[idx[r] * w + c];
}

__global__ void k_lw_to_bf16(long long n, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) pb[i] = __float2bfloat16(p[i]);
}

// x_std = (x - mean)/sd (in place) or y = y*sd + mean (inverse)
__global__ void k_lw_scale(long long n, int w, float* __restrict__ x, const float* __restrict__ mean,
                           const float* __restrict__ sd, int inverse) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int c = (int)(i % w);
  x[i] = inverse ? x[i] * sd[c] + mean[c] : (x[i] - mean[c]) / sd[c];
}

}  // namespace

namespace eb {

struct LW {
  bool ready = false;
  // parameters: per layer W (out x in) and b (out), FP32 master + BF16 copy
  DBuf<float> P, G, M1, M2;
  DBuf<__nv_bfloat16> Pb;
  long long off_w[LW_LAYERS], off_b[LW_LAYERS], nparam = 0;
  std::vector<float> xmean, xsd, ymean, ysd;
  DBuf<float> d_xmean, d_xsd, d_ymean, d_ysd;
  DBuf<float> act, pre, grad;   // activations per layer
  DBuf<float> xbuf, ybuf;
  DBuf<double> loss;
  long long step = 0;
};
static LW& lw() {
  static LW m;
  return m;
}

static void lw_layout(LW& m) {
  long long o = 0;
  for (int l = 0; l < LW_LAYERS; ++l) {
    m.off_w[l] = o;
    o += (long long)lw_out(l) * lw_in(l);
    m.off_b[l] = o;
    o += lw_out(l);
  }
  m.nparam = o;
}

static void lw_init(State& s, LW& m, unsigned long long seed) {
  lw_layout(m);
  std::vector<float> h(m.nparam, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < LW_LAYERS; ++l) {
    const double sc = std::sqrt(2.0 / lw_in(l));   // He initialisation
    std::normal_distribution<double> nd(0.0, sc);
    for (long long k = 0; k < (long long)lw_out(l) * lw_in(l); ++k) h[m.off_w[l] + k] = (float)nd(rng);
  }
  h2d(m.P.ensure(m.nparam), h.data(), m.nparam, s.st);
  m.G.ensure(m.nparam);
  EB_CK(cudaMemsetAsync(m.M1.ensure(m.nparam), 0, m.nparam * sizeof(float), s.st));
  EB_CK(cudaMemsetAsync(m.M2.ensure(m.nparam), 0, m.nparam * sizeof(float), s.st));
  m.Pb.ensure(m.nparam);
  k_lw_to_bf16<<<nblk(m.nparam, 256), 256, 0, s.st>>>(m.nparam, m.P.p, m.Pb.p);
  EB_LAUNCH_CHECK();
  m.step = 0;
  EB_CK(cudaStreamSynchronize(s.st));
}

// Forward pass of B standardised rows in m.xbuf; activations kept for backward.
static void lw_forward(State& s, LW& m, int B) {
  long long aoff = 0;
  const float* X = m.xbuf.p;
  m.act.ensure((size_t)B * (LW_IN + 3 * LW_H + LW_OUT));
  m.pre.ensure((size_t)B * (3 * LW_H + LW_OUT));
  long long poff = 0;
  // act layout: [x (B*LW_IN)] [h1] [h2] [h3] [y]
  EB_CK(cudaMemcpyAsync(m.act.p, X, (size_t)B * LW_IN * sizeof(float), cudaMemcpyDeviceToDevice, s.st));
  aoff = (long long)B * LW_IN;
  const float* in = m.act.p;
  for (int l = 0; l < LW_LAYERS; ++l) {
    const int ni = lw_in(l), no = lw_out(l);
    float* Y = m.act.p + aoff;
    float* Z = m.pre.p + poff;
    dim3 g(nblk(no, 16), nblk(B, 16));
    k_lw_fwd<<<g, 256, 0, s.st>>>(B, ni, no, in, m.Pb.p + m.off_w[l], m.P.p + m.off_b[l], Z, Y, l < LW_LAYERS - 1);
    EB_LAUNCH_CHECK();
    in = Y;
    aoff += (long long)B * no;
    poff += (long long)B * no;
  }
}

static const float* lw_output(LW& m, int B) { return m.act.p + (long long)B * (LW_IN + 3 * LW_H); }

// Backward pass from dY (B x OUT, in m.grad's tail) into m.G.
static void lw_backward(State& s, LW& m, int B, float* dY) {
  m.grad.ensure((size_t)B * LW_H * 2);
  float* dcur = dY;
  long long aoff_in[LW_LAYERS], poff[LW_LAYERS];
  {
    long long a = 0, p = 0;
    for (int l = 0; l < LW_LAYERS; ++l) {
      aoff_in[l] = a;
      a += (long long)B * lw_in(l);
      poff[l] = p;
      p += (long long)B * lw_out(l);
    }
  }
  float* dbuf[2] = {m.grad.p, m.grad.p + (size_t)B * LW_H};
  for (int l = LW_LAYERS - 1; l >= 0; --l) {
    const int ni = lw_in(l), no = lw_out(l);
    k_lw_act_back<<<nblk((long long)B * no, 256), 256, 0, s.st>>>((long long)B * no, m.pre.p + poff[l], dcur,
                                                                  l < LW_LAYERS - 1);
    EB_LAUNCH_CHECK();
    dim3 gw(nblk(ni, 16), nblk(no, 16));
    k_lw_bwd_w<<<gw, 256, 0, s.st>>>(B, ni, no, dcur, m.act.p + aoff_in[l], m.G.p + m.off_w[l], m.G.p + m.off_b[l]);
    EB_LAUNCH_CHECK();
    if (l > 0) {
      float* dX = dbuf[l & 1];
      dim3 gx(nblk(ni, 16), nblk(B, 16));
      k_lw_bwd_x<<<gx, 256, 0, s.st>>>(B, ni, no, dcur, m.Pb.p + m.off_w[l], dX);
      EB_LAUNCH_CHECK();
      dcur = dX;
    }
  }
}

static void lw_standardise(State& s, LW& m, const float* hx, const float* hy, long long ns) {
  auto stats = [&](const float* a, int w, std::vector<float>& mu, std::vector<float>& sd) {
    mu.assign(w, 0.f);
    sd.assign(w, 1.f);
    for (int c = 0; c < w; ++c) {
      double s1 = 0, s2 = 0;
      for (long long i = 0; i < ns; ++i) { double v = a[i * w + c]; s1 += v; s2 += v * v; }
      double mean = s1 / ns, var = std::max(0.0, s2 / ns - mean * mean);
      mu[c] = (float)mean;
      sd[c] = (float)std::max(std::sqrt(var), 1e-6);
    }
  };
  stats(hx, LW_IN, m.xmean, m.xsd);
  stats(hy, LW_OUT, m.ymean, m.ysd);
  h2d(m.d_xmean.ensure(LW_IN), m.xmean.data(), LW_IN, s.st);
  h2d(m.d_xsd.ensure(LW_IN), m.xsd.data(), LW_IN, s.st);
  h2d(m.d_ymean.ensure(LW_OUT), m.ymean.data(), LW_OUT, s.st);
  h2d(m.d_ysd.ensure(LW_OUT), m.ysd.data(), LW_OUT, s.st);
  EB_CK(cudaStreamSynchronize(s.st));
}

// Predicts the encoded density increment (denormalised) of the M bodies of
// the current geometry into d_out, given the previous increment's encoding
// d_hist (M x LW_OUT, or null: none).
void lw_predict_current(State& s, const float* d_hist, float* d_out, bool* ok) {
  LW& m = lw();
  *ok = m.ready && s.pr.M > 0;
  if (!*ok) return;
  const int M = s.pr.M;
  const GeoDev G = s.geo();
  m.xbuf.ensure((size_t)M * LW_IN);
  k_lw_features<<<M, 128, 0, s.st>>>(G, s.pr.P.wall_a, s.pr.P.wall_b, m.xbuf.p, LW_IN);
  EB_LAUNCH_CHECK();
  k_lw_put_hist<<<nblk((long long)M * LW_OUT, 256), 256, 0, s.st>>>(M, d_hist, m.xbuf.p);
  EB_LAUNCH_CHECK();
  k_lw_scale<<<nblk((long long)M * LW_IN, 256), 256, 0, s.st>>>((long long)M * LW_IN, LW_IN, m.xbuf.p, m.d_xmean.p,
                                                               m.d_xsd.p, 0);
  EB_LAUNCH_CHECK();
  lw_forward(s, m, M);
  EB_CK(cudaMemcpyAsync(d_out, lw_output(m, M), (size_t)M * LW_OUT * sizeof(float), cudaMemcpyDeviceToDevice, s.st));
  k_lw_scale<<<nblk((long long)M * LW_OUT, 256), 256, 0, s.st>>>((long long)M * LW_OUT, LW_OUT, d_out, m.d_ymean.p,
                                                                m.d_ysd.p, 1);
  EB_LAUNCH_CHECK();
}

// Adds the learned density increment of every body to d_den (which holds
// the previous step's density; wall entries untouched).
bool lw_guess_increment(State& s, const float* d_hist, double* d_den) {
  static DBuf<float> out;
  bool ok = false;
  out.ensure((size_t)std::max(1, s.pr.M) * LW_OUT);
  lw_predict_current(s, d_hist, out.p, &ok);
  if (!ok) return false;
  k_lw_decode<<<s.pr.M, 128, 0, s.st>>>(s.geo(), out.p, d_den, 1);
  EB_LAUNCH_CHECK();
  return true;
}

// The encoding (LW_OUT per body) of density d on the current geometry.
void lw_encode_current(State& s, const double* d_den, float* d_out) {
  if (s.pr.M == 0) return;
  k_lw_encode<<<s.pr.M, 128, 0, s.st>>>(s.geo(), d_den, d_out);
  EB_LAUNCH_CHECK();
}

int lw_out_width() { return LW_OUT; }

}  // namespace eb

using namespace eb;

namespace {
template <class F>
int guarded4(F&& f) {
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

void host_geometry(State& s, const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                   const double* yy) {
  if (npts <= 0 || nbods <= 0 || nouter <= 0) throw Error(EROSION_BAD_INPUT, "bad sizes");
  Problem pr;
  if (p) pr.P = *p;
  else erosion_default_params(&pr.P);
  pr.P.precond = 0;
  pr.n = (int)npts; pr.M = (int)nbods; pr.nout = (int)nouter;
  size_t nb = (size_t)pr.n * pr.M;
  h2d(s.d_xx.ensure(nb), xx, nb, s.st);
  h2d(s.d_yy.ensure(nb), yy, nb, s.st);
  setup_problem(s, pr, s.d_xx.p, s.d_yy.p);
}
}  // namespace

extern "C" {

int erosion_lw_features(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                        const double* yy, float* feat) {
  return guarded4([&](State& s) {
    host_geometry(s, p, npts, nbods, nouter, xx, yy);
    static DBuf<float> f;
    f.ensure((size_t)nbods * LW_GEO);
    k_lw_features<<<(unsigned)nbods, 128, 0, s.st>>>(s.geo(), s.pr.P.wall_a, s.pr.P.wall_b, f.p, LW_GEO);
    EB_LAUNCH_CHECK();
    d2h(feat, f.p, (size_t)nbods * LW_GEO, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_lw_encode(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                      const double* yy, const double* density, float* targ) {
  return guarded4([&](State& s) {
    host_geometry(s, p, npts, nbods, nouter, xx, yy);
    double* dd = s.d_den.ensure(s.pr.ntot);
    h2d(dd, density, s.pr.ntot, s.st);
    static DBuf<float> t;
    t.ensure((size_t)nbods * LW_OUT);
    k_lw_encode<<<(unsigned)nbods, 128, 0, s.st>>>(s.geo(), dd, t.p);
    EB_LAUNCH_CHECK();
    d2h(targ, t.p, (size_t)nbods * LW_OUT, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_lw_decode(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                      const double* yy, const float* targ, double* density) {
  return guarded4([&](State& s) {
    host_geometry(s, p, npts, nbods, nouter, xx, yy);
    double* dd = s.d_den.ensure(s.pr.ntot);
    EB_CK(cudaMemsetAsync(dd, 0, s.pr.ntot * sizeof(double), s.st));
    static DBuf<float> t;
    h2d(t.ensure((size_t)nbods * LW_OUT), targ, (size_t)nbods * LW_OUT, s.st);
    k_lw_decode<<<(unsigned)nbods, 128, 0, s.st>>>(s.geo(), t.p, dd, 0);
    EB_LAUNCH_CHECK();
    d2h(density, dd, s.pr.ntot, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_lw_dims(int32_t* geo, int32_t* in, int32_t* out) {
  if (geo) *geo = LW_GEO;
  if (in) *in = LW_IN;
  if (out) *out = LW_OUT;
  return EROSION_OK;
}

int erosion_lw_init(uint64_t seed) {
  return guarded4([&](State& s) {
    LW& m = lw();
    lw_init(s, m, seed);
    m.ready = false;
    return EROSION_OK;
  });
}

int64_t erosion_lw_num_params(void) {
  LW& m = lw();
  if (m.nparam == 0) lw_layout(m);
  return m.nparam;
}

int erosion_lw_get_params(float* out) {
  return guarded4([&](State& s) {
    LW& m = lw();
    if (!m.P.p) throw Error(EROSION_BAD_INPUT, "network not initialised");
    d2h(out, m.P.p, m.nparam, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_lw_set_params(const float* in) {
  return guarded4([&](State& s) {
    LW& m = lw();
    if (!m.P.p) lw_init(s, m, 1);
    h2d(m.P.p, in, m.nparam, s.st);
    k_lw_to_bf16<<<nblk(m.nparam, 256), 256, 0, s.st>>>(m.nparam, m.P.p, m.Pb.p);
    EB_LAUNCH_CHECK();
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

// Loss and gradients of the current weights on raw (unstandardised-by-the-
// library) inputs/targets: the rows are used exactly as given.
int erosion_lw_loss_grad(const float* x, const float* y, int64_t nsamples, double* loss, float* grads) {
  return guarded4([&](State& s) {
    LW& m = lw();
    if (!m.P.p) throw Error(EROSION_BAD_INPUT, "network not initialised");
    const int B = (int)nsamples;
    h2d(m.xbuf.ensure((size_t)B * LW_IN), x, (size_t)B * LW_IN, s.st);
    h2d(m.ybuf.ensure((size_t)B * LW_OUT), y, (size_t)B * LW_OUT, s.st);
    lw_forward(s, m, B);
    static DBuf<float> dY;
    dY.ensure((size_t)B * LW_OUT);
    EB_CK(cudaMemsetAsync(m.loss.ensure(1), 0, sizeof(double), s.st));
    k_lw_loss<<<nblk((long long)B * LW_OUT, 256), 256, 0, s.st>>>((long long)B * LW_OUT, LW_OUT, lw_output(m, B),
                                                                  m.ybuf.p, dY.p, m.loss.p);
    EB_LAUNCH_CHECK();
    lw_backward(s, m, B, dY.p);
    double l = 0;
    d2h(&l, m.loss.p, 1, s.st);
    d2h(grads, m.G.p, m.nparam, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    *loss = l / ((double)B * LW_OUT);
    return EROSION_OK;
  });
}

// Trains on (features, targets) pairs: standardisation from the data, then
// `epochs` passes of mini-batch Adam.  final_loss: mean squared error of the
// standardised targets over the last epoch.
int erosion_lw_train(const float* feat, const float* targ, int64_t nsamples, int64_t epochs, int64_t batch, double lr,
                     uint64_t seed, double* final_loss) {
  return guarded4([&](State& s) {
    LW& m = lw();
    if (nsamples <= 0 || epochs <= 0 || batch <= 0) throw Error(EROSION_BAD_INPUT, "bad training sizes");
    lw_init(s, m, seed);
    lw_standardise(s, m, feat, targ, nsamples);
    static DBuf<float> X, Y, dY;
    const long long ns = nsamples;
    h2d(X.ensure((size_t)ns * LW_IN), feat, (size_t)ns * LW_IN, s.st);
    h2d(Y.ensure((size_t)ns * LW_OUT), targ, (size_t)ns * LW_OUT, s.st);
    k_lw_scale<<<nblk(ns * LW_IN, 256), 256, 0, s.st>>>(ns * LW_IN, LW_IN, X.p, m.d_xmean.p, m.d_xsd.p, 0);
    EB_LAUNCH_CHECK();
    k_lw_scale<<<nblk(ns * LW_OUT, 256), 256, 0, s.st>>>(ns * LW_OUT, LW_OUT, Y.p, m.d_ymean.p, m.d_ysd.p, 0);
    EB_LAUNCH_CHECK();
    const int B = (int)std::min<long long>(batch, ns);
    dY.ensure((size_t)B * LW_OUT);
    m.loss.ensure(1);
    double last = 0;
    std::mt19937_64 rng(seed ^ 0x9e3779b97f4a7c15ULL);
    std::vector<long long> order(ns);
    for (long long i = 0; i < ns; ++i) order[i] = i;
    static DBuf<long long> d_idx;
    d_idx.ensure(ns);
    for (long long ep = 0; ep < epochs; ++ep) {
      std::shuffle(order.begin(), order.end(), rng);
      EB_CK(cudaMemsetAsync(m.loss.p, 0, sizeof(double), s.st));
      h2d(d_idx.p, order.data(), ns, s.st);
      m.xbuf.ensure((size_t)B * LW_IN);
      m.ybuf.ensure((size_t)B * LW_OUT);
      for (long long b0 = 0; b0 + B <= ns; b0 += B) {
        k_lw_gather<<<nblk((long long)B * LW_IN, 256), 256, 0, s.st>>>(B, LW_IN, d_idx.p + b0, X.p, m.xbuf.p);
        EB_LAUNCH_CHECK();
        k_lw_gather<<<nblk((long long)B * LW_OUT, 256), 256, 0, s.st>>>(B, LW_OUT, d_idx.p + b0, Y.p, m.ybuf.p);
        EB_LAUNCH_CHECK();
        lw_forward(s, m, B);
        k_lw_loss<<<nblk((long long)B * LW_OUT, 256), 256, 0, s.st>>>((long long)B * LW_OUT, LW_OUT,
                                                                      lw_output(m, B), m.ybuf.p, dY.p, m.loss.p);
        EB_LAUNCH_CHECK();
        lw_backward(s, m, B, dY.p);
        ++m.step;
        const float b1 = 0.9f, b2 = 0.999f;
        const float c1 = 1.f - std::pow(b1, (float)m.step), c2 = 1.f - std::pow(b2, (float)m.step);
        k_lw_adam<<<nblk(m.nparam, 256), 256, 0, s.st>>>(m.nparam, m.P.p, m.G.p, m.M1.p, m.M2.p, m.Pb.p, (float)lr,
                                                         b1, b2, c1, c2, 1e-8f);
        EB_LAUNCH_CHECK();
      }
      double l = 0;
      d2h(&l, m.loss.p, 1, s.st);
      EB_CK(cudaStreamSynchronize(s.st));
      last = l / ((double)(ns / B) * B * LW_OUT);
    }
    m.ready = true;
    if (final_loss) *final_loss = last;
    return EROSION_OK;
  });
}

// Predicted (denormalised) targets of the trained network for raw features.
int erosion_lw_predict(const float* feat, int64_t nsamples, float* out) {
  return guarded4([&](State& s) {
    LW& m = lw();
    if (!m.ready) throw Error(EROSION_BAD_INPUT, "network not trained");
    const int B = (int)nsamples;
    h2d(m.xbuf.ensure((size_t)B * LW_IN), feat, (size_t)B * LW_IN, s.st);
    k_lw_scale<<<nblk((long long)B * LW_IN, 256), 256, 0, s.st>>>((long long)B * LW_IN, LW_IN, m.xbuf.p,
                                                                  m.d_xmean.p, m.d_xsd.p, 0);
    EB_LAUNCH_CHECK();
    lw_forward(s, m, B);
    static DBuf<float> o;
    o.ensure((size_t)B * LW_OUT);
    EB_CK(cudaMemcpyAsync(o.p, lw_output(m, B), (size_t)B * LW_OUT * sizeof(float), cudaMemcpyDeviceToDevice, s.st));
    k_lw_scale<<<nblk((long long)B * LW_OUT, 256), 256, 0, s.st>>>((long long)B * LW_OUT, LW_OUT, o.p, m.d_ymean.p,
                                                                  m.d_ysd.p, 1);
    EB_LAUNCH_CHECK();
    d2h(out, o.p, (size_t)B * LW_OUT, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

}  // extern "C"
