// Device kernels of the boundary operator, its geometry and the Krylov
// solver.  Launch wrappers live in solver.cu.
#pragma once
#include "common.cuh"

// Internal linkage: the translation units that include this header each get
// their own copy of the kernels they launch.
namespace {

// Problem-wide constants of the far-field kernels.
constexpr int FAR_NT = 256;        // CTA shape (threads x targets per thread) that sets the tile
constexpr int FAR_TPT = 2;         //   splits of the shear-stress and target sums
constexpr int FAR_TS = 256;        // sources per shared-memory tile
constexpr int WALL_TS = 32;        // wall nodes per tile (keeps FP32 offsets small)
constexpr int NEAR_NT = 128;       // threads per CTA of the barycentric kernels
constexpr int NEAR_TK = 128;       // source nodes per shared-memory tile
constexpr int BD_NT = 256;         // threads per CTA of the boundary-value kernel

// ---------------------------------------------------------------------------
// Geometry (stokesSolver.f:136-204, :417-457).

// Wall nodes of the superellipse x = a r cos t, y = b r sin t,
// r = (|cos t|^p + |sin t|^p)^(-1/p), t = k 2pi/nout (:182-191).
__global__ void k_wall_nodes(int nout, double a, double b, double p, double* __restrict__ x,
                             double* __restrict__ y) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nout) return;
  double dth = EB_TWOPI / nout;
  double th = k * dth;
  double c = cos(th), s = sin(th);
  double r = pow(pow(fabs(c), p) + pow(fabs(s), p), -1.0 / p);
  x[k] = a * r * c;
  y[k] = b * r * s;
}

// One CTA per curve of length n.  First and second spectral derivatives by
// circulant convolution with dk[m] = (1/2)(-1)^m cot(pi m/n), the matrix of
// fourierDiff (:348-388, even n); then speed, normal (-y', x')/|z'|,
// curvature (y'x'' - x'y'')/|z'|^3 (:447-453), negated on the wall (:195-199).
__global__ void k_geom(const double* __restrict__ x, const double* __restrict__ y, int n,
                       const double* __restrict__ dk, int out_off, int negate,
                       double2* __restrict__ xy, double2* __restrict__ nrm, double* __restrict__ sp,
                       double* __restrict__ cur, double* __restrict__ w, double2* __restrict__ dz,
                       double2* __restrict__ d1tmp) {
  const int c = blockIdx.x;
  const double* xc = x + (size_t)c * n;
  const double* yc = y + (size_t)c * n;
  double2* D1 = d1tmp + (size_t)c * n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double ax = 0.0, ay = 0.0;
    for (int k = 0; k < n; ++k) {
      int m = j - k;
      if (m < 0) m += n;
      double d = __ldg(dk + m);
      ax = fma(d, __ldg(xc + k), ax);
      ay = fma(d, __ldg(yc + k), ay);
    }
    D1[j] = make_double2(ax, ay);
  }
  __syncthreads();
  const double h = EB_TWOPI / n;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    double bx = 0.0, by = 0.0;
    for (int k = 0; k < n; ++k) {
      int m = j - k;
      if (m < 0) m += n;
      double d = __ldg(dk + m);
      double2 q = D1[k];
      bx = fma(d, q.x, bx);
      by = fma(d, q.y, by);
    }
    double2 q = D1[j];
    double Dx = q.x, Dy = q.y, DDx = bx, DDy = by;
    double s = sqrt(Dx * Dx + Dy * Dy);
    double px = -Dy / s, py = Dx / s;
    double cu = (Dy * DDx - Dx * DDy) / (s * s * s);
    if (negate) { px = -px; py = -py; cu = -cu; }
    int g = out_off + c * n + j;
    xy[g] = make_double2(xc[j], yc[j]);
    nrm[g] = make_double2(px, py);
    sp[g] = s;
    cur[g] = cu;
    w[g] = s * h / EB_PI;
    dz[g] = make_double2(Dx * h, Dy * h);
  }
}

// Centroid (plain node mean, :151-160) and mean speed (the body radius of
// matvec_DLP_fmmbary, :697-703) per body.
__global__ void k_body_stats(int n, int nout, const double2* __restrict__ xy, const double* __restrict__ sp,
                             double2* __restrict__ cen, double* __restrict__ rb) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  double sx = 0, sy = 0, ss = 0;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    int g = nout + b * n + k;
    sx += xy[g].x; sy += xy[g].y; ss += sp[g];
  }
  sx = block_sum<256>(sx, sh);
  sy = block_sum<256>(sy, sh);
  ss = block_sum<256>(ss, sh);
  if (threadIdx.x == 0) { cen[b] = make_double2(sx / n, sy / n); rb[b] = ss / n; }
}

// ---------------------------------------------------------------------------
// Per-matvec preparation: one CTA per curve.  Writes
//   ws    = w * sigma               (full strengths: self-curve sums)
//   sq64, sq32: the pair tensors (pair_tensor64/32) of the strengths seen by
//         other curves, v = w * (sigma - rigid part)
// the constraint rows of every body (:1055-1096) and the wall's integral of
// sigma.n for the rank-one term (:1107-1111).  The rigid part of a body's
// density is its speed-weighted projection on the translations and the
// rotation about the speed-weighted centroid: a rigid-motion density has a
// zero double layer outside its curve, so removing it changes the far field
// only at the rounding level while the sums stop cancelling terms of size
// |sigma_rigid| (large for small bodies: the stokeslet/rotlet completion puts
// ~lambda/r and ~xi/r^3 into these modes).  The split is made only when the
// close pairs are masked for the barycentric correction (split_rigid = 1): at a
// few node spacings the trapezoid rule's error on a rigid mode is ~1e-9.
// The FP32 far field's source record of a node: the symmetric tensor S with
// (r.n)(r.v) = r^T S r for the normal n and the weighted strength v,
// (S_xx, 2 S_xy, S_yy) = (n_x v_x, n_x v_y + n_y v_x, n_y v_y), formed in
// FP64 and rounded once.
__device__ __forceinline__ float4 pair_tensor32(double2 nn, double2 v) {
  return make_float4((float)(nn.x * v.x), (float)(nn.x * v.y + nn.y * v.x), (float)(nn.y * v.y), 0.f);
}

__device__ __forceinline__ double4 pair_tensor64(double2 nn, double2 v) {
  return make_double4(nn.x * v.x, nn.x * v.y + nn.y * v.x, nn.y * v.y, 0.0);
}

__global__ void __launch_bounds__(256) k_prep(GeoDev G, const double* __restrict__ den,
                                              double2* __restrict__ ws, double4* __restrict__ sq64,
                                              float4* __restrict__ sq32, double* __restrict__ vel,
                                              double* __restrict__ sigdotn, int split_rigid) {
  __shared__ double sh[32];
  const int c = blockIdx.x;
  const int start = curve_start(G, c), len = curve_len(G, c);
  if (c == 0) {
    double a0 = 0;
    for (int j = threadIdx.x; j < len; j += blockDim.x) {
      int g = start + j;
      double sx = den[ix_of(G, g)], sy = den[iy_of(G, g)];
      double wg = G.w[g];
      double2 v = make_double2(wg * sx, wg * sy);
      ws[g] = v;
      double2 nn = G.nrm[g];
      sq64[g] = pair_tensor64(nn, v);
      sq32[g] = pair_tensor32(nn, v);
      a0 += (nn.x * sx + nn.y * sy) * G.sp[g];
    }
    a0 = block_sum<256>(a0, sh);
    if (threadIdx.x == 0) *sigdotn = a0 * (EB_TWOPI / len);
    return;
  }
  // pass 1: constraint sums and the weighted means
  double a0 = 0, a1 = 0, a2 = 0, s0 = 0, sxw = 0, syw = 0;
  for (int j = threadIdx.x; j < len; j += blockDim.x) {
    int g = start + j;
    double sx = den[ix_of(G, g)], sy = den[iy_of(G, g)];
    double s = G.sp[g];
    double2 p = G.xy[g];
    a0 += sx * s;
    a1 += sy * s;
    a2 += (sx * p.y - sy * p.x) * s;
    s0 += s;
    sxw += s * p.x;
    syw += s * p.y;
  }
  a0 = block_sum<256>(a0, sh);
  a1 = block_sum<256>(a1, sh);
  a2 = block_sum<256>(a2, sh);
  s0 = block_sum<256>(s0, sh);
  sxw = block_sum<256>(sxw, sh);
  syw = block_sum<256>(syw, sh);
  if (threadIdx.x == 0) {
    int b = c - 1;
    vel[ic_of(G, b, 0)] = (-a0) / EB_TWOPI * (EB_TWOPI / len) + den[ic_of(G, b, 0)];
    vel[ic_of(G, b, 1)] = (-a1) / EB_TWOPI * (EB_TWOPI / len) + den[ic_of(G, b, 1)];
    vel[ic_of(G, b, 2)] = (-a2) / EB_TWOPI * (EB_TWOPI / len) + den[ic_of(G, b, 2)];
  }
  const double xb = sxw / s0, yb = syw / s0;
  // pass 2: rotation coefficient about (xb, yb); phi3 = (-(y - yb), x - xb)
  double r0 = 0, r1 = 0;
  for (int j = threadIdx.x; j < len; j += blockDim.x) {
    int g = start + j;
    double sx = den[ix_of(G, g)], sy = den[iy_of(G, g)];
    double s = G.sp[g];
    double2 p = G.xy[g];
    double fx = -(p.y - yb), fy = p.x - xb;
    r0 += s * (fx * sx + fy * sy);
    r1 += s * (fx * fx + fy * fy);
  }
  r0 = block_sum<256>(r0, sh);
  r1 = block_sum<256>(r1, sh);
  double t1 = a0 / s0, t2 = a1 / s0, t3 = r1 > 0 ? r0 / r1 : 0.0;
  if (!split_rigid) t1 = t2 = t3 = 0.0;
  for (int j = threadIdx.x; j < len; j += blockDim.x) {
    int g = start + j;
    double sx = den[ix_of(G, g)], sy = den[iy_of(G, g)];
    double2 p = G.xy[g];
    double wg = G.w[g];
    ws[g] = make_double2(wg * sx, wg * sy);
    double rx = sx - t1 + t3 * (p.y - yb), ry = sy - t2 - t3 * (p.x - xb);
    double2 v = make_double2(wg * rx, wg * ry);
    const double2 nn = G.nrm[g];
    sq64[g] = pair_tensor64(nn, v);
    sq32[g] = pair_tensor32(nn, v);
  }
}

// ---------------------------------------------------------------------------
// Far field, FP64: u_i = sum_{j != i} (r.n_j)(r.w_j sigma_j)/rho^4 r,
// r = x_i - x_j, over every pair of distinct curves except the (target,
// source curve) pairs that the near-field bookkeeping replaces (bit c of
// mask[i]); pairs within a curve are summed by k_self64 with the full density,
// the far field uses the density less its rigid part (see k_prep).  This is the
// sum the reference's FMM approximates (stokesSolver.f:636-680; direct form
// :1563-1584).  Sources are staged tile by tile in shared memory; a tile never
// crosses a curve, so the mask test is one bit per tile and target.  blockIdx.y
// selects a contiguous range of tiles (split-K); partial sums are reduced in a
// fixed order by k_combine.
__device__ __forceinline__ double rcp_or_zero(double r2) { return r2 > 0.0 ? __drcp_rn(r2) : 0.0; }

// 1/r2 for r2 > 0 by Newton-Raphson: the FP32 hardware reciprocal estimate
// (relative error ~2^-23), refined twice by y <- y + y (1 - r2 y) in FP64
// (quadratic convergence: ~2^-46, then below FP64 rounding).  Not correctly
// rounded (a last-bit difference from the division), which the operator's
// 1e-11 parity bound absorbs.
// Valid range: FP32's normal range, 1.2e-38 <= r2 <= 3.4e38 (node distances
// here give r2 ~ 1e-10..1e2).  The seed's argument is clamped to that range,
// so r2 outside it returns a finite value (a wrong one: the seed is then too
// far from 1/r2 for two Newton steps), never the NaN/inf that an
// underflowing or overflowing FP32 conversion would give.
__device__ __forceinline__ double rcp_newton(double r2) {
  float yf;
  const float r2f = fminf(fmaxf(__double2float_rn(r2), 1.17549435e-38f), 3.40282347e38f);
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(r2f));
  double y = (double)yf;
  double e = fma(-r2, y, 1.0);
  y = fma(y, e, y);
  e = fma(-r2, y, 1.0);
  y = fma(y, e, y);
  return r2 > 0.0 ? y : 0.0;
}

// The FP64 hardware reciprocal estimate (rcp.approx.ftz.f64, a coarse
// approximation formed from the upper half of the operand) refined by
// Newton-Raphson steps y <- y + y (1 - r2 y) in FP64.  Each step squares the
// relative error; NSTEP = 2 takes the estimate below FP64 rounding, NSTEP = 1
// leaves a relative error of the order of the square of the estimate's.
// r2 > 0 in the double's normal range (0 for r2 = 0, as rcp_or_zero).
template <int NSTEP>
__device__ __forceinline__ double rcp_newton64(double r2) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(r2));
#pragma unroll
  for (int k = 0; k < NSTEP; ++k) {
    const double e = fma(-r2, y, 1.0);
    y = fma(y, e, y);
  }
  return r2 > 0.0 ? y : 0.0;
}

// One Newton-Raphson step from the FP32 estimate: relative error ~2^-46
// (the estimate's ~2^-23, squared).  Same clamp and range as rcp_newton.
__device__ __forceinline__ double rcp_newton1(double r2) {
  float yf;
  const float r2f = fminf(fmaxf(__double2float_rn(r2), 1.17549435e-38f), 3.40282347e38f);
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(yf) : "f"(r2f));
  double y = (double)yf;
  const double e = fma(-r2, y, 1.0);
  y = fma(y, e, y);
  return r2 > 0.0 ? y : 0.0;
}

// 1/r2 by variant: 0 correctly rounded division, 1 FP32 estimate + 2 Newton
// steps, 3 FP64 estimate + 2 Newton steps (both at FP64 rounding: the
// accurate FP64 operator); 2 FP32 estimate + 1 step, 4 FP64 estimate + 1 step
// (relative error ~1e-14 and ~1e-12 per pair: the fast FP64 operator that the
// mixed-precision solve applies while its residual is still large, where an
// operator error far above FP64 rounding is harmless).
template <int RCP>
__device__ __forceinline__ double rcp_variant(double r2) {
  if constexpr (RCP == 0) return rcp_or_zero(r2);
  else if constexpr (RCP == 1) return rcp_newton(r2);
  else if constexpr (RCP == 2) return rcp_newton1(r2);
  else if constexpr (RCP == 3) return rcp_newton64<2>(r2);
  else return rcp_newton64<1>(r2);
}

// One CTA's share of the FP64 far field: targets of block bx, tiles of split
// 'split'.  Shared by k_far64 and the ensemble kernel k_far64_batch.
template <bool MASK, int NT, int TPT, int RCP>
__device__ __forceinline__ void far64_cta(const GeoDev& G, const double4* __restrict__ sq,
                                          const int4* __restrict__ tiles, const int* __restrict__ split_ptr,
                                          const unsigned* __restrict__ mask, int mw, double2* __restrict__ partial,
                                          int bx, int split, double4* sg, double* sw) {
  const int N = G.N;
  const int i0 = bx * (NT * TPT) + threadIdx.x;
  int it[TPT], cv[TPT];
  double px[TPT], py[TPT], ax[TPT], ay[TPT];
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    int i = i0 + q * NT;
    it[q] = i < N ? i : N - 1;
    cv[q] = it[q] < G.nout ? 0 : 1 + (it[q] - G.nout) / G.n;
    double2 p = G.xy[it[q]];
    px[q] = p.x; py[q] = p.y; ax[q] = 0.0; ay[q] = 0.0;
  }
  const int tb = split_ptr[split], te = split_ptr[split + 1];
  for (int ti = tb; ti < te; ++ti) {
    const int4 T = tiles[ti];
    __syncthreads();
    for (int k = threadIdx.x; k < T.y; k += NT) {
      int g = T.x + k;
      const double2 q = G.xy[g];
      const double4 S = sq[g];
      sg[k] = make_double4(q.x, q.y, S.x, S.y);
      sw[k] = S.z;
    }
    __syncthreads();
    double tx[TPT], ty[TPT];
#pragma unroll
    for (int q = 0; q < TPT; ++q) { tx[q] = 0.0; ty[q] = 0.0; }
#pragma unroll 2
    for (int j = 0; j < T.y; ++j) {
      const double4 s = sg[j];   // x, y, S_xx, 2 S_xy
      const double syy = sw[j];
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        // (r.n)(r.v) = r^T S r = (S_xx r_x + 2 S_xy r_y) r_x + S_yy r_y^2
        const double rx = px[q] - s.x, ry = py[q] - s.y;
        const double ry2 = ry * ry;
        const double rho2 = fma(rx, rx, ry2);
        const double t = fma(s.w, ry, s.z * rx);
        const double qq = fma(t, rx, syy * ry2);
        const double inv = rcp_variant<RCP>(rho2);
        const double c = qq * inv * inv;
        tx[q] = fma(c, rx, tx[q]);
        ty[q] = fma(c, ry, ty[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < TPT; ++q) {
      bool use = T.z != cv[q];
      if (MASK) use = use && !((__ldg(mask + (size_t)it[q] * mw + (T.z >> 5)) >> (T.z & 31)) & 1u);
      if (use) { ax[q] += tx[q]; ay[q] += ty[q]; }
    }
  }
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    int i = i0 + q * NT;
    if (i < N) partial[(size_t)split * N + i] = make_double2(ax[q], ay[q]);
  }
}

template <bool MASK, int NT, int TPT, int RCP>
__global__ void __launch_bounds__(NT, 512 / NT)
k_far64(GeoDev G, const double4* __restrict__ sq, const int4* __restrict__ tiles,
        const int* __restrict__ split_ptr, const unsigned* __restrict__ mask, int mw,
        double2* __restrict__ partial) {
  __shared__ double4 sg[FAR_TS];
  __shared__ double sw[FAR_TS];
  far64_cta<MASK, NT, TPT, RCP>(G, sq, tiles, split_ptr, mask, mw, partial, blockIdx.x, blockIdx.y, sg, sw);
}

// ---------------------------------------------------------------------------
// Far field, FP32 pair terms with FP64 accumulation (the mixed-precision
// operator).  Same sum as k_far64 but over pairs of DIFFERENT curves only (a
// target's own curve is evaluated in FP64 by k_self64) and without the
// near-masked pairs.  Chunks of F32_CHUNK sources are summed in FP32 and each
// chunk sum is added to an FP64 accumulator, so the rounding error of the
// accumulation grows with the chunk length, not with N.
//
// Coordinates: every node is stored as an FP32 offset from the FP64 centre of
// its own tile (tiles never cross a curve and are at most one body or 32 wall
// nodes long).  Per (target, source tile) the centre difference is formed in
// FP64, so r = (c_t - c_s) + (o_t - o_s) is rounded relative to |r|, not to the
// magnitude of the coordinates.
//
// Arithmetic: the pair term (r.n)(r.v) r / rho^4 is evaluated as
// (r^T S r) r / rho^4 with the source's symmetric tensor S (pair_tensor32,
// formed in FP64 by k_prep): t = S_xx r_x + 2 S_xy r_y, q = t r_x + S_yy r_y^2,
// c = (q / rho^2) / rho^2 — 12 lane operations and one reciprocal per pair.
// sm_100's packed FP32 instructions (two lanes per instruction, each lane IEEE
// round-to-nearest exactly like the scalar instruction) process two targets per
// instruction against one source, so every pair costs the same rounded
// operations as the scalar form while the instruction count halves.  The
// source record is duplicated into both lanes when it is staged in shared
// memory: (-x, -x, -y, -y), (S_xx, S_xx, 2 S_xy, 2 S_xy), (S_yy, S_yy).
constexpr int F32_TS = 256;

__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

__device__ __forceinline__ void two_sum_add(float& hi, float& lo, float t) {
  float s = hi + t;
  float bp = s - hi;
  float e = (hi - (s - bp)) + (t - bp);
  hi = s;
  lo += e;
}

// Sources per FP32 partial sum of k_far32: the running FP32 sum of a target is
// added to its FP64 accumulator after every F32_CHUNK sources, so the rounding
// error of the plain FP32 accumulation grows with the chunk length instead of
// the tile length (measured on solution densities: the operator's FP32 error
// is ~2.5x smaller with chunks of 16 than with whole 256-node tiles; an
// emulation of the kernel's arithmetic puts 85% of the remaining error in the
// pair terms themselves).  The FP64 additions run on the FP64 pipe, idle in
// this kernel, instead of a two-sum on the FP32 pipe that bounds it.
#ifndef EROSION_F32_CHUNK
#define EROSION_F32_CHUNK 16
#endif
constexpr int F32_CHUNK = EROSION_F32_CHUNK;

// One CTA's share of the FP32 far field (targets of block bx, tiles of split
// 'split'); shared by k_far32 and the ensemble kernel k_far32_batch.
template <bool MASK, int NT, int TPT, int U>
__device__ __forceinline__ void far32_cta(int N, int nout, int n, const float4* __restrict__ src,
                                          const float2* __restrict__ tgt, const double2* __restrict__ anchor,
                                          const double2* __restrict__ tile_c, const float4* __restrict__ sq32,
                                          const int4* __restrict__ tiles, const int* __restrict__ split_ptr,
                                          const unsigned* __restrict__ mask, int mw, double2* __restrict__ partial,
                                          int bx, int split, float4* s_pos, float4* s_q1, float2* s_q2) {
  static_assert(TPT % 2 == 0, "targets are processed in lane pairs");
  static_assert(F32_CHUNK % U == 0, "the source-loop unroll divides the chunk");
  constexpr int TP = TPT / 2;
  const int i0 = bx * (NT * TPT) + threadIdx.x;
  int it[TPT], cv[TPT];
  double AX[TPT], AY[TPT];   // FP64 accumulators of the chunk sums
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    int i = i0 + q * NT;
    it[q] = i < N ? i : N - 1;
    cv[q] = it[q] < nout ? 0 : 1 + (it[q] - nout) / n;
  }
#pragma unroll
  for (int q = 0; q < TPT; ++q) AX[q] = AY[q] = 0.0;
  const int tb = split_ptr[split], te = split_ptr[split + 1];
  for (int ti = tb; ti < te; ++ti) {
    const int4 T = tiles[ti];
    __syncthreads();
    for (int k = threadIdx.x; k < T.y; k += NT) {
      const float4 a = src[T.x + k];
      const float4 q = sq32[T.x + k];
      s_pos[k] = make_float4(-a.x, -a.x, -a.y, -a.y);
      s_q1[k] = make_float4(q.x, q.x, q.y, q.y);
      s_q2[k] = make_float2(q.z, q.z);
    }
    // pad the last chunk with zero-strength sources far from every target
    // (exactly zero terms)
    const int tlen = (T.y + F32_CHUNK - 1) / F32_CHUNK * F32_CHUNK;
    for (int k = T.y + threadIdx.x; k < tlen; k += NT) {
      s_pos[k] = make_float4(-1e4f, -1e4f, -1e4f, -1e4f);
      s_q1[k] = make_float4(0.f, 0.f, 0.f, 0.f);
      s_q2[k] = make_float2(0.f, 0.f);
    }
    __syncthreads();
    const double2 cs = tile_c[ti];
    float2 PX[TP], PY[TP];
    bool U0[TP], U1[TP];   // false: the pair is masked out of this tile (own curve or near)
#pragma unroll
    for (int p = 0; p < TP; ++p) {
      const int q0 = it[2 * p], q1 = it[2 * p + 1];
      const double2 a0 = anchor[q0], a1 = anchor[q1];
      const float2 o0 = tgt[q0], o1 = tgt[q1];
      PX[p] = make_float2((float)(a0.x - cs.x) + o0.x, (float)(a1.x - cs.x) + o1.x);
      PY[p] = make_float2((float)(a0.y - cs.y) + o0.y, (float)(a1.y - cs.y) + o1.y);
      bool u0 = T.z != cv[2 * p], u1 = T.z != cv[2 * p + 1];
      if (MASK) {
        u0 = u0 && !((__ldg(mask + (size_t)q0 * mw + (T.z >> 5)) >> (T.z & 31)) & 1u);
        u1 = u1 && !((__ldg(mask + (size_t)q1 * mw + (T.z >> 5)) >> (T.z & 31)) & 1u);
      }
      U0[p] = u0;
      U1[p] = u1;
    }
    for (int j0 = 0; j0 < tlen; j0 += F32_CHUNK) {
      float2 TX[TP], TY[TP];
#pragma unroll
      for (int p = 0; p < TP; ++p) TX[p] = TY[p] = make_float2(0.f, 0.f);
#pragma unroll U
      for (int j = j0; j < j0 + F32_CHUNK; ++j) {
        const float4 A = s_pos[j], B = s_q1[j];
        const float2 qyy = s_q2[j];
        const float2 msx = make_float2(A.x, A.y), msy = make_float2(A.z, A.w);
        const float2 qxx = make_float2(B.x, B.y), qxy = make_float2(B.z, B.w);
#pragma unroll
        for (int p = 0; p < TP; ++p) {
          // 12 lane operations and one reciprocal per pair:
          // c = r^T S r / rho^4,  u += c r
          const float2 rx = __fadd2_rn(PX[p], msx);
          const float2 ry = __fadd2_rn(PY[p], msy);
          const float2 ry2 = __fmul2_rn(ry, ry);
          const float2 rho2 = __ffma2_rn(rx, rx, ry2);
          const float2 inv = make_float2(rcp_approx(rho2.x), rcp_approx(rho2.y));
          const float2 t = __ffma2_rn(qxy, ry, __fmul2_rn(qxx, rx));
          const float2 q = __ffma2_rn(t, rx, __fmul2_rn(qyy, ry2));
          const float2 c = __fmul2_rn(__fmul2_rn(q, inv), inv);
          TX[p] = __ffma2_rn(c, rx, TX[p]);
          TY[p] = __ffma2_rn(c, ry, TY[p]);
        }
      }
#pragma unroll
      for (int p = 0; p < TP; ++p) {   // a select, not a product: an own-curve tile holds inf/NaN terms
        if (U0[p]) { AX[2 * p] += (double)TX[p].x; AY[2 * p] += (double)TY[p].x; }
        if (U1[p]) { AX[2 * p + 1] += (double)TX[p].y; AY[2 * p + 1] += (double)TY[p].y; }
      }
    }
  }
#pragma unroll
  for (int q = 0; q < TPT; ++q) {
    int i = i0 + q * NT;
    if (i < N) partial[(size_t)split * N + i] = make_double2(AX[q], AY[q]);
  }
}

// MINB: resident CTAs per SM the kernel is compiled for (the register
// budget: 2 CTAs of 256 threads leave 128 registers a thread, 3 leave 85).
template <bool MASK, int NT, int TPT, int U, int MINB>
__global__ void __launch_bounds__(NT, MINB)
k_far32(int N, int nout, int n, const float4* __restrict__ src, const float2* __restrict__ tgt,
        const double2* __restrict__ anchor, const double2* __restrict__ tile_c, const float4* __restrict__ sq32,
        const int4* __restrict__ tiles, const int* __restrict__ split_ptr, const unsigned* __restrict__ mask, int mw,
        double2* __restrict__ partial) {
  __shared__ float4 s_pos[F32_TS];
  __shared__ float4 s_q1[F32_TS];
  __shared__ float2 s_q2[F32_TS];
  far32_cta<MASK, NT, TPT, U>(N, nout, n, src, tgt, anchor, tile_c, sq32, tiles, split_ptr, mask, mw, partial,
                           blockIdx.x, blockIdx.y, s_pos, s_q1, s_q2);
}

// ---------------------------------------------------------------------------
// Ensemble far field: ONE persistent launch covers the far field of every
// geometry of an ensemble.  Work item = (geometry, target block, tile split);
// items are numbered job by job (FarJob*.item0) and CTAs stride over them.
struct FarJob64 {
  GeoDev G;
  const double4* sq;
  const int4* tiles;
  const int* split_ptr;
  const unsigned* mask;   // nullptr: no near masking
  int mw;
  double2* partial;
  int nbx, nsplit;
  long long item0;
};

struct FarJob32 {
  int N, nout, n;
  const float4* src;
  const float2* tgt;
  const double2* anchor;
  const double2* tile_c;
  const float4* sq32;
  const int4* tiles;
  const int* split_ptr;
  const unsigned* mask;
  int mw;
  double2* partial;
  int nbx, nsplit;
  long long item0;
};

template <class Job>
__device__ __forceinline__ int find_job(const Job* __restrict__ jobs, int njobs, long long item) {
  int lo = 0, hi = njobs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].item0 <= item) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <int NT, int TPT, int RCP>
__global__ void __launch_bounds__(NT, 512 / NT)
k_far64_batch(const FarJob64* __restrict__ jobs, int njobs, long long nitems) {
  __shared__ double4 sg[FAR_TS];
  __shared__ double sw[FAR_TS];
  for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
    const FarJob64 J = jobs[find_job(jobs, njobs, item)];
    const int local = (int)(item - J.item0);
    const int bx = local % J.nbx, q = local / J.nbx;
    if (J.mask) far64_cta<true, NT, TPT, RCP>(J.G, J.sq, J.tiles, J.split_ptr, J.mask, J.mw, J.partial, bx, q, sg, sw);
    else far64_cta<false, NT, TPT, RCP>(J.G, J.sq, J.tiles, J.split_ptr, nullptr, 0, J.partial, bx, q, sg, sw);
    __syncthreads();
  }
}

template <int NT, int TPT, int U, int MINB>
__global__ void __launch_bounds__(NT, MINB)
k_far32_batch(const FarJob32* __restrict__ jobs, int njobs, long long nitems) {
  __shared__ float4 s_pos[F32_TS];
  __shared__ float4 s_q1[F32_TS];
  __shared__ float2 s_q2[F32_TS];
  for (long long item = blockIdx.x; item < nitems; item += gridDim.x) {
    const FarJob32 J = jobs[find_job(jobs, njobs, item)];
    const int local = (int)(item - J.item0);
    const int bx = local % J.nbx, q = local / J.nbx;
    if (J.mask)
      far32_cta<true, NT, TPT, U>(J.N, J.nout, J.n, J.src, J.tgt, J.anchor, J.tile_c, J.sq32, J.tiles, J.split_ptr,
                               J.mask, J.mw, J.partial, bx, q, s_pos, s_q1, s_q2);
    else
      far32_cta<false, NT, TPT, U>(J.N, J.nout, J.n, J.src, J.tgt, J.anchor, J.tile_c, J.sq32, J.tiles, J.split_ptr,
                                nullptr, 0, J.partial, bx, q, s_pos, s_q1, s_q2);
    __syncthreads();
  }
}

// Launch shapes the autotuner chooses from (threads per CTA, targets per
// thread); solver.cu times each on the geometry at hand.
// The third field is a kernel variant: for the FP64 kernels the reciprocal
// (rcp_variant), for the FP32 kernel the unroll factor of the source loop;
// the fourth, for the FP32 kernel, the resident CTAs per SM it is compiled
// for (TPT = 4 fits 80 registers without spills at 3 CTAs of 256 threads).
// Kinds: 0 accurate FP64 (reciprocal at FP64 rounding), 1 FP32, 2 fast FP64.
struct FarShape { int nt, tpt, rcp, minb; };
constexpr FarShape kFar64Shapes[] = {{256, 2, 1}, {128, 4, 1}, {256, 2, 3}, {128, 4, 3}};
constexpr FarShape kFar32Shapes[] = {{256, 4, 2, 2}, {256, 4, 4, 2}, {256, 4, 2, 3}, {256, 4, 4, 3}};
constexpr FarShape kFar64FastShapes[] = {{256, 2, 2}, {128, 4, 2}, {256, 2, 4}, {128, 4, 4}};
constexpr int kNumFar64Shapes = 4, kNumFar32Shapes = 4, kNumFar64FastShapes = 4;
constexpr int kFarKinds = 3;
constexpr FarShape far_shape_of(int kind, int i) {
  return kind == 0 ? kFar64Shapes[i] : (kind == 1 ? kFar32Shapes[i] : kFar64FastShapes[i]);
}
constexpr int far_num_shapes(int kind) {
  return kind == 0 ? kNumFar64Shapes : (kind == 1 ? kNumFar32Shapes : kNumFar64FastShapes);
}

// Tile centres (middle node) and, per node, the FP32 offset from its tile's
// centre plus that centre (the target anchor of k_far32).  One CTA per tile.
__global__ void k_geom32(int ntile, const int4* __restrict__ tiles, const double2* __restrict__ xy,
                         const double2* __restrict__ nrm, double2* __restrict__ tile_c, float4* __restrict__ src,
                         float2* __restrict__ tgt, double2* __restrict__ anchor) {
  const int t = blockIdx.x;
  if (t >= ntile) return;
  const int4 T = tiles[t];
  const double2 c = xy[T.x + T.y / 2];
  if (threadIdx.x == 0) tile_c[t] = c;
  for (int k = threadIdx.x; k < T.y; k += blockDim.x) {
    int g = T.x + k;
    double2 p = xy[g], nn = nrm[g];
    float ox = (float)(p.x - c.x), oy = (float)(p.y - c.y);
    src[g] = make_float4(ox, oy, (float)nn.x, (float)nn.y);
    tgt[g] = make_float2(ox, oy);
    anchor[g] = c;
  }
}

// FP64 pairs within each curve (i != j), with the full density: the
// self-interaction part of the far-field sum.  Task = (first target, count
// <= 256, curve, source chunk); the wall's sources are split into chunks of
// SELF_CHUNK and a body's into chunks of body_chunk, whose partial sums land in
// separate slots (out[slot*N + i]) added in a fixed order by k_combine.
constexpr int SELF_CHUNK = 512;
constexpr int SELF_CHUNK_BODY = 64;
__global__ void __launch_bounds__(256)
k_self64(GeoDev G, const double2* __restrict__ ws, const int4* __restrict__ tasks, double2* __restrict__ out,
         int body_chunk) {
  __shared__ double4 sg[256];
  __shared__ double2 sw[256];
  const int4 tk = tasks[blockIdx.x];   // target start, count, curve, chunk
  const int c = tk.z, chunk = tk.w;
  const int start = curve_start(G, c), len = curve_len(G, c);
  const int csz = c == 0 ? SELF_CHUNK : body_chunk;
  const int kb = chunk * csz, ke = min(len, kb + csz);
  const int i = tk.x + threadIdx.x;
  const bool act = threadIdx.x < tk.y;
  const int ic = act ? i : tk.x;
  const double2 p = G.xy[ic];
  double ax = 0.0, ay = 0.0;
  for (int k0 = kb; k0 < ke; k0 += 256) {
    __syncthreads();
    const int kl = k0 + threadIdx.x;
    if (kl < ke) {
      int g = start + kl;
      double2 q = G.xy[g], nn = G.nrm[g];
      sg[threadIdx.x] = make_double4(q.x, q.y, nn.x, nn.y);
      sw[threadIdx.x] = ws[g];
    }
    __syncthreads();
    const int kt = min(256, ke - k0);
#pragma unroll 4
    for (int j = 0; j < kt; ++j) {
      const double4 s = sg[j];
      const double2 a = sw[j];
      double rx = p.x - s.x, ry = p.y - s.y;
      double rho2 = fma(rx, rx, ry * ry);
      double rdn = fma(rx, s.z, ry * s.w);
      double rds = fma(rx, a.x, ry * a.y);
      double inv = rcp_or_zero(rho2);
      double cc = rdn * rds * inv * inv;
      ax = fma(cc, rx, ax);
      ay = fma(cc, ry, ay);
    }
  }
  if (act) out[(size_t)chunk * G.N + i] = make_double2(ax, ay);
}

// ---------------------------------------------------------------------------
// Block Gauss-Seidel preconditioner (right preconditioning of GMRES):
//   z_wall = -2 v_wall                         (the wall block's jump -1/2 I)
//   t_b    = v_b - A_bw z_wall                 (wall -> body coupling, trapezoid)
//   z_b    = B_b^{-1} t_b                      (exact per-body blocks, FP32)
// B_b is the operator restricted to body b's density and its stokeslet and
// rotlet unknowns (size m = 2n + 3, ordered sigma_x, sigma_y, l1, l2, xi).

// Entries of B_b, FP32, row-major, one CTA per (body, row).
__global__ void __launch_bounds__(256)
k_pc_blocks(GeoDev G, float* __restrict__ B) {
  const int b = blockIdx.x, row = blockIdx.y;
  const int n = G.n, m = 2 * n + 3;
  float* R = B + ((size_t)b * m + row) * m;
  const int base = G.nout + b * n;
  const double2 cb = G.cen[b];
  if (row < 2 * n) {
    const int i = row < n ? row : row - n;   // target node
    const int comp = row < n ? 0 : 1;        // u or v
    const int gi = base + i;
    const double2 p = G.xy[gi];
    for (int col = threadIdx.x; col < m; col += blockDim.x) {
      double v = 0.0;
      if (col < 2 * n) {
        const int j = col < n ? col : col - n;
        const int ccomp = col < n ? 0 : 1;
        const int gj = base + j;
        if (j != i) {
          const double2 q = G.xy[gj], nn = G.nrm[gj];
          const double rx = p.x - q.x, ry = p.y - q.y;
          const double rho2 = rx * rx + ry * ry;
          const double f = (rx * nn.x + ry * nn.y) * G.w[gj] / (rho2 * rho2);
          v = f * (comp == 0 ? rx : ry) * (ccomp == 0 ? rx : ry);
        } else {
          const double2 nn = G.nrm[gi];
          const double k = G.cur[gi] * G.sp[gi] / n;
          if (comp == 0 && ccomp == 0) v = -k * nn.y * nn.y - 0.5;
          else if (comp == 0 && ccomp == 1) v = k * nn.x * nn.y;
          else if (comp == 1 && ccomp == 0) v = k * nn.y * nn.x;
          else v = -k * nn.x * nn.x - 0.5;
        }
      } else {
        const double rx = p.x - cb.x, ry = p.y - cb.y;
        const double rho2 = rx * rx + ry * ry;
        const double lg = log(rho2);
        const int c = col - 2 * n;
        const double q = 0.5 / EB_TWOPI;
        if (c == 0) v = comp == 0 ? q * (-0.5 * lg + rx * rx / rho2) : q * (rx * ry / rho2);
        else if (c == 1) v = comp == 0 ? q * (rx * ry / rho2) : q * (-0.5 * lg + ry * ry / rho2);
        else v = comp == 0 ? ry / rho2 : -rx / rho2;
      }
      R[col] = (float)v;
    }
  } else {
    const int c = row - 2 * n;
    for (int col = threadIdx.x; col < m; col += blockDim.x) {
      double v = 0.0;
      if (col < 2 * n) {
        const int j = col < n ? col : col - n;
        const bool isx = col < n;
        const int gj = base + j;
        const double sp = G.sp[gj];
        const double2 q = G.xy[gj];
        if (c == 0) v = isx ? -sp / n : 0.0;
        else if (c == 1) v = isx ? 0.0 : -sp / n;
        else v = isx ? -q.y * sp / n : q.x * sp / n;
      } else {
        v = (col - 2 * n == c) ? 1.0 : 0.0;
      }
      R[col] = (float)v;
    }
  }
}

// In-place Gauss-Jordan inversion with partial pivoting of a batch of m x m
// FP32 matrices, one CTA per matrix.  A zero pivot sets bad[matrix].
__global__ void __launch_bounds__(1024)
k_gj_inv32(int m, float* __restrict__ B, int* __restrict__ bad) {
  extern __shared__ float gjs[];
  float* prow = gjs;               // pivot row (m)
  float* pcol = gjs + m;           // pivot column (m)
  int* piv = (int*)(gjs + 2 * m);  // row swaps (m)
  __shared__ float rv[32];
  __shared__ int ri[32];
  float* A = B + (size_t)blockIdx.x * m * m;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int k = 0; k < m; ++k) {
    // pivot search over rows k..m-1 of column k
    float best = -1.f;
    int bi = k;
    for (int i = k + tid; i < m; i += nt) {
      float a = fabsf(A[(size_t)i * m + k]);
      if (a > best) { best = a; bi = i; }
    }
    for (int o = 16; o > 0; o >>= 1) {
      float b2 = __shfl_xor_sync(0xffffffffu, best, o);
      int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
      if (b2 > best || (b2 == best && i2 < bi)) { best = b2; bi = i2; }
    }
    if ((tid & 31) == 0) { rv[tid >> 5] = best; ri[tid >> 5] = bi; }
    __syncthreads();
    if (tid < 32) {
      best = tid < (nt >> 5) ? rv[tid] : -1.f;
      bi = tid < (nt >> 5) ? ri[tid] : k;
      for (int o = 16; o > 0; o >>= 1) {
        float b2 = __shfl_xor_sync(0xffffffffu, best, o);
        int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        if (b2 > best || (b2 == best && i2 < bi)) { best = b2; bi = i2; }
      }
      if (tid == 0) { piv[k] = bi; if (!(best > 0.f)) bad[blockIdx.x] = 1; }
    }
    __syncthreads();
    const int p = piv[k];
    if (p != k) {
      for (int j = tid; j < m; j += nt) {
        float t = A[(size_t)k * m + j];
        A[(size_t)k * m + j] = A[(size_t)p * m + j];
        A[(size_t)p * m + j] = t;
      }
      __syncthreads();
    }
    const float d = 1.f / A[(size_t)k * m + k];
    __syncthreads();   // every thread holds the pivot before row k is overwritten
    for (int j = tid; j < m; j += nt) {
      float v = (j == k) ? d : A[(size_t)k * m + j] * d;
      A[(size_t)k * m + j] = v;
      prow[j] = v;
    }
    for (int i = tid; i < m; i += nt) pcol[i] = (i == k) ? 0.f : A[(size_t)i * m + k];
    __syncthreads();
    // rows i != k: a_ij -= a_ik * prow_j (column k: a_ik = -a_ik * d)
    for (int e = tid; e < m * m; e += nt) {
      const int i = e / m, j = e - i * m;
      if (i == k) continue;
      const float f = pcol[i];
      if (j == k) A[(size_t)i * m + j] = -f * d;
      else A[(size_t)i * m + j] -= f * prow[j];
    }
    __syncthreads();
  }
  // undo the row swaps as column swaps, last first
  for (int k = m - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k) {
      for (int i = tid; i < m; i += nt) {
        float t = A[(size_t)i * m + k];
        A[(size_t)i * m + k] = A[(size_t)i * m + p];
        A[(size_t)i * m + p] = t;
      }
    }
    __syncthreads();
  }
}

// Replaces the inverse of every flagged (singular) block by the identity,
// rows blockIdx.y * 8 .. + 7 of body blockIdx.x.
__global__ void __launch_bounds__(256)
k_pc_identity_if_bad(int m, const int* __restrict__ bad, float* __restrict__ B) {
  const int b = blockIdx.x;
  if (!bad[b]) return;
  float* A = B + (size_t)b * m * m;
  const int r0 = blockIdx.y * 8;
  for (int e = threadIdx.x; e < 8 * m; e += blockDim.x) {
    const int r = r0 + e / m, c = e % m;
    if (r < m) A[(size_t)r * m + c] = r == c ? 1.f : 0.f;
  }
}

// Blocked form of k_gj_inv32: the same in-place Gauss-Jordan inversion with
// partial pivoting, the pivots taken pb at a time.  A panel of pb columns is
// loaded into shared memory and eliminated there (pivot search, row scaling
// and elimination of every other row restricted to the panel); the elementary
// row operations of the panel compose into L = I + (P - I_panel) E^T, whose
// panel columns P are exactly what in-place Gauss-Jordan leaves in the panel.
// The other columns then take the whole panel at once: with W the panel's
// pivot rows of those columns (after the panel's row swaps),
//   A[i][j] <- (i a panel pivot row ? 0 : A[i][j]) + sum_k P[i][k] W[k][j],
// one pass over the matrix per panel instead of one per pivot.  Row swaps are
// applied to the non-panel columns in global memory; at the end they are
// undone as column swaps, last first.  Shared memory: m*pb (P) + pb*m (W) +
// m (pivot column) floats + m ints.  A zero pivot sets bad[matrix].
__global__ void __launch_bounds__(512)
k_gj_inv32_blocked(int m, int pb, float* __restrict__ B, int* __restrict__ bad) {
  extern __shared__ float gjb[];
  float* P = gjb;                        // m x pb, row i at P[i * pb]
  float* W = gjb + (size_t)m * pb;       // pb x m
  float* pcol = W + (size_t)pb * m;      // m
  int* piv = (int*)(pcol + m);           // m
  __shared__ float rv[32];
  __shared__ int ri[32];
  __shared__ float dsh;
  float* A = B + (size_t)blockIdx.x * m * m;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int k0 = 0; k0 < m; k0 += pb) {
    const int kb = min(pb, m - k0);
    for (int e = tid; e < m * kb; e += nt) {
      const int i = e / kb, k = e - i * kb;
      P[i * pb + k] = A[(size_t)i * m + k0 + k];
    }
    __syncthreads();
    for (int k = 0; k < kb; ++k) {
      const int kk = k0 + k;
      float best = -1.f;
      int bi = kk;
      for (int i = kk + tid; i < m; i += nt) {
        const float a = fabsf(P[i * pb + k]);
        if (a > best) { best = a; bi = i; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const float b2 = __shfl_xor_sync(0xffffffffu, best, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        if (b2 > best || (b2 == best && i2 < bi)) { best = b2; bi = i2; }
      }
      if ((tid & 31) == 0) { rv[tid >> 5] = best; ri[tid >> 5] = bi; }
      __syncthreads();
      if (tid < 32) {
        best = tid < (nt >> 5) ? rv[tid] : -1.f;
        bi = tid < (nt >> 5) ? ri[tid] : kk;
        for (int o = 16; o > 0; o >>= 1) {
          const float b2 = __shfl_xor_sync(0xffffffffu, best, o);
          const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
          if (b2 > best || (b2 == best && i2 < bi)) { best = b2; bi = i2; }
        }
        if (tid == 0) { piv[kk] = bi; if (!(best > 0.f)) bad[blockIdx.x] = 1; }
      }
      __syncthreads();
      const int p = piv[kk];
      if (p != kk && tid < kb) {
        const float t = P[kk * pb + tid];
        P[kk * pb + tid] = P[p * pb + tid];
        P[p * pb + tid] = t;
      }
      __syncthreads();
      if (tid == 0) dsh = 1.f / P[kk * pb + k];
      for (int i = tid; i < m; i += nt) pcol[i] = P[i * pb + k];
      __syncthreads();
      const float d = dsh;
      if (tid < kb) P[kk * pb + tid] = (tid == k) ? d : P[kk * pb + tid] * d;
      __syncthreads();
      for (int e = tid; e < m * kb; e += nt) {
        const int i = e / kb, j = e - i * kb;
        if (i == kk) continue;
        const float f = pcol[i];
        P[i * pb + j] = (j == k) ? -f * d : P[i * pb + j] - f * P[kk * pb + j];
      }
      __syncthreads();
    }
    // the panel's row swaps, on the other columns
    for (int k = 0; k < kb; ++k) {
      const int kk = k0 + k, p = piv[kk];
      if (p != kk) {
        for (int j = tid; j < m; j += nt) {
          if (j >= k0 && j < k0 + kb) continue;
          const float t = A[(size_t)kk * m + j];
          A[(size_t)kk * m + j] = A[(size_t)p * m + j];
          A[(size_t)p * m + j] = t;
        }
      }
      __syncthreads();
    }
    for (int e = tid; e < kb * m; e += nt) {
      const int k = e / m, j = e - k * m;
      W[e] = (j >= k0 && j < k0 + kb) ? 0.f : A[(size_t)(k0 + k) * m + j];
    }
    __syncthreads();
    for (int i = 0; i < m; ++i) {
      const bool pivot_row = i >= k0 && i < k0 + kb;
      const float* Pi = P + i * pb;
      for (int j = tid; j < m; j += nt) {
        if (j >= k0 && j < k0 + kb) continue;
        float acc = pivot_row ? 0.f : A[(size_t)i * m + j];
        for (int k = 0; k < kb; ++k) acc = fmaf(Pi[k], W[k * m + j], acc);
        A[(size_t)i * m + j] = acc;
      }
    }
    for (int e = tid; e < m * kb; e += nt) {
      const int i = e / kb, k = e - i * kb;
      A[(size_t)i * m + k0 + k] = P[i * pb + k];
    }
    __syncthreads();
  }
  // undo the row swaps as column swaps, last first
  for (int k = m - 1; k >= 0; --k) {
    const int p = piv[k];
    if (p != k) {
      for (int i = tid; i < m; i += nt) {
        const float t = A[(size_t)i * m + k];
        A[(size_t)i * m + k] = A[(size_t)i * m + p];
        A[(size_t)i * m + p] = t;
      }
    }
    __syncthreads();
  }
}

// z_b = B_b^{-1} t_b for every body.  t is gathered from v (the body part of
// the unknown vector) less the wall coupling A_bw z_wall, given as ntw
// partial sums per body node (slot q at tw + q * tw_stride, body-major); z is
// scattered into the same layout.  CTA = (body, 256-row chunk), warp per row.
__global__ void __launch_bounds__(256)
k_pc_apply_bodies(GeoDev G, const float* __restrict__ Binv, const double* __restrict__ v,
                  const double2* __restrict__ tw, long long tw_stride, int ntw, double* __restrict__ z) {
  extern __shared__ float tv[];   // m entries of t_b
  const int b = blockIdx.x, n = G.n, m = 2 * n + 3;
  const long long sb = 2LL * G.nout + 2LL * n * b;      // sigma block of body b
  const long long cbk = 2LL * G.nout + 2LL * n * G.M + 3LL * b;
  for (int r = threadIdx.x; r < m; r += blockDim.x) {
    double t;
    if (r < 2 * n) {
      const int k = r < n ? r : r - n;
      double cpl = 0.0;
      for (int q = 0; q < ntw; ++q) {
        const double2 v2 = tw[q * tw_stride + (size_t)b * n + k];
        cpl += r < n ? v2.x : v2.y;
      }
      t = v[sb + r] - cpl;
    } else {
      t = v[cbk + (r - 2 * n)];
    }
    tv[r] = (float)t;
  }
  __syncthreads();
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int r = blockIdx.y * 8 + wid; r < m; r += gridDim.y * 8) {
    const float* __restrict__ row = Binv + ((size_t)b * m + r) * m;
    float acc = 0.f;
    for (int c = lane; c < m; c += 32) acc = fmaf(__ldg(row + c), tv[c], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) {
      if (r < 2 * n) z[sb + r] = (double)acc;
      else z[cbk + (r - 2 * n)] = (double)acc;
    }
  }
}

// ---------------------------------------------------------------------------
// Coarse correction of the block preconditioner (precond = 2).  Coarse space
// per body b: its rigid-motion densities r1 = (1, 0), r2 = (0, 1),
// r3 = (-(y - yc), x - xc) ((xc, yc) = G.cen[b], the node mean the
// stokeslets/rotlets are centred on) and the unit vectors s1, s2, s3 of its
// stokeslet/rotlet unknowns.  A r_i is non-zero only in b's stokeslet/rotlet
// rows (a rigid motion has no double-layer field; k_prep's constraint rows:
// -(1/n) sum sigma |z'| and -(1/n) sum (sigma_x y - sigma_y x) |z'|), and
// A s_j is the completion field of that unknown at every node (as k_combine
// evaluates it) plus 1 in its own row.  So with coarse coordinates (c_r, c_s)
// the coarse operator Q^T A Q = [[0, Bm], [C, I]]: Bm = the rigid moments
// of the completion fields over every body's nodes (dense, 3M x 3M), C = the
// constraint rows of the rigid densities (3 x 3 per body).

// The completion field at p of unit stokeslet/rotlet unknowns (l1, l2, xi)
// centred at c, as k_combine adds it: u = F * (l1, l2, xi).
__device__ __forceinline__ void cg_fields(double2 p, double2 c, double f[2][3]) {
  const double rx = p.x - c.x, ry = p.y - c.y;
  const double rho2 = rx * rx + ry * ry;
  const double lg = log(rho2), ir = 1.0 / rho2;
  const double k = 0.5 / EB_TWOPI;
  f[0][0] = k * (-0.5 * lg + rx * rx * ir);
  f[1][0] = k * (rx * ry * ir);
  f[0][1] = k * (rx * ry * ir);
  f[1][1] = k * (-0.5 * lg + ry * ry * ir);
  f[0][2] = ry * ir;
  f[1][2] = -rx * ir;
}

// q = Q^T v: per body the sums of v over its nodes against r1, r2, r3, then
// its three stokeslet/rotlet entries.  One CTA per body.
__global__ void __launch_bounds__(256) k_cg_restrict(GeoDev G, const double* __restrict__ v, double* __restrict__ q) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  const double2 c = G.cen[b];
  double a0 = 0, a1 = 0, a2 = 0;
  for (int k = threadIdx.x; k < G.n; k += blockDim.x) {
    const int g = G.nout + b * G.n + k;
    const double2 p = G.xy[g];
    const double vx = v[ix_of(G, g)], vy = v[iy_of(G, g)];
    a0 += vx;
    a1 += vy;
    a2 += -(p.y - c.y) * vx + (p.x - c.x) * vy;
  }
  a0 = block_sum<256>(a0, sh);
  a1 = block_sum<256>(a1, sh);
  a2 = block_sum<256>(a2, sh);
  if (threadIdx.x == 0) {
    q[6 * b] = a0;
    q[6 * b + 1] = a1;
    q[6 * b + 2] = a2;
    q[6 * b + 3] = v[ic_of(G, b, 0)];
    q[6 * b + 4] = v[ic_of(G, b, 1)];
    q[6 * b + 5] = v[ic_of(G, b, 2)];
  }
}

// Bm[(3b + i) * 3M + 3k + j] = r_i^T (field of s_j of body k) over body b's
// nodes, FP32.  CTA = (b, k).
__global__ void __launch_bounds__(128) k_cg_moments(GeoDev G, float* __restrict__ Bm) {
  __shared__ double sh[32];
  const int b = blockIdx.x, kb = blockIdx.y, M3 = 3 * G.M;
  const double2 cb = G.cen[b], ck = G.cen[kb];
  double m[3][3] = {};
  for (int k = threadIdx.x; k < G.n; k += blockDim.x) {
    const double2 p = G.xy[G.nout + b * G.n + k];
    double f[2][3];
    cg_fields(p, ck, f);
    const double ex = -(p.y - cb.y), ey = p.x - cb.x;
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      m[0][j] += f[0][j];
      m[1][j] += f[1][j];
      m[2][j] += ex * f[0][j] + ey * f[1][j];
    }
  }
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      const double t = block_sum<128>(m[i][j], sh);
      if (threadIdx.x == 0) Bm[(size_t)(3 * b + i) * M3 + 3 * kb + j] = (float)t;
    }
}

// Cinv (9 per body, FP64): the inverse of C_b, C_b[row][col] = constraint
// row `row` of A applied to r_col (the rows k_prep writes: -(1/n) sum of
// sigma_x |z'|, of sigma_y |z'|, of (sigma_x y - sigma_y x) |z'|).  A
// singular C_b (not expected for a closed curve) gets the zero inverse.
__global__ void __launch_bounds__(256) k_cg_constraints(GeoDev G, double* __restrict__ Cinv) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  const double2 c = G.cen[b];
  double s0 = 0, sx = 0, sy = 0, sxe = 0, sye = 0, sr = 0;
  for (int k = threadIdx.x; k < G.n; k += blockDim.x) {
    const int g = G.nout + b * G.n + k;
    const double2 p = G.xy[g];
    const double w = G.sp[g];
    s0 += w;
    sx += p.x * w;
    sy += p.y * w;
    sxe += (p.x - c.x) * w;
    sye += (p.y - c.y) * w;
    sr += ((p.y - c.y) * p.y + (p.x - c.x) * p.x) * w;
  }
  s0 = block_sum<256>(s0, sh);
  sx = block_sum<256>(sx, sh);
  sy = block_sum<256>(sy, sh);
  sxe = block_sum<256>(sxe, sh);
  sye = block_sum<256>(sye, sh);
  sr = block_sum<256>(sr, sh);
  if (threadIdx.x != 0) return;
  const double n = G.n;
  // columns: A r1, A r2, A r3 in the three constraint rows
  double C[3][3] = {{-s0 / n, 0.0, sye / n}, {0.0, -s0 / n, -sxe / n}, {-sy / n, sx / n, sr / n}};
  const double det = C[0][0] * (C[1][1] * C[2][2] - C[1][2] * C[2][1]) -
                     C[0][1] * (C[1][0] * C[2][2] - C[1][2] * C[2][0]) +
                     C[0][2] * (C[1][0] * C[2][1] - C[1][1] * C[2][0]);
  double* o = Cinv + 9 * b;
  if (!(fabs(det) > 0.0)) {
    for (int i = 0; i < 9; ++i) o[i] = 0.0;
    return;
  }
  const double id = 1.0 / det;
  o[0] = (C[1][1] * C[2][2] - C[1][2] * C[2][1]) * id;
  o[1] = (C[0][2] * C[2][1] - C[0][1] * C[2][2]) * id;
  o[2] = (C[0][1] * C[1][2] - C[0][2] * C[1][1]) * id;
  o[3] = (C[1][2] * C[2][0] - C[1][0] * C[2][2]) * id;
  o[4] = (C[0][0] * C[2][2] - C[0][2] * C[2][0]) * id;
  o[5] = (C[0][2] * C[1][0] - C[0][0] * C[1][2]) * id;
  o[6] = (C[1][0] * C[2][1] - C[1][1] * C[2][0]) * id;
  o[7] = (C[0][1] * C[2][0] - C[0][0] * C[2][1]) * id;
  o[8] = (C[0][0] * C[1][1] - C[0][1] * C[1][0]) * id;
}

// Coarse solve, stokeslet/rotlet part: c_s = Bm^{-1} q_r (one warp per row
// of the FP32 inverse, FP64 accumulation).  cs[3b + j].
__global__ void __launch_bounds__(256) k_cg_solve_s(int M, const float* __restrict__ Binv,
                                                    const double* __restrict__ q, double* __restrict__ cs) {
  const int M3 = 3 * M;
  const int row = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
  if (row >= M3) return;
  double acc = 0.0;
  for (int c = lane; c < M3; c += 32) acc += (double)Binv[(size_t)row * M3 + c] * q[6 * (c / 3) + (c % 3)];
  acc = warp_sum(acc);
  if (lane == 0) cs[row] = acc;
}

// Coarse solve, rigid part c_r = C_b^{-1} (q_s - c_s), then the coarse
// residual update of the constraint rows: w = v - A Q c there, A Q c = C_b c_r
// + c_s (the rigid densities' constraint rows and the unknowns' own 1).
// One thread per body.  cr[3b + i].
__global__ void k_cg_solve_r(GeoDev G, const double* __restrict__ Cinv, const double* __restrict__ q,
                             const double* __restrict__ cs, double* __restrict__ cr, double* __restrict__ w) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= G.M) return;
  const double* Ci = Cinv + 9 * b;
  double t[3], r[3];
  for (int i = 0; i < 3; ++i) t[i] = q[6 * b + 3 + i] - cs[3 * b + i];
  for (int i = 0; i < 3; ++i) r[i] = Ci[3 * i] * t[0] + Ci[3 * i + 1] * t[1] + Ci[3 * i + 2] * t[2];
  for (int i = 0; i < 3; ++i) cr[3 * b + i] = r[i];
  // C_b r = t exactly when C_b is regular, so the constraint rows of A Q c
  // are t + c_s = q_s; the zero inverse (singular C_b) leaves c_r = 0
  const bool reg = Ci[0] != 0.0 || Ci[4] != 0.0 || Ci[8] != 0.0;
  for (int i = 0; i < 3; ++i) w[ic_of(G, b, i)] -= (reg ? t[i] : 0.0) + cs[3 * b + i];
}

// The density rows of w = v - A Q c: minus the completion field of c_s at
// every node (wall and bodies).  One thread per node, the centres staged in
// shared memory.
__global__ void __launch_bounds__(256) k_cg_field(GeoDev G, const double* __restrict__ cs, double* __restrict__ w) {
  __shared__ double4 sc[256];   // cx, cy, l1, l2
  __shared__ double sxi[256];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < G.N;
  const double2 p = G.xy[act ? i : 0];
  double ux = 0.0, uy = 0.0;
  for (int b0 = 0; b0 < G.M; b0 += 256) {
    __syncthreads();
    const int t = b0 + threadIdx.x;
    if (t < G.M) {
      const double2 c = G.cen[t];
      sc[threadIdx.x] = make_double4(c.x, c.y, cs[3 * t], cs[3 * t + 1]);
      sxi[threadIdx.x] = cs[3 * t + 2];
    }
    __syncthreads();
    const int nb = min(256, G.M - b0);
    for (int j = 0; j < nb; ++j) {
      const double4 q = sc[j];
      double f[2][3];
      cg_fields(p, make_double2(q.x, q.y), f);
      ux += f[0][0] * q.z + f[0][1] * q.w + f[0][2] * sxi[j];
      uy += f[1][0] * q.z + f[1][1] * q.w + f[1][2] * sxi[j];
    }
  }
  if (!act) return;
  w[ix_of(G, i)] -= ux;
  w[iy_of(G, i)] -= uy;
}

// z += Q c: the rigid densities c_r on every body's nodes and c_s in its
// stokeslet/rotlet unknowns.  One CTA per body.
__global__ void __launch_bounds__(256) k_cg_prolong(GeoDev G, const double* __restrict__ cr,
                                                    const double* __restrict__ cs, double* __restrict__ z) {
  const int b = blockIdx.x;
  const double2 c = G.cen[b];
  const double r0 = cr[3 * b], r1 = cr[3 * b + 1], r2 = cr[3 * b + 2];
  for (int k = threadIdx.x; k < G.n; k += blockDim.x) {
    const int g = G.nout + b * G.n + k;
    const double2 p = G.xy[g];
    z[ix_of(G, g)] += r0 - r2 * (p.y - c.y);
    z[iy_of(G, g)] += r1 + r2 * (p.x - c.x);
  }
  if (threadIdx.x < 3) z[ic_of(G, b, threadIdx.x)] += cs[3 * b + threadIdx.x];
}

// z_wall = -2 v_wall, and the FP32 source tensors of w * z_wall on the wall
// (pair_tensor32) for the coupling sum.
__global__ void k_pc_wall(GeoDev G, const double* __restrict__ v, double* __restrict__ z, float4* __restrict__ sq32) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= G.nout) return;
  const double zx = -2.0 * v[g], zy = -2.0 * v[G.nout + g];
  z[g] = zx;
  z[G.nout + g] = zy;
  const double w = G.w[g];
  sq32[g] = pair_tensor32(G.nrm[g], make_double2(w * zx, w * zy));
}

// ---------------------------------------------------------------------------
// Near field: barycentric evaluation (Barnett-Wu-Veerapaneni) of the Stokes
// double layer of one curve as five holomorphic evaluations
// (StokesInteriorDLP/StokesExteriorDLP, stokesSolver.f:4937-5379).

// The five complex fields of one node: x.sigma, sigma_x, sigma_y,
// sigma n_x/(n_x + i n_y), sigma n_y/(n_x + i n_y) (:4984, :4992-4997,
// :5268-5276).
__device__ __forceinline__ void node_fields(const GeoDev& G, const double* __restrict__ den, int g,
                                            double2 f[5]) {
  double sx = den[ix_of(G, g)], sy = den[iy_of(G, g)];
  double2 p = G.xy[g], nn = G.nrm[g];
  f[0] = make_double2(p.x * sx + p.y * sy, 0.0);
  f[1] = make_double2(sx, 0.0);
  f[2] = make_double2(sy, 0.0);
  double2 ninv = cinv(nn);
  f[3] = cmul(make_double2(sx * nn.x, sy * nn.x), ninv);
  f[4] = cmul(make_double2(sx * nn.y, sy * nn.y), ninv);
}

// Boundary values of the five fields on one source curve
// (compute_bdval_in :5103-5146, compute_bdval_ex :5382-5427):
//   S_j = -sum_{k != j} (f_k - f_j) z'_k dt/(z_k - z_j) - dt f'_j
//   interior: -i S_j/(2pi) - f_j        exterior: i S_j/(2pi)
// with f' the spectral derivative.  One CTA per (curve, 256 nodes j).
__global__ void __launch_bounds__(BD_NT)
k_bdval(GeoDev G, const double* __restrict__ den, const int2* __restrict__ work,
        const int* __restrict__ src_curve, const long long* __restrict__ bd_off,
        const double* __restrict__ dker_wall, const double* __restrict__ dker_body,
        double2* __restrict__ bd) {
  __shared__ double2 sz[BD_NT], sdz[BD_NT];
  __shared__ double2 sf[5][BD_NT];
  const int s = work[blockIdx.x].x, j0 = work[blockIdx.x].y;
  const int c = src_curve[s];
  const int start = curve_start(G, c), len = curve_len(G, c);
  const double* __restrict__ dk = (c == 0) ? dker_wall : dker_body;
  const int j = j0 + threadIdx.x;
  const bool act = j < len;
  const int jc = act ? j : len - 1;
  const double2 zj = G.xy[start + jc];
  double2 fj[5];
  node_fields(G, den, start + jc, fj);
  double2 S[5], D[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) { S[q] = make_double2(0, 0); D[q] = make_double2(0, 0); }
  for (int k0 = 0; k0 < len; k0 += BD_NT) {
    __syncthreads();
    const int kl = k0 + threadIdx.x;
    if (kl < len) {
      const int g = start + kl;
      sz[threadIdx.x] = G.xy[g];
      sdz[threadIdx.x] = G.dz[g];
      double2 f[5];
      node_fields(G, den, g, f);
#pragma unroll
      for (int q = 0; q < 5; ++q) sf[q][threadIdx.x] = f[q];
    }
    __syncthreads();
    const int kt = min(BD_NT, len - k0);
    for (int kk = 0; kk < kt; ++kk) {
      const int k = k0 + kk;
      int m = jc - k;
      if (m < 0) m += len;
      const double dd = __ldg(dk + m);
      double2 cc = make_double2(0.0, 0.0);
      if (k != jc) cc = cmul(sdz[kk], cinv(csub(sz[kk], zj)));
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        const double2 fk = sf[q][kk];
        D[q].x = fma(dd, fk.x, D[q].x);
        D[q].y = fma(dd, fk.y, D[q].y);
        const double2 df = csub(fk, fj[q]);
        S[q].x -= df.x * cc.x - df.y * cc.y;
        S[q].y -= df.x * cc.y + df.y * cc.x;
      }
    }
  }
  if (!act) return;
  const double h = EB_TWOPI / len;
  const long long base = bd_off[s];
#pragma unroll
  for (int q = 0; q < 5; ++q) {
    double2 Sq = make_double2(S[q].x - h * D[q].x, S[q].y - h * D[q].y);
    double2 r;
    if (c == 0) r = make_double2(Sq.y / EB_TWOPI - fj[q].x, -Sq.x / EB_TWOPI - fj[q].y);
    else r = make_double2(-Sq.y / EB_TWOPI, Sq.x / EB_TWOPI);
    bd[base + (long long)q * len + j] = r;
  }
}

// Source-curve tile of the barycentric kernels.
struct BaryTile {
  double2 z[NEAR_TK], dz[NEAR_TK], za[NEAR_TK], b[5][NEAR_TK];
};

__device__ __forceinline__ void bary_load_tile(BaryTile& T, const GeoDev& G, int start, int len, int k0,
                                               const double2* __restrict__ bdc, bool ext, double2 a) {
  __syncthreads();
  for (int t = threadIdx.x; t < NEAR_TK; t += blockDim.x) {
    int k = k0 + t;
    if (k < len) {
      int g = start + k;
      double2 z = G.xy[g];
      T.z[t] = z;
      T.dz[t] = G.dz[g];
      T.za[t] = ext ? cinv(csub(z, a)) : make_double2(0, 0);
#pragma unroll
      for (int q = 0; q < 5; ++q) T.b[q][t] = bdc[(long long)q * len + k];
    }
  }
  __syncthreads();
}

// Result of one barycentric Stokes evaluation.
struct DLPVal {
  double ux, uy, u1x, u1y, u2x, u2y;
};

// The coincident-node branch of laplaceExteriorHolomorphic (:5492-5506) for
// field q, evaluated from global memory (taken only when a target lies
// within 1e-10 of a source node).
__device__ double2 bary_coincident(const GeoDev& G, int start, int len, const double2* __restrict__ bdc, int q,
                                   int k, double2 zt, double2 a, double2& tmp1, double2& tmp2) {
  const double2 bk = bdc[(long long)q * len + k];
  const double2 zk = G.xy[start + k];
  for (int l = 0; l < len; ++l) {
    const double2 zl = G.xy[start + l], dzl = G.dz[start + l];
    const double2 bl = bdc[(long long)q * len + l];
    const double2 zla = csub(zl, a), zlt = csub(zl, zt);
    if (l != k) {
      double2 t = csub(cmul(bk, cdiv(csub(zk, a), zla)), bl);
      tmp1 = cadd(tmp1, cdiv(cmul(t, dzl), zlt));
    }
    tmp2 = cadd(tmp2, cmul(cinv(cmul(zla, zlt)), dzl));
  }
  const double2 dk = csub(zk, zt);
  double2 t = csub(cdiv(tmp1, tmp2), cmul(dk, bk));
  t = cdiv(t, cmul(dk, dk));
  t = cdiv(t, csub(zt, a));
  return cmul(t, G.dz[start + k]);
}

// Evaluates the Stokes DLP (and for NDER = 2 its gradient) of source curve c
// at the target zt.  All threads of the CTA call it for the same curve; the
// curve is streamed through shared memory three times (value, first and
// second derivative passes, :5190-5228 / :5468-5525).
template <int NDER>
__device__ DLPVal bary_eval(BaryTile& T, const GeoDev& G, int c, const double2* __restrict__ bdc, double2 zt,
                            bool act) {
  const int start = curve_start(G, c), len = curve_len(G, c);
  const bool ext = c != 0;
  double2 a = make_double2(0, 0);
  if (ext) a = G.cen[c - 1];
  // Pass 1: values.
  double2 den = make_double2(0, 0), num[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) num[q] = make_double2(0, 0);
  for (int k0 = 0; k0 < len; k0 += NEAR_TK) {
    bary_load_tile(T, G, start, len, k0, bdc, ext, a);
    const int kt = min(NEAR_TK, len - k0);
    for (int kk = 0; kk < kt; ++kk) {
      const double2 c1 = cmul(T.dz[kk], cinv(csub(T.z[kk], zt)));
      den = cadd(den, c1);
#pragma unroll
      for (int q = 0; q < 5; ++q) cfma(num[q], T.b[q][kk], c1);
    }
  }
  double2 u[5];
  {
    const double2 dd = ext ? make_double2(den.x, den.y - EB_TWOPI) : den;
    const double2 di = cinv(dd);
#pragma unroll
    for (int q = 0; q < 5; ++q) u[q] = cmul(num[q], di);
  }
  // Pass 2: first derivative.
  double2 den2 = make_double2(0, 0), num2[5];
#pragma unroll
  for (int q = 0; q < 5; ++q) num2[q] = make_double2(0, 0);
  bool coinc = false;
  for (int k0 = 0; k0 < len; k0 += NEAR_TK) {
    bary_load_tile(T, G, start, len, k0, bdc, ext, a);
    const int kt = min(NEAR_TK, len - k0);
    for (int kk = 0; kk < kt; ++kk) {
      const double2 d = csub(T.z[kk], zt);
      const double2 inv = cinv(d);
      const double2 c1 = cmul(T.dz[kk], inv);
      if (ext) {
        den2 = cadd(den2, cmul(c1, T.za[kk]));
        if (cabs2(d) <= 1e-20) { coinc = true; continue; }
      }
      const double2 c2 = cmul(c1, inv);
#pragma unroll
      for (int q = 0; q < 5; ++q) cfma(num2[q], csub(T.b[q][kk], u[q]), c2);
    }
  }
  if (ext && coinc && act) {
#pragma unroll 1
    for (int q = 0; q < 5; ++q) {
      double2 tmp1 = make_double2(0, 0), tmp2 = make_double2(0, 0);
      for (int k = 0; k < len; ++k) {
        const double2 d = csub(G.xy[start + k], zt);
        if (cabs2(d) <= 1e-20) num2[q] = cadd(num2[q], bary_coincident(G, start, len, bdc, q, k, zt, a, tmp1, tmp2));
      }
    }
  }
  double2 du[5];
  double2 fac;
  if (ext) fac = cinv(cmul(csub(zt, a), den2));
  else fac = cinv(den);
#pragma unroll
  for (int q = 0; q < 5; ++q) du[q] = cmul(num2[q], fac);
  DLPVal r;
  r.ux = du[0].x - zt.x * du[1].x - zt.y * du[2].x + u[3].x;
  r.uy = -du[0].y + zt.x * du[1].y + zt.y * du[2].y + u[4].x;
  r.u1x = r.u1y = r.u2x = r.u2y = 0.0;
  if (NDER == 2) {
    // Pass 3: second derivative.
    double2 num3[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) num3[q] = make_double2(0, 0);
    for (int k0 = 0; k0 < len; k0 += NEAR_TK) {
      bary_load_tile(T, G, start, len, k0, bdc, ext, a);
      const int kt = min(NEAR_TK, len - k0);
      for (int kk = 0; kk < kt; ++kk) {
        const double2 d = csub(T.z[kk], zt);
        const double2 inv = cinv(d);
        const double2 c3 = cmul(cmul(cmul(T.dz[kk], inv), inv), inv);
#pragma unroll
        for (int q = 0; q < 5; ++q) {
          double2 t = csub(csub(T.b[q][kk], u[q]), cmul(du[q], d));
          cfma(num3[q], t, c3);
        }
      }
    }
    double2 dd[5];
#pragma unroll
    for (int q = 0; q < 5; ++q) dd[q] = cscale(cmul(num3[q], fac), 2.0);
    r.u1x = dd[0].x - du[1].x - zt.x * dd[1].x - zt.y * dd[2].x + du[3].x;
    r.u1y = -dd[0].y + zt.x * dd[1].y - du[2].x + zt.y * dd[2].y - du[3].y;
    r.u2x = -dd[0].y + du[1].y + zt.x * dd[1].y + zt.y * dd[2].y + du[4].x;
    r.u2y = -dd[0].x + zt.x * dd[1].x + du[2].y + zt.y * dd[2].x - du[4].y;
  }
  return r;
}

// Near-pair list evaluation: CTA = (source s, pairs [p0, p1)), one thread per
// (target, source curve) pair.  Output: (ux, uy) per pair.
__global__ void __launch_bounds__(NEAR_NT)
k_bary_list(GeoDev G, const int4* __restrict__ work, const int* __restrict__ src_curve,
            const long long* __restrict__ bd_off, const double2* __restrict__ bd,
            const int* __restrict__ pair_tgt, const double2* __restrict__ txy, double2* __restrict__ out) {
  __shared__ BaryTile T;
  const int4 wk = work[blockIdx.x];
  const int s = wk.x, p0 = wk.y, p1 = wk.z;
  const int c = src_curve[s];
  const int p = p0 + threadIdx.x;
  const bool act = p < p1;
  const double2 zt = txy[pair_tgt[act ? p : p1 - 1]];
  DLPVal r = bary_eval<1>(T, G, c, bd + bd_off[s], zt, act);
  if (act) out[p] = make_double2(r.ux, r.uy);
}

// ---------------------------------------------------------------------------
// Assembles the boundary operator for every node: far-field partial sums,
// barycentric pairs (in a fixed order per target), the diagonal curvature
// limit and jump (:937-951, :964-985), stokeslets and rotlets of every body
// (:992-1049) and the wall's rank-one term (:1115-1118).
// COMBINE_G consecutive threads share one node: they split the partial-sum
// slots, the near pairs and the bodies of the stokeslet/rotlet sum, and their
// sums meet by warp shuffles (launch nblk(N * COMBINE_G, 256) CTAs of 256).
constexpr int SR_CHUNK = 256;
constexpr int COMBINE_G = 4;
__global__ void __launch_bounds__(256)
k_combine(GeoDev G, const double* __restrict__ den, const double2* __restrict__ partial, int nsplit,
          const int* __restrict__ tptr, const int* __restrict__ tpairs, const double2* __restrict__ pair_out,
          const double* __restrict__ sigdotn, const double2* __restrict__ selfp, int nself, int nself_body,
          double* __restrict__ vel) {
  __shared__ double4 sc[SR_CHUNK];   // cx, cy, stokeslet x, stokeslet y
  __shared__ double sr[SR_CHUNK];    // rotlet
  const long long tid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int g = (int)(tid / COMBINE_G), sub = (int)(tid % COMBINE_G);
  const bool act = g < G.N;
  const int gc = act ? g : G.N - 1;
  const double2 p = G.xy[gc];
  double ux = 0.0, uy = 0.0;
  for (int q = sub; q < nsplit; q += COMBINE_G) {
    double2 v = partial[(size_t)q * G.N + gc];
    ux += v.x; uy += v.y;
  }
  if (selfp) {
    const int ns = gc < G.nout ? nself : nself_body;
    for (int q = sub; q < ns; q += COMBINE_G) {
      double2 v = selfp[(size_t)q * G.N + gc];
      ux += v.x; uy += v.y;
    }
  }
  if (tptr) {
    for (int e = tptr[gc] + sub; e < tptr[gc + 1]; e += COMBINE_G) {
      double2 v = pair_out[tpairs[e]];
      ux += v.x; uy += v.y;
    }
  }
  for (int b0 = 0; b0 < G.M; b0 += SR_CHUNK) {
    __syncthreads();
    for (int t = threadIdx.x; t < SR_CHUNK; t += blockDim.x) {
      int b = b0 + t;
      if (b < G.M) {
        double2 cc = G.cen[b];
        sc[t] = make_double4(cc.x, cc.y, den[ic_of(G, b, 0)], den[ic_of(G, b, 1)]);
        sr[t] = den[ic_of(G, b, 2)];
      }
    }
    __syncthreads();
    const int bt = min(SR_CHUNK, G.M - b0);
    for (int t = sub; t < bt; t += COMBINE_G) {
      const double4 q = sc[t];
      const double rot = sr[t];
      const double rx = p.x - q.x, ry = p.y - q.y;
      const double rho2 = rx * rx + ry * ry;
      const double rd = rx * q.z + ry * q.w;
      const double lg = log(rho2);
      const double ir = 1.0 / rho2;
      ux += 0.5 / EB_TWOPI * (-0.5 * lg * q.z + rd * ir * rx) + rot * ry * ir;
      uy += 0.5 / EB_TWOPI * (-0.5 * lg * q.w + rd * ir * ry) - rot * rx * ir;
    }
  }
#pragma unroll
  for (int o = 1; o < COMBINE_G; o <<= 1) {
    ux += __shfl_xor_sync(0xffffffffu, ux, o);
    uy += __shfl_xor_sync(0xffffffffu, uy, o);
  }
  if (!act || sub != 0) return;
  const long long ixg = ix_of(G, gc), iyg = iy_of(G, gc);
  const double sx = den[ixg], sy = den[iyg];
  const double2 nn = G.nrm[gc];
  const double cu = G.cur[gc], s = G.sp[gc];
  const int nc = gc < G.nout ? G.nout : G.n;
  const double tdd = nn.y * sx - nn.x * sy;
  ux = ux - cu * tdd * nn.y * s / nc;
  uy = uy + cu * tdd * nn.x * s / nc;
  ux -= 0.5 * sx;
  uy -= 0.5 * sy;
  if (gc < G.nout) {
    const double sg = *sigdotn;
    ux += sg * nn.x;
    uy += sg * nn.y;
  }
  vel[ixg] = ux;
  vel[iyg] = uy;
}

// Right-hand side of bd_condition (:208-314).
__global__ void k_rhs(GeoDev G, int ibc, int mode, double wall_b, double* __restrict__ rhs) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < G.M * 3) rhs[2LL * G.nout + 2LL * G.n * G.M + g] = 0.0;
  if (g >= G.N) return;
  const double2 p = G.xy[g];
  double u = 0.0, v = 0.0;
  if (mode == 2) {
    u = 0.0;   // homogeneous data (used to exercise the zero right-hand-side path)
  } else if (mode == 1) {
    const double s1 = 1.0, s2 = 2.0, rot = 3.0;
    double rx = p.x, ry = p.y, rd = rx * s1 + ry * s2, rho2 = rx * rx + ry * ry;
    u = 0.5 / EB_TWOPI * (-0.5 * log(rho2) * s1 + rd / rho2 * rx) + rot * ry / rho2;
    v = 0.5 / EB_TWOPI * (-0.5 * log(rho2) * s2 + rd / rho2 * ry) - rot * rx / rho2;
  } else if (g < G.nout) {
    if (ibc == 0) u = (1.0 + p.y / wall_b) * (1.0 - p.y / wall_b);
    else u = 1.0;
  }
  rhs[ix_of(G, g)] = u;
  rhs[iy_of(G, g)] = v;
}

// ---------------------------------------------------------------------------
// Krylov kernels (tall-skinny products with the basis V, row-major by vector).

// part[j*gridDim.x + blk] = sum over this CTA's rows of V[j] . w, for j < k.
// A warp takes four columns at a time (four independent load streams); each
// column's sum runs in the same order as one column at a time would.
__device__ __forceinline__ void dot_cols_cta(const double* __restrict__ V, long long ldv, int k,
                                             const double* __restrict__ w, long long n, int R,
                                             double* __restrict__ part, double* swv) {
  const long long r0 = (long long)blockIdx.x * R;
  const int rl = (int)max(0LL, min((long long)R, n - r0));
  for (int t = threadIdx.x; t < rl; t += blockDim.x) swv[t] = w[r0 + t];
  __syncthreads();
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (int j0 = 4 * wid; j0 < k; j0 += 4 * nw) {
    const int jn = min(4, k - j0);
    const double* __restrict__ v0 = V + (long long)j0 * ldv + r0;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    if (jn == 4) {
      for (int t = lane; t < rl; t += 32) {
        const double wt = swv[t];
        s0 = fma(__ldg(v0 + t), wt, s0);
        s1 = fma(__ldg(v0 + ldv + t), wt, s1);
        s2 = fma(__ldg(v0 + 2 * ldv + t), wt, s2);
        s3 = fma(__ldg(v0 + 3 * ldv + t), wt, s3);
      }
    } else {
      for (int t = lane; t < rl; t += 32) {
        const double wt = swv[t];
        s0 = fma(__ldg(v0 + t), wt, s0);
        if (jn > 1) s1 = fma(__ldg(v0 + ldv + t), wt, s1);
        if (jn > 2) s2 = fma(__ldg(v0 + 2 * ldv + t), wt, s2);
      }
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    s2 = warp_sum(s2);
    s3 = warp_sum(s3);
    if (lane == 0) {
      double* pj = part + (size_t)j0 * gridDim.x + blockIdx.x;
      pj[0] = s0;
      if (jn > 1) pj[gridDim.x] = s1;
      if (jn > 2) pj[2 * (size_t)gridDim.x] = s2;
      if (jn > 3) pj[3 * (size_t)gridDim.x] = s3;
    }
  }
}

__global__ void __launch_bounds__(256)
k_dot_part(const double* __restrict__ V, long long ldv, int k, const double* __restrict__ w, long long n,
           int R, double* __restrict__ part) {
  extern __shared__ double swv[];
  dot_cols_cta(V, ldv, k, w, n, R, part, swv);
}

// h[j] (+)= sum_b part[j][b]; one warp per j.
__global__ void k_dot_reduce(const double* __restrict__ part, int nb, int k, double* __restrict__ h, int accumulate) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= k) return;
  double s = 0.0;
  for (int b = lane; b < nb; b += 32) s += part[(size_t)j * nb + b];
  s = warp_sum(s);
  if (lane == 0) h[j] = accumulate ? h[j] + s : s;
}

// w[i] += sign * sum_j V[j][i] h[j]
__global__ void __launch_bounds__(256)
k_vh(const double* __restrict__ V, long long ldv, int k, const double* __restrict__ h, double sign,
     double* __restrict__ w, long long n) {
  __shared__ double sh[1024];
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  for (int j0 = 0; j0 < k; j0 += 1024) {
    const int jt = min(1024, k - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < jt; t += blockDim.x) sh[t] = h[j0 + t];
    __syncthreads();
    if (i < n) {
      const double* __restrict__ vp = V + (long long)j0 * ldv + i;
      int j = 0;
      double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0;
      for (; j + 7 < jt; j += 8) {   // eight independent loads in flight
        a0 = fma(__ldg(vp + (long long)(j)*ldv), sh[j], a0);
        a1 = fma(__ldg(vp + (long long)(j + 1) * ldv), sh[j + 1], a1);
        a2 = fma(__ldg(vp + (long long)(j + 2) * ldv), sh[j + 2], a2);
        a3 = fma(__ldg(vp + (long long)(j + 3) * ldv), sh[j + 3], a3);
        a4 = fma(__ldg(vp + (long long)(j + 4) * ldv), sh[j + 4], a4);
        a5 = fma(__ldg(vp + (long long)(j + 5) * ldv), sh[j + 5], a5);
        a6 = fma(__ldg(vp + (long long)(j + 6) * ldv), sh[j + 6], a6);
        a7 = fma(__ldg(vp + (long long)(j + 7) * ldv), sh[j + 7], a7);
      }
      for (; j < jt; ++j) a0 = fma(__ldg(vp + (long long)j * ldv), sh[j], a0);
      acc += ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    }
  }
  if (i < n) w[i] += sign * acc;
}

__global__ void k_scale(double* __restrict__ v, double a, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) v[i] *= a;
}

// r = b - r
__global__ void k_bminus(const double* __restrict__ b, double* __restrict__ r, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) r[i] = b[i] - r[i];
}

// y += a x
__global__ void k_axpy(double a, const double* __restrict__ x, double* __restrict__ y, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}

// out = a (copy) — used to seed the basis from a residual.
__global__ void k_copy(const double* __restrict__ a, double* __restrict__ out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = a[i];
}

// ---------------------------------------------------------------------------
// Arnoldi steps whose column count lives in device memory (*kp), so that one
// captured CUDA graph serves every iteration of a GMRES cycle.

// out = V[:, *kp + off]
__global__ void k_col_get(const double* __restrict__ V, long long ldv, const int* __restrict__ kp, int off,
                          double* __restrict__ out, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = V[(long long)(*kp + off) * ldv + i];
}

// V[:, *kp + off] = in (times *scale when scale is given)
__global__ void k_col_put(double* __restrict__ V, long long ldv, const int* __restrict__ kp, int off,
                          const double* __restrict__ in, const double* __restrict__ scale, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) V[(long long)(*kp + off) * ldv + i] = scale ? in[i] * *scale : in[i];
}

// part[j][b] = partial dot of columns j < *kp with w over the rows of block b
__global__ void __launch_bounds__(256)
k_dot_part_dk(const double* __restrict__ V, long long ldv, const int* __restrict__ kp, const double* __restrict__ w,
              long long n, int R, double* __restrict__ part) {
  extern __shared__ double swv[];
  dot_cols_cta(V, ldv, *kp, w, n, R, part, swv);
}

// h[j] = sum_b part[j][b] for j < *kp (+ koff); one warp per j, grid-stride.
__global__ void k_dot_reduce_dk(const double* __restrict__ part, int nb, const int* __restrict__ kp, int koff,
                                double* __restrict__ h) {
  const int k = *kp + koff;
  const int lane = threadIdx.x & 31;
  for (int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); j < k; j += gridDim.x * (blockDim.x >> 5)) {
    double a = 0.0;
    for (int b = lane; b < nb; b += 32) a += part[(size_t)j * nb + b];
    a = warp_sum(a);
    if (lane == 0) h[j] = a;
  }
}

// w += sign * V[:, 0:*kp] h
__global__ void __launch_bounds__(256)
k_vh_dk(const double* __restrict__ V, long long ldv, const int* __restrict__ kp, const double* __restrict__ h,
        double sign, double* __restrict__ w, long long n) {
  __shared__ double sh[1024];
  const int k = *kp;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double acc = 0.0;
  for (int j0 = 0; j0 < k; j0 += 1024) {
    const int jt = min(1024, k - j0);
    __syncthreads();
    for (int t = threadIdx.x; t < jt; t += blockDim.x) sh[t] = h[j0 + t];
    __syncthreads();
    if (i < n) {
      const double* __restrict__ vp = V + (long long)j0 * ldv + i;
      int j = 0;
      double a0 = 0, a1 = 0, a2 = 0, a3 = 0, a4 = 0, a5 = 0, a6 = 0, a7 = 0;
      for (; j + 7 < jt; j += 8) {   // eight independent loads in flight
        a0 = fma(__ldg(vp + (long long)(j)*ldv), sh[j], a0);
        a1 = fma(__ldg(vp + (long long)(j + 1) * ldv), sh[j + 1], a1);
        a2 = fma(__ldg(vp + (long long)(j + 2) * ldv), sh[j + 2], a2);
        a3 = fma(__ldg(vp + (long long)(j + 3) * ldv), sh[j + 3], a3);
        a4 = fma(__ldg(vp + (long long)(j + 4) * ldv), sh[j + 4], a4);
        a5 = fma(__ldg(vp + (long long)(j + 5) * ldv), sh[j + 5], a5);
        a6 = fma(__ldg(vp + (long long)(j + 6) * ldv), sh[j + 6], a6);
        a7 = fma(__ldg(vp + (long long)(j + 7) * ldv), sh[j + 7], a7);
      }
      for (; j < jt; ++j) a0 = fma(__ldg(vp + (long long)j * ldv), sh[j], a0);
      acc += ((a0 + a1) + (a2 + a3)) + ((a4 + a5) + (a6 + a7));
    }
  }
  if (i < n) w[i] += sign * acc;
}

// The Givens step of one Arnoldi iteration on the device (DHEQR,
// gmres_routines.f:1148, last column).  Column k = *kp of the Hessenberg
// matrix is h1[0..k-1] + h2[0..k-1] (the two Gram-Schmidt passes) with
// subdiagonal sqrt(*hn); the previous rotations (cs[2i], cs[2i+1]) are applied,
// a new rotation zeroes the subdiagonal, the column is stored packed in R
// (column k-1 at offset (k-1)k/2), prod <- prod * s and rho = |prod r0|.
// scale <- 1/sqrt(hn) for the next basis vector.  st: 0 running, 2 breakdown
// (zero diagonal), 3 non-finite.  One thread.
__global__ void k_givens_step(const int* __restrict__ kp, const double* __restrict__ h1,
                              const double* __restrict__ h2, const double* __restrict__ hn, double* __restrict__ cs,
                              double* __restrict__ R, double* __restrict__ prod, const double* __restrict__ r0,
                              double* __restrict__ rho, double* __restrict__ scale, int* __restrict__ st) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const int k = *kp;
  double* col = R + (size_t)(k - 1) * k / 2;
  const double snormw = sqrt(*hn);
  bool finite = isfinite(snormw);
  for (int i = 0; i < k; ++i) {
    col[i] = h1[i] + h2[i];
    finite = finite && isfinite(col[i]);
  }
  if (!finite) { *st = 3; return; }
  for (int kk = 0; kk < k - 1; ++kk) {
    const double c = cs[2 * kk], sn = cs[2 * kk + 1];
    const double t1 = col[kk], t2 = col[kk + 1];
    col[kk] = c * t1 - sn * t2;
    col[kk + 1] = sn * t1 + c * t2;
  }
  const double t1 = col[k - 1], t2 = snormw;
  double c, sn;
  if (t2 == 0.0) { c = 1.0; sn = 0.0; }
  else if (fabs(t2) >= fabs(t1)) { const double t = t1 / t2; sn = -1.0 / sqrt(1.0 + t * t); c = -sn * t; }
  else { const double t = t2 / t1; c = 1.0 / sqrt(1.0 + t * t); sn = -c * t; }
  cs[2 * (k - 1)] = c;
  cs[2 * (k - 1) + 1] = sn;
  col[k - 1] = c * t1 - sn * t2;
  if (col[k - 1] == 0.0) { *st = 2; return; }
  *prod *= sn;
  *rho = fabs(*prod * *r0);
  *scale = snormw > 0.0 ? 1.0 / snormw : 0.0;
  *st = 0;
}

__global__ void k_inc(int* kp) {
  if (threadIdx.x == 0 && blockIdx.x == 0) *kp += 1;
}

}  // namespace
