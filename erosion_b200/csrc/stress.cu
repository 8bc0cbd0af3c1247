// Wall shear stress on the bodies (computeShearStress, stokesSolver.f:3002-3096)
// and velocity/pressure/vorticity at target points (computeQoiTargets,
// :3099-3323).
#include "state.h"
#include "kernels.cuh"
#include <cmath>

namespace eb {

// Offset of curve c's five boundary-value fields in the all-curves buffer.
__device__ __forceinline__ long long bd_all_off(const GeoDev& G, int c) {
  return c == 0 ? 0LL : 5LL * G.nout + 5LL * (c - 1) * G.n;
}

// Barycentric Stokes DLP (NDER = 2: with gradient) of the source curves
// [split_c[y], split_c[y+1]) at the targets of this CTA's task, skipping the
// task's own curve.  Partial sums per split: out[(y*6 + q)*ntar + t] with
// q = ux, uy, u1x, u1y, u2x, u2y.
template <int NDER>
__global__ void __launch_bounds__(NEAR_NT)
k_bary_sum(GeoDev G, const double2* __restrict__ bd_all, const int4* __restrict__ tasks,
           const double2* __restrict__ txy, const int* __restrict__ split_c, int ntar, double* __restrict__ out) {
  __shared__ BaryTile T;
  const int4 tk = tasks[blockIdx.x];
  const int split = blockIdx.y;
  const int t = tk.x + threadIdx.x;
  const bool act = t < tk.y;
  const double2 zt = txy[act ? t : tk.y - 1];
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int c = split_c[split]; c < split_c[split + 1]; ++c) {
    if (c == tk.z) continue;
    DLPVal r = bary_eval<NDER>(T, G, c, bd_all + bd_all_off(G, c), zt, act);
    a[0] += r.ux; a[1] += r.uy; a[2] += r.u1x; a[3] += r.u1y; a[4] += r.u2x; a[5] += r.u2y;
  }
  if (act) {
#pragma unroll
    for (int q = 0; q < 6; ++q) out[((size_t)split * 6 + q) * ntar + t] = a[q];
  }
}

// Self-interaction of each body for the deformation tensor: the odd-even
// trapezoid rule on the subtracted density (:2744-2833) plus the jump term
// from the spectral tangential derivative of sigma (:2933-2958).  One CTA per
// body; out[3][n*M] = E11, E12, E22.
__global__ void __launch_bounds__(256)
k_stress_self(GeoDev G, const double* __restrict__ den, const double* __restrict__ dk, double* __restrict__ out) {
  extern __shared__ double sm[];
  const int n = G.n, b = blockIdx.x, nb = G.n * G.M;
  double* sx = sm;
  double* sy = sm + n;
  double* xs = sm + 2 * n;
  double* ys = sm + 3 * n;
  double* pxs = sm + 4 * n;
  double* pys = sm + 5 * n;
  double* ws = sm + 6 * n;
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    int g = G.nout + b * n + k;
    sx[k] = den[ix_of(G, g)];
    sy[k] = den[iy_of(G, g)];
    double2 p = G.xy[g], nn = G.nrm[g];
    xs[k] = p.x; ys[k] = p.y; pxs[k] = nn.x; pys[k] = nn.y;
    ws[k] = G.w[g];
  }
  __syncthreads();
  for (int k = threadIdx.x; k < n; k += blockDim.x) {
    double e11 = 0, e12 = 0, e22 = 0;
    const double xk = xs[k], yk = ys[k], sxk = sx[k], syk = sy[k];
    for (int j = (k & 1) ? 0 : 1; j < n; j += 2) {
      double rx = xk - xs[j], ry = yk - ys[j];
      double rho2 = rx * rx + ry * ry;
      double ir2 = 1.0 / rho2;
      double ir4 = ir2 * ir2, ir6 = ir4 * ir2;
      double px = pxs[j], py = pys[j];
      double rdotn = rx * px + ry * py;
      double routn = rx * py + ry * px;
      double ssx = sx[j] - sxk, ssy = sy[j] - syk;
      double rdots = rx * ssx + ry * ssy;
      double routs = rx * ssy + ry * ssx;
      double wg = ws[j];
      e11 += 2.0 * 0.5 * (2.0 * rdotn * rdots * ir4 + 2.0 * rdots * ir4 * rx * px + 2.0 * rdotn * ir4 * rx * ssx -
                          8.0 * rdotn * rdots * ir6 * rx * rx) * wg;
      e12 += 2.0 * 0.5 * (rdots * routn * ir4 + rdotn * routs * ir4 - 8.0 * rdotn * rdots * rx * ry * ir6) * wg;
      e22 += 2.0 * 0.5 * (2.0 * rdotn * rdots * ir4 + 2.0 * rdots * ir4 * ry * py + 2.0 * rdotn * ir4 * ry * ssy -
                          8.0 * rdotn * rdots * ir6 * ry * ry) * wg;
    }
    // jump: t = (-py, px) at the target, d(sigma)/ds . t
    double dx = 0, dy = 0;
    for (int j = 0; j < n; ++j) {
      int m = k - j;
      if (m < 0) m += n;
      double d = __ldg(dk + m);
      dx = fma(d, sx[j], dx);
      dy = fma(d, sy[j], dy);
    }
    const int g = G.nout + b * n + k;
    const double spk = G.sp[g];
    const double tx = -pys[k], ty = pxs[k];
    const double dd = (dx / spk) * tx + (dy / spk) * ty;
    e11 += 0.5 * dd * (tx * tx - ty * ty);
    e12 += 0.5 * dd * 2.0 * tx * ty;
    e22 += 0.5 * dd * (-tx * tx + ty * ty);
    const int i = b * n + k;
    out[i] = e11;
    out[nb + i] = e12;
    out[2 * nb + i] = e22;
  }
}

// Trapezoid deformation tensor of every other curve (deformation_on_boundary_trap,
// :2350-2384 for the wall and :2496-2543 for the bodies), as partial sums
// over the far-field tile splits.  out[(split*3 + q)*nb + i].
__global__ void __launch_bounds__(256)
k_stress_trap(GeoDev G, const double* __restrict__ den, const int4* __restrict__ tiles,
              const int* __restrict__ split_ptr, double* __restrict__ out) {
  __shared__ double2 sxy[FAR_TS], sn[FAR_TS], ss[FAR_TS];
  __shared__ double sw[FAR_TS];
  const int nb = G.n * G.M;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < nb;
  const int ic = act ? i : nb - 1;
  const int g = G.nout + ic;
  const int mycurve = 1 + ic / G.n;
  const double2 p = G.xy[g];
  double e11 = 0, e12 = 0, e22 = 0;
  const int split = blockIdx.y;
  for (int ti = split_ptr[split]; ti < split_ptr[split + 1]; ++ti) {
    const int4 T = tiles[ti];
    __syncthreads();
    if (threadIdx.x < T.y) {
      int gs = T.x + threadIdx.x;
      sxy[threadIdx.x] = G.xy[gs];
      sn[threadIdx.x] = G.nrm[gs];
      ss[threadIdx.x] = make_double2(den[ix_of(G, gs)], den[iy_of(G, gs)]);
      sw[threadIdx.x] = G.w[gs];
    }
    __syncthreads();
    if (T.z == mycurve) continue;
    double a11 = 0, a12 = 0, a22 = 0;
    for (int j = 0; j < T.y; ++j) {
      const double2 q = sxy[j], nn = sn[j], s = ss[j];
      double rx = p.x - q.x, ry = p.y - q.y;
      double rho2 = rx * rx + ry * ry;
      double ir2 = 1.0 / rho2, ir4 = ir2 * ir2, ir6 = ir4 * ir2;
      double rdotn = rx * nn.x + ry * nn.y;
      double routn = rx * nn.y + ry * nn.x;
      double rdotden = rx * s.x + ry * s.y;
      double routden = rx * s.y + ry * s.x;
      double wg = sw[j];
      a11 += 0.5 * (2.0 * rdotn * rdotden * ir4 + 2.0 * rdotden * ir4 * rx * nn.x + 2.0 * rdotn * ir4 * rx * s.x -
                    8.0 * rdotn * rdotden * ir6 * rx * rx) * wg;
      a12 += 0.5 * (rdotden * routn * ir4 + rdotn * routden * ir4 - 8.0 * rdotn * rdotden * rx * ry * ir6) * wg;
      a22 += 0.5 * (2.0 * rdotn * rdotden * ir4 + 2.0 * rdotden * ir4 * ry * nn.y + 2.0 * rdotn * ir4 * ry * s.y -
                    8.0 * rdotn * rdotden * ir6 * ry * ry) * wg;
    }
    e11 += a11; e12 += a12; e22 += a22;
  }
  if (act) {
    out[((size_t)split * 3 + 0) * nb + i] = e11;
    out[((size_t)split * 3 + 1) * nb + i] = e12;
    out[((size_t)split * 3 + 2) * nb + i] = e22;
  }
}

// ---- Shear stress with the trapezoid rule wherever it is exact to rounding.
// The reference evaluates every other curve's contribution to a body node by
// the barycentric formulas (deformation_on_boundary, :2707-2727 and
// :2893-2925).  Away from a source curve the trapezoid rule on the same
// density gives the same value up to its quadrature (aliasing) error, which
// for a density with content up to the Nyquist mode decays like
// exp(-pi d / h) with the distance d to the curve and its node spacing h:
// beyond d = STRESS_NEAR_H h it is below 1e-16 of the value.  So the
// barycentric evaluation runs only on the (body node, source curve) pairs
// within that distance, and the trapezoid rule (FP64) on all the others.
constexpr double STRESS_NEAR_H = 12.0;

// Per body node: min over wall nodes j of |x_i - x_j|^2 / h_j^2, with h_j the
// local wall spacing |z'_j| 2 pi / nout.  Wall nodes staged through shared
// memory in chunks.
__global__ void __launch_bounds__(256)
k_stress_wall_dist(GeoDev G, double* __restrict__ d2h) {
  __shared__ double2 sxy[256];
  __shared__ double sh2[256];
  const int nb = G.n * G.M;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double2 p = G.xy[G.nout + (i < nb ? i : nb - 1)];
  const double hs = EB_TWOPI / G.nout;
  double best = 1e300;
  for (int j0 = 0; j0 < G.nout; j0 += 256) {
    __syncthreads();
    const int j = j0 + threadIdx.x;
    if (j < G.nout) {
      sxy[threadIdx.x] = G.xy[j];
      const double h = G.sp[j] * hs;
      sh2[threadIdx.x] = 1.0 / (h * h);
    }
    __syncthreads();
    const int jt = min(256, G.nout - j0);
    for (int k = 0; k < jt; ++k) {
      const double dx = p.x - sxy[k].x, dy = p.y - sxy[k].y;
      best = fmin(best, (dx * dx + dy * dy) * sh2[k]);
    }
  }
  if (i < nb) d2h[i] = best;
}

// Per body: radius of the smallest centroid-centred disc holding its nodes,
// and its node spacing (mean speed x 2 pi / n).
__global__ void __launch_bounds__(256)
k_body_extent(GeoDev G, double2* __restrict__ ext) {
  __shared__ double red[32];
  const int b = blockIdx.x;
  const double2 c = G.cen[b];
  double r = 0.0;
  for (int k = threadIdx.x; k < G.n; k += blockDim.x) {
    const double2 p = G.xy[G.nout + b * G.n + k];
    r = fmax(r, sqrt((p.x - c.x) * (p.x - c.x) + (p.y - c.y) * (p.y - c.y)));
  }
  // block max: within each warp, then across the warps
  for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = r;
  __syncthreads();
  if (threadIdx.x < 32) {
    r = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) r = fmax(r, __shfl_xor_sync(0xffffffffu, r, o));
    if (threadIdx.x == 0) ext[b] = make_double2(r, G.rb[b] * EB_TWOPI / G.n);
  }
}

// Near mask of the stress: bit c of mask[i * mw + c/32] is set when body node
// i lies within STRESS_NEAR_H node spacings of source curve c (its own body
// excluded): for the wall from k_stress_wall_dist, for a body by its bounding
// disc.
__global__ void __launch_bounds__(256)
k_stress_near_mask(GeoDev G, const double* __restrict__ wall_d2h, const double2* __restrict__ ext, int mw,
                   unsigned* __restrict__ mask) {
  const int nb = G.n * G.M;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nb) return;
  const int own = 1 + i / G.n;
  const double2 p = G.xy[G.nout + i];
  for (int w = 0; w < mw; ++w) {
    unsigned bits = 0u;
    for (int q = 0; q < 32; ++q) {
      const int c = 32 * w + q;
      if (c > G.M) break;
      bool near;
      if (c == 0) {
        near = wall_d2h[i] <= STRESS_NEAR_H * STRESS_NEAR_H;
      } else if (c == own) {
        near = false;
      } else {
        const double2 cc = G.cen[c - 1], e = ext[c - 1];
        const double R = e.x + STRESS_NEAR_H * e.y;
        const double dx = p.x - cc.x, dy = p.y - cc.y;
        near = dx * dx + dy * dy <= R * R;
      }
      if (near) bits |= 1u << q;
    }
    mask[(size_t)i * mw + w] = bits;
  }
}

// Barycentric Stokes DLP gradient of the near source curves only: CTA = task
// (up to NEAR_NT nodes of one body); the CTA visits, in curve order, every
// curve that is near for at least one of its nodes, and a node keeps the
// value only for the curves near to it.  out[q * nb + i], q as k_bary_sum
// (one split).
__global__ void __launch_bounds__(NEAR_NT)
k_bary_sum_near(GeoDev G, const double2* __restrict__ bd_all, const int4* __restrict__ tasks,
                const unsigned* __restrict__ mask, int mw, double* __restrict__ out) {
  __shared__ BaryTile T;
  __shared__ unsigned tmask;
  const int nb = G.n * G.M;
  const int4 tk = tasks[blockIdx.x];
  const int t = tk.x + threadIdx.x;
  const bool act = t < tk.y;
  const int tc = act ? t : tk.y - 1;
  const double2 zt = G.xy[G.nout + tc];
  double a[6] = {0, 0, 0, 0, 0, 0};
  for (int w = 0; w < mw; ++w) {
    const unsigned my = act ? mask[(size_t)tc * mw + w] : 0u;
    __syncthreads();
    if (threadIdx.x == 0) tmask = 0u;
    __syncthreads();
    const unsigned wor = __reduce_or_sync(0xffffffffu, my);
    if ((threadIdx.x & 31) == 0 && wor) atomicOr(&tmask, wor);
    __syncthreads();
    unsigned bits = tmask;   // block-uniform
    while (bits) {
      const int q = __ffs(bits) - 1;
      bits &= bits - 1u;
      const int c = 32 * w + q;
      DLPVal r = bary_eval<2>(T, G, c, bd_all + bd_all_off(G, c), zt, act);
      if ((my >> q) & 1u) {
        a[0] += r.ux; a[1] += r.uy; a[2] += r.u1x; a[3] += r.u1y; a[4] += r.u2x; a[5] += r.u2y;
      }
    }
  }
  if (act) {
#pragma unroll
    for (int q = 0; q < 6; ++q) out[(size_t)q * nb + t] = a[q];
  }
}

// Per body: the speed-weighted rigid part of its density, sigma_rigid(x) =
// (t1, t2) + t3 (-(y - yb), x - xb) with (xb, yb) the speed-weighted centroid
// (the split k_prep makes for the far field), as rig[5 b + (0..4)] = t1, t2,
// t3, xb, yb.
__global__ void __launch_bounds__(256)
k_stress_rigid(GeoDev G, const double* __restrict__ den, double* __restrict__ rig) {
  __shared__ double sh[32];
  const int b = blockIdx.x, start = G.nout + b * G.n;
  double a0 = 0, a1 = 0, s0 = 0, sxw = 0, syw = 0;
  for (int j = threadIdx.x; j < G.n; j += blockDim.x) {
    const int g = start + j;
    const double sp = G.sp[g];
    const double2 p = G.xy[g];
    a0 += den[ix_of(G, g)] * sp;
    a1 += den[iy_of(G, g)] * sp;
    s0 += sp;
    sxw += sp * p.x;
    syw += sp * p.y;
  }
  a0 = block_sum<256>(a0, sh);
  a1 = block_sum<256>(a1, sh);
  s0 = block_sum<256>(s0, sh);
  sxw = block_sum<256>(sxw, sh);
  syw = block_sum<256>(syw, sh);
  const double xb = sxw / s0, yb = syw / s0;
  double r0 = 0, r1 = 0;
  for (int j = threadIdx.x; j < G.n; j += blockDim.x) {
    const int g = start + j;
    const double sp = G.sp[g];
    const double2 p = G.xy[g];
    const double fx = -(p.y - yb), fy = p.x - xb;
    r0 += sp * (fx * den[ix_of(G, g)] + fy * den[iy_of(G, g)]);
    r1 += sp * (fx * fx + fy * fy);
  }
  r0 = block_sum<256>(r0, sh);
  r1 = block_sum<256>(r1, sh);
  if (threadIdx.x == 0) {
    rig[5 * b] = a0 / s0;
    rig[5 * b + 1] = a1 / s0;
    rig[5 * b + 2] = r1 > 0 ? r0 / r1 : 0.0;
    rig[5 * b + 3] = xb;
    rig[5 * b + 4] = yb;
  }
}

// Trapezoid deformation tensor of every other curve except the near ones
// (mask as k_stress_near_mask), as partial sums over the far-field tile
// splits: out[(split*3 + q)*nb + i].  The same terms as k_stress_trap, the
// density scaled by the weight when staged and the reciprocal by
// rcp_newton.  A source body's density enters without its rigid part
// (k_stress_rigid): a rigid-motion density has no exterior double layer, and
// at these distances the trapezoid rule's value for it is below 1e-16 of its
// size, while the rigid parts (large for the smallest bodies) would otherwise
// set the rounding error of the sum.
__global__ void __launch_bounds__(256)
k_stress_far(GeoDev G, const double* __restrict__ den, const int4* __restrict__ tiles,
             const int* __restrict__ split_ptr, const unsigned* __restrict__ mask, int mw,
             const double* __restrict__ rig, double* __restrict__ out) {
  __shared__ double4 sg[FAR_TS];   // x, y, nx, ny
  __shared__ double2 ss[FAR_TS];   // w sigma
  const int nb = G.n * G.M;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < nb;
  const int ic = act ? i : nb - 1;
  const int g = G.nout + ic;
  const int mycurve = 1 + ic / G.n;
  const double2 p = G.xy[g];
  double e11 = 0, e12 = 0, e22 = 0;
  const int split = blockIdx.y;
  for (int ti = split_ptr[split]; ti < split_ptr[split + 1]; ++ti) {
    const int4 T = tiles[ti];
    __syncthreads();
    for (int k = threadIdx.x; k < T.y; k += blockDim.x) {
      const int gs = T.x + k;
      const double2 q = G.xy[gs], nn = G.nrm[gs];
      const double wg = G.w[gs];
      sg[k] = make_double4(q.x, q.y, nn.x, nn.y);
      double sx = den[ix_of(G, gs)], sy = den[iy_of(G, gs)];
      if (T.z > 0) {
        const double* R = rig + 5 * (T.z - 1);
        sx -= R[0] - R[2] * (q.y - R[4]);
        sy -= R[1] + R[2] * (q.x - R[3]);
      }
      ss[k] = make_double2(sx * wg, sy * wg);
    }
    __syncthreads();
    if (T.z == mycurve || ((__ldg(mask + (size_t)ic * mw + (T.z >> 5)) >> (T.z & 31)) & 1u)) continue;
    double a11 = 0, a12 = 0, a22 = 0;
#pragma unroll 2
    for (int j = 0; j < T.y; ++j) {
      const double4 q = sg[j];
      const double2 sd = ss[j];
      const double rx = p.x - q.x, ry = p.y - q.y;
      const double inv = rcp_newton(fma(rx, rx, ry * ry));
      const double i4 = inv * inv;
      const double rdn = fma(rx, q.z, ry * q.w), rtn = fma(rx, q.w, ry * q.z);
      const double rds = fma(rx, sd.x, ry * sd.y), rts = fma(rx, sd.y, ry * sd.x);
      const double A = rdn * rds * i4;
      const double C = 4.0 * A * inv;
      a11 += A + i4 * rx * fma(rds, q.z, rdn * sd.x) - C * rx * rx;
      a22 += A + i4 * ry * fma(rds, q.w, rdn * sd.y) - C * ry * ry;
      a12 += 0.5 * i4 * fma(rds, rtn, rdn * rts) - C * rx * ry;
    }
    e11 += a11; e12 += a12; e22 += a22;
  }
  if (act) {
    out[((size_t)split * 3 + 0) * nb + i] = e11;
    out[((size_t)split * 3 + 1) * nb + i] = e12;
    out[((size_t)split * 3 + 2) * nb + i] = e22;
  }
}

// Deformation tensor assembly, stokeslet/rotlet gradients (:2964-2994; the
// trapezoid variant flips the sign of the rotlet's E22 term, :2604-2605),
// traction -2 E n and shear stress tau = f.(p_y, -p_x) (:3075-3092).
// part_b: barycentric partial sums (6 per split, NDER = 2 layout of
// k_bary_sum), part_t: trapezoid partial sums (3 per split, k_stress_trap and
// k_stress_far layout); either count may be zero.
__global__ void __launch_bounds__(256)
k_stress_final(GeoDev G, const double* __restrict__ den, const double* __restrict__ part_b, int nsplit_b,
               const double* __restrict__ part_t, int nsplit_t, int bary, const double* __restrict__ eself,
               double* __restrict__ tau, double* __restrict__ Eout) {
  __shared__ double4 sc[SR_CHUNK];
  __shared__ double sr[SR_CHUNK];
  const int nb = G.n * G.M;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = i < nb;
  const int ic = act ? i : nb - 1;
  double e11 = 0, e12 = 0, e22 = 0;
  for (int s = 0; s < nsplit_b; ++s) {
    const double* P = part_b + (size_t)s * 6 * nb;
    e11 += P[2 * (size_t)nb + ic];
    e12 += 0.5 * (P[3 * (size_t)nb + ic] + P[4 * (size_t)nb + ic]);
    e22 += P[5 * (size_t)nb + ic];
  }
  for (int s = 0; s < nsplit_t; ++s) {
    const double* P = part_t + (size_t)s * 3 * nb;
    e11 += P[ic];
    e12 += P[(size_t)nb + ic];
    e22 += P[2 * (size_t)nb + ic];
  }
  e11 += eself[ic];
  e12 += eself[nb + ic];
  e22 += eself[2 * nb + ic];
  const int g = G.nout + ic;
  const double2 p = G.xy[g];
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
    for (int t = 0; t < bt; ++t) {
      const double4 q = sc[t];
      const double rot = sr[t];
      const double rx = p.x - q.x, ry = p.y - q.y;
      const double rho2 = rx * rx + ry * ry;
      const double rd = rx * q.z + ry * q.w;
      const double ir2 = 1.0 / rho2, ir4 = ir2 * ir2;
      e11 += 0.5 / EB_TWOPI * (rd * ir2 - 2 * rx * rx * rd * ir4);
      e12 -= 1.0 / EB_TWOPI * (rd * ir4 * rx * ry);
      e22 += 0.5 / EB_TWOPI * (rd * ir2 - 2 * ry * ry * rd * ir4);
      e11 -= 2.0 * rot * rx * ry * ir4;
      e12 += rot * (rx * rx - ry * ry) * ir4;
      if (bary) e22 += 2.0 * rot * rx * ry * ir4;
      else e22 -= 2.0 * rot * rx * ry * ir4;
    }
  }
  if (!act) return;
  const double2 nn = G.nrm[g];
  const double tx = -2.0 * e11 * nn.x - 2.0 * e12 * nn.y;
  const double ty = -2.0 * e12 * nn.x - 2.0 * e22 * nn.y;
  tau[i] = tx * nn.y - ty * nn.x;
  if (Eout) {
    Eout[i] = e11;
    Eout[nb + i] = e12;
    Eout[2 * nb + i] = e22;
  }
}

// Trapezoid pressure (always) and velocity/vorticity (ibary = 0) at targets
// from every node (:3170-3197, :3225-3255).  out[(split*4 + q)*ntar + t],
// q = u, v, p, w.
__global__ void __launch_bounds__(256)
k_qoi_trap(GeoDev G, const double* __restrict__ den, const int4* __restrict__ tiles,
           const int* __restrict__ split_ptr, int ntar, const double2* __restrict__ txy, int velocity,
           double* __restrict__ out) {
  __shared__ double2 sxy[FAR_TS], sn[FAR_TS], ss[FAR_TS];
  __shared__ double sw[FAR_TS];
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = t < ntar;
  const double2 p = txy[act ? t : ntar - 1];
  double u = 0, v = 0, pr = 0, w = 0;
  const int split = blockIdx.y;
  for (int ti = split_ptr[split]; ti < split_ptr[split + 1]; ++ti) {
    const int4 T = tiles[ti];
    __syncthreads();
    if (threadIdx.x < T.y) {
      int gs = T.x + threadIdx.x;
      sxy[threadIdx.x] = G.xy[gs];
      sn[threadIdx.x] = G.nrm[gs];
      ss[threadIdx.x] = make_double2(den[ix_of(G, gs)], den[iy_of(G, gs)]);
      sw[threadIdx.x] = G.w[gs];
    }
    __syncthreads();
    for (int j = 0; j < T.y; ++j) {
      const double2 q = sxy[j], nn = sn[j], s = ss[j];
      double rx = p.x - q.x, ry = p.y - q.y;
      double rho2 = rx * rx + ry * ry;
      double rdotn = rx * nn.x + ry * nn.y;
      double rdotden = rx * s.x + ry * s.y;
      double dendotn = nn.x * s.x + nn.y * s.y;
      double wg = sw[j];
      pr += (2.0 * rdotn * rdotden / rho2 / rho2 - dendotn / rho2) * wg;
      if (velocity) {
        double routn = -rx * nn.y + ry * nn.x;
        double routden = -rx * s.y + ry * s.x;
        u += rdotn / rho2 * rdotden / rho2 * rx * wg;
        v += rdotn / rho2 * rdotden / rho2 * ry * wg;
        w += (rdotden * routn + rdotn * routden) / (rho2 * rho2) * wg;
      }
    }
  }
  if (act) {
    out[((size_t)split * 4 + 0) * ntar + t] = u;
    out[((size_t)split * 4 + 1) * ntar + t] = v;
    out[((size_t)split * 4 + 2) * ntar + t] = pr;
    out[((size_t)split * 4 + 3) * ntar + t] = w;
  }
}

// Final assembly at targets: barycentric velocity and vorticity (:3199-3212,
// :3257-3270), stokeslets/rotlets (:3275-3298), and zeroing of targets that
// classifyPointsOld (:4420-4500) puts inside a body (:3301-3309).
__global__ void __launch_bounds__(128)
k_qoi_final(GeoDev G, const double* __restrict__ den, int ntar, const double2* __restrict__ txy,
            const double* __restrict__ ptrap, int ns1, const double* __restrict__ pbary, int ns2, int ibary,
            double* __restrict__ uo, double* __restrict__ vo, double* __restrict__ po, double* __restrict__ wo) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ntar) return;
  double u = 0, v = 0, pr = 0, w = 0;
  for (int s = 0; s < ns1; ++s) {
    u += ptrap[((size_t)s * 4 + 0) * ntar + t];
    v += ptrap[((size_t)s * 4 + 1) * ntar + t];
    pr += ptrap[((size_t)s * 4 + 2) * ntar + t];
    w += ptrap[((size_t)s * 4 + 3) * ntar + t];
  }
  if (ibary) {
    for (int s = 0; s < ns2; ++s) {
      const double* P = pbary + (size_t)s * 6 * ntar;
      u += P[t];
      v += P[(size_t)ntar + t];
      w += P[4 * (size_t)ntar + t] - P[3 * (size_t)ntar + t];
    }
  }
  const double2 p = txy[t];
  if (G.M > 0) {
    for (int b = 0; b < G.M; ++b) {
      const double2 cc = G.cen[b];
      const double s1 = den[ic_of(G, b, 0)], s2 = den[ic_of(G, b, 1)], rot = den[ic_of(G, b, 2)];
      const double rx = p.x - cc.x, ry = p.y - cc.y;
      const double rho2 = rx * rx + ry * ry, rd = rx * s1 + ry * s2;
      u += 0.5 / EB_TWOPI * (-0.5 * log(rho2) * s1 + rd / rho2 * rx);
      v += 0.5 / EB_TWOPI * (-0.5 * log(rho2) * s2 + rd / rho2 * ry);
      pr += 1.0 / EB_TWOPI * rd / rho2;
      w += (ry * s1 - rx * s2) / rho2 / EB_TWOPI;
      u += rot * ry / rho2;
      v -= rot * rx / rho2;
    }
    // classifyPointsOld: nearest body node (first minimum in body-major
    // order) decides the side through the sign of (x_t - x_k).n_k.
    double dmin = 1e10;
    int ind = 0;
    for (int i = 0; i < G.n * G.M; ++i) {
      const double2 q = G.xy[G.nout + i];
      const double d2 = (p.x - q.x) * (p.x - q.x) + (p.y - q.y) * (p.y - q.y);
      if (d2 < dmin) { dmin = d2; ind = i; }
    }
    const double2 q = G.xy[G.nout + ind], nn = G.nrm[G.nout + ind];
    const double vdn = (p.x - q.x) * nn.x + (p.y - q.y) * nn.y;
    if (!(vdn < 0.0)) { u = 0; v = 0; pr = 0; w = 0; }
  }
  uo[t] = u; vo[t] = v; po[t] = pr; wo[t] = w;
}

// ---------------------------------------------------------------------------
// Host side.

// Boundary values of all curves (wall first, then every body).
static void bdval_all(State& s, const double* d_den, DBuf<double2>& bd_all) {
  const Problem& pr = s.pr;
  const GeoDev G = s.geo();
  std::vector<int> curves(pr.M + 1);
  std::vector<long long> off(pr.M + 1);
  std::vector<int2> work;
  for (int c = 0; c <= pr.M; ++c) {
    curves[c] = c;
    off[c] = c == 0 ? 0 : 5LL * pr.nout + 5LL * (c - 1) * pr.n;
    int len = c == 0 ? pr.nout : pr.n;
    for (int j0 = 0; j0 < len; j0 += BD_NT) work.push_back(make_int2(c, j0));
  }
  static DBuf<int> d_curves;
  static DBuf<long long> d_off;
  static DBuf<int2> d_work;
  h2d(d_curves.ensure(curves.size()), curves.data(), curves.size(), s.st);
  h2d(d_off.ensure(off.size()), off.data(), off.size(), s.st);
  h2d(d_work.ensure(work.size()), work.data(), work.size(), s.st);
  bd_all.ensure(5LL * pr.nout + 5LL * pr.n * pr.M);
  k_bdval<<<(unsigned)work.size(), BD_NT, 0, s.st>>>(G, d_den, d_work.p, d_curves.p, d_off.p, s.dker_wall.p,
                                                      s.dker_body.p, bd_all.p);
  EB_LAUNCH_CHECK();
  EB_CK(cudaStreamSynchronize(s.st));   // host vectors go out of scope
}

int eb_num_sms();

// ---------------------------------------------------------------------------
// Pressure on the body boundaries (computePressure, stokesSolver.f:4644-4885).
// Every pair: (2 (r.n)(r.s)/rho^4 - (n.s)/rho^2) w_j with the trapezoid weight
// w = speed (2pi/n_c)/pi.  Targets: body nodes; sources: every tile, split
// over blockIdx.y.  A target's own body uses odd-even quadrature: sources of
// the other index parity only, weight doubled, density minus its value at the
// target (:4728-4787).
__global__ void __launch_bounds__(256)
k_pressure_sum(GeoDev G, const double* __restrict__ den, const int4* __restrict__ tiles,
               const int* __restrict__ split_ptr, double* __restrict__ part) {
  __shared__ double4 sg[FAR_TS];
  __shared__ double2 sd[FAR_TS];
  __shared__ double sw[FAR_TS];
  __shared__ int sl[FAR_TS];
  const int nb = G.n * G.M;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int tc = t < nb ? t : nb - 1;
  const int g = G.nout + tc;
  const int b = tc / G.n, k = tc - b * G.n, curve = 1 + b;
  const double2 p = G.xy[g];
  const double sxk = den[ix_of(G, g)], syk = den[iy_of(G, g)];
  double acc = 0.0;
  const int split = blockIdx.y;
  for (int ti = split_ptr[split]; ti < split_ptr[split + 1]; ++ti) {
    const int4 T = tiles[ti];
    __syncthreads();
    for (int q = threadIdx.x; q < T.y; q += blockDim.x) {
      const int j = T.x + q;
      const double2 xy = G.xy[j], nn = G.nrm[j];
      sg[q] = make_double4(xy.x, xy.y, nn.x, nn.y);
      sd[q] = make_double2(den[ix_of(G, j)], den[iy_of(G, j)]);
      sw[q] = G.w[j];
      sl[q] = j - curve_start(G, T.z);   // index within its curve
    }
    __syncthreads();
    const bool own = T.z == curve;
    for (int q = 0; q < T.y; ++q) {
      if (own && ((sl[q] & 1) == (k & 1))) continue;
      const double4 sq = sg[q];
      const double2 dq = sd[q];
      const double sx = own ? dq.x - sxk : dq.x, sy = own ? dq.y - syk : dq.y;
      const double rx = p.x - sq.x, ry = p.y - sq.y;
      const double rho2 = rx * rx + ry * ry;
      const double rdn = rx * sq.z + ry * sq.w, rds = rx * sx + ry * sy, dn = sq.z * sx + sq.w * sy;
      const double v = (2.0 * rdn * rds / rho2 / rho2 - dn / rho2) * sw[q];
      acc += own ? 2.0 * v : v;
    }
  }
  if (t < nb) part[(size_t)split * nb + t] = acc;
}

// Split sums, the jump -(d sigma/ds . tangent) with the spectral derivative
// (the circulant d[m] of fourierDiff) and the stokeslet pressure
// (r . lambda)/(2 pi rho^2) of every body (:4829-4881); one thread per node.
__global__ void __launch_bounds__(256)
k_pressure_final(GeoDev G, const double* __restrict__ den, const double* __restrict__ part, int nsplit,
                 const double* __restrict__ dk, double* __restrict__ out) {
  const int nb = G.n * G.M;
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb) return;
  const int b = t / G.n, k = t - b * G.n, g = G.nout + t;
  double acc = 0.0;
  for (int q = 0; q < nsplit; ++q) acc += part[(size_t)q * nb + t];
  double dx = 0.0, dy = 0.0;
  for (int j = 0; j < G.n; ++j) {
    int m = k - j;
    if (m < 0) m += G.n;
    const double d = __ldg(dk + m);
    const int gj = G.nout + b * G.n + j;
    dx = fma(d, den[ix_of(G, gj)], dx);
    dy = fma(d, den[iy_of(G, gj)], dy);
  }
  const double2 nn = G.nrm[g];
  const double spd = G.sp[g];
  acc -= (dx / spd) * (-nn.y) + (dy / spd) * nn.x;
  const double2 p = G.xy[g];
  for (int s = 0; s < G.M; ++s) {
    const double2 c = G.cen[s];
    const double rx = p.x - c.x, ry = p.y - c.y;
    acc += (rx * den[ic_of(G, s, 0)] + ry * den[ic_of(G, s, 1)]) / (EB_TWOPI * (rx * rx + ry * ry));
  }
  out[t] = acc;
}

static int source_splits(int ntasks, int ncurves, std::vector<int>& sc) {
  int want = std::max(1, (4 * eb_num_sms() + ntasks - 1) / std::max(ntasks, 1));
  int S = std::max(1, std::min(want, ncurves));
  sc.resize(S + 1);
  for (int q = 0; q <= S; ++q) sc[q] = (int)((long long)q * ncurves / S);
  return S;
}

void body_pressure(State& s, const double* d_den, double* d_p) {
  const Problem& pr = s.pr;
  const GeoDev G = s.geo();
  const int nb = pr.n * pr.M;
  if (nb == 0) return;
  static DBuf<double> part;
  part.ensure((size_t)s.nsplit * nb);
  k_pressure_sum<<<dim3(nblk(nb, 256), s.nsplit), 256, 0, s.st>>>(G, d_den, s.tiles.p, s.split_ptr.p, part.p);
  EB_LAUNCH_CHECK();
  k_pressure_final<<<nblk(nb, 256), 256, 0, s.st>>>(G, d_den, part.p, s.nsplit, s.dker_body.p, d_p);
  EB_LAUNCH_CHECK();
}

void shear_stress(State& s, const double* d_den, double* d_tau, double* d_E) {
  const Problem& pr = s.pr;
  const GeoDev G = s.geo();
  const int nb = pr.n * pr.M;
  if (nb == 0) return;
  static DBuf<double> eself, part;
  static DBuf<double2> bd_all;
  static DBuf<int4> d_tasks;
  static DBuf<int> d_sc;
  eself.ensure(3LL * nb);
  size_t smem = 7 * (size_t)pr.n * sizeof(double);
  if (smem > 48 * 1024) allow_max_dynamic_smem((const void*)k_stress_self);
  k_stress_self<<<pr.M, 256, smem, s.st>>>(G, d_den, s.dker_body.p, eself.p);
  EB_LAUNCH_CHECK();
  const int bary = pr.P.ibary == 1;
  if (bary && pr.P.stress_all_bary) {   // every pair barycentric, as the reference evaluates it
    bdval_all(s, d_den, bd_all);
    std::vector<int4> tasks;
    for (int b = 0; b < pr.M; ++b)
      for (int k0 = 0; k0 < pr.n; k0 += NEAR_NT)
        tasks.push_back(make_int4(b * pr.n + k0, b * pr.n + std::min(pr.n, k0 + NEAR_NT), 1 + b, 0));
    std::vector<int> sc;
    const int nsplit = source_splits((int)tasks.size(), pr.M + 1, sc);
    h2d(d_tasks.ensure(tasks.size()), tasks.data(), tasks.size(), s.st);
    h2d(d_sc.ensure(sc.size()), sc.data(), sc.size(), s.st);
    part.ensure((size_t)nsplit * 6 * nb);
    dim3 grid((unsigned)tasks.size(), nsplit);
    k_bary_sum<2><<<grid, NEAR_NT, 0, s.st>>>(G, bd_all.p, d_tasks.p, s.xy.p + pr.nout, d_sc.p, nb, part.p);
    EB_LAUNCH_CHECK();
    k_stress_final<<<nblk(nb, 256), 256, 0, s.st>>>(G, d_den, part.p, nsplit, nullptr, 0, 1, eself.p, d_tau, d_E);
    EB_LAUNCH_CHECK();
    EB_CK(cudaStreamSynchronize(s.st));
  } else if (bary) {   // barycentric near pairs, trapezoid elsewhere
    static DBuf<double> wall_d2h;
    static DBuf<double2> ext;
    static DBuf<unsigned> smask;
    static DBuf<double> pnear;
    const int mw = (pr.M + 1 + 31) / 32;
    k_stress_wall_dist<<<nblk(nb, 256), 256, 0, s.st>>>(G, wall_d2h.ensure(nb));
    EB_LAUNCH_CHECK();
    k_body_extent<<<pr.M, 256, 0, s.st>>>(G, ext.ensure(pr.M));
    EB_LAUNCH_CHECK();
    k_stress_near_mask<<<nblk(nb, 256), 256, 0, s.st>>>(G, wall_d2h.p, ext.p, mw, smask.ensure((size_t)nb * mw));
    EB_LAUNCH_CHECK();
    bdval_all(s, d_den, bd_all);
    std::vector<int4> tasks;
    for (int b = 0; b < pr.M; ++b)
      for (int k0 = 0; k0 < pr.n; k0 += NEAR_NT)
        tasks.push_back(make_int4(b * pr.n + k0, b * pr.n + std::min(pr.n, k0 + NEAR_NT), 1 + b, 0));
    h2d(d_tasks.ensure(tasks.size()), tasks.data(), tasks.size(), s.st);
    k_bary_sum_near<<<(unsigned)tasks.size(), NEAR_NT, 0, s.st>>>(G, bd_all.p, d_tasks.p, smask.p, mw,
                                                                   pnear.ensure(6LL * nb));
    EB_LAUNCH_CHECK();
    const int nsplit = s.nsplit;
    part.ensure((size_t)nsplit * 3 * nb);
    static DBuf<double> rig;
    k_stress_rigid<<<pr.M, 256, 0, s.st>>>(G, d_den, rig.ensure(5LL * pr.M));
    EB_LAUNCH_CHECK();
    k_stress_far<<<dim3(nblk(nb, 256), nsplit), 256, 0, s.st>>>(G, d_den, s.tiles.p, s.split_ptr.p, smask.p, mw,
                                                                 rig.p, part.p);
    EB_LAUNCH_CHECK();
    k_stress_final<<<nblk(nb, 256), 256, 0, s.st>>>(G, d_den, pnear.p, 1, part.p, nsplit, 1, eself.p, d_tau, d_E);
    EB_LAUNCH_CHECK();
    EB_CK(cudaStreamSynchronize(s.st));   // the task list goes out of scope
  } else {
    const int nsplit = s.nsplit;
    part.ensure((size_t)nsplit * 3 * nb);
    dim3 grid(nblk(nb, 256), nsplit);
    k_stress_trap<<<grid, 256, 0, s.st>>>(G, d_den, s.tiles.p, s.split_ptr.p, part.p);
    EB_LAUNCH_CHECK();
    k_stress_final<<<nblk(nb, 256), 256, 0, s.st>>>(G, d_den, nullptr, 0, part.p, nsplit, 0, eself.p, d_tau, d_E);
    EB_LAUNCH_CHECK();
  }
}

void qoi_targets(State& s, const double* d_den, long long ntar, const double* d_xt, const double* d_yt, double* d_u,
                 double* d_v, double* d_p, double* d_w) {
  const Problem& pr = s.pr;
  const GeoDev G = s.geo();
  if (ntar == 0) return;
  static DBuf<double2> txy, bd_all;
  static DBuf<double> ptrap, pbary;
  static DBuf<int4> d_tasks;
  static DBuf<int> d_sc;
  txy.ensure(ntar);
  {
    std::vector<double> hx(ntar), hy(ntar);
    d2h(hx.data(), d_xt, ntar, s.st);
    d2h(hy.data(), d_yt, ntar, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    std::vector<double2> h(ntar);
    for (long long t = 0; t < ntar; ++t) h[t] = make_double2(hx[t], hy[t]);
    h2d(txy.p, h.data(), ntar, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
  }
  const int ibary = pr.P.ibary == 1;
  ptrap.ensure((size_t)s.nsplit * 4 * ntar);
  dim3 g1(nblk(ntar, 256), s.nsplit);
  k_qoi_trap<<<g1, 256, 0, s.st>>>(G, d_den, s.tiles.p, s.split_ptr.p, (int)ntar, txy.p, !ibary, ptrap.p);
  EB_LAUNCH_CHECK();
  int ns2 = 0;
  if (ibary) {
    bdval_all(s, d_den, bd_all);
    std::vector<int4> tasks;
    for (long long t0 = 0; t0 < ntar; t0 += NEAR_NT)
      tasks.push_back(make_int4((int)t0, (int)std::min<long long>(ntar, t0 + NEAR_NT), -1, 0));
    std::vector<int> sc;
    ns2 = source_splits((int)tasks.size(), pr.M + 1, sc);
    h2d(d_tasks.ensure(tasks.size()), tasks.data(), tasks.size(), s.st);
    h2d(d_sc.ensure(sc.size()), sc.data(), sc.size(), s.st);
    pbary.ensure((size_t)ns2 * 6 * ntar);
    dim3 g2((unsigned)tasks.size(), ns2);
    k_bary_sum<2><<<g2, NEAR_NT, 0, s.st>>>(G, bd_all.p, d_tasks.p, txy.p, d_sc.p, (int)ntar, pbary.p);
    EB_LAUNCH_CHECK();
    EB_CK(cudaStreamSynchronize(s.st));
  }
  k_qoi_final<<<nblk(ntar, 128), 128, 0, s.st>>>(G, d_den, (int)ntar, txy.p, ptrap.p, s.nsplit, pbary.p, ns2, ibary,
                                                  d_u, d_v, d_p, d_w);
  EB_LAUNCH_CHECK();
}

}  // namespace eb

// ===========================================================================
// C ABI
using namespace eb;

namespace {

template <class F>
int guarded2(F&& f) {
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

Problem problem_of(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter) {
  if (npts < 0 || nbods < 0 || nouter < 0 || npts > (1 << 24) || nbods > (1 << 24) || nouter > (1 << 26))
    throw Error(EROSION_BAD_INPUT, "negative or oversized sizes");
  Problem pr;
  if (p) pr.P = *p;
  else erosion_default_params(&pr.P);
  pr.n = (int)npts; pr.M = (int)nbods; pr.nout = (int)nouter;
  return pr;
}

void host_setup(State& s, const Problem& pr, const double* xx, const double* yy, const double* density) {
  size_t nb = (size_t)pr.n * pr.M;
  double* dx = s.d_xx.ensure(std::max<size_t>(nb, 1));
  double* dy = s.d_yy.ensure(std::max<size_t>(nb, 1));
  h2d(dx, xx, nb, s.st);
  h2d(dy, yy, nb, s.st);
  setup_problem(s, pr, dx, dy);
  double* dd = s.d_den.ensure(s.pr.ntot);
  h2d(dd, density, s.pr.ntot, s.st);
}

}  // namespace

extern "C" {

int erosion_shear_stress(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                         const double* yy, const double* density, double* tau, double* E) {
  return guarded2([&](State& s) {
    Problem pr = problem_of(p, npts, nbods, nouter);
    if (pr.M == 0) return EROSION_OK;
    host_setup(s, pr, xx, yy, density);
    const size_t nb = (size_t)s.pr.n * s.pr.M;
    static DBuf<double> dtau, dE;
    dtau.ensure(nb);
    if (E) dE.ensure(3 * nb);
    shear_stress(s, s.d_den.p, dtau.p, E ? dE.p : nullptr);
    d2h(tau, dtau.p, nb, s.st);
    if (E) d2h(E, dE.p, 3 * nb, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_shear_stress_device(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                                const double* d_xx, const double* d_yy, const double* d_density, double* d_tau) {
  return guarded2([&](State& s) {
    Problem pr = problem_of(p, npts, nbods, nouter);
    if (pr.M == 0) return EROSION_OK;
    setup_problem(s, pr, d_xx, d_yy);
    shear_stress(s, d_density, d_tau, nullptr);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

int erosion_pressure(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                     const double* yy, const double* density, double* pressure) {
  return guarded2([&](State& s) {
    Problem pr = problem_of(p, npts, nbods, nouter);
    if (pr.M == 0) return EROSION_OK;
    host_setup(s, pr, xx, yy, density);
    const size_t nb = (size_t)s.pr.n * s.pr.M;
    static DBuf<double> dp;
    dp.ensure(nb);
    body_pressure(s, s.d_den.p, dp.p);
    d2h(pressure, dp.p, nb, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

void computepressure_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter, const double* xx,
                      const double* yy, const double* density, double* pressure) {
  erosion_pressure(nullptr, *npts, *nbods, *nouter, xx, yy, density, pressure);
}

void computeshearstress_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter, const double* xx,
                         const double* yy, const double* density, const int64_t* ibary, double* tau) {
  erosion_params p;
  erosion_default_params(&p);
  p.ibary = (int32_t)*ibary;
  erosion_shear_stress(&p, *npts, *nbods, *nouter, xx, yy, density, tau, nullptr);
}

int erosion_qoi_targets(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter, const double* xx,
                        const double* yy, const double* density, int64_t ntargets, const double* xtar,
                        const double* ytar, double* utar, double* vtar, double* ptar, double* vortar) {
  return guarded2([&](State& s) {
    Problem pr = problem_of(p, npts, nbods, nouter);
    if (ntargets < 0) throw Error(EROSION_BAD_INPUT, "negative target count");
    host_setup(s, pr, xx, yy, density);
    if (ntargets == 0) return EROSION_OK;
    static DBuf<double> buf;
    double* b = buf.ensure(6 * (size_t)ntargets);
    h2d(b, xtar, ntargets, s.st);
    h2d(b + ntargets, ytar, ntargets, s.st);
    qoi_targets(s, s.d_den.p, ntargets, b, b + ntargets, b + 2 * ntargets, b + 3 * ntargets, b + 4 * ntargets,
                b + 5 * ntargets);
    d2h(utar, b + 2 * ntargets, ntargets, s.st);
    d2h(vtar, b + 3 * ntargets, ntargets, s.st);
    d2h(ptar, b + 4 * ntargets, ntargets, s.st);
    d2h(vortar, b + 5 * ntargets, ntargets, s.st);
    EB_CK(cudaStreamSynchronize(s.st));
    return EROSION_OK;
  });
}

void computeqoitargets_(const int64_t* npts, const int64_t* nbods, const int64_t* nouter, const int64_t* ibary,
                        const double* xx, const double* yy, const double* density, const int64_t* ntargets,
                        const double* xtar, const double* ytar, double* utar, double* vtar, double* ptar,
                        double* vortar) {
  erosion_params p;
  erosion_default_params(&p);
  p.ibary = (int32_t)*ibary;
  erosion_qoi_targets(&p, *npts, *nbods, *nouter, xx, yy, density, *ntargets, xtar, ytar, utar, vtar, ptar, vortar);
}

}  // extern "C"
