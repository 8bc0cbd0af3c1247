// Shared device helpers for the B200 Stokes boundary-integral kernels.
#pragma once
#include <cuda_runtime.h>
#include <cstdint>

#define EB_PI 3.141592653589793238462643383279502884
#define EB_TWOPI 6.283185307179586476925286766559005768

// ---------------------------------------------------------------------------
// Layout of one problem on the device.  Nodes are numbered wall first
// (0..nout-1, parameter order), then body b's nodes (nout + b*n + k).  Curves:
// id 0 is the wall, id 1+b is body b.  The unknown vector keeps the
// reference's layout (see include/erosion_b200.h).
struct GeoDev {
  int n, M, nout, N;
  long long ntot;
  const double2* __restrict__ xy;    // node coordinates
  const double2* __restrict__ nrm;   // normals as the reference uses them (wall negated)
  const double* __restrict__ sp;     // |z'(theta)|
  const double* __restrict__ cur;    // curvature (wall negated)
  const double* __restrict__ w;      // far-field weight speed*(2pi/n_c)/pi
  const double2* __restrict__ dz;    // z'(theta) * 2pi/n_c
  const double2* __restrict__ cen;   // body centroids
  const double* __restrict__ rb;     // mean speed per body
};

__device__ __forceinline__ long long ix_of(const GeoDev& G, int g) {
  if (g < G.nout) return g;
  int r = g - G.nout, b = r / G.n, k = r - b * G.n;
  return 2LL * G.nout + 2LL * G.n * b + k;
}
__device__ __forceinline__ long long iy_of(const GeoDev& G, int g) {
  if (g < G.nout) return (long long)G.nout + g;
  int r = g - G.nout, b = r / G.n, k = r - b * G.n;
  return 2LL * G.nout + 2LL * G.n * b + G.n + k;
}
__device__ __forceinline__ long long ic_of(const GeoDev& G, int b, int c) {
  return 2LL * G.nout + 2LL * G.n * G.M + 3LL * b + c;
}
__device__ __forceinline__ int curve_start(const GeoDev& G, int c) { return c == 0 ? 0 : G.nout + (c - 1) * G.n; }
__device__ __forceinline__ int curve_len(const GeoDev& G, int c) { return c == 0 ? G.nout : G.n; }

// ---------------------------------------------------------------------------
// Complex helpers on double2 (x = real, y = imag).
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// a += b * c
__device__ __forceinline__ void cfma(double2& a, double2 b, double2 c) {
  a.x = fma(b.x, c.x, fma(-b.y, c.y, a.x));
  a.y = fma(b.x, c.y, fma(b.y, c.x, a.y));
}
__device__ __forceinline__ double2 cinv(double2 a) {
  double d = 1.0 / fma(a.x, a.x, a.y * a.y);
  return make_double2(a.x * d, -a.y * d);
}
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) { return cmul(a, cinv(b)); }
__device__ __forceinline__ double cabs2(double2 a) { return fma(a.x, a.x, a.y * a.y); }

// ---------------------------------------------------------------------------
// Block reductions (deterministic: fixed tree order).
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) sh[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < NT / 32) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  if (threadIdx.x == 0) sh[0] = r;
  __syncthreads();
  r = sh[0];
  __syncthreads();
  return r;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
