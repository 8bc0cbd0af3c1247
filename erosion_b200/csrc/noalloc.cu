// erosion_matvec_noalloc: the trapezoid-rule boundary operator for callers
// that cannot allocate GPU memory.
//
// Who needs it: a caller that drives its own Krylov loop on the GPU from a
// runtime that owns all device memory (a memory pool that forbids foreign
// cudaMalloc calls, a process whose device memory is fully reserved up front,
// or code that must not synchronise the device the way cudaMalloc/cudaFree
// can) cannot use erosion_matvec, which grows cached device buffers on demand.
// This entry point takes device pointers for its inputs and output, launches
// on the caller's stream, and keeps every intermediate array in one
// fixed-size array of device memory that is part of the library image.
//
// The array (na_scratch, NA_SCRATCH_BYTES = 24 MiB) exists on every GPU that
// loads the library, for as long as the process runs.  It bounds the problem
// size: nouter <= 4096, npts <= 512, nbods <= 128 and
// nouter + npts * nbods <= 32768 nodes; larger problems are rejected with
// EROSION_BAD_INPUT.  Every call shares the array and finds it as the last
// call left it; each call writes every word it later reads, so nothing has to
// start at zero, but two calls whose kernels overlap on the GPU (different
// streams, or different host threads) race on it and corrupt each other.
//
// The first call on a device looks up the array's device address with
// cudaGetSymbolAddress (host code cannot use the array's name as a device
// pointer) and queries the SM count; make that first call before capturing
// any stream.  The computation is the one erosion_matvec performs with
// ibary = 0 and precision = 0 (geometry from spectral derivatives, far field
// with the split-K partial sums, self-curve sums, jump, stokeslets/rotlets,
// constraint rows and the rank-one wall term), by the same kernels.
#include <mutex>

#include "state.h"
#include "kernels.cuh"

namespace {

constexpr int NA_MAX_NODES = 32768;
constexpr int NA_MAX_BODIES = 128;
constexpr int NA_MAX_NPTS = 512;
constexpr int NA_MAX_NOUT = 4096;
constexpr size_t NA_SCRATCH_BYTES = size_t(24) << 20;
constexpr int NA_MAX_DEVICES = 64;

// Per-layout tables the host-side operator builds on the CPU: tiles of the
// far-field sum, their split-K ranges, the self-curve tasks (same order and
// contents as build_tiles in solver.cu) and the two circulant derivative
// kernels d[m] = (1/2)(-1)^m cot(pi m/n) (fourierDiff, stokesSolver.f:348-388).
__global__ void k_na_layout(int nout, int n, int M, int nsplit, int nslots, int4* __restrict__ tiles,
                            int* __restrict__ split_ptr, int4* __restrict__ tasks, double* __restrict__ dker_w,
                            double* __restrict__ dker_b) {
  const int nwt = (nout + WALL_TS - 1) / WALL_TS;
  const int tpb = M > 0 ? (n + FAR_TS - 1) / FAR_TS : 0;
  const int ntile = nwt + M * tpb;
  for (int t = threadIdx.x; t < ntile; t += blockDim.x) {
    if (t < nwt) {
      const int o = t * WALL_TS;
      tiles[t] = make_int4(o, min(WALL_TS, nout - o), 0, 0);
    } else {
      const int r = t - nwt, b = r / tpb, o = (r % tpb) * FAR_TS;
      tiles[t] = make_int4(nout + b * n + o, min(FAR_TS, n - o), 1 + b, 0);
    }
  }
  for (int q = threadIdx.x; q <= nsplit; q += blockDim.x) split_ptr[q] = (int)((long long)q * ntile / nsplit);
  const int wpt = (nout + 255) / 256;
  const int nwtask = nslots * wpt;
  const int bpt = M > 0 ? (n + 255) / 256 : 0;
  for (int t = threadIdx.x; t < nwtask + M * bpt; t += blockDim.x) {
    if (t < nwtask) {
      const int ch = t / wpt, o = (t % wpt) * 256;
      tasks[t] = make_int4(o, min(256, nout - o), 0, ch);
    } else {
      const int r = t - nwtask, b = r / bpt, o = (r % bpt) * 256;
      tasks[t] = make_int4(nout + b * n + o, min(256, n - o), 1 + b, 0);
    }
  }
  for (int m = threadIdx.x; m < nout + n; m += blockDim.x) {
    const int len = m < nout ? nout : n, k = m < nout ? m : m - nout;
    double d = 0.0;
    if (k != 0 && 2 * k != len) {
      const double t = EB_PI * k / len;
      d = 0.5 * ((k & 1) ? -1.0 : 1.0) * cos(t) / sin(t);
    }
    if (m < nout) dker_w[k] = d;
    else dker_b[k] = d;
  }
}

}  // namespace

// The scratch memory of erosion_matvec_noalloc (see the file comment).
static __device__ __align__(256) unsigned char na_scratch[NA_SCRATCH_BYTES];

namespace {

struct NaDevice {
  bool ready = false;
  unsigned char* base = nullptr;   // device address of na_scratch on this device
  int sms = 0;
};
NaDevice g_na[NA_MAX_DEVICES];
std::mutex g_na_mu;

// Bump allocation inside the fixed array, 256-byte aligned.
struct Carve {
  unsigned char* base;
  size_t off = 0;
  template <class T>
  T* take(size_t count) {
    T* p = reinterpret_cast<T*>(base + off);
    off += (count * sizeof(T) + 255) & ~size_t(255);
    return p;
  }
};

// The status channel is per thread and lock-free (set_status), so recording
// an outcome never waits for another thread's call into the library.
int na_fail(int code, const char* msg) {
  eb::set_status(code, msg);
  return code;
}

}  // namespace

using namespace eb;

extern "C" int erosion_matvec_noalloc(const erosion_params* p, int64_t npts, int64_t nbods, int64_t nouter,
                                      const double* d_xx, const double* d_yy, const double* d_den, double* d_vel,
                                      void* stream) {
  if (!p || !d_den || !d_vel || (nbods > 0 && (!d_xx || !d_yy)))
    return na_fail(EROSION_BAD_INPUT, "erosion_matvec_noalloc: null parameter or array pointer");
  if (p->ibary != 0 || p->precision != 0)
    return na_fail(EROSION_BAD_INPUT,
                   "erosion_matvec_noalloc: only the trapezoid FP64 operator (ibary = 0, precision = 0) is "
                   "available without allocation");
  if (nouter < 8 || (nouter & 1) || nouter > NA_MAX_NOUT)
    return na_fail(EROSION_BAD_INPUT, "erosion_matvec_noalloc: nouter must be even, >= 8 and <= 4096");
  if (nbods < 0 || nbods > NA_MAX_BODIES)
    return na_fail(EROSION_BAD_INPUT, "erosion_matvec_noalloc: nbods must be between 0 and 128");
  if (nbods > 0 && (npts < 4 || (npts & 1) || npts > NA_MAX_NPTS))
    return na_fail(EROSION_BAD_INPUT, "erosion_matvec_noalloc: npts must be even, >= 4 and <= 512");
  if (nouter + (nbods > 0 ? npts * nbods : 0) > NA_MAX_NODES)
    return na_fail(EROSION_BAD_INPUT,
                   "erosion_matvec_noalloc: more than 32768 nodes (nouter + npts * nbods) exceeds the fixed "
                   "scratch memory");
  if (!(p->wall_a > 0 && p->wall_b > 0 && p->wall_order > 0))
    return na_fail(EROSION_BAD_INPUT, "erosion_matvec_noalloc: wall semi-axes and order must be positive");
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return na_fail(EROSION_NO_DEVICE, "erosion_matvec_noalloc: no CUDA device");
    }
    // This call shares the caller's stream and the runtime's per-thread error
    // state: an error already pending from the caller's own work is reported
    // (and left pending) instead of being consumed by the launch checks below.
    {
      const cudaError_t pending = cudaPeekAtLastError();
      if (pending != cudaSuccess)
        return na_fail(EROSION_CUDA_ERROR, (std::string("erosion_matvec_noalloc: a CUDA error was already pending "
                                                        "before the call, nothing was launched: ") +
                                            cudaGetErrorString(pending)).c_str());
    }
    int dev = 0;
    EB_CK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NA_MAX_DEVICES) throw Error(EROSION_BAD_INPUT, "erosion_matvec_noalloc: device ordinal");
    NaDevice nd;
    {
      std::lock_guard<std::mutex> lk(g_na_mu);
      if (!g_na[dev].ready) {   // once per device, with that device current
        void* ptr = nullptr;
        EB_CK(cudaGetSymbolAddress(&ptr, na_scratch));
        int sms = 0;
        EB_CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        g_na[dev].base = static_cast<unsigned char*>(ptr);
        g_na[dev].sms = sms;
        g_na[dev].ready = true;
      }
      nd = g_na[dev];
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int n = nbods > 0 ? (int)npts : 2, M = (int)nbods, nout = (int)nouter;
    const int N = nout + n * M;
    const long long ntot = 2LL * N + 3LL * M;
    const int nwt = (nout + WALL_TS - 1) / WALL_TS;
    const int ntile = nwt + (M > 0 ? M * ((n + FAR_TS - 1) / FAR_TS) : 0);
    const int nslots = (nout + SELF_CHUNK - 1) / SELF_CHUNK;
    const int ntask = nslots * ((nout + 255) / 256) + (M > 0 ? M * ((n + 255) / 256) : 0);

    Carve cv{nd.base};
    double* wx = cv.take<double>(nout);
    double* wy = cv.take<double>(nout);
    double* dker_w = cv.take<double>(nout);
    double* dker_b = cv.take<double>(n);
    double2* xy = cv.take<double2>(N);
    double2* nrm = cv.take<double2>(N);
    double2* dz = cv.take<double2>(N);
    double2* d1tmp = cv.take<double2>(N);
    double* sp = cv.take<double>(N);
    double* cur = cv.take<double>(N);
    double* w = cv.take<double>(N);
    double2* cen = cv.take<double2>(std::max(M, 1));
    double* rb = cv.take<double>(std::max(M, 1));
    double2* ws = cv.take<double2>(N);
    double4* sq64 = cv.take<double4>(N);
    float4* sq32 = cv.take<float4>(N);
    double* sigdotn = cv.take<double>(1);
    int4* tiles = cv.take<int4>(ntile);
    int4* tasks = cv.take<int4>(ntask);
    double2* selfsum = cv.take<double2>((size_t)nslots * N);
    // split-K of the far field as the host-side operator chooses it, capped by
    // the room left in the array
    const int TB = (int)nblk(N, FAR_NT * FAR_TPT);
    int nsplit = std::max(1, std::min((int)std::ceil(8.0 * nd.sms / TB), ntile));
    const size_t room = NA_SCRATCH_BYTES - cv.off - 2 * 256 - (size_t)(ntile + 1) * sizeof(int);
    nsplit = std::max(1, std::min<int>(nsplit, (int)(room / ((size_t)N * sizeof(double2)))));
    int* split_ptr = cv.take<int>(nsplit + 1);
    double2* partial = cv.take<double2>((size_t)nsplit * N);
    if (cv.off > NA_SCRATCH_BYTES) throw Error(EROSION_BAD_INPUT, "erosion_matvec_noalloc: scratch layout");

    GeoDev G;
    G.n = n; G.M = M; G.nout = nout; G.N = N; G.ntot = ntot;
    G.xy = xy; G.nrm = nrm; G.sp = sp; G.cur = cur; G.w = w; G.dz = dz; G.cen = cen; G.rb = rb;

    k_na_layout<<<1, 256, 0, st>>>(nout, n, M, nsplit, nslots, tiles, split_ptr, tasks, dker_w, dker_b);
    EB_LAUNCH_CHECK();
    k_wall_nodes<<<nblk(nout, 256), 256, 0, st>>>(nout, p->wall_a, p->wall_b, p->wall_order, wx, wy);
    EB_LAUNCH_CHECK();
    k_geom<<<1, 1024, 0, st>>>(wx, wy, nout, dker_w, 0, 1, xy, nrm, sp, cur, w, dz, d1tmp);
    EB_LAUNCH_CHECK();
    if (M > 0) {
      k_geom<<<M, 256, 0, st>>>(d_xx, d_yy, n, dker_b, nout, 0, xy, nrm, sp, cur, w, dz, d1tmp + nout);
      EB_LAUNCH_CHECK();
      k_body_stats<<<M, 256, 0, st>>>(n, nout, xy, sp, cen, rb);
      EB_LAUNCH_CHECK();
    }
    k_prep<<<M + 1, 256, 0, st>>>(G, d_den, ws, sq64, sq32, d_vel, sigdotn, 0);
    EB_LAUNCH_CHECK();
    k_far64<false, FAR_NT, FAR_TPT, 0><<<dim3((unsigned)TB, (unsigned)nsplit), FAR_NT, 0, st>>>(
        G, sq64, tiles, split_ptr, nullptr, 0, partial);
    EB_LAUNCH_CHECK();
    k_self64<<<ntask, 256, 0, st>>>(G, ws, tasks, selfsum, n);   // one chunk per body
    EB_LAUNCH_CHECK();
    k_combine<<<nblk((long long)N * COMBINE_G, 256), 256, 0, st>>>(G, d_den, partial, nsplit, nullptr, nullptr, nullptr, sigdotn, selfsum,
                                            nslots, 1, d_vel);
    EB_LAUNCH_CHECK();
    set_status(EROSION_OK, "");
    return EROSION_OK;
  } catch (const Error& e) {
    return na_fail(e.code, e.what());
  } catch (const std::exception& e) {
    return na_fail(EROSION_CUDA_ERROR, e.what());
  }
}
