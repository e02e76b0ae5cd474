// Harness kernels on the device: the analytic right-hand side (FishFry.hpp:14-45)
// with an optional seeded sum of Fourier modes, and the error sums against the
// analytic solution (FishFry.hpp:47-101) with a deterministic reduction in
// place of the reference's shared and global FP64 atomics.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <mutex>

#include "ff_status.hpp"

namespace ff {

constexpr int kMaxModes = 64;
constexpr int kSumBlocks = 1184;   // 8 blocks per SM on 148 SMs; fixed, so sums are reproducible
constexpr int kSumThreads = 256;

struct FieldArgs {
  int ni, nj, nk;
  double xlo, ylo, zlo, dx, dy, dz;
  int nmodes;
  ff_mode modes[kMaxModes];
};

// phi factors and their second derivatives, FishFry.hpp:22-41 and :71-86.
struct PointFactors {
  double px, py, pz, dpx, dpy, dpz;
};

__device__ __forceinline__ PointFactors factors(const FieldArgs &a, int i, int j, int k) {
  PointFactors q;
  const double x = a.xlo + i * a.dx;
  const double cx = cos(x), sx = sin(x), ex = exp(sx);
  q.px = cx * ex;
  q.dpx = -ex * sx * cx * (sx + 3.0);
  const double y = a.ylo + j * a.dy;
  const double cy = cos(y), sy = sin(y), ey = exp(cy);
  q.py = sy * ey;
  q.dpy = sy * ey * (sy * sy - 3.0 * cy - 1.0);
  const double z = a.zlo + k * a.dz;
  const double cz = cos(z), sz = sin(z), ez = exp(cz);
  q.pz = cz * ez;
  q.dpz = ez * (3.0 * sz * sz - cz * cz * cz - 1.0);
  return q;
}

// sum over modes of w_m * cos(k_m . x + theta_m), w_m = a_m (f) or -a_m/|k_m|^2 (phi)
__device__ __forceinline__ double modes_sum(const FieldArgs &a, int i, int j, int k, bool solution) {
  double v = 0.0;
  const double x = a.xlo + i * a.dx, y = a.ylo + j * a.dy, z = a.zlo + k * a.dz;
  for (int m = 0; m < a.nmodes; m++) {
    const ff_mode &md = a.modes[m];
    const int k2 = md.kx * md.kx + md.ky * md.ky + md.kz * md.kz;
    if (k2 == 0) continue;
    const double w = solution ? -md.a / (double)k2 : md.a;
    v += w * cos((double)md.kx * x + (double)md.ky * y + (double)md.kz * z + md.theta);
  }
  return v;
}

template <typename T>
__global__ void __launch_bounds__(256) k_init(const FieldArgs a, T *__restrict__ f) {
  const long N = (long)a.ni * a.nj * a.nk;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const int k = (int)(q % a.nk);
    const long ij = q / a.nk;
    const int j = (int)(ij % a.nj);
    const int i = (int)(ij / a.nj);
    const PointFactors p = factors(a, i, j, k);
    double v = p.px * p.py * p.dpz + p.px * p.dpy * p.pz + p.dpx * p.py * p.pz;   // FishFry.hpp:44
    if (a.nmodes) v += modes_sum(a, i, j, k, false);
    f[q] = (T)v;
  }
}

// Stage 1: per-block {sum|d|, sum d^2, max|d|} over a fixed strided slice of
// the points, reduced in a fixed tree.  NaN propagates through the max, as the
// reference's integer atomicMax on the bit pattern does.
template <typename T>
__global__ void __launch_bounds__(kSumThreads) k_diff(const FieldArgs a, const T *__restrict__ phi,
                                                      double *__restrict__ partial) {
  __shared__ double s1[kSumThreads], s2[kSumThreads], sm[kSumThreads];
  const long N = (long)a.ni * a.nj * a.nk;
  double t1 = 0, t2 = 0, tm = 0;
  for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < N; q += (long)gridDim.x * blockDim.x) {
    const int k = (int)(q % a.nk);
    const long ij = q / a.nk;
    const int j = (int)(ij % a.nj);
    const int i = (int)(ij / a.nj);
    const PointFactors p = factors(a, i, j, k);
    double ex = p.px * p.py * p.pz;
    if (a.nmodes) ex += modes_sum(a, i, j, k, true);
    const double d = fabs(ex - (phi ? (double)phi[q] : 0.0));   // FishFry.hpp:89
    t1 += d;
    t2 += d * d;
    tm = (d > tm || d != d) ? d : tm;
  }
  s1[threadIdx.x] = t1;
  s2[threadIdx.x] = t2;
  sm[threadIdx.x] = tm;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
      const double o = sm[threadIdx.x + w];
      if (o > sm[threadIdx.x] || o != o) sm[threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x + 0] = s1[0];
    partial[3 * blockIdx.x + 1] = s2[0];
    partial[3 * blockIdx.x + 2] = sm[0];
  }
}

// Stage 2: one block folds the per-block partials in a fixed order.
__global__ void __launch_bounds__(kSumThreads) k_diff_final(const double *__restrict__ partial, int nb,
                                                            double *__restrict__ out) {
  __shared__ double s1[kSumThreads], s2[kSumThreads], sm[kSumThreads];
  double t1 = 0, t2 = 0, tm = 0;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    t1 += partial[3 * b];
    t2 += partial[3 * b + 1];
    const double o = partial[3 * b + 2];
    tm = (o > tm || o != o) ? o : tm;
  }
  s1[threadIdx.x] = t1;
  s2[threadIdx.x] = t2;
  sm[threadIdx.x] = tm;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
      const double o = sm[threadIdx.x + w];
      if (o > sm[threadIdx.x] || o != o) sm[threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = s1[0];
    out[1] = s2[0];
    out[2] = sm[0];
  }
}

static int field_args(const int n[3], const double xlo[3], const double dx[3], int nmodes, const ff_mode *modes,
                      FieldArgs &a) {
  if (!n || !xlo || !dx) return set_error(FF_ERR_INVALID, "null argument");
  for (int d = 0; d < 3; d++)
    if (n[d] < 1) return set_error(FF_ERR_INVALID, "n[%d] = %d < 1", d, n[d]);
  if (nmodes < 0 || nmodes > kMaxModes || (nmodes > 0 && !modes))
    return set_error(FF_ERR_INVALID, "nmodes = %d outside [0, %d]", nmodes, kMaxModes);
  std::memset(&a, 0, sizeof(a));
  a.ni = n[0];
  a.nj = n[1];
  a.nk = n[2];
  a.xlo = xlo[0];
  a.ylo = xlo[1];
  a.zlo = xlo[2];
  a.dx = dx[0];
  a.dy = dx[1];
  a.dz = dx[2];
  a.nmodes = nmodes;
  for (int m = 0; m < nmodes; m++) a.modes[m] = modes[m];
  return FF_OK;
}

static unsigned grid_for(long N, int threads) {
  long b = (N + threads - 1) / threads;
  return (unsigned)(b < 148L * 32 ? (b < 1 ? 1 : b) : 148L * 32);
}

// ---------------------------------------------------------------------------
// Error sums without any device allocation.
//
// Some callers cannot allocate device memory at the point where they want the
// error norms: a host application whose own pool allocator has already
// reserved the device memory, a time-critical loop where cudaMalloc's implicit
// device synchronisation is not acceptable, or plug-in code that may not call
// the CUDA allocator at all.  For them the partial sums live in a fixed
// file-scope device array instead of a per-call buffer: every GPU that loads
// this library holds it (about 384 KB) until the process exits.
//
// Each block reduces one contiguous chunk of points in a fixed order.  The
// chunk length is a function of N alone (about N / kNoAllocBlocks, a multiple
// of kSumThreads), so small grids still spread over every SM and the
// summation order is the same on every call for a given grid.  The grid is
// limited to kNoAllocMaxPoints = 2^30 points (1024^3); the array holds the
// partials of at most kNoAllocMaxChunks blocks plus the final triple.
constexpr int kNoAllocBlocks = 8 * 148;
constexpr int kNoAllocMaxChunks = 16384;
constexpr long kNoAllocMaxPoints = 1L << 30;
static __device__ __align__(256) double g_noalloc_partials[3 * kNoAllocMaxChunks + 3];

// Chunk length for a grid of N points: ceil(N / kNoAllocBlocks) rounded up to
// a multiple of kSumThreads; chunks = ceil(N / chunk) <= kNoAllocBlocks.
static long noalloc_chunk(long N) {
  long c = (N + kNoAllocBlocks - 1) / kNoAllocBlocks;
  return (c + kSumThreads - 1) / kSumThreads * kSumThreads;
}

template <typename T>
__global__ void __launch_bounds__(kSumThreads) k_diff_chunks(const FieldArgs a, const T *__restrict__ phi,
                                                             long chunk, double *__restrict__ partial) {
  __shared__ double s1[kSumThreads], s2[kSumThreads], sm[kSumThreads];
  const long N = (long)a.ni * a.nj * a.nk;
  const long q0 = (long)blockIdx.x * chunk;
  const long q1 = q0 + chunk < N ? q0 + chunk : N;
  double t1 = 0, t2 = 0, tm = 0;
  for (long q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
    const int k = (int)(q % a.nk);
    const long ij = q / a.nk;
    const int j = (int)(ij % a.nj);
    const int i = (int)(ij / a.nj);
    const PointFactors p = factors(a, i, j, k);
    double ex = p.px * p.py * p.pz;
    if (a.nmodes) ex += modes_sum(a, i, j, k, true);
    const double d = fabs(ex - (phi ? (double)phi[q] : 0.0));
    t1 += d;
    t2 += d * d;
    tm = (d > tm || d != d) ? d : tm;
  }
  s1[threadIdx.x] = t1;
  s2[threadIdx.x] = t2;
  sm[threadIdx.x] = tm;
  __syncthreads();
  for (int w = kSumThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) {
      s1[threadIdx.x] += s1[threadIdx.x + w];
      s2[threadIdx.x] += s2[threadIdx.x + w];
      const double o = sm[threadIdx.x + w];
      if (o > sm[threadIdx.x] || o != o) sm[threadIdx.x] = o;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    partial[3 * blockIdx.x + 0] = s1[0];
    partial[3 * blockIdx.x + 1] = s2[0];
    partial[3 * blockIdx.x + 2] = sm[0];
  }
}

// Device address of g_noalloc_partials on the current device.  The name is a
// host-side stand-in, not a device address, so it is looked up once per
// device (with that device current) and remembered.  A cudaDeviceReset in the
// process makes the remembered address stale (the module is reloaded, perhaps
// elsewhere): the entry point is not for use after a reset.
static int noalloc_partials(double **out) {
  static std::mutex mu;
  static void *addr[256] = {};
  int dev = 0;
  FF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 256) return set_error(FF_ERR_INVALID, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess)
      return set_error(FF_ERR_CUDA, "cudaGetSymbolAddress of the static partial-sum array failed: %s",
                       cudaGetErrorString(e));
    addr[dev] = p;
  }
  *out = static_cast<double *>(addr[dev]);
  return FF_OK;
}

}  // namespace ff

using namespace ff;

extern "C" {

int ff_init_field(const int n[3], const double xlo[3], const double dx[3], int nmodes, const ff_mode *modes,
                  int precision, void *f, void *stream) {
  FieldArgs a;
  int rc = field_args(n, xlo, dx, nmodes, modes, a);
  if (rc != FF_OK) return rc;
  if (!f) return set_error(FF_ERR_INVALID, "ff_init_field: null field");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long N = (long)n[0] * n[1] * n[2];
  if (precision == FF_FP64) k_init<double><<<grid_for(N, 256), 256, 0, st>>>(a, static_cast<double *>(f));
  else if (precision == FF_FP32) k_init<float><<<grid_for(N, 256), 256, 0, st>>>(a, static_cast<float *>(f));
  else return set_error(FF_ERR_INVALID, "ff_init_field: bad precision %d", precision);
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

int ff_error_sums(const int n[3], const double xlo[3], const double dx[3], int nmodes, const ff_mode *modes,
                  int precision, const void *phi, double sums[3], void *stream) {
  FieldArgs a;
  int rc = field_args(n, xlo, dx, nmodes, modes, a);
  if (rc != FF_OK) return rc;
  if (!sums) return set_error(FF_ERR_INVALID, "ff_error_sums: null sums");
  if (precision != FF_FP64 && precision != FF_FP32)
    return set_error(FF_ERR_INVALID, "ff_error_sums: bad precision %d", precision);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // scratch: kSumBlocks partial triples and the final triple, stream-ordered
  double *scratch = nullptr;
  FF_CUDA(cudaMallocAsync(reinterpret_cast<void **>(&scratch), (3 * kSumBlocks + 3) * sizeof(double), st));
  if (precision == FF_FP64)
    k_diff<double><<<kSumBlocks, kSumThreads, 0, st>>>(a, static_cast<const double *>(phi), scratch);
  else
    k_diff<float><<<kSumBlocks, kSumThreads, 0, st>>>(a, static_cast<const float *>(phi), scratch);
  k_diff_final<<<1, kSumThreads, 0, st>>>(scratch, kSumBlocks, scratch + 3 * kSumBlocks);
  cudaError_t e = cudaGetLastError();
  double host[3] = {0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, scratch + 3 * kSumBlocks, sizeof(host), cudaMemcpyDeviceToHost, st);
  cudaError_t ef = cudaFreeAsync(scratch, st);
  if (e == cudaSuccess) e = ef;
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return set_error(FF_ERR_CUDA, "ff_error_sums: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e));
  sums[0] = host[0];
  sums[1] = host[1];
  sums[2] = host[2];
  return FF_OK;
}

int ff_error_sums_noalloc(const int n[3], const double xlo[3], const double dx[3], int nmodes,
                          const ff_mode *modes, int precision, const void *phi, double sums[3], void *stream) {
  FieldArgs a;
  int rc = field_args(n, xlo, dx, nmodes, modes, a);
  if (rc != FF_OK) return rc;
  if (!sums) return set_error(FF_ERR_INVALID, "ff_error_sums_noalloc: null sums");
  if (precision != FF_FP64 && precision != FF_FP32)
    return set_error(FF_ERR_INVALID, "ff_error_sums_noalloc: bad precision %d", precision);
  const long N = (long)n[0] * n[1] * n[2];
  if (N > kNoAllocMaxPoints)
    return set_error(FF_ERR_UNSUPPORTED,
                     "ff_error_sums_noalloc: %ld points exceed the fixed partial-sum array's limit of %ld points", N,
                     kNoAllocMaxPoints);
  const long chunk = noalloc_chunk(N);
  const long chunks = (N + chunk - 1) / chunk;
  if (chunks > kNoAllocMaxChunks)   // cannot happen for N <= kNoAllocMaxPoints; kept as the array's guard
    return set_error(FF_ERR_UNSUPPORTED, "ff_error_sums_noalloc: %ld chunks exceed the fixed array", chunks);
  double *partial = nullptr;
  rc = noalloc_partials(&partial);
  if (rc != FF_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // every slot read below is written by this call first: nothing to clear
  if (precision == FF_FP64)
    k_diff_chunks<double><<<(unsigned)chunks, kSumThreads, 0, st>>>(a, static_cast<const double *>(phi), chunk,
                                                                    partial);
  else
    k_diff_chunks<float><<<(unsigned)chunks, kSumThreads, 0, st>>>(a, static_cast<const float *>(phi), chunk,
                                                                   partial);
  double *total = partial + 3 * kNoAllocMaxChunks;
  k_diff_final<<<1, kSumThreads, 0, st>>>(partial, (int)chunks, total);
  cudaError_t e = cudaGetLastError();
  double host[3] = {0, 0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(host, total, sizeof(host), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return set_error(FF_ERR_CUDA, "ff_error_sums_noalloc: %s (%s)", cudaGetErrorName(e), cudaGetErrorString(e));
  sums[0] = host[0];
  sums[1] = host[1];
  sums[2] = host[2];
  return FF_OK;
}

// SplitMix64 (Steele, Lea and Flood, OOPSLA 2014) as a counter stream, and
// Box-Muller for the normal amplitudes.
int ff_modes_generate(uint64_t seed, int count, int kmax, const int kaxis[3], double sigma, ff_mode *out) {
  if (count < 0 || (count > 0 && !out) || !kaxis) return set_error(FF_ERR_INVALID, "ff_modes_generate: bad argument");
  uint64_t s = seed;
  auto next = [&]() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  auto uniform = [&]() { return (double)(next() >> 11) * 0x1.0p-53; };
  const long kmax2 = (long)kmax * kmax;
  const bool possible = kmax > 0 && (kaxis[0] > 0 || kaxis[1] > 0 || kaxis[2] > 0);
  for (int m = 0; m < count; m++) {
    ff_mode md{0, 0, 0, 0.0, 0.0};
    if (possible) {
      for (;;) {
        const int kx = (int)(next() % (uint64_t)(2 * kaxis[0] + 1)) - kaxis[0];
        const int ky = (int)(next() % (uint64_t)(2 * kaxis[1] + 1)) - kaxis[1];
        const int kz = (int)(next() % (uint64_t)(2 * kaxis[2] + 1)) - kaxis[2];
        const long k2 = (long)kx * kx + (long)ky * ky + (long)kz * kz;
        if (k2 == 0 || k2 > kmax2) continue;
        md.kx = kx;
        md.ky = ky;
        md.kz = kz;
        break;
      }
      const double u1 = 1.0 - uniform();
      const double u2 = uniform();
      md.a = sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
      md.theta = 2.0 * M_PI * uniform();
    }
    out[m] = md;
  }
  return FF_OK;
}

}  // extern "C"
