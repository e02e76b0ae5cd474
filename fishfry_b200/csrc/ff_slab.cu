// Multi-rank solve over an x-slab decomposition: the device phases of one
// rank.  The reference distributes the grid over an mi x mj x mk task grid
// and moves pencils with MPI_Alltoall (ParisPencil.cpp:23-75, :128-421); with
// the task grid (P, 1, 1) its z and y transforms are local and only the x
// pencils need an exchange (its commI, ParisPencil.cpp:236, :312).  This file
// implements that case on GPUs:
//
//   rank r holds planes i in [r*di, r*di + planes) of the real field,
//     di = ceil(n0 / P)                                (ParisPencil.cpp:54)
//   x pencils: rank p holds rows j in [p*djp, p*djp + rows), every i,
//     djp = ceil(n1 / P)                               (ParisPencil.cpp:61)
//   the block of an exchange from rank r to rank p holds the spectrum values
//     of r's planes and p's rows: [i - r*di][j - p*djp][kh], di x djp x nhp
//     complex values (the reference's countI)
//
//   forward  z R2C (density -> potential, the single-grid z pass on the
//            slab) and y forward, whose last stage stores row j of plane i
//            into the block for rank j / djp (pack fused into the y pass)
//   x        on the x pencils (every rank's block from the exchange, one after
//            another: [i][j - p*djp][kh]), forward, filter with the global j,
//            inverse; the last stage stores row i into the block for rank
//            i / di (pack fused into the x pass)
//   backward y inverse reading row j of plane i from the block of rank
//            j / djp (unpack fused into the y pass), z C2R into potential
//
// The destination of every block is a pointer the caller passes, so the
// exchanges can be an all-to-all between separate send and receive buffers or
// stores straight into another rank's buffer.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>

#include "ff_fft.cuh"
#include "ff_plan.hpp"
#include "ff_status.hpp"
#include "ff_tiles.cuh"

namespace ff {

constexpr int kSlabMaxRanks = 64;

template <typename T> struct SlabArgs {
  using C = typename Cplx<T>::type;
  int di, djp;           // planes per rank, pencil rows per rank
  int j0, njg;           // first global row of this rank's pencils; rows of the whole grid
  int nhp;               // row pitch in complex values
  C *dst[kSlabMaxRanks];  // base of the block for each destination rank
};

#define FF_FOR_EACH_SLAB_N(X) X(64) X(128) X(256) X(512)

// y forward of one TMA-loaded tile of the rank's slab (plane o); row j goes
// to the block of rank j / djp.
template <typename T, int N>
__global__ void __launch_bounds__(kZThreads, 3)
    k_slab_yfwd(const __grid_constant__ CUtensorMap tmap, const PassArgs<T> a, const SlabArgs<T> s, int box_rows) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  C *sm = reinterpret_cast<C *>(align128(smraw));
  const int n = N > 0 ? N : a.ax[1].n;
  const int ktiles = (a.nh + W - 1) / W;
  const int o = blockIdx.x / ktiles, kt = blockIdx.x - o * ktiles;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (!tma_tile<C, W, false>(&tmap, sm, &mbar, 0, n, box_rows, o, kt, a.status, a.wait_iters)) return;
  const int kh0 = kt * W;
  auto row_at = [&](int j) {
    const int p = j / s.djp;
    return s.dst[p] + ((long)o * s.djp + (j - p * s.djp)) * s.nhp + kh0;
  };
  PointTile<W, C> tile{sm};
  y_tile_rows<T, W, false, N>(tile, row_at, a, kt, sm);
}

// x pass of one TMA-loaded tile of the rank's pencils (local row o, global
// row s.j0 + o); row i goes to the block of rank i / di.
template <typename T, int N>
__global__ void __launch_bounds__(kZThreads, 3)
    k_slab_x(const __grid_constant__ CUtensorMap tmap, const PassArgs<T> a, const SlabArgs<T> s, int box_rows) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  C *sm = reinterpret_cast<C *>(align128(smraw));
  const int n = N > 0 ? N : a.ax[0].n;
  const int ktiles = (a.nh + W - 1) / W;
  const int o = blockIdx.x / ktiles, kt = blockIdx.x - o * ktiles;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (!tma_tile<C, W, true>(&tmap, sm, &mbar, 0, n, box_rows, o, kt, a.status, a.wait_iters)) return;
  const int kh0 = kt * W;
  const int ncol = min(W, a.nh - kh0);
  auto gst = [&](int i, int c, C v) {
    const int q = i / s.di;
    if (c < ncol) s.dst[q][((long)(i - q * s.di) * s.djp + o) * s.nhp + kh0 + c] = v;
  };
  x_tile_core<T, W, N>(a, s.j0 + o, s.njg, kt, sm, gst);
}

// y inverse of plane o of the rank's slab: row j is read from the block that
// rank j / djp sent (`packed` holds the P blocks one after another); the
// result goes to the slab's spectrum `out`.
template <typename T, int N>
__global__ void __launch_bounds__(kZThreads, 3)
    k_slab_yinv(const typename Cplx<T>::type *__restrict__ packed, typename Cplx<T>::type *out, const PassArgs<T> a,
                const SlabArgs<T> s) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  extern __shared__ unsigned char smraw[];
  C *sm = reinterpret_cast<C *>(align128(smraw));
  const int ktiles = (a.nh + W - 1) / W;
  const int o = blockIdx.x / ktiles, kt = blockIdx.x - o * ktiles;
  const int kh0 = kt * W;
  const int ncol = min(W, a.nh - kh0);
  const long block = (long)s.di * s.djp * s.nhp;
  auto ldg = [&](int j, int c) -> C {
    const int p = j / s.djp;
    return c < ncol ? __ldg(packed + p * block + ((long)o * s.djp + (j - p * s.djp)) * s.nhp + kh0 + c)
                    : mk((T)0, (T)0);
  };
  y_tile<T, W, true, N>(ldg, out, a, o, kt, sm);
}

template <typename T> using SlabYfwdKernel = void (*)(const CUtensorMap, const PassArgs<T>, const SlabArgs<T>, int);
template <typename T> using SlabXKernel = void (*)(const CUtensorMap, const PassArgs<T>, const SlabArgs<T>, int);
template <typename T>
using SlabYinvKernel = void (*)(const typename Cplx<T>::type *, typename Cplx<T>::type *, const PassArgs<T>,
                                const SlabArgs<T>);

template <typename T> static SlabYfwdKernel<T> slab_yfwd_kernel(int n) {
#define FF_CASE(NN) if (n == NN) return k_slab_yfwd<T, NN>;
  FF_FOR_EACH_SLAB_N(FF_CASE)
#undef FF_CASE
  return k_slab_yfwd<T, 0>;
}
template <typename T> static SlabXKernel<T> slab_x_kernel(int n) {
#define FF_CASE(NN) if (n == NN) return k_slab_x<T, NN>;
  FF_FOR_EACH_SLAB_N(FF_CASE)
#undef FF_CASE
  return k_slab_x<T, 0>;
}
template <typename T> static SlabYinvKernel<T> slab_yinv_kernel(int n) {
#define FF_CASE(NN) if (n == NN) return k_slab_yinv<T, NN>;
  FF_FOR_EACH_SLAB_N(FF_CASE)
#undef FF_CASE
  return k_slab_yinv<T, 0>;
}

static int largest_divisor_upto(int n, int cap) {
  for (int d = std::min(n, cap); d >= 1; d--)
    if (n % d == 0) return d;
  return 1;
}

}  // namespace ff

using namespace ff;

struct ff_slab {
  int n[3];
  int precision;
  int P, rank;
  int di, djp;
  int planes, first_plane;   // this rank's planes of the real field
  int rows, first_row;       // this rank's rows of the x pencils
  int nh, nhp;
  double dd[3];              // wavenumber scales of the whole grid (ParisPencil.cpp:9-11)
  size_t block;              // complex values per exchange block
  size_t bytes;              // bytes each of density and potential must hold
  ff_plan *local;            // planes x n1 x n2: z and y passes
  ff_plan *pencil;           // n0 x max(rows, 1) x n2: the x axis tables
  int ybox, xbox;            // TMA box rows of the y and x tiles
  size_t ysmem, xsmem, yismem;
};

namespace ff {

// Kernel arguments of a slab phase; dst (P block pointers) may be NULL for
// a phase that stores no blocks.
template <typename T> static SlabArgs<T> slab_args(const ff_slab *s, void *const *dst) {
  SlabArgs<T> a;
  std::memset(&a, 0, sizeof(a));
  a.di = s->di;
  a.djp = s->djp;
  a.j0 = s->first_row;
  a.njg = s->n[1];
  a.nhp = s->nhp;
  if (dst)
    for (int p = 0; p < s->P; p++) a.dst[p] = static_cast<typename Cplx<T>::type *>(dst[p]);
  return a;
}

// PassArgs of a slab plan with the whole grid's wavenumber scales and 1/N,
// which the local plans (built for their own extents) do not have.
template <typename T> static PassArgs<T> slab_pass_args(const ff_slab *s, const ff_plan *p) {
  PassArgs<T> a = pass_args<T>(p);
  for (int d = 0; d < 3; d++) a.dd[d] = s->dd[d];
  a.invN = 1.0 / (double(s->n[0]) * double(s->n[1]) * double(s->n[2]));
  return a;
}

template <typename T> static int slab_forward(const ff_slab *s, void *density, void *potential, void *const *dst,
                                              cudaStream_t st) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  if (s->planes == 0) return FF_OK;
  int rc = plan_launch_z(s->local, false, density, potential, st);
  if (rc != FF_OK) return rc;
  CUtensorMap map;
  rc = encode_spectrum_map(potential, s->planes, s->n[1], s->nh, s->nhp, sizeof(T), W, s->ybox, false, &map);
  if (rc != FF_OK) return rc;
  const PassArgs<T> a = slab_pass_args<T>(s, s->local);
  const SlabArgs<T> sa = slab_args<T>(s, dst);
  const int ktiles = (s->nh + W - 1) / W;
  slab_yfwd_kernel<T>(s->n[1])<<<s->planes * ktiles, kZThreads, s->ysmem, st>>>(map, a, sa, s->ybox);
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

template <typename T> static int slab_xpass(const ff_slab *s, const void *pencils, void *const *dst,
                                            cudaStream_t st) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  if (s->rows == 0) return FF_OK;
  CUtensorMap map;
  int rc = encode_spectrum_map(const_cast<void *>(pencils), s->n[0], s->djp, s->nh, s->nhp, sizeof(T), W, s->xbox,
                               true, &map);
  if (rc != FF_OK) return rc;
  PassArgs<T> a = slab_pass_args<T>(s, s->pencil);
  a.nj = s->djp;   // the pencil array's row count (its plane pitch)
  const SlabArgs<T> sa = slab_args<T>(s, dst);
  const int ktiles = (s->nh + W - 1) / W;
  slab_x_kernel<T>(s->n[0])<<<s->rows * ktiles, kZThreads, s->xsmem, st>>>(map, a, sa, s->xbox);
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

template <typename T> static int slab_backward(const ff_slab *s, const void *packed, void *density, void *potential,
                                               cudaStream_t st) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  if (s->planes == 0) return FF_OK;
  const PassArgs<T> a = slab_pass_args<T>(s, s->local);
  const SlabArgs<T> sa = slab_args<T>(s, nullptr);
  const int ktiles = (s->nh + W - 1) / W;
  slab_yinv_kernel<T>(s->n[1])<<<s->planes * ktiles, kZThreads, s->yismem, st>>>(
      static_cast<const C *>(packed), static_cast<C *>(density), a, sa);
  FF_CUDA(cudaGetLastError());
  return plan_launch_z(s->local, true, density, potential, st);
}

template <typename T> static int slab_configure(ff_slab *s) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  const int nj = s->n[1], ni = s->n[0];
  s->ybox = largest_divisor_upto(nj, 256);
  s->xbox = largest_divisor_upto(ni, 256);
  s->ysmem = (size_t)nj * W * sizeof(C) + 128;
  s->yismem = s->ysmem;
  s->xsmem = (size_t)ni * W * sizeof(C) + 128;
  size_t avail = 0;
  int rc = allow_dyn_smem_fn(reinterpret_cast<const void *>(slab_yfwd_kernel<T>(nj)), &avail);
  if (rc == FF_OK && s->ysmem > avail) rc = set_error(FF_ERR_UNSUPPORTED, "ff_slab_create: y tile does not fit");
  if (rc == FF_OK) rc = allow_dyn_smem_fn(reinterpret_cast<const void *>(slab_yinv_kernel<T>(nj)), &avail);
  if (rc == FF_OK && s->yismem > avail) rc = set_error(FF_ERR_UNSUPPORTED, "ff_slab_create: y tile does not fit");
  if (rc == FF_OK) rc = allow_dyn_smem_fn(reinterpret_cast<const void *>(slab_x_kernel<T>(ni)), &avail);
  if (rc == FF_OK && s->xsmem > avail) rc = set_error(FF_ERR_UNSUPPORTED, "ff_slab_create: x tile does not fit");
  return rc;
}

}  // namespace ff

extern "C" {

int ff_slab_create(const int n[3], const double lo[3], const double hi[3], int precision, int nranks, int rank,
                   ff_slab **out) {
  if (!n || !lo || !hi || !out) return set_error(FF_ERR_INVALID, "ff_slab_create: null argument");
  *out = nullptr;
  if (nranks < 1 || nranks > kSlabMaxRanks)
    return set_error(FF_ERR_TASKS, "ff_slab_create: %d ranks (1..%d)", nranks, kSlabMaxRanks);
  if (rank < 0 || rank >= nranks) return set_error(FF_ERR_INVALID, "ff_slab_create: rank %d of %d", rank, nranks);
  if (precision != FF_FP64 && precision != FF_FP32)
    return set_error(FF_ERR_INVALID, "ff_slab_create: precision %d", precision);
  for (int d = 0; d < 3; d++) {
    if (n[d] < 1) return set_error(FF_ERR_INVALID, "ff_slab_create: n[%d] = %d < 1", d, n[d]);
    if (n[d] > FF_MAX_AXIS)
      return set_error(FF_ERR_UNSUPPORTED, "ff_slab_create: n[%d] = %d is above %d", d, n[d], FF_MAX_AXIS);
    if (!smooth2357(n[d]))
      return set_error(FF_ERR_UNSUPPORTED, "ff_slab_create: n[%d] = %d has a prime factor above 7", d, n[d]);
  }
  if (n[0] < nranks || n[1] < nranks)   // main.cpp:20 (n >= m) for the slab and the pencils
    return set_error(FF_ERR_TASKS, "ff_slab_create: %d ranks need at least %d points along x and y", nranks, nranks);
  ff_slab *s = new ff_slab();
  std::memset(s, 0, sizeof(*s));
  for (int d = 0; d < 3; d++) s->n[d] = n[d];
  s->precision = precision;
  s->P = nranks;
  s->rank = rank;
  s->di = (n[0] + nranks - 1) / nranks;
  s->djp = (n[1] + nranks - 1) / nranks;
  s->first_plane = std::min(rank * s->di, n[0]);
  s->planes = std::min(s->di, n[0] - s->first_plane);
  s->first_row = std::min(rank * s->djp, n[1]);
  s->rows = std::min(s->djp, n[1] - s->first_row);
  s->nh = n[2] / 2 + 1;
  s->nhp = precision == FF_FP64 ? s->nh : (s->nh + 1) & ~1;
  const size_t csz = precision == FF_FP64 ? 16 : 8;
  s->block = (size_t)s->di * s->djp * s->nhp;
  const size_t real = (size_t)s->planes * n[1] * n[2] * (csz / 2);
  const size_t spec = (size_t)s->planes * n[1] * s->nhp * csz;
  s->bytes = std::max({real, spec, (size_t)nranks * s->block * csz});
  for (int d = 0; d < 3; d++)   // ParisPencil.cpp:9-11; 0 on a one-point axis, as the single-grid plan
    s->dd[d] = n[d] > 1 ? 2.0 * M_PI * double(n[d] - 1) / (double(n[d]) * (hi[d] - lo[d])) : 0.0;
  // the local plans give the passes their axis tables and launch shapes; the
  // wavenumber scales and 1/N of the whole grid are passed to the kernels
  // separately (slab_pass_args)
  const int ln[3] = {std::max(s->planes, 1), n[1], n[2]};
  const int pn[3] = {n[0], std::max(s->rows, 1), n[2]};
  int rc = ff_plan_create(ln, lo, hi, precision, &s->local);
  if (rc == FF_OK) rc = ff_plan_create(pn, lo, hi, precision, &s->pencil);
  if (rc == FF_OK) rc = precision == FF_FP64 ? slab_configure<double>(s) : slab_configure<float>(s);
  if (rc != FF_OK) {
    ff_slab_destroy(s);
    return rc;
  }
  *out = s;
  return FF_OK;
}

int ff_slab_layout(const ff_slab *s, int out[8], size_t *bytes, size_t *block_bytes) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_slab_layout: null slab");
  if (out) {
    const int v[8] = {s->P, s->rank, s->di, s->djp, s->first_plane, s->planes, s->first_row, s->rows};
    for (int q = 0; q < 8; q++) out[q] = v[q];
  }
  if (bytes) *bytes = s->bytes;
  if (block_bytes) *block_bytes = s->block * (s->precision == FF_FP64 ? 16 : 8);
  return FF_OK;
}

static int slab_check_dst(const ff_slab *s, void *const *dst, const char *who) {
  if (!dst) return set_error(FF_ERR_INVALID, "%s: null block pointers", who);
  for (int p = 0; p < s->P; p++)
    if (!dst[p] || ((uintptr_t)dst[p] & 15)) return set_error(FF_ERR_INVALID, "%s: block pointer %d", who, p);
  return FF_OK;
}

int ff_slab_forward(const ff_slab *s, void *density, void *potential, void *const *dst, void *stream) {
  if (!s || !density || !potential) return set_error(FF_ERR_INVALID, "ff_slab_forward: null argument");
  if (((uintptr_t)density | (uintptr_t)potential) & 15)
    return set_error(FF_ERR_INVALID, "ff_slab_forward: buffers must be 16-byte aligned");
  int rc = slab_check_dst(s, dst, "ff_slab_forward");
  if (rc != FF_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return s->precision == FF_FP64 ? slab_forward<double>(s, density, potential, dst, st)
                                 : slab_forward<float>(s, density, potential, dst, st);
}

int ff_slab_xpass(const ff_slab *s, const void *pencils, void *const *dst, void *stream) {
  if (!s || !pencils) return set_error(FF_ERR_INVALID, "ff_slab_xpass: null argument");
  if ((uintptr_t)pencils & 15) return set_error(FF_ERR_INVALID, "ff_slab_xpass: pencils must be 16-byte aligned");
  int rc = slab_check_dst(s, dst, "ff_slab_xpass");
  if (rc != FF_OK) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return s->precision == FF_FP64 ? slab_xpass<double>(s, pencils, dst, st) : slab_xpass<float>(s, pencils, dst, st);
}

int ff_slab_backward(const ff_slab *s, const void *packed, void *density, void *potential, void *stream) {
  if (!s || !packed || !density || !potential) return set_error(FF_ERR_INVALID, "ff_slab_backward: null argument");
  if (((uintptr_t)packed | (uintptr_t)density | (uintptr_t)potential) & 15)
    return set_error(FF_ERR_INVALID, "ff_slab_backward: buffers must be 16-byte aligned");
  if (packed == density) return set_error(FF_ERR_INVALID, "ff_slab_backward: packed and density must differ");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return s->precision == FF_FP64 ? slab_backward<double>(s, packed, density, potential, st)
                                 : slab_backward<float>(s, packed, density, potential, st);
}

int ff_slab_check(const ff_slab *s, void *stream) {
  if (!s) return set_error(FF_ERR_INVALID, "ff_slab_check: null slab");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = take_device_status(s->local, st);
  int rc2 = take_device_status(s->pencil, st);
  return rc != FF_OK ? rc : rc2;
}

int ff_slab_destroy(ff_slab *s) {
  if (!s) return FF_OK;
  int rc = FF_OK;
  if (s->local) rc = ff_plan_destroy(s->local);
  if (s->pencil) {
    int r2 = ff_plan_destroy(s->pencil);
    if (rc == FF_OK) rc = r2;
  }
  delete s;
  return rc;
}

}  // extern "C"
