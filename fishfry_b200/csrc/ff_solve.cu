// The five-pass Poisson solve and its plan: the B200 replacement of
// ParisPencil (ParisPencil.hpp:11-59, ParisPencil.cpp:7-425) on one GPU.
//
// Layout in HBM (x slowest, z fastest, as FishFry.hpp:43 indexes):
//   real field   f[i][j][k]             T = double or float
//   half spectrum S[i][j][kh], kh < nh = nk/2+1, row pitch nhp complex values
// Passes (each reads and writes HBM once; no standalone transposes):
//   1 Z-fwd   density(real) -> potential(S): R2C along z, two real lines per
//             complex transform                            (ParisPencil.cpp:152-165)
//   2 Y-fwd   potential(S) in place: C2C along j, tiles of W kh columns x nj
//             rows read with row stride nhp               (:173-212, transpose :198 fused)
//   3 X       potential(S) in place: C2C forward along i, -1/k^2 * 1/N filter
//             with the zero mode set to 0, C2C inverse along i, in one pass
//                                                          (:221-297, :406-421)
//   4 Y-inv   potential(S) -> density(S)                  (:322-334)
//   5 Z-inv   density(S) -> potential(real): C2R along z  (:368-380)
// The reference's 12 reorder kernels and 6 MPI_Alltoall self-copies reduce to
// the choice of row stride in passes 2-4.

#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "ff_fft.cuh"
#include "ff_status.hpp"

namespace ff {

template <typename T> struct PassArgs {
  using C = typename Cplx<T>::type;
  int ni, nj, nk, nh, nhp;
  AxisDev<C> ax[3];        // 0: x (n = ni), 1: y (nj), 2: z (nk)
  const double *kk[3];     // (min(i, n-i) * dd)^2 per axis; kk[2] indexed by kh
  double invN;             // 1 / (ni*nj*nk)
  double dd[3];            // wavenumber scales (ParisPencil.cpp:9-11)
  int *status;             // device status word (kDev*), 0 = ok
};

constexpr int kZThreads = 256;

// Lengths with compile-time specialised kernels (fully unrolled stages);
// every other length runs the same kernels with the plan read at run time.
#define FF_FOR_EACH_SPECIAL_N(X) X(256) X(512) X(1024)

// Frequency of a last-stage DIF position: arithmetic for compile-time plans,
// one table load per radix group otherwise.
template <int N> struct RevLastOf { using type = RevCT<N>; };
template <> struct RevLastOf<0> { using type = RevLast<0, 0>; };
template <int N, typename C> __device__ __forceinline__ typename RevLastOf<N>::type rev_last(const AxisDev<C> &ax) {
  if constexpr (N > 0) {
    return RevCT<N>{};
  } else {
    const int R = ax.radix[ax.nstages - 1];
    return RevLast<0, 0>{ax.rev, R, ax.n / R};
  }
}

// ------------------------------------------------------------------ pass 1
// Tile: W line pairs (2W consecutive real lines), two line-major buffers A, B
// of pitch P.  Line pair c is transformed as z = f[line a] + i f[line b].
template <typename T, int N>
__global__ void __launch_bounds__(kZThreads) k_zfwd(const T *__restrict__ f, typename Cplx<T>::type *__restrict__ spec,
                                                    const PassArgs<T> a, int W, int P) {
  using C = typename Cplx<T>::type;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *A = reinterpret_cast<C *>(smraw);
  C *B = A + W * P;
  const long nlines = (long)a.ni * a.nj;
  const long line0 = (long)blockIdx.x * (2 * W);
  const int nk = N > 0 ? N : a.nk;
  const AxisDev<C> &ax = a.ax[2];

  // stage 0 reads the two real lines straight from HBM, consecutive threads on
  // consecutive points of one line
  auto ldg = [&](int pos, int c) -> C {
    const long la = line0 + 2 * c;
    T x = 0, y = 0;
    if (la < nlines) x = f[la * nk + pos];
    if (la + 1 < nlines) y = f[(la + 1) * nk + pos];
    return mk(x, y);
  };
  LineTile<C> tA{A, P}, tB{B, P};
  LineTileRev<C, typename RevLastOf<N>::type> tBrev{tB, rev_last<N>(ax)};
  dif_all<N, false, Map::PosFast, 1, kZThreads, true, false>(ax, ldg, tA, tBrev, W);   // B: Z in natural order

  // split: A[k] = (Z[k] + conj Z[n-k]) / 2,  B[k] = (Z[k] - conj Z[n-k]) / (2i)
  const T h = (T)0.5;
  const int nh = a.nh;
  for (int it = threadIdx.x; it < W * nh; it += kZThreads) {
    const int k = it % nh;
    const int c = it / nh;
    const long la = line0 + 2 * c;
    if (la >= nlines) continue;
    const C z = tB(k, c);
    const C w = tB(k == 0 ? 0 : nk - k, c);
    spec[la * a.nhp + k] = mk(h * (z.x + w.x), h * (z.y - w.y));
    if (la + 1 < nlines) spec[(la + 1) * a.nhp + k] = mk(h * (z.y + w.y), h * (w.x - z.x));
  }
}

// ------------------------------------------------------------------ pass 5
template <typename T, int N>
__global__ void __launch_bounds__(kZThreads) k_zinv(const typename Cplx<T>::type *__restrict__ spec, T *__restrict__ out,
                                                    const PassArgs<T> a, int W, int P) {
  using C = typename Cplx<T>::type;
  extern __shared__ __align__(128) unsigned char smraw[];
  C *A = reinterpret_cast<C *>(smraw);
  C *B = A + W * P;
  const long nlines = (long)a.ni * a.nj;
  const long line0 = (long)blockIdx.x * (2 * W);
  const int nk = N > 0 ? N : a.nk;
  const int nh = a.nh;
  const AxisDev<C> &ax = a.ax[2];
  LineTile<C> tA{A, P}, tB{B, P};
  LineTileRev<C, typename RevLastOf<N>::type> tBrev{tB, rev_last<N>(ax)};

  // Z[k] = A[k] + i B[k] over the Hermitian extension, natural order in B; the
  // imaginary parts of the zero and Nyquist terms are dropped, as a C2R
  // transform does.
  for (int it = threadIdx.x; it < W * nh; it += kZThreads) {
    const int k = it % nh;
    const int c = it / nh;
    const long la = line0 + 2 * c;
    C sa = mk((T)0, (T)0), sb = mk((T)0, (T)0);
    if (la < nlines) sa = spec[la * a.nhp + k];
    if (la + 1 < nlines) sb = spec[(la + 1) * a.nhp + k];
    if (k == 0 || 2 * k == nk) {
      tB(k, c, mk(sa.x, sb.x));
    } else {
      tB(k, c, mk(sa.x - sb.y, sa.y + sb.x));
      tB(nk - k, c, mk(sa.x + sb.y, sb.x - sa.y));
    }
  }
  __syncthreads();
  dif_all<N, true, Map::PosFast, 1, kZThreads, true, false>(ax, tB, tA, tBrev, W);   // B: z in natural order

  for (int it = threadIdx.x; it < W * nk; it += kZThreads) {
    const int t = it % nk;
    const int c = it / nk;
    const long la = line0 + 2 * c;
    const C v = tB(t, c);
    if (la < nlines) out[la * nk + t] = v.x;
    if (la + 1 < nlines) out[(la + 1) * nk + t] = v.y;
  }
}

// ------------------------------------------------------------- passes 2-4
// Persistent strided pass.  A tile is W consecutive kh columns of all n rows
// of one plane (y pass: fixed i, rows j; x pass: fixed j, rows i), held
// point-major and brought in by TMA; results leave from registers straight
// to HBM in the last stage.
//
// The last DIF stage of the x forward transform, the filter and the first
// DIT stage of the inverse act on the same register group.
template <int R, int W, int NT, int NC, typename C, typename LD, typename ST, typename FL>
__device__ __forceinline__ void fused_filter_stage(int n_rt, LD &ld, ST &st, FL &filt) {
  const int n = NC ? NC : n_rt;
  auto body = [&](int it) {
    const int c = it % W;
    const int base = (it / W) * R;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = ld(base + r, c);
    Dft<R, false, C>::run(v);
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = filt(base + r, c, v[r]);
    Dft<R, true, C>::run(v);
#pragma unroll
    for (int r = 0; r < R; r++) st(base + r, c, v[r]);
  };
  if constexpr (NC > 0 && (W * (NC / R)) % NT == 0) {
    constexpr int ITER = W * (NC / R) / NT;
#pragma unroll
    for (int q = 0; q < ITER; q++) body((int)threadIdx.x + q * NT);
  } else {
    for (int it = threadIdx.x; it < W * (n / R); it += NT) body(it);
  }
}

// 1/x for x > 0 by two Newton-Raphson steps y <- y + y*(1 - x*y) from the
// single-precision reciprocal (about 2^-23 -> 2^-46 -> full double).
__device__ __forceinline__ double recip_pos(double x) {
  double y = (double)__frcp_rn((float)x);
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// One tile per block: TMA brings the tile into shared memory, the stages run,
// the last stage stores straight to HBM.  Blocks are dispatched in tile order
// (consecutive kh tiles of one plane share DRAM rows), and several blocks per
// SM overlap one another's loads and butterflies.
template <typename T, int W, bool XPASS, bool INV, int NT, int N>
__global__ void __launch_bounds__(NT, NT == 256 ? 3 : 1)
    k_strided(const __grid_constant__ CUtensorMap tmap, typename Cplx<T>::type *dst, const PassArgs<T> a,
              int box_rows) {
  using C = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  const AxisDev<C> &ax = XPASS ? a.ax[0] : a.ax[1];
  const int n = N > 0 ? N : ax.n;
  C *buf = reinterpret_cast<C *>((reinterpret_cast<uintptr_t>(smraw) + 127) & ~uintptr_t(127));
  const int ktiles = (a.nh + W - 1) / W;
  const int t = blockIdx.x;
  const int o = t / ktiles, kt = t - o * ktiles;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
    mbar_expect_tx(&mbar, (uint32_t)(n * W * sizeof(C)));
    for (int q = 0; q < n / box_rows; q++) {
      if (XPASS) tma_load_3d(buf + q * box_rows * W, &tmap, 2 * W * kt, o, q * box_rows, &mbar);
      else tma_load_3d(buf + q * box_rows * W, &tmap, 2 * W * kt, q * box_rows, o, &mbar);
    }
  }
  __syncthreads();   // barrier initialised before anyone polls it
  const bool ok = mbar_wait_bounded(&mbar, 0);
  if (__syncthreads_or(!ok)) {
    // the copy never completed: report and give it a bounded chance to land
    // before the block's shared memory is released
    if (threadIdx.x == 0) {
      atomicExch(a.status, kDevTmaTimeout);
      mbar_wait_bounded(&mbar, 0);
    }
    return;
  }
  const int kh0 = kt * W;
  const int ncol = min(W, a.nh - kh0);
  PointTile<W, C> tile{buf};
  const auto rl = rev_last<N>(ax);
  if (!XPASS) {
    const long base = (long)o * a.nj * a.nhp + kh0;
    const int pitch = a.nhp;
    auto gst = [&](int pos, int c, C v) {
      if (c < ncol) dst[base + (long)rl(pos) * pitch + c] = v;
    };
    dif_all<N, INV, Map::ColFast, W, NT, false, false>(ax, tile, tile, gst, W);
  } else {
    const int j = o;
    const long base = (long)j * a.nhp + kh0;
    const long pitch = (long)a.nj * a.nhp;
    auto gst = [&](int pos, int c, C v) {
      if (c < ncol) dst[base + pos * pitch + c] = v;
    };
    // d = -1/((i2 + j2) + k2) with i2 = (min(i, ni-i)*ddi)^2 etc., as
    // ParisPencil.cpp:276-279 forms it, times 1/N
    const int ni = a.ni;
    const double jd = double(min(j, a.nj - j)) * a.dd[1];
    const double j2 = jd * jd;
    const double ddi = a.dd[0], ddk = a.dd[2];
    const double minvN = -a.invN;
    auto filt = [&](int pos, int c, C v) -> C {
      const int kx = rl(pos);
      const int kh = kh0 + c;
      if (c >= ncol) return v;
      if ((kx | j | kh) == 0) return mk((T)0, (T)0);
      const double id = double(min(kx, ni - kx)) * ddi;
      const double kd = double(kh) * ddk;
      const double d = recip_pos((id * id + j2) + kd * kd) * minvN;
      return cscale(v, (T)d);
    };
    if constexpr (N > 0) {
      constexpr int S = plan_stages(N);
      constexpr int RF = plan_radix(N, S - 1);
      if constexpr (S > 1) {
        dif_ct<N, S - 1, 0, false, Map::ColFast, W, NT, false, true>(ax, tile, tile, tile, W);
        fused_filter_stage<RF, W, NT, N, C>(N, tile, tile, filt);
        __syncthreads();
        dit_ct<N, S - 2, true, Map::ColFast, W, NT, true>(ax, tile, gst, W);
      } else {
        fused_filter_stage<RF, W, NT, N, C>(N, tile, gst, filt);
      }
    } else {
      const int S = ax.nstages;
      if (S > 1) dif_rt<false, Map::ColFast, W, NT, false>(ax, S - 1, tile, tile, tile, W);
      with_radix(ax.radix[S - 1], [&](auto tag) {
        constexpr int R = decltype(tag)::value;
        if (S == 1) fused_filter_stage<R, W, NT, 0, C>(n, tile, gst, filt);
        else fused_filter_stage<R, W, NT, 0, C>(n, tile, tile, filt);
      });
      __syncthreads();
      if (S > 1) dit_rt<true, Map::ColFast, W, NT>(ax, S - 2, tile, gst, W);
    }
  }
}

// ------------------------------------------------------------- plan tables
template <typename C>
__global__ void k_twiddles(int n, C *tw) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)q / (double)n, &s, &c);   // exp(-2*pi*i*q/n) in FP64
    tw[q] = mk((decltype(tw[q].x))c, (decltype(tw[q].x))(-s));
  }
}

// (min(i, n-i) * dd)^2 in FP64, as ParisPencil.cpp:276-278 (sqr of the scaled index).
__global__ void k_wavenumbers(int n, int count, int folded, double dd, double *kk) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
    const double x = double(folded ? min(i, n - i) : i) * dd;
    kk[i] = x * x;
  }
}

}  // namespace ff

// ====================================================================== plan
using namespace ff;

namespace ff {

// Launch shape of a persistent strided pass.
struct StridedCfg {
  int N;          // specialised length of the kernel, 0 = runtime plan
  int threads;    // block size
  int W;          // columns per tile
  int box_rows;   // rows per TMA box (a divisor of n, at most 256)
  size_t smem;    // dynamic shared memory: one tile + alignment slack
  int grid;       // one block per tile
};

}  // namespace ff

struct ff_plan {
  int n[3];
  int precision;
  int nh, nhp;
  double dd[3];
  size_t bytes;
  int device;
  int num_sms;
  void *dmem;
  AxisDev<double2> axd[3];
  AxisDev<float2> axf[3];
  double *kk[3];
  int *status;
  int zN;              // z passes: specialised length, 0 = runtime plan
  int zW, zP;          // z passes: line pairs per block, line pitch in complex values
  size_t zsmem;
  unsigned ztiles;
  StridedCfg ycfg, xcfg;
  cudaEvent_t ev[FF_NUM_PHASES + 1];
};

namespace ff {

bool smooth235(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

// DIF radix order of the device plan (plan_radix in ff_fft.cuh).
static std::vector<int> factor_radices(int n) {
  std::vector<int> r;
  for (int s = 0; s < plan_stages(n); s++) r.push_back(plan_radix(n, s));
  return r;
}

// rev[pos]: frequency held at DIF output position pos.
static std::vector<int> digit_reversal(int n, const std::vector<int> &radix) {
  std::vector<int> rev(n);
  for (int pos = 0; pos < n; pos++) {
    int rem = pos, span = n, kmul = 1, k = 0;
    for (int r : radix) {
      span /= r;
      const int m = rem / span;
      rem %= span;
      k += m * kmul;
      kmul *= r;
    }
    rev[pos] = k;
  }
  return rev;
}

static thread_local char g_err[512];

int set_error(int status, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return status;
}

constexpr size_t kMaxDynSmem = 227 * 1024;   // per-block opt-in shared memory of sm_100

// Raises fn's dynamic shared-memory limit to what is left beside its static
// shared memory; returns that limit in *avail.
template <typename F> static int allow_dyn_smem(F fn, size_t *avail) {
  cudaFuncAttributes fa;
  FF_CUDA(cudaFuncGetAttributes(&fa, fn));
  const size_t lim = kMaxDynSmem - fa.sharedSizeBytes;
  FF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim));
  if (avail) *avail = lim;
  return FF_OK;
}

template <typename T>
using StridedKernel = void (*)(const CUtensorMap, typename Cplx<T>::type *, const PassArgs<T>, int);
template <typename T> using ZFwdKernel = void (*)(const T *, typename Cplx<T>::type *, const PassArgs<T>, int, int);
template <typename T>
using ZInvKernel = void (*)(const typename Cplx<T>::type *, T *, const PassArgs<T>, int, int);

// The specialised length for an axis of n points, or 0 (runtime plan).
static int special_n(int n) {
#define FF_CASE(NN) if (n == NN) return NN;
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return 0;
}

template <typename T> static ZFwdKernel<T> zfwd_kernel(int N) {
#define FF_CASE(NN) if (N == NN) return k_zfwd<T, NN>;
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return k_zfwd<T, 0>;
}
template <typename T> static ZInvKernel<T> zinv_kernel(int N) {
#define FF_CASE(NN) if (N == NN) return k_zinv<T, NN>;
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return k_zinv<T, 0>;
}

// kind: 0 = y forward, 1 = y inverse, 2 = x (forward, filter, inverse);
// 128-byte rows (W = 8 FP64 / 16 FP32), 256 threads.
template <typename T, int N> static StridedKernel<T> strided_n(int kind) {
  constexpr int W = 128 / (2 * (int)sizeof(T));
  return kind == 0 ? k_strided<T, W, false, false, 256, N>
                   : kind == 1 ? k_strided<T, W, false, true, 256, N> : k_strided<T, W, true, false, 256, N>;
}
template <typename T> static StridedKernel<T> strided_kernel(int kind, int N) {
#define FF_CASE(NN) if (N == NN) return strided_n<T, NN>(kind);
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return strided_n<T, 0>(kind);
}

// Largest divisor d of n with d <= cap and d % step == 0 (0 if none).
static int largest_divisor_at_most(int n, int cap, int step) {
  for (int d = std::min(n, cap); d >= 1; d--)
    if (n % d == 0 && d % step == 0) return d;
  return 0;
}

template <typename T> static int configure(ff_plan *p) {
  using C = typename Cplx<T>::type;
  const size_t csz = sizeof(C);
  // z passes: W line pairs, two line-major buffers of pitch P, ~64 KB per block
  const int align = csz == 16 ? 8 : 16;
  p->zN = special_n(p->n[2]);
  p->zP = (p->n[2] + align - 1) / align * align;
  const size_t per_pair = 2 * (size_t)p->zP * csz;
  p->zW = (int)std::max<size_t>(1, std::min<size_t>(8, (64 * 1024) / per_pair));
  p->zsmem = p->zW * per_pair;
  const long npairs = ((long)p->n[0] * p->n[1] + 1) / 2;
  p->ztiles = (unsigned)((npairs + p->zW - 1) / p->zW);
  int rc = allow_dyn_smem(zfwd_kernel<T>(p->zN), nullptr);
  if (rc == FF_OK) rc = allow_dyn_smem(zinv_kernel<T>(p->zN), nullptr);
  if (rc != FF_OK) return rc;
  // strided passes: one tile of W 128-byte columns x n rows per block
  const int W = 128 / (int)csz;
  for (int kind = 0; kind < 3; kind++) {
    StridedCfg &cfg = kind == 2 ? p->xcfg : p->ycfg;
    const int n = kind == 2 ? p->n[0] : p->n[1];
    cfg.N = special_n(n);
    cfg.threads = 256;
    cfg.W = W;
    cfg.box_rows = largest_divisor_at_most(n, 256, 1);
    cfg.smem = (size_t)n * W * csz + 128;
    StridedKernel<T> fn = strided_kernel<T>(kind, cfg.N);
    size_t avail = 0;
    rc = allow_dyn_smem(fn, &avail);
    if (rc != FF_OK) return rc;
    if (cfg.smem > avail) return set_error(FF_ERR_UNSUPPORTED, "no tile shape for an axis of %d points", n);
    const long ktiles = (p->nh + W - 1) / W;
    cfg.grid = (int)((kind == 2 ? p->n[1] : p->n[0]) * ktiles);
  }
  return FF_OK;
}

// cuTensorMapEncodeTiled, fetched from the driver through the runtime.
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void *f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(f);
  }
  return fn;
}

// Tensor map of a half spectrum at `base` viewed as (2*nh reals, nj, ni) with
// row pitch nhp complex values; box = one tile chunk of the y or x pass.
template <typename T> static int spectrum_map(const ff_plan *p, void *base, const StridedCfg &cfg, bool xpass,
                                              CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return set_error(FF_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t csz = 2 * sizeof(T);
  cuuint64_t dims[3] = {(cuuint64_t)2 * p->nh, (cuuint64_t)p->n[1], (cuuint64_t)p->n[0]};
  cuuint64_t strides[2] = {(cuuint64_t)p->nhp * csz, (cuuint64_t)p->nhp * csz * p->n[1]};
  cuuint32_t box[3] = {(cuuint32_t)(2 * cfg.W), xpass ? 1u : (cuuint32_t)cfg.box_rows,
                       xpass ? (cuuint32_t)cfg.box_rows : 1u};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = enc(map, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(FF_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FF_OK;
}

template <typename T> static PassArgs<T> pass_args(const ff_plan *p) {
  PassArgs<T> a;
  a.ni = p->n[0];
  a.nj = p->n[1];
  a.nk = p->n[2];
  a.nh = p->nh;
  a.nhp = p->nhp;
  for (int d = 0; d < 3; d++) {
    if constexpr (sizeof(T) == 8) a.ax[d] = p->axd[d];
    else a.ax[d] = p->axf[d];
    a.kk[d] = p->kk[d];
  }
  a.invN = 1.0 / (double(p->n[0]) * double(p->n[1]) * double(p->n[2]));
  for (int d = 0; d < 3; d++) a.dd[d] = p->dd[d];
  a.status = p->status;
  return a;
}

template <typename T>
static int launch_solve(const ff_plan *p, void *density, void *potential, cudaStream_t st, bool timed) {
  using C = typename Cplx<T>::type;
  const PassArgs<T> a = pass_args<T>(p);
  T *D = static_cast<T *>(density);
  T *P = static_cast<T *>(potential);
  C *Ds = reinterpret_cast<C *>(density);
  C *Ps = reinterpret_cast<C *>(potential);
  CUtensorMap ymapP, xmapP;
  int rc = spectrum_map<T>(p, potential, p->ycfg, false, &ymapP);
  if (rc == FF_OK) rc = spectrum_map<T>(p, potential, p->xcfg, true, &xmapP);
  if (rc != FF_OK) return rc;
  if (timed) FF_CUDA(cudaEventRecord(p->ev[0], st));
  zfwd_kernel<T>(p->zN)<<<p->ztiles, kZThreads, p->zsmem, st>>>(D, Ps, a, p->zW, p->zP);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[1], st));
  strided_kernel<T>(0, p->ycfg.N)<<<p->ycfg.grid, p->ycfg.threads, p->ycfg.smem, st>>>(ymapP, Ps, a,
                                                                                       p->ycfg.box_rows);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[2], st));
  strided_kernel<T>(2, p->xcfg.N)<<<p->xcfg.grid, p->xcfg.threads, p->xcfg.smem, st>>>(xmapP, Ps, a,
                                                                                       p->xcfg.box_rows);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[3], st));
  strided_kernel<T>(1, p->ycfg.N)<<<p->ycfg.grid, p->ycfg.threads, p->ycfg.smem, st>>>(ymapP, Ds, a,
                                                                                       p->ycfg.box_rows);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[4], st));
  zinv_kernel<T>(p->zN)<<<p->ztiles, kZThreads, p->zsmem, st>>>(Ds, P, a, p->zW, p->zP);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[5], st));
  return FF_OK;
}

// Reads and clears the device status word; FF_ERR_TIMEOUT if a bounded wait
// inside a kernel gave up.
static int take_device_status(const ff_plan *p, cudaStream_t st) {
  int h = 0;
  FF_CUDA(cudaMemcpyAsync(&h, p->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  FF_CUDA(cudaStreamSynchronize(st));
  if (h != kDevOk) {
    FF_CUDA(cudaMemsetAsync(p->status, 0, sizeof(int), st));
    FF_CUDA(cudaStreamSynchronize(st));
    return set_error(FF_ERR_TIMEOUT, "a TMA tile load did not complete within its wait limit (device status %d)", h);
  }
  return FF_OK;
}

}  // namespace ff

extern "C" {

const char *ff_version(void) { return "fishfry_b200 0.2 (sm_100a)"; }

const char *ff_last_error(void) { return g_err; }

const char *ff_status_string(int s) {
  switch (s) {
    case FF_OK: return "ok";
    case FF_ERR_INVALID: return "invalid argument";
    case FF_ERR_UNSUPPORTED: return "unsupported size";
    case FF_ERR_BYTES: return "buffer too small";
    case FF_ERR_CUDA: return "CUDA error";
    case FF_ERR_NOMEM: return "out of device memory";
    case FF_ERR_TIMEOUT: return "device wait timed out";
    case FF_ERR_TASKS: return "task grid other than 1x1x1";
    default: return "unknown status";
  }
}

const char *ff_phase_name(int p) {
  // phase names of the reference's stamps (ParisPencil.cpp:142-424) that
  // survive on one GPU, one per pass
  static const char *names[FF_NUM_PHASES] = {"Real-to-complex FFT in Z", "Forward FFT in Y", "X FFTs and filter",
                                             "Backward FFT in Y", "Complex-to-real FFT in Z"};
  return (p >= 0 && p < FF_NUM_PHASES) ? names[p] : "";
}

int ff_plan_create(const int n[3], const double lo[3], const double hi[3], int precision, ff_plan **out) {
  if (!n || !lo || !hi || !out) return set_error(FF_ERR_INVALID, "ff_plan_create: null argument");
  *out = nullptr;
  if (precision != FF_FP64 && precision != FF_FP32)
    return set_error(FF_ERR_INVALID, "ff_plan_create: precision %d is neither FF_FP64 nor FF_FP32", precision);
  for (int d = 0; d < 3; d++) {
    if (n[d] < 1) return set_error(FF_ERR_INVALID, "ff_plan_create: n[%d] = %d < 1", d, n[d]);
    if (n[d] > FF_MAX_AXIS || !smooth235(n[d]))
      return set_error(FF_ERR_UNSUPPORTED, "ff_plan_create: n[%d] = %d is not 2^a 3^b 5^c <= %d", d, n[d],
                       FF_MAX_AXIS);
    if (!(hi[d] > lo[d]) && n[d] > 1)
      return set_error(FF_ERR_INVALID, "ff_plan_create: hi[%d] <= lo[%d]", d, d);
  }
  ff_plan *p = new ff_plan();
  std::memset(p, 0, sizeof(*p));
  for (int d = 0; d < 3; d++) {
    p->n[d] = n[d];
    // ParisPencil.cpp:9-11; a one-point axis (hi == lo) has only wavenumber 0,
    // where the reference's formula would give 0/0
    p->dd[d] = (n[d] > 1) ? 2.0 * M_PI * double(n[d] - 1) / (double(n[d]) * (hi[d] - lo[d])) : 0.0;
  }
  p->precision = precision;
  p->nh = n[2] / 2 + 1;
  // FP32 rows are padded to an even count so every row starts 16-byte aligned
  p->nhp = precision == FF_FP64 ? p->nh : (p->nh + 1) & ~1;
  const size_t csz = precision == FF_FP64 ? 16 : 8;
  const size_t spec = (size_t)n[0] * n[1] * p->nhp * csz;
  const size_t real = (size_t)n[0] * n[1] * n[2] * (csz / 2);
  p->bytes = std::max(spec, real);
  if (cudaGetDevice(&p->device) != cudaSuccess ||
      cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device) != cudaSuccess) {
    delete p;
    return set_error(FF_ERR_CUDA, "ff_plan_create: no current CUDA device");
  }

  // device tables: per axis tw (n complex), rev and ipos (n ints); kk per
  // axis; one status word
  std::vector<int> radix[3], rev[3];
  size_t off = 0;
  size_t o_tw[3], o_tw64[3], o_rev[3], o_ipos[3], o_kk[3];
  auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~size_t(255); return o; };
  for (int d = 0; d < 3; d++) {
    radix[d] = factor_radices(n[d]);
    if ((int)radix[d].size() > kMaxStages) {
      delete p;
      return set_error(FF_ERR_UNSUPPORTED, "ff_plan_create: too many stages");
    }
    rev[d] = digit_reversal(n[d], radix[d]);
    o_tw[d] = take(n[d] * csz);
    o_tw64[d] = precision == FF_FP64 ? o_tw[d] : take(n[d] * sizeof(double2));
    o_rev[d] = take(n[d] * sizeof(int));
    o_ipos[d] = take(n[d] * sizeof(int));
    o_kk[d] = take((d == 2 ? p->nh : n[d]) * sizeof(double));
  }
  const size_t o_status = take(sizeof(int));
  for (int e = 0; e <= FF_NUM_PHASES; e++) {
    if (cudaEventCreate(&p->ev[e]) != cudaSuccess) {
      for (int q = 0; q < e; q++) cudaEventDestroy(p->ev[q]);
      delete p;
      return set_error(FF_ERR_CUDA, "ff_plan_create: cudaEventCreate failed");
    }
  }
  if (cudaMalloc(&p->dmem, off) != cudaSuccess) {
    cudaGetLastError();
    for (int e = 0; e <= FF_NUM_PHASES; e++) cudaEventDestroy(p->ev[e]);
    delete p;
    return set_error(FF_ERR_NOMEM, "ff_plan_create: cudaMalloc(%zu) for plan tables failed", off);
  }
  char *base = static_cast<char *>(p->dmem);
  p->status = reinterpret_cast<int *>(base + o_status);
  int rc = FF_OK;
  if (cudaMemset(p->status, 0, sizeof(int)) != cudaSuccess) rc = set_error(FF_ERR_CUDA, "ff_plan_create: memset");
  for (int d = 0; d < 3 && rc == FF_OK; d++) {
    std::vector<int> ipos(n[d]);
    for (int q = 0; q < n[d]; q++) ipos[rev[d][q]] = q;
    if (cudaMemcpy(base + o_rev[d], rev[d].data(), n[d] * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + o_ipos[d], ipos.data(), n[d] * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error(FF_ERR_CUDA, "ff_plan_create: table upload failed");
    const int blocks = std::min(1024, (n[d] + 255) / 256);
    k_twiddles<<<blocks, 256>>>(n[d], reinterpret_cast<double2 *>(base + o_tw64[d]));
    if (precision == FF_FP32) k_twiddles<<<blocks, 256>>>(n[d], reinterpret_cast<float2 *>(base + o_tw[d]));
    const int cnt = d == 2 ? p->nh : n[d];
    k_wavenumbers<<<std::min(1024, (cnt + 255) / 256), 256>>>(n[d], cnt, d != 2, p->dd[d],
                                                              reinterpret_cast<double *>(base + o_kk[d]));
    p->kk[d] = reinterpret_cast<double *>(base + o_kk[d]);
    AxisDev<double2> ad{};
    AxisDev<float2> af{};
    ad.n = af.n = n[d];
    ad.nstages = af.nstages = (int)radix[d].size();
    for (size_t s = 0; s < radix[d].size(); s++) ad.radix[s] = af.radix[s] = radix[d][s];
    ad.tw = reinterpret_cast<const double2 *>(base + o_tw[d]);
    af.tw = reinterpret_cast<const float2 *>(base + o_tw[d]);
    ad.tw64 = af.tw64 = reinterpret_cast<const double2 *>(base + o_tw64[d]);
    ad.rev = af.rev = reinterpret_cast<const int *>(base + o_rev[d]);
    ad.ipos = af.ipos = reinterpret_cast<const int *>(base + o_ipos[d]);
    p->axd[d] = ad;
    p->axf[d] = af;
  }
  if (rc == FF_OK && cudaGetLastError() != cudaSuccess) rc = set_error(FF_ERR_CUDA, "ff_plan_create: table kernels");
  if (rc == FF_OK && cudaDeviceSynchronize() != cudaSuccess)
    rc = set_error(FF_ERR_CUDA, "ff_plan_create: synchronize failed");
  if (rc == FF_OK) rc = precision == FF_FP64 ? configure<double>(p) : configure<float>(p);
  if (rc != FF_OK) {
    ff_plan_destroy(p);
    return rc;
  }
  *out = p;
  return FF_OK;
}

int ff_plan_bytes(const ff_plan *p, size_t *bytes) {
  if (!p || !bytes) return set_error(FF_ERR_INVALID, "ff_plan_bytes: null argument");
  *bytes = p->bytes;
  return FF_OK;
}

int ff_plan_info(const ff_plan *p, int n[3], int *precision) {
  if (!p) return set_error(FF_ERR_INVALID, "ff_plan_info: null plan");
  if (n)
    for (int d = 0; d < 3; d++) n[d] = p->n[d];
  if (precision) *precision = p->precision;
  return FF_OK;
}

int ff_solve(const ff_plan *p, size_t bytes, void *density, void *potential, void *stream, ff_phase_times *times) {
  if (!p || !density || !potential) return set_error(FF_ERR_INVALID, "ff_solve: null argument");
  if (bytes < p->bytes)   // the reference asserts this (ParisPencil.cpp:101)
    return set_error(FF_ERR_BYTES, "ff_solve: bytes %zu < required %zu", bytes, p->bytes);
  if (density == potential) return set_error(FF_ERR_INVALID, "ff_solve: density and potential must differ");
  if (((uintptr_t)density | (uintptr_t)potential) & 15)
    return set_error(FF_ERR_INVALID, "ff_solve: buffers must be 16-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool timed = times != nullptr;
  int rc = p->precision == FF_FP64 ? launch_solve<double>(p, density, potential, st, timed)
                                   : launch_solve<float>(p, density, potential, st, timed);
  if (rc != FF_OK) return rc;
  if (timed) {
    FF_CUDA(cudaEventSynchronize(p->ev[FF_NUM_PHASES]));
    for (int q = 0; q < FF_NUM_PHASES; q++) {
      float ms = 0;
      FF_CUDA(cudaEventElapsedTime(&ms, p->ev[q], p->ev[q + 1]));
      times->ms[q] = ms;
    }
    float tot = 0;
    FF_CUDA(cudaEventElapsedTime(&tot, p->ev[0], p->ev[FF_NUM_PHASES]));
    times->total_ms = tot;
    return take_device_status(p, st);
  }
  return FF_OK;
}

int ff_plan_check(const ff_plan *p, void *stream) {
  if (!p) return set_error(FF_ERR_INVALID, "ff_plan_check: null plan");
  return take_device_status(p, static_cast<cudaStream_t>(stream));
}

int ff_plan_destroy(ff_plan *p) {
  if (!p) return FF_OK;
  int rc = FF_OK;
  for (int e = 0; e <= FF_NUM_PHASES; e++)
    if (p->ev[e]) cudaEventDestroy(p->ev[e]);
  if (p->dmem && cudaFree(p->dmem) != cudaSuccess) rc = set_error(FF_ERR_CUDA, "ff_plan_destroy: cudaFree failed");
  delete p;
  return rc;
}

}  // extern "C"
