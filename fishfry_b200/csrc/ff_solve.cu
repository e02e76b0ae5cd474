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
};

// ------------------------------------------------------------------ pass 1
template <typename T>
__global__ void __launch_bounds__(kThreads) k_zfwd(const T *__restrict__ f, typename Cplx<T>::type *__restrict__ spec,
                                                   const PassArgs<T> a) {
  using C = typename Cplx<T>::type;
  constexpr int W = TileW<T>::value;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *sm = reinterpret_cast<C *>(smraw);
  const long nlines = (long)a.ni * a.nj;
  const long line0 = (long)blockIdx.x * (2 * W);
  const int nk = a.nk;

  // element pos of pair c: z = f[line a] + i f[line b]
  auto ldg = [&](int pos, int c) -> C {
    const long la = line0 + 2 * c;
    T x = 0, y = 0;
    if (la < nlines) x = f[la * nk + pos];
    if (la + 1 < nlines) y = f[(la + 1) * nk + pos];
    return mk(x, y);
  };
  SmemSt<W, C> sst{sm};
  dif_transform<false, W>(a.ax[2], sm, ldg, sst);

  // split: A[k] = (Z[k] + conj Z[n-k]) / 2,  B[k] = (Z[k] - conj Z[n-k]) / (2i)
  const int *ipos = a.ax[2].ipos;
  const T h = (T)0.5;
  for (int it = threadIdx.x; it < W * a.nh; it += blockDim.x) {
    const int c = it % W;
    const int k = it / W;
    const long la = line0 + 2 * c;
    if (la >= nlines) continue;
    const C z = sm[__ldg(ipos + k) * W + c];
    const C w = sm[__ldg(ipos + (k == 0 ? 0 : nk - k)) * W + c];
    spec[la * a.nhp + k] = mk(h * (z.x + w.x), h * (z.y - w.y));
    if (la + 1 < nlines) spec[(la + 1) * a.nhp + k] = mk(h * (z.y + w.y), h * (w.x - z.x));
  }
}

// ------------------------------------------------------------- passes 2, 4
// Complex transform along y of tile (i = blockIdx.y, kh0 = blockIdx.x*W).
template <typename T, bool INV>
__global__ void __launch_bounds__(kThreads) k_ypass(const typename Cplx<T>::type *src, typename Cplx<T>::type *dst,
                                                    const PassArgs<T> a) {
  using C = typename Cplx<T>::type;
  constexpr int W = TileW<T>::value;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *sm = reinterpret_cast<C *>(smraw);
  const int kh0 = blockIdx.x * W;
  const int ncol = min(W, a.nh - kh0);
  const long base = (long)blockIdx.y * a.nj * a.nhp + kh0;
  const int pitch = a.nhp;
  const int *rev = a.ax[1].rev;
  auto ldg = [&](int pos, int c) -> C { return c < ncol ? src[base + (long)pos * pitch + c] : mk((T)0, (T)0); };
  auto stg = [&](int pos, int c, C v) {
    if (c < ncol) dst[base + (long)__ldg(rev + pos) * pitch + c] = v;
  };
  dif_transform<INV, W>(a.ax[1], sm, ldg, stg);
}

// ------------------------------------------------------------------ pass 3
// Forward transform along x, filter, inverse transform along x, for tile
// (j = blockIdx.y, kh0 = blockIdx.x*W).  DIF forward leaves the spectrum
// digit-reversed in shared memory; the last DIF stage, the filter and the first
// DIT stage of the inverse act on the same register group.
template <int R, int W, typename C, typename LD, typename ST, typename FL>
__device__ __forceinline__ void fused_filter_stage(int n, LD &ld, ST &st, FL &filt) {
  const int items = W * (n / R);
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
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
  }
}

template <typename T>
__global__ void __launch_bounds__(kThreads) k_xpass(typename Cplx<T>::type *data, const PassArgs<T> a) {
  using C = typename Cplx<T>::type;
  constexpr int W = TileW<T>::value;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *sm = reinterpret_cast<C *>(smraw);
  const int j = blockIdx.y;
  const int kh0 = blockIdx.x * W;
  const int ncol = min(W, a.nh - kh0);
  const long base = (long)j * a.nhp + kh0;
  const long pitch = (long)a.nj * a.nhp;
  const AxisDev<C> &ax = a.ax[0];
  const int n = ax.n;
  const int S = ax.nstages;

  auto ldg = [&](int pos, int c) -> C { return c < ncol ? data[base + pos * pitch + c] : mk((T)0, (T)0); };
  auto stg = [&](int pos, int c, C v) {
    if (c < ncol) data[base + pos * pitch + c] = v;
  };
  const double j2 = __ldg(a.kk[1] + j);
  const double *kkx = a.kk[0];
  const double *kkz = a.kk[2];
  const int *rev = ax.rev;
  const double invN = a.invN;
  // d = -1/((i2 + j2) + k2) as ParisPencil.cpp:276-279 forms it, times 1/N
  auto filt = [&](int pos, int c, C v) -> C {
    const int kx = __ldg(rev + pos);
    const int kh = kh0 + c;
    if (c >= ncol) return v;
    if ((kx | j | kh) == 0) return mk((T)0, (T)0);
    const double d = -1.0 / ((__ldg(kkx + kx) + j2) + __ldg(kkz + kh)) * invN;
    return cscale(v, (T)d);
  };

  SmemLd<W, C> sld{sm};
  SmemSt<W, C> sst{sm};
  int L = n;
  for (int s = 0; s < S - 1; s++) {
    with_radix(ax.radix[s], [&](auto tag) {
      constexpr int R = decltype(tag)::value;
      if (s == 0) run_stage<R, false, false, W>(n, L, ax.tw, ldg, sst);
      else run_stage<R, false, false, W>(n, L, ax.tw, sld, sst);
    });
    L /= ax.radix[s];
    __syncthreads();
  }
  with_radix(ax.radix[S - 1], [&](auto tag) {
    constexpr int R = decltype(tag)::value;
    if (S == 1) fused_filter_stage<R, W, C>(n, ldg, stg, filt);
    else fused_filter_stage<R, W, C>(n, sld, sst, filt);
  });
  __syncthreads();
  if (S > 1) dit_stages<true, W>(ax, sm, S - 2, stg);
}

// ------------------------------------------------------------------ pass 5
template <typename T>
__global__ void __launch_bounds__(kThreads) k_zinv(const typename Cplx<T>::type *__restrict__ spec, T *__restrict__ out,
                                                   const PassArgs<T> a) {
  using C = typename Cplx<T>::type;
  constexpr int W = TileW<T>::value;
  extern __shared__ __align__(16) unsigned char smraw[];
  C *sm = reinterpret_cast<C *>(smraw);
  const long nlines = (long)a.ni * a.nj;
  const long line0 = (long)blockIdx.x * (2 * W);
  const int nk = a.nk;
  const int *ipos = a.ax[2].ipos;

  // Z[k] = A[k] + i B[k] over the Hermitian extension; the imaginary parts of
  // the zero and Nyquist terms are dropped, as a C2R transform does.
  for (int it = threadIdx.x; it < W * a.nh; it += blockDim.x) {
    const int c = it % W;
    const int k = it / W;
    const long la = line0 + 2 * c;
    C A = mk((T)0, (T)0), B = mk((T)0, (T)0);
    if (la < nlines) A = spec[la * a.nhp + k];
    if (la + 1 < nlines) B = spec[(la + 1) * a.nhp + k];
    if (k == 0 || 2 * k == nk) {
      sm[__ldg(ipos + k) * W + c] = mk(A.x, B.x);
    } else {
      sm[__ldg(ipos + k) * W + c] = mk(A.x - B.y, A.y + B.x);
      sm[__ldg(ipos + nk - k) * W + c] = mk(A.x + B.y, B.x - A.y);
    }
  }
  __syncthreads();
  auto stg = [&](int pos, int c, C v) {
    const long la = line0 + 2 * c;
    if (la < nlines) out[la * nk + pos] = v.x;
    if (la + 1 < nlines) out[(la + 1) * nk + pos] = v.y;
  };
  dit_stages<true, W>(a.ax[2], sm, a.ax[2].nstages - 1, stg);
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

struct ff_plan {
  int n[3];
  int precision;
  int nh, nhp;
  double dd[3];
  size_t bytes;
  int device;
  void *dmem;
  AxisDev<double2> axd[3];
  AxisDev<float2> axf[3];
  double *kk[3];
  cudaEvent_t ev[FF_NUM_PHASES + 1];
};

namespace ff {

bool smooth235(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

// DIF radix order: 8s first, then a 4 or a 2, then 5s and 3s.
static std::vector<int> factor_radices(int n) {
  std::vector<int> r;
  int twos = 0;
  while (n % 2 == 0) { n /= 2; twos++; }
  while (twos >= 3) { r.push_back(8); twos -= 3; }
  if (twos == 2) r.push_back(4);
  if (twos == 1) r.push_back(2);
  while (n % 5 == 0) { r.push_back(5); n /= 5; }
  while (n % 3 == 0) { r.push_back(3); n /= 3; }
  if (r.empty()) r.push_back(1);
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

template <typename T> static int set_smem_limits() {
  const int lim = 227 * 1024;
  FF_CUDA(cudaFuncSetAttribute(k_zfwd<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  FF_CUDA(cudaFuncSetAttribute(k_ypass<T, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  FF_CUDA(cudaFuncSetAttribute(k_ypass<T, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  FF_CUDA(cudaFuncSetAttribute(k_xpass<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  FF_CUDA(cudaFuncSetAttribute(k_zinv<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
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
  return a;
}

template <typename T>
static int launch_solve(const ff_plan *p, void *density, void *potential, cudaStream_t st, bool timed) {
  using C = typename Cplx<T>::type;
  constexpr int W = TileW<T>::value;
  const PassArgs<T> a = pass_args<T>(p);
  const int ni = p->n[0], nj = p->n[1], nk = p->n[2];
  const long npairs = ((long)ni * nj + 1) / 2;
  const unsigned ztiles = (unsigned)((npairs + W - 1) / W);
  const unsigned ktiles = (unsigned)((p->nh + W - 1) / W);
  T *D = static_cast<T *>(density);
  T *P = static_cast<T *>(potential);
  C *Ds = reinterpret_cast<C *>(density);
  C *Ps = reinterpret_cast<C *>(potential);
  const size_t smz = (size_t)nk * W * sizeof(C);
  const size_t smy = (size_t)nj * W * sizeof(C);
  const size_t smx = (size_t)ni * W * sizeof(C);
  if (timed) FF_CUDA(cudaEventRecord(p->ev[0], st));
  k_zfwd<T><<<ztiles, kThreads, smz, st>>>(D, Ps, a);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[1], st));
  k_ypass<T, false><<<dim3(ktiles, ni), kThreads, smy, st>>>(Ps, Ps, a);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[2], st));
  k_xpass<T><<<dim3(ktiles, nj), kThreads, smx, st>>>(Ps, a);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[3], st));
  k_ypass<T, true><<<dim3(ktiles, ni), kThreads, smy, st>>>(Ps, Ds, a);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[4], st));
  k_zinv<T><<<ztiles, kThreads, smz, st>>>(Ds, P, a);
  FF_CUDA(cudaGetLastError());
  if (timed) FF_CUDA(cudaEventRecord(p->ev[5], st));
  return FF_OK;
}

}  // namespace ff

extern "C" {

const char *ff_version(void) { return "fishfry_b200 0.1 (sm_100a)"; }

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
    // ParisPencil.cpp:9-11
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
  cudaGetDevice(&p->device);

  // device tables: per axis tw (n complex), rev and ipos (n ints); kk per axis
  std::vector<int> radix[3], rev[3];
  size_t off = 0;
  size_t o_tw[3], o_rev[3], o_ipos[3], o_kk[3];
  auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~size_t(255); return o; };
  for (int d = 0; d < 3; d++) {
    radix[d] = factor_radices(n[d]);
    if ((int)radix[d].size() > kMaxStages) {
      delete p;
      return set_error(FF_ERR_UNSUPPORTED, "ff_plan_create: too many stages");
    }
    rev[d] = digit_reversal(n[d], radix[d]);
    o_tw[d] = take(n[d] * csz);
    o_rev[d] = take(n[d] * sizeof(int));
    o_ipos[d] = take(n[d] * sizeof(int));
    o_kk[d] = take((d == 2 ? p->nh : n[d]) * sizeof(double));
  }
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
  int rc = FF_OK;
  for (int d = 0; d < 3 && rc == FF_OK; d++) {
    std::vector<int> ipos(n[d]);
    for (int q = 0; q < n[d]; q++) ipos[rev[d][q]] = q;
    if (cudaMemcpy(base + o_rev[d], rev[d].data(), n[d] * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + o_ipos[d], ipos.data(), n[d] * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error(FF_ERR_CUDA, "ff_plan_create: table upload failed");
    const int blocks = std::min(1024, (n[d] + 255) / 256);
    if (precision == FF_FP64) k_twiddles<<<blocks, 256>>>(n[d], reinterpret_cast<double2 *>(base + o_tw[d]));
    else k_twiddles<<<blocks, 256>>>(n[d], reinterpret_cast<float2 *>(base + o_tw[d]));
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
    ad.rev = af.rev = reinterpret_cast<const int *>(base + o_rev[d]);
    ad.ipos = af.ipos = reinterpret_cast<const int *>(base + o_ipos[d]);
    p->axd[d] = ad;
    p->axf[d] = af;
  }
  if (rc == FF_OK && cudaGetLastError() != cudaSuccess) rc = set_error(FF_ERR_CUDA, "ff_plan_create: table kernels");
  if (rc == FF_OK && cudaDeviceSynchronize() != cudaSuccess)
    rc = set_error(FF_ERR_CUDA, "ff_plan_create: synchronize failed");
  if (rc == FF_OK) rc = precision == FF_FP64 ? set_smem_limits<double>() : set_smem_limits<float>();
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
  }
  return FF_OK;
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
