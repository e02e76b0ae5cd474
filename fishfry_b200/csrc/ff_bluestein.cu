// Bluestein passes of the single-grid solve for axes with a prime factor
// above 7 (the algorithm and its tables are described in ff_bluestein.hpp).
//
// One kernel per pass kind, runtime plans only (M varies with n):
//   z forward / inverse: W line pairs per block in a line-major swizzled tile
//     of pitch P >= M; the lines are read and written with plain loads and
//     stores (the convolution needs M > n rows per line, so the tile is not
//     the line block the bulk copies of the regular z passes move);
//   y forward / inverse, x: W spectrum columns x M rows per block in a
//     point-major tile (W = 8 FP64 / 16 FP32 when it fits, else a quarter of
//     that), rows read and written directly from HBM.
// The x kernel runs the forward transform, stores the filtered spectrum in
// place through its last stage, and runs the inverse on the same tile.

#include <cuda_runtime.h>

#include <algorithm>

#include "ff_bluestein.hpp"
#include "ff_status.hpp"

namespace ff {

namespace {

constexpr int kBsThreads = 256;
constexpr size_t kBsMaxSmem = 227 * 1024;   // per-block opt-in shared memory of sm_100

// The last DIF stage of the forward M-point transform, the product with ghat
// (its conjugate for the inverse direction) and the first DIT stage of the
// inverse M-point transform, on one register group (the span-R stages have
// no twiddles).
template <int R, bool INV, Map MAP, int W, typename C, typename TILE>
__device__ __forceinline__ void bs_mul_stage(int M, const C *__restrict__ ghat, TILE &tile, int ncols) {
  const int nb = M / R;
  for (int it = threadIdx.x; it < ncols * nb; it += kBsThreads) {
    int c, b;
    if (MAP == Map::ColFast) {
      c = it % W;
      b = it / W;
    } else {
      b = it % nb;
      c = it / nb;
    }
    const int base = b * R;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = tile(base + r, c);
    Dft<R, false, C>::run(v);
#pragma unroll
    for (int r = 0; r < R; r++) {
      const C g = __ldg(ghat + base + r);
      v[r] = INV ? cmulc(v[r], g) : cmul(v[r], g);
    }
    Dft<R, true, C>::run(v);
#pragma unroll
    for (int r = 0; r < R; r++) tile(base + r, c, v[r]);
  }
}

// The circular convolution of the tile's lines with the chirp kernel: stage 0
// reads ld0 (the premultiplied line, zero from n to M), the result conv[k]
// (natural order, k < M) leaves through stl(k, c, v) from the last stage.
// INV selects the conjugate kernel.  A block barrier follows.
template <bool INV, Map MAP, int W, bool TWREC0, typename C, typename LD0, typename TILE, typename STL>
__device__ __forceinline__ void bs_core(const BsAxis<C> &bs, LD0 &ld0, TILE &tile, STL &stl, int ncols) {
  constexpr bool TWALL = sizeof(C) == 16;   // FP64: recurrence twiddles in every stage
  const AxisDev<C> &ax = bs.m;
  const int S = ax.nstages;   // n >= 11, so M >= 21: at least two stages
  dif_rt<false, MAP, W, kBsThreads, TWREC0, TWALL>(ax, S - 1, ld0, tile, tile, ncols);
  with_radix(ax.radix[S - 1], [&](auto tag) {
    constexpr int R = decltype(tag)::value;
    bs_mul_stage<R, INV, MAP, W>(ax.n, bs.ghat, tile, ncols);
  });
  __syncthreads();
  dit_rt<true, MAP, W, kBsThreads, TWALL>(ax, S - 2, tile, stl, ncols);
}

// R2C along z (ParisPencil.cpp:152-165) for W line pairs per block.
template <typename T>
__global__ void __launch_bounds__(kBsThreads) k_bs_zfwd(const T *__restrict__ f, typename Cplx<T>::type *spec,
                                                        const PassArgs<T> a, const BsAxis<typename Cplx<T>::type> bs,
                                                        int W, int P) {
  using C = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  LineTile<C> t{reinterpret_cast<C *>(align128(smraw)), P};
  const int nk = a.nk;
  const long nlines = (long)a.ni * a.nj;
  const long line0 = (long)blockIdx.x * (2 * W);
  const C zero = mk((T)0, (T)0);
  // two real lines as one complex line, times the chirp; zero from nk on
  auto ld0 = [&](int pos, int c) -> C {
    if (pos >= nk) return zero;
    const long la = line0 + 2 * c;
    const T x = la < nlines ? f[la * nk + pos] : (T)0;
    const T y = la + 1 < nlines ? f[(la + 1) * nk + pos] : (T)0;
    return cmul(mk(x, y), __ldg(bs.chirp + pos));
  };
  bs_core<false, Map::PosFast, 1, true>(bs, ld0, t, t, W);
  // Z[k] = chirp[k] conv[k]; A[k] = (Z[k] + conj Z[n-k]) / 2,
  // B[k] = (Z[k] - conj Z[n-k]) / (2i)
  const T h = (T)0.5;
  for (int it = threadIdx.x; it < W * a.nh; it += kBsThreads) {
    const int k = it % a.nh;
    const int c = it / a.nh;
    const long la = line0 + 2 * c;
    if (la >= nlines) continue;
    const int kr = k == 0 ? 0 : nk - k;
    const C z = cmul(t(k, c), __ldg(bs.chirp + k));
    const C w = cmul(t(kr, c), __ldg(bs.chirp + kr));
    spec[la * a.nhp + k] = mk(h * (z.x + w.x), h * (z.y - w.y));
    if (la + 1 < nlines) spec[(la + 1) * a.nhp + k] = mk(h * (z.y + w.y), h * (w.x - z.x));
  }
}

// C2R along z (ParisPencil.cpp:368-380) for W line pairs per block.
template <typename T>
__global__ void __launch_bounds__(kBsThreads) k_bs_zinv(const typename Cplx<T>::type *spec, T *__restrict__ out,
                                                        const PassArgs<T> a, const BsAxis<typename Cplx<T>::type> bs,
                                                        int W, int P) {
  using C = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  LineTile<C> t{reinterpret_cast<C *>(align128(smraw)), P};
  const int nk = a.nk;
  const long nlines = (long)a.ni * a.nj;
  const long line0 = (long)blockIdx.x * (2 * W);
  const C zero = mk((T)0, (T)0);
  // Z[k] = A[k] + i B[k] over the Hermitian extension (conj A[n-k] + i conj
  // B[n-k] above n/2; the imaginary parts of the zero and Nyquist terms
  // dropped, as a C2R transform does), times conj chirp[k]
  auto ld0 = [&](int pos, int c) -> C {
    if (pos >= nk) return zero;
    const long la = line0 + 2 * c;
    const bool lo = 2 * pos <= nk;
    const int k = lo ? pos : nk - pos;
    const C sa = la < nlines ? __ldcg(spec + la * a.nhp + k) : zero;
    const C sb = la + 1 < nlines ? __ldcg(spec + (la + 1) * a.nhp + k) : zero;
    C z;
    if (k == 0 || 2 * k == nk) z = mk(sa.x, sb.x);
    else z = lo ? mk(sa.x - sb.y, sa.y + sb.x) : mk(sa.x + sb.y, sb.x - sa.y);
    return cmulc(z, __ldg(bs.chirp + pos));
  };
  bs_core<true, Map::PosFast, 1, true>(bs, ld0, t, t, W);
  for (int it = threadIdx.x; it < W * nk; it += kBsThreads) {
    const int k = it % nk;
    const int c = it / nk;
    const long la = line0 + 2 * c;
    if (la >= nlines) continue;
    const C v = cmulc(t(k, c), __ldg(bs.chirp + k));
    out[la * nk + k] = v.x;
    if (la + 1 < nlines) out[(la + 1) * nk + k] = v.y;
  }
}

// KIND 0: y forward, 1: y inverse (ParisPencil.cpp:173-212, :322-334);
// 2: x forward, filter, x inverse (:221-297, :406-421).  One tile of W
// spectrum columns per block: y tiles are plane i = o with rows j (row
// stride nhp), x tiles plane j = o with rows i (row stride nj*nhp).
template <typename T, int W, int KIND>
__global__ void __launch_bounds__(kBsThreads) k_bs_strided(const typename Cplx<T>::type *src,
                                                           typename Cplx<T>::type *dst, const PassArgs<T> a,
                                                           const BsAxis<typename Cplx<T>::type> bs) {
  using C = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  PointTile<W, C> tile{reinterpret_cast<C *>(align128(smraw))};
  const int n = bs.n;
  const int ktiles = (a.nh + W - 1) / W;
  const int o = blockIdx.x / ktiles;
  const int kt = blockIdx.x - o * ktiles;
  const int kh0 = kt * W;
  const int ncol = min(W, a.nh - kh0);
  const long base = KIND == 2 ? (long)o * a.nhp + kh0 : (long)o * a.nj * a.nhp + kh0;
  const long pitch = KIND == 2 ? (long)a.nj * a.nhp : (long)a.nhp;
  const C zero = mk((T)0, (T)0);
  auto ld0 = [&](int pos, int c) -> C {
    if (pos >= n || c >= ncol) return zero;
    const C v = __ldcg(src + base + pos * pitch + c);
    const C w = __ldg(bs.chirp + pos);
    return KIND == 1 ? cmulc(v, w) : cmul(v, w);
  };
  if constexpr (KIND != 2) {
    auto st = [&](int k, int c, C v) {
      if (k < n && c < ncol) {
        const C w = __ldg(bs.chirp + k);
        dst[base + k * pitch + c] = KIND == 1 ? cmulc(v, w) : cmul(v, w);
      }
    };
    bs_core<KIND == 1, Map::ColFast, W, false>(bs, ld0, tile, st, W);
  } else {
    // d = -1/((i2 + j2) + k2) * 1/N with i2 = (min(i, ni-i)*ddi)^2 etc., as
    // ParisPencil.cpp:276-279 forms it; zero for the zero mode
    const int ni = a.ni;
    const double jd = double(min(o, a.nj - o)) * a.dd[1];
    const double j2 = jd * jd;
    const double ddi = a.dd[0], ddk = a.dd[2];
    const double minvN = -a.invN;
    // The last forward stage leaves X[k] = chirp[k] conv[k]; the inverse
    // transform's input is X[k] d(k) conj chirp[k] = conv[k] d(k), as
    // |chirp| = 1, so that is what it stores (zero from n on).
    auto stf = [&](int k, int c, C v) {
      C r = zero;
      const int kh = kh0 + c;
      if (k < n && (k | o | kh) != 0) {
        const double id = double(min(k, ni - k)) * ddi;
        const double kd = double(kh) * ddk;
        const double d = recip_pos((id * id + j2) + kd * kd) * minvN;
        r = cscale(v, (T)d);
      }
      tile(k, c, r);
    };
    bs_core<false, Map::ColFast, W, false>(bs, ld0, tile, stf, W);
    auto st = [&](int j, int c, C v) {
      if (j < n && c < ncol) dst[base + j * pitch + c] = cmulc(v, __ldg(bs.chirp + j));
    };
    bs_core<true, Map::ColFast, W, false>(bs, tile, tile, st, W);
  }
}

// chirp[j] = exp(-i*pi*j^2/n): the exponent reduced exactly (j^2 mod 2n)
// before FP64 sincospi.
template <typename C> __global__ void k_bs_chirp(int n, C *chirp) {
  using R = typename Real<C>::type;
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const long long q = (long long)j * j % (2LL * n);
    double s, c;
    sincospi((double)q / (double)n, &s, &c);
    chirp[j] = mk((R)c, (R)(-s));
  }
}

// ghat[pos] = G[rev[pos]] / M, G[k] = sum_m g[m] exp(-2*pi*i*m*k/M) over the
// wrapped kernel g[m] = g[M-m] = exp(+i*pi*m^2/n) (m < n):
//   G[k] = 1 + 2 sum_{m=1}^{n-1} exp(i*pi*m^2/n) cos(2*pi*m*k/M),
// a direct FP64 sum (exponents reduced exactly), in blocks of 32 terms.
template <typename C> __global__ void k_bs_ghat(int n, int M, const int *rev, C *ghat) {
  using R = typename Real<C>::type;
  for (int pos = blockIdx.x * blockDim.x + threadIdx.x; pos < M; pos += gridDim.x * blockDim.x) {
    const int k = rev[pos];
    double gx = 1.0, gy = 0.0;
    for (int m0 = 1; m0 < n; m0 += 32) {
      double px = 0.0, py = 0.0;
      for (int m = m0; m < min(n, m0 + 32); m++) {
        const long long q = (long long)m * m % (2LL * n);
        const long long r = (long long)m * k % M;
        double s, c;
        sincospi((double)q / (double)n, &s, &c);
        const double cs = cospi(2.0 * (double)r / (double)M);
        px += c * cs;
        py += s * cs;
      }
      gx += 2.0 * px;
      gy += 2.0 * py;
    }
    ghat[pos] = mk((R)(gx / M), (R)(gy / M));
  }
}

template <typename T, int W> using StridedFn = void (*)(const typename Cplx<T>::type *, typename Cplx<T>::type *,
                                                        const PassArgs<T>, const BsAxis<typename Cplx<T>::type>);

template <typename T, int W> StridedFn<T, W> strided_fn(int kind) {
  return kind == 1 ? k_bs_strided<T, W, 0> : kind == 2 ? k_bs_strided<T, W, 2> : k_bs_strided<T, W, 1>;
}

// Checks that a tile of `need` bytes fits and lets fn use all the dynamic
// shared memory there is: the limit is a property of the kernel, shared by
// every plan, so it is never lowered to one plan's need (a later plan with a
// smaller tile would otherwise break an earlier plan's launches).
template <typename F> int raise_smem(F fn, size_t need) {
  cudaFuncAttributes fa;
  FF_CUDA(cudaFuncGetAttributes(&fa, fn));
  if (need + fa.sharedSizeBytes > kBsMaxSmem)
    return set_error(FF_ERR_UNSUPPORTED, "Bluestein tile of %zu bytes does not fit in shared memory", need);
  FF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(kBsMaxSmem - fa.sharedSizeBytes)));
  return FF_OK;
}

}  // namespace

int bs_padded_length(int n) {
  for (int m = std::max(1, 2 * n - 1);; m++)
    if (smooth2357(m)) return m;
}

template <typename T> int bs_configure(int kind, int ni, int nj, int nh, int M, BsCfg *cfg) {
  using C = typename Cplx<T>::type;
  constexpr int csz = (int)sizeof(C);
  constexpr int WB = 128 / csz, WS = 32 / csz;   // 128- or 32-byte tile rows
  if (kind == 0 || kind == 4) {
    // line pairs of pitch P, about 96 KB per block (at least one pair)
    const int align = csz == 16 ? 8 : 16;
    cfg->P = (M + align - 1) / align * align;
    cfg->W = std::max(1, std::min(8, (96 * 1024) / (cfg->P * csz)));
    cfg->smem = (size_t)cfg->W * cfg->P * csz + 128;
    const long npairs = ((long)ni * nj + 1) / 2;
    cfg->grid = (npairs + cfg->W - 1) / cfg->W;
    return kind == 0 ? raise_smem(k_bs_zfwd<T>, cfg->smem) : raise_smem(k_bs_zinv<T>, cfg->smem);
  }
  if (kind < 1 || kind > 3) return set_error(FF_ERR_INVALID, "bs_configure: pass kind %d", kind);
  cfg->P = 0;
  cfg->W = (size_t)M * WB * csz + 128 <= 200 * 1024 ? WB : WS;
  cfg->smem = (size_t)M * cfg->W * csz + 128;
  const int ktiles = (nh + cfg->W - 1) / cfg->W;
  cfg->grid = (long)(kind == 2 ? nj : ni) * ktiles;
  return cfg->W == WB ? raise_smem(strided_fn<T, WB>(kind), cfg->smem)
                      : raise_smem(strided_fn<T, WS>(kind), cfg->smem);
}

template <typename C> int bs_tables(int n, int M, const int *rev, C *chirp, C *ghat) {
  k_bs_chirp<<<std::min(1024, (n + 255) / 256), 256>>>(n, chirp);
  k_bs_ghat<<<std::min(1024, (M + 127) / 128), 128>>>(n, M, rev, ghat);
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

template <typename T> int bs_launch(int kind, const void *src, void *dst, const PassArgs<T> &a,
                                    const BsAxis<typename Cplx<T>::type> &bs, const BsCfg &cfg, cudaStream_t st) {
  using C = typename Cplx<T>::type;
  constexpr int WB = 128 / (int)sizeof(C), WS = 32 / (int)sizeof(C);
  const unsigned grid = (unsigned)cfg.grid;
  if (kind == 0) {
    k_bs_zfwd<T><<<grid, kBsThreads, cfg.smem, st>>>(static_cast<const T *>(src), static_cast<C *>(dst), a, bs,
                                                     cfg.W, cfg.P);
  } else if (kind == 4) {
    k_bs_zinv<T><<<grid, kBsThreads, cfg.smem, st>>>(static_cast<const C *>(src), static_cast<T *>(dst), a, bs,
                                                     cfg.W, cfg.P);
  } else if (kind >= 1 && kind <= 3) {
    const C *s = static_cast<const C *>(src);
    C *d = static_cast<C *>(dst);
    if (cfg.W == WB) strided_fn<T, WB>(kind)<<<grid, kBsThreads, cfg.smem, st>>>(s, d, a, bs);
    else strided_fn<T, WS>(kind)<<<grid, kBsThreads, cfg.smem, st>>>(s, d, a, bs);
  } else {
    return set_error(FF_ERR_INVALID, "bs_launch: pass kind %d", kind);
  }
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

template int bs_configure<double>(int, int, int, int, int, BsCfg *);
template int bs_configure<float>(int, int, int, int, int, BsCfg *);
template int bs_tables<double2>(int, int, const int *, double2 *, double2 *);
template int bs_tables<float2>(int, int, const int *, float2 *, float2 *);
template int bs_launch<double>(int, const void *, void *, const PassArgs<double> &, const BsAxis<double2> &,
                               const BsCfg &, cudaStream_t);
template int bs_launch<float>(int, const void *, void *, const PassArgs<float> &, const BsAxis<float2> &,
                              const BsCfg &, cudaStream_t);

}  // namespace ff
