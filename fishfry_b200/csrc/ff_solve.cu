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

#include "ff_bluestein.hpp"
#include "ff_fft.cuh"
#include "ff_plan.hpp"
#include "ff_status.hpp"
#include "ff_tiles.cuh"

namespace ff {

// Lengths with compile-time specialised kernels (fully unrolled stages);
// every other length runs the same kernels with the plan read at run time.
#define FF_FOR_EACH_SPECIAL_N(X) X(64) X(128) X(256) X(512) X(1024)

// ------------------------------------------------- unfused pass kernels
// (one launch per pass; used when the fused passes are switched off)
// With BULK (every specialised length, and runtime lengths whose lines are
// whole 16-byte multiples and whose plan has at least two stages) both z
// passes move their line blocks both ways with bulk copies; otherwise the
// threads load the lines, and the inverse stores them.  The spectrum rows
// always leave (forward) and enter (inverse) as 16-byte multiples.
//
// The z passes run blocks of kZPassThreads = 128 threads on tiles of about
// 32 KB, six per SM: more, smaller tiles in flight hide each block's inbound
// copy better than three 64 KB tiles of 256 threads (512^3 FP64 z passes 0.379
// / 0.385 -> 0.337 / 0.321 ms; FP32 0.223 / 0.223 -> 0.204 / 0.201 ms).
constexpr int kZPassThreads = 128;

template <typename T, int N, bool BULK>
__global__ void __launch_bounds__(kZPassThreads, 6) k_zfwd(const T *__restrict__ f, typename Cplx<T>::type *spec,
                                                       const PassArgs<T> a, int W, int P) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  const long nlines = (long)a.ni * a.nj;
  if (BULK && threadIdx.x == 0) {
    // whole lines are 16-byte multiples here
    const long fl = ((long)blockIdx.x + a.l2_ahead) * (2 * W);
    if (a.l2_ahead > 0 && fl < nlines)
      l2_prefetch(f + fl * a.nk, (uint32_t)(min((long)(2 * W), nlines - fl) * a.nk * sizeof(T)));
  }
  const ZTileIO io{&mbar, 0, a.status, a.wait_iters};
  z_fwd_tile<T, N, BULK, true, true, kZPassThreads>(f, spec, a, W, P, (long)blockIdx.x * (2 * W), nlines,
                               reinterpret_cast<typename Cplx<T>::type *>(align128(smraw)), io);
}

template <typename T, int N, bool BULK>
__global__ void __launch_bounds__(kZPassThreads, 6) k_zinv(const typename Cplx<T>::type *spec, T *__restrict__ out,
                                                       const PassArgs<T> a, int W, int P) {
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  const long nlines = (long)a.ni * a.nj;
  // the same L2 hint as the forward pass, on the spectrum rows (contiguous
  // for a block's line pairs)
  if (BULK && threadIdx.x == 32) {
    const long fl = ((long)blockIdx.x + a.l2_ahead) * (2 * W);
    if (a.l2_ahead > 0 && fl < nlines)
      l2_prefetch(spec + fl * a.nhp,
                  (uint32_t)(min((long)(2 * W), nlines - fl) * a.nhp * sizeof(typename Cplx<T>::type)));
  }
  const ZTileIO io{&mbar, 0, a.status, a.wait_iters};
  z_inv_tile<T, N, BULK, true, kZPassThreads>(spec, out, a, W, P, (long)blockIdx.x * (2 * W), nlines,
                         reinterpret_cast<typename Cplx<T>::type *>(align128(smraw)), io);
}

// One TMA-loaded strided tile per block (y forward / inverse or x).  Blocks
// are dispatched in tile order, so the kh tiles of one plane row, which share
// DRAM rows, are fetched together.
template <typename T, int W, bool XPASS, bool INV, int N>
__global__ void __launch_bounds__(kZThreads, 3)
    k_strided(const __grid_constant__ CUtensorMap tmap, typename Cplx<T>::type *dst, const PassArgs<T> a,
              int box_rows) {
  using C = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  C *sm = reinterpret_cast<C *>(align128(smraw));
  const int n = N > 0 ? N : (XPASS ? a.ax[0].n : a.ax[1].n);
  const int ktiles = (a.nh + W - 1) / W;
  const int o = blockIdx.x / ktiles, kt = blockIdx.x - o * ktiles;
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  __syncthreads();
  if (!tma_tile<C, W, XPASS>(&tmap, sm, &mbar, 0, n, box_rows, o, kt, a.status, a.wait_iters)) return;
  if (XPASS) {
    x_tile<T, W, N>(&tmap, a, o, kt, box_rows, sm);
  } else {
    PointTile<W, C> tile{sm};
    y_tile<T, W, INV, N>(tile, dst, a, o, kt, sm);
  }
}

// ---------------------------------------------------------- fused passes
// z forward + y forward (and y inverse + z inverse) in one persistent launch.
// Blocks take tiles from an in-order work queue: the producer tiles of plane
// i (z forward / y inverse) come `lag` planes ahead of its consumer tiles
// (y forward / z inverse), and a consumer tile waits, with an iteration
// limit, until the plane's producer count is complete.  The plane's
// intermediate spectrum is therefore written and read back while it is still
// in L2, and HBM sees the real field once and the spectrum once per
// direction.  Every consumer waits only on tiles handed out before it, so the
// queue cannot deadlock.
struct FuseArgs {
  int *ticket;     // work counter (zeroed before the launch)
  int *done;       // per-plane producer counts (zeroed before the launch)
  int planes;      // ni
  int prod_pp;     // producer tiles per plane
  int cons_pp;     // consumer tiles per plane
  int lag;         // planes between a producer tile and its plane's consumers (<= planes)
  int zW, zP;      // z tile shape
  int box_rows;    // TMA box rows of y tiles
  int wait_iters;  // iteration limit of a dependency wait (0: built-in)
  int target_extra;  // added to every dependency wait's target (0; a test sets 1 to make the waits run out)
};

__device__ __forceinline__ void fuse_decode(const FuseArgs &f, int t, bool &cons, int &plane, int &tile) {
  const int A = f.prod_pp, B = f.cons_pp, L = f.lag;
  const int head = L * A;
  if (t < head) {
    cons = false;
    plane = t / A;
    tile = t - plane * A;
    return;
  }
  t -= head;
  const int mid = (f.planes - L) * (A + B);
  if (t < mid) {
    const int s = t / (A + B), q = t - s * (A + B);
    cons = q >= A;
    plane = cons ? s : L + s;
    tile = cons ? q - A : q;
    return;
  }
  t -= mid;
  cons = true;
  plane = (f.planes - L) + t / B;
  tile = t - (t / B) * B;
}

// Built-in iteration limit of a dependency wait (about a second).
constexpr int kDepWaitIters = 1 << 22;

// Bounded wait for *p >= target (acquire at GPU scope); limit <= 0: the
// built-in kDepWaitIters.
__device__ __forceinline__ bool wait_count(const int *p, int target, int limit) {
  if (limit <= 0) limit = kDepWaitIters;
  for (int i = 0; i < limit; i++) {
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    if (v >= target) return true;
    __nanosleep(128);
  }
  return false;
}

// Publishes this block's finished producer tile of `plane`.
__device__ __forceinline__ void publish(int *done, int plane) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(done + plane, 1);
}

// Waits for all producer tiles of `plane`; false on every thread on timeout,
// and the caller then leaves without touching the plane.
__device__ __forceinline__ bool await_plane(const FuseArgs &fa, int plane, int *status) {
  bool ok = true;
  if (threadIdx.x == 0) {
    ok = wait_count(fa.done + plane, fa.prod_pp + fa.target_extra, fa.wait_iters);
    if (!ok) atomicExch(status, kDevDepTimeout);
  }
  return !__syncthreads_or(!ok);
}

__device__ __forceinline__ int next_ticket(int *ticket, int *s_ticket) {
  __syncthreads();   // the previous tile's shared-memory use is over
  if (threadIdx.x == 0) *s_ticket = atomicAdd(ticket, 1);
  __syncthreads();
  return *s_ticket;
}

template <typename T, int NZ, int NY>
__global__ void __launch_bounds__(kZThreads, 3)
    k_zy_fwd(const T *__restrict__ f, typename Cplx<T>::type *spec, const PassArgs<T> a, const FuseArgs fa) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  extern __shared__ unsigned char smraw[];
  __shared__ int s_ticket;
  C *sm = reinterpret_cast<C *>(align128(smraw));
  const int total = fa.planes * (fa.prod_pp + fa.cons_pp);
  for (;;) {
    const int t = next_ticket(fa.ticket, &s_ticket);
    if (t >= total) break;
    bool cons;
    int plane, tile;
    fuse_decode(fa, t, cons, plane, tile);
    if (!cons) {
      const long first = (long)plane * a.nj;
      z_fwd_tile<T, NZ, false>(f, spec, a, fa.zW, fa.zP, first + (long)tile * 2 * fa.zW, first + a.nj, sm,
                               ZTileIO{nullptr, 0, a.status, 0});
      publish(fa.done, plane);
    } else {
      if (!await_plane(fa, plane, a.status)) break;
      // the plane was written by other blocks moments ago: read it through L2
      const int kh0 = tile * W;
      const int ncol = min(W, a.nh - kh0);
      const long base = (long)plane * a.nj * a.nhp + kh0;
      const int pitch = a.nhp;
      auto ldg = [&](int pos, int c) -> C {
        return c < ncol ? __ldcg(spec + base + (long)pos * pitch + c) : mk((T)0, (T)0);
      };
      y_tile<T, W, false, NY>(ldg, spec, a, plane, tile, sm);
    }
  }
}

template <typename T, int NZ, int NY>
__global__ void __launch_bounds__(kZThreads, 3)
    k_yz_inv(const __grid_constant__ CUtensorMap tmap, typename Cplx<T>::type *specD, T *__restrict__ out,
             const PassArgs<T> a, const FuseArgs fa) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / sizeof(C);
  extern __shared__ unsigned char smraw[];
  __shared__ int s_ticket;
  __shared__ __align__(8) uint64_t mbar;
  C *sm = reinterpret_cast<C *>(align128(smraw));
  const int ny = NY > 0 ? NY : a.nj;
  const int total = fa.planes * (fa.prod_pp + fa.cons_pp);
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  uint32_t loads = 0;   // completed phases of mbar
  for (;;) {
    const int t = next_ticket(fa.ticket, &s_ticket);
    if (t >= total) break;
    bool cons;
    int plane, tile;
    fuse_decode(fa, t, cons, plane, tile);
    if (!cons) {
      // y inverse of a tile of the x pass's output (written by an earlier
      // launch, so TMA may read it)
      fence_proxy_async_smem();
      __syncthreads();
      if (!tma_tile<C, W, false>(&tmap, sm, &mbar, loads & 1, ny, fa.box_rows, plane, tile, a.status,
                                 a.wait_iters))
        break;
      loads++;
      PointTile<W, C> tl{sm};
      y_tile<T, W, true, NY>(tl, specD, a, plane, tile, sm);
      publish(fa.done, plane);
    } else {
      if (!await_plane(fa, plane, a.status)) break;
      const long first = (long)plane * a.nj;
      z_inv_tile<T, NZ, false>(specD, out, a, fa.zW, fa.zP, first + (long)tile * 2 * fa.zW, first + a.nj, sm,
                               ZTileIO{nullptr, 0, a.status, 0});
    }
  }
}

// x pass: forward, filter, inverse; one TMA-loaded tile per block.
template <typename T, int N>
static void launch_x(const CUtensorMap &map, typename Cplx<T>::type *dst, const PassArgs<T> &a, int box_rows,
                     int grid, size_t smem, cudaStream_t st) {
  constexpr int W = 128 / (2 * (int)sizeof(T));
  k_strided<T, W, true, false, N><<<grid, kZThreads, smem, st>>>(map, dst, a, box_rows);
}

// ------------------------------------------------------------- plan tables
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

bool smooth235(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5})
    while (n % p == 0) n /= p;
  return n == 1;
}

bool smooth2357(int n) {
  if (n < 1) return false;
  for (int p : {2, 3, 5, 7})
    while (n % p == 0) n /= p;
  return n == 1;
}

// DIF radix order of the device plan (plan_radix in ff_fft.cuh).
std::vector<int> plan_factor_radices(int n) {
  std::vector<int> r;
  for (int s = 0; s < plan_stages(n); s++) r.push_back(plan_radix(n, s));
  return r;
}

// rev[pos]: frequency held at DIF output position pos.
std::vector<int> plan_digit_reversal(int n, const std::vector<int> &radix) {
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

template <typename T> using ZFwdKernel = void (*)(const T *, typename Cplx<T>::type *, const PassArgs<T>, int, int);
template <typename T>
using ZInvKernel = void (*)(const typename Cplx<T>::type *, T *, const PassArgs<T>, int, int);
template <typename T>
using StridedKernel = void (*)(const CUtensorMap, typename Cplx<T>::type *, const PassArgs<T>, int);
template <typename T>
using FwdKernel = void (*)(const T *, typename Cplx<T>::type *, const PassArgs<T>, const FuseArgs);
template <typename T>
using InvKernel = void (*)(const CUtensorMap, typename Cplx<T>::type *, T *, const PassArgs<T>, const FuseArgs);

// The specialised length for an axis of n points, or 0 (runtime plan).
static int special_n(int n) {
#define FF_CASE(NN) if (n == NN) return NN;
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return 0;
}

// bulk: line blocks by bulk copies (always for specialised lengths)
template <typename T> static ZFwdKernel<T> zfwd_kernel(int N, bool bulk) {
#define FF_CASE(NN) if (N == NN) return k_zfwd<T, NN, true>;
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return bulk ? k_zfwd<T, 0, true> : k_zfwd<T, 0, false>;
}
template <typename T> static ZInvKernel<T> zinv_kernel(int N, bool bulk) {
#define FF_CASE(NN) if (N == NN) return k_zinv<T, NN, true>;
  FF_FOR_EACH_SPECIAL_N(FF_CASE)
#undef FF_CASE
  return bulk ? k_zinv<T, 0, true> : k_zinv<T, 0, false>;
}

// kind: 0 = y forward, 1 = y inverse, 2 = x (forward, filter, inverse);
// N: the compile-time plan (0: runtime plan); W: columns per tile row.
template <typename T, int N, int W> static StridedKernel<T> strided_nw(int kind) {
  return kind == 0 ? k_strided<T, W, false, false, N>
                   : kind == 1 ? k_strided<T, W, false, true, N> : k_strided<T, W, true, false, N>;
}
// Lengths with compile-time strided tiles of 128-byte rows; 1024-point lines
// take 64-byte rows (a 64 KB tile, as a 512-point line's), longer lines than
// 128-byte rows hold take 64- or 32-byte rows with runtime plans.
#define FF_FOR_EACH_STRIDED_N(X) X(64) X(128) X(256) X(512)
template <typename T> static StridedKernel<T> strided_kernel(int kind, int N, int W = 128 / (2 * (int)sizeof(T))) {
  constexpr int WF = 128 / (2 * (int)sizeof(T));
  if (W == WF / 2) return N == 1024 ? strided_nw<T, 1024, WF / 2>(kind) : strided_nw<T, 0, WF / 2>(kind);
  if (W == WF / 4) return strided_nw<T, 0, WF / 4>(kind);
#define FF_CASE(NN) if (N == NN) return strided_nw<T, NN, WF>(kind);
  FF_FOR_EACH_STRIDED_N(FF_CASE)
#undef FF_CASE
  return strided_nw<T, 0, WF>(kind);
}

// (z, y) length pairs with specialised fused kernels; others use (0, 0).
#define FF_FOR_EACH_FUSED_PAIR(X) X(512, 512) X(256, 512) X(256, 256)

static void fused_pair(int nk, int nj, int *NZ, int *NY) {
  *NZ = *NY = 0;
#define FF_CASE(A, B) if (nk == A && nj == B) { *NZ = A; *NY = B; }
  FF_FOR_EACH_FUSED_PAIR(FF_CASE)
#undef FF_CASE
}
template <typename T> static FwdKernel<T> fwd_kernel(int NZ, int NY) {
#define FF_CASE(A, B) if (NZ == A && NY == B) return k_zy_fwd<T, A, B>;
  FF_FOR_EACH_FUSED_PAIR(FF_CASE)
#undef FF_CASE
  return k_zy_fwd<T, 0, 0>;
}
template <typename T> static InvKernel<T> inv_kernel(int NZ, int NY) {
#define FF_CASE(A, B) if (NZ == A && NY == B) return k_yz_inv<T, A, B>;
  FF_FOR_EACH_FUSED_PAIR(FF_CASE)
#undef FF_CASE
  return k_yz_inv<T, 0, 0>;
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
  const int ni = p->n[0], nj = p->n[1], nk = p->n[2];
  int rc = FF_OK;
  // passes along an axis with a prime factor above 7 (pass kind -> axis)
  const int axis_of_kind[5] = {2, 1, 0, 1, 2};
  for (int kind = 0; kind < 5 && rc == FF_OK; kind++)
    if (p->bsM[axis_of_kind[kind]])
      rc = bs_configure<T>(kind, ni, nj, p->nh, p->bsM[axis_of_kind[kind]], &p->bscfg[kind]);
  if (rc != FF_OK) return rc;
  const bool any_bs = p->bsM[0] || p->bsM[1] || p->bsM[2];
  // z tiles: W line pairs, two line-major buffers of pitch P, ~32 KB per
  // block of kZPassThreads threads (six blocks per SM)
  const int align = csz == 16 ? 8 : 16;
  p->zN = special_n(nk);
  p->zP = (nk + align - 1) / align * align;
  const size_t per_pair = 2 * (size_t)p->zP * csz;
  p->zW = (int)std::max<size_t>(1, std::min<size_t>(8, (32 * 1024) / per_pair));
  // A: max(W*P, 2W*nhp) values (stages, then output staging), B: W*P values
  // (+ slack for a copy rounded up to 16 bytes), base alignment; where the
  // forward pass fuses its last stage with the split (z_split_fused) B stages
  // the output and is as large as A
  const size_t a_bytes = (std::max<size_t>((size_t)p->zW * p->zP, 2 * (size_t)p->zW * p->nhp) * csz + 127) & ~size_t(127);
  const bool zfuse = p->zN > 0 && z_split_fused(p->zN, csz);
  p->zsmem = a_bytes + (zfuse ? a_bytes : (size_t)p->zW * p->zP * csz) + 128 + 128;
  const long npairs = ((long)ni * nj + 1) / 2;
  p->ztiles = (unsigned)((npairs + p->zW - 1) / p->zW);
  // line blocks by bulk copies: whole 16-byte multiples, and a first stage
  // that is not the last (the bulk-fed tiles stage their input in the buffer
  // the last stage writes)
  p->zbulk = p->zN > 0 || ((nk * sizeof(T)) % 16 == 0 && plan_stages(nk) >= 2);
  if (!p->bsM[2]) {
    rc = allow_dyn_smem(zfwd_kernel<T>(p->zN, p->zbulk), nullptr);
    if (rc == FF_OK) rc = allow_dyn_smem(zinv_kernel<T>(p->zN, p->zbulk), nullptr);
    if (rc != FF_OK) return rc;
  }
  // strided tiles: W columns of 128-byte rows x n rows, one per block; lines
  // too long for that (above about 1800 points FP64, 3600 FP32) take 64- or
  // 32-byte rows, i.e. half or a quarter of the columns per tile
  const int W = 128 / (int)csz;
  for (int kind = 0; kind < 3; kind++) {
    StridedCfg &cfg = kind == 2 ? p->xcfg : p->ycfg;
    const int n = kind == 2 ? ni : nj;
    if (p->bsM[kind == 2 ? 0 : 1]) continue;
    cfg.N = special_n(n);
    cfg.W = W;
    // 1024-point lines: 64-byte rows, so the tile stays 64 KB and three blocks
    // share an SM (0.63 ms for the 1024x512x256 FP64 x pass, against 0.88 ms
    // for a 1024-row tile split over a 2-block cluster and 1.06 ms for one
    // block of 128-byte rows per SM)
    if (cfg.N == 1024) cfg.W = W / 2;
    while ((size_t)n * cfg.W * csz + 1024 > kMaxDynSmem && cfg.W * csz > 32) {
      cfg.W /= 2;
      cfg.N = 0;
    }
    cfg.box_rows = largest_divisor_at_most(n, 256, 1);
    cfg.smem = (size_t)n * cfg.W * csz + 128;
    size_t avail = 0;
    rc = allow_dyn_smem(strided_kernel<T>(kind, cfg.N, cfg.W), &avail);
    if (rc != FF_OK) return rc;
    if (cfg.smem > avail) return set_error(FF_ERR_UNSUPPORTED, "no tile shape for an axis of %d points", n);
    cfg.grid = (kind == 2 ? nj : ni) * ((p->nh + cfg.W - 1) / cfg.W);
  }
  const int ktiles = (p->nh + W - 1) / W;
  // the fused passes hold a whole y tile of 128-byte rows per block (not with
  // Bluestein axes or narrowed tiles)
  const bool can_fuse = !any_bs && p->ycfg.W == W && p->xcfg.W == W;
  // fused passes: persistent blocks over the in-order tile queue (not with
  // Bluestein axes)
  const int zpp = (nj + 2 * p->zW - 1) / (2 * p->zW);   // z tiles per plane (pairs never cross planes)
  for (int dir = 0; dir < 2 && can_fuse; dir++) {
    FusedCfg &fc = dir == 0 ? p->fwd : p->inv;
    fused_pair(nk, nj, &fc.NZ, &fc.NY);
    fc.smem = std::max(p->zsmem, p->ycfg.smem);
    fc.prod_pp = dir == 0 ? zpp : ktiles;
    fc.cons_pp = dir == 0 ? ktiles : zpp;
    int per_sm = 0;
    size_t avail = 0;
    if (dir == 0) {
      FwdKernel<T> fn = fwd_kernel<T>(fc.NZ, fc.NY);
      rc = allow_dyn_smem(fn, &avail);
      if (rc != FF_OK) return rc;
      if (fc.smem > avail) return set_error(FF_ERR_UNSUPPORTED, "fused pass does not fit (%zu bytes)", fc.smem);
      FF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kZThreads, fc.smem));
    } else {
      InvKernel<T> fn = inv_kernel<T>(fc.NZ, fc.NY);
      rc = allow_dyn_smem(fn, &avail);
      if (rc != FF_OK) return rc;
      if (fc.smem > avail) return set_error(FF_ERR_UNSUPPORTED, "fused pass does not fit (%zu bytes)", fc.smem);
      FF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kZThreads, fc.smem));
    }
    if (per_sm < 1) return set_error(FF_ERR_UNSUPPORTED, "fused pass does not fit on an SM");
    const long total = (long)ni * (fc.prod_pp + fc.cons_pp);
    fc.grid = (int)std::min<long>(total, (long)per_sm * p->num_sms);
    // consumers of plane i are queued once the blocks in flight have moved
    // about 1.5 grids of tiles past its producers
    const int per_plane = fc.prod_pp + fc.cons_pp;
    fc.lag = std::min(ni, std::max(2, (3 * fc.grid + 2 * per_plane - 1) / (2 * per_plane)));
  }
  // The z passes run one tile per block, six blocks per SM, each waiting for
  // its inbound line block.  Block b hints block b + l2_ahead's lines
  // (forward) or spectrum rows (inverse) into L2, so that read is under way
  // while the resident blocks compute and the later bulk copy finds them in
  // L2.  (The same hint on the strided passes' tensor tiles slowed them.)
  const char *ahead = getenv("FF_L2_AHEAD");
  p->l2_ahead = ahead ? std::max(0, atoi(ahead)) : 6 * p->num_sms;
  const char *mode = getenv("FF_PASSES");
  p->fused = mode && strcmp(mode, "3") == 0 && can_fuse;
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

// Tensor map of a half spectrum at `base` (ni planes of nj rows of nh complex
// values, row pitch nhp) viewed as (2*nh reals, nj, ni); box = W columns by
// box_rows rows of one plane (y pass) or box_rows planes of one row (x pass).
int encode_spectrum_map(void *base, int ni, int nj, int nh, int nhp, size_t esz, int W, int box_rows, bool xpass,
                        CUtensorMap *map) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return set_error(FF_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  const cuuint64_t csz = 2 * esz;
  cuuint64_t dims[3] = {(cuuint64_t)2 * nh, (cuuint64_t)nj, (cuuint64_t)ni};
  cuuint64_t strides[2] = {(cuuint64_t)nhp * csz, (cuuint64_t)nhp * csz * nj};
  cuuint32_t box[3] = {(cuuint32_t)(2 * W), xpass ? 1u : (cuuint32_t)box_rows, xpass ? (cuuint32_t)box_rows : 1u};
  cuuint32_t estr[3] = {1, 1, 1};
  const CUtensorMapDataType dt = esz == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
  CUresult r = enc(map, dt, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                   CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return set_error(FF_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return FF_OK;
}

template <typename T> static int spectrum_map(const ff_plan *p, void *base, const StridedCfg &cfg, bool xpass,
                                              CUtensorMap *map) {
  return encode_spectrum_map(base, p->n[0], p->n[1], p->nh, p->nhp, sizeof(T), cfg.W, cfg.box_rows, xpass, map);
}

template <typename T>
static int launch_solve(const ff_plan *p, void *density, void *potential, cudaStream_t st, bool timed,
                        int npass = 5) {
  using C = typename Cplx<T>::type;
  const PassArgs<T> a = pass_args<T>(p);
  T *D = static_cast<T *>(density);
  T *P = static_cast<T *>(potential);
  C *Ds = reinterpret_cast<C *>(density);
  C *Ps = reinterpret_cast<C *>(potential);
  CUtensorMap ymapP, xmapP;
  int rc = FF_OK;
  if (!p->bsM[1]) rc = spectrum_map<T>(p, potential, p->ycfg, false, &ymapP);
  if (rc == FF_OK && !p->bsM[0]) rc = spectrum_map<T>(p, potential, p->xcfg, true, &xmapP);
  if (rc != FF_OK) return rc;
  auto bsax = [&](int d) -> const BsAxis<C> & {
    if constexpr (sizeof(T) == 8) return p->bsd[d];
    else return p->bsf[d];
  };
  int ev = 0;
  if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
  if (p->fused) {
    const int ni = p->n[0];
    FF_CUDA(cudaMemsetAsync(p->counters, 0, (2 + 2 * (size_t)ni) * sizeof(int), st));
    FuseArgs ff{p->counters, p->counters + 2, ni, p->fwd.prod_pp, p->fwd.cons_pp, p->fwd.lag, p->zW, p->zP,
                p->ycfg.box_rows, p->wait_iters, p->dep_extra};
    fwd_kernel<T>(p->fwd.NZ, p->fwd.NY)<<<p->fwd.grid, kZThreads, p->fwd.smem, st>>>(D, Ps, a, ff);
    FF_CUDA(cudaGetLastError());
    if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
    strided_kernel<T>(2, p->xcfg.N, p->xcfg.W)<<<p->xcfg.grid, kZThreads, p->xcfg.smem, st>>>(xmapP, Ps, a, p->xcfg.box_rows);
    FF_CUDA(cudaGetLastError());
    if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
    FuseArgs fi{p->counters + 1, p->counters + 2 + ni, ni, p->inv.prod_pp, p->inv.cons_pp, p->inv.lag, p->zW, p->zP,
                p->ycfg.box_rows, p->wait_iters, p->dep_extra};
    inv_kernel<T>(p->inv.NZ, p->inv.NY)<<<p->inv.grid, kZThreads, p->inv.smem, st>>>(ymapP, Ds, P, a, fi);
    FF_CUDA(cudaGetLastError());
    if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
    return FF_OK;
  }
  // each pass through the Bluestein kernels where its axis needs them
  if (p->bsM[2]) {
    rc = bs_launch<T>(0, D, Ps, a, bsax(2), p->bscfg[0], st);
    if (rc != FF_OK) return rc;
  } else {
    zfwd_kernel<T>(p->zN, p->zbulk)<<<p->ztiles, kZPassThreads, p->zsmem, st>>>(D, Ps, a, p->zW, p->zP);
    FF_CUDA(cudaGetLastError());
  }
  if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
  if (npass == 1) return FF_OK;
  if (p->bsM[1]) {
    rc = bs_launch<T>(1, Ps, Ps, a, bsax(1), p->bscfg[1], st);
    if (rc != FF_OK) return rc;
  } else {
    strided_kernel<T>(0, p->ycfg.N, p->ycfg.W)<<<p->ycfg.grid, kZThreads, p->ycfg.smem, st>>>(ymapP, Ps, a, p->ycfg.box_rows);
    FF_CUDA(cudaGetLastError());
  }
  if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
  if (npass == 2) return FF_OK;
  if (p->bsM[0]) {
    rc = bs_launch<T>(2, Ps, Ps, a, bsax(0), p->bscfg[2], st);
    if (rc != FF_OK) return rc;
  } else {
    strided_kernel<T>(2, p->xcfg.N, p->xcfg.W)<<<p->xcfg.grid, kZThreads, p->xcfg.smem, st>>>(xmapP, Ps, a, p->xcfg.box_rows);
    FF_CUDA(cudaGetLastError());
  }
  if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
  if (npass == 3) return FF_OK;
  if (p->bsM[1]) {
    rc = bs_launch<T>(3, Ps, Ds, a, bsax(1), p->bscfg[3], st);
    if (rc != FF_OK) return rc;
  } else {
    strided_kernel<T>(1, p->ycfg.N, p->ycfg.W)<<<p->ycfg.grid, kZThreads, p->ycfg.smem, st>>>(ymapP, Ds, a, p->ycfg.box_rows);
    FF_CUDA(cudaGetLastError());
  }
  if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
  if (npass == 4) return FF_OK;
  if (p->bsM[2]) {
    rc = bs_launch<T>(4, Ds, P, a, bsax(2), p->bscfg[4], st);
    if (rc != FF_OK) return rc;
  } else {
    zinv_kernel<T>(p->zN, p->zbulk)<<<p->ztiles, kZPassThreads, p->zsmem, st>>>(Ds, P, a, p->zW, p->zP);
    FF_CUDA(cudaGetLastError());
  }
  if (timed) FF_CUDA(cudaEventRecord(p->ev[ev++], st));
  return FF_OK;
}

int allow_dyn_smem_fn(const void *fn, size_t *avail) {
  cudaFuncAttributes fa;
  FF_CUDA(cudaFuncGetAttributes(&fa, fn));
  const size_t lim = kMaxDynSmem - fa.sharedSizeBytes;
  FF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)lim));
  if (avail) *avail = lim;
  return FF_OK;
}

template <typename T> static int launch_z(const ff_plan *p, bool inverse, void *in, void *out, cudaStream_t st) {
  using C = typename Cplx<T>::type;
  const PassArgs<T> a = pass_args<T>(p);
  if (p->bsM[2]) {
    const BsAxis<C> *bs;
    if constexpr (sizeof(T) == 8) bs = &p->bsd[2];
    else bs = &p->bsf[2];
    return bs_launch<T>(inverse ? 4 : 0, in, out, a, *bs, p->bscfg[inverse ? 4 : 0], st);
  }
  if (!inverse)
    zfwd_kernel<T>(p->zN, p->zbulk)<<<p->ztiles, kZPassThreads, p->zsmem, st>>>(static_cast<const T *>(in),
                                                                          static_cast<C *>(out), a, p->zW, p->zP);
  else
    zinv_kernel<T>(p->zN, p->zbulk)<<<p->ztiles, kZPassThreads, p->zsmem, st>>>(static_cast<const C *>(in),
                                                                          static_cast<T *>(out), a, p->zW, p->zP);
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

int plan_launch_z(const ff_plan *p, bool inverse, void *in, void *out, cudaStream_t st) {
  return p->precision == FF_FP64 ? launch_z<double>(p, inverse, in, out, st)
                                 : launch_z<float>(p, inverse, in, out, st);
}

static int plan_phases(const ff_plan *p) { return p->fused ? 3 : 5; }

// Reads and clears the device status word; FF_ERR_TIMEOUT if a bounded wait
// inside a kernel gave up.
int take_device_status(const ff_plan *p, cudaStream_t st) {
  int h = 0;
  FF_CUDA(cudaMemcpyAsync(&h, p->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  FF_CUDA(cudaStreamSynchronize(st));
  if (h != kDevOk) {
    FF_CUDA(cudaMemsetAsync(p->status, 0, sizeof(int), st));
    FF_CUDA(cudaStreamSynchronize(st));
    return set_error(FF_ERR_TIMEOUT, "%s (device status %d)",
                     h == kDevTmaTimeout ? "a TMA tile load did not complete within its wait limit"
                                         : "a fused pass waited too long for a plane's producer tiles",
                     h);
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

const char *ff_phase_name(const ff_plan *p, int q) {
  // the reference's stamp names (ParisPencil.cpp:142-424) for the phases that
  // survive on one GPU; the fused passes join two of them
  static const char *five[5] = {"Real-to-complex FFT in Z", "Forward FFT in Y", "X FFTs and filter",
                                "Backward FFT in Y", "Complex-to-real FFT in Z"};
  static const char *three[3] = {"Real-to-complex FFT in Z + Forward FFT in Y", "X FFTs and filter",
                                 "Backward FFT in Y + Complex-to-real FFT in Z"};
  if (!p || q < 0 || q >= plan_phases(p)) return "";
  return p->fused ? three[q] : five[q];
}

int ff_plan_phases(const ff_plan *p) { return p ? plan_phases(p) : 0; }

int ff_plan_create(const int n[3], const double lo[3], const double hi[3], int precision, ff_plan **out) {
  if (!n || !lo || !hi || !out) return set_error(FF_ERR_INVALID, "ff_plan_create: null argument");
  *out = nullptr;
  if (precision != FF_FP64 && precision != FF_FP32)
    return set_error(FF_ERR_INVALID, "ff_plan_create: precision %d is neither FF_FP64 nor FF_FP32", precision);
  for (int d = 0; d < 3; d++) {
    if (n[d] < 1) return set_error(FF_ERR_INVALID, "ff_plan_create: n[%d] = %d < 1", d, n[d]);
    if (n[d] > FF_MAX_AXIS)
      return set_error(FF_ERR_UNSUPPORTED, "ff_plan_create: n[%d] = %d is above %d", d, n[d], FF_MAX_AXIS);
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

  // device tables: per axis tw (L complex), rev and ipos (L ints) of the
  // axis's transform length L (n, or the padded M of a Bluestein axis), the
  // chirp (n) and kernel transform (M) of a Bluestein axis; kk per axis; one
  // status word
  std::vector<int> radix[3], rev[3];
  int len[3];
  size_t off = 0;
  size_t o_tw[3], o_tw64[3], o_rev[3], o_ipos[3], o_kk[3], o_chirp[3] = {0, 0, 0}, o_ghat[3] = {0, 0, 0};
  auto take = [&](size_t b) { size_t o = off; off += (b + 255) & ~size_t(255); return o; };
  for (int d = 0; d < 3; d++) {
    p->bsM[d] = smooth2357(n[d]) ? 0 : bs_padded_length(n[d]);
    const int L = len[d] = p->bsM[d] ? p->bsM[d] : n[d];
    radix[d] = plan_factor_radices(L);
    if ((int)radix[d].size() > kMaxStages) {
      delete p;
      return set_error(FF_ERR_UNSUPPORTED, "ff_plan_create: too many stages");
    }
    rev[d] = plan_digit_reversal(L, radix[d]);
    o_tw[d] = take(L * csz);
    o_tw64[d] = precision == FF_FP64 ? o_tw[d] : take(L * sizeof(double2));
    o_rev[d] = take(L * sizeof(int));
    o_ipos[d] = take(L * sizeof(int));
    o_kk[d] = take((d == 2 ? p->nh : n[d]) * sizeof(double));
    if (p->bsM[d]) {
      o_chirp[d] = take(n[d] * csz);
      o_ghat[d] = take(L * csz);
    }
  }
  const size_t o_status = take(sizeof(int));
  const size_t o_counters = take((2 + 2 * (size_t)n[0]) * sizeof(int));
  for (int e = 0; e <= FF_MAX_PHASES; e++) {
    if (cudaEventCreate(&p->ev[e]) != cudaSuccess) {
      for (int q = 0; q < e; q++) cudaEventDestroy(p->ev[q]);
      delete p;
      return set_error(FF_ERR_CUDA, "ff_plan_create: cudaEventCreate failed");
    }
  }
  if (cudaMalloc(&p->dmem, off) != cudaSuccess) {
    cudaGetLastError();
    for (int e = 0; e <= FF_MAX_PHASES; e++) cudaEventDestroy(p->ev[e]);
    delete p;
    return set_error(FF_ERR_NOMEM, "ff_plan_create: cudaMalloc(%zu) for plan tables failed", off);
  }
  char *base = static_cast<char *>(p->dmem);
  p->status = reinterpret_cast<int *>(base + o_status);
  p->counters = reinterpret_cast<int *>(base + o_counters);
  int rc = FF_OK;
  if (cudaMemset(p->status, 0, sizeof(int)) != cudaSuccess) rc = set_error(FF_ERR_CUDA, "ff_plan_create: memset");
  for (int d = 0; d < 3 && rc == FF_OK; d++) {
    const int L = len[d];
    std::vector<int> ipos(L);
    for (int q = 0; q < L; q++) ipos[rev[d][q]] = q;
    if (cudaMemcpy(base + o_rev[d], rev[d].data(), L * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + o_ipos[d], ipos.data(), L * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
      rc = set_error(FF_ERR_CUDA, "ff_plan_create: table upload failed");
    const int blocks = std::min(1024, (L + 255) / 256);
    k_twiddles<<<blocks, 256>>>(L, reinterpret_cast<double2 *>(base + o_tw64[d]));
    if (precision == FF_FP32) k_twiddles<<<blocks, 256>>>(L, reinterpret_cast<float2 *>(base + o_tw[d]));
    const int cnt = d == 2 ? p->nh : n[d];
    k_wavenumbers<<<std::min(1024, (cnt + 255) / 256), 256>>>(n[d], cnt, d != 2, p->dd[d],
                                                              reinterpret_cast<double *>(base + o_kk[d]));
    p->kk[d] = reinterpret_cast<double *>(base + o_kk[d]);
    AxisDev<double2> ad{};
    AxisDev<float2> af{};
    ad.n = af.n = L;
    ad.nstages = af.nstages = (int)radix[d].size();
    for (size_t s = 0; s < radix[d].size(); s++) ad.radix[s] = af.radix[s] = radix[d][s];
    ad.tw = reinterpret_cast<const double2 *>(base + o_tw[d]);
    af.tw = reinterpret_cast<const float2 *>(base + o_tw[d]);
    ad.tw64 = af.tw64 = reinterpret_cast<const double2 *>(base + o_tw64[d]);
    ad.rev = af.rev = reinterpret_cast<const int *>(base + o_rev[d]);
    ad.ipos = af.ipos = reinterpret_cast<const int *>(base + o_ipos[d]);
    p->axd[d] = ad;
    p->axf[d] = af;
    if (p->bsM[d] && rc == FF_OK) {
      const int *drev = reinterpret_cast<const int *>(base + o_rev[d]);
      if (precision == FF_FP64) {
        double2 *ch = reinterpret_cast<double2 *>(base + o_chirp[d]), *gh = reinterpret_cast<double2 *>(base + o_ghat[d]);
        rc = bs_tables<double2>(n[d], L, drev, ch, gh);
        p->bsd[d] = BsAxis<double2>{ad, n[d], ch, gh};
      } else {
        float2 *ch = reinterpret_cast<float2 *>(base + o_chirp[d]), *gh = reinterpret_cast<float2 *>(base + o_ghat[d]);
        rc = bs_tables<float2>(n[d], L, drev, ch, gh);
        p->bsf[d] = BsAxis<float2>{af, n[d], ch, gh};
      }
    }
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
    const int np = plan_phases(p);
    FF_CUDA(cudaEventSynchronize(p->ev[np]));
    times->count = np;
    for (int q = 0; q < FF_MAX_PHASES; q++) {
      float ms = 0;
      if (q < np) FF_CUDA(cudaEventElapsedTime(&ms, p->ev[q], p->ev[q + 1]));
      times->ms[q] = ms;
    }
    float tot = 0;
    FF_CUDA(cudaEventElapsedTime(&tot, p->ev[0], p->ev[np]));
    times->total_ms = tot;
    return take_device_status(p, st);
  }
  return FF_OK;
}

int ff_solve_passes(const ff_plan *p, size_t bytes, void *density, void *potential, void *stream, int passes) {
  if (!p || !density || !potential) return set_error(FF_ERR_INVALID, "ff_solve_passes: null argument");
  if (passes < 1 || passes > 5) return set_error(FF_ERR_INVALID, "ff_solve_passes: passes = %d", passes);
  if (p->fused) return set_error(FF_ERR_INVALID, "ff_solve_passes: the plan fuses its passes (FF_PASSES=3)");
  if (bytes < p->bytes) return set_error(FF_ERR_BYTES, "ff_solve_passes: bytes %zu < required %zu", bytes, p->bytes);
  if (density == potential) return set_error(FF_ERR_INVALID, "ff_solve_passes: density and potential must differ");
  if (((uintptr_t)density | (uintptr_t)potential) & 15)
    return set_error(FF_ERR_INVALID, "ff_solve_passes: buffers must be 16-byte aligned");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return p->precision == FF_FP64 ? launch_solve<double>(p, density, potential, st, false, passes)
                                 : launch_solve<float>(p, density, potential, st, false, passes);
}

int ff_plan_check(const ff_plan *p, void *stream) {
  if (!p) return set_error(FF_ERR_INVALID, "ff_plan_check: null plan");
  return take_device_status(p, static_cast<cudaStream_t>(stream));
}

int ff_plan_set_wait_limit(ff_plan *p, int iterations, int target_extra) {
  if (!p) return set_error(FF_ERR_INVALID, "ff_plan_set_wait_limit: null plan");
  if (iterations < 0 || target_extra < 0)
    return set_error(FF_ERR_INVALID, "ff_plan_set_wait_limit: negative argument");
  p->wait_iters = iterations;
  p->dep_extra = target_extra;
  return FF_OK;
}

int ff_plan_destroy(ff_plan *p) {
  if (!p) return FF_OK;
  int rc = FF_OK;
  for (int e = 0; e <= FF_MAX_PHASES; e++)
    if (p->ev[e]) cudaEventDestroy(p->ev[e]);
  if (p->dmem && cudaFree(p->dmem) != cudaSuccess) rc = set_error(FF_ERR_CUDA, "ff_plan_destroy: cudaFree failed");
  delete p;
  return rc;
}

}  // extern "C"
