// Device code of the batch passes: grid descriptors, the column tiles of the
// strided passes, the per-pass persistent kernel and its launch helpers.
// Included by ff_batch_f64.cu and ff_batch_f32.cu, one precision each.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstring>

#include "ff_batch.hpp"
#include "ff_status.hpp"
#include "ff_tiles.cuh"

namespace ff {

// Device descriptor of one grid: its pass arguments, its two buffers and
// the tile shape of each pass.  Copied into shared memory for each tile.
template <typename T> struct alignas(16) GridDesc {
  PassArgs<T> a;
  T *density;
  T *potential;
  TileShape shape[5];
  int box_rows[2];   // rows per TMA box: y pass, x pass
};

// ------------------------------------------------------------ column tiles
// A strided pass over W columns of the flattened column index
// q = plane * nh + kh: y columns are (i, kh) with rows j at stride nhp, x
// columns are (j, kh) with rows i at stride nj*nhp.  Consecutive q of one
// plane are contiguous, so every row access of a warp is coalesced.  The tile
// arrives by asynchronous element copies (every load of the tile in flight at
// once), the stages run in the point-major tile, and the last stage writes
// HBM; all reads of a column precede the first barrier, so src may equal dst.  The x pass runs forward DIF, the -1/k^2 filter fused with the
// last DIF and first DIT stages, and the inverse DIT.  Thread t owns column
// t % W in every stage (column-fastest item order, W divides the block).
template <typename T, int W, bool XPASS, bool INV, int N>
__device__ __forceinline__ void cols_tile(const PassArgs<T> &a, const typename Cplx<T>::type *src,
                                          typename Cplx<T>::type *dst, int tile, typename Cplx<T>::type *sm) {
  using C = typename Cplx<T>::type;
  constexpr int NT = kZThreads;
  static_assert(NT % W == 0, "a thread keeps one column");
  const AxisDev<C> &ax = XPASS ? a.ax[0] : a.ax[1];
  const long rs = XPASS ? (long)a.nj * a.nhp : (long)a.nhp;
  const long ps = XPASS ? (long)a.nhp : (long)a.nj * a.nhp;
  const long ncols = (long)(XPASS ? a.nj : a.ni) * a.nh;
  const long q = (long)tile * W + (int)(threadIdx.x % W);
  const bool valid = q < ncols;
  const int o = valid ? (int)(q / a.nh) : 0;
  const int kh = valid ? (int)(q - (long)o * a.nh) : 0;
  const long cb = (long)o * ps + kh;
  const auto rl = rev_last<N>(ax);
  PointTile<W, C> tl{sm};
  {
    // the whole tile by asynchronous element copies, all in flight at once
    // (measured against loading stage 0 from HBM into registers: FP64 batch
    // x pass 0.87 -> 0.68 ms, y 0.50 -> 0.44 ms)
    const int n = N > 0 ? N : ax.n;
    const int c = threadIdx.x % W;
    for (int pos = threadIdx.x / W; pos < n; pos += NT / W) {
      C *d = sm + pos * W + c;
      if (!valid) *d = mk((T)0, (T)0);
      else if constexpr (sizeof(C) == 16) cp_async16(d, src + cb + (long)pos * rs);
      else cp_async8(d, src + cb + (long)pos * rs);
    }
    cp_async_wait_all();
    __syncthreads();
  }
  // FP64 twiddle powers by recurrence, FP32 by table loads (as the single-grid passes)
  constexpr bool TWR = sizeof(T) == 8;
  if constexpr (!XPASS) {
    auto gst = [&](int pos, int, C v) {
      if (valid) dst[cb + (long)rl(pos) * rs] = v;
    };
    dif_all<N, INV, Map::ColFast, W, NT, false, TWR>(ax, tl, tl, gst, W);
  } else {
    auto gst = [&](int pos, int, C v) {
      if (valid) dst[cb + (long)pos * rs] = v;
    };
    // d = -1/((i2 + j2) + k2) * 1/N as the single-grid x pass (ParisPencil.cpp:276-279)
    const int ni = a.ni;
    const double jd = double(min(o, a.nj - o)) * a.dd[1];
    const double j2 = jd * jd;
    const double ddi = a.dd[0];
    const double kd = double(kh) * a.dd[2];
    const double k2 = kd * kd;
    const double minvN = -a.invN;
    auto filt = [&](int pos, int, C v) -> C {
      const int kx = rl(pos);
      if (!valid) return v;
      if ((kx | o | kh) == 0) return mk((T)0, (T)0);
      const double id = double(min(kx, ni - kx)) * ddi;
      const double d = recip_pos((id * id + j2) + k2) * minvN;
      return cscale(v, (T)d);
    };
    if constexpr (N > 0) {
      constexpr int S = plan_stages(N);
      constexpr int RF = plan_radix(N, S - 1);
      if constexpr (S > 1) {
        dif_ct<N, S - 1, 0, false, Map::ColFast, W, NT, false, TWR>(ax, tl, tl, tl, W);
        fused_filter_stage<RF, W, NT, N, C>(N, tl, tl, filt);
        __syncthreads();
        dit_ct<N, S - 2, true, Map::ColFast, W, NT, TWR>(ax, tl, gst, W);
      } else {
        fused_filter_stage<RF, W, NT, N, C>(N, tl, gst, filt);
      }
    } else {
      const int S = ax.nstages;
      const int n = ax.n;
      if (S > 1) dif_rt<false, Map::ColFast, W, NT, false, TWR>(ax, S - 1, tl, tl, tl, W);
      with_radix(ax.radix[S - 1], [&](auto tag) {
        constexpr int R = decltype(tag)::value;
        if (S == 1) fused_filter_stage<R, W, NT, 0, C>(n, tl, gst, filt);
        else fused_filter_stage<R, W, NT, 0, C>(n, tl, tl, filt);
      });
      __syncthreads();
      if (S > 1) dit_rt<true, Map::ColFast, W, NT, TWR>(ax, S - 2, tl, gst, W);
    }
  }
}

// Strided tile with the column count chosen at run time: W * sizeof(C) is
// 128 * wb bytes.  Shapes whose tile exceeds the block budget are never
// planned and not instantiated.
template <typename T, bool XPASS, bool INV, int N>
__device__ __forceinline__ void cols_tile_w(int wb, const PassArgs<T> &a, const typename Cplx<T>::type *src,
                                            typename Cplx<T>::type *dst, int tile, typename Cplx<T>::type *sm) {
  using C = typename Cplx<T>::type;
  constexpr int W1 = 128 / (int)sizeof(C);
  constexpr bool fit2 = N == 0 || (size_t)N * 256 + 128 <= kBatchSmem;
  constexpr bool fit4 = N == 0 || (size_t)N * 512 + 128 <= kBatchSmem;
  if (wb == 4) {
    if constexpr (fit4) cols_tile<T, 4 * W1, XPASS, INV, N>(a, src, dst, tile, sm);
  } else if (wb == 2) {
    if constexpr (fit2) cols_tile<T, 2 * W1, XPASS, INV, N>(a, src, dst, tile, sm);
  } else {
    cols_tile<T, W1, XPASS, INV, N>(a, src, dst, tile, sm);
  }
}

// One tile of pass KIND of grid descriptor g.  Returns false if a bounded
// wait gave up (the status word is set).  parity tracks the block's
// mbarrier phase across the inbound bulk copies of the z inverse tiles.
// Strided tile of one plane by TMA (the single-grid tile code): W = 128
// bytes of kh columns, all n rows; tile = plane * ktiles + kt.
template <typename T, bool XPASS, bool INV, int N>
__device__ __forceinline__ bool tma_cols_tile(const GridDesc<T> &g, const CUtensorMap *map, int tile,
                                              typename Cplx<T>::type *sm, uint64_t *mbar, uint32_t &parity) {
  using C = typename Cplx<T>::type;
  constexpr int W = 128 / (int)sizeof(C);
  const PassArgs<T> &a = g.a;
  const int n = XPASS ? a.ni : a.nj;
  const int ktiles = (a.nh + W - 1) / W;
  const int o = tile / ktiles, kt = tile - o * ktiles;
  const int box_rows = g.box_rows[XPASS ? 1 : 0];
  if (!tma_tile<C, W, XPASS>(map, sm, mbar, parity, n, box_rows, o, kt, a.status)) return false;
  parity ^= 1u;
  if constexpr (XPASS) {
    x_tile<T, W, N>(map, a, o, kt, box_rows, sm);
  } else {
    PointTile<W, C> t{sm};
    y_tile<T, W, INV, N>(t, reinterpret_cast<C *>(INV ? g.density : g.potential), a, o, kt, sm);
  }
  return true;
}

template <typename T, int KIND>
__device__ __forceinline__ bool batch_tile(const GridDesc<T> &g, const CUtensorMap *maps, int tile,
                                           typename Cplx<T>::type *sm, uint64_t *mbar, uint32_t &parity) {
  using C = typename Cplx<T>::type;
  const PassArgs<T> &a = g.a;
  const TileShape sh = g.shape[KIND];
  if constexpr (KIND == 0 || KIND == 4) {
    const int zW = sh.W;
    const int align = sizeof(C) == 16 ? 8 : 16;
    const int P = (a.nk + align - 1) / align * align;
    const long nlines = (long)a.ni * a.nj;
    const long line0 = (long)tile * 2 * zW;
    const ZTileIO io{mbar, parity, a.status};
    if constexpr (KIND == 0) {
      C *spec = reinterpret_cast<C *>(g.potential);
      if (sh.ct) {
        switch (a.nk) {
#define FF_CASE(NN) \
  case NN: {                                                                              \
    const bool ok = z_fwd_tile<T, NN, true, true, true, kBatchZThreads>(g.density, spec, a, zW, P, line0, nlines, sm, io); \
    parity ^= 1u;                                                                         \
    return ok;                                                                            \
  }
          FF_FOR_EACH_BATCH_N(FF_CASE)
#undef FF_CASE
          default: break;
        }
      }
      if (sh.tma) {
        const bool ok = z_fwd_tile<T, 0, true, true, false, kBatchZThreads>(g.density, spec, a, zW, P, line0, nlines, sm, io);
        parity ^= 1u;
        return ok;
      }
      return z_fwd_tile<T, 0, false, false, false, kBatchZThreads>(g.density, spec, a, zW, P, line0, nlines, sm, io);
    } else {
      const C *spec = reinterpret_cast<const C *>(g.density);
      if (sh.ct) {
        switch (a.nk) {
#define FF_CASE(NN)                                                                       \
  case NN: {                                                                              \
    const bool ok = z_inv_tile<T, NN, true, true, kBatchZThreads>(spec, g.potential, a, zW, P, line0, nlines, sm, io); \
    parity ^= 1u;                                                                         \
    return ok;                                                                            \
  }
          FF_FOR_EACH_BATCH_N(FF_CASE)
#undef FF_CASE
          default: break;
        }
      }
      if (sh.tma) {
        const bool ok = z_inv_tile<T, 0, true, false, kBatchZThreads>(spec, g.potential, a, zW, P, line0, nlines, sm, io);
        parity ^= 1u;
        return ok;
      }
      return z_inv_tile<T, 0, false, false, kBatchZThreads>(spec, g.potential, a, zW, P, line0, nlines, sm, io);
    }
  } else {
    constexpr bool XPASS = KIND == 2;
    constexpr bool INV = KIND == 3;
    const C *src = reinterpret_cast<const C *>(g.potential);
    C *dst = reinterpret_cast<C *>(KIND == 3 ? g.density : g.potential);
    const int wb = sh.W * (int)sizeof(C) / 128;
    const int n = XPASS ? a.ni : a.nj;
    if (sh.tma) {
      const CUtensorMap *map = maps + (XPASS ? 1 : 0);
      // the grid's maps live in global memory and are rewritten when a
      // server slot changes hands
      if (threadIdx.x == 0) tensormap_acquire(map);
      if (sh.ct) {
        switch (n) {
#define FF_CASE(NN) \
  case NN: return tma_cols_tile<T, XPASS, INV, NN>(g, map, tile, sm, mbar, parity);
          FF_FOR_EACH_BATCH_TMA_N(FF_CASE)
#undef FF_CASE
          default: break;
        }
      }
      return tma_cols_tile<T, XPASS, INV, 0>(g, map, tile, sm, mbar, parity);
    }
    if (sh.ct) {
      switch (n) {
#define FF_CASE(NN) \
  case NN: cols_tile_w<T, XPASS, INV, NN>(wb, a, src, dst, tile, sm); return true;
        FF_FOR_EACH_BATCH_N(FF_CASE)
#undef FF_CASE
        default: break;
      }
    }
    cols_tile_w<T, XPASS, INV, 0>(wb, a, src, dst, tile, sm);
    return true;
  }
}

// Persistent pass kernel: blocks take tiles by ticket until the work list is
// exhausted; the tile's grid is found by binary search over the prefix sums.
#ifndef FF_BATCH_MINB
#define FF_BATCH_MINB 6
#endif
template <typename T, int KIND>
__global__ void __launch_bounds__((KIND == 0 || KIND == 4) ? kBatchZThreads : kZThreads,
                                  (KIND == 0 || KIND == 4) ? FF_BATCH_MINB : 3)
    k_batch(const GridDesc<T> *__restrict__ grids, const CUtensorMap *__restrict__ maps, const BatchWork wl) {
  using C = typename Cplx<T>::type;
  extern __shared__ unsigned char smraw[];
  __shared__ __align__(8) uint64_t mbar;
  __shared__ int s_ticket;
  __shared__ GridDesc<T> s_desc;
  C *sm = reinterpret_cast<C *>(align128(smraw));
  if (threadIdx.x == 0) {
    mbar_init(&mbar, 1);
    mbar_init_fence();
  }
  uint32_t parity = 0;
  const int total = __ldg(wl.start + wl.nentry);
  int last_g = -1;
  for (;;) {
    // the previous tile's shared-memory accesses (generic and bulk) are done
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) s_ticket = atomicAdd(wl.ticket, 1);
    __syncthreads();
    const int t = s_ticket;
    if (t >= total) break;
    int lo = 0, hi = wl.nentry - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(wl.start + mid) <= t) lo = mid;
      else hi = mid - 1;
    }
    const int g = wl.entry[lo].x;
    if constexpr (KIND == 0) {
      // forward z pass: hint the lines of the tile claimed about one round
      // later (ticket t + gridDim.x) into L2, where its inbound copy (bulk
      // copy or thread loads) will find them
      const int t2 = t + (int)gridDim.x;
      if (threadIdx.x == 32 && t2 < total) {   // not thread 0, which issues the tile's own copy
        int a2 = lo, b2 = wl.nentry - 1;
        while (a2 < b2) {
          const int mid = (a2 + b2 + 1) >> 1;
          if (__ldg(wl.start + mid) <= t2) a2 = mid;
          else b2 = mid - 1;
        }
        const GridDesc<T> *G = grids + wl.entry[a2].x;
        const int zW = G->shape[0].W;
        const int nk = G->a.nk;
        const long nlines = (long)G->a.ni * G->a.nj;
        const long l0 = (long)(t2 - __ldg(wl.start + a2)) * 2 * zW;
        const long l1 = min(l0 + 2 * zW, nlines);
        // within the buffer: its size is max(real field, half spectrum)
        const size_t cap = max((size_t)nlines * nk * sizeof(T), (size_t)nlines * G->a.nhp * 2 * sizeof(T));
        const size_t b0 = ((size_t)l0 * nk * sizeof(T)) & ~size_t(15);
        const size_t b1 = min(((size_t)l1 * nk * sizeof(T) + 15) & ~size_t(15), cap & ~size_t(15));
        if (b1 > b0) l2_prefetch(reinterpret_cast<const char *>(G->density) + b0, (uint32_t)(b1 - b0));
      }
    }
    if constexpr (KIND == 4) {
      // inverse z pass: the same hint on the spectrum rows of that tile's line
      // pairs (contiguous, nhp complex values per line, in density)
      const int t2 = t + (int)gridDim.x;
      if (threadIdx.x == 32 && t2 < total) {
        int a2 = lo, b2 = wl.nentry - 1;
        while (a2 < b2) {
          const int mid = (a2 + b2 + 1) >> 1;
          if (__ldg(wl.start + mid) <= t2) a2 = mid;
          else b2 = mid - 1;
        }
        const GridDesc<T> *G = grids + wl.entry[a2].x;
        const int zW = G->shape[4].W;
        const long nlines = (long)G->a.ni * G->a.nj;
        const size_t row = (size_t)G->a.nhp * 2 * sizeof(T);
        const long l0 = (long)(t2 - __ldg(wl.start + a2)) * 2 * zW;
        const long l1 = min(l0 + 2 * zW, nlines);
        if (l1 > l0) l2_prefetch(reinterpret_cast<const char *>(G->density) + (size_t)l0 * row, (uint32_t)((size_t)(l1 - l0) * row));
      }
    }
    if (g != last_g) {
      // descriptor of the tile's grid into shared memory (read-only below)
      const int4 *s = reinterpret_cast<const int4 *>(grids + g);
      int4 *d = reinterpret_cast<int4 *>(&s_desc);
      for (int w = threadIdx.x; w < (int)(sizeof(GridDesc<T>) / 16); w += blockDim.x) d[w] = __ldg(s + w);
      __syncthreads();
      last_g = g;
    }
    if (!batch_tile<T, KIND>(s_desc, maps + 2 * g, t - __ldg(wl.start + lo), sm, &mbar, parity)) break;
  }
}

template <typename T, int KIND> static void *batch_kernel_ptr() { return (void *)k_batch<T, KIND>; }

template <typename T> static void *batch_kernel(int kind) {
  switch (kind) {
    case 0: return batch_kernel_ptr<T, 0>();
    case 1: return batch_kernel_ptr<T, 1>();
    case 2: return batch_kernel_ptr<T, 2>();
    case 3: return batch_kernel_ptr<T, 3>();
    default: return batch_kernel_ptr<T, 4>();
  }
}

template <typename T>
int batch_pass_launch(int kind, const void *grids, const CUtensorMap *maps, const BatchWork &wl, int blocks,
                      size_t smem, cudaStream_t st) {
  const GridDesc<T> *g = static_cast<const GridDesc<T> *>(grids);
  switch (kind) {
    case 0: k_batch<T, 0><<<blocks, batch_threads(0), smem, st>>>(g, maps, wl); break;
    case 1: k_batch<T, 1><<<blocks, batch_threads(1), smem, st>>>(g, maps, wl); break;
    case 2: k_batch<T, 2><<<blocks, batch_threads(2), smem, st>>>(g, maps, wl); break;
    case 3: k_batch<T, 3><<<blocks, batch_threads(3), smem, st>>>(g, maps, wl); break;
    default: k_batch<T, 4><<<blocks, batch_threads(4), smem, st>>>(g, maps, wl); break;
  }
  FF_CUDA(cudaGetLastError());
  return FF_OK;
}

template <typename T> int batch_pass_prepare(int kind, size_t smem, int *per_sm) {
  const void *fn = batch_kernel<T>(kind);
  cudaFuncAttributes fa;
  FF_CUDA(cudaFuncGetAttributes(&fa, fn));
  if (fa.sharedSizeBytes + batch_budget(kind) > 227 * 1024)
    return set_error(FF_ERR_UNSUPPORTED, "batch kernel shared memory exceeds the block limit");
  FF_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)batch_budget(kind)));
  FF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, fn, batch_threads(kind), smem));
  return FF_OK;
}

template <typename T> size_t batch_desc_size() { return sizeof(GridDesc<T>); }

template <typename T> void batch_desc_fill(void *dst, const BatchGridHost &h) {
  GridDesc<T> g;
  memset(&g, 0, sizeof(g));
  g.a.ni = h.n[0];
  g.a.nj = h.n[1];
  g.a.nk = h.n[2];
  g.a.nh = h.nh;
  g.a.nhp = h.nhp;
  for (int d = 0; d < 3; d++) {
    if constexpr (sizeof(T) == 8) g.a.ax[d] = h.axd[d];
    else g.a.ax[d] = h.axf[d];
    g.a.kk[d] = nullptr;
    g.a.dd[d] = h.dd[d];
  }
  g.a.invN = h.invN;
  g.a.status = h.status;
  g.a.l2_ahead = 0;
  g.density = static_cast<T *>(h.density);
  g.potential = static_cast<T *>(h.potential);
  for (int k = 0; k < 5; k++) g.shape[k] = h.shape[k];
  g.box_rows[0] = h.box_rows[0];
  g.box_rows[1] = h.box_rows[1];
  memcpy(dst, &g, sizeof(g));
}

#define FF_INSTANTIATE_BATCH(T)                                                                               \
  template int batch_pass_launch<T>(int, const void *, const CUtensorMap *, const BatchWork &, int, size_t,   \
                                    cudaStream_t);                                                          \
  template int batch_pass_prepare<T>(int, size_t, int *);                                                    \
  template size_t batch_desc_size<T>();                                                                      \
  template void batch_desc_fill<T>(void *, const BatchGridHost &);

}  // namespace ff
