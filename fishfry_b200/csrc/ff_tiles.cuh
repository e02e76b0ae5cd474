// Tile-level device code shared by the single-grid passes (ff_solve.cu) and
// the many-grid passes (ff_batch.cu): the per-grid pass arguments, the z
// line-pair tiles (R2C / C2R along z), the fused x filter stage and helpers.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "ff_fft.cuh"

namespace ff {

template <typename T> struct PassArgs {
  using C = typename Cplx<T>::type;
  int ni, nj, nk, nh, nhp;
  AxisDev<C> ax[3];        // 0: x (n = ni), 1: y (nj), 2: z (nk)
  const double *kk[3];     // (min(i, n-i) * dd)^2 per axis; kk[2] indexed by kh
  double invN;             // 1 / (ni*nj*nk)
  double dd[3];            // wavenumber scales (ParisPencil.cpp:9-11)
  int *status;             // device status word (kDev*), 0 = ok
  int l2_ahead;            // z passes: block b prefetches block b + l2_ahead's input into L2 (0: off)
  int wait_iters;          // iteration limit of the first wait for an inbound copy (0: built-in)
};

constexpr int kZThreads = 256;

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

// ------------------------------------------------------------------ z tiles
// A z tile is W line pairs held in two line-major buffers A, B of pitch P.
// Pair c is lines (line0 + 2c, line0 + 2c + 1), transformed as
// z = f[a] + i f[b]; lines at or past `lend` are absent (zero in, no output).
//
// With TMAIO the tile's lines enter and leave by bulk copies between HBM and
// shared memory (the copy engine moves them; the threads only touch shared
// memory), using the buffers as staging.  Forward: the real lines land in B,
// the stages run in A, the last stage writes B, and the output is staged in A.
// Inverse: the spectrum rows land in A, the first stage reads them, the
// stages run in B, the last writes A, and the output lines are staged in B.
// Without TMAIO the first stage reads HBM and the output is written from
// registers.
// A holds max(W*P, 2W*nhp) complex values, B holds W*P (+ 128 bytes slack).
//
// LASTFUSE (single-grid passes, compile-time plans with a radix-8 prefix):
// the last stage is fused with the split (forward) or with the scatter of the
// two real lines (inverse), so the stages' output never goes through shared
// memory in natural order.  Forward: stages in A (LineTileZ), the last stage
// writes the staged spectrum rows into B, which then also holds
// max(W*P, 2W*nhp) values.  Inverse: stages in B (LineTileZ), the last stage
// writes the real lines into A.
struct ZTileIO {
  uint64_t *mbar;      // TMAIO: barrier of the inbound copy
  uint32_t parity;     // TMAIO: its phase
  int *status;         // TMAIO: timeout report
  int wait_iters;      // TMAIO: iteration limit of the wait (0: built-in)
};

// Inbound bulk copy of `bytes` (rounded up to 16) from src into dst, waited
// for on every thread with an iteration limit.  On a timeout the status word
// is set and thread 0 waits again, with the built-in limit, for the copy in
// flight to land before the block may leave (its shared memory is the copy's
// destination).
__device__ __forceinline__ bool bulk_in(void *dst, const void *src, size_t bytes, const ZTileIO &io) {
  if (threadIdx.x == 0) {
    const uint32_t b = (uint32_t)((bytes + 15) & ~size_t(15));
    mbar_expect_tx(io.mbar, b);
    bulk_load(dst, src, b, io.mbar);
  }
  const bool ok = mbar_wait_bounded(io.mbar, io.parity, io.wait_iters);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicExch(io.status, kDevTmaTimeout);
      mbar_wait_bounded(io.mbar, io.parity);
    }
    return false;
  }
  return true;
}

// Outbound bulk copy of the staged bytes; a tail that is not a multiple of 16
// bytes is stored by thread 0 itself.  Waits until the copy has read shared
// memory.  The caller has fenced its shared-memory writes and barriered.
template <typename E>
__device__ __forceinline__ void bulk_out(E *dst, const E *src, size_t count) {
  if (threadIdx.x == 0) {
    const size_t bytes = count * sizeof(E);
    const size_t body = bytes & ~size_t(15);
    if (body) {
      bulk_store(dst, src, (uint32_t)body);
      bulk_commit();
    }
    for (size_t q = body / sizeof(E); q < count; q++) dst[q] = src[q];
    if (body) bulk_wait_read();
  }
}

// The last DIF stage of a compile-time z forward transform fused with the R2C
// split (ParisPencil.cpp:152-165).  An item is the pair of last-stage groups
// whose frequency bases are k0 and nR - k0 (nR = N/RL), so a thread holds
// Z[k] and Z[N-k] of its RL frequency pairs in registers and writes
// A[k] = (Z[k] + conj Z[N-k]) / 2 and B[k] = (Z[k] - conj Z[N-k]) / (2i),
// k <= N/2, into the staging rows [line][kh] (pitch nhp) of `out`: the rows of
// the pair's two lines.  Consecutive threads take consecutive k0, so the
// staging stores are conflict free; LineTileZ spreads the group reads.  The
// two self-paired bases, 0 and nR/2, come after the others.
template <int N, int NT, typename C>
__device__ __forceinline__ void z_split_stage(const LineTileZ<C> &t, C *out, int nhp, int W) {
  using T = typename Real<C>::type;
  constexpr int S = plan_stages(N);
  constexpr int RL = plan_radix(N, S - 1);
  constexpr int nR = N / RL;
  constexpr int NG = nR / 2 - 1;   // bases 1 .. nR/2 - 1 (with their partners)
  static_assert(radix8_prefix(N) && nR >= 4, "fused split needs a radix-8 prefix");
  const T h = (T)0.5;
  auto emit = [&](int c, int k, C p, C q) {   // p = Z[k], q = Z[N - k]
    out[(2 * c) * nhp + k] = mk(h * (p.x + q.x), h * (p.y - q.y));
    out[(2 * c + 1) * nhp + k] = mk(h * (p.y + q.y), h * (q.x - p.x));
  };
  for (int it = threadIdx.x; it < W * (NG + 2); it += NT) {
    if (it < W * NG) {
      const int c = it / NG;
      const int k0 = 1 + (it - c * NG);
      const int g1 = group_of_base<N>(k0), g2 = group_of_base<N>(nR - k0);
      C z1[RL], z2[RL];
#pragma unroll
      for (int r = 0; r < RL; r++) z1[r] = t(g1 * RL + r, c);
      Dft<RL, false, C>::run(z1);
#pragma unroll
      for (int r = 0; r < RL; r++) z2[r] = t(g2 * RL + r, c);
      Dft<RL, false, C>::run(z2);
      // z1[r] = Z[k0 + r nR], z2[r] = Z[nR - k0 + r nR]; N - (k0 + r nR) is
      // the frequency of z2[RL-1-r].  The lower of each pair is k0 + r nR for
      // r < RL/2 and N - k0 - r nR above.
#pragma unroll
      for (int r = 0; r < RL; r++) {
        if (r < RL / 2) emit(c, k0 + r * nR, z1[r], z2[RL - 1 - r]);
        else emit(c, N - k0 - r * nR, z2[RL - 1 - r], z1[r]);
      }
    } else {
      const int q = it - W * NG;
      const int c = q >> 1;
      const int k0 = (q & 1) ? nR / 2 : 0;
      const int g = group_of_base<N>(k0);
      C z[RL];
#pragma unroll
      for (int r = 0; r < RL; r++) z[r] = t(g * RL + r, c);
      Dft<RL, false, C>::run(z);
      if (k0 == 0) {
        // frequencies r nR, N - r nR = (RL - r) nR: r = 0 .. RL/2
#pragma unroll
        for (int r = 0; r <= RL / 2; r++) emit(c, r * nR, z[r], z[(RL - r) % RL]);
      } else {
        // frequencies nR/2 + r nR, N - that = nR/2 + (RL-1-r) nR: r < RL/2
#pragma unroll
        for (int r = 0; r < RL / 2; r++) emit(c, nR / 2 + r * nR, z[r], z[RL - 1 - r]);
      }
    }
  }
}

// The fused last stage and split of the 512-point forward z pass (radix-8
// last stage, nR = 64 frequency bases): one group per thread, all threads
// busy.  A column's 64 groups fill two warps; lane l < 16 holds base
// k0 and lane l + 16 its partner 64 - k0 (warp 0: k0 = 1..16; warp 1:
// k0 = 17..31, and the self-paired bases 0 and 32 in lanes 15 and 31).  Each
// thread needs Z[N - k] for its four outputs k = k0 + r nR (r < 4), which are
// the partner's upper four values: one exchange of four complex values by
// warp shuffles.  The base-0 group pairs with itself shifted by one and
// writes five outputs (0 and N/2 among them).
template <int N, int NT, typename C>
__device__ __forceinline__ void z_split_stage_shfl(const LineTileZ<C> &t, C *out, int nhp, int W) {
  using T = typename Real<C>::type;
  constexpr int S = plan_stages(N);
  constexpr int RL = plan_radix(N, S - 1);
  constexpr int nR = N / RL;
  static_assert(RL == 8 && nR == 64, "the shuffle split is laid out for 64 bases of radix 8");
  const T h = (T)0.5;
  auto emit = [&](int c, int k, C p, C q) {   // p = Z[k], q = Z[N - k]
    out[(2 * c) * nhp + k] = mk(h * (p.x + q.x), h * (p.y - q.y));
    out[(2 * c + 1) * nhp + k] = mk(h * (p.y + q.y), h * (q.x - p.x));
  };
  // W * 64 items are whole warps, so every lane of a warp takes part in the
  // shuffles of an iteration
  for (int it = threadIdx.x; it < W * nR; it += NT) {
    const int c = it >> 6;
    const int u = it & 63;
    const int w = u >> 5, l = u & 31;
    int k0;
    if (l < 16) k0 = w == 0 ? l + 1 : (l < 15 ? 17 + l : 0);
    else k0 = w == 0 ? 63 - (l - 16) : (l < 31 ? 47 - (l - 16) : 32);
    const int g = group_of_base<N>(k0);
    C z[RL];
#pragma unroll
    for (int r = 0; r < RL; r++) z[r] = t(g * RL + r, c);
    Dft<RL, false, C>::run(z);
    // partner's upper half: lane l ^ 16, or the thread's own for the two
    // self-paired bases
    const bool self = (k0 & 31) == 0;
    const int src = self ? (int)(threadIdx.x & 31) : (int)((threadIdx.x & 31) ^ 16);
    C q[RL / 2];
#pragma unroll
    for (int i = 0; i < RL / 2; i++) {
      q[i].x = __shfl_sync(0xffffffffu, z[RL / 2 + i].x, src);
      q[i].y = __shfl_sync(0xffffffffu, z[RL / 2 + i].y, src);
    }
    if (k0 != 0) {
      // N - (k0 + r nR) is the partner's value RL-1-r = q[RL/2-1-r]
#pragma unroll
      for (int r = 0; r < RL / 2; r++) emit(c, k0 + r * nR, z[r], q[RL / 2 - 1 - r]);
    } else {
      // frequencies r nR pair with (RL - r) nR: r = 0 .. RL/2
#pragma unroll
      for (int r = 0; r <= RL / 2; r++) emit(c, r * nR, z[r], z[(RL - r) % RL]);
    }
  }
}

// The last DIF stage of a compile-time z inverse transform fused with the C2R
// output (ParisPencil.cpp:368-380): item (c, k0) transforms the group whose
// outputs are the points k0 + r nR and writes their real and imaginary parts
// to the two real lines of pair c in `raw` (rows of N values).  Consecutive
// threads take consecutive k0, so the stores are conflict free.
template <int N, int NT, typename C>
__device__ __forceinline__ void z_inv_last_stage(const LineTileZ<C> &t, typename Real<C>::type *raw, int W) {
  constexpr int S = plan_stages(N);
  constexpr int RL = plan_radix(N, S - 1);
  constexpr int nR = N / RL;
  static_assert(radix8_prefix(N), "fused last stage needs a radix-8 prefix");
  for (int it = threadIdx.x; it < W * nR; it += NT) {
    const int c = it / nR;
    const int k0 = it - c * nR;
    const int g = group_of_base<N>(k0);
    C z[RL];
#pragma unroll
    for (int r = 0; r < RL; r++) z[r] = t(g * RL + r, c);
    Dft<RL, true, C>::run(z);
#pragma unroll
    for (int r = 0; r < RL; r++) {
      raw[(2 * c) * N + k0 + r * nR] = z[r].x;
      raw[(2 * c + 1) * N + k0 + r * nR] = z[r].y;
    }
  }
}

// R2C along z (ParisPencil.cpp:152-165): the last stage writes Z in natural
// order into B; the split A[k] = (Z[k] + conj Z[n-k]) / 2,
// B[k] = (Z[k] - conj Z[n-k]) / (2i) goes out with consecutive threads on
// consecutive k.
template <typename T, int N, bool TMAIO, bool TMA_OUT = TMAIO, bool LASTFUSE = false, int NT = kZThreads>
__device__ __forceinline__ bool z_fwd_tile(const T *__restrict__ f, typename Cplx<T>::type *spec, const PassArgs<T> &a,
                                           int W, int P, long line0, long lend, typename Cplx<T>::type *sm,
                                           const ZTileIO &io) {
  using C = typename Cplx<T>::type;
  const int nk = N > 0 ? N : a.nk;
  const int nh = a.nh;
  // split/extension loops walk k over nh rounded up to whole 128-byte rows,
  // so each group of lanes that shares a shared-memory wavefront stays in one
  // row (nh = n/2 + 1 is odd; a plain k = it % nh mapping straddles rows)
  constexpr int RA = 128 / (int)sizeof(typename Cplx<T>::type);
  const int nha = N > 0 ? (N / 2 + 1 + RA - 1) / RA * RA : (nh + RA - 1) / RA * RA;
  const int Asz = max(W * P, 2 * W * a.nhp);
  C *A = sm;
  C *B = A + ((Asz * (int)sizeof(C) + 127) & ~127) / (int)sizeof(C);
  const int nl = (int)min((long)(2 * W), lend - line0);
  const AxisDev<C> &ax = a.ax[2];
  LineTile<C> tA{A, P}, tB{B, P};
  LineTileRev<C, typename RevLastOf<N>::type> tBrev{tB, rev_last<N>(ax)};
  if constexpr (TMAIO) {
    T *raw = reinterpret_cast<T *>(B);
    if (!bulk_in(raw, f + line0 * nk, (size_t)nl * nk * sizeof(T), io)) return false;
    auto ld0 = [&](int pos, int c) -> C {
      const int la = 2 * c;
      return mk(la < nl ? raw[la * nk + pos] : (T)0, la + 1 < nl ? raw[(la + 1) * nk + pos] : (T)0);
    };
    if constexpr (LASTFUSE && TMA_OUT && N > 0 && radix8_prefix(N) && z_split_fused(N, sizeof(C))) {
      // stages in A, the fused last stage stages the spectrum rows in B
      LineTileZ<C> tAz{A, P};
      dif_ct<N, plan_stages(N) - 1, 0, false, Map::PosFast, 1, NT, true, true>(ax, ld0, tAz, tAz, W);
      if constexpr (z_split_shfl(N, sizeof(C))) z_split_stage_shfl<N, NT>(tAz, B, a.nhp, W);
      else z_split_stage<N, NT>(tAz, B, a.nhp, W);
      fence_proxy_async_smem();
      __syncthreads();
      bulk_out(spec + line0 * a.nhp, B, (size_t)nl * a.nhp);
      return true;
    }
    dif_all<N, false, Map::PosFast, 1, NT, true, true>(ax, ld0, tA, tBrev, W);
    // split into the staging rows [line][kh] (pitch nhp) in A, then one copy out
    const T h = (T)0.5;
    for (int it = threadIdx.x; it < W * nha; it += NT) {
      const int k = it % nha;
      const int c = it / nha;
      if (k >= nh) continue;
      const C z = tB(k, c);
      const C w = tB(k == 0 ? 0 : nk - k, c);
      A[(2 * c) * a.nhp + k] = mk(h * (z.x + w.x), h * (z.y - w.y));
      A[(2 * c + 1) * a.nhp + k] = mk(h * (z.y + w.y), h * (w.x - z.x));
    }
    fence_proxy_async_smem();
    __syncthreads();
    bulk_out(spec + line0 * a.nhp, A, (size_t)nl * a.nhp);
    return true;
  } else {
    auto ldg = [&](int pos, int c) -> C {
      const long la = line0 + 2 * c;
      T x = 0, y = 0;
      if (la < lend) x = f[la * nk + pos];
      if (la + 1 < lend) y = f[(la + 1) * nk + pos];
      return mk(x, y);
    };
    dif_all<N, false, Map::PosFast, 1, NT, true, true>(ax, ldg, tA, tBrev, W);
    const T h = (T)0.5;
    if constexpr (TMA_OUT) {
      // staged rows [line][kh] (pitch nhp) in A, then one copy out
      for (int it = threadIdx.x; it < W * nha; it += NT) {
        const int k = it % nha;
        const int c = it / nha;
        if (k >= nh) continue;
        const C z = tB(k, c);
        const C w = tB(k == 0 ? 0 : nk - k, c);
        A[(2 * c) * a.nhp + k] = mk(h * (z.x + w.x), h * (z.y - w.y));
        A[(2 * c + 1) * a.nhp + k] = mk(h * (z.y + w.y), h * (w.x - z.x));
      }
      fence_proxy_async_smem();
      __syncthreads();
      bulk_out(spec + line0 * a.nhp, A, (size_t)nl * a.nhp);
    } else {
      for (int it = threadIdx.x; it < W * nha; it += NT) {
        const int k = it % nha;
        const int c = it / nha;
        if (k >= nh) continue;
        const long la = line0 + 2 * c;
        if (la >= lend) continue;
        const C z = tB(k, c);
        const C w = tB(k == 0 ? 0 : nk - k, c);
        spec[la * a.nhp + k] = mk(h * (z.x + w.x), h * (z.y - w.y));
        if (la + 1 < lend) spec[(la + 1) * a.nhp + k] = mk(h * (z.y + w.y), h * (w.x - z.x));
      }
    }
    return true;
  }
}

// C2R along z (ParisPencil.cpp:368-380): Z[k] = A[k] + i B[k] over the
// Hermitian extension in natural order in B (the imaginary parts of the zero
// and Nyquist terms are dropped, as a C2R transform does), inverse DIF into
// natural order in B, real and imaginary parts out to the two lines.
template <typename T, int N, bool TMAIO, bool LASTFUSE = false, int NT = kZThreads>
__device__ __forceinline__ bool z_inv_tile(const typename Cplx<T>::type *spec, T *__restrict__ out,
                                           const PassArgs<T> &a, int W, int P, long line0, long lend,
                                           typename Cplx<T>::type *sm, const ZTileIO &io) {
  using C = typename Cplx<T>::type;
  const int nk = N > 0 ? N : a.nk;
  const int nh = a.nh;
  // split/extension loops walk k over nh rounded up to whole 128-byte rows,
  // so each group of lanes that shares a shared-memory wavefront stays in one
  // row (nh = n/2 + 1 is odd; a plain k = it % nh mapping straddles rows)
  constexpr int RA = 128 / (int)sizeof(typename Cplx<T>::type);
  const int nha = N > 0 ? (N / 2 + 1 + RA - 1) / RA * RA : (nh + RA - 1) / RA * RA;
  const int Asz = max(W * P, 2 * W * a.nhp);
  C *A = sm;
  C *B = A + ((Asz * (int)sizeof(C) + 127) & ~127) / (int)sizeof(C);
  const int nl = (int)min((long)(2 * W), lend - line0);
  const AxisDev<C> &ax = a.ax[2];
  LineTile<C> tA{A, P}, tB{B, P};
  LineTileRev<C, typename RevLastOf<N>::type> tBrev{tB, rev_last<N>(ax)};
  auto hermitian = [&](int k, int c, C sa, C sb) {
    if (k == 0 || 2 * k == nk) {
      tB(k, c, mk(sa.x, sb.x));
    } else {
      tB(k, c, mk(sa.x - sb.y, sa.y + sb.x));
      tB(nk - k, c, mk(sa.x + sb.y, sb.x - sa.y));
    }
  };
  if constexpr (TMAIO) {
    if (!bulk_in(A, spec + line0 * a.nhp, (size_t)nl * a.nhp * sizeof(C), io)) return false;
    // The first stage reads Z straight from the spectrum rows in A, forming
    // the Hermitian extension on the fly (the same values hermitian() writes:
    // Z[k] = A[k] + i B[k] for k <= nk/2, conj A[nk-k] + i conj B[nk-k] above,
    // imaginary parts dropped at k = 0 and nk/2), and writes B; the stages
    // run in B and the last writes natural order into A, whose rows are no
    // longer needed after the first stage.
    auto ldh = [&](int pos, int c) -> C {
      const int la = 2 * c;
      const bool lo = 2 * pos <= nk;
      const int k = lo ? pos : nk - pos;
      const C sa = la < nl ? A[la * a.nhp + k] : mk((T)0, (T)0);
      const C sb = la + 1 < nl ? A[(la + 1) * a.nhp + k] : mk((T)0, (T)0);
      if (k == 0 || 2 * k == nk) return mk(sa.x, sb.x);
      return lo ? mk(sa.x - sb.y, sa.y + sb.x) : mk(sa.x + sb.y, sb.x - sa.y);
    };
    if constexpr (LASTFUSE && N > 0 && radix8_prefix(N)) {
      // stages in B, the fused last stage writes the real lines into A
      LineTileZ<C> tBz{B, P};
      dif_ct<N, plan_stages(N) - 1, 0, true, Map::PosFast, 1, NT, true, true>(ax, ldh, tBz, tBz, W);
      T *rawA = reinterpret_cast<T *>(A);
      z_inv_last_stage<N, NT>(tBz, rawA, W);
      fence_proxy_async_smem();
      __syncthreads();
      bulk_out(out + line0 * nk, rawA, (size_t)nl * nk);
      return true;
    }
    LineTileRev<C, typename RevLastOf<N>::type> tArev{tA, rev_last<N>(ax)};
    dif_all<N, true, Map::PosFast, 1, NT, true, true>(ax, ldh, tB, tArev, W);
    // real lines staged in B, then one copy out
    T *raw = reinterpret_cast<T *>(B);
    for (int it = threadIdx.x; it < W * nk; it += NT) {
      const int t = it % nk;
      const int c = it / nk;
      const C v = tA(t, c);
      raw[(2 * c) * nk + t] = v.x;
      raw[(2 * c + 1) * nk + t] = v.y;
    }
    fence_proxy_async_smem();
    __syncthreads();
    bulk_out(out + line0 * nk, raw, (size_t)nl * nk);
    return true;
  } else {
    for (int it = threadIdx.x; it < W * nha; it += NT) {
      const int k = it % nha;
      const int c = it / nha;
      if (k >= nh) continue;
      const long la = line0 + 2 * c;
      C sa = mk((T)0, (T)0), sb = mk((T)0, (T)0);
      if (la < lend) sa = __ldcg(spec + la * a.nhp + k);
      if (la + 1 < lend) sb = __ldcg(spec + (la + 1) * a.nhp + k);
      hermitian(k, c, sa, sb);
    }
    __syncthreads();
    dif_all<N, true, Map::PosFast, 1, NT, true, true>(ax, tB, tA, tBrev, W);
    for (int it = threadIdx.x; it < W * nk; it += NT) {
      const int t = it % nk;
      const int c = it / nk;
      const long la = line0 + 2 * c;
      const C v = tB(t, c);
      if (la < lend) out[la * nk + t] = v.x;
      if (la + 1 < lend) out[(la + 1) * nk + t] = v.y;
    }
    return true;
  }
}

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

// Parameters of the x pass's filter on one tile (plane j, columns kh0 ..
// kh0 + ncol - 1): d = -1/N / ((i2 + j2) + k2) with i2 = (min(kx, ni - kx)*ddi)^2,
// j2 = (min(j, nj - j)*ddj)^2 and k2 = (kh*ddk)^2, as ParisPencil.cpp:270-284
// forms them (summed in that order), and 0 at the zero mode.
struct XFilter {
  int ni, j, kh0, ncol;
  double j2, ddi, ddk, minvN;
};

// 1/x for x > 0 by two Newton-Raphson steps y <- y + y*(1 - x*y) from the
// hardware's approximate FP64 reciprocal (rcp.approx.ftz.f64; each step
// squares the relative error, so the seed's error of at most about 2^-20
// ends below double rounding).  The seed needs no conversions to and from
// FP32, which ran on the same narrow conversion pipe as the seed itself.
__device__ __forceinline__ double recip_pos(double x) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double e = fma(-x, y, 1.0);
  y = fma(y, e, y);
  e = fma(-x, y, 1.0);
  return fma(y, e, y);
}

// The last DIF stage of the x forward transform, the filter and the first
// DIT stage of the inverse on one register group of R positions base + r of
// an n-point tile.  Their frequencies are k0 + r*kstep with k0 = k0_of(base)
// (the last DIF stage's digit is the slowest digit of the frequency; kstep is
// n/R, or the full line's step when the tile is half of a longer line), so
// the filter needs one frequency lookup per group; the column's k2 is formed
// once per group.
template <int R, int W, int NT, int NC, typename C, typename LD, typename ST, typename K0>
__device__ __forceinline__ void x_filter_stage(int n_rt, LD &ld, ST &st, const XFilter &f, const K0 &k0_of,
                                               int kstep) {
  using T = typename Real<C>::type;
  const int n = NC ? NC : n_rt;
  const int step = kstep;
  // Tiles of 64-byte rows (1024-point lines): a quarter warp holds items b and
  // b + 1, whose rows 2b + r and 2b + 2 + r share banks, so odd items take
  // their two rows in the other order.  Their forward butterfly then gives the
  // same sum and the negated difference, the filter scales them by the same
  // factors, and the inverse butterfly hands back the two outputs swapped,
  // which the swapped stores put in place: bit-identical values.
  constexpr bool kSwap = R == 2 && W * sizeof(C) == 64;
  if constexpr (NC > 0 && std::is_same<C, float2>::value && W % 2 == 0 && PairAccess<LD>::value &&
                PairAccess<ST>::value) {
    // FP32, compile-time plan: two adjacent columns per item, loaded as one
    // 16-byte access; the columns are then finished (filter, inverse
    // butterfly, 8-byte stores) one after the other, which keeps the pair
    // within the register budget (both columns to the end spilled)
    constexpr int WP = W / 2;
    auto body2 = [&](int it) {
      const int c = 2 * (it % WP);
      const int b = it / WP;
      const int base = b * R;
      const int sw = kSwap ? b & 1 : 0;
      float2 u[R], v[R];
#pragma unroll
      for (int r = 0; r < R; r++) {
        const float4 q = ld.ld2(base + (r ^ sw), c);
        u[r] = make_float2(q.x, q.y);
        v[r] = make_float2(q.z, q.w);
      }
      Dft<R, false, float2>::run(u);
      Dft<R, false, float2>::run(v);
      const int k0 = k0_of(base);
      // one column after the other: filter, inverse butterfly, store
      auto finish = [&](float2 *x, int cc) {
        const int kh = f.kh0 + cc;
        const double kd = double(kh) * f.ddk;
        const double k2 = kd * kd;
        const bool live = cc < f.ncol;
#pragma unroll
        for (int r = 0; r < R; r++) {
          const int kx = k0 + r * step;
          const double id = double(min(kx, f.ni - kx)) * f.ddi;
          double d = recip_pos((id * id + f.j2) + k2) * f.minvN;
          if ((kx | f.j | kh) == 0) d = 0.0;
          if (live) x[r] = cscale(x[r], (float)d);
        }
        Dft<R, true, float2>::run(x);
#pragma unroll
        for (int r = 0; r < R; r++) st(base + (r ^ sw), cc, x[r]);
      };
      finish(u, c);
      finish(v, c + 1);
    };
    if constexpr ((WP * (NC / R)) % NT == 0) {
      constexpr int ITER = WP * (NC / R) / NT;
#pragma unroll
      for (int q = 0; q < ITER; q++) body2((int)threadIdx.x + q * NT);
    } else {
      for (int it = threadIdx.x; it < WP * (n / R); it += NT) body2(it);
    }
    return;
  }
  auto body = [&](int it) {
    const int c = it % W;
    const int base = (it / W) * R;
    const int sw = kSwap ? (it / W) & 1 : 0;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = ld(base + (r ^ sw), c);
    Dft<R, false, C>::run(v);
    const int kh = f.kh0 + c;
    const double kd = double(kh) * f.ddk;
    const double k2 = kd * kd;
    const int k0 = k0_of(base);
    const bool live = c < f.ncol;
#pragma unroll
    for (int r = 0; r < R; r++) {
      const int kx = k0 + r * step;
      const double id = double(min(kx, f.ni - kx)) * f.ddi;
      double d = recip_pos((id * id + f.j2) + k2) * f.minvN;
      if ((kx | f.j | kh) == 0) d = 0.0;
      if (live) v[r] = cscale(v[r], (T)d);
    }
    Dft<R, true, C>::run(v);
#pragma unroll
    for (int r = 0; r < R; r++) st(base + (r ^ sw), c, v[r]);
  };
  if constexpr (NC > 0 && (W * (NC / R)) % NT == 0) {
    constexpr int ITER = W * (NC / R) / NT;
#pragma unroll
    for (int q = 0; q < ITER; q++) body((int)threadIdx.x + q * NT);
  } else {
    for (int it = threadIdx.x; it < W * (n / R); it += NT) body(it);
  }
}

__device__ __forceinline__ unsigned char *align128(unsigned char *p) {
  return reinterpret_cast<unsigned char *>((reinterpret_cast<uintptr_t>(p) + 127) & ~uintptr_t(127));
}

// --------------------------------------------------------- strided tiles
// A strided tile is W consecutive kh columns (128-byte rows) of all n rows of
// one plane, held point-major: y tiles are (plane i, rows j), x tiles are
// (plane j, rows i).

// y transform of one tile; stage 0 reads through ld0 (the TMA-filled tile or
// HBM/L2 directly), the last stage stores from registers straight to HBM:
// frequency row j of the tile's columns goes to row_at(j)[0 .. ncol-1].
// Store of a strided pass's last stage: frequency row rl(pos) of the tile's
// columns goes to row_at(row)[c] for c < ncol; FP32 rows also take column
// pairs as one 16-byte store (rows start 16-byte aligned: the FP32 row pitch
// is even and tiles start at even columns).
template <typename C, typename RowAt, typename RL> struct RowStore {
  const RowAt &row_at;
  RL rl;
  int ncol;
  static constexpr bool kPair = std::is_same<C, float2>::value;
  __device__ __forceinline__ void operator()(int pos, int c, C v) const {
    if (c < ncol) row_at(rl(pos))[c] = v;
  }
  __device__ __forceinline__ void st2(int pos, int c, float4 q) const {
    C *p = row_at(rl(pos)) + c;
    if (c + 1 < ncol) *reinterpret_cast<float4 *>(p) = q;
    else if (c < ncol) *reinterpret_cast<float2 *>(p) = make_float2(q.x, q.y);
  }
};

template <typename T, int W, bool INV, int N, typename LD0, typename RowAt>
__device__ __forceinline__ void y_tile_rows(LD0 &ld0, const RowAt &row_at, const PassArgs<T> &a, int kt,
                                            typename Cplx<T>::type *sm) {
  using C = typename Cplx<T>::type;
  const AxisDev<C> &ax = a.ax[1];
  const int ncol = min(W, a.nh - kt * W);
  const auto rl = rev_last<N>(ax);
  PointTile<W, C> tile{sm};
  RowStore<C, RowAt, std::remove_const_t<decltype(rl)>> gst{row_at, rl, ncol};
  dif_all<N, INV, Map::ColFast, W, kZThreads, false, (sizeof(T) == 8)>(ax, ld0, tile, gst, W);
}

// y transform of one tile of plane o, stored into the spectrum dst at the
// same plane and columns.
template <typename T, int W, bool INV, int N, typename LD0>
__device__ __forceinline__ void y_tile(LD0 &ld0, typename Cplx<T>::type *dst, const PassArgs<T> &a, int o, int kt,
                                       typename Cplx<T>::type *sm) {
  using C = typename Cplx<T>::type;
  C *base = dst + (long)o * a.nj * a.nhp + kt * W;
  const int pitch = a.nhp;
  auto row_at = [base, pitch](int j) { return base + (long)j * pitch; };
  y_tile_rows<T, W, INV, N>(ld0, row_at, a, kt, sm);
}

// x transform of one tile in shared memory (plane j of the x pencils,
// columns kt*W ..): forward, filter, inverse.  The filter takes the global
// row jf of an njf-row grid (the plane itself on one GPU).  The last stage
// writes natural order through gst: back into the tile (gst = the tile) or
// straight to HBM.
template <typename T, int W, int N, typename GST>
__device__ __forceinline__ void x_tile_core(const PassArgs<T> &a, int jf, int njf, int kt,
                                            typename Cplx<T>::type *sm, GST &gst) {
  using C = typename Cplx<T>::type;
  constexpr int NT = kZThreads;
  // FP64: twiddle powers by recurrence (fewer table loads); FP32: table loads
  // (FP64-generated values), keeping the FP64 pipe for the filter
  constexpr bool TWX = sizeof(T) == 8;
  const AxisDev<C> &ax = a.ax[0];
  const int n = N > 0 ? N : ax.n;
  const int kh0 = kt * W;
  const int ncol = min(W, a.nh - kh0);
  PointTile<W, C> tile{sm};
  const double jd = double(min(jf, njf - jf)) * a.dd[1];
  const XFilter flt{a.ni, jf, kh0, ncol, jd * jd, a.dd[0], a.dd[2], -a.invN};
  if constexpr (N > 0) {
    constexpr int S = plan_stages(N);
    constexpr int RF = plan_radix(N, S - 1);
    auto k0_of = [](int base) { return rev_ct<N>(base); };
    if constexpr (S > 1) {
      dif_ct<N, S - 1, 0, false, Map::ColFast, W, NT, false, TWX>(ax, tile, tile, tile, W);
      x_filter_stage<RF, W, NT, N, C>(N, tile, tile, flt, k0_of, N / RF);
      __syncthreads();
      dit_ct<N, S - 2, true, Map::ColFast, W, NT, TWX>(ax, tile, gst, W);
    } else {
      x_filter_stage<RF, W, NT, N, C>(N, tile, gst, flt, k0_of, N / RF);
    }
  } else {
    const int S = ax.nstages;
    if (S > 1) dif_rt<false, Map::ColFast, W, NT, false, TWX>(ax, S - 1, tile, tile, tile, W);
    const int *rev = ax.rev;
    auto k0_of = [rev](int base) { return __ldg(rev + base); };
    with_radix(ax.radix[S - 1], [&](auto tag) {
      constexpr int R = decltype(tag)::value;
      if (S == 1) x_filter_stage<R, W, NT, 0, C>(n, tile, gst, flt, k0_of, n / R);
      else x_filter_stage<R, W, NT, 0, C>(n, tile, tile, flt, k0_of, n / R);
    });
    __syncthreads();
    if (S > 1) dit_rt<true, Map::ColFast, W, NT, TWX>(ax, S - 2, tile, gst, W);
  }
}

// x transform of one TMA-filled tile: forward, filter, inverse.  The inverse
// ends in natural order in place, so the finished tile leaves by TMA stores
// of the same boxes it came in with (columns past nh are clipped).
template <typename T, int W, int N>
__device__ __forceinline__ void x_tile(const CUtensorMap *tmap, const PassArgs<T> &a, int j, int kt, int box_rows,
                                       typename Cplx<T>::type *sm) {
  using C = typename Cplx<T>::type;
  const int n = N > 0 ? N : a.ax[0].n;
  PointTile<W, C> tile{sm};
  x_tile_core<T, W, N>(a, j, a.nj, kt, sm, tile);
  fence_proxy_async_smem();
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int q = 0; q < n / box_rows; q++) tma_store_3d(tmap, 2 * W * kt, j, q * box_rows, sm + q * box_rows * W);
    bulk_commit();
    bulk_wait_read();
  }
}

// Loads one strided tile with TMA into sm (boxes of box_rows rows) and waits
// on mb for phase `parity` with an iteration limit.  Returns false on every
// thread if the copy did not complete (the plan status word is set).  The
// caller's earlier shared-memory accesses of sm must be fenced
// (fence_proxy_async_smem) and barriered before the call.
template <typename C, int W, bool XPASS>
__device__ __forceinline__ bool tma_tile(const CUtensorMap *tmap, C *sm, uint64_t *mb, uint32_t parity, int n,
                                         int box_rows, int o, int kt, int *status, int wait_iters = 0) {
  if (threadIdx.x == 0) {
    mbar_expect_tx(mb, (uint32_t)(n * W * sizeof(C)));
    for (int q = 0; q < n / box_rows; q++) {
      if (XPASS) tma_load_3d(sm + q * box_rows * W, tmap, 2 * W * kt, o, q * box_rows, mb);
      else tma_load_3d(sm + q * box_rows * W, tmap, 2 * W * kt, q * box_rows, o, mb);
    }
  }
  const bool ok = mbar_wait_bounded(mb, parity, wait_iters);
  if (__syncthreads_or(!ok)) {
    // report, and give the copy in flight a bounded chance to land before the
    // block's shared memory is released
    if (threadIdx.x == 0) {
      atomicExch(status, kDevTmaTimeout);
      mbar_wait_bounded(mb, parity);
    }
    return false;
  }
  return true;
}


// Twiddle table tw[q] = exp(-2*pi*i*q/n), q < n, from FP64 sincospi.
template <typename C>
__global__ void k_twiddles(int n, C *tw) {
  for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(2.0 * (double)q / (double)n, &s, &c);   // exp(-2*pi*i*q/n) in FP64
    tw[q] = mk((decltype(tw[q].x))c, (decltype(tw[q].x))(-s));
  }
}

}  // namespace ff
