// Shared-memory batched FFT engine for sm_100a.
//
// A thread block owns a tile of W independent lines ("columns") of length n.
// The tile lives in shared memory point-major: element (pos, c) at
// sm[pos*W + c], so that one row of W complex values is exactly 128 bytes
// (W = 8 for FP64, 16 for FP32).  A warp always touches whole rows, which
// keeps every shared-memory access conflict-free for any stage stride.
//
// Transforms are in-place mixed-radix Cooley-Tukey:
//   * decimation in frequency (DIF): natural input, output at position pos
//     holds frequency rev[pos] (mixed-radix digit reversal);
//   * decimation in time (DIT): the transpose, digit-reversed input, natural
//     output.
// Stage s (radix R, span L) works on groups {blk*L + j + r*(L/R)}, r < R.
// The first stage may read straight from global memory and the last stage may
// write straight to global memory (loader / storer functors), so a pass moves
// each element between HBM and the SM once.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace ff {

constexpr int kMaxStages = 16;
constexpr int kThreads = 256;

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

// Columns per tile: one 128-byte shared-memory row.
template <typename T> struct TileW { static constexpr int value = 128 / (2 * sizeof(T)); };

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { return mk(a.x * s, a.y * s); }
// a*b
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a*conj(b)
template <typename C> __device__ __forceinline__ C cmulc(C a, C b) {
  return mk(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// -i*a and +i*a
template <typename C> __device__ __forceinline__ C mul_mi(C a) { return mk(a.y, -a.x); }
template <typename C> __device__ __forceinline__ C mul_pi(C a) { return mk(-a.y, a.x); }
// multiply by -i (forward) or +i (inverse)
template <bool INV, typename C> __device__ __forceinline__ C mul_wi(C a) { return INV ? mul_pi(a) : mul_mi(a); }

template <typename C> struct Real;
template <> struct Real<double2> { using type = double; };
template <> struct Real<float2> { using type = float; };

// Constants from their closed forms: sqrt(1/2); sqrt(3)/2; cos and sin of
// 2*pi/5 and 4*pi/5.
#define FF_SQRT1_2 0.70710678118654752440084436210484903928
#define FF_SQRT3_2 0.86602540378443864676372317075293618347
#define FF_C5_1 0.30901699437494742410229341718281905886
#define FF_C5_2 (-0.80901699437494742410229341718281905886)
#define FF_S5_1 0.95105651629515357211643933337938214340
#define FF_S5_2 0.58778525229247312916870595463907276860

// In-register R-point DFT, y_s = sum_r v_r exp(-+2*pi*i*r*s/R), unnormalised.
template <int R, bool INV, typename C> struct Dft;

template <bool INV, typename C> struct Dft<1, INV, C> {
  static __device__ __forceinline__ void run(C *) {}
};

template <bool INV, typename C> struct Dft<2, INV, C> {
  static __device__ __forceinline__ void run(C *v) {
    const C a = v[0], b = v[1];
    v[0] = cadd(a, b);
    v[1] = csub(a, b);
  }
};

template <bool INV, typename C> struct Dft<3, INV, C> {
  static __device__ __forceinline__ void run(C *v) {
    using T = typename Real<C>::type;
    const C t = cadd(v[1], v[2]);
    const C u = cscale(csub(v[1], v[2]), (T)FF_SQRT3_2);
    const C m = csub(v[0], cscale(t, (T)0.5));
    v[0] = cadd(v[0], t);
    const C iu = mul_wi<INV>(u);   // -i*u forward
    v[1] = cadd(m, iu);
    v[2] = csub(m, iu);
  }
};

template <bool INV, typename C> struct Dft<4, INV, C> {
  static __device__ __forceinline__ void run(C *v) {
    const C t0 = cadd(v[0], v[2]), t1 = csub(v[0], v[2]);
    const C t2 = cadd(v[1], v[3]), t3 = mul_wi<INV>(csub(v[1], v[3]));
    v[0] = cadd(t0, t2);
    v[2] = csub(t0, t2);
    v[1] = cadd(t1, t3);
    v[3] = csub(t1, t3);
  }
};

template <bool INV, typename C> struct Dft<5, INV, C> {
  static __device__ __forceinline__ void run(C *v) {
    using T = typename Real<C>::type;
    const C t1 = cadd(v[1], v[4]), t2 = cadd(v[2], v[3]);
    const C t3 = csub(v[1], v[4]), t4 = csub(v[2], v[3]);
    const C a0 = v[0];
    const C b1 = mk(a0.x + (T)FF_C5_1 * t1.x + (T)FF_C5_2 * t2.x, a0.y + (T)FF_C5_1 * t1.y + (T)FF_C5_2 * t2.y);
    const C b2 = mk(a0.x + (T)FF_C5_2 * t1.x + (T)FF_C5_1 * t2.x, a0.y + (T)FF_C5_2 * t1.y + (T)FF_C5_1 * t2.y);
    const C d1 = mk((T)FF_S5_1 * t3.x + (T)FF_S5_2 * t4.x, (T)FF_S5_1 * t3.y + (T)FF_S5_2 * t4.y);
    const C d2 = mk((T)FF_S5_2 * t3.x - (T)FF_S5_1 * t4.x, (T)FF_S5_2 * t3.y - (T)FF_S5_1 * t4.y);
    v[0] = cadd(a0, cadd(t1, t2));
    const C e1 = mul_wi<INV>(d1), e2 = mul_wi<INV>(d2);   // -i*d forward
    v[1] = cadd(b1, e1);
    v[4] = csub(b1, e1);
    v[2] = cadd(b2, e2);
    v[3] = csub(b2, e2);
  }
};

template <bool INV, typename C> struct Dft<8, INV, C> {
  static __device__ __forceinline__ void run(C *v) {
    using T = typename Real<C>::type;
    // even/odd split into two 4-point DFTs, then w8^s combination
    C e[4] = {v[0], v[2], v[4], v[6]};
    C o[4] = {v[1], v[3], v[5], v[7]};
    Dft<4, INV, C>::run(e);
    Dft<4, INV, C>::run(o);
    const T h = (T)FF_SQRT1_2;
    // w8^1, w8^2, w8^3 with w8 = exp(-i*pi/4) forward, conj inverse
    C o1, o2, o3;
    if (!INV) {
      o1 = mk((o[1].x + o[1].y) * h, (o[1].y - o[1].x) * h);
      o2 = mul_mi(o[2]);
      o3 = mk((o[3].y - o[3].x) * h, -(o[3].x + o[3].y) * h);
    } else {
      o1 = mk((o[1].x - o[1].y) * h, (o[1].x + o[1].y) * h);
      o2 = mul_pi(o[2]);
      o3 = mk(-(o[3].x + o[3].y) * h, (o[3].x - o[3].y) * h);
    }
    v[0] = cadd(e[0], o[0]);
    v[4] = csub(e[0], o[0]);
    v[1] = cadd(e[1], o1);
    v[5] = csub(e[1], o1);
    v[2] = cadd(e[2], o2);
    v[6] = csub(e[2], o2);
    v[3] = cadd(e[3], o3);
    v[7] = csub(e[3], o3);
  }
};

// One axis of a plan as the kernels see it.
template <typename C> struct AxisDev {
  int n;
  int nstages;
  int radix[kMaxStages];   // DIF order: stage 0 spans the whole line
  const C *tw;             // tw[q] = exp(-2*pi*i*q/n), q < n (FP64-generated)
  const int *rev;          // DIF output position -> frequency index
  const int *ipos;         // frequency index -> DIF output position
};

template <bool INV, typename C> __device__ __forceinline__ C twmul(C v, const C *__restrict__ tw, int q) {
  const C w = __ldg(tw + q);
  return INV ? cmulc(v, w) : cmul(v, w);
}

// One stage over all (group, column) items of the tile.
//   DIT = false: DFT then output twiddles (DIF);  DIT = true: input twiddles then DFT.
//   ld(pos, c) -> C,  st(pos, c, C).
template <int R, bool INV, bool DIT, int W, typename C, typename LD, typename ST>
__device__ __forceinline__ void run_stage(int n, int L, const C *__restrict__ tw, LD &ld, ST &st) {
  const int m = L / R;
  const int twstep = n / L;
  const int items = W * (n / R);
  for (int it = threadIdx.x; it < items; it += blockDim.x) {
    const int c = it % W;
    const int b = it / W;
    const int blk = b / m;
    const int j = b - blk * m;
    const int base = blk * L + j;
    C v[R];
#pragma unroll
    for (int r = 0; r < R; r++) v[r] = ld(base + r * m, c);
    if (DIT) {
      if (j != 0) {
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = twmul<INV>(v[r], tw, j * r * twstep);
      }
      Dft<R, INV, C>::run(v);
    } else {
      Dft<R, INV, C>::run(v);
      if (j != 0) {
#pragma unroll
        for (int r = 1; r < R; r++) v[r] = twmul<INV>(v[r], tw, j * r * twstep);
      }
    }
#pragma unroll
    for (int r = 0; r < R; r++) st(base + r * m, c, v[r]);
  }
}

// Calls f(RadixTag<R>) for the runtime radix r.
template <int R> struct RadixTag { static constexpr int value = R; };
template <typename F> __device__ __forceinline__ void with_radix(int r, F &&f) {
  switch (r) {
    case 8: f(RadixTag<8>{}); break;
    case 4: f(RadixTag<4>{}); break;
    case 2: f(RadixTag<2>{}); break;
    case 5: f(RadixTag<5>{}); break;
    case 3: f(RadixTag<3>{}); break;
    default: f(RadixTag<1>{}); break;
  }
}

// Shared-memory accessors of the point-major tile.
template <int W, typename C> struct SmemLd {
  const C *sm;
  __device__ __forceinline__ C operator()(int pos, int c) const { return sm[pos * W + c]; }
};
template <int W, typename C> struct SmemSt {
  C *sm;
  __device__ __forceinline__ void operator()(int pos, int c, C v) const { sm[pos * W + c] = v; }
};

// Full DIF transform of the tile: stage 0 reads through ldg, the last stage
// writes through stg, the stages in between work in shared memory.  Ends with
// a block barrier.
template <bool INV, int W, typename C, typename LDG, typename STG>
__device__ __forceinline__ void dif_transform(const AxisDev<C> &ax, C *sm, LDG &ldg, STG &stg) {
  SmemLd<W, C> sld{sm};
  SmemSt<W, C> sst{sm};
  int L = ax.n;
  for (int s = 0; s < ax.nstages; s++) {
    const bool first = s == 0, last = s == ax.nstages - 1;
    with_radix(ax.radix[s], [&](auto tag) {
      constexpr int R = decltype(tag)::value;
      if (first && last) run_stage<R, INV, false, W>(ax.n, L, ax.tw, ldg, stg);
      else if (first) run_stage<R, INV, false, W>(ax.n, L, ax.tw, ldg, sst);
      else if (last) run_stage<R, INV, false, W>(ax.n, L, ax.tw, sld, stg);
      else run_stage<R, INV, false, W>(ax.n, L, ax.tw, sld, sst);
    });
    L /= ax.radix[s];
    __syncthreads();
  }
}

// DIT stages nstages-1 .. s_end (inclusive) on a digit-reversed tile already in
// shared memory; stage 0 (if s_end == 0) writes through stg.  Ends with a barrier.
template <bool INV, int W, typename C, typename STG>
__device__ __forceinline__ void dit_stages(const AxisDev<C> &ax, C *sm, int s_begin, STG &stg) {
  SmemLd<W, C> sld{sm};
  SmemSt<W, C> sst{sm};
  // span of stage s is n / (r_0 ... r_{s-1})
  for (int s = s_begin; s >= 0; s--) {
    int L = ax.n;
    for (int q = 0; q < s; q++) L /= ax.radix[q];
    with_radix(ax.radix[s], [&](auto tag) {
      constexpr int R = decltype(tag)::value;
      if (s == 0) run_stage<R, INV, true, W>(ax.n, L, ax.tw, sld, stg);
      else run_stage<R, INV, true, W>(ax.n, L, ax.tw, sld, sst);
    });
    __syncthreads();
  }
}

}  // namespace ff
