// Shared-memory batched FFT engine for sm_100a.
//
// A thread block transforms a tile of W independent lines ("columns") of
// length n held in shared memory.  Two tile layouts are used:
//   * point-major  sm[pos*W + c]: one row of W complex values is 128 bytes
//     (W = 8 FP64 / 16 FP32); threads take columns fastest, so a warp always
//     touches whole rows and every access is bank-conflict free.  Used by the
//     strided passes (y and x), whose global rows are W contiguous columns.
//   * line-major   sm[c*P + swz(pos)]: each line contiguous (pitch P), with an
//     XOR swizzle of the element inside every 128-byte row so power-of-two
//     strides are conflict free.  Used by the z passes, whose global lines
//     are contiguous; threads take positions fastest.
//
// Transforms are in-place mixed-radix Cooley-Tukey:
//   * decimation in frequency (DIF): natural input, output at position pos
//     holds frequency rev[pos] (mixed-radix digit reversal);
//   * decimation in time (DIT): the transpose, digit-reversed input, natural
//     output.
// Stage s (radix R, span L) works on groups {blk*L + j + r*(L/R)}, r < R.
// Loads and stores of a stage go through accessor functors, so the first
// stage can read global memory (or another buffer) and the last can write
// global memory (or another buffer) directly.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

namespace ff {

constexpr int kMaxStages = 16;

template <typename T> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };

__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }
__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C, typename S> __device__ __forceinline__ C cscale(C a, S s) { return mk(a.x * s, a.y * s); }
// FP32 complex values as packed pairs: one sm_100 two-wide instruction for
// both components (a - b as the fused a + (-1)*b, exact like the plain
// subtraction).  Each component rounds as the scalar operation does.
template <> __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
template <> __device__ __forceinline__ float2 csub(float2 a, float2 b) {
  return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);
}
template <> __device__ __forceinline__ float2 cscale(float2 a, float s) { return __fmul2_rn(a, make_float2(s, s)); }
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
// cos and sin of 2*pi*k/7, k = 1, 2, 3
#define FF_C7_1 0.62348980185873353052500488400423981063
#define FF_C7_2 (-0.22252093395631440428890256449679475947)
#define FF_C7_3 (-0.90096886790241912623610231950744505117)
#define FF_S7_1 0.78183148246802980870844452667405775023
#define FF_S7_2 0.97492791218182360701813168299393121723
#define FF_S7_3 0.43388373911755812047576833284835875461

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

// 7 points: with t_k = v_k + v_{7-k} and u_k = v_k - v_{7-k} (k = 1..3),
// y_m = v_0 + sum_k cos(2*pi*k*m/7) t_k -+ i sum_k sin(2*pi*k*m/7) u_k and
// y_{7-m} the same with the sign of the sine sum flipped (m = 1..3).
template <bool INV, typename C> struct Dft<7, INV, C> {
  static __device__ __forceinline__ void run(C *v) {
    using T = typename Real<C>::type;
    const C t1 = cadd(v[1], v[6]), t2 = cadd(v[2], v[5]), t3 = cadd(v[3], v[4]);
    const C u1 = csub(v[1], v[6]), u2 = csub(v[2], v[5]), u3 = csub(v[3], v[4]);
    const C a0 = v[0];
    const T c1 = (T)FF_C7_1, c2 = (T)FF_C7_2, c3 = (T)FF_C7_3;
    const T s1 = (T)FF_S7_1, s2 = (T)FF_S7_2, s3 = (T)FF_S7_3;
    // cosine sums (k*m mod 7 folded to 1..3)
    const C b1 = mk(a0.x + c1 * t1.x + c2 * t2.x + c3 * t3.x, a0.y + c1 * t1.y + c2 * t2.y + c3 * t3.y);
    const C b2 = mk(a0.x + c2 * t1.x + c3 * t2.x + c1 * t3.x, a0.y + c2 * t1.y + c3 * t2.y + c1 * t3.y);
    const C b3 = mk(a0.x + c3 * t1.x + c1 * t2.x + c2 * t3.x, a0.y + c3 * t1.y + c1 * t2.y + c2 * t3.y);
    // sine sums: sin(2*pi*j/7) = -sin(2*pi*(7-j)/7) for j > 3
    const C d1 = mk(s1 * u1.x + s2 * u2.x + s3 * u3.x, s1 * u1.y + s2 * u2.y + s3 * u3.y);
    const C d2 = mk(s2 * u1.x - s3 * u2.x - s1 * u3.x, s2 * u1.y - s3 * u2.y - s1 * u3.y);
    const C d3 = mk(s3 * u1.x - s1 * u2.x + s2 * u3.x, s3 * u1.y - s1 * u2.y + s2 * u3.y);
    v[0] = cadd(a0, cadd(t1, cadd(t2, t3)));
    const C e1 = mul_wi<INV>(d1), e2 = mul_wi<INV>(d2), e3 = mul_wi<INV>(d3);   // -i*d forward
    v[1] = cadd(b1, e1);
    v[6] = csub(b1, e1);
    v[2] = cadd(b2, e2);
    v[5] = csub(b2, e2);
    v[3] = cadd(b3, e3);
    v[4] = csub(b3, e3);
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

// ------------------------------------------------------------ radix plan
// Radix order of a DIF transform of length n = 2^a 3^b 5^c 7^d: radix 8
// while three factors of 2 remain, then one 4 or 2, then the 5s, the 3s and
// the 7s; a length of 1 is one stage of radix 1.  Shared by host planning and
// device code, so compile-time specialised kernels and plan tables agree.
__host__ __device__ constexpr int plan_radix(int n, int s) {
  int twos = 0, fives = 0, threes = 0, sevens = 0, m = n;
  while (m > 1 && m % 2 == 0) { m /= 2; twos++; }
  while (m > 1 && m % 5 == 0) { m /= 5; fives++; }
  while (m > 1 && m % 3 == 0) { m /= 3; threes++; }
  while (m > 1 && m % 7 == 0) { m /= 7; sevens++; }
  const int eights = twos / 3, rest = twos % 3;
  if (s < eights) return 8;
  s -= eights;
  if (rest) {
    if (s == 0) return rest == 2 ? 4 : 2;
    s -= 1;
  }
  if (s < fives) return 5;
  s -= fives;
  if (s < threes) return 3;
  s -= threes;
  if (s < sevens) return 7;
  return 1;
}
__host__ __device__ constexpr int plan_stages(int n) {
  int s = 0;
  for (int q = 0, L = n; L > 1; q++) {
    const int r = plan_radix(n, q);
    if (r == 1) break;   // n is not 2^a 3^b 5^c 7^d
    L /= r;
    s++;
  }
  return s > 0 ? s : 1;
}
// Span (sub-transform length) of stage s.
__host__ __device__ constexpr int plan_span(int n, int s) {
  int L = n;
  for (int q = 0; q < s; q++) L /= plan_radix(n, q);
  return L;
}

// One axis of a plan as the kernels see it.
template <typename C> struct AxisDev {
  int n;
  int nstages;
  int radix[kMaxStages];   // DIF order: stage 0 spans the whole line
  const C *tw;             // tw[q] = exp(-2*pi*i*q/n), q < n (FP64-generated, in C's precision)
  const double2 *tw64;     // the same table in FP64
  const int *rev;          // DIF output position -> frequency index
  const int *ipos;         // frequency index -> DIF output position
};

__device__ __forceinline__ double2 to_c(double2 w, double2 *) { return w; }
__device__ __forceinline__ float2 to_c(double2 w, float2 *) { return make_float2((float)w.x, (float)w.y); }

template <bool INV, typename C> __device__ __forceinline__ C twmul(C v, const C *__restrict__ tw, int q) {
  const C w = __ldg(tw + q);
  return INV ? cmulc(v, w) : cmul(v, w);
}

// v[r] *= w^(+-j*r) for r = 1..R-1 with w = exp(-2*pi*i*twstep/n).
//   TWREC = false: one table load per factor (the loads are shared by the
//                  threads of a warp that hold the same j);
//   TWREC = true:  one FP64 table load, the powers by FP64 complex products
//                  (for thread orders in which every lane has its own j).
template <int R, bool INV, bool TWREC, typename C>
__device__ __forceinline__ void apply_twiddles(C *v, int j, int twstep, const C *__restrict__ tw,
                                               const double2 *__restrict__ tw64) {
  if (TWREC) {
    double2 w1 = __ldg(tw64 + j * twstep);
    if (INV) w1.y = -w1.y;
    double2 w = w1;
#pragma unroll
    for (int r = 1; r < R; r++) {
      v[r] = cmul(v[r], to_c(w, (C *)nullptr));
      if (r + 1 < R) w = cmul(w, w1);
    }
  } else {
#pragma unroll
    for (int r = 1; r < R; r++) v[r] = twmul<INV>(v[r], tw, j * r * twstep);
  }
}

// Thread-to-item order of a stage: columns fastest (point-major tiles) or
// butterflies fastest (line-major tiles).
enum class Map { ColFast, PosFast };

// One stage over all (group, column) items of the tile.
//   DIT = false: DFT then output twiddles (DIF);  DIT = true: input twiddles then DFT.
//   ld(pos, c) -> C,  st(pos, c, C).
//   ncols: columns in the tile (must be W for Map::ColFast).
//   NC, LC > 0: compile-time length and span (NC = 0: use n_rt, L_rt);
//   NT > 0: compile-time block size; with NC it fully unrolls the item loop.
//   TWMUL: the twiddle table is TWMUL times longer than n (a sub-transform of
//   a longer line uses that line's table).
// Quotient and remainder by a divisor fixed for a whole stage, from its
// correctly rounded FP32 reciprocal and one correction step: exact for
// 0 <= x < 2^20 (the item indices of a tile), where the FP32 quotient is off
// by less than one.  Compile-time divisors use plain division (the compiler
// turns it into multiplies).
struct StageDiv {
  int d;
  float inv;
  __device__ __forceinline__ explicit StageDiv(int dd) : d(dd), inv(1.0f / (float)dd) {}
  __device__ __forceinline__ int quot(int x, int &rem) const {
    int q = __float2int_rz((float)x * inv);
    int r = x - q * d;
    if (r < 0) { q--; r += d; }
    else if (r >= d) { q++; r -= d; }
    rem = r;
    return q;
  }
};

// Accessors that can move two adjacent FP32 columns (c, c+1 with c even) as
// one 16-byte access declare kPair = true and provide ld2/st2.
template <typename F, typename = void> struct PairAccess : std::false_type {};
template <typename F>
struct PairAccess<F, std::void_t<decltype(F::kPair)>> : std::integral_constant<bool, F::kPair> {};

// A point-major FP32 stage with two adjacent columns per item: the pair moves
// as one 16-byte shared-memory access, and the row group's twiddles are loaded
// (or generated) once for both columns.  Same arithmetic per value as stage().
template <int R, bool INV, bool DIT, int W, int NT, int NC, int LC, bool TWREC, int TWMUL, typename LD, typename ST>
__device__ __forceinline__ void stage_pairs(int n_rt, int L_rt, const AxisDev<float2> &ax, LD &ld, ST &st) {
  constexpr int WP = W / 2;
  const int n = NC ? NC : n_rt;
  const int L = NC ? LC : L_rt;
  const int m = L / R;
  const int twstep = TWMUL * n / L;
  const int nb = n / R;
  const StageDiv dm(NC ? 1 : m);
  const bool has_tw = R > 1 && (NC > 0 ? (LC > R) : (L > R));
  // the last DIF stage of radix 2 on 64-byte rows: odd items read their rows
  // swapped (see stage())
  constexpr bool kSwap = R == 2 && !DIT && W * sizeof(float2) == 64;
  auto body = [&](int it) {
    const int c = 2 * (it % WP);
    const int b = it / WP;
    const int sw = kSwap && m == 1 ? b & 1 : 0;
    int blk, j;
    if (NC) {
      blk = b / m;
      j = b - blk * m;
    } else {
      blk = dm.quot(b, j);
    }
    const int base = blk * L + j;
    float2 w[R > 1 ? R - 1 : 1];
    if constexpr (R > 1) {
      if (has_tw) {
        if constexpr (TWREC) {
          double2 w1 = __ldg(ax.tw64 + j * twstep);
          if (INV) w1.y = -w1.y;
          double2 ww = w1;
#pragma unroll
          for (int r = 1; r < R; r++) {
            w[r - 1] = to_c(ww, (float2 *)nullptr);
            if (r + 1 < R) ww = cmul(ww, w1);
          }
        } else {
#pragma unroll
          for (int r = 1; r < R; r++) {
            w[r - 1] = __ldg(ax.tw + j * r * twstep);
            if (INV) w[r - 1].y = -w[r - 1].y;
          }
        }
      }
    }
    float2 u[R], v[R];
#pragma unroll
    for (int r = 0; r < R; r++) {
      const float4 q = ld.ld2(base + (r ^ sw) * m, c);
      u[r] = make_float2(q.x, q.y);
      v[r] = make_float2(q.z, q.w);
    }
    auto apply = [&](float2 *x) {
#pragma unroll
      for (int r = 1; r < R; r++) x[r] = cmul(x[r], w[r - 1]);
    };
    if (DIT) {
      if (has_tw) {
        apply(u);
        apply(v);
      }
      Dft<R, INV, float2>::run(u);
      Dft<R, INV, float2>::run(v);
    } else {
      Dft<R, INV, float2>::run(u);
      Dft<R, INV, float2>::run(v);
      if (has_tw) {
        apply(u);
        apply(v);
      }
      if (sw) {
        u[R - 1] = make_float2(-u[R - 1].x, -u[R - 1].y);
        v[R - 1] = make_float2(-v[R - 1].x, -v[R - 1].y);
      }
    }
#pragma unroll
    for (int r = 0; r < R; r++) st.st2(base + r * m, c, make_float4(u[r].x, u[r].y, v[r].x, v[r].y));
  };
  if constexpr (NC > 0 && NT > 0 && (WP * (NC / R)) % NT == 0) {
    constexpr int ITER = WP * (NC / R) / NT;
#pragma unroll
    for (int q = 0; q < ITER; q++) body((int)threadIdx.x + q * NT);
  } else {
    const int step = NT > 0 ? NT : (int)blockDim.x;
    for (int it = threadIdx.x; it < WP * nb; it += step) body(it);
  }
}

template <int R, bool INV, bool DIT, Map MAP, int W, int NT, int NC, int LC, bool TWREC, int TWMUL = 1, typename C,
          typename LD, typename ST>
__device__ __forceinline__ void stage(int n_rt, int L_rt, const AxisDev<C> &ax, LD &ld, ST &st, int ncols) {
  // compile-time plans only: a runtime plan instantiates every radix, and the
  // paired registers of all of them spilled
  if constexpr (NC > 0 && std::is_same<C, float2>::value && MAP == Map::ColFast && W % 2 == 0 &&
                PairAccess<LD>::value && PairAccess<ST>::value) {
    stage_pairs<R, INV, DIT, W, NT, NC, LC, TWREC, TWMUL>(n_rt, L_rt, ax, ld, st);
    return;
  }
  const int n = NC ? NC : n_rt;
  const int L = NC ? LC : L_rt;
  const int m = L / R;
  const int twstep = TWMUL * n / L;
  const int nb = n / R;
  // runtime divisors by reciprocal, except on FP64 line-major tiles (their
  // registers are the tightest; measured slower there)
  constexpr bool kRcpDiv = NC == 0 && !(MAP == Map::PosFast && sizeof(C) == 16);
  const StageDiv dm(kRcpDiv ? m : 1), dnb(kRcpDiv ? nb : 1);
  auto body = [&](int it) {
    int c, b;
    if (MAP == Map::ColFast) {
      c = it % W;
      b = it / W;
    } else if (!kRcpDiv) {
      b = it % nb;
      c = it / nb;
    } else {
      c = dnb.quot(it, b);
    }
    int blk, j;
    if (!kRcpDiv) {
      blk = b / m;
      j = b - blk * m;
    } else {
      blk = dm.quot(b, j);
    }
    const int base = blk * L + j;
    C v[R];
    // Stage with twiddles: the factors are fetched before the data loads and
    // applied without a branch (j = 0 reads exp(0) = 1), so their latency
    // overlaps the data loads.  Not for FP64 line-major tiles, where the
    // extra live registers spill.
    constexpr bool kPrefetch = !(MAP == Map::PosFast && sizeof(C) == 16);
    // runtime plans take the same path in every stage that has twiddles
    // (span above the radix); the branch is uniform across the block
    bool pf = false;
    if constexpr (R > 1 && kPrefetch) pf = NC > 0 ? (LC > R) : (L > R);
    if constexpr (R > 1 && kPrefetch) if (pf) {
      if constexpr (TWREC) {
        double2 w1 = __ldg(ax.tw64 + j * twstep);
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = ld(base + r * m, c);
        if (INV) w1.y = -w1.y;
        auto apply = [&] {
          double2 w = w1;
#pragma unroll
          for (int r = 1; r < R; r++) {
            v[r] = cmul(v[r], to_c(w, (C *)nullptr));
            if (r + 1 < R) w = cmul(w, w1);
          }
        };
        if (DIT) { apply(); Dft<R, INV, C>::run(v); }
        else { Dft<R, INV, C>::run(v); apply(); }
      } else {
        C w[R - 1];
#pragma unroll
        for (int r = 1; r < R; r++) w[r - 1] = __ldg(ax.tw + j * r * twstep);
#pragma unroll
        for (int r = 0; r < R; r++) v[r] = ld(base + r * m, c);
        auto apply = [&] {
#pragma unroll
          for (int r = 1; r < R; r++) v[r] = INV ? cmulc(v[r], w[r - 1]) : cmul(v[r], w[r - 1]);
        };
        if (DIT) { apply(); Dft<R, INV, C>::run(v); }
        else { Dft<R, INV, C>::run(v); apply(); }
      }
#pragma unroll
      for (int r = 0; r < R; r++) st(base + r * m, c, v[r]);
      return;
    }
    {
      // The last DIF stage of radix 2 on a point-major tile of 64-byte rows
      // (1024-point lines): a quarter warp holds items b and b + 1, whose rows
      // 2b + r and 2b + 2 + r share banks, so odd items read their two rows
      // in the other order; the butterfly then gives the same sum and the
      // negated difference, which is negated back (exact).
      constexpr bool kSwap = R == 2 && !DIT && MAP == Map::ColFast && W * sizeof(C) == 64;
      const int sw = kSwap && m == 1 ? b & 1 : 0;
#pragma unroll
      for (int r = 0; r < R; r++) v[r] = ld(base + (r ^ sw) * m, c);
      if (DIT) {
        if (j != 0) apply_twiddles<R, INV, TWREC>(v, j, twstep, ax.tw, ax.tw64);
        Dft<R, INV, C>::run(v);
      } else {
        Dft<R, INV, C>::run(v);
        if (j != 0) apply_twiddles<R, INV, TWREC>(v, j, twstep, ax.tw, ax.tw64);
        if (sw) v[R - 1] = mk(-v[R - 1].x, -v[R - 1].y);
      }
#pragma unroll
      for (int r = 0; r < R; r++) st(base + r * m, c, v[r]);
    }
  };
  if constexpr (NC > 0 && NT > 0 && MAP == Map::ColFast && (W * (NC / R)) % NT == 0) {
    constexpr int ITER = W * (NC / R) / NT;
#pragma unroll
    for (int q = 0; q < ITER; q++) body((int)threadIdx.x + q * NT);
  } else {
    const int items = ncols * nb;
    const int step = NT > 0 ? NT : (int)blockDim.x;
    for (int it = threadIdx.x; it < items; it += step) body(it);
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
    case 7: f(RadixTag<7>{}); break;
    default: f(RadixTag<1>{}); break;
  }
}

// ------------------------------------------------------------ accessors
// Point-major tile: element (pos, c) at sm[pos*W + c].
template <int W, typename C> struct PointTile {
  C *sm;
  // columns c, c+1 (c even) of an FP32 tile as one 16-byte access (rows are
  // 16-byte multiples and the tile 128-byte aligned)
  static constexpr bool kPair = std::is_same<C, float2>::value && W % 2 == 0;
  __device__ __forceinline__ C operator()(int pos, int c) const { return sm[pos * W + c]; }
  __device__ __forceinline__ void operator()(int pos, int c, C v) const { sm[pos * W + c] = v; }
  __device__ __forceinline__ float4 ld2(int pos, int c) const {
    return *reinterpret_cast<const float4 *>(sm + pos * W + c);
  }
  __device__ __forceinline__ void st2(int pos, int c, float4 q) const {
    *reinterpret_cast<float4 *>(sm + pos * W + c) = q;
  }
};

// Line-major swizzled tile: element (pos, c) at sm[c*P + swz(pos)]; the
// element index inside each 128-byte row is XORed with the row index (mod 8
// for 16-byte FP64 elements, mod 16 for 8-byte FP32 elements).  Shared memory
// serves 16-byte accesses per quarter warp and 8-byte ones per half warp, so
// unit, 2-, 4-, 8- and row-strided position sets are all conflict free.
// P must be a multiple of 8 (FP64) or 16 (FP32) elements.
__device__ __forceinline__ int swz(int pos, double2 *) { return pos ^ ((pos >> 3) & 7); }
__device__ __forceinline__ int swz(int pos, float2 *) { return pos ^ ((pos >> 4) & 15); }

template <typename C> struct LineTile {
  C *sm;
  int P;
  __device__ __forceinline__ int at(int pos, int c) const { return c * P + swz(pos, (C *)nullptr); }
  __device__ __forceinline__ C operator()(int pos, int c) const { return sm[at(pos, c)]; }
  __device__ __forceinline__ void operator()(int pos, int c, C v) const { sm[at(pos, c)] = v; }
};

// Line-major tile of the compile-time z passes: as LineTile, with an XOR
// swizzle that also folds in higher row bits (t = row of 128 bytes):
//   FP64 (8 elements per row):  pos ^ ((t ^ t>>3 ^ t>>6) & 7)
//   FP32 (16 elements per row): pos ^ ((t ^ t<<1 ^ t>>3) & 15)
// The stages' strided position sets stay conflict free (FP32 ones of stride 8
// too, which LineTile's swizzle serves in two wavefronts), and so, nearly,
// do the fused last stages' reads by consecutive frequency bases, whose
// groups lie at digit-reversed rows (z_split_stage, z_inv_last_stage).
// Chosen with a bank model over the 64- to 1024-point plans.
__device__ __forceinline__ int swz_z(int pos, double2 *) {
  const int t = pos >> 3;
  return pos ^ ((t ^ (t >> 3) ^ (t >> 6)) & 7);
}
__device__ __forceinline__ int swz_z(int pos, float2 *) {
  const int t = pos >> 4;
  return pos ^ ((t ^ (t << 1) ^ (t >> 3)) & 15);
}
template <typename C> struct LineTileZ {
  C *sm;
  int P;
  __device__ __forceinline__ int at(int pos, int c) const { return c * P + swz_z(pos, (C *)nullptr); }
  __device__ __forceinline__ C operator()(int pos, int c) const { return sm[at(pos, c)]; }
  __device__ __forceinline__ void operator()(int pos, int c, C v) const { sm[at(pos, c)] = v; }
};

// Compile-time plans whose stages before the last are all radix 8 (32, 64,
// 128, 256, 512, 1024): the last stage's group g (DIF output positions
// g*RL .. g*RL + RL-1, RL its radix) holds frequencies k0 + r*(N/RL), where
// k0 is g with its S-1 base-8 digits reversed.  The reversal is its own
// inverse: group_of_base(k0) is the group whose frequency base is k0.
__host__ __device__ constexpr bool radix8_prefix(int n) {
  if (n <= 1 || plan_stages(n) < 2) return false;
  for (int s = 0; s + 1 < plan_stages(n); s++)
    if (plan_radix(n, s) != 8) return false;
  return true;
}
// Whether the forward z pass of length n fuses its last stage with the split.
// An item of z_split_stage holds two groups; in FP64 with a radix-8 last
// stage those need more registers than a thread has (spills, and half the
// block idle: 0.411 -> 0.437 ms at 512^3), so 512 points (64 bases) take the
// shuffle form z_split_stage_shfl (ff_tiles.cuh) in both precisions (FP32:
// all threads busy and fewer conflicted reads), and FP64 64 (8 bases) keeps
// the unfused split.
__host__ __device__ constexpr bool z_split_shfl(int n, size_t csz) {
  return csz > 0 && radix8_prefix(n) && plan_radix(n, plan_stages(n) - 1) == 8 && n / 8 == 64;
}
__host__ __device__ constexpr bool z_split_fused(int n, size_t csz) {
  return radix8_prefix(n) && (!(csz == 16 && plan_radix(n, plan_stages(n) - 1) == 8) || z_split_shfl(n, csz));
}

template <int N> __device__ __forceinline__ int group_of_base(int k0) {
  constexpr int D = plan_stages(N) - 1;
  int g = 0;
#pragma unroll
  for (int d = 0; d < D; d++) {
    g = (g << 3) | (k0 & 7);
    k0 >>= 3;
  }
  return g;
}

// Digit reversal of a compile-time plan: the frequency held at DIF output
// position pos (the host builds the same table for runtime plans).
template <int N> __device__ __forceinline__ int rev_ct(int pos) {
  int k = 0, kmul = 1, span = N;
#pragma unroll
  for (int s = 0; s < plan_stages(N); s++) {
    const int r = plan_radix(N, s);
    span /= r;
    const int m = pos / span;
    pos -= m * span;
    k += m * kmul;
    kmul *= r;
  }
  return k;
}

// Frequency index of a position written by the LAST DIF stage (span R):
// rev[base + r] = rev[base] + r*(n/R), so one table load serves the group.
// RC, NRC > 0: compile-time R and n/R.
template <int RC = 0, int NRC = 0> struct RevLast {
  const int *rev;
  int R, nR;
  __device__ __forceinline__ int operator()(int pos) const {
    const int Rv = RC ? RC : R;
    const int r = pos % Rv;
    return __ldg(rev + pos - r) + r * (NRC ? NRC : nR);
  }
};

template <int N> struct RevCT {
  __device__ __forceinline__ int operator()(int pos) const { return rev_ct<N>(pos); }
};

// Line-major tile written at the natural (frequency) index of a DIF output
// position: the out-of-place last stage of a DIF transform.
template <typename C, typename RL> struct LineTileRev {
  LineTile<C> t;
  RL rl;
  __device__ __forceinline__ void operator()(int pos, int c, C v) const { t(rl(pos), c, v); }
};

// ------------------------------------------------------------ stage drivers
// Runtime plan.  DIF stages 0..S-1: stage 0 reads ld0 (with recurrence
// twiddles if TWREC0), stage S-1 writes stl, the others read and write mid.
// A block barrier follows every stage.
template <bool INV, Map MAP, int W, int NT, bool TWREC0, bool TWALL = false, typename C, typename LD0, typename MID,
          typename STL>
__device__ __forceinline__ void dif_rt(const AxisDev<C> &ax, int S, LD0 &ld0, MID &mid, STL &stl, int ncols) {
  int L = ax.n;
  for (int s = 0; s < S; s++) {
    with_radix(ax.radix[s], [&](auto tag) {
      constexpr int R = decltype(tag)::value;
      if (s == 0 && s == S - 1) stage<R, INV, false, MAP, W, NT, 0, 0, TWREC0 || TWALL>(ax.n, L, ax, ld0, stl, ncols);
      else if (s == 0) stage<R, INV, false, MAP, W, NT, 0, 0, TWREC0 || TWALL>(ax.n, L, ax, ld0, mid, ncols);
      else if (s == S - 1) stage<R, INV, false, MAP, W, NT, 0, 0, TWALL>(ax.n, L, ax, mid, stl, ncols);
      else stage<R, INV, false, MAP, W, NT, 0, 0, TWALL>(ax.n, L, ax, mid, mid, ncols);
    });
    L /= ax.radix[s];
    __syncthreads();
  }
}

// Runtime plan.  DIT stages s_begin..0 on a digit-reversed tile in mid;
// stage 0 writes stl.  A block barrier follows every stage.
template <bool INV, Map MAP, int W, int NT, bool TWALL = false, typename C, typename MID, typename STL>
__device__ __forceinline__ void dit_rt(const AxisDev<C> &ax, int s_begin, MID &mid, STL &stl, int ncols) {
  for (int s = s_begin; s >= 0; s--) {
    int L = ax.n;
    for (int q = 0; q < s; q++) L /= ax.radix[q];
    with_radix(ax.radix[s], [&](auto tag) {
      constexpr int R = decltype(tag)::value;
      if (s == 0) stage<R, INV, true, MAP, W, NT, 0, 0, TWALL>(ax.n, L, ax, mid, stl, ncols);
      else stage<R, INV, true, MAP, W, NT, 0, 0, TWALL>(ax.n, L, ax, mid, mid, ncols);
    });
    __syncthreads();
  }
}

// Compile-time plan of length N: DIF stages s..SEND-1 as dif_rt does.
// TWREC0: recurrence twiddles in stage 0; TWALL: in every stage.
// TWMUL: the axis table is TWMUL times longer than N (N is a sub-transform).
template <int N, int SEND, int s, bool INV, Map MAP, int W, int NT, bool TWREC0, bool TWALL, int TWMUL = 1,
          typename C, typename LD0, typename MID, typename STL>
__device__ __forceinline__ void dif_ct(const AxisDev<C> &ax, LD0 &ld0, MID &mid, STL &stl, int ncols) {
  if constexpr (s < SEND) {
    constexpr int R = plan_radix(N, s);
    constexpr int L = plan_span(N, s);
    constexpr bool TWR = TWALL || (TWREC0 && s == 0);
    if constexpr (s == 0 && SEND == 1) stage<R, INV, false, MAP, W, NT, N, L, TWR, TWMUL>(N, L, ax, ld0, stl, ncols);
    else if constexpr (s == 0) stage<R, INV, false, MAP, W, NT, N, L, TWR, TWMUL>(N, L, ax, ld0, mid, ncols);
    else if constexpr (s == SEND - 1) stage<R, INV, false, MAP, W, NT, N, L, TWR, TWMUL>(N, L, ax, mid, stl, ncols);
    else stage<R, INV, false, MAP, W, NT, N, L, TWR, TWMUL>(N, L, ax, mid, mid, ncols);
    __syncthreads();
    dif_ct<N, SEND, s + 1, INV, MAP, W, NT, TWREC0, TWALL, TWMUL>(ax, ld0, mid, stl, ncols);
  }
}

// Compile-time plan of length N: DIT stages s..0 as dit_rt does.
template <int N, int s, bool INV, Map MAP, int W, int NT, bool TWALL, int TWMUL = 1, typename C, typename MID,
          typename STL>
__device__ __forceinline__ void dit_ct(const AxisDev<C> &ax, MID &mid, STL &stl, int ncols) {
  if constexpr (s >= 0) {
    constexpr int R = plan_radix(N, s);
    constexpr int L = plan_span(N, s);
    if constexpr (s == 0) stage<R, INV, true, MAP, W, NT, N, L, TWALL, TWMUL>(N, L, ax, mid, stl, ncols);
    else stage<R, INV, true, MAP, W, NT, N, L, TWALL, TWMUL>(N, L, ax, mid, mid, ncols);
    __syncthreads();
    dit_ct<N, s - 1, INV, MAP, W, NT, TWALL, TWMUL>(ax, mid, stl, ncols);
  }
}

// Full DIF transform (all stages) with a compile-time (N > 0) or runtime plan.
template <int N, bool INV, Map MAP, int W, int NT, bool TWREC0, bool TWALL, typename C, typename LD0, typename MID,
          typename STL>
__device__ __forceinline__ void dif_all(const AxisDev<C> &ax, LD0 &ld0, MID &mid, STL &stl, int ncols) {
  if constexpr (N > 0) dif_ct<N, plan_stages(N), 0, INV, MAP, W, NT, TWREC0, TWALL>(ax, ld0, mid, stl, ncols);
  else dif_rt<INV, MAP, W, NT, TWREC0, TWALL>(ax, ax.nstages, ld0, mid, stl, ncols);
}

// ------------------------------------------------ TMA and mbarrier helpers
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *m, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Orders this thread's earlier generic-proxy shared-memory accesses before
// later async-proxy (TMA) accesses of the same memory.
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// A tensor map in global memory (not a kernel parameter) is written by the
// generic proxy (a copy from the host, possibly over an earlier map at the
// same address) and read by the TMA unit's tensormap proxy: this acquire
// fence, by the thread that issues the copies, orders the two, so the TMA
// does not use a stale descriptor.
__device__ __forceinline__ void tensormap_acquire(const void *map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *m, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *m, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(m)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Built-in iteration limit of the bounded waits (about a second with the
// back-off of mbar_wait_bounded).
constexpr int kWaitIters = 1 << 24;

// Waits for phase `parity` of m with an iteration limit (limit <= 0: the
// built-in kWaitIters); returns false if the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *m, uint32_t parity, int limit = kWaitIters) {
  if (limit <= 0) limit = kWaitIters;
  for (int i = 0; i < limit; i++) {
    if (mbar_try_wait(m, parity)) return true;
    if (i >= 32) __nanosleep(64);
  }
  return false;
}

// 3-D tiled TMA load of one box into shared memory, completing on m.
__device__ __forceinline__ void tma_load_3d(void *dst, const void *tmap, int x, int y, int z, uint64_t *m) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::
          "r"(smem_u32(dst)),
      "l"(tmap), "r"(x), "r"(y), "r"(z), "r"(smem_u32(m))
      : "memory");
}

// 3-D tiled TMA store of one box from shared memory (bulk async-group).
__device__ __forceinline__ void tma_store_3d(const void *tmap, int x, int y, int z, const void *src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(tmap), "r"(x),
               "r"(y), "r"(z), "r"(smem_u32(src))
               : "memory");
}

// Contiguous bulk copies (addresses 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void *dst, const void *src, uint32_t bytes, uint64_t *m) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(m))
               : "memory");
}
__device__ __forceinline__ void bulk_store(void *dst, const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(dst), "r"(smem_u32(src)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// Waits until every committed bulk store of this thread has finished reading
// shared memory (the buffer may then be reused or released).
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }

// L2 prefetch hint of a contiguous range (16-byte aligned, size a multiple of
// 16).  No data reaches shared memory and no completion is tracked.
__device__ __forceinline__ void l2_prefetch(const void *src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

// Element copies from global to shared memory that complete asynchronously
// (all of a thread's copies are in flight together); 16 bytes (.cg, L2 only)
// or 8 bytes (.ca); addresses aligned to the size.  cp_async_wait_all waits
// for this thread's copies; a barrier then publishes them to the block.
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// Device-side status word values (plan status buffer).
enum : int { kDevOk = 0, kDevTmaTimeout = 1, kDevDepTimeout = 2 };

}  // namespace ff
