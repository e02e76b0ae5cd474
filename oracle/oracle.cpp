// CPU oracle for the Fish Fry Poisson solve -- TEST INFRASTRUCTURE ONLY.
// See oracle.h for what each function restates (reference file:line) and who
// may call it.  Plain FP64, OpenMP over lines, FFT written here (mixed-radix
// recursive Cooley-Tukey with specialised radix 2/3/4/5 and a direct DFT for
// any other prime factor, so the oracle accepts every length).

#include "oracle.h"

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

using cd = std::complex<double>;

int g_threads = 0;

int nthreads() {
#ifdef _OPENMP
  return g_threads > 0 ? g_threads : omp_get_max_threads();
#else
  return 1;
#endif
}

// ---------------------------------------------------------------- 1-D FFT
struct Plan1D {
  int n = 0;
  std::vector<int> fac;   // factors, 4 first, then 2, 3, 5, other primes
  std::vector<cd> tw;     // tw[q] = exp(-2*pi*i*q/n), q in [0, n)
};

std::vector<int> factorize(int n) {
  std::vector<int> f;
  while (n % 4 == 0) { f.push_back(4); n /= 4; }
  while (n % 2 == 0) { f.push_back(2); n /= 2; }
  for (int p = 3; n > 1; p += 2) {
    while (n % p == 0) { f.push_back(p); n /= p; }
    if (p * p > n && n > 1) { f.push_back(n); n = 1; }
  }
  return f;
}

// exp(-2*pi*i*q/n) evaluated in long double, then rounded to double.
cd twiddle(long q, long n) {
  long double a = -2.0L * 3.141592653589793238462643383279502884L * (long double)q / (long double)n;
  return cd((double)cosl(a), (double)sinl(a));
}

const Plan1D &get_plan(int n) {
  static std::mutex mu;
  static std::map<int, std::unique_ptr<Plan1D>> cache;
  std::lock_guard<std::mutex> lock(mu);
  auto it = cache.find(n);
  if (it != cache.end()) return *it->second;
  auto p = std::make_unique<Plan1D>();
  p->n = n;
  p->fac = factorize(n);
  p->tw.resize(n);
  for (int q = 0; q < n; q++) p->tw[q] = twiddle(q, n);
  auto &ref = *p;
  cache[n] = std::move(p);
  return ref;
}

// X[k] = sum_t x[t*stride] * w^(sign*t*k) for a sub-transform of length n of
// the plan's full length N.  Decimation in time: the p sub-transforms of the
// strided inputs are written to X[q*m .. q*m+m), then combined in place.
void fft_rec(const cd *x, long stride, cd *X, int n, const int *fac, const Plan1D &P, int sign) {
  if (n == 1) { X[0] = x[0]; return; }
  const int p = fac[0];
  const int m = n / p;
  for (int q = 0; q < p; q++) fft_rec(x + q * stride, stride * p, X + (long)q * m, m, fac + 1, P, sign);
  const int N = P.n;
  const int sN = N / n;   // twiddle stride for length n
  const int sP = N / p;   // twiddle stride for length p
  auto W = [&](long idx) -> cd {   // exp(sign*2*pi*i*idx/N)
    cd w = P.tw[idx % N];
    return sign > 0 ? std::conj(w) : w;
  };
  cd t[64];
  std::vector<cd> big;
  cd *tp = t;
  if (p > 64) { big.resize(p); tp = big.data(); }
  for (int k = 0; k < m; k++) {
    for (int q = 0; q < p; q++) {
      cd y = X[(long)q * m + k];
      tp[q] = (q == 0 || k == 0) ? y : y * W((long)q * k * sN);
    }
    if (p == 2) {
      cd a = tp[0], b = tp[1];
      X[k] = a + b; X[k + m] = a - b;
    } else if (p == 4) {
      cd a = tp[0] + tp[2], b = tp[0] - tp[2];
      cd c = tp[1] + tp[3], d = tp[1] - tp[3];
      // multiply d by -i*sign_fwd: forward (sign=-1) uses -i, inverse +i
      cd dj = sign < 0 ? cd(d.imag(), -d.real()) : cd(-d.imag(), d.real());
      X[k] = a + c; X[k + m] = b + dj; X[k + 2 * m] = a - c; X[k + 3 * m] = b - dj;
    } else {
      // the inputs X[q*m + k] are all held in tp, so the outputs X[k + s*m]
      // (the same locations) can be written directly
      for (int s = 0; s < p; s++) {
        cd acc = tp[0];
        for (int q = 1; q < p; q++) acc += tp[q] * W((long)((q * s) % p) * sP);
        X[k + (long)s * m] = acc;
      }
    }
  }
}

void fft_line(int n, int sign, const cd *in, cd *out) {
  const Plan1D &P = get_plan(n);
  if (in == out) {
    std::vector<cd> tmp(in, in + n);
    fft_rec(tmp.data(), 1, out, n, P.fac.data(), P, sign);
  } else {
    fft_rec(in, 1, out, n, P.fac.data(), P, sign);
  }
}

// ---------------------------------------------------------------- passes
// Half spectrum layout: spec[(i*nj + j)*nh + kh].

// Real-to-complex along z for lines (a, b) packed as z = a + i*b, then split:
// A[k] = (Z[k] + conj(Z[n-k]))/2, B[k] = (Z[k] - conj(Z[n-k]))/(2i).
void r2c_z(int ni, int nj, int nk, const double *f, cd *spec) {
  const int nh = nk / 2 + 1;
  const long nlines = (long)ni * nj;
  const long npairs = (nlines + 1) / 2;
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<cd> z(nk), Z(nk);
#pragma omp for schedule(static)
    for (long pr = 0; pr < npairs; pr++) {
      const long la = 2 * pr, lb = 2 * pr + 1;
      const bool hasb = lb < nlines;
      for (int k = 0; k < nk; k++)
        z[k] = cd(f[la * nk + k], hasb ? f[lb * nk + k] : 0.0);
      fft_line(nk, -1, z.data(), Z.data());
      for (int k = 0; k < nh; k++) {
        const cd zk = Z[k], zn = std::conj(Z[(nk - k) % nk]);
        spec[la * nh + k] = 0.5 * (zk + zn);
        if (hasb) {
          const cd d = zk - zn;
          spec[lb * nh + k] = cd(0.5 * d.imag(), -0.5 * d.real());
        }
      }
    }
  }
}

// Complex-to-real along z: Hermitian extension of each half line (imaginary
// parts of the zero and, for even nk, Nyquist terms are dropped, as a C2R
// transform does), two lines per complex inverse transform, times scale.
void c2r_z(int ni, int nj, int nk, const cd *spec, double scale, double *phi) {
  const int nh = nk / 2 + 1;
  const long nlines = (long)ni * nj;
  const long npairs = (nlines + 1) / 2;
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<cd> Z(nk), z(nk);
#pragma omp for schedule(static)
    for (long pr = 0; pr < npairs; pr++) {
      const long la = 2 * pr, lb = 2 * pr + 1;
      const bool hasb = lb < nlines;
      auto A = [&](int k) { return spec[la * nh + k]; };
      auto B = [&](int k) { return hasb ? spec[lb * nh + k] : cd(0, 0); };
      for (int k = 0; k < nk; k++) {
        cd a, b;
        if (k < nh) { a = A(k); b = B(k); }
        else { a = std::conj(A(nk - k)); b = std::conj(B(nk - k)); }
        if (k == 0 || 2 * k == nk) { a = cd(a.real(), 0); b = cd(b.real(), 0); }
        Z[k] = a + cd(0, 1) * b;
      }
      fft_line(nk, +1, Z.data(), z.data());
      for (int k = 0; k < nk; k++) {
        phi[la * nk + k] = scale * z[k].real();
        if (hasb) phi[lb * nk + k] = scale * z[k].imag();
      }
    }
  }
}

// Complex transform along y (axis 1) or x (axis 0) of the half spectrum.
void c2c_axis(int ni, int nj, int nh, int axis, int sign, cd *spec) {
  const int n = axis == 1 ? nj : ni;
  const long stride = axis == 1 ? (long)nh : (long)nj * nh;
  const int nouter = axis == 1 ? ni : nj;
  const long outer_stride = axis == 1 ? (long)nj * nh : (long)nh;
  const int B = 8;
  const int nblk = (nh + B - 1) / B;
#pragma omp parallel num_threads(nthreads())
  {
    std::vector<cd> buf((size_t)B * n), out(n);
#pragma omp for schedule(static)
    for (long job = 0; job < (long)nouter * nblk; job++) {
      const long o = job / nblk;
      const int k0 = (int)(job % nblk) * B;
      const int w = std::min(B, nh - k0);
      cd *base = spec + o * outer_stride + k0;
      for (int p = 0; p < n; p++)
        for (int c = 0; c < w; c++) buf[(size_t)c * n + p] = base[p * stride + c];
      for (int c = 0; c < w; c++) {
        fft_line(n, sign, &buf[(size_t)c * n], out.data());
        std::copy(out.begin(), out.end(), buf.begin() + (size_t)c * n);
      }
      for (int p = 0; p < n; p++)
        for (int c = 0; c < w; c++) base[p * stride + c] = buf[(size_t)c * n + p];
    }
  }
}

// Spectral filter (ParisPencil.cpp:263-285), single task: global indices
// i, j, kh; d = -1/((min(i,ni-i)*ddi)^2 + (min(j,nj-j)*ddj)^2 + (kh*ddk)^2);
// the zero mode is set to 0.
void filter(int ni, int nj, int nk, const double dd[3], cd *spec) {
  const int nh = nk / 2 + 1;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++) {
      const double ii = (double)std::min(i, ni - i) * dd[0];
      const double jj = (double)std::min(j, nj - j) * dd[1];
      cd *row = spec + ((long)i * nj + j) * nh;
      for (int k = 0; k < nh; k++) {
        if (i || j || k) {
          const double kk = (double)k * dd[2];
          const double d = -1.0 / (ii * ii + jj * jj + kk * kk);
          row[k] = cd(d * row[k].real(), d * row[k].imag());
        } else {
          row[k] = cd(0, 0);
        }
      }
    }
}

// ---------------------------------------------------------------- fields
struct Axis1D {
  std::vector<double> p, dp;   // phi factor and its second derivative
};

// FishFry.hpp:22-41: px = cos x e^{sin x}, py = sin y e^{cos y}, pz = cos z e^{cos z}.
Axis1D axis_factors(int axis, int n, double lo, double d) {
  Axis1D a;
  a.p.resize(n);
  a.dp.resize(n);
  for (int i = 0; i < n; i++) {
    const double x = lo + i * d;
    const double c = std::cos(x), s = std::sin(x);
    if (axis == 0) {
      const double e = std::exp(s);
      a.p[i] = c * e;
      a.dp[i] = -e * s * c * (s + 3.0);
    } else if (axis == 1) {
      const double e = std::exp(c);
      a.p[i] = s * e;
      a.dp[i] = s * e * (s * s - 3.0 * c - 1.0);
    } else {
      const double e = std::exp(c);
      a.p[i] = c * e;
      a.dp[i] = e * (3.0 * s * s - c * c * c - 1.0);
    }
  }
  return a;
}

double mode_value(const orc_mode &m, double x, double y, double z) {
  return std::cos((double)m.kx * x + (double)m.ky * y + (double)m.kz * z + m.theta);
}

int mode_k2(const orc_mode &m) { return m.kx * m.kx + m.ky * m.ky + m.kz * m.kz; }

// SplitMix64 (Steele, Lea and Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014).
struct SplitMix64 {
  uint64_t s;
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * 0x1.0p-53; }
};

}  // namespace

extern "C" {

void orc_set_threads(int n) { g_threads = n; }
int orc_get_threads(void) { return nthreads(); }

int orc_fft1d(int n, int sign, const double *in, double *out) {
  if (n < 1 || (sign != 1 && sign != -1)) return 1;
  fft_line(n, sign, reinterpret_cast<const cd *>(in), reinterpret_cast<cd *>(out));
  return 0;
}

int orc_forward_spectrum(int ni, int nj, int nk, const double *f, double *spec_out) {
  if (ni < 1 || nj < 1 || nk < 1) return 1;
  const int nh = nk / 2 + 1;
  cd *spec = reinterpret_cast<cd *>(spec_out);
  r2c_z(ni, nj, nk, f, spec);
  c2c_axis(ni, nj, nh, 1, -1, spec);
  c2c_axis(ni, nj, nh, 0, -1, spec);
  return 0;
}

int orc_solve(int ni, int nj, int nk, const double lo[3], const double hi[3], const double *f, double *phi) {
  if (ni < 1 || nj < 1 || nk < 1) return 1;
  const int n[3] = {ni, nj, nk};
  double dd[3];
  // ParisPencil.cpp:9-11.  A one-point axis has hi == lo and the reference's
  // formula gives 0/0 = NaN (and a NaN potential); its only wavenumber is 0, so
  // dd = 0 is used there, as the product does.
  for (int a = 0; a < 3; a++)
    dd[a] = n[a] > 1 ? 2.0 * M_PI * double(n[a] - 1) / (double(n[a]) * (hi[a] - lo[a])) : 0.0;
  const int nh = nk / 2 + 1;
  std::vector<cd> spec((size_t)ni * nj * nh);
  r2c_z(ni, nj, nk, f, spec.data());
  c2c_axis(ni, nj, nh, 1, -1, spec.data());
  c2c_axis(ni, nj, nh, 0, -1, spec.data());
  filter(ni, nj, nk, dd, spec.data());
  c2c_axis(ni, nj, nh, 0, +1, spec.data());
  c2c_axis(ni, nj, nh, 1, +1, spec.data());
  const double divN = 1.0 / (double(ni) * double(nj) * double(nk));   // ParisPencil.cpp:408
  c2r_z(ni, nj, nk, spec.data(), divN, phi);
  return 0;
}

void orc_init_f(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                int nmodes, const orc_mode *modes, double *f) {
  const Axis1D X = axis_factors(0, ni, xlo[0], dx[0]);
  const Axis1D Y = axis_factors(1, nj, xlo[1], dx[1]);
  const Axis1D Z = axis_factors(2, nk, xlo[2], dx[2]);
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++)
      for (int k = 0; k < nk; k++) {
        double v = X.p[i] * Y.p[j] * Z.dp[k] + X.p[i] * Y.dp[j] * Z.p[k] + X.dp[i] * Y.p[j] * Z.p[k];
        for (int m = 0; m < nmodes; m++) {
          if (mode_k2(modes[m]) == 0) continue;
          v += modes[m].a * mode_value(modes[m], xlo[0] + i * dx[0], xlo[1] + j * dx[1], xlo[2] + k * dx[2]);
        }
        f[((long)i * nj + j) * nk + k] = v;
      }
}

void orc_phi_exact(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                   int nmodes, const orc_mode *modes, double *phi) {
  const Axis1D X = axis_factors(0, ni, xlo[0], dx[0]);
  const Axis1D Y = axis_factors(1, nj, xlo[1], dx[1]);
  const Axis1D Z = axis_factors(2, nk, xlo[2], dx[2]);
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthreads())
  for (int i = 0; i < ni; i++)
    for (int j = 0; j < nj; j++)
      for (int k = 0; k < nk; k++) {
        double v = X.p[i] * Y.p[j] * Z.p[k];
        for (int m = 0; m < nmodes; m++) {
          const int k2 = mode_k2(modes[m]);
          if (k2 == 0) continue;
          v += -modes[m].a / (double)k2 *
               mode_value(modes[m], xlo[0] + i * dx[0], xlo[1] + j * dx[1], xlo[2] + k * dx[2]);
        }
        phi[((long)i * nj + j) * nk + k] = v;
      }
}

void orc_diff_sums(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                   int nmodes, const orc_mode *modes, const double *phi, double out[3]) {
  std::vector<double> ex((size_t)ni * nj * nk);
  orc_phi_exact(ni, nj, nk, xlo, dx, nmodes, modes, ex.data());
  double s1 = 0, s2 = 0, mx = 0;
  const long N = (long)ni * nj * nk;
#pragma omp parallel for reduction(+ : s1, s2) reduction(max : mx) num_threads(nthreads())
  for (long q = 0; q < N; q++) {
    const double d = std::fabs(ex[q] - (phi ? phi[q] : 0.0));
    s1 += d;
    s2 += d * d;
    mx = std::max(mx, d);
  }
  out[0] = s1;
  out[1] = s2;
  out[2] = mx;
}

void orc_rel_norms(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                   int nmodes, const orc_mode *modes, const double *phi, double out[3]) {
  double scale[3], d[3];
  orc_diff_sums(ni, nj, nk, xlo, dx, nmodes, modes, nullptr, scale);
  orc_diff_sums(ni, nj, nk, xlo, dx, nmodes, modes, phi, d);
  out[0] = d[0] / scale[0];
  out[1] = std::sqrt(d[1] / scale[1]);
  out[2] = d[2] / scale[2];
}

void orc_modes_generate(uint64_t seed, int count, int kmax, const int kaxis[3], double sigma, orc_mode *out) {
  SplitMix64 rng{seed};
  const long kmax2 = (long)kmax * kmax;
  const bool possible = kmax > 0 && (kaxis[0] > 0 || kaxis[1] > 0 || kaxis[2] > 0);
  for (int m = 0; m < count; m++) {
    orc_mode md{0, 0, 0, 0.0, 0.0};
    if (possible) {
      for (;;) {
        const int kx = (int)(rng.next() % (uint64_t)(2 * kaxis[0] + 1)) - kaxis[0];
        const int ky = (int)(rng.next() % (uint64_t)(2 * kaxis[1] + 1)) - kaxis[1];
        const int kz = (int)(rng.next() % (uint64_t)(2 * kaxis[2] + 1)) - kaxis[2];
        const long k2 = (long)kx * kx + (long)ky * ky + (long)kz * kz;
        if (k2 == 0 || k2 > kmax2) continue;
        md.kx = kx; md.ky = ky; md.kz = kz;
        break;
      }
      const double u1 = 1.0 - rng.uniform();
      const double u2 = rng.uniform();
      md.a = sigma * std::sqrt(-2.0 * std::log(u1)) * std::cos(2.0 * M_PI * u2);
      md.theta = 2.0 * M_PI * rng.uniform();
    }
    out[m] = md;
  }
}

}  // extern "C"
