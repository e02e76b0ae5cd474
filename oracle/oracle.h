/*
 * CPU oracle for the Fish Fry periodic Poisson solve -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is the checker, never the product: only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  The product path (fishfry_b200)
 * neither links nor calls it.
 *
 * It restates, in plain FP64 C++ with an FFT written here, the single-task
 * (1x1x1) arithmetic of the reference:
 *   - ParisPencil::ParisPencil  wavenumber scales dd = 2*pi*(n-1)/(n*(hi-lo))
 *                                (ParisPencil.cpp:9-11), nh = nk/2+1 (:18)
 *   - ParisPencil::solve         R2C in z (:165), C2C forward in y (:212) and x
 *                                (:259), filter -1/(kx^2+ky^2+kz^2) with the zero
 *                                mode set to 0 (:263-285), C2C inverse in x (:288)
 *                                and y (:334), C2R in z (:380), times 1/N (:406-421)
 *   - FishFry init kernel        f = px*py*dpz + px*dpy*pz + dpx*py*pz
 *                                (FishFry.hpp:14-45), grid x = -pi + i*2*pi/n
 *                                (FishFry.hpp:109-111,133-134,137-139)
 *   - FishFry diff kernel        sum|d|, sum d^2, max|d| against phi_a=px*py*pz
 *                                (FishFry.hpp:57-101); relative norms use the
 *                                phi=0 pass as scales (FishFry.hpp:146-159,198)
 * The FFT convention matches cuFFT's: unnormalised forward exp(-2*pi*i*jk/n),
 * inverse exp(+...), and the single 1/N applied once at the end.
 *
 * Parity pinning: the relative-norm known answers at 8^3 and 16^3 (truncation
 * dominated, so they pin grid, filter and zero mode) and numpy.fft are checked
 * in tests/test_oracle.py; the reference itself, built from its own sources
 * with a single-rank MPI stub (oracle/ref), is compared on a GPU machine.
 */
#ifndef FISHFRY_ORACLE_H
#define FISHFRY_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* One Fourier mode of the seeded random term: f += a*cos(kx*x+ky*y+kz*z+theta). */
typedef struct {
  int kx, ky, kz;
  double a, theta;
} orc_mode;

/* Number of OpenMP threads the oracle uses (0 = all available). */
void orc_set_threads(int nthreads);
int orc_get_threads(void);

/* 1-D complex DFT of length n (interleaved re,im), sign -1 forward, +1 inverse,
 * unnormalised.  in and out may alias.  Returns 0 on success. */
int orc_fft1d(int n, int sign, const double *in, double *out);

/* Full solve: f real [ni][nj][nk] (k fastest), phi real out.  lo/hi follow the
 * reference constructor (hi is one cell short of the periodic length).
 * Returns 0 on success. */
int orc_solve(int ni, int nj, int nk, const double lo[3], const double hi[3],
              const double *f, double *phi);

/* Forward half spectrum only (after R2C z, C2C y, C2C x): complex
 * [ni][nj][nh] interleaved, nh = nk/2+1.  Used to check the pass sequence. */
int orc_forward_spectrum(int ni, int nj, int nk, const double *f, double *spec);

/* Analytic right-hand side and solution on the reference grid
 * x = xlo + i*dx (FishFry.hpp:22-44 and :71-86), plus the optional modes. */
void orc_init_f(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                int nmodes, const orc_mode *modes, double *f);
void orc_phi_exact(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                   int nmodes, const orc_mode *modes, double *phi);

/* Raw sums against the analytic phi: out = {sum|d|, sum d^2, max|d|}
 * (FishFry.hpp:57-101), and the relative norms {L1, L2, Linf} as printed at
 * FishFry.hpp:198 (scales from a phi=0 pass, FishFry.hpp:146-159). */
void orc_diff_sums(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                   int nmodes, const orc_mode *modes, const double *phi, double out[3]);
void orc_rel_norms(int ni, int nj, int nk, const double xlo[3], const double dx[3],
                   int nmodes, const orc_mode *modes, const double *phi, double out[3]);

/* Seeded random modes (restatement of the product's generator; SplitMix64 +
 * Box-Muller): count modes with integer k, 0 < |k| <= kmax and
 * |k_axis| <= kaxis[axis], amplitude ~ N(0, sigma), phase ~ U[0, 2*pi). */
void orc_modes_generate(uint64_t seed, int count, int kmax, const int kaxis[3],
                        double sigma, orc_mode *out);

#ifdef __cplusplus
}
#endif

#endif
