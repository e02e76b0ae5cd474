// Axes whose length has a prime factor above 7 (single-grid solve).
//
// cuFFT, which the reference calls for every line transform
// (ParisPencil.cpp:78-81 plans, :165/:212/:259/:288/:334/:380 executions),
// accepts any length.  Here an axis of n points with a prime factor above 7
// is transformed by Bluestein's algorithm: with the chirp
// c[j] = exp(-i*pi*j^2/n), the forward DFT is
//   X[k] = c[k] * sum_j (x[j] c[j]) conj c[k-j],
// a circular convolution of M >= 2n-1 points (M = 2^a 3^b 5^c 7^d), computed by
// the same mixed-radix stages as every other axis: an M-point forward DIF
// transform of the premultiplied, zero-padded line, a product with the
// transform of the convolution kernel (one register group, with the last DIF
// and first DIT stages), an M-point inverse DIT transform, and the
// postmultiplication.  The inverse DFT uses the conjugate chirp and kernel.
// Each pass keeps its own work around the transform: the z pass packs two
// real lines into one complex line and splits the result into the two half
// spectra (and the reverse), the x pass applies the filter between its
// forward and inverse transforms.
#pragma once

#include <cuda_runtime.h>

#include "ff_tiles.cuh"

namespace ff {

template <typename C> struct BsAxis {
  AxisDev<C> m;      // plan and twiddle tables of the M-point transforms
  int n;             // axis length
  const C *chirp;    // chirp[j] = exp(-i*pi*j^2/n), j < n (FP64-generated)
  const C *ghat;     // ghat[pos] = G[k]/M for the frequency k at DIF output position pos,
                     // G the M-point DFT of g[m] = conj chirp[|m|] (|m| < n, indices mod M)
};

// Smallest 2^a 3^b 5^c 7^d >= 2n - 1.
int bs_padded_length(int n);

// Launch shape of one Bluestein pass.
struct BsCfg {
  int W;          // z: line pairs per block; y, x: columns per tile
  int P;          // z: line pitch in complex values (multiple of 8 FP64 / 16 FP32)
  size_t smem;    // dynamic shared memory per block
  long grid;      // blocks
};

// Chooses the launch shape of pass `kind` (0 z forward, 1 y forward, 2 x,
// 3 y inverse, 4 z inverse) of an ni x nj x nk plan whose axis for that pass
// is transformed through M points, and raises the kernel's shared-memory
// limit.  FF_OK or an FF_ERR_* status.
template <typename T> int bs_configure(int kind, int ni, int nj, int nh, int M, BsCfg *cfg);

// Device tables of one axis: chirp (n values) and ghat (M values, from the
// M-point plan's digit reversal rev).  Enqueued on the current device's
// default stream.
template <typename C> int bs_tables(int n, int M, const int *rev, C *chirp, C *ghat);

// Pass launches (kind numbering as in bs_configure).  src and dst are the
// pass's input and output arrays as the regular passes use them: z forward
// reads the real field and writes the spectrum; y forward and x work in place
// on the spectrum; y inverse reads one spectrum array and writes the other;
// z inverse reads the spectrum and writes the real field.
template <typename T> int bs_launch(int kind, const void *src, void *dst, const PassArgs<T> &a,
                                    const BsAxis<typename Cplx<T>::type> &bs, const BsCfg &cfg, cudaStream_t st);

}  // namespace ff
