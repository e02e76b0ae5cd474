// The single-grid plan (the state behind ff_plan_create) and the helpers
// that the passes of other forms (the multi-rank slabs) share with it.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include "ff_bluestein.hpp"
#include "ff_fft.cuh"
#include "ff_status.hpp"
#include "ff_tiles.cuh"

namespace ff {

// Launch shape of a strided pass (one TMA tile per block).
struct StridedCfg {
  int N;          // specialised length of the kernel, 0 = runtime plan
  int W;          // columns per tile
  int box_rows;   // rows per TMA box (a divisor of n, at most 256)
  size_t smem;    // dynamic shared memory: one tile + alignment slack
  int grid;       // one block per tile
};

// Launch shape of a fused persistent pass.
struct FusedCfg {
  int NZ, NY;     // specialised z and y lengths of the kernel (0 = runtime plan)
  size_t smem;
  int grid;
  int lag;
  int prod_pp, cons_pp;
};

}  // namespace ff

struct ff_plan {
  int n[3];
  int precision;
  int nh, nhp;
  double dd[3];
  size_t bytes;
  int device;
  int num_sms;
  void *dmem;
  ff::AxisDev<double2> axd[3];
  ff::AxisDev<float2> axf[3];
  double *kk[3];
  int *status;
  int *counters;       // fused passes: 2 tickets + 2 x ni plane counts
  int fused;           // 1: three launches (fused z/y passes), 0: five launches
  int zN;              // z passes: specialised length, 0 = runtime plan
  bool zbulk;          // z passes: line blocks by bulk copies
  int zW, zP;          // z passes: line pairs per block, line pitch in complex values
  size_t zsmem;
  unsigned ztiles;
  int l2_ahead;        // forward z pass: L2 prefetch distance in blocks (0: off)
  int wait_iters;      // bounded device waits: iteration limit of the first wait (0: built-in)
  int dep_extra;       // fused passes: added to every dependency wait's target (test hook, 0)
  ff::StridedCfg ycfg, xcfg;
  ff::FusedCfg fwd, inv;
  // axes with a prime factor above 7: padded convolution length M (0 for a
  // 2^a 3^b 5^c 7^d axis), their tables, and the launch shape of each pass kind
  // (0 z fwd, 1 y fwd, 2 x, 3 y inv, 4 z inv) that transforms such an axis
  int bsM[3];
  ff::BsAxis<double2> bsd[3];
  ff::BsAxis<float2> bsf[3];
  ff::BsCfg bscfg[5];
  cudaEvent_t ev[FF_MAX_PHASES + 1];
};

namespace ff {

// Per-grid pass arguments of a plan.
template <typename T> PassArgs<T> pass_args(const ff_plan *p) {
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
  for (int d = 0; d < 3; d++) a.dd[d] = p->dd[d];
  a.status = p->status;
  a.l2_ahead = p->l2_ahead;
  a.wait_iters = p->wait_iters;
  return a;
}

// Tensor map of a half spectrum at `base` (ni planes of nj rows of nh complex
// values, row pitch nhp) viewed as (2*nh reals, nj, ni); box = W columns by
// box_rows rows of one plane (y pass) or box_rows planes of one row (x pass).
int encode_spectrum_map(void *base, int ni, int nj, int nh, int nhp, size_t esz, int W, int box_rows, bool xpass,
                        CUtensorMap *map);

// Raises fn's dynamic shared-memory limit to what is left beside its static
// shared memory; returns that limit in *avail (may be NULL).
int allow_dyn_smem_fn(const void *fn, size_t *avail);

// The z forward (inverse = false: real field `in` -> half spectrum `out`) or z
// inverse (spectrum `in` -> real field `out`) pass of plan p on stream st,
// through the Bluestein kernels where the z axis needs them.
int plan_launch_z(const ff_plan *p, bool inverse, void *in, void *out, cudaStream_t st);

// Reads and clears the plan's device status word; FF_ERR_TIMEOUT if a
// bounded wait inside a kernel gave up.
int take_device_status(const ff_plan *p, cudaStream_t st);

}  // namespace ff
