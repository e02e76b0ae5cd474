// Many independent grids per launch: host-visible declarations shared by the
// batch translation units (ff_batch.cu host code, ff_batch_f64.cu and
// ff_batch_f32.cu kernels).
//
// A batch runs the same five passes as a single solve (z R2C, y forward,
// x forward + filter + inverse, y inverse, z C2R), but every launch covers
// the tiles of all its grids: one persistent kernel per pass, whose blocks
// take tiles from a ticket counter until the work list is exhausted.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <vector_types.h>

#include <algorithm>
#include <cstddef>
#include <vector>

#include "ff_fft.cuh"

namespace ff {

// Per-block shared-memory budget of the batch kernels (three blocks per SM).
constexpr size_t kBatchSmem = 72 * 1024;
// The z passes (kinds 0 and 4) run blocks of 128 threads on tiles within
// 36 KB, six per SM, as the single-grid z passes do: more, smaller tiles in
// flight hide each block's inbound copy.
constexpr int kBatchZThreads = 128;
constexpr size_t kBatchZSmem = 36 * 1024;
inline int batch_threads(int kind) { return kind == 0 || kind == 4 ? kBatchZThreads : 256; }
inline size_t batch_budget(int kind) { return kind == 0 || kind == 4 ? kBatchZSmem : kBatchSmem; }
inline int batch_blocks_per_sm(int kind) { return kind == 0 || kind == 4 ? 6 : 3; }

// Axis lengths with compile-time specialised batch tiles; others use the
// runtime plan of their axis.
#define FF_FOR_EACH_BATCH_N(X) X(32) X(48) X(64) X(80) X(96) X(128) X(256) X(512)

// Lengths with compile-time specialised one-plane TMA tiles.
#define FF_FOR_EACH_BATCH_TMA_N(X) X(256) X(512)

inline bool batch_special_n(int n) {
#define FF_CASE(NN) if (n == NN) return true;
  FF_FOR_EACH_BATCH_N(FF_CASE)
#undef FF_CASE
  return false;
}

// One launch: tiles of entries e = 0..nentry-1 are numbered start[e] ..
// start[e+1]-1; entry e names (grid, pass).  ticket is zeroed before the
// launch.
struct BatchWork {
  const int2 *entry;
  const int *start;
  int nentry;
  int *ticket;
};

// Tile shape of one pass of one grid: z passes take W line pairs per tile;
// strided passes take W columns (W * sizeof(complex) a multiple of 128
// bytes: 1, 2 or 4 rows of 128 bytes).  ct = 1 selects the compile-time
// specialised tile for the axis length (batch_special_n), 0 the runtime plan.
// Strided passes: tma = 1 (W = 128 bytes of columns) is a tile of W kh
// columns of one plane, loaded by TMA boxes as in the single-grid passes;
// tma = 0 is W columns of the flattened (plane, kh) index, read straight from
// HBM.  z passes of runtime lengths: tma = 1 moves the line blocks by bulk
// copies (compile-time lengths always do).
// order (runtime plans of the owning pass only: z fwd for the z axis, y fwd
// for y, x for x): the radix split of the axis, as batch_radix_order numbers
// it; 0 is the default plan order.
struct TileShape {
  int W;
  int ct;
  int tma;
  int order;
};

// Radix orders the tuner tries for a runtime length: 0 the default plan
// (8s, one 4 or 2, 5s, 3s), 1 the same radices reversed, 2 the odd radices
// first.  Empty if the order repeats a lower-numbered one.
constexpr int kBatchOrders = 3;
std::vector<int> batch_radix_order(int n, int order);

// Shared memory of one tile (bytes, with alignment slack).
inline size_t batch_tile_smem(int kind, int n_axis, int nk, int nhp, int W, size_t csz) {
  if (kind == 0 || kind == 4) {
    const int align = csz == 16 ? 8 : 16;
    const size_t P = (size_t)(nk + align - 1) / align * align;
    const size_t a = std::max<size_t>((size_t)W * P, 2 * (size_t)W * nhp) * csz;
    // a forward tile whose last stage is fused with the split stages the
    // spectrum rows in its second buffer, which is then as large as the first
    const size_t b = kind == 0 && z_split_fused(nk, csz) ? ((a + 127) & ~size_t(127)) : (size_t)W * P * csz;
    return ((a + 127) & ~size_t(127)) + b + 128 + 128;
  }
  return (size_t)n_axis * W * csz + 128;
}

// Launches pass `kind` (0..4) of the precision-T batch kernel; grids points
// at the device array of the batch's grid descriptors.
// maps: per grid two tensor maps of its potential's half spectrum (y boxes,
// x boxes), used by tiles with tma = 1.
template <typename T>
int batch_pass_launch(int kind, const void *grids, const CUtensorMap *maps, const BatchWork &wl, int blocks,
                      size_t smem, cudaStream_t st);
// Raises the pass kernel's shared-memory limit to its budget (batch_budget)
// and reports how many blocks of `smem` bytes fit on one SM.
template <typename T> int batch_pass_prepare(int kind, size_t smem, int *per_sm);
// Size and alignment of the device grid descriptor for precision T.
template <typename T> size_t batch_desc_size();
// Fills the device grid descriptor image at dst (batch_desc_size bytes).
struct BatchGridHost;
template <typename T> void batch_desc_fill(void *dst, const BatchGridHost &g);

// Host description of one grid of a batch (what batch_desc_fill packs).
struct BatchGridHost {
  int n[3];
  int nh, nhp;
  double dd[3];
  double invN;
  AxisDev<double2> axd[3];
  AxisDev<float2> axf[3];
  int *status;
  void *density, *potential;
  TileShape shape[5];
  int box_rows[2];   // rows per TMA box of the y and x passes
};

// Tensor map of a half spectrum (ff_solve.cu).
int encode_spectrum_map(void *base, int ni, int nj, int nh, int nhp, size_t esz, int W, int box_rows, bool xpass,
                        CUtensorMap *map);
// The two tensor maps (y boxes, x boxes) of a grid's potential.
int batch_grid_maps(const BatchGridHost &g, int precision, CUtensorMap maps[2]);

// Host helpers shared by the batch and the server (ff_batch.cu).
int batch_axis_len(const BatchGridHost &g, int kind);
int batch_tiles_of(const BatchGridHost &g, int kind);
size_t batch_shape_smem(int precision, const BatchGridHost &g, int kind, const TileShape &s);
bool batch_shape_valid(int precision, const BatchGridHost &g, int kind, const TileShape &s);
TileShape batch_default_shape(int precision, const BatchGridHost &g, int kind);
// The tuned shape for (precision, kind, axis length) if the tuner has one, else the default.
TileShape batch_shape_for(int precision, const BatchGridHost &g, int kind);
// Device bytes of one axis's tables, and their construction at mem (waits for st).
size_t batch_axis_bytes(int n, int precision);
int batch_axis_build(int n, int precision, int order, void *mem, AxisDev<double2> *ad, AxisDev<float2> *af,
                     cudaStream_t st);
// Dimensions, wavenumber scales (lo/hi: 3 values or NULL), nh/nhp, 1/N.
void batch_grid_init(BatchGridHost &h, const int n[3], const double *lo, const double *hi, int precision);
size_t batch_grid_bytes(const BatchGridHost &h, int precision);
// Axis checks of one grid (status and message as the C ABI reports them).
int batch_check_dims(const int n[3], const double *lo, const double *hi, const char *who, int g);
bool batch_z_bulk_ok(int precision, int nk);

}  // namespace ff
