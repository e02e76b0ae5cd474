// Drop-in replacement of the reference's ParisPencil solver plugin
// (ParisPencil.hpp:11-59) for one B200: same constructor, bytes() and solve()
// signatures, implemented over the fishfry_b200 C ABI (fishfry.h).
//
// Differences a caller can see, all on the single-GPU path:
//   * the task grid m must be 1x1x1 and id 0,0,0 (no MPI decomposition);
//   * stamps hold "Total" plus one entry per device pass.  As in the
//     reference (MPI_Wtime before the first phase and after the final
//     cudaDeviceSynchronize, ParisPencil.cpp:98, :424), stamps.back() -
//     stamps.front() is the host wall time of the whole solve, launches and
//     synchronisation included.  The phases in between are placed by their
//     CUDA-event durations (the solve synchronises once, not after every
//     phase), so the last phase's share also carries that host overhead;
//   * failures print the message and exit with the status code, as the
//     reference's CHECK does (gpu.hpp:69-87).
#pragma once

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <utility>
#include <vector>

#include "TimeStamp.hpp"
#include "fishfry.h"

class ParisPencil {
 public:
  // n: global points per dimension; lo/hi: physical bounds with hi one cell
  // short of the period; m: task grid (must be 1x1x1); id: task coordinates.
  ParisPencil(const int n[3], const double lo[3], const double hi[3], const int m[3], const int id[3])
      : plan_(nullptr), bytes_(0) {
    if (m[0] != 1 || m[1] != 1 || m[2] != 1 || id[0] != 0 || id[1] != 0 || id[2] != 0)
      fail(FF_ERR_TASKS, "ParisPencil: this build runs one task on one GPU (m must be 1x1x1)");
    check(ff_plan_create(n, lo, hi, FF_FP64, &plan_), __LINE__);
    check(ff_plan_bytes(plan_, &bytes_), __LINE__);
  }

  ~ParisPencil() { ff_plan_destroy(plan_); }

  ParisPencil(const ParisPencil &) = delete;
  ParisPencil &operator=(const ParisPencil &) = delete;

  // Bytes needed for each of the density and potential arrays.
  size_t bytes() const { return bytes_; }

  // Solves lap(potential) = density on the periodic grid.  density and
  // potential are device arrays of at least bytes() bytes; density is used as
  // a work array.  Blocks until the result is in potential.
  void solve(size_t bytes, double *density, double *potential, std::vector<TimeStamp> &stamps) const {
    stamps.clear();
    const double t0 = wtime();
    stamps.push_back({"Total", t0});
    ff_phase_times times;
    check(ff_solve(plan_, bytes, density, potential, nullptr, &times), __LINE__);
    const double t1 = wtime();   // after the solve's synchronisation
    double t = t0;
    for (int p = 0; p < times.count; p++) {
      t += 1e-3 * times.ms[p];
      stamps.push_back({ff_phase_name(plan_, p), p + 1 == times.count ? std::max(t, t1) : t});
    }
  }

 private:
  static double wtime() {
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
  }
  [[noreturn]] static void fail(int status, const char *msg) {
    fprintf(stderr, "%s\n", msg);
    fflush(stderr);
    exit(status);
  }
  static void check(int status, int line) {
    if (status == FF_OK) return;
    fprintf(stderr, "FISHFRY ERROR AT LINE %d OF FILE '%s': %s: %s\n", line, __FILE__, ff_status_string(status),
            ff_last_error());
    fflush(stderr);
    exit(status);
  }

  ff_plan *plan_;
  size_t bytes_;
};
