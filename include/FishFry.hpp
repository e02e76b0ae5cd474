// Single-GPU benchmark harness FishFry<P> (the reference's FishFry.hpp:103-246
// without MPI): sets f on the device, times P::solve, and prints per run the
// time, points/s and relative L1/L2/Linf error of phi against the analytic
// solution, then the per-phase table, in the reference's printf formats
// (FishFry.hpp:129, :198-200, :206-226).
//
// P is any class with the reference plugin interface
//   P(const int n[3], const double lo[3], const double hi[3], const int m[3], const int id[3]);
//   size_t bytes() const;
//   void solve(size_t bytes, double *density, double *potential, std::vector<TimeStamp> &stamps) const;
// With one task the MPI reductions of the reference (FishFry.hpp:153-154,
// :195-196, :220-222) are local values: min = avg = max.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <typeinfo>
#include <vector>

#include "TimeStamp.hpp"
#include "fishfry.h"

template <typename P>
class FishFry {
 public:
  FishFry(const int nTasks[3], const int nPoints[3])
      : totalPoints_(double(nPoints[0]) * double(nPoints[1]) * double(nPoints[2])),
        bytes_(0), f_(nullptr), phi_(nullptr), scales_{0, 0, 0} {
    for (int d = 0; d < 3; d++) {
      n_[d] = nPoints[d];
      dx_[d] = 2.0 * M_PI / nPoints[d];   // FishFry.hpp:109-111
      xlo_[d] = -M_PI;                    // FishFry.hpp:133, :137-139 with id = 0
    }
    printf("FishFry<%s>: %dx%dx%d points over %dx%dx%d MPI processes\n", typeid(P).name(), nPoints[0], nPoints[1],
           nPoints[2], nTasks[0], nTasks[1], nTasks[2]);
    fflush(stdout);
    const int id[] = {0, 0, 0};
    const double lo[] = {-M_PI, -M_PI, -M_PI};
    const double hi[] = {M_PI - dx_[0], M_PI - dx_[1], M_PI - dx_[2]};   // FishFry.hpp:134
    poisson_.reset(new P(nPoints, lo, hi, nTasks, id));

    bytes_ = std::max(poisson_->bytes(), size_t(n_[0]) * n_[1] * n_[2] * sizeof(double));   // FishFry.hpp:141
    check(cudaMalloc(&f_, bytes_));
    check(cudaMalloc(&phi_, bytes_));

    double s[3];
    status(ff_error_sums(n_, xlo_, dx_, 0, nullptr, FF_FP64, nullptr, s, nullptr));   // phi = 0 pass
    scales_[0] = 1.0 / s[0];
    scales_[1] = 1.0 / s[1];
    scales_[2] = 1.0 / s[2];
  }

  ~FishFry() {
    poisson_.reset();
    cudaFree(phi_);
    cudaFree(f_);
  }

  void run(const int nIters) {
    std::vector<TimeStamp> totalStamps;
    for (int i = 0; i <= nIters; i++) {
      status(ff_init_field(n_, xlo_, dx_, 0, nullptr, FF_FP64, f_, nullptr));
      check(cudaDeviceSynchronize());

      std::vector<TimeStamp> stamps;
      poisson_->solve(bytes_, f_, phi_, stamps);
      const double time = stamps.back().second - stamps.front().second;
      if (i == 0) {
        totalStamps = stamps;
        for (auto &s : totalStamps) s.second = 0;
      } else {
        for (size_t j = 0; j < stamps.size(); j++) totalStamps.at(j).second += stamps.at(j).second;
      }

      double d[3];
      status(ff_error_sums(n_, xlo_, dx_, 0, nullptr, FF_FP64, phi_, d, nullptr));
      printf("%d: Time %10.4e Rate %10.4e L_1 %10.4e L_2 %10.4e L_\\inf %10.4e", i, time, totalPoints_ / time,
             d[0] * scales_[0], sqrt(d[1] * scales_[1]), d[2] * scales_[2]);
      if (i == 0) printf(" (warmup, ignored)");
      printf("\n");
      fflush(stdout);
    }

    printf("\nTimes Averaged across Iterations\n");
    printf("Min Rank   | Avg Rank   | Max Rank   (%%Total) | Phase\n");
    printf("--------------------------------------------------------\n");
    const double perIter = 1.0 / double(nIters);
    double percent = 0;
    for (size_t i = 0; i < totalStamps.size(); i++) {
      const double dt = (i == 0) ? totalStamps.back().second - totalStamps.front().second
                                 : totalStamps[i].second - totalStamps[i - 1].second;
      const double t = perIter * dt;
      if (i == 0) percent = 100.0 / t;
      printf("%10.4e | %10.4e | %10.4e (%5.1f%%) | %s\n", t, t, t, t * percent, totalStamps[i].first.c_str());
    }
    fflush(stdout);
  }

 private:
  static void check(cudaError_t e) {
    if (e == cudaSuccess) return;
    fprintf(stderr, "CUDA ERROR: %s %s\n", cudaGetErrorName(e), cudaGetErrorString(e));
    fflush(stderr);
    exit(e);
  }
  static void status(int s) {
    if (s == FF_OK) return;
    fprintf(stderr, "FISHFRY ERROR: %s: %s\n", ff_status_string(s), ff_last_error());
    fflush(stderr);
    exit(s);
  }

  int n_[3];
  double dx_[3], xlo_[3];
  double totalPoints_;
  std::unique_ptr<P> poisson_;
  size_t bytes_;
  double *f_, *phi_;
  double scales_[3];
};
