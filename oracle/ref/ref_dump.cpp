// Runs the reference's own solve on one GPU and writes f and phi to a file:
// the reference's ParisPencil (compiled from its ParisPencil.cpp) and its
// FishFry.hpp init kernel, set up exactly as FishFry's constructor does
// (FishFry.hpp:108-139) for a 1x1x1 task grid.  Test infrastructure only.
//   ref_dump nx ny nz out.bin     -> int32 n[3], float64 f[N], float64 phi[N]
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "FishFry.hpp"
#include "ParisPencil.hpp"

int main(int argc, char **argv) {
  if (argc < 5) {
    fprintf(stderr, "usage: %s nx ny nz out.bin\n", argv[0]);
    return 1;
  }
  const int n[3] = {atoi(argv[1]), atoi(argv[2]), atoi(argv[3])};
  const int m[3] = {1, 1, 1}, id[3] = {0, 0, 0};
  const double dx[3] = {2.0 * M_PI / n[0], 2.0 * M_PI / n[1], 2.0 * M_PI / n[2]};
  const double lo[3] = {-M_PI, -M_PI, -M_PI};
  const double hi[3] = {M_PI - dx[0], M_PI - dx[1], M_PI - dx[2]};
  ParisPencil p(n, lo, hi, m, id);
  const size_t N = size_t(n[0]) * n[1] * n[2];
  const size_t bytes = std::max(p.bytes(), N * sizeof(double));
  double *f = nullptr, *phi = nullptr;
  CHECK(cudaMalloc(&f, bytes));
  CHECK(cudaMalloc(&phi, bytes));
  const dim3 nt(8, 8, 8);
  const dim3 nb((n[2] + 7) / 8, (n[1] + 7) / 8, (n[0] + 7) / 8);
  init<<<nb, nt>>>(n[0], n[1], n[2], lo[0], lo[1], lo[2], dx[0], dx[1], dx[2], f);
  CHECK(cudaGetLastError());
  CHECK(cudaDeviceSynchronize());
  std::vector<double> hf(N), hp(N);
  CHECK(cudaMemcpy(hf.data(), f, N * sizeof(double), cudaMemcpyDeviceToHost));
  std::vector<TimeStamp> stamps;
  p.solve(bytes, f, phi, stamps);
  CHECK(cudaMemcpy(hp.data(), phi, N * sizeof(double), cudaMemcpyDeviceToHost));
  FILE *o = fopen(argv[4], "wb");
  if (!o) return 2;
  fwrite(n, sizeof(int), 3, o);
  fwrite(hf.data(), sizeof(double), N, o);
  fwrite(hp.data(), sizeof(double), N, o);
  fclose(o);
  printf("ref_dump %dx%dx%d solve %.4e s\n", n[0], n[1], n[2], stamps.back().second - stamps.front().second);
  CHECK(cudaFree(phi));
  CHECK(cudaFree(f));
  return 0;
}
