// fishfry: the benchmark driver on one B200 (the reference's main.cpp:1-51
// without MPI).  Arguments as the reference: mx my mz nx ny nz [runs]
// (main.cpp:15-23); the task grid must be 1 1 1.

#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "FishFry.hpp"
#include "ParisPencil.hpp"

int main(int argc, char **argv) {
  int nTasks[] = {0, 0, 0};
  int nPoints[] = {0, 0, 0};
  int nIters = 1;
  if (argc <= 6) {
    fprintf(stderr, "usage: %s mx my mz nx ny nz [runs]\n", argv[0]);
    return 1;
  }
  for (int i = 0; i < 3; i++) nTasks[i] = atoi(argv[i + 1]);
  for (int i = 0; i < 3; i++) nPoints[i] = atoi(argv[i + 4]);
  if (argc > 7) nIters = atoi(argv[7]);
  if (nTasks[0] <= 0 || nTasks[1] <= 0 || nTasks[2] <= 0) {
    fprintf(stderr, "task counts must be positive\n");
    return 1;
  }
  if (nTasks[0] * nTasks[1] * nTasks[2] != 1) {   // main.cpp:18 asserts product == MPI size (1 here)
    fprintf(stderr, "this build runs one task on one GPU: mx*my*mz must be 1\n");
    return FF_ERR_TASKS;
  }
  if (nPoints[0] < nTasks[0] || nPoints[1] < nTasks[1] || nPoints[2] < nTasks[2]) {   // main.cpp:20
    fprintf(stderr, "points per dimension must be at least the task count\n");
    return 1;
  }
  if (nIters < 1) {
    fprintf(stderr, "runs must be at least 1\n");
    return 1;
  }
  int nd = 0;
  if (cudaGetDeviceCount(&nd) != cudaSuccess || nd < 1) {
    fprintf(stderr, "no CUDA device\n");
    return 1;
  }
  if (nd > 1) {   // main.cpp:35-44, rank 0 takes device 0
    cudaSetDevice(0);
    printf("# Task %d with node rank %d using device %d (%d devices per node)\n", 0, 0, 0, nd);
    fflush(stdout);
  }
  FishFry<ParisPencil>(nTasks, nPoints).run(nIters);
  return 0;
}
