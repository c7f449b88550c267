// Stand-in for the CUDA samples' helper_cuda.h, which the reference's
// src/main.cu includes (src/main.cu:3) and which CUDA no longer ships.  The
// reference uses only checkCudaErrors from it: report a failed runtime call
// and exit, as the samples' macro does.
#ifndef OCTMPS_BASELINE_HELPER_CUDA_H
#define OCTMPS_BASELINE_HELPER_CUDA_H

#include <cstdio>
#include <cstdlib>

#include <cuda_runtime.h>

#define checkCudaErrors(val) octmps_baseline_check((val), #val, __FILE__, __LINE__)

inline void octmps_baseline_check(cudaError_t e, const char *call, const char *file, int line) {
    if (e != cudaSuccess) {
        fprintf(stderr, "CUDA error %d (%s) at %s:%d: %s\n", (int)e, cudaGetErrorString(e), file,
                line, call);
        exit(1);
    }
}

#endif
