// post_fast.cu -- the fast-math post-processing kernels (post_kernels.cuh
// with FAST): this file is compiled with --use_fast_math, the recipe the
// reference builds its own post kernels with (CudaModularProgram.h:133-157),
// so contractions and approximations follow that build.
#include "post_kernels.cuh"

int cr_launch_post_fast(const CrPostParams& p, void* stream) {
    launch_post<true>(p, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
