// post.cu -- the IEEE post-processing kernels (post_kernels.cuh) and the
// launch entry, which hands CR_POST_FAST_MATH passes to post_fast.cu.
#include "post_kernels.cuh"

int cr_launch_post_fast(const CrPostParams& p, void* stream);

int cr_launch_post(const CrPostParams& p, void* stream) {
    if (p.fast) return cr_launch_post_fast(p, stream);
    launch_post<false>(p, (cudaStream_t)stream);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
