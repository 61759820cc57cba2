/* Stand-in for the CUDA-samples header that the reference includes
 * (the samples tree is not installed in this image).  Only the one macro the
 * reference uses (plus two printing helpers) is provided.  Part of the oracle build recipe; test
 * infrastructure only. */
#ifndef GNSS_REFSHIM_HELPER_CUDA_H
#define GNSS_REFSHIM_HELPER_CUDA_H
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#define checkCudaErrors(val)                                                            \
    do {                                                                                \
        cudaError_t e_ = (val);                                                         \
        if (e_ != cudaSuccess) {                                                        \
            std::fprintf(stderr, "CUDA error %d (%s) at %s:%d\n", (int)e_,               \
                         cudaGetErrorString(e_), __FILE__, __LINE__);                   \
            std::exit(1);                                                               \
        }                                                                               \
    } while (0)
/* used only for printing device properties (iofuncs.cu:21-51) */
#ifndef SPRINTF
#define SPRINTF sprintf
#endif
static inline int _ConvertSMVer2Cores(int major, int minor) {
    (void)minor;
    return major >= 8 ? 128 : 64;   /* informational only */
}
#endif
