// The batched kernels for systems of order up to 64: a CTA of 64 threads (a thread per row, as
// in batched.cu's build for n <= 256), so that eight systems run per SM instead of two and no
// thread of a CTA idles on a small system. batched.cu's plans hand these kernels the systems of
// n <= 64 and run them beside the 256-thread kernel.
#define RM_BT_NS bt64
#define RM_BT_NMAX 64
#define RM_BT_MIN_BLOCKS 8
#include "batched_kernels.cuh"
