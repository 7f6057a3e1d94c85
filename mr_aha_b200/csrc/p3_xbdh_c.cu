// Instantiations of the half-length pass 3 (passes3.cuh) for list C
// (N = 128, 64).
#include "passes3.cuh"

int mr_launch_xbdh_c(const mr_x_args &a, cudaStream_t s, bool *found) {
    const int N = a.n_in;
    *found = false;
    MR_XH_LIST_C(MR_XH_DISPATCH)
    return MR_SUCCESS;
}
