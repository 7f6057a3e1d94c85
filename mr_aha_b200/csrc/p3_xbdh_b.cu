// Instantiations of the half-length pass 3 (passes3.cuh) for list B
// (N = 256, 192).
#include "passes3.cuh"

int mr_launch_xbdh_b(const mr_x_args &a, cudaStream_t s, bool *found) {
    const int N = a.n_in;
    *found = false;
    MR_XH_LIST_B(MR_XH_DISPATCH)
    return MR_SUCCESS;
}
