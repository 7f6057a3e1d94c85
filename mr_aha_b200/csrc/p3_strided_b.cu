// Instantiations of the specialised strided passes for the lengths of list B
// (passes3.cuh): the grids of uneven batches (256, 384, 512 points in plane,
// 8 to 32 along z).
#include "passes3.cuh"

int mr_launch_strided3_b(int dir, int lmode, int smode, const mr_strided_args &a,
                         cudaStream_t s, bool *found) {
    const int M = a.ax.M, XT = a.xt;
    *found = false;
    MR_S3_LIST_B(MR_S3_DISPATCH)
    return MR_SUCCESS;
}
