// Instantiations of the half-length strided passes (passes3.cuh): y lines of
// M = 2N points that read (forward) or write (inverse) only the N image rows.
#include "passes3.cuh"

int mr_half_strided_xt(int N, int want) {
    // `want` when instantiated, else the widest instantiated tile of this
    // length within half the shared memory (two CTAs per SM); 0 if none
    if (mr_env_int("MR_AHA_B200_NO_HALF", 0) || mr_env_int("MR_AHA_B200_NO_FIXED", 0)) return 0;
    int best = 0;
#define MR_SH_PICK(n, xt)                                                                    \
    if (N == n) {                                                                            \
        if (want == xt) return xt;                                                           \
        if ((size_t)2 * n * xt * sizeof(float2) <= (size_t)mr_smem_limit() / 2 && xt > best) \
            best = xt;                                                                       \
    }
    MR_SH_LIST(MR_SH_PICK)
#undef MR_SH_PICK
    return best;
}

int mr_half_strided_list(int N, int *xt, int max) {
    int n = 0;
#define MR_SH_LISTPICK(nn, w) \
    if (N == nn && n < max) xt[n++] = w;
    MR_SH_LIST(MR_SH_LISTPICK)
#undef MR_SH_LISTPICK
    return n;
}

int mr_launch_strided_half(int dir, const mr_strided_args &a, cudaStream_t s) {
    const int N = a.ax.M / 2, XT = a.xt;
    if (a.ax.M != 2 * N || (dir < 0 ? a.n_in : a.n_out) != N)
        MR_FAIL(MR_ERR_INTERNAL, "half-length strided pass needs M = 2N image rows");
#define MR_SH_CASE(n, xt)                                                      \
    if (N == n && XT == xt) {                                                  \
        return dir < 0 ? launch_sh<-1, n, xt>(a, s) : launch_sh<1, n, xt>(a, s); \
    }
    MR_SH_LIST(MR_SH_CASE)
#undef MR_SH_CASE
    MR_FAIL(MR_ERR_INTERNAL, "no half-length strided pass for N = %d, tile %d", N, XT);
}
