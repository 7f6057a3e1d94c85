// Passes with a compile-time-specialised FFT (fftfix.cuh) for the common
// lengths of the plans: the same data flow as the in-place kernels of
// passes2.cu, with the transform length, tile width / coil count and rank as
// template parameters. The plan uses these kernels when its geometry matches
// an instantiated configuration (mr_fixed_*), else the generic ones. Kernel
// templates and configuration lists: passes3.cuh.
#include "passes3.cuh"


namespace {
// Shared memory a tile may take: half the per-block limit (two CTAs per SM)
// unless MR_AHA_B200_FULL_TILES is set.
size_t tile_budget(bool half) { return (size_t)mr_smem_limit() / (half ? 2 : 1); }
bool half_tiles() { return mr_env_int("MR_AHA_B200_FULL_TILES", 0) == 0; }
}  // namespace

int mr_fixed_strided_xt(int M, int smode, int want) {
    // `want` when it is instantiated and fits; else the widest instantiated
    // tile of this length for the store mode within the tile budget, the
    // full limit when no tile fits half of it
    int best = 0;
    if (want > 0) {
#define MR_S3_WANT(m, xt)                                                      \
        if (M == m && want == xt &&                                            \
            (size_t)m * xt * sizeof(float2) * (smode == MR_SM_COILSUM ? 2 : 1) <= \
                (size_t)mr_smem_limit())                                       \
            return xt;
        MR_S3_LIST(MR_S3_WANT)
#undef MR_S3_WANT
    }
    for (int pass = 0; pass < 2 && best == 0; ++pass) {
        const size_t budget = tile_budget(pass == 0 && half_tiles());
#define MR_S3_PICK(m, xt)                                                 \
        if (M == m) {                                                     \
            size_t b = (size_t)m * xt * sizeof(float2);                   \
            if (smode == MR_SM_COILSUM) b += (size_t)m * xt * sizeof(float2); \
            if (b <= budget && xt > best) best = xt;                      \
        }
        MR_S3_LIST(MR_S3_PICK)
#undef MR_S3_PICK
    }
    return best;
}

int mr_launch_strided3(int dir, int lmode, int smode, const mr_strided_args &a, cudaStream_t s) {
    const int M = a.ax.M, XT = a.xt;
    bool fnd = false;
    bool *found = &fnd;
    MR_S3_LIST_A(MR_S3_DISPATCH)
    const int rc = mr_launch_strided3_b(dir, lmode, smode, a, s, found);
    if (fnd) return rc;
    MR_FAIL(MR_ERR_INTERNAL, "no specialised strided pass for M = %d, tile %d", M, XT);
}

int mr_fixed_xbd_coils(int M, int L) {
    // the most coils per tile within the tile budget (as above)
    int nc = 0;
    for (int pass = 0; pass < 2 && nc == 0; ++pass) {
        const size_t budget = tile_budget(pass == 0 && half_tiles());
#define MR_X3_PICK(m, l, c)                                                         \
        if (M == m && L == l && (size_t)c * l * odd_stride<m>() * sizeof(float2) <= budget && \
            c > nc)                                                                 \
            nc = c;
        MR_X3_LIST(MR_X3_PICK)
#undef MR_X3_PICK
    }
    return nc;
}

int mr_launch_xbd3(const mr_x_args &a, cudaStream_t s) {
    const int M = a.ax.M;
#define MR_X3_CASE(m, l, c)                                                     \
    if (M == m && a.L == l && a.nc == c) {                                      \
        switch (a.K.kf) {                                                       \
            case MR_KF_F32: return launch_x3<m, l, c, MR_KF_F32>(a, s);         \
            case MR_KF_BF16: return launch_x3<m, l, c, MR_KF_BF16>(a, s);       \
            default: return launch_x3<m, l, c, MR_KF_I16>(a, s);                \
        }                                                                       \
    }
    MR_X3_LIST(MR_X3_CASE)
#undef MR_X3_CASE
    MR_FAIL(MR_ERR_INTERNAL, "no specialised block-diagonal pass for M = %d, L = %d", M, a.L);
}

int mr_fixed_xbdh_coils(int M, int n_in, int L) {
    if (M != 2 * n_in || mr_env_int("MR_AHA_B200_NO_HALF", 0)) return 0;
    const int N = n_in;
    int nc = 0;
#define MR_XH_PICK(n, l, c)                                                                  \
    if (N == n && L == l && (size_t)2 * c * l * odd_stride<n>() * sizeof(float2) <=          \
                                (size_t)mr_smem_limit() && c > nc)                           \
        nc = c;
    MR_XH_LIST(MR_XH_PICK)
#undef MR_XH_PICK
    return nc;
}

int mr_launch_xbdh(const mr_x_args &a, cudaStream_t s) {
    const int N = a.n_in;
    if (a.ax.M != 2 * N || a.n_out != N || a.shift_out != a.shift_in)
        MR_FAIL(MR_ERR_INTERNAL, "half-length block-diagonal pass needs M = 2 N and equal windows");
    bool fnd = false;
    bool *found = &fnd;
    MR_XH_LIST_A(MR_XH_DISPATCH)
    int rc = mr_launch_xbdh_b(a, s, found);
    if (fnd) return rc;
    rc = mr_launch_xbdh_c(a, s, found);
    if (fnd) return rc;
    MR_FAIL(MR_ERR_INTERNAL, "no half-length block-diagonal pass for N = %d, L = %d", N, a.L);
}

int mr_fixed_strided_list(int M, int smode, int *xt, int max) {
    // every instantiated tile width of this length that fits the per-block
    // shared memory limit, for the autotuner
    int n = 0;
#define MR_S3_LISTPICK(m, w)                                                                \
    if (M == m && n < max &&                                                                \
        (size_t)m * w * sizeof(float2) * (smode == MR_SM_COILSUM ? 2 : 1) <=                \
            (size_t)mr_smem_limit())                                                        \
        xt[n++] = w;
    MR_S3_LIST(MR_S3_LISTPICK)
#undef MR_S3_LISTPICK
    return n;
}

int mr_fixed_xbd_list(int M, int L, int *nc, int max) {
    int n = 0;
#define MR_X3_LISTPICK(m, l, c)                                                             \
    if (M == m && L == l && n < max &&                                                      \
        (size_t)c * l * odd_stride<m>() * sizeof(float2) <= (size_t)mr_smem_limit())        \
        nc[n++] = c;
    MR_X3_LIST(MR_X3_LISTPICK)
#undef MR_X3_LISTPICK
    return n;
}
