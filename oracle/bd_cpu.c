/*
 * CPU restatement (FP32, OpenMP) of the packed Hermitian block multiply of
 * the Toeplitz apply, for the timed CPU baseline. TEST / MEASUREMENT
 * INFRASTRUCTURE ONLY: the shipped library never links this file.
 *
 * At every location q, the rank row vector v of one coil is multiplied from
 * the right by the Hermitian block of that location, y_c = sum_r v_r A_rc,
 * with A held as one packed triangle whose component t is element (r, c)
 * (lower: t = c*L - c*(c-1)/2 + (r - c), r >= c; upper: t = c*(c+1)/2 + r,
 * r <= c), following the reference's src/cuda/mr_kernels_bd.cu:56-139 and
 * include/mr_aha/mr_aha.h:300-317. Arrays are interleaved complex64:
 * v, y: [L][nloc]; K: [ntri][nloc] (already in the spectrum's index order).
 */
#include <stdint.h>
#include <string.h>

void bd_cpu_apply(const float *v, float *y, const float *K, int64_t nloc, int L, int upper) {
    const int64_t ntri = (int64_t)L * (L + 1) / 2;
#pragma omp parallel for schedule(static)
    for (int64_t q = 0; q < nloc; ++q) {
        float vr[512][2], yr[512][2];
        for (int l = 0; l < L; ++l) {
            vr[l][0] = v[2 * (l * nloc + q)];
            vr[l][1] = v[2 * (l * nloc + q) + 1];
            yr[l][0] = 0.f;
            yr[l][1] = 0.f;
        }
        int64_t t = 0;
        for (int c = 0; c < L; ++c) {
            const int r0 = upper ? 0 : c;
            const int r1 = upper ? c + 1 : L;
            for (int r = r0; r < r1; ++r, ++t) {
                const float ar = K[2 * (t * nloc + q)], ai = K[2 * (t * nloc + q) + 1];
                /* y_c += a v_r */
                yr[c][0] += ar * vr[r][0] - ai * vr[r][1];
                yr[c][1] += ar * vr[r][1] + ai * vr[r][0];
                if (r != c) { /* y_r += conj(a) v_c */
                    yr[r][0] += ar * vr[c][0] + ai * vr[c][1];
                    yr[r][1] += ar * vr[c][1] - ai * vr[c][0];
                }
            }
        }
        (void)ntri;
        for (int l = 0; l < L; ++l) {
            y[2 * (l * nloc + q)] = yr[l][0];
            y[2 * (l * nloc + q) + 1] = yr[l][1];
        }
    }
}
