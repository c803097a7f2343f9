/* cholqr2! through the C ABI from plain C: what a `ccall` binding does, with
 * no Python in between. Builds a seeded N x k ComplexF64 matrix with a column
 * scale (condition about 1e3), orthonormalizes it on the device with
 * fb_zcholqr2 and, from page-locked host panels, with fb_zcholqr2_staged,
 * and checks ||Q^H Q - I||_F <= 1e-12, ||Y - Q R||_F / ||Y||_F <= 1e-13 and
 * that the two paths agree to the bit. Also checks the statuses of bad
 * arguments. Without a device it checks the statuses only.
 * Exit status 0 on success. */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "funicular_b200.h"

#define CHECK(call)                                                                      \
    do {                                                                                 \
        int st_ = (call);                                                                \
        if (st_ != FB_OK) {                                                              \
            fprintf(stderr, "%s:%d: %s -> %d (%s)\n", __FILE__, __LINE__, #call, st_,   \
                    fb_last_error());                                                    \
            return 1;                                                                    \
        }                                                                                \
    } while (0)

static uint64_t lcg = 0x9E3779B97F4A7C15ull;
static double uniform(void) {
    lcg = lcg * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(lcg >> 11) * 0x1.0p-53 - 0.5;
}

static int statuses_without_work(void) {
    fb_z128 one = {1.0, 0.0};
    if (fb_zgram(NULL, 1, NULL, 1, NULL, 1, -1, 2, 2, one, one, NULL, 0, NULL) != FB_EDIM) return 1;
    if (fb_last_error()[0] == '\0') return 1;
    if (fb_ztrsm_right_upper(NULL, 1, -3, 2, NULL, 1, NULL, 0, NULL) != FB_EDIM) return 1;
    if (fb_zcholqr2(NULL, 1, 0, 4, NULL, 4, NULL, NULL, NULL, 0, NULL) != FB_EINVAL) return 1;
    int blocks = 0;
    CHECK(fb_zcholqr2_staged_blocks(10000000, 64, &blocks));
    if (blocks < 1 || blocks > 8) return 1;
    return 0;
}

int main(void) {
    if (fb_abi_version() != FB_ABI_VERSION) { fprintf(stderr, "ABI version\n"); return 1; }
    if (statuses_without_work()) { fprintf(stderr, "status checks failed\n"); return 1; }
    int devices = 0;
    CHECK(fb_device_count(&devices));
    if (devices == 0) { printf("statuses ok, no device\n"); return 0; }

    const int64_t N = 200003;
    const int k = 24, w = 8, npanels = 3;
    const size_t bytes = (size_t)N * k * sizeof(fb_z128);
    fb_z128* A = malloc(bytes);
    for (int j = 0; j < k; ++j) {
        const double scale = pow(10.0, -3.0 * j / (k - 1));
        for (int64_t i = 0; i < N; ++i) A[i + j * N] = (fb_z128){scale * uniform(), scale * uniform()};
    }
    void *Yd, *Rd, *Y2, *R2, *ws, *slab;
    CHECK(fb_alloc_device(&Yd, bytes));
    CHECK(fb_alloc_device(&Y2, bytes));
    CHECK(fb_alloc_device(&Rd, (size_t)k * k * sizeof(fb_z128)));
    CHECK(fb_alloc_device(&R2, (size_t)k * k * sizeof(fb_z128)));
    size_t wbytes = 0, sbytes = 0;
    CHECK(fb_zcholqr2_workspace_size(N, k, &wbytes));
    CHECK(fb_zcholqr2_staged_workspace_size(N, k, FB_C128, &sbytes));
    if (sbytes > wbytes) wbytes = sbytes;
    CHECK(fb_alloc_device(&ws, wbytes + 256));
    void* wsa = (void*)(((uintptr_t)ws + 255) & ~(uintptr_t)255);

    /* Device-resident chain. */
    CHECK(fb_copy2d(Yd, N * sizeof(fb_z128), A, N * sizeof(fb_z128), N * sizeof(fb_z128), k, NULL));
    int info = -1, passes = 0;
    CHECK(fb_zcholqr2((fb_z128*)Yd, N, N, k, (fb_z128*)Rd, k, &info, &passes, wsa, wbytes, NULL));
    fb_z128* Q = malloc(bytes);
    fb_z128* R = malloc((size_t)k * k * sizeof(fb_z128));
    CHECK(fb_copy2d(Q, N * sizeof(fb_z128), Yd, N * sizeof(fb_z128), N * sizeof(fb_z128), k, NULL));
    CHECK(fb_copy2d(R, k * sizeof(fb_z128), Rd, k * sizeof(fb_z128), k * sizeof(fb_z128), k, NULL));

    /* The same matrix in page-locked panels of width 8, staged. */
    CHECK(fb_alloc_host_slab(&slab, bytes));
    fb_z128* P = slab;
    memcpy(P, A, bytes);
    fb_z128* panels[3];
    int64_t lds[3];
    int cols[3];
    for (int p = 0; p < npanels; ++p) { panels[p] = P + (int64_t)p * w * N; lds[p] = N; cols[p] = w; }
    int info2 = -1, passes2 = 0;
    CHECK(fb_zcholqr2_staged((void* const*)panels, FB_C128, lds, cols, npanels, (fb_z128*)Y2, N, N, k,
                             (fb_z128*)R2, k, 0.0, &info2, &passes2, wsa, wbytes, NULL));
    fb_z128* Rs = malloc((size_t)k * k * sizeof(fb_z128));
    CHECK(fb_copy2d(Rs, k * sizeof(fb_z128), R2, k * sizeof(fb_z128), k * sizeof(fb_z128), k, NULL));
    if (memcmp(P, Q, bytes) != 0 || memcmp(Rs, R, (size_t)k * k * sizeof(fb_z128)) != 0) {
        fprintf(stderr, "staged and resident results differ\n");
        return 1;
    }

    /* ||Q^H Q - I||_F and ||A - Q R||_F / ||A||_F on the host. */
    double orth = 0.0;
    for (int a = 0; a < k; ++a)
        for (int b = 0; b < k; ++b) {
            double re = 0.0, im = 0.0;
            for (int64_t i = 0; i < N; ++i) {
                const fb_z128 x = Q[i + a * N], y = Q[i + b * N];
                re += x.re * y.re + x.im * y.im;
                im += x.re * y.im - x.im * y.re;
            }
            re -= (a == b);
            orth += re * re + im * im;
        }
    orth = sqrt(orth);
    double num = 0.0, den = 0.0;
    for (int64_t i = 0; i < N; ++i)
        for (int j = 0; j < k; ++j) {
            double re = 0.0, im = 0.0;
            for (int l = 0; l <= j; ++l) {
                const fb_z128 q = Q[i + l * N], r = R[l + j * k];
                re += q.re * r.re - q.im * r.im;
                im += q.re * r.im + q.im * r.re;
            }
            const fb_z128 y = A[i + j * N];
            num += (y.re - re) * (y.re - re) + (y.im - im) * (y.im - im);
            den += y.re * y.re + y.im * y.im;
        }
    const double recon = sqrt(num / den);
    printf("info %d passes %d orth %.3e recon %.3e\n", info, passes, orth, recon);
    if (info != 0 || passes != 2 || info2 != 0 || !(orth <= 1e-12) || !(recon <= 1e-13)) return 1;
    CHECK(fb_free_device(Yd));
    CHECK(fb_free_device(Y2));
    CHECK(fb_free_device(Rd));
    CHECK(fb_free_device(R2));
    CHECK(fb_free_device(ws));
    CHECK(fb_free_host_slab(slab));
    free(A); free(Q); free(R); free(Rs);
    return 0;
}
