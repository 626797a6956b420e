/* A C caller of libxk.so, compiled by the tests with gcc against include/xk.h.
 *
 *   xk_abi_check <case file>
 *
 * The case file holds whitespace-separated numbers: n_rays, then the 12 ray
 * columns (x y z nx ny nz nl es_re es_im ep_re ep_im energy) of n_rays values
 * each, then n_pix and the 3 pixel columns. The program prints the library
 * version, then either "no-device" (xk_init and xk_kirchhoff_auto both report
 * XK_ERR_NO_DEVICE) or, per pixel, the field of xk_diffraction_integral on
 * XK_PATH_F64 and XK_PATH_F32PR and of xk_kirchhoff_gpu on the f32 records
 * ("f64 i es_re es_im ep_re ep_im", "f32pr ...", "gpu ..."). Exit status 0
 * on success, 1 on any unexpected status. */
#include <stdio.h>
#include <stdlib.h>

#include "xk.h"

static double* read_col(FILE* f, size_t n) {
    double* v = (double*)calloc(n ? n : 1, sizeof(double));
    for (size_t i = 0; i < n; ++i)
        if (fscanf(f, "%lf", &v[i]) != 1) {
            fprintf(stderr, "short case file\n");
            exit(1);
        }
    return v;
}

static int fail(const char* what, int rc, const xk_ctx* ctx) {
    fprintf(stderr, "%s: status %d (%s) %s\n", what, rc, xk_status_string(rc),
            ctx ? xk_last_error(ctx) : "");
    return 1;
}

static void print_field(const char* tag, size_t m, const xk_field* f) {
    for (size_t i = 0; i < m; ++i)
        printf("%s %zu %.17g %.17g %.17g %.17g\n", tag, i, f->es_re[i], f->es_im[i],
               f->ep_re[i], f->ep_im[i]);
}

int main(int argc, char** argv) {
    if (argc != 2) {
        fprintf(stderr, "usage: %s case-file\n", argv[0]);
        return 2;
    }
    FILE* f = fopen(argv[1], "r");
    if (!f) {
        perror(argv[1]);
        return 2;
    }
    size_t n = 0, m = 0;
    if (fscanf(f, "%zu", &n) != 1) return 2;
    double* rc[12];
    for (int c = 0; c < 12; ++c) rc[c] = read_col(f, n);
    if (fscanf(f, "%zu", &m) != 1) return 2;
    double* pc[3];
    for (int c = 0; c < 3; ++c) pc[c] = read_col(f, m);
    fclose(f);

    printf("version %s\n", xk_version());
    xk_rays rays = {rc[0], rc[1], rc[2], rc[3], rc[4], rc[5], rc[6],
                    rc[7], rc[8], rc[9], rc[10], rc[11]};
    xk_pixels pix = {pc[0], pc[1], pc[2]};

    /* GpuRay / GpuPixel records (src/gpu/kirchhoff.rs:20-45) of the same case. */
    xk_gpu_ray* gr = (xk_gpu_ray*)calloc(n ? n : 1, sizeof(xk_gpu_ray));
    xk_gpu_pixel* gp = (xk_gpu_pixel*)calloc(m ? m : 1, sizeof(xk_gpu_pixel));
    for (size_t i = 0; i < n; ++i) {
        xk_gpu_ray r = {(float)rc[0][i], (float)rc[1][i],  (float)rc[2][i], (float)rc[3][i],
                        (float)rc[4][i], (float)rc[5][i],  (float)rc[6][i], (float)rc[11][i],
                        (float)rc[7][i], (float)rc[8][i],  (float)rc[9][i], (float)rc[10][i]};
        gr[i] = r;
    }
    for (size_t i = 0; i < m; ++i) {
        xk_gpu_pixel p = {(float)pc[0][i], (float)pc[1][i], (float)pc[2][i], 0.0f};
        gp[i] = p;
    }
    double* gout = (double*)calloc(4 * (m ? m : 1), sizeof(double));

    xk_ctx* ctx = NULL;
    int st = xk_init(0, &ctx);
    if (st == XK_ERR_NO_DEVICE) {
        int st2 = xk_kirchhoff_auto(gr, n, gp, m, gout);
        if (st2 != XK_ERR_NO_DEVICE) return fail("xk_kirchhoff_auto without a device", st2, NULL);
        printf("no-device\n");
        return 0;
    }
    if (st != XK_OK) return fail("xk_init", st, NULL);
    printf("device %s\n", xk_device_name(ctx));

    double* o[4];
    for (int c = 0; c < 4; ++c) o[c] = (double*)calloc(m ? m : 1, sizeof(double));
    xk_field field = {o[0], o[1], o[2], o[3]};
    const int paths[2] = {XK_PATH_F64, XK_PATH_F32PR};
    const char* tags[2] = {"f64", "f32pr"};
    for (int k = 0; k < 2; ++k) {
        xk_stats stats;
        st = xk_diffraction_integral(ctx, &rays, n, &pix, m, &field, paths[k], &stats);
        if (st != XK_OK) return fail("xk_diffraction_integral", st, ctx);
        print_field(tags[k], m, &field);
    }
    st = xk_kirchhoff_gpu(ctx, gr, n, gp, m, gout);
    if (st != XK_OK) return fail("xk_kirchhoff_gpu", st, ctx);
    for (size_t i = 0; i < m; ++i)
        printf("gpu %zu %.17g %.17g %.17g %.17g\n", i, gout[4 * i], gout[4 * i + 1],
               gout[4 * i + 2], gout[4 * i + 3]);
    /* A mismatched call is refused with a status, not a crash. */
    st = xk_diffraction_integral(ctx, NULL, n, &pix, m, &field, XK_PATH_F64, NULL);
    if (st != XK_ERR_INVALID) return fail("null rays not refused", st, ctx);
    xk_destroy(ctx);
    printf("done\n");
    return 0;
}
