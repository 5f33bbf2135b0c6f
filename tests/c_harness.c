/* A plain C caller of the library's C ABI (include/inmsom_gpu.h), with
 * Fortran-layout arrays (column-major, 1-based positions in the argument
 * lists), as a Fortran or C host program would call it: no Python, no
 * torch.  It runs without a GPU: the device entry point must fail cleanly
 * with INMSOM_ECUDA and a message (or, with a device, succeed and be
 * finalised); the host-side entries run end to end:
 *   wdstd8 -> rdstd8 (Service/input_output_data.f90:329-527),
 *   ctl_file_write -> ctl_file_read (Service/rw_ctl_file.f90:1-566),
 *   pwdstd by two row strips == wdstd of the whole field (:206-327, 657-819),
 *   the error code and message of a missing file.
 * Usage: c_harness <scratch directory>; prints "ok" and exits 0. */
#include "inmsom_gpu.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define NX 14
#define NY 11
#define NZ 3

static int failures = 0;
#define CHECK(cond, what)                                                        \
    do {                                                                         \
        if (!(cond)) {                                                           \
            fprintf(stderr, "FAIL line %d: %s (%s)\n", __LINE__, what,           \
                    inmsom_gpu_last_error());                                    \
            failures++;                                                          \
        }                                                                        \
    } while (0)

/* field(i, j, k), 1-based */
#define AT(f, i, j, k) (f)[((i) - 1) + NX * (((j) - 1) + NY * ((k) - 1))]
#define LU(i, j) lu[((i) - 1) + NX * ((j) - 1)]

static long file_size(const char *path)
{
    FILE *f = fopen(path, "rb");
    long n;
    if (!f) return -1;
    fseek(f, 0, SEEK_END);
    n = ftell(f);
    fclose(f);
    return n;
}

static int same_files(const char *a, const char *b)
{
    FILE *fa = fopen(a, "rb"), *fb = fopen(b, "rb");
    int ca, cb, same = fa && fb;
    while (same) {
        ca = fgetc(fa);
        cb = fgetc(fb);
        if (ca != cb) same = 0;
        if (ca == EOF || cb == EOF) break;
    }
    if (fa) fclose(fa);
    if (fb) fclose(fb);
    return same;
}

int main(int argc, char **argv)
{
    static double field[NX * NY * NZ], back[NX * NY * NZ];
    static float lu[NX * NY], f4[NX * NY * NZ], strip[NX * NY * NZ];
    char path[1024];
    int i, j, k, rc;
    if (argc < 2) {
        fprintf(stderr, "usage: %s <scratch directory>\n", argv[0]);
        return 2;
    }
    const char *dir = argv[1];

    /* the device entry: a serial 10 x 7 basin, arrays 1..14 x 1..11 */
    {
        inmsom_bounds b = {3, 12, 3, 9, 1, 14, 1, 11, 3, 12, 3, 9, 0, 0};
        inmsom_consts c = {0.05, 9.8, 1025.0, 1};
        inmsom_ctx *ctx = NULL;
        rc = inmsom_gpu_init(&ctx, &b, &c, 0, 0);
        if (rc == INMSOM_OK) {
            CHECK(inmsom_gpu_finalize(ctx) == INMSOM_OK, "finalize");
            printf("device present\n");
        } else {
            CHECK(rc == INMSOM_ECUDA, "init without a device returns INMSOM_ECUDA");
            CHECK(strlen(inmsom_gpu_last_error()) > 0, "init without a device leaves a message");
        }
        CHECK(inmsom_gpu_init(NULL, &b, &c, 0, 0) == INMSOM_EARG, "init with no context pointer");
    }

    /* wdstd8 -> rdstd8 of levels 1..3 of the interior box 3..12 x 3..9 */
    for (k = 1; k <= NZ; k++)
        for (j = 1; j <= NY; j++)
            for (i = 1; i <= NX; i++) AT(field, i, j, k) = sin(0.37 * i + 1.3 * j) * (k + 0.25);
    for (j = 1; j <= NY; j++)
        for (i = 1; i <= NX; i++) LU(i, j) = ((i * 7 + j * 3) % 5 == 0) ? 0.0f : 1.0f;
    memcpy(back, field, sizeof field);
    CHECK(inmsom_wdstd8(dir, "h8.dat", 2, field, lu, NX, NY, NZ, 3, 12, 3, 9, 1, NZ) == INMSOM_OK, "wdstd8");
    snprintf(path, sizeof path, "%s/h8.dat", dir);
    CHECK(file_size(path) == 2L * NZ * 10 * 7 * 8, "two fields of three 10 x 7 FP64 records");
    for (k = 1; k <= NZ; k++)
        for (j = 3; j <= 9; j++)
            for (i = 3; i <= 12; i++) AT(back, i, j, k) = -5.0;
    CHECK(inmsom_rdstd8(dir, "h8.dat", 2, back, lu, NX, NY, NZ, 3, 12, 3, 9, 1, NZ) == INMSOM_OK, "rdstd8");
    for (k = 1; k <= NZ; k++)
        for (j = 1; j <= NY; j++)
            for (i = 1; i <= NX; i++) {
                const int inbox = i >= 3 && i <= 12 && j >= 3 && j <= 9;
                const double want = inbox && LU(i, j) < 0.5f ? 0.0 : AT(field, i, j, k);
                if (AT(back, i, j, k) != want) {
                    CHECK(0, "rdstd8 gives back what wdstd8 wrote");
                    i = NX + 1, j = NY + 1, k = NZ + 1;
                }
            }

    /* the descriptor of an FP32 copy and its reading */
    {
        const double x0 = 27.5, y0 = 40.9, z0[NZ] = {5.0, 15.0, 30.0};
        char datname[256], title[256], varname[2 * 32];
        double xs[16], ys[16], zs[8], hx, hy, hz;
        float undef, ht;
        int nx, ny, nz, nt, xt, yt, zt, nvar, yr, y, mo, d, h, mn, inform = 0;
        snprintf(path, sizeof path, "%s/h4.dat", dir);
        CHECK(inmsom_ctl_file_write(path, -1.0e32f, 10, 7, NZ, 2, 0, &x0, 0.5, 0, &y0, 0.25, 1, z0, 1.0, 0, 2001,
                                    7, 15, 6, 0, 21600.0f, "Harness field, 1", "hf") == INMSOM_OK,
              "ctl_file_write");
        snprintf(path, sizeof path, "%s/h4.ctl", dir);
        rc = inmsom_ctl_file_read(path, datname, (int)sizeof datname, &undef, &nx, &ny, &nz, &nt, &xt, xs, 16, &hx,
                                  &yt, ys, 16, &hy, &zt, zs, 8, &hz, &nvar, &yr, &y, &mo, &d, &h, &mn, &ht, title,
                                  (int)sizeof title, varname, 32, 2, &inform);
        CHECK(rc == INMSOM_OK, "ctl_file_read");
        CHECK(strcmp(datname, "h4.dat") == 0 && strcmp(varname, "hf") == 0, "names read back");
        CHECK(nx == 10 && ny == 7 && nz == NZ && nt == 2 && xt == 0 && zt == 1 && yr == 0, "dimensions read back");
        CHECK(y == 2001 && mo == 7 && d == 15 && h == 6 && mn == 0 && ht == 21600.0f, "calendar read back");
        CHECK(fabs(xs[9] - (27.5 + 9 * 0.5)) < 1e-12 && zs[2] == 30.0 && undef == -1.0e32f, "axes read back");
        CHECK(inform == 8, "eight definitions counted");
    }

    /* two row strips by pwdstd give the file wdstd writes for the field */
    for (k = 0; k < NX * NY * NZ; k++) f4[k] = (float)field[k];
    memcpy(strip, f4, sizeof f4);
    CHECK(inmsom_wdstd(dir, "whole.dat", 1, f4, lu, NX, NY, NZ, 3, 12, 3, 9, 1, NZ) == INMSOM_OK, "wdstd");
    {
        /* strips 3..5 and 6..9 of the interior; each rank's arrays are its
         * rows with two halo rows, taken from the whole field */
        const int rows[2][2] = {{3, 5}, {6, 9}};
        int s;
        for (s = 0; s < 2; s++) {
            const int y1 = rows[s][0] - 2, y2 = rows[s][1] + 2, ny = y2 - y1 + 1;
            inmsom_bounds b = {3, 12, rows[s][0], rows[s][1], 1, 14, y1, y2, 3, 12, 3, 9, 0, 0};
            float *loc = malloc(sizeof(float) * NX * ny * NZ), *lmask = malloc(sizeof(float) * NX * ny);
            for (k = 1; k <= NZ; k++)
                for (j = y1; j <= y2; j++)
                    for (i = 1; i <= NX; i++) loc[(i - 1) + NX * ((j - y1) + ny * (k - 1))] = AT(strip, i, j, k);
            for (j = y1; j <= y2; j++)
                for (i = 1; i <= NX; i++) lmask[(i - 1) + NX * (j - y1)] = LU(i, j);
            CHECK(inmsom_pwdstd(&b, dir, "strips.dat", 1, loc, lmask, NX, NY, NZ, 3, 12, 3, 9, 1, NZ) == INMSOM_OK,
                  "pwdstd");
            free(loc);
            free(lmask);
        }
    }
    {
        char a[1024], b2[1024];
        snprintf(a, sizeof a, "%s/whole.dat", dir);
        snprintf(b2, sizeof b2, "%s/strips.dat", dir);
        CHECK(file_size(a) == (long)NZ * 70 * 4 && same_files(a, b2), "the strips' file equals wdstd's");
    }

    /* a missing file */
    CHECK(inmsom_rdstd8(dir, "missing.dat", 1, back, lu, NX, NY, NZ, 3, 12, 3, 9, 1, 1) == INMSOM_EIO,
          "a missing file is INMSOM_EIO");
    CHECK(strstr(inmsom_gpu_last_error(), "missing.dat") != NULL, "the message names the file");

    if (failures) return 1;
    printf("ok\n");
    return 0;
}
