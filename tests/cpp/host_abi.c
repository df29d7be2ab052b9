/*
 * host_abi.c -- the C ABI from plain C (no C++, no Python, no GPU).
 *
 * Built with gcc against include/ and libmtb.so by tests/test_capi.py.  It
 * calls the host-side entry points: the baseline-major record order of
 * mt-imager's visibility ingest (SortIndex.cpp:46-87) on a hand-made antenna
 * table, a column gather in that order (SortedStorage.h:205-246), the status
 * strings, and parameter refusals that happen before any device work
 * (grid, engine, FITS and TOPO -> LSRK entry points).
 * Prints "ok" and exits 0 when every check holds.
 */
#include <stdio.h>
#include <string.h>

#include "mtb.h"
#include "mtb_engine.h"
#include "mtb_fits.h"

#define CHECK(c)                                                      \
    do {                                                              \
        if (!(c)) {                                                   \
            fprintf(stderr, "check failed at line %d: %s\n", __LINE__, #c); \
            return 1;                                                 \
        }                                                             \
    } while (0)

int main(void)
{
    /* 3 antennas; rows in time order with one autocorrelation.
     * baseline number nA*nA - a1*nA - a2 - 1: (0,1) -> 7, (0,2) -> 6, (1,2) -> 3 */
    const int a1[] = {0, 0, 1, 1, 0, 0, 1};
    const int a2[] = {1, 2, 2, 1, 1, 2, 2};
    const int want[] = {2, 6, 1, 5, 0, 4};   /* (1,2) rows, then (0,2), then (0,1), time order kept */
    int index[7], n = -1;
    CHECK(mtb_sort_index(a1, a2, 7, 3, index, &n) == MTB_OK);
    CHECK(n == 6);
    for (int k = 0; k < n; k++) CHECK(index[k] == want[k]);

    /* antenna id out of range: refused */
    const int bad[] = {0, 3};
    const int ok2[] = {1, 1};
    CHECK(mtb_sort_index(bad, ok2, 2, 3, index, &n) == MTB_ERR_BAD_PARAM);

    /* gather a [row][2] float column in the sorted order, second value only */
    float col[7][2];
    for (int r = 0; r < 7; r++) {
        col[r][0] = (float)r;
        col[r][1] = 10.0f * (float)r;
    }
    float out[6];
    CHECK(mtb_gather_rows(col, sizeof(col[0]), sizeof(float), sizeof(float), want, 6, out, 2) == MTB_OK);
    for (int k = 0; k < 6; k++) CHECK(out[k] == 10.0f * (float)want[k]);

    /* status strings and version */
    CHECK(strcmp(mtb_status_string(MTB_OK), "ok") == 0);
    CHECK(mtb_status_string(MTB_ERR_CUDA) != NULL && mtb_status_string(MTB_ERR_CUDA)[0] != '\0');
    CHECK(mtb_version() >= 100);

    /* host-side refusals before any device work */
    mtb_grid_params gp;
    memset(&gp, 0, sizeof(gp));
    gp.nx = gp.ny = 1024;
    gp.npol = 3;
    gp.sampling = 4;
    gp.wplanes = 1;
    gp.u_increment = gp.v_increment = gp.w_sq_increment = 1.0;
    int conv_info[2] = {7, 0};
    size_t bytes = 0;
    CHECK(mtb_grid_workspace_size(&gp, conv_info, 100, &bytes) == MTB_ERR_BAD_SHAPE);
    /* the per-call delta grid: FP32 pairs by default, none without grid_lo */
    gp.npol = 4;
    CHECK(mtb_grid_delta_bytes(&gp, &bytes) == MTB_OK && bytes == (size_t)1024 * 1024 * 4 * 8);
    gp.no_grid_lo = 1;
    CHECK(mtb_grid_delta_bytes(&gp, &bytes) == MTB_OK && bytes == 0);
    mtb_finalize_params fp = {1024, 1024, 4, 8, 2, 0, NULL};   /* pol_type 2: neither linear nor circular */
    CHECK(mtb_finalize_workspace_size(&fp, &bytes) == MTB_ERR_BAD_PARAM);
    fp.pol_type = MTB_POL_LINEAR;
    CHECK(mtb_finalize_planes_bytes(&fp, &bytes) == MTB_OK && bytes == (size_t)4 * 1024 * 1024 * 16);
    mtb_wkernel_params wp;
    memset(&wp, 0, sizeof(wp));
    wp.nx = wp.ny = 256;
    wp.l_increment = wp.m_increment = 1e-5;
    wp.wplanes = 32;
    wp.sampling = 8;
    wp.trial_support = 32;                           /* even: refused */
    mtb_wkernel_info info;
    CHECK(mtb_wkernel_query(&wp, &info) == MTB_ERR_BAD_PARAM);
    CHECK(mtb_engine_destroy(NULL) == MTB_ERR_NULL);
    CHECK(mtb_engine_cancel(NULL, 1) == MTB_ERR_NULL);
    CHECK(strcmp(mtb_status_string(MTB_ERR_CANCELLED), "request cancelled") == 0);
    CHECK(mtb_fits_create(NULL, NULL, NULL) != MTB_OK);

    /* TOPO -> LSRK conversion: the parameter block from C and its refusals */
    mtb_lsrk_params lp;
    memset(&lp, 0, sizeof(lp));
    lp.site_itrf[0] = 5109360.133;
    lp.site_itrf[1] = 2006852.586;
    lp.site_itrf[2] = -3238948.127;
    lp.ra = 1.2;
    lp.dec = -0.8;
    lp.tt_minus_time = 69.184;
    size_t lws = 0;
    CHECK(mtb_lsrk_workspace_size(-1, &lws) == MTB_ERR_BAD_PARAM);
    CHECK(mtb_lsrk_freq_over_c(NULL, NULL, 1, NULL, 1, NULL, 1, NULL, NULL, 0, NULL) == MTB_ERR_NULL);
    CHECK(mtb_lsrk_freq_over_c(&lp, NULL, 4, NULL, 1, NULL, 3, NULL, NULL, 0, NULL) == MTB_ERR_BAD_PARAM);
    CHECK(mtb_lsrk_freq_over_c(&lp, NULL, 4, NULL, 0, NULL, 4, NULL, NULL, 0, NULL) == MTB_OK);
    CHECK(mtb_lsrk_freq_over_c(&lp, NULL, 4, NULL, 2, NULL, 4, NULL, NULL, 0, NULL) == MTB_ERR_NULL);

    printf("ok\n");
    return 0;
}
