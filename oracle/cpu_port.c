/*
 * cpu_port.c -- TEST/MEASUREMENT INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * mt-imager ships only a GPU gridder, so the CPU baseline that bench.py times
 * on the host cores is this OpenMP C transcription of the reference's
 * per-chunk gridding semantics, in FP32 like the reference:
 *   preprocess    mt-imager/lib/operators/WProjPreProcessUVW.cu:112-324
 *   compression   CreateCompressionPlan.cu:32-67, CompressVisibilties.cu:41-74
 *   gridding      ConvolutionGridder.cu:130-181, 394-442 (complex MAC, no conjugate)
 *   normaliser    WImager.cpp:196-197 (sum of ConvolutionFunctionSum)
 * Only bench.py's cpu_baseline and reference legs load it.  The gridding loop
 * splits grid rows across threads so no two threads write one cell.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

int port_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* Threads of the following parallel regions (a launcher may have set
 * OMP_NUM_THREADS=1 for every process). */
void port_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

/* vis, grid: float complex interleaved.  stats[4]: gridded, compressed
 * records, gridded, compressed points.  Returns 0. */
int port_grid_chunk(int R, int P, const float *uvw, const float *freq, const float *vis,
                    const float *weights, const int *flags, int nw, float w_inc, const int *conv_info,
                    const float *conv_sums, const float *table, int s, int nv, int nu, float du, float dv,
                    float *grid, float *norm, long long *stats)
{
    int T = (s % 2) ? s : s + 1;
    int *loc = (int *)malloc(sizeof(int) * 2 * (size_t)R);    /* corner x, y */
    int *ci = (int *)malloc(sizeof(int) * (size_t)R);
    int *sup = (int *)malloc(sizeof(int) * (size_t)R);
    int *tg = (int *)malloc(sizeof(int) * (size_t)R);
    float *im = (float *)malloc(sizeof(float) * (size_t)R);
    float *cv = (float *)malloc(sizeof(float) * 2 * P * (size_t)R);
    double nacc[4] = {0, 0, 0, 0};
#pragma omp parallel for reduction(+ : nacc[:4]) schedule(static)
    for (int r = 0; r < R; r++) {
        int g = 0;
        for (int p = 0; p < P; p++) if (flags[(size_t)r * P + p] == 0) g = 1;
        int cx = 0, cy = 0, c = 0, S = 0;
        float imm = 1.0f, cs = 0.0f;
        if (g) {
            float u = uvw[r], v = uvw[(size_t)R + r], w = uvw[2 * (size_t)R + r], f = freq[r];
            if (w < 0.0f) { u = -u; v = -v; imm = -1.0f; }
            float wpf = roundf(sqrtf(fabsf((w * f) / w_inc)));
            int k = (wpf > (float)(nw - 1) || wpf != wpf) ? nw - 1 : (int)wpf;
            S = conv_info[2 * k];
            c = conv_info[2 * k + 1];
            float pv = (v * f / dv) + (float)(nv / 2), pu = (u * f / du) + (float)(nu / 2);
            float lx = roundf(pu), ly = roundf(pv);
            cx = (int)lx - S / 2; cy = (int)ly - S / 2;
            if (cy < 0 || cy > (nv - 1) - S || cx < 0 || cx > nu - 1 - S) {
                g = 0;
            } else {
                int ox = (int)roundf((lx - pu) * (float)s) + s / 2, oy = (int)roundf((ly - pv) * (float)s) + s / 2;
                if (s % 2) {
                    ox = ox < 0 ? 0 : (ox == s ? s - 1 : ox);
                    oy = oy < 0 ? 0 : (oy == s ? s - 1 : oy);
                }
                cs = conv_sums[(size_t)k * T * T + oy * T + ox];
                c += oy * S * S * T + ox * S * S;
            }
        }
        if (!g) { S = 0; c = 0; cx = cy = 0; cs = 0.0f; }
        loc[2 * (size_t)r] = cx; loc[2 * (size_t)r + 1] = cy;
        ci[r] = c; sup[r] = S; tg[r] = g; im[r] = imm;
        for (int p = 0; p < P; p++) nacc[p] += cs * weights[(size_t)r * P + p] * (1.0f - (float)flags[(size_t)r * P + p]);
    }
    for (int p = 0; p < P; p++) norm[p] += (float)nacc[p];
    /* compression flags: compare with the previous record's stored values */
    char *comp = (char *)calloc((size_t)R, 1);
#pragma omp parallel for schedule(static)
    for (int r = 1; r < R; r++) {
        int pc = tg[r - 1] ? ci[r - 1] : 0;
        int py = tg[r - 1] ? loc[2 * (size_t)(r - 1) + 1] * nu + loc[2 * (size_t)(r - 1)] : 0;
        if (tg[r] && ci[r] == pc && loc[2 * (size_t)r + 1] * nu + loc[2 * (size_t)r] == py) comp[r] = 1;
    }
    long long st[4] = {0, 0, 0, 0};
#pragma omp parallel for reduction(+ : st[:4]) schedule(static)
    for (int g = 0; g < R; g++) {
        if (!tg[g]) continue;
        long long s2 = (long long)sup[g] * sup[g];
        if (comp[g]) { st[1]++; st[3] += s2; continue; }
        st[0]++; st[2] += s2;
        for (int q = 0; q < 2 * P; q++) cv[(size_t)g * 2 * P + q] = 0.0f;
        int r = g;
        do {
            for (int p = 0; p < P; p++) {
                float wt = weights[(size_t)r * P + p] * (1.0f - (float)flags[(size_t)r * P + p]);
                cv[(size_t)g * 2 * P + 2 * p] += vis[(size_t)r * 2 * P + 2 * p] * wt;
                cv[(size_t)g * 2 * P + 2 * p + 1] += vis[(size_t)r * 2 * P + 2 * p + 1] * wt * im[r];
            }
            r++;
        } while (r < R && comp[r]);
    }
    for (int i = 0; i < 4; i++) stats[i] += st[i];
#pragma omp parallel
    {
        int nt = 1, t = 0;
#ifdef _OPENMP
        nt = omp_get_num_threads();
        t = omp_get_thread_num();
#endif
        int y0 = (int)((long)nv * t / nt), y1 = (int)((long)nv * (t + 1) / nt);
        for (int r = 0; r < R; r++) {
            if (!tg[r] || comp[r]) continue;
            int S = sup[r], cx = loc[2 * (size_t)r], cy = loc[2 * (size_t)r + 1];
            if (cy + S <= y0 || cy >= y1) continue;
            const float *V = cv + (size_t)r * 2 * P;
            for (int sy = 0; sy < S; sy++) {
                int y = cy + sy;
                if (y < y0 || y >= y1) continue;
                const float *tb = table + 2 * ((size_t)ci[r] + (size_t)sy * S);
                float *gr = grid + ((size_t)y * nu + cx) * 2 * P;
                for (int sx = 0; sx < S; sx++) {
                    float cr = tb[2 * sx], cim = tb[2 * sx + 1];
                    float *gc = gr + (size_t)sx * 2 * P;
                    for (int p = 0; p < P; p++) {
                        float vr = V[2 * p], vi = V[2 * p + 1];
                        gc[2 * p] += vr * cr - vi * cim;
                        gc[2 * p + 1] += vi * cr + vr * cim;
                    }
                }
            }
        }
    }
    free(loc); free(ci); free(sup); free(tg); free(im); free(cv); free(comp);
    return 0;
}
