// Host side of visibility ingest: the baseline-major record order of
// mt-imager's VisibilityManager and the row gathers that apply it
// (include/mtb.h).  No kernels; no GPU needed.
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

#include "mtb.h"

// Counting sort on the baseline number nA*nA - a1*nA - a2 - 1
// (code/mt-imager/lib/components/VisibilityManager/SortIndex.cpp:46-87):
// autocorrelations dropped, rows of one baseline kept in their original order.
extern "C" int mtb_sort_index(const int *antenna1, const int *antenna2, int nrows, int nantennas, int *index,
                              int *nsorted) {
    if (!nsorted || (nrows > 0 && (!antenna1 || !antenna2 || !index))) return MTB_ERR_NULL;
    if (nrows < 0 || nantennas < 1 || nantennas > 46340) return MTB_ERR_BAD_PARAM;
    const long long nb = (long long)nantennas * nantennas;
    for (int i = 0; i < nrows; i++)
        if (antenna1[i] < 0 || antenna1[i] >= nantennas || antenna2[i] < 0 || antenna2[i] >= nantennas)
            return MTB_ERR_BAD_PARAM;
    std::vector<int> start((size_t)nb + 1, 0);
    for (int i = 0; i < nrows; i++)
        if (antenna1[i] != antenna2[i]) start[(size_t)(nb - (long long)antenna1[i] * nantennas - antenna2[i] - 1) + 1]++;
    for (long long b = 0; b < nb; b++) start[(size_t)b + 1] += start[(size_t)b];
    const int kept = start[(size_t)nb];
    for (int i = 0; i < nrows; i++)
        if (antenna1[i] != antenna2[i]) index[start[(size_t)(nb - (long long)antenna1[i] * nantennas - antenna2[i] - 1)]++] = i;
    *nsorted = kept;
    return MTB_OK;
}

// out[k * row_bytes ...] = in[index[k] * in_stride + offset ...] for k < n,
// split over `threads` host threads (0: the hardware's, at most 16).
extern "C" int mtb_gather_rows(const void *in, size_t in_stride, size_t offset, size_t row_bytes, const int *index,
                               int n, void *out, int threads) {
    if (n < 0) return MTB_ERR_BAD_PARAM;
    if (n == 0) return MTB_OK;
    if (!in || !index || !out) return MTB_ERR_NULL;
    if (row_bytes == 0 || offset + row_bytes > in_stride) return MTB_ERR_BAD_PARAM;
    if (threads <= 0) {
        const int hw = (int)std::thread::hardware_concurrency();
        threads = std::max(1, std::min(16, hw));
    }
    threads = std::max(1, std::min(threads, n / 65536 + 1));
    const char *src = (const char *)in + offset;
    char *dst = (char *)out;
    auto part = [&](int k0, int k1) {
        if (row_bytes == 4) {
            for (int k = k0; k < k1; k++) std::memcpy(dst + (size_t)k * 4, src + (size_t)index[k] * in_stride, 4);
        } else {
            for (int k = k0; k < k1; k++)
                std::memcpy(dst + (size_t)k * row_bytes, src + (size_t)index[k] * in_stride, row_bytes);
        }
    };
    std::vector<std::thread> th;
    for (int t = 1; t < threads; t++)
        th.emplace_back(part, (int)((long long)n * t / threads), (int)((long long)n * (t + 1) / threads));
    part(0, (int)((long long)n / threads));
    for (auto &x : th) x.join();
    return MTB_OK;
}
