// Images one chunk of records with the C++ host API (include/mtb.hpp):
//   image_one <in.bin> <out.bin>
// in.bin:  int32 nx, ny, npol, wplanes, sampling, pol_type, compensated, R;
//          float64 l_increment; then float32 uvw[3][R], freq[R],
//          complex64 vis[R][P], float32 weights[R][P], int32 flags[R][P]
// out.bin: float32 image[P][ny][nx] followed by uint64 gridded_records,
//          compressed_records
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "mtb.hpp"

template <class T>
static void read(FILE *f, T *p, size_t n) {
    if (fread(p, sizeof(T), n, f) != n) {
        fprintf(stderr, "short read\n");
        exit(2);
    }
}

int main(int argc, char **argv) {
    if (argc != 3) return 2;
    FILE *f = fopen(argv[1], "rb");
    if (!f) return 2;
    int h[8];
    read(f, h, 8);
    double dl;
    read(f, &dl, 1);
    const int nx = h[0], ny = h[1], P = h[2], nw = h[3], s = h[4], pol = h[5], comp = h[6], R = h[7];
    std::vector<float> uvw(3 * (size_t)R), freq(R), vis(2 * (size_t)R * P), wt((size_t)R * P);
    std::vector<int> fl((size_t)R * P);
    read(f, uvw.data(), uvw.size());
    read(f, freq.data(), freq.size());
    read(f, vis.data(), vis.size());
    read(f, wt.data(), wt.size());
    read(f, fl.data(), fl.size());
    fclose(f);
    try {
        cudaStream_t st;
        mtb::cuda_check(cudaStreamCreate(&st), "stream");
        mtb_wkernel_params kp{nx, ny, dl, dl, nw, s, 0, 0, 0.0};
        auto k = mtb::KernelTable::build(kp, st);
        // FP64 per-call delta grid: an order-independent, reproducible image
        mtb::Imager im(k, P, pol, comp != 0, st, nullptr, /*exact_delta=*/true);
        mtb::DeviceArray<float> d_uvw(uvw.size(), st), d_freq(freq.size(), st), d_vis(vis.size(), st),
            d_wt(wt.size(), st), d_img((size_t)P * nx * ny, st);
        mtb::DeviceArray<int> d_fl(fl.size(), st);
        cudaMemcpyAsync(d_uvw.data(), uvw.data(), uvw.size() * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_freq.data(), freq.data(), freq.size() * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_vis.data(), vis.data(), vis.size() * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_wt.data(), wt.data(), wt.size() * 4, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_fl.data(), fl.data(), fl.size() * 4, cudaMemcpyHostToDevice, st);
        im.grid(d_uvw.data(), d_freq.data(), d_vis.data(), d_wt.data(), d_fl.data(), R);
        im.finalize(d_img.data());
        std::vector<float> img((size_t)P * nx * ny);
        mtb::cuda_check(cudaMemcpyAsync(img.data(), d_img.data(), img.size() * 4, cudaMemcpyDeviceToHost, st),
                        "D2H");
        mtb_grid_stats stats = im.stats();
        FILE *o = fopen(argv[2], "wb");
        fwrite(img.data(), 4, img.size(), o);
        unsigned long long st2[2] = {stats.gridded_records, stats.compressed_records};
        fwrite(st2, 8, 2, o);
        fclose(o);
    } catch (const std::exception &e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
