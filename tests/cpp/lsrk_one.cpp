// TOPO -> LSRK nu/c with the C++ host API (include/mtb.hpp, mtb::FrequencyConverter):
//   lsrk_one <in.bin> <out.bin>
// in.bin:  int32 nrows, nchan, n, has_index; float64 site_itrf[3], ra, dec,
//          tt_minus_time, ut1_minus_time; float64 time[nrows], chan_hz[nchan];
//          int32 index[n] when has_index
// out.bin: float32 nu_over_c[nchan][n]
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
    int h[4];
    read(f, h, 4);
    const int nrows = h[0], nchan = h[1], n = h[2], has_index = h[3];
    double g[7];
    read(f, g, 7);
    std::vector<double> time(nrows), chan(nchan);
    std::vector<int> index(has_index ? n : 0);
    read(f, time.data(), time.size());
    read(f, chan.data(), chan.size());
    read(f, index.data(), index.size());
    fclose(f);
    try {
        cudaStream_t st;
        mtb::cuda_check(cudaStreamCreate(&st), "stream");
        mtb_lsrk_params p{{g[0], g[1], g[2]}, g[3], g[4], g[5], g[6]};
        mtb::FrequencyConverter conv(p, st);
        mtb::DeviceArray<double> d_time(time.size(), st), d_chan(chan.size(), st);
        mtb::DeviceArray<int> d_index(index.size(), st);
        mtb::DeviceArray<float> d_out((size_t)nchan * n, st);
        mtb::cuda_check(cudaMemcpyAsync(d_time.data(), time.data(), time.size() * 8, cudaMemcpyHostToDevice, st), "H2D");
        mtb::cuda_check(cudaMemcpyAsync(d_chan.data(), chan.data(), chan.size() * 8, cudaMemcpyHostToDevice, st), "H2D");
        if (has_index)
            mtb::cuda_check(cudaMemcpyAsync(d_index.data(), index.data(), index.size() * 4, cudaMemcpyHostToDevice, st),
                            "H2D");
        conv.convert(d_time.data(), nrows, d_chan.data(), nchan, has_index ? d_index.data() : nullptr, n, d_out.data());
        std::vector<float> out((size_t)nchan * n);
        mtb::cuda_check(cudaMemcpyAsync(out.data(), d_out.data(), out.size() * 4, cudaMemcpyDeviceToHost, st), "D2H");
        mtb::cuda_check(cudaStreamSynchronize(st), "sync");
        FILE *o = fopen(argv[2], "wb");
        fwrite(out.data(), 4, out.size(), o);
        fclose(o);
    } catch (const std::exception &e) {
        fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
