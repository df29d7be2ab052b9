// Drives the GAFW operators of mt-imager_b200/gafw_adapter/ the way GAFW's engine
// does -- validate(ValidationData &) to learn the outputs and the scratch, then
// submitToGPU(GPUSubmissionData &) with engine-allocated arrays, an int buffer
// size and the timing events -- and compares every output with the direct
// C-ABI call on the same inputs.
//   gafw_adapter <dir>
// dir/params.txt: nx ny dl nw sampling R P; dir/uvw.f32 [3][R], freq.f32 [R],
// vis.c64 [R][P], weights.f32 [R][P], flags.i32 [R][P].
// Prints "all match" and exits 0, or names the first mismatch and exits 1.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mtb_gafw_operators.h"

using namespace GAFW;
using namespace GAFW::GPU;
using namespace GAFW::GeneralImplimentation;
using GAFW::Tools::CppProperties::Properties;

static void cu(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "%s: %s\n", what, cudaGetErrorString(e));
        exit(2);
    }
}
static void ok(int rc, const char *what) {
    if (rc != MTB_OK) {
        fprintf(stderr, "%s: %s\n", what, mtb_status_string(rc));
        exit(2);
    }
}

template <class T>
static std::vector<T> load(const std::string &path, size_t n) {
    std::vector<T> v(n);
    FILE *f = fopen(path.c_str(), "rb");
    if (!f || fread(v.data(), sizeof(T), n, f) != n) {
        fprintf(stderr, "cannot read %s\n", path.c_str());
        exit(2);
    }
    fclose(f);
    return v;
}

static size_t type_size(StoreType t) {
    switch (t) {
    case real_int: case real_uint: case real_float: return 4;
    case real_double: case complex_float: case real_longint: case real_ulongint: return 8;
    case complex_double: return 16;
    case real_shortint: case real_ushortint: return 2;
    default: return 0;
    }
}

// One array as the engine holds it.
struct Buf {
    void *p = nullptr;
    ArrayDimensions dim;
    StoreType type = StoreTypeUnknown;
    size_t bytes() const { return (size_t)dim.getTotalNoOfElements() * type_size(type); }
};

static Buf device(const void *host, size_t bytes, const ArrayDimensions &dim, StoreType t, cudaStream_t st) {
    Buf b;
    b.dim = dim;
    b.type = t;
    cu(cudaMalloc(&b.p, bytes ? bytes : 1), "cudaMalloc");
    if (host && bytes) cu(cudaMemcpyAsync(b.p, host, bytes, cudaMemcpyHostToDevice, st), "H2D");
    return b;
}

template <class T>
static std::vector<T> host(const void *d, size_t n, cudaStream_t st) {
    std::vector<T> v(n);
    if (n) cu(cudaMemcpyAsync(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost, st), "D2H");
    cu(cudaStreamSynchronize(st), "sync");
    return v;
}

static bool fail(const std::string &what) {
    printf("FAILED: %s\n", what.c_str());
    return false;
}

static bool same_bytes(const void *da, const void *db, size_t bytes, cudaStream_t st, const std::string &what) {
    std::vector<unsigned char> a = host<unsigned char>(da, bytes, st), b = host<unsigned char>(db, bytes, st);
    if (std::memcmp(a.data(), b.data(), bytes) != 0) return fail(what + " differs");
    return true;
}

// The engine's part for one operator: validate (outputs allocated by the
// engine unless `outs` already holds them, as for an accumulating array the
// engine keeps), scratch of the validated size, submit on `st` with the
// events, and the end event recorded by the operator.
struct Run {
    cudaStream_t st;
    cudaEvent_t start, end;

    void operator()(GPUArrayOperator &op, const std::vector<Buf> &ins, std::vector<Buf> &outs, size_t nouts) {
        std::vector<Array> in_a(ins.size()), out_a(nouts);
        op.inputs.clear();
        op.outputs.clear();
        for (size_t i = 0; i < ins.size(); i++) {
            in_a[i].setDimensions(ins[i].dim);
            in_a[i].setType(ins[i].type);
            op.inputs.push_back(&in_a[i]);
        }
        for (size_t i = 0; i < nouts; i++) op.outputs.push_back(&out_a[i]);
        ValidationData vd;
        op.validate(vd);
        const bool fresh = outs.empty();
        for (size_t i = 0; i < nouts; i++) {
            Buf b;
            b.dim = out_a[i].getDimensions();
            b.type = out_a[i].getType();
            if (fresh) {
                b = device(nullptr, b.bytes(), b.dim, b.type, st);
                outs.push_back(b);
            } else if (outs[i].bytes() != b.bytes()) {
                fprintf(stderr, "%s: output %zu changed size\n", op.name.c_str(), i);
                exit(2);
            }
        }
        if (vd.bufferSize > (size_t)0x7fffffff) {
            fprintf(stderr, "%s: scratch does not fit an int\n", op.name.c_str());
            exit(2);
        }
        void *scratch = nullptr;
        cu(cudaMalloc(&scratch, vd.bufferSize ? vd.bufferSize : 1), "scratch");
        std::vector<GPUArrayDescriptor> din(ins.size()), dout(nouts);
        for (size_t i = 0; i < ins.size(); i++) din[i] = GPUArrayDescriptor{ins[i].p, ins[i].dim, ins[i].type};
        for (size_t i = 0; i < nouts; i++) dout[i] = GPUArrayDescriptor{outs[i].p, outs[i].dim, outs[i].type};
        GPUSubmissionData d;
        d.noOfInputs = (int)din.size();
        d.inputs = din.data();
        d.noOfOutputs = (int)dout.size();
        d.outputs = dout.data();
        d.stream = st;
        d.startEvent = &start;
        d.endEvent = &end;
        d.params = op.params;
        d.bufferGPUPointer = scratch;
        d.buffersize = (int)vd.bufferSize;
        op.submitToGPU(d);
        if (!d.endEventRecorded) {
            fprintf(stderr, "%s: end event not recorded\n", op.name.c_str());
            exit(2);
        }
        cu(cudaEventSynchronize(end), "end event");
        float ms = 0.0f;
        cu(cudaEventElapsedTime(&ms, start, end), "elapsed");
        cu(cudaFree(scratch), "free scratch");
    }
};

int main(int argc, char **argv) {
    if (argc != 2) return 2;
    const std::string dir = argv[1];
    int nx, ny, nw, s, R, P;
    double dl;
    {
        FILE *f = fopen((dir + "/params.txt").c_str(), "r");
        if (!f || fscanf(f, "%d %d %lf %d %d %d %d", &nx, &ny, &dl, &nw, &s, &R, &P) != 7) return 2;
        fclose(f);
    }
    const std::vector<float> uvw = load<float>(dir + "/uvw.f32", 3 * (size_t)R);
    const std::vector<float> freq = load<float>(dir + "/freq.f32", R);
    const std::vector<float> vis = load<float>(dir + "/vis.c64", 2 * (size_t)R * P);
    const std::vector<float> wt = load<float>(dir + "/weights.f32", (size_t)R * P);
    const std::vector<int> fl = load<int>(dir + "/flags.i32", (size_t)R * P);

    Run run;
    cu(cudaStreamCreate(&run.st), "stream");
    cu(cudaEventCreate(&run.start), "event");
    cu(cudaEventCreate(&run.end), "event");
    cudaStream_t st = run.st;
    bool good = true;
    try {
        // ---- WProjectionConvFunction against mtb_wkernel_build
        mtb_gafw::MtbWProjectionConvFunction wk(nullptr, "wkernels");
        wk.params.set("image.nx", nx, Properties::Int);
        wk.params.set("image.ny", ny, Properties::Int);
        wk.params.set("image.lintervalsize", dl, Properties::Double);
        wk.params.set("image.mintervalsize", dl, Properties::Double);
        wk.params.set("wproj.wplanes", nw, Properties::Int);
        wk.params.set("wproj.convFunction.sampling", s, Properties::Int);
        wk.params.set("wproj.convFunction.trialsupport", 0, Properties::Int);
        wk.params.set("wproj.convFunction.maxsupport", 0, Properties::Int);
        wk.params.set("wproj.wmax", 0.0, Properties::Double);
        std::vector<Buf> kt;
        run(wk, {}, kt, 3);

        mtb_wkernel_params kp{nx, ny, dl, dl, nw, s, 0, 0, 0.0};
        mtb_wkernel_info info;
        ok(mtb_wkernel_query(&kp, &info), "query");
        Buf kws = device(nullptr, info.workspace_bytes, ArrayDimensions(1, 1), real_float, st);
        Buf table = device(nullptr, info.table_capacity * 8, ArrayDimensions(1, (int)info.table_capacity),
                           complex_float, st);
        Buf dci = device(nullptr, (size_t)nw * 2 * 4, ArrayDimensions(2, nw, 2), real_int, st);
        Buf sums = device(nullptr, (size_t)nw * info.T * info.T * 4, ArrayDimensions(2, nw, info.T * info.T),
                          real_float, st);
        std::vector<int> hci((size_t)nw * 2);
        size_t elems = 0;
        ok(mtb_wkernel_build(&kp, kws.p, info.workspace_bytes, table.p, info.table_capacity, (int *)dci.p,
                             hci.data(), (float *)sums.p, &elems, (mtb_stream_t)st),
           "mtb_wkernel_build");
        good = good && same_bytes(kt[0].p, table.p, elems * 8, st, "WProjectionConvFunction table");
        good = good && same_bytes(kt[1].p, dci.p, (size_t)nw * 2 * 4, st, "WProjectionConvFunction convInfo");
        good = good && same_bytes(kt[2].p, sums.p, sums.bytes(), st, "WProjectionConvFunction sums");

        // ---- the gridding parameters as the adapter reads them (float properties)
        auto grid_keys = [&](Properties &pr) {
            pr.set("ConvolutionFunction.sampling", s, Properties::Int);
            pr.set("ConvolutionFunction.wsquareincrement", info.w_sq_increment, Properties::Float);
            pr.set("uvImage.u_increment", info.u_increment, Properties::Float);
            pr.set("uvImage.v_increment", info.v_increment, Properties::Float);
            pr.set("uvImage.rows", ny, Properties::Int);
            pr.set("uvImage.columns", nx, Properties::Int);
            pr.set("ConvolutionFunction.maxsupport", info.support_cap, Properties::Int);
        };
        mtb_grid_params gp;
        std::memset(&gp, 0, sizeof(gp));
        gp.nx = nx;
        gp.ny = ny;
        gp.npol = P;
        gp.sampling = s;
        gp.wplanes = nw;
        gp.u_increment = (float)info.u_increment;
        gp.v_increment = (float)info.v_increment;
        gp.w_sq_increment = (float)info.w_sq_increment;

        Buf d_uvw = device(uvw.data(), uvw.size() * 4, ArrayDimensions(2, 3, R), real_float, st);
        Buf d_freq = device(freq.data(), freq.size() * 4, ArrayDimensions(1, R), real_float, st);
        Buf d_vis = device(vis.data(), vis.size() * 4, ArrayDimensions(2, R, P), complex_float, st);
        Buf d_wt = device(wt.data(), wt.size() * 4, ArrayDimensions(2, R, P), real_float, st);
        Buf d_fl = device(fl.data(), fl.size() * 4, ArrayDimensions(2, R, P), real_int, st);

        // ---- PreProcessUVW against mtb_preprocess_uvw
        mtb_gafw::MtbPreProcessUVW pre(nullptr, "preprocess");
        grid_keys(pre.params);
        std::vector<Buf> po;
        run(pre, {kt[1], kt[2], d_uvw, d_freq, d_wt, d_fl}, po, 7);
        {
            mtb_grid_params p = gp;
            p.no_grid_lo = 1;
            size_t ws = 0;
            ok(mtb_grid_workspace_size(&p, hci.data(), R, &ws), "workspace");
            Buf w = device(nullptr, ws, ArrayDimensions(1, 1), real_float, st);
            std::vector<Buf> ref;
            for (size_t i = 0; i < po.size(); i++) ref.push_back(device(nullptr, po[i].bytes(), po[i].dim, po[i].type, st));
            ok(mtb_preprocess_uvw(&p, (const int *)dci.p, hci.data(), (const float *)sums.p, (const float *)d_uvw.p,
                                  (const float *)d_freq.p, (const float *)d_wt.p, (const int *)d_fl.p, R,
                                  (int *)ref[0].p, (int *)ref[1].p, (int *)ref[2].p, (int *)ref[3].p,
                                  (int *)ref[4].p, (float *)ref[5].p, (float *)ref[6].p, w.p, ws,
                                  (mtb_stream_t)st),
               "mtb_preprocess_uvw");
            for (size_t i = 0; i < po.size(); i++)
                good = good && same_bytes(po[i].p, ref[i].p, po[i].bytes(), st,
                                          "PreProcessUVW output " + std::to_string(i));
        }

        // ---- GridChunk over two chunks against two mtb_grid calls
        const int R1 = R / 2;
        const int cr[2] = {0, R1}, cn[2] = {R1, R - R1};
        std::vector<Buf> go;
        Buf g_ref = device(nullptr, (size_t)nx * ny * P * 8, ArrayDimensions(3, ny, nx, P), complex_float, st);
        Buf lo_ref = device(nullptr, g_ref.bytes(), g_ref.dim, complex_float, st);
        Buf n_ref = device(nullptr, (size_t)P * 4, ArrayDimensions(1, P), real_float, st);
        Buf s_ref = device(nullptr, 32, ArrayDimensions(1, 4), real_ulongint, st);
        for (int c = 0; c < 2; c++) {
            const int n = cn[c];
            std::vector<float> cu_uvw(3 * (size_t)n);
            for (int a = 0; a < 3; a++)
                std::memcpy(&cu_uvw[(size_t)a * n], &uvw[(size_t)a * R + cr[c]], (size_t)n * 4);
            Buf c_uvw = device(cu_uvw.data(), cu_uvw.size() * 4, ArrayDimensions(2, 3, n), real_float, st);
            Buf c_freq = device(&freq[cr[c]], (size_t)n * 4, ArrayDimensions(1, n), real_float, st);
            Buf c_vis = device(&vis[2 * (size_t)cr[c] * P], (size_t)n * P * 8, ArrayDimensions(2, n, P),
                               complex_float, st);
            Buf c_wt = device(&wt[(size_t)cr[c] * P], (size_t)n * P * 4, ArrayDimensions(2, n, P), real_float, st);
            Buf c_fl = device(&fl[(size_t)cr[c] * P], (size_t)n * P * 4, ArrayDimensions(2, n, P), real_int, st);
            mtb_gafw::MtbGridChunk gc(nullptr, "grid");
            grid_keys(gc.params);
            gc.params.set("initialize_output", c == 0 ? 1.0 : 0.0, Properties::Bool);
            run(gc, {kt[0], kt[1], kt[2], c_uvw, c_freq, c_vis, c_wt, c_fl}, go, 5);

            mtb_grid_params p = gp;
            p.initialize_output = c == 0 ? 1 : 0;
            size_t ws = 0;
            ok(mtb_grid_workspace_size(&p, hci.data(), n, &ws), "workspace");
            Buf w = device(nullptr, ws, ArrayDimensions(1, 1), real_float, st);
            ok(mtb_grid(&p, table.p, (const int *)dci.p, hci.data(), (const float *)sums.p, (const float *)c_uvw.p,
                        (const float *)c_freq.p, c_vis.p, (const float *)c_wt.p, (const int *)c_fl.p, n, g_ref.p,
                        lo_ref.p, (float *)n_ref.p, (mtb_grid_stats *)s_ref.p, w.p, ws, (mtb_stream_t)st),
               "mtb_grid");
            cu(cudaStreamSynchronize(st), "sync");
            for (Buf *b : {&c_uvw, &c_freq, &c_vis, &c_wt, &c_fl, &w}) cudaFree(b->p);
        }
        good = good && same_bytes(go[2].p, n_ref.p, n_ref.bytes(), st, "GridChunk normaliser");
        good = good && same_bytes(go[3].p, s_ref.p, 32, st, "GridChunk statistics");
        {
            // The per-call delta grid gathers flushes with atomics: the grids
            // agree to the rounding of that FP32 sum.
            const size_t n = (size_t)nx * ny * P * 2;
            std::vector<float> g = host<float>(go[0].p, n, st), lo = host<float>(go[1].p, n, st);
            std::vector<float> gr = host<float>(g_ref.p, n, st), lr = host<float>(lo_ref.p, n, st);
            double peak = 0.0, err = 0.0;
            for (size_t i = 0; i < n; i++) {
                const double a = (double)g[i] + lo[i], b = (double)gr[i] + lr[i];
                peak = std::fmax(peak, std::fabs(b));
                err = std::fmax(err, std::fabs(a - b));
            }
            if (!(peak > 0.0) || err > 2e-6 * peak) good = fail("GridChunk grid differs: " + std::to_string(err) +
                                                              " of peak " + std::to_string(peak));
        }

        // ---- ImageFinalizer against mtb_finalize on the adapter's grid
        mtb_gafw::MtbImageFinalizer fin(nullptr, "finalize");
        fin.params.set("ConvolutionFunction.sampling", s, Properties::Int);
        fin.params.set("PolarizationType", MTB_POL_LINEAR, Properties::Int);
        std::vector<Buf> fo;
        run(fin, {go[0], go[1], go[2]}, fo, 2);
        {
            mtb_finalize_params p;
            std::memset(&p, 0, sizeof(p));
            p.nx = nx;
            p.ny = ny;
            p.npol = P;
            p.sampling = s;
            p.pol_type = MTB_POL_LINEAR;
            size_t ws = 0;
            ok(mtb_finalize_workspace_size(&p, &ws), "finalize workspace");
            Buf w = device(nullptr, ws, ArrayDimensions(1, 1), real_float, st);
            Buf img = device(nullptr, fo[0].bytes(), fo[0].dim, real_float, st);
            ok(mtb_finalize(&p, go[0].p, go[1].p, (const float *)go[2].p, (float *)img.p, w.p, ws, (mtb_stream_t)st),
               "mtb_finalize");
            good = good && same_bytes(fo[0].p, img.p, img.bytes(), st, "ImageFinalizer image");
        }
    } catch (const std::exception &e) {
        printf("FAILED: exception %s\n", e.what());
        return 1;
    }
    if (!good) return 1;
    printf("all match\n");
    return 0;
}
