/*
 * ref_harness.cu -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * Drives mt-imager's own operator code (compiled unchanged from the reference
 * tree by oracle/build_ref.py against the GAFW stand-in in oracle/ref_stubs/)
 * through the operator graphs of the imaging modules, so that golden vectors
 * can be produced by the reference itself on a GPU.  The output is used only
 * to pin the FP64 oracle and the product path in tests/ (fixtures under
 * tests/golden/); nothing in mt-imager_b200/ links or loads it.
 *
 * Each entry point allocates its own device buffers (every buffer padded and
 * zeroed, so a kernel that reads a few elements past an array's end reads
 * zeros), copies host inputs in, calls the operators' submitToGPU in the
 * order the module wires them, checks the preconditions under which the
 * reference's kernels stay in bounds before launching them, and copies the
 * outputs back.  Failures return non-zero with a message.
 *
 * Operator graph of one WImager chunk: code/mt-imager/lib/components/
 * WImager.cpp:167-234 (PreProcessUVW, AccumulatedSum, CreateIndexAndReorder,
 * ValueChangeDetect, AccumulatedSum, CreateBlockDataIndex,
 * NotSameSupportManipulate, AccumulatedSum, CreateBlockDataIndex,
 * CreateCompressionPlan, CompressVisibilities, ConvolutionGridder).
 */
#include "GPUafw.h"
#include "ImagerOperators.h"
#include "AccumulatedSum.h"
#include "SingleMultiply.h"
#include "ValueChangeDetect.h"
#include "ZeroToCentre2DShift.h"

#include <cufft.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

using GAFW::ArrayDimensions;
using GAFW::GeneralImplimentation::StoreType;
using namespace GAFW::GeneralImplimentation;
using GAFW::GPU::GPUArrayDescriptor;
using GAFW::GPU::GPUSubmissionData;

// ---- constructors, destructors and validate() of the operators: in mt-imager
// they live in the operators' .cpp files together with GAFW's validation
// logic, which the harness does not use (it sizes every buffer itself).
#define MTREF_OP(NS, C)                                                                    \
    NS::C::C(GAFW::GPU::GPUFactory *f, std::string n) : GAFW::GPU::GPUArrayOperator(f, n) {} \
    NS::C::~C() {}                                                                         \
    void NS::C::validate() {}
MTREF_OP(mtimager, WProjPreProcessUVW)
MTREF_OP(mtimager, CreateIndexAndReorder)
MTREF_OP(mtimager, CreateBlockIndex)
MTREF_OP(mtimager, NotSameSupportManipulate)
MTREF_OP(mtimager, CreateCompressionPlan)
MTREF_OP(mtimager, CompressVisibilities)
MTREF_OP(mtimager, ConvolutionGridder)
MTREF_OP(GAFW::GPU::StandardOperators, AccumulatedSum)
MTREF_OP(GAFW::GPU::StandardOperators, ValueChangeDetect)
MTREF_OP(mtimager, CasaGridSF)
MTREF_OP(mtimager, WProjPreFFTConvFunc)
MTREF_OP(mtimager, ConvFunctionSupportFind)
MTREF_OP(mtimager, ConvFunctionReOrganize)
MTREF_OP(mtimager, SumConvolutionFunctions)
MTREF_OP(mtimager, PreIFFTUVCorrection)
MTREF_OP(mtimager, SincCorrector)
MTREF_OP(GAFW::GPU::StandardOperators, ZeroToCentre2DShift)
MTREF_OP(GAFW::GPU::StandardOperators, SingleMultiply)
mtimager::PostIFFTStokesConverter::PostIFFTStokesConverter(GAFW::GPU::GPUFactory *f, std::string n)
    : GAFW::GPU::GPUArrayOperator(f, n) {}
mtimager::PostIFFTStokesConverter::~PostIFFTStokesConverter() {}
void mtimager::PostIFFTStokesConverter::validate(GAFW::GPU::ValidationData &) {}

// ConvolutionGridder creates a texture object per submission and hands it to
// the engine for release after the run (ConvolutionGridder.cpp:56-59).
void mtimager::ConvolutionGridder::postRunExecute(void *p) {
    Texture *t = (Texture *)p;
    if (t) {
        cudaDestroyTextureObject(t->object);
        delete t;
    }
}

namespace {

const size_t kPad = 1 << 20;   // bytes of zeroed slack after every buffer

struct DevArray {
    void *d = nullptr;
    size_t bytes = 0;
    std::vector<unsigned> dims;
    StoreType type = real_float;
    DevArray(const std::vector<unsigned> &dims, StoreType type, size_t elem_bytes) : dims(dims), type(type) {
        size_t n = 1;
        for (unsigned x : dims) n *= x;
        bytes = n * elem_bytes;
        checkCudaError(cudaMalloc(&d, bytes + kPad), "cudaMalloc");
        checkCudaError(cudaMemset(d, 0, bytes + kPad), "cudaMemset");
    }
    ~DevArray() {
        if (d) cudaFree(d);
    }
    GPUArrayDescriptor desc() const {
        GPUArrayDescriptor g;
        g.pointer = d;
        g.dim = ArrayDimensions(dims);
        g.type = type;
        return g;
    }
    void upload(const void *h) { checkCudaError(cudaMemcpy(d, h, bytes, cudaMemcpyHostToDevice), "upload"); }
    void download(void *h) const { checkCudaError(cudaMemcpy(h, d, bytes, cudaMemcpyDeviceToHost), "download"); }
};

typedef std::unique_ptr<DevArray> Arr;
Arr make(std::vector<unsigned> dims, StoreType t, size_t eb) { return Arr(new DevArray(dims, t, eb)); }

struct Runner {
    cudaStream_t stream = 0;
    cudaEvent_t ev0, ev1;          // handed to the operators (GPUSubmissionData)
    cudaEvent_t t0, t1;            // the harness's own span around each submission
    double chain_ms = 0.0;         // sum of the submissions' spans
    float own_ms = 0.0f;           // the last operator's own start..end events, when it records both
    GAFW::GPU::GPUDeviceDescriptor device;
    Runner() {
        checkCudaError(cudaStreamCreate(&stream), "stream");
        checkCudaError(cudaEventCreate(&ev0), "event");
        checkCudaError(cudaEventCreate(&ev1), "event");
        checkCudaError(cudaEventCreate(&t0), "event");
        checkCudaError(cudaEventCreate(&t1), "event");
    }
    ~Runner() {
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        cudaStreamDestroy(stream);
    }
    // One submitToGPU with the engine's bookkeeping: events, post-run hook,
    // and the error check GPUEngine makes after every submission.
    void submit(GAFW::GPU::GPUArrayOperator &op, const std::vector<const DevArray *> &in,
                const std::vector<const DevArray *> &out, const GAFW::Tools::CppProperties::Properties &params) {
        std::vector<GPUArrayDescriptor> di, dout;
        for (auto *a : in) di.push_back(a->desc());
        for (auto *a : out) dout.push_back(a->desc());
        GPUSubmissionData d;
        d.noOfInputs = (int)di.size();
        d.inputs = di.data();
        d.noOfOutputs = (int)dout.size();
        d.outputs = dout.data();
        d.stream = stream;
        void *post = nullptr;
        d.postExecutePointer = &post;
        d.startEvent = &ev0;
        d.endEvent = &ev1;
        d.params = params;
        d.deviceDescriptor = &device;
        checkCudaError(cudaEventRecord(t0, stream), "event");
        op.submitToGPU(d);
        checkCudaError(cudaEventRecord(t1, stream), "event");
        checkCudaError(cudaGetLastError(), "launch of " + op.nickname);
        checkCudaError(cudaStreamSynchronize(stream), "run of " + op.nickname);
        float ms = 0.0f;
        checkCudaError(cudaEventElapsedTime(&ms, t0, t1), "elapsed");
        chain_ms += ms;
        own_ms = ms;
        if (d.endEventRecorded && cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) own_ms = ms;
        if (post) op.postRunExecute(post);
    }
};

// The multiFFT2D / IFFT2D operators: one 2-D single-precision complex FFT per
// plane of a [planes][rows][cols] array with a cufftPlan2d(rows, cols, C2C)
// plan (std/MultiFFT2D.cpp:77-116 forward, std/IFFT2D.cpp:73-111 inverse,
// unnormalised).  Their sources also carry GAFW validation code, so the
// harness issues the same cuFFT calls itself.
void fft_planes(const DevArray &in, const DevArray &out, int direction, cudaStream_t stream) {
    const ArrayDimensions d(in.dims);
    const int rows = (int)d.getNoOfRows(), cols = (int)d.getNoOfColumns();
    const int planes = (int)(d.getTotalNoOfElements() / (unsigned)(rows * cols));
    cufftHandle plan;
    if (cufftPlan2d(&plan, rows, cols, CUFFT_C2C) != CUFFT_SUCCESS) throw GAFW::GeneralException("cufftPlan2d");
    cufftSetStream(plan, stream);
    for (int i = 0; i < planes; i++) {
        cufftComplex *a = (cufftComplex *)in.d + (size_t)i * rows * cols;
        cufftComplex *b = (cufftComplex *)out.d + (size_t)i * rows * cols;
        if (cufftExecC2C(plan, a, b, direction) != CUFFT_SUCCESS) {
            cufftDestroy(plan);
            throw GAFW::GeneralException("cufftExecC2C");
        }
    }
    checkCudaError(cudaStreamSynchronize(stream), "fft");
    cufftDestroy(plan);
}

int fail(char *err, int errlen, const char *msg) {
    if (err && errlen > 0) {
        std::strncpy(err, msg, errlen - 1);
        err[errlen - 1] = 0;
    }
    return 1;
}

// Spans of the last mtref_grid_chunk call (milliseconds).
float g_gridder_ms = 0.0f;   // ConvolutionGridder's own start..end events: its two kernels
float g_chain_ms = 0.0f;     // every operator of the chunk's graph, PreProcessUVW to the gridder

}  // namespace

extern "C" {

/* One WImager chunk through mt-imager's operators.
 *   table        complex64 [table_elems] (AmalgamatedConvFunction)
 *   conv_info    int [wplanes][2] {support, first element}
 *   conv_sums    float [wplanes][T*T]
 *   uvw float [3][R], freq float [R] (nu/c), vis complex64 [R][P],
 *   weights float [R][P], flags int [R][P]
 *   grid         complex64 [ny][nx][P], in/out (accumulated unless initialize)
 *   pre_*        the seven PreProcessUVW outputs (may be NULL) */
int mtref_grid_chunk(int nx, int ny, int npol, int sampling, int wplanes, float u_increment, float v_increment,
                     float w_sq_increment, const void *table, int table_elems, const int *conv_info,
                     const float *conv_sums, const float *uvw, const float *freq, const void *vis,
                     const float *weights, const int *flags, int R, int initialize, void *grid,
                     int *pre_gridding_data, int *pre_conv_index, int *pre_to_grid, int *pre_to_compress,
                     int *pre_support, float *pre_take_conjugate, float *pre_conv_sum, char *err, int errlen) {
    try {
        if (npol != 1 && npol != 2 && npol != 4) return fail(err, errlen, "npol must be 1, 2 or 4");
        if (R < 2048) return fail(err, errlen, "the reference plan kernels need at least 2048 records");
        // ConvolutionGridder reads the table through a linear texture whose
        // creation it does not check (ConvolutionGridder.cu:520-534)
        {
            int dev = 0, width = 0;
            checkCudaError(cudaGetDevice(&dev), "device");
            checkCudaError(cudaDeviceGetAttribute(&width, cudaDevAttrMaxTexture1DLinearWidth, dev), "attribute");
            if (table_elems <= 0 || table_elems > width)
                return fail(err, errlen, "kernel table larger than a linear texture");
        }
        const unsigned U = (unsigned)R, P = (unsigned)npol, W = (unsigned)wplanes;
        const unsigned T = (unsigned)(sampling % 2 ? sampling : sampling + 1);
        Runner run;
        // inputs (GAFW dimensions, slowest first)
        Arr a_info = make({W, 2}, real_int, 4), a_sums = make({W, T * T}, real_float, 4);
        Arr a_uvw = make({3, U}, real_float, 4), a_freq = make({U}, real_float, 4);
        Arr a_wt = make({U, P}, real_float, 4), a_fl = make({U, P}, real_int, 4);
        Arr a_vis = make({U, 2 * P}, real_float, 4);
        Arr a_table = make({(unsigned)table_elems}, complex_float, 8);
        a_info->upload(conv_info);
        a_sums->upload(conv_sums);
        a_uvw->upload(uvw);
        a_freq->upload(freq);
        a_wt->upload(weights);
        a_fl->upload(flags);
        a_vis->upload(vis);
        a_table->upload(table);
        // PreProcessUVW outputs (WProjPreProcessUVW.cpp:70-84)
        Arr g_data = make({U, 4}, real_int, 4), g_cidx = make({U}, real_int, 4), g_tog = make({U}, real_int, 4);
        Arr g_toc = make({U}, real_int, 4), g_sup = make({U}, real_int, 4), g_conj = make({U}, real_float, 4);
        Arr g_csum = make({P, U}, real_float, 4);
        GAFW::Tools::CppProperties::Properties pp;
        pp.set("ConvolutionFunction.sampling", sampling);
        pp.set("ConvolutionFunction.wsquareincrement", w_sq_increment);
        pp.set("uvImage.u_increment", u_increment);
        pp.set("uvImage.v_increment", v_increment);
        pp.set("uvImage.rows", ny);
        pp.set("uvImage.columns", nx);
        mtimager::WProjPreProcessUVW pre(nullptr, "PreProcessUVW");
        run.submit(pre, {a_info.get(), a_sums.get(), a_uvw.get(), a_freq.get(), a_wt.get(), a_fl.get()},
                   {g_data.get(), g_cidx.get(), g_tog.get(), g_toc.get(), g_sup.get(), g_conj.get(), g_csum.get()},
                   pp);
        if (pre_gridding_data) g_data->download(pre_gridding_data);
        if (pre_conv_index) g_cidx->download(pre_conv_index);
        if (pre_to_grid) g_tog->download(pre_to_grid);
        if (pre_to_compress) g_toc->download(pre_to_compress);
        if (pre_support) g_sup->download(pre_support);
        if (pre_take_conjugate) g_conj->download(pre_take_conjugate);
        if (pre_conv_sum) g_csum->download(pre_conv_sum);

        GAFW::Tools::CppProperties::Properties none, with_support;
        with_support.set("with_support", 1);
        GAFW::GPU::StandardOperators::AccumulatedSum acc(nullptr, "GridIndexAccumulate");
        Arr grid_acc = make({U}, real_int, 4);
        run.submit(acc, {g_tog.get()}, {grid_acc.get()}, none);
        // CreateBlockIndex writes a sentinel over the last run's entry when
        // every record is gridded (CreateBlockIndex.cu:61-68): keep one out.
        {
            int last_acc = 0, last_tog = 0;
            checkCudaError(cudaMemcpy(&last_acc, (int *)grid_acc->d + (R - 1), 4, cudaMemcpyDeviceToHost), "read");
            checkCudaError(cudaMemcpy(&last_tog, (int *)g_tog->d + (R - 1), 4, cudaMemcpyDeviceToHost), "read");
            if (last_acc + last_tog >= R) return fail(err, errlen, "every record gridded: reference plan edge case");
        }
        mtimager::CreateIndexAndReorder reorder(nullptr, "CreateIndexAndReorder");
        Arr d_index = make({U}, real_int, 4), d_sup = make({U}, real_int, 4), d_cidx = make({U}, real_int, 4);
        run.submit(reorder, {g_tog.get(), grid_acc.get(), g_sup.get(), g_cidx.get()},
                   {d_index.get(), d_sup.get(), d_cidx.get()}, none);
        GAFW::GPU::StandardOperators::ValueChangeDetect change(nullptr, "NotSameSupportDetect");
        Arr nss = make({U}, real_int, 4), nss_acc = make({U}, real_int, 4);
        run.submit(change, {d_sup.get()}, {nss.get()}, none);
        GAFW::GPU::StandardOperators::AccumulatedSum acc1(nullptr, "NotSameSupportAccumulate");
        run.submit(acc1, {nss.get()}, {nss_acc.get()}, none);
        mtimager::CreateBlockIndex block1(nullptr, "CreateBlockDataIndex");
        block1.params = with_support;
        Arr bdi1 = make({U + 1, 2}, real_int, 4);
        run.submit(block1, {nss.get(), nss_acc.get(), d_sup.get()}, {bdi1.get()}, none);
        // NotSameSupportManipulate reads a 1025-entry shared table whose last
        // entry is only loaded when it lies inside the records
        // (NotSameSupportManipulate.cu:62-80): require the plan to end at
        // least 1025 entries before the last record.
        {
            int last_entry = 0;
            checkCudaError(cudaMemcpy(&last_entry, (int *)bdi1->d + 2 * R, 4, cudaMemcpyDeviceToHost), "read");
            if (last_entry < 0 || last_entry + 1100 >= R)
                return fail(err, errlen, "too many support runs for the reference plan kernels");
        }
        mtimager::NotSameSupportManipulate manip(nullptr, "NotSameSupportManipulate");
        Arr nss2 = make({U}, real_int, 4), nss2_acc = make({U}, real_int, 4);
        run.submit(manip, {nss.get(), bdi1.get()}, {nss2.get()}, none);
        GAFW::GPU::StandardOperators::AccumulatedSum acc2(nullptr, "NotSameSupportAccumulate2");
        run.submit(acc2, {nss2.get()}, {nss2_acc.get()}, none);
        mtimager::CreateBlockIndex block2(nullptr, "CreateBlockDataIndex2");
        block2.params = with_support;
        Arr bdi2 = make({U + 1, 2}, real_int, 4);
        run.submit(block2, {nss2.get(), nss2_acc.get(), d_sup.get()}, {bdi2.get()}, none);
        mtimager::CreateCompressionPlan cplan(nullptr, "CreateCompressionPlan");
        Arr plan = make({U + 1}, real_int, 4);
        run.submit(cplan, {d_index.get(), grid_acc.get(), g_toc.get()}, {plan.get()}, none);
        mtimager::CompressVisibilities comp(nullptr, "CompressVisibilities");
        Arr cvis = make({U, 2 * P}, real_float, 4);
        run.submit(comp, {d_index.get(), plan.get(), a_vis.get(), g_conj.get(), a_wt.get(), a_fl.get()},
                   {cvis.get()}, none);
        mtimager::ConvolutionGridder gridder(nullptr, "ConvolutionGridder");
        Arr g = make({(unsigned)ny, (unsigned)nx, P}, complex_float, 8);
        if (!initialize) g->upload(grid);
        GAFW::Tools::CppProperties::Properties gp;
        gp.set("initialize_output", initialize ? 1 : 0);
        run.submit(gridder, {bdi2.get(), d_index.get(), g_data.get(), cvis.get(), a_table.get(), d_cidx.get()},
                   {g.get()}, gp);
        g->download(grid);
        g_gridder_ms = run.own_ms;
        g_chain_ms = (float)run.chain_ms;
    } catch (const std::exception &e) {
        return fail(err, errlen, e.what());
    }
    return 0;
}

/* Device time of the last successful mtref_grid_chunk: the ConvolutionGridder
 * operator's kernels (its own events) and the whole operator graph of the
 * chunk (each submission's span, summed; the harness synchronises between
 * them as GAFW's engine does not). */
int mtref_last_chunk_ms(float *gridder_ms, float *chain_ms) {
    if (gridder_ms) *gridder_ms = g_gridder_ms;
    if (chain_ms) *chain_ms = g_chain_ms;
    return 0;
}

/* WProjectionConvFunction::calculate (WProjectionConvFunction.cpp:186-291)
 * with the per-plane chain of WPlaneConvFunctionCalculator
 * (WPlaneConvFunctionCalculator.cpp:36-66): casagridsf (generate) ->
 * WProjPreFFTConvFunc -> multiFFT2D -> ZeroToCentre2DShift -> SingleMultiply ->
 * ConvFunctionSupportFind; then ConvFunctionReOrganize per plane,
 * concatenation and SumConvolutionFunctions.  The scalars follow the module:
 * w_max = 0.25 / l_increment and the plane spacing in float
 * (WProjectionConvFunction.cpp:105-112), w_k = k^2 * increment in float
 * (:238), the divisor read from the unshifted w = 0 FFT at [0][0]
 * (WPlaneConvFunctionCalculator.cpp:128-142), supports capped at S_t - 2.
 *   table       out complex64 [table_capacity]
 *   conv_info   out int [wplanes][2], conv_sums out float [wplanes][T*T]
 *   table_elems out: elements written; divisor out: {re, im} */
int mtref_wkernels(int nx, int ny, double l_increment, double m_increment, int wplanes, int sampling, void *table,
                   int table_capacity, int *conv_info, float *conv_sums, int *table_elems, float *divisor,
                   char *err, int errlen) {
    try {
        Runner run;
        int st = std::min(nx, ny) / sampling;
        if (st % 2 == 0) st++;
        const unsigned S_t = (unsigned)st, PS = S_t * (unsigned)sampling;
        const int T = sampling % 2 ? sampling : sampling + 1;
        const float maxW = 0.25 / l_increment;
        const float wIncrement = wplanes == 1 ? 1.0f : maxW / (float)((wplanes - 1) * (wplanes - 1));
        GAFW::Tools::CppProperties::Properties taper_p, screen_p, find_p, none;
        typedef GAFW::Tools::CppProperties::Properties PR;
        taper_p.set("lmPlanePostCorrection", 1, PR::Bool);
        taper_p.set("generate", 1, PR::Bool);
        screen_p.set("sampling", sampling, PR::Int);
        screen_p.set("support", st, PR::Int);
        screen_p.set("total_l", l_increment * nx, PR::Double);
        screen_p.set("total_m", m_increment * ny, PR::Double);
        screen_p.set("lwimager-removeedge", 0, PR::Bool);
        find_p.set("ConvolutionFunction.sampling", sampling, PR::Int);
        find_p.set("ConvolutionFunction.takeaszero", 1e-3f, PR::Float);
        Arr taper = make({S_t, S_t}, real_float, 4);
        Arr screen = make({PS, PS}, complex_float, 8), fftd = make({PS, PS}, complex_float, 8);
        Arr shifted = make({PS, PS}, complex_float, 8), normed = make({PS, PS}, complex_float, 8);
        Arr sup = make({1}, real_float, 4);
        mtimager::CasaGridSF taper_op(nullptr, "taper");
        run.submit(taper_op, {}, {taper.get()}, taper_p);
        mtimager::WProjPreFFTConvFunc screen_op(nullptr, "preFFTConvFunction");
        screen_op.params = screen_p;    // read through getBoolParameter (WProjPreFFTconvFunc.cu:141)
        // divisor: the w = 0 plane's FFT at the origin, before the shift
        screen_p.set("w", 0.0f, PR::Float);
        run.submit(screen_op, {taper.get()}, {screen.get()}, screen_p);
        fft_planes(*screen, *fftd, CUFFT_FORWARD, run.stream);
        float dv[2];
        checkCudaError(cudaMemcpy(dv, fftd->d, 8, cudaMemcpyDeviceToHost), "read divisor");
        divisor[0] = dv[0];
        divisor[1] = dv[1];
        if (dv[1] > 1e-3) return fail(err, errlen, "w=0 origin has a non-zero imaginary part");
        const float multiplier = 1 / dv[0];
        GAFW::Tools::CppProperties::Properties mult_p;
        mult_p.set("multiplier.value", multiplier, PR::Float);
        GAFW::GPU::StandardOperators::ZeroToCentre2DShift shift_op(nullptr, "convFuncZeroShift");
        GAFW::GPU::StandardOperators::SingleMultiply mult_op(nullptr, "convNormalizer");
        mtimager::ConvFunctionSupportFind find_op(nullptr, "supportfind");
        mtimager::ConvFunctionReOrganize org_op(nullptr, "convFuncOrganise");
        int offset = 0;
        for (int k = 0; k < wplanes; k++) {
            const float w = k * k * wIncrement;
            screen_p.set("w", w, PR::Float);
            run.submit(screen_op, {taper.get()}, {screen.get()}, screen_p);
            fft_planes(*screen, *fftd, CUFFT_FORWARD, run.stream);
            run.submit(shift_op, {fftd.get()}, {shifted.get()}, none);
            run.submit(mult_op, {shifted.get()}, {normed.get()}, mult_p);
            run.submit(find_op, {normed.get()}, {sup.get()}, find_p);
            float fs = 0;
            checkCudaError(cudaMemcpy(&fs, sup->d, 4, cudaMemcpyDeviceToHost), "read support");
            int S = (int)fs;
            if (S > st - 2) S = st - 2;
            if (S < 1) return fail(err, errlen, "plane without support");
            const unsigned n = (unsigned)(T * T * S * S);
            if (offset + (int)n > table_capacity) return fail(err, errlen, "table capacity too small");
            Arr plane = make({n}, complex_float, 8);
            GAFW::Tools::CppProperties::Properties org_p;
            org_p.set("ConvolutionFunction.sampling", sampling, PR::Int);
            org_p.set("ConvolutionFunction.support", S, PR::Int);
            run.submit(org_op, {normed.get()}, {plane.get()}, org_p);
            checkCudaError(cudaMemcpy((char *)table + (size_t)offset * 8, plane->d, (size_t)n * 8,
                                      cudaMemcpyDeviceToHost), "read plane");
            conv_info[2 * k] = S;
            conv_info[2 * k + 1] = offset;
            offset += (int)n;
        }
        *table_elems = offset;
        Arr info = make({(unsigned)wplanes, 2}, real_int, 4), all = make({(unsigned)offset}, complex_float, 8);
        Arr sums = make({(unsigned)wplanes, (unsigned)(T * T)}, real_float, 4);
        info->upload(conv_info);
        all->upload(table);
        GAFW::Tools::CppProperties::Properties sum_p;
        sum_p.set("sampling", sampling, PR::Int);
        mtimager::SumConvolutionFunctions sum_op(nullptr, "SumConvolutionFunctions");
        run.submit(sum_op, {info.get(), all.get()}, {sums.get()}, sum_p);
        sums->download(conv_sums);
    } catch (const std::exception &e) {
        return fail(err, errlen, e.what());
    }
    return 0;
}

/* mode=normal kernels (OnlyTaperConvFunction.cpp:29-99): casagridsf (uv
 * gridding function, complex output) -> ConvFunctionReOrganize ->
 * SumConvolutionFunctions with convInfo = {support, 0}.
 *   table out complex64 [T*T*support*support], conv_sums out float [T*T] */
int mtref_taper_kernel(int support, int sampling, void *table, float *conv_sums, char *err, int errlen) {
    try {
        typedef GAFW::Tools::CppProperties::Properties PR;
        Runner run;
        const int T = sampling % 2 ? sampling : sampling + 1;
        const unsigned size = (unsigned)(support * sampling + (sampling % 2 ? 0 : 1));
        const unsigned n = (unsigned)(T * T * support * support);
        Arr full = make({size, size}, complex_float, 8), org = make({n}, complex_float, 8);
        Arr info = make({1, 2}, real_int, 4), sums = make({1, (unsigned)(T * T)}, real_float, 4);
        PR taper_p, org_p, sum_p;
        taper_p.set("lmPlanePostCorrection", 0, PR::Bool);
        taper_p.set("generate", 1, PR::Bool);
        taper_p.set("support", support, PR::Int);
        taper_p.set("sampling", sampling, PR::Int);
        mtimager::CasaGridSF taper_op(nullptr, "taper");
        run.submit(taper_op, {}, {full.get()}, taper_p);
        org_p.set("ConvolutionFunction.sampling", sampling, PR::Int);
        org_p.set("ConvolutionFunction.support", support, PR::Int);
        mtimager::ConvFunctionReOrganize org_op(nullptr, "convFuncOrganise");
        run.submit(org_op, {full.get()}, {org.get()}, org_p);
        const int ci[2] = {support, 0};
        info->upload(ci);
        sum_p.set("sampling", sampling, PR::Int);
        mtimager::SumConvolutionFunctions sum_op(nullptr, "SumConvolutionFunctions");
        run.submit(sum_op, {info.get(), org.get()}, {sums.get()}, sum_p);
        org->download(table);
        sums->download(conv_sums);
    } catch (const std::exception &e) {
        return fail(err, errlen, e.what());
    }
    return 0;
}

/* ImageFinalizer (ImageFinalizer.cpp:31-44): PreIFFTUVCorrection -> IFFT2D ->
 * ZeroToCentre2DShift -> StokesConverter -> casagridsf (lmPlanePostCorrection)
 * -> SincCorrector.
 *   grid        complex64 [ny][nx][P]; normalizer float [P]
 *   image       out float [P][ny][nx] */
int mtref_finalize(int nx, int ny, int npol, int sampling, int pol_type, const void *grid, const float *normalizer,
                   float *image, char *err, int errlen) {
    try {
        typedef GAFW::Tools::CppProperties::Properties PR;
        Runner run;
        const unsigned P = (unsigned)npol, X = (unsigned)nx, Y = (unsigned)ny;
        Arr g = make({Y, X, P}, complex_float, 8), prep = make({P, Y, X}, complex_float, 8);
        Arr ifft = make({P, Y, X}, complex_float, 8), shifted = make({P, Y, X}, complex_float, 8);
        Arr norm = make({P}, real_float, 4), stokes = make({P, Y, X}, real_float, 4);
        Arr tapered = make({P, Y, X}, real_float, 4), fin = make({P, Y, X}, real_float, 4);
        g->upload(grid);
        norm->upload(normalizer);
        PR none, stokes_p, taper_p, sinc_p;
        stokes_p.set("PolarizationType", pol_type, PR::Int);
        taper_p.set("lmPlanePostCorrection", 1, PR::Bool);
        taper_p.set("generate", 0, PR::Bool);
        taper_p.set("sampling", 1, PR::Int);
        sinc_p.set("sampling", sampling, PR::Int);
        mtimager::PreIFFTUVCorrection pre_op(nullptr, "FFTPrepare");
        run.submit(pre_op, {g.get()}, {prep.get()}, none);
        fft_planes(*prep, *ifft, CUFFT_INVERSE, run.stream);
        GAFW::GPU::StandardOperators::ZeroToCentre2DShift shift_op(nullptr, "Shift");
        run.submit(shift_op, {ifft.get()}, {shifted.get()}, none);
        mtimager::PostIFFTStokesConverter stokes_op(nullptr, "StokesConversion");
        run.submit(stokes_op, {shifted.get(), norm.get()}, {stokes.get()}, stokes_p);
        mtimager::CasaGridSF taper_op(nullptr, "TaperCorrection");
        run.submit(taper_op, {stokes.get()}, {tapered.get()}, taper_p);
        mtimager::SincCorrector sinc_op(nullptr, "SincCorrection");
        run.submit(sinc_op, {tapered.get()}, {fin.get()}, sinc_p);
        fin->download(image);
    } catch (const std::exception &e) {
        return fail(err, errlen, e.what());
    }
    return 0;
}

}  // extern "C"
