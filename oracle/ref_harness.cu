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
#include "ValueChangeDetect.h"

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
    cudaEvent_t ev0, ev1;
    GAFW::GPU::GPUDeviceDescriptor device;
    Runner() {
        checkCudaError(cudaStreamCreate(&stream), "stream");
        checkCudaError(cudaEventCreate(&ev0), "event");
        checkCudaError(cudaEventCreate(&ev1), "event");
    }
    ~Runner() {
        cudaEventDestroy(ev0);
        cudaEventDestroy(ev1);
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
        op.submitToGPU(d);
        checkCudaError(cudaGetLastError(), "launch of " + op.nickname);
        checkCudaError(cudaStreamSynchronize(stream), "run of " + op.nickname);
        if (post) op.postRunExecute(post);
    }
};

int fail(char *err, int errlen, const char *msg) {
    if (err && errlen > 0) {
        std::strncpy(err, msg, errlen - 1);
        err[errlen - 1] = 0;
    }
    return 1;
}

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
    } catch (const std::exception &e) {
        return fail(err, errlen, e.what());
    }
    return 0;
}

}  // extern "C"
