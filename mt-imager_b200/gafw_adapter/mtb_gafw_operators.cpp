// GAFW operators over the mtb C ABI (mtb_gafw_operators.h).
#include "mtb_gafw_operators.h"

#include <climits>
#include <cstring>
#include <vector>

using namespace GAFW;
using namespace GAFW::GPU;
using namespace GAFW::GeneralImplimentation;
using GAFW::Tools::CppProperties::Properties;

// A status code as the exception GAFW expects (GPUafw.h:28-33): CUDA failures
// as CudaException, FFT and kernel-generation failures as GeneralException,
// everything a caller can fix as ValidationException.
#define MTB_GAFW_TRY(call, where)                                                                 \
    do {                                                                                          \
        const int mtb_rc_ = (call);                                                               \
        if (mtb_rc_ != MTB_OK) {                                                                  \
            const std::string mtb_msg_ = std::string(where) + ": " + mtb_status_string(mtb_rc_);   \
            if (mtb_rc_ == MTB_ERR_CUDA) throw CudaException(mtb_msg_, cudaGetLastError());        \
            if (mtb_rc_ == MTB_ERR_CUFFT || mtb_rc_ == MTB_ERR_KERNEL) throw GeneralException(mtb_msg_); \
            throw ValidationException(mtb_msg_);                                                  \
        }                                                                                         \
    } while (0)

namespace mtb_gafw {
namespace {

// GAFW hands the scratch size to submitToGPU as an int (GPUSubmissionData.h:42)
const size_t kMaxScratch = (size_t)INT_MAX;

int columns(Array *a) { return (int)a->getDimensions().getNoOfColumns(); }
int rows(Array *a) { return (int)a->getDimensions().getNoOfRows(); }

// mtb_grid_params from the PreProcessUVW keys (WImager.cpp:186-191) and the
// shapes of the inputs: planes = rows of the position array, polarisations =
// columns of the weights.
mtb_grid_params grid_params(const Properties &pr, int wplanes, int npol) {
    mtb_grid_params p;
    std::memset(&p, 0, sizeof(p));
    p.nx = pr.getIntProperty("uvImage.columns");
    p.ny = pr.getIntProperty("uvImage.rows");
    p.npol = npol;
    p.sampling = pr.getIntProperty("ConvolutionFunction.sampling");
    p.wplanes = wplanes;
    p.u_increment = pr.getFloatProperty("uvImage.u_increment");
    p.v_increment = pr.getFloatProperty("uvImage.v_increment");
    p.w_sq_increment = pr.getFloatProperty("ConvolutionFunction.wsquareincrement");
    return p;
}

// convInfo with every plane at the largest support a plane can have: an upper
// bound of the scratch before the table exists (mtb_grid sizes its plan from
// the supports).
std::vector<int> worst_conv_info(int wplanes, int max_support) {
    int S = max_support < 1 ? 1 : (max_support > 255 ? 255 : max_support);
    if (S % 2 == 0) S--;
    std::vector<int> ci((size_t)wplanes * 2, 0);
    for (int k = 0; k < wplanes; k++) ci[2 * (size_t)k] = S;
    return ci;
}

// The position array (convInfo) read back to the host on the operator's stream.
std::vector<int> host_conv_info(const GPUArrayDescriptor &d, cudaStream_t st) {
    const size_t n = (size_t)d.dim.getTotalNoOfElements();
    std::vector<int> h(n);
    checkCudaError(cudaMemcpyAsync(h.data(), d.pointer, n * sizeof(int), cudaMemcpyDeviceToHost, st),
                   "reading ConvolutionFunctionPosition");
    checkCudaError(cudaStreamSynchronize(st), "reading ConvolutionFunctionPosition");
    return h;
}

void set_out(Array *a, const ArrayDimensions &d, StoreType t) {
    a->setDimensions(d);
    a->setType(t);
}

// The operator's timing span, as the reference's operators record it
// (CompressVisibilties.cu:82-96): the engine records the end itself when an
// operator has not.
void record_start(GPUSubmissionData &d) {
    if (d.startEvent) checkCudaError(cudaEventRecord(*d.startEvent, d.stream), "Unable to record event");
}
void record_end(GPUSubmissionData &d) {
    if (d.endEvent) {
        checkCudaError(cudaEventRecord(*d.endEvent, d.stream), "Unable to record event");
        d.endEventRecorded = true;
    }
}

}  // namespace

// ------------------------------------------------------------ PreProcessUVW --
MtbPreProcessUVW::MtbPreProcessUVW(GPUFactory *factory, std::string nickname)
    : GPUArrayOperator(factory, nickname, "Operator::PreProcessUVW") {}

void MtbPreProcessUVW::validate(ValidationData &data) {
    if (this->inputs.size() != 6) throw ValidationException("PreProcessUVW expects six inputs");
    if (this->outputs.size() != 7) throw ValidationException("PreProcessUVW expects seven outputs");
    this->checkParameter("ConvolutionFunction.sampling", Properties::Int);
    this->checkParameter("ConvolutionFunction.wsquareincrement", Properties::Float);
    this->checkParameter("uvImage.u_increment", Properties::Float);
    this->checkParameter("uvImage.v_increment", Properties::Float);
    this->checkParameter("uvImage.rows", Properties::Int);
    this->checkParameter("uvImage.columns", Properties::Int);
    this->checkParameter("ConvolutionFunction.maxsupport", Properties::Int);
    const int P = columns(this->inputs[4]);
    const int R = columns(this->inputs[2]);
    const int nw = rows(this->inputs[0]);
    mtb_grid_params p = grid_params(this->params, nw, P);
    p.no_grid_lo = 1;                         // preprocessing holds no delta grid
    const std::vector<int> ci = worst_conv_info(nw, this->params.getIntProperty("ConvolutionFunction.maxsupport"));
    size_t bytes = 0;
    MTB_GAFW_TRY(mtb_grid_workspace_size(&p, ci.data(), R, &bytes), "PreProcessUVW");
    if (bytes > kMaxScratch) throw ValidationException("PreProcessUVW: chunk too large for an int scratch size");
    data.bufferMode = Buffer::Buffer_Normal;
    data.bufferSize = bytes;
    // WProjPreProcessUVW.cpp:66-85
    set_out(this->outputs[0], ArrayDimensions(2, R, 4), real_int);
    set_out(this->outputs[1], ArrayDimensions(1, R), real_int);
    set_out(this->outputs[2], ArrayDimensions(1, R), real_int);
    set_out(this->outputs[3], ArrayDimensions(1, R), real_int);
    set_out(this->outputs[4], ArrayDimensions(1, R), real_int);
    set_out(this->outputs[5], ArrayDimensions(1, R), real_float);
    set_out(this->outputs[6], ArrayDimensions(2, P, R), real_float);
}

void MtbPreProcessUVW::submitToGPU(GPUSubmissionData &d) {
    const int P = (int)d.inputs[4].dim.getNoOfColumns();
    const int R = (int)d.inputs[2].dim.getNoOfColumns();
    const int nw = (int)d.inputs[0].dim.getNoOfRows();
    mtb_grid_params p = grid_params(d.params, nw, P);
    p.no_grid_lo = 1;
    const std::vector<int> ci = host_conv_info(d.inputs[0], d.stream);
    record_start(d);
    MTB_GAFW_TRY(mtb_preprocess_uvw(&p, (const int *)d.inputs[0].pointer, ci.data(), (const float *)d.inputs[1].pointer,
                                    (const float *)d.inputs[2].pointer, (const float *)d.inputs[3].pointer,
                                    (const float *)d.inputs[4].pointer, (const int *)d.inputs[5].pointer, R,
                                    (int *)d.outputs[0].pointer, (int *)d.outputs[1].pointer,
                                    (int *)d.outputs[2].pointer, (int *)d.outputs[3].pointer,
                                    (int *)d.outputs[4].pointer, (float *)d.outputs[5].pointer,
                                    (float *)d.outputs[6].pointer, d.bufferGPUPointer, (size_t)d.buffersize,
                                    (mtb_stream_t)d.stream),
                 "PreProcessUVW");
    record_end(d);
}

// ---------------------------------------------------------------- GridChunk --
MtbGridChunk::MtbGridChunk(GPUFactory *factory, std::string nickname)
    : GPUArrayOperator(factory, nickname, "Operator::mtb::GridChunk") {}

void MtbGridChunk::validate(ValidationData &data) {
    if (this->inputs.size() != 8) throw ValidationException("mtb::GridChunk expects eight inputs");
    if (this->outputs.size() != 5) throw ValidationException("mtb::GridChunk expects five outputs");
    this->checkParameter("ConvolutionFunction.sampling", Properties::Int);
    this->checkParameter("ConvolutionFunction.wsquareincrement", Properties::Float);
    this->checkParameter("uvImage.u_increment", Properties::Float);
    this->checkParameter("uvImage.v_increment", Properties::Float);
    this->checkParameter("uvImage.rows", Properties::Int);
    this->checkParameter("uvImage.columns", Properties::Int);
    this->checkParameter("ConvolutionFunction.maxsupport", Properties::Int);
    this->checkParameter("initialize_output", Properties::Bool);
    const int P = columns(this->inputs[6]);
    const int R = columns(this->inputs[3]);
    const int nw = rows(this->inputs[1]);
    mtb_grid_params p = grid_params(this->params, nw, P);
    p.external_delta = 1;                     // the delta grid is output 4
    const std::vector<int> ci = worst_conv_info(nw, this->params.getIntProperty("ConvolutionFunction.maxsupport"));
    size_t bytes = 0, delta = 0;
    MTB_GAFW_TRY(mtb_grid_workspace_size(&p, ci.data(), R, &bytes), "mtb::GridChunk");
    MTB_GAFW_TRY(mtb_grid_delta_bytes(&p, &delta), "mtb::GridChunk");
    if (bytes > kMaxScratch) throw ValidationException("mtb::GridChunk: chunk too large for an int scratch size");
    data.bufferMode = Buffer::Buffer_Normal;
    data.bufferSize = bytes;
    // Grid and its compensation term as WImager.cpp:230-234 declares the Grid
    set_out(this->outputs[0], ArrayDimensions(3, p.ny, p.nx, P), complex_float);
    set_out(this->outputs[1], ArrayDimensions(3, p.ny, p.nx, P), complex_float);
    set_out(this->outputs[2], ArrayDimensions(1, P), real_float);
    set_out(this->outputs[3], ArrayDimensions(1, 4), real_ulongint);
    const bool fp64 = delta == (size_t)p.nx * p.ny * P * 2 * sizeof(double);
    set_out(this->outputs[4], ArrayDimensions(3, p.ny, p.nx, 2 * P), fp64 ? real_double : real_float);
}

void MtbGridChunk::submitToGPU(GPUSubmissionData &d) {
    const int P = (int)d.inputs[6].dim.getNoOfColumns();
    const int R = (int)d.inputs[3].dim.getNoOfColumns();
    const int nw = (int)d.inputs[1].dim.getNoOfRows();
    mtb_grid_params p = grid_params(d.params, nw, P);
    p.initialize_output = d.params.getBoolProperty("initialize_output") ? 1 : 0;
    p.external_delta = 1;
    p.d_delta = d.outputs[4].pointer;
    const std::vector<int> ci = host_conv_info(d.inputs[1], d.stream);
    record_start(d);
    MTB_GAFW_TRY(mtb_grid(&p, d.inputs[0].pointer, (const int *)d.inputs[1].pointer, ci.data(),
                          (const float *)d.inputs[2].pointer, (const float *)d.inputs[3].pointer,
                          (const float *)d.inputs[4].pointer, d.inputs[5].pointer, (const float *)d.inputs[6].pointer,
                          (const int *)d.inputs[7].pointer, R, d.outputs[0].pointer, d.outputs[1].pointer,
                          (float *)d.outputs[2].pointer, (mtb_grid_stats *)d.outputs[3].pointer, d.bufferGPUPointer,
                          (size_t)d.buffersize, (mtb_stream_t)d.stream),
                 "mtb::GridChunk");
    record_end(d);
}

// ----------------------------------------------------------- ImageFinalizer --
MtbImageFinalizer::MtbImageFinalizer(GPUFactory *factory, std::string nickname)
    : GPUArrayOperator(factory, nickname, "Operator::mtb::ImageFinalizer") {}

static mtb_finalize_params finalize_params(const Properties &pr, const ArrayDimensions &grid) {
    mtb_finalize_params p;
    std::memset(&p, 0, sizeof(p));
    p.ny = (int)grid.getZ();
    p.nx = (int)grid.getY();
    p.npol = (int)grid.getX();
    p.sampling = pr.getIntProperty("ConvolutionFunction.sampling");
    p.pol_type = pr.getIntProperty("PolarizationType");
    p.external_planes = 1;                    // the FFT planes are output 1
    return p;
}

void MtbImageFinalizer::validate(ValidationData &data) {
    if (this->inputs.size() != 3) throw ValidationException("mtb::ImageFinalizer expects three inputs");
    if (this->outputs.size() != 2) throw ValidationException("mtb::ImageFinalizer expects two outputs");
    this->checkParameter("ConvolutionFunction.sampling", Properties::Int);
    this->checkParameter("PolarizationType", Properties::Int);
    if (this->inputs[0]->getDimensions().getNoOfDimensions() != 3)
        throw ValidationException("mtb::ImageFinalizer: the grid is [rows][columns][polarisations]");
    mtb_finalize_params p = finalize_params(this->params, this->inputs[0]->getDimensions());
    size_t bytes = 0;
    MTB_GAFW_TRY(mtb_finalize_workspace_size(&p, &bytes), "mtb::ImageFinalizer");
    if (bytes > kMaxScratch) throw ValidationException("mtb::ImageFinalizer: FFT work area too large for an int");
    data.bufferMode = Buffer::Buffer_Normal;
    data.bufferSize = bytes;
    set_out(this->outputs[0], ArrayDimensions(3, p.npol, p.ny, p.nx), real_float);
    set_out(this->outputs[1], ArrayDimensions(3, p.npol, p.ny, p.nx), complex_double);
}

void MtbImageFinalizer::submitToGPU(GPUSubmissionData &d) {
    mtb_finalize_params p = finalize_params(d.params, d.inputs[0].dim);
    p.d_planes = d.outputs[1].pointer;
    record_start(d);
    MTB_GAFW_TRY(mtb_finalize(&p, d.inputs[0].pointer, d.inputs[1].pointer, (const float *)d.inputs[2].pointer,
                              (float *)d.outputs[0].pointer, d.bufferGPUPointer, (size_t)d.buffersize,
                              (mtb_stream_t)d.stream),
                 "mtb::ImageFinalizer");
    record_end(d);
}

// -------------------------------------------------- WProjectionConvFunction --
MtbWProjectionConvFunction::MtbWProjectionConvFunction(GPUFactory *factory, std::string nickname)
    : GPUArrayOperator(factory, nickname, "Operator::mtb::WProjectionConvFunction") {}

static mtb_wkernel_params wkernel_params(const Properties &pr) {
    mtb_wkernel_params p;
    std::memset(&p, 0, sizeof(p));
    p.nx = pr.getIntProperty("image.nx");
    p.ny = pr.getIntProperty("image.ny");
    p.l_increment = pr.getDoubleProperty("image.lintervalsize");
    p.m_increment = pr.getDoubleProperty("image.mintervalsize");
    p.wplanes = pr.getIntProperty("wproj.wplanes");
    p.sampling = pr.getIntProperty("wproj.convFunction.sampling");
    p.trial_support = pr.getIntProperty("wproj.convFunction.trialsupport");
    p.max_support = pr.getIntProperty("wproj.convFunction.maxsupport");
    p.w_max = pr.getDoubleProperty("wproj.wmax");
    return p;
}

void MtbWProjectionConvFunction::validate(ValidationData &data) {
    if (!this->inputs.empty()) throw ValidationException("mtb::WProjectionConvFunction takes no inputs");
    if (this->outputs.size() != 3) throw ValidationException("mtb::WProjectionConvFunction expects three outputs");
    this->checkParameter("image.nx", Properties::Int);
    this->checkParameter("image.ny", Properties::Int);
    this->checkParameter("image.lintervalsize", Properties::Double);
    this->checkParameter("image.mintervalsize", Properties::Double);
    this->checkParameter("wproj.wplanes", Properties::Int);
    this->checkParameter("wproj.convFunction.sampling", Properties::Int);
    this->checkParameter("wproj.convFunction.trialsupport", Properties::Int);
    this->checkParameter("wproj.convFunction.maxsupport", Properties::Int);
    this->checkParameter("wproj.wmax", Properties::Double);
    const mtb_wkernel_params p = wkernel_params(this->params);
    mtb_wkernel_info info;
    MTB_GAFW_TRY(mtb_wkernel_query(&p, &info), "mtb::WProjectionConvFunction");
    if (info.workspace_bytes > kMaxScratch)
        throw ValidationException("mtb::WProjectionConvFunction: work area too large for an int");
    if (info.table_capacity > (size_t)INT_MAX)
        throw ValidationException("mtb::WProjectionConvFunction: table too large for GAFW array dimensions");
    data.bufferMode = Buffer::Buffer_Normal;
    data.bufferSize = info.workspace_bytes;
    set_out(this->outputs[0], ArrayDimensions(1, (int)info.table_capacity), complex_float);
    set_out(this->outputs[1], ArrayDimensions(2, p.wplanes, 2), real_int);
    set_out(this->outputs[2], ArrayDimensions(2, p.wplanes, info.T * info.T), real_float);
}

void MtbWProjectionConvFunction::submitToGPU(GPUSubmissionData &d) {
    const mtb_wkernel_params p = wkernel_params(d.params);
    std::vector<int> ci((size_t)p.wplanes * 2);
    size_t elems = 0;
    record_start(d);
    MTB_GAFW_TRY(mtb_wkernel_build(&p, d.bufferGPUPointer, (size_t)d.buffersize, d.outputs[0].pointer,
                                   (size_t)d.outputs[0].dim.getTotalNoOfElements(), (int *)d.outputs[1].pointer,
                                   ci.data(), (float *)d.outputs[2].pointer, &elems, (mtb_stream_t)d.stream),
                 "mtb::WProjectionConvFunction");
    record_end(d);
}

GPUArrayOperator *create_operator(GPUFactory *factory, const std::string &nickname, const std::string &name) {
    if (name == "PreProcessUVW") return new MtbPreProcessUVW(factory, nickname);
    if (name == "mtb::GridChunk") return new MtbGridChunk(factory, nickname);
    if (name == "mtb::ImageFinalizer") return new MtbImageFinalizer(factory, nickname);
    if (name == "mtb::WProjectionConvFunction") return new MtbWProjectionConvFunction(factory, nickname);
    return nullptr;
}

}  // namespace mtb_gafw
