/*
 * mtb_gafw_operators.h -- GAFW operators over the mtb C ABI.
 *
 * The drop-in for mt-imager's dataflow: GAFW::GPU::GPUArrayOperator subclasses
 * (code/gafw/Implimentation/GPUImplimentation/GPUArrayOperator.h:27-43) that
 * mt-imager's operator factory hands out by name
 * (code/mt-imager/lib/operators/ImagerFactoryHelper.cpp:45-87: add the names
 * below to createOperator).  Each one declares its outputs and its scratch in
 * validate(ValidationData &), enqueues the library's work on the engine's
 * stream in submitToGPU(GPUSubmissionData &), and turns status codes into the
 * exceptions GAFW expects (CudaException, ValidationException, GeneralException:
 * GPUafw.h:28-33, GAFWValidationException.h:29).
 *
 *   "PreProcessUVW"        MtbPreProcessUVW: the reference operator's inputs,
 *                          outputs and parameters (WProjPreProcessUVW.cpp:39-86,
 *                          WImager.cpp:167-172, 186-191), one call of
 *                          mtb_preprocess_uvw.
 *   "mtb::GridChunk"       MtbGridChunk: one WImager chunk, the operator graph of
 *                          WImager.cpp:167-234 from PreProcessUVW to
 *                          ConvolutionGridder and the normaliser / statistics sums,
 *                          one call of mtb_grid.
 *   "mtb::ImageFinalizer"  MtbImageFinalizer: ImageFinalizer.cpp:31-44, one call of
 *                          mtb_finalize.
 *   "mtb::WProjectionConvFunction"  MtbWProjectionConvFunction: the tables
 *                          WProjectionConvFunction::calculate builds
 *                          (WProjectionConvFunction.cpp:186-291), one call of
 *                          mtb_wkernel_build.
 *
 * Scratch and GAFW's int buffer size.  GAFW allocates an operator's scratch with
 * the size_t that validate() asks for, but hands its size to submitToGPU as an
 * int (GPUSubmissionData.h:42).  The two large work areas of the path are
 * therefore outputs of their operators, arrays the engine owns and can keep
 * reusable as it keeps the grid (WImager.cpp:226-234): the gridder's per-call
 * delta grid (mtb_grid_params.external_delta) and the finaliser's FP64 FFT planes
 * (mtb_finalize_params.external_planes).  validate() refuses a configuration
 * whose remaining scratch does not fit an int.
 *
 * Host reads.  mtb_grid and mtb_preprocess_uvw plan with the per-plane supports
 * on the host; submitToGPU reads the convInfo input back (a few hundred bytes)
 * and synchronises the stream once per call for it, as the reference's own
 * FFT and support operators synchronise.  mtb_wkernel_build synchronises once
 * to bring the supports to the host (WPlaneConvFunctionCalculator.cpp:117-126
 * does so once per plane).
 */
#ifndef MTB_GAFW_OPERATORS_H
#define MTB_GAFW_OPERATORS_H

#include <string>
#include <vector>

#include "GPUafw.h"
#include "mtb.h"

namespace mtb_gafw {

// Inputs 0..5: ConvolutionFunctionPosition (int [nw][2]), ConvolutionFunctionSums
// (float [nw][T*T]), UVWData (float [3][R]), LSRK frequencies (float [R]),
// weights (float [R][P]), flags (int [R][P]).  Outputs 0..6: GriddingData
// (int [R][4]), GriddingDataConvolutionIndex, ToGridIndicator,
// ToCompressIndicator, GriddingDataSupport (int [R]), TakeConjugateIndicator
// (float [R]), ConvolutionFunctionSum (float [P][R]).  Parameters:
// ConvolutionFunction.sampling (Int), ConvolutionFunction.wsquareincrement
// (Float), uvImage.u_increment, uvImage.v_increment (Float), uvImage.rows,
// uvImage.columns (Int), ConvolutionFunction.maxsupport (Int: the largest
// support a plane can have, which sizes the scratch before the table exists).
class MtbPreProcessUVW : public GAFW::GPU::GPUArrayOperator {
public:
    MtbPreProcessUVW(GAFW::GPU::GPUFactory *factory, std::string nickname);
    virtual void validate(GAFW::GPU::ValidationData &data);
    virtual void submitToGPU(GAFW::GPU::GPUSubmissionData &data);
};

// Inputs 0..7: ConvolutionFunction (complex float, the table), its Position and
// Sums arrays, UVWData, LSRK frequencies, Visibilities (complex float [R][P]),
// weights, flags (as for MtbPreProcessUVW).  Outputs 0..4: Grid (complex float
// [ny][nx][P]), GridCompensation (the same: the two-float grid's lower part),
// NormalizerValue (float [P]), Statistics (unsigned long [4]: gridded records,
// compressed records, gridded points, compressed points), DeltaGrid (float or
// double [ny][nx][2P]: the call's delta grid, kept by nobody).  Outputs 0..3
// accumulate over chunks; the engine keeps them reusable.  Parameters: those of
// MtbPreProcessUVW and initialize_output (Bool).
class MtbGridChunk : public GAFW::GPU::GPUArrayOperator {
public:
    MtbGridChunk(GAFW::GPU::GPUFactory *factory, std::string nickname);
    virtual void validate(GAFW::GPU::ValidationData &data);
    virtual void submitToGPU(GAFW::GPU::GPUSubmissionData &data);
};

// Inputs 0..2: Grid, GridCompensation, NormalizerValue (the outputs of
// MtbGridChunk).  Outputs 0..1: the Stokes image (float [P][ny][nx]) and
// FinalizePlanes (complex double [P][ny][nx], kept by nobody).  Parameters:
// ConvolutionFunction.sampling (Int, the SincCorrector's sampling),
// PolarizationType (Int: 0 linear, 1 circular).
class MtbImageFinalizer : public GAFW::GPU::GPUArrayOperator {
public:
    MtbImageFinalizer(GAFW::GPU::GPUFactory *factory, std::string nickname);
    virtual void validate(GAFW::GPU::ValidationData &data);
    virtual void submitToGPU(GAFW::GPU::GPUSubmissionData &data);
};

// No inputs.  Outputs 0..2: ConvolutionFunction (complex float
// [table_capacity]; the planes' tables concatenated from element 0),
// ConvolutionFunctionPosition (int [nw][2]), ConvolutionFunctionSums (float
// [nw][T*T]).  Parameters: image.nx, image.ny (Int), image.lintervalsize,
// image.mintervalsize (Double, radians), wproj.wplanes,
// wproj.convFunction.sampling, wproj.convFunction.trialsupport,
// wproj.convFunction.maxsupport (Int; 0 selects the reference's rules),
// wproj.wmax (Double; 0: the reference's rule).
class MtbWProjectionConvFunction : public GAFW::GPU::GPUArrayOperator {
public:
    MtbWProjectionConvFunction(GAFW::GPU::GPUFactory *factory, std::string nickname);
    virtual void validate(GAFW::GPU::ValidationData &data);
    virtual void submitToGPU(GAFW::GPU::GPUSubmissionData &data);
};

// The operator for `name` (the names above), or NULL: the lines a maintainer
// adds to ImagerFactoryHelper::createOperator.
GAFW::GPU::GPUArrayOperator *create_operator(GAFW::GPU::GPUFactory *factory, const std::string &nickname,
                                             const std::string &name);

}  // namespace mtb_gafw

#endif
