/*
 * GPUafw.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A minimal stand-in for the GAFW engine headers, written for this project,
 * so that mt-imager's own operator sources (their kernels and submitToGPU
 * launch code) compile unchanged outside GAFW and can be driven by
 * oracle/ref_harness.cu to produce reference outputs, and so that the GAFW
 * operator adapter (mt-imager_b200/gafw_adapter/) compiles and runs in the
 * tests.  Only the names those sources use are provided; the interface
 * mirrors GAFW's
 * (gafw/Implimentation/GPUImplimentation/GPUafw.h:28-70,
 *  GPUSubmissionData.h:27-47, GPUArrayOperator.h:27-43,
 *  gafw/pil/ArrayDimensions.h:31-83, GeneralImplimentation/Array.h:59-78,
 *  GeneralImplimentation/ArrayOperator.h:41-91,
 *  GeneralImplimentation/GAFWValidationException.h:29-45) because the operator
 * sources are written against it.  The engine itself (scheduling, memory, validation)
 * is not reproduced: the harness allocates every buffer and calls
 * submitToGPU directly.
 */
#ifndef MTREF_GPUAFW_STUB_H
#define MTREF_GPUAFW_STUB_H

#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

typedef unsigned int uint;

class CudaException : public std::runtime_error {
public:
    CudaException(const std::string &msg, cudaError_t err)
        : std::runtime_error(msg + ": " + cudaGetErrorString(err)), err(err) {}
    cudaError_t err;
};

#define checkCudaError(x, msg)                                    \
    {                                                             \
        cudaError_t _mtref_err_ = (x);                            \
        if (_mtref_err_ != cudaSuccess) throw CudaException(msg, _mtref_err_); \
    }

namespace GAFW {

class GeneralException : public std::runtime_error {
public:
    explicit GeneralException(const std::string &msg) : std::runtime_error(msg) {}
};

// Dimensions listed slowest first; the last one is X (columns).
class ArrayDimensions {
public:
    ArrayDimensions() {}
    explicit ArrayDimensions(const std::vector<unsigned> &d) : dims(d) {}
    ArrayDimensions(int noOfDims, int dim0 = 0, int dim1 = 0, int dim2 = 0, int dim3 = 0, int dim4 = 0) {
        const int d[5] = {dim0, dim1, dim2, dim3, dim4};
        for (int i = 0; i < noOfDims && i < 5; i++) dims.push_back((unsigned)d[i]);
    }
    int getNoOfDimensions() const { return (int)dims.size(); }
    unsigned getNoOfColumns() const { return dims.empty() ? 0 : dims.back(); }
    unsigned getNoOfRows() const { return dims.size() < 2 ? 1 : dims[dims.size() - 2]; }
    unsigned getX() const { return getNoOfColumns(); }
    unsigned getY() const { return getNoOfRows(); }
    unsigned getZ() const { return dims.size() < 3 ? 1 : dims[dims.size() - 3]; }
    unsigned getTotalNoOfElements() const {
        unsigned n = dims.empty() ? 0 : 1;
        for (unsigned d : dims) n *= d;
        return n;
    }
    std::vector<unsigned> dims;
};

namespace GeneralImplimentation {
enum StoreType { real_int, real_uint, real_float, real_double, complex_float, complex_double, real_longint,
                 real_ulongint, real_shortint, real_ushortint, StoreTypeUnknown };

// An operator's input or output as validate() sees it.
class Array {
public:
    ArrayDimensions getDimensions() { return dim; }
    void setDimensions(ArrayDimensions d) { dim = d; }
    StoreType getType() { return type; }
    void setType(StoreType t) { type = t; }
    bool isDefined() { return dim.getNoOfDimensions() > 0; }
    ArrayDimensions dim;
    StoreType type = StoreTypeUnknown;
};

class GAFWValidationException : public GeneralException {
public:
    GAFWValidationException(std::string desc, void *, int linenumber, std::string file)
        : GeneralException(desc + " (" + file + ":" + std::to_string(linenumber) + ")") {}
};
}  // namespace GeneralImplimentation

namespace Tools { namespace CppProperties {
class Properties {
public:
    enum PropertyType { Int, Float, Double, Bool, Complex };
    int getIntProperty(const std::string &k) const { return (int)get(k).value; }
    float getFloatProperty(const std::string &k) const { return (float)get(k).value; }
    double getDoubleProperty(const std::string &k) const { return get(k).value; }
    bool getBoolProperty(const std::string &k) const { return get(k).value != 0.0; }
    std::complex<float> getComplexProperty(const std::string &k) const {
        return std::complex<float>((float)get(k).value, 0.0f);
    }
    PropertyType getPropertyType(const std::string &k) const { return get(k).type; }
    void set(const std::string &k, double v, PropertyType t = Double) { values[k] = Entry{v, t}; }

private:
    struct Entry {
        double value;
        PropertyType type;
    };
    const Entry &get(const std::string &k) const {
        auto it = values.find(k);
        if (it == values.end()) throw GeneralException("property not set: " + k);
        return it->second;
    }
    std::map<std::string, Entry> values;
};
}}  // namespace Tools::CppProperties

namespace GPU {
class GPUFactory;

namespace Buffer {
enum BufferType { Buffer_Normal, Buffer_DeallocBeforeSubmit, Buffer_UnkownSize };
}

typedef struct {
    void *pointer;
    GAFW::ArrayDimensions dim;
    GAFW::GeneralImplimentation::StoreType type;
} GPUArrayDescriptor;

// Launch shape covering a rows x columns array with 16 x 16 thread blocks
// (small enough for every operator kernel's register use on sm_100a).
class GPUDeviceDescriptor {
public:
    int getBestThreadsAndBlocksDim(const int rows, const int columns, dim3 &blocks, dim3 &threads) {
        threads = dim3(16, 16, 1);
        blocks = dim3((unsigned)(columns + 15) / 16, (unsigned)(rows + 15) / 16, 1);
        if (blocks.x == 0) blocks.x = 1;
        if (blocks.y == 0) blocks.y = 1;
        return 0;
    }
};

class ValidationData {
public:
    Buffer::BufferType bufferMode = Buffer::Buffer_Normal;
    size_t bufferSize = 0;
};

class GPUSubmissionData {
public:
    int noOfInputs = 0;
    GPUArrayDescriptor *inputs = nullptr;
    int noOfOutputs = 0;
    GPUArrayDescriptor *outputs = nullptr;
    cudaStream_t stream = 0;
    void **postExecutePointer = nullptr;
    cudaEvent_t *startEvent = nullptr;
    cudaEvent_t *endEvent = nullptr;
    bool endEventRecorded = false;
    GAFW::Tools::CppProperties::Properties params;
    void *bufferGPUPointer = nullptr;
    int buffersize = 0;
    GPUDeviceDescriptor *deviceDescriptor = nullptr;
};

class GPUArrayOperator {
public:
    enum LogCategory { other, execution, execution_submission };
    GPUArrayOperator(GPUFactory *, std::string nickname, std::string name = "GPUMatrixOperator")
        : nickname(nickname), name(name) {}
    virtual ~GPUArrayOperator() {}
    virtual void validate() {}
    virtual void validate(ValidationData &) {}
    virtual void submitToGPU(GPUSubmissionData &data) = 0;
    virtual void postRunExecute(void *) {}
    bool getBoolParameter(const std::string &k) const { return params.getBoolProperty(k); }
    void logDebug(int, const std::string &) {}
    void logWarn(int, const std::string &) {}
    void logInfo(int, const std::string &) {}
    GAFW::Tools::CppProperties::Properties params;
    std::string nickname, name;
    std::vector<GAFW::GeneralImplimentation::Array *> inputs;
    std::vector<GAFW::GeneralImplimentation::Array *> outputs;
    // throws unless the parameter is set with this type
    void checkParameter(std::string param, GAFW::Tools::CppProperties::Properties::PropertyType type) {
        if (params.getPropertyType(param) != type)
            throw GAFW::GeneralImplimentation::GAFWValidationException("parameter " + param + " has another type",
                                                                       this, __LINE__, __FILE__);
    }
};
}  // namespace GPU
}  // namespace GAFW

#define ValidationException(description) \
    GAFW::GeneralImplimentation::GAFWValidationException(description, this, __LINE__, __FILE__)

#endif
