/*
 * mtimager.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * Stand-in for mt-imager's master header (code/mt-imager/lib/mtimager.h),
 * which pulls in casacore for the MeasurementSet reader.  The operator
 * sources compiled by oracle/build_ref.py only need the polarisation type
 * (mtimager.h:30-37), declared here with the same names and values.
 */
#ifndef MTREF_MTIMAGER_STUB_H
#define MTREF_MTIMAGER_STUB_H
#include "GPUafw.h"

namespace mtimager {
namespace PolarizationType {
enum Type { Linear, Circular };
}
}  // namespace mtimager

#endif
