/*
 * gafw.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 * Stand-in for GAFW's public header; everything the compiled operator
 * sources need is in the GPUafw.h stand-in next to this file.
 */
#ifndef MTREF_GAFW_STUB_H
#define MTREF_GAFW_STUB_H
#include "GPUafw.h"
#endif
