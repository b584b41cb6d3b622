/* calc_numerical_flux.h - forwarding header with the reference's file name (its include/calc_numerical_flux.h):
 * host code written against the reference's headers compiles unchanged against
 * libcbns_b200 when this directory precedes the reference's include directory. */
#ifndef CBNS_COMPAT_CALC_NUMERICAL_FLUX_H_
#define CBNS_COMPAT_CALC_NUMERICAL_FLUX_H_
#include "../block3d_cuda.h"
#endif
