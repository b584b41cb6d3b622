/* get_conservative.h - forwarding header with the reference's file name (its include/get_conservative.h):
 * host code written against the reference's headers compiles unchanged against
 * libcbns_b200 when this directory precedes the reference's include directory. */
#ifndef CBNS_COMPAT_GET_CONSERVATIVE_H_
#define CBNS_COMPAT_GET_CONSERVATIVE_H_
#include "../block3d_cuda.h"
#endif
