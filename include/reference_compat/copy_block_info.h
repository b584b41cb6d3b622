/* copy_block_info.h - forwarding header with the reference's file name (its include/copy_block_info.h):
 * host code written against the reference's headers compiles unchanged against
 * libcbns_b200 when this directory precedes the reference's include directory. */
#ifndef CBNS_COMPAT_COPY_BLOCK_INFO_H_
#define CBNS_COMPAT_COPY_BLOCK_INFO_H_
#include "../block3d_cuda.h"
#endif
