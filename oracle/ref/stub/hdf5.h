/* Stand-in for <hdf5.h> when building the reference's CPU path without
 * libhdf5: the reference header io/hdf5_file.h only needs the handle type.
 * The hdf5_file class itself is implemented in oracle/ref/hdf5_file_shim.cpp
 * on top of nebula_b200/csrc/h5lite. */
#pragma once
#include <stdint.h>
typedef int64_t hid_t;
