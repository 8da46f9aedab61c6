// The reference includes CUB from a 3rdparty/cub submodule checkout
// (<cub/cub/cub.cuh>); the submodule is not vendored.  This forwards to the
// CUB that ships with the CUDA toolkit.
#include <cub/cub.cuh>
