/* Build shim: rocHPL device files include <hip/hip_runtime.h>; under nvcc the
 * CUDA runtime (pulled in by the shim hpl.hpp) provides everything they use. */
#pragma once
#include <cuda_runtime.h>
