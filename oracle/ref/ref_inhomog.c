/* TEST INFRASTRUCTURE ONLY: compiles the reference's inhomogeneous drift-diffusion
 * kernels (StochasticInhomogeneousDriftDiffusion.cl, helpers.cl) unchanged for the CPU,
 * with the float overloads OpenCL gives its math functions. */
#include "cl_shim.h"
#include <tgmath.h>   /* OpenCL's math overloads: tanh of a float is the float tanh */
#define min(a, b) fminf((a), (b))
#include "StochasticInhomogeneousDriftDiffusion.cl"
