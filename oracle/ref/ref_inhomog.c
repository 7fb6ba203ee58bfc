/* TEST INFRASTRUCTURE ONLY: compiles the reference's inhomogeneous drift-diffusion
 * kernels (StochasticInhomogeneousDriftDiffusion.cl, helpers.cl) unchanged for the CPU. */
#include "cl_shim.h"
#define min(a, b) fminf((a), (b))
#include "StochasticInhomogeneousDriftDiffusion.cl"
