/* TEST INFRASTRUCTURE ONLY: compiles the reference's homogeneous stochastic
 * diffusion kernels (StochasticHomogeneousDiffusion.cl) unchanged for the CPU. */
#include "cl_shim.h"
#include "StochasticHomogeneousDiffusion.cl"
