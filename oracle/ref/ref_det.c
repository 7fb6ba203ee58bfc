/* TEST INFRASTRUCTURE ONLY: compiles the reference's deterministic diffusion
 * kernels (Deterministic.cl) unchanged for the CPU.  The RK4 and alpha-QSS
 * reaction kernels need generated right-hand sides and stay out (GPGMP_NUM_REACTIONS 0). */
#include "cl_shim.h"
#define GPGMP_SOLVER_DETERMINISTIC_RK4
#include "Deterministic.cl"
