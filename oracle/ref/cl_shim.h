/*
 * oracle/ref/cl_shim.h -- TEST INFRASTRUCTURE ONLY (builds the reference checker).
 *
 * Lets the reference's OpenCL C kernel sources compile unchanged as C for the CPU:
 * address-space qualifiers become empty, work-item queries read variables the
 * driver sets before each call, vector types become structs, and the model
 * constants that Solver::oclGenerateHeader (Solver.cpp:449-567) would print into
 * the program header become variables set from the model at run time, with the
 * same printed precision.  The address macros repeat the ones that header
 * defines (Solver.cpp:470-477).  Kernels that need a work-group barrier run with
 * a local size of 1.
 */
#ifndef GPGMP_CL_SHIM_H
#define GPGMP_CL_SHIM_H
#include <stddef.h>
#include <stdint.h>
#include <math.h>

#define __kernel
#define __global
#define __local
#define __constant
#define CLK_LOCAL_MEM_FENCE 0
#define barrier(x) ((void)0)

typedef float Real;
typedef struct { int x, y; } int2;
typedef struct { int x, y, z, w; } int4;
typedef struct { float x, y, z, w; } float4;

#include <Random123/threefry.h>

#define M_RAN_INVM32 2.32830643653869628906e-010

extern size_t shim_gid[2], shim_gsize[2], shim_lid[2], shim_lsize[2], shim_group[2], shim_ngroups[2];
static inline size_t get_global_id(int d) { return shim_gid[d]; }
static inline size_t get_global_size(int d) { return shim_gsize[d]; }
static inline size_t get_local_id(int d) { return shim_lid[d]; }
static inline size_t get_local_size(int d) { return shim_lsize[d]; }
static inline size_t get_group_id(int d) { return shim_group[d]; }
static inline size_t get_num_groups(int d) { return shim_ngroups[d]; }

#define get_global_area_2d (GridModelWidth * GridModelHeight)
#define get_local_area_2d  (get_local_size(0)  * get_local_size(1))
#define get_global_id_2d   (get_global_id(0) + (get_global_id(1) * GridModelWidth))
#define get_local_id_2d    (get_local_id(0)  + (get_local_id(1)  * get_local_size(0)))
#define get_block_id_2d    (get_group_id(0)  + (get_group_id(1)  * get_num_groups(0)))
#define get_global_id_for_species_2d(SPECIES_INDEX) (get_global_id_2d + (SPECIES_INDEX*get_global_area_2d))
#define get_local_id_for_species_2d(SPECIES_INDEX) (get_local_id_2d + (SPECIES_INDEX*get_local_area_2d))

#define GPGMP_DIMENSIONALITY 3
#define GPGMP_NUM_REACTIONS 0
#define GPGMP_NUM_SPECIES ((int)NumSpecies)
#define GPGMP_STATE_TYPE int
#define GPGMP_SOLVER_STOCHASTIC_INHOMOGENEOUS

extern size_t GridModelWidth, GridModelHeight, NumReactions, NumSpecies;
extern Real PhysicalModelWidth, PhysicalModelHeight, PhysicalCellWidth, PhysicalCellHeight, StayProbability;
extern int BoundaryMaskX1, BoundaryMaskX2, BoundaryMaskY1, BoundaryMaskY2;

#endif
