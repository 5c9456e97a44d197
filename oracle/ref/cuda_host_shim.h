/* Host-compilation shim for slices of the reference's CUDA sources.
 *
 * Test infrastructure only: lets g++ compile reference functions that are
 * marked __global__/__device__ so their CPU behaviour can be checked against
 * the oracle.  A kernel compiled through this shim runs as ONE thread
 * (threadIdx = blockIdx = 0, blockDim = gridDim = 1); only grid-stride loops
 * without __syncthreads (e.g. BotomUp-rtree.cu:73-94) are correct that way.
 */
#ifndef PRT_CUDA_HOST_SHIM_H
#define PRT_CUDA_HOST_SHIM_H
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>
#include <float.h>
#include <algorithm>
#include <vector>
using namespace std;

#define __global__
#define __device__
#define __host__
#define __constant__

struct prt_shim_dim3 { unsigned int x, y, z; };
static const prt_shim_dim3 threadIdx = {0u, 0u, 0u};
static const prt_shim_dim3 blockIdx = {0u, 0u, 0u};
static const prt_shim_dim3 blockDim = {1u, 1u, 1u};
static const prt_shim_dim3 gridDim = {1u, 1u, 1u};
#endif
