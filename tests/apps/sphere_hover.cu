// CUDA side of sphere_drop's hover hook: adds a constant force to one object.
#include "kernel/CUDAKernelFunction/myUtility/myVec.h"

__global__ void addConstantForce(double3* force, int index, double3 f) { force[index] += f; }

extern "C" void launchAddConstantForce(double3* force, int index, double3 f, cudaStream_t stream)
{
    addConstantForce<<<1, 1, 0, stream>>>(force, index, f);
}
