/*
 * cuda_host.h -- lets the reference's CUDA kernel source compile as host C++
 * so that its own code can serve as the oracle's pin.  TEST INFRASTRUCTURE
 * ONLY (see ref_driver.cpp); the product never includes it.
 *
 * Force-included (g++ -include) ahead of gpu_blastp_kernel.cu:
 *   - the CUDA qualifiers (__global__, __device__, __shared__, __constant__)
 *     expand to nothing, so the kernel and its three extenders become plain
 *     functions and the constant arrays plain globals;
 *   - gridDim/blockDim are process globals and blockIdx/threadIdx are
 *     thread-local: ref_driver.cpp runs one POSIX thread per CUDA thread of a
 *     block, and __syncthreads() is a barrier across those threads;
 *   - `texture<...>` is an empty class template, so the unused legacy texture
 *     reference declared at gpu_blastp_kernel.h:37 compiles as an unused
 *     global object instead of being removed from the source.
 */
#ifndef BLASTP_REFSHIM_CUDA_HOST_H
#define BLASTP_REFSHIM_CUDA_HOST_H

#include <pthread.h>

#define __global__
#define __device__
#define __host__
#define __shared__
#define __constant__

struct uint3 { unsigned int x, y, z; };
typedef uint3 dim3;

extern dim3 gridDim;
extern dim3 blockDim;
extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern pthread_barrier_t refshim_block_barrier;

static inline void __syncthreads(void) { pthread_barrier_wait(&refshim_block_barrier); }

enum cudaTextureReadMode { cudaReadModeElementType = 0, cudaReadModeNormalizedFloat = 1 };
template <class T, int dim, enum cudaTextureReadMode mode> struct texture {};

#endif
