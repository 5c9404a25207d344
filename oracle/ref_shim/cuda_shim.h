/* Host build of the reference's device functions (test infrastructure only).
 *
 * Force-included before device_function.cu when oracle/Makefile's ref_harness
 * target compiles that file with g++ for the CPU, so that the oracle's fold,
 * field and smart-MC energy can be checked against the reference's own
 * functions.  It maps the CUDA qualifiers to nothing, gives the launch
 * coordinates as host globals the harness sets, and stands in for the few
 * CUDA/cuRAND calls the file makes: normals come from a queue the harness
 * fills (so the reference's trial uses chosen numbers), uniforms are a fixed
 * value, atomics are plain read-modify-writes (one host thread). */
#pragma once
#include <assert.h>
#include <math.h>
#include <stdbool.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include <vector>

#define __device__
#define __global__
#define __host__
#define __forceinline__ inline

struct dim3 {
    unsigned int x = 0, y = 0, z = 0;
};
struct float4 {
    float x, y, z, w;
};
struct double4 {
    double x, y, z, w;
};

extern dim3 blockIdx, threadIdx, gridDim, blockDim;

/* cuRAND stand-ins */
struct curandStatePhilox4_32_10_t {
    unsigned int unused;
};
typedef curandStatePhilox4_32_10_t curandStatePhilox4_32_10;
void curand_init(unsigned long long seed, unsigned long long seq, unsigned long long off, curandStatePhilox4_32_10_t* s);
float curand_uniform(curandStatePhilox4_32_10_t* s);
double curand_uniform_double(curandStatePhilox4_32_10_t* s);
float4 curand_normal4(curandStatePhilox4_32_10_t* s);
double4 curand_normal4_double(curandStatePhilox4_32_10_t* s);

/* CUDA intrinsics used by the file, for one host thread */
inline void __syncthreads() {}
inline void __threadfence() {}
inline int atomicAdd(int* a, int v) {
    const int o = *a;
    *a = o + v;
    return o;
}
inline unsigned long long atomicCAS(unsigned long long* a, unsigned long long cmp, unsigned long long v) {
    const unsigned long long o = *a;
    if (o == cmp) *a = v;
    return o;
}
inline float atomicExch(float* a, float v) {
    const float o = *a;
    *a = v;
    return o;
}
inline long long __double_as_longlong(double d) {
    long long r;
    memcpy(&r, &d, sizeof r);
    return r;
}
inline double __longlong_as_double(long long v) {
    double r;
    memcpy(&r, &v, sizeof r);
    return r;
}

/* types named by gpu_info.h */
struct cudaDeviceProp {
    char name[256];
};
typedef void* cudaStream_t;

/* the reference's bounds check traps the GPU (asm("trap;")); on the host it aborts */
#define asm(text) abort()
