// Accuracy of the library's reciprocal square root (necg::rsq) and reciprocal
// (necg::rcp) against IEEE 1/sqrt(x) and 1/x, over 2^24 inputs with random
// mantissas and exponents in [-40, 40].  Prints the largest distances in units
// in the last place.  Test infrastructure: built and run by
// tests/test_gpu_special.py.
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include "necg_math.cuh"

__device__ __forceinline__ uint64_t mix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ unsigned long long ulps(double a, double b) {
    const long long d = (long long)__double_as_longlong(a) - (long long)__double_as_longlong(b);
    return d < 0 ? (unsigned long long)-d : (unsigned long long)d;
}
__global__ void probe(long long n, unsigned long long *out) {
    unsigned long long ms = 0, mr = 0;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const uint64_t r = mix((uint64_t)i);
        const double x = ldexp(1.0 + (double)(r >> 11) * 0x1.0p-53, (int)((r & 0x7ff) % 81) - 40);
        const unsigned long long s = ulps(necg::rsq(x), 1.0 / sqrt(x));
        const unsigned long long c = ulps(necg::rcp(x), 1.0 / x);
        if (s > ms) ms = s;
        if (c > mr) mr = c;
    }
    atomicMax(out, ms);
    atomicMax(out + 1, mr);
}
int main() {
    unsigned long long *d = nullptr, h[2] = {0, 0};
    if (cudaMalloc(&d, sizeof(h)) != cudaSuccess || cudaMemset(d, 0, sizeof(h)) != cudaSuccess) return 1;
    probe<<<148 * 8, 256>>>(1ll << 24, d);
    if (cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost) != cudaSuccess) return 2;
    cudaFree(d);
    printf("rsq_max_ulp %llu rcp_max_ulp %llu\n", h[0], h[1]);
    return 0;
}
