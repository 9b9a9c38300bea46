// Shared device helpers for the AFQMC walker-step engine (sm_100a).
//
// Complex numbers are stored interleaved as double2 (x = real, y = imag),
// the same memory layout as std::complex<double> in the reference's
// TensorHao (common/tensorHao/include/tensor_core.h:83-91), so walker
// matrices move between host and device without reformatting.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

typedef double2 zd;

#define HD __host__ __device__ __forceinline__

HD zd zmk(double r, double i) { return make_double2(r, i); }
HD zd zadd(zd a, zd b) { return make_double2(a.x + b.x, a.y + b.y); }
HD zd zsub(zd a, zd b) { return make_double2(a.x - b.x, a.y - b.y); }
HD zd zmul(zd a, zd b) { return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); }
HD zd zconj(zd a) { return make_double2(a.x, -a.y); }
HD zd zneg(zd a) { return make_double2(-a.x, -a.y); }
HD zd zscale(zd a, double s) { return make_double2(a.x * s, a.y * s); }
// acc += a * b
HD void zfma(zd &acc, zd a, zd b)
{
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
}
HD double zabs(zd a) { return hypot(a.x, a.y); }
HD double zcabs1(zd a) { return fabs(a.x) + fabs(a.y); }
HD zd zdiv(zd a, zd b)
{
    // Smith's algorithm (robust complex division)
    if (fabs(b.y) <= fabs(b.x)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.y + b.x * r;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}
HD zd zexp(zd a)
{
    double e = exp(a.x), s, c;
    sincos(a.y, &s, &c);
    return make_double2(e * c, e * s);
}
HD zd zlog(zd a) { return make_double2(log(zabs(a)), atan2(a.y, a.x)); }
HD bool zeq0(zd a) { return a.x == 0.0 && a.y == 0.0; }

// ---------------------------------------------------------------------------
// Counter-based random numbers (replaces the reference's SPRNG stream,
// common/randomHao/source/random_hao.cpp:73-85).  Uniform number k of the
// stream `seed` is the SplitMix64 output for state mix(seed) + (k+1)*golden;
// any position of the stream is computable independently, so each walker
// reads its own slice of the reference's sequential, walker-major stream.
// ---------------------------------------------------------------------------
HD uint64_t rng_mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
HD double rng_uniform(uint64_t seed, uint64_t k)
{
    uint64_t b = rng_mix64(rng_mix64(seed) + (k + 1ULL) * 0x9E3779B97F4A7C15ULL);
    return (double)(b >> 11) * 0x1.0p-53;
}
// gaussianHao(): Box-Muller from draws k (log) and k+1 (cos), u==0 -> 1e-300.
HD double rng_gaussian(uint64_t seed, uint64_t k)
{
    double u1 = rng_uniform(seed, k);
    if (u1 == 0.0) u1 += 1e-300;
    double u2 = rng_uniform(seed, k + 1);
    return sqrt(-2.0 * log(u1)) * cos(2.0 * 3.14159265358979324 * u2);
}

// ---------------------------------------------------------------------------
// Block reductions (deterministic: fixed tree order for a fixed blockDim).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v)
{
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
// Sum over the block; every thread receives the result.  scratch >= 32 doubles.
__device__ __forceinline__ double block_sum(double v, double *scratch)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < nw ? scratch[lane] : 0.0;
        r = warp_sum(r);
        if (lane == 0) scratch[0] = r;
    }
    __syncthreads();
    r = scratch[0];
    __syncthreads();
    return r;
}
__device__ __forceinline__ double block_max(double v, double *scratch)
{
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_max(v);
    __syncthreads();
    if (lane == 0) scratch[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = lane < nw ? scratch[lane] : -1e308;
        r = warp_max(r);
        if (lane == 0) scratch[0] = r;
    }
    __syncthreads();
    r = scratch[0];
    __syncthreads();
    return r;
}
__device__ __forceinline__ zd block_zsum(zd v, double *scratch)
{
    double r = block_sum(v.x, scratch);
    double i = block_sum(v.y, scratch);
    return make_double2(r, i);
}

// Per-walker status bits written by the kernels (never a trap or abort).
enum {
    ST_SINGULAR = 1,     // zero pivot in the overlap LU
    ST_NONFINITE = 2,    // NaN/Inf in a walker quantity
    ST_TAYLOR_CAP = 4,   // Taylor series hit the order cap before converging
    ST_ZERO_NORM = 8,    // zero column norm in Gram-Schmidt
};
