// Device helpers shared by the libvv kernels: complex arithmetic on double2,
// deterministic block reductions and the bounded-wait error flag.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define VV_DEV __device__ __forceinline__

// n / d by one wide multiply with m = ceil(2^32 / d): floor(n m / 2^32)
// equals floor(n / d) whenever n d < 2^32 (the excess n (m - 2^32/d) / 2^32
// stays below 1/d).  For the pad-slot index r / CH of the staged tridiagonal
// lines (r < nv, CH = ceil(nv / 32): exact for nv below 370,000).
struct FastDiv {
    unsigned long long m;
    VV_DEV explicit FastDiv(unsigned d) : m((0xFFFFFFFFull + d) / d) {}
    VV_DEV unsigned operator()(unsigned n) const { return (unsigned)(((unsigned long long)n * m) >> 32); }
};

VV_DEV double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
VV_DEV double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
VV_DEV double2 c_mul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
VV_DEV double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
VV_DEV double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
// multiply by a complex number that is given as (real scalar) * (complex lam)
VV_DEV double2 c_rmul(double2 lam, double s) { return make_double2(lam.x * s, lam.y * s); }

// float2 counterparts (single-precision complex)
VV_DEV float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
VV_DEV float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
VV_DEV float2 c_mul(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
VV_DEV float2 c_conj(float2 a) { return make_float2(a.x, -a.y); }
VV_DEV float2 c_scale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
VV_DEV float2 c_rmul(float2 lam, float s) { return make_float2(lam.x * s, lam.y * s); }

// complex type of a real type
template <typename R> struct Cplx;
template <> struct Cplx<double> { using type = double2; };
template <> struct Cplx<float> { using type = float2; };
template <typename C> VV_DEV C c_make(double x, double y);
template <> VV_DEV double2 c_make<double2>(double x, double y) { return make_double2(x, y); }
template <> VV_DEV float2 c_make<float2>(double x, double y) { return make_float2((float)x, (float)y); }

// Warp sum of a double (all lanes get the result).
VV_DEV double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
VV_DEV double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
VV_DEV double warp_min(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum; result valid in linear thread 0.  `sh` must hold
// (threads per block)/32 doubles.  Works for 1-D and 2-D blocks.
VV_DEV double block_sum(double v, double* sh) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y;
    const int lane = tid & 31, wid = tid >> 5;
    const int nw = (blockDim.x * blockDim.y + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0) {
        r = (lane < nw) ? sh[lane] : 0.0;
        r = warp_sum(r);
    }
    return r;
}

// Neumaier compensated accumulator.
struct KSum {
    double s, c;
    VV_DEV void init() { s = 0.0; c = 0.0; }
    VV_DEV void add(double x) {
        double t = s + x;
        if (fabs(s) >= fabs(x)) c += (s - t) + x; else c += (x - t) + s;
        s = t;
    }
    VV_DEV double value() const { return s + c; }
};

// Asynchronous global -> shared copies (cp.async, sm_80+): a zero src_bytes
// fills the destination with zeros and reads nothing.
VV_DEV void cp_async_16(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
VV_DEV void cp_async_8(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
VV_DEV void cp_async_4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, 4;\n" ::"r"(s), "l"(gmem));
}
// one element of 4, 8 or 16 bytes
template <typename E>
VV_DEV void cp_async_elem(E* smem, const E* gmem) {
    static_assert(sizeof(E) == 4 || sizeof(E) == 8 || sizeof(E) == 16, "cp.async copies 4, 8 or 16 bytes");
    if (sizeof(E) == 16) cp_async_16(smem, gmem, 16);
    else if (sizeof(E) == 8) cp_async_8(smem, gmem, 8);
    else cp_async_4(smem, gmem);
}
// the waits clobber memory so that no shared-memory read moves above them
VV_DEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
VV_DEV void cp_async_wait2() { asm volatile("cp.async.wait_group 2;\n" ::: "memory"); }
VV_DEV void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
VV_DEV void cp_async_wait0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
