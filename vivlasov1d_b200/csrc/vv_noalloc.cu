// Invariants of a distribution function without a context and without any
// device allocation (vv_invariants_noalloc).
//
// The context entry point vv_invariants keeps its scratch (the x profile of
// phi, one row of partial sums per reduction block, the final sums) in
// buffers that vv_create allocates together with the whole solver: the GMRES
// basis, spectra and factorised preconditioner, some thirty-odd fields of
// nx*nv doubles, plus an autotuning pass.  A caller that only wants the
// diagnostics of fields it already holds on the device cannot afford that
// in several situations:
//   * a monitor or logging hook called between the steps of a running solve,
//     where cudaMalloc/cudaFree would synchronise the device and stall the
//     solve it is observing;
//   * a process whose device memory is fully reserved by another allocator
//     (a framework's caching pool), where a new cudaMalloc fails;
//   * analysis code that opens fields produced elsewhere (another process,
//     a checkpoint loaded by another library) and has no solver to build.
// Here the scratch lives in one file-scope __device__ array of fixed size,
// so the call allocates nothing.  What that costs:
//   * nx is limited to VV_NOALLOC_MAX_NX (the x profile of phi is kept in
//     the array); larger grids are refused with VV_ERR_UNSUPPORTED before
//     any device work;
//   * the array is one per device and shared by every caller in the
//     process: calls whose kernels overlap in time on the same device (from
//     two host threads, or on two streams without ordering between them)
//     overwrite each other's partial sums.  Serialise them (one stream, or a
//     synchronisation between calls).
//   * the first call on each device (and the first after that device's CUDA
//     context was destroyed and re-created) looks the array's address up
//     (cudaGetSymbolAddress), which may load the library's device code; make
//     that first call before any stream capture begins on that device.
// No part of the array has to start at zero: every word a kernel reads in a
// call was written earlier in the same call.
//
// The sums follow distribution_function.pyx:130-306, hamiltonian.pyx:67-124
// and potential.pyx:48-59 (vlasov/core) with the same compensated FP64
// accumulation, block shape and block count as vv_invariants.
#include "vv.h"
#include "vv_common.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>

namespace {

constexpr int NA_THREADS = 256;          // threads of the reduction blocks
constexpr int NA_PROFILE_THREADS = 1024; // threads of the one-block x profile
constexpr int NA_MAX_BLOCKS = 592;       // reduction blocks at most (4 x 148 SMs)
constexpr int NA_SUMS = 13;              // mass, L1..L6, L8, S, Ekin, Ep1, Ep2, P
constexpr int NA_ROWS = NA_SUMS + 2;     // + min, max

// scratch layout (doubles)
constexpr size_t NA_MEAN = 0;            // mean of phi
constexpr size_t NA_FE = 1;              // field energy
constexpr size_t NA_OUT = 16;            // NA_ROWS final values
constexpr size_t NA_HEAD = 32;           // words copied back to the host
constexpr size_t NA_PART = 64;           // NA_ROWS x blocks partial sums
constexpr size_t NA_H1 = NA_PART + (size_t)NA_ROWS * NA_MAX_BLOCKS;  // nx: phi - mean(phi)
constexpr size_t NA_WORDS = NA_H1 + VV_NOALLOC_MAX_NX;               // 25,328 doubles, about 198 KiB

// one block: h1 = phi - mean(phi), field energy 0.5 q sum (dphi)^2 / hx
__global__ void __launch_bounds__(NA_PROFILE_THREADS)
k_na_profile(const double* __restrict__ phi, int nx, double charge, double hx, double* __restrict__ s) {
    __shared__ double red[NA_PROFILE_THREADS / 32];
    __shared__ double mean_s;
    double t = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) t += phi[i];
    t = block_sum(t, red);
    if (threadIdx.x == 0) mean_s = t / nx;
    __syncthreads();
    double* h1 = s + NA_H1;
    double w = 0.0;
    for (int i = threadIdx.x; i < nx; i += blockDim.x) {
        h1[i] = phi[i] - mean_s;
        const double d = phi[(i + 1) % nx] - phi[i];
        w += d * d;
    }
    w = block_sum(w, red);
    if (threadIdx.x == 0) {
        s[NA_MEAN] = mean_s;
        s[NA_FE] = 0.5 * charge * w / hx;
    }
}

// per block: compensated partial sums of the 13 integrands, min and max of f.
// v_j = vmin + j hv and h0_j = (v_j^2 / 2) m are formed with the rounding of
// the host tables of vv_create (no fused multiply-add).
__global__ void __launch_bounds__(NA_THREADS)
k_na_partial(const double* __restrict__ f, int nx, int nv, double vmin, double hv, double mass,
             const double* __restrict__ h2, double* __restrict__ s) {
    __shared__ double sh[NA_THREADS / 32];
    __shared__ double shm[NA_THREADS / 32], shx[NA_THREADS / 32];
    const double* h1 = s + NA_H1;
    double* part = s + NA_PART;
    KSum acc[NA_SUMS];
#pragma unroll
    for (int q = 0; q < NA_SUMS; ++q) acc[q].init();
    double fmn = INFINITY, fmx = -INFINITY;
    const size_t n = (size_t)nx * nv;
    for (size_t idx = blockIdx.x * (size_t)NA_THREADS + threadIdx.x; idx < n; idx += (size_t)gridDim.x * NA_THREADS) {
        const int j = (int)(idx / nx), i = (int)(idx - (size_t)j * nx);
        const double vj = __dadd_rn(vmin, __dmul_rn((double)j, hv));
        const double h0j = __dmul_rn(__dmul_rn(0.5, __dmul_rn(vj, vj)), mass);
        const double fv = f[idx];
        fmn = fmin(fmn, fv);
        fmx = fmax(fmx, fv);
        acc[9].add(fv * h0j);
        acc[10].add(fv * h1[i]);
        if (h2) acc[11].add(fv * h2[i]);
        if (j < nv - 1) {
            // mass by the cell average of the four corners, as the reference
            const int ip = (i + 1 == nx) ? 0 : i + 1;
            const double s4 = ((fv + f[(size_t)j * nx + ip]) + f[(size_t)(j + 1) * nx + ip]) + f[(size_t)(j + 1) * nx + i];
            acc[0].add(s4);
            const double f2 = fv * fv, f3 = f2 * fv, f4 = f2 * f2;
            acc[1].add(fabs(fv));
            acc[2].add(f2);
            acc[3].add(f3);
            acc[4].add(f4);
            acc[5].add(f4 * fv);
            acc[6].add(f3 * f3);
            acc[7].add(f4 * f4);
            const double fe = fv <= 0.0 ? 1e-15 : fv;
            acc[8].add(fe * log(fe));
            acc[12].add(fv * vj);
        }
    }
    for (int q = 0; q < NA_SUMS; ++q) {
        const double t = block_sum(acc[q].value(), sh);
        if (threadIdx.x == 0) part[(size_t)q * gridDim.x + blockIdx.x] = t;
        __syncthreads();
    }
    double m = warp_min(fmn), x = warp_max(fmx);
    if ((threadIdx.x & 31) == 0) {
        shm[threadIdx.x >> 5] = m;
        shx[threadIdx.x >> 5] = x;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < NA_THREADS / 32; ++w) {
            m = fmin(m, shm[w]);
            x = fmax(x, shx[w]);
        }
        part[(size_t)NA_SUMS * gridDim.x + blockIdx.x] = m;
        part[(size_t)(NA_SUMS + 1) * gridDim.x + blockIdx.x] = x;
    }
}

// one block: the NA_ROWS final values from the np partial rows
__global__ void __launch_bounds__(NA_THREADS) k_na_final(int np, double* __restrict__ s) {
    __shared__ double sh[NA_THREADS / 32];
    const double* part = s + NA_PART;
    double* out = s + NA_OUT;
    for (int q = 0; q < NA_SUMS; ++q) {
        KSum a;
        a.init();
        for (int b = threadIdx.x; b < np; b += NA_THREADS) a.add(part[(size_t)q * np + b]);
        const double t = block_sum(a.value(), sh);
        if (threadIdx.x == 0) out[q] = t;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double m = INFINITY, x = -INFINITY;
        for (int b = 0; b < np; ++b) {
            m = fmin(m, part[(size_t)NA_SUMS * np + b]);
            x = fmax(x, part[(size_t)(NA_SUMS + 1) * np + b]);
        }
        out[NA_SUMS] = m;
        out[NA_SUMS + 1] = x;
    }
}

}  // namespace

// the scratch of every vv_invariants_noalloc call on a device
static __device__ __align__(256) double g_scratch[NA_WORDS];

namespace {

// device address of g_scratch, looked up once per device and CUDA context:
// a context destroyed and re-created (cudaDeviceReset, a driver-API context
// of its own) reloads the module, so the address of the old context is not
// reused -- the context's process-unique id (cuCtxGetId) keys the cache
constexpr int NA_MAX_DEVICES = 64;
struct ScratchOf {
    unsigned long long ctx_id;
    double* ptr;
};
std::mutex g_setup_mu;
ScratchOf g_scratch_of[NA_MAX_DEVICES] = {};

typedef int (*ctx_get_current_fn)(void**);
typedef int (*ctx_get_id_fn)(void*, unsigned long long*);

// id of the context current on this thread (0 if none or not available)
unsigned long long current_ctx_id() {
    static ctx_get_current_fn get_current = nullptr;
    static ctx_get_id_fn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void* f1 = nullptr;
        void* f2 = nullptr;
        cudaDriverEntryPointQueryResult q1, q2;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) == cudaSuccess &&
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) == cudaSuccess &&
            q1 == cudaDriverEntryPointSuccess && q2 == cudaDriverEntryPointSuccess) {
            get_current = (ctx_get_current_fn)f1;
            get_id = (ctx_get_id_fn)f2;
        }
        looked_up = true;
    }
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

int scratch_for_current_device(double** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return VV_ERR_CUDA;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return VV_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    unsigned long long id = current_ctx_id();
    ScratchOf& e = g_scratch_of[dev];
    if (!e.ptr || id == 0 || e.ctx_id != id) {
        // set-up on this device and context (the lookup makes the runtime's
        // context current if no call on this thread has done so yet)
        double* p = nullptr;
        if (cudaGetSymbolAddress((void**)&p, g_scratch) != cudaSuccess || !p) return VV_ERR_CUDA;
        if (id == 0) id = current_ctx_id();
        e.ptr = p;
        e.ctx_id = id;
    }
    *out = e.ptr;
    return VV_OK;
}

}  // namespace

extern "C" int vv_invariants_noalloc(const vv_grid* g, const double* f, const double* phi, const double* h2,
                                     void* cuda_stream, vv_invariant_set* out) {
    if (!g || !f || !phi || !out) return VV_ERR_ARG;
    if (g->nx < 4 || g->nv < 5 || !(g->L > 0.0) || !(g->vmax > g->vmin)) return VV_ERR_ARG;
    if (g->nx > VV_NOALLOC_MAX_NX) return VV_ERR_UNSUPPORTED;
    double* s = nullptr;
    int st = scratch_for_current_device(&s);
    if (st != VV_OK) return st;
    const cudaStream_t stream = (cudaStream_t)cuda_stream;
    const int nx = g->nx, nv = g->nv;
    const double hx = g->L / nx;
    const double hv = (g->vmax - g->vmin) / (nv - 1);
    const size_t n = (size_t)nx * nv;
    const int np = (int)std::max<size_t>(
        1, std::min<size_t>((n + (size_t)NA_THREADS * 8 - 1) / ((size_t)NA_THREADS * 8), (size_t)NA_MAX_BLOCKS));
    k_na_profile<<<1, NA_PROFILE_THREADS, 0, stream>>>(phi, nx, g->charge, hx, s);
    if (cudaGetLastError() != cudaSuccess) return VV_ERR_CUDA;
    k_na_partial<<<np, NA_THREADS, 0, stream>>>(f, nx, nv, g->vmin, hv, g->mass, h2, s);
    if (cudaGetLastError() != cudaSuccess) return VV_ERR_CUDA;
    k_na_final<<<1, NA_THREADS, 0, stream>>>(np, s);
    if (cudaGetLastError() != cudaSuccess) return VV_ERR_CUDA;
    double head[NA_HEAD];
    if (cudaMemcpyAsync(head, s, sizeof head, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return VV_ERR_CUDA;
    const double* r = head + NA_OUT;
    const double hxhv = hx * hv;
    out->mass = r[0] * 0.25 * hx * hv;
    out->L1 = hxhv * r[1];
    out->L2 = hxhv * r[2];
    out->L3 = hxhv * r[3];
    out->L4 = hxhv * r[4];
    out->L5 = hxhv * r[5];
    out->L6 = hxhv * r[6];
    out->L8 = hxhv * r[7];
    out->entropy = -hx * hv * r[8];
    out->E_kin = r[9] * hx * hv;
    out->E_pot = (r[10] + r[11]) * hx * hv;
    out->energy = out->E_kin + 0.5 * out->E_pot;
    out->momentum = r[12] * g->mass * hx * hv;
    out->Lmin = r[13] * hx * hv;
    out->Lmax = r[14] * hx * hv;
    out->field_energy = head[NA_FE];
    return VV_OK;
}
