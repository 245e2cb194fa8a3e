// fvm_noalloc.cu -- fvm_state_max_noalloc: the maximum temperature or local
// Mach number of a flow state that lives in the caller's own device memory,
// computed without allocating anything.
//
// Who needs this: a caller that keeps states outside any solve handle (a
// checkpoint held on the device, states gathered from several solves, the
// output of another solver in the same layout) and runs where it may not
// allocate -- for instance a process whose device memory is fully committed
// to solve instances up front, so a per-call cudaMalloc could fail or stall the
// device.  The handle-based fvm_max_temperature / fvm_max_mach need a handle,
// and creating one allocates the whole solve.
//
// How: the same per-cell quantity as k_max_reduce (fvm_aux.cu), one CTA per
// grid row.  Each CTA writes its row maximum into a fixed file-scope device
// array; the last CTA to arrive reduces the row maxima and stores the result
// in the same array.  The array's size caps the number of rows; larger grids
// are rejected before anything is launched.
#include <cuda.h>

#include <cstdio>
#include <mutex>

#include "fvm_handle.h"
#include "fvm_tma.cuh"

namespace fvm {
namespace {

constexpr int kNoAllocMaxRows = 16384;              // row maxima the scratch holds (64 KiB)
constexpr int kResultWord = kNoAllocMaxRows;        // float bits of the final maximum
constexpr int kArrivalWord = kNoAllocMaxRows + 32;  // CTA arrival counter (own 128-byte line)
constexpr int kScratchWords = kNoAllocMaxRows + 64;
constexpr int kMaxDevices = 64;
constexpr int kThreads = 256;

}  // namespace

// Word layout: [0, kNoAllocMaxRows) row maxima (float bits), kResultWord the
// result, kArrivalWord the arrival counter.  Only the arrival counter must be
// zero when a launch starts.  The host clears it with a 4-byte memset on the
// call's stream before every launch, so a launch that never finished (its
// context torn down mid-flight, say) cannot leave a count behind that would
// make a later launch pick the wrong last CTA.  The last CTA also sets it back
// to zero.  Row maxima are written before they are read in each launch, so
// they need no initial value.
static __device__ __align__(256) unsigned int g_noalloc_scratch[kScratchWords];

// what = 0: temperature, what = 1: local Mach number, cell by cell as
// k_max_reduce computes them (reference getMaxTemperature, src/solver.cu:2835-2867,
// and computeMachNumberKernel, src/solver.cu:2782-2794).  Launched with one
// CTA per row (gridDim.x = ny <= kNoAllocMaxRows) and kThreads threads.
__global__ void __launch_bounds__(kThreads)
    k_state_max_rows(int what, int nx, size_t pitch, size_t plane, const float *U, unsigned int *scratch) {
    const int j = blockIdx.x;
    const float *row = U + (size_t)j * pitch;
    float m = 0.0f;
    for (int i = threadIdx.x; i < nx; i += kThreads) {
        float u, v, p, T;
        const float rho = row[i];
        prim_from_cons(rho, row[plane + i], row[2 * plane + i], row[3 * plane + i], row[4 * plane + i], u, v, p, T);
        if (what == 0) {
            m = fmaxf(m, T);
        } else {
            float rho_val = rho + 1e-10f;
            float speed = sqrtf(u * u + v * v);
            float cs = sqrtf(GAMMA * p / rho_val);
            m = fmaxf(m, speed / (cs + 1e-10f));
        }
    }
    __shared__ float ws[kThreads / 32];
    __shared__ bool is_last;
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = 0.0f;
        for (int k = 0; k < kThreads / 32; k++) mm = fmaxf(mm, ws[k]);
        scratch[j] = __float_as_uint(mm);
        __threadfence();
        const unsigned int prev = atomicAdd(&scratch[kArrivalWord], 1u);
        is_last = (prev == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    float mm = 0.0f;
    for (int r = threadIdx.x; r < (int)gridDim.x; r += kThreads) mm = fmaxf(mm, __uint_as_float(__ldcg(&scratch[r])));
    mm = warp_max(mm);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = mm;
    __syncthreads();
    if (threadIdx.x == 0) {
        float r = 0.0f;
        for (int k = 0; k < kThreads / 32; k++) r = fmaxf(r, ws[k]);
        scratch[kResultWord] = __float_as_uint(r);
        scratch[kArrivalWord] = 0u;
    }
}

}  // namespace fvm

using namespace fvm;

// Device address of g_noalloc_scratch.  The address belongs to one CUDA
// context's copy of this module, not to a device index: after
// cudaDeviceReset, or with another context made current on the same device,
// the old address is stale.  So the cache is keyed on the current context's
// unique id (cuCtxGetId; ids are never reused within a process), and the
// lookup is repeated whenever the id changes.
namespace {
typedef CUresult (*PFN_ctxGetCurrent_t)(CUcontext *);
typedef CUresult (*PFN_ctxGetId_t)(CUcontext, unsigned long long *);
struct ScratchSlot {
    unsigned long long ctx_id = 0;
    unsigned int *addr = nullptr;
};
std::mutex g_scratch_mu;
ScratchSlot g_scratch_slot[kMaxDevices];

template <class F>
F driver_fn(const char *name) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint(name, &p, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
        return nullptr;
    return reinterpret_cast<F>(p);
}
}  // namespace

static int noalloc_err(int code, const char *fmt, long long a, long long b) {
    char buf[256];
    snprintf(buf, sizeof buf, fmt, a, b);
    return fvm_internal_set_error(code, buf);
}

extern "C" int fvm_state_max_noalloc(const float *state, int nx, int ny, size_t pitch, size_t plane, int what,
                                     float *out, void *stream) {
    if (!state || !out) return fvm_internal_set_error(FVM_ERR_INVALID, "fvm_state_max_noalloc: null pointer");
    if (what != 0 && what != 1)
        return fvm_internal_set_error(FVM_ERR_INVALID,
                                      "fvm_state_max_noalloc: what must be 0 (temperature) or 1 (Mach)");
    if (nx <= 0 || ny <= 0)
        return noalloc_err(FVM_ERR_INVALID, "fvm_state_max_noalloc: empty grid %lld x %lld", nx, ny);
    if (ny > kNoAllocMaxRows)
        return noalloc_err(FVM_ERR_INVALID,
                           "fvm_state_max_noalloc: ny = %lld rows exceeds the fixed scratch of %lld rows", ny,
                           kNoAllocMaxRows);
    if (pitch < (size_t)nx)
        return noalloc_err(FVM_ERR_INVALID, "fvm_state_max_noalloc: pitch %lld < nx %lld", (long long)pitch, nx);
    if (plane < pitch * (size_t)(ny - 1) + (size_t)nx)
        return noalloc_err(FVM_ERR_INVALID, "fvm_state_max_noalloc: plane %lld floats < the %lld a plane spans",
                           (long long)plane, (long long)(pitch * (size_t)(ny - 1) + (size_t)nx));
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices)
        return noalloc_err(FVM_ERR_UNSUPPORTED, "fvm_state_max_noalloc: device %lld beyond the %lld supported", dev,
                           kMaxDevices);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the call ends with a copy into pageable host memory and a stream
    // synchronize, neither of which a capturing stream allows
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if ((e = cudaStreamIsCapturing(st, &cap)) != cudaSuccess)
        return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    if (cap != cudaStreamCaptureStatusNone)
        return fvm_internal_set_error(FVM_ERR_STATE, "fvm_state_max_noalloc: the stream is being captured");
    static const PFN_ctxGetCurrent_t ctx_current = driver_fn<PFN_ctxGetCurrent_t>("cuCtxGetCurrent");
    static const PFN_ctxGetId_t ctx_id_of = driver_fn<PFN_ctxGetId_t>("cuCtxGetId");
    if (!ctx_current || !ctx_id_of)
        return fvm_internal_set_error(FVM_ERR_UNSUPPORTED, "fvm_state_max_noalloc: cuCtxGetId unavailable");
    CUcontext ctx = nullptr;
    if (ctx_current(&ctx) != CUDA_SUCCESS)
        return fvm_internal_set_error(FVM_ERR_CUDA, "fvm_state_max_noalloc: cuCtxGetCurrent failed");
    if (!ctx) {
        // no context current on this thread yet: the runtime's symbol lookup
        // makes the device's primary context current (allocating nothing)
        unsigned int *probe = nullptr;
        if ((e = cudaGetSymbolAddress((void **)&probe, g_noalloc_scratch)) != cudaSuccess)
            return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
        if (ctx_current(&ctx) != CUDA_SUCCESS || !ctx)
            return fvm_internal_set_error(FVM_ERR_CUDA, "fvm_state_max_noalloc: no current CUDA context");
    }
    unsigned long long ctx_id = 0;
    if (ctx_id_of(ctx, &ctx_id) != CUDA_SUCCESS)
        return fvm_internal_set_error(FVM_ERR_CUDA, "fvm_state_max_noalloc: cuCtxGetId failed");
    unsigned int *scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_scratch_mu);
        ScratchSlot &slot = g_scratch_slot[dev];
        if (slot.addr == nullptr || slot.ctx_id != ctx_id) {
            e = cudaGetSymbolAddress((void **)&scratch, g_noalloc_scratch);
            if (e != cudaSuccess) return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
            slot.addr = scratch;
            slot.ctx_id = ctx_id;
        }
        scratch = slot.addr;
    }
    if ((e = cudaMemsetAsync(scratch + kArrivalWord, 0, sizeof(unsigned int), st)) != cudaSuccess)
        return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    k_state_max_rows<<<ny, kThreads, 0, st>>>(what, nx, pitch, plane, state, scratch);
    if ((e = cudaGetLastError()) != cudaSuccess) return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    e = cudaMemcpyAsync(out, scratch + kResultWord, sizeof(float), cudaMemcpyDeviceToHost, st);
    if (e != cudaSuccess) return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fvm_internal_set_error(FVM_ERR_CUDA, cudaGetErrorString(e));
    return FVM_OK;
}
