// noalloc.cu -- the incremental walk decision without any device allocation.
//
// Some callers cannot call cudaMalloc: a serving loop that reserves all of its
// device memory at start-up and forbids allocation afterwards (cudaMalloc
// synchronizes the device and fragments the pool), or a plugin living inside a
// host framework that owns every device allocation.  For them,
// dyg_incremental_walk_noalloc runs the same walk kernel as
// dyg_incremental_batch on caller-provided device buffers and keeps its scratch
// (one 64-bit winner key per edge plus the kernel's counters) in the
// file-scope device array below.  It tests the batch against H and reports
// found_at / conductance / accepted; it does not append the accepted edges to
// H (that commit needs sort buffers sized by the batch).
//
// The array exists once per device that loads this library and stays
// allocated until the process exits.  Every call on a device shares it and
// it keeps the last call's contents, so each call clears the keys and
// counters it uses; calls whose work overlaps on the GPU (different streams,
// or different host threads) race on it and must be serialized by the
// caller.  The first call on a device looks up the array's device address
// with cudaGetSymbolAddress (set-up), and so does the first call after the
// device's context was replaced (cudaDeviceReset destroys the array with the
// context; the address is cached together with the context's unique id and
// looked up again when the id changes).  Make those calls before any stream
// capture.
#include <cuda.h>

#include <mutex>

#include "dyg_internal.cuh"

namespace dyg {

constexpr uint32_t kNoallocMaxEdges = DYG_NOALLOC_MAX_EDGES;
constexpr uint32_t kNoallocScalars = 16;

// keys[0 .. kNoallocMaxEdges), then the walk kernel's counters.
static __device__ __align__(256) unsigned long long
    g_noalloc_scratch[kNoallocMaxEdges + kNoallocScalars];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
unsigned long long *g_scratch_addr[kMaxDevices] = {nullptr};
unsigned long long g_scratch_ctx[kMaxDevices] = {0};

// Unique id of the context current on this thread (cuCtxGetId, reached through
// the runtime's driver entry points, so no libcuda link is needed); 0 when the
// driver does not provide it.
unsigned long long current_context_id() {
    typedef CUresult (*GetCurrent)(CUcontext *);
    typedef CUresult (*GetId)(CUcontext, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
        cudaGetLastError();
    });
    if (!get_current || !get_id) return 0ull;
    CUcontext c = nullptr;
    unsigned long long id = 0ull;
    if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0ull;
    return id;
}

// Device address of g_noalloc_scratch on `dev` (which must be current).  In
// host code the symbol's name is only a host-side stand-in, so the address is
// looked up once per device and context.
dyg_status scratch_on(int dev, unsigned long long **out) {
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("device ordinal out of range for the no-allocation path");
        return DYG_EINVAL;
    }
    std::lock_guard<std::mutex> lk(g_setup_mu);
    const unsigned long long ctx = current_context_id();
    if (!g_scratch_addr[dev] || (ctx && ctx != g_scratch_ctx[dev])) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            cudaGetLastError();
            set_error(std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                      cudaGetErrorString(e));
            return DYG_ECUDA;
        }
        g_scratch_addr[dev] = static_cast<unsigned long long *>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_addr[dev];
    return DYG_OK;
}

// found_at = winner's step or -1; -2 marks an edge whose endpoint is not a
// vertex of H (its walkers did not run).
__global__ void k_noalloc_decode(const unsigned long long *keys, const uint32_t *src,
                                 const uint32_t *dst, uint32_t n, uint32_t nv, int32_t *found,
                                 float *cond, uint8_t *acc) {
    const uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    if (src[e] >= nv || dst[e] >= nv) {
        if (found) found[e] = -2;
        if (cond) cond[e] = 0.f;
        if (acc) acc[e] = 0;
        return;
    }
    const unsigned long long k = keys[e];
    if (found) found[e] = key_found(k);
    if (cond) cond[e] = k ? __uint_as_float((uint32_t)(k >> 32)) : 0.f;
    if (acc) acc[e] = k ? 0 : 1;
}

}  // namespace
}  // namespace dyg

extern "C" dyg_status dyg_incremental_walk_noalloc(const dyg_graph *H, const uint32_t *src,
                                                   const uint32_t *dst, const float *w,
                                                   uint32_t n, uint64_t first_update_id,
                                                   const dyg_walk_params *p, int32_t *found_at,
                                                   float *conductance, uint8_t *accepted,
                                                   dyg_stream_t stream) {
    using namespace dyg;
    set_error("");
    if (!H || !p || (n && (!src || !dst || !w))) {
        set_error("NULL argument");
        return DYG_EINVAL;
    }
    if (n > kNoallocMaxEdges) {
        set_error("dyg_incremental_walk_noalloc: batch of " + std::to_string(n) +
                  " edges exceeds the maximum of " + std::to_string(kNoallocMaxEdges));
        return DYG_EINVAL;
    }
    if (p->walkers == 0 || p->walkers % 32 != 0 || p->walkers > 1024 || p->max_steps < 1 ||
        p->max_steps > 0x3FFFFF || p->transition > DYG_TRANSITION_WEIGHTED) {
        set_error("invalid walk parameters (walkers: multiple of 32 up to 1024; max_steps >= 1)");
        return DYG_EINVAL;
    }
    if (n == 0) return DYG_OK;
    int prev = -1;
    if (cudaGetDevice(&prev) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaGetDevice failed");
        return DYG_ECUDA;
    }
    const bool switch_dev = prev != H->device;
    if (switch_dev && cudaSetDevice(H->device) != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaSetDevice failed");
        return DYG_ECUDA;
    }
    dyg_status rc = DYG_OK;
    const void *ptrs[] = {src, dst, w, found_at, conductance, accepted};
    for (const void *q : ptrs) {
        if (!q || rc != DYG_OK) continue;
        const PtrPlace at = ptr_place(q, H->device);
        if (at == kOnOtherDevice) {
            set_error("dyg_incremental_walk_noalloc: a pointer is device memory of another GPU "
                      "than the graph's");
            rc = DYG_EINVAL;
        } else if (at != kOnDevice) {
            set_error("dyg_incremental_walk_noalloc takes device pointers only");
            rc = DYG_EINVAL;
        }
    }
    unsigned long long *scratch = nullptr;
    if (rc == DYG_OK) rc = scratch_on(H->device, &scratch);
    cudaStream_t st = (cudaStream_t)stream;
    if (rc == DYG_OK) {
        unsigned long long *keys = scratch;
        unsigned long long *scalars = scratch + kNoallocMaxEdges;
        cudaError_t e = cudaMemsetAsync(keys, 0, sizeof(unsigned long long) * n, st);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(scalars, 0, sizeof(unsigned long long) * kNoallocScalars, st);
        if (e != cudaSuccess) rc = cuda_fail(e, "cudaMemsetAsync", __FILE__, __LINE__);
        if (rc == DYG_OK) {
            WalkJob job{nullptr, src, dst, w, nullptr, (unsigned long long)first_update_id, nullptr, n,
                        kDomainIncr};
            rc = launch_walk_scalars(H->g, job, *p, true, keys, scalars, st);
        }
        if (rc == DYG_OK) {
            k_noalloc_decode<<<(n + 255) / 256, 256, 0, st>>>(keys, src, dst, n, H->g.n, found_at,
                                                              conductance, accepted);
            count_launch();
            const cudaError_t le = cudaGetLastError();
            if (le != cudaSuccess) rc = cuda_fail(le, "k_noalloc_decode", __FILE__, __LINE__);
        }
    }
    if (switch_dev) cudaSetDevice(prev);
    return rc;
}
