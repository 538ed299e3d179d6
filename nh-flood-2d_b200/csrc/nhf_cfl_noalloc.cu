// nhf_cfl_noalloc: the CFL candidate of the current state without any device
// allocation, for callers that cannot allocate GPU memory.
//
// Some hosts reserve their whole device-memory budget once at start-up and
// forbid allocation afterwards (for example a serving process that admits
// flood solves against a fixed HBM budget, or a model coupler that hands out
// pre-sized pools to its components). nhf_create allocates per-handle
// scratch, so such a caller could not even ask "what time step would this
// state allow?". This entry point answers it using only caller-owned inputs
// and outputs plus one fixed scratch array compiled into the library.
//
// The scratch is the file-scope array below: 32,769 64-bit words (256 KiB +
// 8 bytes) per device, held by every GPU that loads the library until the
// process exits. Words [0, 32768) hold one packed per-block minimum each and
// the last word is the completion ticket. One block covers 2,048 sides, so
// the entry point accepts at most 32,768 * 2,048 = 67,108,864 sides and
// rejects larger meshes with NHF_EINVAL.
//
// Host code must not take the array's name as a device address (in host code
// it names a host-side stand-in). On the first call on each device, with that
// device current, the entry point looks up the device address with
// cudaGetSymbolAddress and caches it; that first call should therefore come
// before any stream capture. Every later call checks that the cached address
// is still device memory of the current context (cudaPointerGetAttributes) and
// looks it up again if not, so a context torn down by cudaDeviceReset does not
// leave a stale address behind. All calls share the array and it keeps the
// last call's contents: each call clears the ticket before its kernel runs,
// and calls whose kernels overlap on the GPU race on the array, so serialise
// them (one stream, or events between streams). The inputs and outputs must
// be device (or managed) memory; a host pointer is refused with NHF_EINVAL
// before any launch. Error messages are kept per host thread.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/nhflood.h"
#include "nhf_common.cuh"

namespace {

using nhf::cfl_face_depth;
using nhf::cfl_value;

constexpr int kNoAllocSlots = 32768;
constexpr int kThreads = 256;
constexpr int kSidesPerThread = 8;
constexpr int kSidesPerBlock = kThreads * kSidesPerThread;
constexpr long long kMaxSides = (long long)kNoAllocSlots * kSidesPerBlock;
constexpr unsigned long long kEmpty = 0xFFFFFFFFFFFFFFFFULL;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned long long g_cfl_scratch[kNoAllocSlots + 1];

std::mutex g_setup_mutex;
unsigned long long *g_scratch_address[kMaxDevices] = {};
thread_local std::string g_error;  // the calling thread's last failure

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_error = buf;
    return code;
}

// Same arithmetic as compute_cfl (solver_compact.py:617-641), through the same
// helpers as the handle entry point's k_cfl: interior sides only, face depth
// floor 0.01, packed (cfl bits << 32 | side) minimum so that ties resolve to
// the lowest side id.
__global__ void __launch_bounds__(kThreads)
k_cfl_noalloc(const int32_t *topology, const float *bed, const float *depth, const float *length,
              const float *q, int32_t s_num, float afa, float g, unsigned long long *scratch,
              int32_t blocks, float *ndt_out, int32_t *arg_out)
{
    __shared__ unsigned long long sh[kThreads / 32];
    __shared__ bool last;
    unsigned long long best = kEmpty;
    const long long base = 1 + (long long)blockIdx.x * kSidesPerBlock;
    for (int k = 0; k < kSidesPerThread; ++k) {
        long long si = base + (long long)k * kThreads + threadIdx.x;
        if (si >= s_num) break;
        int el = topology[3 * si + 1], eh = topology[3 * si + 2];
        if (el == 0 || eh == 0) continue;
        float h = cfl_face_depth(bed[el], depth[el], bed[eh], depth[eh]);
        float cfl = cfl_value(afa, g, length[si], q[si], h);
        unsigned long long key = ((unsigned long long)__float_as_uint(cfl) << 32) | (unsigned long long)si;
        best = key < best ? key : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_down_sync(0xffffffffu, best, o);
        best = w < best ? w : best;
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = best;
    __syncthreads();
    if (warp == 0) {
        best = lane < kThreads / 32 ? sh[lane] : kEmpty;
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long w = __shfl_down_sync(0xffffffffu, best, o);
            best = w < best ? w : best;
        }
        if (lane == 0) {
            scratch[blockIdx.x] = best;
            __threadfence();
            unsigned long long ticket = atomicAdd(&scratch[kNoAllocSlots], 1ULL);
            last = ticket == (unsigned long long)(blocks - 1);
        }
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    // The last block reduces the per-block minima (min is order free).
    unsigned long long total = kEmpty;
    for (int b = threadIdx.x; b < blocks; b += kThreads) {
        unsigned long long v = *((volatile unsigned long long *)&scratch[b]);
        total = v < total ? v : total;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_down_sync(0xffffffffu, total, o);
        total = w < total ? w : total;
    }
    if (lane == 0) sh[warp] = total;
    __syncthreads();
    if (threadIdx.x == 0) {
        total = kEmpty;
        for (int w = 0; w < kThreads / 32; ++w) total = sh[w] < total ? sh[w] : total;
        if (total == kEmpty) {
            *ndt_out = __uint_as_float(0x7f800000u);
            *arg_out = 0;
        } else {
            *ndt_out = __uint_as_float((uint32_t)(total >> 32));
            *arg_out = (int32_t)(total & 0xffffffffu);
        }
        scratch[kNoAllocSlots] = 0ULL;
    }
}

int scratch_for_current_device(unsigned long long **out)
{
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return fail(NHF_ECUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
    if (device < 0 || device >= kMaxDevices) return fail(NHF_EINVAL, "device %d beyond %d devices", device, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_address[device]) {
        // still device memory of the current context? (not after cudaDeviceReset)
        cudaPointerAttributes attr{};
        if (cudaPointerGetAttributes(&attr, g_scratch_address[device]) != cudaSuccess ||
            attr.type != cudaMemoryTypeDevice || attr.device != device) {
            cudaGetLastError();
            g_scratch_address[device] = nullptr;
        }
    }
    if (!g_scratch_address[device]) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_cfl_scratch);
        if (e != cudaSuccess)
            return fail(NHF_ECUDA, "cudaGetSymbolAddress(g_cfl_scratch) failed: %s", cudaGetErrorString(e));
        g_scratch_address[device] = (unsigned long long *)ptr;
    }
    *out = g_scratch_address[device];
    return NHF_OK;
}

// Inputs and outputs must be memory the kernel can address: device or managed.
int check_device_pointer(const void *p, const char *name)
{
    cudaPointerAttributes attr{};
    cudaError_t e = cudaPointerGetAttributes(&attr, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(NHF_EINVAL, "nhf_cfl_noalloc: %s is not a CUDA pointer (%s)", name, cudaGetErrorString(e));
    }
    if (attr.type != cudaMemoryTypeDevice && attr.type != cudaMemoryTypeManaged)
        return fail(NHF_EINVAL, "nhf_cfl_noalloc: %s is not device memory", name);
    return NHF_OK;
}

}  // namespace

extern "C" {

const char *nhf_cfl_noalloc_error(void) { return g_error.c_str(); }

int nhf_cfl_noalloc(const int32_t *topology, const float *bed, const float *depth, const float *length,
                    const float *q, int32_t s_num, float afa, float g, void *stream, float *ndt_out,
                    int32_t *arg_out)
{
    if (!topology || !bed || !depth || !length || !q || !ndt_out || !arg_out)
        return fail(NHF_EINVAL, "nhf_cfl_noalloc: null pointer argument");
    if (s_num < 1) return fail(NHF_EINVAL, "nhf_cfl_noalloc: s_num must be at least 1 (sentinel side 0)");
    if ((long long)s_num - 1 > kMaxSides)
        return fail(NHF_EINVAL, "nhf_cfl_noalloc: %d sides exceed the %lld-side limit of its fixed scratch",
                    s_num - 1, kMaxSides);
    if (!(afa > 0.0f) || !(g > 0.0f)) return fail(NHF_EINVAL, "nhf_cfl_noalloc: afa and g must be positive");
    const void *pointers[7] = {topology, bed, depth, length, q, ndt_out, arg_out};
    const char *names[7] = {"topology", "bed", "depth", "length", "q", "ndt_out", "arg_out"};
    for (int i = 0; i < 7; ++i) {
        int rc = check_device_pointer(pointers[i], names[i]);
        if (rc) return rc;
    }
    unsigned long long *scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    int blocks = (int)(((long long)s_num - 1 + kSidesPerBlock - 1) / kSidesPerBlock);
    if (blocks < 1) blocks = 1;
    cudaError_t e = cudaMemsetAsync(scratch + kNoAllocSlots, 0, sizeof(unsigned long long), s);
    if (e != cudaSuccess) return fail(NHF_ECUDA, "clearing the ticket failed: %s", cudaGetErrorString(e));
    k_cfl_noalloc<<<blocks, kThreads, 0, s>>>(topology, bed, depth, length, q, s_num, afa, g, scratch, blocks,
                                             ndt_out, arg_out);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(NHF_ECUDA, "k_cfl_noalloc launch failed: %s", cudaGetErrorString(e));
    return NHF_OK;
}

}  // extern "C"
