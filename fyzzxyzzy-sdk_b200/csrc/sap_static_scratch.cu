// Sweep-and-prune overlap pairs of one scene's finite shapes, computed
// without allocating memory.
//
// The world's broadphase (broadphase.cu) keeps its sort keys, sweep records
// and per-owner pair buckets in buffers the world allocates when a scene is
// uploaded or when the pair budget grows.  Some callers cannot allocate at
// the point where they need a pair set: a frame loop that shares the GPU with
// other work and must not take the device-wide synchronisation that
// cudaMalloc / cudaFree imply, or a process that runs under a fixed device
// memory budget reserved up front.  This entry point serves them: the same
// sort + sweep + canonical owner-bucket emission as the world's broadphase,
// in one CTA, with its working set in a fixed file-scope device array
// instead of allocated buffers.
//
// Pair semantics follow the reference's full sweep (src/native/scene.cpp,
// Scene::update_pairs 2635-2704): two finite shapes pair when their encoded
// bounds overlap on all three axes, they belong to different bodies and at
// least one body is dynamic.  Output is (a, b) with a < b, ascending.
//
// Limits and sharing:
//  * at most kStaticSapMaxShapes shapes per call (larger inputs are rejected
//    before anything is launched);
//  * every call on a device uses the same scratch array, so calls whose
//    kernels may overlap in time (different streams, different host threads
//    without ordering) race and corrupt each other's results; order them on
//    one stream;
//  * the first call on a device resolves the scratch array's address with
//    cudaGetSymbolAddress (which loads this module on that device) and
//    raises the kernel's dynamic shared-memory limit; make that first call
//    before any stream capture on the device.  The resolved address is kept
//    per CUDA context, so a context made after cudaDeviceReset resolves it
//    again on its first call;
//  * when the pair total exceeds the caller's capacity, only whole owner
//    buckets that end within the capacity are written: the list is then a
//    prefix of the full canonical list (deterministic), and the total tells
//    the caller how much room a complete list needs.
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>
#include <initializer_list>
#include <mutex>
#include "fyzz_b200.h"

namespace fyzz::b200 {
namespace {

constexpr uint32_t kStaticSapMaxShapes = FYZZ_B200_STATIC_SAP_MAX_SHAPES;
static_assert(kStaticSapMaxShapes == 8192u, "the rejection message states the limit");
constexpr int kThreads = 1024;
// Sorted (min x << 32 | shape) keys live in shared memory: 8 bytes a shape.
constexpr size_t kMaxSortSmem = size_t(kStaticSapMaxShapes) * sizeof(unsigned long long);
static_assert(kMaxSortSmem <= 227u * 1024u, "sort keys must fit one CTA's shared memory");

// Scratch layout, 32 bytes a shape (256 KiB at the maximum):
//   rec  uint4  sorted-order (min y, max y, min z, max z)
//   meta uint2  sorted-order (max x, body | dynamic << 31)
//   cnt  u32    pairs owned by each shape      -- must start at zero; the
//                                                 kernel clears it first
//   off  u32    bucket offsets (written by the kernel's scan before use)
constexpr size_t kRecOff = 0;
constexpr size_t kMetaOff = kRecOff + size_t(kStaticSapMaxShapes) * 16;
constexpr size_t kCntOff = kMetaOff + size_t(kStaticSapMaxShapes) * 8;
constexpr size_t kOffOff = kCntOff + size_t(kStaticSapMaxShapes) * 4;
constexpr size_t kScratchBytes = kOffOff + size_t(kStaticSapMaxShapes) * 4;

static __device__ __align__(256) unsigned char g_sap_scratch[kScratchBytes];

// Block-wide exclusive scan of cnt[0, n) into off[0, n); returns the total.
__device__ uint32_t block_scan(const uint32_t* cnt, uint32_t* off, uint32_t n) {
    __shared__ uint32_t warp_sum[kThreads / 32];
    __shared__ uint32_t total;
    const uint32_t chunk = (n + kThreads - 1) / kThreads;
    const uint32_t b = threadIdx.x * chunk;
    const uint32_t e = b + chunk < n ? b + chunk : n;
    uint32_t local = 0;
    for (uint32_t i = b; i < e; ++i) local += __ldcg(cnt + i);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t incl = local;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= uint32_t(d)) incl += v;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = warp_sum[lane];
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t v = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= uint32_t(d)) w += v;
        }
        warp_sum[lane] = w;                  // inclusive over warps
        if (lane == 31) total = w;
    }
    __syncthreads();
    uint32_t run = (warp ? warp_sum[warp - 1] : 0u) + incl - local;
    for (uint32_t i = b; i < e; ++i) {
        off[i] = run;
        run += __ldcg(cnt + i);
    }
    __syncthreads();
    return total;
}

// One CTA: sort min-x endpoints, gather the sweep records, count pairs per
// owner (the lower shape id), scan, fill the owner buckets, sort each bucket
// by partner.  bounds: n x 6 encoded values (min x, y, z, max x, y, z), the
// layout fyzz_b200_read_encoded_bounds produces.
__global__ void __launch_bounds__(kThreads) k_sap_static(const uint32_t* __restrict__ bounds,
                                                         const uint32_t* __restrict__ body,
                                                         uint32_t n, uint32_t* __restrict__ pairs,
                                                         uint32_t cap, uint32_t* __restrict__ count,
                                                         unsigned char* scratch) {
    extern __shared__ unsigned long long sk[];
    __shared__ uint32_t s_total;
    uint4* rec = reinterpret_cast<uint4*>(scratch + kRecOff);
    uint2* meta = reinterpret_cast<uint2*>(scratch + kMetaOff);
    uint32_t* cnt = reinterpret_cast<uint32_t*>(scratch + kCntOff);
    uint32_t* off = reinterpret_cast<uint32_t*>(scratch + kOffOff);
    uint32_t m = 1;
    while (m < n) m <<= 1;
    for (uint32_t i = threadIdx.x; i < n; i += kThreads) cnt[i] = 0u;
    for (uint32_t i = threadIdx.x; i < m; i += kThreads)
        sk[i] = i < n ? (static_cast<unsigned long long>(bounds[6 * size_t(i)]) << 32) | i : ~0ull;
    __syncthreads();
    // bitonic sort by (min x, shape id), the reference's endpoint order
    for (uint32_t k = 2; k <= m; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = threadIdx.x; i < m; i += kThreads) {
                const uint32_t ixj = i ^ j;
                if (ixj > i) {
                    const unsigned long long a = sk[i], c = sk[ixj];
                    const bool up = (i & k) == 0;
                    if ((a > c) == up) { sk[i] = c; sk[ixj] = a; }
                }
            }
            __syncthreads();
        }
    for (uint32_t i = threadIdx.x; i < n; i += kThreads) {
        const uint32_t id = uint32_t(sk[i]);
        const uint32_t* bd = bounds + 6 * size_t(id);
        rec[i] = make_uint4(bd[1], bd[4], bd[2], bd[5]);
        meta[i] = make_uint2(bd[3], body[id]);
    }
    __syncthreads();
    for (int fill = 0; fill < 2; ++fill) {
        for (uint32_t i = threadIdx.x; i < n; i += kThreads) {
            const uint32_t id = uint32_t(sk[i]);
            const uint4 a = rec[i];
            const uint2 am = meta[i];
            const uint32_t abody = am.y & 0x7fffffffu;
            const bool adyn = (am.y >> 31) != 0u;
            for (uint32_t j = i + 1; j < n; ++j) {
                const unsigned long long kj = sk[j];
                if (uint32_t(kj >> 32) > am.x) break;
                const uint2 bm = meta[j];
                if ((bm.y & 0x7fffffffu) == abody) continue;
                if (!adyn && (bm.y >> 31) == 0u) continue;
                const uint4 c = rec[j];
                if (a.x > c.y || c.x > a.y || a.z > c.w || c.z > a.w) continue;
                const uint32_t other = uint32_t(kj);
                const uint32_t owner = id < other ? id : other;
                const uint32_t partner = id < other ? other : id;
                if (!fill) {
                    atomicAdd(cnt + owner, 1u);
                } else {
                    // bucket [off[owner], off[owner + 1]): written only when
                    // all of it fits, so a truncated list is a canonical prefix
                    const uint32_t end = owner + 1 < n ? __ldcg(off + owner + 1) : s_total;
                    if (end <= cap) {
                        const uint32_t pos = __ldcg(off + owner) + atomicSub(cnt + owner, 1u) - 1u;
                        pairs[2 * size_t(pos)] = owner;
                        pairs[2 * size_t(pos) + 1] = partner;
                    }
                }
            }
        }
        __syncthreads();
        if (!fill) {
            const uint32_t total = block_scan(cnt, off, n);
            if (threadIdx.x == 0) {
                *count = total;
                s_total = total;
            }
            __syncthreads();
        }
    }
    // each written owner bucket [off[o], off[o + 1]) sorted by partner
    // (insertion sort; buckets are short)
    for (uint32_t o = threadIdx.x; o < n; o += kThreads) {
        const uint32_t begin = __ldcg(off + o);
        const uint32_t end = o + 1 < n ? __ldcg(off + o + 1) : s_total;
        const uint32_t c = end - begin;
        if (c < 2 || end > cap) continue;
        uint32_t* p = pairs + 2 * size_t(begin) + 1;
        for (uint32_t i = 1; i < c; ++i) {
            const uint32_t v = p[2 * size_t(i)];
            uint32_t j = i;
            while (j > 0 && p[2 * size_t(j - 1)] > v) { p[2 * size_t(j)] = p[2 * size_t(j - 1)]; --j; }
            p[2 * size_t(j)] = v;
        }
    }
}

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
unsigned char* g_scratch[kMaxDevices] = {};
void* g_scratch_ctx[kMaxDevices] = {};       // the CUDA context g_scratch[dev] was resolved in
using CtxGetCurrent = int (*)(void**);       // the driver's cuCtxGetCurrent
CtxGetCurrent g_ctx_get = nullptr;

// Copies a message into the caller's buffer (no formatting, no allocation).
void put_message(char* out, size_t len, const char* a, const char* b = "") {
    if (!out || len == 0) return;
    size_t k = 0;
    for (const char* s : {a, b})
        for (; *s && k + 1 < len; ++s) out[k++] = *s;
    out[k] = '\0';
}

// Once per device (per CUDA context of the device: a context made after
// cudaDeviceReset loads this module again), with that device current:
// resolve the scratch array's address and allow the kernel the shared
// memory its largest sort needs.
int setup_device(int dev, unsigned char** out, char* msg, size_t msg_len) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_ctx_get) {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        const cudaError_t e = cudaGetDriverEntryPoint("cuCtxGetCurrent", &fn, cudaEnableDefault, &q);
        if (e != cudaSuccess || q != cudaDriverEntryPointSuccess || !fn) {
            put_message(msg, msg_len, "cuCtxGetCurrent unavailable: ", cudaGetErrorString(e));
            return FYZZ_B200_RUNTIME_ERROR;
        }
        g_ctx_get = reinterpret_cast<CtxGetCurrent>(fn);
    }
    void* ctx = nullptr;
    if (g_ctx_get(&ctx) != 0 || !ctx) {
        put_message(msg, msg_len, "no current CUDA context");
        return FYZZ_B200_RUNTIME_ERROR;
    }
    if (!g_scratch[dev] || g_scratch_ctx[dev] != ctx) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_sap_scratch);
        if (e != cudaSuccess || !p) {
            put_message(msg, msg_len, "cudaGetSymbolAddress failed: ", cudaGetErrorString(e));
            return FYZZ_B200_RUNTIME_ERROR;
        }
        e = cudaFuncSetAttribute(k_sap_static, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(kMaxSortSmem));
        if (e != cudaSuccess) {
            put_message(msg, msg_len, "cudaFuncSetAttribute failed: ", cudaGetErrorString(e));
            return FYZZ_B200_RUNTIME_ERROR;
        }
        g_scratch[dev] = static_cast<unsigned char*>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch[dev];
    return FYZZ_B200_OK;
}

}  // namespace
}  // namespace fyzz::b200

extern "C" int fyzz_b200_sap_pairs_static_scratch(const uint32_t* bounds_dev, const uint32_t* body_dev,
                                                  uint32_t n_shapes, uint32_t* pairs_dev,
                                                  uint32_t pair_cap, uint32_t* count_dev, void* stream,
                                                  char* message, size_t message_len) {
    using namespace fyzz::b200;
    put_message(message, message_len, "");
    if (n_shapes > kStaticSapMaxShapes) {
        put_message(message, message_len,
                    "n_shapes exceeds FYZZ_B200_STATIC_SAP_MAX_SHAPES (the fixed scratch array "
                    "holds 8192 shapes); split the scene or use the world's broadphase");
        return FYZZ_B200_INVALID_ARGUMENT;
    }
    if (!count_dev || (n_shapes && (!bounds_dev || !body_dev)) || (pair_cap && !pairs_dev)) {
        put_message(message, message_len, "null device pointer");
        return FYZZ_B200_INVALID_ARGUMENT;
    }
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        put_message(message, message_len, "no usable current CUDA device: ", cudaGetErrorString(e));
        return FYZZ_B200_RUNTIME_ERROR;
    }
    unsigned char* scratch = nullptr;
    if (const int rc = setup_device(dev, &scratch, message, message_len)) return rc;
    uint32_t m = 1;
    while (m < n_shapes) m <<= 1;
    k_sap_static<<<1, kThreads, size_t(m) * sizeof(unsigned long long),
                   static_cast<cudaStream_t>(stream)>>>(bounds_dev, body_dev, n_shapes, pairs_dev,
                                                        pair_cap, count_dev, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        put_message(message, message_len, "launch failed: ", cudaGetErrorString(e));
        return FYZZ_B200_RUNTIME_ERROR;
    }
    return FYZZ_B200_OK;
}
