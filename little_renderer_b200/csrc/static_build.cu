// static_build.cu - lrc_build_static: the BVH builder for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: a host program that hands out all of its device memory up
// front from its own pool (a game engine's or a framework's allocator) cannot have a library
// allocate behind its back, since the allocation can fail against that budget; and in a frame
// loop that rebuilds a top-level tree every frame, cudaMalloc's implicit device synchronisation
// would stall the frame. For them this entry point runs the same builder as lrc_build with its
// scratch memory in one fixed device array of this file, which every GPU that loads the library
// holds until the process exits. The caller passes inputs and outputs as device pointers.
#include "lrc_internal.cuh"

namespace {

// the builder's scratch for up to LRC_STATIC_MAX_ITEMS items (the largest need, 63-bit keys with
// PLOC, is about 5.9 MB), then the status word
constexpr size_t STATIC_SCRATCH_BYTES = LRC_STATIC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_static_scratch[STATIC_SCRATCH_BYTES + 256];

// per device: the array's device address (cudaGetSymbolAddress, with that device current) and the
// SM count; filled by the first call on the device
constexpr int MAX_DEVICES = 64;
void *g_scratch_addr[MAX_DEVICES];
int g_num_sms[MAX_DEVICES];

}  // namespace

extern "C" int lrc_build_static(const lrc_build_params *p, const float *boxes, uint32_t *nodes, uint32_t *aux,
                                void *cuda_stream) {
    if (!p || (p->key_bits != 30 && p->key_bits != 63)) return LRC_E_INVALID;
    if (p->n > LRC_STATIC_MAX_ITEMS) return LRC_E_TOO_BIG;
    if (p->n == 0) return LRC_OK;
    if (!boxes || !nodes || !aux) return LRC_E_INVALID;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return LRC_E_NODEVICE;
    }
    if (dev < 0 || dev >= MAX_DEVICES) return LRC_E_INVALID;
    if (!g_scratch_addr[dev]) {
        // set-up, once per device: host code only knows the array's host-side stand-in; its
        // device address comes from the runtime
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_static_scratch);
        if (e != cudaSuccess || !ptr) {
            cudaGetLastError();
            return LRC_E_CUDA;
        }
        int sms = 0;
        e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e != cudaSuccess || sms <= 0) {
            cudaGetLastError();
            return LRC_E_CUDA;
        }
        g_num_sms[dev] = sms;
        g_scratch_addr[dev] = ptr;
    }
    if (lrc::build_scratch_bytes(p->n, p->key_bits, p->builder) > STATIC_SCRATCH_BYTES) return LRC_E_TOO_BIG;
    char *scratch = static_cast<char *>(g_scratch_addr[dev]);
    uint32_t *status = reinterpret_cast<uint32_t *>(scratch + STATIC_SCRATCH_BYTES);
    cudaStream_t st = static_cast<cudaStream_t>(cuda_stream);
    // what must start at zero is cleared here (the status word) or by the builder itself (its
    // histograms, look-back words, counters and exchange words): the array keeps the last call's data
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess)
        e = lrc::build_device(*p, boxes, reinterpret_cast<lrc::Node *>(nodes) + p->node0, aux + p->ref0, scratch,
                              STATIC_SCRATCH_BYTES, status, g_num_sms[dev], st);
    uint32_t word = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&word, status, sizeof(word), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return LRC_E_CUDA;
    }
    return word ? LRC_E_TIMEOUT : LRC_OK;
}
