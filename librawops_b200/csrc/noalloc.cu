// Reduced-level (mip 1/2) RAW render that allocates nothing.
//
// re_render_raw needs device scratch for the native-resolution footprint of a
// reduced request and allocates it per call from the stream-ordered pool.
// Some callers cannot allocate device memory at render time -- a plug-in
// running inside a host application's render callback whose device memory is
// budgeted up front, a real-time preview thread that must not take the
// allocator's locks or risk an out-of-memory in mid-frame.  This variant keeps
// its scratch in a fixed file-scope device array instead, so a call makes no
// cudaMalloc/cudaFree and uses no allocating library routine.
//
// The array holds kNoAllocMaxNativePixels native float32 RGB pixels (12 MiB)
// plus one status word, on every GPU that loads the library, until the process
// exits.  All calls share it and it keeps the last call's contents: the status
// word is cleared at the start of every call, and calls that overlap on the GPU
// (concurrent streams, or threads without ordering) race on it.  The first call
// on a device looks up the array's device address (cudaGetSymbolAddress) with
// that device current; make that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "re_device.cuh"

namespace re {
cudaError_t launch_demosaic(uint32_t demosaic, const DevRaw& raw, int ox, int oy, int ow, int oh,
                            int stage_end, const DevProgram& P, float* out, size_t out_stride,
                            uint32_t* status, unsigned long long* ties, cudaStream_t stream,
                            uint32_t* launches, uint8_t* dirs = nullptr);
cudaError_t launch_mip_reduce(const float* native, int nw, int nh, size_t native_stride, int mip,
                              int ow, int oh, int stage_begin, int stage_end, const DevProgram& P,
                              float* out, size_t out_stride, uint32_t* status, cudaStream_t stream,
                              uint32_t* launches);
void set_last_error(const std::string& msg);
re_status render_plan(const re_image* img, const re_render_desc* desc, re_rect viewport, uint32_t mip,
                      uint32_t quality, DevProgram& P, re_rect& native, const DevRaw** raw);
re_status status_key_to_error(uint32_t key);
}  // namespace re

using namespace re;

namespace {

constexpr size_t kNoAllocMaxNativePixels = size_t(1) << 20;   // 1,048,576 native pixels
constexpr size_t kScratchFloats = kNoAllocMaxNativePixels * 3 + 64;

// Static scratch: [0, 64) floats hold the status word, the rest the native footprint.
static __device__ __align__(256) float g_noalloc_scratch[kScratchFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
float* g_scratch_ptr[kMaxDevices] = {};

re_status scratch_for_current_device(float** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(e));
        return RE_CUDA_ERROR;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        set_last_error("device ordinal beyond the no-allocation scratch table");
        return RE_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            set_last_error(std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            return RE_CUDA_ERROR;
        }
        g_scratch_ptr[dev] = static_cast<float*>(p);
    }
    *out = g_scratch_ptr[dev];
    return RE_OK;
}

}  // namespace

extern "C" {

size_t re_render_raw_reduced_noalloc_max_native_pixels(void) { return kNoAllocMaxNativePixels; }

re_status re_render_raw_reduced_noalloc(const re_image* image, const re_render_desc* desc, re_rect viewport,
                                        uint32_t mip, float* out, size_t out_row_stride, void* stream_) {
    // Same argument rules as re_render_raw: a null output is accepted for an
    // empty viewport, which renders nothing.
    if (!image || !desc || (!out && viewport.width && viewport.height)) {
        set_last_error("null render arguments");
        return RE_INVALID_ARGUMENT;
    }
    if (mip < 1 || mip > 2) {
        set_last_error("the no-allocation render covers reduced levels (mip 1 or 2, Preview) only");
        return RE_INVALID_ARGUMENT;
    }
    DevProgram P;
    re_rect native;
    const DevRaw* raw = nullptr;
    re_status s = render_plan(image, desc, viewport, mip, 0, P, native, &raw);
    if (s) return s;
    if (out_row_stride < (size_t)viewport.width * 3) {
        set_last_error("output row stride too small");
        return RE_INVALID_ARGUMENT;
    }
    if (!viewport.width || !viewport.height) return RE_OK;
    if ((size_t)native.width * native.height > kNoAllocMaxNativePixels) {
        set_last_error("native footprint of " + std::to_string((size_t)native.width * native.height) +
                       " pixels exceeds the no-allocation limit of " + std::to_string(kNoAllocMaxNativePixels) +
                       " pixels");
        return RE_LENGTH_ERROR;
    }
    float* scratch = nullptr;
    s = scratch_for_current_device(&scratch);
    if (s) return s;
    cudaStream_t stream = (cudaStream_t)stream_;
    uint32_t* status = reinterpret_cast<uint32_t*>(scratch);
    float* nat = scratch + 64;
    const size_t nstride = (size_t)native.width * 3;
    cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), stream);
    if (e == cudaSuccess)
        e = launch_demosaic(desc->demosaic, *raw, (int)native.x, (int)native.y, (int)native.width,
                            (int)native.height, P.anchor + 1, P, nat, nstride, status, nullptr, stream, nullptr);
    if (e == cudaSuccess)
        e = launch_mip_reduce(nat, (int)native.width, (int)native.height, nstride, (int)mip, (int)viewport.width,
                              (int)viewport.height, P.anchor + 1, (int)P.count, P, out, out_row_stride, status,
                              stream, nullptr);
    uint32_t key = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(&key, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) {
        set_last_error(std::string("no-allocation render: ") + cudaGetErrorString(e));
        return RE_CUDA_ERROR;
    }
    return status_key_to_error(key);
}

}  // extern "C"
