// mk_multigrid_apply_noalloc: the multigrid apply for callers that cannot allocate device
// memory (see include/markovkit_b200.h). The cycle's work vectors live in one file-scope
// device array instead of the hierarchy's own buffers.
#include "capi_internal.hpp"

#include <mutex>

namespace {

// 64 MiB per GPU that loads the library, held until the process exits
constexpr std::size_t kNoAllocScratchBytes = std::size_t(64) << 20;
__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void *g_scratch_addr[kMaxDevices] = {};

// The array's device address on the current device. In host code the symbol's name is only a
// host-side stand-in, so the address is looked up once per device, with that device current.
void *scratch_on_current_device() {
    int dev = -1;
    mkb::check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        throw mkb::Error(MK_EINVAL, "device ordinal out of range");
    }
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_addr[dev]) {
        void *ptr = nullptr;
        mkb::check_cuda(cudaGetSymbolAddress(&ptr, g_noalloc_scratch), "cudaGetSymbolAddress");
        g_scratch_addr[dev] = ptr;
    }
    return g_scratch_addr[dev];
}

} // namespace

extern "C" int mk_multigrid_apply_noalloc(mk_multigrid mg, const double *d_b, double *d_x,
                                          void *stream) {
    return mkb::capi::guarded([&] {
        MK_REQUIRE(mg && d_b && d_x, "null argument");
        const std::size_t need = mg->mg->scratch_bytes();
        if (need > kNoAllocScratchBytes) {
            throw mkb::Error(MK_EINVAL,
                             "mk_multigrid_apply_noalloc: this hierarchy needs " +
                                 std::to_string(need) +
                                 " bytes of work vectors; the static scratch holds 64 MiB");
        }
        void *scratch = scratch_on_current_device();
        mg->mg->apply_in(d_b, d_x, scratch, kNoAllocScratchBytes, mkb::capi::as_stream(stream));
    });
}
