// chx_noalloc.cu -- the full path sum for callers that cannot allocate.
//
// chx_chi_full needs scratch memory (the staged pair records and the
// per-CTA partial spectra) that its caller allocates. Some callers cannot
// allocate device memory: a host that embeds this library through a foreign
// function interface and has no device allocator of its own, or code that
// runs where allocating is not allowed (inside a host callback, or next to a
// component that owns the device allocator and its memory budget). For them
// chx_chi_full_noalloc runs the same computation with its scratch in
// g_noalloc_scratch below: a fixed array in device memory that the library
// reserves on every GPU that loads it, for as long as the process lives.
//
// Host code cannot use the array's name as a device address (on the host it
// names a host-side stand-in), so the first call on each device asks the
// runtime for the array's device address (cudaGetSymbolAddress, with that
// device current) and keeps it; later calls on that device reuse it, so calls
// must not span a reset of the device (the module may load elsewhere). Because
// that first call may load the module, it should come before any stream
// capture. All calls on a device share the one array and it keeps the last
// call's contents: the error word that must start at zero is cleared by each
// call, and calls that overlap on the GPU (different streams, or different
// host threads) race on the array and must be serialised by the caller. The
// error word sits in the array, where the caller cannot read it, so a device
// error reaches the caller as NaN in every chi value of the call (the final
// reduction of chx_chi_full checks the word).
#include <mutex>
#include "chx_common.cuh"

namespace chx {

// The fixed scratch: 32 MiB, 256-byte aligned.
constexpr size_t kNoallocScratchBytes = (size_t)32 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[kMaxDevices];

// Device address of g_noalloc_scratch on the current device (set up once).
static int noalloc_scratch(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "chi_full_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("chi_full_noalloc: device ordinal %d beyond %d", dev, kMaxDevices);
        return CHX_ERR_UNSUPPORTED;
    }
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "chi_full_noalloc: cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return CHX_OK;
}

}  // namespace chx

using namespace chx;

extern "C" {

int64_t chx_chi_full_noalloc_max_bytes(void) { return (int64_t)kNoallocScratchBytes; }

int chx_chi_full_noalloc(const chx_pairs_t *P, const double *pos, const int *species, int nconf,
                         int precision, double *chi, void *stream) {
    CHX_REQUIRE(P && pos && species && chi && nconf > 0, "chi_full_noalloc: bad arguments");
    int64_t need = chx_chi_full_scratch_bytes(P, nconf);
    if (need < 0) {
        set_error("chi_full_noalloc: bad pair set");
        return CHX_ERR_ARG;
    }
    if (need > (int64_t)kNoallocScratchBytes) {
        set_error("chi_full_noalloc: %lld bytes of scratch needed for %d configurations of %d "
                  "pairs, the fixed array holds %lld; use chx_chi_full with a caller buffer or "
                  "fewer configurations per call",
                  (long long)need, nconf, P->npairs, (long long)kNoallocScratchBytes);
        return CHX_ERR_SCRATCH;
    }
    void *scratch = nullptr;
    int rc = noalloc_scratch(&scratch);
    if (rc != CHX_OK) return rc;
    return chx_chi_full(P, pos, species, nconf, precision, chi, scratch,
                        (int64_t)kNoallocScratchBytes, stream);
}

}  // extern "C"
