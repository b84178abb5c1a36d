// noalloc.cu -- a CIC density entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc or cudaFree during a
// run.  One kind manages all device memory itself: fs2's own core reserves
// its working memory up front through its Mem arena, and a framework's
// caching allocator may own the whole device.  The other kind calls from
// inside a tight time loop, where cudaFree's implicit device-wide
// synchronisation is not acceptable.  fs2g_cic_density_noalloc serves them:
// the deterministic CIC density, the same kernels as
// fs2g_pm_compute_density in FS2G_DEPOSIT_DETERMINISTIC mode, with every
// scratch buffer (sort keys and values, cell runs, per-cell sums, CUB's
// temporary storage, the error word) placed in one file-scope __device__
// array of fixed size.
//
// That array is part of the module: every GPU that loads the library holds
// it (FS2G_NOALLOC_SCRATCH_BYTES, about 19 MiB) until the process exits.
// In host code its name is only a host-side stand-in; the device address
// comes from cudaGetSymbolAddress, taken once per device on that device's
// first call (with the device current) and cached.
#include <mutex>
#include "internal.h"

namespace fs2g {
namespace {

constexpr size_t kMaxNp = FS2G_NOALLOC_MAX_PARTICLES;
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t b) { return (b + kAlign - 1)/kAlign*kAlign; }

// layout of the scratch array (byte offsets, each 256-aligned)
constexpr size_t kKeys = 0;
constexpr size_t kKeysAlt = kKeys + align_up(4*kMaxNp);
constexpr size_t kIdx = kKeysAlt + align_up(4*kMaxNp);
constexpr size_t kIdxAlt = kIdx + align_up(4*kMaxNp);
constexpr size_t kUkeys = kIdxAlt + align_up(4*kMaxNp);
constexpr size_t kStarts = kUkeys + align_up(4*kMaxNp);
constexpr size_t kNruns = kStarts + align_up(4*(kMaxNp + 2));
constexpr size_t kErr = kNruns + kAlign;
constexpr size_t kSums = kErr + kAlign;
constexpr size_t kTemp = kSums + align_up(32*kMaxNp);
constexpr size_t kTempBytes = size_t(4) << 20;     // CUB temporary storage
constexpr size_t kTotal = kTemp + kTempBytes;
static_assert(kTotal == FS2G_NOALLOC_SCRATCH_BYTES,
              "FS2G_NOALLOC_SCRATCH_BYTES in fs2gpu.h must match the layout");

// the scratch: one copy per device, for the life of the process
static __device__ __align__(256) unsigned char g_noalloc_scratch[kTotal];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char* g_addr[kMaxDevices] = {nullptr};

// device address of the scratch on the current device (set-up on first use)
unsigned char* scratch_address(int device) {
  std::lock_guard<std::mutex> lock(g_mutex);
  if(g_addr[device]) return g_addr[device];
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if(e != cudaSuccess) {
    (void) cudaGetLastError();
    throw Error{FS2G_ERR_CUDA, std::string("cudaGetSymbolAddress of the "
                "no-alloc scratch failed: ") + cudaGetErrorString(e)};
  }
  g_addr[device] = (unsigned char*) ptr;
  return g_addr[device];
}

}  // namespace
}  // namespace fs2g

using namespace fs2g;

extern "C" int fs2g_cic_density_noalloc(const float* x0, const float* x1,
                                        const float* x2, size_t np,
                                        float* mesh, int n, double boxsize,
                                        double pm_factor, void* cuda_stream) {
  if(np > kMaxNp)
    return fail(FS2G_ERR_VALUE, "fs2g_cic_density_noalloc: np = " +
                std::to_string(np) + " exceeds its fixed scratch, which holds "
                "at most FS2G_NOALLOC_MAX_PARTICLES = " +
                std::to_string(kMaxNp) + " particles");
  if(n < 2 || (unsigned long long) n*n*n >= 0xffffffffull)
    return fail(FS2G_ERR_VALUE, "fs2g_cic_density_noalloc: n must be >= 2 "
                "with n^3 < 2^32");
  if(!mesh || (np > 0 && (!x0 || !x1 || !x2)))
    return fail(FS2G_ERR_VALUE, "fs2g_cic_density_noalloc: null pointer");
  if(!(boxsize > 0))
    return fail(FS2G_ERR_VALUE, "fs2g_cic_density_noalloc: boxsize must be "
                "positive");
  try {
    int dev = 0;
    FS2G_CUDA(cudaGetDevice(&dev));
    if(dev < 0 || dev >= kMaxDevices)
      throw Error{FS2G_ERR_VALUE, "device index beyond the no-alloc table"};
    unsigned char* base = scratch_address(dev);
    if(density_deterministic_temp_bytes(kMaxNp, n) > kTempBytes)
      throw Error{FS2G_ERR_VALUE, "CUB temporary storage for this size "
                  "exceeds the no-alloc scratch"};
    DetScratch sc;
    sc.keys = (uint32_t*)(base + kKeys);
    sc.keys_alt = (uint32_t*)(base + kKeysAlt);
    sc.idx = (uint32_t*)(base + kIdx);
    sc.idx_alt = (uint32_t*)(base + kIdxAlt);
    sc.ukeys = (uint32_t*)(base + kUkeys);
    sc.starts = (uint32_t*)(base + kStarts);
    sc.nruns = (uint32_t*)(base + kNruns);
    sc.err = (int*)(base + kErr);
    sc.sums = (float*)(base + kSums);
    sc.temp = base + kTemp;
    sc.temp_bytes = kTempBytes;
    cudaStream_t s = (cudaStream_t) cuda_stream;
    // the array keeps the previous call's contents: zero what must start at 0
    FS2G_CUDA(cudaMemsetAsync(sc.err, 0, 2*sizeof(int), s));
    FS2G_CUDA(cudaMemsetAsync(sc.starts, 0, 4*(np + 2), s));
    const float dx_inv = (float) n / (float) boxsize;            // py/pm.cpp:77
    const float fac = (float)(pm_factor*pm_factor*pm_factor);    // py/pm.cpp:78
    FS2G_CUDA(density_deterministic_on(s, x0, x1, x2, np, mesh, n, dx_inv,
                                       fac, sc));
    FS2G_CUDA(cudaStreamSynchronize(s));
    int err[2] = {0, 0};
    FS2G_CUDA(cudaMemcpy(err, sc.err, sizeof(err), cudaMemcpyDeviceToHost));
    if(err[0] == DEV_POSITION_OUT_OF_RANGE)
      throw Error{FS2G_ERR_DEVICE, "particle " + std::to_string(err[1]) +
                  " lies below -1 cell: wrap positions into the box first"};
    return FS2G_OK;
  }
  catch(const Error& e) { return fail(e.code, e.msg); }
  catch(const std::exception& e) { return fail(FS2G_ERR_RUNTIME, e.what()); }
}
