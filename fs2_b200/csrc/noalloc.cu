// noalloc.cu -- a CIC density entry point that allocates no device memory.
//
// Some callers cannot let a library call cudaMalloc or cudaFree during a
// run.  One kind manages all device memory itself: fs2's own core reserves
// its working memory up front through its Mem arena, and a framework's
// caching allocator may own the whole device.  The other kind calls from
// inside a tight time loop, where cudaFree's implicit device-wide
// synchronisation is not acceptable.  fs2g_cic_density_noalloc serves them:
// the deterministic CIC density, the same kernels as
// fs2g_pm_compute_density in FS2G_DEPOSIT_DETERMINISTIC mode (the binned,
// fixed-point deposit of deposit_binned.cu), with every scratch buffer (bin
// counts and cursors, bin entries, CUB's scan storage, the error word)
// placed in one file-scope __device__ array of fixed size.
//
// That array is part of the module: every GPU that loads the library holds
// it (FS2G_NOALLOC_SCRATCH_BYTES, about 10 MiB) until the process exits.
// In host code its name is only a host-side stand-in; the device address
// comes from cudaGetSymbolAddress, taken on a device's first call (with the
// device current) and cached together with the id of the CUDA context it
// belongs to, so that a new context on that device (after cudaDeviceReset)
// is looked up again instead of reusing a stale address.
#include <cuda.h>
#include <mutex>
#include "internal.h"

namespace fs2g {
namespace {

constexpr size_t kMaxNp = FS2G_NOALLOC_MAX_PARTICLES;
constexpr int kMaxN = FS2G_NOALLOC_MAX_MESH;
constexpr size_t kMaxTiles =
    (size_t)((kMaxN + BIN_TX - 1)/BIN_TX)*((kMaxN + BIN_TY - 1)/BIN_TY)*
    ((kMaxN + BIN_TZ - 1)/BIN_TZ);
constexpr size_t kAlign = 256;
constexpr size_t align_up(size_t b) { return (b + kAlign - 1)/kAlign*kAlign; }

// layout of the scratch array (byte offsets, each 256-aligned)
constexpr size_t kCounts = 0;
constexpr size_t kCursor = kCounts + align_up(4*kMaxTiles);
constexpr size_t kIdx = kCursor + align_up(4*kMaxTiles);
constexpr size_t kErr = kIdx + align_up(4*8*kMaxNp);   // 8 bins per particle
constexpr size_t kTemp = kErr + kAlign;
constexpr size_t kTempBytes = size_t(1) << 20;     // CUB scan storage
constexpr size_t kTotal = kTemp + kTempBytes;
static_assert(kTotal == FS2G_NOALLOC_SCRATCH_BYTES,
              "FS2G_NOALLOC_SCRATCH_BYTES in fs2gpu.h must match the layout");

// the scratch: one copy per device, for the life of the process
static __device__ __align__(256) unsigned char g_noalloc_scratch[kTotal];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
unsigned char* g_addr[kMaxDevices] = {nullptr};
unsigned long long g_ctx_id[kMaxDevices] = {0};

// id of the current CUDA context (cuCtxGetCurrent and cuCtxGetId through
// the runtime's driver entry points; 0 if unavailable or no context)
unsigned long long current_context_id() {
  typedef CUresult (*GetCurrent)(CUcontext*);
  typedef CUresult (*GetId)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static bool looked_up = false;
  if(!looked_up) {
    cudaDriverEntryPointQueryResult q;
    void* f = nullptr;
    if(cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q)
       == cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent) f;
    f = nullptr;
    if(cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q)
       == cudaSuccess && q == cudaDriverEntryPointSuccess)
      get_id = (GetId) f;
    (void) cudaGetLastError();
    looked_up = true;
  }
  CUcontext ctx = nullptr;
  unsigned long long id = 0;
  if(get_current && get_id && get_current(&ctx) == CUDA_SUCCESS && ctx &&
     get_id(ctx, &id) == CUDA_SUCCESS)
    return id;
  return 0;
}

// set-up, once per device (and per context on it): the scratch's device
// address, and the shared-memory limit of the deposit kernel.  Called with
// the device current.
unsigned char* scratch_address(int device) {
  std::lock_guard<std::mutex> lock(g_mutex);
  const unsigned long long id = current_context_id();
  if(g_addr[device] && id != 0 && g_ctx_id[device] == id)
    return g_addr[device];
  void* ptr = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
  if(e != cudaSuccess) {
    (void) cudaGetLastError();
    throw Error{FS2G_ERR_CUDA, std::string("cudaGetSymbolAddress of the "
                "no-alloc scratch failed: ") + cudaGetErrorString(e)};
  }
  FS2G_CUDA(deposit_binned_set_smem_limits());
  g_addr[device] = (unsigned char*) ptr;
  // the context is current now (the symbol lookup initialises it)
  g_ctx_id[device] = current_context_id();
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
  if(n < 2 || n > kMaxN)
    return fail(FS2G_ERR_VALUE, "fs2g_cic_density_noalloc: n = " +
                std::to_string(n) + " outside 2 .. FS2G_NOALLOC_MAX_MESH = " +
                std::to_string(kMaxN));
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
    const BinGeom g = bin_geometry(n);
    if(bin_scan_temp_bytes(g.ntx*g.nty*g.ntz) > kTempBytes)
      throw Error{FS2G_ERR_VALUE, "CUB scan storage for this mesh exceeds "
                  "the no-alloc scratch"};
    BinScratch sc;
    sc.counts = (uint32_t*)(base + kCounts);
    sc.cursor = (uint32_t*)(base + kCursor);
    sc.idx = (uint32_t*)(base + kIdx);
    sc.temp = base + kTemp;
    sc.temp_bytes = kTempBytes;
    int* err = (int*)(base + kErr);
    cudaStream_t s = (cudaStream_t) cuda_stream;
    // the array keeps the previous call's contents: zero what must start at
    // 0 (the deposit zeroes the bin counts itself)
    FS2G_CUDA(cudaMemsetAsync(err, 0, 2*sizeof(int), s));
    const float dx_inv = (float) n / (float) boxsize;            // py/pm.cpp:77
    const float fac = (float)(pm_factor*pm_factor*pm_factor);    // py/pm.cpp:78
    // wrap = false: the positions are only read
    FS2G_CUDA(deposit_binned_on(s, const_cast<float*>(x0),
                                const_cast<float*>(x1), const_cast<float*>(x2),
                                np, mesh, n, dx_inv, fac, (float) boxsize,
                                false, sc, err));
    FS2G_CUDA(cudaStreamSynchronize(s));
    int herr[2] = {0, 0};
    FS2G_CUDA(cudaMemcpy(herr, err, sizeof(herr), cudaMemcpyDeviceToHost));
    if(herr[0] == DEV_POSITION_OUT_OF_RANGE)
      throw Error{FS2G_ERR_DEVICE, "particle " + std::to_string(herr[1]) +
                  " lies below -1 cell: wrap positions into the box first"};
    return FS2G_OK;
  }
  catch(const Error& e) { return fail(e.code, e.msg); }
  catch(const std::exception& e) { return fail(FS2G_ERR_RUNTIME, e.what()); }
}
