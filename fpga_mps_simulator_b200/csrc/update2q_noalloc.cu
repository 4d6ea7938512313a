// Allocation-free entry point of the batched two-site update.
//
// mpsb_update2q_batch needs a caller-provided device workspace (the per-pair
// record and the unrotated copy of theta).  Some callers cannot provide one:
// a host runtime that hands this library only buffers registered up front
// and owns the rest of device memory (an FFI host whose pool may not be
// grown), or a time-critical loop in which a cudaMalloc / cudaFree would
// synchronise the device and is therefore forbidden.  For them,
// mpsb_update2q_batch_noalloc runs the same kernels with the scratch placed in
// a file-scope device array of MPSB_NOALLOC_SCRATCH_BYTES, which every GPU
// that loads this library holds until the process exits.  The call itself
// allocates nothing (no cudaMalloc, no cudaFree, no allocating library call).
//
// The array's name is only a host-side stand-in in host code, so its device
// address is looked up once per device with cudaGetSymbolAddress while that
// device is current; the first call on a device does this set-up, which is
// why that first call should come before any stream capture on the device.
// The address is kept per device ordinal for the life of the process: it
// assumes the device keeps one primary context throughout.  After a
// cudaDeviceReset the module is loaded again and the kept address is stale,
// so this entry must not be used across a device reset.
// All calls share the one array and it keeps the last call's contents; the
// kernels write every scratch byte they later read within the same call, so
// nothing has to be cleared between calls.  Two calls whose kernels overlap
// on the GPU (different streams, or different host threads) race on the
// array: serialise them on one stream.
#include "mpsb_common.cuh"

#include <mutex>

namespace mpsb {

size_t upd_workspace_bytes(int npairs, int chi_cap);
int launch_update2q(int, const mpsb_chain *, const mpsb_pair *, int, const double2 *, int, double, int, void *,
                    double *, int32_t *, double *, int32_t *, cudaStream_t);

static __device__ __align__(256) unsigned char g_noalloc_scratch[MPSB_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
void *g_noalloc_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device (set up once per device).
int noalloc_scratch(void **out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(MPSB_ENODEV, "no CUDA device");
    if (dev < 0 || dev >= kMaxDevices)
        return set_error(MPSB_EINVAL, "device ordinal %d beyond the %d the no-alloc entry tracks", dev, kMaxDevices);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (g_noalloc_ptr[dev] == nullptr) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || p == nullptr)
            return set_error(MPSB_ELAUNCH, "cudaGetSymbolAddress(no-alloc scratch) on device %d: %s", dev,
                             cudaGetErrorString(e));
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return MPSB_OK;
}
}  // namespace

}  // namespace mpsb

using namespace mpsb;

extern "C" int mpsb_update2q_batch_noalloc(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs,
                                           const mpsb_c128 *gates, int precision, int chi_cap, double tol,
                                           int max_sweeps, double *spectra, int32_t *kept, double *trunc,
                                           int32_t *status, mpsb_stream_t stream) {
    if (npairs < 0) return set_error(MPSB_EINVAL, "npairs=%d < 0", npairs);
    if (npairs == 0) return MPSB_OK;
    if (!chains || !pairs || !gates || !status)
        return set_error(MPSB_EINVAL, "null chains/pairs/gates/status pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (!valid_precision(precision)) return set_error(MPSB_EINVAL, "unknown precision %d", precision);
    const size_t need = upd_workspace_bytes(npairs, chi_cap);
    if (need > (size_t)MPSB_NOALLOC_SCRATCH_BYTES)
        return set_error(MPSB_EWORKSPACE,
                         "no-alloc update: %d pairs at chi_cap=%d need %zu scratch bytes, more than the fixed "
                         "%zu; split the batch or use mpsb_update2q_batch with a workspace",
                         npairs, chi_cap, need, (size_t)MPSB_NOALLOC_SCRATCH_BYTES);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    void *scratch = nullptr;
    rc = noalloc_scratch(&scratch);
    if (rc) return rc;
    if (max_sweeps <= 0) max_sweeps = 40;
    if (tol <= 0.0) tol = default_tol(precision);
    return launch_update2q(precision, chains, pairs, npairs, reinterpret_cast<const double2 *>(gates), chi_cap, tol,
                           max_sweeps, scratch, spectra, kept, trunc, status, reinterpret_cast<cudaStream_t>(stream));
}
