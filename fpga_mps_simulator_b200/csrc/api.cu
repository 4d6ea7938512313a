// C ABI of libmpsb200 (declared in include/mpsb200.h): argument checks,
// error reporting and dispatch to the kernels.
#include "mpsb_common.cuh"

#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>

namespace mpsb {

static thread_local char g_err[512] = "";

int set_error(int code, const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

int check_launch(const char *what) {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(MPSB_ELAUNCH, "%s: %s", what, cudaGetErrorString(e));
    return MPSB_OK;
}

// The current device must be an sm_100 part, and the chain table (when
// given) must be device memory of that device: every kernel launches on the
// current device, so a table on another GPU would be read through a wrong
// address space rather than refused.
int check_device(const void *table, void *stream) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(MPSB_ENODEV, "no CUDA device");
    int major = 0;
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major != 10) return set_error(MPSB_ENODEV, "device %d has compute capability %d.x; sm_100 required", dev, major);
    // (skipped while the stream is being captured into a graph, where only
    // stream-ordered work belongs)
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (table && cudaStreamIsCapturing(reinterpret_cast<cudaStream_t>(stream), &cap) == cudaSuccess &&
        cap == cudaStreamCaptureStatusNone) {
        cudaPointerAttributes at{};
        const cudaError_t e = cudaPointerGetAttributes(&at, table);
        if (e != cudaSuccess) {
            cudaGetLastError();  // clear the error this query leaves behind
            return set_error(MPSB_EINVAL, "chain table %p is not a CUDA pointer (%s)", table, cudaGetErrorString(e));
        }
        if (at.type != cudaMemoryTypeDevice && at.type != cudaMemoryTypeManaged)
            return set_error(MPSB_EINVAL, "chain table %p is not device memory", table);
        if (at.device != dev)
            return set_error(MPSB_ENODEV, "chain table lives on device %d but device %d is current", at.device, dev);
    }
    return MPSB_OK;
}

// The dynamic shared-memory limit is a per-device attribute of a kernel, so
// the largest size enabled so far is remembered per (kernel, device), under a
// lock (host threads may launch concurrently).  Called before each launch;
// only a size above the remembered one reaches cudaFuncSetAttribute.  (Any
// non-zero size is set: the default limit is 48 KB minus the kernel's static
// shared memory, which several kernels here use.)
int ensure_smem(const void *kernel, size_t bytes, const char *what) {
    if (bytes == 0) return MPSB_OK;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return set_error(MPSB_ENODEV, "no CUDA device");
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> enabled;
    std::lock_guard<std::mutex> lock(mu);
    size_t &have = enabled[std::make_pair(kernel, dev)];
    if (bytes <= have) return MPSB_OK;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) != cudaSuccess)
        return check_launch(what);
    have = bytes;
    return MPSB_OK;
}

// kernels (update2q.cu, readout.cu)
size_t upd_workspace_bytes(int npairs, int chi_cap);
int launch_update2q(int, const mpsb_chain *, const mpsb_pair *, int, const double2 *, int, double, int, void *,
                    double *, int32_t *, double *, int32_t *, cudaStream_t);
int launch_apply1q(const mpsb_chain *, const mpsb_site_op *, int, const double2 *, int, cudaStream_t);
int launch_statevector(const mpsb_chain *, int, int, double2 *, double2 *, size_t, cudaStream_t);
int launch_amplitude(const mpsb_chain *, int, int, const uint8_t *, int, double2 *, double *, cudaStream_t);
size_t expect_workspace_bytes(int nchains, int n, int chi_cap, int nctas);
int launch_expect(const mpsb_chain *, int, int, int, const int32_t *, const int32_t *, const double2 *, int,
                  double *, void *, int, cudaStream_t);
int launch_fp64_probe(long long iters, int blocks, int threads, double *sink, cudaStream_t s);
int launch_tf32_probe(long long iters, int blocks, double *sink, cudaStream_t s);
int launch_theta2q(int, const mpsb_chain *, const mpsb_pair *, int, const double2 *, int, double2 *, int32_t *,
                   cudaStream_t);
int launch_overlap(const mpsb_chain *, const mpsb_chain *, int, int, double2 *, double *, void *, cudaStream_t);

size_t upd_flow_workspace_bytes(int nitems, int chi_cap, int precision, int threads, int nclusters);
int upd_flow_clusters(int chi_cap, int precision, int threads);
int launch_update2q_flow(const mpsb_chain *, int, const mpsb_flow_item *, int, const int32_t *, const int32_t *,
                         const double2 *, int, int, double, int, int, int, int, void *, size_t, double *, int32_t *,
                         double *, int32_t *, cudaStream_t);
size_t upd_tape_bytes(int npairs, int chi_cap);
int launch_update2q_taped(int, const mpsb_chain *, const mpsb_pair *, int, const double2 *, int, double, int,
                          void *, void *, double *, int32_t *, double *, int32_t *, cudaStream_t);
size_t bwd_workspace_bytes(int npairs, int chi_cap);
int launch_update2q_backward(const mpsb_chain *, const mpsb_chain *, const mpsb_pair *, int, const double2 *, int,
                             const void *, double2 *, void *, int32_t *, double, double, cudaStream_t);
int launch_apply1q_backward(const mpsb_chain *, const mpsb_chain *, const mpsb_site_op *, int, const double2 *,
                            double2 *, cudaStream_t);
size_t mpo_grad_workspace_bytes(int nchains, int n, int chi_cap, int D);
int launch_mpo_energy_grad(const mpsb_chain *, int, int, int, const double2 *, int, const double *, double *,
                           const mpsb_chain *, void *, cudaStream_t);

size_t sample_workspace_bytes(int n, int chi_cap);
int launch_sample(const mpsb_chain *, int, int, int, const double *, int, uint8_t *, void *, cudaStream_t);
int launch_reset(const mpsb_chain *, const mpsb_site_op *, int, cudaStream_t);
size_t canon_workspace_bytes(int nchains, int chi_cap);
int launch_canonicalize(const mpsb_chain *, const int32_t *, int, int, int, int, int, void *, cudaStream_t);

static int expect_ctas() {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return 2 * sms;
}

}  // namespace mpsb

using namespace mpsb;

extern "C" {

const char *mpsb_version(void) { return "libmpsb200 1.0 (sm_100a)"; }

const char *mpsb_last_error(void) { return g_err; }

size_t mpsb_update2q_workspace_bytes(int npairs, int chi_cap) {
    if (npairs < 0 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    return upd_workspace_bytes(npairs, chi_cap);
}

int mpsb_update2q_batch(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs, const mpsb_c128 *gates,
                        int precision, int chi_cap, double tol, int max_sweeps, void *workspace,
                        size_t workspace_bytes, double *spectra, int32_t *kept, double *trunc, int32_t *status,
                        mpsb_stream_t stream) {
    if (npairs < 0) return set_error(MPSB_EINVAL, "npairs=%d < 0", npairs);
    if (npairs == 0) return MPSB_OK;
    if (!chains || !pairs || !gates || !status || !workspace)
        return set_error(MPSB_EINVAL, "null chains/pairs/gates/status/workspace pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (!valid_precision(precision))
        return set_error(MPSB_EINVAL, "unknown precision %d", precision);
    const size_t need = upd_workspace_bytes(npairs, chi_cap);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return set_error(MPSB_EINVAL, "workspace must be 256-byte aligned");
    int rc = check_device(chains, stream);
    if (rc) return rc;
    if (max_sweeps <= 0) max_sweeps = 40;
    if (tol <= 0.0) tol = default_tol(precision);
    return launch_update2q(precision, chains, pairs, npairs, reinterpret_cast<const double2 *>(gates), chi_cap, tol,
                           max_sweeps, workspace, spectra, kept, trunc, status,
                           reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_update2q_flow_workspace_bytes(int nitems, int chi_cap, int precision, int threads, int nclusters) {
    if (nitems < 0 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    if (!valid_precision(precision)) return 0;
    return upd_flow_workspace_bytes(nitems, chi_cap, precision, threads, nclusters);
}

int mpsb_update2q_flow_clusters(int chi_cap, int precision, int threads) {
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (!valid_precision(precision))
        return set_error(MPSB_EINVAL, "unknown precision %d", precision);
    int rc = check_device(nullptr, nullptr);
    if (rc) return rc;
    return upd_flow_clusters(chi_cap, precision, threads);
}

int mpsb_update2q_flow(const mpsb_chain *chains, int nchains, const mpsb_flow_item *items, int nitems,
                       const int32_t *chain_order, const int32_t *chain_offsets, const mpsb_c128 *gates,
                       int precision, int chi_cap, double tol, int max_sweeps, int threads, int nclusters,
                       int poll_limit, void *workspace, size_t workspace_bytes, double *spectra, int32_t *kept,
                       double *trunc, int32_t *status, mpsb_stream_t stream) {
    if (nitems < 0 || nchains < 0) return set_error(MPSB_EINVAL, "nitems=%d / nchains=%d < 0", nitems, nchains);
    if (nitems == 0) return MPSB_OK;
    if (!chains || !items || !chain_order || !chain_offsets || !gates || !status || !workspace)
        return set_error(MPSB_EINVAL, "null chains/items/chain_order/chain_offsets/gates/status/workspace pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (!valid_precision(precision))
        return set_error(MPSB_EINVAL, "unknown precision %d", precision);
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
        return set_error(MPSB_EINVAL, "workspace must be 256-byte aligned");
    int rc = check_device(chains, stream);
    if (rc) return rc;
    if (max_sweeps <= 0) max_sweeps = 40;
    if (tol <= 0.0) tol = default_tol(precision);
    return launch_update2q_flow(chains, nchains, items, nitems, chain_order, chain_offsets,
                                reinterpret_cast<const double2 *>(gates), precision, chi_cap, tol, max_sweeps,
                                threads, nclusters, poll_limit, workspace, workspace_bytes, spectra, kept, trunc,
                                status, reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_contract2q_batch(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs, const mpsb_c128 *gates,
                          int precision, int chi_cap, mpsb_c128 *theta, int32_t *status, mpsb_stream_t stream) {
    if (npairs < 0) return set_error(MPSB_EINVAL, "npairs=%d < 0", npairs);
    if (npairs == 0) return MPSB_OK;
    if (!chains || !pairs || !gates || !theta || !status)
        return set_error(MPSB_EINVAL, "null chains/pairs/gates/theta/status pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (!valid_precision(precision)) return set_error(MPSB_EINVAL, "unknown precision %d", precision);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_theta2q(precision, chains, pairs, npairs, reinterpret_cast<const double2 *>(gates), chi_cap,
                          reinterpret_cast<double2 *>(theta), status, reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_apply1q_batch(const mpsb_chain *chains, const mpsb_site_op *ops, int nops, const mpsb_c128 *gates,
                       int chi_cap, mpsb_stream_t stream) {
    if (nops < 0) return set_error(MPSB_EINVAL, "nops=%d < 0", nops);
    if (nops == 0) return MPSB_OK;
    if (!chains || !ops || !gates) return set_error(MPSB_EINVAL, "null chains/ops/gates pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_apply1q(chains, ops, nops, reinterpret_cast<const double2 *>(gates), chi_cap,
                          reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_statevector(const mpsb_chain *chain_dev, int n, int chi_cap, mpsb_c128 *out, mpsb_c128 *scratch,
                     size_t scratch_bytes, mpsb_stream_t stream) {
    if (!chain_dev || !out || !scratch) return set_error(MPSB_EINVAL, "null chain/out/scratch pointer");
    if (n < 1 || n > 24) return set_error(MPSB_EINVAL, "statevector needs 1 <= n <= 24, got %d", n);
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    int rc = check_device(chain_dev, stream);
    if (rc) return rc;
    return launch_statevector(chain_dev, n, chi_cap, reinterpret_cast<double2 *>(out),
                              reinterpret_cast<double2 *>(scratch), scratch_bytes,
                              reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_amplitude(const mpsb_chain *chains, int chain, int n, const uint8_t *bits, int nbits, int chi_cap,
                   mpsb_c128 *out, double *log_abs, mpsb_stream_t stream) {
    if (!chains || !bits || !out) return set_error(MPSB_EINVAL, "null chains/bits/out pointer");
    if (nbits < 0 || n < 1 || chain < 0) return set_error(MPSB_EINVAL, "bad nbits/n/chain");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_amplitude(chains, chain, n, bits, nbits, reinterpret_cast<double2 *>(out), log_abs,
                            reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_expect_workspace_bytes(int nchains, int n, int chi_cap) {
    if (nchains < 0 || n < 1 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    return expect_workspace_bytes(nchains, n, chi_cap, expect_ctas());
}

int mpsb_expect_local(const mpsb_chain *chains, int nchains, int n, int chi_cap, const int32_t *sites,
                      const int32_t *two_site, const mpsb_c128 *ops, int nterms, double *out, void *workspace,
                      size_t workspace_bytes, mpsb_stream_t stream) {
    if (nchains < 0 || nterms < 0 || n < 1) return set_error(MPSB_EINVAL, "bad nchains/nterms/n");
    if (nchains == 0 || nterms == 0) return MPSB_OK;
    if (!chains || !sites || !two_site || !ops || !out || !workspace)
        return set_error(MPSB_EINVAL, "null pointer argument");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    const int nctas = expect_ctas();
    const size_t need = expect_workspace_bytes(nchains, n, chi_cap, nctas);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_expect(chains, nchains, n, chi_cap, sites, two_site, reinterpret_cast<const double2 *>(ops),
                         nterms, out, workspace, nctas, reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_overlap(const mpsb_chain *a, const mpsb_chain *b, int n, int chi_cap, mpsb_c128 *out, double *out_log,
                 void *workspace, size_t workspace_bytes, mpsb_stream_t stream) {
    if (!a || !b || !out || !out_log || !workspace) return set_error(MPSB_EINVAL, "null pointer argument");
    if (n < 1) return set_error(MPSB_EINVAL, "n=%d < 1", n);
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    const size_t need = 2 * (size_t)chi_cap * chi_cap * sizeof(double2);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    int rc = check_device(a, stream);
    if (rc) return rc;
    return launch_overlap(a, b, n, chi_cap, reinterpret_cast<double2 *>(out), out_log, workspace,
                          reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_sample_workspace_bytes(int n, int chi_cap) {
    if (n < 1 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    return sample_workspace_bytes(n, chi_cap);
}

int mpsb_sample(const mpsb_chain *chains, int chain, int n, int chi_cap, const double *uniforms, int shots,
                uint8_t *bits, void *workspace, size_t workspace_bytes, mpsb_stream_t stream) {
    if (!chains || !workspace || (shots > 0 && (!uniforms || !bits)))
        return set_error(MPSB_EINVAL, "null chains/uniforms/bits/workspace pointer");
    if (chain < 0 || n < 1 || shots < 0) return set_error(MPSB_EINVAL, "bad chain/n/shots");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    const size_t need = sample_workspace_bytes(n, chi_cap);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_sample(chains, chain, n, chi_cap, uniforms, shots, bits, workspace,
                         reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_reset_batch(const mpsb_chain *chains, const mpsb_site_op *ops, int nops, int chi_cap,
                     mpsb_stream_t stream) {
    if (nops < 0) return set_error(MPSB_EINVAL, "nops=%d < 0", nops);
    if (nops == 0) return MPSB_OK;
    if (!chains || !ops) return set_error(MPSB_EINVAL, "null chains/ops pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_reset(chains, ops, nops, reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_canonicalize_workspace_bytes(int nchains, int chi_cap) {
    if (nchains < 0 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    return canon_workspace_bytes(nchains, chi_cap);
}

int mpsb_canonicalize(const mpsb_chain *chains, const int32_t *chain_ids, int nchains, int lo, int hi, int direction,
                      int chi_cap, void *workspace, size_t workspace_bytes, mpsb_stream_t stream) {
    if (nchains < 0) return set_error(MPSB_EINVAL, "nchains=%d < 0", nchains);
    if (nchains == 0 || hi < lo) return MPSB_OK;
    if (!chains || !chain_ids || !workspace) return set_error(MPSB_EINVAL, "null chains/chain_ids/workspace pointer");
    if (lo < 0) return set_error(MPSB_EINVAL, "lo=%d < 0", lo);
    if (direction != 0 && direction != 1) return set_error(MPSB_EINVAL, "direction must be 0 (left) or 1 (right)");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    const size_t need = canon_workspace_bytes(nchains, chi_cap);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_canonicalize(chains, chain_ids, nchains, lo, hi, direction, chi_cap, workspace,
                               reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_update2q_tape_bytes(int npairs, int chi_cap) {
    if (npairs < 0 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    return upd_tape_bytes(npairs, chi_cap);
}

int mpsb_update2q_batch_taped(const mpsb_chain *chains, const mpsb_pair *pairs, int npairs, const mpsb_c128 *gates,
                              int precision, int chi_cap, double tol, int max_sweeps, void *workspace,
                              size_t workspace_bytes, void *tape, size_t tape_bytes, double *spectra, int32_t *kept,
                              double *trunc, int32_t *status, mpsb_stream_t stream) {
    if (npairs < 0) return set_error(MPSB_EINVAL, "npairs=%d < 0", npairs);
    if (npairs == 0) return MPSB_OK;
    if (!chains || !pairs || !gates || !status || !workspace || !tape)
        return set_error(MPSB_EINVAL, "null chains/pairs/gates/status/workspace/tape pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (!valid_precision(precision))
        return set_error(MPSB_EINVAL, "unknown precision %d", precision);
    const size_t need = upd_workspace_bytes(npairs, chi_cap);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    const size_t tneed = upd_tape_bytes(npairs, chi_cap);
    if (tape_bytes < tneed) return set_error(MPSB_EWORKSPACE, "tape of %zu bytes < %zu needed", tape_bytes, tneed);
    if (((reinterpret_cast<uintptr_t>(workspace) | reinterpret_cast<uintptr_t>(tape)) & 255) != 0)
        return set_error(MPSB_EINVAL, "workspace and tape must be 256-byte aligned");
    int rc = check_device(chains, stream);
    if (rc) return rc;
    if (max_sweeps <= 0) max_sweeps = 40;
    if (tol <= 0.0) tol = default_tol(precision);
    return launch_update2q_taped(precision, chains, pairs, npairs, reinterpret_cast<const double2 *>(gates), chi_cap, tol,
                                 max_sweeps, workspace, tape, spectra, kept, trunc, status,
                                 reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_update2q_backward_workspace_bytes(int npairs, int chi_cap) {
    if (npairs < 0 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT) return 0;
    return bwd_workspace_bytes(npairs, chi_cap);
}

int mpsb_update2q_backward_batch(const mpsb_chain *pre, const mpsb_chain *cot, const mpsb_pair *pairs, int npairs,
                                 const mpsb_c128 *gates, int chi_cap, const void *tape, size_t tape_bytes,
                                 mpsb_c128 *gate_grads, void *workspace, size_t workspace_bytes, int32_t *status,
                                 mpsb_stream_t stream) {
    if (npairs < 0) return set_error(MPSB_EINVAL, "npairs=%d < 0", npairs);
    if (npairs == 0) return MPSB_OK;
    if (!pre || !cot || !pairs || !gates || !tape || !workspace || !status)
        return set_error(MPSB_EINVAL, "null pre/cot/pairs/gates/tape/workspace/status pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (tape_bytes < upd_tape_bytes(npairs, chi_cap))
        return set_error(MPSB_EWORKSPACE, "tape of %zu bytes < %zu needed", tape_bytes, upd_tape_bytes(npairs, chi_cap));
    const size_t need = bwd_workspace_bytes(npairs, chi_cap);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)  // its L2 lines are discarded per pair
        return set_error(MPSB_EINVAL, "workspace must be 256-byte aligned");
    int rc = check_device(pre, stream);
    if (rc) return rc;
    return launch_update2q_backward(pre, cot, pairs, npairs, reinterpret_cast<const double2 *>(gates), chi_cap, tape,
                                    reinterpret_cast<double2 *>(gate_grads), workspace, status, 1.0e-6, 1.0e-12,
                                    reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_apply1q_backward_batch(const mpsb_chain *pre, const mpsb_chain *cot, const mpsb_site_op *ops, int nops,
                                const mpsb_c128 *gates, int chi_cap, mpsb_c128 *gate_grads, mpsb_stream_t stream) {
    if (nops < 0) return set_error(MPSB_EINVAL, "nops=%d < 0", nops);
    if (nops == 0) return MPSB_OK;
    if (!pre || !cot || !ops || !gates) return set_error(MPSB_EINVAL, "null pre/cot/ops/gates pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    int rc = check_device(pre, stream);
    if (rc) return rc;
    return launch_apply1q_backward(pre, cot, ops, nops, reinterpret_cast<const double2 *>(gates),
                                   reinterpret_cast<double2 *>(gate_grads), reinterpret_cast<cudaStream_t>(stream));
}

size_t mpsb_mpo_grad_workspace_bytes(int nchains, int n, int chi_cap, int mpo_bond) {
    if (nchains < 0 || n < 1 || chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT || mpo_bond < 1 || mpo_bond > 16) return 0;
    return mpo_grad_workspace_bytes(nchains, n, chi_cap, mpo_bond);
}

int mpsb_mpo_energy_grad(const mpsb_chain *chains, int nchains, int n, int chi_cap, const mpsb_c128 *mpo,
                         int mpo_bond, const double *weights, double *loss, const mpsb_chain *cot, void *workspace,
                         size_t workspace_bytes, mpsb_stream_t stream) {
    if (nchains < 0 || n < 1) return set_error(MPSB_EINVAL, "bad nchains/n");
    if (nchains == 0) return MPSB_OK;
    if (!chains || !mpo || !cot || !workspace) return set_error(MPSB_EINVAL, "null chains/mpo/cot/workspace pointer");
    if (chi_cap < 1 || chi_cap > MPSB_CHI_LIMIT)
        return set_error(MPSB_EINVAL, "chi_cap=%d outside [1, %d]", chi_cap, MPSB_CHI_LIMIT);
    if (mpo_bond < 1 || mpo_bond > 16) return set_error(MPSB_EINVAL, "mpo bond %d outside [1, 16]", mpo_bond);
    const size_t need = mpo_grad_workspace_bytes(nchains, n, chi_cap, mpo_bond);
    if (workspace_bytes < need)
        return set_error(MPSB_EWORKSPACE, "workspace of %zu bytes < %zu needed", workspace_bytes, need);
    int rc = check_device(chains, stream);
    if (rc) return rc;
    return launch_mpo_energy_grad(chains, nchains, n, chi_cap, reinterpret_cast<const double2 *>(mpo), mpo_bond,
                                  weights, loss, cot, workspace, reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_fp64_probe(int64_t iters, int blocks, int threads, double *sink, mpsb_stream_t stream) {
    if (iters < 1 || blocks < 1 || threads < 32 || threads > 1024 || !sink)
        return set_error(MPSB_EINVAL, "bad probe arguments");
    int rc = check_device(nullptr, stream);
    if (rc) return rc;
    return launch_fp64_probe(iters, blocks, threads, sink, reinterpret_cast<cudaStream_t>(stream));
}

int mpsb_tf32_probe(int64_t iters, int blocks, double *sink, mpsb_stream_t stream) {
    // (the cap keeps one CTA's MMA chain, ~5 ms at the TF32 peak, far inside
    // the bounded completion wait)
    if (iters < 1 || iters > 65536 || blocks < 1 || !sink) return set_error(MPSB_EINVAL, "bad probe arguments");
    int rc = check_device(nullptr, stream);
    if (rc) return rc;
    return launch_tf32_probe(iters, blocks, sink, reinterpret_cast<cudaStream_t>(stream));
}

}  // extern "C"
