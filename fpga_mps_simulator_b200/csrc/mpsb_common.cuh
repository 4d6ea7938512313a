// Shared device helpers for libmpsb200: complex128 arithmetic on double2,
// warp reductions, error plumbing.  sm_100a only.
#pragma once

#include <cuda_runtime.h>
#include <cooperative_groups.h>
#include <stdint.h>

#include "mpsb200.h"

namespace mpsb {
namespace cg = cooperative_groups;

#if defined(__CUDA_ARCH__) && (__CUDA_ARCH__ < 1000)
#error "libmpsb200 is built for sm_100a only"
#endif

// ---------------------------------------------------------------- complex
__device__ __forceinline__ double2 c_make(double re, double im) { return make_double2(re, im); }
__device__ __forceinline__ double2 c_add(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 c_sub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 c_conj(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 c_scale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 c_mul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// acc + a * b
__device__ __forceinline__ double2 c_fma(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
// acc + conj(a) * b
__device__ __forceinline__ double2 c_cfma(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(-a.y, b.x, acc.y);
    return acc;
}
__device__ __forceinline__ double c_abs2(double2 a) { return fma(a.x, a.x, a.y * a.y); }
__device__ __forceinline__ bool c_finite(double2 a) { return isfinite(a.x) && isfinite(a.y); }

__device__ __forceinline__ double2 ld_c(const mpsb_c128 *p) {
    return __ldg(reinterpret_cast<const double2 *>(p));
}

// ---------------------------------------------------------------- warp
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Largest bond a two-site update of this chain may form: its chi_max, the
// device limit MPSB_CHI_LIMIT and the Schmidt-rank bound 2^(n/2) of the
// middle cut (no bond of an n-site chain can exceed it).
__host__ __device__ inline int keep_limit(const mpsb_chain &ch) {
    const int schmidt = ch.n >= 14 ? (1 << 7) : (ch.n < 2 ? 1 : (1 << (ch.n / 2)));
    int k = ch.chi_max < MPSB_CHI_LIMIT ? ch.chi_max : MPSB_CHI_LIMIT;
    return k < schmidt ? k : schmidt;
}

__host__ __device__ inline bool valid_precision(int p) {
    return p == MPSB_FP64 || p == MPSB_MIXED_TF32X3 || p == MPSB_TF32X3_ALL;
}
// Jacobi off-diagonal tolerance of a form when the caller passes none: the
// tensor-core forms' theta carries ~1e-7 relative rounding, so they stop at 1e-9.
__host__ __device__ inline double default_tol(int p) { return p == MPSB_FP64 ? 1.0e-14 : 1.0e-9; }

// Per-pair bookkeeping written by the update kernel, folded into norm_log by
// a second kernel in pair order.
struct PairRec {
    double d_trunc;   // 0.5*log(1 - dropped/total) (0 when nothing dropped)
    double d_norm;    // log(norm of kept S) (0 when norm <= 1e-15)
    double discarded; // dropped/total
    int32_t keep;
    int32_t status;
};

// Adjoint tape of one two-site update, per pair, in double2 units with
// Q = (2 chi_cap)^2:
//   [0, Q)       X = U S V^H, the matrix the update factorised (theta, or
//                theta^H when chi_r > chi_l), R x C row-major
//   [Q, 2Q)      singular vectors times S in decreasing order of S_k: either
//                u_k S_k at [Q + k R, Q + (k + 1) R), or (side flag set, the
//                QR-preconditioned factorisation) v_k S_k at
//                [Q + k C, Q + (k + 1) C)
//   [2Q, 2Q+72)  144 doubles: S[0..128), then keep, the kept-norm divisor,
//                R, C, the side flag and the number of Jacobi sweeps
// rounded up to a multiple of 16 double2 (256 bytes).
constexpr int kTapeMetaKeep = 128, kTapeMetaDiv = 129, kTapeMetaRows = 130, kTapeMetaCols = 131;
constexpr int kTapeMetaSide = 132;
constexpr int kTapeMetaSweeps = 133;  // Jacobi sweeps taken (the final one, with no rotation above the stop bound, included)
__host__ __device__ inline long long tape_stride(int chi_cap) {
    const long long q = (long long)(2 * chi_cap) * (2 * chi_cap);
    return (2 * q + 72 + 15) & ~15LL;
}

}  // namespace mpsb

// host-side error helpers (defined in api.cu)
namespace mpsb {
int set_error(int code, const char *fmt, ...);
int check_launch(const char *what);
int check_device(const void *table, void *stream);
int ensure_smem(const void *kernel, size_t bytes, const char *what);
}  // namespace mpsb
