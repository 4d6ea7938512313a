// CTA-wide tiled complex FP64 GEMM on arbitrary operand accessors, shared by
// the adjoint and measurement kernels.  sm_100a only.
#pragma once

#include "mpsb_common.cuh"

namespace mpsb {

constexpr int kCtaGemmThreads = 256;
constexpr int kGT = 64;  // output tile edge
constexpr int kGK = 16;  // k chunk staged in shared memory

struct GemmSmem {
    double2 a[kGK][kGT + 1];
    double2 b[kGK][kGT + 1];
};

// out(i, j, sum_k a(i, k) b(k, j)) for i < m, j < n, k < kk, by all 256
// threads of the CTA (each owns 4 x 4 outputs of a 64 x 64 tile).  AK / BJ
// choose which index runs fastest across threads while a tile is staged, so
// that row-major and transposed operands both load contiguously.  The next
// k chunk's operands are fetched into registers while the current chunk
// computes (the operands come from L2 through the accessors; waiting on them
// right before the FMAs was the kernels' top stall).
template <bool AK, bool BJ, class FA, class FB, class FO>
__device__ void cta_cgemm(int m, int n, int kk, FA fa, FB fb, FO out, GemmSmem &sm) {
    constexpr int kPer = kGK * kGT / kCtaGemmThreads;  // elements of each operand per thread and chunk
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
    auto a_at = [&](int q, int &ii, int &kq) {
        const int e = tid + q * kCtaGemmThreads;
        if (AK) {
            kq = e & (kGK - 1);
            ii = e >> 4;
        } else {
            ii = e & (kGT - 1);
            kq = e >> 6;
        }
    };
    auto b_at = [&](int q, int &jj, int &kb) {
        const int e = tid + q * kCtaGemmThreads;
        if (BJ) {
            jj = e & (kGT - 1);
            kb = e >> 6;
        } else {
            kb = e & (kGK - 1);
            jj = e >> 4;
        }
    };
    for (int i0 = 0; i0 < m; i0 += kGT) {
        for (int j0 = 0; j0 < n; j0 += kGT) {
            double2 acc[4][4];
#pragma unroll
            for (int qi = 0; qi < 4; ++qi)
#pragma unroll
                for (int qj = 0; qj < 4; ++qj) acc[qi][qj] = make_double2(0.0, 0.0);
            double2 ra[kPer], rb[kPer];
            auto fetch = [&](int k0) {
#pragma unroll
                for (int q = 0; q < kPer; ++q) {
                    int ii, kq, jj, kb;
                    a_at(q, ii, kq);
                    b_at(q, jj, kb);
                    const int gi = i0 + ii, gk = k0 + kq, gj = j0 + jj, gk2 = k0 + kb;
                    ra[q] = (gi < m && gk < kk) ? fa(gi, gk) : make_double2(0.0, 0.0);
                    rb[q] = (gj < n && gk2 < kk) ? fb(gk2, gj) : make_double2(0.0, 0.0);
                }
            };
            fetch(0);
            for (int k0 = 0; k0 < kk; k0 += kGK) {
                __syncthreads();  // the previous chunk's reads of the tiles are done
#pragma unroll
                for (int q = 0; q < kPer; ++q) {
                    int ii, kq, jj, kb;
                    a_at(q, ii, kq);
                    b_at(q, jj, kb);
                    sm.a[kq][ii] = ra[q];
                    sm.b[kb][jj] = rb[q];
                }
                __syncthreads();
                if (k0 + kGK < kk) fetch(k0 + kGK);
#pragma unroll 4
                for (int kq = 0; kq < kGK; ++kq) {
                    double2 av[4], bv[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        av[q] = sm.a[kq][ty + 16 * q];
                        bv[q] = sm.b[kq][tx + 16 * q];
                    }
#pragma unroll
                    for (int qi = 0; qi < 4; ++qi)
#pragma unroll
                        for (int qj = 0; qj < 4; ++qj) acc[qi][qj] = c_fma(av[qi], bv[qj], acc[qi][qj]);
                }
            }
#pragma unroll
            for (int qi = 0; qi < 4; ++qi)
#pragma unroll
                for (int qj = 0; qj < 4; ++qj) {
                    const int i = i0 + ty + 16 * qi, j = j0 + tx + 16 * qj;
                    if (i < m && j < n) out(i, j, acc[qi][qj]);
                }
        }
    }
    __syncthreads();
}

}  // namespace mpsb
