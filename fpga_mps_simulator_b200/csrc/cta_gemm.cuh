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

// FP64 tensor-core MMA (the sm_80+ mma.sync shape; tcgen05 has no FP64
// kind): D = A B + D for an 8 x 8 block, k = 4.  Fragments: a = A[g][t4],
// b = B[t4][g], d = D[g][2 t4 + {0, 1}] with g = lane / 4, t4 = lane % 4.
__device__ __forceinline__ void dmma_m8n8k4(double &d0, double &d1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d0), "+d"(d1)
        : "d"(a), "d"(b));
}

// out(i, j, sum_k a(i, k) b(k, j)) for i < m, j < n, k < kk, by all 256
// threads of the CTA: warp w owns rows 8w..8w+7 of a 64 x 64 tile, as eight
// 8 x 8 blocks computed with FP64 tensor-core MMAs (a complex k4 step is four
// real MMAs: Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br).  AK / BJ
// choose which index runs fastest across threads while a tile is staged, so
// that row-major and transposed operands both load contiguously.  The next
// k chunk's operands are fetched into registers while the current chunk
// computes (the operands come from L2 through the accessors; waiting on them
// right before the FMAs was the kernels' top stall).
template <bool AK, bool BJ, class FA, class FB, class FO>
__device__ void cta_cgemm(int m, int n, int kk, FA fa, FB fb, FO out, GemmSmem &sm) {
    constexpr int kPer = kGK * kGT / kCtaGemmThreads;  // elements of each operand per thread and chunk
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t4 = lane & 3;
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
            double cr[8][2], ci[8][2];  // warp's 8 x 64 strip: 8 blocks of 8 x 8, real and imaginary
#pragma unroll
            for (int cb = 0; cb < 8; ++cb) cr[cb][0] = cr[cb][1] = ci[cb][0] = ci[cb][1] = 0.0;
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
#pragma unroll
                for (int k4 = 0; k4 < kGK; k4 += 4) {
                    const double2 av = sm.a[k4 + t4][8 * warp + g];
                    const double nai = -av.y;
#pragma unroll
                    for (int cb = 0; cb < 8; ++cb) {
                        const double2 bv = sm.b[k4 + t4][8 * cb + g];
                        dmma_m8n8k4(cr[cb][0], cr[cb][1], av.x, bv.x);
                        dmma_m8n8k4(cr[cb][0], cr[cb][1], nai, bv.y);
                        dmma_m8n8k4(ci[cb][0], ci[cb][1], av.x, bv.y);
                        dmma_m8n8k4(ci[cb][0], ci[cb][1], av.y, bv.x);
                    }
                }
            }
            const int i = i0 + 8 * warp + g;
#pragma unroll
            for (int cb = 0; cb < 8; ++cb)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int j = j0 + 8 * cb + 2 * t4 + h;
                    if (i < m && j < n) out(i, j, make_double2(cr[cb][h], ci[cb][h]));
                }
        }
    }
    __syncthreads();
}

}  // namespace mpsb
