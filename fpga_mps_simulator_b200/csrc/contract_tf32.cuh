// Theta of the mixed-precision two-site update on the fifth-generation tensor
// cores: T = A_mat x B_mat as a complex 3M product (three real GEMMs:
// P1 = Re A Re B, P2 = Im A Im B, P3 = (Re A + Im A)(Re B + Im B); then
// Re T = P1 - P2, Im T = P3 - P1 - P2), each real GEMM in split-precision
// 3xTF32 (a b ~ a_hi b_hi + a_hi b_lo + a_lo b_hi, FP32 accumulation in
// TMEM; at M = 128 the two correction terms in an accumulator bank of their
// own, added in FP64 on read-back).  The 4x4 gate is then mixed in FP64 while reading the accumulators
// back, and the result lands in the Jacobi slots exactly like the FP64 path.
//
// Included by update2q.cu only.  One CTA issues its own cta_group::1 MMAs
// (M = 128, K = 8 per instruction, N <= 64); operands are staged in shared
// memory in the canonical K-major no-swizzle layout: 8-row x 16-byte core
// matrices, K-chunks of one row group contiguous (leading byte offset 128 B,
// stride byte offset K/4 * 128 B).
#pragma once

#include "mpsb_common.cuh"

namespace mpsb {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// tf32 rounding (round to nearest, ties away) of an fp32 value, bits returned.
__device__ __forceinline__ uint32_t to_tf32(float f) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(f));
    return r;
}

// hi/lo tf32 split of a double: hi = tf32(x), lo = tf32(x - hi).
__device__ __forceinline__ void split_tf32(double x, uint32_t &hi, uint32_t &lo) {
    hi = to_tf32(static_cast<float>(x));
    lo = to_tf32(static_cast<float>(x - static_cast<double>(__uint_as_float(hi))));
}

// Shared-memory matrix descriptor (tcgen05), K-major, no swizzle, version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo_bytes >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor: D f32, A and B tf32, both K-major, M (64 or 128), N.
__device__ __forceinline__ uint32_t make_idesc_tf32(int m, int n) {
    return (1u << 4) | (2u << 7) | (2u << 10) | (static_cast<uint32_t>(n >> 3) << 17) |
           (static_cast<uint32_t>(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t *mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}

// Bounded wait for the given phase parity of an mbarrier.  Returns false on
// timeout (the caller records it and still releases its resources).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity) {
    const uint32_t addr = smem_u32(mbar);
    for (uint32_t polls = 0; polls < (1u << 24); ++polls) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Warp-wide TMEM allocation of `ncols` columns (power of two >= 32); the base
// address is written to *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive fp32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = __uint_as_float(r[k]);
}

// Byte offset of element (row, k) in the canonical layout with kc = K/4 chunks per row group.
__device__ __forceinline__ uint32_t core_off(int row, int k, int kc) {
    return static_cast<uint32_t>(((row >> 3) * kc + (k >> 2)) * 128 + (row & 7) * 16 + (k & 3) * 4);
}

}  // namespace tc

// Shapes of one CTA's GEMM.  Rows ("m", up to mt, padded to the MMA height
// mt: 128 above chi_cap 32, 64 at or below it) run over the index the CTA
// does not split, columns ("n", up to 64, padded to 16) over its share of the
// split index, K over the shared bond chi_m (padded to 8):
//   X = M   (no transpose): m = 2a + p (all a), n = 2(d - idx0) + q
//   X = M^H (transpose):    m = 2d + q (all d), n = 2(a - idx0) + p
// The accumulator of an M = 128 MMA holds row m in TMEM lane m; that of an
// M = 64 MMA (one CTA) holds row m = m0 + 16 m1 (m0 < 16, m1 < 4) in lane
// m0 + 32 m1, the first half of each warp's 32-lane quarter.
// corr: the correction products hi*lo and lo*hi accumulate in a second bank
// of accumulators 3 npad columns on (M = 128 tiles), so the fp32 rounding of
// the large hi*hi sum does not also swallow the low bits of the corrections;
// the two banks are added in FP64 on read-back.
struct TcShape {
    int mvalid, nvalid, kpad, npad, mt;
    bool corr;
};
__device__ __forceinline__ int tmem_lane_of_row(int m, int mt) { return mt == 128 ? m : (m & 15) + 32 * (m >> 4); }

// Operand value of the real product `prod` (0: Re, 1: Im, 2: Re + Im).
__device__ __forceinline__ double part(double2 v, int prod) {
    return prod == 0 ? v.x : (prod == 1 ? v.y : v.x + v.y);
}

// Stage the hi/lo tf32 operands of product `prod` into shared memory:
// Ahi | Alo (128 x kpad each) then Bhi | Blo (npad x kpad each).
// COHERENT (the persistent kernel): the sites were written by other CTAs of
// the same launch, so they are read through L2 rather than L1.
template <int NT, bool COHERENT = false>
__device__ void stage_operands(unsigned char *buf, const double2 *A, const double2 *B, int cl, int cm, int cr,
                               bool trans, int idx0, const TcShape &sh, int prod, int tid) {
    auto ld = [](const double2 *q) -> double2 {
        if constexpr (COHERENT)
            return __ldcg(q);
        else
            return *q;
    };
    const int kc = sh.kpad >> 2;
    const uint32_t abytes = static_cast<uint32_t>(sh.mt) * sh.kpad * 4u;
    const uint32_t bbytes = static_cast<uint32_t>(sh.npad) * sh.kpad * 4u;
    unsigned char *ahi = buf, *alo = buf + abytes, *bhi = buf + 2 * abytes, *blo = buf + 2 * abytes + bbytes;
    // A operand: rows m < mt, one 16-byte chunk (4 k) per thread-iteration
    const int achunks = sh.mt * kc;
    for (int e = tid; e < achunks; e += NT) {
        const int r8 = e & 7, c = (e >> 3) % kc, g = (e >> 3) / kc;
        const int m = g * 8 + r8, k0 = c * 4;
        uint32_t h[4], l[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            double v = 0.0;
            if (m < sh.mvalid && k < cm) {
                if (!trans) {  // A[a, p, k] with m = 2a + p
                    v = part(ld(A + (size_t)m * cm + k), prod);
                } else {       // B[k, q, d] with m = 2d + q
                    v = part(ld(B + (size_t)(2 * k + (m & 1)) * cr + (m >> 1)), prod);
                }
            }
            tc::split_tf32(v, h[q], l[q]);
        }
        const uint32_t off = static_cast<uint32_t>((g * kc + c) * 128 + r8 * 16);
        *reinterpret_cast<uint4 *>(ahi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(alo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
    // B operand: rows n < npad
    const int bchunks = sh.npad * kc;
    for (int e = tid; e < bchunks; e += NT) {
        const int r8 = e & 7, c = (e >> 3) % kc, g = (e >> 3) / kc;
        const int n = g * 8 + r8, k0 = c * 4;
        uint32_t h[4], l[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const int k = k0 + q;
            double v = 0.0;
            if (n < sh.nvalid && k < cm) {
                if (!trans) {  // B[k, q, d] with n = 2(d - idx0) + q
                    v = part(ld(B + (size_t)(2 * k + (n & 1)) * cr + idx0 + (n >> 1)), prod);
                } else {       // A[a, p, k] with n = 2(a - idx0) + p
                    v = part(ld(A + (size_t)(2 * (idx0 + (n >> 1)) + (n & 1)) * cm + k), prod);
                }
            }
            tc::split_tf32(v, h[q], l[q]);
        }
        const uint32_t off = static_cast<uint32_t>((g * kc + c) * 128 + r8 * 16);
        *reinterpret_cast<uint4 *>(bhi + off) = make_uint4(h[0], h[1], h[2], h[3]);
        *reinterpret_cast<uint4 *>(blo + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

// One thread issues the 3xTF32 MMAs of a product into accumulator column `dcol`.
__device__ __forceinline__ void issue_product(unsigned char *buf, uint32_t tmem, int dcol, const TcShape &sh) {
    const int kc = sh.kpad >> 2;
    const uint32_t abytes = static_cast<uint32_t>(sh.mt) * sh.kpad * 4u;
    const uint32_t bbytes = static_cast<uint32_t>(sh.npad) * sh.kpad * 4u;
    const uint32_t ahi = tc::smem_u32(buf), alo = ahi + abytes, bhi = ahi + 2 * abytes, blo = bhi + bbytes;
    const uint32_t sbo = static_cast<uint32_t>(kc) * 128u;
    const uint32_t idesc = tc::make_idesc_tf32(sh.mt, sh.npad);
    const uint32_t d = tmem + static_cast<uint32_t>(dcol);
    const uint32_t dc = sh.corr ? d + static_cast<uint32_t>(3 * sh.npad) : d;  // correction bank
    for (int s = 0; s < (sh.kpad >> 3); ++s) {
        const uint32_t step = static_cast<uint32_t>(s) * 256u;  // two 16-byte K chunks per K = 8 step
        tc::mma_tf32(d, tc::make_desc(ahi + step, 128, sbo), tc::make_desc(bhi + step, 128, sbo), idesc, s > 0);
        tc::mma_tf32(dc, tc::make_desc(ahi + step, 128, sbo), tc::make_desc(blo + step, 128, sbo), idesc,
                     (sh.corr && s == 0) ? 0u : 1u);
        tc::mma_tf32(dc, tc::make_desc(alo + step, 128, sbo), tc::make_desc(bhi + step, 128, sbo), idesc, 1);
    }
}

// Read the three accumulators back, form T = P1 - P2 + i (P3 - P1 - P2),
// apply the gate in FP64 and write theta into the Jacobi slots (X) and the
// workspace copy (x0), in the same positions the FP64 path uses.  Warp w
// reads TMEM lanes 32 (w & 3) .. +31 and 16-column chunks w >> 2,
// w >> 2 + NT / 128, ...; its lanes hold rows m = 32 (w & 3) + lane (M = 128)
// or, in lanes 0..15, rows m = 16 (w & 3) + lane (M = 64).  The two values of
// a row pair (m, m ^ 1) meet by shuffle.  Rows no warp reads (M = 64 with two
// warps: rows 32..63) must be padding (mvalid <= 32).
template <int NT, bool WRITE_X = true>
__device__ void read_theta(uint32_t tmem, const TcShape &sh, const double2 *g, bool trans, int cr, int C,
                           int idx0, int nidx, int w, int wmax, int rpad, double2 *X, double2 *x0, int tid,
                           int &nonfin) {
    const int warp = tid >> 5, lane = tid & 31;
    const int qr = warp & 3;
    const int m = sh.mt == 128 ? 32 * qr + lane : 16 * qr + lane;
    const bool mval = m < sh.mvalid && (sh.mt == 128 || lane < 16);
    const int nchunks = sh.npad >> 4;
    constexpr int kChunkStride = NT >= 256 ? NT / 128 : 1;
    for (int ch = warp >> 2; ch < nchunks; ch += kChunkStride) {
        const uint32_t base = tmem + (static_cast<uint32_t>(32 * qr) << 16) + static_cast<uint32_t>(16 * ch);
        float p1[16], p2[16], p3[16];
        double d1[16], d2[16], d3[16];
        tc::tmem_ld16(base, p1);
        tc::tmem_ld16(base + static_cast<uint32_t>(sh.npad), p2);
        tc::tmem_ld16(base + static_cast<uint32_t>(2 * sh.npad), p3);
#pragma unroll
        for (int q = 0; q < 16; ++q) {
            d1[q] = p1[q];
            d2[q] = p2[q];
            d3[q] = p3[q];
        }
        if (sh.corr) {  // add the correction bank in FP64
            tc::tmem_ld16(base + static_cast<uint32_t>(3 * sh.npad), p1);
            tc::tmem_ld16(base + static_cast<uint32_t>(4 * sh.npad), p2);
            tc::tmem_ld16(base + static_cast<uint32_t>(5 * sh.npad), p3);
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                d1[q] += p1[q];
                d2[q] += p2[q];
                d3[q] += p3[q];
            }
        }
#pragma unroll
        for (int jj = 0; jj < 8; ++jj) {
            // own row m: columns n = 16 ch + 2 jj + {0, 1}
            const double o0r = d1[2 * jj] - d2[2 * jj];
            const double o0i = d3[2 * jj] - d1[2 * jj] - d2[2 * jj];
            const double o1r = d1[2 * jj + 1] - d2[2 * jj + 1];
            const double o1i = d3[2 * jj + 1] - d1[2 * jj + 1] - d2[2 * jj + 1];
            const double q0r = __shfl_xor_sync(0xffffffffu, o0r, 1), q0i = __shfl_xor_sync(0xffffffffu, o0i, 1);
            const double q1r = __shfl_xor_sync(0xffffffffu, o1r, 1), q1i = __shfl_xor_sync(0xffffffffu, o1i, 1);
            const int col = 8 * ch + jj;  // index within the CTA's share (dd or aa)
            if (!mval || col >= nidx) continue;
            const int lo = m & 1;
            const double2 own0 = make_double2(o0r, o0i), own1 = make_double2(o1r, o1i);
            const double2 oth0 = make_double2(q0r, q0i), oth1 = make_double2(q1r, q1i);
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                // !trans: row m = 2a + p holds s0 = p, t = s1; trans: row m = 2d + q holds s1 = q, t = s0
                const int s0 = trans ? t : lo, s1 = trans ? lo : t;
                const int srow = 2 * s0 + s1;
                double2 v = make_double2(0.0, 0.0);
#pragma unroll
                for (int pp = 0; pp < 2; ++pp) {
#pragma unroll
                    for (int qq = 0; qq < 2; ++qq) {
                        // T_{pp qq}: the row bit of m is p (!trans) or q (trans), the column bit the other one
                        const int rowbit = trans ? qq : pp, colbit = trans ? pp : qq;
                        const double2 tv = (rowbit == lo) ? (colbit ? own1 : own0) : (colbit ? oth1 : oth0);
                        v = c_fma(g[4 * srow + 2 * pp + qq], tv, v);
                    }
                }
                nonfin |= !c_finite(v);
                int r, j, xcol;
                if (!trans) {
                    const int a = m >> 1, d = idx0 + col;
                    r = 2 * a + s0;
                    j = 2 * col + s1;
                    xcol = s1 * cr + d;
                } else {
                    const int d = m >> 1, a = idx0 + col;
                    r = s1 * cr + d;
                    j = 2 * col + s0;
                    xcol = 2 * a + s0;
                    v = c_conj(v);
                }
                const int slot = j >= w, jl = j - slot * w;
                if constexpr (WRITE_X) X[(size_t)(slot * wmax + jl) * rpad + r] = v;
                x0[(size_t)r * C + xcol] = v;
            }
        }
    }
}

// Whole mixed-precision contraction of one CTA.  Returns false when an
// mbarrier wait timed out (the caller reports MPSB_ST_TIMEOUT); TMEM is
// released on every path.  Called once per CTA (a CTA may allocate TMEM
// only until it relinquishes the permit).  COHERENT: read the sites through
// L2 (the dataflow kernel, where other clusters of the launch wrote them).
// WRITE_X = false (the contraction-only kernel): theta goes to x0 alone, so
// the shared memory holds just the operand staging area.
template <int NT, bool COHERENT = false, bool WRITE_X = true>
__device__ bool contract_mixed(unsigned char *opbuf, uint64_t *mbar, uint32_t *tmem_slot, const double2 *A,
                               const double2 *B, const double2 *g, int cl, int cm, int cr, bool trans, int idx0,
                               int nidx, int C, int w, int wmax, int rpad, double2 *X, double2 *x0, int tid,
                               int &nonfin) {
    TcShape sh;
    sh.mvalid = trans ? 2 * cr : 2 * cl;
    sh.nvalid = 2 * nidx;
    sh.npad = max(16, (sh.nvalid + 15) & ~15);
    sh.kpad = (cm + 7) & ~7;
    sh.mt = rpad > 64 ? 128 : 64;  // rows of a column: 128 above chi_cap 32, at most 64 below
    // (the 64-row tiles run three CTAs per SM, whose TMEM must fit together:
    // one bank there)
    sh.corr = sh.mt == 128;
    const int need = (sh.corr ? 6 : 3) * sh.npad;
    const uint32_t ncols = need <= 32 ? 32u : need <= 64 ? 64u : need <= 128 ? 128u : need <= 256 ? 256u : 512u;
    if ((tid >> 5) == 0) tc::tmem_alloc(tmem_slot, ncols);
    if (tid == 0) {
        tc::mbar_init(mbar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    for (int prod = 0; prod < 3; ++prod) {
        stage_operands<NT, COHERENT>(opbuf, A, B, cl, cm, cr, trans, idx0, sh, prod, tid);
        tc::fence_proxy_async();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            issue_product(opbuf, tmem, prod * sh.npad, sh);
            tc::mma_commit(mbar);
        }
        ok = tc::mbar_wait(mbar, static_cast<uint32_t>(prod & 1)) && ok;
        __syncthreads();
    }
    tc::fence_after_sync();
    // the operand staging area overlaps the Jacobi slots: clear them before writing theta
    if constexpr (WRITE_X)
        for (int e = tid; e < 2 * wmax * rpad; e += NT) X[e] = make_double2(0.0, 0.0);
    __syncthreads();
    if (ok) read_theta<NT, WRITE_X>(tmem, sh, g, trans, cr, C, idx0, nidx, w, wmax, rpad, X, x0, tid, nonfin);
    tc::fence_before_sync();
    __syncthreads();
    if ((tid >> 5) == 0) tc::tmem_free(tmem, ncols);
    return ok;
}

}  // namespace mpsb
