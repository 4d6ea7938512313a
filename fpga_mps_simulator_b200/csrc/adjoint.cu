// Hand-written adjoint of the MPS two-site update, of single-site gates, and
// of a normalised matrix-product-operator energy, for sm_100a.
//
// The reference engine (mps_core.py of nasir26/fpga-mps-simulator) has no
// gradients; these kernels differentiate exactly the forward the fused update
// kernel computes (mps_core.py:326-350 with the keep / renormalise rule of
// mps_core.py:277-300).  Convention: for a real loss L the cotangent of a
// complex array z is z_bar = dL/dRe z + i dL/dIm z, so y = W x gives
// x_bar = W^H y_bar.
//
// Two-site update backward (persistent grid, one pair per CTA at a time).
// The forward's Jacobi factorised X = theta (or theta^H when chi_r > chi_l), R x C with R >= C,
// as X = U S V^H; the tape holds X, the converged columns u_k S_k in
// decreasing order of S_k, and the spectrum.  The kept triplets carry the
// cotangents, the discarded ones none; the exact derivative is the thin-SVD
// backward over the kept triplets and every discarded triplet whose value is
// above `retain` times the smallest kept one and above theta's rounding
// floor (the rest act as an exact null space, an O((s_j / s_i)^2)
// approximation that also avoids dividing by vanishing singular values):
//   X_bar = U G' V^H + [U_bar S^-1 | 0] V^H + U_K S_K^-1 V_bar^H
//   G'_ij = s_j F_ij (P - P^H)_ij + s_i F_ij (Q - Q^H)_ij
//           - [j < K] P_ij / s_j - [i < K] conj(Q_ji) / s_i          (i != j)
//   G'_ii = S_bar_i + i (Im P_ii - Im Q_ii) / (2 s_i) - P_ii / s_i - conj(Q_ii) / s_i
//   P = U^H U_bar, Q = V^H V_bar,
//   F_ij = (s_j^2 - s_i^2) / ((s_j^2 - s_i^2)^2 + (b s_0^2)^2)     (Lorentzian-broadened)
// The cotangents of the sqrt(S) split and of the kept-norm renormalisation
// give U_bar, V_bar and S_bar; then theta_bar = G^H M_bar, A_bar = theta_bar
// B^H and B_bar = A^H theta_bar.  All matrices of one pair live in a
// per-CTA global scratch (L2-resident at these sizes) and are combined by a
// 64 x 64 tiled complex FP64 GEMM run by the whole CTA.
#include "mpsb_common.cuh"
#include "cta_gemm.cuh"

#include <algorithm>
#include <climits>

namespace mpsb {

constexpr int kBwdThreads = kCtaGemmThreads;

// ------------------------------------------------------------------ two-site
struct BwdParams {
    const mpsb_chain *pre;   // pre-update state: sites A, B and the bonds
    const mpsb_chain *cot;   // cotangent slots (same slot layout), updated in place
    const mpsb_pair *pairs;
    int npairs;
    const double2 *gates;
    const double2 *tape;
    long long tape_stride;
    double2 *gate_grads;     // optional: 16 per pair (index pr.out)
    double2 *ws;
    long long ws_stride;
    int32_t *status;
    int chi_cap;
    double retain;
    double broaden;
    int pqg_in_smem;         // P, Q and G' in dynamic shared memory (chi_cap <= 32) instead of the scratch
};

// The per-pair scratch is dead once a pair is done: drop its lines from L2
// without writing them back (the next pair writes every element before it
// reads it).  Without this, the tapes streaming through L2 evicted the dirty
// scratch to DRAM -- most of the backward's DRAM writes.
__device__ __forceinline__ void discard_l2(const double2 *base, size_t n_elems, int tid, int nthreads) {
    const char *b = reinterpret_cast<const char *>(base);
    const size_t lines = n_elems * sizeof(double2) / 128;
    for (size_t l = tid; l < lines; l += nthreads)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(b + l * 128) : "memory");
}

// Tape elements are read once per backward: streaming loads (evict first).
__device__ __forceinline__ double2 ld_tape(const double2 *p) { return __ldcs(p); }

// One pair; every early exit is block-uniform.  `base` is this CTA's scratch.
__device__ __forceinline__ void backward_pair(const BwdParams &p, const int pi, double2 *base) {
    __shared__ GemmSmem sm;
    __shared__ double sS[128], sSb[128];
    __shared__ int s_rp, s_bad;
    __shared__ double2 s_gate[16];
    __shared__ double2 s_red[kBwdThreads / 32][16];
    const int tid = threadIdx.x;
    const mpsb_pair pr = p.pairs[pi];
    const mpsb_chain ch = p.pre[pr.chain];
    const mpsb_chain cc = p.cot[pr.chain];
    const int site = pr.site;
    const long long Qn = (long long)(2 * p.chi_cap) * (2 * p.chi_cap);
    const double2 *X = p.tape + (size_t)pi * p.tape_stride;
    const double2 *Xs = X + Qn;
    const double *meta = reinterpret_cast<const double *>(X + 2 * Qn);

    int cl = 0, cm = 0, cr = 0;
    bool bad = site < 0 || site + 2 > ch.n;
    if (!bad) {
        cl = ch.bonds[site];
        cm = ch.bonds[site + 1];
        cr = ch.bonds[site + 2];
        bad = cl < 1 || cm < 1 || cr < 1 || cl > p.chi_cap || cm > p.chi_cap || cr > p.chi_cap;
    }
    const bool trans = cr > cl;
    const int R = trans ? 2 * cr : 2 * cl;
    const int C = trans ? 2 * cl : 2 * cr;
    const int K = bad ? 0 : (int)meta[kTapeMetaKeep];
    if (!bad)
        bad = (int)meta[kTapeMetaRows] != R || (int)meta[kTapeMetaCols] != C || K < 1 || K > C ||
              K > ch.chi_max;
    if (bad) {
        if (tid == 0) p.status[pr.out] = MPSB_ST_BADDIM;
        return;
    }
    const double div = meta[kTapeMetaDiv];
    for (int j = tid; j < 128; j += kBwdThreads) sS[j] = j < C ? meta[j] : 0.0;
    if (tid < 16) s_gate[tid] = p.gates[(size_t)pr.gate * 16 + tid];
    __syncthreads();
    if (tid == 0) {
        int rp = K;
        // discarded triplets below the rounding floor of theta (~64 eps S_0) carry
        // no accurate vectors: they join the null space with the rest
        const double thr = fmax(p.retain * sS[K - 1], 1.5e-14 * sS[0]);
        while (rp < C && sS[rp] > thr && sS[rp] > 0.0) ++rp;
        s_rp = rp;
        s_bad = !(sS[K - 1] > 0.0) || !(div > 0.0);
    }
    __syncthreads();
    const int rp = s_rp;
    double2 *Acot = reinterpret_cast<double2 *>(cc.sites + (size_t)site * cc.slot_elems);
    double2 *Bcot = reinterpret_cast<double2 *>(cc.sites + (size_t)(site + 1) * cc.slot_elems);
    if (s_bad) {  // all-zero theta: no direction to differentiate along
        for (int e = tid; e < 2 * cl * cm; e += kBwdThreads) Acot[e] = make_double2(0.0, 0.0);
        for (int e = tid; e < 2 * cm * cr; e += kBwdThreads) Bcot[e] = make_double2(0.0, 0.0);
        if (tid == 0) p.status[pr.out] = MPSB_ST_NONFINITE;
        return;
    }
    const double2 *Asite = reinterpret_cast<const double2 *>(ch.sites + (size_t)site * ch.slot_elems);
    const double2 *Bsite = reinterpret_cast<const double2 *>(ch.sites + (size_t)(site + 1) * ch.slot_elems);

    extern __shared__ __align__(16) double2 bwd_dyn[];
    double2 *U = base;                       // R x rp
    double2 *V = base + Qn;                  // C x rp
    double2 *Ub = base + 2 * Qn;             // R x K
    double2 *Vb = base + 2 * Qn + Qn / 2;    // C x K
    double2 *const pqg = p.pqg_in_smem ? bwd_dyn : base + 3 * Qn;
    double2 *Pm = pqg;                       // rp x K
    double2 *Qm = pqg + Qn / 2;              // rp x K
    double2 *Gm = pqg + Qn;                  // rp x rp
    double2 *T = base + 5 * Qn;              // R x rp
    double2 *Mb = base + 6 * Qn;             // 2cl x 2cr
    double2 *Th = base + 7 * Qn;             // 2cl x 2cr (gate cotangent only)

    // 1. cotangents of the kept factors (split: A' = U_M sqrt(s), B' = sqrt(s) V_M^H), X frame
    {
        const int twocl = 2 * cl, twocr = 2 * cr;
        double2 *dA = trans ? Vb : Ub;
        double2 *dB = trans ? Ub : Vb;
        for (int e = tid; e < twocl * K; e += kBwdThreads) {
            const int k = e % K;
            dA[e] = c_scale(Acot[e], sqrt(sS[k] / div));
        }
        for (int e = tid; e < twocr * K; e += kBwdThreads) {
            const int col = e / K, k = e - col * K;
            dB[e] = c_scale(c_conj(Bcot[(size_t)k * twocr + col]), sqrt(sS[k] / div));
        }
    }
    if (meta[kTapeMetaSide] != 0.0) {
        // 2'. V = Vs / S (the QR-preconditioned forward taped the right side)
        for (int e = tid; e < C * rp; e += kBwdThreads) {
            const int i = e / rp, j = e - i * rp;
            V[e] = c_scale(ld_tape(Xs + (size_t)j * C + i), 1.0 / sS[j]);
        }
        __syncthreads();
        // 3'. U = X V S^-1   (R x rp)
        cta_cgemm<true, true>(
            R, rp, C, [&](int r, int k) { return ld_tape(X + (size_t)r * C + k); },
            [&](int k, int j) { return V[(size_t)k * rp + j]; },
            [&](int r, int j, double2 v) { U[(size_t)r * rp + j] = c_scale(v, 1.0 / sS[j]); }, sm);
    } else {
        // 2. U = Xs / S
        for (int e = tid; e < R * rp; e += kBwdThreads) {
            const int r = e / rp, j = e - r * rp;
            U[e] = c_scale(ld_tape(Xs + (size_t)j * R + r), 1.0 / sS[j]);
        }
        __syncthreads();
        // 3. V = X^H U S^-1   (C x rp)
        cta_cgemm<false, true>(
            C, rp, R, [&](int i, int k) { return c_conj(ld_tape(X + (size_t)k * C + i)); },
            [&](int k, int j) { return U[(size_t)k * rp + j]; },
            [&](int i, int j, double2 v) { V[(size_t)i * rp + j] = c_scale(v, 1.0 / sS[j]); }, sm);
    }
    // 4. P = U^H U_bar, Q = V^H V_bar   (rp x K)
    cta_cgemm<false, true>(
        rp, K, R, [&](int i, int k) { return c_conj(U[(size_t)k * rp + i]); },
        [&](int k, int j) { return Ub[(size_t)k * K + j]; },
        [&](int i, int j, double2 v) { Pm[(size_t)i * K + j] = v; }, sm);
    cta_cgemm<false, true>(
        rp, K, C, [&](int i, int k) { return c_conj(V[(size_t)k * rp + i]); },
        [&](int k, int j) { return Vb[(size_t)k * K + j]; },
        [&](int i, int j, double2 v) { Qm[(size_t)i * K + j] = v; }, sm);
    // 5. S_bar from s_bar (split) through the kept-norm renormalisation s = S / div
    if (tid == 0) {
        double dot = 0.0;
        for (int k = 0; k < K; ++k) {
            const double s = sS[k] / div;
            const double sb = (Pm[(size_t)k * K + k].x + Qm[(size_t)k * K + k].x) / (2.0 * s);
            sSb[k] = sb;
            dot = fma(s, sb, dot);
        }
        for (int k = 0; k < K; ++k) sSb[k] = (sSb[k] - (sS[k] / div) * dot) / div;
    }
    __syncthreads();
    // 6. G' (rp x rp)
    {
        const double eps = (p.broaden * sS[0] * sS[0]) * (p.broaden * sS[0] * sS[0]);
        for (int e = tid; e < rp * rp; e += kBwdThreads) {
            const int i = e / rp, j = e - i * rp;
            const double2 zero = make_double2(0.0, 0.0);
            const double2 pij = j < K ? Pm[(size_t)i * K + j] : zero;
            const double2 qij = j < K ? Qm[(size_t)i * K + j] : zero;
            const double2 pji = i < K ? Pm[(size_t)j * K + i] : zero;
            const double2 qji = i < K ? Qm[(size_t)j * K + i] : zero;
            double2 g = zero;
            if (i != j) {
                const double dd = sS[j] * sS[j] - sS[i] * sS[i];
                const double F = dd / fma(dd, dd, eps);
                g = c_add(c_scale(c_sub(pij, c_conj(pji)), sS[j] * F), c_scale(c_sub(qij, c_conj(qji)), sS[i] * F));
            } else if (i < K) {
                g = make_double2(sSb[i], 0.5 * (pij.y - qij.y) / sS[i]);
            }
            if (j < K) g = c_sub(g, c_scale(pij, 1.0 / sS[j]));
            if (i < K) g = c_sub(g, c_scale(c_conj(qji), 1.0 / sS[i]));
            Gm[e] = g;
        }
    }
    __syncthreads();
    // 7. T = U G' + [U_bar S^-1 | 0]   (R x rp)
    cta_cgemm<true, true>(
        R, rp, rp, [&](int i, int k) { return U[(size_t)i * rp + k]; },
        [&](int k, int j) { return Gm[(size_t)k * rp + j]; },
        [&](int i, int j, double2 v) {
            if (j < K) v = c_add(v, c_scale(Ub[(size_t)i * K + j], 1.0 / sS[j]));
            T[(size_t)i * rp + j] = v;
        },
        sm);
    // 8. X_bar = T V^H + U_K S_K^-1 V_bar^H, stored as M_bar (theta frame)
    {
        const int twocr = 2 * cr;
        cta_cgemm<true, false>(
            R, C, rp + K,
            [&](int i, int k) {
                return k < rp ? T[(size_t)i * rp + k] : c_scale(U[(size_t)i * rp + (k - rp)], 1.0 / sS[k - rp]);
            },
            [&](int k, int j) { return k < rp ? c_conj(V[(size_t)j * rp + k]) : c_conj(Vb[(size_t)j * K + (k - rp)]); },
            [&](int i, int j, double2 v) {
                if (!trans)
                    Mb[(size_t)i * twocr + j] = v;
                else
                    Mb[(size_t)j * twocr + i] = c_conj(v);
            },
            sm);
    }
    // 9. gate: theta_bar = G^H theta'_bar; optional G_bar = theta'_bar theta^H
    const bool want_gate = p.gate_grads != nullptr;
    if (want_gate) {
        cta_cgemm<true, true>(
            2 * cl, 2 * cr, cm, [&](int i, int k) { return Asite[(size_t)i * cm + k]; },
            [&](int k, int j) { return Bsite[(size_t)k * 2 * cr + j]; },
            [&](int i, int j, double2 v) { Th[(size_t)i * 2 * cr + j] = v; }, sm);
    }
    {
        double2 gpart[16];
#pragma unroll
        for (int q = 0; q < 16; ++q) gpart[q] = make_double2(0.0, 0.0);
        for (int e = tid; e < cl * cr; e += kBwdThreads) {
            const int a = e / cr, c = e - a * cr;
            double2 tp[4], th[4];
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                const size_t idx = (size_t)(2 * a + (t >> 1)) * 2 * cr + (size_t)(t & 1) * cr + c;
                tp[t] = Mb[idx];
                if (want_gate) th[t] = Th[idx];
            }
            if (want_gate) {
#pragma unroll
                for (int t = 0; t < 4; ++t)
#pragma unroll
                    for (int s = 0; s < 4; ++s) gpart[t * 4 + s] = c_fma(tp[t], c_conj(th[s]), gpart[t * 4 + s]);
            }
#pragma unroll
            for (int s = 0; s < 4; ++s) {
                double2 acc = make_double2(0.0, 0.0);
#pragma unroll
                for (int t = 0; t < 4; ++t) acc = c_cfma(s_gate[t * 4 + s], tp[t], acc);
                Mb[(size_t)(2 * a + (s >> 1)) * 2 * cr + (size_t)(s & 1) * cr + c] = acc;
            }
        }
        if (want_gate) {
            const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                double2 v = gpart[q];
                v.x = warp_sum(v.x);
                v.y = warp_sum(v.y);
                if (lane == 0) s_red[warp][q] = v;
            }
            __syncthreads();
            if (tid < 16) {
                double2 v = make_double2(0.0, 0.0);
                for (int w = 0; w < kBwdThreads / 32; ++w) v = c_add(v, s_red[w][tid]);
                p.gate_grads[(size_t)pr.out * 16 + tid] = v;
            }
        }
    }
    __syncthreads();
    // 10. A_bar = theta_bar B^H (2cl x cm), B_bar = A^H theta_bar (cm x 2cr)
    {
        const int twocr = 2 * cr;
        cta_cgemm<true, false>(
            2 * cl, cm, twocr, [&](int i, int k) { return Mb[(size_t)i * twocr + k]; },
            [&](int k, int j) { return c_conj(Bsite[(size_t)j * twocr + k]); },
            [&](int i, int j, double2 v) { Acot[(size_t)i * cm + j] = v; }, sm);
        cta_cgemm<false, true>(
            cm, twocr, 2 * cl, [&](int i, int k) { return c_conj(Asite[(size_t)k * cm + i]); },
            [&](int k, int j) { return Mb[(size_t)k * twocr + j]; },
            [&](int i, int j, double2 v) { Bcot[(size_t)i * twocr + j] = v; }, sm);
    }
    __syncthreads();
    discard_l2(base, (size_t)8 * Qn, tid, kBwdThreads);
    if (tid == 0) p.status[pr.out] = 0;
}

// Persistent grid (one CTA per SM at most): a CTA walks pairs blockIdx.x,
// blockIdx.x + gridDim.x, ... and reuses ONE scratch region, so the live
// scratch is gridDim.x regions (L2-resident) instead of one per pair.
__global__ void __launch_bounds__(kBwdThreads, 1) update2q_backward_kernel(const BwdParams p) {
    double2 *base = p.ws + (size_t)blockIdx.x * p.ws_stride;
    for (int pi = blockIdx.x; pi < p.npairs; pi += gridDim.x) {
        backward_pair(p, pi, base);
        __syncthreads();  // shared tiles and scratch are reused by the next pair
    }
}

// ------------------------------------------------------------------ one-site
// A' = G A on the physical index: A_bar = G^H A'_bar (in place), G_bar = sum A'_bar A^H.
__global__ void __launch_bounds__(128) apply1q_backward_kernel(const mpsb_chain *pre, const mpsb_chain *cot,
                                                               const mpsb_site_op *ops, int nops, const double2 *gates,
                                                               double2 *gate_grads) {
    __shared__ double2 red[4][4];
    const int q = blockIdx.x, tid = threadIdx.x;
    if (q >= nops) return;
    const mpsb_site_op op = ops[q];
    const mpsb_chain ch = pre[op.chain], cc = cot[op.chain];
    const int cl = ch.bonds[op.site], cr = ch.bonds[op.site + 1];
    const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)op.site * ch.slot_elems);
    double2 *Ab = reinterpret_cast<double2 *>(cc.sites + (size_t)op.site * cc.slot_elems);
    double2 g[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) g[e] = gates[(size_t)op.gate * 4 + e];
    double2 part[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int e = tid; e < cl * cr; e += blockDim.x) {
        const int l = e / cr, r = e - l * cr;
        const size_t i0 = (size_t)l * 2 * cr + r, i1 = i0 + cr;
        const double2 b0 = Ab[i0], b1 = Ab[i1];
        const double2 a0 = A[i0], a1 = A[i1];
        part[0] = c_fma(b0, c_conj(a0), part[0]);
        part[1] = c_fma(b0, c_conj(a1), part[1]);
        part[2] = c_fma(b1, c_conj(a0), part[2]);
        part[3] = c_fma(b1, c_conj(a1), part[3]);
        // A_bar[s] = sum_t conj(G[t, s]) A'_bar[t]
        Ab[i0] = c_cfma(g[2], b1, c_cfma(g[0], b0, make_double2(0, 0)));
        Ab[i1] = c_cfma(g[3], b1, c_cfma(g[1], b0, make_double2(0, 0)));
    }
    if (gate_grads) {
        const int lane = tid & 31, warp = tid >> 5;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            double2 v = part[e];
            v.x = warp_sum(v.x);
            v.y = warp_sum(v.y);
            if (lane == 0) red[warp][e] = v;
        }
        __syncthreads();
        if (tid < 4) {
            double2 v = make_double2(0, 0);
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = c_add(v, red[w][tid]);
            gate_grads[(size_t)q * 4 + tid] = v;
        }
    }
}

// ------------------------------------------------------------------ MPO energy
// Environments of <psi|H|psi> for an MPO W (n sites, bond D, W[k][a][b][s][t]
// acting as |s><t|) whose state D-1 is the left boundary ("nothing placed")
// and state 0 the right boundary ("complete"), with W[k][D-1][D-1] = W[k][0][0]
// = identity, so that the D-1 component of a left environment and the 0
// component of a right one are the plain norm environments.  Each
// environment is rescaled by the trace of its norm component as it is built;
// every quantity formed from one left and one right environment is then a
// ratio in which the scales cancel.
struct EnvParams {
    const mpsb_chain *chains;
    int nchains, n, chi_cap, D;
    const double2 *mpo;       // n * D * D * 4
    double2 *L, *R;           // per chain (n + 1) * D * chi_cap^2
    double2 *scratch;         // per CTA: 2 * D * 2 chi_cap^2
    long long env_stride, scratch_stride;
};

__device__ __forceinline__ double2 W_at(const EnvParams &p, int k, int a, int b, int s, int t) {
    return p.mpo[((((size_t)k * p.D + a) * p.D + b) * 2 + s) * 2 + t];
}

// blockIdx.x = chain * 2 + direction (0 = left sweep, 1 = right sweep)
__global__ void __launch_bounds__(kBwdThreads, 1) mpo_env_kernel(const EnvParams p) {
    __shared__ GemmSmem sm;
    __shared__ double s_tr;
    const int c = blockIdx.x >> 1, dir = blockIdx.x & 1, tid = threadIdx.x;
    const mpsb_chain ch = p.chains[c];
    const int D = p.D, n = p.n;
    const long long Q1 = (long long)p.chi_cap * p.chi_cap;
    double2 *envs = (dir == 0 ? p.L : p.R) + (size_t)c * p.env_stride;
    double2 *T1 = p.scratch + (size_t)blockIdx.x * p.scratch_stride;
    double2 *T2 = T1 + (size_t)D * 2 * Q1;
    if (dir == 0) {
        for (int a = tid; a < D; a += kBwdThreads) envs[(size_t)a * Q1] = make_double2(a == D - 1 ? 1.0 : 0.0, 0.0);
        __syncthreads();
        for (int k = 0; k < n; ++k) {
            const int xk = ch.bonds[k], xk1 = ch.bonds[k + 1];
            const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems);
            const double2 *Lk = envs + (size_t)k * D * Q1;
            double2 *Lk1 = envs + (size_t)(k + 1) * D * Q1;
            // T1[(a, x)][(t, v)] = sum_y L[a][x][y] A[y][(t, v)]
            cta_cgemm<true, true>(
                D * xk, 2 * xk1, xk,
                [&](int i, int kk) { return Lk[(size_t)(i / xk) * Q1 + (size_t)(i % xk) * xk + kk]; },
                [&](int kk, int j) { return A[(size_t)kk * 2 * xk1 + j]; },
                [&](int i, int j, double2 v) { T1[(size_t)i * 2 * xk1 + j] = v; }, sm);
            // T2[(b, x)][(s, v)] = sum_{a, t} W[a][b][s][t] T1[(a, x)][(t, v)]
            for (int e = tid; e < D * xk * 2 * xk1; e += kBwdThreads) {
                const int b = e / (xk * 2 * xk1), rem = e - b * (xk * 2 * xk1);
                const int x = rem / (2 * xk1), sv = rem - x * 2 * xk1, s = sv / xk1, v = sv - s * xk1;
                double2 acc = make_double2(0.0, 0.0);
                for (int a = 0; a < D; ++a)
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const double2 w = W_at(p, k, a, b, s, t);
                        if (w.x != 0.0 || w.y != 0.0)
                            acc = c_fma(w, T1[((size_t)a * xk + x) * 2 * xk1 + (size_t)t * xk1 + v], acc);
                    }
                T2[e] = acc;
            }
            __syncthreads();
            // L'[b][u][v] = sum_{(x, s)} conj(A[(x, s)][u]) T2[b][(x, s)][v]
            for (int b = 0; b < D; ++b) {
                const double2 *T2b = T2 + (size_t)b * xk * 2 * xk1;
                double2 *Lb = Lk1 + (size_t)b * Q1;
                cta_cgemm<false, true>(
                    xk1, xk1, 2 * xk, [&](int i, int kk) { return c_conj(A[(size_t)kk * xk1 + i]); },
                    [&](int kk, int j) { return T2b[(size_t)kk * xk1 + j]; },
                    [&](int i, int j, double2 v) { Lb[(size_t)i * xk1 + j] = v; }, sm);
            }
            if (tid == 0) {
                double tr = 0.0;
                const double2 *Ln = Lk1 + (size_t)(D - 1) * Q1;
                for (int u = 0; u < xk1; ++u) tr += Ln[(size_t)u * xk1 + u].x;
                s_tr = tr > 0.0 ? 1.0 / tr : 1.0;
            }
            __syncthreads();
            const double sc = s_tr;
            for (int b = 0; b < D; ++b)
                for (int e = tid; e < xk1 * xk1; e += kBwdThreads) {
                    double2 *q = Lk1 + (size_t)b * Q1 + e;
                    *q = c_scale(*q, sc);
                }
            __syncthreads();
        }
    } else {
        double2 *Rn = envs + (size_t)n * D * Q1;
        for (int a = tid; a < D; a += kBwdThreads) Rn[(size_t)a * Q1] = make_double2(a == 0 ? 1.0 : 0.0, 0.0);
        __syncthreads();
        for (int k = n - 1; k >= 0; --k) {
            const int xk = ch.bonds[k], xk1 = ch.bonds[k + 1];
            const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems);
            const double2 *Rk1 = envs + (size_t)(k + 1) * D * Q1;
            double2 *Rk = envs + (size_t)k * D * Q1;
            // T1[b][(y, t)][u] = sum_v A[(y, t)][v] R'[b][u][v]
            for (int b = 0; b < D; ++b) {
                const double2 *Rb = Rk1 + (size_t)b * Q1;
                double2 *T1b = T1 + (size_t)b * 2 * xk * xk1;
                cta_cgemm<true, false>(
                    2 * xk, xk1, xk1, [&](int i, int kk) { return A[(size_t)i * xk1 + kk]; },
                    [&](int kk, int j) { return Rb[(size_t)j * xk1 + kk]; },
                    [&](int i, int j, double2 v) { T1b[(size_t)i * xk1 + j] = v; }, sm);
            }
            // T2[a][(y, s)][u] = sum_{b, t} W[a][b][s][t] T1[b][(y, t)][u]
            for (int e = tid; e < D * 2 * xk * xk1; e += kBwdThreads) {
                const int a = e / (2 * xk * xk1), rem = e - a * (2 * xk * xk1);
                const int ys = rem / xk1, u = rem - ys * xk1, y = ys >> 1, s = ys & 1;
                double2 acc = make_double2(0.0, 0.0);
                for (int b = 0; b < D; ++b)
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const double2 w = W_at(p, k, a, b, s, t);
                        if (w.x != 0.0 || w.y != 0.0)
                            acc = c_fma(w, T1[(size_t)b * 2 * xk * xk1 + (size_t)(2 * y + t) * xk1 + u], acc);
                    }
                T2[e] = acc;
            }
            __syncthreads();
            // R[a][x][y] = sum_{(s, u)} conj(A[x][(s, u)]) T2[a][(y, s)][u]
            for (int a = 0; a < D; ++a) {
                const double2 *T2a = T2 + (size_t)a * 2 * xk * xk1;
                double2 *Ra = Rk + (size_t)a * Q1;
                cta_cgemm<true, false>(
                    xk, xk, 2 * xk1, [&](int i, int kk) { return c_conj(A[(size_t)i * 2 * xk1 + kk]); },
                    [&](int kk, int j) { return T2a[(size_t)j * 2 * xk1 + kk]; },
                    [&](int i, int j, double2 v) { Ra[(size_t)i * xk + j] = v; }, sm);
            }
            if (tid == 0) {
                double tr = 0.0;
                for (int u = 0; u < xk; ++u) tr += Rk[(size_t)u * xk + u].x;
                s_tr = tr > 0.0 ? 1.0 / tr : 1.0;
            }
            __syncthreads();
            const double sc = s_tr;
            for (int a = 0; a < D; ++a)
                for (int e = tid; e < xk * xk; e += kBwdThreads) {
                    double2 *q = Rk + (size_t)a * Q1 + e;
                    *q = c_scale(*q, sc);
                }
            __syncthreads();
        }
    }
}

struct GradParams {
    EnvParams e;
    const mpsb_chain *cot;
    const double *weights;
    double *loss;
    double2 *scratch;          // per (chain, site) CTA
    long long scratch_stride;
};

// One CTA per (chain, site): cotangent 2 w (H_eff A - L N_eff A) / <A, N_eff A>,
// with L = <H> / <1> from the completed left environment.
__global__ void __launch_bounds__(kBwdThreads, 1) mpo_grad_kernel(const GradParams g) {
    __shared__ GemmSmem sm;
    __shared__ double s_part[kBwdThreads / 32];
    const EnvParams &p = g.e;
    const int c = blockIdx.x / p.n, k = blockIdx.x - c * p.n, tid = threadIdx.x;
    const mpsb_chain ch = p.chains[c];
    const int D = p.D;
    const long long Q1 = (long long)p.chi_cap * p.chi_cap;
    const int xk = ch.bonds[k], xk1 = ch.bonds[k + 1];
    const double2 *Lk = p.L + (size_t)c * p.env_stride + (size_t)k * D * Q1;
    const double2 *Rk1 = p.R + (size_t)c * p.env_stride + (size_t)(k + 1) * D * Q1;
    const double2 *Lend = p.L + (size_t)c * p.env_stride + (size_t)p.n * D * Q1;
    const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems);
    double2 *out = reinterpret_cast<double2 *>(g.cot[c].sites + (size_t)k * g.cot[c].slot_elems);
    double2 *T1 = g.scratch + (size_t)blockIdx.x * g.scratch_stride;
    double2 *T2 = T1 + (size_t)D * 2 * Q1;
    double2 *HA = T2 + (size_t)D * 2 * Q1;
    double2 *NA = HA + 2 * Q1;
    const double energy = Lend[0].x / Lend[(size_t)(D - 1) * Q1].x;
    if (k == 0 && tid == 0 && g.loss) g.loss[c] = energy;
    cta_cgemm<true, true>(
        D * xk, 2 * xk1, xk, [&](int i, int kk) { return Lk[(size_t)(i / xk) * Q1 + (size_t)(i % xk) * xk + kk]; },
        [&](int kk, int j) { return A[(size_t)kk * 2 * xk1 + j]; },
        [&](int i, int j, double2 v) { T1[(size_t)i * 2 * xk1 + j] = v; }, sm);
    for (int e = tid; e < D * xk * 2 * xk1; e += kBwdThreads) {
        const int b = e / (xk * 2 * xk1), rem = e - b * (xk * 2 * xk1);
        const int x = rem / (2 * xk1), sv = rem - x * 2 * xk1, s = sv / xk1, v = sv - s * xk1;
        double2 acc = make_double2(0.0, 0.0);
        for (int a = 0; a < D; ++a)
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                const double2 w = W_at(p, k, a, b, s, t);
                if (w.x != 0.0 || w.y != 0.0)
                    acc = c_fma(w, T1[((size_t)a * xk + x) * 2 * xk1 + (size_t)t * xk1 + v], acc);
            }
        T2[e] = acc;
    }
    __syncthreads();
    // HA[(x, s)][u] = sum_{(b, v)} T2[b][x][(s, v)] R[b][u][v]
    cta_cgemm<true, false>(
        2 * xk, xk1, D * xk1,
        [&](int i, int kk) {
            const int b = kk / xk1, v = kk - b * xk1;
            return T2[(size_t)b * xk * 2 * xk1 + (size_t)(i >> 1) * 2 * xk1 + (size_t)(i & 1) * xk1 + v];
        },
        [&](int kk, int j) {
            const int b = kk / xk1, v = kk - b * xk1;
            return Rk1[(size_t)b * Q1 + (size_t)j * xk1 + v];
        },
        [&](int i, int j, double2 v) { HA[(size_t)i * xk1 + j] = v; }, sm);
    // NA[(x, s)][u] = sum_v T1[D-1][x][(s, v)] R[0][u][v]
    cta_cgemm<true, false>(
        2 * xk, xk1, xk1,
        [&](int i, int kk) {
            return T1[((size_t)(D - 1) * xk + (i >> 1)) * 2 * xk1 + (size_t)(i & 1) * xk1 + kk];
        },
        [&](int kk, int j) { return Rk1[(size_t)j * xk1 + kk]; },
        [&](int i, int j, double2 v) { NA[(size_t)i * xk1 + j] = v; }, sm);
    // <A, N_eff A>
    double part = 0.0;
    for (int e = tid; e < 2 * xk * xk1; e += kBwdThreads) part += c_cfma(A[e], NA[e], make_double2(0, 0)).x;
    part = warp_sum(part);
    if ((tid & 31) == 0) s_part[tid >> 5] = part;
    __syncthreads();
    double nk = 0.0;
    for (int w = 0; w < kBwdThreads / 32; ++w) nk += s_part[w];
    const double wgt = g.weights ? g.weights[c] : 1.0;
    const double f = nk != 0.0 ? 2.0 * wgt / nk : 0.0;
    for (int e = tid; e < 2 * xk * xk1; e += kBwdThreads)
        out[e] = c_scale(c_sub(HA[e], c_scale(NA[e], energy)), f);
}

// ------------------------------------------------------------------ host
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// CTAs of the persistent backward grid: every resident CTA on the device
// (no cap while no device answers the query).
static int bwd_grid_cap() {
    static int cap = 0;
    if (cap == 0) {
        int dev = 0, sms = 0, per_sm = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, update2q_backward_kernel, kBwdThreads, 0) !=
                cudaSuccess ||
            sms < 1 || per_sm < 1) {
            cudaGetLastError();
            return INT_MAX;
        }
        cap = sms * per_sm;
    }
    return cap;
}

size_t bwd_workspace_bytes(int npairs, int chi_cap) {
    const size_t q = (size_t)(2 * chi_cap) * (2 * chi_cap);
    return (size_t)std::min(npairs, bwd_grid_cap()) * 8 * q * sizeof(double2);
}

int launch_update2q_backward(const mpsb_chain *pre, const mpsb_chain *cot, const mpsb_pair *pairs, int npairs,
                             const double2 *gates, int chi_cap, const void *tape, double2 *gate_grads, void *ws,
                             int32_t *status, double retain, double broaden, cudaStream_t s) {
    if (npairs == 0) return MPSB_OK;
    BwdParams p;
    p.pre = pre;
    p.cot = cot;
    p.pairs = pairs;
    p.npairs = npairs;
    p.gates = gates;
    p.tape = reinterpret_cast<const double2 *>(tape);
    p.tape_stride = tape_stride(chi_cap);
    p.gate_grads = gate_grads;
    p.ws = reinterpret_cast<double2 *>(ws);
    p.ws_stride = 8LL * (2 * chi_cap) * (2 * chi_cap);
    p.status = status;
    p.chi_cap = chi_cap;
    p.retain = retain;
    p.broaden = broaden;
    // P, Q (rp x K each, <= Q/2) and G' (rp x rp, <= Q) fit in shared memory up to chi_cap = 32
    p.pqg_in_smem = chi_cap <= 32 ? 1 : 0;
    const size_t dyn = p.pqg_in_smem ? (size_t)2 * (2 * chi_cap) * (2 * chi_cap) * sizeof(double2) : 0;
    const int rc = ensure_smem(reinterpret_cast<const void *>(update2q_backward_kernel), dyn,
                               "cudaFuncSetAttribute(update2q_backward)");
    if (rc) return rc;
    update2q_backward_kernel<<<std::min(npairs, bwd_grid_cap()), kBwdThreads, dyn, s>>>(p);
    return check_launch("update2q_backward_kernel");
}

int launch_apply1q_backward(const mpsb_chain *pre, const mpsb_chain *cot, const mpsb_site_op *ops, int nops,
                            const double2 *gates, double2 *gate_grads, cudaStream_t s) {
    if (nops == 0) return MPSB_OK;
    apply1q_backward_kernel<<<nops, 128, 0, s>>>(pre, cot, ops, nops, gates, gate_grads);
    return check_launch("apply1q_backward_kernel");
}

static void mpo_layout(int nchains, int n, int chi_cap, int D, size_t *env_bytes, size_t *env_scr, size_t *grad_scr) {
    const size_t q1 = (size_t)chi_cap * chi_cap;
    *env_bytes = align256((size_t)nchains * (n + 1) * D * q1 * sizeof(double2));
    *env_scr = align256((size_t)nchains * 2 * (2 * D * 2 * q1) * sizeof(double2));
    *grad_scr = (size_t)nchains * n * (2 * D * 2 * q1 + 4 * q1) * sizeof(double2);
}

size_t mpo_grad_workspace_bytes(int nchains, int n, int chi_cap, int D) {
    size_t eb, es, gs;
    mpo_layout(nchains, n, chi_cap, D, &eb, &es, &gs);
    return 2 * eb + es + gs;
}

int launch_mpo_energy_grad(const mpsb_chain *chains, int nchains, int n, int chi_cap, const double2 *mpo, int D,
                           const double *weights, double *loss, const mpsb_chain *cot, void *ws, cudaStream_t s) {
    size_t eb, es, gs;
    mpo_layout(nchains, n, chi_cap, D, &eb, &es, &gs);
    const size_t q1 = (size_t)chi_cap * chi_cap;
    EnvParams e;
    e.chains = chains;
    e.nchains = nchains;
    e.n = n;
    e.chi_cap = chi_cap;
    e.D = D;
    e.mpo = mpo;
    char *b = static_cast<char *>(ws);
    e.L = reinterpret_cast<double2 *>(b);
    e.R = reinterpret_cast<double2 *>(b + eb);
    e.scratch = reinterpret_cast<double2 *>(b + 2 * eb);
    e.env_stride = (long long)(n + 1) * D * q1;
    e.scratch_stride = 2LL * D * 2 * q1;
    mpo_env_kernel<<<2 * nchains, kBwdThreads, 0, s>>>(e);
    int rc = check_launch("mpo_env_kernel");
    if (rc) return rc;
    GradParams g;
    g.e = e;
    g.cot = cot;
    g.weights = weights;
    g.loss = loss;
    g.scratch = reinterpret_cast<double2 *>(b + 2 * eb + es);
    g.scratch_stride = 2LL * D * 2 * q1 + 4 * q1;
    mpo_grad_kernel<<<nchains * n, kBwdThreads, 0, s>>>(g);
    return check_launch("mpo_grad_kernel");
}

}  // namespace mpsb
