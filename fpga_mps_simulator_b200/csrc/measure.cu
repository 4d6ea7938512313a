// Measurement on device-resident chains: conditional shot sampling and the
// site reset of the reference's execution engine.  sm_100a only.
//
// Sampling follows MPSState.sample (mps_core.py:354-419): right environments
// R[i] = sum_s A[s] R[i+1] A[s]^H, each divided by its trace (when > 1e-300),
// then per shot a left-to-right sweep with the row vector v (v = [1] at the
// left boundary): w_s = v A[:, s, :], p_s = Re(w_s R[i+1] w_s^H), clipped at 0,
// normalised (0.5 / 0.5 when the total is below 1e-15), outcome drawn, v =
// w_outcome / |w_outcome| when that norm exceeds 1e-15.  The draw consumes one
// caller-supplied uniform u per (shot, site): outcome = 1 exactly when
// u >= p_0 / (p_0 + p_1), which is how numpy's Generator.choice(2, p=...)
// (the reference's draw) turns its one uniform into an index (normalised
// cumulative sum, searchsorted side='right').  Given the uniforms of the same
// seeded generator the shots therefore match the reference's, up to
// decisions within rounding of a threshold.
//
// Reset follows the 'reset' branch of _run_circuit_fpga
// (fpga_mps_simulator.py:530-552): zero the sigma = 1 half of the site tensor,
// divide by the Frobenius norm of what is left when it exceeds 1e-15, else
// replace the tensor by zeros with a 1 at [0, 0, 0].
#include "mpsb_common.cuh"
#include "cta_gemm.cuh"

namespace mpsb {

// One CTA per chain: R[n] = [[1]], R[i] from R[i+1], stored at
// envs + i * chi_cap^2 as (bonds[i] x bonds[i]) row-major, ket index first
// (the orientation of mps_core.py:360-368).
__global__ void __launch_bounds__(kCtaGemmThreads, 1)
    sample_env_kernel(const mpsb_chain *chains, int chain, int n, int chi_cap, double2 *envs, double2 *tmp) {
    __shared__ GemmSmem sm;
    __shared__ double s_scale;
    const mpsb_chain ch = chains[chain];
    const size_t q1 = (size_t)chi_cap * chi_cap;
    const int tid = threadIdx.x;
    if (tid == 0) envs[(size_t)n * q1] = make_double2(1.0, 0.0);
    __syncthreads();
    for (int i = n - 1; i >= 0; --i) {
        const int cl = ch.bonds[i], cr = ch.bonds[i + 1];
        const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)i * ch.slot_elems);
        const double2 *R = envs + (size_t)(i + 1) * q1;
        double2 *Rn = envs + (size_t)i * q1;
        // T[(a, s)][c] = sum_b A[(a, s)][b] R[b][c]
        cta_cgemm<true, true>(
            2 * cl, cr, cr, [&](int r, int k) { return A[(size_t)r * cr + k]; },
            [&](int k, int c) { return R[(size_t)k * cr + c]; },
            [&](int r, int c, double2 v) { tmp[(size_t)r * cr + c] = v; }, sm);
        // R'[a][b] = sum_{(s, c)} T[a][(s, c)] conj(A[b][(s, c)])
        cta_cgemm<true, false>(
            cl, cl, 2 * cr, [&](int a, int k) { return tmp[(size_t)a * 2 * cr + k]; },
            [&](int k, int b) { return c_conj(A[(size_t)b * 2 * cr + k]); },
            [&](int a, int b, double2 v) { Rn[(size_t)a * cl + b] = v; }, sm);
        if (tid == 0) {
            double tr = 0.0;
            for (int a = 0; a < cl; ++a) tr += Rn[(size_t)a * cl + a].x;
            s_scale = tr > 1e-300 ? tr : 0.0;
        }
        __syncthreads();
        const double tr = s_scale;
        if (tr != 0.0)
            for (int e = tid; e < cl * cl; e += kCtaGemmThreads) Rn[e] = make_double2(Rn[e].x / tr, Rn[e].y / tr);
        __syncthreads();
    }
}

constexpr int kShotWarps = 4;

// One warp per shot.  bits: shots x n bytes, byte i = outcome of site i.
__global__ void __launch_bounds__(32 * kShotWarps)
    sample_kernel(const mpsb_chain *chains, int chain, int n, int chi_cap, const double2 *envs,
                  const double *uniforms, int shots, uint8_t *bits) {
    __shared__ double2 sv[kShotWarps][64], sw[kShotWarps][2][64];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int shot = blockIdx.x * kShotWarps + warp;
    if (shot >= shots) return;
    const mpsb_chain ch = chains[chain];
    const size_t q1 = (size_t)chi_cap * chi_cap;
    double2 *v = sv[warp];
    if (lane == 0) v[0] = make_double2(1.0, 0.0);
    __syncwarp();
    for (int i = 0; i < n; ++i) {
        const int cl = ch.bonds[i], cr = ch.bonds[i + 1];
        const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)i * ch.slot_elems);
        const double2 *R = envs + (size_t)(i + 1) * q1;
        // w_s[c] = sum_b v[b] A[b][s][c]
        for (int c = lane; c < cr; c += 32) {
            double2 w0 = make_double2(0.0, 0.0), w1 = w0;
            for (int b = 0; b < cl; ++b) {
                const double2 vb = v[b];
                w0 = c_fma(vb, A[(size_t)b * 2 * cr + c], w0);
                w1 = c_fma(vb, A[(size_t)b * 2 * cr + cr + c], w1);
            }
            sw[warp][0][c] = w0;
            sw[warp][1][c] = w1;
        }
        __syncwarp();
        // p_s = Re sum_b w_s[b] sum_c R[b][c] conj(w_s[c])
        double pp[2];
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            const double2 *w = sw[warp][s];
            double part = 0.0;
            for (int b = lane; b < cr; b += 32) {
                double2 t = make_double2(0.0, 0.0);
                for (int c = 0; c < cr; ++c) t = c_fma(R[(size_t)b * cr + c], c_conj(w[c]), t);
                part += c_mul(w[b], t).x;
            }
            pp[s] = warp_sum(part);
        }
        double p0 = fmax(pp[0], 0.0), p1 = fmax(pp[1], 0.0);
        const double tot = p0 + p1;
        if (tot < 1e-15) {
            p0 = 0.5;
            p1 = 0.5;
        } else {
            p0 /= tot;
            p1 /= tot;
        }
        const double cdf0 = p0 / (p0 + p1);
        const int o = uniforms[(size_t)shot * n + i] >= cdf0 ? 1 : 0;
        if (lane == 0) bits[(size_t)shot * n + i] = (uint8_t)o;
        // v = w_o / |w_o|
        const double2 *w = sw[warp][o];
        double nn = 0.0;
        for (int c = lane; c < cr; c += 32) nn += c_abs2(w[c]);
        const double nrm = sqrt(warp_sum(nn));
        __syncwarp();
        for (int c = lane; c < cr; c += 32) {
            const double2 x = w[c];
            v[c] = nrm > 1e-15 ? make_double2(x.x / nrm, x.y / nrm) : x;
        }
        __syncwarp();
    }
}

// One CTA per op.
__global__ void __launch_bounds__(128) reset_kernel(const mpsb_chain *chains, const mpsb_site_op *ops, int nops) {
    __shared__ double red[4];
    const int q = blockIdx.x, tid = threadIdx.x;
    if (q >= nops) return;
    const mpsb_site_op op = ops[q];
    const mpsb_chain ch = chains[op.chain];
    const int cl = ch.bonds[op.site], cr = ch.bonds[op.site + 1];
    double2 *t = reinterpret_cast<double2 *>(ch.sites + (size_t)op.site * ch.slot_elems);
    double part = 0.0;
    for (int e = tid; e < cl * cr; e += blockDim.x) {
        const int l = e / cr, r = e - l * cr;
        part += c_abs2(t[(size_t)l * 2 * cr + r]);
    }
    part = warp_sum(part);
    if ((tid & 31) == 0) red[tid >> 5] = part;
    __syncthreads();
    const double nm = sqrt(red[0] + red[1] + red[2] + red[3]);
    for (int e = tid; e < cl * 2 * cr; e += blockDim.x) {
        const int s = (e / cr) & 1;
        double2 x = t[e];
        if (nm > 1e-15)
            x = s ? make_double2(0.0, 0.0) : make_double2(x.x / nm, x.y / nm);
        else
            x = make_double2(e == 0 ? 1.0 : 0.0, 0.0);
        t[e] = x;
    }
}

// ------------------------------------------------------------------ host
size_t sample_workspace_bytes(int n, int chi_cap) {
    const size_t q1 = (size_t)chi_cap * chi_cap;
    return ((size_t)(n + 1) * q1 + 2 * q1) * sizeof(double2);
}

int launch_sample(const mpsb_chain *chains, int chain, int n, int chi_cap, const double *uniforms, int shots,
                  uint8_t *bits, void *ws, cudaStream_t s) {
    const size_t q1 = (size_t)chi_cap * chi_cap;
    double2 *envs = reinterpret_cast<double2 *>(ws);
    double2 *tmp = envs + (size_t)(n + 1) * q1;
    sample_env_kernel<<<1, kCtaGemmThreads, 0, s>>>(chains, chain, n, chi_cap, envs, tmp);
    int rc = check_launch("sample_env_kernel");
    if (rc || shots == 0) return rc;
    sample_kernel<<<(shots + kShotWarps - 1) / kShotWarps, 32 * kShotWarps, 0, s>>>(chains, chain, n, chi_cap, envs,
                                                                                     uniforms, shots, bits);
    return check_launch("sample_kernel");
}

int launch_reset(const mpsb_chain *chains, const mpsb_site_op *ops, int nops, cudaStream_t s) {
    if (nops == 0) return MPSB_OK;
    reset_kernel<<<nops, 128, 0, s>>>(chains, ops, nops);
    return check_launch("reset_kernel");
}


// ============================================================ canonical forms
// left_normalize_site / right_normalize_site of mps_core.py:221-252 as one
// sweep per chain (one CTA per chain, sites in order).  The QR follows
// LAPACK's zgeqr2 + zung2r, the routines numpy.linalg.qr calls: for column
// j, alpha = M[j][j], x = M[j+1:, j]; unless x = 0 and alpha is real,
// beta = -sign(Re alpha) |(alpha, x)|, tau = ((beta - Re alpha) / beta,
// -Im alpha / beta), x /= (alpha - beta), M[j][j] = beta, and
// H^H = I - conj(tau) v v^H (v = [1; x]) is applied to the columns on the
// right; R is the upper triangle, Q = H(0) ... H(k-1) applied to the leading
// k columns of the identity.  The matrix lives column-major in shared memory
// (at most 128 x 64 complex); R goes to a per-chain global scratch.

namespace {
constexpr int kQrThreads = 256;

struct QrSmem {
    double2 *A;    // rows x cols, column-major, leading dimension ld
    double2 *R;    // k x cols, row-major (global scratch)
    double2 *tau;  // k
    double *red;   // kQrThreads / 32
    int ld;
};

__device__ double block_sum(double v, double *red) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < kQrThreads / 32; ++w) t += red[w];
    return t;
}

// Householder QR of the rows x cols matrix in S.A; leaves R in S.R (k x cols)
// and Q (rows x k) in S.A.  Returns k = min(rows, cols).
__device__ int cta_qr(QrSmem &S, int rows, int cols) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int k = min(rows, cols);
    const int ld = S.ld;
    for (int j = 0; j < k; ++j) {
        double xs = 0.0;
        for (int r = j + 1 + tid; r < rows; r += kQrThreads) xs += c_abs2(S.A[(size_t)j * ld + r]);
        const double xnorm2 = block_sum(xs, S.red);
        const double2 alpha = S.A[(size_t)j * ld + j];
        double2 tau = make_double2(0.0, 0.0);
        double2 scale = make_double2(0.0, 0.0);
        double beta = 0.0;
        const bool identity = xnorm2 == 0.0 && alpha.y == 0.0;
        if (!identity) {
            const double nrm = sqrt(fma(alpha.x, alpha.x, fma(alpha.y, alpha.y, xnorm2)));
            beta = alpha.x >= 0.0 ? -nrm : nrm;
            tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
            const double2 d = make_double2(alpha.x - beta, alpha.y);  // 1 / (alpha - beta)
            const double dd = fma(d.x, d.x, d.y * d.y);
            scale = make_double2(d.x / dd, -d.y / dd);
        }
        __syncthreads();
        if (!identity) {
            for (int r = j + 1 + tid; r < rows; r += kQrThreads)
                S.A[(size_t)j * ld + r] = c_mul(S.A[(size_t)j * ld + r], scale);
            if (tid == 0) S.A[(size_t)j * ld + j] = make_double2(beta, 0.0);
        }
        if (tid == 0) S.tau[j] = tau;
        __syncthreads();
        if (!identity) {
            // columns c > j: w = v^H M[:, c]; M[:, c] -= conj(tau) v w
            const double2 ctau = c_conj(tau);
            for (int c = j + 1 + warp; c < cols; c += kQrThreads / 32) {
                double2 w = make_double2(0.0, 0.0);
                for (int r = j + lane; r < rows; r += 32) {
                    const double2 v = r == j ? make_double2(1.0, 0.0) : S.A[(size_t)j * ld + r];
                    w = c_cfma(v, S.A[(size_t)c * ld + r], w);
                }
                w.x = warp_sum(w.x);
                w.y = warp_sum(w.y);
                const double2 f = c_mul(ctau, w);
                for (int r = j + lane; r < rows; r += 32) {
                    const double2 v = r == j ? make_double2(1.0, 0.0) : S.A[(size_t)j * ld + r];
                    S.A[(size_t)c * ld + r] = c_sub(S.A[(size_t)c * ld + r], c_mul(v, f));
                }
            }
        }
        __syncthreads();
    }
    // R = upper triangle (k x cols)
    for (int e = tid; e < k * cols; e += kQrThreads) {
        const int i = e / cols, c = e - i * cols;
        S.R[e] = c >= i ? S.A[(size_t)c * ld + i] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    // Q: zung2r on the leading k columns
    for (int i = k - 1; i >= 0; --i) {
        const double2 tau = S.tau[i];
        if (i < k - 1) {
            if (tid == 0) S.A[(size_t)i * ld + i] = make_double2(1.0, 0.0);
            __syncthreads();
            for (int c = i + 1 + warp; c < k; c += kQrThreads / 32) {
                double2 w = make_double2(0.0, 0.0);
                for (int r = i + lane; r < rows; r += 32) w = c_cfma(S.A[(size_t)i * ld + r], S.A[(size_t)c * ld + r], w);
                w.x = warp_sum(w.x);
                w.y = warp_sum(w.y);
                const double2 f = c_mul(tau, w);
                for (int r = i + lane; r < rows; r += 32)
                    S.A[(size_t)c * ld + r] = c_sub(S.A[(size_t)c * ld + r], c_mul(S.A[(size_t)i * ld + r], f));
            }
            __syncthreads();
        }
        const double2 mt = make_double2(-tau.x, -tau.y);
        for (int r = i + 1 + tid; r < rows; r += kQrThreads) S.A[(size_t)i * ld + r] = c_mul(S.A[(size_t)i * ld + r], mt);
        if (tid == 0) S.A[(size_t)i * ld + i] = make_double2(1.0 - tau.x, -tau.y);
        for (int r = tid; r < i; r += kQrThreads) S.A[(size_t)i * ld + r] = make_double2(0.0, 0.0);
        __syncthreads();
    }
    return k;
}
}  // namespace

// Dynamic shared memory: the matrix (2 chi_cap x chi_cap), tau, the reduction
// slots (R goes to global scratch: 192 KB + the GEMM tiles would not fit).
size_t canon_smem_bytes(int chi_cap) {
    const size_t rows = 2 * (size_t)chi_cap, cols = chi_cap;
    return (rows * cols + cols) * sizeof(double2) + (kQrThreads / 32) * sizeof(double);
}

// dir = 0: left_normalize_site(i) for i = lo .. hi (R absorbed into i + 1 when it exists);
// dir = 1: right_normalize_site(i) for i = hi .. lo (L absorbed into i - 1 when it exists).
// scratch: per chain 3 chi_cap^2 complex (the absorbed neighbour, then R).
__global__ void __launch_bounds__(kQrThreads, 1)
    canon_kernel(const mpsb_chain *chains, const int32_t *ids, int lo, int hi, int dir, int chi_cap,
                 double2 *scratch) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ GemmSmem gsm;
    const mpsb_chain ch = chains[ids[blockIdx.x]];
    double2 *tmp = scratch + (size_t)blockIdx.x * 3 * chi_cap * chi_cap;
    QrSmem S;
    S.ld = 2 * chi_cap;
    S.A = reinterpret_cast<double2 *>(smem_raw);
    S.R = tmp + (size_t)2 * chi_cap * chi_cap;
    S.tau = S.A + (size_t)2 * chi_cap * chi_cap;
    S.red = reinterpret_cast<double *>(S.tau + chi_cap);
    const int tid = threadIdx.x;
    const int n = ch.n;
    if (lo < 0 || hi >= n) return;  // the host validates; never index outside the chain
    for (int step = 0; step <= hi - lo; ++step) {
        const int i = dir == 0 ? lo + step : hi - step;
        const int cl = ch.bonds[i], cr = ch.bonds[i + 1];
        double2 *A = reinterpret_cast<double2 *>(ch.sites + (size_t)i * ch.slot_elems);
        int rows, cols;
        if (dir == 0) {  // M = A as (2 cl) x cr
            rows = 2 * cl;
            cols = cr;
            for (int e = tid; e < rows * cols; e += kQrThreads) {
                const int r = e / cols, c = e - r * cols;
                S.A[(size_t)c * S.ld + r] = A[e];
            }
        } else {  // M^H with M = A as cl x (2 cr)
            rows = 2 * cr;
            cols = cl;
            for (int e = tid; e < cl * rows; e += kQrThreads) {
                const int c = e / rows, r = e - c * rows;
                S.A[(size_t)c * S.ld + r] = c_conj(A[e]);
            }
        }
        __syncthreads();
        const int k = cta_qr(S, rows, cols);
        if (dir == 0) {
            // site i = Q as (cl, 2, k)
            for (int e = tid; e < rows * k; e += kQrThreads) {
                const int r = e / k, c = e - r * k;
                A[e] = S.A[(size_t)c * S.ld + r];
            }
            if (i + 1 < n) {  // site i+1 = R (k x cr) . B (cr x 2 c2)
                const int c2 = ch.bonds[i + 2];
                const double2 *B = reinterpret_cast<const double2 *>(ch.sites + (size_t)(i + 1) * ch.slot_elems);
                cta_cgemm<true, true>(
                    k, 2 * c2, cr, [&](int a, int b) { return S.R[(size_t)a * cols + b]; },
                    [&](int b, int c) { return B[(size_t)b * 2 * c2 + c]; },
                    [&](int a, int c, double2 v) { tmp[(size_t)a * 2 * c2 + c] = v; }, gsm);
                double2 *Bw = reinterpret_cast<double2 *>(ch.sites + (size_t)(i + 1) * ch.slot_elems);
                for (int e = tid; e < k * 2 * c2; e += kQrThreads) Bw[e] = tmp[e];
            }
            if (tid == 0) ch.bonds[i + 1] = k;
        } else {
            // site i = Q^H as (k, 2, cr)
            for (int e = tid; e < k * rows; e += kQrThreads) {
                const int a = e / rows, r = e - a * rows;
                A[e] = c_conj(S.A[(size_t)a * S.ld + r]);
            }
            if (i - 1 >= 0) {  // site i-1 = P (2 c0 x cl) . L (cl x k), L = R^H
                const int c0 = ch.bonds[i - 1];
                const double2 *P = reinterpret_cast<const double2 *>(ch.sites + (size_t)(i - 1) * ch.slot_elems);
                cta_cgemm<true, false>(
                    2 * c0, k, cl, [&](int a, int b) { return P[(size_t)a * cl + b]; },
                    [&](int b, int c) { return c_conj(S.R[(size_t)c * cols + b]); },
                    [&](int a, int c, double2 v) { tmp[(size_t)a * k + c] = v; }, gsm);
                double2 *Pw = reinterpret_cast<double2 *>(ch.sites + (size_t)(i - 1) * ch.slot_elems);
                for (int e = tid; e < 2 * c0 * k; e += kQrThreads) Pw[e] = tmp[e];
            }
            if (tid == 0) ch.bonds[i] = k;
        }
        __syncthreads();
    }
}

size_t canon_workspace_bytes(int nchains, int chi_cap) {
    return (size_t)nchains * 3 * chi_cap * chi_cap * sizeof(double2);
}

int launch_canonicalize(const mpsb_chain *chains, const int32_t *ids, int nchains, int lo, int hi, int dir,
                        int chi_cap, void *ws, cudaStream_t s) {
    if (nchains == 0 || hi < lo) return MPSB_OK;
    const size_t smem = canon_smem_bytes(chi_cap);
    const int rc = ensure_smem(reinterpret_cast<const void *>(canon_kernel), smem, "cudaFuncSetAttribute(canon)");
    if (rc) return rc;
    canon_kernel<<<nchains, kQrThreads, smem, s>>>(chains, ids, lo, hi, dir, chi_cap,
                                                   reinterpret_cast<double2 *>(ws));
    return check_launch("canon_kernel");
}

}  // namespace mpsb
