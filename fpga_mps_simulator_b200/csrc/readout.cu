// Single-site gates and read-out of device-resident MPS chains.
//
// apply1q:      A'[l,s',r] = sum_s G[s',s] A[l,s,r]          (mps_core.py:267-273)
// statevector:  left-to-right contraction, exp(norm_log), Qiskit order (mps_core.py:433-461)
// amplitude:    <b|psi> by a product of matrices A_k[:, b_k, :], same convention
// expectations: left/right transfer environments (the contraction of
//               mps_core.py:364, trace-normalised per site) and local terms.
#include "mpsb_common.cuh"
#include "cta_gemm.cuh"

namespace mpsb {

// ------------------------------------------------------------- apply 1q
__global__ void apply1q_kernel(const mpsb_chain *chains, const mpsb_site_op *ops, const double2 *gates,
                               int chi_cap) {
    const mpsb_site_op op = ops[blockIdx.x];
    const mpsb_chain ch = chains[op.chain];
    if (op.site < 0 || op.site >= ch.n) return;
    const int cl = ch.bonds[op.site], cr = ch.bonds[op.site + 1];
    if (cl < 1 || cr < 1 || cl > chi_cap || cr > chi_cap) return;
    double2 *A = reinterpret_cast<double2 *>(ch.sites + (size_t)op.site * ch.slot_elems);
    const double2 g0 = __ldg(gates + 4 * op.gate + 0), g1 = __ldg(gates + 4 * op.gate + 1);
    const double2 g2 = __ldg(gates + 4 * op.gate + 2), g3 = __ldg(gates + 4 * op.gate + 3);
    for (int e = threadIdx.x; e < cl * cr; e += blockDim.x) {
        const int a = e / cr, b = e - a * cr;
        double2 *p0 = A + (size_t)(2 * a) * cr + b;
        double2 *p1 = p0 + cr;
        const double2 x0 = *p0, x1 = *p1;
        *p0 = c_fma(g1, x1, c_mul(g0, x0));
        *p1 = c_fma(g3, x1, c_mul(g2, x0));
    }
}

int launch_apply1q(const mpsb_chain *chains, const mpsb_site_op *ops, int nops, const double2 *gates,
                   int chi_cap, cudaStream_t s) {
    if (nops == 0) return MPSB_OK;
    apply1q_kernel<<<nops, 256, 0, s>>>(chains, ops, gates, chi_cap);
    return check_launch("apply1q_kernel");
}

// ------------------------------------------------------------- statevector
// psi_out[(x, s), d] = sum_c psi_in[x, c] A[c, s, d]; x < P rows.  Site 0
// starts from psi = A_0[0, :, :].  Dimensions are read on the device.
__global__ void sv_step_kernel(const mpsb_chain *ch_p, int k, long long P, long long cap, const double2 *psi_in,
                               double2 *psi_out) {
    const mpsb_chain ch = *ch_p;
    const int cin = ch.bonds[k], cout = ch.bonds[k + 1];
    const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems);
    // a valid chain has bonds[k+1] <= 2^(n-k-1), so 2 P cout <= 2^n = cap; never write past the buffer
    if (P * 2 * cout > cap || (long long)P * cin > cap) return;
    const long long total = P * 2 * cout;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long x = e / (2 * cout);
        const int rem = (int)(e - x * 2 * cout);
        const int s = rem / cout, d = rem - s * cout;
        double2 acc = make_double2(0, 0);
        if (k == 0) {
            acc = A[s * cout + d];
        } else {
            const double2 *pin = psi_in + x * cin;
            for (int c = 0; c < cin; ++c) acc = c_fma(pin[c], A[(size_t)(2 * c + s) * cout + d], acc);
        }
        psi_out[e] = acc;
    }
}

__global__ void sv_final_kernel(const mpsb_chain *ch_p, int n, const double2 *psi, double2 *out) {
    const double scale = exp(*ch_p->norm_log);
    const long long N = 1ll << n;
    for (long long x = blockIdx.x * (long long)blockDim.x + threadIdx.x; x < N;
         x += (long long)gridDim.x * blockDim.x) {
        // psi index x has site 0 as the most significant bit; Qiskit puts qubit 0 at bit 0
        const long long y = (long long)(__brevll((unsigned long long)x) >> (64 - n));
        out[y] = c_scale(psi[x], scale);
    }
}

int launch_statevector(const mpsb_chain *ch_dev, int n, int chi_cap, double2 *out, double2 *scratch,
                       size_t scratch_bytes, cudaStream_t s) {
    const size_t need = (size_t)2 * ((size_t)1 << n) * sizeof(double2);
    if (scratch_bytes < need) return set_error(MPSB_EWORKSPACE, "statevector scratch needs %zu bytes", need);
    double2 *bufs[2] = {scratch, scratch + ((size_t)1 << n)};
    long long P = 1;
    for (int k = 0; k < n; ++k) {
        // rows after this step: 2P; columns <= min(chi_cap, 2^(n-k-1))
        const long long right = (n - k - 1) >= 30 ? (1ll << 30) : (1ll << (n - k - 1));
        const long long cols = right < chi_cap ? right : chi_cap;
        const long long total = 2 * P * cols;
        const int blocks = (int)((total + 255) / 256 > 4096 ? 4096 : (total + 255) / 256);
        sv_step_kernel<<<blocks, 256, 0, s>>>(ch_dev, k, P, 1ll << n, bufs[(k + 1) & 1], bufs[k & 1]);
        int rc = check_launch("sv_step_kernel");
        if (rc) return rc;
        P *= 2;
    }
    const long long N = 1ll << n;
    const int blocks = (int)((N + 255) / 256 > 4096 ? 4096 : (N + 255) / 256);
    sv_final_kernel<<<blocks, 256, 0, s>>>(ch_dev, n, bufs[(n - 1) & 1], out);
    return check_launch("sv_final_kernel");
}

// ------------------------------------------------------------- amplitudes
// One CTA per basis state; the row vector is renormalised every site and the
// log-scale accumulated so that long chains do not underflow.
__global__ void amplitude_kernel(const mpsb_chain *chains, int chain, int n, const uint8_t *bits,
                                 double2 *out, double *log_abs) {
    extern __shared__ double2 vbuf[];  // 2 * 64
    __shared__ double red[8];
    const mpsb_chain ch = chains[chain];
    const uint8_t *b = bits + (size_t)blockIdx.x * n;
    double2 *v = vbuf, *vn = vbuf + 64;
    const int tid = threadIdx.x;
    if (tid == 0) v[0] = make_double2(1.0, 0.0);
    double lscale = 0.0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const int cin = ch.bonds[k], cout = ch.bonds[k + 1];
        const int s = b[k] ? 1 : 0;
        const double2 *A = reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems);
        double part = 0.0;
        if (tid < cout) {
            double2 acc = make_double2(0, 0);
            for (int c = 0; c < cin; ++c) acc = c_fma(v[c], A[(size_t)(2 * c + s) * cout + tid], acc);
            vn[tid] = acc;
            part = c_abs2(acc);
        }
        part = warp_sum(part);
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        double nrm2 = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) nrm2 += red[q];
        const double inv = nrm2 > 0.0 ? rsqrt(nrm2) : 1.0;
        if (nrm2 > 0.0) lscale += 0.5 * log(nrm2);
        if (tid < cout) v[tid] = c_scale(vn[tid], inv);
        __syncthreads();
    }
    if (tid == 0) {
        const double nl = *ch.norm_log;
        const double2 a = v[0];
        const double mag = sqrt(c_abs2(a));
        if (log_abs) log_abs[blockIdx.x] = (mag > 0.0) ? log(mag) + lscale + nl : -INFINITY;
        out[blockIdx.x] = c_scale(a, exp(lscale + nl));
    }
}

int launch_amplitude(const mpsb_chain *chains, int chain, int n, const uint8_t *bits, int nbits,
                     double2 *out, double *log_abs, cudaStream_t s) {
    if (nbits == 0) return MPSB_OK;
    amplitude_kernel<<<nbits, 64, 128 * sizeof(double2), s>>>(chains, chain, n, bits, out, log_abs);
    return check_launch("amplitude_kernel");
}

// ------------------------------------------------------------- environments
// Left:  E_{k+1}[c,d] = sum_{x,y,s,t} conj(A[x,s,c]) O[s,t] E_k[x,y] A[y,t,d]
// Right: F_k[c,d]     = sum_{x,y,s}   conj(A[c,s,x]) A[d,s,y] F_{k+1}[x,y]
// (bra index first; O = identity for the plain environments).  The
// intermediate T lives in global scratch so shared memory stays at two
// chi x chi matrices (128 KB at chi = 64).
struct EnvStepArgs {
    const double2 *A;
    int cl, cr;
};

// T[x, t, d] = sum_y E[x, y] A[y, t, d];  E'[c, d] = sum_{x,s,t} conj(A[x,s,c]) O[s,t] T[x,t,d]
__device__ void left_step(const double2 *E, const EnvStepArgs &a, const double2 *O, double2 *T, double2 *Eout,
                          int tid, int nth) {
    const int cl = a.cl, cr = a.cr;
    for (int e = tid; e < cl * 2 * cr; e += nth) {
        const int x = e / (2 * cr), rem = e - x * 2 * cr;
        double2 acc = make_double2(0, 0);
        for (int y = 0; y < cl; ++y) acc = c_fma(E[x * cl + y], a.A[(size_t)y * 2 * cr + rem], acc);
        T[e] = acc;
    }
    __threadfence_block();
    __syncthreads();
    for (int e = tid; e < cr * cr; e += nth) {
        const int c = e / cr, d = e - c * cr;
        double2 acc = make_double2(0, 0);
        for (int x = 0; x < cl; ++x) {
            const double2 a0 = a.A[(size_t)(2 * x) * cr + c], a1 = a.A[(size_t)(2 * x + 1) * cr + c];
            const double2 t0 = T[(size_t)(2 * x) * cr + d], t1 = T[(size_t)(2 * x + 1) * cr + d];
            if (O) {
                const double2 o0 = c_fma(O[1], t1, c_mul(O[0], t0));
                const double2 o1 = c_fma(O[3], t1, c_mul(O[2], t0));
                acc = c_cfma(a0, o0, acc);
                acc = c_cfma(a1, o1, acc);
            } else {
                acc = c_cfma(a0, t0, acc);
                acc = c_cfma(a1, t1, acc);
            }
        }
        Eout[e] = acc;
    }
    __threadfence_block();
    __syncthreads();
}

// T[d, s, x] = sum_y A[d, s, y] F[x, y];  F'[c, d] = sum_{s, x} conj(A[c, s, x]) T[d, s, x]
__device__ void right_step(const double2 *F, const EnvStepArgs &a, double2 *T, double2 *Fout, int tid, int nth) {
    const int cl = a.cl, cr = a.cr;
    for (int e = tid; e < cl * 2 * cr; e += nth) {
        const int ds = e / cr, x = e - ds * cr;
        double2 acc = make_double2(0, 0);
        const double2 *arow = a.A + (size_t)ds * cr;
        for (int y = 0; y < cr; ++y) acc = c_fma(arow[y], F[x * cr + y], acc);
        T[e] = acc;
    }
    __threadfence_block();
    __syncthreads();
    for (int e = tid; e < cl * cl; e += nth) {
        const int c = e / cl, d = e - c * cl;
        double2 acc = make_double2(0, 0);
        for (int x = 0; x < cr; ++x) {
            acc = c_cfma(a.A[(size_t)(2 * c) * cr + x], T[(size_t)(2 * d) * cr + x], acc);
            acc = c_cfma(a.A[(size_t)(2 * c + 1) * cr + x], T[(size_t)(2 * d + 1) * cr + x], acc);
        }
        Fout[e] = acc;
    }
    __threadfence_block();
    __syncthreads();
}

__device__ double block_sum(double v, double *red, int tid, int nth) {
    v = warp_sum(v);
    __syncthreads();
    if ((tid & 31) == 0) red[tid >> 5] = v;
    __syncthreads();
    double s = 0.0;
    for (int q = 0; q < nth / 32; ++q) s += red[q];
    __syncthreads();
    return s;
}

__device__ void trace_normalise(double2 *E, int dim, double *red, int tid, int nth) {
    double part = 0.0;
    for (int c = tid; c < dim; c += nth) part += E[c * dim + c].x;
    const double tr = block_sum(part, red, tid, nth);
    if (tr > 0.0) {
        const double inv = 1.0 / tr;
        for (int e = tid; e < dim * dim; e += nth) E[e] = c_scale(E[e], inv);
    }
    __syncthreads();
}

// Two CTAs per chain, one per direction: left environments envL[k] (k = 0..n) and right
// environments envR[k], chi_cap x chi_cap each, trace-normalised per site.
// The environment sweeps' steps as two CTA GEMMs each on the FP64
// tensor-core MMA (the whole 256-thread CTA; T in global scratch):
//   left:  T[x, (t,d)] = sum_y E[x,y] A[y,(t,d)];  E'[c,d] = sum_(x,s) conj(A[(x,s),c]) T[(x,s),d]
//   right: T[(d,s), x] = sum_y A[(d,s),y] F[x,y];  F'[c,d] = sum_(s,x) conj(A[c,(s,x)]) T[d,(s,x)]
// (the loops of left_step / right_step for the plain environments, 7-8x
// fewer cycles per step at chi = 64).
__device__ void left_env_step_mma(const double2 *E, const EnvStepArgs &a, double2 *T, double2 *Eout,
                                  GemmSmem &sm) {
    const int cl = a.cl, cr = a.cr, twocr = 2 * cr;
    cta_cgemm<true, true>(
        cl, twocr, cl, [&](int x, int y) { return E[x * cl + y]; },
        [&](int y, int j) { return a.A[(size_t)y * twocr + j]; },
        [&](int x, int j, double2 v) { T[(size_t)x * twocr + j] = v; }, sm);
    __threadfence_block();
    __syncthreads();
    cta_cgemm<false, true>(
        cr, cr, 2 * cl, [&](int c, int k) { return c_conj(a.A[(size_t)k * cr + c]); },
        [&](int k, int d) { return T[(size_t)k * cr + d]; }, [&](int c, int d, double2 v) { Eout[c * cr + d] = v; },
        sm);
    __syncthreads();
}

__device__ void right_env_step_mma(const double2 *F, const EnvStepArgs &a, double2 *T, double2 *Fout,
                                   GemmSmem &sm) {
    const int cl = a.cl, cr = a.cr, twocr = 2 * cr;
    cta_cgemm<true, false>(
        2 * cl, cr, cr, [&](int i, int y) { return a.A[(size_t)i * cr + y]; },
        [&](int y, int x) { return F[x * cr + y]; }, [&](int i, int x, double2 v) { T[(size_t)i * cr + x] = v; },
        sm);
    __threadfence_block();
    __syncthreads();
    cta_cgemm<true, false>(
        cl, cl, twocr, [&](int c, int k) { return c_conj(a.A[(size_t)c * twocr + k]); },
        [&](int k, int d) { return T[(size_t)d * twocr + k]; }, [&](int c, int d, double2 v) { Fout[c * cl + d] = v; },
        sm);
    __syncthreads();
}

__global__ void environments_kernel(const mpsb_chain *chains, int n, int chi_cap, double2 *envL, double2 *envR,
                                    double2 *tscr) {
    __shared__ GemmSmem gsm;
    extern __shared__ __align__(16) unsigned char sm[];
    double2 *E = reinterpret_cast<double2 *>(sm);
    double2 *En = E + chi_cap * chi_cap;
    __shared__ double red[32];
    const int tid = threadIdx.x, nth = blockDim.x;
    const int chain = blockIdx.x >> 1;
    const bool left = (blockIdx.x & 1) == 0;  // CTA 2c sweeps left to right, CTA 2c + 1 right to left
    const mpsb_chain ch = chains[chain];
    const size_t es = (size_t)chi_cap * chi_cap;
    double2 *L = envL + (size_t)chain * (n + 1) * es;
    double2 *Rv = envR + (size_t)chain * (n + 1) * es;
    double2 *T = tscr + (size_t)blockIdx.x * 2 * es;
    if (left) {
        if (tid == 0) {
            E[0] = make_double2(1.0, 0.0);
            L[0] = E[0];
        }
        __syncthreads();
        for (int k = 0; k < n; ++k) {
            EnvStepArgs a{reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems), ch.bonds[k],
                          ch.bonds[k + 1]};
            left_env_step_mma(E, a, T, En, gsm);
            trace_normalise(En, a.cr, red, tid, nth);
            for (int e = tid; e < a.cr * a.cr; e += nth) {
                E[e] = En[e];
                L[(size_t)(k + 1) * es + e] = En[e];
            }
            __syncthreads();
        }
        return;
    }
    if (tid == 0) {
        E[0] = make_double2(1.0, 0.0);
        Rv[(size_t)n * es] = E[0];
    }
    __syncthreads();
    for (int k = n - 1; k >= 0; --k) {
        EnvStepArgs a{reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems), ch.bonds[k],
                      ch.bonds[k + 1]};
        right_env_step_mma(E, a, T, En, gsm);
        trace_normalise(En, a.cl, red, tid, nth);
        for (int e = tid; e < a.cl * a.cl; e += nth) {
            E[e] = En[e];
            Rv[(size_t)k * es + e] = En[e];
        }
        __syncthreads();
    }
}

// Closure of one site between a left matrix E (cl x cl) and a right matrix
// F (cr x cr): S[s][t] = sum_{x,d} P[x,s,d] T[x,t,d] with
// P[x,s,d] = sum_c conj(A[x,s,c]) F[c,d] and T[x,t,d] = sum_y E[x,y] A[y,t,d],
// so that <O> = sum_{st} O[s,t] S[s][t] and the norm is S[0][0] + S[1][1].
__device__ void site_closure(const double2 *E, const double2 *A, const double2 *F, int cl, int cr, double *red,
                             int tid, int nth, double2 S[4]) {
    double2 acc[4] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int e = tid; e < cl * cr; e += nth) {
        const int x = e / cr, d = e - x * cr;
        double2 p0 = make_double2(0, 0), p1 = p0, t0 = p0, t1 = p0;
        for (int c = 0; c < cr; ++c) {
            const double2 f = F[c * cr + d];
            p0 = c_cfma(A[(size_t)(2 * x) * cr + c], f, p0);
            p1 = c_cfma(A[(size_t)(2 * x + 1) * cr + c], f, p1);
        }
        for (int y = 0; y < cl; ++y) {
            const double2 ev = E[x * cl + y];
            t0 = c_fma(ev, A[(size_t)(2 * y) * cr + d], t0);
            t1 = c_fma(ev, A[(size_t)(2 * y + 1) * cr + d], t1);
        }
        acc[0] = c_fma(p0, t0, acc[0]);
        acc[1] = c_fma(p0, t1, acc[1]);
        acc[2] = c_fma(p1, t0, acc[2]);
        acc[3] = c_fma(p1, t1, acc[3]);
    }
    for (int q = 0; q < 4; ++q) {
        S[q].x = block_sum(acc[q].x, red, tid, nth);
        S[q].y = block_sum(acc[q].y, red, tid, nth);
    }
}

// Persistent CTAs over (chain, term).  Two-site terms first fold site k
// with O1 (numerator) and with the identity (denominator) into scratch.
__global__ void terms_kernel(const mpsb_chain *chains, int nchains, int n, int chi_cap, const double2 *envL,
                             const double2 *envR, const int32_t *sites, const int32_t *two_site,
                             const double2 *ops, int nterms, double *out, double2 *scr) {
    __shared__ double2 O[8];
    __shared__ double red[32];
    const int tid = threadIdx.x, nth = blockDim.x;
    const size_t es = (size_t)chi_cap * chi_cap;
    double2 *T = scr + (size_t)blockIdx.x * 4 * es;
    double2 *En = T + 2 * es;
    double2 *Ed = En + es;
    for (int job = blockIdx.x; job < nchains * nterms; job += gridDim.x) {
        const int chain = job / nterms, t = job - chain * nterms;
        const mpsb_chain ch = chains[chain];
        const int k = sites[t];
        const bool two = two_site[t] != 0;
        __syncthreads();
        if (k < 0 || k + (two ? 1 : 0) >= n) {
            if (tid == 0) out[job] = 0.0;
            continue;
        }
        if (tid < 8) O[tid] = ops[(size_t)8 * t + tid];
        __syncthreads();
        const double2 *L = envL + ((size_t)chain * (n + 1) + k) * es;
        const int last = two ? k + 1 : k;
        const double2 *F = envR + ((size_t)chain * (n + 1) + last + 1) * es;
        const double2 *Alast = reinterpret_cast<const double2 *>(ch.sites + (size_t)last * ch.slot_elems);
        const int cl = ch.bonds[last], cr = ch.bonds[last + 1];
        double2 S[4], Sd[4];
        const double2 *Olast = O + (two ? 4 : 0);
        if (!two) {
            site_closure(L, Alast, F, cl, cr, red, tid, nth, S);
            Sd[0] = S[0];
            Sd[3] = S[3];
        } else {
            EnvStepArgs a{reinterpret_cast<const double2 *>(ch.sites + (size_t)k * ch.slot_elems), ch.bonds[k],
                          ch.bonds[k + 1]};
            left_step(L, a, O, T, En, tid, nth);
            left_step(L, a, nullptr, T, Ed, tid, nth);
            site_closure(En, Alast, F, cl, cr, red, tid, nth, S);
            site_closure(Ed, Alast, F, cl, cr, red, tid, nth, Sd);
        }
        if (tid == 0) {
            double2 num = make_double2(0, 0);
            for (int q = 0; q < 4; ++q) num = c_fma(Olast[q], S[q], num);
            const double den = Sd[0].x + Sd[3].x;
            out[job] = den != 0.0 ? num.x / den : 0.0;
        }
    }
}

size_t expect_workspace_bytes(int nchains, int n, int chi_cap, int nctas) {
    const size_t es = (size_t)chi_cap * chi_cap * sizeof(double2);
    return (size_t)2 * nchains * (n + 1) * es + (size_t)nchains * 4 * es + (size_t)nctas * 4 * es;
}

int launch_expect(const mpsb_chain *chains, int nchains, int n, int chi_cap, const int32_t *sites,
                  const int32_t *two_site, const double2 *ops, int nterms, double *out, void *ws, int nctas,
                  cudaStream_t s) {
    if (nchains == 0 || nterms == 0) return MPSB_OK;
    const size_t es = (size_t)chi_cap * chi_cap;
    double2 *envL = reinterpret_cast<double2 *>(ws);
    double2 *envR = envL + (size_t)nchains * (n + 1) * es;
    double2 *tscr = envR + (size_t)nchains * (n + 1) * es;
    double2 *cscr = tscr + (size_t)nchains * 4 * es;  // 2 es of T per environment CTA, two CTAs per chain
    const size_t smem_env = 2 * es * sizeof(double2);
    int rc = ensure_smem(reinterpret_cast<const void *>(environments_kernel), smem_env,
                         "cudaFuncSetAttribute(environments)");
    if (rc) return rc;
    environments_kernel<<<2 * nchains, 256, smem_env, s>>>(chains, n, chi_cap, envL, envR, tscr);
    rc = check_launch("environments_kernel");
    if (rc) return rc;
    const int grid = nchains * nterms < nctas ? nchains * nterms : nctas;
    terms_kernel<<<grid, 256, 0, s>>>(chains, nchains, n, chi_cap, envL, envR, sites, two_site, ops, nterms, out,
                                      cscr);
    return check_launch("terms_kernel");
}

// ------------------------------------------------------------- overlap
// <a|b> of two chains of equal length: E_{k+1}[c, d] = sum_{x,y,s}
// conj(A_k[x,s,c]) E_k[x,y] B_k[y,s,d], rescaled by its largest magnitude
// each site (the scale is returned as a log).  One CTA; T in global scratch.
__global__ void __launch_bounds__(kCtaGemmThreads, 1)
    overlap_kernel(const mpsb_chain *pa, const mpsb_chain *pb, int n, int chi_cap, double2 *out, double *out_log,
                   double2 *tscr) {
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ GemmSmem gsm;
    double2 *E = reinterpret_cast<double2 *>(sm);
    double2 *En = E + chi_cap * chi_cap;
    __shared__ double red[32];
    const int tid = threadIdx.x, nth = blockDim.x;
    const mpsb_chain a = *pa, b = *pb;
    if (tid == 0) E[0] = make_double2(1.0, 0.0);
    double lg = 0.0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const int cla = a.bonds[k], cra = a.bonds[k + 1], clb = b.bonds[k], crb = b.bonds[k + 1];
        const double2 *A = reinterpret_cast<const double2 *>(a.sites + (size_t)k * a.slot_elems);
        const double2 *B = reinterpret_cast<const double2 *>(b.sites + (size_t)k * b.slot_elems);
        // T[x, (t, d)] = sum_y E[x, y] B[y, (t, d)]
        cta_cgemm<true, true>(
            cla, 2 * crb, clb, [&](int i, int kk) { return E[i * clb + kk]; },
            [&](int kk, int j) { return B[(size_t)kk * 2 * crb + j]; },
            [&](int i, int j, double2 v) { tscr[(size_t)i * 2 * crb + j] = v; }, gsm);
        // E'[c, d] = sum_{(x, s)} conj(A[(x, s), c]) T[(x, s), d]
        double part = 0.0;
        cta_cgemm<false, true>(
            cra, crb, 2 * cla, [&](int i, int kk) { return c_conj(A[(size_t)kk * cra + i]); },
            [&](int kk, int j) { return tscr[(size_t)kk * crb + j]; },
            [&](int i, int j, double2 v) {
                En[i * crb + j] = v;
                part = fmax(part, c_abs2(v));
            },
            gsm);
        // block max
        for (int o = 16; o > 0; o >>= 1) part = fmax(part, __shfl_xor_sync(0xffffffffu, part, o));
        if ((tid & 31) == 0) red[tid >> 5] = part;
        __syncthreads();
        double mx = 0.0;
        for (int q = 0; q < nth / 32; ++q) mx = fmax(mx, red[q]);
        const double sc = mx > 0.0 ? rsqrt(mx) : 1.0;
        if (mx > 0.0) lg -= log(sc);
        for (int e = tid; e < cra * crb; e += nth) E[e] = c_scale(En[e], sc);
        __syncthreads();
    }
    if (tid == 0) {
        out[0] = E[0];
        out_log[0] = lg + *a.norm_log + *b.norm_log;
    }
}

int launch_overlap(const mpsb_chain *a, const mpsb_chain *b, int n, int chi_cap, double2 *out, double *out_log,
                   void *ws, cudaStream_t s) {
    const size_t smem = 2 * (size_t)chi_cap * chi_cap * sizeof(double2);
    const int rc = ensure_smem(reinterpret_cast<const void *>(overlap_kernel), smem, "cudaFuncSetAttribute(overlap)");
    if (rc) return rc;
    overlap_kernel<<<1, kCtaGemmThreads, smem, s>>>(a, b, n, chi_cap, out, out_log, reinterpret_cast<double2 *>(ws));
    return check_launch("overlap_kernel");
}

// ------------------------------------------------------------- FP64 probe
// Eight independent FMA chains per thread; the caller times the launch.
__global__ void fp64_probe_kernel(long long iters, double *sink) {
    double a0 = threadIdx.x * 1e-9, a1 = a0 + 1e-10, a2 = a0 + 2e-10, a3 = a0 + 3e-10;
    double a4 = a0 + 4e-10, a5 = a0 + 5e-10, a6 = a0 + 6e-10, a7 = a0 + 7e-10;
    const double m = 0.999999999, c = 1e-12;
    for (long long it = 0; it < iters; ++it) {
        a0 = fma(a0, m, c); a1 = fma(a1, m, c); a2 = fma(a2, m, c); a3 = fma(a3, m, c);
        a4 = fma(a4, m, c); a5 = fma(a5, m, c); a6 = fma(a6, m, c); a7 = fma(a7, m, c);
    }
    const double r = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (r == 12345.678) sink[0] = r;  // keeps the chains live
}

int launch_fp64_probe(long long iters, int blocks, int threads, double *sink, cudaStream_t s) {
    fp64_probe_kernel<<<blocks, threads, 0, s>>>(iters, sink);
    return check_launch("fp64_probe_kernel");
}

}  // namespace mpsb
