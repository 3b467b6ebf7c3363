// Transpose-free QMR (Freund, SIAM J. Sci. Comput. 14:470, 1993) for all columns of the
// block-sparse Green function at once, each column with its own scalars; the reference calls
// the same algorithm from the external library tfQMRgpu (include/green_action.hxx:216).
//
// Two precisions:
//  * FP64: every vector and the solution in FP64; a column has converged when its QMR residual
//    bound tau*sqrt(m+1) falls below the tolerance (the test tfQMRgpu applies);
//  * FP32 recurrences with an FP64 solution and residual replacement: the vectors W, U, V, D,
//    A U are FP32 and the operator is the FP32 action; the solution is accumulated in FP64
//    (X64 += X32 at every replacement, X32 = 0).  A replacement recomputes the true residual of
//    the FP64 solution with the FP64 action, R = B - A X64, and restarts the recurrence of W
//    from it: with the CGS iterate  x~ = x + theta^2 eta d  of the QMR iterate x,
//    W = R - theta^2 eta A d  (A d with the FP32 action) is the true residual of x~.  The QMR
//    smoothing (tau, theta, eta, D) and the search directions (U2, V) are kept, so the Krylov
//    space is not restarted (residual replacement after Sleijpen & van der Vorst, Computing 56,
//    1996, and van der Vorst & Ye, SIAM J. Sci. Comput. 22, 2000).  A column has converged when
//    its true FP64 residual at a replacement is below the tolerance.  Each source cube (64
//    columns) asks for a replacement when the largest residual estimate of its active columns
//    has fallen by update_factor since its last one, when all of them are below the tolerance,
//    or after update_gap iterations.  The CGS-type recurrences of tfQMR amplify the FP32
//    rounding strongly where the energy lies close to the spectrum: a source cube whose largest
//    true residual has not halved over stall_limit replacements (or is not finite) leaves the FP32
//    recurrences, and all such sources then continue as FP64 tfQMR from their FP64 solution
//    (on A d = B - A X64, to half the tolerance; sources whose true residual is then still above
//    the tolerance restart from their solution, at most kRestarts times).
//
// One iteration = two operator applications.  The BLAS-1 work is fused so that every vector
// is streamed as few times as possible:
//   K_A   U2 = U1 - a V                 and |W - a AU1|^2
//   K_C   W  = W - a (AU1 + AU2)        and |W|^2, rt^H W
//   K_DX  D, X advanced by both half steps at once;  U1 = W + b U2
//   K_E   V  = AU1 + b (AU2 + b V)      and rt^H V
// (U1 = y_{2n-1}, U2 = y_{2n}, AU1 = A y_{2n-1}, AU2 = A y_{2n}, V = v_{n-1} in Freund's
// notation).  The shadow residual rt is a counter-based random vector regenerated on the fly.
// K_A, K_C and K_E move 16 bytes per thread and access (K_A16 ...; K_DX32 in the FP32
// recurrences); the scalar kernels remain as alternatives.
//
// Work units and reductions: every vector kernel runs one CTA per (source cube, chunk of its
// blocks); the column sums of a unit go to a slot of their own, and the last CTA of a source to
// finish (a ticket counter) adds the slots in chunk order, so every inner product is the same in
// every run, and then advances the scalar recurrences of the source's 64 columns.
//
// Retirement: a source whose 64 columns have all finished is skipped by every vector kernel and
// by every kernel of the action (DevicePlan::retire), so finished columns cost nothing.
//
// Batches: a plan built by GreenPlan::replicate holds several (energy, k-point) pairs as
// independent sources of one block-sparse system; solve_batched solves them in waves.
#include "solver.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace a43g {

#define A43G_CUDA_TRY_RC(call) do { cudaError_t e_ = (call); if (cudaSuccess != e_) { \
    ::a43g::set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); return A43G_ERR_CUDA; } } while (0)

namespace {

constexpr int kBlk = 8192;
constexpr int kCoef = 14;     // alpha, beta, the five complex K_DX coefficients
constexpr int kSlots = 8;     // column sums per unit and column (at most 5 are used)
constexpr int kRestarts = 3;  // FP64 continuation: restarts of sources whose true residual is above the tolerance

struct ColState {
    double rho_re, rho_im;       // rho = rt^H w
    double al_re, al_im;         // alpha
    double be_re, be_im;         // beta
    double eta_re, eta_im;       // eta of the last half step
    double kd1_re, kd1_im;       // D coefficient of the first half step
    double et1_re, et1_im;       // eta of the first half step
    double tau, theta;           // tau, theta of the last half step
    double bnorm;                // |b| of the column
    // combined coefficients of K_DX (X and D advanced over both half steps)
    double cu1x_re, cu1x_im, cu2x_re, cu2x_im, cdx_re, cdx_im;
    double cu1d_re, cu1d_im, cdd_re, cdd_im;
    double rhop_re, rhop_im;     // rho of the previous iteration (beta after a replacement)
    double cup_re, cup_im;       // theta^2 eta:  x~ - x = cup d
    double scale;                // estimate correction (true residual / estimate at a replacement, >= 1)
    double res;                  // true relative residual at the last replacement, or at the end
    int32_t m;                   // half steps done
    int32_t status;              // 0 active, 1 converged, 2 breakdown, 3 idle (zero column), 5 left the
                                 // FP32 recurrences for FP64
    int32_t conv1;               // converged in the first half step of this iteration (FP64)
    int32_t pad;
};

struct SrcState {
    int32_t it;                  // iterations done while the source was active
    int32_t since;               // iterations since its last replacement
    int32_t upd;                 // replacement in this iteration
    int32_t updates;             // replacements done
    int32_t done;                // no active column left
    int32_t stall;               // replacements since its largest true residual last halved
    int32_t fallback;            // left the FP32 recurrences for FP64
    int32_t nonfinite;           // ... with a residual that was not finite
    double est_ref;              // largest true residual of its active columns at the last replacement
    double best;                 // smallest such residual so far
};

struct Ctl {
    int32_t n_active;            // sources with an active column
    int32_t breakdowns;
    int32_t pad[2];
};

struct Ctx {
    uint32_t const *src_start, *src_blocks;
    uint32_t const *subset;
    uint8_t const *active;       // retirement flags read by the vector kernels (nullptr: all)
    uint8_t *src_active;         // the flags the action reads, cleared when a source retires
    uint8_t *upd;                // per source: replacement in this iteration
    uint32_t nch, ncol;          // chunks per source, columns (sources * 64)
    double *part;                // [units][kSlots][64] column sums per unit
    uint32_t *tickets;           // [sources]
    ColState *cs;
    SrcState *ss;
    Ctl *ctl;
    double *cd;                  // [kCoef][ncol] coefficients for the FP64 vector kernels
    float *cf;                   // [kCoef][ncol] the same in FP32
    uint32_t seed;
    double tol, delta;
    int32_t gap, mixed, retire;
    int32_t stall_limit;         // replacements without progress of the true residual before FP64
    int32_t abs_tol;             // the tolerance is absolute (the FP64 continuation of unit columns)
    int32_t vec16;               // K_A, K_C, K_E with 16-byte accesses (else the scalar kernels)
};

__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    // murmur3 finaliser as a counter-based generator
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
    return h;
}

// shadow residual element for (block, reim, i, j): uniform in [-1, 1); FP32 sweeps use the
// same values rounded to FP32
__device__ __forceinline__ double shadow(uint32_t seed, uint32_t idx) {
    return double(int32_t(mix32(idx*0x9E3779B9u + seed))) * (1.0/2147483648.0);
}
__device__ __forceinline__ float shadow32(uint32_t seed, uint32_t idx) {
    return float(int32_t(mix32(idx*0x9E3779B9u + seed))) * (1.0f/2147483648.0f);
}
template <typename T> __device__ __forceinline__ T shadow_t(uint32_t seed, uint32_t idx);
template <> __device__ __forceinline__ float shadow_t<float>(uint32_t seed, uint32_t idx) { return shadow32(seed, idx); }
template <> __device__ __forceinline__ double shadow_t<double>(uint32_t seed, uint32_t idx) { return shadow(seed, idx); }

// the blocks [lo, hi) of src_blocks that unit u works on; false for a skipped source
__device__ __forceinline__ bool unit_range(Ctx const &c, uint8_t const *active, uint32_t u, uint32_t &s,
                                           uint32_t &lo, uint32_t &hi) {
    s = u/c.nch;
    uint32_t const q = u - s*c.nch;
    if (active && !active[s]) return false;
    uint32_t const a = c.src_start[s], n = c.src_start[s + 1] - a;
    lo = a + uint32_t((uint64_t(n)*q)/c.nch);
    hi = a + uint32_t((uint64_t(n)*(q + 1))/c.nch);
    return true;
}

// Column sums of one unit (thread (q, j) holds its row group's share v[] of column j) into the
// unit's slot; true in the last CTA of the source to finish, whose threads 0..63 then hold the
// fixed-order total over all units of the source in out[].  Called by all 256 threads.
template <int NC>
__device__ bool reduce_source(Ctx const &c, uint32_t u, uint32_t s, double const (&v)[NC], double (&out)[NC]) {
    __shared__ double red[4][64][NC];
    __shared__ uint32_t ticket;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
#pragma unroll
    for (int k = 0; k < NC; ++k) red[q][j][k] = v[k];
    __syncthreads();
    if (0 == q) {
#pragma unroll
        for (int k = 0; k < NC; ++k)
            c.part[(size_t(u)*kSlots + k)*64 + j] = ((red[0][j][k] + red[1][j][k]) + red[2][j][k]) + red[3][j][k];
    }
    __threadfence();
    __syncthreads();
    if (0 == threadIdx.x) ticket = atomicAdd(&c.tickets[s], 1u);
    __syncthreads();
    if (ticket + 1 != c.nch) return false;            // uniform over the CTA
    __threadfence();
    // thread (q, j) adds the units q, q + 4, ... of the source into four interleaved partial
    // sums (independent loads in flight), combined in a fixed order, then the four q's sums
    double acc4[4][NC];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int k = 0; k < NC; ++k) acc4[u][k] = 0;
    uint32_t i = q;
    for (; i + 12 < c.nch; i += 16) {
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            size_t const base = size_t(s)*c.nch + i + 4*u;
#pragma unroll
            for (int k = 0; k < NC; ++k) acc4[u][k] += __ldcg(&c.part[(base*kSlots + k)*64 + j]);
        }
    }
    for (; i < c.nch; i += 4) {
        size_t const base = size_t(s)*c.nch + i;
#pragma unroll
        for (int k = 0; k < NC; ++k) acc4[0][k] += __ldcg(&c.part[(base*kSlots + k)*64 + j]);
    }
    double acc[NC];
#pragma unroll
    for (int k = 0; k < NC; ++k) acc[k] = ((acc4[0][k] + acc4[1][k]) + acc4[2][k]) + acc4[3][k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NC; ++k) red[q][j][k] = acc[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < NC; ++k) out[k] = ((red[0][j][k] + red[1][j][k]) + red[2][j][k]) + red[3][j][k];
    if (0 == threadIdx.x) c.tickets[s] = 0u;
    return true;
}

__device__ __forceinline__ void cdiv(double ar, double ai, double br, double bi, double &r, double &i) {
    double const d = br*br + bi*bi;
    r = (ar*br + ai*bi)/d; i = (ai*br - ar*bi)/d;
}

__device__ __forceinline__ void freeze(ColState &s) {
    s.al_re = s.al_im = s.be_re = s.be_im = 0;
    s.cu1x_re = s.cu1x_im = s.cu2x_re = s.cu2x_im = s.cdx_re = s.cdx_im = 0;
    s.cu1d_re = s.cu1d_im = s.cdd_re = s.cdd_im = 0;
    s.cup_re = s.cup_im = 0;
}

__device__ __forceinline__ void store_coef(Ctx const &c, uint32_t col, ColState const &s) {
    double const v[kCoef] = {s.al_re, s.al_im, s.be_re, s.be_im, s.cu1x_re, s.cu1x_im, s.cu2x_re, s.cu2x_im,
                             s.cdx_re, s.cdx_im, s.cu1d_re, s.cu1d_im, s.cdd_re, s.cdd_im};
#pragma unroll
    for (int i = 0; i < kCoef; ++i) { c.cd[size_t(i)*c.ncol + col] = v[i]; c.cf[size_t(i)*c.ncol + col] = float(v[i]); }
}

template <typename T> __device__ __forceinline__ T coef(Ctx const &c, int i, uint32_t col);
template <> __device__ __forceinline__ float coef<float>(Ctx const &c, int i, uint32_t col) { return c.cf[size_t(i)*c.ncol + col]; }
template <> __device__ __forceinline__ double coef<double>(Ctx const &c, int i, uint32_t col) { return c.cd[size_t(i)*c.ncol + col]; }

// ------------------------------------------------------------------ per-source steps
// Called by all threads of the last CTA of source s; thread j < 64 owns column s*64 + j.

// a source without active columns is done: counted once, and retired if retirement is on
__device__ void finish_source(Ctx const &c, uint32_t s, bool any_active, bool count_iteration) {
    if (0 != threadIdx.x) return;
    SrcState &src = c.ss[s];
    if (count_iteration) src.it += 1;
    if (!any_active && !src.done) {
        src.done = 1;
        atomicSub(&c.ctl->n_active, 1);
        if (c.retire) c.src_active[s] = 0;
    }
}

// r = |W|^2, rt^H W, rt^H V
__device__ void step_init(Ctx const &c, uint32_t s, double const (&r)[5]) {
    int const j = threadIdx.x;
    bool act = false;
    if (j < 64) {
        uint32_t const col = s*64 + j;
        ColState st{};
        double const bn = sqrt(r[0]);
        st.bnorm = bn; st.tau = bn; st.scale = 1; st.res = (bn > 0) ? 1.0 : 0.0;
        st.rho_re = r[1]; st.rho_im = r[2]; st.rhop_re = r[1]; st.rhop_im = r[2];
        double const sr = r[3], si = r[4];
        if (!(bn > 0)) { st.status = 3; freeze(st); }
        else if (sr*sr + si*si == 0.0 || r[1]*r[1] + r[2]*r[2] == 0.0) { st.status = 2; freeze(st); atomicAdd(&c.ctl->breakdowns, 1); }
        else { cdiv(st.rho_re, st.rho_im, sr, si, st.al_re, st.al_im); st.status = 0; }
        c.cs[col] = st;
        store_coef(c, col, st);
        act = (0 == st.status);
    }
    bool const any = __syncthreads_or(act);
    if (0 == threadIdx.x) {
        SrcState z{}; z.est_ref = 1.0; z.best = 1e300;
        c.ss[s] = z;
        c.upd[s] = 0;
    }
    __syncthreads();
    finish_source(c, s, any, false);
}

// first half step m = 2n-1: r = |w_{2n-1}|^2
__device__ void step_half1(Ctx const &c, uint32_t s, double const (&r)[1]) {
    int const j = threadIdx.x;
    if (j >= 64) return;
    uint32_t const col = s*64 + j;
    ColState st = c.cs[col];
    st.conv1 = 0;
    if (0 == st.status) {
        double const wn = sqrt(r[0]);
        int const m = st.m + 1;
        double const th = wn/st.tau;
        double const c2 = 1.0/(1.0 + th*th);
        double const tau = st.tau*th*sqrt(c2);
        // kd = theta_{m-1}^2 eta_{m-1} / alpha ; eta = c^2 alpha
        double kr, ki; cdiv(st.theta*st.theta*st.eta_re, st.theta*st.theta*st.eta_im, st.al_re, st.al_im, kr, ki);
        st.kd1_re = kr; st.kd1_im = ki;
        st.et1_re = c2*st.al_re; st.et1_im = c2*st.al_im;
        st.theta = th; st.tau = tau; st.m = m;
        st.eta_re = st.et1_re; st.eta_im = st.et1_im;
        if (!c.mixed && tau*sqrt(double(m) + 1.0) <= c.tol*(c.abs_tol ? 1.0 : st.bnorm)) st.conv1 = 1;
    }
    c.cs[col] = st;
}

// second half step m = 2n: r = |w_{2n}|^2, rt^H w_{2n}; coefficients of K_DX, beta; the
// replacement decision of the source (FP32 recurrences)
__device__ void step_half2(Ctx const &c, uint32_t s, double const (&r)[3]) {
    __shared__ double est_max[64];
    __shared__ int below[64];
    int const j = threadIdx.x;
    bool act = false;
    if (j < 64) {
        uint32_t const col = s*64 + j;
        ColState st = c.cs[col];
        double est = 0;
        if (0 != st.status) {
            freeze(st);
        } else if (st.conv1) {
            // X = X0 + et1 (U1 + kd1 D0); the column is done
            double const k1r = st.kd1_re, k1i = st.kd1_im, e1r = st.et1_re, e1i = st.et1_im;
            st.cu1x_re = e1r; st.cu1x_im = e1i; st.cu2x_re = st.cu2x_im = 0;
            st.cdx_re = e1r*k1r - e1i*k1i; st.cdx_im = e1r*k1i + e1i*k1r;
            st.cu1d_re = st.cu1d_im = st.cdd_re = st.cdd_im = 0;
            st.be_re = st.be_im = 0; st.al_re = st.al_im = 0;
            st.status = 1;
            st.res = st.tau*sqrt(double(st.m) + 1.0)/st.bnorm;
        } else {
            double const wn = sqrt(r[0]), rnr = r[1], rni = r[2];
            int const m = st.m + 1;
            double const k1r = st.kd1_re, k1i = st.kd1_im, e1r = st.et1_re, e1i = st.et1_im;
            double const th = wn/st.tau;
            double const c2 = 1.0/(1.0 + th*th);
            double const tau = st.tau*th*sqrt(c2);
            double k2r, k2i; cdiv(st.theta*st.theta*st.eta_re, st.theta*st.theta*st.eta_im, st.al_re, st.al_im, k2r, k2i);
            double const e2r = c2*st.al_re, e2i = c2*st.al_im;
            // D2 = U2 + kd2 D1 = U2 + kd2 U1 + kd2 kd1 D0
            // X2 = X0 + et1 D1 + et2 D2 = X0 + (et1 + et2 kd2) U1 + et2 U2 + (et1 kd1 + et2 kd2 kd1) D0
            double const kkr = k2r*k1r - k2i*k1i, kki = k2r*k1i + k2i*k1r;       // kd2 kd1
            double const ekr = e2r*k2r - e2i*k2i, eki = e2r*k2i + e2i*k2r;       // et2 kd2
            st.cu1x_re = e1r + ekr; st.cu1x_im = e1i + eki;
            st.cu2x_re = e2r; st.cu2x_im = e2i;
            double const a1r = e1r*k1r - e1i*k1i, a1i = e1r*k1i + e1i*k1r;       // et1 kd1
            double const a2r = e2r*kkr - e2i*kki, a2i = e2r*kki + e2i*kkr;       // et2 kd2 kd1
            st.cdx_re = a1r + a2r; st.cdx_im = a1i + a2i;
            st.cu1d_re = k2r; st.cu1d_im = k2i;
            st.cdd_re = kkr; st.cdd_im = kki;
            st.theta = th; st.tau = tau; st.eta_re = e2r; st.eta_im = e2i; st.m = m;
            st.cup_re = th*th*e2r; st.cup_im = th*th*e2i;
            // beta = rho_n / rho_{n-1}
            double br, bi; cdiv(rnr, rni, st.rho_re, st.rho_im, br, bi);
            st.rhop_re = st.rho_re; st.rhop_im = st.rho_im;
            st.be_re = br; st.be_im = bi; st.rho_re = rnr; st.rho_im = rni;
            double const bound = tau*sqrt(double(m) + 1.0);
            est = bound/st.bnorm*st.scale;
            if (!c.mixed && bound <= c.tol*(c.abs_tol ? 1.0 : st.bnorm)) {
                st.status = 1; st.be_re = st.be_im = 0; st.al_re = st.al_im = 0;
                st.res = bound/st.bnorm;
            } else if (rnr*rnr + rni*rni == 0.0) {
                st.status = 2; st.be_re = st.be_im = 0; st.al_re = st.al_im = 0; atomicAdd(&c.ctl->breakdowns, 1);
            }
        }
        c.cs[col] = st;
        store_coef(c, col, st);
        act = (0 == st.status);
        est_max[j] = act ? est : 0.0;
        below[j] = act ? (est <= c.tol) : 1;
    }
    if (!c.mixed) return;
    bool const any = __syncthreads_or(act);
    if (0 == threadIdx.x) {
        double e = 0; int all = 1;
        for (int k = 0; k < 64; ++k) { e = fmax(e, est_max[k]); all &= below[k]; }
        SrcState &src = c.ss[s];
        int const u = any && (e < c.delta*src.est_ref || all || src.since + 1 >= c.gap);
        src.upd = u;
        c.upd[s] = uint8_t(u);
    }
}

// end of an iteration: r = rt^H v_n; alpha = rho / (rt^H v_n)
__device__ void step_alpha(Ctx const &c, uint32_t s, double const (&r)[2]) {
    int const j = threadIdx.x;
    bool act = false;
    if (j < 64) {
        uint32_t const col = s*64 + j;
        ColState st = c.cs[col];
        double const sr = r[0], si = r[1];
        if (0 != st.status) freeze(st);
        else if (sr*sr + si*si == 0.0) { st.status = 2; freeze(st); atomicAdd(&c.ctl->breakdowns, 1); }
        else cdiv(st.rho_re, st.rho_im, sr, si, st.al_re, st.al_im);
        c.cs[col] = st;
        store_coef(c, col, st);
        act = (0 == st.status);
    }
    bool const any = __syncthreads_or(act);
    if (0 == threadIdx.x) {
        SrcState &src = c.ss[s];
        src.since = src.upd ? 0 : src.since + 1;
        src.upd = 0;
        c.upd[s] = 0;
    }
    finish_source(c, s, any, true);
}

// residual replacement: r = |B - A X64|^2, rt^H W with the new W
__device__ void step_replace(Ctx const &c, uint32_t s, double const (&r)[3]) {
    __shared__ double resmax[64];
    int const j = threadIdx.x;
    bool act = false;
    if (j < 64) {
        uint32_t const col = s*64 + j;
        ColState st = c.cs[col];
        double const res = (st.bnorm > 0) ? sqrt(r[0])/st.bnorm : 0.0;
        if (0 == st.status) {
            st.res = res;
            if (res <= c.tol) {
                st.status = 1; freeze(st);
            } else {
                double const est = st.tau*sqrt(double(st.m) + 1.0)/st.bnorm;
                st.scale = fmax(1.0, res/fmax(est, 1e-300));
                double const rnr = r[1], rni = r[2];
                if (rnr*rnr + rni*rni == 0.0) {
                    st.status = 2; freeze(st); atomicAdd(&c.ctl->breakdowns, 1);
                } else {
                    double br, bi; cdiv(rnr, rni, st.rhop_re, st.rhop_im, br, bi);
                    st.be_re = br; st.be_im = bi; st.rho_re = rnr; st.rho_im = rni;
                }
            }
        }
        c.cs[col] = st;
        store_coef(c, col, st);
        act = (0 == st.status);
        resmax[j] = act ? res : 0.0;
    }
    bool any = __syncthreads_or(act);
    __shared__ int fb;
    if (0 == threadIdx.x) {
        double e = 0;
        bool finite = true;
        for (int k = 0; k < 64; ++k) { e = fmax(e, resmax[k]); finite = finite && isfinite(resmax[k]); }
        SrcState &src = c.ss[s];
        src.est_ref = e;
        src.updates += 1;
        // progress: the largest true residual halved since the best one so far (slower progress
        // is slower than the FP64 recurrences, whose iterations cost 2.7 times as much)
        if (e < 0.5*src.best) { src.best = e; src.stall = 0; } else src.stall += 1;
        fb = any && (!finite || src.stall >= c.stall_limit);
        if (fb) { src.fallback = 1; src.nonfinite = !finite; }
    }
    __syncthreads();
    if (fb) {
        // the FP32 recurrences stopped making progress: the active columns continue in FP64
        if (j < 64) {
            ColState &st = c.cs[s*64 + j];
            if (0 == st.status) { st.status = 5; freeze(st); store_coef(c, s*64 + j, st); }
        }
        any = false;
    }
    // a source that finished here is retired now; its last iteration counts
    finish_source(c, s, any, !any);
}

// final true residuals: r = |B - A X|^2
__device__ void step_final(Ctx const &c, uint32_t s, double const (&r)[1]) {
    int const j = threadIdx.x;
    if (j >= 64) return;
    uint32_t const col = s*64 + j;
    c.cs[col].res = sqrt(r[0]);      // |b| = 1: the right-hand sides are unit columns
}

// ------------------------------------------------------------------ vector kernels
// one CTA of 256 threads per unit; thread (q, j): column j, rows q*16 .. q*16+15, re and im

template <typename T>
__global__ void k_set_diag(T *W, T *U1, uint32_t const *subset, uint32_t ncols_blk) {
    uint32_t const c = blockIdx.x; int const i = threadIdx.x;
    if (c < ncols_blk) {
        size_t const o = size_t(subset[c])*kBlk + size_t(i)*64 + i;
        W[o] = T(1); U1[o] = T(1);
    }
}

// initial reductions: |W|^2, rt^H W, rt^H V
template <typename T>
__global__ void __launch_bounds__(256) k_init_dots(T const *W, T const *V, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    double v[5] = {0, 0, 0, 0, 0};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
#pragma unroll 4
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            uint32_t const idx = uint32_t(o);
            double const tr = double(shadow_t<T>(c.seed, idx)), ti = double(shadow_t<T>(c.seed, idx + 4096u));
            double const xr = W[o], xi = W[o + 4096], yr = V[o], yi = V[o + 4096];
            v[0] += xr*xr + xi*xi;
            v[1] += tr*xr + ti*xi; v[2] += tr*xi - ti*xr;     // conj(rt) w
            v[3] += tr*yr + ti*yi; v[4] += tr*yi - ti*yr;
        }
    }
    double out[5];
    if (reduce_source<5>(c, blockIdx.x, s, v, out)) step_init(c, s, out);
}

// K_A: U2 = U1 - alpha V ; |W - alpha AU1|^2
template <typename T>
__global__ void __launch_bounds__(256) k_A(T *U2, T const *U1, T const *V, T const *W, T const *AU1, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    uint32_t const col = s*64 + j;
    T const ar = coef<T>(c, 0, col), ai = coef<T>(c, 1, col);
    double n2 = 0;
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        T n2t = T(0);                 // 16-row partial sums in the vector precision
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            T const vr = V[o], vi = V[o + 4096];
            U2[o] = fma(ai, vi, fma(-ar, vr, U1[o]));
            U2[o + 4096] = fma(-ai, vr, fma(-ar, vi, U1[o + 4096]));
            T const ur = AU1[o], ui = AU1[o + 4096];
            T const wr = fma(ai, ui, fma(-ar, ur, W[o])), wi = fma(-ai, ur, fma(-ar, ui, W[o + 4096]));
            n2t = fma(wr, wr, fma(wi, wi, n2t));
        }
        n2 += double(n2t);
    }
    double const v[1] = {n2};
    double out[1];
    if (reduce_source<1>(c, blockIdx.x, s, v, out)) step_half1(c, s, out);
}

// K_C: W = W - alpha (AU1 + AU2) ; |W|^2 and rt^H W
template <typename T>
__global__ void __launch_bounds__(256) k_C(T *W, T const *AU1, T const *AU2, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    uint32_t const col = s*64 + j;
    T const ar = coef<T>(c, 0, col), ai = coef<T>(c, 1, col);
    double v[3] = {0, 0, 0};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        T n2 = T(0), dr = T(0), di = T(0);
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            T const sr = AU1[o] + AU2[o], si = AU1[o + 4096] + AU2[o + 4096];
            T const wr = fma(ai, si, fma(-ar, sr, W[o])), wi = fma(-ai, sr, fma(-ar, si, W[o + 4096]));
            W[o] = wr; W[o + 4096] = wi;
            uint32_t const idx = uint32_t(o);
            T const tr = shadow_t<T>(c.seed, idx), ti = shadow_t<T>(c.seed, idx + 4096u);
            n2 = fma(wr, wr, fma(wi, wi, n2));
            dr = fma(tr, wr, fma(ti, wi, dr)); di = fma(tr, wi, fma(-ti, wr, di));
        }
        v[0] += double(n2); v[1] += double(dr); v[2] += double(di);
    }
    double out[3];
    if (reduce_source<3>(c, blockIdx.x, s, v, out)) step_half2(c, s, out);
}

// K_DX: X += cu1x U1 + cu2x U2 + cdx D ; D = U2 + cu1d U1 + cdd D ; U1 = W + beta U2
template <typename T>
__global__ void __launch_bounds__(256) k_DX(T *X, T *D, T *U1, T const *U2, T const *W, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    uint32_t const col = s*64 + j;
    T const g_r = coef<T>(c, 2, col), g_i = coef<T>(c, 3, col);
    T const a_r = coef<T>(c, 4, col), a_i = coef<T>(c, 5, col);
    T const b_r = coef<T>(c, 6, col), b_i = coef<T>(c, 7, col);
    T const c_r = coef<T>(c, 8, col), c_i = coef<T>(c, 9, col);
    T const d_r = coef<T>(c, 10, col), d_i = coef<T>(c, 11, col);
    T const e_r = coef<T>(c, 12, col), e_i = coef<T>(c, 13, col);
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
#pragma unroll 4
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            T const u1r = U1[o], u1i = U1[o + 4096], u2r = U2[o], u2i = U2[o + 4096];
            T const dr = D[o], di = D[o + 4096];
            T xr = X[o], xi = X[o + 4096];
            xr = fma(a_r, u1r, fma(-a_i, u1i, xr)); xi = fma(a_r, u1i, fma(a_i, u1r, xi));
            xr = fma(b_r, u2r, fma(-b_i, u2i, xr)); xi = fma(b_r, u2i, fma(b_i, u2r, xi));
            xr = fma(c_r, dr, fma(-c_i, di, xr));   xi = fma(c_r, di, fma(c_i, dr, xi));
            X[o] = xr; X[o + 4096] = xi;
            D[o] = fma(d_r, u1r, fma(-d_i, u1i, fma(e_r, dr, fma(-e_i, di, u2r))));
            D[o + 4096] = fma(d_r, u1i, fma(d_i, u1r, fma(e_r, di, fma(e_i, dr, u2i))));
            U1[o] = fma(g_r, u2r, fma(-g_i, u2i, W[o]));
            U1[o + 4096] = fma(g_r, u2i, fma(g_i, u2r, W[o + 4096]));
        }
    }
}

// K_DX in FP32 with 16-byte accesses: thread (column group of 4, row group of 4 rows); each row
// moves 10 float4 loads and 6 float4 stores
__device__ __forceinline__ float4 ld4(float const *p) { return *reinterpret_cast<float4 const*>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4*>(p) = v; }
__device__ __forceinline__ float4 ldc4(Ctx const &c, int i, uint32_t col) { return ld4(c.cf + size_t(i)*c.ncol + col); }

__global__ void __launch_bounds__(256, 2) k_DX32(float *X, float *D, float *U1, float const *U2, float const *W,
                                                 Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const cg = threadIdx.x & 15, rg = threadIdx.x >> 4;
    int const j0 = cg*4;
    uint32_t const col = s*64 + j0;
    float4 const g_r = ldc4(c, 2, col), g_i = ldc4(c, 3, col);
    float4 const a_r = ldc4(c, 4, col), a_i = ldc4(c, 5, col);
    float4 const b_r = ldc4(c, 6, col), b_i = ldc4(c, 7, col);
    float4 const c_r = ldc4(c, 8, col), c_i = ldc4(c, 9, col);
    float4 const d_r = ldc4(c, 10, col), d_i = ldc4(c, 11, col);
    float4 const e_r = ldc4(c, 12, col), e_i = ldc4(c, 13, col);
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
#pragma unroll 2
        for (int i = rg*4; i < rg*4 + 4; ++i) {
            size_t const o = b*kBlk + i*64 + j0;
            float4 const u1r = ld4(U1 + o), u1i = ld4(U1 + o + 4096), u2r = ld4(U2 + o), u2i = ld4(U2 + o + 4096);
            float4 const dr = ld4(D + o), di = ld4(D + o + 4096), wr = ld4(W + o), wi = ld4(W + o + 4096);
            float4 xr = ld4(X + o), xi = ld4(X + o + 4096);
            float4 nd_r, nd_i, nu_r, nu_i;
#define A43G_DX_LANE(f) \
            xr.f = fmaf(a_r.f, u1r.f, fmaf(-a_i.f, u1i.f, xr.f)); xi.f = fmaf(a_r.f, u1i.f, fmaf(a_i.f, u1r.f, xi.f)); \
            xr.f = fmaf(b_r.f, u2r.f, fmaf(-b_i.f, u2i.f, xr.f)); xi.f = fmaf(b_r.f, u2i.f, fmaf(b_i.f, u2r.f, xi.f)); \
            xr.f = fmaf(c_r.f, dr.f, fmaf(-c_i.f, di.f, xr.f));   xi.f = fmaf(c_r.f, di.f, fmaf(c_i.f, dr.f, xi.f)); \
            nd_r.f = fmaf(d_r.f, u1r.f, fmaf(-d_i.f, u1i.f, fmaf(e_r.f, dr.f, fmaf(-e_i.f, di.f, u2r.f)))); \
            nd_i.f = fmaf(d_r.f, u1i.f, fmaf(d_i.f, u1r.f, fmaf(e_r.f, di.f, fmaf(e_i.f, dr.f, u2i.f)))); \
            nu_r.f = fmaf(g_r.f, u2r.f, fmaf(-g_i.f, u2i.f, wr.f)); \
            nu_i.f = fmaf(g_r.f, u2i.f, fmaf(g_i.f, u2r.f, wi.f));
            A43G_DX_LANE(x) A43G_DX_LANE(y) A43G_DX_LANE(z) A43G_DX_LANE(w)
#undef A43G_DX_LANE
            st4(X + o, xr); st4(X + o + 4096, xi);
            st4(D + o, nd_r); st4(D + o + 4096, nd_i);
            st4(U1 + o, nu_r); st4(U1 + o + 4096, nu_i);
        }
    }
}

// K_E: V = AU1 + beta (AU2 + beta V) ; rt^H V
template <typename T>
__global__ void __launch_bounds__(256) k_E(T *V, T const *AU1, T const *AU2, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    uint32_t const col = s*64 + j;
    T const fr = coef<T>(c, 2, col), fi = coef<T>(c, 3, col);
    double v[2] = {0, 0};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        T dr = T(0), di = T(0);
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            T const vr = V[o], vi = V[o + 4096];
            T const t1r = fma(-fi, vi, fma(fr, vr, AU2[o])), t1i = fma(fi, vr, fma(fr, vi, AU2[o + 4096]));
            T const sr = fma(-fi, t1i, fma(fr, t1r, AU1[o])), si = fma(fi, t1r, fma(fr, t1i, AU1[o + 4096]));
            V[o] = sr; V[o + 4096] = si;
            uint32_t const idx = uint32_t(o);
            T const tr = shadow_t<T>(c.seed, idx), ti = shadow_t<T>(c.seed, idx + 4096u);
            dr = fma(tr, sr, fma(ti, si, dr)); di = fma(tr, si, fma(-ti, sr, di));
        }
        v[0] += double(dr); v[1] += double(di);
    }
    double out[2];
    if (reduce_source<2>(c, blockIdx.x, s, v, out)) step_alpha(c, s, out);
}

// ------------------------------------------------------------------ 16-byte vector kernels
// K_A, K_C and K_E with 16-byte accesses (the scalar kernels above move 4 or 8 bytes per thread
// and access): thread (row group rg, column group cg) owns N = 16/sizeof(T) consecutive columns
// of RP rows of every block of its unit.  The column sums of the row groups are folded in a fixed
// order into the (q, j) layout of reduce_source, so the results are reproducible.
template <typename T> struct Lanes {
    static constexpr int N = 16/int(sizeof(T));       // columns per thread
    static constexpr int CG = 64/N, RG = 256/CG;       // column groups, row groups
    static constexpr int RP = 64/RG;                   // rows per thread and block
    T v[N];
};
template <typename T> __device__ __forceinline__ Lanes<T> ldl(T const *p) {
    Lanes<T> r;
    if constexpr (sizeof(T) == 4) { float4 const a = *reinterpret_cast<float4 const*>(p); r.v[0] = a.x; r.v[1] = a.y; r.v[2] = a.z; r.v[3] = a.w; }
    else { double2 const a = *reinterpret_cast<double2 const*>(p); r.v[0] = a.x; r.v[1] = a.y; }
    return r;
}
template <typename T> __device__ __forceinline__ void stl(T *p, Lanes<T> const &r) {
    if constexpr (sizeof(T) == 4) *reinterpret_cast<float4*>(p) = make_float4(r.v[0], r.v[1], r.v[2], r.v[3]);
    else *reinterpret_cast<double2*>(p) = make_double2(r.v[0], r.v[1]);
}
template <typename T> __device__ __forceinline__ Lanes<T> coefl(Ctx const &c, int i, uint32_t col) {
    if constexpr (sizeof(T) == 4) return ldl<float>(c.cf + size_t(i)*c.ncol + col);
    else return ldl<double>(c.cd + size_t(i)*c.ncol + col);
}

// a[n][k]: this thread's sums of its column n; v[k]: thread (q, j)'s share for reduce_source
template <typename T, int NC>
__device__ __forceinline__ void fold_lanes(double const (&a)[Lanes<T>::N][NC], double (&v)[NC]) {
    using L = Lanes<T>;
    __shared__ double sm[L::RG][64][NC];
    int const cg = threadIdx.x % L::CG, rg = threadIdx.x/L::CG;
#pragma unroll
    for (int n = 0; n < L::N; ++n)
#pragma unroll
        for (int k = 0; k < NC; ++k) sm[rg][cg*L::N + n][k] = a[n][k];
    __syncthreads();
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    constexpr int PER = L::RG/4;                       // row groups per q
#pragma unroll
    for (int k = 0; k < NC; ++k) {
        double t = sm[q*PER][j][k];
#pragma unroll
        for (int r = 1; r < PER; ++r) t += sm[q*PER + r][j][k];
        v[k] = t;
    }
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_A16(T *U2, T const *U1, T const *V, T const *W, T const *AU1, Ctx const c) {
    using L = Lanes<T>;
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const cg = threadIdx.x % L::CG, rg = threadIdx.x/L::CG, j0 = cg*L::N;
    uint32_t const col = s*64 + j0;
    L const ar = coefl<T>(c, 0, col), ai = coefl<T>(c, 1, col);
    double a[L::N][1] = {};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        T n2[L::N] = {};
#pragma unroll 2
        for (int i = rg*L::RP; i < rg*L::RP + L::RP; ++i) {
            size_t const o = b*kBlk + i*64 + j0;
            L const vr = ldl(V + o), vi = ldl(V + o + 4096), u1r = ldl(U1 + o), u1i = ldl(U1 + o + 4096);
            L const ur = ldl(AU1 + o), ui = ldl(AU1 + o + 4096), wr = ldl(W + o), wi = ldl(W + o + 4096);
            L u2r, u2i;
#pragma unroll
            for (int n = 0; n < L::N; ++n) {
                u2r.v[n] = fma(ai.v[n], vi.v[n], fma(-ar.v[n], vr.v[n], u1r.v[n]));
                u2i.v[n] = fma(-ai.v[n], vr.v[n], fma(-ar.v[n], vi.v[n], u1i.v[n]));
                T const xr = fma(ai.v[n], ui.v[n], fma(-ar.v[n], ur.v[n], wr.v[n]));
                T const xi = fma(-ai.v[n], ur.v[n], fma(-ar.v[n], ui.v[n], wi.v[n]));
                n2[n] = fma(xr, xr, fma(xi, xi, n2[n]));
            }
            stl(U2 + o, u2r); stl(U2 + o + 4096, u2i);
        }
#pragma unroll
        for (int n = 0; n < L::N; ++n) a[n][0] += double(n2[n]);
    }
    double v[1], out[1];
    fold_lanes<T, 1>(a, v);
    if (reduce_source<1>(c, blockIdx.x, s, v, out)) step_half1(c, s, out);
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_C16(T *W, T const *AU1, T const *AU2, Ctx const c) {
    using L = Lanes<T>;
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const cg = threadIdx.x % L::CG, rg = threadIdx.x/L::CG, j0 = cg*L::N;
    uint32_t const col = s*64 + j0;
    L const ar = coefl<T>(c, 0, col), ai = coefl<T>(c, 1, col);
    double a[L::N][3] = {};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        T n2[L::N] = {}, dr[L::N] = {}, di[L::N] = {};
#pragma unroll 2
        for (int i = rg*L::RP; i < rg*L::RP + L::RP; ++i) {
            size_t const o = b*kBlk + i*64 + j0;
            L const a1r = ldl(AU1 + o), a1i = ldl(AU1 + o + 4096), a2r = ldl(AU2 + o), a2i = ldl(AU2 + o + 4096);
            L wr = ldl(W + o), wi = ldl(W + o + 4096);
#pragma unroll
            for (int n = 0; n < L::N; ++n) {
                T const sr = a1r.v[n] + a2r.v[n], si = a1i.v[n] + a2i.v[n];
                T const xr = fma(ai.v[n], si, fma(-ar.v[n], sr, wr.v[n]));
                T const xi = fma(-ai.v[n], sr, fma(-ar.v[n], si, wi.v[n]));
                wr.v[n] = xr; wi.v[n] = xi;
                uint32_t const idx = uint32_t(o) + uint32_t(n);
                T const tr = shadow_t<T>(c.seed, idx), ti = shadow_t<T>(c.seed, idx + 4096u);
                n2[n] = fma(xr, xr, fma(xi, xi, n2[n]));
                dr[n] = fma(tr, xr, fma(ti, xi, dr[n])); di[n] = fma(tr, xi, fma(-ti, xr, di[n]));
            }
            stl(W + o, wr); stl(W + o + 4096, wi);
        }
#pragma unroll
        for (int n = 0; n < L::N; ++n) { a[n][0] += double(n2[n]); a[n][1] += double(dr[n]); a[n][2] += double(di[n]); }
    }
    double v[3], out[3];
    fold_lanes<T, 3>(a, v);
    if (reduce_source<3>(c, blockIdx.x, s, v, out)) step_half2(c, s, out);
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_E16(T *V, T const *AU1, T const *AU2, Ctx const c) {
    using L = Lanes<T>;
    uint32_t s, lo, hi;
    if (!unit_range(c, c.active, blockIdx.x, s, lo, hi)) return;
    int const cg = threadIdx.x % L::CG, rg = threadIdx.x/L::CG, j0 = cg*L::N;
    uint32_t const col = s*64 + j0;
    L const fr = coefl<T>(c, 2, col), fi = coefl<T>(c, 3, col);
    double a[L::N][2] = {};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        T dr[L::N] = {}, di[L::N] = {};
#pragma unroll 2
        for (int i = rg*L::RP; i < rg*L::RP + L::RP; ++i) {
            size_t const o = b*kBlk + i*64 + j0;
            L vr = ldl(V + o), vi = ldl(V + o + 4096);
            L const a1r = ldl(AU1 + o), a1i = ldl(AU1 + o + 4096), a2r = ldl(AU2 + o), a2i = ldl(AU2 + o + 4096);
#pragma unroll
            for (int n = 0; n < L::N; ++n) {
                T const t1r = fma(-fi.v[n], vi.v[n], fma(fr.v[n], vr.v[n], a2r.v[n]));
                T const t1i = fma(fi.v[n], vr.v[n], fma(fr.v[n], vi.v[n], a2i.v[n]));
                T const sr = fma(-fi.v[n], t1i, fma(fr.v[n], t1r, a1r.v[n]));
                T const si = fma(fi.v[n], t1r, fma(fr.v[n], t1i, a1i.v[n]));
                vr.v[n] = sr; vi.v[n] = si;
                uint32_t const idx = uint32_t(o) + uint32_t(n);
                T const tr = shadow_t<T>(c.seed, idx), ti = shadow_t<T>(c.seed, idx + 4096u);
                dr[n] = fma(tr, sr, fma(ti, si, dr[n])); di[n] = fma(tr, si, fma(-ti, sr, di[n]));
            }
            stl(V + o, vr); stl(V + o + 4096, vi);
        }
#pragma unroll
        for (int n = 0; n < L::N; ++n) { a[n][0] += double(dr[n]); a[n][1] += double(di[n]); }
    }
    double v[2], out[2];
    fold_lanes<T, 2>(a, v);
    if (reduce_source<2>(c, blockIdx.x, s, v, out)) step_alpha(c, s, out);
}

// ------------------------------------------------------------------ residual replacement
// (FP32 recurrences; the units of sources without a replacement in this iteration return at once)

// X64 += X32, X32 = 0
__global__ void __launch_bounds__(256) k_flush(double *X64, float *X32, Ctx const c, uint8_t const *sel) {
    uint32_t s, lo, hi;
    if (!unit_range(c, sel, blockIdx.x, s, lo, hi)) return;
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        for (int t = threadIdx.x; t < kBlk/4; t += blockDim.x) {
            float4 const x = ld4(X32 + b*kBlk + 4*t);
            double2 *p = reinterpret_cast<double2*>(X64 + b*kBlk + 4*t);
            double2 a = p[0], d = p[1];
            a.x += x.x; a.y += x.y; d.x += x.z; d.y += x.w;
            p[0] = a; p[1] = d;
            st4(X32 + b*kBlk + 4*t, make_float4(0.f, 0.f, 0.f, 0.f));
        }
    }
}

// R = B - AX64 (B: unit diagonal block of the source); W = R - cup AD; |R|^2 and rt^H W
__global__ void __launch_bounds__(256) k_replace(float *W, double const *AX64, float const *AD, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.upd, blockIdx.x, s, lo, hi)) return;
    if (c.active && !c.active[s]) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    uint32_t const col = s*64 + j;
    double const pr = c.cs[col].cup_re, pi = c.cs[col].cup_im;
    uint32_t const diag = c.subset[s];
    double v[3] = {0, 0, 0};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        bool const isdiag = (b == diag);
#pragma unroll 4
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            double const rr = ((isdiag && i == j) ? 1.0 : 0.0) - AX64[o], ri = -AX64[o + 4096];
            double const dr = AD[o], di = AD[o + 4096];
            float const wr = float(rr - (pr*dr - pi*di)), wi = float(ri - (pr*di + pi*dr));
            W[o] = wr; W[o + 4096] = wi;
            uint32_t const idx = uint32_t(o);
            double const tr = shadow32(c.seed, idx), ti = shadow32(c.seed, idx + 4096u);
            v[0] += rr*rr + ri*ri;
            v[1] += tr*double(wr) + ti*double(wi); v[2] += tr*double(wi) - ti*double(wr);
        }
    }
    double out[3];
    if (reduce_source<3>(c, blockIdx.x, s, v, out)) step_replace(c, s, out);
}

// U1 = W + beta U2 after a replacement (the new beta)
__global__ void __launch_bounds__(256) k_U1(float *U1, float const *W, float const *U2, Ctx const c) {
    uint32_t s, lo, hi;
    if (!unit_range(c, c.upd, blockIdx.x, s, lo, hi)) return;
    if (c.active && !c.active[s]) return;
    int const cg = threadIdx.x & 15, rg = threadIdx.x >> 4;
    uint32_t const col = s*64 + cg*4;
    float4 const g_r = ldc4(c, 2, col), g_i = ldc4(c, 3, col);
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        for (int i = rg*4; i < rg*4 + 4; ++i) {
            size_t const o = b*kBlk + i*64 + cg*4;
            float4 const u2r = ld4(U2 + o), u2i = ld4(U2 + o + 4096), wr = ld4(W + o), wi = ld4(W + o + 4096);
            float4 nr, ni;
#define A43G_U1_LANE(f) nr.f = fmaf(g_r.f, u2r.f, fmaf(-g_i.f, u2i.f, wr.f)); ni.f = fmaf(g_r.f, u2i.f, fmaf(g_i.f, u2r.f, wi.f));
            A43G_U1_LANE(x) A43G_U1_LANE(y) A43G_U1_LANE(z) A43G_U1_LANE(w)
#undef A43G_U1_LANE
            st4(U1 + o, nr); st4(U1 + o + 4096, ni);
        }
    }
}

// |B - AX|^2 per column of every source (final residuals; AX in FP64)
__global__ void __launch_bounds__(256) k_final(double const *AX, Ctx const c, uint8_t const *sel) {
    uint32_t s, lo, hi;
    if (!unit_range(c, sel, blockIdx.x, s, lo, hi)) return;
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    uint32_t const diag = c.subset[s];
    double v[1] = {0};
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        bool const isdiag = (b == diag);
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = b*kBlk + i*64 + j;
            double const rr = ((isdiag && i == j) ? 1.0 : 0.0) - AX[o], ri = -AX[o + 4096];
            v[0] += rr*rr + ri*ri;
        }
    }
    double out[1];
    if (reduce_source<1>(c, blockIdx.x, s, v, out)) step_final(c, s, out);
}

// FP64 continuation of the sources flagged in sel: W = U1 = B - AX, with a source whose FP64
// solution is not finite restarted from zero (W = U1 = B, X = 0)
__global__ void __launch_bounds__(256) k_start64(double *W, double *U1, double *X, double const *AX, Ctx const c,
                                                 uint8_t const *sel) {
    uint32_t s, lo, hi;
    if (!unit_range(c, sel, blockIdx.x, s, lo, hi)) return;
    uint32_t const diag = c.subset[s];
    int const bad = c.ss[s].nonfinite;               // the FP32 phase's record, uniform
    for (uint32_t k = lo; k < hi; ++k) {
        size_t const b = c.src_blocks[k];
        bool const isdiag = (b == diag);
        for (int t = threadIdx.x; t < kBlk; t += blockDim.x) {
            int const reim = t >> 12, i = (t >> 6) & 63, j = t & 63;
            double const one = (isdiag && 0 == reim && i == j) ? 1.0 : 0.0;
            double const r = bad ? one : one - AX[b*kBlk + t];
            W[b*kBlk + t] = r; U1[b*kBlk + t] = r;
            if (bad) X[b*kBlk + t] = 0.0;
        }
    }
}

// sums[0] += |X64 + X32 - Xref|^2, sums[1] += |Xref|^2 over all blocks (X32 may be null)
__global__ void __launch_bounds__(256) k_trace(double const *X64, float const *X32, double const *Xref, size_t n,
                                               double *sums) {
    double e = 0, r = 0;
    for (size_t i = size_t(blockIdx.x)*blockDim.x + threadIdx.x; i < n; i += size_t(gridDim.x)*blockDim.x) {
        double const x = X64[i] + (X32 ? double(X32[i]) : 0.0), y = Xref[i];
        e += (x - y)*(x - y); r += y*y;
    }
    __shared__ double se[8], sr[8];
    for (int o = 16; o > 0; o >>= 1) { e += __shfl_xor_sync(0xffffffffu, e, o); r += __shfl_xor_sync(0xffffffffu, r, o); }
    if (0 == (threadIdx.x & 31)) { se[threadIdx.x >> 5] = e; sr[threadIdx.x >> 5] = r; }
    __syncthreads();
    if (0 == threadIdx.x) {
        double a = 0, b = 0;
        for (int w = 0; w < 8; ++w) { a += se[w]; b += sr[w]; }
        atomicAdd(sums, a); atomicAdd(sums + 1, b);   // a diagnostic: the summation order may vary
    }
}

// rho[c][i] = X[subset[c]][re, im][i][i] / pi
template <typename T>
__global__ void k_export_rho(double *rho, T const *X, uint32_t const *subset, uint32_t ncols_blk) {
    uint32_t const c = blockIdx.x; int const i = threadIdx.x;
    if (c >= ncols_blk) return;
    size_t const o = size_t(subset[c])*kBlk + size_t(i)*64 + i;
    double const f = 1.0/3.14159265358979323846;
    rho[2*(size_t(c)*64 + i)] = double(X[o])*f;
    rho[2*(size_t(c)*64 + i) + 1] = double(X[o + 4096])*f;
}

// chunks per source: at least one CTA per SM for a lone source, about eight per SM in total
uint32_t chunks_for(DevicePlan const &dp) {
    uint32_t const n = std::max(1u, dp.nCols);
    uint32_t const want = std::max<uint32_t>(148u, (148u*8u + n - 1)/n);
    return std::max(1u, std::min(want, std::max(1u, dp.max_src_blocks)));
}

} // namespace

bool TfqmrVectors::alloc(size_t nreals, size_t elem_bytes, bool with_x) {
    if (n == nreals && elem == elem_bytes && W.ptr && (!with_x || X.ptr)) return true;
    n = nreals; elem = elem_bytes;
    size_t const b = std::max<size_t>(16, nreals*elem_bytes);
    if (!with_x) X.release();
    return (!with_x || X.alloc(b)) && W.alloc(b) && U1.alloc(b) && U2.alloc(b) && V.alloc(b) && D.alloc(b) &&
           AU1.alloc(b) && AU2.alloc(b);
}

void TfqmrVectors::release() {
    X.release(); W.release(); U1.release(); U2.release(); V.release(); D.release();
    AU1.release(); AU2.release(); n = 0; elem = 0;
}

SolverWorkspace::~SolverWorkspace() {
    if (host_ctl) cudaFreeHost(host_ctl);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
}

namespace {

// restores the plan's retirement state (all sources active, retirement off) on every exit
struct RetireGuard {
    DevicePlan &dp;
    cudaStream_t st;
    ~RetireGuard() {
        dp.retire = false;
        if (dp.src_active.ptr) cudaMemsetAsync(dp.src_active.ptr, 1, std::max<uint32_t>(dp.nCols, 1), st);
    }
};

struct Prepared {
    Ctx c;
    uint32_t units = 0;
};

bool prepare(DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt, bool mixed, bool retire,
             Prepared &p) {
    uint32_t const nsrc = dp.nCols, ncol = nsrc*64;
    uint32_t const nch = chunks_for(dp);
    uint32_t const units = nsrc*nch;
    auto r256 = [](size_t n) { return (n + 255) & ~size_t(255); };
    size_t const bytes = r256(size_t(ncol)*sizeof(ColState)) + r256(size_t(ncol)*kCoef*sizeof(double)) +
                         r256(size_t(ncol)*kCoef*sizeof(float)) + r256(size_t(nsrc)*sizeof(SrcState)) +
                         r256(nsrc) + r256(sizeof(Ctl));
    if (!ws.state.alloc(bytes)) return false;
    if (!ws.part.alloc(std::max<size_t>(16, size_t(units)*kSlots*64*sizeof(double)))) return false;
    if (!ws.tickets.alloc(std::max<size_t>(16, size_t(nsrc)*sizeof(uint32_t)))) return false;
    if (!ws.host_ctl) A43G_CUDA_TRY(cudaMallocHost(&ws.host_ctl, 64));
    if (!ws.ev0) { A43G_CUDA_TRY(cudaEventCreate(&ws.ev0)); A43G_CUDA_TRY(cudaEventCreate(&ws.ev1)); }
    char *q = static_cast<char*>(ws.state.ptr);
    auto take = [&](size_t n) { char *r = q; q += (n + 255) & ~size_t(255); return r; };
    Ctx &c = p.c;
    c = Ctx{};
    c.cs = reinterpret_cast<ColState*>(take(size_t(ncol)*sizeof(ColState)));
    c.cd = reinterpret_cast<double*>(take(size_t(ncol)*kCoef*sizeof(double)));
    c.cf = reinterpret_cast<float*>(take(size_t(ncol)*kCoef*sizeof(float)));
    c.ss = reinterpret_cast<SrcState*>(take(size_t(nsrc)*sizeof(SrcState)));
    c.upd = reinterpret_cast<uint8_t*>(take(nsrc));
    c.ctl = reinterpret_cast<Ctl*>(take(sizeof(Ctl)));
    c.src_start = dptr<uint32_t>(dp.src_start);
    c.src_blocks = dptr<uint32_t>(dp.src_blocks);
    c.subset = dptr<uint32_t>(dp.subset_dev);
    c.src_active = dptr<uint8_t>(dp.src_active);
    c.active = retire ? c.src_active : nullptr;
    c.nch = nch; c.ncol = ncol;
    c.part = dptr<double>(ws.part);
    c.tickets = dptr<uint32_t>(ws.tickets);
    c.seed = uint32_t(opt.seed*2654435761ull + 12345u);
    c.tol = opt.tolerance;
    c.delta = (opt.update_factor > 0 && opt.update_factor < 1) ? opt.update_factor : 0.1;
    c.gap = (opt.update_gap > 0) ? opt.update_gap : 10;
    c.mixed = mixed ? 1 : 0;
    c.retire = retire ? 1 : 0;
    c.stall_limit = 3;
    {
        // vector kernels with 16-byte accesses (default) or the scalar ones ("0")
        char const *v = std::getenv("A43G_VEC16");
        c.vec16 = (v && 0 == std::strcmp(v, "0")) ? 0 : 1;
    }
    c.abs_tol = 0;
    p.units = units;
    return true;
}

// the operator on the solver's vectors with the source selection `sel` (nullptr: all sources)
template <typename T>
bool apply(DevicePlan &dp, T *y, T const *x, uint8_t const *sel, bool retire, cudaStream_t st) {
    // the action's kernels read DevicePlan::src_active when retire is set; a replacement runs the
    // action on the sources flagged in upd instead, through a temporary swap of the buffer pointer
    void *const keep = dp.src_active.ptr;
    bool const keep_retire = dp.retire;
    if (sel) { dp.src_active.ptr = const_cast<uint8_t*>(sel); dp.retire = true; }
    else dp.retire = retire;
    bool const ok = launch_action<T>(dp, y, x, dptr<uint16_t>(dp.colindx), st);
    dp.src_active.ptr = keep;
    dp.retire = keep_retire;
    return ok;
}

// the solver's operator: A, or A M^-1 with the cube-diagonal preconditioner from the right
// (M^-1 x into the workspace's scratch of the precision, on the same sources)
template <typename T>
bool apply_op(DevicePlan &dp, SolverWorkspace &ws, T *y, T const *x, uint8_t const *sel, bool retire,
              cudaStream_t st) {
    if (!ws.use_pc) return apply<T>(dp, y, x, sel, retire, st);
    T *t = (sizeof(T) == 8) ? reinterpret_cast<T*>(ws.PT64.ptr) : reinterpret_cast<T*>(ws.PT32.ptr);
    uint8_t const *act = sel ? sel : (retire ? dptr<uint8_t>(dp.src_active) : nullptr);
    if (!precond_apply<T>(dp, ws.pc, t, x, act, st)) return false;
    return apply<T>(dp, y, t, sel, retire, st);
}

struct Result { int iterations = 0; double applications = 0; };

// tfQMR on vectors of precision T whose W, U1 hold B and D, X are zero; mixed: X is X32 and the
// solution accumulates in X64 (with AX64 the FP64 scratch of the replacements)
// mask: the sources that take part (the others are padding of a batch, or sources an earlier
// phase has finished), retired before the first kernel
template <typename T>
bool run(DevicePlan &dp, SolverWorkspace &ws, TfqmrVectors &v, Prepared &p, T *X, int maxit, int check_every,
         double *X64, double *AX64, cudaStream_t st, Result &res, int echo, std::vector<uint8_t> const &mask,
         SolveTrace *trace = nullptr) {
    Ctx const &c = p.c;
    uint32_t const nsrc = dp.nCols;
    bool const mixed = c.mixed != 0;
    bool const retire = c.retire != 0;
    T *W = dptr<T>(v.W), *U1 = dptr<T>(v.U1), *U2 = dptr<T>(v.U2), *V = dptr<T>(v.V);
    T *D = dptr<T>(v.D), *AU1 = dptr<T>(v.AU1), *AU2 = dptr<T>(v.AU2);
    uint32_t live = 0;
    for (auto f : mask) live += f ? 1u : 0u;
    bool const partial = live < nsrc;
    Ctl init{}; init.n_active = int32_t(live);
    A43G_CUDA_TRY(cudaMemsetAsync(ws.state.ptr, 0, ws.state.bytes, st));
    A43G_CUDA_TRY(cudaMemcpyAsync(c.ctl, &init, sizeof(Ctl), cudaMemcpyHostToDevice, st));
    A43G_CUDA_TRY(cudaMemsetAsync(ws.tickets.ptr, 0, size_t(nsrc)*sizeof(uint32_t), st));
    A43G_CUDA_TRY(cudaMemcpyAsync(dp.src_active.ptr, mask.data(), nsrc, cudaMemcpyHostToDevice, st));
    // V = A U1
    if (!apply_op<T>(dp, ws, AU1, U1, nullptr, retire, st)) return false;
    A43G_CUDA_TRY(cudaMemcpyAsync(V, AU1, v.n*sizeof(T), cudaMemcpyDeviceToDevice, st));
    res.applications += 1;
    {   // the sources outside the mask are skipped by the initial reductions too
        Ctx ci = c;
        if (partial) ci.active = c.src_active;
        k_init_dots<T><<<p.units, 256, 0, st>>>(W, V, ci);
    }
    count_launch();
    auto iteration = [&]() -> bool {
        if (c.vec16) k_A16<T><<<p.units, 256, 0, st>>>(U2, U1, V, W, AU1, c);
        else k_A<T><<<p.units, 256, 0, st>>>(U2, U1, V, W, AU1, c);
        count_launch();
        if (!apply_op<T>(dp, ws, AU2, U2, nullptr, retire, st)) return false;
        if (c.vec16) k_C16<T><<<p.units, 256, 0, st>>>(W, AU1, AU2, c);
        else k_C<T><<<p.units, 256, 0, st>>>(W, AU1, AU2, c);
        count_launch();
        if constexpr (sizeof(T) == 4) k_DX32<<<p.units, 256, 0, st>>>(X, D, U1, U2, W, c);
        else k_DX<T><<<p.units, 256, 0, st>>>(X, D, U1, U2, W, c);
        count_launch();
        if constexpr (sizeof(T) == 4) {
            if (mixed) {
                // residual replacement of the sources flagged in upd (the launches of the other
                // sources' units return at once)
                k_flush<<<p.units, 256, 0, st>>>(X64, X, c, c.upd);
                count_launch();
                if (!apply_op<double>(dp, ws, AX64, X64, c.upd, retire, st)) return false;
                if (!apply_op<float>(dp, ws, AU1, D, c.upd, retire, st)) return false;    // A d (AU1 is free here)
                k_replace<<<p.units, 256, 0, st>>>(W, AX64, AU1, c);
                count_launch();
                k_U1<<<p.units, 256, 0, st>>>(U1, W, U2, c);
                count_launch();
            }
        }
        if (!apply_op<T>(dp, ws, AU1, U1, nullptr, retire, st)) return false;
        if (c.vec16) k_E16<T><<<p.units, 256, 0, st>>>(V, AU1, AU2, c);
        else k_E<T><<<p.units, 256, 0, st>>>(V, AU1, AU2, c);
        count_launch();
        return true;
    };
    // one iteration captured as a CUDA graph and replayed (not on the legacy default stream,
    // which cannot be captured)
    cudaGraphExec_t exec = nullptr;
    uint64_t per_iteration = 0;
    if (st != nullptr && !std::getenv("A43G_NO_GRAPH")) {
        uint64_t const l0 = launches_so_far();
        cudaGraph_t graph = nullptr;
        A43G_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        bool const ok = iteration();
        cudaError_t const e = cudaStreamEndCapture(st, &graph);
        if (!ok || cudaSuccess != e || !graph) {
            if (graph) cudaGraphDestroy(graph);
            set_error(std::string("capture of the tfQMR iteration: ") + cudaGetErrorString(e));
            return false;
        }
        cudaError_t const ei = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (cudaSuccess != ei) { set_error(std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ei)); return false; }
        per_iteration = launches_so_far() - l0;
        count_launches(uint64_t(0) - per_iteration);   // captured, not launched: counted per replay
    }
    struct GraphGuard { cudaGraphExec_t &e; ~GraphGuard() { if (e) cudaGraphExecDestroy(e); } } guard{exec};
    int it = 0;
    int const every = std::max(1, check_every);
    int const tevery = trace ? std::max(1, trace->every) : 0;
    for (it = 1; it <= maxit; ++it) {
        if (exec) {
            A43G_CUDA_TRY(cudaGraphLaunch(exec, st));
            count_launches(per_iteration);
        } else if (!iteration()) {
            return false;
        }
        res.applications += 2;
        bool const sample = trace && (0 == (res.iterations + it) % tevery);
        if (sample) {
            // the current solution: X64 plus the FP32 correction of the recurrences
            double const *x64 = X64 ? X64 : reinterpret_cast<double const*>(X);
            float const *x32 = (sizeof(T) == 4) ? reinterpret_cast<float const*>(X) : nullptr;
            A43G_CUDA_TRY(cudaMemsetAsync(ws.trace_sums.ptr, 0, 16, st));
            k_trace<<<148*8, 256, 0, st>>>(x64, x32, trace->Xref, v.n, dptr<double>(ws.trace_sums));
            count_launch();
            A43G_CUDA_TRY(cudaMemcpyAsync(reinterpret_cast<char*>(ws.host_ctl) + 32, ws.trace_sums.ptr, 16,
                                          cudaMemcpyDeviceToHost, st));
        }
        if (sample || 0 == it % every || it == maxit) {
            A43G_CUDA_TRY(cudaMemcpyAsync(ws.host_ctl, c.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
            A43G_CUDA_TRY(cudaStreamSynchronize(st));
            Ctl const *h = reinterpret_cast<Ctl const*>(ws.host_ctl);
            if (sample) {
                double const *q = reinterpret_cast<double const*>(reinterpret_cast<char const*>(ws.host_ctl) + 32);
                trace->rows.push_back(double(res.iterations + it));
                trace->rows.push_back(q[1] > 0 ? std::sqrt(q[0]/q[1]) : 0.0);
                trace->rows.push_back(double(h->n_active));
            }
            if (echo > 1) {
                std::printf("# tfqmr<%s> iteration %d: %d of %u sources active, %d breakdowns\n",
                            mixed ? "f32+f64" : "f64", it, h->n_active, nsrc, h->breakdowns);
                std::fflush(stdout);
            }
            if (0 == h->n_active) break;
        }
    }
    res.iterations += std::min(it, maxit);
    A43G_CUDA_TRY(cudaGetLastError());
    // the host copy of the mask must outlive the asynchronous copy above
    A43G_CUDA_TRY(cudaStreamSynchronize(st));
    return true;
}

// The FP64 solution X64 and the recurrence vectors of the precision: FP64 tfQMR keeps its
// solution in X64 and uses AU1 as the scratch of its final residual (8 FP64 vectors); the FP32
// recurrences have their own X (X32) and the FP64 scratch AX64 of the replacements (8 FP32 and
// 2 FP64 vectors).  Vectors of the other precision are released first when the free memory does
// not hold both (large plans: 9 FP64 vectors of the 300,960-block cell fill 178 GB).
bool ensure_vectors(SolverWorkspace &ws, DevicePlan &dp, bool mixed) {
    size_t const n = size_t(dp.nnzb)*kBlk;
    size_t need = 0;
    if (ws.X64.bytes < n*8) need += n*8;
    if (mixed) {
        if (ws.AX64.bytes < n*8) need += n*8;
        if (!ws.v32.W.ptr || ws.v32.n != n) need += 8*n*4;
    } else if (!ws.v64.W.ptr || ws.v64.n != n) {
        need += 7*n*8;
    }
    size_t freeb = 0, total = 0;
    if (need && cudaSuccess == cudaMemGetInfo(&freeb, &total) && freeb < need + (size_t(512) << 20)) {
        if (mixed) ws.v64.release(); else { ws.v32.release(); ws.AX64.release(); }
    }
    if (!ws.X64.alloc(n*8)) return false;
    if (mixed) return ws.AX64.alloc(n*8) && ws.v32.alloc(n, 4, true);
    return ws.v64.alloc(n, 8, false);
}

} // namespace

size_t solve_bytes(DevicePlan const &dp, int precision, bool precondition) {
    // FP64: X64 and 7 recurrence vectors; FP32: 8 FP32 vectors, X64 and AX64, or, for sources
    // continued in FP64, X64 and 7 FP64 vectors (the larger of the two); the preconditioner's
    // scratch: one vector of each precision in use
    size_t const n = size_t(dp.nnzb)*kBlk;
    size_t const pc = precondition ? ((A43G_F32 == precision) ? n*(8 + 4) : n*8) : 0;
    return pc + ((A43G_F32 == precision) ? n*std::max(8*4 + 2*8, 8 + 7*8) : n*(8*8));
}

int solve(GreenPlan &hp, DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt,
          void *Xout, double *rho, a43g_solve_stats_t *stats, cudaStream_t st, SourceStats *per_source,
          SolveTrace *trace) {
    *stats = a43g_solve_stats_t{};
    if (0 == dp.nnzb) { stats->converged = 1; return A43G_OK; }
    if (!(opt.tolerance > 0) || opt.max_iterations < 1) { set_error("tolerance must be > 0 and max_iterations >= 1"); return A43G_ERR_ARGUMENT; }
    if (A43G_F64 != opt.precision && A43G_F32 != opt.precision) { set_error("precision must be A43G_F64 or A43G_F32"); return A43G_ERR_ARGUMENT; }
    (void)hp;
    bool const mixed = (A43G_F32 == opt.precision);
    // the FP32 recurrences always retire finished sources (stalled sources leave them retired and
    // continue in FP64 on their own); A43G_SOLVE_NO_RETIRE applies to FP64 solves
    bool const retire = mixed || 0 == (opt.flags & A43G_SOLVE_NO_RETIRE);
    uint32_t const nsrc = dp.nCols;
    uint32_t const live = (per_source && per_source->live_sources) ? std::min(per_source->live_sources, nsrc) : nsrc;
    std::vector<uint8_t> mask(nsrc, 0);
    std::fill(mask.begin(), mask.begin() + live, uint8_t(1));
    if (!ensure_vectors(ws, dp, mixed)) return A43G_ERR_MEMORY;
    if (trace && (!trace->Xref || !ws.trace_sums.alloc(16))) return trace->Xref ? A43G_ERR_MEMORY : A43G_ERR_ARGUMENT;
    // right preconditioning: the recurrences see A M^-1 and the solution is M^-1 of theirs
    ws.use_pc = 0 != (opt.flags & A43G_SOLVE_PRECONDITION);
    if (ws.use_pc) {
        if (trace) { set_error("a traced solve takes no preconditioner"); return A43G_ERR_UNSUPPORTED; }
        size_t const nr = size_t(dp.nnzb)*kBlk;
        if (!ws.PT64.alloc(nr*8) || (mixed && !ws.PT32.alloc(nr*4))) return A43G_ERR_MEMORY;
        if (int const rc = precond_setup(hp, dp, ws.pc, st); A43G_OK != rc) return rc;
    }
    // projector scratch for both precisions before the iteration is captured (no allocation
    // may happen inside a stream capture)
    if (!ensure_dyadic_scratch(dp, 8) || !ensure_prj_part(dp, 8)) return A43G_ERR_MEMORY;
    Prepared p;
    if (!prepare(dp, ws, opt, mixed, retire || live < nsrc, p)) return A43G_ERR_MEMORY;
    RetireGuard rg{dp, st};
    size_t const n = size_t(dp.nnzb)*kBlk;
    A43G_CUDA_TRY_RC(cudaEventRecord(ws.ev0, st));
    Result res;
    double *X64 = dptr<double>(ws.X64);
    std::vector<SrcState> ss1;                  // the FP32 phase's per-source results
    std::vector<int> it1(nsrc, 0);
    if (mixed) {
        auto &v = ws.v32;
        for (DeviceBuffer *b : {&v.W, &v.U1, &v.D, &v.X}) A43G_CUDA_TRY_RC(cudaMemsetAsync(b->ptr, 0, n*4, st));
        A43G_CUDA_TRY_RC(cudaMemsetAsync(X64, 0, n*8, st));
        k_set_diag<float><<<nsrc, 64, 0, st>>>(dptr<float>(v.W), dptr<float>(v.U1), dptr<uint32_t>(dp.subset_dev), nsrc);
        count_launch();
        if (!run<float>(dp, ws, v, p, dptr<float>(v.X), opt.max_iterations, opt.check_every, X64,
                        dptr<double>(ws.AX64), st, res, opt.echo, mask, trace))
            return A43G_ERR_CUDA;
        // the rest of every column's FP32 correction into the FP64 solution
        k_flush<<<p.units, 256, 0, st>>>(X64, dptr<float>(v.X), p.c, nullptr);
        count_launch();
        ss1.resize(nsrc);
        A43G_CUDA_TRY_RC(cudaMemcpyAsync(ss1.data(), p.c.ss, nsrc*sizeof(SrcState), cudaMemcpyDeviceToHost, st));
        A43G_CUDA_TRY_RC(cudaStreamSynchronize(st));
        // sources whose FP32 recurrences stalled, or that ran out of iterations, continue in FP64
        // from their FP64 solution: tfQMR on (H - E S) X = B with the initial guess X64
        std::vector<uint8_t> fb(nsrc, 0);
        uint32_t nfb = 0;
        for (uint32_t k = 0; k < live; ++k) {
            it1[k] = ss1[k].done ? ss1[k].it : res.iterations;
            if (ss1[k].fallback) { fb[k] = 1; ++nfb; }
        }
        int left = opt.max_iterations - res.iterations;
        if (nfb && left > 0) {
            // the FP32 set is done with: released first where both sets do not fit
            size_t freeb = 0, total = 0;
            if ((!ws.v64.W.ptr || ws.v64.n != n) && cudaSuccess == cudaMemGetInfo(&freeb, &total) &&
                freeb < 7*n*8 + (size_t(512) << 20)) {
                A43G_CUDA_TRY_RC(cudaStreamSynchronize(st));
                v.release();
                ws.AX64.release();
            }
            if (!ws.v64.alloc(n, 8, false)) return A43G_ERR_MEMORY;
            auto &w = ws.v64;
            Prepared p2;
            a43g_solve_options_t o2 = opt;
            if (!prepare(dp, ws, o2, false, true, p2)) return A43G_ERR_MEMORY;
            p2.c.abs_tol = 1;
            // the QMR bound decides when an FP64 run stops; aiming at half the tolerance leaves
            // room for the gap between the bound and the true residual
            p2.c.tol = 0.5*opt.tolerance;
            std::vector<uint8_t> cont = fb;
            std::vector<ColState> cs2;
            for (int restart = 0; ; ++restart) {
                // A X64 of the continuing sources (their blocks only) into AU1
                A43G_CUDA_TRY_RC(cudaMemcpyAsync(dp.src_active.ptr, cont.data(), nsrc, cudaMemcpyHostToDevice, st));
                if (!apply_op<double>(dp, ws, dptr<double>(w.AU1), X64, nullptr, true, st)) return A43G_ERR_CUDA;
                res.applications += 1;
                if (restart > 0) {
                    // the true residual of each source the last run finished: sources still above
                    // the tolerance (rounding in the recurrences can hold the true residual above
                    // the bound) restart from their solution, at most kRestarts times
                    k_final<<<p2.units, 256, 0, st>>>(dptr<double>(w.AU1), p2.c, dptr<uint8_t>(dp.src_active));
                    count_launch();
                    cs2.resize(size_t(nsrc)*64);
                    A43G_CUDA_TRY_RC(cudaMemcpyAsync(cs2.data(), p2.c.cs, cs2.size()*sizeof(ColState),
                                                     cudaMemcpyDeviceToHost, st));
                    A43G_CUDA_TRY_RC(cudaStreamSynchronize(st));
                    uint32_t again = 0;
                    for (uint32_t k = 0; k < live; ++k) {
                        if (!cont[k]) continue;
                        double r = 0;
                        for (int j = 0; j < 64; ++j) r = std::max(r, cs2[size_t(k)*64 + j].res);
                        cont[k] = (std::isfinite(r) && r > opt.tolerance) ? 1 : 0;
                        again += cont[k];
                    }
                    left = opt.max_iterations - res.iterations;
                    if (0 == again || left <= 0 || restart > kRestarts) break;
                    A43G_CUDA_TRY_RC(cudaMemcpyAsync(dp.src_active.ptr, cont.data(), nsrc, cudaMemcpyHostToDevice, st));
                }
                // R = B - A X64 of the continuing sources into W and U1; D = 0
                A43G_CUDA_TRY_RC(cudaMemsetAsync(w.D.ptr, 0, n*8, st));
                k_start64<<<p2.units, 256, 0, st>>>(dptr<double>(w.W), dptr<double>(w.U1), X64, dptr<double>(w.AU1),
                                                   p2.c, dptr<uint8_t>(dp.src_active));
                count_launch();
                int const it0 = res.iterations;
                if (!run<double>(dp, ws, w, p2, X64, left, opt.check_every, nullptr, nullptr, st, res, opt.echo, cont,
                                 trace))
                    return A43G_ERR_CUDA;
                std::vector<SrcState> ss2(nsrc);
                A43G_CUDA_TRY_RC(cudaMemcpyAsync(ss2.data(), p2.c.ss, nsrc*sizeof(SrcState), cudaMemcpyDeviceToHost, st));
                A43G_CUDA_TRY_RC(cudaStreamSynchronize(st));
                for (uint32_t k = 0; k < live; ++k) if (cont[k]) it1[k] += ss2[k].done ? ss2[k].it : res.iterations - it0;
            }
        }
    } else {
        auto &v = ws.v64;
        for (DeviceBuffer *b : {&v.W, &v.U1, &v.D}) A43G_CUDA_TRY_RC(cudaMemsetAsync(b->ptr, 0, n*8, st));
        A43G_CUDA_TRY_RC(cudaMemsetAsync(X64, 0, n*8, st));
        k_set_diag<double><<<nsrc, 64, 0, st>>>(dptr<double>(v.W), dptr<double>(v.U1), dptr<uint32_t>(dp.subset_dev), nsrc);
        count_launch();
        if (!run<double>(dp, ws, v, p, X64, opt.max_iterations, opt.check_every, nullptr, nullptr, st, res, opt.echo,
                         mask, trace))
            return A43G_ERR_CUDA;
    }
    if (trace) {
        // the error of the final FP64 solution
        A43G_CUDA_TRY_RC(cudaMemsetAsync(ws.trace_sums.ptr, 0, 16, st));
        k_trace<<<148*8, 256, 0, st>>>(X64, nullptr, trace->Xref, n, dptr<double>(ws.trace_sums));
        count_launch();
        double q[2] = {0, 0};
        A43G_CUDA_TRY_RC(cudaMemcpyAsync(q, ws.trace_sums.ptr, 16, cudaMemcpyDeviceToHost, st));
        A43G_CUDA_TRY_RC(cudaStreamSynchronize(st));
        trace->rows.push_back(double(res.iterations));
        trace->rows.push_back(q[1] > 0 ? std::sqrt(q[0]/q[1]) : 0.0);
        trace->rows.push_back(0.0);
    }
    if (ws.use_pc) {
        // the solution of the original system: X = M^-1 Y (in place, every block)
        if (!precond_apply<double>(dp, ws.pc, X64, X64, nullptr, st)) return A43G_ERR_CUDA;
    }
    // true residual of every column's FP64 solution (the whole operator, no source skipped), in
    // whichever FP64 scratch the solve holds
    double *AXs = ws.AX64.ptr ? dptr<double>(ws.AX64) : dptr<double>(ws.v64.AU1);
    dp.retire = false;
    if (!launch_action<double>(dp, AXs, X64, dptr<uint16_t>(dp.colindx), st)) return A43G_ERR_CUDA;
    res.applications += 1;
    k_final<<<p.units, 256, 0, st>>>(AXs, p.c, nullptr);
    count_launch();
    if (Xout) A43G_CUDA_TRY_RC(cudaMemcpyAsync(Xout, X64, n*8, cudaMemcpyDeviceToDevice, st));
    if (rho) {
        double *rb = AXs;                        // the residual scratch is free again
        k_export_rho<double><<<nsrc, 64, 0, st>>>(rb, X64, dptr<uint32_t>(dp.subset_dev), nsrc);
        count_launch();
        A43G_CUDA_TRY_RC(cudaMemcpyAsync(rho, rb, size_t(nsrc)*128*8, cudaMemcpyDeviceToHost, st));
    }
    A43G_CUDA_TRY_RC(cudaEventRecord(ws.ev1, st));
    // per-column and per-source results
    std::vector<ColState> cs(size_t(nsrc)*64);
    std::vector<SrcState> ss(nsrc);
    Ctl ctl{};
    A43G_CUDA_TRY_RC(cudaMemcpyAsync(cs.data(), p.c.cs, cs.size()*sizeof(ColState), cudaMemcpyDeviceToHost, st));
    A43G_CUDA_TRY_RC(cudaMemcpyAsync(ss.data(), p.c.ss, ss.size()*sizeof(SrcState), cudaMemcpyDeviceToHost, st));
    A43G_CUDA_TRY_RC(cudaMemcpyAsync(&ctl, p.c.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, st));
    if (cudaSuccess != cudaEventSynchronize(ws.ev1) || cudaSuccess != cudaStreamSynchronize(st)) {
        set_error(std::string("solve: ") + cudaGetErrorString(cudaGetLastError()));
        return A43G_ERR_CUDA;
    }
    float ms = 0; cudaEventElapsedTime(&ms, ws.ev0, ws.ev1);
    if (!mixed) for (uint32_t k = 0; k < live; ++k) it1[k] = ss[k].done ? ss[k].it : res.iterations;
    double rmax = 0;
    int updates = 0;
    for (size_t k = 0; k < size_t(live)*64; ++k) rmax = std::max(rmax, std::isfinite(cs[k].res) ? cs[k].res : 1e300);
    if (mixed) for (uint32_t k = 0; k < live; ++k) updates = std::max(updates, ss1[k].updates);
    int fallbacks = 0;
    if (mixed) for (uint32_t k = 0; k < live; ++k) fallbacks += ss1[k].fallback;
    stats->seconds = ms*1e-3;
    stats->iterations = res.iterations;
    stats->refinements = updates;
    stats->breakdowns = ctl.breakdowns;
    stats->residual_max = rmax;
    stats->operator_applications = res.applications;
    stats->converged = (rmax <= opt.tolerance) ? 1 : 0;
    stats->fp64_sources = fallbacks;
    double est = 0;
    for (size_t k = 0; k < size_t(live)*64; ++k)
        if (cs[k].bnorm > 0) est = std::max(est, cs[k].tau*std::sqrt(double(cs[k].m) + 1.0)/cs[k].bnorm);
    stats->residual_estimate = est;
    if (per_source) {
        per_source->iterations.assign(it1.begin(), it1.end());
        per_source->residual.assign(nsrc, 0.0);
        per_source->updates.assign(nsrc, 0);
        per_source->fallback.assign(nsrc, 0);
        for (uint32_t k = 0; k < nsrc; ++k) {
            if (mixed) { per_source->updates[k] = ss1[k].updates; per_source->fallback[k] = ss1[k].fallback; }
            for (int j = 0; j < 64; ++j) {
                double const r = cs[size_t(k)*64 + j].res;
                per_source->residual[k] = std::max(per_source->residual[k], std::isfinite(r) ? r : 1e300);
            }
        }
    }
    if (opt.echo > 0)
        std::printf("# tfqmr<%s> %d iterations, %d replacements, %d sources continued in FP64, true residual %.3e (tolerance %.1e)\n",
                    mixed ? "f32+f64" : "f64", res.iterations, updates, fallbacks, rmax, opt.tolerance);
    cudaError_t const e = cudaGetLastError();
    if (cudaSuccess != e) { set_error(std::string("solve: ") + cudaGetErrorString(e)); return A43G_ERR_CUDA; }
    return A43G_OK;
}

} // namespace a43g

namespace a43g {

// Solves of many (energy, k-point) pairs on the geometry of the one-pair plan hp, in waves of
// up to `wave` pairs: each wave is one block-sparse system (GreenPlan::replicate) whose sources
// retire as they finish.  The last wave is filled up with copies of its last pair whose sources
// are retired from the start.
int solve_batched(GreenPlan &hp, DevicePlan &dp, BatchCache &bc, a43g_solve_options_t const &opt,
                  int32_t n, double const *energies, double const *kpoints, double dVol,
                  double *rho, a43g_solve_stats_t *stats, cudaStream_t st) {
    if (n <= 0) return A43G_OK;
    if (hp.npairs != 1) { set_error("solve_batched needs a one-pair plan"); return A43G_ERR_ARGUMENT; }
    for (int32_t i = 0; i < n; ++i)
        for (int d = 0; d < 3; ++d)
            if (!(std::abs(kpoints[3*i + d]) < 0.503)) { set_error("k-point components must be below 0.503 (units of 2 pi / cell)"); return A43G_ERR_ARGUMENT; }
    uint32_t const nsrc = hp.nCols;
    uint32_t wave = opt.batch > 0 ? uint32_t(opt.batch) : 0;
    if (0 == wave) {
        // as many pairs as fit 85 % of the free memory next to what the batch plan holds already
        size_t freeb = 0, total = 0;
        if (cudaSuccess != cudaMemGetInfo(&freeb, &total)) { set_error("cudaMemGetInfo"); return A43G_ERR_CUDA; }
        bool const pcf = 0 != (opt.flags & A43G_SOLVE_PRECONDITION);
        size_t const held = bc.npairs ? solve_bytes(*bc.dev, opt.precision, pcf) : 0;
        size_t const per = solve_bytes(dp, opt.precision, pcf) + size_t(dp.nnzb)*kBlk*2 + (size_t(64) << 20);
        wave = uint32_t(std::max<size_t>(1, (size_t(0.85*double(freeb + held)))/per));
    }
    wave = std::min<uint32_t>(wave, uint32_t(n));
    wave = std::min<uint32_t>(wave, 65535u/std::max(1u, nsrc));
    if (wave < 1) { set_error("a pair has more sources than a batch holds"); return A43G_ERR_UNSUPPORTED; }
    if (bc.npairs != wave) {
        bc.ws.reset(); bc.dev.reset(); bc.npairs = 0;    // release the old batch first
        auto const err = bc.host.replicate(hp, wave);
        if (!err.empty()) { set_error(err); return A43G_ERR_ARGUMENT; }
        bc.dev.reset(new DevicePlan());
        bc.ws.reset(new SolverWorkspace());
        bc.dev->prj_chunk = dp.prj_chunk; bc.dev->add_blocks = dp.add_blocks;
        if (!upload_plan(bc.host, *bc.dev)) return A43G_ERR_CUDA;
        bc.dev->local_variant = dp.local_variant; bc.dev->use_tc = dp.use_tc;
        bc.npairs = wave;
    }
    // the caller's potential and atom matrices as they are now
    bc.host.Vcell = hp.Vcell;
    bc.host.AtomMatricesIn = hp.AtomMatricesIn;
    for (int32_t w0 = 0; w0 < n; w0 += int32_t(wave)) {
        uint32_t const live = std::min<uint32_t>(wave, uint32_t(n - w0));
        for (uint32_t p = 0; p < wave; ++p) {
            uint32_t const i = w0 + std::min(p, live - 1);
            auto const err = bc.host.set_pair(p, energies[2*i], energies[2*i + 1], dVol, kpoints + 3*size_t(i));
            if (!err.empty()) { set_error(err); return A43G_ERR_ARGUMENT; }
        }
        if (!upload_values(bc.host, *bc.dev)) return A43G_ERR_CUDA;
        a43g_solve_stats_t ws_stats{};
        SourceStats per;
        per.live_sources = live*nsrc;
        std::vector<double> rb(rho ? size_t(wave)*nsrc*128 : 0);
        a43g_solve_options_t o = opt;
        o.flags &= ~A43G_SOLVE_NO_RETIRE;            // padding sources are retired from the start
        int const rc = solve(bc.host, *bc.dev, *bc.ws, o, nullptr, rho ? rb.data() : nullptr, &ws_stats, st, &per);
        if (rc) return rc;
        for (uint32_t p = 0; p < live; ++p) {
            a43g_solve_stats_t &s = stats[w0 + p];
            s = ws_stats;
            int it = 0, upd = 0, fb = 0; double r = 0;
            for (uint32_t k = 0; k < nsrc; ++k) {
                it = std::max(it, per.iterations[p*nsrc + k]);
                upd = std::max(upd, per.updates[p*nsrc + k]);
                fb += per.fallback[p*nsrc + k];
                r = std::max(r, per.residual[p*nsrc + k]);
            }
            s.iterations = it; s.refinements = upd; s.residual_max = r; s.fp64_sources = fb;
            s.converged = (r <= opt.tolerance) ? 1 : 0;
            if (rho) std::memcpy(rho + (size_t(w0) + p)*nsrc*128, rb.data() + size_t(p)*nsrc*128, size_t(nsrc)*128*8);
        }
    }
    return A43G_OK;
}

} // namespace a43g
