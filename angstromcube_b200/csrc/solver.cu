// Transpose-free QMR (Freund, SIAM J. Sci. Comput. 14:470, 1993) for all columns of the
// block-sparse Green function at once, each column with its own scalars, plus mixed
// precision (FP32 sweeps inside FP64 residual refinement).
//
// One iteration = two operator applications.  The BLAS-1 work is fused so that every vector
// is streamed as few times as possible:
//   K_A   U2 = U1 - a V                 and |W - a AU1|^2
//   K_C   W  = W - a (AU1 + AU2)        and |W|^2, rt^H W
// (U1 = y_{2n-1}, U2 = y_{2n}, AU1 = A y_{2n-1}, AU2 = A y_{2n}, V = v_{n-1} in Freund's notation)
//   K_DX  D, X advanced by both half steps at once;  U1 = W + b U2
//   K_E   V  = AU1 + b (AU2 + b V)      and rt^H V
// The shadow residual rt is a counter-based random vector regenerated on the fly, so it is
// never stored.  FP32 sweeps do the vector arithmetic in FP32 and accumulate the inner
// products in FP64.  Per-column reductions end in double atomics; the scalar recurrences run in
// FP64 in one thread per column.  Finished columns (converged or broken down) get zero
// coefficients, which freezes X and keeps all vectors finite.
#include "solver.hpp"

#include <algorithm>
#include <cstdlib>
#include <cmath>
#include <cstdio>
#include <vector>

namespace a43g {

namespace {

constexpr int kBlk = 8192;

struct ColState {
    double rho_re, rho_im;       // rho_{n-1} = rt^H w
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
    double tau_ref;              // stall detection: tau at the last halving, and its half step
    int32_t m_ref;
    int32_t status;              // 0 active, 1 converged, 2 breakdown, 3 idle (zero column), 4 stalled
    int32_t conv1;               // converged in the first half step of this iteration
};

struct Acc { double n2, re, im, pad; };   // per-column reduction accumulator

__device__ __forceinline__ uint32_t mix32(uint32_t h) {
    // murmur3 finaliser as a counter-based generator
    h ^= h >> 16; h *= 0x85ebca6bu; h ^= h >> 13; h *= 0xc2b2ae35u; h ^= h >> 16;
    return h;
}

// shadow residual element for (block, reim, i, j): uniform in [-1, 1)
__device__ __forceinline__ double shadow(uint32_t seed, uint32_t idx) {
    return double(int32_t(mix32(idx*0x9E3779B9u + seed))) * (1.0/2147483648.0);
}

// the same element in FP32 (the double value above rounded to float)
__device__ __forceinline__ float shadow32(uint32_t seed, uint32_t idx) {
    return float(int32_t(mix32(idx*0x9E3779B9u + seed))) * (1.0f/2147483648.0f);
}

template <typename T>
__device__ __forceinline__ void cmul(double ar, double ai, T br, T bi, double &r, double &i) {
    r = ar*double(br) - ai*double(bi); i = ar*double(bi) + ai*double(br);
}

// block-local reduction of up to 3 values per column over the 4 row groups, then atomics
__device__ __forceinline__ void reduce_cols(double (*red)[64][3], int q, int j, double v0, double v1, double v2,
                                            Acc *acc, int ncomp) {
    red[q][j][0] = v0; red[q][j][1] = v1; red[q][j][2] = v2;
    __syncthreads();
    if (0 == q) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int k = 0; k < 4; ++k) { s0 += red[k][j][0]; s1 += red[k][j][1]; s2 += red[k][j][2]; }
        atomicAdd(&acc->n2, s0);
        if (ncomp > 1) { atomicAdd(&acc->re, s1); atomicAdd(&acc->im, s2); }
    }
    __syncthreads();
}

// ------------------------------------------------------------------ vector kernels
// grid-stride over blocks; thread (q, j): column j, rows q*16 .. q*16+15, re and im

template <typename T>
__global__ void k_set_diag(T *W, T *U1, uint32_t const *subset, uint32_t ncols_blk) {
    uint32_t const c = blockIdx.x; int const i = threadIdx.x;
    if (c < ncols_blk) {
        size_t const o = size_t(subset[c])*kBlk + size_t(i)*64 + i;
        W[o] = T(1); U1[o] = T(1);
    }
}

// initial reductions: |W|^2, rt^H W and rt^H V
template <typename T>
__global__ void __launch_bounds__(256) k_init_dots(T const *W, T const *V, uint32_t nnzb, uint16_t const *colindx,
                                                   Acc *accW, Acc *accV, uint32_t seed) {
    __shared__ double red[4][64][3];
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const c = colindx[b];
        double n2 = 0, wr = 0, wi = 0, vr = 0, vi = 0;
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j;
            uint32_t const idx = uint32_t(o);
            // FP32 sweeps use the shadow vector rounded to FP32 throughout
            double const tr = (sizeof(T) == 4) ? double(shadow32(seed, idx)) : shadow(seed, idx);
            double const ti = (sizeof(T) == 4) ? double(shadow32(seed, idx + 4096u)) : shadow(seed, idx + 4096u);
            double const xr = W[o], xi = W[o + 4096], yr = V[o], yi = V[o + 4096];
            n2 += xr*xr + xi*xi;
            wr += tr*xr + ti*xi; wi += tr*xi - ti*xr;     // conj(rt) w
            vr += tr*yr + ti*yi; vi += tr*yi - ti*yr;
        }
        reduce_cols(red, q, j, n2, wr, wi, &accW[c*64 + j], 3);
        reduce_cols(red, q, j, 0.0, vr, vi, &accV[c*64 + j], 3);
    }
}

// K_A: U2 = U1 - alpha V ; acc |W - alpha AU1|^2
template <typename T>
__global__ void __launch_bounds__(256) k_A(T *U2, T const *U1, T const *V, T const *W, T const *AU1, uint32_t nnzb,
                                           uint16_t const *colindx, ColState const *cs, Acc *acc,
                                           float const *cf, uint32_t ncol) {
    __shared__ double red[4][64][3];
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const col = colindx[b]*64 + j;
        double n2 = 0;
        if constexpr (sizeof(T) == 4) {
            // FP32 sweep: vector arithmetic in FP32, 32-term partial sums in FP32, the rest in FP64
            float const fr = cf[col], fi = cf[ncol + col];
            float n2f = 0.f;
#pragma unroll 8
            for (int i = q*16; i < q*16 + 16; ++i) {
                size_t const o = size_t(b)*kBlk + i*64 + j;
                float const vr = V[o], vi = V[o + 4096];
                U2[o] = fmaf(fi, vi, fmaf(-fr, vr, U1[o]));
                U2[o + 4096] = fmaf(-fi, vr, fmaf(-fr, vi, U1[o + 4096]));
                float const ur = AU1[o], ui = AU1[o + 4096];
                float const wr = fmaf(fi, ui, fmaf(-fr, ur, W[o])), wi = fmaf(-fi, ur, fmaf(-fr, ui, W[o + 4096]));
                n2f = fmaf(wr, wr, fmaf(wi, wi, n2f));
            }
            n2 = double(n2f);
        } else {
        double const ar = cs[col].al_re, ai = cs[col].al_im;
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j;
            T const vr = V[o], vi = V[o + 4096];
            double avr, avi; cmul(ar, ai, vr, vi, avr, avi);
            U2[o] = T(double(U1[o]) - avr); U2[o + 4096] = T(double(U1[o + 4096]) - avi);
            double aur, aui; cmul(ar, ai, AU1[o], AU1[o + 4096], aur, aui);
            double const wr = double(W[o]) - aur, wi = double(W[o + 4096]) - aui;
            n2 += wr*wr + wi*wi;
        }
        }
        reduce_cols(red, q, j, n2, 0.0, 0.0, &acc[col], 1);
    }
}

// K_C: W = W - alpha (AU1 + AU2) ; acc |W|^2 and rt^H W
template <typename T>
__global__ void __launch_bounds__(256) k_C(T *W, T const *AU1, T const *AU2, uint32_t nnzb,
                                           uint16_t const *colindx, ColState const *cs, Acc *acc, uint32_t seed,
                                           float const *cf, uint32_t ncol) {
    __shared__ double red[4][64][3];
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const col = colindx[b]*64 + j;
        double const ar = (sizeof(T) == 8) ? cs[col].al_re : 0.0, ai = (sizeof(T) == 8) ? cs[col].al_im : 0.0;
        double n2 = 0, dr = 0, di = 0;
        if constexpr (sizeof(T) == 4) {
            float const fr = cf[col], fi = cf[ncol + col];
            float n2f = 0.f, drf = 0.f, dif = 0.f;
#pragma unroll 8
            for (int i = q*16; i < q*16 + 16; ++i) {
                size_t const o = size_t(b)*kBlk + i*64 + j;
                float const sr = AU1[o] + AU2[o], si = AU1[o + 4096] + AU2[o + 4096];
                float const wr = fmaf(fi, si, fmaf(-fr, sr, W[o])), wi = fmaf(-fi, sr, fmaf(-fr, si, W[o + 4096]));
                W[o] = wr; W[o + 4096] = wi;
                uint32_t const idx = uint32_t(o);
                float const tr = shadow32(seed, idx), ti = shadow32(seed, idx + 4096u);
                n2f = fmaf(wr, wr, fmaf(wi, wi, n2f));
                drf = fmaf(tr, wr, fmaf(ti, wi, drf)); dif = fmaf(tr, wi, fmaf(-ti, wr, dif));
            }
            n2 = double(n2f); dr = double(drf); di = double(dif);
        } else
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j;
            double const sr = double(AU1[o]) + double(AU2[o]), si = double(AU1[o + 4096]) + double(AU2[o + 4096]);
            double const wr = double(W[o]) - (ar*sr - ai*si), wi = double(W[o + 4096]) - (ar*si + ai*sr);
            T const tr_ = T(wr), ti_ = T(wi);
            W[o] = tr_; W[o + 4096] = ti_;
            double const xr = tr_, xi = ti_;
            uint32_t const idx = uint32_t(o);
            double const tr = shadow(seed, idx), ti = shadow(seed, idx + 4096u);
            n2 += xr*xr + xi*xi;
            dr += tr*xr + ti*xi; di += tr*xi - ti*xr;
        }
        reduce_cols(red, q, j, n2, dr, di, &acc[col], 3);
    }
}

// K_DX: X += cu1x U1 + cu2x U2 + cdx D ; D = U2 + cu1d U1 + cdd D ; U1 = W + beta U2
// (X may be kept in FP64 while the recurrence vectors are FP32: the solution then carries no
// FP32 rounding, which lowers the residual floor of an FP32 sweep)
template <typename T, typename TX>
__global__ void __launch_bounds__(256) k_DX(TX *X, T *D, T *U1, T const *U2, T const *W, uint32_t nnzb,
                                            uint16_t const *colindx, ColState const *cs, float const *cf, uint32_t ncol) {
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const col = colindx[b]*64 + j;
        if constexpr (sizeof(T) == 4 && sizeof(TX) == 4) {
            float const g_r = cf[2*size_t(ncol) + col], g_i = cf[3*size_t(ncol) + col];
            float const a_r = cf[4*size_t(ncol) + col], a_i = cf[5*size_t(ncol) + col];
            float const b_r = cf[6*size_t(ncol) + col], b_i = cf[7*size_t(ncol) + col];
            float const c_r = cf[8*size_t(ncol) + col], c_i = cf[9*size_t(ncol) + col];
            float const d_r = cf[10*size_t(ncol) + col], d_i = cf[11*size_t(ncol) + col];
            float const e_r = cf[12*size_t(ncol) + col], e_i = cf[13*size_t(ncol) + col];
#pragma unroll 8
            for (int i = q*16; i < q*16 + 16; ++i) {
                size_t const o = size_t(b)*kBlk + i*64 + j;
                float const u1r = U1[o], u1i = U1[o + 4096], u2r = U2[o], u2i = U2[o + 4096];
                float const dr = D[o], di = D[o + 4096];
                float xr = X[o], xi = X[o + 4096];
                xr = fmaf(a_r, u1r, fmaf(-a_i, u1i, xr)); xi = fmaf(a_r, u1i, fmaf(a_i, u1r, xi));
                xr = fmaf(b_r, u2r, fmaf(-b_i, u2i, xr)); xi = fmaf(b_r, u2i, fmaf(b_i, u2r, xi));
                xr = fmaf(c_r, dr, fmaf(-c_i, di, xr));   xi = fmaf(c_r, di, fmaf(c_i, dr, xi));
                X[o] = xr; X[o + 4096] = xi;
                D[o] = fmaf(d_r, u1r, fmaf(-d_i, u1i, fmaf(e_r, dr, fmaf(-e_i, di, u2r))));
                D[o + 4096] = fmaf(d_r, u1i, fmaf(d_i, u1r, fmaf(e_r, di, fmaf(e_i, dr, u2i))));
                U1[o] = fmaf(g_r, u2r, fmaf(-g_i, u2i, W[o]));
                U1[o + 4096] = fmaf(g_r, u2i, fmaf(g_i, u2r, W[o + 4096]));
            }
        } else {
        ColState const &s = cs[col];
        double const ax_r = s.cu1x_re, ax_i = s.cu1x_im, bx_r = s.cu2x_re, bx_i = s.cu2x_im, cx_r = s.cdx_re, cx_i = s.cdx_im;
        double const ad_r = s.cu1d_re, ad_i = s.cu1d_im, cd_r = s.cdd_re, cd_i = s.cdd_im;
        double const be_r = s.be_re, be_i = s.be_im;
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j;
            double const u1r = U1[o], u1i = U1[o + 4096], u2r = U2[o], u2i = U2[o + 4096];
            double const dr = D[o], di = D[o + 4096];
            double const xr = double(X[o]) + (ax_r*u1r - ax_i*u1i) + (bx_r*u2r - bx_i*u2i) + (cx_r*dr - cx_i*di);
            double const xi = double(X[o + 4096]) + (ax_r*u1i + ax_i*u1r) + (bx_r*u2i + bx_i*u2r) + (cx_r*di + cx_i*dr);
            X[o] = TX(xr); X[o + 4096] = TX(xi);
            D[o] = T(u2r + (ad_r*u1r - ad_i*u1i) + (cd_r*dr - cd_i*di));
            D[o + 4096] = T(u2i + (ad_r*u1i + ad_i*u1r) + (cd_r*di + cd_i*dr));
            double const wr = W[o], wi = W[o + 4096];
            U1[o] = T(wr + (be_r*u2r - be_i*u2i));
            U1[o + 4096] = T(wi + (be_r*u2i + be_i*u2r));
        }
        }
    }
}

// K_DX of an FP32 sweep with 16-byte accesses: thread (column group of 4, row group of 4 rows);
// each row moves 10 float4 loads and 6 float4 stores, and the 12 coefficients of its 4 columns
// are 12 float4 loads per block
__device__ __forceinline__ float4 ld4(float const *p) { return *reinterpret_cast<float4 const*>(p); }
__device__ __forceinline__ void st4(float *p, float4 v) { *reinterpret_cast<float4*>(p) = v; }

__global__ void __launch_bounds__(256, 2) k_DX32(float *X, float *D, float *U1, float const *U2, float const *W,
                                                 uint32_t nnzb, uint16_t const *colindx, float const *cf, uint32_t ncol) {
    int const cg = threadIdx.x & 15, rg = threadIdx.x >> 4;
    int const j0 = cg*4;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const col = colindx[b]*64 + j0;
        float4 const g_r = ld4(cf + 2*size_t(ncol) + col), g_i = ld4(cf + 3*size_t(ncol) + col);
        float4 const a_r = ld4(cf + 4*size_t(ncol) + col), a_i = ld4(cf + 5*size_t(ncol) + col);
        float4 const b_r = ld4(cf + 6*size_t(ncol) + col), b_i = ld4(cf + 7*size_t(ncol) + col);
        float4 const c_r = ld4(cf + 8*size_t(ncol) + col), c_i = ld4(cf + 9*size_t(ncol) + col);
        float4 const d_r = ld4(cf + 10*size_t(ncol) + col), d_i = ld4(cf + 11*size_t(ncol) + col);
        float4 const e_r = ld4(cf + 12*size_t(ncol) + col), e_i = ld4(cf + 13*size_t(ncol) + col);
#pragma unroll 2
        for (int i = rg*4; i < rg*4 + 4; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j0;
            float4 const u1r = ld4(U1 + o), u1i = ld4(U1 + o + 4096), u2r = ld4(U2 + o), u2i = ld4(U2 + o + 4096);
            float4 const dr = ld4(D + o), di = ld4(D + o + 4096), wr = ld4(W + o), wi = ld4(W + o + 4096);
            float4 xr = ld4(X + o), xi = ld4(X + o + 4096);
            float4 nd_r, nd_i, nu_r, nu_i;
#define A43G_DX_LANE(c) \
            xr.c = fmaf(a_r.c, u1r.c, fmaf(-a_i.c, u1i.c, xr.c)); xi.c = fmaf(a_r.c, u1i.c, fmaf(a_i.c, u1r.c, xi.c)); \
            xr.c = fmaf(b_r.c, u2r.c, fmaf(-b_i.c, u2i.c, xr.c)); xi.c = fmaf(b_r.c, u2i.c, fmaf(b_i.c, u2r.c, xi.c)); \
            xr.c = fmaf(c_r.c, dr.c, fmaf(-c_i.c, di.c, xr.c));   xi.c = fmaf(c_r.c, di.c, fmaf(c_i.c, dr.c, xi.c)); \
            nd_r.c = fmaf(d_r.c, u1r.c, fmaf(-d_i.c, u1i.c, fmaf(e_r.c, dr.c, fmaf(-e_i.c, di.c, u2r.c)))); \
            nd_i.c = fmaf(d_r.c, u1i.c, fmaf(d_i.c, u1r.c, fmaf(e_r.c, di.c, fmaf(e_i.c, dr.c, u2i.c)))); \
            nu_r.c = fmaf(g_r.c, u2r.c, fmaf(-g_i.c, u2i.c, wr.c)); \
            nu_i.c = fmaf(g_r.c, u2i.c, fmaf(g_i.c, u2r.c, wi.c));
            A43G_DX_LANE(x) A43G_DX_LANE(y) A43G_DX_LANE(z) A43G_DX_LANE(w)
#undef A43G_DX_LANE
            st4(X + o, xr); st4(X + o + 4096, xi);
            st4(D + o, nd_r); st4(D + o + 4096, nd_i);
            st4(U1 + o, nu_r); st4(U1 + o + 4096, nu_i);
        }
    }
}

// K_E: V = AU1 + beta (AU2 + beta V) ; acc rt^H V
template <typename T>
__global__ void __launch_bounds__(256) k_E(T *V, T const *AU1, T const *AU2, uint32_t nnzb,
                                           uint16_t const *colindx, ColState const *cs, Acc *acc, uint32_t seed,
                                           float const *cf, uint32_t ncol) {
    __shared__ double red[4][64][3];
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const col = colindx[b]*64 + j;
        double const br = (sizeof(T) == 8) ? cs[col].be_re : 0.0, bi = (sizeof(T) == 8) ? cs[col].be_im : 0.0;
        double dr = 0, di = 0;
        if constexpr (sizeof(T) == 4) {
            float const fr = cf[2*size_t(ncol) + col], fi = cf[3*size_t(ncol) + col];
            float drf = 0.f, dif = 0.f;
#pragma unroll 8
            for (int i = q*16; i < q*16 + 16; ++i) {
                size_t const o = size_t(b)*kBlk + i*64 + j;
                float const vr = V[o], vi = V[o + 4096];
                float const t1r = fmaf(-fi, vi, fmaf(fr, vr, AU2[o])), t1i = fmaf(fi, vr, fmaf(fr, vi, AU2[o + 4096]));
                float const sr = fmaf(-fi, t1i, fmaf(fr, t1r, AU1[o])), si = fmaf(fi, t1r, fmaf(fr, t1i, AU1[o + 4096]));
                V[o] = sr; V[o + 4096] = si;
                uint32_t const idx = uint32_t(o);
                float const tr = shadow32(seed, idx), ti = shadow32(seed, idx + 4096u);
                drf = fmaf(tr, sr, fmaf(ti, si, drf)); dif = fmaf(tr, si, fmaf(-ti, sr, dif));
            }
            dr = double(drf); di = double(dif);
        } else
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j;
            double const vr = V[o], vi = V[o + 4096];
            double const tr1 = double(AU2[o]) + (br*vr - bi*vi), ti1 = double(AU2[o + 4096]) + (br*vi + bi*vr);
            double const nr = double(AU1[o]) + (br*tr1 - bi*ti1), ni = double(AU1[o + 4096]) + (br*ti1 + bi*tr1);
            T const sr = T(nr), si = T(ni);
            V[o] = sr; V[o + 4096] = si;
            uint32_t const idx = uint32_t(o);
            double const tr = shadow(seed, idx), ti = shadow(seed, idx + 4096u);
            dr += tr*double(sr) + ti*double(si); di += tr*double(si) - ti*double(sr);
        }
        reduce_cols(red, q, j, 0.0, dr, di, &acc[col], 3);
    }
}

// ------------------------------------------------------------------ scalar kernels (one thread per column)

__device__ __forceinline__ void cdiv(double ar, double ai, double br, double bi, double &r, double &i) {
    double const d = br*br + bi*bi;
    r = (ar*br + ai*bi)/d; i = (ai*br - ar*bi)/d;
}

__device__ __forceinline__ void freeze(ColState &s) {
    s.al_re = s.al_im = s.be_re = s.be_im = 0;
    s.cu1x_re = s.cu1x_im = s.cu2x_re = s.cu2x_im = s.cdx_re = s.cdx_im = 0;
    s.cu1d_re = s.cu1d_im = s.cdd_re = s.cdd_im = 0;
}

// the coefficients the FP32 vector kernels use, as float columns cf[i][ncol] (coalesced loads):
// alpha, beta, and the five complex K_DX coefficients
constexpr int kCoef = 14;
__device__ __forceinline__ void store_coef(float *cf, uint32_t ncol, uint32_t c, ColState const &s) {
    double const v[kCoef] = {s.al_re, s.al_im, s.be_re, s.be_im, s.cu1x_re, s.cu1x_im, s.cu2x_re, s.cu2x_im,
                             s.cdx_re, s.cdx_im, s.cu1d_re, s.cu1d_im, s.cdd_re, s.cdd_im};
#pragma unroll
    for (int i = 0; i < kCoef; ++i) cf[size_t(i)*ncol + c] = float(v[i]);
}

__global__ void s_init(ColState *cs, Acc *accW, Acc *accV, uint32_t ncol, int32_t *counters, float *cf) {
    uint32_t const c = blockIdx.x*blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    ColState s{};
    double const bn = sqrt(accW[c].n2);
    s.bnorm = bn; s.tau = bn; s.theta = 0; s.eta_re = s.eta_im = 0;
    s.tau_ref = bn; s.m_ref = 0;
    s.rho_re = accW[c].re; s.rho_im = accW[c].im;
    double const sr = accV[c].re, si = accV[c].im;
    if (!(bn > 0)) { s.status = 3; freeze(s); }
    else if (sr*sr + si*si == 0.0 || s.rho_re*s.rho_re + s.rho_im*s.rho_im == 0.0) { s.status = 2; freeze(s); atomicAdd(&counters[1], 1); }
    else { cdiv(s.rho_re, s.rho_im, sr, si, s.al_re, s.al_im); s.status = 0; }
    cs[c] = s;
    store_coef(cf, ncol, c, s);
    accW[c] = Acc{0, 0, 0, 0}; accV[c] = Acc{0, 0, 0, 0};
}

// first half step m = 2n-1
// the iteration number n (1-based) is counters[2] + 1: s_alpha advances it at the end of each
// iteration, so a captured iteration replays unchanged
__global__ void s_half1(ColState *cs, Acc *acc, uint32_t ncol, int32_t const *counters, double tol) {
    uint32_t const c = blockIdx.x*blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    int const m = 2*(counters[2] + 1) - 1;
    ColState s = cs[c];
    double const wn = sqrt(acc[c].n2);
    acc[c].n2 = 0;
    s.conv1 = 0;
    if (0 != s.status) { cs[c] = s; return; }
    double const th = wn/s.tau;
    double const c2 = 1.0/(1.0 + th*th);
    double const tau = s.tau*th*sqrt(c2);
    // kd = theta_{m-1}^2 eta_{m-1} / alpha ; eta = c^2 alpha
    double kr, ki; cdiv(s.theta*s.theta*s.eta_re, s.theta*s.theta*s.eta_im, s.al_re, s.al_im, kr, ki);
    s.kd1_re = kr; s.kd1_im = ki;
    s.et1_re = c2*s.al_re; s.et1_im = c2*s.al_im;
    s.theta = th; s.tau = tau;
    s.eta_re = s.et1_re; s.eta_im = s.et1_im;
    if (tau*sqrt(double(m) + 1.0) <= tol*s.bnorm) s.conv1 = 1;
    cs[c] = s;
}

// second half step m = 2n: coefficients of K_DX, beta, rho; counts active columns
// stall_level > 0 (FP32 correction sweeps only): a column whose estimate is already below
// stall_level and whose tau has not halved within stall_window half steps has reached the
// rounding floor of the sweep; it is frozen like a converged one (the refinement step then
// restarts from the true FP64 residual)
__global__ void s_half2(ColState *cs, Acc *acc, uint32_t ncol, double tol, int32_t *counters,
                        double stall_level, int stall_window, float *cf) {
    uint32_t const c = blockIdx.x*blockDim.x + threadIdx.x;
    if (c >= ncol) return;
    int const m = 2*(counters[2] + 1);
    ColState s = cs[c];
    double const wn = sqrt(acc[c].n2), rnr = acc[c].re, rni = acc[c].im;
    acc[c] = Acc{0, 0, 0, 0};
    if (0 != s.status) { freeze(s); cs[c] = s; store_coef(cf, ncol, c, s); return; }
    // first-half coefficients: D1 = U1 + kd1 D0 ; X1 = X0 + et1 D1
    double const k1r = s.kd1_re, k1i = s.kd1_im, e1r = s.et1_re, e1i = s.et1_im;
    if (s.conv1) {
        // X = X0 + et1 (U1 + kd1 D0); the column is done
        s.cu1x_re = e1r; s.cu1x_im = e1i; s.cu2x_re = s.cu2x_im = 0;
        s.cdx_re = e1r*k1r - e1i*k1i; s.cdx_im = e1r*k1i + e1i*k1r;
        s.cu1d_re = s.cu1d_im = s.cdd_re = s.cdd_im = 0;
        s.be_re = s.be_im = 0; s.al_re = s.al_im = 0;
        s.status = 1;
        cs[c] = s;
        store_coef(cf, ncol, c, s);
        return;
    }
    double const th = wn/s.tau;
    double const c2 = 1.0/(1.0 + th*th);
    double const tau = s.tau*th*sqrt(c2);
    double k2r, k2i; cdiv(s.theta*s.theta*s.eta_re, s.theta*s.theta*s.eta_im, s.al_re, s.al_im, k2r, k2i);
    double const e2r = c2*s.al_re, e2i = c2*s.al_im;
    // D2 = U2 + kd2 D1 = U2 + kd2 U1 + kd2 kd1 D0
    // X2 = X0 + et1 D1 + et2 D2 = X0 + (et1 + et2 kd2) U1 + et2 U2 + (et1 kd1 + et2 kd2 kd1) D0
    double const kkr = k2r*k1r - k2i*k1i, kki = k2r*k1i + k2i*k1r;       // kd2 kd1
    double const ekr = e2r*k2r - e2i*k2i, eki = e2r*k2i + e2i*k2r;       // et2 kd2
    s.cu1x_re = e1r + ekr; s.cu1x_im = e1i + eki;
    s.cu2x_re = e2r; s.cu2x_im = e2i;
    double const a1r = e1r*k1r - e1i*k1i, a1i = e1r*k1i + e1i*k1r;       // et1 kd1
    double const a2r = e2r*kkr - e2i*kki, a2i = e2r*kki + e2i*kkr;       // et2 kd2 kd1
    s.cdx_re = a1r + a2r; s.cdx_im = a1i + a2i;
    s.cu1d_re = k2r; s.cu1d_im = k2i;
    s.cdd_re = kkr; s.cdd_im = kki;
    s.theta = th; s.tau = tau; s.eta_re = e2r; s.eta_im = e2i;
    // beta = rho_n / rho_{n-1}
    double br, bi; cdiv(rnr, rni, s.rho_re, s.rho_im, br, bi);
    s.be_re = br; s.be_im = bi; s.rho_re = rnr; s.rho_im = rni;
    double const est = tau*sqrt(double(m) + 1.0);
    if (tau <= 0.5*s.tau_ref) { s.tau_ref = tau; s.m_ref = m; }
    if (est <= tol*s.bnorm) {
        s.status = 1; s.be_re = s.be_im = 0; s.al_re = s.al_im = 0;
    } else if (stall_level > 0 && m - s.m_ref > (est <= stall_level*s.bnorm ? stall_window : 4*stall_window)) {
        // FP32 sweep: no halving of tau for stall_window half steps below the stall level, or
        // for four times as long above it (a sweep that lost its way; the refinement restarts it)
        s.status = 4; s.be_re = s.be_im = 0; s.al_re = s.al_im = 0;
    } else if (rnr*rnr + rni*rni == 0.0) {
        s.status = 2; s.be_re = s.be_im = 0; s.al_re = s.al_im = 0; atomicAdd(&counters[1], 1);
    } else {
        atomicAdd(&counters[0], 1);
    }
    cs[c] = s;
    store_coef(cf, ncol, c, s);
}

// alpha = rho / (rt^H V)
__global__ void s_alpha(ColState *cs, Acc *acc, uint32_t ncol, int32_t *counters, float *cf) {
    uint32_t const c = blockIdx.x*blockDim.x + threadIdx.x;
    if (0 == c) counters[2] += 1;                   // next iteration (read only by later kernels)
    if (c >= ncol) return;
    ColState s = cs[c];
    double const sr = acc[c].re, si = acc[c].im;
    acc[c] = Acc{0, 0, 0, 0};
    // the K_DX coefficients have been applied: finished columns keep all-zero coefficients
    if (0 != s.status) { freeze(s); cs[c] = s; store_coef(cf, ncol, c, s); return; }
    if (sr*sr + si*si == 0.0) { s.status = 2; freeze(s); atomicAdd(&counters[1], 1); cs[c] = s; store_coef(cf, ncol, c, s); return; }
    cdiv(s.rho_re, s.rho_im, sr, si, s.al_re, s.al_im);
    cs[c] = s;
    store_coef(cf, ncol, c, s);
}

__global__ void s_estimate(ColState const *cs, uint32_t ncol, int m, double *out) {
    // max over active or converged columns of tau sqrt(m+1)/|b|
    __shared__ double r[256];
    double v = 0;
    for (uint32_t c = threadIdx.x; c < ncol; c += blockDim.x)
        if (cs[c].bnorm > 0) v = fmax(v, cs[c].tau*sqrt(double(m) + 1.0)/cs[c].bnorm);
    r[threadIdx.x] = v;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) { if (threadIdx.x < k) r[threadIdx.x] = fmax(r[threadIdx.x], r[threadIdx.x + k]); __syncthreads(); }
    if (0 == threadIdx.x) *out = r[0];
}

// ------------------------------------------------------------------ refinement helpers

// R = B - AX (FP64) and per-column |R|^2 into colnorm (atomics)
__global__ void __launch_bounds__(256) k_residual(double *R, double const *AX, uint32_t nnzb, uint16_t const *colindx,
                                                  uint32_t const *subset, double *colnorm) {
    __shared__ double red[4][64];
    int const j = threadIdx.x & 63, q = threadIdx.x >> 6;
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        uint32_t const c = colindx[b];
        bool const diag = (subset[c] == b);
        double n2 = 0;
#pragma unroll 8
        for (int i = q*16; i < q*16 + 16; ++i) {
            size_t const o = size_t(b)*kBlk + i*64 + j;
            double const rr = ((diag && i == j) ? 1.0 : 0.0) - AX[o], ri = -AX[o + 4096];
            R[o] = rr; R[o + 4096] = ri;
            n2 += rr*rr + ri*ri;
        }
        red[q][j] = n2;
        __syncthreads();
        if (0 == q) atomicAdd(&colnorm[c*64 + j], red[0][j] + red[1][j] + red[2][j] + red[3][j]);
        __syncthreads();
    }
}

// W = U1 = (T) R, D = 0  (right-hand side of a correction sweep)
template <typename T>
__global__ void __launch_bounds__(256) k_set_from(T *W, T *U1, T *D, double const *R, size_t n) {
    for (size_t e = blockIdx.x*size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x)*blockDim.x) {
        T const r = T(R[e]);
        W[e] = r; U1[e] = r; D[e] = T(0);
    }
}

// X64 += (double) dX  (end of an FP32 correction sweep)
template <typename T>
__global__ void __launch_bounds__(256) k_accumulate(double *X64, T const *dX, size_t n) {
    for (size_t e = blockIdx.x*size_t(blockDim.x) + threadIdx.x; e < n; e += size_t(gridDim.x)*blockDim.x)
        X64[e] += double(dX[e]);
}

__global__ void k_max_ratio(double const *colnorm, uint32_t ncol, double *out) {
    __shared__ double r[256];
    double v = 0;
    for (uint32_t c = threadIdx.x; c < ncol; c += blockDim.x) v = fmax(v, sqrt(colnorm[c]));
    r[threadIdx.x] = v;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) { if (threadIdx.x < k) r[threadIdx.x] = fmax(r[threadIdx.x], r[threadIdx.x + k]); __syncthreads(); }
    if (0 == threadIdx.x) *out = r[0];
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

unsigned grid_for(uint32_t nnzb) { return std::max(1u, std::min<uint32_t>(nnzb, 148u*8)); }

} // namespace

bool TfqmrVectors::alloc(size_t nreals, size_t elem_bytes) {
    if (n == nreals && elem == elem_bytes && X.ptr) return true;
    n = nreals; elem = elem_bytes;
    size_t const b = std::max<size_t>(16, nreals*elem_bytes);
    return X.alloc(b) && W.alloc(b) && U1.alloc(b) && U2.alloc(b) && V.alloc(b) && D.alloc(b) &&
           AU1.alloc(b) && AU2.alloc(b);
}

void TfqmrVectors::release() {
    X.release(); W.release(); U1.release(); U2.release(); V.release(); D.release();
    AU1.release(); AU2.release(); Rt.release(); n = 0; elem = 0;
}

SolverWorkspace::~SolverWorkspace() {
    if (host_counters) cudaFreeHost(host_counters);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
}

namespace {

// half steps without a halving of tau after which a column of an FP32 sweep counts as stalled
constexpr int kStallWindow = 60;

struct InnerResult { int iterations = 0; int converged = 0; int breakdowns = 0; double estimate = 0; double applications = 0; };

// tfQMR on the vectors of precision T whose W, U1 hold the right-hand side and D is zero;
// the solution is accumulated into Xs (precision TX), which holds the starting guess of the
// correction (zero for a plain solve)
template <typename T, typename TX>
bool tfqmr_inner(DevicePlan &dp, SolverWorkspace &ws, TfqmrVectors &v, TX *Xs, double tol, int maxit, int check_every,
                 uint32_t seed, cudaStream_t st, InnerResult &res, int echo, double stall_level = 0) {
    uint32_t const nnzb = dp.nnzb, ncol = dp.nCols*64;
    uint16_t const *ci = dptr<uint16_t>(dp.colindx);
    auto *cs = dptr<ColState>(ws.colstate);
    Acc *accA = (Acc*)(cs + ncol);     // two accumulator banks after the states
    auto *accB = accA + ncol;
    float *cf = reinterpret_cast<float*>(accB + ncol);   // kCoef float columns for the FP32 kernels
    int32_t *cnt = dptr<int32_t>(ws.counters);
    unsigned const g = grid_for(nnzb), gs = (ncol + 255)/256;
    TX *X = Xs;
    T *W = dptr<T>(v.W), *U1 = dptr<T>(v.U1), *U2 = dptr<T>(v.U2), *V = dptr<T>(v.V);
    T *D = dptr<T>(v.D), *AU1 = dptr<T>(v.AU1), *AU2 = dptr<T>(v.AU2);
    A43G_CUDA_TRY(cudaMemsetAsync(accA, 0, 2*size_t(ncol)*sizeof(Acc), st));
    A43G_CUDA_TRY(cudaMemsetAsync(cnt, 0, 4*sizeof(int32_t), st));
    // V = A U1
    if (!launch_action<T>(dp, AU1, U1, ci, st)) return false;
    A43G_CUDA_TRY(cudaMemcpyAsync(V, AU1, v.n*sizeof(T), cudaMemcpyDeviceToDevice, st));
    res.applications += 1;
    k_init_dots<T><<<g, 256, 0, st>>>(W, V, nnzb, ci, accA, accB, seed);
    count_launch();
    s_init<<<gs, 256, 0, st>>>(cs, accA, accB, ncol, cnt, cf);
    count_launch();
    // one iteration; counters[0] counts the columns still active after it
    auto iteration = [&]() -> bool {
        A43G_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int32_t), st));
        k_A<T><<<g, 256, 0, st>>>(U2, U1, V, W, AU1, nnzb, ci, cs, accA, cf, ncol);
        count_launch();
        s_half1<<<gs, 256, 0, st>>>(cs, accA, ncol, cnt, tol);
        count_launch();
        if (!launch_action<T>(dp, AU2, U2, ci, st)) return false;
        k_C<T><<<g, 256, 0, st>>>(W, AU1, AU2, nnzb, ci, cs, accA, seed, cf, ncol);
        count_launch();
        s_half2<<<gs, 256, 0, st>>>(cs, accA, ncol, tol, cnt, stall_level, kStallWindow, cf);
        count_launch();
        if constexpr (sizeof(T) == 4 && sizeof(TX) == 4)
            k_DX32<<<g, 256, 0, st>>>(X, D, U1, U2, W, nnzb, ci, cf, ncol);
        else
            k_DX<T, TX><<<g, 256, 0, st>>>(X, D, U1, U2, W, nnzb, ci, cs, cf, ncol);
        count_launch();
        if (!launch_action<T>(dp, AU1, U1, ci, st)) return false;
        k_E<T><<<g, 256, 0, st>>>(V, AU1, AU2, nnzb, ci, cs, accA, seed, cf, ncol);
        count_launch();
        s_alpha<<<gs, 256, 0, st>>>(cs, accA, ncol, cnt, cf);
        count_launch();
        return true;
    };
    // the iteration is captured once into a CUDA graph and replayed (one launch instead of
    // about 25 per iteration); not on the legacy default stream, which cannot be captured
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
    uint64_t const captured = per_iteration;
    int it = 0;
    for (it = 1; it <= maxit; ++it) {
        bool const check = (0 == it % check_every) || (it == maxit);
        if (exec) {
            A43G_CUDA_TRY(cudaGraphLaunch(exec, st));
            count_launches(captured);
        } else if (!iteration()) {
            return false;
        }
        res.applications += 2;
        if (check) {
            A43G_CUDA_TRY(cudaMemcpyAsync(ws.host_counters, cnt, 4*sizeof(int32_t), cudaMemcpyDeviceToHost, st));
            A43G_CUDA_TRY(cudaStreamSynchronize(st));
            if (echo > 1) {
                double *est = dptr<double>(ws.colnorm) + ncol;
                s_estimate<<<1, 256, 0, st>>>(cs, ncol, 2*it, est);
                count_launch();
                double e = 0;
                A43G_CUDA_TRY(cudaMemcpyAsync(&e, est, sizeof(double), cudaMemcpyDeviceToHost, st));
                A43G_CUDA_TRY(cudaStreamSynchronize(st));
                std::printf("# tfqmr<%s> iteration %d: %d of %u columns active, %d breakdowns, estimate %.3e\n",
                            sizeof(T) == 8 ? "f64" : "f32", it, ws.host_counters[0], ncol, ws.host_counters[1], e);
                std::fflush(stdout);
            }
            if (0 == ws.host_counters[0]) break;
        }
    }
    res.iterations += std::min(it, maxit);
    A43G_CUDA_TRY(cudaGetLastError());
    double *est = dptr<double>(ws.colnorm) + ncol;     // one spare double after the column norms
    s_estimate<<<1, 256, 0, st>>>(cs, ncol, 2*std::min(it, maxit), est);
    count_launch();
    A43G_CUDA_TRY(cudaMemcpyAsync(ws.host_counters, cnt, 4*sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    double e = 0;
    A43G_CUDA_TRY(cudaMemcpyAsync(&e, est, sizeof(double), cudaMemcpyDeviceToHost, st));
    A43G_CUDA_TRY(cudaStreamSynchronize(st));
    res.estimate = e;
    res.breakdowns += ws.host_counters[1];
    res.converged = (e <= tol) ? 1 : 0;
    if (echo > 0) std::printf("# tfqmr<%s> %d iterations, residual estimate %.3e (tolerance %.1e)\n",
                              sizeof(T) == 8 ? "f64" : "f32", std::min(it, maxit), e, tol);
    return true;
}

bool workspace_common(DevicePlan &dp, SolverWorkspace &ws) {
    size_t const ncol = size_t(dp.nCols)*64;
    if (!ws.colstate.alloc(ncol*(sizeof(ColState) + 2*sizeof(Acc) + kCoef*sizeof(float)))) return false;
    if (!ws.counters.alloc(64)) return false;
    if (!ws.colnorm.alloc((ncol + 8)*sizeof(double))) return false;
    if (!ws.host_counters) A43G_CUDA_TRY(cudaMallocHost(&ws.host_counters, 64));
    if (!ws.ev0) { A43G_CUDA_TRY(cudaEventCreate(&ws.ev0)); A43G_CUDA_TRY(cudaEventCreate(&ws.ev1)); }
    return true;
}

// true relative residual max_col |B - A X| / |B| for an FP64 solution X64 (|B col| = 1); R64 receives B - AX
bool residual64(DevicePlan &dp, SolverWorkspace &ws, double const *X64, double *R64, double *AX64, cudaStream_t st,
                double &rmax, double &applications) {
    uint32_t const ncol = dp.nCols*64;
    if (!launch_action<double>(dp, AX64, X64, dptr<uint16_t>(dp.colindx), st)) return false;
    applications += 1;
    double *cn = dptr<double>(ws.colnorm);
    A43G_CUDA_TRY(cudaMemsetAsync(cn, 0, (ncol + 8)*sizeof(double), st));
    k_residual<<<grid_for(dp.nnzb), 256, 0, st>>>(R64, AX64, dp.nnzb, dptr<uint16_t>(dp.colindx),
                                                  dptr<uint32_t>(dp.subset_dev), cn);
                                                  count_launch();
    k_max_ratio<<<1, 256, 0, st>>>(cn, ncol, cn + ncol);
    count_launch();
    A43G_CUDA_TRY(cudaMemcpyAsync(&rmax, cn + ncol, sizeof(double), cudaMemcpyDeviceToHost, st));
    A43G_CUDA_TRY(cudaStreamSynchronize(st));
    return true;
}

} // namespace

int solve(GreenPlan &hp, DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt,
          void *Xout, double *rho, a43g_solve_stats_t *stats, cudaStream_t st) {
    *stats = a43g_solve_stats_t{};
    if (0 == dp.nnzb) { stats->converged = 1; return A43G_OK; }
    if (!(opt.tolerance > 0) || opt.max_iterations < 1) { set_error("tolerance must be > 0 and max_iterations >= 1"); return A43G_ERR_ARGUMENT; }
    if (!dp.subset_dev.ptr) {
        std::vector<uint32_t> sub(hp.subset.begin(), hp.subset.end());
        if (!dp.subset_dev.alloc(std::max<size_t>(16, sub.size()*4))) return A43G_ERR_MEMORY;
        if (cudaSuccess != cudaMemcpy(dp.subset_dev.ptr, sub.data(), sub.size()*4, cudaMemcpyHostToDevice)) { set_error("copy of subset"); return A43G_ERR_CUDA; }
    }
    if (!workspace_common(dp, ws)) return A43G_ERR_MEMORY;
    size_t const n = size_t(dp.nnzb)*kBlk;
    int const check = std::max(1, opt.check_every);
    uint32_t const seed = uint32_t(opt.seed*2654435761ull + 12345u);
    cudaEventRecord(ws.ev0, st);
    InnerResult res;
    unsigned const g = grid_for(dp.nnzb);
    if (A43G_F64 == opt.precision) {
        if (!ws.v64.alloc(n, 8)) return A43G_ERR_MEMORY;
        auto &v = ws.v64;
        // W = U1 = B (unit diagonal blocks), D = X = 0
        for (DeviceBuffer *b : {&v.W, &v.U1, &v.D, &v.X})
            if (cudaSuccess != cudaMemsetAsync(b->ptr, 0, n*8, st)) { set_error("memset"); return A43G_ERR_CUDA; }
        k_set_diag<double><<<dp.nCols, 64, 0, st>>>(dptr<double>(v.W), dptr<double>(v.U1), dptr<uint32_t>(dp.subset_dev), dp.nCols);
        count_launch();
        if (!tfqmr_inner<double, double>(dp, ws, v, dptr<double>(v.X), opt.tolerance, opt.max_iterations, check, seed, st, res, opt.echo)) return A43G_ERR_CUDA;
        // true residual of the FP64 solution (uses U2/AU1 as scratch)
        double rmax = 0;
        if (!residual64(dp, ws, dptr<double>(v.X), dptr<double>(v.U2), dptr<double>(v.AU1), st, rmax, res.applications)) return A43G_ERR_CUDA;
        stats->residual_max = rmax;
        stats->refinements = 0;
        if (Xout) cudaMemcpyAsync(Xout, v.X.ptr, n*8, cudaMemcpyDeviceToDevice, st);
        if (rho) {
            DeviceBuffer rb; if (!rb.alloc(size_t(dp.nCols)*128*8)) return A43G_ERR_MEMORY;
            k_export_rho<double><<<dp.nCols, 64, 0, st>>>(dptr<double>(rb), dptr<double>(v.X), dptr<uint32_t>(dp.subset_dev), dp.nCols);
            count_launch();
            cudaMemcpyAsync(rho, rb.ptr, size_t(dp.nCols)*128*8, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
        }
    } else if (A43G_F32 == opt.precision) {
        // mixed precision: X64 = 0, R64 = B; repeat: solve A dX = R in FP32, X64 += dX, R64 = B - A X64
        if (!ws.v32.alloc(n, 4)) return A43G_ERR_MEMORY;
        if (!ws.X64.alloc(n*8) || !ws.R64.alloc(n*8) || !ws.AX64.alloc(n*8)) return A43G_ERR_MEMORY;
        double *X64 = dptr<double>(ws.X64), *R64 = dptr<double>(ws.R64), *AX64 = dptr<double>(ws.AX64);
        if (cudaSuccess != cudaMemsetAsync(X64, 0, n*8, st)) { set_error("memset"); return A43G_ERR_CUDA; }
        auto &v = ws.v32;
        double rmax = 1.0;
        // R64 = B - A*0 = B
        if (!residual64(dp, ws, X64, R64, AX64, st, rmax, res.applications)) return A43G_ERR_CUDA;
        int const maxref = std::max(1, opt.max_refinements);
        double const inner_tol = (opt.inner_tolerance > 0) ? opt.inner_tolerance : 1e-4;
        int ref = 0, first_sweep = 0;
        for (ref = 0; ref < maxref && rmax > opt.tolerance; ++ref) {
            k_set_from<float><<<g*8, 256, 0, st>>>(dptr<float>(v.W), dptr<float>(v.U1), dptr<float>(v.D), R64, n);
            count_launch();
            if (cudaSuccess != cudaMemsetAsync(v.X.ptr, 0, n*4, st)) { set_error("memset"); return A43G_ERR_CUDA; }
            int left = opt.max_iterations - res.iterations;
            if (left < 1) break;
            // a correction sweep that needs far more iterations than the first one has stagnated
            // at the FP32 rounding floor: end it, recompute the true residual and restart (with a
            // new shadow vector), which is cheaper than letting it run
            if (ref > 0) left = std::min(left, std::max(2*first_sweep, 100));
            // relative inner tolerance, not tighter than needed for the outer target
            double const itol = std::max(inner_tol, 0.5*opt.tolerance/rmax);
            // FP32 correction sweep (keeping its solution in FP64 does not lower the FP32 residual
            // floor, measured, so the correction is accumulated once per sweep)
            // columns stalled below 10x the sweep tolerance end the sweep (FP32 rounding floor)
            if (!tfqmr_inner<float, float>(dp, ws, v, dptr<float>(v.X), itol, left, check, seed + 7919u*uint32_t(ref + 1), st, res,
                                           opt.echo, 10*itol)) return A43G_ERR_CUDA;
            if (0 == ref) first_sweep = res.iterations;
            k_accumulate<float><<<g*8, 256, 0, st>>>(X64, dptr<float>(v.X), n);
            count_launch();
            if (!residual64(dp, ws, X64, R64, AX64, st, rmax, res.applications)) return A43G_ERR_CUDA;
            if (opt.echo > 0) std::printf("# refinement %d: FP64 residual %.3e after %d iterations in total\n",
                                          ref + 1, rmax, res.iterations);
        }
        stats->refinements = ref;
        stats->residual_max = rmax;
        if (Xout) cudaMemcpyAsync(Xout, X64, n*8, cudaMemcpyDeviceToDevice, st);
        if (rho) {
            DeviceBuffer rb; if (!rb.alloc(size_t(dp.nCols)*128*8)) return A43G_ERR_MEMORY;
            k_export_rho<double><<<dp.nCols, 64, 0, st>>>(dptr<double>(rb), X64, dptr<uint32_t>(dp.subset_dev), dp.nCols);
            count_launch();
            cudaMemcpyAsync(rho, rb.ptr, size_t(dp.nCols)*128*8, cudaMemcpyDeviceToHost, st);
            cudaStreamSynchronize(st);
        }
    } else {
        set_error("precision must be A43G_F64 or A43G_F32");
        return A43G_ERR_ARGUMENT;
    }
    cudaEventRecord(ws.ev1, st);
    if (cudaSuccess != cudaEventSynchronize(ws.ev1)) { set_error("event synchronize"); return A43G_ERR_CUDA; }
    float ms = 0; cudaEventElapsedTime(&ms, ws.ev0, ws.ev1);
    stats->seconds = ms*1e-3;
    stats->iterations = res.iterations;
    stats->breakdowns = res.breakdowns;
    stats->residual_estimate = res.estimate;
    stats->operator_applications = res.applications;
    stats->converged = (stats->residual_max <= opt.tolerance) ? 1 : 0;
    cudaError_t const e = cudaGetLastError();
    if (cudaSuccess != e) { set_error(std::string("solve: ") + cudaGetErrorString(e)); return A43G_ERR_CUDA; }
    return A43G_OK;
}

int solve_batched(GreenPlan &hp, DevicePlan &dp, SolverWorkspace &ws, a43g_solve_options_t const &opt,
                  int32_t n, double const *energies, double const *kpoints, double dVol,
                  double *rho, a43g_solve_stats_t *stats, cudaStream_t st) {
    for (int32_t i = 0; i < n; ++i) {
        hp.set_energy(energies[2*i], energies[2*i + 1], dVol);
        auto const err = hp.set_kpoint(kpoints + 3*i);
        if (!err.empty()) { set_error(err); return A43G_ERR_ARGUMENT; }
        if (!upload_values(hp, dp)) return A43G_ERR_CUDA;
        int const rc = solve(hp, dp, ws, opt, nullptr, rho ? rho + size_t(i)*dp.nCols*128 : nullptr, &stats[i], st);
        if (rc) return rc;
    }
    return A43G_OK;
}

} // namespace a43g
