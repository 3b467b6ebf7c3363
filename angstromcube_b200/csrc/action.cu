// The Green-function action y = (H - E S) x on sm_100a.
//
//  * local part (potential V - E and the finite-difference kinetic energy) in ONE pass:
//    local_fused_kernel walks the z-lines of cubes of one source column block, keeps the
//    z-stencil window in registers and stages the current cube and its four x/y neighbour
//    cubes in shared memory, so y is written exactly once per block (the reference makes
//    four passes that re-read and re-write y, include/green_action.hxx:159-167).
//    Plans with a 17-point stencil in some direction use the generic per-direction kernels.
//  * dyadic part (PAW projectors): projection, atom-matrix multiply, addition
//    (include/green_dyadic.hxx:856-922), with the image/atom coefficient scratch owned by
//    the plan instead of being allocated on every call.
#include "device.cuh"

#include <algorithm>

namespace a43g {

namespace {

constexpr int kBlockReals = 8192;   // 2 x 64 x 64

template <typename T>
struct Stencil9 { T c[3][5]; };      // per direction, c[0] centre ... c[4] distance 4

template <typename T>
Stencil9<T> make_stencil9(DevicePlan const &dp) {
    // 8th-order second derivative {-14350, 8064, -1008, 128, -9}/5040 times -1/(2h^2),
    // formed in double and rounded to real_t as include/green_kinetic.hxx:37-42 does
    Stencil9<T> s;
    double const w[5] = {-14350, 8064, -1008, 128, -9};
    for (int d = 0; d < 3; ++d) {
        double const norm = dp.prefactor[d]/5040.;
        for (int k = 0; k < 5; ++k) s.c[d][k] = T(w[k]*norm);
        if (dp.FD_range[d] < 1) for (int k = 0; k < 5; ++k) s.c[d][k] = T(0);
    }
    return s;
}

// energy and Bloch phases of one (energy, k-point) pair of a batch plan
template <typename T>
struct PairArgs { T E_re, E_im; T ph[3][2][2]; };

template <typename T>
struct LocalArgs {
    Stencil9<T> st;
    T E_re, E_im;
    T ph[3][2][2];                   // Bloch phases [dd][left,right][re,im]
    PairArgs<T> const *pairs;        // batch plan: per-pair values (nullptr: the values above)
    uint16_t const *colindx;         // block -> source column (batch plans and retirement)
    uint8_t const *active;           // per-source flag: 0 = retired, skip (nullptr: all active)
    uint32_t nsrc_pair;              // sources per pair
};

// the values of the pair that owns block b (uniform over a CTA that works on one z-line: the
// lines of a batch plan never mix sources); false if b's source is retired
template <typename T>
__device__ __forceinline__ bool line_args(LocalArgs<T> &a, int32_t b) {
    if (!a.colindx) return true;
    uint32_t const s = a.colindx[b];
    if (a.active && !a.active[s]) return false;
    if (a.pairs) {
        PairArgs<T> const &q = a.pairs[s/a.nsrc_pair];
        a.E_re = q.E_re; a.E_im = q.E_im;
#pragma unroll
        for (int d = 0; d < 3; ++d)
#pragma unroll
            for (int u = 0; u < 2; ++u) { a.ph[d][u][0] = q.ph[d][u][0]; a.ph[d][u][1] = q.ph[d][u][1]; }
    }
    return true;
}

// 4 consecutive points (x = 0..3 of one (z, y) row) of one column from shared memory
template <typename T> struct Row4 { T v[4]; };
template <typename T>
__device__ __forceinline__ Row4<T> lds_row(T const *p) {
    Row4<T> r;
    if (sizeof(T) == 4) {
        float4 const a = *reinterpret_cast<float4 const*>(p);
        r.v[0] = T(a.x); r.v[1] = T(a.y); r.v[2] = T(a.z); r.v[3] = T(a.w);
    } else {
        double2 const a = *reinterpret_cast<double2 const*>(p), b = *reinterpret_cast<double2 const*>(p + 2);
        r.v[0] = T(a.x); r.v[1] = T(a.y); r.v[2] = T(b.x); r.v[3] = T(b.y);
    }
    return r;
}
template <typename T>
__device__ __forceinline__ void sts_row(T *p, T const (&v)[4]) {
    if (sizeof(T) == 4) {
        *reinterpret_cast<float4*>(p) = make_float4(float(v[0]), float(v[1]), float(v[2]), float(v[3]));
    } else {
        *reinterpret_cast<double2*>(p) = make_double2(double(v[0]), double(v[1]));
        *reinterpret_cast<double2*>(p + 2) = make_double2(double(v[2]), double(v[3]));
    }
}

// 4 contiguous values from global memory (one potential row)
template <typename T>
__device__ __forceinline__ Row4<T> lds_row_global(T const *__restrict__ p) {
    Row4<T> r;
    if (sizeof(T) == 4) {
        float4 const a = __ldg(reinterpret_cast<float4 const*>(p));
        r.v[0] = T(a.x); r.v[1] = T(a.y); r.v[2] = T(a.z); r.v[3] = T(a.w);
    } else {
        double2 const a = __ldg(reinterpret_cast<double2 const*>(p)), b = __ldg(reinterpret_cast<double2 const*>(p) + 1);
        r.v[0] = T(a.x); r.v[1] = T(a.y); r.v[2] = T(b.x); r.v[3] = T(b.y);
    }
    return r;
}

// the row (z, y) = r of one cube (encoded e) for column col: 4 points x = 0..3, real and
// imaginary part, optionally rotated by a Bloch phase (pr, pi)
template <typename T>
__device__ __forceinline__ void load_row(T const *__restrict__ x, int32_t e, T pr, T pi, int r, int col,
                                         T (&re)[4], T (&im)[4]) {
    if (-1 == e) {
#pragma unroll
        for (int i = 0; i < 4; ++i) { re[i] = T(0); im[i] = T(0); }
        return;
    }
    T const *b = x + size_t(nbr_block(e))*kBlockReals + (r*4)*64 + col;
#pragma unroll
    for (int i = 0; i < 4; ++i) { re[i] = __ldg(b + i*64); im[i] = __ldg(b + 4096 + i*64); }
    if (e < -1) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            T const a = pr*re[i] - pi*im[i], c = pr*im[i] + pi*re[i];
            re[i] = a; im[i] = c;
        }
    }
}

// list entry (inzb+1, 0, -(inzb+1)) to neighbour code (>= 0 plain, -1 zero, <= -2 phase)
__device__ __forceinline__ int32_t list_code(int32_t entry) {
    return (entry > 0) ? entry - 1 : ((entry < 0) ? -(-entry - 1) - 2 : -1);
}

// One CTA per (z-line of cubes, slice of S columns).  Thread (j, r) owns row r = (z, y) of
// every cube of the line for column j: the x-stencil runs in registers (with the x-neighbour
// rows loaded directly), the y- and z-stencils read whole rows from shared memory, where the
// previous, current and next cube of the line and the two y-neighbour cubes are staged.
// Shared rows are padded to 68 points, so the 128-bit row accesses of a quarter warp hit
// distinct banks.
template <typename T, int S>
__global__ void __launch_bounds__(S*16)
local_fused_kernel(T *__restrict__ y, T const *__restrict__ x,
                   uint32_t const *__restrict__ zstart, int32_t const *__restrict__ zlist,
                   int32_t const *__restrict__ nbr, int32_t const *__restrict__ veff,
                   T const *__restrict__ Vcell, LocalArgs<T> a)
{
    constexpr int NSL = 64/S, PAD = 68;
    __shared__ __align__(16) T sm[5][2][S][PAD];   // slots: 3 rotating z-slots, y-, y+
    int const line = blockIdx.x/NSL, slice = blockIdx.x % NSL;
    int const j = threadIdx.x % S, r = threadIdx.x/S;       // r = z*4 + y
    int const zq = r >> 2, yq = r & 3, col = slice*S + j;
    int32_t const *L = zlist + zstart[line];
    int n = 0;
    while (L[4 + n] > 0) ++n;        // lists end with 4 non-positive entries
    if (0 == n || !line_args(a, L[4] - 1)) return;           // uniform over the CTA
    T const (&cx)[5] = a.st.c[0];
    T const (&cy)[5] = a.st.c[1];
    T const (&cz)[5] = a.st.c[2];
    T const c0 = cx[0] + cy[0] + cz[0];

    T cre[4], cim[4], nre[4], nim[4];
    {   // left z-halo into slot 0, first cube into slot 1
        T pre[4], pim[4];
        load_row(x, list_code(L[3]), a.ph[2][0][0], a.ph[2][0][1], r, col, pre, pim);
        sts_row(&sm[0][0][j][r*4], pre); sts_row(&sm[0][1][j][r*4], pim);
    }
    load_row(x, L[4] - 1, T(0), T(0), r, col, cre, cim);
    sts_row(&sm[1][0][j][r*4], cre); sts_row(&sm[1][1][j][r*4], cim);
    int sp = 0, sc = 1, sn = 2;                      // rotating slots: previous, current, next cube

    for (int k = 0; k < n; ++k) {
        int32_t const b = L[4 + k] - 1;
        int32_t const *nb = nbr + 6*size_t(b);
        int32_t const exm = nb[0], exp_ = nb[1], eym = nb[2], eyp = nb[3];
        load_row(x, list_code(L[5 + k]), a.ph[2][1][0], a.ph[2][1][1], r, col, nre, nim);
        T ymr[4], ymi[4], ypr[4], ypi[4];
        load_row(x, eym, a.ph[1][0][0], a.ph[1][0][1], r, col, ymr, ymi);
        load_row(x, eyp, a.ph[1][1][0], a.ph[1][1][1], r, col, ypr, ypi);
        T lr[12], li[12];                            // x-line: left row | own row | right row
        load_row(x, exm, a.ph[0][0][0], a.ph[0][0][1], r, col, *reinterpret_cast<T(*)[4]>(&lr[0]), *reinterpret_cast<T(*)[4]>(&li[0]));
        load_row(x, exp_, a.ph[0][1][0], a.ph[0][1][1], r, col, *reinterpret_cast<T(*)[4]>(&lr[8]), *reinterpret_cast<T(*)[4]>(&li[8]));
#pragma unroll
        for (int i = 0; i < 4; ++i) { lr[4 + i] = cre[i]; li[4 + i] = cim[i]; }
        __syncthreads();                             // previous step finished reading the slots
        sts_row(&sm[sn][0][j][r*4], nre); sts_row(&sm[sn][1][j][r*4], nim);
        sts_row(&sm[3][0][j][r*4], ymr); sts_row(&sm[3][1][j][r*4], ymi);
        sts_row(&sm[4][0][j][r*4], ypr); sts_row(&sm[4][1][j][r*4], ypi);
        __syncthreads();
        T accr[4], acci[4];
        {
            int32_t const iloc = veff[b];
            T V[4];
            if (iloc < 0) { V[0] = V[1] = V[2] = V[3] = T(0); }
            else { Row4<T> const v = lds_row_global(Vcell + size_t(iloc)*64 + r*4); V[0] = v.v[0]; V[1] = v.v[1]; V[2] = v.v[2]; V[3] = v.v[3]; }
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                T const Vt = V[i] - a.E_re;
                accr[i] = Vt*cre[i] + a.E_im*cim[i] + c0*cre[i];
                acci[i] = Vt*cim[i] - a.E_im*cre[i] + c0*cim[i];
            }
        }
        // x direction in registers
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int d = 1; d <= 4; ++d) {
                accr[i] += cx[d]*(lr[4 + i - d] + lr[4 + i + d]);
                acci[i] += cx[d]*(li[4 + i - d] + li[4 + i + d]);
            }
        // y and z directions: whole rows from shared memory
#pragma unroll
        for (int d = 1; d <= 4; ++d) {
            int const ym = yq - d, yp = yq + d, zm = zq - d, zp = zq + d;
            int const s_ym = (ym < 0) ? 3 : sc, s_yp = (yp > 3) ? 4 : sc;
            int const s_zm = (zm < 0) ? sp : sc, s_zp = (zp > 3) ? sn : sc;
            int const o_ym = (zq*4 + (ym & 3))*4, o_yp = (zq*4 + (yp & 3))*4;
            int const o_zm = ((zm & 3)*4 + yq)*4, o_zp = ((zp & 3)*4 + yq)*4;
            Row4<T> const r1 = lds_row(&sm[s_ym][0][j][o_ym]), r2 = lds_row(&sm[s_yp][0][j][o_yp]);
            Row4<T> const r3 = lds_row(&sm[s_zm][0][j][o_zm]), r4 = lds_row(&sm[s_zp][0][j][o_zp]);
            Row4<T> const i1 = lds_row(&sm[s_ym][1][j][o_ym]), i2 = lds_row(&sm[s_yp][1][j][o_yp]);
            Row4<T> const i3 = lds_row(&sm[s_zm][1][j][o_zm]), i4 = lds_row(&sm[s_zp][1][j][o_zp]);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                accr[i] += cy[d]*(r1.v[i] + r2.v[i]) + cz[d]*(r3.v[i] + r4.v[i]);
                acci[i] += cy[d]*(i1.v[i] + i2.v[i]) + cz[d]*(i3.v[i] + i4.v[i]);
            }
        }
        T *yb = y + size_t(b)*kBlockReals + (r*4)*64 + col;
#pragma unroll
        for (int i = 0; i < 4; ++i) { yb[i*64] = accr[i]; yb[4096 + i*64] = acci[i]; }
        int const t = sp; sp = sc; sc = sn; sn = t;  // rotate the z-slots
#pragma unroll
        for (int i = 0; i < 4; ++i) { cre[i] = nre[i]; cim[i] = nim[i]; }
    }
}

// The same fused local operator with the global loads of every step issued one step ahead:
// the neighbour codes of the whole z-line are read into shared memory once, so the rows of cube
// k+1 (its z-successor, its y and x neighbours and its potential row) are requested before cube
// k is computed and arrive while it is.  Bloch phases are applied when the rows are consumed.
// Lines of at most kMaxLine cubes (the host checks).
constexpr int kMaxLine = 128;

template <typename T> struct Rows { T re[4], im[4]; };

template <typename T>
__device__ __forceinline__ void row_raw(T const *__restrict__ x, int32_t e, int r, int col, Rows<T> &o) {
    if (-1 == e) {
#pragma unroll
        for (int i = 0; i < 4; ++i) { o.re[i] = T(0); o.im[i] = T(0); }
        return;
    }
    T const *b = x + size_t(nbr_block(e))*kBlockReals + (r*4)*64 + col;
#pragma unroll
    for (int i = 0; i < 4; ++i) { o.re[i] = __ldg(b + i*64); o.im[i] = __ldg(b + 4096 + i*64); }
}

template <typename T>
__device__ __forceinline__ void row_phase(int32_t e, T pr, T pi, Rows<T> &o) {
    if (e < -1) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            T const a = pr*o.re[i] - pi*o.im[i], c = pr*o.im[i] + pi*o.re[i];
            o.re[i] = a; o.im[i] = c;
        }
    }
}

template <typename T, int S>
__global__ void __launch_bounds__(S*16, 2)
local_fused_pf_kernel(T *__restrict__ y, T const *__restrict__ x,
                      uint32_t const *__restrict__ zstart, int32_t const *__restrict__ zlist,
                      int32_t const *__restrict__ nbr, int32_t const *__restrict__ veff,
                      T const *__restrict__ Vcell, LocalArgs<T> a)
{
    constexpr int NSL = 64/S, PAD = 68;
    __shared__ __align__(16) T sm[5][2][S][PAD];   // slots: 3 rotating z-slots, y-, y+
    __shared__ int32_t code[kMaxLine][8];           // per step: block, x-, x+, y-, y+, veff, z-next
    __shared__ int32_t zleft, nline;
    int const line = blockIdx.x/NSL, slice = blockIdx.x % NSL;
    int const tid = threadIdx.x, j = tid % S, r = tid/S;       // r = z*4 + y
    int const zq = r >> 2, yq = r & 3, col = slice*S + j;
    int32_t const *L = zlist + zstart[line];
    if (0 == tid) {
        int n = 0;
        while (L[4 + n] > 0) ++n;                   // lists end with 4 non-positive entries
        nline = n; zleft = list_code(L[3]);
    }
    __syncthreads();
    int const n = nline;
    if (0 == n || !line_args(a, L[4] - 1)) return;  // uniform: nothing on this line, or retired
    for (int k = tid; k < n; k += S*16) {
        int32_t const b = L[4 + k] - 1;
        int32_t const *nb = nbr + 6*size_t(b);
        code[k][0] = b; code[k][1] = nb[0]; code[k][2] = nb[1]; code[k][3] = nb[2]; code[k][4] = nb[3];
        code[k][5] = veff[b]; code[k][6] = list_code(L[5 + k]);
    }
    __syncthreads();
    T const (&cx)[5] = a.st.c[0];
    T const (&cy)[5] = a.st.c[1];
    T const (&cz)[5] = a.st.c[2];
    T const c0 = cx[0] + cy[0] + cz[0];

    Rows<T> cur;                                     // own row of the current cube
    {
        Rows<T> h;
        row_raw(x, zleft, r, col, h);
        row_phase(zleft, a.ph[2][0][0], a.ph[2][0][1], h);
        sts_row(&sm[0][0][j][r*4], h.re); sts_row(&sm[0][1][j][r*4], h.im);
    }
    row_raw(x, code[0][0], r, col, cur);
    sts_row(&sm[1][0][j][r*4], cur.re); sts_row(&sm[1][1][j][r*4], cur.im);
    // rows of step 0 requested before the loop
    Rows<T> pz, pym, pyp, pxm, pxp;
    Row4<T> pV;
    auto request = [&](int k) {
        row_raw(x, code[k][6], r, col, pz);
        row_raw(x, code[k][3], r, col, pym);
        row_raw(x, code[k][4], r, col, pyp);
        row_raw(x, code[k][1], r, col, pxm);
        row_raw(x, code[k][2], r, col, pxp);
        int32_t const iloc = code[k][5];
        if (iloc < 0) { pV.v[0] = pV.v[1] = pV.v[2] = pV.v[3] = T(0); }
        else pV = lds_row_global(Vcell + size_t(iloc)*64 + r*4);
    };
    request(0);
    int sp = 0, sc = 1, sn = 2;
    for (int k = 0; k < n; ++k) {
        int32_t const b = code[k][0];
        row_phase(code[k][6], a.ph[2][1][0], a.ph[2][1][1], pz);
        row_phase(code[k][3], a.ph[1][0][0], a.ph[1][0][1], pym);
        row_phase(code[k][4], a.ph[1][1][0], a.ph[1][1][1], pyp);
        row_phase(code[k][1], a.ph[0][0][0], a.ph[0][0][1], pxm);
        row_phase(code[k][2], a.ph[0][1][0], a.ph[0][1][1], pxp);
        __syncthreads();                             // previous step finished reading the slots
        sts_row(&sm[sn][0][j][r*4], pz.re);  sts_row(&sm[sn][1][j][r*4], pz.im);
        sts_row(&sm[3][0][j][r*4], pym.re);  sts_row(&sm[3][1][j][r*4], pym.im);
        sts_row(&sm[4][0][j][r*4], pyp.re);  sts_row(&sm[4][1][j][r*4], pyp.im);
        __syncthreads();
        T lr[12], li[12];                            // x-line: left row | own row | right row
        T V[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            lr[i] = pxm.re[i]; li[i] = pxm.im[i];
            lr[4 + i] = cur.re[i]; li[4 + i] = cur.im[i];
            lr[8 + i] = pxp.re[i]; li[8 + i] = pxp.im[i];
            V[i] = pV.v[i];
        }
        Rows<T> const nextc = pz;
        if (k + 1 < n) request(k + 1);               // arrives while this cube is computed
        T accr[4], acci[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            T const Vt = V[i] - a.E_re;
            accr[i] = Vt*cur.re[i] + a.E_im*cur.im[i] + c0*cur.re[i];
            acci[i] = Vt*cur.im[i] - a.E_im*cur.re[i] + c0*cur.im[i];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int d = 1; d <= 4; ++d) {
                accr[i] += cx[d]*(lr[4 + i - d] + lr[4 + i + d]);
                acci[i] += cx[d]*(li[4 + i - d] + li[4 + i + d]);
            }
#pragma unroll
        for (int d = 1; d <= 4; ++d) {
            int const ym = yq - d, yp = yq + d, zm = zq - d, zp = zq + d;
            int const s_ym = (ym < 0) ? 3 : sc, s_yp = (yp > 3) ? 4 : sc;
            int const s_zm = (zm < 0) ? sp : sc, s_zp = (zp > 3) ? sn : sc;
            int const o_ym = (zq*4 + (ym & 3))*4, o_yp = (zq*4 + (yp & 3))*4;
            int const o_zm = ((zm & 3)*4 + yq)*4, o_zp = ((zp & 3)*4 + yq)*4;
            Row4<T> const r1 = lds_row(&sm[s_ym][0][j][o_ym]), r2 = lds_row(&sm[s_yp][0][j][o_yp]);
            Row4<T> const r3 = lds_row(&sm[s_zm][0][j][o_zm]), r4 = lds_row(&sm[s_zp][0][j][o_zp]);
            Row4<T> const i1 = lds_row(&sm[s_ym][1][j][o_ym]), i2 = lds_row(&sm[s_yp][1][j][o_yp]);
            Row4<T> const i3 = lds_row(&sm[s_zm][1][j][o_zm]), i4 = lds_row(&sm[s_zp][1][j][o_zp]);
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                accr[i] += cy[d]*(r1.v[i] + r2.v[i]) + cz[d]*(r3.v[i] + r4.v[i]);
                acci[i] += cy[d]*(i1.v[i] + i2.v[i]) + cz[d]*(i3.v[i] + i4.v[i]);
            }
        }
        T *yb = y + size_t(b)*kBlockReals + (r*4)*64 + col;
#pragma unroll
        for (int i = 0; i < 4; ++i) { yb[i*64] = accr[i]; yb[4096 + i*64] = acci[i]; }
        int const t = sp; sp = sc; sc = sn; sn = t;  // rotate the z-slots
        cur = nextc;
    }
}

// Pencil variant (FP32): one CTA per (z-line, slice of S = 32 columns); thread (zq, j) owns the
// four y-rows (zq, y = 0..3) of every cube of the line for column j, so one warp covers 32
// consecutive columns of one z-plane (128-byte loads and stores).  The x- and y-stencils run in
// registers: the x- and y-neighbour rows come straight from global memory (the L2) and are
// applied in scatter form as they arrive.  Only the z-stencil reads shared memory, where the
// previous, current and next cube of the line are staged as 16-byte rows, [slot][plane][row][S]
// (a quarter warp reads 128 contiguous bytes: no bank conflicts).  Per output point this reads
// half the shared-memory bytes of the row kernel above and passes a barrier a quarter as often.
// The z-successor of the next cube is requested one step ahead.
constexpr int kPencilS = 32;
constexpr int kPencilSmem = 3*2*16*kPencilS*16;   // bytes of the three z-slots

struct Quad { float v[2][16]; };                 // [plane][y*4 + x] of one z-plane of a cube

__device__ __forceinline__ void quad_raw(float const *__restrict__ x, int32_t e, int zq, int col, Quad &q) {
    if (-1 == e) {
#pragma unroll
        for (int i = 0; i < 16; ++i) { q.v[0][i] = 0.f; q.v[1][i] = 0.f; }
        return;
    }
    float const *b = x + size_t(nbr_block(e))*kBlockReals + (zq*16)*64 + col;
#pragma unroll
    for (int i = 0; i < 16; ++i) { q.v[0][i] = __ldg(b + i*64); q.v[1][i] = __ldg(b + 4096 + i*64); }
}

__device__ __forceinline__ void quad_phase(int32_t e, float pr, float pi, Quad &q) {
    if (e < -1) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float const a = pr*q.v[0][i] - pi*q.v[1][i], c = pr*q.v[1][i] + pi*q.v[0][i];
            q.v[0][i] = a; q.v[1][i] = c;
        }
    }
}

__global__ void __launch_bounds__(4*kPencilS, 4)
local_pencil_kernel(float *__restrict__ y, float const *__restrict__ x,
                    uint32_t const *__restrict__ zstart, int32_t const *__restrict__ zlist,
                    int32_t const *__restrict__ nbr, int32_t const *__restrict__ veff,
                    float const *__restrict__ Vcell, LocalArgs<float> a)
{
    constexpr int S = kPencilS, NSL = 64/S;
    extern __shared__ __align__(16) float4 slot4[];   // [3][2][16][S]
    __shared__ int32_t code[kMaxLine][8];              // per step: block, x-, x+, y-, y+, veff, z-next
    __shared__ int32_t zleft, nline;
    int const line = blockIdx.x/NSL, slice = blockIdx.x % NSL;
    int const tid = threadIdx.x, j = tid % S, zq = tid/S, col = slice*S + j;
    int32_t const *L = zlist + zstart[line];
    if (0 == tid) {
        int n = 0;
        while (L[4 + n] > 0) ++n;                   // lists end with 4 non-positive entries
        nline = n; zleft = list_code(L[3]);
    }
    __syncthreads();
    int const n = nline;
    if (0 == n || !line_args(a, L[4] - 1)) return;  // uniform: nothing on this line, or retired
    for (int k = tid; k < n; k += 4*S) {
        int32_t const b = L[4 + k] - 1;
        int32_t const *nb = nbr + 6*size_t(b);
        code[k][0] = b; code[k][1] = nb[0]; code[k][2] = nb[1]; code[k][3] = nb[2]; code[k][4] = nb[3];
        code[k][5] = veff[b]; code[k][6] = list_code(L[5 + k]);
    }
    auto srow = [&](int slot, int pl, int row) -> float4 & { return slot4[((slot*2 + pl)*16 + row)*S + j]; };
    auto put = [&](int slot, Quad const &q) {
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int pl = 0; pl < 2; ++pl)
                srow(slot, pl, zq*4 + yy) = make_float4(q.v[pl][yy*4], q.v[pl][yy*4 + 1], q.v[pl][yy*4 + 2], q.v[pl][yy*4 + 3]);
    };
    float const (&cx)[5] = a.st.c[0];
    float const (&cy)[5] = a.st.c[1];
    float const (&cz)[5] = a.st.c[2];
    float const c0 = cx[0] + cy[0] + cz[0];
    __syncthreads();                                // code[] complete
    {
        Quad h;
        quad_raw(x, zleft, zq, col, h);
        quad_phase(zleft, a.ph[2][0][0], a.ph[2][0][1], h);
        put(0, h);
        quad_raw(x, code[0][0], zq, col, h);
        put(1, h);
    }
    Quad nx;                                        // rows of the z-successor, one step ahead
    quad_raw(x, code[0][6], zq, col, nx);
    int sp = 0, sc = 1, sn = 2;
    for (int k = 0; k < n; ++k) {
        int32_t const b = code[k][0];
        quad_phase(code[k][6], a.ph[2][1][0], a.ph[2][1][1], nx);   // only the line end has a phase
        __syncthreads();                            // the previous step finished reading slot sn
        put(sn, nx);
        __syncthreads();
        if (k + 1 < n) quad_raw(x, code[k + 1][6], zq, col, nx);   // arrives during this step
        Quad cur;
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int pl = 0; pl < 2; ++pl) {
                float4 const v = srow(sc, pl, zq*4 + yy);
                cur.v[pl][yy*4] = v.x; cur.v[pl][yy*4 + 1] = v.y; cur.v[pl][yy*4 + 2] = v.z; cur.v[pl][yy*4 + 3] = v.w;
            }
        float acc[2][16];
        // potential and centre
        int32_t const iloc = code[k][5];
        float V[16];
        if (iloc < 0) {
#pragma unroll
            for (int i = 0; i < 16; ++i) V[i] = 0.f;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 const v = __ldg(reinterpret_cast<float4 const*>(Vcell + size_t(iloc)*64 + zq*16 + q*4));
                V[q*4] = v.x; V[q*4 + 1] = v.y; V[q*4 + 2] = v.z; V[q*4 + 3] = v.w;
            }
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float const Vt = V[i] - a.E_re;
            acc[0][i] = Vt*cur.v[0][i] + a.E_im*cur.v[1][i] + c0*cur.v[0][i];
            acc[1][i] = Vt*cur.v[1][i] - a.E_im*cur.v[0][i] + c0*cur.v[1][i];
        }
        // y-stencil inside the cube
#pragma unroll
        for (int pl = 0; pl < 2; ++pl)
#pragma unroll
            for (int yy = 0; yy < 4; ++yy)
#pragma unroll
                for (int yo = 0; yo < 4; ++yo) {
                    if (yo == yy) continue;
                    int const d = (yo > yy) ? yo - yy : yy - yo;
#pragma unroll
                    for (int i = 0; i < 4; ++i) acc[pl][yy*4 + i] += cy[d]*cur.v[pl][yo*4 + i];
                }
        // x-stencil: the rows of the x-neighbours at (zq, yy)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
            Rows<float> xm, xp;
            row_raw(x, code[k][1], zq*4 + yy, col, xm);
            row_raw(x, code[k][2], zq*4 + yy, col, xp);
            row_phase(code[k][1], a.ph[0][0][0], a.ph[0][0][1], xm);
            row_phase(code[k][2], a.ph[0][1][0], a.ph[0][1][1], xp);
            float lr[12], li[12];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                lr[i] = xm.re[i]; li[i] = xm.im[i];
                lr[4 + i] = cur.v[0][yy*4 + i]; li[4 + i] = cur.v[1][yy*4 + i];
                lr[8 + i] = xp.re[i]; li[8 + i] = xp.im[i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int d = 1; d <= 4; ++d) {
                    acc[0][yy*4 + i] += cx[d]*(lr[4 + i - d] + lr[4 + i + d]);
                    acc[1][yy*4 + i] += cx[d]*(li[4 + i - d] + li[4 + i + d]);
                }
        }
        // y-neighbour cubes: row yo of y- sits at y = yo - 4, row yo of y+ at y = yo + 4
#pragma unroll
        for (int yo = 0; yo < 4; ++yo) {
            Rows<float> ym, yp;
            row_raw(x, code[k][3], zq*4 + yo, col, ym);
            row_raw(x, code[k][4], zq*4 + yo, col, yp);
            row_phase(code[k][3], a.ph[1][0][0], a.ph[1][0][1], ym);
            row_phase(code[k][4], a.ph[1][1][0], a.ph[1][1][1], yp);
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) {
                if (yy <= yo) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        acc[0][yy*4 + i] += cy[yy - yo + 4]*ym.re[i];
                        acc[1][yy*4 + i] += cy[yy - yo + 4]*ym.im[i];
                    }
                }
                if (yy >= yo) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        acc[0][yy*4 + i] += cy[yo + 4 - yy]*yp.re[i];
                        acc[1][yy*4 + i] += cy[yo + 4 - yy]*yp.im[i];
                    }
                }
            }
        }
        // z-stencil from the three staged cubes (previous, current, next)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int d = 1; d <= 4; ++d) {
                int const zm = zq - d, zp = zq + d;
                int const s_m = (zm < 0) ? sp : sc, s_p = (zp > 3) ? sn : sc;
                int const r_m = (zm & 3)*4 + yy, r_p = (zp & 3)*4 + yy;
#pragma unroll
                for (int pl = 0; pl < 2; ++pl) {
                    float4 const m = srow(s_m, pl, r_m), p = srow(s_p, pl, r_p);
                    acc[pl][yy*4 + 0] += cz[d]*(m.x + p.x);
                    acc[pl][yy*4 + 1] += cz[d]*(m.y + p.y);
                    acc[pl][yy*4 + 2] += cz[d]*(m.z + p.z);
                    acc[pl][yy*4 + 3] += cz[d]*(m.w + p.w);
                }
            }
        float *yb = y + size_t(b)*kBlockReals + (zq*16)*64 + col;
#pragma unroll
        for (int i = 0; i < 16; ++i) { yb[i*64] = acc[0][i]; yb[4096 + i*64] = acc[1][i]; }
        int const t = sp; sp = sc; sc = sn; sn = t;  // rotate the z-slots
    }
}

// Pencil variant in FP64: the pencil kernel's mapping with the two planes on two threads.  One
// CTA of 128 threads per (z-line, slice of 16 columns); thread (zq, plane, j) owns one plane (re
// or im) of the four y-rows (zq, y = 0..3) of every cube of the line for column j, so a warp is
// one z-plane: 16 consecutive columns of the real plane and the same columns of the imaginary
// plane (two 128-byte segments per load).  The only couplings of the planes, -i Im(E) x and the
// Bloch phases of halo cubes, take the partner plane's values by a warp shuffle (lane ^ 16).
// Registers hold the same number of values as the FP32 kernel's, at twice the bytes.
constexpr int kPencil64S = 16;
constexpr int kPencil64Smem = 3*2*16*kPencil64S*32;   // bytes of the three z-slots (double4 rows)

struct Quad64 { double v[16]; };                     // one plane of [y*4 + x] of one z-plane of a cube

__device__ __forceinline__ void quad64_raw(double const *__restrict__ x, int32_t e, int zq, int pl, int col, Quad64 &q) {
    if (-1 == e) {
#pragma unroll
        for (int i = 0; i < 16; ++i) q.v[i] = 0.0;
        return;
    }
    double const *b = x + size_t(nbr_block(e))*kBlockReals + pl*4096 + (zq*16)*64 + col;
#pragma unroll
    for (int i = 0; i < 16; ++i) q.v[i] = __ldg(b + i*64);
}

// rotation by the Bloch phase (pr, pi) of a halo cube, uniform over the CTA: re' = pr re - pi im,
// im' = pr im + pi re, with the other plane from the partner lane
__device__ __forceinline__ double phase64(double v, int pl, double pr, double pi) {
    double const w = __shfl_xor_sync(0xffffffffu, v, 16);
    return pr*v + (pl ? pi : -pi)*w;
}

__global__ void __launch_bounds__(8*kPencil64S, 3)
local_pencil64_kernel(double *__restrict__ y, double const *__restrict__ x,
                      uint32_t const *__restrict__ zstart, int32_t const *__restrict__ zlist,
                      int32_t const *__restrict__ nbr, int32_t const *__restrict__ veff,
                      double const *__restrict__ Vcell, LocalArgs<double> a)
{
    constexpr int S = kPencil64S, NSL = 64/S;
    extern __shared__ __align__(16) double4 slot64[];  // [3][2][16][S]
    __shared__ int32_t code[kMaxLine][8];              // per step: block, x-, x+, y-, y+, veff, z-next
    __shared__ int32_t zleft, nline;
    int const line = blockIdx.x/NSL, slice = blockIdx.x % NSL;
    int const tid = threadIdx.x, lane = tid & 31, zq = tid >> 5;
    int const pl = lane >> 4, j = lane & 15, col = slice*S + j;
    int32_t const *L = zlist + zstart[line];
    if (0 == tid) {
        int n = 0;
        while (L[4 + n] > 0) ++n;                   // lists end with 4 non-positive entries
        nline = n; zleft = list_code(L[3]);
    }
    __syncthreads();
    int const n = nline;
    if (0 == n || !line_args(a, L[4] - 1)) return;  // uniform: nothing on this line, or retired
    for (int k = tid; k < n; k += 8*S) {
        int32_t const b = L[4 + k] - 1;
        int32_t const *nb = nbr + 6*size_t(b);
        code[k][0] = b; code[k][1] = nb[0]; code[k][2] = nb[1]; code[k][3] = nb[2]; code[k][4] = nb[3];
        code[k][5] = veff[b]; code[k][6] = list_code(L[5 + k]);
    }
    auto srow = [&](int slot, int plane, int row) -> double4 & { return slot64[((slot*2 + plane)*16 + row)*S + j]; };
    auto put = [&](int slot, Quad64 const &q) {
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
            srow(slot, pl, zq*4 + yy) = make_double4(q.v[yy*4], q.v[yy*4 + 1], q.v[yy*4 + 2], q.v[yy*4 + 3]);
    };
    auto qphase = [&](int32_t e, double pr, double pi, Quad64 &q) {
        if (e < -1) {
#pragma unroll
            for (int i = 0; i < 16; ++i) q.v[i] = phase64(q.v[i], pl, pr, pi);
        }
    };
    double const (&cx)[5] = a.st.c[0];
    double const (&cy)[5] = a.st.c[1];
    double const (&cz)[5] = a.st.c[2];
    double const c0 = cx[0] + cy[0] + cz[0];
    double const Eim = pl ? -a.E_im : a.E_im;       // re: + Im(E) im, im: - Im(E) re
    __syncthreads();                                // code[] complete
    {
        Quad64 h;
        quad64_raw(x, zleft, zq, pl, col, h);
        qphase(zleft, a.ph[2][0][0], a.ph[2][0][1], h);
        put(0, h);
        quad64_raw(x, code[0][0], zq, pl, col, h);
        put(1, h);
    }
    Quad64 nx;                                      // rows of the z-successor, one step ahead
    quad64_raw(x, code[0][6], zq, pl, col, nx);
    int sp = 0, sc = 1, sn = 2;
    for (int k = 0; k < n; ++k) {
        int32_t const b = code[k][0];
        qphase(code[k][6], a.ph[2][1][0], a.ph[2][1][1], nx);       // only the line end has a phase
        __syncthreads();                            // the previous step finished reading slot sn
        put(sn, nx);
        __syncthreads();
        if (k + 1 < n) quad64_raw(x, code[k + 1][6], zq, pl, col, nx);   // arrives during this step
        double cur[16];
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
            double4 const v = srow(sc, pl, zq*4 + yy);
            cur[yy*4] = v.x; cur[yy*4 + 1] = v.y; cur[yy*4 + 2] = v.z; cur[yy*4 + 3] = v.w;
        }
        double acc[16];
        // potential and centre; the other plane of the own points from the partner lane
        int32_t const iloc = code[k][5];
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            double const V = (iloc < 0) ? 0.0 : __ldg(Vcell + size_t(iloc)*64 + zq*16 + i);
            double const w = __shfl_xor_sync(0xffffffffu, cur[i], 16);
            acc[i] = (V - a.E_re)*cur[i] + Eim*w + c0*cur[i];
        }
        // y-stencil inside the cube
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int yo = 0; yo < 4; ++yo) {
                if (yo == yy) continue;
                int const d = (yo > yy) ? yo - yy : yy - yo;
#pragma unroll
                for (int i = 0; i < 4; ++i) acc[yy*4 + i] += cy[d]*cur[yo*4 + i];
            }
        // x-stencil: the rows of the x-neighbours at (zq, yy)
        int32_t const exm = code[k][1], exp_ = code[k][2], eym = code[k][3], eyp = code[k][4];
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
            double xm[4], xp[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                xm[i] = (-1 == exm) ? 0.0 : __ldg(x + size_t(nbr_block(exm))*kBlockReals + pl*4096 + (zq*16 + yy*4 + i)*64 + col);
                xp[i] = (-1 == exp_) ? 0.0 : __ldg(x + size_t(nbr_block(exp_))*kBlockReals + pl*4096 + (zq*16 + yy*4 + i)*64 + col);
            }
            if (exm < -1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) xm[i] = phase64(xm[i], pl, a.ph[0][0][0], a.ph[0][0][1]);
            }
            if (exp_ < -1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) xp[i] = phase64(xp[i], pl, a.ph[0][1][0], a.ph[0][1][1]);
            }
            double l[12];
#pragma unroll
            for (int i = 0; i < 4; ++i) { l[i] = xm[i]; l[4 + i] = cur[yy*4 + i]; l[8 + i] = xp[i]; }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int d = 1; d <= 4; ++d) acc[yy*4 + i] += cx[d]*(l[4 + i - d] + l[4 + i + d]);
        }
        // y-neighbour cubes: row yo of y- sits at y = yo - 4, row yo of y+ at y = yo + 4
#pragma unroll
        for (int yo = 0; yo < 4; ++yo) {
            double ym[4], yp[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                ym[i] = (-1 == eym) ? 0.0 : __ldg(x + size_t(nbr_block(eym))*kBlockReals + pl*4096 + (zq*16 + yo*4 + i)*64 + col);
                yp[i] = (-1 == eyp) ? 0.0 : __ldg(x + size_t(nbr_block(eyp))*kBlockReals + pl*4096 + (zq*16 + yo*4 + i)*64 + col);
            }
            if (eym < -1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) ym[i] = phase64(ym[i], pl, a.ph[1][0][0], a.ph[1][0][1]);
            }
            if (eyp < -1) {
#pragma unroll
                for (int i = 0; i < 4; ++i) yp[i] = phase64(yp[i], pl, a.ph[1][1][0], a.ph[1][1][1]);
            }
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) {
                if (yy <= yo) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) acc[yy*4 + i] += cy[yy - yo + 4]*ym[i];
                }
                if (yy >= yo) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) acc[yy*4 + i] += cy[yo + 4 - yy]*yp[i];
                }
            }
        }
        // z-stencil from the three staged cubes (previous, current, next)
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int d = 1; d <= 4; ++d) {
                int const zm = zq - d, zp = zq + d;
                int const s_m = (zm < 0) ? sp : sc, s_p = (zp > 3) ? sn : sc;
                int const r_m = (zm & 3)*4 + yy, r_p = (zp & 3)*4 + yy;
                double4 const m = srow(s_m, pl, r_m), p = srow(s_p, pl, r_p);
                acc[yy*4 + 0] += cz[d]*(m.x + p.x);
                acc[yy*4 + 1] += cz[d]*(m.y + p.y);
                acc[yy*4 + 2] += cz[d]*(m.z + p.z);
                acc[yy*4 + 3] += cz[d]*(m.w + p.w);
            }
        double *yb = y + size_t(b)*kBlockReals + pl*4096 + (zq*16)*64 + col;
#pragma unroll
        for (int i = 0; i < 16; ++i) yb[i*64] = acc[i];
        int const t = sp; sp = sc; sc = sn; sn = t;  // rotate the z-slots
    }
}

// Pencils with staged lateral cubes (FP32): the thread mapping and arithmetic of
// local_pencil_kernel, but the four x- and y-neighbour cubes of step k + 1 are copied into shared
// memory with 16-byte cp.async while step k is computed, so the stencil reads only shared memory
// and registers and the neighbour rows' L2 latency is hidden behind a whole step.  The lateral
// stage holds [2 steps][x-, x+, y-, y+][re, im][64 rows][32 columns]; one CTA per SM.
constexpr int kStageLat = 4*2*64*kPencilS;                       // floats of one step's laterals
constexpr int kStageSmem = kPencilSmem + 2*kStageLat*4;          // bytes: z-slots + two lateral steps

__device__ __forceinline__ uint32_t smem_addr_u32(void const *p) { return uint32_t(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void cp_async16_cg(void *dst, void const *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_addr_u32(dst)), "l"(src) : "memory");
}

__global__ void __launch_bounds__(4*kPencilS, 1)
local_stage_kernel(float *__restrict__ y, float const *__restrict__ x,
                   uint32_t const *__restrict__ zstart, int32_t const *__restrict__ zlist,
                   int32_t const *__restrict__ nbr, int32_t const *__restrict__ veff,
                   float const *__restrict__ Vcell, LocalArgs<float> a)
{
    constexpr int S = kPencilS, NSL = 64/S;
    extern __shared__ __align__(16) float4 slot4[];   // [3][2][16][S] float4, then the lateral stages
    float *lat = reinterpret_cast<float*>(slot4 + 3*2*16*S);
    __shared__ int32_t code[kMaxLine][8];              // per step: block, x-, x+, y-, y+, veff, z-next
    __shared__ int32_t zleft, nline;
    int const line = blockIdx.x/NSL, slice = blockIdx.x % NSL;
    int const tid = threadIdx.x, j = tid % S, zq = tid/S, col = slice*S + j;
    int32_t const *L = zlist + zstart[line];
    if (0 == tid) {
        int n = 0;
        while (L[4 + n] > 0) ++n;                   // lists end with 4 non-positive entries
        nline = n; zleft = list_code(L[3]);
    }
    __syncthreads();
    int const n = nline;
    if (0 == n || !line_args(a, L[4] - 1)) return;  // uniform: nothing on this line, or retired
    for (int k = tid; k < n; k += 4*S) {
        int32_t const b = L[4 + k] - 1;
        int32_t const *nb = nbr + 6*size_t(b);
        code[k][0] = b; code[k][1] = nb[0]; code[k][2] = nb[1]; code[k][3] = nb[2]; code[k][4] = nb[3];
        code[k][5] = veff[b]; code[k][6] = list_code(L[5 + k]);
    }
    __syncthreads();                                // code[] complete
    // the four lateral cubes of step k into stage st: 1024 16-byte pieces each, 8 per thread
    auto issue = [&](int k, int st) {
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            int32_t const e = code[k][1 + l];
            if (-1 == e) continue;                  // no cube: read as zeros, nothing to copy
            float const *src = x + size_t(nbr_block(e))*kBlockReals + slice*S;
            float *dst = lat + (st*4 + l)*2*64*S;
#pragma unroll
            for (int q = 0; q < 2*64*(S/4)/(4*S); ++q) {
                int const c = q*4*S + tid;          // piece: (plane*64 + row)*(S/4) + quad
                int const pr = c/(S/4), qd = c % (S/4);
                cp_async16_cg(dst + pr*S + qd*4, src + pr*64 + qd*4);
            }
        }
    };
    auto srow = [&](int slot, int pl, int row) -> float4 & { return slot4[((slot*2 + pl)*16 + row)*S + j]; };
    auto put = [&](int slot, Quad const &q) {
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int pl = 0; pl < 2; ++pl)
                srow(slot, pl, zq*4 + yy) = make_float4(q.v[pl][yy*4], q.v[pl][yy*4 + 1], q.v[pl][yy*4 + 2], q.v[pl][yy*4 + 3]);
    };
    // row (zq, r4) of lateral l of stage st: 4 x-points, re and im, with the Bloch phase of its code
    auto lrow = [&](int st, int l, int r4, int32_t e, float pr, float pi, Rows<float> &o) {
        if (-1 == e) {
#pragma unroll
            for (int i = 0; i < 4; ++i) { o.re[i] = 0.f; o.im[i] = 0.f; }
            return;
        }
        float const *b = lat + (st*4 + l)*2*64*S + (zq*16 + r4*4)*S + j;
#pragma unroll
        for (int i = 0; i < 4; ++i) { o.re[i] = b[i*S]; o.im[i] = b[64*S + i*S]; }
        row_phase(e, pr, pi, o);
    };
    float const (&cx)[5] = a.st.c[0];
    float const (&cy)[5] = a.st.c[1];
    float const (&cz)[5] = a.st.c[2];
    float const c0 = cx[0] + cy[0] + cz[0];
    issue(0, 0);
    asm volatile("cp.async.commit_group;" ::: "memory");
    {
        Quad h;
        quad_raw(x, zleft, zq, col, h);
        quad_phase(zleft, a.ph[2][0][0], a.ph[2][0][1], h);
        put(0, h);
        quad_raw(x, code[0][0], zq, col, h);
        put(1, h);
    }
    Quad nx;                                        // rows of the z-successor, one step ahead
    quad_raw(x, code[0][6], zq, col, nx);
    int sp = 0, sc = 1, sn = 2;
    for (int k = 0; k < n; ++k) {
        int32_t const b = code[k][0];
        int const st = k & 1;
        quad_phase(code[k][6], a.ph[2][1][0], a.ph[2][1][1], nx);   // only the line end has a phase
        __syncthreads();                            // step k-1 finished reading slot sn and stage st^1
        if (k + 1 < n) issue(k + 1, st ^ 1);
        asm volatile("cp.async.commit_group;" ::: "memory");
        put(sn, nx);
        asm volatile("cp.async.wait_group 1;" ::: "memory");   // this thread's copies of step k landed
        __syncthreads();                            // ... and everybody else's; slot sn written
        if (k + 1 < n) quad_raw(x, code[k + 1][6], zq, col, nx);   // arrives during this step
        Quad cur;
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int pl = 0; pl < 2; ++pl) {
                float4 const v = srow(sc, pl, zq*4 + yy);
                cur.v[pl][yy*4] = v.x; cur.v[pl][yy*4 + 1] = v.y; cur.v[pl][yy*4 + 2] = v.z; cur.v[pl][yy*4 + 3] = v.w;
            }
        float acc[2][16];
        int32_t const iloc = code[k][5];
        float V[16];
        if (iloc < 0) {
#pragma unroll
            for (int i = 0; i < 16; ++i) V[i] = 0.f;
        } else {
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 const v = __ldg(reinterpret_cast<float4 const*>(Vcell + size_t(iloc)*64 + zq*16 + q*4));
                V[q*4] = v.x; V[q*4 + 1] = v.y; V[q*4 + 2] = v.z; V[q*4 + 3] = v.w;
            }
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            float const Vt = V[i] - a.E_re;
            acc[0][i] = Vt*cur.v[0][i] + a.E_im*cur.v[1][i] + c0*cur.v[0][i];
            acc[1][i] = Vt*cur.v[1][i] - a.E_im*cur.v[0][i] + c0*cur.v[1][i];
        }
#pragma unroll
        for (int pl = 0; pl < 2; ++pl)
#pragma unroll
            for (int yy = 0; yy < 4; ++yy)
#pragma unroll
                for (int yo = 0; yo < 4; ++yo) {
                    if (yo == yy) continue;
                    int const d = (yo > yy) ? yo - yy : yy - yo;
#pragma unroll
                    for (int i = 0; i < 4; ++i) acc[pl][yy*4 + i] += cy[d]*cur.v[pl][yo*4 + i];
                }
        int32_t const exm = code[k][1], exp_ = code[k][2], eym = code[k][3], eyp = code[k][4];
#pragma unroll
        for (int yy = 0; yy < 4; ++yy) {
            Rows<float> xm, xp;
            lrow(st, 0, yy, exm, a.ph[0][0][0], a.ph[0][0][1], xm);
            lrow(st, 1, yy, exp_, a.ph[0][1][0], a.ph[0][1][1], xp);
            float lr[12], li[12];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                lr[i] = xm.re[i]; li[i] = xm.im[i];
                lr[4 + i] = cur.v[0][yy*4 + i]; li[4 + i] = cur.v[1][yy*4 + i];
                lr[8 + i] = xp.re[i]; li[8 + i] = xp.im[i];
            }
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int d = 1; d <= 4; ++d) {
                    acc[0][yy*4 + i] += cx[d]*(lr[4 + i - d] + lr[4 + i + d]);
                    acc[1][yy*4 + i] += cx[d]*(li[4 + i - d] + li[4 + i + d]);
                }
        }
#pragma unroll
        for (int yo = 0; yo < 4; ++yo) {
            Rows<float> ym, yp;
            lrow(st, 2, yo, eym, a.ph[1][0][0], a.ph[1][0][1], ym);
            lrow(st, 3, yo, eyp, a.ph[1][1][0], a.ph[1][1][1], yp);
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) {
                if (yy <= yo) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        acc[0][yy*4 + i] += cy[yy - yo + 4]*ym.re[i];
                        acc[1][yy*4 + i] += cy[yy - yo + 4]*ym.im[i];
                    }
                }
                if (yy >= yo) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        acc[0][yy*4 + i] += cy[yo + 4 - yy]*yp.re[i];
                        acc[1][yy*4 + i] += cy[yo + 4 - yy]*yp.im[i];
                    }
                }
            }
        }
#pragma unroll
        for (int yy = 0; yy < 4; ++yy)
#pragma unroll
            for (int d = 1; d <= 4; ++d) {
                int const zm = zq - d, zp = zq + d;
                int const s_m = (zm < 0) ? sp : sc, s_p = (zp > 3) ? sn : sc;
                int const r_m = (zm & 3)*4 + yy, r_p = (zp & 3)*4 + yy;
#pragma unroll
                for (int pl = 0; pl < 2; ++pl) {
                    float4 const m = srow(s_m, pl, r_m), p = srow(s_p, pl, r_p);
                    acc[pl][yy*4 + 0] += cz[d]*(m.x + p.x);
                    acc[pl][yy*4 + 1] += cz[d]*(m.y + p.y);
                    acc[pl][yy*4 + 2] += cz[d]*(m.z + p.z);
                    acc[pl][yy*4 + 3] += cz[d]*(m.w + p.w);
                }
            }
        float *yb = y + size_t(b)*kBlockReals + (zq*16)*64 + col;
#pragma unroll
        for (int i = 0; i < 16; ++i) { yb[i*64] = acc[0][i]; yb[4096 + i*64] = acc[1][i]; }
        int const t = sp; sp = sc; sc = sn; sn = t;  // rotate the z-slots
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// ---------------------------------------------------------------- generic local path

// y = (V - E) x for every block (include/green_potential.hxx:15-139, collinear)
template <typename T>
__global__ void __launch_bounds__(256)
potential_kernel(T *__restrict__ y, T const *__restrict__ x, int32_t const *__restrict__ veff,
                 T const *__restrict__ Vcell, uint32_t nnzb, LocalArgs<T> const a0)
{
    for (uint32_t b = blockIdx.x; b < nnzb; b += gridDim.x) {
        LocalArgs<T> a = a0;
        if (!line_args(a, int32_t(b))) continue;          // uniform: the CTA works on block b
        T const Er = a.E_re, Ei = a.E_im;
        int32_t const iloc = veff[b];
        T const *xb = x + size_t(b)*kBlockReals;
        T *yb = y + size_t(b)*kBlockReals;
        for (int t = threadIdx.x; t < 4096; t += blockDim.x) {
            int const i = t >> 6;
            T const Vt = ((iloc < 0) ? T(0) : Vcell[size_t(iloc)*64 + i]) - Er;
            T const xr = xb[t], xi = xb[4096 + t];
            yb[t] = Vt*xr + Ei*xi;
            yb[4096 + t] = Vt*xi - Ei*xr;
        }
    }
}

// y += T_dd x along the lists of one direction; NH halo cubes (1: 9-point, 2: 17-point stencil).
// One CTA per (list, cross-section row i16), 64 threads = columns, each for re and im.
template <typename T>
struct Coef17 { T c[9]; };

template <typename T, int NH>
__global__ void __launch_bounds__(64)
kinetic_list_kernel(T *__restrict__ y, T const *__restrict__ x, uint32_t const *__restrict__ lstart,
                    int32_t const *__restrict__ lists, int stride, Coef17<T> const coef, int dd,
                    LocalArgs<T> a)
{
    constexpr int W = 4*(2*NH + 1);   // window points: NH cubes left, current, NH right
    constexpr int R = 4*NH;           // stencil reach in points
    int const i16 = blockIdx.y, col = threadIdx.x;
    int const base = (16 == stride) ? i16 : ((4 == stride) ? (16*(i16 >> 2) + (i16 & 3)) : 4*i16);
    int32_t const *L = lists + lstart[blockIdx.x];
    int n = 0;
    while (L[4 + n] > 0) ++n;
    if (0 == n || !line_args(a, L[4] - 1)) return;      // uniform: empty list, or a retired source
    T const plr = a.ph[dd][0][0], pli = a.ph[dd][0][1], prr = a.ph[dd][1][0], pri = a.ph[dd][1][1];
    T c[R + 1];
#pragma unroll
    for (int k = 0; k <= R; ++k) c[k] = coef.c[k];
    T wr[W], wi[W];
    // cube at list position p (0-based among the cubes), with halo handling at both ends
    auto fetch = [&](int p, int slot) {
        int32_t entry = 0; T pr = T(1), pi = T(0);
        if (p >= 0 && p < n) entry = L[4 + p];
        else if (1 == NH && -1 == p) { entry = L[3]; pr = plr; pi = pli; }
        else if (1 == NH && n == p) { entry = L[4 + n]; pr = prr; pi = pri; }
        if (0 == entry) {
#pragma unroll
            for (int i4 = 0; i4 < 4; ++i4) { wr[slot*4 + i4] = T(0); wi[slot*4 + i4] = T(0); }
            return;
        }
        int32_t const b = (entry > 0) ? entry - 1 : -entry - 1;
        T const *xb = x + size_t(b)*kBlockReals + base*64 + col;
#pragma unroll
        for (int i4 = 0; i4 < 4; ++i4) {
            T const r = xb[i4*stride*64], i = xb[4096 + i4*stride*64];
            if (entry < 0) { wr[slot*4 + i4] = pr*r - pi*i; wi[slot*4 + i4] = pr*i + pi*r; }
            else { wr[slot*4 + i4] = r; wi[slot*4 + i4] = i; }
        }
    };
#pragma unroll
    for (int s = 0; s < 2*NH + 1; ++s) fetch(s - NH, s);
    for (int k = 0; k < n; ++k) {
        int32_t const b = L[4 + k] - 1;
        T *yb = y + size_t(b)*kBlockReals + base*64 + col;
#pragma unroll
        for (int i4 = 0; i4 < 4; ++i4) {
            int const p = 4*NH + i4;
            T sr = c[0]*wr[p], si = c[0]*wi[p];
#pragma unroll
            for (int d = 1; d <= R; ++d) { sr += c[d]*(wr[p - d] + wr[p + d]); si += c[d]*(wi[p - d] + wi[p + d]); }
            yb[i4*stride*64] += sr;
            yb[4096 + i4*stride*64] += si;
        }
#pragma unroll
        for (int q = 0; q < W - 4; ++q) { wr[q] = wr[q + 4]; wi[q] = wi[q + 4]; }
        fetch(k + 1 + NH, 2*NH);
    }
}

// ---------------------------------------------------------------- dyadic part

__host__ __device__ constexpr int nsho_c(int L) { return ((L + 1)*(L + 2)*(L + 3))/6; }
__host__ __device__ constexpr int n2ho_c(int L) { return ((L + 1)*(L + 2))/2; }

// Projector tables of one (atom image, target row) slot staged in shared memory: the 1D
// Hermite-Gauss functions H[nu][dir][i4] (unnormalized, H_0 = exp(-xi^2/2) inside the
// projection radius, H_{n+1} = xi H_n - n/2 H_{n-1}, include/green_dyadic.hxx:33-107) and
// the 64-point spherical mask, both precomputed by the plan builder.
template <typename T, int LM>
__device__ __forceinline__ void stage_table(T (*H)[3][4], double const *__restrict__ slot_H, int stride,
                                            uint32_t slot, int lmax, int tid) {
    if (tid < (lmax + 1)*12) (&H[0][0][0])[tid] = T(slot_H[size_t(slot)*stride + tid]);
}

// apc[(i0 + sho)*nrhs + s][reim][j] = sum over the blocks of source s near image a of the
// masked projector functions times x (include/green_dyadic.hxx:112-288), for images whose
// basis size is exactly L (the host launches one grid per distinct L).  Sum-factorized:
// contract x, then y, then z.  One CTA per work item (image, source, chunk of at most 16
// blocks of its list), 128 threads = (reim, column); the chunks of one (image, source) are
// summed with atomics into the zeroed coefficients.
template <typename T, int L>
__global__ void __launch_bounds__(128)
sho_project_kernel(T *__restrict__ apc, T const *__restrict__ x, uint32_t nrhs,
                   uint32_t const *__restrict__ items,
                   uint32_t const *__restrict__ prj_col, uint64_t const *__restrict__ prj_coloff,
                   uint32_t const *__restrict__ prj_slot,
                   double const *__restrict__ slot_H, uint64_t const *__restrict__ slot_mask, int stride,
                   uint32_t const *__restrict__ img_starts)
{
    constexpr int NS = nsho_c(L), N2 = n2ho_c(L);
    __shared__ T Hs[2][L + 1][3][4];
    uint32_t const *item = items + 4*size_t(blockIdx.x);
    uint32_t const a = item[0], s = item[1], k0 = item[2], k1 = item[3];
    int const tid = threadIdx.x;
    int const reim = tid >> 6, j = tid & 63;
    uint64_t const off = prj_coloff[s];
    T acc[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) acc[i] = T(0);
    int buf = 0;
    for (uint32_t k = k0; k < k1; ++k, buf ^= 1) {
        uint32_t const b = prj_col[off + k];
        uint32_t const slot = prj_slot[off + k];
        stage_table<T, L>(Hs[buf], slot_H, stride, slot, L, tid);
        uint64_t const mask = slot_mask[slot];
        __syncthreads();             // double-buffered tables: one barrier per block
        T (*H)[3][4] = Hs[buf];
        T const *xb = x + size_t(b)*kBlockReals + reim*4096 + j;
        for (int z = 0; z < 4; ++z) {
            if (0 == ((mask >> (16*z)) & 0xffffu)) continue;
            T byx[N2];
#pragma unroll
            for (int i = 0; i < N2; ++i) byx[i] = T(0);
            for (int yy = 0; yy < 4; ++yy) {
                unsigned const row = unsigned(mask >> (16*z + 4*yy)) & 0xfu;
                if (0 == row) continue;
                T ax[L + 1];
#pragma unroll
                for (int i = 0; i <= L; ++i) ax[i] = T(0);
#pragma unroll
                for (int xx = 0; xx < 4; ++xx) {
                    if ((row >> xx) & 1u) {
                        T const ps = xb[((z*4 + yy)*4 + xx)*64];
#pragma unroll
                        for (int ix = 0; ix <= L; ++ix) ax[ix] += ps*H[ix][0][xx];
                    }
                }
#pragma unroll
                for (int iy = 0, iyx = 0; iy <= L; ++iy) {
                    T const hy = H[iy][1][yy];
#pragma unroll
                    for (int ix = 0; ix <= L - iy; ++ix, ++iyx) byx[iyx] += ax[ix]*hy;
                }
            }
#pragma unroll
            for (int iz = 0, sho = 0; iz <= L; ++iz) {
                T const hz = H[iz][2][z];
#pragma unroll
                for (int iy = 0; iy <= L - iz; ++iy) {
                    int const iyx = iy*(2*L + 3 - iy)/2;
#pragma unroll
                    for (int ix = 0; ix <= L - iz - iy; ++ix, ++sho) acc[sho] += byx[iyx + ix]*hz;
                }
            }
        }
    }
    T *out = apc + (size_t(img_starts[a])*nrhs + s)*128 + reim*64 + j;
#pragma unroll
    for (int sho = 0; sho < NS; ++sho) atomicAdd(out + size_t(sho)*nrhs*128, acc[sho]);
}

// aac[(a0 + c)*nrhs + s] = sum over the images i of atom A of phase_i * apc[(i0 + c)*nrhs + s]
// (collect) in double (include/green_dyadic.hxx:600-702).  Grid (nAtoms, nrhs), 64 threads.
// per-source selection of the pair values of a batch plan (image phases and atom matrices
// stored [pair][...]) and the retirement flags (nullptr: every source active)
struct DyadicPairs {
    uint32_t nsrc_pair;              // sources per pair (= nrhs for a one-pair plan)
    size_t img_stride, mat_stride;   // doubles per pair of img_phase and of the atom matrices
    uint8_t const *active;
};

template <typename T>
__global__ void __launch_bounds__(64)
sho_collect_kernel(double *__restrict__ aac, T const *__restrict__ apc, uint32_t nrhs,
                   uint32_t const *__restrict__ atom_starts, int8_t const *__restrict__ atom_lmax,
                   uint32_t const *__restrict__ sum_start, uint32_t const *__restrict__ sum_col,
                   uint32_t const *__restrict__ img_starts, double const *__restrict__ img_phase,
                   DyadicPairs const bp)
{
    int const A = blockIdx.x, s = blockIdx.y, j = threadIdx.x;
    if (bp.active && !bp.active[s]) return;
    img_phase += (s/bp.nsrc_pair)*bp.img_stride;
    int const nc = nsho_c(atom_lmax[A]);
    size_t const a0 = atom_starts[A];
    for (int c = 0; c < nc; ++c) {
        double re = 0, im = 0;
        for (uint32_t k = sum_start[A]; k < sum_start[A + 1]; ++k) {
            uint32_t const i = sum_col[k];
            double const pr = img_phase[4*i], pi = img_phase[4*i + 1];
            T const *src = apc + ((size_t(img_starts[i]) + c)*nrhs + s)*128;
            double const xr = double(src[j]), xi = double(src[64 + j]);
            re += pr*xr - pi*xi;
            im += pr*xi + pi*xr;
        }
        double *dst = aac + ((a0 + c)*nrhs + s)*128;
        dst[j] = re; dst[64 + j] = im;
    }
}

// out[(a0 + i)*nrhs + s] = sum_k M_A[i][k] in[(a0 + k)*nrhs + s], complex, accumulated in
// double (include/green_dyadic.hxx:740-826).  Grid (nAtoms, nrhs), 64 threads.
template <typename Tin, typename Tout>
__global__ void __launch_bounds__(64)
sho_mul_kernel(Tout *__restrict__ out, Tin const *__restrict__ in, uint32_t nrhs,
               uint32_t const *__restrict__ atom_starts, int8_t const *__restrict__ atom_lmax,
               double const *__restrict__ mats, uint32_t const *__restrict__ mat_off, DyadicPairs const bp)
{
    int const A = blockIdx.x, s = blockIdx.y, j = threadIdx.x;
    if (bp.active && !bp.active[s]) return;
    mats += (s/bp.nsrc_pair)*bp.mat_stride;
    int const nc = nsho_c(atom_lmax[A]);
    size_t const a0 = atom_starts[A];
    double const *Mr = mats + mat_off[A], *Mi = Mr + nc*nc;
    constexpr int R = 8;                       // output rows per pass: each input value is loaded once per R rows
    for (int i0 = 0; i0 < nc; i0 += R) {
        double re[R], im[R];
#pragma unroll
        for (int r = 0; r < R; ++r) { re[r] = 0; im[r] = 0; }
        for (int k = 0; k < nc; ++k) {
            Tin const *src = in + ((a0 + k)*nrhs + s)*128;
            double const xr = double(src[j]), xi = double(src[64 + j]);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                int const i = (i0 + r < nc) ? i0 + r : nc - 1;   // clamped rows are not stored
                double const mr = __ldg(Mr + i*nc + k), mi = __ldg(Mi + i*nc + k);
                re[r] += mr*xr - mi*xi;
                im[r] += mr*xi + mi*xr;
            }
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (i0 + r >= nc) break;
            Tout *dst = out + ((a0 + i0 + r)*nrhs + s)*128;
            dst[j] = Tout(re[r]); dst[64 + j] = Tout(im[r]);
        }
    }
}

// cad[(i0 + c)*nrhs + s] = conj(phase_i) * cadd[(a0 + c)*nrhs + s] for every image i of atom A
// (broadcast, include/green_dyadic.hxx:683-694).  Grid (nAtoms, nrhs), 64 threads.
template <typename T>
__global__ void __launch_bounds__(64)
sho_broadcast_kernel(T *__restrict__ cad, double const *__restrict__ cadd, uint32_t nrhs,
                     uint32_t const *__restrict__ atom_starts, int8_t const *__restrict__ atom_lmax,
                     uint32_t const *__restrict__ sum_start, uint32_t const *__restrict__ sum_col,
                     uint32_t const *__restrict__ img_starts, double const *__restrict__ img_phase,
                     DyadicPairs const bp)
{
    int const A = blockIdx.x, s = blockIdx.y, j = threadIdx.x;
    if (bp.active && !bp.active[s]) return;
    img_phase += (s/bp.nsrc_pair)*bp.img_stride;
    int const nc = nsho_c(atom_lmax[A]);
    size_t const a0 = atom_starts[A];
    for (uint32_t k = sum_start[A]; k < sum_start[A + 1]; ++k) {
        uint32_t const i = sum_col[k];
        double const pr = img_phase[4*i], pi = -img_phase[4*i + 1];
        for (int c = 0; c < nc; ++c) {
            double const *src = cadd + ((a0 + c)*nrhs + s)*128;
            double const xr = src[j], xi = src[64 + j];
            T *dst = cad + ((size_t(img_starts[i]) + c)*nrhs + s)*128;
            dst[j] = T(pr*xr - pi*xi);
            dst[64 + j] = T(pr*xi + pi*xr);
        }
    }
}

// The atom-matrix chain in one kernel (collect, multiply, broadcast of the three kernels above),
// per (atom, source, half of the 64 columns): the coefficients of the atom's images summed with
// their Bloch phases into shared memory, multiplied by M_A (complex, FP64) and written to every
// image with the conjugate phase.  Warp g of the four works on rows g, g + 4, ... (M_A's rows are
// uniform over a warp), lane j on column half*32 + j.  Plans without periodic images take no
// phases (the reference's direct path).  nSHO <= 56.
constexpr int kAtomRows = 56;

template <typename T>
__global__ void __launch_bounds__(128)
sho_atom_kernel(T *__restrict__ cad, T const *__restrict__ apc, uint32_t nrhs,
                int8_t const *__restrict__ atom_lmax, uint32_t const *__restrict__ sum_start,
                uint32_t const *__restrict__ sum_col, uint32_t const *__restrict__ img_starts,
                double const *__restrict__ img_phase, double const *__restrict__ mats,
                uint32_t const *__restrict__ mat_off, int use_phase, DyadicPairs const bp)
{
    __shared__ double sre[kAtomRows][32], sim[kAtomRows][32];
    constexpr int kImg = 32;                          // images of the atom staged in shared memory
    __shared__ uint32_t simg[kImg];
    __shared__ double sph[kImg][2];
    int const A = blockIdx.x, s = blockIdx.y, half = blockIdx.z;
    int const j = threadIdx.x & 31, g = threadIdx.x >> 5, col = half*32 + j;
    if (bp.active && !bp.active[s]) return;
    img_phase += (s/bp.nsrc_pair)*bp.img_stride;
    mats += (s/bp.nsrc_pair)*bp.mat_stride;
    int const nc = nsho_c(atom_lmax[A]);
    uint32_t const k0 = sum_start[A], k1 = sum_start[A + 1];
    // the atom's images (their coefficient start and phase) once, instead of a chain of three
    // dependent loads per row and image
    for (uint32_t k = k0 + threadIdx.x; k < k1 && k < k0 + kImg; k += blockDim.x) {
        uint32_t const i = sum_col[k];
        simg[k - k0] = img_starts[i];
        sph[k - k0][0] = img_phase[4*i]; sph[k - k0][1] = img_phase[4*i + 1];
    }
    __syncthreads();
    auto image = [&](uint32_t k, uint32_t &start, double &pr, double &pi) {
        if (k - k0 < uint32_t(kImg)) { start = simg[k - k0]; pr = sph[k - k0][0]; pi = sph[k - k0][1]; }
        else { uint32_t const i = sum_col[k]; start = img_starts[i]; pr = img_phase[4*i]; pi = img_phase[4*i + 1]; }
    };
    for (int c = g; c < nc; c += 4) {
        double re = 0, im = 0;
        for (uint32_t k = k0; k < k1; ++k) {
            uint32_t start; double pr, pi;
            image(k, start, pr, pi);
            T const *src = apc + ((size_t(start) + c)*nrhs + s)*128;
            double const xr = double(src[col]), xi = double(src[64 + col]);
            if (use_phase) {
                re += pr*xr - pi*xi;
                im += pr*xi + pi*xr;
            } else {
                re += xr; im += xi;
            }
        }
        sre[c][j] = re; sim[c][j] = im;
    }
    __syncthreads();
    double const *Mr = mats + mat_off[A], *Mi = Mr + nc*nc;
    for (int r = g; r < nc; r += 4) {
        double re = 0, im = 0;
        for (int k = 0; k < nc; ++k) {
            double const mr = __ldg(Mr + r*nc + k), mi = __ldg(Mi + r*nc + k);
            double const xr = sre[k][j], xi = sim[k][j];
            re += mr*xr - mi*xi;
            im += mr*xi + mi*xr;
        }
        for (uint32_t k = k0; k < k1; ++k) {
            uint32_t start; double pr, pi;
            image(k, start, pr, pi);
            pi = -pi;
            T *dst = cad + ((size_t(start) + r)*nrhs + s)*128;
            if (use_phase) {
                dst[col] = T(pr*re - pi*im);
                dst[64 + col] = T(pr*im + pi*re);
            } else {
                dst[col] = T(re); dst[64 + col] = T(im);
            }
        }
    }
}

// y[b] += sum over the images a near block b of the masked projector functions times
// cad[a, rhs(b)] (include/green_dyadic.hxx:325-518); sum-factorized over z, y, x.
// One CTA per block, 128 threads = (reim, column); only masked points are written.
template <typename T>
__global__ void __launch_bounds__(128)
sho_add_kernel(T *__restrict__ y, T const *__restrict__ cad, uint32_t nrhs, uint32_t nnzb,
               uint16_t const *__restrict__ colIndex, uint32_t const *__restrict__ add_start,
               uint32_t const *__restrict__ add_col, uint32_t const *__restrict__ add_slot,
               double const *__restrict__ slot_H, uint64_t const *__restrict__ slot_mask, int stride,
               int8_t const *__restrict__ img_lmax, uint32_t const *__restrict__ img_starts)
{
    constexpr int LM = 7;
    __shared__ T Hs[2][LM + 1][3][4];
    uint32_t const b = blockIdx.x;
    if (add_start[b] >= add_start[b + 1]) return;
    int const tid = threadIdx.x, reim = tid >> 6, j = tid & 63;
    uint32_t const s = colIndex[b];
    T acc[64];
#pragma unroll
    for (int i = 0; i < 64; ++i) acc[i] = T(0);
    uint64_t mask_all = 0;
    int buf = 0;
    for (uint32_t k = add_start[b]; k < add_start[b + 1]; ++k, buf ^= 1) {
        uint32_t const a = add_col[k], slot = add_slot[k];
        int const lmax = img_lmax[a];
        stage_table<T, LM>(Hs[buf], slot_H, stride, slot, lmax, tid);
        uint64_t const mask = slot_mask[slot];
        __syncthreads();
        if (!mask) continue;
        mask_all |= mask;
        T (*H)[3][4] = Hs[buf];
        T const *c = cad + (size_t(img_starts[a])*nrhs + s)*128 + reim*64 + j;
        int sho = 0;
        for (int iz = 0; iz <= lmax; ++iz) {
            T byx[4][4];
#pragma unroll
            for (int yy = 0; yy < 4; ++yy)
#pragma unroll
                for (int xx = 0; xx < 4; ++xx) byx[yy][xx] = T(0);
            for (int iy = 0; iy <= lmax - iz; ++iy) {
                T ax[4] = {T(0), T(0), T(0), T(0)};
                for (int ix = 0; ix <= lmax - iz - iy; ++ix, ++sho) {
                    T const ca = c[size_t(sho)*nrhs*128];
#pragma unroll
                    for (int xx = 0; xx < 4; ++xx) ax[xx] += H[ix][0][xx]*ca;
                }
#pragma unroll
                for (int yy = 0; yy < 4; ++yy) {
                    T const hy = H[iy][1][yy];
#pragma unroll
                    for (int xx = 0; xx < 4; ++xx) byx[yy][xx] += hy*ax[xx];
                }
            }
#pragma unroll
            for (int z = 0; z < 4; ++z) {
                T const hz = H[iz][2][z];
#pragma unroll
                for (int yy = 0; yy < 4; ++yy)
#pragma unroll
                    for (int xx = 0; xx < 4; ++xx) {
                        int const p = (z*4 + yy)*4 + xx;
                        if ((mask >> p) & 1) acc[p] += hz*byx[yy][xx];
                    }
            }
        }
    }
    T *yb = y + size_t(b)*kBlockReals + reim*4096 + j;
#pragma unroll
    for (int p = 0; p < 64; ++p) if ((mask_all >> p) & 1) yb[p*64] += acc[p];
}

DyadicPairs dyadic_pairs(DevicePlan const &dp) {
    DyadicPairs bp;
    bp.nsrc_pair = dp.nsrc_pair ? dp.nsrc_pair : std::max(1u, dp.nCols);
    bp.img_stride = (dp.npairs > 1) ? size_t(dp.nAI)*4 : 0;
    bp.mat_stride = (dp.npairs > 1) ? dp.mat_stride : 0;
    bp.active = dp.retire ? dptr<uint8_t>(dp.src_active) : nullptr;
    return bp;
}

template <typename T> T const *vcell(DevicePlan &dp);
template <> double const *vcell<double>(DevicePlan &dp) { return dptr<double>(dp.Vcell64); }
template <> float const *vcell<float>(DevicePlan &dp) { return dptr<float>(dp.Vcell32); }

template <typename T, int L>
void launch_project_L(DevicePlan &dp, T const *x, cudaStream_t st) {
    auto const &g = dp.prj_items[L];
    if (0 == g.count) return;
    sho_project_kernel<T, L><<<g.count, 128, 0, st>>>(
        dptr<T>(dp.apc), x, dp.nCols, dptr<uint32_t>(g.items),
        dptr<uint32_t>(dp.prj_col), dptr<uint64_t>(dp.prj_coloff),
        dptr<uint32_t>(dp.prj_slot), dptr<double>(dp.slot_H), dptr<uint64_t>(dp.slot_mask), dp.table_stride,
        dptr<uint32_t>(dp.img_starts));
        count_launch();
}

} // namespace

bool prepare_local_kernels() {
    // the pencil kernel's three z-slots are 48 KB of dynamic shared memory beside its static part
    A43G_CUDA_TRY(cudaFuncSetAttribute(local_pencil_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPencilSmem));
    A43G_CUDA_TRY(cudaFuncSetAttribute(local_stage_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStageSmem));
    A43G_CUDA_TRY(cudaFuncSetAttribute(local_pencil64_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPencil64Smem));
    return true;
}

// kernel arguments of the local part: stencil, energy and phases of a one-pair plan, or the
// per-pair table of a batch plan; the source flags when some sources are retired
template <typename T>
LocalArgs<T> local_args(DevicePlan const &dp) {
    LocalArgs<T> a;
    a.st = make_stencil9<T>(dp);
    a.E_re = T(dp.E_re); a.E_im = T(dp.E_im);
    for (int d = 0; d < 3; ++d) for (int s = 0; s < 2; ++s) for (int c = 0; c < 2; ++c) a.ph[d][s][c] = T(dp.phase[d][s][c]);
    bool const batch = dp.npairs > 1;
    a.pairs = batch ? dptr<PairArgs<T>>(sizeof(T) == 8 ? dp.pair_args64 : dp.pair_args32) : nullptr;
    a.active = dp.retire ? dptr<uint8_t>(dp.src_active) : nullptr;
    a.colindx = (batch || a.active) ? dptr<uint16_t>(dp.colindx) : nullptr;
    a.nsrc_pair = dp.nsrc_pair ? dp.nsrc_pair : dp.nCols;
    return a;
}

template <typename T>
bool launch_local(DevicePlan &dp, T *y, T const *x, cudaStream_t st) {
    if (0 == dp.nnzb) return true;
    LocalArgs<T> a = local_args<T>(dp);
    if (dp.fused_local) {
        constexpr int S = (sizeof(T) == 8) ? 8 : 16;
        unsigned const nblk = dp.nlists[2]*(64/S);
        if constexpr (sizeof(T) == 4) {
            if (dp.nlists[2] && dp.max_zline <= kMaxLine && 3 == dp.local_variant &&
                0 == (reinterpret_cast<uintptr_t>(x) & 15u)) {
                local_stage_kernel<<<dp.nlists[2]*(64/kPencilS), 4*kPencilS, kStageSmem, st>>>(y, x,
                    dptr<uint32_t>(dp.lists_start[2]), dptr<int32_t>(dp.lists[2]), dptr<int32_t>(dp.nbr),
                    dptr<int32_t>(dp.veff_index), vcell<T>(dp), a);
                count_launch();
                A43G_CUDA_TRY(cudaGetLastError());
                return true;
            }
            if (dp.nlists[2] && dp.max_zline <= kMaxLine && (2 == dp.local_variant || 3 == dp.local_variant)) {
                local_pencil_kernel<<<dp.nlists[2]*(64/kPencilS), 4*kPencilS, kPencilSmem, st>>>(y, x,
                    dptr<uint32_t>(dp.lists_start[2]), dptr<int32_t>(dp.lists[2]), dptr<int32_t>(dp.nbr),
                    dptr<int32_t>(dp.veff_index), vcell<T>(dp), a);
                count_launch();
                A43G_CUDA_TRY(cudaGetLastError());
                return true;
            }
        }
        if constexpr (sizeof(T) == 8) {
            if (dp.nlists[2] && dp.max_zline <= kMaxLine && dp.local64_pencils) {
                local_pencil64_kernel<<<dp.nlists[2]*(64/kPencil64S), 8*kPencil64S, kPencil64Smem, st>>>(y, x,
                    dptr<uint32_t>(dp.lists_start[2]), dptr<int32_t>(dp.lists[2]), dptr<int32_t>(dp.nbr),
                    dptr<int32_t>(dp.veff_index), vcell<T>(dp), a);
                count_launch();
                A43G_CUDA_TRY(cudaGetLastError());
                return true;
            }
        }
        if (nblk && sizeof(T) == 4 && dp.max_zline <= kMaxLine && 0 == dp.local_variant) {
            local_fused_pf_kernel<T, S><<<nblk, S*16, 0, st>>>(y, x, dptr<uint32_t>(dp.lists_start[2]),
                dptr<int32_t>(dp.lists[2]), dptr<int32_t>(dp.nbr), dptr<int32_t>(dp.veff_index), vcell<T>(dp), a);
            count_launch();
        } else if (nblk) {
            local_fused_kernel<T, S><<<nblk, S*16, 0, st>>>(y, x, dptr<uint32_t>(dp.lists_start[2]),
                dptr<int32_t>(dp.lists[2]), dptr<int32_t>(dp.nbr), dptr<int32_t>(dp.veff_index), vcell<T>(dp), a);
            count_launch();
        }
    } else {
        unsigned const nb = std::min<uint32_t>(dp.nnzb, 148u*16);
        potential_kernel<T><<<nb, 256, 0, st>>>(y, x, dptr<int32_t>(dp.veff_index), vcell<T>(dp), dp.nnzb, a);
        count_launch();
        for (int d = 0; d < 3; ++d) {
            int const nFD = dp.FD_range[d];
            if (nFD < 1 || 0 == dp.nlists[d]) continue;
            dim3 const grid(dp.nlists[d], 16);
            // 8th order {-14350, 8064, -1008, 128, -9}/5040 or 16th order
            // {-924708642, 538137600, -94174080, 22830080, -5350800, 1053696, -156800, 15360, -735}/302702400,
            // times -1/(2h^2) (include/green_kinetic.hxx:37-42, 215-225)
            Coef17<T> coef;
            if (8 == nFD) {
                double const w[9] = {-924708642, 538137600, -94174080, 22830080, -5350800, 1053696, -156800, 15360, -735};
                double const norm = dp.prefactor[d]/302702400.;
                for (int k = 0; k < 9; ++k) coef.c[k] = T(w[k]*norm);
            } else {
                double const w[5] = {-14350, 8064, -1008, 128, -9};
                double const norm = dp.prefactor[d]/5040.;
                for (int k = 0; k < 9; ++k) coef.c[k] = T(k < 5 ? w[k]*norm : 0.0);
            }
            if (8 == nFD) kinetic_list_kernel<T, 2><<<grid, 64, 0, st>>>(y, x, dptr<uint32_t>(dp.lists_start[d]),
                              dptr<int32_t>(dp.lists[d]), 1 << (2*d), coef, d, a);
            else kinetic_list_kernel<T, 1><<<grid, 64, 0, st>>>(y, x, dptr<uint32_t>(dp.lists_start[d]),
                              dptr<int32_t>(dp.lists[d]), 1 << (2*d), coef, d, a);
            count_launch();
        }
    }
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

template <typename T>
bool launch_dyadic(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t st) {
    if (dp.nAI < 1 || dp.nCols < 1) return true;
    if (!ensure_dyadic_scratch(dp, sizeof(T))) return false;
    // both FP32 projector paths stage x with 16-byte loads; other x take the generic kernels
    bool const aligned16 = 0 == (reinterpret_cast<uintptr_t>(x) & 15u);
    bool const tc = (sizeof(T) == 4) && dp.use_tc && aligned16 && tc_projector_supported(dp);
    bool const simt = !tc && simt_projector_supported(dp, x, y, sizeof(T));
    if (tc) {
        if (!launch_project_tc(dp, (float const*)x, st)) return false;
    } else if (simt) {
        if (!launch_project_simt<T>(dp, x, st)) return false;
    } else {
        // coefficients of images without any block stay zero
        A43G_CUDA_TRY(cudaMemsetAsync(dp.apc.ptr, 0, size_t(dp.ncoeffI)*dp.nCols*128*sizeof(T), st));
        launch_project_L<T, 0>(dp, x, st); launch_project_L<T, 1>(dp, x, st);
        launch_project_L<T, 2>(dp, x, st); launch_project_L<T, 3>(dp, x, st);
        launch_project_L<T, 4>(dp, x, st); launch_project_L<T, 5>(dp, x, st);
        launch_project_L<T, 6>(dp, x, st); launch_project_L<T, 7>(dp, x, st);
    }
    dim3 const ga(dp.nAtoms, dp.nCols);
    if (dp.lmax_max <= 5 && !dp.atom_chain3) {
        sho_atom_kernel<T><<<dim3(dp.nAtoms, dp.nCols, 2), 128, 0, st>>>(dptr<T>(dp.cad), dptr<T>(dp.apc), dp.nCols,
            dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.sum_start), dptr<uint32_t>(dp.sum_col),
            dptr<uint32_t>(dp.img_starts), dptr<double>(dp.img_phase), dptr<double>(dp.atom_mat),
            dptr<uint32_t>(dp.atom_mat_off), dp.nAI > dp.nAtoms ? 1 : 0, dyadic_pairs(dp));
        count_launch();
    } else if (dp.nAI > dp.nAtoms) {
        sho_collect_kernel<T><<<ga, 64, 0, st>>>(dptr<double>(dp.aac), dptr<T>(dp.apc), dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.sum_start),
            dptr<uint32_t>(dp.sum_col), dptr<uint32_t>(dp.img_starts), dptr<double>(dp.img_phase), dyadic_pairs(dp));
        count_launch();
        sho_mul_kernel<double, double><<<ga, 64, 0, st>>>(dptr<double>(dp.cadd), dptr<double>(dp.aac), dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<double>(dp.atom_mat), dptr<uint32_t>(dp.atom_mat_off), dyadic_pairs(dp));
        count_launch();
        sho_broadcast_kernel<T><<<ga, 64, 0, st>>>(dptr<T>(dp.cad), dptr<double>(dp.cadd), dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.sum_start),
            dptr<uint32_t>(dp.sum_col), dptr<uint32_t>(dp.img_starts), dptr<double>(dp.img_phase), dyadic_pairs(dp));
        count_launch();
    } else {
        sho_mul_kernel<T, T><<<ga, 64, 0, st>>>(dptr<T>(dp.cad), dptr<T>(dp.apc), dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<double>(dp.atom_mat), dptr<uint32_t>(dp.atom_mat_off), dyadic_pairs(dp));
        count_launch();
    }
    if (tc) {
        if (!launch_add_tc(dp, (float*)y, colIndex, st)) return false;
    } else if (simt) {
        if (!launch_add_simt<T>(dp, y, colIndex, st)) return false;
    } else {
        sho_add_kernel<T><<<dp.nnzb, 128, 0, st>>>(y, dptr<T>(dp.cad), dp.nCols, dp.nnzb, colIndex,
            dptr<uint32_t>(dp.add_start), dptr<uint32_t>(dp.add_col), dptr<uint32_t>(dp.add_slot),
            dptr<double>(dp.slot_H), dptr<uint64_t>(dp.slot_mask), dp.table_stride,
            dptr<int8_t>(dp.img_lmax), dptr<uint32_t>(dp.img_starts));
        count_launch();
    }
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

template <typename T>
bool launch_action(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t st) {
    if (!launch_local<T>(dp, y, x, st)) return false;
    return launch_dyadic<T>(dp, y, x, colIndex, st);
}

// ---------------------------------------------------------------- pieces of the dyadic part with
// caller-given buffers and tables (FP64), for the vector-Jacobian products

namespace {
template <typename T, int L>
void project_into_L(DevicePlan &dp, T *apc, T const *x, double const *table, cudaStream_t st) {
    auto const &g = dp.prj_items[L];
    if (0 == g.count) return;
    sho_project_kernel<T, L><<<g.count, 128, 0, st>>>(
        apc, x, dp.nCols, dptr<uint32_t>(g.items), dptr<uint32_t>(dp.prj_col), dptr<uint64_t>(dp.prj_coloff),
        dptr<uint32_t>(dp.prj_slot), table, dptr<uint64_t>(dp.slot_mask), dp.table_stride, dptr<uint32_t>(dp.img_starts));
    count_launch();
}

// generic projection (zeroes apc, then atomics per work item) into a caller-given buffer
template <typename T>
bool project_into(DevicePlan &dp, T *apc, T const *x, double const *table, cudaStream_t st) {
    A43G_CUDA_TRY(cudaMemsetAsync(apc, 0, size_t(dp.ncoeffI)*dp.nCols*128*sizeof(T), st));
    project_into_L<T, 0>(dp, apc, x, table, st); project_into_L<T, 1>(dp, apc, x, table, st);
    project_into_L<T, 2>(dp, apc, x, table, st); project_into_L<T, 3>(dp, apc, x, table, st);
    project_into_L<T, 4>(dp, apc, x, table, st); project_into_L<T, 5>(dp, apc, x, table, st);
    project_into_L<T, 6>(dp, apc, x, table, st); project_into_L<T, 7>(dp, apc, x, table, st);
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}
} // namespace

bool launch_project_with(DevicePlan &dp, double *apc, double const *x, double const *table, cudaStream_t st) {
    return project_into<double>(dp, apc, x, table, st);
}

bool launch_collect_with(DevicePlan &dp, double *aac, double const *apc, double const *img_phase, cudaStream_t st) {
    dim3 const ga(dp.nAtoms, dp.nCols);
    sho_collect_kernel<double><<<ga, 64, 0, st>>>(aac, apc, dp.nCols, dptr<uint32_t>(dp.atom_starts),
        dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.sum_start), dptr<uint32_t>(dp.sum_col),
        dptr<uint32_t>(dp.img_starts), img_phase, dyadic_pairs(dp));
    count_launch();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

bool launch_mul_with(DevicePlan &dp, double *out, double const *in, cudaStream_t st) {
    dim3 const ga(dp.nAtoms, dp.nCols);
    sho_mul_kernel<double, double><<<ga, 64, 0, st>>>(out, in, dp.nCols, dptr<uint32_t>(dp.atom_starts),
        dptr<int8_t>(dp.atom_lmax), dptr<double>(dp.atom_mat), dptr<uint32_t>(dp.atom_mat_off), dyadic_pairs(dp));
    count_launch();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

// the whole action with the dyadic coefficients in caller-given scratch (generic kernels only)
template <typename T>
bool launch_action_scratch(DevicePlan &dp, T *y, T const *x, uint16_t const *colIndex, cudaStream_t st,
                           DyadicScratch const &sc) {
    if (!launch_local<T>(dp, y, x, st)) return false;
    if (dp.nAI < 1 || dp.nCols < 1) return true;
    T *apc = static_cast<T*>(sc.apc), *cad = static_cast<T*>(sc.cad);
    if (!project_into<T>(dp, apc, x, dptr<double>(dp.slot_H), st)) return false;
    dim3 const ga(dp.nAtoms, dp.nCols);
    if (dp.nAI > dp.nAtoms) {
        sho_collect_kernel<T><<<ga, 64, 0, st>>>(sc.aac, apc, dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.sum_start),
            dptr<uint32_t>(dp.sum_col), dptr<uint32_t>(dp.img_starts), dptr<double>(dp.img_phase), dyadic_pairs(dp));
        count_launch();
        sho_mul_kernel<double, double><<<ga, 64, 0, st>>>(sc.cadd, sc.aac, dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<double>(dp.atom_mat), dptr<uint32_t>(dp.atom_mat_off), dyadic_pairs(dp));
        count_launch();
        sho_broadcast_kernel<T><<<ga, 64, 0, st>>>(cad, sc.cadd, dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.sum_start),
            dptr<uint32_t>(dp.sum_col), dptr<uint32_t>(dp.img_starts), dptr<double>(dp.img_phase), dyadic_pairs(dp));
        count_launch();
    } else {
        sho_mul_kernel<T, T><<<ga, 64, 0, st>>>(cad, apc, dp.nCols,
            dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<double>(dp.atom_mat), dptr<uint32_t>(dp.atom_mat_off), dyadic_pairs(dp));
        count_launch();
    }
    sho_add_kernel<T><<<dp.nnzb, 128, 0, st>>>(y, cad, dp.nCols, dp.nnzb, colIndex,
        dptr<uint32_t>(dp.add_start), dptr<uint32_t>(dp.add_col), dptr<uint32_t>(dp.add_slot),
        dptr<double>(dp.slot_H), dptr<uint64_t>(dp.slot_mask), dp.table_stride,
        dptr<int8_t>(dp.img_lmax), dptr<uint32_t>(dp.img_starts));
    count_launch();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

template bool launch_action_scratch<double>(DevicePlan &, double *, double const *, uint16_t const *, cudaStream_t, DyadicScratch const &);
template bool launch_action_scratch<float>(DevicePlan &, float *, float const *, uint16_t const *, cudaStream_t, DyadicScratch const &);

template bool launch_local<double>(DevicePlan &, double *, double const *, cudaStream_t);
template bool launch_local<float>(DevicePlan &, float *, float const *, cudaStream_t);
template bool launch_dyadic<double>(DevicePlan &, double *, double const *, uint16_t const *, cudaStream_t);
template bool launch_dyadic<float>(DevicePlan &, float *, float const *, uint16_t const *, cudaStream_t);
template bool launch_action<double>(DevicePlan &, double *, double const *, uint16_t const *, cudaStream_t);
template bool launch_action<float>(DevicePlan &, float *, float const *, uint16_t const *, cudaStream_t);

} // namespace a43g
