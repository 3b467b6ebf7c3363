// Projector contraction of the action on the CUDA cores (FP32 and FP64), sum-factorized
// (include/green_dyadic.hxx:112-288 projection, :325-518 addition).
//
// The projector functions are separable on the spherical mask,
//     P_(ix,iy,iz)(x, y, z) = H_ix(x) H_iy(y) H_iz(z)   for points inside the projection radius,
// so one (block, image) pair costs 64*(L+1) + 16*(L+1)(L+2)/2 + 4*nSHO fused multiply-adds per
// column instead of 64*nSHO for the dense product (944 instead of 3584 at numax 5).
//
// Both kernels keep the 1D tables of the current (image, row) slot and the per-thread partial
// sums in registers (loops fully unrolled for the basis size L), one thread per (real/imaginary
// plane, right-hand-side column):
//   * projection: one CTA per work item (image, source, up to 16 blocks of its list); the
//     blocks stream through a double-buffered shared-memory stage filled with cp.async
//     (16-byte copies, so x must be 16-byte aligned), and the partial coefficients of the item
//     are added to the zeroed image coefficients with one atomic per coefficient;
//   * addition: one CTA per block b, summing the contributions of all images near b in
//     registers and updating y[b] once; the coefficients of the next image are staged in shared
//     memory with cp.async while the current one is applied (16-byte copies of rows that start
//     on 512-byte boundaries of the plan's coefficient array).
#include "device.cuh"

#include <algorithm>

namespace a43g {

namespace {

constexpr int kBlk = 8192;            // floats per block: 2 planes x 64 points x 64 columns
constexpr int kThreads = 128;

__host__ __device__ constexpr int nsho_of(int L) { return ((L + 1)*(L + 2)*(L + 3))/6; }
__host__ __device__ constexpr int n2_of(int L) { return ((L + 1)*(L + 2))/2; }

__device__ __forceinline__ uint32_t smem_addr(void const *p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void cp_async16(void *dst, void const *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// the 1D tables of one slot, H[nu][dir][i] at tab[(nu*3 + dir)*4 + i], dir 0/1/2 = x/y/z, staged in
// shared memory: FP32 copies them into registers, FP64 (twice the registers) reads them in place
template <typename T, int L> struct Tables;
template <int L> struct Tables<float, L> {
    float h[L + 1][3][4];
    __device__ __forceinline__ void load(float const *tab) {
#pragma unroll
        for (int nu = 0; nu <= L; ++nu)
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                float4 const v = *reinterpret_cast<float4 const*>(tab + (nu*3 + d)*4);
                h[nu][d][0] = v.x; h[nu][d][1] = v.y; h[nu][d][2] = v.z; h[nu][d][3] = v.w;
            }
    }
    __device__ __forceinline__ float operator()(int nu, int d, int i) const { return h[nu][d][i]; }
};
template <int L> struct Tables<double, L> {
    double const *p;
    __device__ __forceinline__ void load(double const *tab) { p = tab; }
    __device__ __forceinline__ double operator()(int nu, int d, int i) const { return p[(nu*3 + d)*4 + i]; }
};

__device__ __forceinline__ float fmat(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmat(double a, double b, double c) { return fma(a, b, c); }

// CTAs per SM the kernels are compiled for (FP64 needs twice the registers and shared memory)
template <typename T> struct Occ { static constexpr int project = 3, add = 2; };
template <> struct Occ<double> { static constexpr int project = 1, add = 1; };

__device__ __forceinline__ void cp_async8(void *dst, void const *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(smem_addr(dst)), "l"(src) : "memory");
}

// ---------------------------------------------------------------- projection

// Work item w = (image a, source s, list positions [k0, k1)) of group (first, count): the items of
// one (image, source) pair.  A group of one item writes its coefficients directly; otherwise
// every item stores its partial sums in part[w] and the last item of the group to finish (ticket
// counter) adds the partials in item order, so the result does not depend on the order in which
// the items ran, and resets the counter for the next call.
// ZS threads share a column and split its z-planes (FP64: one CTA of 128 threads per SM would
// leave one warp per scheduler); their partial coefficients are added in a fixed order at the end.
template <typename T, int L, int ZS = int(sizeof(T))/4>
__global__ void __launch_bounds__(kThreads*ZS, Occ<T>::project)
sho_project_simt_kernel(T *__restrict__ apc, T const *__restrict__ x, uint32_t nrhs,
                       uint32_t const *__restrict__ items, uint32_t const *__restrict__ prj_col,
                       uint64_t const *__restrict__ prj_coloff, uint32_t const *__restrict__ prj_slot,
                       T const *__restrict__ slot_H, uint64_t const *__restrict__ slot_mask, int stride,
                       uint32_t const *__restrict__ img_starts, uint8_t const *__restrict__ active,
                       T *__restrict__ part, uint32_t *__restrict__ tickets)
{
    constexpr int NS = nsho_of(L), N2 = n2_of(L);
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *xs = reinterpret_cast<T*>(smem_raw);           // [2][kBlk]
    uint32_t const *item = items + 8*size_t(blockIdx.x);
    uint32_t const a = item[0], s = item[1], k0 = item[2], k1 = item[3];
    uint32_t const g_first = item[4], g_count = item[5], g_id = item[6], g_part = item[7];
    if (active && !active[s]) return;                 // uniform: a retired source
    constexpr int NT = kThreads*ZS, NZ = 4/ZS;         // threads, z-planes per thread
    int const tid = threadIdx.x, zh = tid/kThreads, reim = (tid >> 6) & 1, j = tid & 63;
    uint64_t const off = prj_coloff[s];

    __shared__ __align__(16) T tbuf[2][(L + 1)*12];       // 1D tables of the staged blocks' slots
    __shared__ uint64_t mbuf[2];                           // and their masks
    // block, table and mask of list position k go to shared memory ahead of use; the block and
    // slot indices are loaded one position earlier still
    auto stage = [&](uint32_t b, uint32_t slot, int buf) {
        char const *src = reinterpret_cast<char const*>(x + size_t(b)*kBlk);
        char *dst = reinterpret_cast<char*>(xs + buf*kBlk);
#pragma unroll
        for (int r = 0; r < kBlk*int(sizeof(T))/(16*NT); ++r) {
            int const o = (r*NT + tid)*16;
            cp_async16(dst + o, src + o);
        }
        constexpr int TE = 16/int(sizeof(T));          // table elements per 16-byte copy
        if (tid < (L + 1)*12/TE) cp_async16(&tbuf[buf][tid*TE], slot_H + size_t(slot)*stride + tid*TE);
        if (tid == NT - 1) cp_async8(&mbuf[buf], slot_mask + slot);
    };

    T acc[NS];
#pragma unroll
    for (int i = 0; i < NS; ++i) acc[i] = T(0);

    stage(prj_col[off + k0], prj_slot[off + k0], 0);
    cp_async_commit();
    uint32_t nb = 0, ns = 0;
    if (k0 + 1 < k1) { nb = prj_col[off + k0 + 1]; ns = prj_slot[off + k0 + 1]; }
    int buf = 0;
    for (uint32_t k = k0; k < k1; ++k, buf ^= 1) {
        if (k + 1 < k1) stage(nb, ns, buf ^ 1);
        cp_async_commit();
        if (k + 2 < k1) { nb = prj_col[off + k + 2]; ns = prj_slot[off + k + 2]; }   // for the next iteration
        cp_async_wait1();                            // block k has landed (this thread's copies)
        __syncthreads();                             // ... and everybody else's
        Tables<T, L> t;
        t.load(tbuf[buf]);
        // the x-functions of the slot in registers (FP64 reads the other tables in place)
        T tx[L + 1][4];
#pragma unroll
        for (int ix = 0; ix <= L; ++ix)
#pragma unroll
            for (int xx = 0; xx < 4; ++xx) tx[ix][xx] = t(ix, 0, xx);
        uint64_t const mask = mbuf[buf];
        T const *xb = xs + buf*kBlk + reim*4096 + j;
#pragma unroll
        for (int zl = 0; zl < NZ; ++zl) {
            int const z = zh*NZ + zl;
            if (0 == ((mask >> (16*z)) & 0xffffu)) continue;     // uniform per thread: plane outside the sphere
            T byx[N2];
#pragma unroll
            for (int i = 0; i < N2; ++i) byx[i] = T(0);
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) {
                T ax[L + 1];
#pragma unroll
                for (int i = 0; i <= L; ++i) ax[i] = T(0);
#pragma unroll
                for (int xx = 0; xx < 4; ++xx) {
                    int const p = (z*4 + yy)*4 + xx;
                    T const v = ((mask >> p) & 1u) ? xb[p*64] : T(0);
#pragma unroll
                    for (int ix = 0; ix <= L; ++ix) ax[ix] = fmat(v, tx[ix][xx], ax[ix]);
                }
#pragma unroll
                for (int iy = 0, iyx = 0; iy <= L; ++iy) {
                    T const hy = t(iy, 1, yy);
#pragma unroll
                    for (int ix = 0; ix <= L - iy; ++ix, ++iyx) byx[iyx] = fmat(ax[ix], hy, byx[iyx]);
                }
            }
#pragma unroll
            for (int iz = 0, sho = 0; iz <= L; ++iz) {
                T const hz = t(iz, 2, z);
#pragma unroll
                for (int iy = 0; iy <= L - iz; ++iy) {
                    int const iyx = iy*(2*L + 3 - iy)/2;
#pragma unroll
                    for (int ix = 0; ix <= L - iz - iy; ++ix, ++sho) acc[sho] = fmat(byx[iyx + ix], hz, acc[sho]);
                }
            }
        }
        __syncthreads();                             // buffer buf is free for block k + 2
    }
    if constexpr (ZS > 1) {
        // the partial sums of the other z-planes, through the (now free) block stage, added in
        // the order of the planes
        cp_async_wait0();
        __syncthreads();
        if (zh > 0) {
#pragma unroll
            for (int sho = 0; sho < NS; ++sho) xs[(size_t(zh - 1)*NS + sho)*128 + reim*64 + j] = acc[sho];
        }
        __syncthreads();
        if (zh > 0) return;
        for (int h = 1; h < ZS; ++h) {
#pragma unroll
            for (int sho = 0; sho < NS; ++sho) acc[sho] += xs[(size_t(h - 1)*NS + sho)*128 + reim*64 + j];
        }
    }
    T *out = apc + (size_t(img_starts[a])*nrhs + s)*128 + reim*64 + j;
    if (1 == g_count) {
#pragma unroll
        for (int sho = 0; sho < NS; ++sho) out[size_t(sho)*nrhs*128] = acc[sho];
        return;
    }
    // partial sums of this item: part[(g_part + position in group)][sho][128]
    uint32_t const q = blockIdx.x - g_first;
    T *mine = part + (size_t(g_part) + q)*NS*128 + reim*64 + j;
#pragma unroll
    for (int sho = 0; sho < NS; ++sho) mine[size_t(sho)*128] = acc[sho];
    __threadfence();                                  // partials visible before the ticket
    __shared__ uint32_t ticket;
    if constexpr (ZS > 1) {
        // the remaining threads of the first z-group only (the others have returned)
        asm volatile("bar.sync 1, %0;" :: "n"(kThreads) : "memory");
        if (0 == tid) ticket = atomicAdd(&tickets[g_id], 1u);
        asm volatile("bar.sync 1, %0;" :: "n"(kThreads) : "memory");
    } else {
        __syncthreads();
        if (0 == tid) ticket = atomicAdd(&tickets[g_id], 1u);
        __syncthreads();
    }
    if (ticket + 1 != g_count) return;                // uniform: not the last item of the group
    __threadfence();
    T const *pg = part + size_t(g_part)*NS*128 + reim*64 + j;
#pragma unroll 4
    for (int sho = 0; sho < NS; ++sho) {
        T sum = T(0);
        for (uint32_t i = 0; i < g_count; ++i) sum += __ldcg(pg + (size_t(i)*NS + sho)*128);
        out[size_t(sho)*nrhs*128] = sum;
    }
    if (0 == tid) tickets[g_id] = 0u;                 // ready for the next call
}

// ---------------------------------------------------------------- addition

// contribution of one image with basis size L to the 64 point sums of this thread
// ZS threads share a column and split its x-points (FP64: the 64 sums of one thread would not
// fit the registers): thread zh owns x = zh*(4/ZS) ... of every (z, y) row, so each stage of
// the contraction (x, then y, then z) is split between them without repeating any work.  The
// sums are ordered acc[(z*4 + y)*(4/ZS) + x - zh*(4/ZS)].
// UZ: the z-orders unrolled (tables and coefficient offsets known at compile time) or one at a
// time (fewer registers)
template <typename T, int L, bool FULL, int ZS, bool UZ>
__device__ __forceinline__ void add_image(T (&acc)[64/ZS], Tables<T, L> const &t, uint64_t mask,
                                          T const *__restrict__ c, size_t cstride, int zh) {
    constexpr int kUnrollZ = UZ ? L + 1 : 1;
    constexpr int NX = 4/ZS;                                   // x-points of this thread
    int const x0 = (1 == ZS) ? 0 : zh*NX;
    int sho = 0;
#pragma unroll kUnrollZ
    for (int iz = 0; iz <= L; ++iz) {
        T byx[4*NX];
#pragma unroll
        for (int i = 0; i < 4*NX; ++i) byx[i] = T(0);
#pragma unroll
        for (int iy = 0; iy <= L - iz; ++iy) {
            T ax[NX];
#pragma unroll
            for (int xl = 0; xl < NX; ++xl) ax[xl] = T(0);
#pragma unroll
            for (int ix = 0; ix <= L - iz - iy; ++ix, ++sho) {
                T const cv = c[size_t(sho)*cstride];
#pragma unroll
                for (int xl = 0; xl < NX; ++xl) ax[xl] = fmat(t(ix, 0, x0 + xl), cv, ax[xl]);
            }
#pragma unroll
            for (int yy = 0; yy < 4; ++yy) {
                T const hy = t(iy, 1, yy);
#pragma unroll
                for (int xl = 0; xl < NX; ++xl) byx[yy*NX + xl] = fmat(hy, ax[xl], byx[yy*NX + xl]);
            }
        }
#pragma unroll
        for (int z = 0; z < 4; ++z) {
            T const hz = t(iz, 2, z);
#pragma unroll
            for (int q = 0; q < 4*NX; ++q) {
                int const pl = z*4*NX + q, p = z*16 + (q/NX)*4 + x0 + (q % NX);
                if (FULL) acc[pl] = fmat(hz, byx[q], acc[pl]);
                else acc[pl] = ((mask >> p) & 1u) ? fmat(hz, byx[q], acc[pl]) : acc[pl];
            }
        }
    }
}

template <typename T, int L, int ZS, bool UZ>
__device__ __forceinline__ void add_image_L(T (&acc)[64/ZS], T const *__restrict__ tab, uint64_t mask,
                                            T const *__restrict__ c, size_t cstride, int zh) {
    Tables<T, L> t;
    t.load(tab);
    if (~0ull == mask) add_image<T, L, true, ZS, UZ>(acc, t, mask, c, cstride, zh);
    else add_image<T, L, false, ZS, UZ>(acc, t, mask, c, cstride, zh);
}

// LMAX: largest basis size of the plan (the instantiation has no larger one).  One CTA walks the
// blocks [b0, b1) (consecutive, same order as y) and treats their (block, image) pairs as one
// stream: the coefficients, table and mask of the next pair are staged while the current pair is
// applied, and the y values of the next block with atoms are staged during the whole of the
// current block, so neither the start of a block nor its final y update waits for memory.
template <typename T, int LMAX, int ZS = int(sizeof(T))/4, bool UZ = true>
__global__ void __launch_bounds__(kThreads*ZS, Occ<T>::add)
sho_add_simt_kernel(T *__restrict__ y, T const *__restrict__ cad, uint32_t nrhs, uint32_t nnzb,
                    uint32_t blocks_per_cta, uint16_t const *__restrict__ colIndex,
                    uint32_t const *__restrict__ add_start, uint4 const *__restrict__ info,
                    T const *__restrict__ slot_H, uint64_t const *__restrict__ slot_mask, int stride,
                    uint8_t const *__restrict__ active)
{
    constexpr int NCMAX = nsho_of(LMAX);
    constexpr int TE = 16/int(sizeof(T));                  // elements per 16-byte copy
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T *cbuf = reinterpret_cast<T*>(smem_raw);              // [2][NCMAX][128] coefficients of two pairs
    T *ybuf = cbuf + 2*NCMAX*128;                          // [8192] y of the current block
    __shared__ __align__(16) T tbuf[2][(LMAX + 1)*12];
    __shared__ uint64_t mbuf[2];
    uint32_t const b0 = blockIdx.x*blocks_per_cta, b1 = min(b0 + blocks_per_cta, nnzb);
    if (b0 >= b1) return;
    uint32_t const T0 = add_start[b0], T1 = add_start[b1];
    if (T0 >= T1) return;                                  // no atoms near any of these blocks
    constexpr int NT = kThreads*ZS, NP = 64/ZS;             // threads, point sums per thread
    int const tid = threadIdx.x, zh = tid/kThreads, reim = (tid >> 6) & 1, j = tid & 63;
    size_t const cstride = size_t(nrhs)*128;

    // the block owning pair t: blocks are visited in order, skipping blocks without pairs
    uint32_t bb = b0;
    while (add_start[bb + 1] <= T0) ++bb;
    uint32_t s = colIndex[bb];
    uint32_t bend = add_start[bb + 1];                     // first pair of the next block

    // pairs of a retired source stage nothing and carry an empty mask: no work, no y update
    auto stage_pair = [&](uint4 const inf, uint32_t src_col, int buf) {
        if (active && !active[src_col]) {
            if (tid == NT - 1) mbuf[buf] = 0;
            return;
        }
        int const L = int(inf.z), nc = nsho_of(L);
        T const *src = cad + (size_t(inf.y)*nrhs + src_col)*128;
        T *dst = cbuf + buf*NCMAX*128;
        constexpr int CPR = 128/TE;                        // 16-byte copies per coefficient row
        for (int q = tid; q < nc*CPR; q += NT) {
            int const row = q/CPR, part = (q % CPR)*TE;
            cp_async16(dst + row*128 + part, src + size_t(row)*cstride + part);
        }
        if (tid < (L + 1)*12/TE) cp_async16(&tbuf[buf][tid*TE], slot_H + size_t(inf.x)*stride + tid*TE);
        if (tid == NT - 1) cp_async8(&mbuf[buf], slot_mask + inf.x);
    };
    auto stage_y = [&](uint32_t blk) {
        if (active && !active[colIndex[blk]]) return;
        T const *src = y + size_t(blk)*kBlk;
#pragma unroll
        for (int r = 0; r < kBlk/(TE*NT); ++r) {
            int const o = (r*NT + tid)*TE;
            cp_async16(ybuf + o, src + o);
        }
    };
    // the source column of the pair after t (it may belong to a later block)
    auto column_of = [&](uint32_t t) -> uint32_t {
        uint32_t c = bb;
        while (add_start[c + 1] <= t) ++c;
        return colIndex[c];
    };

    T acc[NP];
#pragma unroll
    for (int i = 0; i < NP; ++i) acc[i] = T(0);
    uint64_t mask_all = 0;
    uint4 const zero4 = make_uint4(0u, 0u, 0u, 0u);
    uint4 cur = info[T0];
    stage_y(bb);
    stage_pair(cur, s, 0);
    cp_async_commit();
    uint4 nxt = (T0 + 1 < T1) ? info[T0 + 1] : zero4;
    int buf = 0;
    for (uint32_t t = T0; t < T1; ++t, buf ^= 1) {
        if (t + 1 < T1) stage_pair(nxt, (t + 1 < bend) ? s : column_of(t + 1), buf ^ 1);
        cp_async_commit();
        uint4 const after = (t + 2 < T1) ? info[t + 2] : zero4;
        cp_async_wait1();
        __syncthreads();
        uint64_t const mask = mbuf[buf];
        if (mask) {
            mask_all |= mask;
            T const *tab = tbuf[buf];
            T const *c = cbuf + buf*NCMAX*128 + reim*64 + j;
            int const L = int(cur.z);                      // uniform over the CTA
            if (L == LMAX) add_image_L<T, LMAX, ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 0 && L == 0) add_image_L<T, 0, ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 1 && L == 1) add_image_L<T, (LMAX > 1 ? 1 : 0), ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 2 && L == 2) add_image_L<T, (LMAX > 2 ? 2 : 0), ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 3 && L == 3) add_image_L<T, (LMAX > 3 ? 3 : 0), ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 4 && L == 4) add_image_L<T, (LMAX > 4 ? 4 : 0), ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 5 && L == 5) add_image_L<T, (LMAX > 5 ? 5 : 0), ZS, UZ>(acc, tab, mask, c, 128, zh);
            else if (LMAX > 6 && L == 6) add_image_L<T, (LMAX > 6 ? 6 : 0), ZS, UZ>(acc, tab, mask, c, 128, zh);
        }
        cur = nxt; nxt = after;
        if (t + 1 == bend) {
            // last pair of block bb: y[bb] = staged y + sums on the points inside the spheres
            cp_async_wait0();
            __syncthreads();
            T const *yb_s = ybuf + reim*4096 + j;
            T *yb = y + size_t(bb)*kBlk + reim*4096 + j;
#pragma unroll
            for (int pl = 0; pl < NP; ++pl) {
                int const p = (pl/(4/ZS))*4 + zh*(4/ZS) + pl % (4/ZS);   // this thread's points
                if ((mask_all >> p) & 1u) yb[p*64] = yb_s[p*64] + acc[pl];
                acc[pl] = T(0);
            }
            mask_all = 0;
            __syncthreads();                               // ybuf free
            if (t + 1 < T1) {
                ++bb;
                while (add_start[bb + 1] <= t + 1) ++bb;
                s = colIndex[bb];
                bend = add_start[bb + 1];
                stage_y(bb);                               // lands during the pairs of block bb
            }
        }
        __syncthreads();                                   // buffers buf are free for pair t + 2
    }
}

template <typename T> T const *simt_table(DevicePlan const &dp);
template <> float const *simt_table<float>(DevicePlan const &dp) { return dptr<float>(dp.slot_H32); }
template <> double const *simt_table<double>(DevicePlan const &dp) { return dptr<double>(dp.slot_H); }

template <typename T, int L>
void launch_project_L(DevicePlan &dp, T const *x, cudaStream_t st) {
    auto const &g = dp.prj_items[L];
    if (0 == g.count) return;
    constexpr int smem = 2*kBlk*int(sizeof(T));         // double-buffered block stage
    sho_project_simt_kernel<T, L><<<g.count, kThreads*(int(sizeof(T))/4), smem, st>>>(
        dptr<T>(dp.apc), x, dp.nCols, dptr<uint32_t>(g.items8), dptr<uint32_t>(dp.prj_col),
        dptr<uint64_t>(dp.prj_coloff), dptr<uint32_t>(dp.prj_slot), simt_table<T>(dp),
        dptr<uint64_t>(dp.slot_mask), dp.table_stride, dptr<uint32_t>(dp.img_starts),
        dp.retire ? dptr<uint8_t>(dp.src_active) : nullptr, dptr<T>(dp.prj_part), dptr<uint32_t>(g.tickets));
    count_launch();
}

template <typename T, int LMAX>
void launch_add_L(DevicePlan &dp, T *y, uint16_t const *colIndex, cudaStream_t st) {
    constexpr int smem = (2*nsho_of(LMAX)*128 + kBlk)*int(sizeof(T));
    constexpr int ZS = int(sizeof(T))/4;
    uint32_t const per_cta = std::max<uint32_t>(1, dp.add_blocks);
    unsigned const grid = (dp.nnzb + per_cta - 1)/per_cta;
    auto *k = sho_add_simt_kernel<T, LMAX, ZS, true>;
    if (sizeof(T) == 8 && !dp.add64_unrolled) k = sho_add_simt_kernel<T, LMAX, ZS, false>;
    k<<<grid, kThreads*ZS, smem, st>>>(y, dptr<T>(dp.cad), dp.nCols, dp.nnzb, per_cta,
        colIndex, dptr<uint32_t>(dp.add_start), dptr<uint4>(dp.add_info), simt_table<T>(dp),
        dptr<uint64_t>(dp.slot_mask), dp.table_stride, dp.retire ? dptr<uint8_t>(dp.src_active) : nullptr);
}

template <typename T, int L>
void set_smem_attributes() {
    cudaFuncSetAttribute(sho_project_simt_kernel<T, L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         2*kBlk*int(sizeof(T)));
    cudaFuncSetAttribute(sho_add_simt_kernel<T, L, int(sizeof(T))/4, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (2*nsho_of(L)*128 + kBlk)*int(sizeof(T)));
    if (sizeof(T) == 8)
        cudaFuncSetAttribute(sho_add_simt_kernel<T, L, int(sizeof(T))/4, false>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (2*nsho_of(L)*128 + kBlk)*int(sizeof(T)));
}

} // namespace

bool prepare_simt_kernels() {
    // the dynamic shared memory the kernels need beyond 48 KB (per device: called with the
    // device current, before any launch and outside stream capture)
    set_smem_attributes<float, 0>(); set_smem_attributes<float, 1>(); set_smem_attributes<float, 2>();
    set_smem_attributes<float, 3>(); set_smem_attributes<float, 4>(); set_smem_attributes<float, 5>();
    set_smem_attributes<float, 6>(); set_smem_attributes<float, 7>();
    set_smem_attributes<double, 0>(); set_smem_attributes<double, 1>(); set_smem_attributes<double, 2>();
    set_smem_attributes<double, 3>(); set_smem_attributes<double, 4>(); set_smem_attributes<double, 5>();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

bool simt_projector_supported(DevicePlan const &dp, void const *x, void const *y, size_t real_bytes) {
    // 16-byte staging copies; the FP64 addition stages up to numax 5 (shared memory)
    int const lmax_limit = (8 == real_bytes) ? 5 : 7;
    return dp.slot_H32.ptr && dp.lmax_max <= lmax_limit && 0 == (reinterpret_cast<uintptr_t>(x) & 15u) &&
           0 == (reinterpret_cast<uintptr_t>(y) & 15u);
}

template <typename T>
bool launch_project_simt(DevicePlan &dp, T const *x, cudaStream_t st) {
    // every (image, source) pair with blocks is written by its items; images without blocks of a
    // source keep zero coefficients
    if (!ensure_prj_part(dp, sizeof(T))) return false;
    A43G_CUDA_TRY(cudaMemsetAsync(dp.apc.ptr, 0, size_t(dp.ncoeffI)*dp.nCols*128*sizeof(T), st));
    launch_project_L<T, 0>(dp, x, st); launch_project_L<T, 1>(dp, x, st);
    launch_project_L<T, 2>(dp, x, st); launch_project_L<T, 3>(dp, x, st);
    launch_project_L<T, 4>(dp, x, st); launch_project_L<T, 5>(dp, x, st);
    if constexpr (sizeof(T) == 4) {
        launch_project_L<T, 6>(dp, x, st); launch_project_L<T, 7>(dp, x, st);
    }
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

// (FP64 up to numax 5: its two coefficient stages and y fit 227 KB of shared memory)
template <typename T>
bool launch_add_simt(DevicePlan &dp, T *y, uint16_t const *colIndex, cudaStream_t st) {
    switch (dp.lmax_max) {
        case 0: launch_add_L<T, 0>(dp, y, colIndex, st); break;
        case 1: launch_add_L<T, 1>(dp, y, colIndex, st); break;
        case 2: launch_add_L<T, 2>(dp, y, colIndex, st); break;
        case 3: launch_add_L<T, 3>(dp, y, colIndex, st); break;
        case 4: launch_add_L<T, 4>(dp, y, colIndex, st); break;
        case 5: launch_add_L<T, 5>(dp, y, colIndex, st); break;
        default:
            if constexpr (sizeof(T) == 4) {
                if (6 == dp.lmax_max) launch_add_L<T, 6>(dp, y, colIndex, st);
                else launch_add_L<T, 7>(dp, y, colIndex, st);
            }
            break;
    }
    count_launch();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

template bool launch_project_simt<float>(DevicePlan &, float const *, cudaStream_t);
template bool launch_project_simt<double>(DevicePlan &, double const *, cudaStream_t);
template bool launch_add_simt<float>(DevicePlan &, float *, uint16_t const *, cudaStream_t);
template bool launch_add_simt<double>(DevicePlan &, double *, uint16_t const *, cudaStream_t);

} // namespace a43g
