// FP32 projector contraction of the action on the sm_100a tensor cores (tcgen05, kind::tf32,
// 3xTF32 split precision, FP32 accumulation in TMEM).
//
// Projection (include/green_dyadic.hxx:112-288), one CTA per (atom image a, source s):
//     C^T[(reim, j), sho] = sum over the blocks b of s near a:  X[b]^T (128 x 64) . P[a,b]^T (64 x 64)
//   M = 128 (real and imaginary planes x 64 source columns), N = 64 (nSHO <= 56 padded),
//   K = 64 grid points per block.
// Addition (include/green_dyadic.hxx:325-518), one CTA per block b:
//     D[(reim, j), i] = sum over the images a near b:  Cad[a, s]^T (128 x 64) . P[a,b] (64 x 64)
//   and y[b] += D^T on the points inside the projection spheres.
// P[sho][i] = H_ix(x_i) H_iy(y_i) H_iz(z_i) on the mask (tables of the plan), 0 elsewhere.
// Each operand x is split x = hi + lo with hi = TF32(x); C = A_hi B_hi + A_hi B_lo + A_lo B_hi.
// Both operands are K-major in shared memory (no swizzle; an MN-major TF32 A operand in this
// layout produced zeros on B200, so the data tiles are transposed while they are staged).
// Operands are staged by all threads into shared memory (double-buffered stages), one thread
// issues the MMAs and commits them to an mbarrier; every wait is bounded and a timeout is
// recorded in the device error flag instead of hanging.
#include "device.cuh"
#include "tc_sm100.cuh"

namespace a43g {

namespace {

constexpr int kThreads = 256;
constexpr int kA = 32768;            // bytes of one 128 x 64 FP32 operand
constexpr int kB = 16384;            // bytes of one 64 x 64 FP32 operand
constexpr int kStage = 2*kA + 2*kB;  // A_hi, A_lo, B_hi, B_lo
constexpr int kRaw = 32768;          // one FP32 block as it is in memory, prefetched by cp.async
constexpr int kSmem = 2*kStage + kRaw;        // 224 KB of the 227 KB a CTA may use
constexpr uint64_t kWaitNs = 500000000ull;    // 0.5 s per wait: far beyond any MMA latency
constexpr uint32_t kIdesc = tc::idesc_tf32(128, 64, false, false);  // A and B K-major

// byte offset of element (m, k) of a 128 x 64 K-major operand (core matrices 8 m x 4 k;
// K chunks 2048 bytes apart, 8-row groups 128 bytes apart)
__device__ __forceinline__ uint32_t offA(int m, int k) { return ((k >> 2)*16 + (m >> 3))*128 + ((m & 7)*4 + (k & 3))*4; }
// byte offset of element (n, k) of a 64 x 64 K-major operand (core matrices 8 n x 4 k)
__device__ __forceinline__ uint32_t offB(int n, int k) { return ((k >> 2)*8 + (n >> 3))*128 + ((n & 7)*4 + (k & 3))*4; }

// issue the 8 K-steps x 3 split products of one 64-deep chunk
__device__ __forceinline__ void issue_mmas(uint32_t tmem, uint32_t sA_hi, uint32_t sA_lo, uint32_t sB_hi,
                                           uint32_t sB_lo, bool first) {
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        uint64_t const ah = tc::smem_desc(sA_hi + s*4096, 2048, 128), al = tc::smem_desc(sA_lo + s*4096, 2048, 128);
        uint64_t const bh = tc::smem_desc(sB_hi + s*2048, 1024, 128), bl = tc::smem_desc(sB_lo + s*2048, 1024, 128);
        tc::mma_tf32(tmem, ah, bh, kIdesc, (first && 0 == s) ? 0u : 1u);
        tc::mma_tf32(tmem, ah, bl, kIdesc, 1u);
        tc::mma_tf32(tmem, al, bh, kIdesc, 1u);
    }
}

// stage a 128 x 64 FP32 matrix, element (m = reim*64 + j, k) at src[reim*plane + k*ld_k + j]
// (shared memory), as the split K-major operand; rows k >= kmax are zero.  Thread (m, kh)
// gathers column m for the 32 values k = kh*32 ... (scalar loads, consecutive m in consecutive
// banks) and stores 4 k-values per 16-byte chunk: the 8 threads of a store phase write the 8
// rows of one core matrix, 128 contiguous bytes, so neither loads nor stores conflict.
__device__ __forceinline__ void stage_A(char *sA_hi, char *sA_lo, float const *src, size_t plane,
                                        size_t ld_k, int kmax, int tid) {
    static_assert(kThreads == 256, "one thread per (row, half of K)");
    int const m = tid & 127, kh = tid >> 7;
    float const *col = src + (m >> 6)*plane + (m & 63);
#pragma unroll
    for (int c = 0; c < 8; ++c) {                    // 4 k-values per chunk
        int const k0 = kh*32 + c*4;
        float v[4];
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) v[kk] = (k0 + kk < kmax) ? col[size_t(k0 + kk)*ld_k] : 0.f;
        float4 h, l;
        tc::split_tf32(v[0], h.x, l.x); tc::split_tf32(v[1], h.y, l.y);
        tc::split_tf32(v[2], h.z, l.z); tc::split_tf32(v[3], h.w, l.w);
        uint32_t const o = offA(m, k0);
        *reinterpret_cast<float4*>(sA_hi + o) = h;
        *reinterpret_cast<float4*>(sA_lo + o) = l;
    }
}

struct ShoIdx { uint8_t ix[64], iy[64], iz[64]; };

__device__ __forceinline__ void fill_sho_index(ShoIdx &t, int lmax, int tid) {
    if (0 == tid) {
        int sho = 0;
        for (int iz = 0; iz <= lmax; ++iz)
            for (int iy = 0; iy <= lmax - iz; ++iy)
                for (int ix = 0; ix <= lmax - iz - iy; ++ix, ++sho) { t.ix[sho] = ix; t.iy[sho] = iy; t.iz[sho] = iz; }
    }
}

__device__ __forceinline__ float pval(float const (*H)[3][4], ShoIdx const &t, uint64_t mask, int sho, int nsho, int i) {
    if (sho >= nsho || !((mask >> i) & 1)) return 0.f;
    return H[t.ix[sho]][0][i & 3]*H[t.iy[sho]][1][(i >> 2) & 3]*H[t.iz[sho]][2][i >> 4];
}

__device__ __forceinline__ void record_error(int *err, int code) { atomicCAS(err, 0, code); }

__device__ __forceinline__ void cp_async16(void *dst, void const *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async8(void *dst, void const *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" :: "r"(tc::smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// ---------------------------------------------------------------- projection

__global__ void __launch_bounds__(kThreads, 1)
sho_project_tc_kernel(float *__restrict__ apc, float const *__restrict__ x, uint32_t nrhs,
                      uint32_t const *__restrict__ images, uint32_t nAI, uint32_t const *__restrict__ prj_start,
                      uint32_t const *__restrict__ prj_col, uint64_t const *__restrict__ prj_coloff,
                      uint32_t const *__restrict__ prj_slot, float const *__restrict__ slot_H,
                      uint64_t const *__restrict__ slot_mask, int stride, uint32_t const *__restrict__ img_starts,
                      int8_t const *__restrict__ img_lmax, int *err)
{
    extern __shared__ __align__(128) char smem[];
    __shared__ __align__(16) float Hs[2][8][3][4];
    __shared__ ShoIdx sidx;
    __shared__ uint64_t mbar[2];
    __shared__ uint64_t mk[2];
    __shared__ uint32_t tmem_base;
    int const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t const a = images[blockIdx.x];
    int const s = blockIdx.y;
    int const lmax = img_lmax[a], nsho = ((lmax + 1)*(lmax + 2)*(lmax + 3))/6;
    uint32_t const *start = prj_start + size_t(s)*(nAI + 1);
    uint64_t const off = prj_coloff[s];
    uint32_t const k0 = start[a], k1 = start[a + 1];
    float *out = apc + (size_t(img_starts[a])*nrhs + s)*128;
    if (*(int const volatile*)err) return;             // an earlier CTA timed out: results are void
    if (k0 == k1) {                                  // no block: zero coefficients
        for (int e = tid; e < nsho*128; e += kThreads) out[size_t(e >> 7)*nrhs*128 + (e & 127)] = 0.f;
        return;
    }
    fill_sho_index(sidx, lmax, tid);
    if (0 == warp) tc::tmem_alloc(&tmem_base, 64);
    if (0 == tid) { tc::mbar_init(&mbar[0], 1); tc::mbar_init(&mbar[1], 1); }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    uint32_t const tmem = tmem_base;
    bool ok = true;
    int issued = 0;                                  // commits issued (block-uniform)
    float *raw = reinterpret_cast<float*>(smem + 2*kStage);
    // block k (as stored), its 1D tables and mask go to shared memory one block ahead
    auto prefetch = [&](uint32_t k, int st) {
        float const *src = x + size_t(prj_col[off + k])*8192;
        uint32_t const slot = prj_slot[off + k];
#pragma unroll
        for (int r = 0; r < kRaw/(16*kThreads); ++r) {
            int const o = (r*kThreads + tid)*4;
            cp_async16(raw + o, src + o);
        }
        if (tid < (lmax + 1)*3) cp_async16(&Hs[st][0][0][0] + tid*4, slot_H + size_t(slot)*stride + tid*4);
        if (tid == kThreads - 1) cp_async8(&mk[st], slot_mask + slot);
        cp_async_commit();
    };
    prefetch(k0, 0);
    for (uint32_t k = k0; k < k1; ++k) {
        int const it = int(k - k0), st = it & 1;
        char *sA_hi = smem + st*kStage, *sA_lo = sA_hi + kA, *sB_hi = sA_lo + kA, *sB_lo = sB_hi + kB;
        if (it >= 2) {                               // stage st is free once the MMAs of it-2 completed
            bool w = true;
            if (0 == tid) w = tc::mbar_wait(&mbar[st], uint32_t((it - 2) >> 1) & 1u, kWaitNs, err);
            ok = __syncthreads_and(w);               // block-uniform decision
            if (!ok) break;
        }
        cp_async_wait0();                            // block k, its tables and mask have landed
        __syncthreads();
        uint64_t const mask = mk[st];
        stage_A(sA_hi, sA_lo, raw, 4096, 64, 64, tid);   // A = X^T: m = (reim, j), k = point i
        __syncthreads();                             // raw is free: fetch the next block meanwhile
        if (k + 1 < k1) prefetch(k + 1, st ^ 1);
        // B = P^T: n = sho, k = point i; float4 along k
#pragma unroll 2
        for (int r = 0; r < 1024/kThreads; ++r) {
            int const q = r*kThreads + tid;
            int const n = ((q >> 3) & 7)*8 + (q & 7), kc = q >> 6;
            float4 v;
            v.x = pval(Hs[st], sidx, mask, n, nsho, kc*4 + 0); v.y = pval(Hs[st], sidx, mask, n, nsho, kc*4 + 1);
            v.z = pval(Hs[st], sidx, mask, n, nsho, kc*4 + 2); v.w = pval(Hs[st], sidx, mask, n, nsho, kc*4 + 3);
            float4 h, l;
            tc::split_tf32(v.x, h.x, l.x); tc::split_tf32(v.y, h.y, l.y);
            tc::split_tf32(v.z, h.z, l.z); tc::split_tf32(v.w, h.w, l.w);
            uint32_t const o = offB(n, kc*4);
            *reinterpret_cast<float4*>(sB_hi + o) = h;
            *reinterpret_cast<float4*>(sB_lo + o) = l;
        }
        tc::fence_smem_to_async();
        __syncthreads();
        if (0 == tid) {
            tc::fence_after_sync();
            issue_mmas(tmem, tc::smem_u32(sA_hi), tc::smem_u32(sA_lo), tc::smem_u32(sB_hi), tc::smem_u32(sB_lo), 0 == it);
            tc::commit(&mbar[st]);
        }
        ++issued;
    }
    cp_async_wait0();                                // no copy outstanding when the CTA ends
    int const last = issued - 1;
    if (last >= 0) {
        bool w = ok;
        if (0 == tid && ok) w = tc::mbar_wait(&mbar[last & 1], uint32_t(last >> 1) & 1u, kWaitNs, err);
        ok = __syncthreads_and(w);
    }
    if (!ok && 0 == tid && last >= 0) {
        record_error(err, 1);
        // give the tensor core a bounded grace period before the TMEM is released
        tc::mbar_wait(&mbar[last & 1], uint32_t(last >> 1) & 1u, kWaitNs, err);
    }
    tc::fence_after_sync();
    if (ok) {
        // warps w and w+4 share TMEM lane quarter w%4: columns 0-31 and 32-63
        float v[32];
        int const quarter = warp & 3, half = warp >> 2;
        uint32_t const taddr = tmem + (uint32_t(quarter*32) << 16) + uint32_t(half*32);
        tc::tmem_ld_32x32b_x32(taddr, v);
        int const m = quarter*32 + lane;
#pragma unroll
        for (int c = 0; c < 32; ++c)
            if (half*32 + c < nsho) out[size_t(half*32 + c)*nrhs*128 + m] = v[c];
    }
    tc::fence_before_sync();
    __syncthreads();
    if (0 == warp) tc::tmem_dealloc(tmem, 64);
}

// ---------------------------------------------------------------- addition

__global__ void __launch_bounds__(kThreads, 1)
sho_add_tc_kernel(float *__restrict__ y, float const *__restrict__ cad, uint32_t nrhs,
                  uint16_t const *__restrict__ colIndex, uint32_t const *__restrict__ add_start,
                  uint32_t const *__restrict__ add_col, uint32_t const *__restrict__ add_slot,
                  float const *__restrict__ slot_H, uint64_t const *__restrict__ slot_mask, int stride,
                  int8_t const *__restrict__ img_lmax, uint32_t const *__restrict__ img_starts, int *err)
{
    extern __shared__ __align__(128) char smem[];
    __shared__ __align__(16) float Hs[2][8][3][4];
    __shared__ ShoIdx sidx[2];
    __shared__ uint64_t mbar[2];
    __shared__ uint64_t mk[2];
    __shared__ int lm[2];
    __shared__ uint32_t tmem_base;
    int const tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    uint32_t const b = blockIdx.x;
    uint32_t const k0 = add_start[b], k1 = add_start[b + 1];
    if (k0 == k1 || *(int const volatile*)err) return;
    uint32_t const s = colIndex[b];
    if (0 == warp) tc::tmem_alloc(&tmem_base, 64);
    if (0 == tid) { tc::mbar_init(&mbar[0], 1); tc::mbar_init(&mbar[1], 1); }
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    uint32_t const tmem = tmem_base;
    uint64_t mask_all = 0;
    bool ok = true;
    int issued = 0;                                  // commits issued (block-uniform)
    float *raw = reinterpret_cast<float*>(smem + 2*kStage);
    size_t const cstride = size_t(nrhs)*128;
    // coefficients (nSHO rows of 128 floats), tables and mask of image k go to shared memory
    // one image ahead
    auto prefetch = [&](uint32_t k, int st) {
        uint32_t const a = add_col[k], slot = add_slot[k];
        int const lmax = img_lmax[a], nsho = ((lmax + 1)*(lmax + 2)*(lmax + 3))/6;
        float const *src = cad + (size_t(img_starts[a])*nrhs + s)*128;
        for (int q = tid; q < nsho*32; q += kThreads) {
            int const row = q >> 5, part = (q & 31)*4;
            cp_async16(raw + row*128 + part, src + size_t(row)*cstride + part);
        }
        if (tid < (lmax + 1)*3) cp_async16(&Hs[st][0][0][0] + tid*4, slot_H + size_t(slot)*stride + tid*4);
        if (tid == kThreads - 1) cp_async8(&mk[st], slot_mask + slot);
        fill_sho_index(sidx[st], lmax, tid);
        if (0 == tid) lm[st] = lmax;
        cp_async_commit();
    };
    prefetch(k0, 0);
    for (uint32_t k = k0; k < k1; ++k) {
        int const it = int(k - k0), st = it & 1;
        char *sA_hi = smem + st*kStage, *sA_lo = sA_hi + kA, *sB_hi = sA_lo + kA, *sB_lo = sB_hi + kB;
        if (it >= 2) {                               // stage st is free once the MMAs of it-2 completed
            bool w = true;
            if (0 == tid) w = tc::mbar_wait(&mbar[st], uint32_t((it - 2) >> 1) & 1u, kWaitNs, err);
            ok = __syncthreads_and(w);               // block-uniform decision
            if (!ok) break;
        }
        cp_async_wait0();                            // coefficients, tables and mask of image k
        __syncthreads();
        int const lmax = lm[st], nsho = ((lmax + 1)*(lmax + 2)*(lmax + 3))/6;
        uint64_t const mask = mk[st];
        mask_all |= mask;
        // A = Cad^T: m = (reim, j), k = sho (rows beyond nsho zero)
        stage_A(sA_hi, sA_lo, raw, 64, 128, nsho, tid);
        __syncthreads();                             // raw is free: fetch the next image meanwhile
        if (k + 1 < k1) prefetch(k + 1, st ^ 1);
        // B = P: n = point i, k = sho; float4 along sho
#pragma unroll 2
        for (int r = 0; r < 1024/kThreads; ++r) {
            int const q = r*kThreads + tid;
            int const n = ((q >> 3) & 7)*8 + (q & 7), kc = q >> 6;
            float4 v;
            v.x = pval(Hs[st], sidx[st], mask, kc*4 + 0, nsho, n); v.y = pval(Hs[st], sidx[st], mask, kc*4 + 1, nsho, n);
            v.z = pval(Hs[st], sidx[st], mask, kc*4 + 2, nsho, n); v.w = pval(Hs[st], sidx[st], mask, kc*4 + 3, nsho, n);
            float4 h, l;
            tc::split_tf32(v.x, h.x, l.x); tc::split_tf32(v.y, h.y, l.y);
            tc::split_tf32(v.z, h.z, l.z); tc::split_tf32(v.w, h.w, l.w);
            uint32_t const o = offB(n, kc*4);
            *reinterpret_cast<float4*>(sB_hi + o) = h;
            *reinterpret_cast<float4*>(sB_lo + o) = l;
        }
        tc::fence_smem_to_async();
        __syncthreads();
        if (0 == tid) {
            tc::fence_after_sync();
            issue_mmas(tmem, tc::smem_u32(sA_hi), tc::smem_u32(sA_lo), tc::smem_u32(sB_hi), tc::smem_u32(sB_lo), 0 == it);
            tc::commit(&mbar[st]);
        }
        ++issued;
    }
    cp_async_wait0();                                // no copy outstanding when the CTA ends
    int const last = issued - 1;
    if (last >= 0) {
        bool w = ok;
        if (0 == tid && ok) w = tc::mbar_wait(&mbar[last & 1], uint32_t(last >> 1) & 1u, kWaitNs, err);
        ok = __syncthreads_and(w);
    }
    if (!ok && 0 == tid && last >= 0) {
        record_error(err, 2);
        // give the tensor core a bounded grace period before the TMEM is released
        tc::mbar_wait(&mbar[last & 1], uint32_t(last >> 1) & 1u, kWaitNs, err);
    }
    tc::fence_after_sync();
    if (ok && mask_all) {
        float v[32];
        int const quarter = warp & 3, half = warp >> 2;
        uint32_t const taddr = tmem + (uint32_t(quarter*32) << 16) + uint32_t(half*32);
        tc::tmem_ld_32x32b_x32(taddr, v);
        int const m = quarter*32 + lane, reim = m >> 6, j = m & 63;
        float *yb = y + size_t(b)*8192 + reim*4096 + size_t(half*32)*64 + j;
        uint32_t const mk = uint32_t(mask_all >> (half*32));
#pragma unroll
        for (int i = 0; i < 32; ++i)
            if ((mk >> i) & 1u) yb[i*64] += v[i];
    }
    tc::fence_before_sync();
    __syncthreads();
    if (0 == warp) tc::tmem_dealloc(tmem, 64);
}

} // namespace

namespace { bool g_tc_ready[64] = {}; }   // per device: the kernels got their shared memory

bool tc_projector_supported(DevicePlan const &dp) {
    int dev = 0;
    if (cudaSuccess != cudaGetDevice(&dev) || dev < 0 || dev >= 64 || !g_tc_ready[dev]) return false;
    return dp.lmax_max >= 0 && dp.lmax_max <= 5;
}

bool prepare_tc_kernels() {
    // a device on which the kernels cannot get their shared memory keeps the CUDA-core projector
    int dev = 0;
    if (cudaSuccess != cudaGetDevice(&dev) || dev < 0 || dev >= 64) return true;
    bool const ok = cudaSuccess == cudaFuncSetAttribute(sho_project_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem) &&
                    cudaSuccess == cudaFuncSetAttribute(sho_add_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmem);
    if (!ok) cudaGetLastError();                     // clear the error: the rest of the library is unaffected
    g_tc_ready[dev] = ok;
    return true;
}

bool launch_project_tc(DevicePlan &dp, float const *x, cudaStream_t st) {
    for (int L = 0; L < 8; ++L) {
        auto const &g = dp.img_group[L];
        if (0 == g.count) continue;
        dim3 const grid(g.count, dp.nCols);
        sho_project_tc_kernel<<<grid, kThreads, kSmem, st>>>(dptr<float>(dp.apc), x, dp.nCols,
            dptr<uint32_t>(g.images), dp.nAI, dptr<uint32_t>(dp.prj_start), dptr<uint32_t>(dp.prj_col),
            dptr<uint64_t>(dp.prj_coloff), dptr<uint32_t>(dp.prj_slot), dptr<float>(dp.slot_H32),
            dptr<uint64_t>(dp.slot_mask), dp.table_stride, dptr<uint32_t>(dp.img_starts), dptr<int8_t>(dp.img_lmax),
            dptr<int>(dp.dev_error));
        count_launch();
    }
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

bool launch_add_tc(DevicePlan &dp, float *y, uint16_t const *colIndex, cudaStream_t st) {
    sho_add_tc_kernel<<<dp.nnzb, kThreads, kSmem, st>>>(y, dptr<float>(dp.cad), dp.nCols, colIndex,
        dptr<uint32_t>(dp.add_start), dptr<uint32_t>(dp.add_col), dptr<uint32_t>(dp.add_slot),
        dptr<float>(dp.slot_H32), dptr<uint64_t>(dp.slot_mask), dp.table_stride, dptr<int8_t>(dp.img_lmax),
        dptr<uint32_t>(dp.img_starts), dptr<int>(dp.dev_error));
    count_launch();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

} // namespace a43g
