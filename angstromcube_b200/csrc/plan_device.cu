// Plan construction on the GPU: the atom-image x target-row overlap test of the dyadic plan
// (src/dyadic_plan.cxx:264-401 runs it as a serial loop over images and rows; the host builder
// restates that loop).  One thread per (candidate image, row), one ballot word per 32 rows; the
// double expressions are written with explicitly rounded operations in the host loop's order
// (no contraction into FMA), so the hit sets are bit-identical to the host's.
#include "device.cuh"
#include "plan.hpp"

#include <algorithm>

namespace a43g {

namespace {

__device__ __forceinline__ double sqr(double x) { return __dmul_rn(x, x); }

// bits[c][w]: bit r of word w is row 32 w + r of candidate c0 + c
__global__ void __launch_bounds__(256)
image_rows_kernel(uint32_t *__restrict__ bits, uint32_t nwords, double const *__restrict__ pos,
                  double const *__restrict__ r2p, double const *__restrict__ r2p_plus,
                  float const *__restrict__ rowpos, uint32_t nRows, double hx, double hy, double hz, size_t c0)
{
    size_t const c = c0 + blockIdx.y;
    uint32_t const ir = blockIdx.x*blockDim.x + threadIdx.x;
    bool hit = false;
    if (ir < nRows) {
        double const h[3] = {hx, hy, hz};
        double const p[3] = {pos[3*c], pos[3*c + 1], pos[3*c + 2]};
        float const t[3] = {rowpos[4*size_t(ir)], rowpos[4*size_t(ir) + 1], rowpos[4*size_t(ir) + 2]};
        // centre distance: sum over d of ((t*4f + 2.0) h - p)^2
        double dc2 = 0;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            double const a = __dsub_rn(__dmul_rn(__dadd_rn(double(t[d]*4.f), 2.0), h[d]), p[d]);
            dc2 = __dadd_rn(dc2, sqr(a));
        }
        if (!(dc2 > r2p_plus[c])) {
            double d2c[3][2];
#pragma unroll
            for (int d = 0; d < 3; ++d)
#pragma unroll
                for (int ii = 0; ii < 2; ++ii) {
                    double const x = __dadd_rn(__dadd_rn(__dmul_rn(double(t[d]), 4.0), double(ii*3)), 0.5);
                    d2c[d][ii] = sqr(__dsub_rn(__dmul_rn(x, h[d]), p[d]));
                }
            double const lim = r2p[c];
#pragma unroll
            for (int i8 = 0; i8 < 8; ++i8)
                hit |= (__dadd_rn(__dadd_rn(d2c[0][i8 & 1], d2c[1][(i8 & 2) >> 1]), d2c[2][i8 >> 2]) < lim);
        }
    }
    uint32_t const word = __ballot_sync(0xffffffffu, hit);
    if (0 == (threadIdx.x & 31) && (ir >> 5) < nwords) bits[size_t(blockIdx.y)*nwords + (ir >> 5)] = word;
}

} // namespace

std::string image_rows_on_device(ImageRowsTask const &t, std::vector<std::vector<uint32_t>> &hits) {
    hits.assign(t.ncand, {});
    if (0 == t.ncand || 0 == t.nRows) return "";
    uint32_t const nwords = (t.nRows + 31)/32;
    // candidates per launch: grid y <= 65535 and at most 256 MB of bits
    size_t const chunk = std::min<size_t>({t.ncand, 65535, std::max<size_t>(1, (size_t(256) << 20)/(size_t(nwords)*4))});
    DeviceBuffer dpos, dr2p, dr2pp, drows, dbits;
    if (!dpos.alloc(t.ncand*3*8) || !dr2p.alloc(t.ncand*8) || !dr2pp.alloc(t.ncand*8) ||
        !drows.alloc(size_t(t.nRows)*4*4) || !dbits.alloc(chunk*nwords*4))
        return "device plan construction: out of device memory";
    if (cudaSuccess != cudaMemcpy(dpos.ptr, t.pos, t.ncand*3*8, cudaMemcpyHostToDevice) ||
        cudaSuccess != cudaMemcpy(dr2p.ptr, t.r2p, t.ncand*8, cudaMemcpyHostToDevice) ||
        cudaSuccess != cudaMemcpy(dr2pp.ptr, t.r2p_plus, t.ncand*8, cudaMemcpyHostToDevice) ||
        cudaSuccess != cudaMemcpy(drows.ptr, t.rowCubePos, size_t(t.nRows)*4*4, cudaMemcpyHostToDevice))
        return "device plan construction: upload of the inputs failed";
    std::vector<uint32_t> bits(chunk*nwords);
    for (size_t c0 = 0; c0 < t.ncand; c0 += chunk) {
        size_t const nc = std::min(chunk, t.ncand - c0);
        dim3 const grid((t.nRows + 255)/256, uint32_t(nc));
        image_rows_kernel<<<grid, 256>>>(dptr<uint32_t>(dbits), nwords, dptr<double>(dpos), dptr<double>(dr2p),
                                         dptr<double>(dr2pp), dptr<float>(drows), t.nRows, t.hg[0], t.hg[1],
                                         t.hg[2], c0);
        count_launch();
        if (cudaSuccess != cudaGetLastError() ||
            cudaSuccess != cudaMemcpy(bits.data(), dbits.ptr, nc*nwords*4, cudaMemcpyDeviceToHost))
            return std::string("device plan construction: ") + cudaGetErrorString(cudaGetLastError());
        for (size_t c = 0; c < nc; ++c) {
            auto &h = hits[c0 + c];
            for (uint32_t w = 0; w < nwords; ++w)
                for (uint32_t m = bits[c*nwords + w]; m; m &= m - 1) h.push_back(32*w + uint32_t(__builtin_ctz(m)));
        }
    }
    return "";
}

} // namespace a43g
