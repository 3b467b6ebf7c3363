// Atomic density matrices Im <p_i|G|p_j> from a Green function (green_dyadic::
// get_projection_coefficients, include/green_dyadic.hxx:1062-1088, and its SHOprj_right,
// :925-1060): the left index of G is projected onto every atom image's SHO functions with the
// action's own projection and image sums (the coefficients green_dyadic::multiply exports), then
// the right index, the points of each source cube, is contracted with the same functions
// evaluated at the source cube's points, summed over the source cubes, multiplied by the image's
// Bloch phase, and the imaginary part is accumulated onto the atom.  The reference computes the
// contraction on the CPU and only for plans without periodic images (nAtomImages == nAtoms);
// here it is one CTA per (atom image, left SHO index) on the GPU, with the same restriction.
#include "device.cuh"
#include "density_matrix.hpp"

namespace a43g {

namespace {

__host__ __device__ constexpr int nsho_dm(int L) { return ((L + 1)*(L + 2)*(L + 3))/6; }

// CTA (image a, left index isho), thread jsho: sum over the source cubes s and the masked points
// p of the source cube of aac[(a0 + isho)*nrhs + s][re, im][p] * H_jsho(p), then Im(phase * sum)
__global__ void __launch_bounds__(128)
sho_right_kernel(double *__restrict__ out, double const *__restrict__ aac, uint32_t nrhs,
                 uint32_t const *__restrict__ img_starts, int8_t const *__restrict__ img_lmax,
                 uint32_t const *__restrict__ img_index, double const *__restrict__ img_phase,
                 uint64_t const *__restrict__ out_off, double const *__restrict__ srcH,
                 uint64_t const *__restrict__ srcMask, int stride)
{
    constexpr int LM = 7;
    __shared__ double H[(LM + 1)*12];
    __shared__ double pre[64], pim[64];
    __shared__ uint64_t msk;
    uint32_t const a = blockIdx.x;
    int const isho = blockIdx.y, t = threadIdx.x;
    int const lmax = img_lmax[a], nc = nsho_dm(lmax);
    if (isho >= nc) return;                         // uniform over the CTA
    // quantum numbers of jsho = t in the zyx order of the SHO index
    int ix = 0, iy = 0, iz = 0;
    {
        int k = 0;
        bool found = false;
        for (int z = 0; z <= lmax && !found; ++z)
            for (int y = 0; y <= lmax - z && !found; ++y)
                for (int x = 0; x <= lmax - z - y; ++x, ++k)
                    if (k == t) { ix = x; iy = y; iz = z; found = true; break; }
    }
    double sr = 0, si = 0;
    size_t const a0 = img_starts[a];
    for (uint32_t s = 0; s < nrhs; ++s) {
        __syncthreads();                            // the previous source's stage is consumed
        for (int i = t; i < (lmax + 1)*12; i += blockDim.x) H[i] = srcH[(size_t(a)*nrhs + s)*stride + i];
        if (t < 64) {
            double const *c = aac + ((a0 + isho)*nrhs + s)*128;
            pre[t] = c[t]; pim[t] = c[64 + t];
        }
        if (0 == t) msk = srcMask[size_t(a)*nrhs + s];
        __syncthreads();
        if (t < nc && msk) {
            for (int p = 0; p < 64; ++p) {
                if (0 == ((msk >> p) & 1u)) continue;
                int const z4 = p >> 4, y4 = (p >> 2) & 3, x4 = p & 3;
                double const f = H[(ix*3 + 0)*4 + x4]*H[(iy*3 + 1)*4 + y4]*H[(iz*3 + 2)*4 + z4];
                sr += pre[p]*f; si += pim[p]*f;
            }
        }
    }
    if (t < nc) {
        double const pr = img_phase[4*size_t(a)], pi = img_phase[4*size_t(a) + 1];
        out[out_off[img_index[a]] + size_t(isho)*nc + t] = sr*pi + si*pr;   // Im((sr + i si)(pr + i pi))
    }
}

} // namespace

int projection_coefficients(GreenPlan const &hp, DevicePlan &dp, DensityWorkspace &ws, double const *G,
                            double *out, cudaStream_t st) {
    if (hp.nAtomImages != hp.nAtoms) {
        set_error("atomic density matrices need a plan without periodic atom images (nAtomImages == nAtoms), "
                  "as the reference's get_projection_coefficients does");
        return A43G_ERR_UNSUPPORTED;
    }
    if (hp.nAtoms < 1 || hp.nCols < 1) return A43G_OK;
    if (hp.table_lmax > 7) { set_error("projector basis sizes above numax 7 are not supported"); return A43G_ERR_UNSUPPORTED; }
    size_t const nI = size_t(dp.ncoeffI)*dp.nCols*128, nA = size_t(dp.ncoeffA)*dp.nCols*128;
    if (!ws.ready) {
        std::vector<double> H;
        std::vector<uint64_t> mask;
        hp.source_tables(H, mask);
        std::vector<uint64_t> off(hp.nAtoms + 1, 0);
        for (uint32_t ia = 0; ia < hp.nAtoms; ++ia) { int const n = nsho(hp.AtomLmax[ia]); off[ia + 1] = off[ia] + size_t(n)*n; }
        ws.nout = off[hp.nAtoms];
        ws.stride = (hp.table_lmax + 1)*12;
        if (!ws.srcH.alloc(std::max<size_t>(16, H.size()*8)) || !ws.srcMask.alloc(std::max<size_t>(16, mask.size()*8)) ||
            !ws.out_off.alloc(off.size()*8) || !ws.out.alloc(std::max<size_t>(16, ws.nout*8)) ||
            !ws.img_index.alloc(std::max<size_t>(16, hp.AtomImageIndex.size()*4)))
            return A43G_ERR_MEMORY;
        if (cudaSuccess != cudaMemcpy(ws.srcH.ptr, H.data(), H.size()*8, cudaMemcpyHostToDevice) ||
            cudaSuccess != cudaMemcpy(ws.srcMask.ptr, mask.data(), mask.size()*8, cudaMemcpyHostToDevice) ||
            cudaSuccess != cudaMemcpy(ws.out_off.ptr, off.data(), off.size()*8, cudaMemcpyHostToDevice) ||
            cudaSuccess != cudaMemcpy(ws.img_index.ptr, hp.AtomImageIndex.data(), hp.AtomImageIndex.size()*4,
                                      cudaMemcpyHostToDevice)) {
            set_error("upload of the source-cube projector tables");
            return A43G_ERR_CUDA;
        }
        ws.ready = true;
    }
    if (!ws.apc.alloc(std::max<size_t>(16, nI*8)) || !ws.aac.alloc(std::max<size_t>(16, nA*8))) return A43G_ERR_MEMORY;
    // <p|G: the image projections and their phase-weighted sums onto the atoms
    if (!launch_project_with(dp, dptr<double>(ws.apc), G, dptr<double>(dp.slot_H), st)) return A43G_ERR_CUDA;
    if (!launch_collect_with(dp, dptr<double>(ws.aac), dptr<double>(ws.apc), dptr<double>(dp.img_phase), st))
        return A43G_ERR_CUDA;
    dim3 const grid(dp.nAI, uint32_t(nsho(dp.lmax_max)));
    sho_right_kernel<<<grid, 128, 0, st>>>(dptr<double>(ws.out), dptr<double>(ws.aac), dp.nCols,
        dptr<uint32_t>(dp.img_starts), dptr<int8_t>(dp.img_lmax), dptr<uint32_t>(ws.img_index),
        dptr<double>(dp.img_phase), dptr<uint64_t>(ws.out_off), dptr<double>(ws.srcH), dptr<uint64_t>(ws.srcMask),
        ws.stride);
    count_launch();
    if (cudaSuccess != cudaGetLastError()) { set_error("launch of the density-matrix kernel"); return A43G_ERR_CUDA; }
    if (cudaSuccess != cudaMemcpyAsync(out, ws.out.ptr, ws.nout*8, cudaMemcpyDeviceToHost, st) ||
        cudaSuccess != cudaStreamSynchronize(st)) {
        set_error("copy of the atomic density matrices");
        return A43G_ERR_CUDA;
    }
    return A43G_OK;
}

} // namespace a43g
