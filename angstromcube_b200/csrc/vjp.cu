// Vector-Jacobian products of the action (FP64).  The reference has no derivatives; these
// kernels give the gradients of the bilinear form
//     F = sum over blocks b and source columns c of  L[b]^T (H - E S) G[b]      (no conjugation)
// with respect to the local potential, the atom matrices and the atom positions.  With G the
// Green function and L the solution of the adjoint system (the solve at conj(E), conjugated),
// -F derivatives are the derivatives of any linear functional of G, e.g. of the density.
//
//   dF/dV[cell][i]  = sum over blocks b with veff[b] = cell, columns j:  L[b][i][j] G[b][i][j]
//   dF/dM_A[m][n]   = sum over columns:  l_A[m] g_A[n]
//   dF/dR_A[d]      = sum over columns, m:  dl_A,d[m] (M_A g_A)[m] + l_A[m] (M_A dg_A,d)[m]
// where g_A = sum_i ph_i P_i G (the collected projection, include/green_dyadic.hxx:600-702),
// l_A = sum_i conj(ph_i) P_i L (the transpose of the addition), and dg, dl the same with the
// projector functions of direction d differentiated with respect to the atom position.
#include "device.cuh"
#include "vjp.hpp"

#include <algorithm>
#include <cstring>
#include <vector>

#define VJP_TRY(call) do { cudaError_t e_ = (call); if (cudaSuccess != e_) { \
    ::a43g::set_error(std::string(#call) + ": " + cudaGetErrorString(e_)); return A43G_ERR_CUDA; } } while (0)

namespace a43g {

namespace {

constexpr int kBlk = 8192;

// dV (complex, [ncells][64][2]) += sum over columns of L G, one CTA (64 threads = columns) per block
__global__ void __launch_bounds__(64) vjp_potential_kernel(double *__restrict__ dV, double const *__restrict__ L,
                                                           double const *__restrict__ G, int32_t const *__restrict__ veff,
                                                           uint32_t nnzb) {
    uint32_t const b = blockIdx.x;
    int const cell = veff[b];
    if (cell < 0) return;
    __shared__ double red[2][2][64];
    int const j = threadIdx.x, lane = j & 31, w = j >> 5;
    double const *lb = L + size_t(b)*kBlk, *gb = G + size_t(b)*kBlk;
    for (int i = 0; i < 64; ++i) {
        double const lr = lb[i*64 + j], li = lb[4096 + i*64 + j];
        double const gr = gb[i*64 + j], gi = gb[4096 + i*64 + j];
        double re = lr*gr - li*gi, im = lr*gi + li*gr;
        for (int o = 16; o > 0; o >>= 1) {
            re += __shfl_xor_sync(0xffffffffu, re, o);
            im += __shfl_xor_sync(0xffffffffu, im, o);
        }
        if (0 == lane) { red[w][0][i] = re; red[w][1][i] = im; }
    }
    __syncthreads();
    double *out = dV + (size_t(cell)*64 + j)*2;
    atomicAdd(out, red[0][0][j] + red[1][0][j]);
    atomicAdd(out + 1, red[0][1][j] + red[1][1][j]);
}

// dM[A][m][n] (complex) = sum over (s, j) of l[(a0+m)][s][j] g[(a0+n)][s][j];
// grid (nAtoms, max nSHO), threads n
__global__ void vjp_matrix_kernel(double *__restrict__ dM, double const *__restrict__ l, double const *__restrict__ g,
                                  uint32_t nrhs, uint32_t const *__restrict__ atom_starts,
                                  int8_t const *__restrict__ atom_lmax, uint32_t const *__restrict__ mat_off) {
    int const A = blockIdx.x, m = blockIdx.y, n = threadIdx.x;
    int const L = atom_lmax[A], nc = ((L + 1)*(L + 2)*(L + 3))/6;
    if (m >= nc || n >= nc) return;
    size_t const a0 = atom_starts[A];
    double re = 0, im = 0;
    for (uint32_t s = 0; s < nrhs; ++s) {
        double const *lp = l + ((a0 + m)*nrhs + s)*128, *gp = g + ((a0 + n)*nrhs + s)*128;
        for (int j = 0; j < 64; ++j) {
            double const lr = lp[j], li = lp[64 + j], gr = gp[j], gi = gp[64 + j];
            re += lr*gr - li*gi; im += lr*gi + li*gr;
        }
    }
    // complex matrices of atom A start at mat_off[A] (re plane, then im plane): same order here
    double *out = dM + mat_off[A];
    out[size_t(m)*nc + n] = re;
    out[size_t(nc)*nc + size_t(m)*nc + n] = im;
}

// dR[A][d] (complex) += sum over (m, s, j) of a[m][s][j] b[m][s][j] for the pairs of coefficient
// arrays given; grid (nAtoms), 256 threads
__global__ void __launch_bounds__(256) vjp_dot_kernel(double *__restrict__ out, double const *__restrict__ a,
                                                      double const *__restrict__ b, uint32_t nrhs,
                                                      uint32_t const *__restrict__ atom_starts,
                                                      int8_t const *__restrict__ atom_lmax, int d) {
    int const A = blockIdx.x;
    int const L = atom_lmax[A], nc = ((L + 1)*(L + 2)*(L + 3))/6;
    size_t const a0 = atom_starts[A];
    size_t const n = size_t(nc)*nrhs*64;
    double re = 0, im = 0;
    for (size_t e = threadIdx.x; e < n; e += blockDim.x) {
        size_t const row = e >> 6, j = e & 63;        // row = m*nrhs + s
        size_t const o = (a0*nrhs + row)*128 + j;
        double const ar = a[o], ai = a[o + 64], br = b[o], bi = b[o + 64];
        re += ar*br - ai*bi; im += ar*bi + ai*br;
    }
    __shared__ double r[2][256];
    r[0][threadIdx.x] = re; r[1][threadIdx.x] = im;
    __syncthreads();
    for (int k = 128; k > 0; k >>= 1) {
        if (threadIdx.x < k) { r[0][threadIdx.x] += r[0][threadIdx.x + k]; r[1][threadIdx.x] += r[1][threadIdx.x + k]; }
        __syncthreads();
    }
    if (0 == threadIdx.x) { out[(size_t(A)*3 + d)*2] += r[0][0]; out[(size_t(A)*3 + d)*2 + 1] += r[1][0]; }
}

template <typename T>
bool upload(DeviceBuffer &b, std::vector<T> const &v, cudaStream_t st) {
    size_t const n = std::max<size_t>(16, v.size()*sizeof(T));
    if (!b.alloc(n)) return false;
    if (!v.empty()) A43G_CUDA_TRY(cudaMemcpyAsync(b.ptr, v.data(), v.size()*sizeof(T), cudaMemcpyHostToDevice, st));
    return true;
}

} // namespace

int vjp(GreenPlan const &hp, DevicePlan &dp, VjpWorkspace &ws, double const *L, double const *G,
        double *dV, double *dM, double *dR, cudaStream_t st) {
    size_t const ncells = hp.ncells();
    if (dV) {
        if (!ws.dV.alloc(std::max<size_t>(16, ncells*64*2*sizeof(double)))) return A43G_ERR_MEMORY;
        if (cudaSuccess != cudaMemsetAsync(ws.dV.ptr, 0, ncells*64*2*sizeof(double), st)) { set_error("memset"); return A43G_ERR_CUDA; }
        if (dp.nnzb) {
            vjp_potential_kernel<<<dp.nnzb, 64, 0, st>>>(dptr<double>(ws.dV), L, G, dptr<int32_t>(dp.veff_index), dp.nnzb);
            count_launch();
        }
    }
    bool const atoms = dp.nAI > 0 && dp.nCols > 0 && dp.nAtoms > 0;
    size_t const nmat = hp.AtomMatOffset.empty() ? 0 : hp.AtomMatOffset.back();
    size_t const nI = size_t(dp.ncoeffI)*dp.nCols*128, nA = size_t(dp.ncoeffA)*dp.nCols*128;
    if (atoms && (dM || dR)) {
        // conjugated image phases (transpose of the broadcast)
        std::vector<double> phc(hp.AtomImagePhase);
        for (size_t a = 0; a < phc.size()/4; ++a) phc[4*a + 1] = -phc[4*a + 1];
        if (!upload(ws.phase_conj, phc, st)) return A43G_ERR_CUDA;
        for (DeviceBuffer *b : {&ws.apc, &ws.lA, &ws.gA})
            if (!b->alloc(std::max<size_t>(16, std::max(nI, nA)*sizeof(double)))) return A43G_ERR_MEMORY;
        double *apc = dptr<double>(ws.apc), *lA = dptr<double>(ws.lA), *gA = dptr<double>(ws.gA);
        double const *H = dptr<double>(dp.slot_H);
        if (!launch_project_with(dp, apc, L, H, st) || !launch_collect_with(dp, lA, apc, dptr<double>(ws.phase_conj), st)) return A43G_ERR_CUDA;
        if (!launch_project_with(dp, apc, G, H, st) || !launch_collect_with(dp, gA, apc, dptr<double>(dp.img_phase), st)) return A43G_ERR_CUDA;
        if (dM) {
            if (!ws.dM.alloc(std::max<size_t>(16, nmat*sizeof(double)))) return A43G_ERR_MEMORY;
            if (cudaSuccess != cudaMemsetAsync(ws.dM.ptr, 0, nmat*sizeof(double), st)) { set_error("memset"); return A43G_ERR_CUDA; }
            int nmax = 0;
            for (auto l : hp.AtomLmax) nmax = std::max(nmax, ((l + 1)*(l + 2)*(l + 3))/6);
            dim3 const grid(dp.nAtoms, nmax);
            vjp_matrix_kernel<<<grid, std::max(32, ((nmax + 31)/32)*32), 0, st>>>(dptr<double>(ws.dM), lA, gA, dp.nCols,
                dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), dptr<uint32_t>(dp.atom_mat_off));
            count_launch();
        }
        if (dR) {
            if (!ws.tables_ready) {
                for (int d = 0; d < 3; ++d) if (!upload(ws.slot_Hd[d], hp.position_derivative_tables(d), st)) return A43G_ERR_CUDA;
                ws.tables_ready = true;
            }
            for (DeviceBuffer *b : {&ws.Mg, &ws.dl, &ws.dg, &ws.Mdg})
                if (!b->alloc(std::max<size_t>(16, nA*sizeof(double)))) return A43G_ERR_MEMORY;
            if (!ws.dR.alloc(std::max<size_t>(16, size_t(dp.nAtoms)*6*sizeof(double)))) return A43G_ERR_MEMORY;
            if (cudaSuccess != cudaMemsetAsync(ws.dR.ptr, 0, size_t(dp.nAtoms)*6*sizeof(double), st)) { set_error("memset"); return A43G_ERR_CUDA; }
            double *Mg = dptr<double>(ws.Mg), *dl = dptr<double>(ws.dl), *dg = dptr<double>(ws.dg), *Mdg = dptr<double>(ws.Mdg);
            if (!launch_mul_with(dp, Mg, gA, st)) return A43G_ERR_CUDA;
            for (int d = 0; d < 3; ++d) {
                double const *Hd = dptr<double>(ws.slot_Hd[d]);
                if (!launch_project_with(dp, apc, L, Hd, st) || !launch_collect_with(dp, dl, apc, dptr<double>(ws.phase_conj), st)) return A43G_ERR_CUDA;
                if (!launch_project_with(dp, apc, G, Hd, st) || !launch_collect_with(dp, dg, apc, dptr<double>(dp.img_phase), st)) return A43G_ERR_CUDA;
                if (!launch_mul_with(dp, Mdg, dg, st)) return A43G_ERR_CUDA;
                vjp_dot_kernel<<<dp.nAtoms, 256, 0, st>>>(dptr<double>(ws.dR), dl, Mg, dp.nCols, dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), d);
                count_launch();
                vjp_dot_kernel<<<dp.nAtoms, 256, 0, st>>>(dptr<double>(ws.dR), lA, Mdg, dp.nCols, dptr<uint32_t>(dp.atom_starts), dptr<int8_t>(dp.atom_lmax), d);
                count_launch();
            }
        }
    }
    VJP_TRY(cudaGetLastError());
    if (dV) VJP_TRY(cudaMemcpyAsync(dV, ws.dV.ptr, ncells*64*2*sizeof(double), cudaMemcpyDeviceToHost, st));
    if (dM) {
        if (atoms) { VJP_TRY(cudaMemcpyAsync(dM, ws.dM.ptr, nmat*sizeof(double), cudaMemcpyDeviceToHost, st)); }
        else std::memset(dM, 0, nmat*sizeof(double));
    }
    if (dR) {
        if (atoms) { VJP_TRY(cudaMemcpyAsync(dR, ws.dR.ptr, size_t(dp.nAtoms)*6*sizeof(double), cudaMemcpyDeviceToHost, st)); }
        else std::memset(dR, 0, size_t(dp.nAtoms)*6*sizeof(double));
    }
    VJP_TRY(cudaStreamSynchronize(st));
    return A43G_OK;
}

} // namespace a43g
