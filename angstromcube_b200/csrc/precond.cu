// Cube-diagonal preconditioner: set-up on the host, application on the device (precond.hpp).
#include "precond.hpp"

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

namespace a43g {

namespace {

// eigenvalues lam[k] and eigenvectors V[i][k] of a symmetric 4x4 matrix (cyclic Jacobi rotations)
void jacobi4(double const (&A0)[4][4], double (&lam)[4], double (&V)[4][4]) {
    double A[4][4];
    for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) { A[i][j] = A0[i][j]; V[i][j] = (i == j) ? 1.0 : 0.0; }
    for (int sweep = 0; sweep < 50; ++sweep) {
        double off = 0;
        for (int i = 0; i < 4; ++i)
            for (int j = i + 1; j < 4; ++j) off += A[i][j]*A[i][j];
        if (off < 1e-30) break;
        for (int p = 0; p < 4; ++p)
            for (int q = p + 1; q < 4; ++q) {
                if (A[p][q] == 0.0) continue;
                double const theta = (A[q][q] - A[p][p])/(2*A[p][q]);
                double const t = (theta >= 0 ? 1.0 : -1.0)/(std::fabs(theta) + std::sqrt(theta*theta + 1));
                double const c = 1/std::sqrt(t*t + 1), s = t*c;
                for (int k = 0; k < 4; ++k) {            // A = J^T A J
                    double const akp = A[k][p], akq = A[k][q];
                    A[k][p] = c*akp - s*akq; A[k][q] = s*akp + c*akq;
                }
                for (int k = 0; k < 4; ++k) {
                    double const apk = A[p][k], aqk = A[q][k];
                    A[p][k] = c*apk - s*aqk; A[q][k] = s*apk + c*aqk;
                }
                for (int k = 0; k < 4; ++k) {
                    double const vkp = V[k][p], vkq = V[k][q];
                    V[k][p] = c*vkp - s*vkq; V[k][q] = s*vkp + c*vkq;
                }
            }
    }
    for (int k = 0; k < 4; ++k) lam[k] = A[k][k];
}

// the finite-difference weights of the distances 0..3 inside a cube (8th or 16th order) times
// the direction's prefactor -1/(2 h^2); zero where the direction has no kinetic term
void fd_weights(KineticLists const &kl, double (&w)[4]) {
    double const w8[4] = {-14350, 8064, -1008, 128}, w16[4] = {-924708642, 538137600, -94174080, 22830080};
    for (int k = 0; k < 4; ++k) w[k] = 0;
    if (kl.FD_range >= 8) for (int k = 0; k < 4; ++k) w[k] = kl.prefactor*w16[k]/302702400.;
    else if (kl.FD_range >= 1) for (int k = 0; k < 4; ++k) w[k] = kl.prefactor*w8[k]/5040.;
}

template <typename T> struct QOf;
template <> struct QOf<double> { using type = PrecondQ; };
template <> struct QOf<float> { using type = PrecondQf; };

// One CTA of 128 threads per half block (32 columns); thread (z-plane zq, column j) holds the
// real and imaginary parts of its plane's 16 points.  The x- and y-transforms run in registers,
// the z-transform through shared memory; each half block is read completely before it is
// written, so y may be x.
template <typename T>
__global__ void __launch_bounds__(128)
k_precond(T *y, T const *x, uint32_t nnzb, int32_t const *__restrict__ veff, uint32_t ncells,
          T const *__restrict__ tab, uint16_t const *__restrict__ colindx, uint32_t nsrc_pair,
          uint8_t const *__restrict__ active, typename QOf<T>::type const Q)
{
    __shared__ T sm[2][4][16][32];                   // [re, im][z][y*4 + x][column of the half]
    int const zq = threadIdx.x >> 5, jl = threadIdx.x & 31;
    for (uint32_t item = blockIdx.x; item < 2*nnzb; item += gridDim.x) {
        uint32_t const b = item >> 1;
        int const j = int(item & 1u)*32 + jl;
        uint32_t const s = colindx[b];
        if (active && !active[s]) continue;          // uniform over the CTA
        int32_t const cell = veff[b];
        T const *d = tab + ((size_t(s/nsrc_pair)*(ncells + 1) + (cell < 0 ? ncells : uint32_t(cell)))*64)*2;
        T re[16], im[16];
        T const *xb = x + size_t(b)*8192 + (zq*16)*64 + j;
#pragma unroll
        for (int i = 0; i < 16; ++i) { re[i] = xb[i*64]; im[i] = xb[4096 + i*64]; }
        // forward transform along x, then y (Q^T)
        auto fwd4 = [&](T (&v)[16], int dir) {
            T out[16];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int kk = 0; kk < 4; ++kk) {
                    T t = T(0);
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        int const idx = (0 == dir) ? a*4 + i : i*4 + a;     // dir 0: along x, 1: along y
                        t += T(Q.q[dir][i][kk])*v[idx];
                    }
                    out[(0 == dir) ? a*4 + kk : kk*4 + a] = t;
                }
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = out[i];
        };
        auto bwd4 = [&](T (&v)[16], int dir) {
            T out[16];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    T t = T(0);
#pragma unroll
                    for (int kk = 0; kk < 4; ++kk) {
                        int const idx = (0 == dir) ? a*4 + kk : kk*4 + a;
                        t += T(Q.q[dir][i][kk])*v[idx];
                    }
                    out[(0 == dir) ? a*4 + i : i*4 + a] = t;
                }
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = out[i];
        };
        fwd4(re, 0); fwd4(im, 0); fwd4(re, 1); fwd4(im, 1);
        // along z through shared memory, scaled, and back
        __syncthreads();                             // the previous block's last reads are done
#pragma unroll
        for (int i = 0; i < 16; ++i) { sm[0][zq][i][jl] = re[i]; sm[1][zq][i][jl] = im[i]; }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            T tr = T(0), ti = T(0);
#pragma unroll
            for (int z = 0; z < 4; ++z) {
                T const qz = T(Q.q[2][z][zq]);
                tr += qz*sm[0][z][i][jl]; ti += qz*sm[1][z][i][jl];
            }
            T const dr = d[2*(zq*16 + i)], di = d[2*(zq*16 + i) + 1];
            re[i] = tr*dr - ti*di; im[i] = tr*di + ti*dr;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; ++i) { sm[0][zq][i][jl] = re[i]; sm[1][zq][i][jl] = im[i]; }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 16; ++i) {
            T tr = T(0), ti = T(0);
#pragma unroll
            for (int z = 0; z < 4; ++z) {
                T const qz = T(Q.q[2][zq][z]);
                tr += qz*sm[0][z][i][jl]; ti += qz*sm[1][z][i][jl];
            }
            re[i] = tr; im[i] = ti;
        }
        bwd4(re, 1); bwd4(im, 1); bwd4(re, 0); bwd4(im, 0);
        T *yb = y + size_t(b)*8192 + (zq*16)*64 + j;
#pragma unroll
        for (int i = 0; i < 16; ++i) { yb[i*64] = re[i]; yb[4096 + i*64] = im[i]; }
    }
}

} // namespace

namespace {
bool upload_tables(BlockPreconditioner &pc, std::vector<double> const &t64, std::vector<float> const &t32,
                   cudaStream_t st) {
    size_t const n = t64.size();
    A43G_CUDA_TRY(cudaMemcpyAsync(pc.tab64.ptr, t64.data(), n*8, cudaMemcpyHostToDevice, st));
    A43G_CUDA_TRY(cudaMemcpyAsync(pc.tab32.ptr, t32.data(), n*4, cudaMemcpyHostToDevice, st));
    A43G_CUDA_TRY(cudaStreamSynchronize(st));      // the host tables go out of scope
    return true;
}
} // namespace

int precond_setup(GreenPlan const &hp, DevicePlan const &dp, BlockPreconditioner &pc, cudaStream_t st) {
    (void)dp;
    double lam[3][4];
    for (int d = 0; d < 3; ++d) {
        double w[4];
        fd_weights(hp.kinetic[d], w);
        double A[4][4], V[4][4];
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 4; ++k) A[i][k] = w[i > k ? i - k : k - i];
        jacobi4(A, lam[d], V);
        for (int i = 0; i < 4; ++i)
            for (int k = 0; k < 4; ++k) { pc.Q.q[d][i][k] = V[i][k]; pc.Qf.q[d][i][k] = float(V[i][k]); }
    }
    uint32_t const ncells = uint32_t(hp.ncells());
    uint32_t const npairs = std::max(1u, hp.npairs);
    pc.ncells = ncells; pc.npairs = npairs;
    pc.nsrc_pair = (hp.npairs > 1) ? hp.nsrc_pair : std::max(1u, hp.nCols);
    std::vector<double> vbar(size_t(ncells) + 1, 0.0);
    for (uint32_t c = 0; c < ncells && hp.Vcell.size() >= size_t(ncells)*64; ++c) {
        double sum = 0;
        for (int p = 0; p < 64; ++p) sum += hp.Vcell[size_t(c)*64 + p];
        vbar[c] = sum/64;
    }
    size_t const n = size_t(npairs)*(ncells + 1)*64*2;
    std::vector<double> t64(n);
    std::vector<float> t32(n);
    for (uint32_t pr = 0; pr < npairs; ++pr) {
        double const Er = (hp.npairs > 1) ? hp.pair_E[2*pr] : hp.E_re;
        double const Ei = (hp.npairs > 1) ? hp.pair_E[2*pr + 1] : hp.E_im;
        for (uint32_t c = 0; c <= ncells; ++c)
            for (int z = 0; z < 4; ++z)
                for (int yy = 0; yy < 4; ++yy)
                    for (int xx = 0; xx < 4; ++xx) {
                        int const p = (z*4 + yy)*4 + xx;
                        std::complex<double> const den(lam[2][z] + lam[1][yy] + lam[0][xx] + vbar[c] - Er, -Ei);
                        std::complex<double> const v = (0.0 == std::abs(den)) ? std::complex<double>(INFINITY, 0) : 1.0/den;
                        if (!std::isfinite(v.real()) || !std::isfinite(v.imag()) ||
                            !std::isfinite(float(v.real())) || !std::isfinite(float(v.imag()))) {
                            set_error("preconditioner: the cube model is singular at this energy "
                                      "(a real energy on one of its eigenvalues)");
                            return A43G_ERR_ARGUMENT;
                        }
                        size_t const o = ((size_t(pr)*(ncells + 1) + c)*64 + p)*2;
                        t64[o] = v.real(); t64[o + 1] = v.imag();
                        t32[o] = float(v.real()); t32[o + 1] = float(v.imag());
                    }
    }
    if (!pc.tab64.alloc(n*8) || !pc.tab32.alloc(n*4)) return A43G_ERR_MEMORY;
    return upload_tables(pc, t64, t32, st) ? A43G_OK : A43G_ERR_CUDA;
}

template <typename T>
bool precond_apply(DevicePlan const &dp, BlockPreconditioner const &pc, T *y, T const *x, uint8_t const *active,
                   cudaStream_t st) {
    if (0 == dp.nnzb) return true;
    unsigned const grid = uint32_t(std::min<uint64_t>(2ull*dp.nnzb, 148ull*16));
    T const *tab = (sizeof(T) == 8) ? reinterpret_cast<T const*>(pc.tab64.ptr) : reinterpret_cast<T const*>(pc.tab32.ptr);
    if constexpr (sizeof(T) == 8)
        k_precond<double><<<grid, 128, 0, st>>>(y, x, dp.nnzb, dptr<int32_t>(dp.veff_index), pc.ncells, tab,
                                                dptr<uint16_t>(dp.colindx), pc.nsrc_pair, active, pc.Q);
    else
        k_precond<float><<<grid, 128, 0, st>>>(y, x, dp.nnzb, dptr<int32_t>(dp.veff_index), pc.ncells, tab,
                                               dptr<uint16_t>(dp.colindx), pc.nsrc_pair, active, pc.Qf);
    count_launch();
    A43G_CUDA_TRY(cudaGetLastError());
    return true;
}

template bool precond_apply<double>(DevicePlan const &, BlockPreconditioner const &, double *, double const *,
                                    uint8_t const *, cudaStream_t);
template bool precond_apply<float>(DevicePlan const &, BlockPreconditioner const &, float *, float const *,
                                   uint8_t const *, cudaStream_t);

} // namespace a43g
