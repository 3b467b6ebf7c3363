/* TEST INFRASTRUCTURE ONLY -- the oracle (see green_oracle.h).
 *
 * Each function restates one part of the reference's action in plain C, written for
 * clarity rather than speed, and cites the reference lines it follows.  Parity of this
 * restatement is pinned against the reference's own CPU build (oracle/_ref) and against
 * the reference's analytic finite-difference known answers (src/green_kinetic.cxx:59-226).
 */
#include "green_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define BLK 8192 /* doubles per block: 2 x 64 x 64 */
#define AT(buf, inzb, reim, i, j) (buf)[(size_t)(inzb)*BLK + (size_t)(reim)*4096 + (size_t)(i)*64 + (j)]

static int nsho(int numax) { return ((1 + numax)*(2 + numax)*(3 + numax))/6; } /* include/sho_tools.hxx:21 */

/* include/green_potential.hxx:15-139 (Potential kernel, collinear, no confinement):
 *   y = (V(r_i) - Re E) x + i (-Im E) x  evaluated per complex element. */
void oracle_potential(const oracle_plan_t *p, double *y, const double *x)
{
    for (uint32_t b = 0; b < p->nnzb; ++b) {
        int32_t const iloc = p->veff_index[b];
        for (int i = 0; i < 64; ++i) {
            double const V = (iloc < 0) ? 0.0 : p->Vcell[(size_t)iloc*64 + i];
            double const Vt = V - p->E_re;
            for (int j = 0; j < 64; ++j) {
                double const xr = AT(x, b, 0, i, j), xi = AT(x, b, 1, i, j);
                /* (Vt - i Ei)(xr + i xi) = Vt xr + Ei xi + i (Vt xi - Ei xr) */
                AT(y, b, 0, i, j) = Vt*xr + p->E_im*xi;
                AT(y, b, 1, i, j) = Vt*xi - p->E_im*xr;
            }
        }
    }
}

/* 1D finite-difference second derivative along the lists of direction dd.
 * include/green_kinetic.hxx:23-195 (Laplace8th, 9-point stencil, halo cubes with Bloch phase)
 * and :199-329 (Laplace16th, 17-point stencil, isolated only), dispatched as in :342-367.
 * The list of one chain is [4 halo entries | n cube entries | 4 halo entries]; restated here
 * as a 1D line of 4*(n + 2*nh) points padded with the halo cubes (nh = 1 or 2). */
void oracle_kinetic(const oracle_plan_t *p, int dd, double *y, const double *x)
{
    int const nFD = p->FD_range[dd];
    if (nFD < 1) return;
    int const sixteenth = (8 == nFD);
    int const R = sixteenth ? 8 : 4;           /* stencil reach in grid points */
    double c[9];
    if (sixteenth) {
        static const double w[9] = {-924708642, 538137600, -94174080, 22830080, -5350800,
                                    1053696, -156800, 15360, -735};   /* / 302702400 */
        double const norm = p->kinetic_prefactor[dd]/302702400.;
        for (int k = 0; k <= 8; ++k) c[k] = w[k]*norm;
    } else {
        static const double w[5] = {-14350, 8064, -1008, 128, -9};    /* / 5040 */
        double const norm = p->kinetic_prefactor[dd]/5040.;
        for (int k = 0; k <= 4; ++k) c[k] = w[k]*norm;
    }
    int const stride = 1 << (2*dd);
    for (uint32_t il = 0; il < p->nlists[dd]; ++il) {
        const int32_t *list = p->lists[dd] + p->lists_start[dd][il];
        int const len = (int)(p->lists_start[dd][il + 1] - p->lists_start[dd][il]);
        int n = 0; /* number of cube entries, they start at list[4] and end before the first entry <= 0 */
        while (4 + n < len && list[4 + n] > 0) ++n;
        if (n < 1) continue;
        int const nh = R/4;                     /* halo cubes on each side */
        int const npts = 4*(n + 2*nh);
        double *line = (double*)malloc(sizeof(double)*2*(size_t)npts);
        double *out  = (double*)malloc(sizeof(double)*2*(size_t)npts);
        for (int i16 = 0; i16 < 16; ++i16) {
            int const base = (16 == stride) ? i16 : ((4 == stride) ? (16*(i16 >> 2) + (i16 & 3)) : 4*i16);
            for (int j = 0; j < 64; ++j) {
                memset(line, 0, sizeof(double)*2*(size_t)npts);
                for (int ic = 0; ic < n; ++ic) {
                    int const b = list[4 + ic] - 1;
                    for (int i4 = 0; i4 < 4; ++i4)
                        for (int ri = 0; ri < 2; ++ri)
                            line[2*(4*(nh + ic) + i4) + ri] = AT(x, b, ri, base + stride*i4, j);
                }
                if (!sixteenth) {
                    /* left halo: list[3] (<0: periodic image times phase[0]);
                     * right halo: the entry that ends the chain (<0: image times phase[1]) */
                    int32_t const hl = list[3], hr = list[4 + n];
                    for (int side = 0; side < 2; ++side) {
                        int32_t const h = side ? hr : hl;
                        if (h >= 0) continue;          /* 0: zero (isolated/vacuum) */
                        int const b = -h - 1;
                        double const pr = p->phase[dd][side][0], pi = p->phase[dd][side][1];
                        int const off = side ? 4*(nh + n) : 0;
                        for (int i4 = 0; i4 < 4; ++i4) {
                            double const xr = AT(x, b, 0, base + stride*i4, j), xi = AT(x, b, 1, base + stride*i4, j);
                            line[2*(off + i4) + 0] = pr*xr - pi*xi;
                            line[2*(off + i4) + 1] = pr*xi + pi*xr;
                        }
                    }
                }
                for (int ip = 4*nh; ip < 4*(nh + n); ++ip) {
                    for (int ri = 0; ri < 2; ++ri) {
                        double s = c[0]*line[2*ip + ri];
                        for (int k = 1; k <= R; ++k) s += c[k]*(line[2*(ip - k) + ri] + line[2*(ip + k) + ri]);
                        out[2*ip + ri] = s;
                    }
                }
                for (int ic = 0; ic < n; ++ic) {
                    int const b = list[4 + ic] - 1;
                    for (int i4 = 0; i4 < 4; ++i4)
                        for (int ri = 0; ri < 2; ++ri)
                            AT(y, b, ri, base + stride*i4, j) += out[2*(4*(nh + ic) + i4) + ri];
                }
            }
        }
        free(line); free(out);
    }
}

/* include/green_dyadic.hxx:33-107 (Hermite_polynomials_1D): unnormalized Hermite-Gauss
 * functions H_0 = exp(-xi^2/2) (0 outside the projection radius), H_{n+1} = xi H_n - n/2 H_{n-1},
 * xi = ((cube*4 + i4 + 1/2) h - R_atom)/sigma; xi^2 is exported in float for the mask. */
void oracle_hermite_1d(double H[8][3][4], float xi2[3][4], int lmax, const double xyza[4],
                       const float xyzc[3], const double hxyz[4])
{
    double const R2 = hxyz[3]*hxyz[3];
    double const sigma_inverse = xyza[3]*xyza[3];
    for (int d = 0; d < 3; ++d) {
        for (int i4 = 0; i4 < 4; ++i4) {
            double const xi = sigma_inverse*(((double)xyzc[d]*4 + i4 + 0.5)*hxyz[d] - xyza[d]);
            double const x2 = xi*xi;
            xi2[d][i4] = (float)x2;
            double hm = 0, h = (x2 < R2) ? exp(-0.5*x2) : 0;
            H[0][d][i4] = h;
            for (int nu = 0; nu < lmax; ++nu) {
                double const hp = xi*h - 0.5*nu*hm;
                H[nu + 1][d][i4] = hp;
                hm = h; h = hp;
            }
        }
    }
}

/* spherical mask of include/green_dyadic.hxx:218-239 / 472-492, evaluated in float exactly
 * as there: ((xi2_z - R2) + xi2_y) + xi2_x < 0 */
static int inside_mask(const float xi2[3][4], float R2f, int x, int y, int z)
{
    float const d2z = xi2[2][z] - R2f;
    float const d2yz = xi2[1][y] + d2z;
    float const d2xyz = xi2[0][x] + d2yz;
    return d2xyz < 0;
}

/* product of the three 1D functions for SHO index (ix,iy,iz) at point (x,y,z) */
static double hprod(double H[8][3][4], int ix, int iy, int iz, int x, int y, int z)
{
    return H[ix][0][x]*H[iy][1][y]*H[iz][2][z];
}

/* include/green_dyadic.hxx:856-922 (multiply): SHOprj (:112-288), then either
 * SHOsum-collect (:600-702) + SHOmul<double> (:740-826) + SHOsum-broadcast when there are
 * periodic images, or SHOmul directly; then SHOadd (:325-518). */
void oracle_dyadic(const oracle_plan_t *p, double *y, const double *x, double *apc_out, double *cad_out)
{
    uint32_t const nAI = p->nAtomImages, nA = p->nAtoms, nrhs = p->nCols;
    if (nAI < 1 || nrhs < 1) return;
    size_t const ncI = p->AtomImageStarts[nAI], ncA = p->AtomStarts[nA];
    double *apc = (double*)calloc(ncI*nrhs*128, sizeof(double)); /* [(i0+sho)*nrhs + s][2][64] */
    double *cad = (double*)calloc(ncI*nrhs*128, sizeof(double));
    float const R2f = (float)(p->grid_spacing[3]*p->grid_spacing[3]);
    double H[8][3][4]; float xi2[3][4];

    /* projection: apc[a,sho,s] = sum over blocks b of rhs s near image a, points inside the mask */
    for (uint32_t s = 0; s < nrhs; ++s) {
        const uint32_t *start = p->SHOprj_start + (size_t)s*(nAI + 1);
        const uint32_t *cols = p->SHOprj_col + p->SHOprj_coloff[s];
        for (uint32_t a = 0; a < nAI; ++a) {
            int const lmax = p->AtomImageLmax[a];
            for (uint32_t k = start[a]; k < start[a + 1]; ++k) {
                uint32_t const b = cols[k];
                float const *cp = p->rowCubePos + 4*(size_t)p->rowindx[b];
                oracle_hermite_1d(H, xi2, lmax, p->AtomImagePos + 4*a, cp, p->grid_spacing);
                int sho = 0;
                for (int iz = 0; iz <= lmax; ++iz)
                for (int iy = 0; iy <= lmax - iz; ++iy)
                for (int ix = 0; ix <= lmax - iz - iy; ++ix, ++sho) {
                    double *c = apc + ((p->AtomImageStarts[a] + sho)*(size_t)nrhs + s)*128;
                    for (int z = 0; z < 4; ++z) for (int yy = 0; yy < 4; ++yy) for (int xx = 0; xx < 4; ++xx) {
                        if (!inside_mask(xi2, R2f, xx, yy, z)) continue;
                        double const h = hprod(H, ix, iy, iz, xx, yy, z);
                        int const i64 = (z*4 + yy)*4 + xx;
                        for (int ri = 0; ri < 2; ++ri)
                            for (int j = 0; j < 64; ++j) c[ri*64 + j] += h*AT(x, b, ri, i64, j);
                    }
                }
            }
        }
    }
    if (apc_out) memcpy(apc_out, apc, sizeof(double)*ncI*nrhs*128);

    /* atom matrices: cad = M (sum over images phase * apc); broadcast with the conjugate phase */
    double *aac = (double*)calloc((ncA ? ncA : 1)*nrhs*128, sizeof(double));
    double *add = (double*)calloc((ncA ? ncA : 1)*nrhs*128, sizeof(double));
    int const with_images = (nAI > nA);
    for (uint32_t A = 0; A < nA; ++A) {
        int const nc = nsho(p->AtomLmax[A]);
        size_t const a0 = p->AtomStarts[A];
        if (with_images) {
            for (uint32_t k = p->SHOsum_start[A]; k < p->SHOsum_start[A + 1]; ++k) {
                uint32_t const ai = p->SHOsum_col[k];
                double const pr = p->AtomImagePhase[4*ai], pi = p->AtomImagePhase[4*ai + 1];
                size_t const i0 = p->AtomImageStarts[ai];
                for (int c = 0; c < nc; ++c) for (uint32_t s = 0; s < nrhs; ++s) {
                    double *dst = aac + ((a0 + c)*nrhs + s)*128;
                    const double *src = apc + ((i0 + c)*nrhs + s)*128;
                    for (int j = 0; j < 64; ++j) {
                        dst[j]      += pr*src[j] - pi*src[64 + j];
                        dst[64 + j] += pr*src[64 + j] + pi*src[j];
                    }
                }
            }
        } else {
            memcpy(aac + a0*nrhs*128, apc + a0*nrhs*128, sizeof(double)*nc*nrhs*128);
        }
    }
    size_t moff = 0;
    for (uint32_t A = 0; A < nA; ++A) {
        int const nc = nsho(p->AtomLmax[A]);
        size_t const a0 = p->AtomStarts[A];
        const double *Mr = p->AtomMatrices + moff, *Mi = Mr + (size_t)nc*nc;
        for (uint32_t s = 0; s < nrhs; ++s)
            for (int i = 0; i < nc; ++i) {
                double *dst = add + ((a0 + i)*nrhs + s)*128;
                for (int k = 0; k < nc; ++k) {
                    double const mr = Mr[i*nc + k], mi = Mi[i*nc + k];
                    const double *src = aac + ((a0 + k)*nrhs + s)*128;
                    for (int j = 0; j < 64; ++j) {
                        dst[j]      += mr*src[j] - mi*src[64 + j];
                        dst[64 + j] += mr*src[64 + j] + mi*src[j];
                    }
                }
            }
        moff += 2*(size_t)nc*nc;
    }
    if (with_images) {
        for (uint32_t A = 0; A < nA; ++A) {
            int const nc = nsho(p->AtomLmax[A]);
            size_t const a0 = p->AtomStarts[A];
            for (uint32_t k = p->SHOsum_start[A]; k < p->SHOsum_start[A + 1]; ++k) {
                uint32_t const ai = p->SHOsum_col[k];
                double const pr = p->AtomImagePhase[4*ai], pi = -p->AtomImagePhase[4*ai + 1];
                size_t const i0 = p->AtomImageStarts[ai];
                for (int c = 0; c < nc; ++c) for (uint32_t s = 0; s < nrhs; ++s) {
                    const double *src = add + ((a0 + c)*nrhs + s)*128;
                    double *dst = cad + ((i0 + c)*nrhs + s)*128;
                    for (int j = 0; j < 64; ++j) {
                        dst[j]      = pr*src[j] - pi*src[64 + j];
                        dst[64 + j] = pr*src[64 + j] + pi*src[j];
                    }
                }
            }
        }
    } else {
        memcpy(cad, add, sizeof(double)*ncA*nrhs*128);
    }
    if (cad_out) memcpy(cad_out, cad, sizeof(double)*ncI*nrhs*128);

    /* addition: y[b] += sum over images a near block b of P_a(points) cad[a, rhs(b)] */
    for (uint32_t b = 0; b < p->nnzb; ++b) {
        uint32_t const s = p->colindx[b];
        float const *cp = p->rowCubePos + 4*(size_t)p->rowindx[b];
        for (uint32_t k = p->SHOadd_start[b]; k < p->SHOadd_start[b + 1]; ++k) {
            uint32_t const a = p->SHOadd_col[k];
            int const lmax = p->AtomImageLmax[a];
            oracle_hermite_1d(H, xi2, lmax, p->AtomImagePos + 4*a, cp, p->grid_spacing);
            for (int z = 0; z < 4; ++z) for (int yy = 0; yy < 4; ++yy) for (int xx = 0; xx < 4; ++xx) {
                if (!inside_mask(xi2, R2f, xx, yy, z)) continue;
                int const i64 = (z*4 + yy)*4 + xx;
                int sho = 0;
                for (int iz = 0; iz <= lmax; ++iz)
                for (int iy = 0; iy <= lmax - iz; ++iy)
                for (int ix = 0; ix <= lmax - iz - iy; ++ix, ++sho) {
                    double const h = hprod(H, ix, iy, iz, xx, yy, z);
                    const double *c = cad + ((p->AtomImageStarts[a] + sho)*(size_t)nrhs + s)*128;
                    for (int ri = 0; ri < 2; ++ri)
                        for (int j = 0; j < 64; ++j) AT(y, b, ri, i64, j) += h*c[ri*64 + j];
                }
            }
        }
    }
    free(apc); free(cad); free(aac); free(add);
}

/* include/green_action.hxx:159-171: potential assigns y, then kinetic x, y, z, then dyadic */
void oracle_action(const oracle_plan_t *p, double *y, const double *x)
{
    oracle_potential(p, y, x);
    for (int dd = 0; dd < 3; ++dd) oracle_kinetic(p, dd, y, x);
    oracle_dyadic(p, y, x, NULL, NULL);
}

/* src/kinetic_plan.cxx:214-269 (set_phase): left phase exp(2 pi i angle), right phase its
 * conjugate; angles on the 15-degree grid use exact values sin(k 15deg) from the table
 * {0, (sqrt3-1) sqrt(1/2)/2, 1/2, sqrt(1/2), sqrt3/2, (sqrt3+1) sqrt(1/2)/2, 1}. */
double oracle_set_phase(double phase[2][2], double angle)
{
    double const arg = 2*3.14159265358979323846*angle;
    double cs = cos(arg), sn = sin(arg), dev = 0;
    double const a24 = angle*24;
    int const k = (int)a24;
    if (a24 == k) {
        double const sh = sqrt(0.5), s3 = sqrt(3);
        double const T[7] = {0.0, (s3 - 1)*sh*.5, .5, sh, s3*.5, (s3 + 1)*sh*.5, 1.0};
        int const k24 = ((k % 24) + 24) % 24;   /* angle in 15 degree steps, [0, 24) */
        int const q = k24/6, r = k24 % 6;        /* quadrant and remainder */
        int const is = (q & 1) ? 6 - r : r;      /* |sin| index */
        sn = ((q < 2) ? 1 : -1)*T[is];
        cs = ((q == 1 || q == 2) ? -1 : 1)*T[6 - is];
        dev = fmax(fabs(cs - cos(arg)), fabs(sn - sin(arg)));
    }
    phase[0][0] = cs; phase[0][1] = sn;
    phase[1][0] = cs; phase[1][1] = -sn;
    return dev;
}
