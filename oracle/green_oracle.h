/* TEST INFRASTRUCTURE ONLY -- the oracle.
 *
 * Plain-C restatement of AngstromCube's Green-function action Y = (H - E S) X
 * (real-space/AngstromCube, include/green_action.hxx:140-176) in FP64, complex
 * (R1C2 = 2), collinear (Noco = 1).  Blocks are double[nnzb][2][64][64]:
 * [block][re,im][target point i64][source column j64], columns fastest.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg call this.
 */
#ifndef GREEN_ORACLE_H
#define GREEN_ORACLE_H
#include <stdint.h>

typedef struct {
    uint32_t nnzb, nRows, nCols;
    const uint16_t *colindx;       /* [nnzb] source cube column of each block */
    const uint32_t *rowindx;       /* [nnzb] target cube row of each block */
    const int32_t  *veff_index;    /* [nnzb] cell-cube index of the potential, -1: none */
    const double   *Vcell;         /* [ncells][64] local potential */
    double E_re, E_im;             /* energy parameter */
    /* kinetic: finite-difference lists per direction (src/kinetic_plan.cxx:38-210) */
    uint32_t nlists[3];
    const uint32_t *lists_start[3];/* [nlists+1] */
    const int32_t  *lists[3];      /* entries: inzb+1, 0 (zero cube), -(inzb+1) (periodic image) */
    double kinetic_prefactor[3];   /* -0.5/h^2 */
    int32_t FD_range[3];           /* 4: 8th order, 8: 16th order, <1: off */
    double phase[3][2][2];         /* [dd][left,right][re,im] Bloch phases */
    /* dyadic (include/dyadic_plan.hxx:14-47) */
    uint32_t nAtoms, nAtomImages;
    const uint32_t *AtomStarts;    /* [nAtoms+1] */
    const int8_t   *AtomLmax;      /* [nAtoms] */
    const double   *AtomMatrices;  /* concatenated [nAtoms][2][nc][nc] (re, im), dVol included */
    const uint32_t *AtomImageStarts; /* [nAI+1] */
    const double   *AtomImagePos;  /* [nAI][4] x,y,z,1/sqrt(sigma) */
    const int8_t   *AtomImageLmax; /* [nAI] */
    const double   *AtomImagePhase;/* [nAI][4] */
    const double   *grid_spacing;  /* [4] hx,hy,hz, projection radius in sigma */
    const float    *rowCubePos;    /* [nRows][4] */
    const uint32_t *SHOprj_start;  /* [nCols][nAI+1] (each rhs its own CSR over images) */
    const uint32_t *SHOprj_col;    /* concatenated over rhs, entries inzb */
    const uint64_t *SHOprj_coloff; /* [nCols] offset of each rhs in SHOprj_col */
    const uint32_t *SHOadd_start;  /* [nnzb+1] */
    const uint32_t *SHOadd_col;    /* entries: atom image index */
    const uint32_t *SHOsum_start;  /* [nAtoms+1] */
    const uint32_t *SHOsum_col;    /* entries: atom image index */
} oracle_plan_t;

#ifdef __cplusplus
extern "C" {
#endif
/* y = (V - E) x, assigns every block of y */
void oracle_potential(const oracle_plan_t *p, double *y, const double *x);
/* y += T_dd x along the lists of one direction */
void oracle_kinetic(const oracle_plan_t *p, int dd, double *y, const double *x);
/* y += sum_a P_a M_a P_a^T x  (projection, atom-matrix multiply, addition);
 * apc/aac: optional outputs of the image projection coefficients [ncoeff_images*nCols][2][64]
 * and of the addition coefficients (may be NULL) */
void oracle_dyadic(const oracle_plan_t *p, double *y, const double *x, double *apc, double *cad);
/* the full action in the reference's order: potential, kinetic x,y,z, dyadic */
void oracle_action(const oracle_plan_t *p, double *y, const double *x);
/* 1D unnormalized Hermite-Gauss functions H[nu][dir][i4] and float xi^2[dir][i4] of one
 * (atom image, target cube) pair */
void oracle_hermite_1d(double H[8][3][4], float xi2[3][4], int lmax, const double xyza[4],
                       const float xyzc[3], const double hxyz[4]);
/* kinetic_plan::set_phase restated: phase[2][2] for a phase angle in units of 2 pi */
double oracle_set_phase(double phase[2][2], double angle);
#ifdef __cplusplus
}
#endif
#endif
